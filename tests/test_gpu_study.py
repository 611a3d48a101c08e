"""Study loops on the device against the reference.

Topology: the reference's own optimizeTopology (oracle/_ref, native/src/fea/topology.cpp:103-183,
with runTopology's solve) and ps_topology_run on the same inputs; the per-iteration compliance,
volume and design change must agree (each solve stops at rel. res. 1e-5, so the two designs differ
by solver rounding that the optimisation carries along, ~1e-5 relative per iteration).

Break test: a restatement of breakTest (native/src/fea/static_study.cpp:199-279) composed of the
reference's own solver calls (VoxelFEA solve with warm start, stresses, pruneFloating) against
ps_break_test: load factors, solved-voxel counts and cracked voxels per step."""
import numpy as np
import pytest

import oracle
import psfea
import voxel_models as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def check_topology(m, fill, keep, max_iter, **kw):
    d_ref, h_ref = oracle.topology(m.dims, fill, m.nu, m.bc, m.f, keep=keep, max_iter=max_iter, **kw)
    d, h = psfea.topology_run(m.dims, fill, m.nu, m.bc, m.f, keep=keep, max_iter=max_iter, **kw)
    assert len(h) == len(h_ref)
    for row, (it, c, v, ch) in zip(h, h_ref):
        assert row["it"] == it
        assert rel(row["compliance"], c) < 1e-3, (row, c)
        assert abs(row["volume"] - v) < 1e-3, (row, v)
        assert abs(row["change"] - ch) < 2e-2, (row, ch)
        assert row["solve_status"] == psfea.PS_OK
    assert np.abs(d - d_ref).max() < 0.1 and abs(d.mean() - d_ref.mean()) < 1e-3
    assert np.all(d[fill == 0] == 0)
    return h


def test_topology_cantilever_matches_reference():
    m = W.cantilever(24, 8, 8, coarsest_max_dof=1100)
    h = check_topology(m, np.ones(24 * 8 * 8, np.float32), None, 8, vol_frac=0.4)
    assert h[-1]["compliance"] < 0.5 * h[0]["compliance"]


def test_topology_with_kept_voxels_and_partial_fill_matches_reference():
    """Voxels at the support kept solid, a partially filled design domain (fill < 1 on one layer
    and a void pocket), a tighter budget and a wider filter."""
    m = W.cantilever(20, 10, 6, coarsest_max_dof=1100)
    nx, ny, nz = m.dims
    fill = np.ones((nz, ny, nx), np.float32)
    fill[:, :, nx // 2] = 0.5
    fill[2:4, 3:6, 5:9] = 0
    keep = np.zeros((nz, ny, nx), np.uint8)
    keep[:, :, 0] = 1
    check_topology(m, fill.ravel(), keep.ravel(), 6, vol_frac=0.3, rmin=2.0)


def reference_break(m, E, h, strength, principal, max_steps):
    """breakTest (static_study.cpp:199-279) composed of the reference's own calls."""
    held = W.held_nodes(m.dims, m.bc)
    dens, _ = oracle.prune("reference", m.dims, m.density, held)
    nx, ny, nz = m.dims
    NX, NY = nx + 1, ny + 1
    off = np.array([0, 1, 1 + NX, NX, NX * NY, 1 + NX * NY, 1 + NX + NX * NY, NX + NX * NY])
    fm = np.linalg.norm(m.f.reshape(-1, 3), axis=1)
    x0, steps, reason, peak = None, [], "step limit", 0.0
    for step in range(max_steps):
        if not (dens > 0).any():
            reason = "separated" if step else "unsupported load"
            break
        R = oracle.OracleModel("reference", m.dims, dens, m.nu, m.bc, 1100)
        act = R.active(0)
        if R.level_info(0)["nElems"] == 0 or fm[act == 0].sum() / fm.sum() > 0.5:
            reason = "separated" if step else "unsupported load"
            break
        u, it, res, conv = R.solve(m.f, 1e-6, 3000, x0)
        if not conv:
            reason = "solver did not converge"
            break
        vm, p1, _ = R.stresses(u / (E * h), E, h, True)
        nodal = p1 if principal else vm
        x0 = u
        solved = np.nonzero(dens > 0)[0]
        i, j, k = solved % nx, (solved // nx) % ny, solved // (nx * ny)
        base = i + NX * (j + NY * k)
        measure = nodal[base[:, None] + off[None, :]].max(axis=1)
        smax = float(measure.max())
        if not smax > 0:
            reason = "no stress"
            break
        lam = strength / smax
        peak = max(peak, lam)
        cap = max(1, int(round(0.02 * len(solved) ** (2.0 / 3))))
        order = np.argsort(-measure, kind="stable")
        cracked = [int(solved[q]) for q in order if measure[q] >= 0.95 * smax][:cap]
        nxt = dens.copy()
        nxt[cracked] = 0
        dens, _ = oracle.prune("reference", m.dims, nxt, held)
        steps.append({"lambda": lam, "voxels": len(solved), "cracked": sorted(cracked),
                      "candidates": int((measure >= 0.95 * smax).sum()), "cap": cap})
    return steps, dens, peak, reason


@pytest.mark.parametrize("principal", [False, True])
def test_break_test_matches_reference(principal):
    m = W.l_bracket(48, 16, 24, holes=3, seed=5)
    E, h = 70e9, 0.5e-3
    strength = 250e6
    ref_steps, ref_dens, ref_peak, ref_reason = reference_break(m, E, h, strength, principal, 4)
    out = psfea.break_test(m.dims, m.density, m.nu, m.bc, m.f, E, h, strength, principal=principal, max_steps=4)
    assert out["reason"] == ref_reason and len(out["steps"]) == len(ref_steps)
    for s, r, cr in zip(out["steps"], ref_steps, out["cracked"]):
        assert s["voxels"] == r["voxels"]
        assert rel(s["lambda"], r["lambda"]) < 1e-4, (s, r["lambda"])
        if r["candidates"] <= r["cap"]:  # the cracked set does not depend on the order of equal measures
            assert sorted(cr.tolist()) == r["cracked"]
        else:
            assert len(cr) == len(r["cracked"])
    assert rel(out["peak"], ref_peak) < 1e-4
    if all(r["candidates"] <= r["cap"] for r in ref_steps):
        assert np.array_equal(out["density"], ref_dens)


def test_prune_floating_on_the_device_matches_the_library_and_reference():
    """ps_prune_floating_dev (union-find components) keeps exactly the voxels of the host
    breadth-first search and of the reference's prune fixture: random sparse grids, a gyroid sheet
    with floating fragments, a grid with nothing held."""
    import torch
    from conftest import golden
    dev = torch.device("cuda", 0)

    def run(dims, d, held):
        dd = torch.from_numpy(np.ascontiguousarray(d, np.float32)).to(dev)
        hh = torch.from_numpy(np.ascontiguousarray(held, np.uint8)).to(dev)
        out = torch.full_like(dd, float("nan"))
        rem = psfea.prune_floating_dev(dims, dd.data_ptr(), hh.data_ptr(), out.data_ptr())
        return out.cpu().numpy(), rem

    g = golden("prune")
    for d, h, dims in ((g["d1"], g["h1"], (4, 1, 1)), (g["d2"], g["h2"], tuple(g["dims2"]))):
        o, r = run(dims, d, h)
        o_ref, r_ref = oracle.prune("reference", dims, d, h)
        assert np.array_equal(o, o_ref) and r == r_ref
    rng = np.random.default_rng(8)
    for dims in ((64, 48, 40), (17, 9, 13), (1, 1, 1), (200, 3, 2)):
        nx, ny, nz = dims
        for frac in (0.3, 0.55):
            d = (rng.random(nx * ny * nz) < frac).astype(np.float32) * (0.5 + rng.random(nx * ny * nz).astype(np.float32))
            held = (rng.random((nx + 1) * (ny + 1) * (nz + 1)) < 0.01).astype(np.uint8)
            o, r = run(dims, d, held)
            o_lib, r_lib = psfea.prune_floating(dims, d, held)
            assert np.array_equal(o, o_lib) and r == r_lib, (dims, frac)
    m = W.gyroid(96, 96, 48)
    t = lambda n: 2 * np.pi * (np.arange(n) + 0.5) / 24
    val = (np.sin(t(96))[None, None, :] * np.cos(t(96))[None, :, None] + np.sin(t(96))[None, :, None] * np.cos(t(48))[:, None, None]
           + np.sin(t(48))[:, None, None] * np.cos(t(96))[None, None, :])
    raw = (np.abs(val) < 0.3).astype(np.float32).ravel()
    held = W.held_nodes((96, 96, 48), m.bc)
    o, r = run((96, 96, 48), raw, held)
    assert np.array_equal(o, m.density) and r == m.meta["removed"]
    o, r = run((96, 96, 48), raw, np.zeros_like(held))
    assert not o.any() and r == int((raw > 0).sum())
