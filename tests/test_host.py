"""CPU-side checks of the product library: it loads, exports every symbol include/ps_fea.h
declares, and its host-side hierarchy build (no GPU) matches the reference's golden vectors."""
import os
import re

import numpy as np
import pytest

import psfea
from conftest import ROOT, golden
import voxel_models as W

MODELS = ["cantilever_32x8x8", "cantilever_64x16x16", "lbracket_32x16x16", "simp_16x8x8", "lbracket_24x12x12_loose", "gyroid_48x48x24",
          "box_request_20_28"]


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ps_fea.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(psfea.lib, n), n
    assert set(names) == set(psfea.EXPORTS)


@pytest.mark.parametrize("nu", [0.3, 0.33, 0.34, 0.36])
def test_element_matrix(nu):
    g = golden("element")
    K, cs = psfea.element_matrix(nu)
    Kr = g[f"K_{nu}"]
    assert np.abs(K - Kr).max() <= 1e-14 * np.abs(Kr).max()
    assert np.array_equal(K, K.T)
    if nu == 0.3:
        assert np.abs(cs - g["cornerStress_0.3"]).max() <= 1e-14 * np.abs(cs).max()


def test_invalid_inputs_raise_like_the_reference():
    for nu in (-1, 0.5, float("nan"), float("inf")):  # test/fea.test.js:128
        with pytest.raises(ValueError, match="Poisson"):
            psfea.element_matrix(nu)
        with pytest.raises(ValueError, match="Poisson"):
            psfea.Hierarchy((1, 1, 1), np.ones(1, np.float32), nu, np.ones(24, np.uint8))
    bc = np.zeros(3 * 5 * 2 * 2, np.uint8)
    with pytest.raises(ValueError, match="between zero and one"):
        psfea.Hierarchy((4, 1, 1), np.array([1, 2, 0, 1], np.float32), 0.3, bc)
    with pytest.raises(ValueError, match="do not match"):
        psfea.Hierarchy((4, 1, 1), np.ones(3, np.float32), 0.3, bc)
    with pytest.raises(ValueError, match="three positive"):
        psfea.Hierarchy((0, 1, 1), np.ones(0, np.float32), 0.3, np.zeros(12, np.uint8))


def test_prune_matches_reference():
    g = golden("prune")
    o1, r1 = psfea.prune_floating((4, 1, 1), g["d1"], g["h1"])
    assert np.array_equal(o1, g["o1"]) and r1 == 1
    o2, r2 = psfea.prune_floating(tuple(g["dims2"]), g["d2"], g["h2"])
    assert np.array_equal(o2, g["o2"]) and r2 == int(g["r2"])


def test_model_generators_prune_like_the_library():
    """The generators' pruning (connected-component labelling, no library needed, so the reference
    arm of the benchmark can build its inputs without loading the product) keeps exactly the voxels
    the library's breadth-first search keeps: on the reference's prune cases, on a gyroid sheet with
    floating fragments and on random sparse grids."""
    g = golden("prune")
    for d, h, dims in ((g["d1"], g["h1"], (4, 1, 1)), (g["d2"], g["h2"], tuple(g["dims2"]))):
        o, r = W.prune_floating(dims, d, h)
        o_lib, r_lib = psfea.prune_floating(dims, d, h)
        assert np.array_equal(o, o_lib) and r == r_lib
    rng = np.random.default_rng(4)
    for dims in ((48, 48, 24), (17, 9, 13), (1, 1, 1)):
        nx, ny, nz = dims
        for frac in (0.35, 0.6):
            d = (rng.random(nx * ny * nz) < frac).astype(np.float32) * rng.random(nx * ny * nz).astype(np.float32)
            held = (rng.random((nx + 1) * (ny + 1) * (nz + 1)) < 0.02).astype(np.uint8)
            o, r = W.prune_floating(dims, d, held)
            o_lib, r_lib = psfea.prune_floating(dims, d, held)
            assert np.array_equal(o, o_lib) and r == r_lib, (dims, frac)
    m = W.gyroid(48, 48, 24)
    t = lambda n: 2 * np.pi * (np.arange(n) + 0.5) / 24
    val = (np.sin(t(48))[None, None, :] * np.cos(t(48))[None, :, None] + np.sin(t(48))[None, :, None] * np.cos(t(24))[:, None, None]
           + np.sin(t(24))[:, None, None] * np.cos(t(48))[None, None, :])
    raw = (np.abs(val) < 0.3).astype(np.float32).ravel()
    o_lib, r_lib = psfea.prune_floating((48, 48, 24), raw, W.held_nodes((48, 48, 24), m.bc))
    assert np.array_equal(m.density, o_lib) and m.meta["removed"] == r_lib


@pytest.mark.parametrize("name", MODELS)
def test_hierarchy_matches_reference(name):
    """Fixed-DOF masks, voxel/element indexing and level sizes bit-exact on every level."""
    g = golden(name)
    H = psfea.Hierarchy(tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    assert H.n_levels == int(g["levels"])
    for l in range(H.n_levels):
        info = H.level_info(l)
        assert [info[k] for k in ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")] == list(g[f"info_{l}"])
        assert np.array_equal(np.packbits(H.fixed(l)), g[f"fixed_{l}"])


@pytest.mark.parametrize("model", ["l_bracket", "gyroid", "simp"])
def test_own_matrices_match_oracle(model):
    """Galerkin matrices against the oracle's, on an L-bracket, a gyroid (a few hundred classes of
    equal child patterns over thousands of voxels: computed once per class, then copied) and the
    graded SIMP grid (180 k mostly distinct matrices on level 1: the class search stops early)."""
    import oracle
    m = {"l_bracket": lambda: W.l_bracket(32, 16, 16, holes=3), "gyroid": lambda: W.gyroid(48, 48, 24),
         "simp": lambda: W.simp(nrhs=1)}[model]()
    H = psfea.Hierarchy(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    for l in range(1, H.n_levels):
        a, b = H.own(l), P.own(l)
        assert a.shape == b.shape
        if a.size:
            assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
        assert np.abs(H.kb(l) - P.kb(l)).max() <= 1e-13 * np.abs(P.kb(l)).max()


def test_workloads_are_deterministic_and_loaded_as_specified():
    c = W.cantilever()
    assert c.dims == (64, 16, 16) and abs(c.f.sum() + 256.0) < 1e-9
    assert c.bc.reshape(17, 17, 65, 3)[:, :, 0].all() and c.bc.sum() == 3 * 17 * 17
    a, b = W.l_bracket(64, 32, 32, holes=8), W.l_bracket(64, 32, 32, holes=8)
    assert np.array_equal(a.density, b.density) and np.array_equal(a.f, b.f)
    assert abs(a.f.sum() + 500.0) < 1e-9
    s = W.simp(16, 8, 8, nrhs=4)
    assert s.f.shape[0] == 4 and np.allclose(np.linalg.norm(s.f.reshape(4, -1, 3).sum(axis=1), axis=1), 1.0)
    assert s.density.min() >= 1e-9 and s.density.max() <= 1.0


def test_no_device_is_reported_not_faked(have_gpu):
    if have_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(psfea.SolverError, match="ENODEV"):
        psfea.VoxelFEA((4, 1, 1), np.ones(4, np.float32), 0.3, np.zeros(3 * 5 * 2 * 2, np.uint8))


def test_device_hierarchy_build_needs_a_device(have_gpu):
    """The device Galerkin build reports the missing device; the host build of the same model works."""
    if have_gpu:
        pytest.skip("a GPU is present")
    dims, dens, bc = (4, 2, 2), np.ones(16, np.float32), np.zeros(3 * 5 * 3 * 3, np.uint8)
    bc[:3 * 5 * 3] = 1
    with pytest.raises(psfea.SolverError, match="ENODEV"):
        psfea.Hierarchy(dims, dens, 0.3, bc, device=True)
    assert psfea.Hierarchy(dims, dens, 0.3, bc).n_levels >= 1


def test_server_needs_a_device(have_gpu):
    if have_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(psfea.SolverError, match="ENODEV"):
        psfea.Server()


def test_study_loops_validate_their_inputs_then_need_a_device(have_gpu):
    """The study entry points reject invalid options with the reference's messages before they
    look for a device (topology.hpp:38-48; static_study.cpp:201)."""
    if have_gpu:
        pytest.skip("a GPU is present")
    m = W.cantilever(8, 2, 2, coarsest_max_dof=1100)
    fill = np.ones(8 * 2 * 2, np.float32)
    with pytest.raises(ValueError, match="invalid topology options"):
        psfea.topology_run(m.dims, fill, m.nu, m.bc, m.f, vol_frac=0)
    with pytest.raises(ValueError, match="invalid topology options"):
        psfea.topology_run(m.dims, fill, m.nu, m.bc, m.f, rmin=-1)
    with pytest.raises(psfea.SolverError, match="ENODEV"):
        psfea.topology_run(m.dims, fill, m.nu, m.bc, m.f, max_iter=2)
    with pytest.raises(ValueError, match="Failure strength must be positive"):
        psfea.break_test(m.dims, m.density, m.nu, m.bc, m.f, 200e9, 1e-3, strength=0)
    with pytest.raises(psfea.SolverError, match="ENODEV"):
        psfea.break_test(m.dims, m.density, m.nu, m.bc, m.f, 200e9, 1e-3, strength=100e6)
