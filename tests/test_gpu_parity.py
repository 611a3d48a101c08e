"""GPU parity: the CUDA path, called through the C ABI, against the CPU oracle and the
reference's golden vectors on the same seeded inputs."""
import ctypes
import numpy as np
import pytest

import oracle
import psfea
from conftest import golden
import voxel_models as W

pytestmark = pytest.mark.gpu

MODELS = ["cantilever_32x8x8", "cantilever_64x16x16", "lbracket_32x16x16", "simp_16x8x8", "lbracket_24x12x12_loose", "gyroid_48x48x24",
          "box_request_20_28"]
U_TOL = 1e-6   # displacement relative L2 against the reference


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def make(g):
    return psfea.VoxelFEA(tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))


@pytest.mark.parametrize("name", MODELS)
def test_apply_fp64_every_level(name):
    g = golden(name)
    S = make(g)
    assert rel(S.apply(g["apply_x"]), g["apply_y"]) < 1e-13
    assert rel(S.apply(g["apply_x"], raw=True), g["apply_y_raw"]) < 1e-13
    P = oracle.OracleModel("port", tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    rng = np.random.default_rng(1)
    for l in range(S.n_levels):
        x = rng.standard_normal(S.level_info(l)["nDof"])
        assert rel(S.apply(x, level=l), P.apply(x, level=l)) < 1e-12
        assert np.array_equal(S.fixed(l), P.fixed(l))


@pytest.mark.parametrize("name", MODELS)
@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32", "half"])
def test_solve_matches_reference(name, precision):
    g = golden(name)
    S = make(g)
    tol = float(g["tol"])
    r = S.solve(g["f"], tol=tol, max_iter=3000, precision=precision)
    assert r.status == psfea.PS_OK and r.converged
    assert r.residual <= 10 * tol
    # an independent FP64 check of the residual with the oracle's operator
    P = oracle.OracleModel("port", tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    fixed = P.fixed(0).astype(bool)
    res = g["f"] - P.apply(r.u)
    res[fixed] = 0
    ff = np.where(fixed, 0, g["f"])
    assert np.linalg.norm(res) / np.linalg.norm(ff) <= 10 * tol
    assert rel(r.u, g["u"]) < (U_TOL if tol <= 1e-8 else 1e-4)
    if precision in ("fp64", "mixed"):  # the FP64 Krylov recurrence: the reference's iteration count
        it = int(g["iterations"])
        assert abs(r.iterations - it) <= max(2, 0.15 * it)
    assert np.all(r.u[fixed] == 0)


@pytest.mark.parametrize("name", MODELS[:3])
def test_stresses_and_reactions(name):
    g = golden(name)
    S = make(g)
    E, h = float(g["E"]), float(g["h"])
    vm, p1, p3 = S.stresses(g["u"] / (E * h), E, h)
    assert rel(vm, g["vm"]) < 1e-6 and rel(p1, g["p1"]) < 1e-6 and rel(p3, g["p3"]) < 1e-6
    vm2, n1, n3 = S.stresses(g["u"] / (E * h), E, h, principals=False)
    assert np.array_equal(vm, vm2) and n1 is None
    R = S.reactions(g["u"], g["f"])
    assert np.abs(R - g["reactions"]).max() <= 1e-6 * max(1.0, np.abs(g["reactions"]).max())


def test_precondition_close_to_oracle_and_linear():
    g = golden("lbracket_32x16x16")
    S = make(g)
    P = oracle.OracleModel("port", tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    r = P.apply(g["apply_x"])
    z = S.precondition(r)
    zo = P.precondition(r)
    # one FP32 V-cycle, different summation order: measured on a B200 6.8e-6 against the reference's
    # own V-cycle and 1.9e-5 against the restatement on this model (the golden models: 2e-6 - 9.5e-5)
    assert rel(z, zo) < 1e-4
    R = oracle.OracleModel("reference", tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    assert rel(z, R.precondition(r)) < 1e-4
    # r is scaled by 1 / max|r| before the FP32 cycle: scaling by 2 is exact
    assert np.array_equal(S.precondition(2 * r), 2 * z)
    assert np.allclose([S.lmax(l) for l in range(S.n_levels - 1)], g["lmax"], rtol=1e-9)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32", "half"])
def test_solve_after_other_calls_on_the_handle(precision):
    """Calls made before a solve on the same handle (product, preconditioner, stresses, reactions,
    a warm-started solve) must leave nothing behind that changes the solve: same iterations and
    bitwise the same displacements as on a fresh handle."""
    g = golden("gyroid_48x48x24")
    fresh = make(g).solve(g["f"], tol=1e-8, max_iter=3000, precision=precision)
    S = make(g)
    x = np.random.default_rng(5).standard_normal(S.n_dof) * 1e3
    S.apply(x)
    S.apply(x, raw=True)
    S.precondition(x)
    E, h = float(g["E"]), float(g["h"])
    S.stresses(x, E, h)
    S.reactions(x, g["f"])
    S.solve(g["f"], tol=1e-3, max_iter=3000, x0=x, precision=precision)
    r = S.solve(g["f"], tol=1e-8, max_iter=3000, precision=precision)
    assert r.converged and r.iterations == fresh.iterations
    assert np.array_equal(r.u, fresh.u)
    assert rel(r.u, g["u"]) < U_TOL


def test_warm_start_zero_load_and_errors():
    g = golden("cantilever_32x8x8")
    S = make(g)
    r = S.solve(g["f"], tol=1e-8, max_iter=3000, x0=g["u"])
    assert r.converged and r.iterations <= 1
    z = S.solve(np.zeros_like(g["f"]), tol=1e-8, x0=g["u"])
    assert z.converged and not z.u.any() and z.iterations == 0  # voxel_fea.cpp:880-884
    bad = g["f"].copy()
    bad[5] = np.nan
    with pytest.raises(ValueError, match="finite"):
        S.solve(bad)
    with pytest.raises(ValueError, match="wrong size"):
        S.solve(g["f"][:-3])
    few = S.solve(g["f"], tol=1e-12, max_iter=3)
    assert few.status == psfea.PS_NOT_CONVERGED and few.iterations == 3 and not few.converged


def test_cancel_flag():
    g = golden("cantilever_64x16x16")
    S = make(g)
    flag = ctypes.c_int32(1)
    r = S.solve(g["f"], tol=1e-12, max_iter=3000, cancel=flag)
    assert r.status == psfea.PS_CANCELLED and not r.converged


def test_mechanism_does_not_hang():
    """No supports at all: K is singular; the solve must end (breakdown or the cap), not hang."""
    m = W.cantilever(8, 4, 4)
    bc = np.zeros_like(m.bc)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, bc, 100)
    r = S.solve(m.f, tol=1e-10, max_iter=200)
    assert r.status in (psfea.PS_BREAKDOWN, psfea.PS_NOT_CONVERGED, psfea.PS_OK)


def test_bitwise_reproducible():
    g = golden("lbracket_32x16x16")
    S = make(g)
    a = S.solve(g["f"], tol=1e-8, max_iter=3000)
    b = S.solve(g["f"], tol=1e-8, max_iter=3000)
    assert np.array_equal(a.u, b.u) and a.iterations == b.iterations


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_pointer_solve_on_a_caller_stream(precision):
    """ps_fea_solve_dev with f, x0 and u in the caller's device memory (the reference's dense
    layout), on the caller's stream: the same iterations and bitwise the same displacements as
    the host-buffer solve."""
    import torch

    g = golden("lbracket_32x16x16")
    S = make(g)
    host = S.solve(g["f"], tol=1e-8, max_iter=3000, precision=precision)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    S.set_stream(stream.cuda_stream)
    f = torch.from_numpy(g["f"]).to(dev)
    u = torch.full_like(f, float("nan"))
    r = S.solve_dev(f.data_ptr(), u.data_ptr(), tol=1e-8, max_iter=3000, precision=precision)
    torch.cuda.synchronize()
    assert r.converged and r.iterations == host.iterations
    assert np.array_equal(u.cpu().numpy(), host.u)
    # a warm start from the solution, also in device memory
    u2 = torch.zeros_like(f)
    r2 = S.solve_dev(f.data_ptr(), u2.data_ptr(), tol=1e-8, max_iter=3000, precision=precision, x0_ptr=u.data_ptr())
    torch.cuda.synchronize()
    assert r2.converged and r2.iterations <= 1
    assert rel(u2.cpu().numpy(), host.u) < 1e-8
    S.set_stream(0)


def test_solve_batch_contexts_match_single(monkeypatch):
    """The batch as concurrent single-solve contexts (the FP32-Krylov form's batch, and any form's
    with PSFEA_BATCH_MODE=contexts): each result is the single solve's."""
    monkeypatch.setenv("PSFEA_BATCH_MODE", "contexts")
    m = W.simp(16, 8, 8, nrhs=3)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc)
    rs = S.solve_batch(m.f, tol=1e-8, max_iter=3000)
    for q in range(3):
        one = S.solve(m.f[q], tol=1e-8, max_iter=3000)
        assert rs[q].converged and rel(rs[q].u, one.u) < 1e-12


def test_full_size_l_bracket_residual():
    """The benchmark model itself (256x128x128, 12.8 M DOF): every precision reaches rel. res.
    1e-8 by the oracle's own FP64 operator. The model is ill-conditioned (the holes leave thin
    ligaments), so a residual of 1e-8 pins the displacements only to ~3e-4 (measured on a B200 for
    all forms); the solutions are compared with an FP64 solve driven to 1e-11, and the reduced-
    precision ones must be as close to it as the plain FP64 one (within 3x)."""
    m = W.l_bracket()
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    fixed = P.fixed(0).astype(bool)
    ff = np.where(fixed, 0, m.f)
    truth = S.solve(m.f, tol=1e-11, max_iter=8000, precision="fp64")
    assert truth.converged
    err = {}
    for prec in ("fp64", "mixed", "fp32"):
        r = S.solve(m.f, tol=1e-8, max_iter=8000, precision=prec)
        assert r.converged, (prec, r.iterations, r.residual)
        res = m.f - P.apply(r.u)
        res[fixed] = 0
        assert np.linalg.norm(res) / np.linalg.norm(ff) <= 1e-7
        err[prec] = rel(r.u, truth.u)
    assert err["fp64"] < 1e-3 and err["mixed"] < max(1e-4, 3 * err["fp64"]) and err["fp32"] < max(1e-4, 3 * err["fp64"]), err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_boundary_nodes_in_the_smoother(monkeypatch, precision):
    """32-bit tiles that leave their boundary nodes to the list kernel (PSFEA_TILE_SPLIT32, a bit
    per level) give the same V-cycle up to FP32 summation order, and solves that match the
    oracle. Tiles forced onto levels of any size, so levels 0 and 1 of a 128x64x64 L-bracket
    both take the tiled path."""
    m = W.l_bracket(128, 64, 64, holes=16, seed=3)
    monkeypatch.setenv("PSFEA_TILE_MIN_NODES", "0")
    monkeypatch.setenv("PSFEA_TILE_SPLIT32", "0")
    A = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    monkeypatch.setenv("PSFEA_TILE_SPLIT32", "-1")
    B = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    r = A.apply(np.random.default_rng(7).standard_normal(A.n_dof))
    za, zb = A.precondition(r), B.precondition(r)
    assert rel(zb, za) < 1e-5
    ra = A.solve(m.f, tol=1e-8, max_iter=3000, precision=precision)
    rb = B.solve(m.f, tol=1e-8, max_iter=3000, precision=precision)
    assert ra.converged and rb.converged
    assert abs(ra.iterations - rb.iterations) <= 2
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    fixed = P.fixed(0).astype(bool)
    res = m.f - P.apply(rb.u)
    res[fixed] = 0
    assert np.linalg.norm(res) / np.linalg.norm(np.where(fixed, 0, m.f)) <= 1e-7
    assert rel(rb.u, ra.u) < 1e-5


@pytest.mark.parametrize("model,precision", [("gyroid", "fp64"), ("gyroid", "fp32"), ("simp", "fp64"), ("simp", "fp32"),
                                             ("lbracket", "mixed")])
def test_assembled_stencils_on_every_galerkin_level(monkeypatch, model, precision):
    """The assembled stencils of the Galerkin levels (FP32 in the FP64-Krylov forms, FP16 in the
    FP32-Krylov ones), forced onto every level >= 1 whatever its size and on both the untiled levels
    (every active node) and a split tiled level (its boundary nodes), against the per-voxel gather
    (PSFEA_STENCIL_LEVELS=0): the same solution to the solve tolerance, iteration counts within 15 %,
    and a true FP64 residual by the oracle's operator."""
    m = {"gyroid": lambda: W.gyroid(64, 64, 32), "simp": lambda: W.simp(32, 16, 16, nrhs=1),
         "lbracket": lambda: W.l_bracket(128, 64, 64, holes=16, seed=3)}[model]()
    f = m.f if m.f.ndim == 1 else m.f[0]
    monkeypatch.setenv("PSFEA_TILE_MIN_NODES", "20000")  # level 1 of the L-bracket tiled (and split)
    monkeypatch.setenv("PSFEA_STENCIL_LEVELS", "0")
    A = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    monkeypatch.setenv("PSFEA_STENCIL_LEVELS", "-1")
    monkeypatch.setenv("PSFEA_STENCIL_MIN_NODES", "1")
    B = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    ra = A.solve(f, tol=1e-8, max_iter=3000, precision=precision)
    rb = B.solve(f, tol=1e-8, max_iter=3000, precision=precision)
    assert ra.converged and rb.converged, (ra.iterations, rb.iterations)
    assert abs(ra.iterations - rb.iterations) <= max(2, 0.15 * ra.iterations), (ra.iterations, rb.iterations)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    fixed = P.fixed(0).astype(bool)
    res = f - P.apply(rb.u)
    res[fixed] = 0
    assert np.linalg.norm(res) / np.linalg.norm(np.where(fixed, 0, f)) <= 1e-7
    assert rel(rb.u, ra.u) < 1e-5
    # the stencils are made once per model and form: a second solve repeats the first bitwise
    rc = B.solve(f, tol=1e-8, max_iter=3000, precision=precision)
    assert rc.iterations == rb.iterations and np.array_equal(rc.u, rb.u)


def test_solve_into_a_pinned_caller_buffer():
    """solve(out=...) writes u into the caller's array (here pinned host memory) and returns it:
    bitwise the same as a solve into a new array; a buffer of the wrong type is refused."""
    import torch

    g = golden("cantilever_32x8x8")
    S = make(g)
    a = S.solve(g["f"], tol=1e-8, max_iter=3000)
    buf = torch.empty(S.n_dof, dtype=torch.float64, pin_memory=True).numpy()
    b = S.solve(g["f"], tol=1e-8, max_iter=3000, out=buf)
    assert b.u is buf and np.array_equal(buf, a.u) and b.iterations == a.iterations
    with pytest.raises(ValueError, match="out"):
        S.solve(g["f"], out=np.zeros(S.n_dof, np.float32))


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_one_device_copy_per_class_of_galerkin_matrices(monkeypatch, precision):
    """One device copy per class of bitwise-equal Galerkin matrices (the default; PSFEA_OWN_DEDUP=0
    uploads one per voxel, as the host holds them) (the
    gyroid's and the L-bracket's coarse levels hold tens to hundreds of distinct ones among
    thousands) and points the voxel words at them: the operator on every level and the solves are
    bitwise the same, in less device memory. The tiled L-bracket puts level 1 (own matrices) on
    the tiles and the boundary-node list kernel."""
    g = golden("gyroid_48x48x24")
    tiled = W.l_bracket(128, 64, 64, holes=16, seed=3)
    cases = [(lambda: make(g), g["f"], {}),
             (lambda: psfea.VoxelFEA(tiled.dims, tiled.density, tiled.nu, tiled.bc, tiled.coarsest_max_dof), tiled.f,
              {"PSFEA_TILE_MIN_NODES": "0"})]
    rng = np.random.default_rng(3)
    for build, f, env in cases:
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        monkeypatch.setenv("PSFEA_OWN_DEDUP", "0")
        A = build()
        monkeypatch.setenv("PSFEA_OWN_DEDUP", "1")
        B = build()
        assert B.device_bytes < A.device_bytes
        for l in range(A.n_levels):
            x = rng.standard_normal(A.level_info(l)["nDof"])
            assert np.array_equal(A.apply(x, level=l), B.apply(x, level=l))
        r = A.apply(rng.standard_normal(A.n_dof))
        assert np.array_equal(A.precondition(r), B.precondition(r))
        ra = A.solve(f, tol=1e-8, max_iter=3000, precision=precision)
        rb = B.solve(f, tol=1e-8, max_iter=3000, precision=precision)
        assert ra.converged and rb.iterations == ra.iterations and np.array_equal(ra.u, rb.u)
        for k in env:
            monkeypatch.delenv(k)
