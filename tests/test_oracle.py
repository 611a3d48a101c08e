"""The CPU oracle (oracle/psoracle.cpp) pinned against the reference's golden vectors
(tests/golden/, written by the reference itself) and, where oracle/_ref is built, against the
reference run side by side."""
import numpy as np
import pytest

import oracle
from conftest import golden
from psfea import workloads as W

MODELS = ["cantilever_32x8x8", "cantilever_64x16x16", "lbracket_32x16x16", "simp_16x8x8", "lbracket_24x12x12_loose", "gyroid_48x48x24",
          "box_request_20_28"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("nu", [0.3, 0.33, 0.34, 0.36])
def test_element_matches_reference(nu):
    g = golden("element")
    K, cs, gb = oracle.element("port", nu)
    Kr = g[f"K_{nu}"]
    assert np.abs(K - Kr).max() <= 1e-14 * np.abs(Kr).max()
    assert np.array_equal(K, K.T)  # exact symmetry (native/tests/test_fea.cpp:20-21)
    for d in range(3):  # rigid-body translations (native/tests/test_fea.cpp:14-19)
        assert np.abs(K[:, d::3].sum(axis=1)).max() < 1e-12
    if nu == 0.3:
        assert np.abs(cs - g["cornerStress_0.3"]).max() <= 1e-14 * np.abs(cs).max()
        assert np.abs(gb - g["gaussB_0.3"]).max() <= 1e-14 * np.abs(gb).max()
        Kt, _, _ = oracle.element("port", 0.3, modes=False)
        assert np.abs(Kt - g["K_trilinear_0.3"]).max() <= 1e-14 * np.abs(Kt).max()


def test_element_rejects_bad_nu():
    for nu in (0.5, -1.0, float("nan")):
        with pytest.raises(ValueError):
            oracle.element("port", nu)


def test_prune_matches_reference():
    g = golden("prune")
    o1, r1 = oracle.prune("port", (4, 1, 1), g["d1"], g["h1"])
    assert np.array_equal(o1, g["o1"]) and r1 == int(g["r1"]) == 1
    o2, r2 = oracle.prune("port", tuple(g["dims2"]), g["d2"], g["h2"])
    assert np.array_equal(o2, g["o2"]) and r2 == int(g["r2"])


def _model(g):
    return oracle.OracleModel("port", tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))


@pytest.mark.parametrize("name", MODELS)
def test_hierarchy_bit_exact(name):
    g = golden(name)
    M = _model(g)
    assert M.n_levels == int(g["levels"])
    for l in range(M.n_levels):
        info = M.level_info(l)
        assert [info[k] for k in ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")] == list(g[f"info_{l}"])
        assert np.array_equal(np.packbits(M.fixed(l)), g[f"fixed_{l}"])
        assert np.array_equal(M.kidx(l), g[f"kidx_{l}"])
        assert np.array_equal(M.elems(l), g[f"elems_{l}"])


@pytest.mark.parametrize("name", MODELS)
def test_apply_and_solve_match_reference(name):
    g = golden(name)
    M = _model(g)
    y = M.apply(g["apply_x"])
    assert rel(y, g["apply_y"]) < 1e-13
    assert rel(M.apply(g["apply_x"], raw=True), g["apply_y_raw"]) < 1e-13
    tol = float(g["tol"])
    u, it, res, conv = M.solve(g["f"], tol, 3000)
    assert conv and res <= 10 * tol
    assert abs(it - int(g["iterations"])) <= 2
    assert rel(u, g["u"]) < 1e-6
    M.prepare()
    assert np.allclose([M.lmax(l) for l in range(M.n_levels - 1)], g["lmax"], rtol=1e-10)
    E, h = float(g["E"]), float(g["h"])
    vm, p1, p3 = M.stresses(u / (E * h), E, h)
    assert rel(vm, g["vm"]) < 1e-5 and rel(p1, g["p1"]) < 1e-5 and rel(p3, g["p3"]) < 1e-5
    R = M.reactions(u, g["f"])
    assert np.abs(R - g["reactions"]).max() <= 1e-6 * max(1.0, np.abs(g["reactions"]).max())


def test_cantilever_against_beam_theory():
    """native/tests/test_fea.cpp:59-100: n = 4 through the thickness, tip within 6% of
    Timoshenko, reaction 100 N within 0.1%."""
    n, Lm, b, F, E, nu = 4, 0.1, 0.01, 100.0, 200e9, 0.3
    h = b / n
    nx = int(round(Lm / h))
    NX, NY, NZ = nx + 1, n + 1, n + 1
    density = np.ones(nx * n * n, np.float32)
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    bc[:, :, 0, :] = 1
    f = np.zeros((NZ, NY, NX, 3))
    w = np.ones(n + 1)
    w[0] = w[-1] = 0.5
    f[:, :, nx, 1] = -F * np.outer(w, w) / (n * n)
    M = oracle.OracleModel("port", (nx, n, n), density, nu, bc.ravel(), 1100)
    u, it, res, conv = M.solve(f.ravel(), 1e-7, 500)
    assert conv
    tip = (u.reshape(NZ, NY, NX, 3)[:, :, nx, 1] / (E * h)).mean()
    I, G = b ** 4 / 12, E / (2 * (1 + nu))
    expected = -F * Lm ** 3 / (3 * E * I) - F * Lm / ((5 / 6) * G * b * b)
    assert abs(tip / expected - 1) < 0.06
    assert abs(M.reactions(u)[1] - 100) < 0.1


@pytest.mark.skipif(not oracle.available("reference"), reason="oracle/_ref not built here")
def test_port_against_reference_side_by_side():
    m = W.l_bracket(40, 20, 20, holes=4, seed=11)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc)
    R = oracle.OracleModel("reference", m.dims, m.density, m.nu, m.bc)
    for l in range(R.n_levels):
        assert np.array_equal(P.fixed(l), R.fixed(l))
        if R.level_info(l)["nOwn"]:
            assert np.abs(P.own(l) - R.own(l)).max() <= 1e-6 * np.abs(R.own(l)).max()
    up, itp, rp, _ = P.solve(m.f, 1e-8, 3000)
    ur, itr, rr, _ = R.solve(m.f, 1e-8, 3000)
    # the FP32 V-cycle rounds differently, so long runs drift by a few iterations
    assert rel(up, ur) < 1e-6 and abs(itp - itr) <= max(3, 0.15 * itr)
