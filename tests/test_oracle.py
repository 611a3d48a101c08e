"""The CPU oracle (oracle/psoracle.cpp) pinned against the reference's golden vectors
(tests/golden/, written by the reference itself) and, where oracle/_ref is built, against the
reference run side by side."""
import numpy as np
import pytest

import oracle
import known_answers as KA
from conftest import golden
import voxel_models as W

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
    # the Gauss-point strain matrices reproduce the condensed stiffness (test_fea.cpp:24-38):
    # K = sum over the 8 points of B^T D B / 8, D the isotropic elasticity matrix for E = 1
    lam, mu = nu / ((1 + nu) * (1 - 2 * nu)), 1 / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    Ks = sum(B.T @ D @ B for B in gb) / 8
    assert np.abs(Ks - K).max() < 1e-12 * np.abs(K).max()
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


@pytest.mark.parametrize("n", [2, 4, 8])
def test_cantilever_against_beam_theory(n):
    """native/tests/test_fea.cpp:91-100: n = 2, 4, 8 through the thickness, tip within 6% of
    Timoshenko, reaction 100 N within 0.1%."""
    dims, density, bc, f, h = KA.beam(n)
    M = oracle.OracleModel("port", dims, density, 0.3, bc)
    u, it, res, conv = M.solve(f, 1e-7, 500)
    assert conv
    assert abs(KA.beam_tip(u, dims, 200e9, h) / KA.timoshenko_tip() - 1) < 0.06
    assert abs(M.reactions(u)[1] - 100) < 0.1
    if n == 8:  # test_fea.cpp:102-113: mid-span surface stress M c / I = 30 MPa, peak near 60 MPa
        vm, _, _ = M.stresses(u / (200e9 * h), 200e9, h)
        assert abs(vm[KA.beam_mid_node(n, dims[0])] / 30e6 - 1) < 0.05
        assert 0.95 * 60e6 < vm.max() < 1.4 * 60e6


@pytest.mark.parametrize("sigma", [KA.KNOWN_TENSOR, KA.GENERAL_TENSOR])
def test_principal_stresses_of_a_known_tensor(sigma):
    """test_fea.cpp:40-47 through the stress recovery: a linear displacement field with the
    known uniform stress gives that stress's von Mises and principal values at every node."""
    dims, E, nu, h = (6, 5, 4), 200e9, 0.3, 1e-3
    bc = np.zeros((5, 6, 7, 3), np.uint8)
    bc[:, :, 0, :] = 1  # supports play no part in stress recovery
    M = oracle.OracleModel("port", dims, np.ones(120, np.float32), nu, bc.ravel())
    vm, p1, p3 = M.stresses(KA.uniform_stress_field(dims, h, sigma, E, nu), E, h)
    pr = KA.principals(sigma)
    if sigma is KA.KNOWN_TENSOR:
        assert np.allclose(pr, KA.KNOWN_PRINCIPALS, rtol=0, atol=1e-3)
    scale = np.abs(sigma).max()
    assert np.abs(vm - KA.von_mises(sigma)).max() < 1e-6 * scale
    assert np.abs(p1 - pr[0]).max() < 1e-6 * scale and np.abs(p3 - pr[2]).max() < 1e-6 * scale


def test_reaction_includes_loads_on_held_nodes():
    """test_fea.cpp:124-132: one voxel, every DOF held, -100 N on a held DOF: the reaction is
    exactly (0, 100, 0)."""
    M = oracle.OracleModel("port", (1, 1, 1), np.ones(1, np.float32), 0.3, np.ones(24, np.uint8))
    f = np.zeros(24)
    f[1] = -100
    u, it, res, conv = M.solve(f, 1e-6, 500)
    assert conv and not u.any()
    assert list(M.reactions(u, f)) == [0, 100, 0]


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
