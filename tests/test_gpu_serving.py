"""Serving (ps_server_*): requests submitted together run concurrently on the GPU, admitted by
device-memory footprint; every result equals the same model solved alone through ps_fea_solve
(same kernels, launch shapes and deterministic reductions: bit-identical), and the memory budget
is honoured."""
import numpy as np
import pytest

import oracle
import psfea
import voxel_models as W

pytestmark = pytest.mark.gpu


def requests(n, seed=17):
    return [W.box_with_voids(W.Rng(seed * 7919 + q), lo=12, hi=36) for q in range(n)]


@pytest.mark.parametrize("precision", ["mixed", "fp64", "fp32"])
def test_results_identical_alone_and_in_the_mix(precision):
    models = requests(8)
    srv = psfea.Server(max_active=8, build_threads=4)
    ids = [srv.submit(m.dims, m.density, m.nu, m.bc, m.f, tol=1e-8, precision=precision, coarsest_max_dof=300) for m in models]
    out = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == len(models)
    for m, r in zip(models, out):
        assert r["status"] == psfea.PS_OK and r["converged"], r
        alone = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, 300).solve(m.f, tol=1e-8, max_iter=5000, precision=precision)
        assert alone.iterations == r["iterations"]
        assert np.array_equal(alone.u, r["u"])
        assert r["total_s"] >= r["solve_s"] >= 0


def test_budget_admits_one_at_a_time():
    models = requests(4, seed=3)
    srv = psfea.Server(budget_bytes=1, max_active=8, build_threads=2)  # every request is oversized: each runs alone
    ids = [srv.submit(m.dims, m.density, m.nu, m.bc, m.f, tol=1e-6) for m in models]
    out = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    assert all(r["converged"] for r in out)
    assert stats["peak_active"] == 1 and stats["device_bytes_in_use"] == 0


def test_bad_request_fails_alone():
    m = requests(1, seed=5)[0]
    srv = psfea.Server(max_active=4)
    bad = srv.submit(m.dims, m.density * 0 + 2.0, m.nu, m.bc, m.f)  # density above one
    good = srv.submit(m.dims, m.density, m.nu, m.bc, m.f, tol=1e-6)
    rb, rg = srv.wait(bad), srv.wait(good)
    srv.close()
    assert rb["status"] == psfea.PS_EINVAL
    assert rg["converged"]


def test_served_stream_requests_match_the_reference_solver():
    """Requests drawn like the serving stream's (boxes with spherical voids, the three materials,
    one face held, a traction on the opposite one; 24-56 voxels per axis here), served with the
    bench's mixed form and with the drop-in, against the reference's own VoxelFEA::solve (compiled
    from its sources) on the same arrays: the level-0 fixed mask bit-exact, the displacements
    within 1e-6 relative L2 with both solvers driven to rel. res. 1e-10, the FP64-Krylov iteration
    counts within 15 % of the reference's."""
    models = [W.box_with_voids(W.Rng(5 * 1000003 + q), lo=24, hi=56) for q in range(4)]
    out = {}
    for precision in ("mixed", "fp64"):
        srv = psfea.Server(max_active=4, build_threads=2)
        ids = [srv.submit(m.dims, m.density, m.nu, m.bc, m.f, tol=1e-10, max_iter=5000, precision=precision, coarsest_max_dof=300)
               for m in models]
        out[precision] = [srv.wait(i) for i in ids]
        srv.close()
    for q, m in enumerate(models):
        ref = oracle.OracleModel("reference", m.dims, m.density, m.nu, m.bc, 300)
        u_ref, it_ref, res_ref, conv_ref = ref.solve(m.f, 1e-10, 5000)
        S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, 300)
        np.testing.assert_array_equal(S.fixed(0), ref.fixed(0))
        S.close()
        for precision in ("mixed", "fp64"):
            r = out[precision][q]
            assert r["status"] == psfea.PS_OK and r["converged"], (q, precision, r["status"])
            err = float(np.linalg.norm(r["u"] - u_ref) / np.linalg.norm(u_ref))
            assert err <= 1e-6, (q, m.dims, precision, err, r["iterations"], it_ref, res_ref, conv_ref)
            assert abs(r["iterations"] - it_ref) <= 0.15 * it_ref + 1, (q, precision, r["iterations"], it_ref)
        ref.close()
