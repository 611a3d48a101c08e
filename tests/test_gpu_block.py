"""Block (multi-RHS) solves and block preconditioning on the GPU.

ps_fea_solve_batch runs the FP64-Krylov forms in blocks of up to 32 right-hand sides whose kernels
take the whole block; every right-hand side must reach the result of its own single solve (and of
the oracle) with the same tolerance as single solves, converge on its own, and keep its own
iteration count. ps_fea_precondition_block must give each vector the single-vector V-cycle up to
FP32 summation order."""
import numpy as np
import pytest

import oracle
import psfea
import voxel_models as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def random_loads(m, nrhs, seed):
    """nrhs load vectors: each a random direction times the model's own load pattern magnitude,
    spread over the loaded nodes of m.f (or of its first right-hand side)"""
    base = m.f if m.f.ndim == 1 else m.f[0]
    mag = np.linalg.norm(base.reshape(-1, 3), axis=1)
    rng = np.random.default_rng(seed)
    F = np.zeros((nrhs, base.size))
    for q in range(nrhs):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        F[q] = (mag[:, None] * d[None, :]).ravel()
    return F


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_block_matches_single_and_oracle(precision):
    m = W.simp(16, 8, 8, nrhs=5)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    rs = S.solve_batch(m.f, tol=1e-8, max_iter=3000, precision=precision)
    for q in range(5):
        one = S.solve(m.f[q], tol=1e-8, max_iter=3000, precision=precision)
        uo, ito, _, _ = P.solve(m.f[q], 1e-8, 3000)
        assert rs[q].converged and rs[q].residual <= 1e-7, (q, rs[q])
        assert rel(rs[q].u, uo) < 1e-6 and rel(rs[q].u, one.u) < 1e-6, q
        assert abs(rs[q].iterations - one.iterations) <= max(2, 0.15 * one.iterations)
        assert abs(rs[q].iterations - ito) <= max(2, 0.15 * ito)


@pytest.mark.parametrize("nrhs", [12, 40])
def test_block_widths_and_remainders(nrhs):
    """12 right-hand sides: one 16-wide block; 40: a 32-wide block and a remainder of 8 in it.
    The L-bracket exercises uniform (stencil) nodes, boundary nodes and Galerkin levels."""
    m = W.l_bracket(64, 32, 32, holes=6, seed=4)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    F = random_loads(m, nrhs, seed=nrhs)
    rs = S.solve_batch(F, tol=1e-8, max_iter=3000, precision="fp64")
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    fixed = P.fixed(0).astype(bool)
    for q in (0, nrhs // 2, nrhs - 1):
        one = S.solve(F[q], tol=1e-8, max_iter=3000, precision="fp64")
        assert rs[q].converged
        # the true residual by the oracle's operator
        res = F[q] - P.apply(rs[q].u)
        res[fixed] = 0
        assert np.linalg.norm(res) / np.linalg.norm(np.where(fixed, 0, F[q])) <= 1e-7
        assert rel(rs[q].u, one.u) < 1e-5, q
        assert abs(rs[q].iterations - one.iterations) <= max(2, 0.15 * one.iterations)
    assert all(r.converged for r in rs)


def test_block_zero_load_warm_start_and_cap():
    """A zero right-hand side gives exact zeros (after a warm start, too); the others are unaffected;
    an iteration cap stops every right-hand side with NOT_CONVERGED and a true residual."""
    m = W.cantilever(32, 8, 8, coarsest_max_dof=1100)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    F = np.stack([m.f, np.zeros_like(m.f), 2 * m.f])
    x0 = np.stack([np.zeros_like(m.f), np.ones_like(m.f), np.zeros_like(m.f)])
    rs = S.solve_batch(F, tol=1e-10, max_iter=3000, X0=x0)
    assert np.all(rs[1].u == 0) and rs[1].converged and rs[1].iterations == 0
    assert rel(rs[2].u, 2 * rs[0].u) < 1e-8
    one = S.solve(m.f, tol=1e-10, max_iter=3000)
    assert rel(rs[0].u, one.u) < 1e-8
    capped = S.solve_batch(F[[0, 2]], tol=1e-12, max_iter=3)
    for r in capped:
        assert r.status == psfea.PS_NOT_CONVERGED and r.iterations == 3 and 0 < r.residual < 1


def test_block_single_level_model():
    """A model small enough to be its own coarsest level: the block's direct FP64 solve."""
    m = W.cantilever(4, 2, 2, coarsest_max_dof=1100)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    assert S.n_levels == 1
    F = np.stack([m.f, -3 * m.f])
    rs = S.solve_batch(F, tol=1e-10, max_iter=100)
    one = S.solve(m.f, tol=1e-10, max_iter=100)
    assert rel(rs[0].u, one.u) < 1e-10 and rel(rs[1].u, -3 * one.u) < 1e-10


def test_precondition_block_matches_single():
    """Each vector of the block gets the single-vector preconditioner (the same V-cycle; the FP32
    sums run in another order, so agreement is to FP32 rounding, measured ~1e-6)."""
    import torch
    m = W.l_bracket(64, 32, 32, holes=6, seed=4)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    rng = np.random.default_rng(3)
    R = np.stack([S.apply(rng.standard_normal(S.n_dof)) for _ in range(6)])
    R[2] = 0.0  # a zero vector gives z = 0
    dev = torch.device("cuda", 0)
    r_dev = torch.from_numpy(R).to(dev)
    z_dev = torch.full_like(r_dev, float("nan"))
    S.precondition_block(6, r_dev.data_ptr(), z_dev.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    Z = z_dev.cpu().numpy()
    assert np.all(Z[2] == 0)
    for k in (0, 1, 3, 5):
        z1 = S.precondition(R[k])
        assert rel(Z[k], z1) < 1e-4, (k, rel(Z[k], z1))
    # linear: scaling a vector scales its result
    r_dev[1] *= 4.0
    S.precondition_block(6, r_dev.data_ptr(), z_dev.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    assert rel(z_dev[1].cpu().numpy(), 4 * Z[1]) < 1e-12


def test_mixed_block_on_the_tensor_cores_matches_the_oracle(monkeypatch):
    """A 32-wide mixed block with PSFEA_BLOCK_TC=1 runs its finest-level V-cycle operator on the tensor cores (TF32 with
    the translation removed per voxel): every right-hand side must still match the oracle's solve to
    1e-6, with the iteration count of its CUDA-core block (PSFEA_BLOCK_TC=0) within 15 %."""
    m = W.simp(24, 12, 12, nrhs=20, seed=11)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    monkeypatch.setenv("PSFEA_BLOCK_TC", "1")
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    tc = S.solve_batch(m.f, tol=1e-8, max_iter=3000, precision="mixed")
    monkeypatch.setenv("PSFEA_BLOCK_TC", "0")
    S0 = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    cc = S0.solve_batch(m.f, tol=1e-8, max_iter=3000, precision="mixed")
    for q in range(20):
        assert tc[q].converged and tc[q].residual <= 1e-7, (q, tc[q].iterations, tc[q].residual)
        if q % 5 == 0:
            uo, _, _, _ = P.solve(m.f[q], 1e-8, 3000)
            assert rel(tc[q].u, uo) < 1e-6, q
        assert abs(tc[q].iterations - cc[q].iterations) <= max(2, 0.15 * cc[q].iterations), (q, tc[q].iterations, cc[q].iterations)
