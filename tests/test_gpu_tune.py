"""Autotuning on the GPU: the chosen configuration is one of the candidates, solves with it still
match the oracle, the process's cache serves a second model with the same signature without
trials, and ps_fea_create_tuned returns a working handle for one of the coarsening depths."""
import numpy as np
import pytest

import oracle
import psfea
import voxel_models as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_autotune_chooses_a_candidate_and_keeps_parity(monkeypatch):
    monkeypatch.setenv("PSFEA_TILE_MIN_NODES", "0")  # tiled levels even on a small model: the tile flags are tuned too
    m = W.l_bracket(64, 32, 32, holes=4, seed=9)
    S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    t = S.autotune(m.f, tol=1e-8, force=True)
    assert 1 <= t["smoother_degree"] <= 4 and t["trials"] >= 5 and not t["cached"]
    assert 0 < t["best_seconds"] <= t["default_seconds"]
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    uo, _, _, _ = P.solve(m.f, 1e-10, 5000)
    for prec in ("fp64", "mixed"):
        r = S.solve(m.f, tol=1e-10, max_iter=5000, precision=prec)  # the tuned degree (smoother_degree left at 0)
        assert r.converged and rel(r.u, uo) < 1e-6
    # the same model again: the cached choice, no trials
    S2 = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    t2 = S2.autotune(m.f, tol=1e-8)
    assert t2["cached"] and t2["trials"] == 0
    assert (t2["smoother_degree"], t2["split_levels"], t2["inner64"]) == (t["smoother_degree"], t["split_levels"], t["inner64"])


def test_create_tuned_picks_a_depth():
    m = W.cantilever(48, 12, 12, coarsest_max_dof=1100)
    S, t = psfea.VoxelFEA.create_tuned(m.dims, m.density, m.nu, m.bc, m.f, tol=1e-8, force=True)
    assert t["coarsest_max_dof"] in (300, 1100, 3000)
    P = oracle.OracleModel("port", m.dims, m.density, m.nu, m.bc, int(t["coarsest_max_dof"]))
    assert S.n_levels == P.n_levels
    uo, _, _, _ = P.solve(m.f, 1e-10, 5000)
    r = S.solve(m.f, tol=1e-10, max_iter=5000)
    assert r.converged and rel(r.u, uo) < 1e-6
