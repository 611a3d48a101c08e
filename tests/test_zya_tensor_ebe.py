"""The tensor-core element-block operator (tcgen05, TF32 with an optional 3-term split) in the
reduced-precision forms: with it on the finest level (PSFEA_EBE=1) the mixed and FP32-Krylov solves
must still match the reference's golden displacements to 1e-6 at rel. res. 1e-8, with iteration
counts near the reference's, and its smoothing step must match the CUDA-core one."""
import numpy as np
import pytest

import psfea
from conftest import golden

pytestmark = pytest.mark.gpu

MODELS = ["cantilever_64x16x16", "lbracket_32x16x16", "simp_16x8x8", "gyroid_48x48x24", "box_request_20_28"]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def make(g):
    return psfea.VoxelFEA(tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))


@pytest.mark.parametrize("split", ["1", "3"])
@pytest.mark.parametrize("name", MODELS)
def test_ebe_solves_match_reference(monkeypatch, name, split):
    g = golden(name)
    monkeypatch.setenv("PSFEA_EBE", "1")
    monkeypatch.setenv("PSFEA_EBE_SPLIT", split)
    S = make(g)
    tol = float(g["tol"])
    it_ref = int(g["iterations"])
    for prec in ("mixed", "fp32"):
        r = S.solve(g["f"], tol=tol, max_iter=3000, precision=prec)
        assert r.converged and r.residual <= 10 * tol, (prec, r.iterations, r.residual)
        assert rel(r.u, g["u"]) < (1e-6 if tol <= 1e-8 else 1e-4), (prec, rel(r.u, g["u"]))
        if prec == "mixed":
            assert abs(r.iterations - it_ref) <= max(2, 0.2 * it_ref), (r.iterations, it_ref)


def test_ebe_step_matches_cuda_core_step(monkeypatch):
    """One V-cycle of the mixed form through the public solve: a single CG iteration from the same
    start gives the same iterate with the tensor-core product as with the CUDA-core one, to the
    split's rounding (3 terms: ~1e-6; the residual after one iteration is compared)."""
    g = golden("lbracket_32x16x16")
    base = make(g)
    r0 = base.solve(g["f"], tol=1e-14, max_iter=1, precision="mixed")
    monkeypatch.setenv("PSFEA_EBE", "1")
    monkeypatch.setenv("PSFEA_EBE_SPLIT", "3")
    S = make(g)
    r1 = S.solve(g["f"], tol=1e-14, max_iter=1, precision="mixed")
    assert rel(r1.u, r0.u) < 1e-5
    assert abs(r1.residual - r0.residual) <= 1e-4 * r0.residual
