"""Galerkin coarsening on the device against the host build.

The device engine (galerkin.cu) forms every own coarse matrix with the host loop's FP64 products and
sums in the host's order, so the hierarchies must agree bitwise: own matrices, uniform elements
and fixed masks of every level. PSFEA_DEVICE_GALERKIN_MIN=0 hands every level with own matrices to
the device (by default only levels with >= 4096 classes of child patterns go there)."""
import time

import numpy as np
import pytest

import psfea
import voxel_models as W

pytestmark = pytest.mark.gpu


def _models():
    g = W.gyroid(96, 96, 48)  # own children from level 2 on (the full two-stage product)
    return {
        "simp_48x24x24": W.simp(48, 24, 24, nrhs=1),  # graded: every coarse matrix distinct
        "gyroid_96x96x48": g,
        "l_bracket_64x32x32": W.l_bracket(64, 32, 32, holes=4),
    }


def _assert_same(a, b):
    assert a.n_levels == b.n_levels
    for l in range(a.n_levels):
        assert a.level_info(l) == b.level_info(l)
        np.testing.assert_array_equal(a.fixed(l), b.fixed(l))
        np.testing.assert_array_equal(a.kb(l), b.kb(l))
        oa, ob = a.own(l), b.own(l)
        assert oa.shape == ob.shape
        # bitwise, NaN-safe
        np.testing.assert_array_equal(oa.view(np.uint32), ob.view(np.uint32))


@pytest.mark.parametrize("name", ["simp_48x24x24", "gyroid_96x96x48", "l_bracket_64x32x32"])
def test_device_galerkin_bitwise_every_level(name, monkeypatch):
    monkeypatch.setenv("PSFEA_DEVICE_GALERKIN_MIN", "0")
    m = _models()[name]
    h = psfea.Hierarchy(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    d = psfea.Hierarchy(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof, device=True)
    assert any(h.level_info(l)["nOwn"] for l in range(h.n_levels))
    _assert_same(h, d)


def test_device_galerkin_full_size_simp():
    """The SIMP grid of the batched benchmark (192x96x96, graded densities): its levels 1 and 2 go
    to the device under the default threshold; bitwise the host's. Prints the two build times."""
    m = W.simp(nrhs=1)
    t0 = time.perf_counter()
    h = psfea.Hierarchy(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    t1 = time.perf_counter()
    d = psfea.Hierarchy(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof, device=True)
    t2 = time.perf_counter()
    _assert_same(h, d)
    print(f"SIMP 192x96x96 hierarchy: host {t1 - t0:.3f} s, device Galerkin {t2 - t1:.3f} s")


def test_solver_built_with_device_galerkin_solves_bitwise_the_same(monkeypatch):
    m = W.simp(48, 24, 24, nrhs=1)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("PSFEA_DEVICE_GALERKIN", flag)
        monkeypatch.setenv("PSFEA_DEVICE_GALERKIN_MIN", "0")
        S = psfea.VoxelFEA(m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
        out[flag] = S.solve(m.f[0], tol=1e-8, max_iter=3000, precision="fp64")
        S.close()
    a, b = out["0"], out["1"]
    assert a.converged and b.converged
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.u, b.u)
