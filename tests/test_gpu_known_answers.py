"""The reference's known-answer tests for the solve (native/tests/test_fea.cpp, test_gpu.cpp,
test/fea.test.js), run on the CUDA path through the C ABI: beam theory for the clamped bar, the
mid-span bending stress, the principal stresses of a known tensor through the stress recovery,
the reaction of loads put directly on held nodes, the GPU solve against the CPU solver, and a
zero load after a warm start."""
import numpy as np
import pytest

import known_answers as KA
import oracle
import psfea

pytestmark = pytest.mark.gpu

E, NU = 200e9, 0.3


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
@pytest.mark.parametrize("n", [2, 4, 8])
def test_cantilever_against_beam_theory(n, precision):
    """test_fea.cpp:91-100: tip within 6% of Timoshenko, reaction 100 N within 0.1%; every
    precision form, at the reference's tolerance 1e-7 (its iteration cap of 500 for the FP64
    Krylov forms)."""
    dims, density, bc, f, h = KA.beam(n)
    S = psfea.VoxelFEA(dims, density, NU, bc)
    r = S.solve(f, tol=1e-7, max_iter=500 if precision != "fp32" else 3000, precision=precision)
    assert r.status == psfea.PS_OK and r.converged
    assert abs(KA.beam_tip(r.u, dims, E, h) / KA.timoshenko_tip() - 1) < 0.06
    assert abs(S.reactions(r.u)[1] - 100) < 1e-3 * 100
    if n == 8:  # test_fea.cpp:102-113: surface stress M c / I = 30 MPa at mid-span, peak near 60 MPa
        vm, _, _ = S.stresses(r.u / (E * h), E, h)
        assert abs(vm[KA.beam_mid_node(n, dims[0])] / 30e6 - 1) < 0.05
        assert 0.95 * 60e6 < vm.max() < 1.4 * 60e6


def test_large_cantilever():
    """test_fea.cpp:134-141: 200 x 20 x 20 voxels (80,000) converge; the tip stays within 6% of
    Timoshenko."""
    dims, density, bc, f, h = KA.beam(20)
    S = psfea.VoxelFEA(dims, density, NU, bc)
    r = S.solve(f, tol=1e-7, max_iter=500)
    assert r.converged
    assert abs(KA.beam_tip(r.u, dims, E, h) / KA.timoshenko_tip() - 1) < 0.06


@pytest.mark.parametrize("sigma", [KA.KNOWN_TENSOR, KA.GENERAL_TENSOR])
def test_principal_stresses_of_a_known_tensor(sigma):
    """test_fea.cpp:40-47 through the device stress recovery: the linear displacement field of a
    known uniform stress gives its von Mises and principal values at every node."""
    dims, h = (6, 5, 4), 1e-3
    bc = np.zeros((5, 6, 7, 3), np.uint8)
    bc[:, :, 0, :] = 1  # supports play no part in stress recovery
    S = psfea.VoxelFEA(dims, np.ones(120, np.float32), NU, bc.ravel())
    vm, p1, p3 = S.stresses(KA.uniform_stress_field(dims, h, sigma, E, NU), E, h)
    pr = KA.principals(sigma)
    scale = np.abs(sigma).max()
    assert np.abs(vm - KA.von_mises(sigma)).max() < 1e-6 * scale
    assert np.abs(p1 - pr[0]).max() < 1e-6 * scale and np.abs(p3 - pr[2]).max() < 1e-6 * scale


def test_reaction_includes_loads_on_held_nodes():
    """test_fea.cpp:124-132: one voxel, every DOF held, -100 N on a held DOF: no free load, a
    zero solution, and exactly (0, 100, 0) as the reaction."""
    S = psfea.VoxelFEA((1, 1, 1), np.ones(1, np.float32), NU, np.ones(24, np.uint8))
    f = np.zeros(24)
    f[1] = -100
    r = S.solve(f)
    assert r.converged and r.iterations == 0 and not r.u.any()
    assert list(S.reactions(r.u, f)) == [0, 100, 0]


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
@pytest.mark.parametrize("n", [4, 10])
def test_gpu_matches_cpu_solver(n, precision):
    """test_gpu.cpp:13-53: the clamped bar with -100 N spread evenly over the tip nodes, at rel.
    res. 1e-8: the GPU displacements within 1e-6 of the CPU solver's in the max norm."""
    dims, density, bc, _, h = KA.beam(n)
    nx = dims[0]
    NX, NY, NZ = nx + 1, n + 1, n + 1
    f = np.zeros((NZ, NY, NX, 3))
    f[:, :, nx, 1] = -100.0 / (NY * NZ)
    f = f.ravel()
    P = oracle.OracleModel("port", dims, density, NU, bc)
    a, _, _, conv = P.solve(f, 1e-8, 500)
    assert conv
    S = psfea.VoxelFEA(dims, density, NU, bc)
    r = S.solve(f, tol=1e-8, max_iter=3000, precision=precision)
    assert r.converged
    assert np.abs(r.u - a).max() / np.abs(a).max() < 1e-6


def test_zero_load_clears_a_warm_start():
    """test/fea.test.js:145-152: one voxel, the even corner nodes held, a zero load from a warm
    start of 10 everywhere: converged, every displacement exactly 0."""
    bc = np.zeros(24, np.uint8)
    for node in range(0, 8, 2):
        bc[3 * node:3 * node + 3] = 1
    S = psfea.VoxelFEA((1, 1, 1), np.ones(1, np.float32), NU, bc)
    r = S.solve(np.zeros(24), x0=np.full(24, 10.0))
    assert r.converged and np.all(r.u == 0)
