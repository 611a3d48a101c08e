"""Models and closed-form answers of the reference's own known-answer tests for the solve
(native/tests/test_fea.cpp), shared by the oracle tests and the GPU tests."""
import numpy as np


def beam(n, Lm=0.1, b=0.01, F=100.0):
    """test_fea.cpp:58-89: a bar of length Lm along x and square section b, n voxels through the
    thickness, the x = 0 face held, a tip load F in -y spread over the x = nx face with trapezoid
    weights (1/2 on the face's edges). Returns dims, density, bc, f and the voxel size h."""
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
    return (nx, n, n), density, bc.ravel(), f.ravel(), h


def beam_tip(u, dims, E, h):
    """Mean y displacement (m) of the tip face; u in the solver's units (E = 1, h = 1)."""
    nx, ny, nz = dims
    return float((u.reshape(nz + 1, ny + 1, nx + 1, 3)[:, :, nx, 1] / (E * h)).mean())


def timoshenko_tip(Lm=0.1, b=0.01, F=100.0, E=200e9, nu=0.3):
    """Tip deflection of a clamped square bar: bending plus shear with k = 5/6 (test_fea.cpp:85-86)."""
    I, G = b ** 4 / 12, E / (2 * (1 + nu))
    return -F * Lm ** 3 / (3 * E * I) - F * Lm / ((5 / 6) * G * b * b)


def beam_mid_node(n, nx):
    """The mid-span node on the top surface (+y), half way through z (test_fea.cpp:104-105)."""
    NX, NY = nx + 1, n + 1
    return nx // 2 + NX * (n + NY * (n // 2))


def uniform_stress_field(dims, h, sigma, E, nu):
    """Physical displacements (m) of the linear field whose strain is uniform with the stress
    sigma = (sxx, syy, szz, sxy, syz, szx) in Pa: eps = C^-1 sigma, u = eps x. Trilinear hex8
    elements reproduce a linear field exactly, so every node's stress is sigma."""
    sxx, syy, szz, sxy, syz, szx = sigma
    G = E / (2 * (1 + nu))
    exx = (sxx - nu * (syy + szz)) / E
    eyy = (syy - nu * (szz + sxx)) / E
    ezz = (szz - nu * (sxx + syy)) / E
    gxy, gyz, gzx = sxy / G, syz / G, szx / G
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz + 1) * h, np.arange(ny + 1) * h, np.arange(nx + 1) * h, indexing="ij")
    u = np.stack([exx * x + 0.5 * gxy * y + 0.5 * gzx * z,
                  0.5 * gxy * x + eyy * y + 0.5 * gyz * z,
                  0.5 * gzx * x + 0.5 * gyz * y + ezz * z], axis=-1)
    return u.ravel()


def von_mises(sigma):
    sxx, syy, szz, sxy, syz, szx = sigma
    return float(np.sqrt(sxx ** 2 + syy ** 2 + szz ** 2 - sxx * syy - syy * szz - szz * sxx + 3 * (sxy ** 2 + syz ** 2 + szx ** 2)))


def principals(sigma):
    """Principal stresses, largest first, as eigenvalues of the symmetric tensor."""
    sxx, syy, szz, sxy, syz, szx = sigma
    return np.linalg.eigvalsh(np.array([[sxx, sxy, szx], [sxy, syy, syz], [szx, syz, szz]]))[::-1]


# test_fea.cpp:40-47: principals 15 + r, 10 and 15 - r with r = hypot(35, 30) (in MPa here)
KNOWN_TENSOR = (50e6, -20e6, 10e6, 30e6, 0.0, 0.0)
KNOWN_PRINCIPALS = (15e6 + np.hypot(35e6, 30e6), 10e6, 15e6 - np.hypot(35e6, 30e6))
GENERAL_TENSOR = (42e6, -17e6, 23e6, 11e6, -29e6, 7e6)
