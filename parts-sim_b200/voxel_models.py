"""Seeded synthetic voxel models of the benchmark shapes (numpy; host-side set-up, not the solve).

Each generator returns a ``Model`` with the solver's inputs in the reference's layout
(native/src/fea/voxel_fea.hpp:132-137): ``density`` per voxel ``i + nx*(j + ny*k)`` (0 = empty),
``bc`` per DOF ``3*(i + NX*(j + NY*k)) + d`` (1 = held), and loads ``f`` per DOF in N, in the
solver's normalised units (E = 1, voxel size 1: ``u_physical = u / (E*h)``,
native/src/fea/voxel_fea.hpp:17-18). The same arrays feed the GPU solver and the CPU oracle, so
the mask, indexing and load vector are identical by construction.

Random numbers come from a counter-based splitmix64 stream, so every model is reproducible from
its seed on any machine.
"""
from dataclasses import dataclass, field

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class Rng:
    """splitmix64 stream (Steele, Lea & Flood 2014): value i is mix(seed + (i + 1) * golden)."""

    def __init__(self, seed):
        self.state = np.uint64(seed)
        self.count = 0

    def u64(self, n):
        with np.errstate(over="ignore"):
            i = np.arange(self.count + 1, self.count + 1 + n, dtype=np.uint64)
            z = self.state + i * _GOLD
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        self.count += n
        return z

    def uniform(self, n, lo=0.0, hi=1.0):
        u = (self.u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def normal(self, n):
        """Box-Muller pairs."""
        m = (n + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log1p(-u1))
        out = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
        return out[:n]


@dataclass
class Model:
    name: str
    dims: tuple            # voxel counts (nx, ny, nz)
    density: np.ndarray    # float32 [nx*ny*nz]
    bc: np.ndarray         # uint8 [3*NX*NY*NZ]
    f: np.ndarray          # float64 [3*NX*NY*NZ] or [nrhs, 3*NX*NY*NZ]
    nu: float
    E: float               # Pa, for physical displacements / stresses
    h: float               # m, voxel size
    coarsest_max_dof: int = 1100
    meta: dict = field(default_factory=dict)

    @property
    def nodes(self):
        nx, ny, nz = self.dims
        return (nx + 1, ny + 1, nz + 1)

    @property
    def n_dof(self):
        NX, NY, NZ = self.nodes
        return 3 * NX * NY * NZ

    def node(self, i, j, k):
        NX, NY, _ = self.nodes
        return i + NX * (j + NY * k)


def _edge_weights(n):
    """Trapezoid weights of the n+1 nodes along an edge of n voxels (0.5 at both ends)."""
    w = np.ones(n + 1)
    w[0] = w[-1] = 0.5
    return w


def held_nodes(dims, bc):
    """Per node: 1 if any of its DOFs is held."""
    nx, ny, nz = dims
    return (np.asarray(bc).reshape(-1, 3).max(axis=1) > 0).astype(np.uint8)


def prune_floating(dims, density, held_node):
    """Voxels face-connected (6-neighbourhood) to a voxel with a held corner node survive; the
    rest become empty (the rule of native/src/fea/voxel_fea.cpp:1086-1119). The reference walks the
    voxels breadth-first from the held ones; the same set is every 6-connected component of the
    solid that contains such a voxel, found here by connected-component labelling.
    ``held_node``: per node, nonzero where any DOF is held. Returns (density, removed)."""
    from scipy import ndimage
    nx, ny, nz = dims
    d = np.asarray(density, np.float32).reshape(nz, ny, nx)
    held = np.asarray(held_node).reshape(nz + 1, ny + 1, nx + 1) > 0
    touch = np.zeros((nz, ny, nx), bool)
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                touch |= held[dk:dk + nz, dj:dj + ny, di:di + nx]
    solid = d > 0
    labels, _ = ndimage.label(solid)  # default structure: the 6 face neighbours
    keep_ids = np.unique(labels[solid & touch])
    keep = np.zeros(int(labels.max()) + 1, bool)
    keep[keep_ids] = True
    keep[0] = False
    reach = keep[labels]
    out = np.where(reach, d, 0).astype(np.float32).ravel()
    return out, int(solid.sum() - reach.sum())


def _face_load(dims, density, axis, side, value_per_voxel):
    """Consistent nodal loads of a uniform traction on one outer grid face of the solid voxels:
    each loaded voxel face gives a quarter of its load to each of its 4 corner nodes.
    ``axis`` 0/1/2 = x/y/z, ``side`` 0 = the low face, 1 = the high face; ``value_per_voxel`` is a
    3-vector of N per voxel face. Returns (f, number of loaded faces)."""
    nx, ny, nz = dims
    d = np.asarray(density, np.float32).reshape(nz, ny, nx)
    f = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    ax = 2 - axis  # array axis in (k, j, i) order
    layer = [slice(None)] * 3
    layer[ax] = 0 if side == 0 else dims[axis] - 1
    solid = (d[tuple(layer)] > 0).astype(np.float64)  # 2D over the two in-plane axes
    nodal = np.zeros((solid.shape[0] + 1, solid.shape[1] + 1))
    for a in (0, 1):
        for b in (0, 1):
            nodal[a:a + solid.shape[0], b:b + solid.shape[1]] += 0.25 * solid
    plane = [slice(None)] * 3
    plane[ax] = 0 if side == 0 else dims[axis]
    for c in range(3):
        f[..., c][tuple(plane)] += nodal * value_per_voxel[c]
    return f.reshape(-1), int(solid.sum())


def cantilever(nx=64, ny=16, nz=16, traction=1e6, h=1e-3, E=200e9, nu=0.3, coarsest_max_dof=1300):
    """Steel cantilever: x = 0 face fully held; uniform traction in -z on the x = nx face.
    Tip nodes get traction*h^2 times trapezoid weights (w = 1/2 on face edges), which is the
    consistent load of native/tests/test_fea.cpp:65-71. With 1 MPa on 16x16 voxels of 1 mm the
    total is -256 N. coarsest_max_dof 1300 gives the 3-level hierarchy."""
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    density = np.ones(nx * ny * nz, np.float32)
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    bc[:, :, 0, :] = 1
    f = np.zeros((NZ, NY, NX, 3))
    f[:, :, nx, 2] = -traction * h * h * np.outer(_edge_weights(nz), _edge_weights(ny))
    return Model("cantilever", (nx, ny, nz), density, bc.ravel(), f.ravel(), nu, E, h, coarsest_max_dof,
                 {"traction_Pa": traction, "total_N": float(f.sum())})


def l_bracket(nx=256, ny=128, nz=128, holes=64, seed=2, h=0.5e-3, E=70e9, nu=0.33, load=500.0):
    """Aluminium L-bracket: solid except the quadrant x > 96 and z > 48 (voxel centres, scaled
    with the grid), minus ``holes`` cylinders along y (radius U[3, 8] voxels, centres uniform over
    the solid x-z region, by rejection), the y = 0 face held, and ``load`` N in -z spread evenly
    over the solid top faces of an 8x8-voxel patch at the arm tip (the z = 48 face, largest x,
    centred in y), each face's share split 1/4 per corner node."""
    sx, sz = nx / 256.0, nz / 128.0
    xq, zq = 96 * sx, 48 * sz
    rng = Rng(seed)
    i = np.arange(nx) + 0.5
    k = np.arange(nz) + 0.5
    X, Z = np.meshgrid(i, k, indexing="xy")  # [nz, nx]
    solid = ~((X > xq) & (Z > zq))
    cyl = []
    while len(cyl) < holes:
        c = rng.uniform(3)
        cx, cz, r = c[0] * nx, c[1] * nz, 3 + 5 * c[2]
        if cx > xq and cz > zq:
            continue
        cyl.append((cx, cz, r))
    for cx, cz, r in cyl:
        solid &= (X - cx) ** 2 + (Z - cz) ** 2 >= r * r
    d2 = solid.astype(np.float32)  # [nz, nx]
    density = np.repeat(d2[:, None, :], ny, axis=1).ravel()  # [nz, ny, nx]
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    bc[:, 0, :, :] = 1
    density, removed = prune_floating((nx, ny, nz), density, held_nodes((nx, ny, nz), bc))
    # load patch on top of the arm: voxel layer just below z = zq, x in [nx-8, nx), y centred
    kz = int(round(zq)) - 1
    d3 = density.reshape(nz, ny, nx)
    pi0, pj0 = nx - 8, ny // 2 - 4
    patch = d3[kz, pj0:pj0 + 8, pi0:pi0 + 8] > 0
    nface = int(patch.sum())
    f = np.zeros((NZ, NY, NX, 3))
    if nface:
        per = load / nface
        for a in (0, 1):
            for b in (0, 1):
                f[kz + 1, pj0 + a:pj0 + a + 8, pi0 + b:pi0 + b + 8, 2] -= 0.25 * per * patch
    return Model("l_bracket", (nx, ny, nz), density, bc.ravel(), f.ravel(), nu, E, h, 1100,
                 {"holes": cyl, "removed": removed, "loaded_faces": nface, "total_N": float(f.sum())})


def _gauss_smooth(g, sigma):
    """Separable Gaussian filter (truncated at 4 sigma), edges clamped."""
    rad = int(np.ceil(4 * sigma))
    x = np.arange(-rad, rad + 1)
    w = np.exp(-0.5 * (x / sigma) ** 2)
    w /= w.sum()
    out = g
    for axis in range(3):
        n = out.shape[axis]
        idx = np.clip(np.arange(-rad, n + rad), 0, n - 1)
        padded = np.take(out, idx, axis=axis)
        acc = np.zeros_like(out)
        for t, wt in enumerate(w):
            sl = [slice(None)] * 3
            sl[axis] = slice(t, t + n)
            acc += wt * padded[tuple(sl)]
        out = acc
    return out


def simp(nx=192, ny=96, nz=96, nrhs=32, seed=3, nu=0.3, E=1.0, h=1.0):
    """SIMP-like graded grid with MBB supports and ``nrhs`` unit loads.
    g ~ N(0,1) per voxel, Gaussian-smoothed (sigma 4 voxels, clamped edges), normalised to unit std;
    rho = clamp(0.5 + 0.5 g, 1e-3, 1); density = 1e-9 + rho^3 (1 - 1e-9).
    Supports: u_x = 0 on the x = 0 plane (symmetry); u_z = 0 on the bottom edge line x = nx, z = 0
    (roller), plus u_y = 0 on that line so the y translation is held too (loads have y parts).
    Loads: unit force spread evenly over the top centre line nodes (x = 0, z = nz), one direction
    per right-hand side, uniform on the unit sphere."""
    rng = Rng(seed)
    g = rng.normal(nx * ny * nz).reshape(nz, ny, nx)
    g = _gauss_smooth(g, 4.0)
    g = (g - g.mean()) / g.std()
    rho = np.clip(0.5 + 0.5 * g, 1e-3, 1.0)
    density = (1e-9 + rho ** 3 * (1 - 1e-9)).astype(np.float32).ravel()
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    bc[:, :, 0, 0] = 1
    bc[0, :, nx, 2] = 1
    bc[0, :, nx, 1] = 1
    dirs = rng.normal(3 * nrhs).reshape(nrhs, 3)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    f = np.zeros((nrhs, NZ, NY, NX, 3))
    for q in range(nrhs):
        f[q, nz, :, 0, :] = dirs[q] / NY
    return Model("simp", (nx, ny, nz), density, bc.ravel(), f.reshape(nrhs, -1), nu, E, h, 1100, {"dirs": dirs})


def gyroid(nx=384, ny=384, nz=192, period=24, thickness=0.3, pressure=5e6, h=1e-3, E=114e9, nu=0.34):
    """Gyroid sheet lattice: solid where |sin x cos y + sin y cos z + sin z cos x| < thickness with
    x = 2 pi (i + 1/2) / period (same for y, z); bottom z = 0 face held; ``pressure`` in -z on the
    solid top faces (consistent nodal weights); floating fragments pruned."""
    t = lambda n: 2 * np.pi * (np.arange(n) + 0.5) / period
    x = t(nx)[None, None, :]
    y = t(ny)[None, :, None]
    z = t(nz)[:, None, None]
    val = np.sin(x) * np.cos(y) + np.sin(y) * np.cos(z) + np.sin(z) * np.cos(x)
    density = (np.abs(val) < thickness).astype(np.float32).ravel()
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    bc[0] = 1
    density, removed = prune_floating((nx, ny, nz), density, held_nodes((nx, ny, nz), bc))
    f, nface = _face_load((nx, ny, nz), density, 2, 1, (0.0, 0.0, -pressure * h * h))
    return Model("gyroid", (nx, ny, nz), density, bc.ravel(), f, nu, E, h, 1100, {"removed": removed, "loaded_faces": nface})


MATERIALS = ((200e9, 0.30), (70e9, 0.33), (3.5e9, 0.36))


def box_with_voids(rng, lo=24, hi=160, solid_target=0.6, h=1e-3):
    """One serving request: per-axis size log-uniform in [lo, hi] voxels, spherical voids with
    radius U[2, 10] voxels placed until the solid fraction reaches ``solid_target``, material
    drawn from MATERIALS, one random face held and a uniform traction with a random direction and
    log-uniform magnitude in [0.1, 10] MPa on the opposite face; floating fragments pruned."""
    u = rng.uniform(3)
    dims = tuple(int(round(np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * v))) for v in u)
    nx, ny, nz = dims
    solid = np.ones((nz, ny, nx), bool)
    total = nx * ny * nz
    removed = 0
    # voids in rounds (each round's centres drawn at once); a round stops at the target
    while total - removed > solid_target * total:
        c = rng.uniform(4 * 32).reshape(32, 4)
        for cx, cy, cz, cr in c:
            cx, cy, cz, r = cx * nx, cy * ny, cz * nz, 2 + 8 * cr
            k0, k1 = max(0, int(cz - r)), min(nz, int(cz + r) + 1)
            j0, j1 = max(0, int(cy - r)), min(ny, int(cy + r) + 1)
            i0, i1 = max(0, int(cx - r)), min(nx, int(cx + r) + 1)
            zz = (np.arange(k0, k1) + 0.5 - cz)[:, None, None] ** 2
            yy = (np.arange(j0, j1) + 0.5 - cy)[None, :, None] ** 2
            xx = (np.arange(i0, i1) + 0.5 - cx)[None, None, :] ** 2
            m = zz + yy + xx < r * r
            sub = solid[k0:k1, j0:j1, i0:i1]
            removed += int((sub & m).sum())
            sub &= ~m
            if total - removed <= solid_target * total:
                break
    mat = MATERIALS[int(rng.uniform(1)[0] * 3) % 3]
    face = int(rng.uniform(1)[0] * 6) % 6
    axis, side = face // 2, face % 2
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    bc = np.zeros((NZ, NY, NX, 3), np.uint8)
    sl = [slice(None)] * 3
    sl[2 - axis] = 0 if side == 0 else dims[axis]
    bc[tuple(sl)] = 1
    held = bc.reshape(-1, 3).max(axis=1)
    density, nrem = prune_floating(dims, solid.astype(np.float32).ravel(), held)
    d = rng.normal(3)
    d /= np.linalg.norm(d)
    mag = np.exp(np.log(0.1e6) + (np.log(10e6) - np.log(0.1e6)) * rng.uniform(1)[0])
    f, nface = _face_load(dims, density, axis, 1 - side, d * mag * h * h)
    return Model("request", dims, density, bc.ravel(), f, mat[1], mat[0], h, 300,
                 {"face": face, "traction_Pa": mag, "removed": nrem})


def serving_stream(n=512, rate=200.0, seed=5):
    """``n`` requests with Poisson arrival times at ``rate`` per second: a generator of
    (t_arrival, Model), each request from its own sub-seed (so any prefix is reproducible)."""
    rng = Rng(seed)
    gaps = -np.log1p(-rng.uniform(n)) / rate
    t = np.cumsum(gaps)
    for q in range(n):
        yield float(t[q]), box_with_voids(Rng(seed * 1000003 + q))
