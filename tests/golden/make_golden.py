"""Writes the golden fixtures in this folder from the reference's own solver.

The reference (native/src/fea/*.cpp of Parts Sim) is compiled from its sources by
``make -C oracle`` into oracle/_ref/libpsref.so; this script runs it on small seeded models and
stores inputs and outputs as compressed .npz files. Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

The fixtures are committed; the tests read them, never the reference itself. Names given on the
command line limit the run to those fixtures (``element``, ``prune`` or a model name).
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "parts-sim_b200"))

import oracle  # noqa: E402
import voxel_models as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def element_fixture():
    out = {}
    for nu in (0.3, 0.33, 0.34, 0.36):
        K, cs, gb = oracle.element("reference", nu)
        out[f"K_{nu}"] = K
        if nu == 0.3:
            out["cornerStress_0.3"] = cs
            out["gaussB_0.3"] = gb
    K, _, _ = oracle.element("reference", 0.3, modes=False)
    out["K_trilinear_0.3"] = K
    np.savez_compressed(os.path.join(OUT, "element.npz"), **out)


def model_fixture(name, m, tol=1e-8, rhs=0):
    f = m.f if m.f.ndim == 1 else m.f[rhs]
    R = oracle.OracleModel("reference", m.dims, m.density, m.nu, m.bc, m.coarsest_max_dof)
    out = {"dims": np.array(m.dims, np.int32), "density": m.density, "bc": m.bc, "f": f, "nu": np.float64(m.nu),
           "E": np.float64(m.E), "h": np.float64(m.h), "coarsest": np.int64(m.coarsest_max_dof), "tol": np.float64(tol)}
    out["levels"] = np.int64(R.n_levels)
    for l in range(R.n_levels):
        info = R.level_info(l)
        out[f"info_{l}"] = np.array([info[k] for k in ("nx", "ny", "nz", "nNodes", "nDof", "freeDof", "nElems", "nOwn", "coarse_m")],
                                    np.int64)
        out[f"fixed_{l}"] = np.packbits(R.fixed(l))
        out[f"kidx_{l}"] = R.kidx(l)
        out[f"elems_{l}"] = R.elems(l)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(R.n_dof)
    out["apply_x"] = x
    out["apply_y"] = R.apply(x)
    out["apply_y_raw"] = R.apply(x, raw=True)
    u, it, res, conv = R.solve(f, tol, 3000)
    out["u"] = u
    out["iterations"] = np.int64(it)
    out["residual"] = np.float64(res)
    out["converged"] = np.int64(conv)
    R.prepare()
    out["lmax"] = np.array([R.lmax(l) for l in range(R.n_levels - 1)])
    uphys = u / (m.E * m.h)
    vm, p1, p3 = R.stresses(uphys, m.E, m.h, True)
    out["vm"], out["p1"], out["p3"] = vm, p1, p3
    out["reactions"] = R.reactions(u, f)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    print(name, m.dims, "levels", R.n_levels, "it", it, "res", res, "conv", conv)


def prune_fixture():
    # the reference's own test case (native/tests/test_fea.cpp:115-122) plus a seeded 3D one
    d1 = np.array([1, 1, 0, 1], np.float32)
    h1 = np.zeros(5 * 2 * 2, np.uint8)
    h1[0] = 1
    o1, r1 = oracle.prune("reference", (4, 1, 1), d1, h1)
    rng = np.random.default_rng(3)
    dims = (12, 10, 8)
    d2 = (rng.random(12 * 10 * 8) < 0.55).astype(np.float32)
    h2 = np.zeros(13 * 11 * 9, np.uint8)
    h2[: 13 * 11] = 1  # the k = 0 plane
    o2, r2 = oracle.prune("reference", dims, d2, h2)
    np.savez_compressed(os.path.join(OUT, "prune.npz"), d1=d1, h1=h1, o1=o1, r1=np.int64(r1), d2=d2, h2=h2, o2=o2, r2=np.int64(r2),
                        dims2=np.array(dims, np.int32))


if __name__ == "__main__":
    if not oracle.available("reference"):
        sys.exit("oracle/_ref/libpsref.so is missing: run `make -C oracle` where the reference sources are present")
    models = {
        "cantilever_32x8x8": lambda: W.cantilever(32, 8, 8, coarsest_max_dof=1100),
        "cantilever_64x16x16": W.cantilever,
        "lbracket_32x16x16": lambda: W.l_bracket(32, 16, 16, holes=3),
        "simp_16x8x8": lambda: W.simp(16, 8, 8, nrhs=1),
        "lbracket_24x12x12_loose": lambda: (W.l_bracket(24, 12, 12, holes=2), 1e-6),
        # the lattice and the serving-stream shapes, small
        "gyroid_48x48x24": lambda: W.gyroid(48, 48, 24),
        "box_request_20_28": lambda: W.box_with_voids(W.Rng(11), lo=20, hi=28),
    }
    want = sys.argv[1:] or ["element", "prune"] + list(models)
    if "element" in want:
        element_fixture()
    if "prune" in want:
        prune_fixture()
    for name, make in models.items():
        if name in want:
            m = make()
            m, tol = m if isinstance(m, tuple) else (m, 1e-8)
            model_fixture(name, m, tol=tol)
