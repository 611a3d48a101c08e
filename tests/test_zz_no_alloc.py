"""The allocation-free entry point, ps_fea_apply_dot_noalloc: for callers that cannot allocate
device memory during a call (their device memory belongs to another allocator or a fixed budget,
or they must not stall on the synchronisation a cudaMalloc can cause). Its product y = K x and
dot x.y, computed with the library's static device scratch, must equal what the allocating entry
point ps_fea_apply returns, on two calls in a row. Collected last on purpose: it needs nothing the
other tests leave behind and passes alone in a fresh process as well."""
import numpy as np
import pytest

import psfea
from conftest import golden

pytestmark = pytest.mark.gpu


def test_apply_dot_noalloc_matches_apply_twice():
    import torch

    g = golden("cantilever_64x16x16")
    S = psfea.VoxelFEA(tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))
    n = S.n_dof
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(12)
    y_dev = torch.empty(n, dtype=torch.float64, device=dev)
    dot_dev = torch.empty(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        x = rng.standard_normal(n)
        x_dev = torch.from_numpy(x).to(dev)
        y_dev.fill_(float("nan"))
        dot_dev.fill_(float("nan"))
        torch.cuda.synchronize()
        S.apply_dot_noalloc(x_dev.data_ptr(), y_dev.data_ptr(), dot_dev.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        y = y_dev.cpu().numpy()
        y_ref = S.apply(x)  # the allocating entry point
        assert np.linalg.norm(y - y_ref) <= 1e-13 * np.linalg.norm(y_ref), call
        d_ref = float(np.dot(x, y_ref))
        assert abs(float(dot_dev.item()) - d_ref) <= 1e-12 * abs(d_ref), call
