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


def _model():
    g = golden("cantilever_64x16x16")
    return psfea.VoxelFEA(tuple(g["dims"]), g["density"], float(g["nu"]), g["bc"], int(g["coarsest"]))


def _check(S, x, y, dot, call):
    y_ref = S.apply(x)  # the allocating entry point
    assert np.linalg.norm(y - y_ref) <= 1e-13 * np.linalg.norm(y_ref), call
    d_ref = float(np.dot(x, y_ref))
    assert abs(dot - d_ref) <= 1e-12 * abs(d_ref), call


def test_apply_dot_noalloc_matches_apply_twice():
    import torch

    S = _model()
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
        _check(S, x, y_dev.cpu().numpy(), float(dot_dev.item()), call)


@pytest.mark.parametrize("which", ["side", "default"])
def test_apply_dot_noalloc_is_stream_ordered(which):
    """The fill of x, two calls back to back and the copies of y and x.y all queued on one caller
    stream (a side stream, or PyTorch's default stream, which it reports as 0), with a single
    synchronisation at the end: the calls must be ordered after the model's uploads and the fill,
    and before the copies."""
    import torch

    S = _model()  # created just before: its uploads may still be in flight
    n = S.n_dof
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(13)
    xs = [torch.from_numpy(rng.standard_normal(n)).pin_memory() for _ in range(2)]
    stream = torch.cuda.Stream(dev) if which == "side" else torch.cuda.default_stream(dev)
    outs = []
    with torch.cuda.stream(stream):
        x_dev = torch.empty(n, dtype=torch.float64, device=dev)
        y_dev = torch.empty(n, dtype=torch.float64, device=dev)
        dot_dev = torch.empty(1, dtype=torch.float64, device=dev)
        for call in range(2):
            x_dev.copy_(xs[call], non_blocking=True)
            y_dev.fill_(float("nan"))
            S.apply_dot_noalloc(x_dev.data_ptr(), y_dev.data_ptr(), dot_dev.data_ptr(), stream.cuda_stream)
            y_host = torch.empty(n, dtype=torch.float64).pin_memory()
            d_host = torch.empty(1, dtype=torch.float64).pin_memory()
            y_host.copy_(y_dev, non_blocking=True)
            d_host.copy_(dot_dev, non_blocking=True)
            outs.append((y_host, d_host))
    stream.synchronize()
    for call, (y, d) in enumerate(outs):
        _check(S, xs[call].numpy(), y.numpy(), float(d[0]), call)
