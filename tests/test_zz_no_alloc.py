"""chns_dfft_noalloc: the 2D r2c transform for callers that cannot allocate
device memory (it keeps its intermediate field in a fixed device array).

It must give what the allocating entry point chns_dfft gives, on consecutive
calls that reuse the shared array.  This file is named so that pytest collects
it last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dfft_noalloc_matches_dfft_on_consecutive_calls():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    import chns_b200

    L = chns_b200.load_library()
    stream = torch.cuda.current_stream()
    # two calls in a row: different sizes and data share the one scratch array
    for n, seed in ((512, 1), (64, 2), (512, 3)):
        rng = np.random.default_rng(seed)
        x = rng.standard_normal((n, n))
        with chns_b200.Context(dict(model=0, nx=n, ny=n, dt=1e-3, nu=0.01)) as ctx:
            ref = ctx.dfft(x)
        xd = torch.from_numpy(x).cuda()
        out = torch.full((n, n // 2 + 1, 2), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.chns_dfft_noalloc(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(out.data_ptr()), n,
                                 ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, chns_b200.STATUS.get(rc, rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128)[..., 0]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= 1e-13, (n, err)
        assert err <= 1e-13 and np.linalg.norm(got - np.fft.rfft2(x)) <= 1e-13 * np.linalg.norm(ref)


def test_dfft_noalloc_rejects_sizes_beyond_the_maximum():
    import torch

    import chns_b200

    L = chns_b200.load_library()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    for n in (1024, 48, 16):
        assert L.chns_dfft_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), n, None) == -5
