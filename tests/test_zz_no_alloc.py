"""chns_dfft_noalloc: the 2D r2c transform for callers that cannot allocate
device memory (code inside another library's allocator or memory pool, or whose
device memory a host application hands out); it keeps its intermediate field in
a fixed device array.

It must give what the allocating entry point chns_dfft gives, on consecutive
calls that reuse the shared array, at every supported size, and it must take no
device memory once its first call has set the device up.  This file is named so
that pytest collects it last."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIZES = (32, 64, 128, 256, 512)


def _call(L, xd, out, n, stream):
    rc = L.chns_dfft_noalloc(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(out.data_ptr()), n,
                             ctypes.c_void_p(stream.cuda_stream))
    return rc


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
        rc = _call(L, xd, out, n, stream)
        assert rc == 0, chns_b200.STATUS.get(rc, rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128)[..., 0]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= 1e-13, (n, err)
        assert np.linalg.norm(got - np.fft.rfft2(x)) <= 1e-13 * np.linalg.norm(ref)


def test_dfft_noalloc_every_size_twice_takes_no_device_memory():
    """Every supported n, two rounds; the device's free memory after the second
    round equals that after the first (the set-up loads every size's kernels, so
    a first call at a new size loads no module either)."""
    import torch

    import chns_b200

    L = chns_b200.load_library()
    stream = torch.cuda.current_stream()
    xs, refs, outs = {}, {}, {}
    for n in SIZES:
        x = np.random.default_rng(100 + n).standard_normal((n, n))
        with chns_b200.Context(dict(model=0, nx=n, ny=n, dt=1e-3, nu=0.01)) as ctx:
            refs[n] = ctx.dfft(x)
        xs[n] = torch.from_numpy(x).cuda()
        outs[n] = torch.empty((n, n // 2 + 1, 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free = []
    for rnd in range(2):
        for n in SIZES:
            outs[n].fill_(float("nan"))
            assert _call(L, xs[n], outs[n], n, stream) == 0
            torch.cuda.synchronize()
            got = outs[n].cpu().numpy().view(np.complex128)[..., 0]
            err = np.linalg.norm(got - refs[n]) / np.linalg.norm(refs[n])
            assert err <= 1e-13, (rnd, n, err)
        free.append(torch.cuda.mem_get_info()[0])
    assert free[1] == free[0], free


_FIRST_CALL = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import chns_b200
L = chns_b200.load_library()
n = 512
x = np.random.default_rng(7).standard_normal((n, n))
side = torch.cuda.Stream()  # created non-blocking by torch: not ordered after the legacy stream
with torch.cuda.stream(side):
    xd = torch.from_numpy(x).to("cuda", non_blocking=False)
    out = torch.full((n, n // 2 + 1, 2), float("nan"), dtype=torch.float64, device="cuda")
side.synchronize()
rc = L.chns_dfft_noalloc(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(out.data_ptr()), n,
                         ctypes.c_void_p(side.cuda_stream))
assert rc == 0, rc
side.synchronize()
got = out.cpu().numpy().view(np.complex128)[..., 0]
ref = np.fft.rfft2(x)
err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
assert err <= 1e-13, err
print("first call ok", err)
"""


def test_dfft_noalloc_first_call_on_a_nonblocking_stream():
    """The very first call of a fresh process, on a non-blocking stream: the
    set-up's twiddle upload must have landed before the transform reads it."""
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, os.path.join(ROOT, "ternary-chns_b200")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "first call ok" in r.stdout


def test_dfft_noalloc_rejects_sizes_beyond_the_maximum():
    import torch

    import chns_b200

    L = chns_b200.load_library()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    for n in (1024, 48, 16):
        assert L.chns_dfft_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), n, None) == -5
