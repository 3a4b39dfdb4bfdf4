"""Slab-decomposed 2D transforms over the ranks of a torch.distributed group.

The reference runs its transforms under FFTW-MPI (fft.c:11-31, plans
main.c:193-194): rank r of P holds local_nx = nx / P x-rows of each real field,
x = r local_nx .. (r + 1) local_nx - 1, and the same kx-rows of its spectrum in
FFTW's layout.  ``SlabFFT`` is that dfft / ifft with one GPU per rank: the local
phases are this library's kernels (chns_slab_* in include/chns.h) and the two
global transposes of each transform are ``all_to_all_single`` exchanges of equal
blocks -- NCCL over NVLink on a "nccl" group, through host memory on a "gloo"
group.  There is no CPU transform: without the built library or a GPU every call
raises.
"""
from __future__ import annotations

import ctypes

from . import ChnsError, load_library

_bound = False


def _bind(L):
    global _bound
    if _bound:
        return
    vp, sz, ip = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.chns_slab_create.argtypes = [ip, ip, ip, ctypes.POINTER(vp)]
    L.chns_slab_destroy.argtypes = [vp]
    L.chns_slab_destroy.restype = None
    L.chns_slab_sizes.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(sz)]
    for f in ("chns_slab_dfft_x", "chns_slab_dfft_unpack", "chns_slab_ifft_pack", "chns_slab_ifft_x"):
        getattr(L, f).argtypes = [vp, vp, vp, vp]
    L.chns_slab_dfft_y.argtypes = [vp, vp, sz, vp, vp]
    L.chns_slab_ifft_y.argtypes = [vp, vp, vp, sz, vp]
    _bound = True


class SlabFFT:
    """dfft / ifft of an n x n field distributed by x-rows over a process group.

    ``dfft(real)``: real is this rank's (local_nx, m) float64 CUDA tensor, m >= n
    (the reference's in-place rows have m = n + 2; only the first n columns are
    read); returns the rank's (local_nx, n/2+1) complex128 spectrum, kx-rows
    rank * local_nx ..., unnormalised (fft.c:11-14).  ``ifft(spec, out=None)``:
    the inverse with the reference's 1/(nx ny) (fft.c:16-31), into ``out``
    (local_nx, m >= n; its first n columns are written) or a new (local_nx, n)
    tensor.  Every rank of the group calls each method with its own slab.
    """

    def __init__(self, n: int, group=None):
        import torch
        import torch.distributed as dist

        self.L = load_library()
        _bind(self.L)
        self.group = group
        self.nranks = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.n = n
        self.device = torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        rc = self.L.chns_slab_create(n, self.nranks, self.rank, ctypes.byref(h))
        if rc != 0:
            raise ChnsError(rc, "chns_slab_create")
        self.handle = h
        lnx, rows, ex = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        rc = self.L.chns_slab_sizes(h, ctypes.byref(lnx), ctypes.byref(rows), ctypes.byref(ex))
        if rc != 0:
            raise ChnsError(rc, "chns_slab_sizes")
        self.local_nx, self.rows_per_rank, self.exchange_complex = lnx.value, rows.value, ex.value
        # two exchange buffers of complex doubles (as float64 pairs)
        self._buf = [torch.empty(2 * self.exchange_complex, dtype=torch.float64, device=self.device) for _ in range(2)]
        self.device_exchange = dist.get_backend(group) == "nccl"

    def close(self):
        if getattr(self, "handle", None):
            self.L.chns_slab_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _exchange(self, send, recv):
        import torch.distributed as dist

        if self.device_exchange:
            dist.all_to_all_single(recv, send, group=self.group)
        else:
            host = send.cpu()  # synchronises the stream the phase ran on
            out = host.new_empty(host.shape)
            dist.all_to_all_single(out, host, group=self.group)
            recv.copy_(out)

    def _check(self, rc, what):
        if rc != 0:
            raise ChnsError(rc, what)

    def dfft(self, real):
        import torch

        if real.dtype != torch.float64 or real.device != self.device or real.dim() != 2:
            raise ValueError("real must be a 2-D float64 tensor on this rank's GPU")
        if real.shape[0] != self.local_nx or real.shape[1] < self.n or real.stride(1) != 1:
            raise ValueError(f"real must be ({self.local_nx}, >= {self.n}) with unit column stride")
        a, b = self._buf
        spec = torch.empty((self.local_nx, self.n // 2 + 1), dtype=torch.complex128, device=self.device)
        st = self._stream()
        self._check(self.L.chns_slab_dfft_y(self.handle, ctypes.c_void_p(real.data_ptr()), real.stride(0),
                                            ctypes.c_void_p(a.data_ptr()), st), "chns_slab_dfft_y")
        self._exchange(a, b)
        self._check(self.L.chns_slab_dfft_x(self.handle, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                            st), "chns_slab_dfft_x")
        self._exchange(a, b)
        self._check(self.L.chns_slab_dfft_unpack(self.handle, ctypes.c_void_p(b.data_ptr()),
                                                 ctypes.c_void_p(spec.data_ptr()), st), "chns_slab_dfft_unpack")
        return spec

    def ifft(self, spec, out=None):
        import torch

        if spec.dtype != torch.complex128 or spec.device != self.device or \
                tuple(spec.shape) != (self.local_nx, self.n // 2 + 1) or not spec.is_contiguous():
            raise ValueError(f"spec must be a contiguous ({self.local_nx}, {self.n // 2 + 1}) complex128 CUDA tensor")
        if out is None:
            out = torch.empty((self.local_nx, self.n), dtype=torch.float64, device=self.device)
        elif out.dtype != torch.float64 or out.device != self.device or out.shape[0] != self.local_nx or \
                out.shape[1] < self.n or out.stride(1) != 1:
            raise ValueError(f"out must be ({self.local_nx}, >= {self.n}) float64 on this rank's GPU")
        a, b = self._buf
        st = self._stream()
        self._check(self.L.chns_slab_ifft_pack(self.handle, ctypes.c_void_p(spec.data_ptr()),
                                               ctypes.c_void_p(a.data_ptr()), st), "chns_slab_ifft_pack")
        self._exchange(a, b)
        self._check(self.L.chns_slab_ifft_x(self.handle, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                            st), "chns_slab_ifft_x")
        self._exchange(a, b)
        self._check(self.L.chns_slab_ifft_y(self.handle, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                            out.stride(0), st), "chns_slab_ifft_y")
        return out
