"""Slab-decomposed transforms (chns_b200.slab.SlabFFT over the chns_slab_* C
ABI): the reference's FFTW-MPI dfft/ifft (fft.c:11-31, slabs main.c:43-46) with
one rank per slab of x-rows.  Each case starts its ranks as separate processes;
the ranks of one case share this GPU, which is possible because the exchanges of
a "gloo" group go through host memory (no kernel of one rank waits on another);
the "nccl" case runs one rank, so its all-to-all stays on the device.

Checked on every rank against numpy's rfft2 of the whole field (the rank's
kx-rows) and for the round trip: relative L2 <= 1e-13 (FP64), the padding
columns of the reference's in-place rows neither read nor written."""
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RANK = r"""
import os, sys
import numpy as np
import torch
import torch.distributed as dist
sys.path.insert(0, sys.argv[1])
n = int(sys.argv[2]); backend = sys.argv[3]
torch.cuda.set_device(0)
dist.init_process_group(backend, timeout=__import__("datetime").timedelta(seconds=60))
from chns_b200.slab import SlabFFT
rank, P = dist.get_rank(), dist.get_world_size()
full = np.random.default_rng(11).standard_normal((n, n))
ref = np.fft.rfft2(full)
s = SlabFFT(n)
lnx = s.local_nx
rows = slice(rank * lnx, (rank + 1) * lnx)
# the reference's in-place rows: n reals and 2 padding columns (NaN: never read)
real = torch.full((lnx, n + 2), float("nan"), dtype=torch.float64, device="cuda")
real[:, :n] = torch.from_numpy(full[rows])
spec = s.dfft(real)
got = spec.cpu().numpy()
e1 = np.linalg.norm(got - ref[rows]) / np.linalg.norm(ref[rows])
out = torch.full((lnx, n + 2), 7.0, dtype=torch.float64, device="cuda")
s.ifft(spec, out=out)
back = out.cpu().numpy()
e2 = np.linalg.norm(back[:, :n] - full[rows]) / np.linalg.norm(full[rows])
pad_ok = bool(np.all(back[:, n:] == 7.0))
# a second transform reuses the plan's buffers
spec2 = s.dfft(real)
e3 = np.linalg.norm(spec2.cpu().numpy() - got) / np.linalg.norm(got)
s.close()
dist.barrier()
dist.destroy_process_group()
assert e1 <= 1e-13 and e2 <= 1e-13 and e3 == 0.0 and pad_ok, (rank, e1, e2, e3, pad_ok)
print(f"rank {rank}/{P} ok {e1:.2e} {e2:.2e}")
"""


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("n,world,backend", [(64, 2, "gloo"), (128, 4, "gloo"), (512, 2, "gloo"),
                                             (256, 1, "nccl")])
def test_slab_fft_matches_numpy(n, world, backend):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE=str(world),
                   LOCAL_RANK="0", NCCL_NVLS_ENABLE="0")
        procs.append(subprocess.Popen([sys.executable, "-c", _RANK, os.path.join(ROOT, "ternary-chns_b200"), str(n),
                                       backend], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            outs.append(p.communicate(timeout=240)[0])
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    for r, (p, o) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, f"rank {r}:\n{o}"
        assert f"rank {r}/{world} ok" in o, o

