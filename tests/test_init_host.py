"""The host half of CHNS_INIT_C_NOISE: the ternary noise is the C library's
rand() sequence after srand(seed), two draws per grid point in row-major order
(init.c:264-292).  Pinned here on the CPU: those draws, put through the oracle's
dfft and truncation, reproduce the reference's own init() state bit for bit
(tests/golden/init_ref.npz, seed 10 as in the reference on rank 0)."""
import ctypes
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def libc_draws(seed: int, count: int) -> np.ndarray:
    libc = ctypes.CDLL("libc.so.6")
    libc.srandom.argtypes = [ctypes.c_uint]
    libc.random.restype = ctypes.c_long
    libc.srandom(seed)
    return np.array([libc.random() for _ in range(count)], dtype=np.float64)


@pytest.mark.parametrize("name", ["ter32", "terdef64"])
def test_noise_draws_match_reference_init(name):
    import oracle as O

    z = np.load(os.path.join(HERE, "golden", "init_ref.npz"))
    p = json.loads(str(z[f"{name}_params"]))
    n = p["nx"]
    r = libc_draws(10, 2 * n * n).reshape(n, n, 2)
    rand_max = 2147483647.0
    phi1 = (1.0 / 4.0) + 0.001 * (r[..., 0] / rand_max)
    phi2 = (1.0 / 4.0) + 0.001 * (r[..., 1] / rand_max)
    o = O.Oracle(p)
    o.set_phase_real(phi1, phi2)
    st = o.get_state()
    assert np.array_equal(st[1], z[f"{name}_state1"])
    assert np.array_equal(st[2], z[f"{name}_state2"])
