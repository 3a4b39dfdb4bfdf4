"""Failure detection without a GPU fault: the failure is made on the host (a NaN
put into the initial state, a configuration that blows up in the reference's own
scheme) and the library reports it through its status codes."""
import math

import numpy as np
import pytest

from _golden import load_small

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("field", [0, 1])
def test_nan_in_the_state_is_reported(chns, prec, field):
    g = load_small("bin32")
    st = [a.copy() for a in g["init"]]
    st[field][3, 2] = complex(float("nan"), 0.0)
    with chns.Context(dict(g["params"], precision=prec)) as c:
        c.set_state(*g["init"])
        c.check()  # clean
        c.step(2)
        c.check()
        c.set_state(*st)
        with pytest.raises(chns.ChnsError) as e:
            c.check()
        assert e.value.status == -3
        c.step(3)  # the NaN spreads through the transforms; the step itself does not fail
        with pytest.raises(chns.ChnsError) as e:
            c.check()
        assert e.value.status == -3
        # the context stays usable: a clean state checks clean again
        c.set_state(*g["init"])
        c.step(1)
        c.check()


def test_blow_up_is_reported_by_check_and_diagnostics(chns):
    """Ternary 512^2 at dt = 5e-4 diverges within a few steps in the reference's
    scheme (NaN by step 5 there); the GPU step diverges the same way."""
    n = 512
    lx = 2 * math.pi
    p = dict(model=2, nx=n, ny=n, lx=lx, dt=5e-4, nu=0.01, epsilon=2 * lx / n, sigma12=0.2, sigma13=0.3,
             sigma23=0.25)
    p["lambda"] = 0.005
    rng = np.random.default_rng(4)
    with chns.Context(p) as c:
        c.set_phase_real(1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)), 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n)))
        c.check()
        c.step(40)
        with pytest.raises(chns.ChnsError) as e:
            c.check()
        assert e.value.status == -3
        fe, ke, rc = c.diagnostics()
        assert rc == -3


@pytest.mark.parametrize("prec", [0, 1])
def test_tile_wait_that_runs_out_is_reported_and_recoverable(chns, prec):
    """The bounded wait of the row kernels for their TMA tiles, made to run out
    on the GPU without a fault: chns_debug_tile_waits stops the tile copies (no
    copy is in flight, so the barriers are ones nothing completes) and bounds
    each wait to 16 polls.  The step's results are garbage; chns_synchronize
    returns CHNS_ERR_TIMEOUT; with the hook off and the flag cleared the same
    context steps exactly as a fresh one."""
    import ctypes

    from chns_b200 import configs

    L = chns.load_library()
    L.chns_debug_tile_waits.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    p, (c_real,) = configs.binary_spinodal(256, prec)
    with chns.Context(p) as ref:
        ref.set_phase_real(c_real)
        st0 = ref.get_state()
        ref.step(5)
        want = ref.get_state()
    with chns.Context(p) as c:
        assert c.tma_tiles()
        c.set_state(*st0)
        assert L.chns_debug_tile_waits(c.handle, 16, 1) == 0
        c.step(2)
        with pytest.raises(chns.ChnsError) as e:
            c.synchronize()
        assert e.value.status == -4
        c.synchronize()  # the flag was cleared by the report
        assert L.chns_debug_tile_waits(c.handle, 0, 0) == 0
        c.set_state(*st0)
        c.step(5)
        c.synchronize()
        for a, b in zip(c.get_state(), want):
            assert np.array_equal(a, b)
    assert L.chns_debug_tile_waits(None, 0, 0) == -1
