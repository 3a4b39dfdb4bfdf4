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
