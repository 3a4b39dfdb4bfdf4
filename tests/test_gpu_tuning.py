"""The autotuner's run-time launch-shape choices (chns_tune_override: rows per
TMA box of the row kernels' tiles, the P1 split, P4's grad c from P2's real-space
copy or from its own transform, programmatic dependent launches) change no result
bit: every
choice gives the state of the tuned default bit for bit, on grids whose tiles
take one or several boxes, in both precisions and with the smooth filter."""
import math

import numpy as np
import pytest

import make_golden as MG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


def _run(chns, p, steps, ph, w):
    with chns.Context(p) as c:
        MG.apply_initial(c, p["model"], ph[0], ph[1], w)
        c.step(steps)
        c.check()
        return c.get_state()


@pytest.mark.parametrize("model,n,prec,filt", [(1, 256, 1, 0), (2, 512, 0, 0), (1, 2048, 1, 0), (1, 1024, 2, 0),
                                              (2, 256, 1, 1), (1, 4096, 1, 0)])
def test_launch_shapes_change_no_bit(chns, model, n, prec, filt):
    lx = 2 * math.pi
    p = dict(model=model, nx=n, ny=n, lx=lx, ly=lx, dt=1e-6, nu=0.01, epsilon=2 * lx / n, sigma=0.2,
             sigma12=0.2, sigma13=0.3, sigma23=0.25, precision=prec, coef_mode=1, filter=filt)
    p["lambda"] = 0.005
    p1, p2, w = MG.initial_state(model, n, lx, 500 + n, 501 + n, 8.0, 0.1)
    ref = _run(chns, p, 3, (p1, p2), w)
    try:
        for knob, values in ((chns.TUNE_TMA_BOX_ROWS, (64, 128, 256, 8)), (chns.TUNE_P1_SPLIT, (0, 1)),
                             (chns.TUNE_P4_GRAD, (0, 1)), (chns.TUNE_PDL, (0, 1))):
            for v in values:
                chns.tune_override(knob, v)
                got = _run(chns, p, 3, (p1, p2), w)
                for a, b in zip(got, ref):
                    assert np.array_equal(a, b), (knob, v)
            chns.tune_override(knob, -1)
    finally:
        chns.tune_override(chns.TUNE_TMA_BOX_ROWS, -1)
        chns.tune_override(chns.TUNE_P1_SPLIT, -1)
        chns.tune_override(chns.TUNE_P4_GRAD, -1)
        chns.tune_override(chns.TUNE_PDL, -1)
