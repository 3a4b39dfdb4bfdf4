"""init.c on the device (chns_init_vorticity / chns_init_phase) against the
reference's own init() (tests/golden/init_ref.npz: ZERO_INIT vorticity with the
binary drop and the ternary srand(10) noise, TG_INIT, and the k-space shell
vorticity of the branch selected by neither macro).  FP64 relative L2
<= 1e-13 (the GPU's tanh, sin and cos and the FFT differ from the host's in the
last bits); FP32 contexts <= 1e-6."""
import json
import os

import numpy as np
import pytest

from _golden import rel_l2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {  # name: (vorticity kind, phase kind or None)
    "bin32": (0, 0), "ter32": (0, 1), "bindef64": (0, 0), "terdef64": (0, 1), "nstg32": (1, None),
    "bintg64": (1, 0), "nssh32": (2, None), "binsh64": (2, 0),
}


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_init_matches_reference(chns, name, prec):
    z = np.load(os.path.join(HERE, "golden", "init_ref.npz"))
    p = dict(json.loads(str(z[f"{name}_params"])), precision=prec)
    want = [z[k] for k in sorted(z.files) if k.startswith(name + "_state")]
    wk, ck = CASES[name]
    tol = 1e-13 if prec == 0 else 1e-6
    with chns.Context(p) as c:
        # start from garbage so that every field is really written
        c.set_state(*[np.full(c.shape, 3.0 + 1.0j) for _ in want])
        c.init_vorticity(wk, 1.0)
        if ck is not None:
            c.init_phase(ck, 10)
        got = c.get_state()
    assert len(got) == len(want)
    for k, (a, b) in enumerate(zip(got, want)):
        if np.linalg.norm(b) == 0:
            assert np.linalg.norm(a) == 0, (name, k)
        else:
            assert rel_l2(a, b) <= tol, (name, k, rel_l2(a, b))


def test_init_phase_keeps_vorticity_and_rejects_wrong_model(chns):
    z = np.load(os.path.join(HERE, "golden", "init_ref.npz"))
    p = json.loads(str(z["bintg64_params"]))
    with chns.Context(p) as c:
        c.init_vorticity(1, 1.0)
        w0 = c.get_state()[0]
        c.init_phase(0)
        assert np.array_equal(c.get_state()[0], w0)
        with pytest.raises(chns.ChnsError):
            c.init_phase(1)  # the noise is the ternary model's
        with pytest.raises(chns.ChnsError):
            c.init_vorticity(7)
