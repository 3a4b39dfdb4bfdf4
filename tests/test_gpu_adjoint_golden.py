"""chns_adjoint (FP64, 12 steps, bin64, ter64 and ns32, coef_mode 1) against the golden
gradients of tests/golden/adjoint_*.npz: the exact gradients of the discrete map,
by reverse mode through a torch restatement of the reference step that is pinned on
the CPU against the C restatement (tests/test_oracle_adjoint.py).  The hand-written
adjoint transposes the same operations, so it must agree to round-off rather than
to the 1e-6 of central differences: J to 1e-12, the state and parameter gradients
to 1e-9 relative L2."""
import json
import os

import numpy as np
import pytest

from _golden import load_small, rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


@pytest.mark.parametrize("name", ["bin64", "ter64", "ns32"])
def test_adjoint_equals_golden_gradients(chns, name):
    z = np.load(os.path.join(HERE, "golden", f"adjoint_{name}.npz"))
    p = json.loads(str(z["params"]))
    p["precision"] = chns.FP64
    init = load_small(name)["init"]
    with chns.Context(p) as c:
        c.set_state(*init)
        J, gw, gc, gp = c.adjoint(int(z["steps"]), 5)
    gcs = [] if p["model"] == 0 else [gc] if p["model"] == 1 else list(gc)
    assert len(gcs) == len(z["g_c"])
    assert J == pytest.approx(float(z["J"]), rel=1e-12)
    assert rel_l2(gw, z["g_w"]) <= 1e-9
    for k, g in enumerate(gcs):
        assert rel_l2(g, z["g_c"][k]) <= 1e-9, k
    npar = len(z["g_params"])
    assert np.allclose(gp[:npar], z["g_params"], rtol=1e-9, atol=0)
