"""CPU tests of the adjoint's checker: oracle/torch_step.py restates the reference step
(pure Navier-Stokes, binary and ternary, coef_mode 1) in torch so that reverse mode gives the exact
gradient of the discrete map.  Pinned here against the C restatement:

* forward: 12 steps from the golden initial states equal the C restatement's to
  1e-14 relative L2;
* gradients: directional derivatives along seeded random directions of every
  state field, and the derivatives with respect to every parameter, equal central
  differences of the C restatement's loss to 1e-6 relative (each step size chosen
  where the difference quotient is accurate: the loss is nearly linear in omega and
  in nu, so those take larger steps);
* the golden gradients tests/golden/adjoint_*.npz (tests/golden/make_adjoint_golden.py)
  are reproduced to 1e-12.

The gradients are with respect to the stored real and imaginary parts of the
initial spectral state (g = dJ/dRe + i dJ/dIm), the convention of chns_adjoint."""
import json
import os
import sys

import numpy as np
import pytest

import oracle as O
from _golden import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_adjoint_golden as MA  # noqa: E402

torch = pytest.importorskip("torch")
import torch_step as TS  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _lib():
    O.build_oracle_lib()


def _loss_of_c_oracle(p, state, steps):
    """The loss of the C restatement's final state (torch only evaluates it)."""
    o = O.Oracle(p)
    o.set_state(*state)
    o.step(steps)
    fin = [torch.from_numpy(a) for a in o.get_state()]
    prm = {k: torch.tensor(float(p[k]), dtype=torch.float64) for k in TS.PARAM_NAMES[p["model"]]}
    with torch.no_grad():
        return float(TS.TorchStep(p).loss(fin, prm))


def _rdot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


@pytest.mark.parametrize("name", MA.CASES)
def test_torch_forward_equals_c_restatement(name):
    p, init = MA.case(name)
    o = O.Oracle(p)
    o.set_state(*init)
    o.step(MA.STEPS)
    want = o.get_state()
    got = TS.forward(p, init, MA.STEPS)
    for a, b, s0 in zip(want, got, init):
        assert rel_l2(b, a) <= 1e-14
        assert rel_l2(a, s0) >= 1e-4  # the state moved: the comparison is not of the initial state


@pytest.mark.parametrize("name", MA.CASES)
def test_gradients_equal_central_differences_of_c_restatement(name):
    p, init = MA.case(name)
    J, gw, gcs, gp = TS.gradient(p, init, MA.STEPS)
    assert J == pytest.approx(_loss_of_c_oracle(p, init, MA.STEPS), rel=1e-14)
    rng = np.random.default_rng(3)
    for k, g in enumerate([gw] + gcs):
        d = rng.standard_normal(init[k].shape) + 1j * rng.standard_normal(init[k].shape)
        d *= np.abs(init[k]).max() / np.abs(d).max()
        # the phase-field losses are nearly linear in omega; the pure Navier-Stokes one is not
        h = 1e-2 if k == 0 and p["model"] != 0 else 1e-6
        plus = [s + h * d if i == k else s for i, s in enumerate(init)]
        minus = [s - h * d if i == k else s for i, s in enumerate(init)]
        fd = (_loss_of_c_oracle(p, plus, MA.STEPS) - _loss_of_c_oracle(p, minus, MA.STEPS)) / (2 * h)
        assert abs(_rdot(g, d) - fd) <= 1e-6 * abs(fd), (name, k, _rdot(g, d), fd)
    for i, nm in enumerate(TS.PARAM_NAMES[p["model"]]):
        h = (1e-4 if p["model"] == 0 else 1e-1 if nm == "nu" else 1e-6) * abs(p[nm])
        fd = (_loss_of_c_oracle(dict(p, **{nm: p[nm] + h}), init, MA.STEPS)
              - _loss_of_c_oracle(dict(p, **{nm: p[nm] - h}), init, MA.STEPS)) / (2 * h)
        assert abs(gp[i] - fd) <= 1e-6 * abs(fd), (name, nm, gp[i], fd)


@pytest.mark.parametrize("name", MA.CASES)
def test_golden_gradients_reproduce(name):
    z = np.load(os.path.join(HERE, "golden", f"adjoint_{name}.npz"))
    assert json.loads(str(z["params"])) == MA.case(name)[0]
    got = MA.compute(name)
    assert got["J"] == pytest.approx(float(z["J"]), rel=1e-13)
    assert rel_l2(got["g_w"], z["g_w"]) <= 1e-12
    assert rel_l2(got["g_c"], z["g_c"]) <= 1e-12
    assert np.allclose(got["g_params"], z["g_params"], rtol=1e-12, atol=0)


def test_state_gradients_are_hermitian_in_the_real_columns():
    """Only the real fields reach the loss, so the gradient with respect to the
    ky = 0 column is Hermitian (g[n - i, 0] = conj g[i, 0]), like the fields'."""
    z = np.load(os.path.join(HERE, "golden", "adjoint_bin64.npz"))
    for g in (z["g_w"], z["g_c"][0]):
        col = g[:, 0]
        n = col.shape[0]
        mirror = np.conj(col[(-np.arange(n)) % n])
        assert np.abs(col - mirror).max() <= 1e-12 * np.abs(g).max()
