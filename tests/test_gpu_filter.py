"""Contexts with the SMOOTH_FILTER truncation (chns_params.filter =
CHNS_FILTER_SMOOTH: the reference built with SMOOTH_FILTER, macro.h:15,
functions.c:69-72) on the GPU.

The small configurations (nssf32, binsf64, tersf64, binsfdef64) also run through
the golden tests of test_gpu_parity (right-hand side within 1e-12, 20 steps within
1e-11 of the reference built with the macro, diagnostics, phase init) and binsf64
through the drop-in test.  Here: the large-grid kernels, where every G row is live
and the row kernels' tiles hold all n/2+1 rows, against the oracle run live on the
same inputs (FP64 within 1e-11 relative L2); FP32 and FP32_STATE64 against FP64
(1e-5); ensembles of filtered members; and the refusal of the adjoint."""
import math
import os

import numpy as np
import pytest

import make_golden as MG
from _golden import load_small, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


def _params(model, n, **kw):
    lx = 2 * math.pi
    p = dict(model=model, nx=n, ny=n, lx=lx, ly=lx, nu=0.01, epsilon=2.0 * lx / n, filter=1)
    if model == 1:
        p.update(dt=2e-6, nu=1e-3, sigma=0.1)
        p["lambda"] = 1e-3
    elif model == 2:
        p.update(dt=5e-6, sigma12=0.2, sigma13=0.3, sigma23=0.25, xlambda=2.0)
        p["lambda"] = 0.005
    else:
        p.update(dt=1e-3)
    p.update(kw)
    return p


@pytest.mark.parametrize("model,n,steps", [(2, 1024, 2), (1, 2048, 2), (1, 4096, 1), (0, 512, 3)])
def test_large_grids_match_the_oracle(chns, model, n, steps):
    """Spinodal noise plus random low-k vorticity, stepped by the GPU and by the
    oracle (the C restatement, checked bitwise against the reference built with
    SMOOTH_FILTER): every field within 1e-11 relative L2."""
    import oracle as O

    p = _params(model, n)
    p1, p2, w = MG.initial_state(model, n, p["lx"], 200 + n, 300 + n, 8.0, 0.1)
    o = O.Oracle(p, nthreads=min(16, os.cpu_count() or 1))
    MG.apply_initial(o, model, p1, p2, w)
    st0 = o.get_state()
    o.step(steps)
    with chns.Context(p) as c:
        assert c.tma_tiles()
        c.set_state(*st0)
        c.step(steps)
        c.check()
        for k, (a, b) in enumerate(zip(c.get_state(), o.get_state())):
            assert rel_l2(a, b) <= 1e-11, (model, n, k, rel_l2(a, b))


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("name", ["binsf64", "tersf64"])
def test_fp32_close_to_fp64(chns, name, prec):
    g = load_small(name)
    p = g["params"]
    with chns.Context(p) as a, chns.Context(dict(p, precision=prec, coef_mode=1)) as b:
        a.set_state(*g["init"])
        b.set_state(*g["init"])
        a.step(20)
        b.step(20)
        for x, y in zip(b.get_state(), a.get_state()):
            assert rel_l2(x, y) <= 1e-5, (name, prec, rel_l2(x, y))


@pytest.mark.parametrize("prec", [1, 2])
def test_fp32_large_grid_close_to_fp64(chns, prec):
    """The FP32 row and spectral kernels at 4096^2 with full-height tiles."""
    p = _params(1, 4096)
    p1, _, w = MG.initial_state(1, 4096, p["lx"], 401, 402, 8.0, 0.1)
    with chns.Context(p) as a, chns.Context(dict(p, precision=prec)) as b:
        for c in (a, b):
            MG.apply_initial(c, 1, p1, None, w)
            c.step(3)
            c.check()
        for x, y in zip(b.get_state(), a.get_state()):
            assert rel_l2(x, y) <= 1e-5, (prec, rel_l2(x, y))


def test_filter_differs_from_the_sharp_cut(chns):
    """The switch reaches the kernels: the same 20 steps with the sharp cut end
    about 1% away, and match the sharp cut's own golden run."""
    g = load_small("binsf64")
    sharp = load_small("bin64")
    p = dict(g["params"])
    p.pop("filter")
    assert p == sharp["params"]
    with chns.Context(p) as c:
        c.set_state(*g["init"])
        c.step(20)
        st = c.get_state()
    for a, b, s in zip(st, g["final"], sharp["final"]):
        assert rel_l2(a, b) > 1e-4
    with chns.Context(p) as c:
        c.set_state(*sharp["init"])
        c.step(20)
        for a, b in zip(c.get_state(), sharp["final"]):
            assert rel_l2(a, b) <= 1e-11


def test_ensemble_of_filtered_members_matches_lone_contexts(chns):
    g = load_small("tersf64")
    p = g["params"]
    members = [p, dict(p, dt=p["dt"] * 0.5)]
    with chns.Ensemble(members) as ens:
        assert not ens.persistent
        with pytest.raises(chns.ChnsError):
            ens.persistent = True  # the persistent kernel runs the sharp cut only
        for m in ens.members:
            m.set_state(*g["init"])
        ens.step(5)
        ens.synchronize()
        got = [m.get_state() for m in ens.members]
    for k, q in enumerate(members):
        with chns.Context(q) as c:
            c.set_state(*g["init"])
            c.step(5)
            for a, b in zip(got[k], c.get_state()):
                assert np.array_equal(a, b)


def test_adjoint_is_refused(chns):
    g = load_small("binsf64")
    with chns.Context(g["params"]) as c:
        c.set_state(*g["init"])
        with pytest.raises(chns.ChnsError) as e:
            c.adjoint(4, 2)
        assert e.value.status == -5
