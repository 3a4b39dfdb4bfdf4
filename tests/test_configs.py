"""The named run configurations (chns_b200.configs): parameters accepted by the C
ABI's validation (no GPU needed), seeded initial states reproducible, and every
ensemble member well posed (all spreading coefficients gamma_i >= 0.1)."""
import ctypes

import numpy as np


def test_configs_validate_and_repeat():
    import chns_b200 as C
    from chns_b200 import configs

    L = C.load_library()
    cases = [configs.binary_spinodal(64)[0], configs.ternary_spinodal(64)[0],
             configs.binary_kolmogorov(64)[0], configs.binary_adjoint(64)[0]]
    cases += [p for p, _ in configs.ternary_ensemble()[:3]]
    for p in cases:
        q = dict(p, nx=8192, ny=8192)  # an unsupported size is rejected before CUDA is touched
        h = ctypes.c_void_p()
        assert L.chns_create(ctypes.byref(C.make_params(q)), ctypes.byref(h)) == -5
    a = configs.binary_kolmogorov(64)
    b = configs.binary_kolmogorov(64)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert np.array_equal(configs.binary_adjoint(32)[1], configs.binary_adjoint(32)[1])


def test_ensemble_members_are_well_posed():
    from chns_b200 import configs

    members = configs.ternary_ensemble()
    assert [p["nx"] for p, _ in members].count(256) == 32
    assert [p["nx"] for p, _ in members].count(512) == 24
    assert [p["nx"] for p, _ in members].count(1024) == 8
    for p, (c1, c2) in members:
        s12, s13, s23 = p["sigma12"], p["sigma13"], p["sigma23"]
        assert 0.15 <= min(s12, s13, s23) and max(s12, s13, s23) <= 0.35
        assert min(s12 + s13 - s23, s12 + s23 - s13, s13 + s23 - s12) >= 0.1
        assert abs(c1.mean() - 1 / 3) < 1e-3 and np.abs(c1 - 1 / 3).max() <= 0.02
    assert len({(p["sigma12"], p["sigma13"]) for p, _ in members}) == len(members)
