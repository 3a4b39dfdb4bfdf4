"""The literal drop-in: the reference's own sources with etd2rk.c replaced by
ternary-chns_b200/csrc/etd2rk_dropin.c (same signature, GPU step), driven like
the reference (oracle/ref_harness.c), against the reference's golden vectors."""
import os

import pytest

import oracle as O
from _golden import load_small, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", O.build_ref.DROPIN_CONFIGS)
def test_reference_main_loop_with_gpu_etd2rk(name):
    path = O.build_ref.lib_path(name, dropin=True)
    if not os.path.isfile(path):
        pytest.fail(f"{path} missing: build it with oracle/build_ref.py where the reference sources exist")
    g = load_small(name)
    R = O.RefLib(name, dropin=True)
    R.set_state(*g["init"])
    R.step(g["steps"])  # t += dt; etd2rk(cwz, cphi...) -> the GPU through include/chns.h
    for k, (a, b) in enumerate(zip(R.get_state(), g["final"])):
        assert rel_l2(a, b) <= 1e-11, (name, k, rel_l2(a, b))
