"""Field files in the reference's format (write_array.c / read_array.c): raw FP64
nx x ny, x the slow index.  The dumps hold the reference's ifft of the state
(restated by the oracle; FP64 relative L2 <= 1e-13), with DUMP_REAL_MPI's
truncation when asked; reading a phase file equals chns_set_phase_real on the
same array, bit for bit; unreadable files give CHNS_ERR_IO."""
import ctypes

import numpy as np
import pytest

from _golden import load_small, rel_l2

pytestmark = pytest.mark.gpu
NAMES = {0: ["vort/wz"], 1: ["vort/wz", "phase_field/phi"],
         2: ["vort/wz", "phase_field/phi1", "phase_field/phi2"]}


@pytest.fixture(scope="module")
def chns():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    import chns_b200

    chns_b200.load_library()
    return chns_b200


@pytest.mark.parametrize("truncate", [False, True])
@pytest.mark.parametrize("name", ["ns32", "bin32", "ter32", "terdef64"])
def test_dumps_match_reference_ifft(chns, tmp_path, name, truncate):
    import oracle as O

    g = load_small(name)
    p = g["params"]
    n = p["nx"]
    ref = O.Oracle(p)
    with chns.Context(p) as c:
        c.set_state(*g["final"])
        c.write_fields(str(tmp_path), 12, truncate=truncate)
    for k, stem in enumerate(NAMES[p["model"]]):
        path = tmp_path / f"{stem}.12"
        assert path.stat().st_size == n * n * 8
        got = np.fromfile(path, dtype=np.float64).reshape(n, n)
        spec = ref.truncation(g["final"][k]) if truncate else g["final"][k]
        want = ref.ifft(spec)
        assert rel_l2(got, want) <= 1e-13, (stem, rel_l2(got, want))


def test_read_phase_equals_set_phase_real(chns, tmp_path):
    g = load_small("ter32")
    p = g["params"]
    n = p["nx"]
    rng = np.random.default_rng(5)
    a = 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n))
    b = 1 / 3 + 0.02 * rng.uniform(-1, 1, (n, n))
    a.tofile(tmp_path / "phi1.in")
    b.tofile(tmp_path / "phi2.in")
    with chns.Context(p) as c1, chns.Context(p) as c2:
        c1.read_phase(str(tmp_path / "phi1.in"), str(tmp_path / "phi2.in"))
        c2.set_phase_real(a, b)
        for x, y in zip(c1.get_state(), c2.get_state()):
            assert np.array_equal(x, y)
        # a short file and a missing one
        a[: n // 2].tofile(tmp_path / "short.in")
        with pytest.raises(chns.ChnsError) as e:
            c1.read_phase(str(tmp_path / "short.in"), str(tmp_path / "phi2.in"))
        assert e.value.status == -7
        with pytest.raises(chns.ChnsError) as e:
            c1.read_phase(str(tmp_path / "missing.in"), str(tmp_path / "phi2.in"))
        assert e.value.status == -7


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["bin32", "ter32", "ns32"])
def test_checkpoint_resume_is_bit_exact(chns, tmp_path, name, prec):
    g = load_small(name)
    p = dict(g["params"], precision=prec)
    path = str(tmp_path / "run.ckpt")
    with chns.Context(p) as a:
        a.set_state(*g["init"])
        a.step(7)
        a.save(path)
        a.step(9)
        want = a.get_state()
    with chns.Context(p) as b:
        b.load(path)
        b.step(9)
        got = b.get_state()
    for x, y in zip(got, want):
        assert np.array_equal(x, y)
    # a context with other parameters refuses the file
    with chns.Context(dict(p, dt=p["dt"] * 2)) as c:
        with pytest.raises(chns.ChnsError) as e:
            c.load(path)
        assert e.value.status == -1


@pytest.mark.parametrize("name", ["bin32", "ter32", "ns32"])
def test_logs_write_the_reference_files(chns, tmp_path, name):
    from chns_b200 import logs

    g = load_small(name)
    p = g["params"]
    with chns.Context(p) as c:
        c.set_state(*g["init"])
        lg = logs.Logs(c, str(tmp_path))
        lg.record(0.0)
        c.step(2)
        lg.record(2 * p["dt"])
    names = {0: ["ken_t.dat"], 1: ["free_en_t.dat", "ken_t.dat", "gamma.dat"],
             2: ["free_en_t.dat", "ken_t.dat", "gamma1.dat", "gamma2.dat"]}[p["model"]]
    for nm in names:
        lines = open(tmp_path / "data" / nm).read().splitlines()
        assert len(lines) == 2, nm
    for i in (0, 1):
        for stem in ("spectrum", "Xspectrum", "Yspectrum"):
            assert (tmp_path / "spectra" / f"{stem}.{i}").stat().st_size > 0


def test_pinned_host_arrays(chns):
    g = load_small("ter32")
    p = g["params"]
    with chns.Context(p) as c:
        bufs = [a.copy() for a in g["init"]]
        for b in bufs:
            c.pin_host(b)
        c.pin_host(bufs[0])  # again: accepted
        c.set_state(*bufs)
        c.step(g["steps"])
        out = [np.empty_like(b) for b in bufs]
        for o in out:
            c.pin_host(o)
        c.L.chns_get_state(c.handle, *[ctypes.c_void_p(o.ctypes.data) for o in out], 0)
        for o, ref in zip(out, g["final"]):
            assert rel_l2(o, ref) <= 1e-11
        for b in bufs + out:
            c.unpin_host(b)
        with pytest.raises(chns.ChnsError):
            c.unpin_host(bufs[0])
