"""The reference arm of bench.py (`--impl reference`): the reference's own etd2rk()
(oracle/_ref, compiled from the reference's C sources) timed on the host cores,
printing the bench's JSON line with `"impl": "reference"`.  Under torchrun only
rank 0 runs it; the other ranks exit 0 without work.  CPU only."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


def _ref_built(name):
    import oracle as O

    return os.path.isfile(O.build_ref.lib_path(name))


def test_reference_arm_json_line():
    if not _ref_built("bin256"):
        pytest.skip("oracle/_ref/bin256 not built (no reference sources here)")
    r = _run({}, "--n", "256", "--steps", "2", "--warmup", "1")
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference"
    assert d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2
    assert d["warmup"] >= 3  # at least three untimed steps, whatever was asked
    assert d["ms_per_step"] == pytest.approx(1e3 / d["value"], rel=1e-3)
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_no_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--n", "256", "--steps", "2")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
