"""Autotuner and its cache file on the GPU.

In a child process with NOTORIOUS_FFT_TUNE_CACHE pointing at a temporary file
(the cache is loaded once per process): tune two (kind, N) pairs, check that
the file records them for this GPU, that notorious_fft_tune_lookup returns the
same splits, and that a ragged batch planned with the cached splits still
matches the oracle.  Entries of other GPUs are kept when the file is
rewritten.  (A cached split this build cannot run falls back to the default
schedule; the emulator test covers that.)
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys, json, numpy as np
sys.path.insert(0, sys.argv[1])
from notorious_fft import load
lib = load(False)
lib.autotune("dft", 1 << 15)
lib.autotune("realdft", 1 << 14)
res = {"dft": lib.tune_lookup("dft", 1 << 15), "realdft": lib.tune_lookup("realdft", 1 << 14),
       "absent": lib.tune_lookup("dct2", 1 << 16)}
kinds, Ns = ["dft", "realdft", "dct2", "dft"], [1 << 15, 1 << 14, 1 << 16, 1 << 15]
b = lib.mkbatch(kinds, Ns)
x = np.random.default_rng(3).uniform(-1, 1, b.in_size)
y = np.zeros(b.out_size)
b.execute(x, y)
np.savez(sys.argv[2], x=x, y=y)
print(json.dumps(res))
'''


def test_autotune_cache(tmp_path, lib_d, oracle_d):
    cache = tmp_path / "tune.json"
    # an entry of another GPU, which must survive the rewrite
    cache.write_text('{"format": "notorious_fft tune cache 1", "entries": [\n'
                     '{"device": "some other GPU", "key": "f64:dft:32768", "split": [5, 10], "us": 1.0}\n]}\n')
    out = tmp_path / "out.npz"
    env = dict(os.environ, NOTORIOUS_FFT_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "notorious-fft_b200"), str(out)], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert sum(res["dft"]) == 15 and sum(res["realdft"]) == 13     # complex length of realdft is N/2
    assert res["absent"] == []
    text = cache.read_text()
    assert "some other GPU" in text                                # other devices' entries are kept
    entries = [json.loads(l.rstrip(",")) for l in text.splitlines() if l.startswith('{"device"')]
    mine = {e["key"]: e for e in entries if e["device"] != "some other GPU"}
    assert mine["f64:dft:32768"]["split"] == res["dft"]
    assert mine["f64:realdft:16384"]["split"] == res["realdft"]
    d = np.load(out)
    x, y = d["x"], d["y"]
    n = 1 << 15
    xc = x[: 2 * n][0::2] + 1j * x[: 2 * n][1::2]
    assert rel_l2(y[: 2 * n][0::2] + 1j * y[: 2 * n][1::2], oracle_d.transform("dft", xc)) <= 3e-15 * 15


CHILD_PLAN = r'''
import sys, json, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
from notorious_fft import load
from oracle import Oracle, rel_l2
lib = load(False)
o = Oracle()
n = 1 << 14
with lib.mkaux("dft", [n]) as a:
    before = a.schedule()
lib.autotune("dft", n)
tuned = lib.tune_lookup_plan("dft", n)
res = {"before": before, "tuned": tuned}
rng = np.random.default_rng(5)
for m in (n, 1 << 16):
    x = rng.uniform(-1, 1, (3, m)) + 1j * rng.uniform(-1, 1, (3, m))
    with lib.mkaux("dft", [m]) as a:
        y = np.zeros_like(x)
        a.batched("dft", x, y, 3, m, m)
        res[f"sched{m}"] = a.schedule()
        res[f"err{m}"] = max(rel_l2(y[b], o.transform("dft", x[b])) for b in range(3))
print(json.dumps(res))
'''


def test_standalone_plans_use_the_tuned_schedule(tmp_path, lib_d):
    """notorious_fft_autotune also tunes standalone plans; a later mkaux runs the
    cached schedule (first child).  A hand-written entry for this GPU (its tag
    taken from the file the first child wrote) with split [10, 6] and 256-thread
    kernels changes the schedule a plain 2^16 mkaux runs (second child), and
    both results match the oracle."""
    cache = tmp_path / "tune.json"
    env = dict(os.environ, NOTORIOUS_FFT_TUNE_CACHE=str(cache))
    args = [sys.executable, "-c", CHILD_PLAN, os.path.join(ROOT, "notorious-fft_b200"), os.path.join(ROOT, "oracle")]
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["tuned"] is not None
    split, logt = res["tuned"]
    assert res["sched16384"][1] == logt
    if split:
        assert res["sched16384"][0] == split
    assert res["err16384"] <= 1e-13 * 14 and res["err65536"] <= 1e-13 * 16
    assert res["sched65536"][0] == [8, 8]                     # no entry: the default schedule
    entries = [json.loads(l.rstrip(",")) for l in cache.read_text().splitlines() if l.startswith('{"device"')]
    tag = entries[0]["device"]
    entries.append({"device": tag, "key": "f64:plan:dft:65536", "split": [10, 6], "logt": 8, "us": 1.0})
    cache.write_text('{"format": "notorious_fft tune cache 1", "entries": [\n' +
                     ",\n".join(json.dumps(e) for e in entries) + "\n]}\n")
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["sched65536"] == [[10, 6], 8]
    assert res["err65536"] <= 1e-13 * 16
