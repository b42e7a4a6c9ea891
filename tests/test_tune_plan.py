"""Standalone plans consult the tune cache (CPU, emulator build).

A child process with NOTORIOUS_FFT_TUNE_CACHE pointing at a hand-written
cache file (the cache is loaded once per process) builds plain mkaux_* plans:
a cached split and thread count must become the schedule the plan runs
(notorious_fft_aux_schedule), an entry whose split the planner cannot run
keeps the default schedule, and the results still match the oracle.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TAG = "emulated sm_100 sm_100 driver 0"

CHILD = r'''
import sys, json, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
from notorious_fft import Library
from oracle import Oracle, rel_l2
L = Library(sys.argv[3])
o = Oracle()
out = {}
rng = np.random.default_rng(4)
for fam, n, kind in (("dft", 1 << 16, "dft"), ("realdft", 1 << 14, "realdft"), ("t2t3", 4096, "dct2"),
                     ("dft", 1 << 15, "dft")):
    with L.mkaux(fam, [n]) as a:
        sched = a.schedule()
        x = rng.uniform(-1, 1, n) + (1j * rng.uniform(-1, 1, n) if fam == "dft" else 0)
        err = rel_l2(a(kind, x), o.transform(kind, x))
    out[f"{fam}:{n}"] = {"split": sched[0], "logt": sched[1], "err": err,
                         "lookup": L.tune_lookup_plan(kind, n)}
print(json.dumps(out))
'''


def test_plans_use_cached_schedules(tmp_path):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "emu")], check=True)
    cache = tmp_path / "tune.json"
    entries = [
        {"device": TAG, "key": "f64:plan:dft:65536", "split": [10, 6], "logt": 8, "us": 1.0},
        {"device": TAG, "key": "f64:plan:realdft:16384", "split": [], "logt": 7, "us": 1.0},
        {"device": TAG, "key": "f64:plan:t2t3:4096", "split": [15, 1], "logt": 0, "us": 1.0},   # not runnable
        {"device": "some other GPU", "key": "f64:plan:dft:32768", "split": [5, 10], "logt": 7, "us": 1.0},
    ]
    cache.write_text('{"format": "notorious_fft tune cache 1", "entries": [\n' +
                     ",\n".join(json.dumps(e) for e in entries) + "\n]}\n")
    env = dict(os.environ, NOTORIOUS_FFT_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "notorious-fft_b200"),
                        os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "emu", "_build", "libnfft_emu_d.so")],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["dft:65536"]["split"] == [10, 6] and res["dft:65536"]["logt"] == 8
    assert res["dft:65536"]["lookup"] == [[10, 6], 8]
    assert res["realdft:16384"]["split"] == [13] and res["realdft:16384"]["logt"] == 7   # default split, tuned threads
    assert res["t2t3:4096"]["split"] == [11]                                              # fallback to the default
    assert res["dft:32768"]["split"] == [8, 7] and res["dft:32768"]["logt"] == 0          # other GPU's entry ignored
    assert res["dft:32768"]["lookup"] is None
    for k, v in res.items():
        assert v["err"] <= 1e-13 * 16, (k, v["err"])
