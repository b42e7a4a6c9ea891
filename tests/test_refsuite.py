"""The reference project's own test programs, run unchanged.

tests/test_notoriousfft.c and tests/test_notoriousfft.cpp of
NotoriousLOB/Notorious-FFT (its C API suite, :672-780, and its C++17 wrapper
suite, :543-621) are compiled from the reference sources by
tests/refsuite/Makefile against this repository's include/notorious_fft.h.
Their oracle, minfft, is absent here (fetched unpinned at configure time,
CMakeLists.txt:113-129); tests/refsuite/minfft_oracle.c stands in for it,
answering with this repository's long-double oracle.

* CPU: the same programs linked with the reference itself must pass every
  case -- this pins the stand-in.
* GPU: linked with libnotorious_fft.so, every case must pass on the B200
  (host pointers, the drop-in's synchronous path), with the same case count.
"""
import os
import re
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
B = os.path.join(HERE, "refsuite", "_build")
# case counts of the reference's programs (every case printed as PASS/FAIL)
EXPECTED = {"c": 138, "cpp": 150}


def _run(exe):
    if not os.path.exists(exe):
        pytest.skip("reference test programs not built (needs the reference sources; tests/refsuite/Makefile)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    m = re.search(r"Results: (\d+) passed, (\d+) failed", r.stdout)
    assert m, r.stdout[-2000:] + r.stderr[-2000:]
    return r.returncode, int(m.group(1)), int(m.group(2)), r.stdout


@pytest.mark.parametrize("lang", ["c", "cpp"])
def test_reference_passes_its_suite_through_the_minfft_stand_in(lang):
    rc, passed, failed, out = _run(os.path.join(B, f"reference_{lang}"))
    assert rc == 0 and failed == 0, "\n".join(l for l in out.splitlines() if "FAIL" in l)
    assert passed == EXPECTED[lang]


@pytest.mark.gpu
@pytest.mark.parametrize("lang", ["c", "cpp"])
def test_reference_suite_against_the_drop_in(lang):
    rc, passed, failed, out = _run(os.path.join(B, f"test_notoriousfft_{lang}"))
    assert rc == 0 and failed == 0, "\n".join(l for l in out.splitlines() if "FAIL" in l)
    assert passed == EXPECTED[lang]
