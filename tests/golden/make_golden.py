"""Generate tests/golden/reference_outputs.npz from the reference itself.

Runs the reference's own C API, compiled from its sources by oracle/Makefile
into oracle/_ref/libref_{d_avx2,d_scalar,s_scalar}.so, on the cases of the
reference's test suite (tests/test_notoriousfft.c: the sin fixture of :45-48,
the 1-D size list of :673, the 2-D / 3-D shapes of :716-766, the Bluestein
sizes of :770) plus a few larger seeded cases and the N-D edge shapes whose
length-1 axes exercise the reference's recursion quirks.

    make -C oracle && python tests/golden/make_golden.py

Only this container has the reference sources; the fixture file is committed
and travels instead.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import KINDS, Reference, ref_fill  # noqa: E402

REF_SIZES = [1, 2, 4, 8, 16, 32, 64, 128, 256, 1024]
BLUESTEIN = [3, 5, 6, 7, 10, 12, 15, 20, 100]
ND_2D = [(4, 4), (8, 16), (32, 32)]
ND_3D = [(4, 4, 4), (4, 8, 8)]
EDGE = [(1, 8), (8, 1), (2, 1, 4), (16, 1, 1), (1, 1)]
LARGE = {"dft": [4096], "invdft": [2048], "realdft": [8192], "dct2": [4096], "dst2": [2048], "dct4": [4096]}


def inputs_for(kind, dims, single, rng=None):
    total = int(np.prod(dims))
    rdt = np.float32 if single else np.float64
    cdt = np.complex64 if single else np.complex128
    if rng is not None:
        if kind in ("dft", "invdft"):
            return (rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims)).astype(cdt)
        return rng.uniform(-1, 1, dims).astype(rdt)
    if kind in ("dft", "invdft"):
        f = ref_fill(2 * total)
        return (f[0::2] + 1j * f[1::2]).reshape(dims).astype(cdt)
    if kind == "invrealdft":
        return None
    return ref_fill(total).reshape(dims).astype(rdt)


def main():
    out = {}
    refs = {v: Reference(v) for v in ("d_avx2", "d_scalar", "s_scalar")}
    for variant, ref in refs.items():
        single = ref.single
        for n in REF_SIZES:
            for k in KINDS:
                if k == "invrealdft":
                    if n == 1:
                        continue
                    x = ref.run("realdft", inputs_for("realdft", (n,), single), (n,))
                else:
                    x = inputs_for(k, (n,), single)
                y = ref.run(k, x, (n,))
                out[f"{variant}/{k}/{n}/x"] = x
                out[f"{variant}/{k}/{n}/y"] = y
        if variant == "d_avx2":
            for dims in ND_2D + ND_3D + EDGE:
                kinds = ["dft", "invdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4"]
                if dims in ND_3D:
                    kinds = ["dft", "invdft", "dct2"]
                for k in kinds:
                    x = inputs_for(k, dims, False)
                    y = ref.run(k, x, dims)
                    tag = "x".join(map(str, dims))
                    out[f"{variant}/{k}/{tag}/x"] = x
                    out[f"{variant}/{k}/{tag}/y"] = y
            rng = np.random.default_rng(12345)
            for k, sizes in LARGE.items():
                for n in sizes:
                    x = inputs_for(k, (n,), False, rng)
                    out[f"{variant}/{k}/{n}/x"] = x
                    out[f"{variant}/{k}/{n}/y"] = ref.run(k, x, (n,))
        if variant == "d_scalar":
            # the only reference build whose Bluestein path is correct
            for n in BLUESTEIN:
                for k in ("dft", "invdft"):
                    x = inputs_for(k, (n,), False)
                    out[f"{variant}/{k}/{n}/x"] = x
                    out[f"{variant}/{k}/{n}/y"] = ref.run(k, x, (n,))
    path = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {len(out)} arrays to {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
