"""Generate tests/golden/ref_fft.npz from the reference's own CPU FFT.

The reference's Source/FastFourierTransformCPU/FastFourierTransform.cpp is
compiled unmodified from the reference checkout by oracle/Makefile into
oracle/_ref/libreffft.so; this script runs it on seeded inputs and stores
inputs and outputs. Run it where the reference sources are present:

    python tests/golden/make_golden.py

The fixture pins the oracle's FFT restatement (PI_MODE_REPO must reproduce
these bits) without needing the reference on the machine that runs tests.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_fft.npz"


def main() -> None:
    O.build(with_ref=True)
    if not O.ref_available():
        raise SystemExit("reference sources not available: cannot regenerate the golden vectors")
    rng = np.random.default_rng(20240530)
    data = {"pi_repo": np.float64(O.ref().ref_pi())}
    for n in (2, 8, 64, 512, 2048):
        z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        data[f"fft_in_{n}"] = z
        data[f"fft_out_{n}"] = O.ref_fft(z)
        data[f"ifft_out_{n}"] = O.ref_fft(z, inverse=True)
    # the survey's known answer: forward FFT of 0..7
    data["fft_ramp8_out"] = O.ref_fft(np.arange(8.0))
    # rows filtered along the reference's path with its FFT
    for m, filt in ((367, O.RAM_LAK), (768, O.SHEPP_LOGAN), (384, O.HANN)):
        rows = rng.standard_normal((4, m)).astype(np.float32)
        rows += np.linspace(0, 3, m, dtype=np.float32)  # a DC-heavy component
        data[f"filter_in_{m}_{filt}"] = rows
        data[f"filter_out_{m}_{filt}"] = O.ref_filter_rows(rows, filt)
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
