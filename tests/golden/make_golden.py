"""Generate the golden fixtures under tests/golden/ (run where the reference
headers exist: `make -C oracle` first builds oracle/_ref/libref_parafaft.so).

Each case runs the reference's own orchestrator — ParaFaFT_C2C<D, OracleBackend>
or ParaFaFT_R2C<D, OracleBackend> compiled from the reference headers
(oracle/ref_parafaft.cpp) — on an input from the reference tests' generators
(test/test_helpers.hpp:106-219), and stores the forward result in ParaFaFT's
final layout together with a checksum of the input. The matrix follows the
reference test registrations (test/CMakeLists.txt:215-271) at reduced N so the
fixtures stay small.

Usage: python tests/golden/make_golden.py
"""
import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden_cases.npz"

CASES = [
    # (name, kind, D, N, shape_id)
    ("c2c_d2_n32_gauss", "c2c", 2, 32, O.SHAPE_GAUSSIAN),
    ("c2c_d2_n32_step", "c2c", 2, 32, O.SHAPE_STEP),
    ("c2c_d3_n16_gauss", "c2c", 3, 16, O.SHAPE_GAUSSIAN),
    ("c2c_d3_n16_poly", "c2c", 3, 16, O.SHAPE_RANDOM_POLY),
    ("c2c_d4_n8_step", "c2c", 4, 8, O.SHAPE_STEP),
    ("c2c_d5_n4_poly", "c2c", 5, 4, O.SHAPE_RANDOM_POLY),
    ("r2c_d2_n32_gauss", "r2c", 2, 32, O.SHAPE_GAUSSIAN),
    ("r2c_d3_n16_step", "r2c", 3, 16, O.SHAPE_STEP),
    ("r2c_d3_n16_poly", "r2c", 3, 16, O.SHAPE_RANDOM_POLY),
    ("r2c_d4_n8_gauss", "r2c", 4, 8, O.SHAPE_GAUSSIAN),
]


def run_case(kind, D, N, shape_id):
    shape = (N,) * D
    x = O.shape_data(N, D, shape_id)
    f = O.RefParaFaFT(kind, shape)
    if kind == "c2c":
        buf = np.zeros(f.required_size, np.complex128)
        buf[:x.size] = x.ravel()
        f.forward(buf)
        out = buf[:x.size].reshape(f.shapes()[2]).copy()
    else:
        buf = np.zeros(f.required_size, np.float64)
        p = O.pad_real(x)
        buf[:p.size] = p
        f.forward(buf)
        out = O.complex_view(buf[:p.size], shape).copy()
    return x, out


def main():
    arrays = {}
    for name, kind, D, N, sid in CASES:
        x, out = run_case(kind, D, N, sid)
        arrays[f"{name}__output"] = out
        arrays[f"{name}__input_sha256"] = np.frombuffer(
            hashlib.sha256(np.ascontiguousarray(x).tobytes()).digest(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
