"""Generate ``sobol_directions.h``: 32 direction numbers for the first 256
Sobol dimensions (Joe & Kuo, "new-joe-kuo-6.21201" primitive polynomials and
initial direction numbers).

The polynomials and initial values are read from the copy of the Joe-Kuo
table that SciPy ships (``scipy/stats/_sobol_direction_numbers.npz``); the
expansion below is the standard Bratley-Fox recurrence

    m_i = 2 a_1 m_{i-1} ^ 4 a_2 m_{i-2} ^ ... ^ 2^{s-1} a_{s-1} m_{i-s+1}
          ^ 2^s m_{i-s} ^ m_{i-s},        V_i = m_i << (32 - i),

written here from the published method.  256 dimensions matches the table
size of the ``sobol_burley`` crate the reference calls (dimensions beyond it
wrap with a seed offset, crates/mc-core/src/runtime/cpu.rs:5406-5431).

Run: ``python montepath_b200/csrc/gen_sobol_directions.py``.
"""

from __future__ import annotations

import os

import numpy as np

DIMS = 256
BITS = 32


def direction_numbers(dims: int = DIMS) -> np.ndarray:
    import scipy.stats

    path = os.path.join(os.path.dirname(scipy.stats.__file__), "_sobol_direction_numbers.npz")
    table = np.load(path)
    poly = table["poly"].astype(np.int64)
    vinit = table["vinit"].astype(np.int64)
    out = np.zeros((dims, BITS), dtype=np.uint64)
    for d in range(dims):
        if d == 0:
            m = [1] * BITS
        else:
            p = int(poly[d])
            s = p.bit_length() - 1
            m = [int(vinit[d][i]) for i in range(s)]
            # a_k for k = 1..s-1: coefficient of x^{s-k}
            a = [(p >> (s - k)) & 1 for k in range(1, s)]
            for i in range(s, BITS):
                value = m[i - s] ^ (m[i - s] << s)
                for k in range(1, s):
                    if a[k - 1]:
                        value ^= m[i - k] << k
                m.append(value)
        for j in range(BITS):
            out[d, j] = (m[j] << (BITS - 1 - j)) & 0xFFFFFFFF
    return out


def main() -> None:
    v = direction_numbers()
    here = os.path.dirname(os.path.abspath(__file__))
    lines = [
        "/* Generated by gen_sobol_directions.py -- do not edit.",
        " * Sobol direction numbers V[dim][bit] (bit 0 = most significant), first 256",
        " * dimensions of the Joe-Kuo new-joe-kuo-6.21201 table. */",
        "#pragma once",
        "#include <stdint.h>",
        f"#define MPC_SOBOL_DIMS {DIMS}",
        f"static const uint32_t kSobolDirections[{DIMS}][{BITS}] = {{",
    ]
    for d in range(DIMS):
        row = ", ".join(f"0x{int(x):08x}u" for x in v[d])
        lines.append(f"  {{{row}}},")
    lines.append("};")
    with open(os.path.join(here, "sobol_directions.h"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
