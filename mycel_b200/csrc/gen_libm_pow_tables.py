"""Generate libm_pow_tables.h: the lookup tables of the host C library's pow (GNU libc 2.28 and later,
whose pow comes from Arm's optimized-routines, 2018), rebuilt from the construction rules published with
that algorithm rather than copied.

Log table (128 entries). x = 2^k z with z in [OFF, 2 OFF), OFF = 0x1.69555p-1; the bit range of z is split
into 128 equal subintervals i = ((bits(z) - bits(OFF)) >> 45) mod 128. For the centre m of subinterval i:
    1/c      = m < 1 ? round(128 / m) / 128 : round(256 / m) / 256
    logc     = round(2^43 log c) / 2^43
    logctail = (double)(log c - logc)
so z/c - 1 is exact in double and k ln2hi + logc adds without rounding.

Exp table (128 entries). 2^(j/128) = H_j (1 + T_j) with H_j = (double) 2^(j/128) and T_j = (double)
(2^(j/128)/H_j - 1); the table stores bits(T_j) and bits(H_j) - (j << 45).

Run: python gen_libm_pow_tables.py  (writes the header beside this script).
"""
from __future__ import annotations

import os
import struct
from decimal import Decimal, getcontext

getcontext().prec = 80

N = 128
OFF = 0x3FE6955500000000


def bits_to_double(u: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", u & 0xFFFFFFFFFFFFFFFF))[0]


def double_to_bits(d: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def dec(d: float) -> Decimal:
    return Decimal(d)  # exact


def round_half_even(q: Decimal) -> int:
    return int(q.to_integral_value())  # ROUND_HALF_EVEN is the decimal default


def nearest_double(q: Decimal) -> float:
    """Round an exact decimal to the nearest double (ties to even)."""
    f = float(q)  # Python's float(Decimal) rounds correctly
    return f


def log_table():
    rows = []
    for i in range(N):
        lo = bits_to_double(OFF + (i << 45))
        hi = bits_to_double(OFF + ((i + 1) << 45))
        m = (dec(lo) + dec(hi)) / 2
        if m < 1:
            invc = Decimal(round_half_even(Decimal(N) / m)) / N
        else:
            invc = Decimal(round_half_even(Decimal(2 * N) / m)) / (2 * N)
        invc_d = float(invc)
        assert Decimal(invc_d) == invc
        logc_exact = -(invc.ln())
        logc = Decimal(round_half_even(logc_exact * (Decimal(2) ** 43))) / (Decimal(2) ** 43)
        logc_d = float(logc)
        assert Decimal(logc_d) == logc
        tail = nearest_double(logc_exact - logc)
        rows.append((invc_d, logc_d, tail))
    return rows


def exp_table():
    out = []
    for j in range(N):
        v = (Decimal(2) ** (Decimal(j) / N))
        h = nearest_double(v)
        t = nearest_double(v / dec(h) - 1)
        out.append(double_to_bits(t))
        out.append((double_to_bits(h) - (j << 45)) & 0xFFFFFFFFFFFFFFFF)
    return out


def main():
    lt = log_table()
    et = exp_table()
    here = os.path.dirname(os.path.abspath(__file__))
    lines = [
        "// Generated by gen_libm_pow_tables.py: the lookup tables of the host C library's pow, rebuilt from the",
        "// algorithm's published construction rules (see that script). Do not edit by hand.",
        "#pragma once",
        "#include <stdint.h>",
        "",
        "namespace mycel {",
        "namespace libm_pow {",
        "",
        "// {1/c, logc, logctail} for the 128 subintervals of [0x1.69555p-1, 0x1.69555p0)",
        "MYCEL_POW_TABLE_QUAL double kLogTab[128][3] = {",
    ]
    for a, b, c in lt:
        lines.append(f"    {{{a.hex()}, {b.hex()}, {c.hex()}}},")
    lines += ["};", "", "// bits(T_j), bits(H_j) - (j << 45) for 2^(j/128) = H_j (1 + T_j)",
              "MYCEL_POW_TABLE_QUAL uint64_t kExpTab[256] = {"]
    for k in range(0, len(et), 2):
        lines.append(f"    0x{et[k]:016x}ULL, 0x{et[k + 1]:016x}ULL,")
    lines += ["};", "", "}  // namespace libm_pow", "}  // namespace mycel", ""]
    with open(os.path.join(here, "libm_pow_tables.h"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
