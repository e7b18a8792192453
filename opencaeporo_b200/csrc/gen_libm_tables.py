"""Writes flash_libm_tables.h: the tables of the flash kernels' table-driven
exponential and logarithm (flash_libm.cuh), computed in 60-digit decimal
arithmetic and split into double-precision head and tail parts.

  exp: T_j = 2^(j/32), j = 0..31, as (head, tail) with head = RN(T_j).
  log: for the 128 intervals of the reduced argument m in [sqrt(2)/2, sqrt(2))
       (64 intervals of width 2^-7 on [0.5, 1), 64 of width 2^-6 on [1, 2),
       of which the first half-range and the second are used), a reciprocal
       c_j of the interval's midpoint rounded to 10 significant bits (c = 1
       for the two intervals that touch m = 1), and -ln(c_j) as (head, tail)
       with the head rounded to a multiple of 2^-42, so that k ln2_head +
       head is exact for every exponent k.

    python opencaeporo_b200/csrc/gen_libm_tables.py   # rewrites the header
"""
import math
import os
from decimal import Decimal, getcontext

getcontext().prec = 60
HERE = os.path.dirname(os.path.abspath(__file__))


def split(v: Decimal, quantum=None):
    if quantum is None:
        h = float(v)
    else:
        h = float((v / quantum).to_integral_value() * quantum)
    return h, float(v - Decimal(h))


def main():
    lines = ["// flash_libm_tables.h -- generated by gen_libm_tables.py; do not edit.",
             "#pragma once", "", "namespace ocpf {", ""]
    exp_rows = []
    for j in range(32):
        v = (Decimal(2) ** (Decimal(j) / 32))
        h, t = split(v)
        exp_rows.append(f"    {h.hex()}, {t.hex()},")
    lines.append("// 2^(j/32): head, tail")
    lines.append("__device__ __align__(16) const double kExpTable[64] = {")
    lines += exp_rows
    lines.append("};")
    lines.append("")
    q = Decimal(2) ** -42
    log_rows = []
    for j in range(128):
        lo = Decimal("0.5") + Decimal(j) / 128 if j < 64 else Decimal(1) + Decimal(j - 64) / 64
        w = Decimal(1) / 128 if j < 64 else Decimal(1) / 64
        mc = lo + w / 2
        c = float(Decimal(1) / mc)
        fr, ex = math.frexp(c)
        c = math.ldexp(round(fr * 1024.0) / 1024.0, ex)
        if j in (63, 64):
            c = 1.0
        L = -Decimal(c).ln()
        h, t = split(L, q)
        log_rows.append(f"    {c.hex()}, {h.hex()}, {t.hex()}, 0x0p+0,")
    lines.append("// per interval j: c_j, -ln(c_j) head (a multiple of 2^-42), tail, padding")
    lines.append("__device__ __align__(16) const double kLogTable[512] = {")
    lines += log_rows
    lines.append("};")
    ln2 = Decimal(2).ln()
    h, t = split(ln2, q)
    lines.append("")
    lines.append(f"constexpr double kLn2Head = {h.hex()};  // ln 2 rounded to a multiple of 2^-42")
    lines.append(f"constexpr double kLn2Tail = {t.hex()};")
    l32 = ln2 / 32
    h, t = split(l32)
    lines.append(f"constexpr double kLn2By32Head = {h.hex()};  // RN(ln 2 / 32)")
    lines.append(f"constexpr double kLn2By32Tail = {t.hex()};")
    lines.append(f"constexpr double k32ByLn2 = {float(Decimal(32) / ln2).hex()};  // RN(32 / ln 2)")
    lines += ["", "}  // namespace ocpf", ""]
    with open(os.path.join(HERE, "flash_libm_tables.h"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
