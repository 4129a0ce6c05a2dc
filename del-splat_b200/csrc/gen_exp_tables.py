"""Writes exp_tables.cuh: the constants of the blend's correctly rounded exp.

    python del-splat_b200/csrc/gen_exp_tables.py

Every constant is derived here from ln 2 evaluated to 60 significant digits
(Python's decimal module), then rounded to the stated precision:

* K64 = 64/ln2 rounded to float (any rounding works: it only picks k).
* C1, C2: ln2/64 split into two parts of at most 11 significant bits each, so
  that k*C1 and k*C2 are exact floats for |k| < 2^13; C3 is the rest,
  rounded to float.
* TH[j] + TL[j]: 2^(j/64) as an unevaluated sum of two floats (TH the
  nearest float, TL the nearest float to the remainder); the table stores
  TH[j] and TL[j] / TH[j] (rounded to float), the low part relative to the
  high one, so that it joins the reduction's correction term.
* TD[j]: 2^(j/64) rounded to double; L1D + L2D: ln2/64 split for the
  double-precision path (L1D has 38 significant bits, so k*L1D is exact for
  |k| < 2^15).
"""
from __future__ import annotations

import math
import os
import struct
from decimal import Decimal, getcontext

getcontext().prec = 60
LN2 = Decimal(2).ln()


def _f32(d: Decimal) -> float:
    """Nearest float32 to d: the float32 rounding of float(d), or one of its
    two float32 neighbours if double rounding moved it (finite d only)."""
    c = struct.unpack("f", struct.pack("f", float(d)))[0]
    if c == 0.0:
        return 0.0
    u = struct.unpack("<i", struct.pack("<f", c))[0]
    best = c
    for cu in (u - 1, u + 1):
        cf = struct.unpack("<f", struct.pack("<i", cu))[0]
        if abs(Decimal(cf) - d) < abs(Decimal(best) - d):
            best = cf
    return best


def _bits(d: Decimal, bits: int) -> Decimal:
    """d rounded to `bits` significant bits."""
    e = math.floor(math.log2(abs(float(d))))
    scale = Decimal(2) ** (bits - 1 - e)
    return (d * scale).to_integral_value() / scale


def tables() -> dict:
    l64 = LN2 / 64
    c1 = _bits(l64, 11)
    c2 = _bits(l64 - c1, 11)
    c3 = _f32(l64 - c1 - c2)
    th, tl, tlr, td = [], [], [], []
    for j in range(64):
        t = (Decimal(j) / 64 * LN2).exp()
        hi = _f32(t)
        th.append(hi)
        tl.append(_f32(t - Decimal(hi)))
        tlr.append(_f32(Decimal(tl[-1]) / Decimal(hi)))
        td.append(float(t))  # float(Decimal) rounds to the nearest double
    l1d = _bits(l64, 38)
    return dict(K64=_f32(Decimal(64) / LN2), C1=float(c1), C2=float(c2), C3=c3, TH=th, TL=tl, TLR=tlr, TD=td,
                K64D=float(Decimal(64) / LN2), L1D=float(l1d), L2D=float(l64 - l1d))


def render(t: dict) -> str:
    fl = lambda v: v.hex() + "f"  # noqa: E731
    lines = [
        "// exp_tables.cuh -- generated by gen_exp_tables.py; do not edit.",
        "// Constants of expf_cr (common.cuh): 64/ln2, ln2/64 in three parts,",
        "// 2^(j/64) as (float, relative float remainder) and as doubles.",
        "#pragma once",
        "namespace dsplat {",
        f"constexpr float kExpK64 = {fl(t['K64'])};",
        f"constexpr float kExpC1 = {fl(t['C1'])}, kExpC2 = {fl(t['C2'])}, kExpC3 = {fl(t['C3'])};",
        f"constexpr double kExpK64d = {t['K64D'].hex()}, kExpL1d = {t['L1D'].hex()}, kExpL2d = {t['L2D'].hex()};",
        "// 2^(j/64) = hi (1 + rel): {hi, rel}",
        "static __device__ const float2 g_exp2_64[64] = {",
    ]
    lines += [f"    {{{fl(h)}, {fl(r)}}}," for h, r in zip(t["TH"], t["TLR"])]
    lines += ["};", "static __device__ const double g_exp2_64d[64] = {"]
    lines += [f"    {v.hex()}," for v in t["TD"]]
    lines += ["};", "}  // namespace dsplat", ""]
    return "\n".join(lines)


if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "exp_tables.cuh")
    with open(out, "w") as f:
        f.write(render(tables()))
    print(out)
