#!/usr/bin/env python
"""Writes fb_ghost_tables.h: the constant tables of the GhostPanels fill's
ln and cos/sin (fb_ghost.cu), shared with the fill's C restatement in the
oracle so both round every entry the same way.

    python gen_ghost_tables.py > fb_ghost_tables.h

Values come from mpmath at 60 digits, each rounded once to the nearest
double (Python's float() of an mpmath value rounds to nearest).

ln. x = 2^e m with m in (sqrt(1/2), sqrt(2)]. m >= 1: bin j = the top 8
bits of m's fraction, j in [0, 106], centre c = 1 + j/256 (its left end,
so bin 0 has c = 1). m < 1 (m in [1/2, 1) as a double): bin j = the top 8
bits of its fraction, j in [105, 255], c = (1 + (j + 1)/256) / 2 (its right
end, so bin 255 has c = 1). Table entry: inv = fl(1 / c) and
lninv = fl(-ln(inv)) for that double inv, so ln m = lninv + log1p(m inv - 1).
Upper bins sit at index j, lower ones at index 107 + (j - 105).

cos/sin. 2 pi u with u = b 2^-53, b < 2^53: bin j = b >> 45, centre
theta_j = 2 pi (j + 1/2) / 256; table entry (fl(cos theta_j), fl(sin theta_j)).
"""
import mpmath

mpmath.mp.dps = 60

UPPER = range(0, 107)     # m in [1, sqrt 2]: fraction bits top 8 in 0..106
LOWER = range(105, 256)   # m in (sqrt(1/2), 1): fraction bits top 8 in 105..255


def hexd(x: float) -> str:
    return float(x).hex()


def ln_entries():
    out = []
    for j in UPPER:
        c = mpmath.mpf(1) + mpmath.mpf(j) / 256
        inv = float(1 / c) if j else 1.0
        out.append((inv, float(-mpmath.log(mpmath.mpf(inv))) if j else 0.0))
    for j in LOWER:
        c = (mpmath.mpf(1) + mpmath.mpf(j + 1) / 256) / 2
        inv = float(1 / c) if j != 255 else 1.0
        out.append((inv, float(-mpmath.log(mpmath.mpf(inv))) if j != 255 else 0.0))
    return out


def trig_entries():
    out = []
    for j in range(256):
        t = 2 * mpmath.pi * (mpmath.mpf(j) + mpmath.mpf(1) / 2) / 256
        out.append((float(mpmath.cos(t)), float(mpmath.sin(t))))
    return out


def main():
    ln2 = mpmath.log(2)
    ln2_hi = float(mpmath.floor(ln2 * 2 ** 44) / 2 ** 44)   # 44 fraction bits: e * ln2_hi exact for |e| < 2^8
    ln2_lo = float(ln2 - mpmath.mpf(ln2_hi))
    two_pi = float(2 * mpmath.pi)
    lines = [
        "// Generated by gen_ghost_tables.py: the constant tables of the GhostPanels",
        "// fill's ln and cos/sin (fb_ghost.cu and the oracle's C restatement).",
        "// Do not edit; regenerate.",
        "#pragma once",
        "",
        f"#define FB_GHOST_LN2_HI {hexd(ln2_hi)}",
        f"#define FB_GHOST_LN2_LO {hexd(ln2_lo)}",
        f"#define FB_GHOST_TWO_PI {hexd(two_pi)}",
        "#define FB_GHOST_LN_UPPER_BINS 107",
        "#define FB_GHOST_LN_LOWER_FIRST 105",
        f"#define FB_GHOST_LN_ENTRIES {len(UPPER) + len(LOWER)}",
        "",
        "// (inv, lninv) per ln bin, interleaved.",
        "FB_GHOST_TABLE_QUALIFIER double fb_ghost_ln_table[2 * FB_GHOST_LN_ENTRIES] = {",
    ]
    for inv, lninv in ln_entries():
        lines.append(f"    {hexd(inv)}, {hexd(lninv)},")
    lines += ["};", "", "// (cos, sin) of 2 pi (j + 1/2) / 256, interleaved.",
              "FB_GHOST_TABLE_QUALIFIER double fb_ghost_trig_table[2 * 256] = {"]
    for c, s in trig_entries():
        lines.append(f"    {hexd(c)}, {hexd(s)},")
    lines += ["};", ""]
    print("\n".join(lines))


if __name__ == "__main__":
    main()
