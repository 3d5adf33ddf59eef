"""Generates crmath_tables.h: the constant tables of the correctly rounded
FP64 exp / log / sin / cos in crmath.cuh, from 300-bit mpmath evaluations.

Every table value is written as a C99 hexadecimal literal, so the header is
exact.  Run:  python gen_crmath_tables.py > crmath_tables.h
"""
import mpmath as mp

mp.mp.prec = 300


def hexd(v):
    """Round an mpf to the nearest double and print it as a hex literal."""
    return float(v).hex() if v != 0 else "0x0.0p+0"


def dd(v):
    hi = float(v)
    lo = float(v - mp.mpf(hi))
    return hi, lo


def split_bits(v, bits):
    """Leading `bits` significant bits of v (truncated), as a double."""
    if v == 0:
        return 0.0
    e = int(mp.floor(mp.log(abs(v), 2)))
    scale = mp.mpf(2) ** (bits - 1 - e)
    return float(mp.floor(v * scale) / scale) if v > 0 else float(mp.ceil(v * scale) / scale)


def emit_dd_array(name, vals, out):
    out.append(f"#define {name}_INIT {{ \\")
    for v in vals:
        hi, lo = dd(v)
        out.append(f"    {hexd(mp.mpf(hi))}, {hexd(mp.mpf(lo))}, \\")
    out.append("}")


def main():
    out = ["// Generated by gen_crmath_tables.py (mpmath, 300-bit arithmetic): do not edit.",
           "// Pairs are double-double values (hi, lo) with |lo| <= ulp(hi)/2.",
           "#pragma once", ""]
    ln2 = mp.log(2)
    # exp: x = k ln2 / 4096 + r, k = 4096 m + 64 j2 + j1
    L = ln2 / 4096
    L1 = split_bits(L, 30)
    L2 = split_bits(L - L1, 30)
    L3 = float(L - L1 - L2)
    out.append(f"#define CR_EXP_INVL {hexd(4096 / ln2)}")
    out.append(f"#define CR_EXP_L1 {hexd(mp.mpf(L1))}")
    out.append(f"#define CR_EXP_L2 {hexd(mp.mpf(L2))}")
    out.append(f"#define CR_EXP_L3 {hexd(mp.mpf(L3))}")
    emit_dd_array("CR_EXP_T1", [mp.mpf(2) ** (mp.mpf(j) / 4096) for j in range(64)], out)
    emit_dd_array("CR_EXP_T2", [mp.mpf(2) ** (mp.mpf(j) / 64) for j in range(64)], out)
    # log: m in [1, 2), j = top 7 mantissa bits, inv_j with 8 significant bits
    invs, es, ts = [], [], []
    for j in range(128):
        c = 1 + (mp.mpf(j) + mp.mpf("0.5")) / 128
        if j == 0:
            inv = mp.mpf(1)
        elif j == 127:
            inv = mp.mpf("0.5")
        else:
            inv = mp.nint(256 / c) / 256
        e = 1 if c > mp.sqrt(2) else 0
        invs.append(inv)
        es.append(e)
        ts.append(-mp.log(inv * 2 ** e))
        # |r| < 2^-7 on the whole bin and r exact: checked here
        for m in (1 + mp.mpf(j) / 128, 1 + mp.mpf(j + 1) / 128 - mp.mpf(2) ** -52):
            assert abs(m * inv - 1) < mp.mpf(2) ** -7, (j, m * inv - 1)
    out.append("#define CR_LOG_INV_INIT { \\")
    out.extend(f"    {hexd(v)}, \\" for v in invs)
    out.append("}")
    out.append("#define CR_LOG_E_INIT { \\")
    out.append("    " + ", ".join(str(e) for e in es) + " \\")
    out.append("}")
    emit_dd_array("CR_LOG_T", ts, out)
    out.append(f"#define CR_LN2_HI {hexd(mp.mpf(dd(ln2)[0]))}")
    out.append(f"#define CR_LN2_LO {hexd(mp.mpf(dd(ln2)[1]))}")
    for k in (3, 5):
        hi, lo = dd(mp.mpf(1) / k)
        out.append(f"#define CR_INV{k}_HI {hexd(mp.mpf(hi))}")
        out.append(f"#define CR_INV{k}_LO {hexd(mp.mpf(lo))}")
    # sin / cos: x = k pi/2 + r, r = j/256 + t
    pio2 = mp.pi / 2
    parts = []
    rem = pio2
    for bits in (32, 32, 32, 32):
        p = split_bits(rem, bits)
        parts.append(p)
        rem -= p
    parts.append(float(rem))
    for i, p in enumerate(parts):
        out.append(f"#define CR_PIO2_{i + 1} {hexd(mp.mpf(p))}")
    out.append(f"#define CR_2OPI {hexd(2 / mp.pi)}")
    nsc = 202
    out.append(f"#define CR_SC_N {nsc}")
    emit_dd_array("CR_SIN_T", [mp.sin(mp.mpf(j) / 256) for j in range(nsc)], out)
    emit_dd_array("CR_COS_T", [mp.cos(mp.mpf(j) / 256) for j in range(nsc)], out)
    for k in (2, 6):
        hi, lo = dd(mp.mpf(1) / k)
        out.append(f"#define CR_INV{k}_HI {hexd(mp.mpf(hi))}")
        out.append(f"#define CR_INV{k}_LO {hexd(mp.mpf(lo))}")
    # Taylor coefficients 1/k! (plain doubles, the tails only)
    for k in range(3, 12):
        out.append(f"#define CR_IFACT{k} {hexd(1 / mp.factorial(k))}")
    for k in range(7, 16, 2):
        out.append(f"#define CR_INVODD{k} {hexd(mp.mpf(1) / k)}")
    print("\n".join(out))


if __name__ == "__main__":
    main()
