/* Test infrastructure only: the CPU restatement the GhostPanels device fill
 * is checked against, bit for bit. Nothing in the product links this file.
 *
 * The reference fills ghost column col with randn!(Xoshiro(hash(col, seed)))
 * on the host (src/ghosts.jl:97-103), a stream defined only within one Julia
 * version (src/ghosts.jl:34-38), and no golden vectors exist for it; Julia is
 * not installed here. The B200 fill therefore defines its own entries, and
 * this file states them independently of the CUDA source:
 *
 *   (x0, x1, x2, x3) = Philox4x32-10((row_lo, row_hi, col_lo, col_hi), (seed_lo, seed_hi))
 *   u1 = ((x0:x1 >> 11) + 1) 2^-53,  u2 = (x2:x3 >> 11) 2^-53
 *   complex: sqrt(-ln u1) (cos 2 pi u2, sin 2 pi u2);  real: sqrt(-2 ln u1) cos 2 pi u2
 *
 * Philox4x32-10 follows Salmon et al., SC 2011 (checked here against the
 * published known-answer vectors). ln and cos/sin are table driven:
 *   ln x, x = 2^e m, m in (sqrt(1/2), sqrt(2)]: bin of m's top 8 fraction bits
 *     gives (inv, lninv) with lninv = ln(1/inv); r = fma(m, inv, -1);
 *     ln x = fma(e, ln2_hi, lninv) + fma(e, ln2_lo, log1p(r)), log1p to r^8;
 *   cos/sin of 2 pi u, u = b 2^-53: bin j = b >> 45 gives (cos, sin) of its
 *     centre; the rest a = 2 pi (u - centre) by series to a^7 and a^6 and the
 *     angle sum.
 * The tables come from the product's generated fb_ghost_tables.h (constants
 * only; every operation is restated here), so both round alike. Build with
 * -ffp-contract=off so nothing else is contracted.
 * Parity with the reference's values: unpinned (see above). */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define FB_GHOST_TABLE_QUALIFIER static const
#include "../funicular.jl_b200/csrc/fb_ghost_tables.h"

static void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n[4];
    n[0] = hi1 ^ c[1] ^ k0;
    n[1] = lo1;
    n[2] = hi0 ^ c[3] ^ k1;
    n[3] = lo0;
    memcpy(c, n, sizeof n);
}

void ghost_oracle_philox(uint32_t out[4], const uint32_t ctr[4], const uint32_t key[2]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        philox_round(c, k0, k1);
    }
    memcpy(out, c, sizeof c);
}

static double ln_pos(double x) {
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    int e = (int)((bits >> 52) & 0x7ff) - 1023;
    const uint64_t mb = (bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mb, sizeof m);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    uint64_t m_bits;
    memcpy(&m_bits, &m, sizeof m_bits);
    const int j = (int)((m_bits >> 44) & 0xff);
    const int idx = m >= 1.0 ? j : FB_GHOST_LN_UPPER_BINS + (j - FB_GHOST_LN_LOWER_FIRST);
    const double inv = fb_ghost_ln_table[2 * idx], lninv = fb_ghost_ln_table[2 * idx + 1];
    const double r = fma(m, inv, -1.0);
    /* log1p(r) = r + r^2 (-1/2 + r (1/3 + r (-1/4 + ... - r/8))) */
    static const double coef[7] = {-1.0 / 8.0, 1.0 / 7.0, -1.0 / 6.0, 1.0 / 5.0, -1.0 / 4.0, 1.0 / 3.0, -0.5};
    double p = coef[0];
    for (int i = 1; i < 7; ++i) p = fma(p, r, coef[i]);
    const double l1p = fma(r * r, p, r);
    const double hi = fma((double)e, FB_GHOST_LN2_HI, lninv);
    const double lo = fma((double)e, FB_GHOST_LN2_LO, l1p);
    return hi + lo;
}

static void cos_sin_2pi(uint64_t b, double* c, double* s) {
    const int j = (int)(b >> 45);
    const long long f = (long long)(b & ((1ULL << 45) - 1)) - (1LL << 44);
    const double a = ((double)f * 0x1.0p-53) * FB_GHOST_TWO_PI;
    const double a2 = a * a;
    double ps = fma(a2, -1.0 / 5040.0, 1.0 / 120.0);
    ps = fma(ps, a2, -1.0 / 6.0);
    const double sa = fma(a * a2, ps, a);
    double pc = fma(a2, -1.0 / 720.0, 1.0 / 24.0);
    pc = fma(pc, a2, -0.5);
    const double cm1 = a2 * pc;
    const double C = fb_ghost_trig_table[2 * j], S = fb_ghost_trig_table[2 * j + 1];
    *c = C + fma(C, cm1, -(S * sa));
    *s = S + fma(S, cm1, C * sa);
}

/* Entry (row, col) of the ghost matrix as (re, im); im = 0 for a real one.
 * narrow rounds both through single precision. */
void ghost_oracle_entry(uint64_t seed, int64_t row, int64_t col, int is_complex, int narrow, double out[2]) {
    const uint32_t ctr[4] = {(uint32_t)row, (uint32_t)((uint64_t)row >> 32), (uint32_t)col,
                             (uint32_t)((uint64_t)col >> 32)};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    ghost_oracle_philox(x, ctr, key);
    const uint64_t a = ((uint64_t)x[0] << 32) | x[1];
    const uint64_t b = ((uint64_t)x[2] << 32) | x[3];
    const double u1 = (double)((a >> 11) + 1) * 0x1.0p-53;
    double c, s;
    cos_sin_2pi(b >> 11, &c, &s);
    const double l = ln_pos(u1);
    double re, im;
    if (is_complex) {
        const double rad = sqrt(-l);
        re = rad * c;
        im = rad * s;
    } else {
        re = sqrt(-2.0 * l) * c;
        im = 0.0;
    }
    if (narrow) {
        re = (double)(float)re;
        im = (double)(float)im;
    }
    out[0] = re;
    out[1] = im;
}

/* The rows x cols block at (row0, col0), column-major with leading dimension
 * ld, as interleaved (re, im) pairs when complex and plain doubles when real. */
void ghost_oracle_fill(double* dst, int64_t ld, int64_t rows, int64_t cols, int64_t row0, int64_t col0,
                       uint64_t seed, int is_complex, int narrow) {
    for (int64_t j = 0; j < cols; ++j)
        for (int64_t i = 0; i < rows; ++i) {
            double v[2];
            ghost_oracle_entry(seed, row0 + i, col0 + j, is_complex, narrow, v);
            if (is_complex) {
                dst[2 * (i + j * ld)] = v[0];
                dst[2 * (i + j * ld) + 1] = v[1];
            } else {
                dst[i + j * ld] = v[0];
            }
        }
}

/* The ln and cos/sin above, exposed for accuracy tests against libm. */
double ghost_oracle_ln(double x) { return ln_pos(x); }

/* u must be a multiple of 2^-53 in [0, 1), as every u2 of the fill is. */
void ghost_oracle_cos_sin_2pi(double u, double out[2]) {
    cos_sin_2pi((uint64_t)(u * 0x1.0p53), &out[0], &out[1]);
}
