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
 * published known-answer vectors). ln, cos and sin are series with 1/n and
 * 1/n! coefficients evaluated with explicit fma; build with
 * -ffp-contract=off so nothing else is contracted.
 * Parity with the reference's values: unpinned (see above). */
#include <math.h>
#include <stdint.h>
#include <string.h>

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
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    static const double inv_odd[9] = {1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0,
                                      1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0};
    double p = inv_odd[0];
    for (int i = 1; i < 9; ++i) p = fma(p, z, inv_odd[i]);
    const double t = s + s;
    const double lnm = fma(t * z, p, t);
    return fma((double)e, 0.6931471805599453, lnm);
}

static void cos_sin_2pi(double u, double* c, double* s) {
    const double t = 4.0 * u;
    const double qf = floor(t + 0.5);
    const double r = t - qf;
    const int q = ((int)qf) & 3;
    const double a = r * 1.5707963267948966;
    const double a2 = a * a;
    /* sin: a + a^3 (-1/3! + a^2 (1/5! - ...)), down from 1/17!. */
    static const double sin_coef[8] = {1.0 / 355687428096000.0, -1.0 / 1307674368000.0, 1.0 / 6227020800.0,
                                       -1.0 / 39916800.0,       1.0 / 362880.0,         -1.0 / 5040.0,
                                       1.0 / 120.0,             -1.0 / 6.0};
    /* cos: 1 - a^2/2 + a^4 (1/4! - a^2 (1/6! - ...)), down from -1/18!. */
    static const double cos_coef[8] = {-1.0 / 6402373705728000.0, 1.0 / 20922789888000.0, -1.0 / 87178291200.0,
                                       1.0 / 479001600.0,         -1.0 / 3628800.0,       1.0 / 40320.0,
                                       -1.0 / 720.0,              1.0 / 24.0};
    double sp = sin_coef[0], cp = cos_coef[0];
    for (int i = 1; i < 8; ++i) {
        sp = fma(sp, a2, sin_coef[i]);
        cp = fma(cp, a2, cos_coef[i]);
    }
    const double sa = fma(a * a2, sp, a);
    const double ca = fma(a2 * a2, cp, fma(a2, -0.5, 1.0));
    switch (q) {
        case 0: *c = ca; *s = sa; break;
        case 1: *c = -sa; *s = ca; break;
        case 2: *c = -ca; *s = -sa; break;
        default: *c = sa; *s = -ca; break;
    }
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
    const double u2 = (double)(b >> 11) * 0x1.0p-53;
    double c, s;
    cos_sin_2pi(u2, &c, &s);
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

void ghost_oracle_cos_sin_2pi(double u, double out[2]) { cos_sin_2pi(u, &out[0], &out[1]); }
