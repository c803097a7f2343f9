// The device fill behind GhostPanels (src/ghosts.jl:53-122). The reference
// draws column col from randn!(Xoshiro(hash(col, hash(seed)))), one sequential
// stream per column, on the host, and then uploads the panel. Here entry
// (row, col) is a pure function of (seed, row, col), so any block of rows of
// any panel is generated where it is needed, in device memory, by as many
// threads as there are entries, and nothing crosses the bus:
//
//   (x0, x1, x2, x3) = Philox4x32-10(counter = (row, col), key = seed)
//   u1 = (top 53 bits of x0:x1 + 1) 2^-53 in (0, 1]
//   u2 = (top 53 bits of x2:x3) 2^-53      in [0, 1)
//   complex: re + i im = sqrt(-ln u1) (cos 2 pi u2 + i sin 2 pi u2)  (each N(0, 1/2))
//   real:    sqrt(-2 ln u1) cos 2 pi u2                              (N(0, 1))
//
// Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC 2011); its ten
// round keys depend on the seed alone and are made on the host. The
// transform is Box and Muller (1958). ln, cos and sin are this file's own,
// table driven: ln m = ln(1/inv) + log1p(m inv - 1) with (inv, ln(1/inv)) of
// the 8-bit bin m falls in and a degree-8 series for log1p on |r| < 2^-8;
// cos and sin of 2 pi u by the angle sum from the centre of u's 8-bit bin,
// the remaining angle below 2 pi 2^-9 taken to a^7 (sin) and a^6 (cos).
// The tables (fb_ghost_tables.h) are generated to the nearest double from
// 60-digit values. Only + - * sqrt and explicit fma are used, and this file
// is compiled with -fmad=false, so every entry rounds the same way on any
// IEEE machine: the oracle's C restatement reproduces it bit for bit.
#include "fb_common.cuh"

#define FB_GHOST_TABLE_QUALIFIER static __device__ const
#include "fb_ghost_tables.h"

namespace fb {
namespace ghost {

constexpr uint32_t PHILOX_M0 = 0xD2511F53u, PHILOX_M1 = 0xCD9E8D57u;
constexpr uint32_t PHILOX_W0 = 0x9E3779B9u, PHILOX_W1 = 0xBB67AE85u;

// The ten round keys of a seed: key k_r = seed + r W (per 32-bit half).
struct RoundKeys {
    uint32_t k0[10], k1[10];
};

static RoundKeys round_keys(uint64_t seed) {
    RoundKeys rk;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        rk.k0[r] = k0;
        rk.k1[r] = k1;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    return rk;
}

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], const RoundKeys& rk) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t lo0 = PHILOX_M0 * c[0], hi0 = __umulhi(PHILOX_M0, c[0]);
        const uint32_t lo1 = PHILOX_M1 * c[2], hi1 = __umulhi(PHILOX_M1, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ rk.k0[round], n2 = hi0 ^ c[3] ^ rk.k1[round];
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}

// The tables, staged in shared memory by each CTA.
constexpr int LN_DOUBLES = 2 * FB_GHOST_LN_ENTRIES;
constexpr int TRIG_DOUBLES = 2 * 256;

// ln u for u = n 2^-53, 1 <= n <= 2^53, read straight from the integer (the
// exponent and fraction bits u has as a double, without converting):
// u = 2^e m with m in (sqrt(1/2), sqrt(2)].
__device__ __forceinline__ double ln_u53(uint64_t n, const double* __restrict__ lnt) {
    const int lz = __clzll((long long)n);
    int e = 10 - lz;                                          // 63 - lz - 53
    const uint64_t frac = ((n << lz) >> 11) & 0x000fffffffffffffull;
    double m = __longlong_as_double((long long)(frac | 0x3ff0000000000000ull));
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    const int j = (int)((__double_as_longlong(m) >> 44) & 0xff);
    const int idx = m >= 1.0 ? j : FB_GHOST_LN_UPPER_BINS + (j - FB_GHOST_LN_LOWER_FIRST);
    const double inv = lnt[2 * idx], lninv = lnt[2 * idx + 1];
    const double r = fma(m, inv, -1.0);
    double p = -1.0 / 8.0;
    p = fma(p, r, 1.0 / 7.0);
    p = fma(p, r, -1.0 / 6.0);
    p = fma(p, r, 1.0 / 5.0);
    p = fma(p, r, -1.0 / 4.0);
    p = fma(p, r, 1.0 / 3.0);
    p = fma(p, r, -0.5);
    const double l1p = fma(r * r, p, r);
    const double hi = fma((double)e, FB_GHOST_LN2_HI, lninv);
    const double lo = fma((double)e, FB_GHOST_LN2_LO, l1p);
    return hi + lo;
}

// (cos, sin) of 2 pi u, u = b 2^-53 with b < 2^53: bin j = b >> 45 (centre
// theta_j = 2 pi (j + 1/2) / 256), a = 2 pi (u - centre) in [-2 pi 2^-9,
// 2 pi 2^-9).
__device__ __forceinline__ void cos_sin_2pi(uint64_t b, const double* __restrict__ trig, double& c, double& s) {
    const int j = (int)(b >> 45);
    const long long f = (long long)(b & ((1ull << 45) - 1)) - (1ll << 44);
    const double a = ((double)f * 0x1.0p-53) * FB_GHOST_TWO_PI;
    const double a2 = a * a;
    double ps = fma(a2, -1.0 / 5040.0, 1.0 / 120.0);
    ps = fma(ps, a2, -1.0 / 6.0);
    const double sa = fma(a * a2, ps, a);
    double pc = fma(a2, -1.0 / 720.0, 1.0 / 24.0);
    pc = fma(pc, a2, -0.5);
    const double cm1 = a2 * pc;
    const double C = trig[2 * j], S = trig[2 * j + 1];
    c = C + fma(C, cm1, -(S * sa));
    s = S + fma(S, cm1, C * sa);
}

// The two 53-bit integers of an entry: u1 = n1 2^-53 in (0, 1], u2 = b2 2^-53.
__device__ __forceinline__ void uniforms(const RoundKeys& rk, int64_t row, int64_t col, uint64_t& n1, uint64_t& b2) {
    uint32_t c[4] = {(uint32_t)row, (uint32_t)((uint64_t)row >> 32), (uint32_t)col, (uint32_t)((uint64_t)col >> 32)};
    philox4x32_10(c, rk);
    const uint64_t a = ((uint64_t)c[0] << 32) | c[1];
    const uint64_t b = ((uint64_t)c[2] << 32) | c[3];
    n1 = (a >> 11) + 1;
    b2 = b >> 11;
}

template <typename D>
__device__ __forceinline__ void store(D* p, double re, double im);
template <> __device__ __forceinline__ void store<double2>(double2* p, double re, double im) { *p = make_double2(re, im); }
template <> __device__ __forceinline__ void store<float2>(float2* p, double re, double im) {
    *p = make_float2(__double2float_rn(re), __double2float_rn(im));
}
template <> __device__ __forceinline__ void store<double>(double* p, double re, double) { *p = re; }
template <> __device__ __forceinline__ void store<float>(float* p, double re, double) { *p = __double2float_rn(re); }

// One thread per entry of a column block, rows fastest so stores coalesce.
// narrow rounds each value through single precision before it is stored,
// which is what a narrowed host tier holds (src/ghosts.jl:109).
template <typename D, bool COMPLEX>
__global__ void __launch_bounds__(256) ghost_fill_kernel(D* __restrict__ dst, int64_t ld, int64_t rows, int64_t cols,
                                                         int64_t row0, int64_t col0, const RoundKeys rk, int narrow) {
    __shared__ double lnt[LN_DOUBLES];
    __shared__ double trig[TRIG_DOUBLES];
    for (int e = threadIdx.x; e < LN_DOUBLES; e += blockDim.x) lnt[e] = fb_ghost_ln_table[e];
    for (int e = threadIdx.x; e < TRIG_DOUBLES; e += blockDim.x) trig[e] = fb_ghost_trig_table[e];
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = blockIdx.y; j < cols; j += gridDim.y) {
        D* column = dst + j * ld;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) {
            double c, s;
            uint64_t n1, b2;
            uniforms(rk, row0 + i, col0 + j, n1, b2);
            cos_sin_2pi(b2, trig, c, s);
            const double l = ln_u53(n1, lnt);
            double re, im;
            if (COMPLEX) {
                const double rad = sqrt(-l);
                re = rad * c;
                im = rad * s;
            } else {
                re = sqrt(-2.0 * l) * c;
                im = 0.0;
            }
            if (narrow) {
                re = (double)__double2float_rn(re);
                im = (double)__double2float_rn(im);
            }
            store<D>(column + i, re, im);
        }
    }
}

template <typename D, bool COMPLEX>
static int launch_fill(void* dst, int64_t ld, int64_t rows, int64_t cols, int64_t row0, int64_t col0, uint64_t seed,
                       int narrow, cudaStream_t stream) {
    int64_t gx = (rows + 255) / 256;
    const int64_t gy = cols < 65535 ? cols : 65535;
    // Enough CTAs to fill every SM several times over, whatever the shape.
    const int64_t want = (int64_t)sm_count() * 16;
    const int64_t cap_x = (want + gy - 1) / gy;
    if (gx > cap_x) gx = cap_x;
    if (gx < 1) gx = 1;
    ghost_fill_kernel<D, COMPLEX><<<dim3((unsigned)gx, (unsigned)gy), 256, 0, stream>>>(
        static_cast<D*>(dst), ld, rows, cols, row0, col0, round_keys(seed), narrow);
    FB_LAUNCHED("ghost_fill_kernel");
    return FB_OK;
}

}  // namespace ghost
}  // namespace fb

using namespace fb;

extern "C" {

int fb_ghost_fill(void* dst, int dst_type, int64_t ld, int64_t rows, int64_t cols, int64_t row0, int64_t col0,
                  uint64_t seed, int value_type, fb_queue_t queue) {
    if (rows < 0 || cols < 0) { set_error(FB_EDIM, "fb_ghost_fill: negative size"); return FB_EDIM; }
    if (row0 < 0 || col0 < 0) { set_error(FB_EDIM, "fb_ghost_fill: negative row or column offset"); return FB_EDIM; }
    const bool dst_complex = dst_type == FB_C128 || dst_type == FB_C64;
    const bool value_complex = value_type == FB_C128 || value_type == FB_C64;
    const bool known = dst_type >= FB_C128 && dst_type <= FB_F32 && value_type >= FB_C128 && value_type <= FB_F32;
    if (!known || dst_complex != value_complex) {
        set_error(FB_EINVAL, "fb_ghost_fill: element types %d (storage) and %d (values) must both be known and both "
                  "complex or both real", dst_type, value_type);
        return FB_EINVAL;
    }
    if (rows == 0 || cols == 0) return FB_OK;
    if (!dst) { set_error(FB_EINVAL, "fb_ghost_fill: NULL destination"); return FB_EINVAL; }
    if (ld < rows) { set_error(FB_EDIM, "fb_ghost_fill: leading dimension %lld is smaller than rows %lld",
                               (long long)ld, (long long)rows); return FB_EDIM; }
    const int narrow = (value_type == FB_C64 || value_type == FB_F32) ? 1 : 0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(queue);
    switch (dst_type) {
        case FB_C128: return ghost::launch_fill<double2, true>(dst, ld, rows, cols, row0, col0, seed, narrow, s);
        case FB_C64: return ghost::launch_fill<float2, true>(dst, ld, rows, cols, row0, col0, seed, narrow, s);
        case FB_F64: return ghost::launch_fill<double, false>(dst, ld, rows, cols, row0, col0, seed, narrow, s);
        default: return ghost::launch_fill<float, false>(dst, ld, rows, cols, row0, col0, seed, narrow, s);
    }
}

}  // extern "C"
