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
// Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC 2011); the
// transform is Box and Muller (1958). ln, cos and sin are this file's own
// (series about 1 and about 0 with 1/n and 1/n! coefficients, below), built
// from + - * / sqrt and explicit fma only, and this file is compiled with
// -fmad=false, so every entry rounds the same way on any IEEE machine: the
// oracle's C restatement reproduces it bit for bit.
#include "fb_common.cuh"

namespace fb {
namespace ghost {

constexpr uint32_t PHILOX_M0 = 0xD2511F53u, PHILOX_M1 = 0xCD9E8D57u;
constexpr uint32_t PHILOX_W0 = 0x9E3779B9u, PHILOX_W1 = 0xBB67AE85u;

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t lo0 = PHILOX_M0 * c[0], hi0 = __umulhi(PHILOX_M0, c[0]);
        const uint32_t lo1 = PHILOX_M1 * c[2], hi1 = __umulhi(PHILOX_M1, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += PHILOX_W0; k1 += PHILOX_W1;
    }
}

// ln x for a positive normal x: x = 2^e m with m in (sqrt(1/2), sqrt(2)],
// ln m = 2 atanh(s) with s = (m - 1) / (m + 1), |s| < 0.1716, summed to s^19.
__device__ __forceinline__ double ln_pos(double x) {
    const long long bits = __double_as_longlong(x);
    int e = (int)((bits >> 52) & 0x7ff) - 1023;
    double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    double p = 1.0 / 19.0;
    p = fma(p, z, 1.0 / 17.0);
    p = fma(p, z, 1.0 / 15.0);
    p = fma(p, z, 1.0 / 13.0);
    p = fma(p, z, 1.0 / 11.0);
    p = fma(p, z, 1.0 / 9.0);
    p = fma(p, z, 1.0 / 7.0);
    p = fma(p, z, 1.0 / 5.0);
    p = fma(p, z, 1.0 / 3.0);
    const double t = s + s;
    const double lnm = fma(t * z, p, t);
    return fma((double)e, 0.6931471805599453, lnm);
}

// (cos, sin) of 2 pi u for u in [0, 1): quadrant q = round(4u), a = (4u - q) pi/2
// in [-pi/4, pi/4], Taylor series to a^17 and a^18.
__device__ __forceinline__ void cos_sin_2pi(double u, double& c, double& s) {
    const double t = 4.0 * u;
    const double qf = floor(t + 0.5);
    const double r = t - qf;
    const int q = ((int)qf) & 3;
    const double a = r * 1.5707963267948966;
    const double a2 = a * a;
    double sp = 1.0 / 355687428096000.0;
    sp = fma(sp, a2, -1.0 / 1307674368000.0);
    sp = fma(sp, a2, 1.0 / 6227020800.0);
    sp = fma(sp, a2, -1.0 / 39916800.0);
    sp = fma(sp, a2, 1.0 / 362880.0);
    sp = fma(sp, a2, -1.0 / 5040.0);
    sp = fma(sp, a2, 1.0 / 120.0);
    sp = fma(sp, a2, -1.0 / 6.0);
    const double sa = fma(a * a2, sp, a);
    double cp = -1.0 / 6402373705728000.0;
    cp = fma(cp, a2, 1.0 / 20922789888000.0);
    cp = fma(cp, a2, -1.0 / 87178291200.0);
    cp = fma(cp, a2, 1.0 / 479001600.0);
    cp = fma(cp, a2, -1.0 / 3628800.0);
    cp = fma(cp, a2, 1.0 / 40320.0);
    cp = fma(cp, a2, -1.0 / 720.0);
    cp = fma(cp, a2, 1.0 / 24.0);
    const double ca = fma(a2 * a2, cp, fma(a2, -0.5, 1.0));
    switch (q) {
        case 0: c = ca; s = sa; break;
        case 1: c = -sa; s = ca; break;
        case 2: c = -ca; s = -sa; break;
        default: c = sa; s = -ca; break;
    }
}

__device__ __forceinline__ void uniforms(uint64_t seed, int64_t row, int64_t col, double& u1, double& u2) {
    uint32_t c[4] = {(uint32_t)row, (uint32_t)((uint64_t)row >> 32), (uint32_t)col, (uint32_t)((uint64_t)col >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((uint64_t)c[0] << 32) | c[1];
    const uint64_t b = ((uint64_t)c[2] << 32) | c[3];
    u1 = (double)((a >> 11) + 1) * 0x1.0p-53;
    u2 = (double)(b >> 11) * 0x1.0p-53;
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
                                                         int64_t row0, int64_t col0, uint64_t seed, int narrow) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = blockIdx.y; j < cols; j += gridDim.y) {
        D* column = dst + j * ld;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) {
            double u1, u2, c, s;
            uniforms(seed, row0 + i, col0 + j, u1, u2);
            cos_sin_2pi(u2, c, s);
            const double l = ln_pos(u1);
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
        static_cast<D*>(dst), ld, rows, cols, row0, col0, seed, narrow);
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
