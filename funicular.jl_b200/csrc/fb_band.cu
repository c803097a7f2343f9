// A Hermitian band operator, the dense-in-its-band G of the differentiation
// workload (S = Q^H (G Q) with G Hermitian of bandwidth kd): Y <- G X for the
// columns of a device panel, the panel-capable mul! of apply_operator!
// (src/operator.jl:80-87).
//
// G is stored by diagonals: column d (0 <= d <= kd) of the N x (kd + 1)
// matrix Dg holds the d-th superdiagonal, Dg[i + d ld] = G[i, i + d]; the
// subdiagonals are their conjugates, G[i, i - d] = conj(Dg[i - d + d ld]), and
// the imaginary part of the main diagonal is ignored. Both reads of a
// diagonal are coalesced across consecutive rows, unlike LAPACK's band
// storage, which keeps a column of G contiguous.
//
// A thread owns one row and CB columns of the output; the blocks of one row
// tile run side by side over the column chunks, so each diagonal entry
// comes from DRAM once and from L2 for the other chunks, and the X rows of
// the band come from L1.
#include "fb_common.cuh"

namespace fb {

constexpr int HB_ROWS = 128;
constexpr int HB_CB = 4;

__device__ __forceinline__ z64 zconj_b(z64 a) { return zmake(a.x, -a.y); }

__global__ void __launch_bounds__(HB_ROWS)
hband_kernel(z64* __restrict__ Y, int64_t ldy, const z64* __restrict__ X, int64_t ldx, const z64* __restrict__ Dg,
             int64_t lddg, int64_t N, int kd, int cols) {
    const int c0 = blockIdx.x * HB_CB;
    const int64_t tiles = (N + HB_ROWS - 1) / HB_ROWS;
    for (int64_t tile = blockIdx.y; tile < tiles; tile += gridDim.y) {
        const int64_t i = tile * HB_ROWS + threadIdx.x;
        if (i >= N) continue;
        const z64* x[HB_CB];
#pragma unroll
        for (int c = 0; c < HB_CB; ++c) x[c] = X + (int64_t)(c0 + c < cols ? c0 + c : c0) * ldx;
        z64 acc[HB_CB];
        const double g0 = __ldg(&Dg[i].x);
#pragma unroll
        for (int c = 0; c < HB_CB; ++c) {
            const z64 v = __ldg(x[c] + i);
            acc[c] = zmake(g0 * v.x, g0 * v.y);
        }
        for (int d = 1; d <= kd; ++d) {
            if (i + d < N) {
                const z64 g = __ldg(Dg + i + (int64_t)d * lddg);
#pragma unroll
                for (int c = 0; c < HB_CB; ++c) zmac(acc[c], g, __ldg(x[c] + i + d));
            }
            if (i - d >= 0) {
                const z64 g = zconj_b(__ldg(Dg + (i - d) + (int64_t)d * lddg));
#pragma unroll
                for (int c = 0; c < HB_CB; ++c) zmac(acc[c], g, __ldg(x[c] + i - d));
            }
        }
#pragma unroll
        for (int c = 0; c < HB_CB; ++c)
            if (c0 + c < cols) Y[i + (int64_t)(c0 + c) * ldy] = acc[c];
    }
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zhband_apply(fb_z128* Y, int64_t ldy, const fb_z128* X, int64_t ldx, const fb_z128* Dg, int64_t lddg,
                    int64_t N, int kd, int cols, fb_queue_t queue) {
    if (N < 0 || kd < 0 || cols < 0) {
        set_error(FB_EINVAL, "fb_zhband_apply: N = %lld, kd = %d, cols = %d", (long long)N, kd, cols);
        return FB_EINVAL;
    }
    if (N == 0 || cols == 0) return FB_OK;
    if (!Y || !X || !Dg) { set_error(FB_EINVAL, "fb_zhband_apply: NULL matrix"); return FB_EINVAL; }
    if (ldy < N || ldx < N || lddg < N) {
        set_error(FB_EDIM, "fb_zhband_apply: leading dimensions %lld, %lld, %lld below N = %lld", (long long)ldy,
                  (long long)ldx, (long long)lddg, (long long)N);
        return FB_EDIM;
    }
    if (((uintptr_t)Y | (uintptr_t)X | (uintptr_t)Dg) & 15) {
        set_error(FB_EINVAL, "fb_zhband_apply: pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    const char* y0 = reinterpret_cast<const char*>(Y);
    const char* x0 = reinterpret_cast<const char*>(X);
    const size_t ybytes = ((size_t)(cols - 1) * ldy + N) * 16, xbytes = ((size_t)(cols - 1) * ldx + N) * 16;
    if (y0 < x0 + xbytes && x0 < y0 + ybytes) {
        set_error(FB_EINVAL, "fb_zhband_apply: the output overlaps the input");
        return FB_EINVAL;
    }
    const int64_t chunks = (cols + HB_CB - 1) / HB_CB;
    if (chunks > 65535) { set_error(FB_ENOTSUP, "fb_zhband_apply: more than %d columns", 65535 * HB_CB); return FB_ENOTSUP; }
    int64_t tiles = (N + HB_ROWS - 1) / HB_ROWS;
    if (tiles > 65535) tiles = 65535;
    hband_kernel<<<dim3((unsigned)chunks, (unsigned)tiles), HB_ROWS, 0, stream_of(queue)>>>(
        reinterpret_cast<z64*>(Y), ldy, reinterpret_cast<const z64*>(X), ldx, reinterpret_cast<const z64*>(Dg), lddg,
        N, kd, cols);
    FB_LAUNCHED("hband_kernel");
    return FB_OK;
}

}  // extern "C"
