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
// For kd <= 64 the product runs on the FP64 tensor cores (DMMA m8n8k4 on
// the real form of the complex product): a CTA owns 256 rows, a warp 16 of
// them (two 8-row m-tiles), and the band of those rows, columns
// i - kd .. i + 15 + kd, is the MMA A operand (entries of G, loaded once per
// k-step and reused for every n-tile) against the real form of X as the B
// operand, each B entry serving both m-tiles. The X rows the CTA's band
// reaches (256 + 2 kd of them) are staged in shared memory 32 columns at
// a time, column-major with a padded column length so that one fragment load
// (two rows by four columns) touches 32 distinct banks. A wider band falls
// back to the FP64-pipe kernel below: a thread owns one row and CB columns of
// the output; the blocks of one row tile run side by side over the column
// chunks, so each diagonal entry comes from DRAM once and from L2 for the
// other chunks, and the X rows of the band come from L1.
#include "fb_common.cuh"
#include "fb_tma.cuh"

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

constexpr int HBT_MT = 2;                  // 8-row m-tiles a warp owns
constexpr int HBT_WROWS = 8 * HBT_MT;      // rows a warp owns
constexpr int HBT_WARPS = 16;
constexpr int HBT_ROWS = HBT_WARPS * HBT_WROWS;  // rows a CTA owns
constexpr int HBT_COLS = 32;               // columns of X staged at a time (8 n-tiles)
constexpr int HBT_KDMAX = 64;
constexpr int HBT_AHEAD = 2;               // k-steps of band entries loaded ahead (32 products)

// Column length of the staged X tile: HBT_ROWS + 2 kd rows, padded to 2 mod 8 so
// that the four columns a fragment load reads start 8 banks apart.
__host__ __device__ inline int hbt_pitch(int kd) {
    int r = HBT_ROWS + 2 * kd;
    while ((r & 7) != 2) ++r;
    return r;
}

// Part p of G[i][j], zero outside the matrix and the band. The lanes of a
// warp fall on different sides of the diagonal, so the entry is found without
// branching: one address (the superdiagonal entry for j >= i, the conjugate
// of the mirrored one for j < i) and one predicated load.
__device__ __forceinline__ double band_part(const double* __restrict__ Dg, int64_t lddg, int64_t N, int kd, int64_t i,
                                            int64_t j, int p) {
    const int64_t d = j - i;
    const int64_t ad = d < 0 ? -d : d;
    const bool live = i < N && j >= 0 && j < N && ad <= kd && !(d == 0 && p);
    const int64_t at = 2 * ((d >= 0 ? i : j) + ad * lddg) + p;
    const double v = live ? __ldg(Dg + at) : 0.0;
    return (d < 0 && p) ? -v : v;
}

__global__ void __launch_bounds__(HBT_WARPS * 32, 1)
hband_dmma_kernel(z64* __restrict__ Y, int64_t ldy, const z64* __restrict__ X, int64_t ldx,
                  const z64* __restrict__ Dg, int64_t lddg, int64_t N, int kd, int cols) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    z64* xs = reinterpret_cast<z64*>(smem_raw);   // HBT_COLS columns of `pitch` rows
    const int pitch = hbt_pitch(kd);
    const int staged = HBT_ROWS + 2 * kd;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rr = lane >> 2, kr = lane & 3, nr = lane >> 2;
    const int p = kr & 1, o = nr & 1, cq = lane & 3;
    // The B entry this lane supplies: part (p ^ o) of X[row][col], negated
    // for (p, o) = (1, 0): the real form of the complex product.
    const int bpart = p ^ o;
    const double bsign = (p == 1 && o == 0) ? -1.0 : 1.0;
    const int nsteps = kd + HBT_WROWS / 2;         // k-steps of a warp's band: 2 kd + 16 columns
    const int64_t tiles = (N + HBT_ROWS - 1) / HBT_ROWS;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t i0 = tile * HBT_ROWS;
        const int64_t xrow0 = i0 - kd;             // first staged row (may be negative: zeros)
        const int64_t wi0 = i0 + HBT_WROWS * warp; // this warp's first row
        for (int c0 = 0; c0 < cols; c0 += HBT_COLS) {
            __syncthreads();   // the previous chunk's fragments have all been read
            for (int e = threadIdx.x; e < staged * HBT_COLS; e += blockDim.x) {
                const int r = e % staged, c = e / staged;
                const int64_t gr = xrow0 + r;
                z64 v = zmake(0.0, 0.0);
                if (gr >= 0 && gr < N && c0 + c < cols) v = X[gr + (int64_t)(c0 + c) * ldx];
                xs[c * pitch + r] = v;
            }
            __syncthreads();
            double acc[HBT_MT][8][2];
#pragma unroll
            for (int m = 0; m < HBT_MT; ++m)
#pragma unroll
                for (int t = 0; t < 8; ++t) acc[m][t][0] = acc[m][t][1] = 0.0;
            if (wi0 < N) {
                // k-step s covers columns jb, jb + 1 with jb = wi0 - kd + 2 s
                // (the union of the m-tiles' bands); this lane's A entry of
                // m-tile m is G[wi0 + 8 m + rr][jb + (kr >> 1)], part p. The
                // entries of the next HBT_AHEAD steps are in flight.
                const double* dg = reinterpret_cast<const double*>(Dg);
                const int64_t j0 = wi0 - kd + (kr >> 1);
                double ring[HBT_MT][HBT_AHEAD];
#pragma unroll
                for (int m = 0; m < HBT_MT; ++m)
#pragma unroll
                    for (int q = 0; q < HBT_AHEAD; ++q)
                        ring[m][q] = band_part(dg, lddg, N, kd, wi0 + 8 * m + rr, j0 + 2 * q, p);
                // One k-step against the eight n-tiles: B is rows jb + (kr >> 1)
                // of the staged tile, columns 4 t + (nr >> 1); each B entry
                // serves every m-tile.
                auto step = [&](int st, const double (&a)[HBT_MT]) {
                    const int lr = (int)(wi0 - xrow0) - kd + 2 * st + (kr >> 1);
                    const double* xb = reinterpret_cast<const double*>(xs + (nr >> 1) * pitch + lr) + bpart;
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        const double b = bsign * xb[2 * (4 * t) * pitch];
#pragma unroll
                        for (int m = 0; m < HBT_MT; ++m) dmma_884(acc[m][t][0], acc[m][t][1], a[m], b);
                    }
                };
                int s = 0;
                for (; s + HBT_AHEAD <= nsteps; s += HBT_AHEAD) {
#pragma unroll
                    for (int q = 0; q < HBT_AHEAD; ++q) {
                        double a[HBT_MT];
#pragma unroll
                        for (int m = 0; m < HBT_MT; ++m) {
                            a[m] = ring[m][q];
                            ring[m][q] = band_part(dg, lddg, N, kd, wi0 + 8 * m + rr, j0 + 2 * (s + q + HBT_AHEAD), p);
                        }
                        step(s + q, a);
                    }
                }
#pragma unroll
                for (int q = 0; q < HBT_AHEAD; ++q)
                    if (s + q < nsteps) {
                        double a[HBT_MT];
#pragma unroll
                        for (int m = 0; m < HBT_MT; ++m) a[m] = ring[m][q];
                        step(s + q, a);
                    }
            }
#pragma unroll
            for (int m = 0; m < HBT_MT; ++m) {
                const int64_t row = wi0 + 8 * m + rr;
                if (row >= N) continue;
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int col = c0 + 4 * t + cq;
                    if (col < cols) Y[row + (int64_t)col * ldy] = zmake(acc[m][t][0], acc[m][t][1]);
                }
            }
        }
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
    if (kd <= HBT_KDMAX) {
        const size_t smem = (size_t)hbt_pitch(kd) * HBT_COLS * sizeof(z64);
        FB_CUDA(cudaFuncSetAttribute(hband_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(hband_dmma_kernel)");
        const int64_t tiles = (N + HBT_ROWS - 1) / HBT_ROWS;
        int64_t grid = (int64_t)sm_count() * 4;
        if (grid > tiles) grid = tiles;
        hband_dmma_kernel<<<(unsigned)grid, HBT_WARPS * 32, smem, stream_of(queue)>>>(
            reinterpret_cast<z64*>(Y), ldy, reinterpret_cast<const z64*>(X), ldx, reinterpret_cast<const z64*>(Dg),
            lddg, N, kd, cols);
        FB_LAUNCHED("hband_dmma_kernel");
        return FB_OK;
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
