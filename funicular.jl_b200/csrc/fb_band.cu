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
// reaches (256 + 2 kd of them) are staged in shared memory 16 columns at
// a time, column-major with a padded column length so that one fragment load
// (two rows by four columns) touches 32 distinct banks, in two buffers: one
// CTA an SM copies the next stage with cp.async while its warps multiply
// the current one, so the tensor pipe does not wait for the copies. Signs
// of the real form are flipped on the integer pipe, leaving the FP64 pipe,
// which the MMAs share, to the MMAs. A wider band falls
// back to the FP64-pipe kernel below: a thread owns one row and CB columns of
// the output; the blocks of one row tile run side by side over the column
// chunks, so each diagonal entry comes from DRAM once and from L2 for the
// other chunks, and the X rows of the band come from L1.
#include <type_traits>

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
constexpr int HBT_COLS = 16;               // columns of X a stage holds
constexpr int HBT_NT = HBT_COLS / 4;       // n-tiles of a stage
constexpr int HBT_STAGES = 2;
constexpr int HBT_KDMAX = 64;

// Column length of a staged X block: HBT_ROWS + 2 HBT_KDMAX rows (any band
// up to HBT_KDMAX fits), padded to 2 mod 8 so that the four columns a
// fragment load reads start 8 banks apart. Fixed, so fragment loads take
// their column offsets as immediates.
constexpr int hbt_pitch_for(int rows) { return (rows & 7) == 2 ? rows : hbt_pitch_for(rows + 1); }
constexpr int HBT_PITCH = hbt_pitch_for(HBT_ROWS + 2 * HBT_KDMAX);
constexpr size_t HBT_SMEM = (size_t)HBT_STAGES * HBT_PITCH * HBT_COLS * sizeof(z64);

// One 16-byte copy from global to shared memory that completes
// asynchronously (cp.async, cached in L2 only); src_bytes = 0 reads nothing
// and writes zeros.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)),
                 "l"(__cvta_generic_to_global(src)), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// x with its sign bit flipped where flip has it set: a negation that takes
// an integer instruction instead of the FP64 pipe the MMAs run on.
__device__ __forceinline__ double flip_sign(double x, unsigned flip) {
    return __hiloint2double(__double2hiint(x) ^ (int)flip, __double2loint(x));
}

// The A operand of the band product, one lane's entries k-step after
// k-step. Lane (rr, kr) of m-tile m supplies part p = kr & 1 of G[i][j] with
// i = wi0 + 8 m + rr and j = j0 + 2 s, j0 = wi0 - kd + (kr >> 1), at k-step s,
// so its diagonal is d = j - i = dd + 2 s - 8 m, dd = (kr >> 1) - rr - kd,
// whatever the tile. The entry is Dg[i, d] for d >= 0 and conj(Dg[j, -d])
// for d < 0: in doubles, base + P_m for d >= 0 and base + Q_m for d < 0, with
// base = Dg + 2 wi0 and offsets that advance by fixed strides from one k-step
// to the next (Off = int when every offset a unit reaches fits 32 bits).
// Which steps are live (the column in the matrix, |d| <= kd, the row in the
// matrix, not the imaginary part of the main diagonal), where d turns
// non-negative and where it is zero depend on the lane and m alone, or once
// per unit on the tile's edges, so a step tests two integer ranges. entry()
// gives the value as stored; the conjugation (the sign of part 1 where
// d < 0) is applied by sign() when the entry is used, so nothing waits on a
// load before the step that multiplies it.
template <typename Off>
struct BandFeed {
    const double* base;
    Off P[HBT_MT], Q[HBT_MT];
    Off dP, dQ;
    int s;                  // k-step of the next entries
    int L[HBT_MT];          // live steps: L <= s <= L + W, s != Z
    unsigned W[HBT_MT];
    int Z[HBT_MT];
    int S[HBT_MT];          // first step with d >= 0
    int T[HBT_MT];          // steps below T take a flipped sign (S for part 1, none for part 0)

    __device__ __forceinline__ void start(const double* __restrict__ Dg, int64_t wi0, int rr, int kr, int kd,
                                          int64_t N, int64_t lddg) {
        const int p = kr & 1;
        const int dd = (kr >> 1) - rr - kd;
        const int64_t j0 = wi0 - kd + (kr >> 1);
        base = Dg + 2 * wi0;
        dP = (Off)(4 * lddg);
        dQ = (Off)(4 - 4 * lddg);
        s = 0;
        // The column j0 + 2 s lies in the matrix for first <= s <= last.
        const int64_t first = j0 >= 0 ? 0 : (1 - j0) >> 1;
        const int64_t last64 = (N - 1 - j0) >> 1;
        const int lo = (int)(first < 4096 ? first : 4096);
        const int hi = (int)(last64 < 4096 ? (last64 < -1 ? -1 : last64) : 4096);
        constexpr int NEVER = 1 << 30;
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m) {
            const int e = 8 * m - dd;   // d = 2 s - e
            P[m] = (Off)(2 * (8 * m + rr) + p - 2 * lddg * e);
            Q[m] = (Off)(2 * (j0 - wi0) + p + 2 * lddg * e);
            S[m] = (e + 1) >> 1;
            T[m] = p ? S[m] : -NEVER;
            Z[m] = (p && !(e & 1)) ? e >> 1 : -NEVER;
            const int sa = (e - kd + 1) >> 1, sb = (e + kd) >> 1;   // |2 s - e| <= kd
            const int l = sa > lo ? sa : lo, h = sb < hi ? sb : hi;
            const bool any = h >= l && wi0 + 8 * m + rr < N;
            L[m] = any ? l : NEVER;
            W[m] = any ? (unsigned)(h - l) : 0u;
        }
    }
    // Part p of m-tile m's entry at step s, as stored.
    __device__ __forceinline__ double entry(int m) const {
        const bool live = (unsigned)(s - L[m]) <= W[m] && s != Z[m];
        const Off at = s < S[m] ? Q[m] : P[m];
        return live ? __ldg(base + at) : 0.0;
    }
    // The sign flip that turns m-tile m's stored entry at step st into G's.
    __device__ __forceinline__ unsigned sign(int st, int m) const { return st < T[m] ? 0x80000000u : 0u; }
    __device__ __forceinline__ void advance() {
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m) {
            P[m] += dP;
            Q[m] += dQ;
        }
        ++s;
    }
};

// Whether every offset BandFeed<int> forms stays in 32 bits: |offset| is at
// most 2 lddg (kd + 24) + 2 (kd + 40) over the steps a unit reaches.
__host__ __device__ inline bool hbt_offsets_fit_int(int64_t lddg, int kd) {
    return 2 * lddg * (int64_t)(kd + 32) + 4096 < ((int64_t)1 << 31);
}

// Copies rows xrow0 .. xrow0 + staged - 1 of columns c0 .. c0 + HBT_COLS - 1
// of X into a stage buffer (column-major, HBT_PITCH rows a column), zeros for
// rows outside the matrix and columns past `cols`.
__device__ __forceinline__ void hbt_stage(z64* __restrict__ xs, int staged, const z64* __restrict__ X,
                                          int64_t ldx, int64_t N, int cols, int64_t xrow0, int c0) {
#pragma unroll 1
    for (int c = 0; c < HBT_COLS; ++c) {
        const bool col_live = c0 + c < cols;
        const z64* column = X + (int64_t)(col_live ? c0 + c : 0) * ldx;
        for (int r = threadIdx.x; r < staged; r += blockDim.x) {
            const int64_t gr = xrow0 + r;
            const bool live = col_live && gr >= 0 && gr < N;
            cp_async16(xs + c * HBT_PITCH + r, live ? column + gr : X, live ? 16 : 0);
        }
    }
}

// One CTA an SM walks units (a tile of HBT_ROWS rows, a stage of HBT_COLS
// columns), the tile's columns in order, then its next tile. The X rows the
// next unit reaches are copied into the other stage buffer while this unit's
// MMAs run. A warp's window of k-steps (2 kd + 16 columns) is the union of its
// two m-tiles' bands: m-tile m's rows 8 m .. 8 m + 7 reach k-steps
// 4 m .. 4 m + kd + 3, so the window runs in three phases (m-tile 0 alone,
// both, m-tile 1 alone), each a straight loop, and no MMA multiplies a
// k-step outside its m-tile's band.
template <typename Off>
__global__ void __launch_bounds__(HBT_WARPS * 32, 1)
hband_dmma_kernel(z64* __restrict__ Y, int64_t ldy, const z64* __restrict__ X, int64_t ldx,
                  const z64* __restrict__ Dg, int64_t lddg, int64_t N, int kd, int cols) {
    static_assert(HBT_MT == 2, "the phases below are written for two m-tiles a warp");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    z64* xs0 = reinterpret_cast<z64*>(smem_raw);   // HBT_STAGES buffers of HBT_COLS columns of HBT_PITCH rows
    constexpr int pitch = HBT_PITCH;
    constexpr int stage_elems = HBT_PITCH * HBT_COLS;
    const int staged = HBT_ROWS + 2 * kd;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rr = lane >> 2, kr = lane & 3, nr = lane >> 2;
    const int p = kr & 1, o = nr & 1, cq = lane & 3;
    // The B entry this lane supplies: part (p ^ o) of X[row][col], negated
    // for (p, o) = (1, 0): the real form of the complex product.
    const int bpart = p ^ o;
    const unsigned bflip = (p == 1 && o == 0) ? 0x80000000u : 0u;
    const int64_t tiles = (N + HBT_ROWS - 1) / HBT_ROWS;
    const int nchunks = (cols + HBT_COLS - 1) / HBT_COLS;
    const int64_t mine = (int64_t)blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t units = mine * nchunks;
    auto unit_row0 = [&](int64_t u) { return ((int64_t)blockIdx.x + (u / nchunks) * gridDim.x) * HBT_ROWS; };
    auto unit_col0 = [&](int64_t u) { return (int)(u % nchunks) * HBT_COLS; };
    const double* dg = reinterpret_cast<const double*>(Dg);

    if (units > 0) hbt_stage(xs0, staged, X, ldx, N, cols, unit_row0(0) - kd, unit_col0(0));
    cp_async_commit();
    for (int64_t u = 0; u < units; ++u) {
        const int64_t i0 = unit_row0(u);
        const int c0 = unit_col0(u);
        const int64_t wi0 = i0 + HBT_WROWS * warp;   // this warp's first row
        BandFeed<Off> feed;
        feed.start(dg, wi0, rr, kr, kd, N, lddg);
        // The band entries of k-steps s and s + 1 (the next two to multiply);
        // the first two do not depend on the stage, so they load across the
        // wait.
        double e0[HBT_MT], e1[HBT_MT];
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m) e0[m] = feed.entry(m);
        feed.advance();
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m) e1[m] = feed.entry(m);
        feed.advance();
        // One barrier a unit: past it, unit u's copies (the only group in
        // flight) are visible to every warp, and every warp has finished
        // unit u - 1, so unit u + 1 may land in the buffer that unit read.
        cp_async_wait<0>();
        __syncthreads();
        if (u + 1 < units) {
            hbt_stage(xs0 + ((u + 1) & 1) * stage_elems, staged, X, ldx, N, cols, unit_row0(u + 1) - kd,
                      unit_col0(u + 1));
            cp_async_commit();
        }
        const z64* xs = xs0 + (u & 1) * stage_elems;
        double acc[HBT_MT][HBT_NT][2];
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m)
#pragma unroll
            for (int t = 0; t < HBT_NT; ++t) acc[m][t][0] = acc[m][t][1] = 0.0;
        if (wi0 < N) {
            // k-steps [sb, se) with m-tiles MLO..MHI multiplying: B is local
            // rows HBT_WROWS warp + 2 s + (kr >> 1) of the stage, columns
            // 4 t + (nr >> 1), each B entry serving every multiplying m-tile;
            // the entries of step s + 2 load while step s multiplies.
            const double* xb0 = reinterpret_cast<const double*>(xs + (nr >> 1) * pitch + HBT_WROWS * warp + (kr >> 1)) +
                                bpart;
            auto phase = [&](auto mlo, auto mhi, int sb, int se) {
                constexpr int MLO = decltype(mlo)::value, MHI = decltype(mhi)::value;
#pragma unroll 2
                for (int s = sb; s < se; ++s) {
                    double a[HBT_MT];
#pragma unroll
                    for (int m = 0; m < HBT_MT; ++m) {
                        a[m] = flip_sign(e0[m], feed.sign(s, m));
                        e0[m] = e1[m];
                        e1[m] = feed.entry(m);
                    }
                    feed.advance();
                    const double* xb = xb0 + 4 * s;
                    double b[HBT_NT];
#pragma unroll
                    for (int t = 0; t < HBT_NT; ++t) b[t] = flip_sign(xb[2 * (4 * t) * pitch], bflip);
#pragma unroll
                    for (int m = MLO; m <= MHI; ++m)
#pragma unroll
                        for (int t = 0; t < HBT_NT; ++t) dmma_884(acc[m][t][0], acc[m][t][1], a[m], b[t]);
                }
            };
            phase(std::integral_constant<int, 0>(), std::integral_constant<int, 0>(), 0, 4);
            phase(std::integral_constant<int, 0>(), std::integral_constant<int, 1>(), 4, kd + 4);
            phase(std::integral_constant<int, 1>(), std::integral_constant<int, 1>(), kd + 4, kd + 8);
        }
#pragma unroll
        for (int m = 0; m < HBT_MT; ++m) {
            const int64_t row = wi0 + 8 * m + rr;
            if (row >= N) continue;
#pragma unroll
            for (int t = 0; t < HBT_NT; ++t) {
                const int col = c0 + 4 * t + cq;
                if (col < cols) Y[row + (int64_t)col * ldy] = zmake(acc[m][t][0], acc[m][t][1]);
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
        const bool narrow = hbt_offsets_fit_int(lddg, kd);
        auto kernel = narrow ? hband_dmma_kernel<int> : hband_dmma_kernel<int64_t>;
        FB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HBT_SMEM),
                "cudaFuncSetAttribute(hband_dmma_kernel)");
        const int64_t tiles = (N + HBT_ROWS - 1) / HBT_ROWS;
        int64_t grid = (int64_t)sm_count();   // one CTA an SM (its shared memory), each walking its tiles
        if (grid > tiles) grid = tiles;
        kernel<<<(unsigned)grid, HBT_WARPS * 32, HBT_SMEM, stream_of(queue)>>>(
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
