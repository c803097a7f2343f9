// The tensor-core right product D <- beta D + A1 L + A2 C (fb_rmul.cuh).
//
// A team of one or two warps owns 8 rows at a time, each warp a contiguous
// share of the output n-tiles. A warp streams the rows' entries one k-step
// (two complex columns) at a time, loading each entry of A1 and A2 once (the
// second warp of a team finds them in L1), and keeps its n-tiles in its
// accumulators, so each output entry is written once. The loads run two
// groups of four k-steps ahead of the products; the group after that waits for
// the products of the current one, which bounds the registers the prefetch
// holds.
#include "fb_rmul.cuh"
#include "fb_tma.cuh"

namespace fb {

constexpr int RM_THREADS = 512;
// Warps that share one 8-row unit, each taking a contiguous share of the
// output n-tiles: wide factors split in two, which halves the accumulators a
// thread holds and lets 16 warps run on an SM instead of 8.
__host__ __device__ constexpr int rm_split(int ntn) { return ntn >= 8 ? 2 : 1; }

template <int NTK, int NTN>
__global__ void __launch_bounds__(RM_THREADS, 1)
rmul_dmma_kernel(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2, int64_t rows,
                 int K, int n, const double* __restrict__ gdense, const double* __restrict__ glower,
                 const z64* __restrict__ Cm, int64_t ldcm, z64 beta,
                 int use_beta, int zero, int inplace, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    constexpr int NS = 2 * NTK;               // k-steps
    constexpr int NT = NTN;                   // output n-tiles
    constexpr int SPLIT = rm_split(NTN);      // warps sharing one 8-row unit
    constexpr int NH = (NT + SPLIT - 1) / SPLIT;  // n-tiles of one warp
    constexpr int G = 4;                      // k-steps whose inputs are loaded together
    constexpr int NG = (NS + G - 1) / G;
    constexpr bool SQUARE = NTK == NTN;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* fd = reinterpret_cast<double*>(smem_raw);
    double* fl = fd + dense_frag_doubles(NTK, NTN);
    const bool lower = SQUARE && A1 != nullptr;
    if (gdense == nullptr) {
        // The factor given as a K x n matrix (the plain product A2 C): every
        // CTA lays out the fragments of the whole template-sized factor
        // itself, zero past K and n.
        for (int e = threadIdx.x; e < dense_frag_doubles(NTK, NTN); e += blockDim.x) {
            const int l = e & 31, q = e >> 5;
            const int s = q / NTN, t = q - s * NTN;
            fd[e] = frag_entry(Cm, ldcm, K, n, s, t, l, 1.0);
        }
    } else {
        const double2* s2 = reinterpret_cast<const double2*>(gdense);
        double2* d2 = reinterpret_cast<double2*>(fd);
        for (int e = threadIdx.x; e < dense_frag_doubles(NTK, NTN) / 2; e += blockDim.x) d2[e] = s2[e];
        if (lower) {
            const double2* l2 = reinterpret_cast<const double2*>(glower);
            double2* dl = reinterpret_cast<double2*>(fl);
            for (int e = threadIdx.x; e < lower_frag_doubles(NTN) / 2; e += blockDim.x) dl[e] = l2[e];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rr = lane >> 2, cq = lane & 3, acol = cq >> 1;
    const int apart = lane & 1;
    const int64_t units = (rows + 7) / 8;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const int t0 = (int)(gw % SPLIT) * NH;    // this warp's first n-tile
    const int64_t teams = (int64_t)gridDim.x * (blockDim.x >> 5) / SPLIT;
    for (int64_t u = gw / SPLIT; u < units; u += teams) {
        const int64_t row = u * 8 + rr;
        const bool live = row < rows;
        const int64_t r0 = live ? row : 0;
        // This lane's entries of k-steps gG .. gG + G - 1 of both inputs.
        auto load_group = [&](int g, double (&b2)[G], double (&b1)[G], const z64* p2, const z64* p1) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const int s = g * G + j;
                const int col = 2 * s + acol;
                const bool ok = s < NS && live && col < K;
                b2[j] = ok ? reinterpret_cast<const double*>(p2 + (int64_t)col * lda2)[apart] : 0.0;
                b1[j] = (ok && lower) ? reinterpret_cast<const double*>(p1 + (int64_t)col * lda1)[apart] : 0.0;
            }
        };
        double acc[NH][2];
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const int col = 4 * (t0 + h) + cq;
            z64 d = zmake(0.0, 0.0);
            if (use_beta && live && col < n) d = zmul(beta, D[r0 + (int64_t)col * ldd]);
            acc[h][0] = d.x;
            acc[h][1] = d.y;
        }
        const z64* p2 = A2 + r0;
        const z64* p1 = lower ? A1 + r0 : A2 + r0;
        double c2[G], c1[G], n2[G], n1[G];
        load_group(0, c2, c1, p2, p1);
        load_group(1, n2, n1, p2, p1);
        // Two groups of loads in flight: group g + 2 is issued once group
        // g's products are done, so its registers are not held any longer.
#pragma unroll
        for (int g = 0; g < NG; ++g) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const int s = g * G + j;
                if (s >= NS) break;
                // This step's fragments are read once the previous step's
                // first product is done, not hoisted further ahead.
                const double step_chain = acc[0][0];
                const double* fp = hold(fd + (s * NT + t0) * 32 + lane, step_chain, zero);
#pragma unroll
                for (int h = 0; h < NH; ++h)
                    if (SPLIT == 1 || t0 + h < NT) dmma_884(acc[h][0], acc[h][1], c2[j], fp[h * 32]);
                if (SQUARE && lower) {
                    const double* lp = hold(fl + (lower_step_offset(s) + t0) * 32 + lane, step_chain, zero);
#pragma unroll
                    for (int h = 0; h < NH; ++h)
                        if (t0 + h <= s / 2 && t0 + h < NT) dmma_884(acc[h][0], acc[h][1], c1[j], lp[h * 32]);
                }
            }
#pragma unroll
            for (int j = 0; j < G; ++j) {
                c2[j] = n2[j];
                c1[j] = n1[j];
            }
            if (g + 2 < NG) {
                const double chain = acc[0][0];
                load_group(g + 2, n2, n1, hold(p2, chain, zero), hold(p1, chain, zero));
            }
        }
        // When D is one of the inputs, the other warp of the team may still be
        // reading these rows: both finish reading before either writes.
        if (SPLIT > 1 && inplace) asm volatile("bar.sync %0, %1;" ::"r"(1 + warp / SPLIT), "r"(32 * SPLIT) : "memory");
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const int col = 4 * (t0 + h) + cq;
            if (live && col < n && t0 + h < NT) D[row + (int64_t)col * ldd] = zmake(acc[h][0], acc[h][1]);
        }
    }
}

// The same product on the FP64 pipes, for factors past 64: a thread per row,
// output columns in order, so D may be the same matrix as A1 (column j of the
// result reads columns l >= j of A1 only) but must not overlap A2.
__global__ void __launch_bounds__(128)
rmul_rows_kernel(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* __restrict__ A2, int64_t lda2,
                 int64_t rows, int K, int n, const z64* __restrict__ L, int64_t ldl, const z64* __restrict__ C,
                 int64_t ldc, z64 beta, int use_beta, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
        for (int j = 0; j < n; ++j) {
            z64 acc = use_beta ? zmul(beta, D[r + (int64_t)j * ldd]) : zmake(0.0, 0.0);
            if (A1)
                for (int l = j; l < K; ++l) zmac(acc, A1[r + (int64_t)l * lda1], __ldg(L + l + (int64_t)j * ldl));
            for (int l = 0; l < K; ++l) zmac(acc, A2[r + (int64_t)l * lda2], __ldg(C + l + (int64_t)j * ldc));
            D[r + (int64_t)j * ldd] = acc;
        }
    }
}

template <int NTK, int NTN>
static int launch_rmul_dmma(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2,
                            int64_t rows, int K, int n, const double* fdense, const double* flower, z64 beta,
                            int use_beta, cudaStream_t stream, const ChainStatus* st, int gate,
                            const z64* Cm = nullptr, int64_t ldcm = 0) {
    const bool lower = NTK == NTN && A1 != nullptr;
    const size_t smem = (size_t)(dense_frag_doubles(NTK, NTN) + (lower ? lower_frag_doubles(NTN) : 0)) * sizeof(double);
    FB_CUDA(cudaFuncSetAttribute(rmul_dmma_kernel<NTK, NTN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(rmul_dmma_kernel)");
    int per_sm = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rmul_dmma_kernel<NTK, NTN>, RM_THREADS, smem),
            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    const int64_t units = (rows + 7) / 8;
    const int teams_per_cta = RM_THREADS / 32 / rm_split(NTN);
    int64_t need = (units + teams_per_cta - 1) / teams_per_cta;
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    const int inplace = (D == A1 || D == A2) ? 1 : 0;
    rmul_dmma_kernel<NTK, NTN><<<(unsigned)grid, RM_THREADS, smem, stream>>>(
        D, ldd, lower ? A1 : nullptr, lda1, A2, lda2, rows, K, n, fdense, flower, Cm, ldcm, beta, use_beta, 0, inplace,
        st, gate);
    FB_LAUNCHED("rmul_dmma_kernel");
    return FB_OK;
}

// D <- beta D (when use_beta) + A C for a K x n factor C given as a matrix,
// K, n <= 64, on the tensor cores. The template is the smallest one that
// holds the factor: square when K and n take the same number of 4-column
// tiles or K takes fewer (K padded with zeros), 64 rows of K otherwise.
int rmul_matrix_enqueue(z64* D, int64_t ldd, const z64* A, int64_t lda, int64_t rows, int K, int n, const z64* C,
                        int64_t ldc, z64 beta, int use_beta, cudaStream_t stream) {
    if (rows == 0 || n == 0) return FB_OK;
    if (K < 1 || K > RM_KMAX || n > RM_KMAX) {
        set_error(FB_EINVAL, "rmul: a %d x %d factor is past the 64 x 64 the tensor-core product takes", K, n);
        return FB_EINVAL;
    }
    const int ntk = (K + 3) / 4, ntn = (n + 3) / 4;
    if (ntk <= ntn) {
        switch (ntn) {
#define FB_RM_MSQ(t) \
    case t: return launch_rmul_dmma<t, t>(D, ldd, nullptr, 0, A, lda, rows, K, n, nullptr, nullptr, beta, use_beta, stream, nullptr, GATE_ALWAYS, C, ldc);
            FB_RM_MSQ(1) FB_RM_MSQ(2) FB_RM_MSQ(3) FB_RM_MSQ(4) FB_RM_MSQ(5) FB_RM_MSQ(6) FB_RM_MSQ(7) FB_RM_MSQ(8)
            FB_RM_MSQ(9) FB_RM_MSQ(10) FB_RM_MSQ(11) FB_RM_MSQ(12) FB_RM_MSQ(13) FB_RM_MSQ(14) FB_RM_MSQ(15)
            FB_RM_MSQ(16)
#undef FB_RM_MSQ
        }
    } else {
        switch (ntn) {
#define FB_RM_MWIDE(t) \
    case t: return launch_rmul_dmma<16, t>(D, ldd, nullptr, 0, A, lda, rows, K, n, nullptr, nullptr, beta, use_beta, stream, nullptr, GATE_ALWAYS, C, ldc);
            FB_RM_MWIDE(1) FB_RM_MWIDE(2) FB_RM_MWIDE(3) FB_RM_MWIDE(4) FB_RM_MWIDE(5) FB_RM_MWIDE(6) FB_RM_MWIDE(7)
            FB_RM_MWIDE(8) FB_RM_MWIDE(9) FB_RM_MWIDE(10) FB_RM_MWIDE(11) FB_RM_MWIDE(12) FB_RM_MWIDE(13)
            FB_RM_MWIDE(14) FB_RM_MWIDE(15)
#undef FB_RM_MWIDE
        }
    }
    set_error(FB_EINVAL, "rmul: no template for a %d x %d factor", K, n);
    return FB_EINVAL;
}

int rmul_enqueue(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2, int64_t rows,
                 int K, int n, const z64* L, int64_t ldl, const z64* C, int64_t ldc, const double* fdense,
                 const double* flower, z64 beta, int use_beta, cudaStream_t stream, const ChainStatus* st, int gate) {
    if (rows == 0 || n == 0) return FB_OK;
    if (A1 && K != n) { set_error(FB_EINVAL, "rmul: a lower triangular factor is square, got %d x %d", K, n); return FB_EINVAL; }
    const int ntk = (K + 3) / 4, ntn = (n + 3) / 4;
    if (K <= RM_KMAX && n <= RM_KMAX && (ntk == ntn || ntk == RM_KMAX / 4)) {
        if (ntk == ntn) {
            switch (ntn) {
#define FB_RM_SQ(t) \
    case t: return launch_rmul_dmma<t, t>(D, ldd, A1, lda1, A2, lda2, rows, K, n, fdense, flower, beta, use_beta, stream, st, gate);
                FB_RM_SQ(1) FB_RM_SQ(2) FB_RM_SQ(3) FB_RM_SQ(4) FB_RM_SQ(5) FB_RM_SQ(6) FB_RM_SQ(7) FB_RM_SQ(8)
                FB_RM_SQ(9) FB_RM_SQ(10) FB_RM_SQ(11) FB_RM_SQ(12) FB_RM_SQ(13) FB_RM_SQ(14) FB_RM_SQ(15) FB_RM_SQ(16)
#undef FB_RM_SQ
            }
        } else {
            switch (ntn) {
#define FB_RM_WIDE(t) \
    case t: return launch_rmul_dmma<16, t>(D, ldd, nullptr, 0, A2, lda2, rows, K, n, fdense, nullptr, beta, use_beta, stream, st, gate);
                FB_RM_WIDE(1) FB_RM_WIDE(2) FB_RM_WIDE(3) FB_RM_WIDE(4) FB_RM_WIDE(5) FB_RM_WIDE(6) FB_RM_WIDE(7)
                FB_RM_WIDE(8) FB_RM_WIDE(9) FB_RM_WIDE(10) FB_RM_WIDE(11) FB_RM_WIDE(12) FB_RM_WIDE(13)
                FB_RM_WIDE(14) FB_RM_WIDE(15)
#undef FB_RM_WIDE
            }
        }
    }
    int64_t grid = (int64_t)sm_count() * 8;
    int64_t need = (rows + 127) / 128;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    rmul_rows_kernel<<<(unsigned)grid, 128, 0, stream>>>(D, ldd, A1, lda1, A2, lda2, rows, K, n, L, ldl, C, ldc, beta,
                                                         use_beta, st, gate);
    FB_LAUNCHED("rmul_rows_kernel");
    return FB_OK;
}

}  // namespace fb
