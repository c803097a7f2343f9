// The adjoints of cholqr2! and project: the hand-written backward pass of
// the differentiable range finder. The reference has no rrule
// (Project.toml:6-9 has no ChainRulesCore); these kernels are what its
// ChainRulesCore.rrule methods would call.
//
// cholqr2! computes the thin QR factorization Y = Q R with Q^H Q = I and R
// upper triangular with a real positive diagonal (src/panelblas.jl:130-146).
// For a real loss with cotangents Qbar and Rbar the cotangent of Y is
//     Ybar = (Qbar + Q H) R^-H,  H = copyltu(R Rbar^H - Qbar^H Q),
// copyltu(M) being the Hermitian matrix with M's strictly lower triangle
// below the diagonal, its conjugate transpose above and Re diag(M) on it.
// Q is never stored: with Q = Y R^-1,
//     Qbar^H Q = (Qbar^H Y) R^-1,    Ybar = Qbar R^-H + Y (R^-1 H R^-H),
// so the backward pass is one cross Gram Qbar^H Y (two N x k reads), a k x k
// prep on one CTA, and one fused pass that reads Qbar and Y and writes Ybar
// (three N x k sweeps): 80 N k bytes in all.
//
// project (src/panelblas.jl:268-301) computes S = Q^H (G Q); for a cotangent
// Sbar the cotangent of Q is Qbar = (G Q) Sbar^H + (G^H Q) Sbar, which is
// (G Q)(Sbar + Sbar^H) when G is Hermitian. The caller applies the operator;
// this file does the N x k by k x k products.
//
// The fused pass: D <- beta D + A1 L + A2 C, A1 and A2 N x k, L lower
// triangular and C dense k x k, on the FP64 tensor cores (DMMA m8n8k4 on the
// real form of the complex product, as the triangular solver does) for
// k <= 64. A warp owns 8 rows at a time; it streams their entries one k-step
// (two complex columns) at a time and keeps every output n-tile in its
// accumulators, so each input entry is read once and each output written
// once. L and C sit in shared memory as MMA B fragments ordered by k-step,
// L keeping only the n-tiles on or below its diagonal.
#include "fb_common.cuh"
#include "fb_tma.cuh"

namespace fb {

int gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, const z64* B, int64_t ldb,
                 int64_t rows, int kA, int kB, z64 alpha, z64 beta, bool hermitian,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream,
                 const ChainStatus* st, int gate);
size_t gram_workspace_size(int64_t rows, int kA, int kB, bool hermitian);

constexpr int AD_KMAX = 64;       // widest k of the tensor-core pass
constexpr int AD_THREADS = 256;   // threads of the tensor-core pass
constexpr int PREP_THREADS = 1024;

// B fragments of one dense k x k factor: NT n-tiles x 2 NT k-steps x 32 lanes.
__host__ __device__ inline int dense_frag_doubles(int nt) { return 64 * nt * nt; }
// Of a lower triangular one: k-step s holds n-tiles 0 .. s/2.
__host__ __device__ inline int lower_frag_doubles(int nt) { return 32 * nt * (nt + 1); }
__host__ __device__ inline int lower_step_offset(int s) {
    const int m = s >> 1;
    return (s & 1) ? (m + 1) * (m + 1) : m * (m + 1);
}

// Entry (kr, nr) of the real 8 x 8 form of a complex 4 x 4 block M: kr = 2 i + p
// (row i of M, part p of the input entry it multiplies), nr = 2 j + o (column
// j, part o of the output).
__device__ __forceinline__ double real_part_of(z64 m, int p, int o) {
    return o == 0 ? (p == 0 ? m.x : -m.y) : (p == 0 ? m.y : m.x);
}

// The B fragment entry of `lane` for k-step s and n-tile t of a column-major
// k x k matrix M (zero past k): lane & 3 is the real k index inside the
// step, lane >> 2 the real n index inside the tile.
__device__ __forceinline__ double frag_entry(const z64* M, int k, int s, int t, int lane) {
    const int kr = lane & 3, nr = lane >> 2;
    const int i = 2 * s + (kr >> 1), p = kr & 1;
    const int j = 4 * t + (nr >> 1), o = nr & 1;
    return (i < k && j < k) ? real_part_of(M[i + (int64_t)j * k], p, o) : 0.0;
}

__device__ void build_dense_frags(double* frag, const z64* M, int k, int nt) {
    for (int e = threadIdx.x; e < dense_frag_doubles(nt); e += blockDim.x) {
        const int lane = e & 31, q = e >> 5;
        const int s = q / nt, t = q - s * nt;
        frag[e] = frag_entry(M, k, s, t, lane);
    }
}

__device__ void build_lower_frags(double* frag, const z64* M, int k, int nt) {
    for (int e = threadIdx.x; e < lower_frag_doubles(nt); e += blockDim.x) {
        const int lane = e & 31, q = e >> 5;
        int s = 0;
        while (lower_step_offset(s + 1) <= q) ++s;
        frag[e] = frag_entry(M, k, s, q - lower_step_offset(s), lane);
    }
}

__device__ __forceinline__ z64 zconj(z64 a) { return zmake(a.x, -a.y); }

// The k x k half of the cholqr2! adjoint, one CTA. Matrices are column-major
// with leading dimension k in the workspace. X = Qbar^H Y (NULL when Qbar is
// zero), Rbar may be NULL (zero). Writes L = R^-H and C = R^-1 H R^-H, and
// their fragments when k <= 64.
__global__ void __launch_bounds__(PREP_THREADS, 1)
cholqr2_adjoint_prep_kernel(const z64* __restrict__ R, int64_t ldr, const z64* __restrict__ Rbar, int64_t ldrb,
                            const z64* __restrict__ X, int k, z64* Rinv, z64* P, z64* H, z64* T, z64* L, z64* C,
                            double* fdense, double* flower) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const int64_t kk = (int64_t)k * k;
    // R^-1 by rows from the bottom, a thread per column:
    // Rinv[i][j] = (delta_ij - sum_{i<l<=j} R[i][l] Rinv[l][j]) / R[i][i].
    for (int64_t e = tid; e < kk; e += nth) Rinv[e] = zmake(0.0, 0.0);
    __syncthreads();
    for (int i = k - 1; i >= 0; --i) {
        const z64 d = R[i + (int64_t)i * ldr];
        const double s = 1.0 / fma(d.x, d.x, d.y * d.y);
        const z64 dinv = zmake(d.x * s, -d.y * s);
        for (int j = i + tid; j < k; j += nth) {
            z64 acc = zmake(j == i ? 1.0 : 0.0, 0.0);
            for (int l = i + 1; l <= j; ++l) zmsub(acc, R[i + (int64_t)l * ldr], Rinv[l + (int64_t)j * k]);
            Rinv[i + (int64_t)j * k] = zmul(acc, dinv);
        }
        __syncthreads();
    }
    // P = Qbar^H Q = X R^-1; M = R Rbar^H - P on and below the diagonal (the
    // part copyltu reads), kept in P.
    for (int64_t e = tid; e < kk; e += nth) {
        const int i = (int)(e % k), j = (int)(e / k);
        if (i < j) continue;
        z64 m = zmake(0.0, 0.0);
        if (Rbar)
            for (int l = i; l < k; ++l) zmac(m, R[i + (int64_t)l * ldr], zconj(Rbar[j + (int64_t)l * ldrb]));
        if (X)
            for (int l = 0; l <= j; ++l) zmsub(m, X[i + (int64_t)l * k], Rinv[l + (int64_t)j * k]);
        P[e] = m;
    }
    __syncthreads();
    // H = copyltu(M).
    for (int64_t e = tid; e < kk; e += nth) {
        const int i = (int)(e % k), j = (int)(e / k);
        H[e] = i > j ? P[e] : (i < j ? zconj(P[j + (int64_t)i * k]) : zmake(P[e].x, 0.0));
    }
    __syncthreads();
    // T = H R^-H: T[i][j] = sum_{l>=j} H[i][l] conj(Rinv[j][l]); L = R^-H.
    for (int64_t e = tid; e < kk; e += nth) {
        const int i = (int)(e % k), j = (int)(e / k);
        z64 t = zmake(0.0, 0.0);
        for (int l = j; l < k; ++l) zmac(t, H[i + (int64_t)l * k], zconj(Rinv[j + (int64_t)l * k]));
        T[e] = t;
        L[e] = i >= j ? zconj(Rinv[j + (int64_t)i * k]) : zmake(0.0, 0.0);
    }
    __syncthreads();
    // C = R^-1 T: C[i][j] = sum_{l>=i} Rinv[i][l] T[l][j].
    for (int64_t e = tid; e < kk; e += nth) {
        const int i = (int)(e % k), j = (int)(e / k);
        z64 c = zmake(0.0, 0.0);
        for (int l = i; l < k; ++l) zmac(c, Rinv[i + (int64_t)l * k], T[l + (int64_t)j * k]);
        C[e] = c;
    }
    __syncthreads();
    if (k <= AD_KMAX) {
        const int nt = (k + 3) / 4;
        build_dense_frags(fdense, C, k, nt);
        build_lower_frags(flower, L, k, nt);
    }
}

// The k x k half of the project adjoint, one CTA: C1 = Sbar^H + Sbar when
// `hermitian` (G Hermitian: one product), else C1 = Sbar^H and C2 = Sbar.
__global__ void __launch_bounds__(PREP_THREADS, 1)
project_adjoint_prep_kernel(const z64* __restrict__ Sbar, int64_t ldsb, int k, int hermitian, z64* C1, z64* C2,
                            double* f1, double* f2) {
    const int64_t kk = (int64_t)k * k;
    for (int64_t e = threadIdx.x; e < kk; e += blockDim.x) {
        const int i = (int)(e % k), j = (int)(e / k);
        const z64 s = Sbar[i + (int64_t)j * ldsb];
        const z64 sh = zconj(Sbar[j + (int64_t)i * ldsb]);
        C1[e] = hermitian ? zmake(s.x + sh.x, s.y + sh.y) : sh;
        C2[e] = s;
    }
    __syncthreads();
    if (k <= AD_KMAX) {
        const int nt = (k + 3) / 4;
        build_dense_frags(f1, C1, k, nt);
        if (!hermitian) build_dense_frags(f2, C2, k, nt);
    }
}

// D <- beta D + A1 L + A2 C on the FP64 tensor cores (k <= 4 NT). A1 may be
// NULL (no L term). D may be the same matrix as A1 or A2: a warp reads all of
// its rows' inputs before it writes their outputs.
template <int NT>
__global__ void __launch_bounds__(AD_THREADS, 1)
rmul_dmma_kernel(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2, int64_t rows,
                 int k, const double* __restrict__ gdense, const double* __restrict__ glower, z64 beta,
                 int use_beta, int zero) {
    constexpr int NS = 2 * NT;          // k-steps
    constexpr int G = 4;                // k-steps whose inputs are loaded together
    constexpr int NG = (NS + G - 1) / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* fd = reinterpret_cast<double*>(smem_raw);
    double* fl = fd + dense_frag_doubles(NT);
    const bool lower = A1 != nullptr;
    {
        const double2* s2 = reinterpret_cast<const double2*>(gdense);
        double2* d2 = reinterpret_cast<double2*>(fd);
        for (int e = threadIdx.x; e < dense_frag_doubles(NT) / 2; e += blockDim.x) d2[e] = s2[e];
        if (lower) {
            const double2* l2 = reinterpret_cast<const double2*>(glower);
            double2* dl = reinterpret_cast<double2*>(fl);
            for (int e = threadIdx.x; e < lower_frag_doubles(NT) / 2; e += blockDim.x) dl[e] = l2[e];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rr = lane >> 2, cq = lane & 3, acol = cq >> 1, apart = lane & 1;
    const int64_t units = (rows + 7) / 8;
    const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; u < units; u += warps_total) {
        const int64_t row = u * 8 + rr;
        const bool live = row < rows;
        const int64_t r0 = live ? row : 0;
        // This lane's entries of k-steps gG .. gG + G - 1 of both inputs.
        auto load_group = [&](int g, double (&b2)[G], double (&b1)[G], const z64* p2, const z64* p1) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
                const int s = g * G + j;
                const int col = 2 * s + acol;
                const bool ok = s < NS && live && col < k;
                b2[j] = ok ? reinterpret_cast<const double*>(p2 + (int64_t)col * lda2)[apart] : 0.0;
                b1[j] = (ok && lower) ? reinterpret_cast<const double*>(p1 + (int64_t)col * lda1)[apart] : 0.0;
            }
        };
        double acc[NT][2];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const int col = 4 * t + cq;
            z64 d = zmake(0.0, 0.0);
            if (use_beta && live && col < k) d = zmul(beta, D[r0 + (int64_t)col * ldd]);
            acc[t][0] = d.x;
            acc[t][1] = d.y;
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
                const double* fp = fd + s * NT * 32 + lane;
#pragma unroll
                for (int t = 0; t < NT; ++t) dmma_884(acc[t][0], acc[t][1], c2[j], fp[t * 32]);
                if (lower) {
                    const double* lp = fl + lower_step_offset(s) * 32 + lane;
#pragma unroll
                    for (int t = 0; t <= s / 2; ++t) dmma_884(acc[t][0], acc[t][1], c1[j], lp[t * 32]);
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
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const int col = 4 * t + cq;
            if (live && col < k) D[row + (int64_t)col * ldd] = zmake(acc[t][0], acc[t][1]);
        }
    }
}

// The same product on the FP64 pipes for k > 64: a thread per row, output
// columns in order, so D may be the same matrix as A1 (column j of the
// result reads columns l >= j of A1 only) but must not overlap A2.
__global__ void __launch_bounds__(128)
rmul_rows_kernel(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* __restrict__ A2, int64_t lda2,
                 int64_t rows, int k, const z64* __restrict__ L, const z64* __restrict__ C, z64 beta, int use_beta) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
        for (int j = 0; j < k; ++j) {
            z64 acc = use_beta ? zmul(beta, D[r + (int64_t)j * ldd]) : zmake(0.0, 0.0);
            if (A1)
                for (int l = j; l < k; ++l) zmac(acc, A1[r + (int64_t)l * lda1], __ldg(L + l + (int64_t)j * k));
            for (int l = 0; l < k; ++l) zmac(acc, A2[r + (int64_t)l * lda2], __ldg(C + l + (int64_t)j * k));
            D[r + (int64_t)j * ldd] = acc;
        }
    }
}

template <int NT>
static int launch_rmul_dmma(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2,
                            int64_t rows, int k, const double* fdense, const double* flower, z64 beta, int use_beta,
                            cudaStream_t stream) {
    const size_t smem = (size_t)(dense_frag_doubles(NT) + (A1 ? lower_frag_doubles(NT) : 0)) * sizeof(double);
    FB_CUDA(cudaFuncSetAttribute(rmul_dmma_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(rmul_dmma_kernel)");
    int per_sm = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rmul_dmma_kernel<NT>, AD_THREADS, smem),
            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    const int64_t units = (rows + 7) / 8;
    int64_t need = (units + AD_THREADS / 32 - 1) / (AD_THREADS / 32);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    rmul_dmma_kernel<NT><<<(unsigned)grid, AD_THREADS, smem, stream>>>(D, ldd, A1, lda1, A2, lda2, rows, k, fdense,
                                                                       flower, beta, use_beta, 0);
    FB_LAUNCHED("rmul_dmma_kernel");
    return FB_OK;
}

// D <- beta D + A1 L + A2 C with L, C (and their fragments when k <= 64) in
// the workspace.
static int rmul_enqueue(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2,
                        int64_t rows, int k, const z64* L, const z64* C, const double* fdense,
                        const double* flower, z64 beta, int use_beta, cudaStream_t stream) {
    if (rows == 0 || k == 0) return FB_OK;
    if (k <= AD_KMAX) {
        switch ((k + 3) / 4) {
#define FB_RM_CASE(n) \
    case n: return launch_rmul_dmma<n>(D, ldd, A1, lda1, A2, lda2, rows, k, fdense, flower, beta, use_beta, stream);
            FB_RM_CASE(1) FB_RM_CASE(2) FB_RM_CASE(3) FB_RM_CASE(4) FB_RM_CASE(5) FB_RM_CASE(6)
            FB_RM_CASE(7) FB_RM_CASE(8) FB_RM_CASE(9) FB_RM_CASE(10) FB_RM_CASE(11) FB_RM_CASE(12)
            FB_RM_CASE(13) FB_RM_CASE(14) FB_RM_CASE(15) FB_RM_CASE(16)
#undef FB_RM_CASE
        }
    }
    int64_t grid = (int64_t)sm_count() * 8;
    int64_t need = (rows + 127) / 128;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    rmul_rows_kernel<<<(unsigned)grid, 128, 0, stream>>>(D, ldd, A1, lda1, A2, lda2, rows, k, L, C, beta, use_beta);
    FB_LAUNCHED("rmul_rows_kernel");
    return FB_OK;
}

// Workspace of the cholqr2! adjoint: six k x k matrices, the fragments, the
// cross Gram's scratch.
struct AdjointLayout {
    size_t X, Rinv, P, H, T, L, C, fdense, flower, gram, gram_bytes, total;
};

static AdjointLayout adjoint_layout(int64_t N, int k) {
    AdjointLayout a{};
    const size_t mat = align_up((size_t)k * k * sizeof(z64), 256);
    const int nt = (k + 3) / 4;
    size_t off = 0;
    a.X = off; off += mat;
    a.Rinv = off; off += mat;
    a.P = off; off += mat;
    a.H = off; off += mat;
    a.T = off; off += mat;
    a.L = off; off += mat;
    a.C = off; off += mat;
    a.fdense = off; off += k <= AD_KMAX ? align_up((size_t)dense_frag_doubles(nt) * sizeof(double), 256) : 0;
    a.flower = off; off += k <= AD_KMAX ? align_up((size_t)lower_frag_doubles(nt) * sizeof(double), 256) : 0;
    a.gram = off;
    a.gram_bytes = align_up(gram_workspace_size(N, k, k, false), 256);
    off += a.gram_bytes;
    a.total = off;
    return a;
}

struct ProjectLayout {
    size_t C1, C2, f1, f2, total;
};

static ProjectLayout project_layout(int k) {
    ProjectLayout p{};
    const size_t mat = align_up((size_t)k * k * sizeof(z64), 256);
    const size_t frag = k <= AD_KMAX ? align_up((size_t)dense_frag_doubles((k + 3) / 4) * sizeof(double), 256) : 0;
    p.C1 = 0;
    p.C2 = mat;
    p.f1 = 2 * mat;
    p.f2 = 2 * mat + frag;
    p.total = 2 * mat + 2 * frag;
    return p;
}

static bool overlaps(const void* a, int64_t lda, const void* b, int64_t ldb, int64_t rows, int cols) {
    if (!a || !b || cols == 0 || rows == 0) return false;
    const char* a0 = static_cast<const char*>(a);
    const char* b0 = static_cast<const char*>(b);
    const size_t abytes = ((size_t)(cols - 1) * lda + rows) * sizeof(z64);
    const size_t bbytes = ((size_t)(cols - 1) * ldb + rows) * sizeof(z64);
    return a0 < b0 + bbytes && b0 < a0 + abytes;
}

static bool misaligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) != 0; }

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zcholqr2_adjoint_workspace_size(int64_t N, int k, size_t* bytes) {
    if (!bytes || N < 0 || k < 0) { set_error(FB_EINVAL, "fb_zcholqr2_adjoint_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = (N == 0 || k == 0) ? 0 : adjoint_layout(N, k).total;
    return FB_OK;
}

int fb_zcholqr2_adjoint(fb_z128* Ybar, int64_t ldyb, const fb_z128* Y, int64_t ldy, const fb_z128* R, int64_t ldr,
                        const fb_z128* Qbar, int64_t ldqb, const fb_z128* Rbar, int64_t ldrb, int64_t N, int k,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (N < 0 || k < 0) {
        set_error(FB_EDIM, "the adjoint of cholqr2! takes an N x k matrix, got %lld x %d", (long long)N, k);
        return FB_EDIM;
    }
    if (N == 0 || k == 0) return FB_OK;
    if (!Ybar || !Y || !R) { set_error(FB_EINVAL, "fb_zcholqr2_adjoint: NULL Ybar, Y or R"); return FB_EINVAL; }
    if (ldyb < N || ldy < N || ldr < k || (Qbar && ldqb < N) || (Rbar && ldrb < k)) {
        set_error(FB_EDIM, "fb_zcholqr2_adjoint: leading dimension too small for an %lld x %d matrix", (long long)N, k);
        return FB_EDIM;
    }
    if (misaligned(Ybar) || misaligned(Y) || misaligned(R) || misaligned(Qbar) || misaligned(Rbar)) {
        set_error(FB_EINVAL, "fb_zcholqr2_adjoint: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    if (overlaps(Ybar, ldyb, Y, ldy, N, k)) {
        set_error(FB_EINVAL, "fb_zcholqr2_adjoint: Ybar overlaps Y (Y is read after Ybar is written)");
        return FB_EINVAL;
    }
    if (Qbar && overlaps(Ybar, ldyb, Qbar, ldqb, N, k) && !(Ybar == Qbar && ldyb == ldqb)) {
        set_error(FB_EINVAL, "fb_zcholqr2_adjoint: Ybar must be Qbar itself or not overlap it");
        return FB_EINVAL;
    }
    const AdjointLayout lay = adjoint_layout(N, k);
    if (!workspace || workspace_bytes < lay.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        set_error(FB_ENOMEM, "fb_zcholqr2_adjoint: workspace of %zu bytes, need %zu (256-byte aligned)",
                  workspace_bytes, lay.total);
        return FB_ENOMEM;
    }
    cudaStream_t stream = stream_of(queue);
    char* ws = static_cast<char*>(workspace);
    auto mat = [&](size_t off) { return reinterpret_cast<z64*>(ws + off); };
    const z64* Yz = reinterpret_cast<const z64*>(Y);
    const z64* Qb = reinterpret_cast<const z64*>(Qbar);
    if (Qb)
        FB_TRY(gram_enqueue(mat(lay.X), k, Qb, ldqb, Yz, ldy, N, k, k, zmake(1.0, 0.0), zmake(0.0, 0.0), false,
                            ws + lay.gram, lay.gram_bytes, stream, nullptr, GATE_ALWAYS));
    double* fdense = reinterpret_cast<double*>(ws + lay.fdense);
    double* flower = reinterpret_cast<double*>(ws + lay.flower);
    cholqr2_adjoint_prep_kernel<<<1, PREP_THREADS, 0, stream>>>(
        reinterpret_cast<const z64*>(R), ldr, reinterpret_cast<const z64*>(Rbar), ldrb, Qb ? mat(lay.X) : nullptr, k,
        mat(lay.Rinv), mat(lay.P), mat(lay.H), mat(lay.T), mat(lay.L), mat(lay.C), fdense, flower);
    FB_LAUNCHED("cholqr2_adjoint_prep_kernel");
    return rmul_enqueue(reinterpret_cast<z64*>(Ybar), ldyb, Qb, ldqb, Yz, ldy, N, k, mat(lay.L), mat(lay.C), fdense,
                        flower, zmake(0.0, 0.0), 0, stream);
}

int fb_zproject_adjoint_workspace_size(int k, size_t* bytes) {
    if (!bytes || k < 0) { set_error(FB_EINVAL, "fb_zproject_adjoint_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = k == 0 ? 0 : project_layout(k).total;
    return FB_OK;
}

int fb_zproject_adjoint(fb_z128* Qbar, int64_t ldqb, const fb_z128* GQ, int64_t ldgq, const fb_z128* GhQ,
                        int64_t ldghq, const fb_z128* Sbar, int64_t ldsb, int64_t N, int k, int accumulate,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (N < 0 || k < 0) {
        set_error(FB_EDIM, "the adjoint of project takes an N x k matrix, got %lld x %d", (long long)N, k);
        return FB_EDIM;
    }
    if (N == 0 || k == 0) return FB_OK;
    if (!Qbar || !GQ || !Sbar) { set_error(FB_EINVAL, "fb_zproject_adjoint: NULL Qbar, GQ or Sbar"); return FB_EINVAL; }
    if (ldqb < N || ldgq < N || ldsb < k || (GhQ && ldghq < N)) {
        set_error(FB_EDIM, "fb_zproject_adjoint: leading dimension too small for an %lld x %d matrix", (long long)N, k);
        return FB_EDIM;
    }
    if (misaligned(Qbar) || misaligned(GQ) || misaligned(GhQ) || misaligned(Sbar)) {
        set_error(FB_EINVAL, "fb_zproject_adjoint: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    if (overlaps(Qbar, ldqb, GQ, ldgq, N, k) || (GhQ && overlaps(Qbar, ldqb, GhQ, ldghq, N, k))) {
        set_error(FB_EINVAL, "fb_zproject_adjoint: Qbar overlaps an operator image");
        return FB_EINVAL;
    }
    const ProjectLayout lay = project_layout(k);
    if (!workspace || workspace_bytes < lay.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        set_error(FB_ENOMEM, "fb_zproject_adjoint: workspace of %zu bytes, need %zu (256-byte aligned)",
                  workspace_bytes, lay.total);
        return FB_ENOMEM;
    }
    cudaStream_t stream = stream_of(queue);
    char* ws = static_cast<char*>(workspace);
    z64* C1 = reinterpret_cast<z64*>(ws + lay.C1);
    z64* C2 = reinterpret_cast<z64*>(ws + lay.C2);
    double* f1 = reinterpret_cast<double*>(ws + lay.f1);
    double* f2 = reinterpret_cast<double*>(ws + lay.f2);
    const int hermitian = GhQ == nullptr;
    project_adjoint_prep_kernel<<<1, PREP_THREADS, 0, stream>>>(reinterpret_cast<const z64*>(Sbar), ldsb, k,
                                                                hermitian, C1, C2, f1, f2);
    FB_LAUNCHED("project_adjoint_prep_kernel");
    z64* Qb = reinterpret_cast<z64*>(Qbar);
    FB_TRY(rmul_enqueue(Qb, ldqb, nullptr, 0, reinterpret_cast<const z64*>(GQ), ldgq, N, k, nullptr, C1, f1, nullptr,
                        zmake(1.0, 0.0), accumulate ? 1 : 0, stream));
    if (!hermitian)
        FB_TRY(rmul_enqueue(Qb, ldqb, nullptr, 0, reinterpret_cast<const z64*>(GhQ), ldghq, N, k, nullptr, C2, f2,
                            nullptr, zmake(1.0, 0.0), 1, stream));
    return FB_OK;
}

}  // extern "C"
