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
// The fused pass is the tensor-core right product of fb_rmul.cuh with L = R^-H
// (lower triangular) and C = R^-1 H R^-H.
#include "fb_rmul.cuh"

namespace fb {

int gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, const z64* B, int64_t ldb,
                 int64_t rows, int kA, int kB, z64 alpha, z64 beta, bool hermitian,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream,
                 const ChainStatus* st, int gate);
size_t gram_workspace_size(int64_t rows, int kA, int kB, bool hermitian);

constexpr int PREP_THREADS = 1024;

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
    if (k <= RM_KMAX) {
        build_dense_frags(fdense, C, k, k, k, 1.0);
        build_lower_frags(flower, L, k, k);
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
    if (k <= RM_KMAX) {
        build_dense_frags(f1, C1, k, k, k, 1.0);
        if (!hermitian) build_dense_frags(f2, C2, k, k, k, 1.0);
    }
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
    a.fdense = off; off += k <= RM_KMAX ? align_up((size_t)dense_frag_doubles(nt, nt) * sizeof(double), 256) : 0;
    a.flower = off; off += k <= RM_KMAX ? align_up((size_t)lower_frag_doubles(nt) * sizeof(double), 256) : 0;
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
    const int nt = (k + 3) / 4;
    const size_t frag = k <= RM_KMAX ? align_up((size_t)dense_frag_doubles(nt, nt) * sizeof(double), 256) : 0;
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
    return rmul_enqueue(reinterpret_cast<z64*>(Ybar), ldyb, Qb, ldqb, Yz, ldy, N, k, k, mat(lay.L), k, mat(lay.C), k,
                        fdense, flower, zmake(0.0, 0.0), 0, stream, nullptr, GATE_ALWAYS);
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
    FB_TRY(rmul_enqueue(Qb, ldqb, nullptr, 0, reinterpret_cast<const z64*>(GQ), ldgq, N, k, k, nullptr, 0, C1, k, f1,
                        nullptr, zmake(1.0, 0.0), accumulate ? 1 : 0, stream, nullptr, GATE_ALWAYS));
    if (!hermitian)
        FB_TRY(rmul_enqueue(Qb, ldqb, nullptr, 0, reinterpret_cast<const z64*>(GhQ), ldghq, N, k, k, nullptr, 0, C2, k,
                            f2, nullptr, zmake(1.0, 0.0), 1, stream, nullptr, GATE_ALWAYS));
    return FB_OK;
}

}  // extern "C"
