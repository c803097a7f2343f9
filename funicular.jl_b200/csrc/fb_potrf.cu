// cholesky_upper (src/panelblas.jl:148-155) as one CTA on the device: the
// k x k Cholesky of a Hermitian Gram matrix, the shifted retry, and the
// R2 * R product of cholqr2! (src/panelblas.jl:133,136), all FP64.
//
// The factorization is right-looking on the upper triangle, held in shared
// memory when it fits (k <= 112) and in workspace memory otherwise. Pivot
// test as LAPACK's zpotrf makes it: the factorization fails as soon as a
// pivot is not > 0 (this also catches NaN). On failure the matrix is reloaded
// with s = 11 N k eps(Float64) ||G||_F added to the diagonal and factored
// again; a second failure is reported, not shifted further.
//
// The shifted CholeskyQR3 of Fukaya, Kannan, Nakatsukasa, Zhang and Yamamoto
// (SIAM J. Sci. Comput. 2020) shifts its first pass unconditionally: with a
// unit roundoff u > 0 the kernel factors G + s I once, s = 11 (N k + k (k+1))
// u ||G||_F (||G||_F bounds ||Y||_2^2 from above, which keeps s inside the
// range the analysis allows for the condition numbers it targets).
#include "fb_factor.cuh"

namespace fb {

constexpr int POTRF_THREADS = 512;
constexpr int POTRF_SMEM_MAX_K = 112;

__global__ void __launch_bounds__(POTRF_THREADS, 1)
potrf_kernel(const z64* __restrict__ G, int64_t ldg, int k, int64_t N,
             z64* __restrict__ U, int64_t ldu, const z64* __restrict__ Rin, int64_t ldrin,
             z64* __restrict__ Rout, int64_t ldrout, z64* __restrict__ gwork,
             ChainStatus* st, int pass, int gate, double forced_u) {
    if (gated_off(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_scratch[33];
    const bool in_smem = k <= POTRF_SMEM_MAX_K;
    z64* W = in_smem ? reinterpret_cast<z64*>(smem_raw) : gwork;  // row-major k x k, upper part used
    const int tid = threadIdx.x, nt = blockDim.x;
    const int kk = k * k;
    auto g = [&](int i, int j) { return G[i + (int64_t)j * ldg]; };
    const double gnorm = hermitian_fro(g, k, red_scratch);
    bool shifted = false;
    double shift = 0.0;
    const bool ok = factor_shifted(g, k, N, gnorm, forced_u, W, shifted, shift);

    if (tid == 0 && st) {
        st->shifted[pass] = shifted ? 1 : 0;
        st->shift[pass] = shift;
        st->norm[pass] = gnorm;
        if (!ok) st->failed = pass;
    }
    if (!ok) return;

    for (int e = tid; e < kk; e += nt) {
        int j = e / k, i = e - j * k;  // column-major walk of U: coalesced stores
        U[i + (int64_t)j * ldu] = (i <= j) ? W[i * k + j] : zmake(0.0, 0.0);
    }
    if (Rout) {
        for (int e = tid; e < kk; e += nt) {
            int j = e / k, i = e - j * k;
            z64 acc = zmake(0.0, 0.0);
            if (i <= j) {
                if (Rin) {
                    for (int m = i; m <= j; ++m) zmac(acc, W[i * k + m], Rin[m + (int64_t)j * ldrin]);
                } else {
                    acc = W[i * k + j];
                }
            }
            Rout[i + (int64_t)j * ldrout] = acc;
        }
    }
}

size_t potrf_gwork_bytes(int k) { return k > POTRF_SMEM_MAX_K ? (size_t)k * k * sizeof(z64) : 0; }

int potrf_enqueue(const z64* G, int64_t ldg, int k, int64_t N, z64* U, int64_t ldu,
                  const z64* Rin, int64_t ldrin, z64* Rout, int64_t ldrout, z64* gwork,
                  ChainStatus* st, int pass, int gate, cudaStream_t stream, double forced_u) {
    size_t smem = k <= POTRF_SMEM_MAX_K ? (size_t)k * k * sizeof(z64) : 0;
    if (smem > 0) {
        FB_CUDA(cudaFuncSetAttribute(potrf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(potrf_kernel)");
    }
    potrf_kernel<<<1, POTRF_THREADS, smem, stream>>>(G, ldg, k, N, U, ldu, Rin, ldrin, Rout, ldrout, gwork, st,
                                                     pass, gate, forced_u);
    FB_LAUNCHED("potrf_kernel");
    return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zpotrf_workspace_size(int k, size_t* bytes) {
    if (!bytes || k < 0) { set_error(FB_EINVAL, "fb_zpotrf_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = align_up(sizeof(ChainStatus), 256) + align_up(potrf_gwork_bytes(k), 256);
    return FB_OK;
}

static int potrf_call(fb_z128* U, int64_t ldu, const fb_z128* G, int64_t ldg, int k, int64_t N,
                      const fb_z128* Rin, int64_t ldrin, fb_z128* Rout, int64_t ldrout,
                      int* shifted, double* shift, void* workspace, size_t workspace_bytes, fb_queue_t queue,
                      double forced_u) {
    if (k < 0 || N < 0) { set_error(FB_EINVAL, "fb_zpotrf_shifted: negative size"); return FB_EINVAL; }
    if (k == 0) {
        if (shifted) *shifted = 0;
        if (shift) *shift = 0.0;
        return FB_OK;
    }
    if (!U || !G || (Rin && !Rout)) { set_error(FB_EINVAL, "fb_zpotrf_shifted: NULL matrix"); return FB_EINVAL; }
    if (ldu < k || ldg < k || (Rin && ldrin < k) || (Rout && ldrout < k)) {
        set_error(FB_EDIM, "fb_zpotrf_shifted: leading dimension smaller than k=%d", k);
        return FB_EDIM;
    }
    if (Rin && Rout && Rin == Rout) {
        set_error(FB_EINVAL, "fb_zpotrf_shifted: Rout must not alias Rin");
        return FB_EINVAL;
    }
    size_t need = 0;
    fb_zpotrf_workspace_size(k, &need);
    if (!workspace || workspace_bytes < need) {
        set_error(FB_ENOMEM, "fb_zpotrf_shifted: workspace of %zu bytes, need %zu", workspace_bytes, need);
        return FB_ENOMEM;
    }
    cudaStream_t stream = stream_of(queue);
    ChainStatus* st = static_cast<ChainStatus*>(workspace);
    z64* gwork = reinterpret_cast<z64*>(static_cast<char*>(workspace) + align_up(sizeof(ChainStatus), 256));
    FB_CUDA(cudaMemsetAsync(st, 0, sizeof(ChainStatus), stream), "cudaMemsetAsync");
    FB_TRY(potrf_enqueue(reinterpret_cast<const z64*>(G), ldg, k, N, reinterpret_cast<z64*>(U), ldu,
                         reinterpret_cast<const z64*>(Rin), ldrin, reinterpret_cast<z64*>(Rout), ldrout, gwork, st,
                         1, GATE_ALWAYS, stream, forced_u));
    ChainStatus host{};
    FB_CUDA(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
    FB_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    if (shifted) *shifted = host.shifted[1];
    if (shift) *shift = host.shift[1];
    if (host.failed) {
        set_error(FB_ENOTSPD,
                  "the %dx%d Gram matrix is not positive definite even after a shift of %.17g, so the columns are "
                  "numerically dependent: a zero column, a duplicated one, or a condition number past 4.5e15. "
                  "Drop the dependent columns before orthonormalizing",
                  k, k, host.shift[1]);
        return FB_ENOTSPD;
    }
    return FB_OK;
}

int fb_zpotrf_shifted(fb_z128* U, int64_t ldu, const fb_z128* G, int64_t ldg, int k, int64_t N,
                      const fb_z128* Rin, int64_t ldrin, fb_z128* Rout, int64_t ldrout,
                      int* shifted, double* shift, void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    return potrf_call(U, ldu, G, ldg, k, N, Rin, ldrin, Rout, ldrout, shifted, shift, workspace, workspace_bytes,
                      queue, 0.0);
}

int fb_zpotrf_forced_shift(fb_z128* U, int64_t ldu, const fb_z128* G, int64_t ldg, int k, int64_t N,
                           const fb_z128* Rin, int64_t ldrin, fb_z128* Rout, int64_t ldrout, double unit_roundoff,
                           double* shift, void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (!(unit_roundoff > 0.0 && unit_roundoff < 1.0)) {
        set_error(FB_EINVAL, "fb_zpotrf_forced_shift: the unit roundoff must lie in (0, 1), got %g", unit_roundoff);
        return FB_EINVAL;
    }
    return potrf_call(U, ldu, G, ldg, k, N, Rin, ldrin, Rout, ldrout, nullptr, shift, workspace, workspace_bytes,
                      queue, unit_roundoff);
}

}  // extern "C"
