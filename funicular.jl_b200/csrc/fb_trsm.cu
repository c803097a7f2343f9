// rdiv_upper! (src/kernels.jl:90-124) for k > 64 and rightmul_gemm!
// (src/kernels.jl:57-88): dst <- A C. (k <= 64 goes to the tensor-core
// solvers in fb_trsm_dmma.cu.)
//
// Past 64 columns the solve goes by 64-column blocks: for block b,
//     Y_b <- Y_b - sum_{c<b} X_c R_cb    (the tensor-core right product of
//                                         fb_rmul.cuh, one launch per c),
//     X_b  = Y_b R_bb^-1                 (the k <= 64 solver),
// so every flop still runs on the FP64 tensor cores. A prep kernel lays out
// -R_cb as MMA fragments for every pair c < b; each diagonal block gets the
// k <= 64 solver's own plan and fragments, so its path (one product by the
// inverse, blocked, or substitution) is chosen for that block alone.
#include "fb_common.cuh"
#include "fb_rmul.cuh"

namespace fb {

constexpr int TB_COLS = 64;  // columns of a block of the blocked solve

int trsm_dmma_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                      size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate);
size_t trsm_workspace_bytes_small(int k);

static int trsm_blocks(int k) { return (k + TB_COLS - 1) / TB_COLS; }
static size_t trsm_diag_bytes() { return align_up(trsm_workspace_bytes_small(TB_COLS), 256); }
static size_t trsm_pair_bytes() { return align_up((size_t)dense_frag_doubles(TB_COLS / 4, TB_COLS / 4) * sizeof(double), 256); }

size_t trsm_workspace_bytes(int k) {
    if (k <= TB_COLS) return trsm_workspace_bytes_small(k);
    const size_t nb = trsm_blocks(k);
    return nb * trsm_diag_bytes() + nb * (nb - 1) / 2 * trsm_pair_bytes();
}

// Block p = b (b - 1) / 2 + c of the grid lays out -R_cb (64 x width of b).
__global__ void __launch_bounds__(256)
trsm_pairs_prep_kernel(const z64* __restrict__ R, int64_t ldr, int k, double* frags, size_t pair_doubles,
                       const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    const int p = blockIdx.x;
    int b = 1;
    while ((b + 1) * b / 2 <= p) ++b;
    const int c = p - b * (b - 1) / 2;
    const int width = (k - TB_COLS * b) < TB_COLS ? k - TB_COLS * b : TB_COLS;
    build_dense_frags(frags + p * pair_doubles, R + (int64_t)TB_COLS * c + (int64_t)TB_COLS * b * ldr, ldr, TB_COLS,
                      width, -1.0);
}

int trsm_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                 size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate) {
    if (rows == 0 || k == 0) return FB_OK;
    if (k <= TB_COLS) return trsm_dmma_enqueue(Y, ldy, rows, k, R, ldr, workspace, workspace_bytes, stream, st, gate);
    if (!workspace || workspace_bytes < trsm_workspace_bytes(k)) {
        set_error(FB_ENOMEM, "rdiv_upper!: workspace of %zu bytes, need %zu", workspace_bytes, trsm_workspace_bytes(k));
        return FB_ENOMEM;
    }
    const int nb = trsm_blocks(k);
    char* ws = static_cast<char*>(workspace);
    double* pairs = reinterpret_cast<double*>(ws + (size_t)nb * trsm_diag_bytes());
    const size_t pair_doubles = trsm_pair_bytes() / sizeof(double);
    trsm_pairs_prep_kernel<<<nb * (nb - 1) / 2, 256, 0, stream>>>(R, ldr, k, pairs, pair_doubles, st, gate);
    FB_LAUNCHED("trsm_pairs_prep_kernel");
    for (int b = 0; b < nb; ++b) {
        const int width = k - TB_COLS * b < TB_COLS ? k - TB_COLS * b : TB_COLS;
        z64* Yb = Y + (int64_t)TB_COLS * b * ldy;
        for (int c = 0; c < b; ++c) {
            const double* frag = pairs + (size_t)(b * (b - 1) / 2 + c) * pair_doubles;
            FB_TRY(rmul_enqueue(Yb, ldy, nullptr, 0, Y + (int64_t)TB_COLS * c * ldy, ldy, rows, TB_COLS, width,
                                nullptr, 0, nullptr, 0, frag, nullptr, zmake(1.0, 0.0), 1, stream, st, gate));
        }
        FB_TRY(trsm_dmma_enqueue(Yb, ldy, rows, width, R + (int64_t)TB_COLS * b * (1 + ldr), ldr,
                                 ws + (size_t)b * trsm_diag_bytes(), trsm_diag_bytes(), stream, st, gate));
    }
    return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_ztrsm_workspace_size(int k, size_t* bytes) {
    if (!bytes || k < 0) { set_error(FB_EINVAL, "fb_ztrsm_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = trsm_workspace_bytes(k);
    return FB_OK;
}

int fb_ztrsm_right_upper(fb_z128* Y, int64_t ldy, int64_t rows, int k,
                         const fb_z128* R, int64_t ldr, void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (rows < 0 || k < 0) {
        set_error(FB_EDIM, "a %lld x %d block cannot be divided by a triangular factor", (long long)rows, k);
        return FB_EDIM;
    }
    if (rows == 0 || k == 0) return FB_OK;
    if (!Y || !R) { set_error(FB_EINVAL, "fb_ztrsm_right_upper: NULL matrix"); return FB_EINVAL; }
    if (ldy < rows || ldr < k) {
        set_error(FB_EDIM, "fb_ztrsm_right_upper: leading dimension too small (ldy=%lld for %lld rows, ldr=%lld for k=%d)",
                  (long long)ldy, (long long)rows, (long long)ldr, k);
        return FB_EDIM;
    }
    if (((uintptr_t)Y | (uintptr_t)R) & 15) {
        set_error(FB_EINVAL, "fb_ztrsm_right_upper: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    return trsm_enqueue(reinterpret_cast<z64*>(Y), ldy, rows, k, reinterpret_cast<const z64*>(R), ldr,
                        workspace, workspace_bytes, stream_of(queue), nullptr, GATE_ALWAYS);
}

int fb_zgemm_right(fb_z128* dst, int64_t ldd, const fb_z128* A, int64_t lda, int64_t rows, int s,
                   const fb_z128* C, int64_t ldc, int r, fb_queue_t queue) {
    if (rows < 0 || s < 0 || r < 0) {
        set_error(FB_EDIM, "cannot multiply a %lld x %d block by a %d x %d factor", (long long)rows, s, s, r);
        return FB_EDIM;
    }
    if (rows == 0 || r == 0) return FB_OK;
    if (!dst || (s > 0 && (!A || !C))) { set_error(FB_EINVAL, "fb_zgemm_right: NULL matrix"); return FB_EINVAL; }
    if (ldd < rows || (s > 0 && (lda < rows || ldc < s))) {
        set_error(FB_EDIM, "fb_zgemm_right: leading dimension too small");
        return FB_EDIM;
    }
    if (((uintptr_t)dst | (uintptr_t)A | (uintptr_t)C) & 15) {
        set_error(FB_EINVAL, "fb_zgemm_right: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    z64* D = reinterpret_cast<z64*>(dst);
    const z64* Az = reinterpret_cast<const z64*>(A);
    const z64* Cz = reinterpret_cast<const z64*>(C);
    cudaStream_t stream = stream_of(queue);
    if (s == 0) {
        FB_CUDA(cudaMemset2DAsync(D, ldd * sizeof(z64), 0, rows * sizeof(z64), r, stream), "cudaMemset2DAsync");
        return FB_OK;
    }
    // On the FP64 tensor cores (the right product of fb_rmul.cu), in blocks of
    // at most 64 x 64 of the factor: output columns 64 at a time, and the s
    // columns of A 64 at a time, each block accumulated onto the output (the
    // first overwrites it, NaN included).
    for (int j0 = 0; j0 < r; j0 += RM_KMAX) {
        const int nb = r - j0 < RM_KMAX ? r - j0 : RM_KMAX;
        for (int i0 = 0; i0 < s; i0 += RM_KMAX) {
            const int kb = s - i0 < RM_KMAX ? s - i0 : RM_KMAX;
            FB_TRY(rmul_matrix_enqueue(D + (int64_t)j0 * ldd, ldd, Az + (int64_t)i0 * lda, lda, rows, kb, nb,
                                       Cz + i0 + (int64_t)j0 * ldc, ldc, zmake(1.0, 0.0), i0 > 0 ? 1 : 0, stream));
        }
    }
    return FB_OK;
}

}  // extern "C"
