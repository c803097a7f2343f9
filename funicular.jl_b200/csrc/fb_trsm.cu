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

// dst <- A C. A thread owns a row and produces its outputs TB columns at a
// time: a loop over the s columns of A (read from the row) accumulates
// the block against row i of C, staged in shared memory.
constexpr int TB = 16;

__global__ void __launch_bounds__(128)
gemm_right_kernel(z64* __restrict__ D, int64_t ldd, const z64* __restrict__ A, int64_t lda,
                  int64_t rows, int s, const z64* __restrict__ C, int64_t ldc, int r) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    z64* Cs = reinterpret_cast<z64*>(smem_raw);  // s x rp, row-major, zero past r
    const int rp = (r + TB - 1) / TB * TB;
    for (int e = threadIdx.x; e < s * rp; e += blockDim.x) {
        int i = e / rp, j = e - i * rp;
        Cs[e] = (j < r) ? C[i + (int64_t)j * ldc] : zmake(0.0, 0.0);
    }
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += stride) {
        const z64* arow = A + row;
        for (int j0 = 0; j0 < rp; j0 += TB) {
            z64 acc[TB];
#pragma unroll
            for (int c = 0; c < TB; ++c) acc[c] = zmake(0.0, 0.0);
#pragma unroll 2
            for (int i = 0; i < s; ++i) {
                const z64 a = arow[(int64_t)i * lda];
                const z64* Ci = Cs + i * rp + j0;
#pragma unroll
                for (int c = 0; c < TB; ++c) zmac(acc[c], a, Ci[c]);
            }
#pragma unroll
            for (int c = 0; c < TB; ++c)
                if (j0 + c < r) D[row + (int64_t)(j0 + c) * ldd] = acc[c];
        }
    }
}

// Factors too large for shared memory: the same loop, C through the
// read-only cache.
__global__ void gemm_right_generic_kernel(z64* __restrict__ D, int64_t ldd, const z64* __restrict__ A, int64_t lda,
                                          int64_t rows, int s, const z64* __restrict__ C, int64_t ldc, int r) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += stride) {
        for (int j = 0; j < r; ++j) {
            z64 acc = zmake(0.0, 0.0);
            for (int i = 0; i < s; ++i) zmac(acc, A[row + (int64_t)i * lda], __ldg(C + i + (int64_t)j * ldc));
            D[row + (int64_t)j * ldd] = acc;
        }
    }
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
    const int threads = 128;
    const int rp = (r + TB - 1) / TB * TB;
    size_t smem = (size_t)s * rp * sizeof(z64);
    int64_t need = (rows + threads - 1) / threads;
    if (smem <= 227 * 1024) {
        FB_CUDA(cudaFuncSetAttribute(gemm_right_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                "cudaFuncSetAttribute(gemm_right_kernel)");
        int per_sm = 0;
        FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gemm_right_kernel, threads, smem),
                "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        if (per_sm < 1) per_sm = 1;
        int64_t grid = (int64_t)sm_count() * per_sm;
        if (grid > need) grid = need;
        gemm_right_kernel<<<(unsigned)grid, threads, smem, stream>>>(D, ldd, Az, lda, rows, s, Cz, ldc, r);
        FB_LAUNCHED("gemm_right_kernel");
        return FB_OK;
    }
    int64_t grid = (int64_t)sm_count() * 8;
    if (grid > need) grid = need;
    gemm_right_generic_kernel<<<(unsigned)grid, threads, 0, stream>>>(D, ldd, Az, lda, rows, s, Cz, ldc, r);
    FB_LAUNCHED("gemm_right_generic_kernel");
    return FB_OK;
}

}  // extern "C"
