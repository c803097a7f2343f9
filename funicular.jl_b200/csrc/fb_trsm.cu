// rdiv_upper! (src/kernels.jl:90-124) for k > 64 and rightmul_gemm!
// (src/kernels.jl:57-88): dst <- A C. (k <= 64 goes to the tensor-core
// solvers in fb_trsm_dmma.cu.)
//
// Both are row-independent, so a thread owns a row. For k <= 64 the row lives
// in registers for the whole solve, and the substitution runs right-looking:
// once column j of the result is known it is subtracted from every later
// column, which gives the FP64 pipe long runs of independent fused
// multiply-adds. R sits in shared memory and every thread of a warp reads the
// same entry at the same time, so each read is one broadcast. Loads and
// stores of a row are one column at a time across the warp: 32 consecutive
// rows of a column-major block, 512 contiguous bytes per warp instruction.
// The grid is persistent (a few CTAs per SM) so R is staged once per CTA.
#include "fb_common.cuh"

namespace fb {

__device__ __forceinline__ z64 zrecip(z64 d) {
    double s = 1.0 / fma(d.x, d.x, d.y * d.y);
    return zmake(d.x * s, -d.y * s);
}

// The solve goes 16 columns at a time. For block b a thread first takes the
// finished columns 0..16b-1 of its own row off the block (left-looking: the
// row is read back, these are values this thread has just written), then
// solves the block's own 16 x 16 triangle right-looking. Sixteen columns of
// state keep the thread near 100 registers, so a warp scheduler has several
// warps to choose from while one waits on memory.
constexpr int TB = 16;

template <int J>
__device__ __forceinline__ void solve_block(z64 (&y)[TB], const z64* Rb, int ld, const z64* dinv) {
    if constexpr (J < TB) {
        z64 q = zmul(y[J], dinv[J]);
        y[J] = q;
#pragma unroll
        for (int l = J + 1; l < TB; ++l) zmsub(y[l], q, Rb[J * ld + l]);
        solve_block<J + 1>(y, Rb, ld, dinv);
    }
}

// R is staged row-major in shared memory (ld = kp, k rounded up to 16, zero
// outside the upper triangle and past k; the reciprocal diagonal apart).
__global__ void __launch_bounds__(128)
trsm_rows_kernel(z64* __restrict__ Y, int64_t ldy, int64_t rows, int k,
                 const z64* __restrict__ R, int64_t ldr, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kp = (k + TB - 1) / TB * TB;
    z64* Rs = reinterpret_cast<z64*>(smem_raw);
    z64* dinv = Rs + (size_t)kp * kp;
    for (int e = threadIdx.x; e < kp * kp; e += blockDim.x) {
        int j = e / kp, l = e - j * kp;
        z64 v = zmake(0.0, 0.0);
        if (j < k && l < k && j < l) v = R[j + (int64_t)l * ldr];
        Rs[e] = v;
    }
    for (int j = threadIdx.x; j < kp; j += blockDim.x)
        dinv[j] = (j < k) ? zrecip(R[j + (int64_t)j * ldr]) : zmake(0.0, 0.0);
    __syncthreads();

    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += stride) {
        z64* row = Y + r;
        for (int b0 = 0; b0 < kp; b0 += TB) {
            z64 y[TB];
#pragma unroll
            for (int c = 0; c < TB; ++c) y[c] = (b0 + c < k) ? row[(int64_t)(b0 + c) * ldy] : zmake(0.0, 0.0);
#pragma unroll 2
            for (int i = 0; i < b0; ++i) {
                const z64 q = row[(int64_t)i * ldy];
                const z64* Ri = Rs + i * kp + b0;
#pragma unroll
                for (int c = 0; c < TB; ++c) zmsub(y[c], q, Ri[c]);
            }
            solve_block<0>(y, Rs + b0 * kp + b0, kp, dinv + b0);
#pragma unroll
            for (int c = 0; c < TB; ++c)
                if (b0 + c < k) row[(int64_t)(b0 + c) * ldy] = y[c];
        }
    }
}

int trsm_dmma_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                      size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate);
size_t trsm_workspace_bytes(int k);

int trsm_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                 size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate) {
    if (rows == 0 || k == 0) return FB_OK;
    if (k <= 64) return trsm_dmma_enqueue(Y, ldy, rows, k, R, ldr, workspace, workspace_bytes, stream, st, gate);
    const int threads = 128;
    const int kp = (k + TB - 1) / TB * TB;
    size_t smem = ((size_t)kp * kp + kp) * sizeof(z64);
    if (smem > 227 * 1024) {
        set_error(FB_ENOTSUP, "rdiv_upper!: k = %d is past the %d columns whose factor fits in shared memory", k, 112);
        return FB_ENOTSUP;
    }
    FB_CUDA(cudaFuncSetAttribute(trsm_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(trsm_rows_kernel)");
    int per_sm = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsm_rows_kernel, threads, smem),
            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    int64_t need = (rows + threads - 1) / threads;
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    trsm_rows_kernel<<<(unsigned)grid, threads, smem, stream>>>(Y, ldy, rows, k, R, ldr, st, gate);
    FB_LAUNCHED("trsm_rows_kernel");
    return FB_OK;
}

// dst <- A C. A thread owns a row and produces its outputs 16 columns at a
// time: a loop over the s columns of A (read from the row) accumulates
// the block against row i of C, staged in shared memory.
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
