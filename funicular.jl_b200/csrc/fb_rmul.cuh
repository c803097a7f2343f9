// Right products of a tall N x K block by a small K x n factor on the FP64
// tensor cores (DMMA m8n8k4 on the real form of the complex product):
//     D <- beta D + A1 L + A2 C,
// with L lower triangular (K = n) and C dense. The factors travel as MMA B
// fragments that a prep kernel builds in device memory and each CTA stages in
// shared memory: for k-step s (two complex rows of the factor) and n-tile t
// (four complex columns), the 32 lanes' entries are consecutive. Used by the
// adjoint pullbacks (fb_adjoint.cu) and by the off-diagonal updates of the
// blocked triangular solve (fb_trsm.cu).
#pragma once

#include "fb_common.cuh"

namespace fb {

constexpr int RM_KMAX = 64;  // widest K and n of the tensor-core product

// B fragments of a dense K x n factor: 2 ntk k-steps x ntn n-tiles x 32 lanes.
__host__ __device__ inline int dense_frag_doubles(int ntk, int ntn) { return 64 * ntk * ntn; }
// Of a lower triangular k x k one: k-step s holds n-tiles 0 .. s/2.
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

// The B fragment entry of `lane` for k-step s and n-tile t of scale * M, M
// K x n column-major with leading dimension ldm, zero past its edges: lane & 3
// is the real k index inside the step, lane >> 2 the real n index inside the
// tile.
__device__ __forceinline__ double frag_entry(const z64* M, int64_t ldm, int K, int n, int s, int t, int lane,
                                             double scale) {
    const int kr = lane & 3, nr = lane >> 2;
    const int i = 2 * s + (kr >> 1), p = kr & 1;
    const int j = 4 * t + (nr >> 1), o = nr & 1;
    return (i < K && j < n) ? scale * real_part_of(M[i + (int64_t)j * ldm], p, o) : 0.0;
}

// Run by every thread of one CTA.
__device__ inline void build_dense_frags(double* frag, const z64* M, int64_t ldm, int K, int n, double scale) {
    const int ntk = (K + 3) / 4, ntn = (n + 3) / 4;
    for (int e = threadIdx.x; e < dense_frag_doubles(ntk, ntn); e += blockDim.x) {
        const int lane = e & 31, q = e >> 5;
        const int s = q / ntn, t = q - s * ntn;
        frag[e] = frag_entry(M, ldm, K, n, s, t, lane, scale);
    }
}

__device__ inline void build_lower_frags(double* frag, const z64* M, int64_t ldm, int k) {
    const int nt = (k + 3) / 4;
    for (int e = threadIdx.x; e < lower_frag_doubles(nt); e += blockDim.x) {
        const int lane = e & 31, q = e >> 5;
        int s = 0;
        while (lower_step_offset(s + 1) <= q) ++s;
        frag[e] = frag_entry(M, ldm, k, k, s, q - lower_step_offset(s), lane, 1.0);
    }
}

// D <- beta D (when use_beta) + A1 L + A2 C for rows x K inputs and a K x n
// output. A1 may be NULL; when it is not, K == n. With K, n <= 64 the product
// runs on the tensor cores from the fragments (fdense of C, flower of L);
// otherwise on the FP64 pipes from L and C themselves (column-major, leading
// dimensions ldl and ldc). D may be the same matrix as A1 (or A2 on the
// tensor-core path); it must not otherwise overlap them.
int rmul_enqueue(z64* D, int64_t ldd, const z64* A1, int64_t lda1, const z64* A2, int64_t lda2, int64_t rows,
                 int K, int n, const z64* L, int64_t ldl, const z64* C, int64_t ldc, const double* fdense,
                 const double* flower, z64 beta, int use_beta, cudaStream_t stream, const ChainStatus* st, int gate);

// D <- beta D (when use_beta) + A C, A rows x K, C a K x n device matrix
// (leading dimension ldc), K and n at most 64, on the tensor cores: each CTA
// lays out C's fragments in shared memory itself. D must not overlap A.
int rmul_matrix_enqueue(z64* D, int64_t ldd, const z64* A, int64_t lda, int64_t rows, int K, int n, const z64* C,
                        int64_t ldc, z64 beta, int use_beta, cudaStream_t stream);

}  // namespace fb
