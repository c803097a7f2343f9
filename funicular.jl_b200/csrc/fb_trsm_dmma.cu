// rdiv_upper! (src/kernels.jl:90-124) on the FP64 tensor cores, k <= 64.
//
// Y <- Y R^-1 is solved by column blocks of 8: for block b,
//     X_b = (Y_b - sum_{c<b} X_c R_cb) inv(R_bb),
// so every flop is in 8 x 8 complex products (DMMA m8n8k4 on the real form
// of the complex product), the diagonal blocks entering through their
// inverses. That costs 14 % more flops than substitution and makes the error
// of block b grow with cond(R_bb) instead of staying at a few eps; each CTA
// therefore estimates cond_1(R_bb) of every diagonal block while it builds
// the inverses, and if one exceeds TR_COND_LIMIT the whole CTA solves its rows
// by plain substitution instead (the reference's ztrsm arithmetic).
//
// A warp owns rows for the whole solve (16 in the blocked path: two 8-row
// units sharing every B fragment; 8 in the product by the inverse), so warps
// never wait for one another. The solved blocks of its rows stay in
// registers, already in the MMA A-operand layout; results leave the
// accumulators (C layout) through a small per-warp shared buffer that
// transposes them into that layout.
// Every CTA first expands R into "fragment order" in shared memory: for each
// pair of column blocks (c <= b), the 16 x 16 real matrix of the product
// with -R_cb (c < b) or inv(R_bb) (c = b), laid out so that each lane's MMA B
// operand is one consecutive 8-byte load.
#include "fb_factor.cuh"
#include "fb_tma.cuh"

namespace fb {

constexpr int TR_THREADS = 256;

// Substitution for rows in [first, rows) step `stride`: the fallback.
__device__ void trsm_substitute_rows(z64* __restrict__ Y, int64_t ldy, int64_t rows, int k,
                                     const z64* __restrict__ R, int64_t ldr, int64_t first, int64_t stride) {
    for (int64_t r = first; r < rows; r += stride) {
        z64* row = Y + r;
        for (int j = 0; j < k; ++j) {
            z64 acc = row[(int64_t)j * ldy];
            for (int i = 0; i < j; ++i) zmsub(acc, row[(int64_t)i * ldy], __ldg(R + i + (int64_t)j * ldr));
            row[(int64_t)j * ldy] = zmul(acc, zrecip_d(__ldg(R + j + (int64_t)j * ldr)));
        }
    }
}

// One CTA: inv(R) in shared memory, the condition numbers, the choice of
// path, and the chosen path's B fragments in the workspace.
//   inverse:    cond_1(R) <= TR_INV_COND_LIMIT: Y inv(R) as one product
//               (fragments of inv(R), n-tile t holding k-steps 0..2t+1);
//   blocked:    otherwise, if every diagonal 8 x 8 block has cond_1 up to
//               TR_COND_LIMIT (fragments of -R_cb and inv(R_bb));
//   substitute: otherwise, plain substitution (no fragments).
// inv(R) is computed by rows from the bottom, every column of a row at once,
// four threads to a column sharing the dot product.
__global__ void __launch_bounds__(256, 1)
trsm_prep_kernel(const z64* __restrict__ R, int64_t ldr, int k, TrsmPlan* plan, double* __restrict__ frag,
                 const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    constexpr int LD = TR_PREP_LD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    z64* Rs = reinterpret_cast<z64*>(smem_raw);   // KP x KP, padded with the identity
    z64* Xs = Rs + TR_KMAX * LD;                   // inv(R)
    const int tid = threadIdx.x;
    const int KP = (k + TR_NB - 1) / TR_NB * TR_NB;
    for (int e = tid; e < KP * KP; e += blockDim.x) {
        const int i = e / KP, j = e - i * KP;
        z64 v = zmake(i == j ? 1.0 : 0.0, 0.0);
        if (i < k && j < k && i <= j) v = R[i + (int64_t)j * ldr];
        Rs[i * LD + j] = v;
        Xs[i * LD + j] = zmake(0.0, 0.0);
    }
    __syncthreads();
    solve_plan(Rs, Xs, k, plan, frag);
}

// Plain substitution, a thread per row (the reference's ztrsm arithmetic),
// for a factor whose diagonal blocks are too ill-conditioned to invert.
__global__ void __launch_bounds__(256)
trsm_subst_kernel(z64* __restrict__ Y, int64_t ldy, int64_t rows, int k, const z64* __restrict__ R, int64_t ldr,
                  const TrsmPlan* plan, const ChainStatus* st, int gate) {
    if (gated_off(st, gate) || plan->path != PATH_SUBSTITUTE) return;
    trsm_substitute_rows(Y, ldy, rows, k, R, ldr, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                         (int64_t)gridDim.x * blockDim.x);
}

__device__ __forceinline__ void copy_frags(double* dst, const double* __restrict__ src, int n) {
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    for (int e = threadIdx.x; e < n / 2; e += blockDim.x) d2[e] = s2[e];
    __syncthreads();
}

// Y R^-1 as one product by inv(R) (path inverse): a warp owns 8 rows, loads
// them once in the MMA A layout and writes each 4-column n-tile of the result
// straight from the accumulators; n-tile t needs k-steps 0..2t+1 only.
template <int NT>
__global__ void __launch_bounds__(TR_THREADS, 2)
trsm_inv_kernel(z64* __restrict__ Y, int64_t ldy, int64_t rows, int k, const TrsmPlan* plan,
                const double* __restrict__ gfrag, const ChainStatus* st, int gate, int zero) {
    if (gated_off(st, gate) || plan->path != PATH_INVERSE) return;
    constexpr int KP = 4 * NT;
    constexpr int NS = KP / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* frag = reinterpret_cast<double*>(smem_raw);
    copy_frags(frag, gfrag, 32 * NT * (NT + 1));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cq = lane & 3, acol = cq >> 1, apart = lane & 1, rr = lane >> 2;
    const int64_t units = (rows + 7) / 8;
    const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; u < units; u += warps_total) {
        const int64_t row = u * 8 + rr;
        const bool live = row < rows;
        z64* yrow = Y + (live ? row : 0);
        double a[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int col = 2 * s + acol;
            a[s] = (live && col < k) ? reinterpret_cast<const double*>(yrow + (int64_t)col * ldy)[apart] : 0.0;
        }
        // The loads of n-tile t wait for the result of n-tile t - 2 and,
        // inside a tile, each group of eight for the group before: two tiles
        // in flight, and no more fragments in registers than that needs.
        double chain = 0.0, done1 = 0.0, done2 = 0.0;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            double acc[2][2] = {};
            const double* fp = frag + 32 * t * (t + 1) + lane;
            chain = done2;
#pragma unroll
            for (int s = 0; s <= 2 * t + 1; ++s) {
                if ((s & 7) == 0) fp = hold(fp, chain, zero);
                const double bv = fp[s * 32];
                if ((s & 7) == 0) chain = bv;
                dmma_884(acc[s & 1][0], acc[s & 1][1], a[s], bv);
            }
            const int col = 4 * t + cq;
            const z64 x = zmake(acc[0][0] + acc[1][0], acc[0][1] + acc[1][1]);
            if (live && col < k) yrow[(int64_t)col * ldy] = x;
            done2 = done1;
            done1 = x.x;
        }
    }
}

// The blocked solve (path blocked) with two adjacent 8-row units a warp (16
// rows): every B fragment read from shared memory feeds one MMA of each unit,
// which halves the fragment traffic per MMA against one unit a warp (whose
// shared pipe and tensor pipe both ran near their limits: 6.91 ms against
// 6.40 ms at N = 1e7, k = 64), and each warp carries the independent MMA
// chains of two units. The solved blocks of both units stay in registers (64
// doubles a lane at k = 64), so a CTA of eight warps runs alone on an SM.
constexpr int TR2_THREADS = 256;

template <int NBLK>
__global__ void __launch_bounds__(TR2_THREADS, 1)
trsm_dmma2_kernel(z64* __restrict__ Y, int64_t ldy, int64_t rows, int k, const TrsmPlan* plan,
                  const double* __restrict__ gfrag, const ChainStatus* st, int gate) {
    if (gated_off(st, gate) || plan->path != PATH_BLOCKED) return;
    constexpr int NPAIRS = NBLK * (NBLK + 1) / 2;
    constexpr int NCH = 4;                   // accumulator chains per unit and n-tile
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* frag = reinterpret_cast<double*>(smem_raw);
    z64* tbuf = reinterpret_cast<z64*>(frag + NPAIRS * TR_FRAG);
    copy_frags(frag, gfrag, NPAIRS * TR_FRAG);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    z64* bufs[2] = {tbuf + (2 * warp) * TR_BUF, tbuf + (2 * warp + 1) * TR_BUF};
    const int rr = lane >> 2;            // row of the 8 this lane's fragments belong to
    const int cq = lane & 3;             // C layout: complex column within a 4-column n-tile
    const int acol = cq >> 1;            // A layout: which of the k-step's two columns
    const int apart = lane & 1;          // A layout: re or im
    const int64_t units = (rows + 7) / 8;
    const int64_t pairs = (units + 1) / 2;
    const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);

    // Y of (unit, block) in the C layout, zero past the matrix.
    auto load_y = [&](int64_t unit, int b, z64 (&v)[2]) {
        const int64_t row = unit * 8 + rr;
        const bool ok_row = unit < units && row < rows;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int col = TR_NB * b + 4 * t + cq;
            v[t] = (ok_row && col < k) ? Y[row + (int64_t)col * ldy] : zmake(0.0, 0.0);
        }
    };
    // Pair p holds units 2p and 2p + 1. The Y blocks of the next two steps
    // are always in flight for both units (a step is one column block of the
    // pair, and the prefetch runs on into the warp's next pairs). Block b is
    // read from slot b & 1; with an odd block count the prefetch leaves the
    // next pair's blocks 0 and 1 in slots 1 and 0, so the slots are swapped at
    // the end of each pair.
    int64_t pr = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    z64 yq[2][2][2];   // [slot][unit][n-tile]
#pragma unroll
    for (int v = 0; v < 2; ++v) {
        load_y(2 * pr + v, 0, yq[0][v]);
        load_y(2 * (pr + (1 / NBLK) * warps_total) + v, 1 % NBLK, yq[1][v]);
    }
    for (; pr < pairs; pr += warps_total) {
        double xa[NBLK][2][4];
#pragma unroll
        for (int b = 0; b < NBLK; ++b) {
            double acc[2][NCH][2][2];
            const int slot = b & 1;
#pragma unroll
            for (int v = 0; v < 2; ++v)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    acc[v][0][t][0] = yq[slot][v][t].x;
                    acc[v][0][t][1] = yq[slot][v][t].y;
#pragma unroll
                    for (int h = 1; h < NCH; ++h) acc[v][h][t][0] = acc[v][h][t][1] = 0.0;
                }
#pragma unroll
            for (int v = 0; v < 2; ++v)
                load_y(2 * (pr + ((b + 2) / NBLK) * warps_total) + v, (b + 2) % NBLK, yq[slot][v]);
            // Y_b - sum_{c<b} X_c R_cb, each fragment serving both units.
#pragma unroll
            for (int c = 0; c < b; ++c) {
                const double* fp = frag + pair_index(c, b) * TR_FRAG + lane;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int h = (c * 4 + s) % NCH;
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const double bv = fp[(s * 2 + t) * 32];
                        dmma_884(acc[0][h][t][0], acc[0][h][t][1], xa[c][0][s], bv);
                        dmma_884(acc[1][h][t][0], acc[1][h][t][1], xa[c][1][s], bv);
                    }
                }
            }
            // Transpose T_b from the C layout into the A layout.
#pragma unroll
            for (int v = 0; v < 2; ++v)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    double re = acc[v][0][t][0], im = acc[v][0][t][1];
#pragma unroll
                    for (int h = 1; h < NCH; ++h) {
                        re += acc[v][h][t][0];
                        im += acc[v][h][t][1];
                    }
                    bufs[v][tbuf_index(rr, 4 * t + cq)] = zmake(re, im);
                }
            __syncwarp();
            double ta[2][4];
#pragma unroll
            for (int v = 0; v < 2; ++v)
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    ta[v][s] = reinterpret_cast<const double*>(&bufs[v][tbuf_index(rr, 2 * s + acol)])[apart];
            __syncwarp();
            // X_b = T_b inv(R_bb), inv(R_bb) upper triangular (k-steps 2, 3
            // skip n-tile 0).
            double xb[2][2][2][2] = {};
            const double* fd = frag + pair_index(b, b) * TR_FRAG + lane;
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int t = 0; t < 2; ++t)
                    if (2 * s <= 4 * t + 3) {
                        const double bv = fd[(s * 2 + t) * 32];
                        dmma_884(xb[0][s & 1][t][0], xb[0][s & 1][t][1], ta[0][s], bv);
                        dmma_884(xb[1][s & 1][t][0], xb[1][s & 1][t][1], ta[1][s], bv);
                    }
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const int64_t row = (2 * pr + v) * 8 + rr;
                const bool live = row < rows;
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const z64 x = zmake(xb[v][0][t][0] + xb[v][1][t][0], xb[v][0][t][1] + xb[v][1][t][1]);
                    const int col = TR_NB * b + 4 * t + cq;
                    if (live && col < k) Y[row + (int64_t)col * ldy] = x;
                    if (b + 1 < NBLK) bufs[v][tbuf_index(rr, 4 * t + cq)] = x;
                }
            }
            if (b + 1 < NBLK) {
                __syncwarp();
#pragma unroll
                for (int v = 0; v < 2; ++v)
#pragma unroll
                    for (int s = 0; s < 4; ++s)
                        xa[b][v][s] = reinterpret_cast<const double*>(&bufs[v][tbuf_index(rr, 2 * s + acol)])[apart];
                __syncwarp();
            }
        }
        if (NBLK & 1) {
#pragma unroll
            for (int v = 0; v < 2; ++v)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const z64 tmp = yq[0][v][t];
                    yq[0][v][t] = yq[1][v][t];
                    yq[1][v][t] = tmp;
                }
        }
    }
}

template <int NBLK>
static int launch_trsm_dmma2(z64* Y, int64_t ldy, int64_t rows, int k, const TrsmPlan* plan, const double* frag,
                             cudaStream_t stream, const ChainStatus* st, int gate) {
    constexpr int NPAIRS = NBLK * (NBLK + 1) / 2;
    const size_t smem = (size_t)NPAIRS * TR_FRAG * sizeof(double) + (TR2_THREADS / 32) * 2 * TR_BUF * sizeof(z64);
    FB_CUDA(cudaFuncSetAttribute(trsm_dmma2_kernel<NBLK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(trsm_dmma2_kernel)");
    int per_sm = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsm_dmma2_kernel<NBLK>, TR2_THREADS, smem),
            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    const int64_t pairs = ((rows + 7) / 8 + 1) / 2;
    int64_t need = (pairs + TR2_THREADS / 32 - 1) / (TR2_THREADS / 32);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    trsm_dmma2_kernel<NBLK><<<(unsigned)grid, TR2_THREADS, smem, stream>>>(Y, ldy, rows, k, plan, frag, st, gate);
    FB_LAUNCHED("trsm_dmma2_kernel");
    return FB_OK;
}

template <int NT>
static int launch_trsm_inv(z64* Y, int64_t ldy, int64_t rows, int k, const TrsmPlan* plan, const double* frag,
                           cudaStream_t stream, const ChainStatus* st, int gate) {
    const size_t smem = (size_t)32 * NT * (NT + 1) * sizeof(double);
    FB_CUDA(cudaFuncSetAttribute(trsm_inv_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(trsm_inv_kernel)");
    int per_sm = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsm_inv_kernel<NT>, TR_THREADS, smem),
            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    const int64_t units = (rows + 7) / 8;
    int64_t need = (units + TR_THREADS / 32 - 1) / (TR_THREADS / 32);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    trsm_inv_kernel<NT><<<(unsigned)grid, TR_THREADS, smem, stream>>>(Y, ldy, rows, k, plan, frag, st, gate, 0);
    FB_LAUNCHED("trsm_inv_kernel");
    return FB_OK;
}


size_t trsm_workspace_bytes_small(int k) {
    return k <= TR_KMAX ? (size_t)TR_PLAN_BYTES + (size_t)TR_FRAG_DOUBLES * sizeof(double) : 0;
}

// Prep, then all three solvers; the plan the prep writes lets exactly one of
// them work, so the choice of path costs no host round trip.
int trsm_dmma_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                      size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate) {
    if (k > TR_KMAX) { set_error(FB_ENOTSUP, "trsm_dmma: k = %d is past %d", k, TR_KMAX); return FB_ENOTSUP; }
    if (!workspace || workspace_bytes < trsm_workspace_bytes_small(k)) {
        set_error(FB_ENOMEM, "rdiv_upper!: workspace of %zu bytes, need %zu", workspace_bytes,
                  trsm_workspace_bytes_small(k));
        return FB_ENOMEM;
    }
    TrsmPlan* plan = static_cast<TrsmPlan*>(workspace);
    double* frag = reinterpret_cast<double*>(static_cast<char*>(workspace) + TR_PLAN_BYTES);
    const size_t prep_smem = (size_t)2 * TR_KMAX * (TR_KMAX + 1) * sizeof(z64);
    FB_CUDA(cudaFuncSetAttribute(trsm_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)prep_smem),
            "cudaFuncSetAttribute(trsm_prep_kernel)");
    trsm_prep_kernel<<<1, 256, prep_smem, stream>>>(R, ldr, k, plan, frag, st, gate);
    FB_LAUNCHED("trsm_prep_kernel");
    int status = FB_OK;
    switch ((k + 3) / 4) {
#define FB_INV_CASE(n) case n: status = launch_trsm_inv<n>(Y, ldy, rows, k, plan, frag, stream, st, gate); break;
        FB_INV_CASE(1) FB_INV_CASE(2) FB_INV_CASE(3) FB_INV_CASE(4) FB_INV_CASE(5) FB_INV_CASE(6)
        FB_INV_CASE(7) FB_INV_CASE(8) FB_INV_CASE(9) FB_INV_CASE(10) FB_INV_CASE(11) FB_INV_CASE(12)
        FB_INV_CASE(13) FB_INV_CASE(14) FB_INV_CASE(15) FB_INV_CASE(16)
#undef FB_INV_CASE
    }
    FB_TRY(status);
    switch ((k + TR_NB - 1) / TR_NB) {
#define FB_BLK_CASE(n) case n: status = launch_trsm_dmma2<n>(Y, ldy, rows, k, plan, frag, stream, st, gate); break;
        FB_BLK_CASE(1) FB_BLK_CASE(2) FB_BLK_CASE(3) FB_BLK_CASE(4)
        FB_BLK_CASE(5) FB_BLK_CASE(6) FB_BLK_CASE(7) FB_BLK_CASE(8)
#undef FB_BLK_CASE
    }
    FB_TRY(status);
    int64_t grid = (int64_t)sm_count() * 4;
    int64_t need = (rows + 255) / 256;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    trsm_subst_kernel<<<(unsigned)grid, 256, 0, stream>>>(Y, ldy, rows, k, R, ldr, plan, st, gate);
    FB_LAUNCHED("trsm_subst_kernel");
    return FB_OK;
}

}  // namespace fb
