// The Gram matrix G = Y^H Y (gram_accumulate!, src/kernels.jl:22-55, with
// A === B) on the integer tensor cores: an Ozaki-style split of every FP64
// entry into 8-bit slices whose products are exact in 32-bit integer
// accumulators, recovered to FP64 with power-of-two weights.
//
// Real form. With W the 2N x k real matrix holding Re Y and Im Y in
// alternating rows (exactly the interleaved ComplexF64 layout of a column) and
// JW the same with each (re, im) pair turned into (im, -re):
//   [W JW]^T W = [Re G ; -Im G]      (a 128 x 64 product for k <= 64).
// The MMA operand A is [W_t ; JW_t] (128 rows, slice t), operand B the W
// slices stacked along N, so one MMA of A slice t against B slices 1..7-t
// lands in the accumulators of the groups g = t + u it feeds.
//
// Slices. Column j carries a power-of-two scale 2^E_j with |entries| <=
// 2^(E_j - 1); an entry x becomes the integer x_int = rint(x 2^(55 - E_j)),
// |x_int| <= 2^54, written as seven signed bytes
//   x_int = d_1 2^48 + sum_{t=2..7} d_t 2^(8 (7 - t)),  d_1 in [-64, 64], d_t in [-128, 127]
// (the low bytes of x_int + 0x808080808080, each minus 128). A product of two
// entries is 2^(E_a + E_b - 110) sum_{t,u} d_t e_u 2^(8 (14 - t - u)); the 28
// terms with t + u <= 8 are kept, the rest lie below 2^-51 of the leading
// term. Group g = t + u owns 64 accumulator columns of tensor memory, 448 in
// all.
//
// Scales adapt as the rows stream: a stage whose column maximum exceeds the
// current limit, or one that would let an int32 accumulator overflow (every
// 8192 rows), first drains the accumulators into this CTA's FP64 partial in
// global memory, then rescales. The partials of all CTAs are summed in a
// fixed order by the reduce kernel, so results are deterministic.
//
// Roles (one CTA per SM, 192 threads): warps 0-3 read FP64 tiles from shared
// memory, slice them into the MMA operand layout and drain tensor memory
// (warp w owns lanes 32w..32w+31); warp 4 issues the MMAs; warp 5 keeps a
// ring of TMA tile loads in flight. Every wait is bounded.
#include "fb_umma.cuh"

namespace fb {
namespace ozaki {

constexpr int SLICES = 7;
constexpr int ROWS = 16;                        // complex rows per stage: K = 32 bytes
constexpr int FSTAGES = 4;                      // FP64 ring depth
constexpr int FBYTES = ROWS * 64 * 16;          // 16 KB: 16 rows x 64 columns
constexpr int ATILE = 128 * 32;                 // one A slice tile: 128 rows x 32 bytes
constexpr int BTILE = SLICES * 64 * 32;         // B: 7 x 64 rows x 32 bytes
constexpr int SBYTES = SLICES * ATILE + BTILE;  // one slice buffer, 42 KB
constexpr int SBUFS = 2;
constexpr int TMEM_COLS = 512;
constexpr int EPOCH_STAGES = 8192 / ROWS;       // int32 headroom: 7 x 2^14 x 2 x 8192 < 2^31
constexpr int HEADROOM = 1;                     // spare exponent bits above the stage maximum
constexpr int E_UNSET = -4000;                  // column seen only zeros so far
constexpr int THREADS = 192;
constexpr uint64_t BIAS = 0x0000808080808080ull;

constexpr size_t OFF_F = 0;
constexpr size_t OFF_S = OFF_F + (size_t)FSTAGES * FBYTES;
constexpr size_t OFF_MAX = OFF_S + (size_t)SBUFS * SBYTES;  // double [2][64]
constexpr size_t OFF_BAR = OFF_MAX + 2 * 64 * 8;            // 12 mbarriers
constexpr size_t OFF_MISC = OFF_BAR + 16 * 8;
constexpr size_t MISC_BYTES = 512;                          // flags, TMEM slot, column exponents
constexpr size_t SMEM_BYTES = OFF_MISC + MISC_BYTES + 1024;  // + alignment slack

struct Flags {
    int timeout;
    int nonfinite;
};

__device__ __forceinline__ uint32_t sw32_offset(uint32_t row, uint32_t chunk) {
    return row * 32 + ((chunk ^ ((row >> 2) & 1)) << 4);
}

// 2^e as a double for e in the normal range, 0 below it.
__device__ __forceinline__ double pow2(int e) {
    if (e < -1022) return 0.0;
    if (e > 1023) e = 1023;
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// K-major operand tile with 32-byte rows and the 32-byte swizzle: eight-row
// groups 256 bytes apart, layout type 6 = SWIZZLE_32B.
__device__ __forceinline__ uint64_t desc_sw32(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;           // leading byte offset, unused when swizzled
    d |= (uint64_t)(256 >> 4) << 32;  // stride byte offset: eight 32-byte rows
    d |= (uint64_t)1 << 46;           // version
    d |= (uint64_t)6 << 61;           // SWIZZLE_32B
    return d;
}

// Byte p of each of four 64-bit values, packed low to high.
__device__ __forceinline__ uint32_t gather_byte(const uint64_t (&y)[4], int p) {
    const int half = p >> 2, b = p & 3;
    const uint32_t w0 = half ? (uint32_t)(y[0] >> 32) : (uint32_t)y[0];
    const uint32_t w1 = half ? (uint32_t)(y[1] >> 32) : (uint32_t)y[1];
    const uint32_t w2 = half ? (uint32_t)(y[2] >> 32) : (uint32_t)y[2];
    const uint32_t w3 = half ? (uint32_t)(y[3] >> 32) : (uint32_t)y[3];
    const uint32_t sel = (uint32_t)b | ((uint32_t)(b + 4) << 4);
    const uint32_t lo = __byte_perm(w0, w1, sel);
    const uint32_t hi = __byte_perm(w2, w3, sel);
    return __byte_perm(lo, hi, 0x5410);
}

// The seven slice words of four biased integers: slice 1 is byte 6 as is,
// slices 2..7 are bytes 5..0 with the bias bit flipped back.
__device__ __forceinline__ void slice_words(const uint64_t (&y)[4], uint32_t (&w)[SLICES]) {
    w[0] = gather_byte(y, 6);
#pragma unroll
    for (int t = 1; t < SLICES; ++t) w[t] = gather_byte(y, 6 - t) ^ 0x80808080u;
}

__global__ void __launch_bounds__(THREADS, 1)
ozaki_gram_kernel(const __grid_constant__ CUtensorMap tm, int64_t rows, int64_t chunk_rows,
                  double* __restrict__ partial, Flags* __restrict__ flags, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* fp_full = reinterpret_cast<uint64_t*>(smem + OFF_BAR);
    uint64_t* fp_empty = fp_full + FSTAGES;
    uint64_t* sl_full = fp_empty + FSTAGES;
    uint64_t* sl_empty = sl_full + SBUFS;
    int* misc = reinterpret_cast<int*>(smem + OFF_MISC);
    volatile int* fresh_flag = misc;           // [SBUFS]
    volatile int* abort_flag = misc + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc + 4);
    int* Es = misc + 8;                        // [64] scale exponents for the drain
    double* colmax = reinterpret_cast<double*>(smem + OFF_MAX);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = (int64_t)blockIdx.x * chunk_rows;
    const int64_t row_end = min(rows, row0 + chunk_rows);
    const int nstages = (int)((row_end - row0 + ROWS - 1) / ROWS);
    double* P = partial + (size_t)blockIdx.x * (128 * 64);

    if (threadIdx.x == 0) {
        for (int b = 0; b < FSTAGES; ++b) {
            mbar_init(&fp_full[b], 1);
            mbar_init(&fp_empty[b], 128);
        }
        for (int b = 0; b < SBUFS; ++b) {
            mbar_init(&sl_full[b], 128);
            mbar_init(&sl_empty[b], 1);
        }
        *abort_flag = 0;
        for (int c = 0; c < 64; ++c) Es[c] = E_UNSET;
        mbar_fence_init();
    }
    if (warp == 0) umma::tmem_alloc(tmem_slot, TMEM_COLS);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = *tmem_slot;

    if (warp == 5) {
        // ---- producer: FP64 tiles, two 8-row boxes per stage ----
        if (lane == 0) {
            tma_prefetch_map(&tm);
            int issued = 0;
            for (int s = 0; s < nstages; ++s) {
                const int b = s % FSTAGES;
                if (s >= FSTAGES && !mbar_wait(&fp_empty[b], ((s / FSTAGES) - 1) & 1)) {
                    atomicExch(&flags->timeout, 1);
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                mbar_arrive_expect_tx(&fp_full[b], FBYTES);
                const int x = (int)(2 * (row0 + (int64_t)s * ROWS));
                unsigned char* dst = smem + OFF_F + (size_t)b * FBYTES;
                tma_load_2d(dst, &tm, x, 0, &fp_full[b]);
                tma_load_2d(dst + FBYTES / 2, &tm, x + 16, 0, &fp_full[b]);
                issued = s + 1;
            }
            // After an abort, let the copies still in flight land before the
            // shared memory they write goes away.
            for (int s = issued > FSTAGES ? issued - FSTAGES : 0; *abort_flag && s < issued; ++s)
                mbar_wait(&fp_full[s % FSTAGES], (s / FSTAGES) & 1);
        }
    } else if (warp == 4) {
        // ---- MMA issuer ----
        if (lane == 0) {
            int issued = 0;
            for (int s = 0; s < nstages; ++s) {
                const int b = s % SBUFS;
                if (!mbar_wait(&sl_full[b], (s / SBUFS) & 1) || *abort_flag) {
                    atomicExch(&flags->timeout, 1);
                    *abort_flag = 1;
                    break;
                }
                umma::fence_after_sync();
                const bool fresh = fresh_flag[b] != 0;
                const uint32_t abase = smem_u32(smem + OFF_S + (size_t)b * SBYTES);
                const uint32_t bbase = abase + SLICES * ATILE;
#pragma unroll
                for (int t = 0; t < SLICES; ++t) {
                    const int ntot = 64 * (SLICES - t);
                    const uint64_t da = desc_sw32(abase + t * ATILE);
#pragma unroll
                    for (int off = 0; off < ntot; off += 256) {
                        const int n = ntot - off < 256 ? ntot - off : 256;
                        umma::mma_s8(taddr + 64 * t + off, da, desc_sw32(bbase + off * 32),
                                     umma::idesc_s8s8_s32(128, n), !(fresh && t == 0));
                    }
                }
                umma::commit(&sl_empty[b]);
                issued = s + 1;
            }
            // After an abort, wait for the MMAs in flight before tensor memory
            // is released.
            if (*abort_flag && issued > 0) mbar_wait(&sl_empty[(issued - 1) % SBUFS], ((issued - 1) / SBUFS) & 1);
        }
    } else {
        // ---- slicers and drains: warps 0..3, thread tid owns TMEM lane tid ----
        const int tid = threadIdx.x;
        const int j = tid & 63, h = tid >> 6;
        int E = E_UNSET;            // scale exponent of column j
        int epoch_start = 0;
        bool initialized = false;   // P written at least once
        bool bad = false;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;

        // A CTA-uniform OR over the 128 slicer threads; also a barrier.
        auto any = [](bool p) -> bool {
            uint32_t q;
            asm volatile(
                "{\n\t.reg .pred a, b;\n\t"
                "setp.ne.u32 a, %1, 0;\n\t"
                "barrier.cta.red.or.pred b, 1, 128, a;\n\t"
                "selp.u32 %0, 1, 0, b;\n\t}"
                : "=r"(q)
                : "r"((uint32_t)p)
                : "memory");
            return q != 0;
        };
        auto fail = [&]() {
            atomicExch(&flags->timeout, 1);
            *abort_flag = 1;
        };

        // Adds the accumulators of the epoch that ended with last_stage into
        // P, row tid of the 128 x 64 partial. False if the MMAs never finished.
        auto drain = [&](int last_stage) -> bool {
            // Every MMA up to last_stage has finished once its commit arrived.
            if (!mbar_wait(&sl_empty[last_stage % SBUFS], (last_stage / SBUFS) & 1)) return false;
            umma::fence_after_sync();
            const int m = tid;
            const int Em = Es[m & 63];
#pragma unroll 1
            for (int c = 0; c < 2; ++c) {
                double acc[32];
#pragma unroll
                for (int i = 0; i < 32; ++i) acc[i] = 0.0;
#pragma unroll 1
                for (int g = 0; g < SLICES; ++g) {
                    uint32_t r[32];
                    umma::tmem_ld32(taddr + lane_base + 64 * g + 32 * c, r);
                    umma::tmem_wait_ld();
                    const double w = pow2(-8 * (g + 2));
#pragma unroll
                    for (int i = 0; i < 32; ++i) acc[i] = fma((double)(int)r[i], w, acc[i]);
                }
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const int n = 32 * c + i;
                    const int En = Es[n];
                    double v = 0.0;
                    if (Em != E_UNSET && En != E_UNSET) v = acc[i] * pow2(Em + En + 2);
                    double* dst = P + (size_t)n * 128 + m;
                    *dst = initialized ? *dst + v : v;
                }
            }
            initialized = true;
            umma::fence_before_sync();
            return true;
        };

        // Every decision that can end the loop is taken by all 128 threads
        // together (any), so none of them is ever left waiting at a barrier.
        int s = 0;
        for (; s < nstages; ++s) {
            const int fb = s % FSTAGES, sb = s % SBUFS;
            const bool landed = mbar_wait(&fp_full[fb], (s / FSTAGES) & 1);
            // Eight complex rows of column j from box h.
            double v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.0;
            if (landed) {
                const unsigned char* box = smem + OFF_F + (size_t)fb * FBYTES + (size_t)h * (FBYTES / 2) + j * 128;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const double2 z = *reinterpret_cast<const double2*>(box + ((r ^ (j & 7)) << 4));
                    v[2 * r] = z.x;
                    v[2 * r + 1] = z.y;
                }
                mbar_arrive(&fp_empty[fb]);
                double mx = 0.0;
                bool finite = true;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    mx = fmax(mx, fabs(v[i]));
                    finite &= isfinite(v[i]);
                }
                if (!finite) bad = true;
                colmax[h * 64 + j] = mx;
            }
            if (any(!landed || *abort_flag)) { fail(); break; }
            const double cm = fmax(colmax[j], colmax[64 + j]);
            const int need = cm > 0.0 ? ilogb(cm) + 2 + HEADROOM : E_UNSET;
            const bool over = cm > 0.0 && (E == E_UNSET || need > E);
            bool fresh = s == 0;
            if (any(over || (s - epoch_start >= EPOCH_STAGES))) {
                const bool drained = s > epoch_start ? drain(s - 1) : true;
                if (any(!drained)) { fail(); break; }
                if (over) E = E == E_UNSET ? need : max(E, need);
                if (h == 0) Es[j] = E;
                epoch_start = s;
                fresh = true;
            }
            // The slice buffer is free once the MMAs of stage s - 2 finished.
            const bool free_buf = s < SBUFS || mbar_wait(&sl_empty[sb], ((s - SBUFS) / SBUFS) & 1);
            if (any(!free_buf)) { fail(); break; }
            // Scale and split.
            const double sc = E == E_UNSET ? 0.0 : pow2(55 - E);
            unsigned char* sbuf = smem + OFF_S + (size_t)sb * SBYTES;
            // W row j: K values re0 im0 .. re7 im7; JW row 64 + j: im0 -re0 ..
            // Four K values (two complex rows) at a time, so only their
            // integers are live at once.
            uint32_t wW[4][SLICES], wJ[4][SLICES];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long long r0 = __double2ll_rn(v[4 * q] * sc), i0 = __double2ll_rn(v[4 * q + 1] * sc);
                const long long r1 = __double2ll_rn(v[4 * q + 2] * sc), i1 = __double2ll_rn(v[4 * q + 3] * sc);
                const uint64_t yw[4] = {(uint64_t)r0 + BIAS, (uint64_t)i0 + BIAS, (uint64_t)r1 + BIAS,
                                        (uint64_t)i1 + BIAS};
                const uint64_t yj[4] = {(uint64_t)i0 + BIAS, (uint64_t)(-r0) + BIAS, (uint64_t)i1 + BIAS,
                                        (uint64_t)(-r1) + BIAS};
                slice_words(yw, wW[q]);
                slice_words(yj, wJ[q]);
            }
#pragma unroll
            for (int t = 0; t < SLICES; ++t) {
                const uint4 ww = make_uint4(wW[0][t], wW[1][t], wW[2][t], wW[3][t]);
                const uint4 wj = make_uint4(wJ[0][t], wJ[1][t], wJ[2][t], wJ[3][t]);
                unsigned char* at = sbuf + t * ATILE;
                *reinterpret_cast<uint4*>(at + sw32_offset(j, h)) = ww;
                *reinterpret_cast<uint4*>(at + sw32_offset(64 + j, h)) = wj;
                *reinterpret_cast<uint4*>(sbuf + SLICES * ATILE + sw32_offset(64 * t + j, h)) = ww;
            }
            umma::fence_smem_to_async();
            if (tid == 0) fresh_flag[sb] = fresh ? 1 : 0;
            mbar_arrive(&sl_full[sb]);
        }
        if (s == nstages && nstages > 0) {
            if (any(!drain(nstages - 1))) fail();
        }
        if (bad) atomicExch(&flags->nonfinite, 1);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (warp == 0) umma::tmem_dealloc(taddr, TMEM_COLS);
}

// G = alpha (sum over CTAs) + beta C: Re G[a][b] = P[b][a], Im G[a][b] =
// -P[b][64 + a]. Re comes out symmetric to the bit (its slice products are
// symmetric integers); Im is made antisymmetric to the bit by taking half the
// difference of the two mirrored sums, since the slices of -x are not the
// negated slices of x and so the kept products differ in their last bits.
__global__ void ozaki_gram_reduce_kernel(z64* __restrict__ C, int64_t ldc, int k, int nctas,
                                         const double* __restrict__ partial, const Flags* __restrict__ flags,
                                         z64 alpha, z64 beta, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    const int lane = threadIdx.x & 31;
    const int64_t entry = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (entry >= (int64_t)k * k) return;
    const int a = (int)(entry % k), b = (int)(entry / k);
    double re = 0.0, im_ab = 0.0, im_ba = 0.0;
    for (int c = lane; c < nctas; c += 32) {
        const double* p = partial + (size_t)c * (128 * 64);
        re += p[(size_t)b * 128 + a];
        im_ab -= p[(size_t)b * 128 + 64 + a];
        im_ba -= p[(size_t)a * 128 + 64 + b];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, off);
        im_ab += __shfl_down_sync(0xffffffffu, im_ab, off);
        im_ba += __shfl_down_sync(0xffffffffu, im_ba, off);
    }
    if (lane != 0) return;
    double im = a == b ? 0.0 : 0.5 * (im_ab - im_ba);
    if (flags->timeout || flags->nonfinite) re = im = __longlong_as_double(0x7ff8000000000000ll);
    z64 out = zmul(alpha, zmake(re, im));
    z64* dst = C + a + (int64_t)b * ldc;
    if (beta.x != 0.0 || beta.y != 0.0) zmac(out, beta, *dst);
    *dst = out;
}

struct Shape {
    int nctas;
    int64_t chunk_rows;
};

static Shape shape_of(int64_t rows) {
    Shape s{};
    const int64_t sms = sm_count();
    const int64_t stages = (rows + ROWS - 1) / ROWS;
    const int64_t per = (stages + sms - 1) / sms;
    s.chunk_rows = per * ROWS;
    s.nctas = s.chunk_rows > 0 ? (int)((rows + s.chunk_rows - 1) / s.chunk_rows) : 0;
    return s;
}

}  // namespace ozaki

size_t ozaki_gram_workspace_size(int64_t rows) {
    const ozaki::Shape s = ozaki::shape_of(rows);
    return align_up(sizeof(ozaki::Flags), 256) + (size_t)(s.nctas > 0 ? s.nctas : 1) * 128 * 64 * sizeof(double);
}

// C = alpha A^H A + beta C for a rows x k matrix A, k <= 64, on the integer
// tensor cores. workspace: ozaki_gram_workspace_size(rows) bytes.
int ozaki_gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, int64_t rows, int k, z64 alpha, z64 beta,
                       void* workspace, size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st,
                       int gate) {
    if (k < 1 || k > 64) {
        set_error(FB_ENOTSUP, "the tensor-core Gram handles 1 <= k <= 64, got k = %d", k);
        return FB_ENOTSUP;
    }
    if (rows > ((int64_t)1 << 30)) {
        set_error(FB_ENOTSUP, "the tensor-core Gram handles at most 2^30 rows, got %lld", (long long)rows);
        return FB_ENOTSUP;
    }
    const size_t need = ozaki_gram_workspace_size(rows);
    if (!workspace || workspace_bytes < need) {
        set_error(FB_ENOMEM, "tensor-core gram: workspace of %zu bytes is smaller than the %zu bytes needed",
                  workspace_bytes, need);
        return FB_ENOMEM;
    }
    const ozaki::Shape s = ozaki::shape_of(rows);
    ozaki::Flags* flags = static_cast<ozaki::Flags*>(workspace);
    double* partial = reinterpret_cast<double*>(static_cast<char*>(workspace) + align_up(sizeof(ozaki::Flags), 256));
    FB_CUDA(cudaMemsetAsync(flags, 0, sizeof(ozaki::Flags), stream), "cudaMemsetAsync");
    if (s.nctas > 0) {
        CUtensorMap tm;
        FB_TRY(encode_panel_map(&tm, A, rows, k, lda, 64));
        FB_CUDA(cudaFuncSetAttribute(ozaki::ozaki_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ozaki::SMEM_BYTES), "cudaFuncSetAttribute");
        ozaki::ozaki_gram_kernel<<<s.nctas, ozaki::THREADS, ozaki::SMEM_BYTES, stream>>>(
            tm, rows, s.chunk_rows, partial, flags, st, gate);
        FB_LAUNCHED("ozaki_gram_kernel");
    } else {
        FB_CUDA(cudaMemsetAsync(partial, 0, 128 * 64 * sizeof(double), stream), "cudaMemsetAsync");
    }
    const int64_t threads = (int64_t)k * k * 32;
    ozaki::ozaki_gram_reduce_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
        C, ldc, k, s.nctas > 0 ? s.nctas : 1, partial, flags, alpha, beta, st, gate);
    FB_LAUNCHED("ozaki_gram_reduce_kernel");
    return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zgram_tc_workspace_size(int64_t rows, int k, size_t* bytes) {
    if (!bytes || rows < 0 || k < 0) { set_error(FB_EINVAL, "fb_zgram_tc_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = ozaki_gram_workspace_size(rows);
    return FB_OK;
}

int fb_zgram_tc(fb_z128* C, int64_t ldc, const fb_z128* A, int64_t lda, int64_t rows, int k, fb_z128 alpha,
                fb_z128 beta, void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (rows < 0 || k < 0) { set_error(FB_EDIM, "fb_zgram_tc: negative size"); return FB_EDIM; }
    if (k == 0) return FB_OK;
    if (!C || (!A && rows > 0)) { set_error(FB_EINVAL, "fb_zgram_tc: NULL matrix"); return FB_EINVAL; }
    if (ldc < k || (rows > 0 && lda < rows)) { set_error(FB_EDIM, "fb_zgram_tc: leading dimension too small"); return FB_EDIM; }
    if ((uintptr_t)A & 15) { set_error(FB_EINVAL, "fb_zgram_tc: A must be 16-byte aligned"); return FB_EINVAL; }
    return ozaki_gram_enqueue(reinterpret_cast<z64*>(C), ldc, reinterpret_cast<const z64*>(A), lda, rows, k,
                              zmake(alpha.re, alpha.im), zmake(beta.re, beta.im), workspace, workspace_bytes,
                              stream_of(queue), nullptr, GATE_ALWAYS);
}

}  // extern "C"
