// The Gram matrix G = Y^H Y (gram_accumulate!, src/kernels.jl:22-55, with
// A === B) on the integer tensor cores: an Ozaki-style split of every FP64
// entry into 8-bit slices whose products are exact in 32-bit integer
// accumulators, recovered to FP64 with power-of-two weights.
//
// Real form. With W the 2N x k real matrix holding Re Y and Im Y in
// alternating rows (exactly the interleaved ComplexF64 layout of a column) and
// JW the same with each (re, im) pair turned into (im, -re):
//   [W JW]^T W = [Re G ; -Im G]      (a 128 x 64 product for k <= 64).
// The MMA operand A holds the slices of W and JW, 128 rows, in tensor memory;
// operand B holds the W slices stacked along N in shared memory, so one MMA
// of A slice t against B slices 1..7-t lands in the accumulators of the groups
// g = t + u it feeds. Keeping A in tensor memory halves the shared-memory
// traffic of the products, which bounds this kernel.
//
// Slices. Column j carries a power-of-two scale 2^E_j with |entries| <
// 2^(E_j - 1); an entry x becomes the integer x_int = rint(x 2^(51 - E_j)),
// |x_int| <= 2^50, written as seven signed bytes on a grid of 8-bit steps
//   x_int = sum_{t=1..7} d_t 2^(52 - 8 t),   d_t in [-128, 127],
// the last one a multiple of 16 (it carries the lowest 4 bits). One FMA makes
// them: m = fma(x, 2^(51 - E_j), 2^52 + 2^51 + B) is exact, its 52 mantissa
// bits are x_int + B + 2^51 with B = 0x80808080808 biasing every digit by
// half its range, and the bytes of m << 4 are the digits, each plus 128: the
// slices are read straight out of the double's bit pattern, and its exponent
// field tells whether x was in range. A product of two entries is
// 2^(E_a + E_b - 102) sum_{t,u} d_t e_u 2^(104 - 8 (t + u)); the 28 terms
// with t + u <= 8 are kept, the rest lie below 2^-50 of the leading term. Group g = t + u owns 64 accumulator columns of tensor memory (448 in
// all), the A slices the next 56.
//
// Scales adapt as the rows stream: a stage with an entry its column's scale
// cannot hold, or one that would let an int32 accumulator overflow (every
// 8192 rows), first drains the accumulators into this CTA's FP64 partial in
// global memory, then rescales with HEADROOM spare bits. The partials of all
// CTAs are summed in a fixed order by the reduce kernel, so results are
// deterministic.
//
// Rows of A (tensor memory lanes): lane 32q + l holds W column 16q + l for
// l < 16 and JW column 16q + l - 16 for l >= 16, so one warp writes both rows
// of a column and its two halves read the same FP64 values (a broadcast).
//
// Roles (one CTA per SM, 576 threads): warps 0-15 slice (warp w writes lane
// quarter w % 4, K bytes 8 (w / 4)..+7 of every A slice) and drain (lane
// quarter w % 4, accumulator columns 16 (w / 4)..+15 of every group); warp 16
// issues the MMAs; warp 17 keeps a ring of TMA tile loads in flight. Every
// wait is bounded.
#include "fb_umma.cuh"

namespace fb {
namespace ozaki {

constexpr int SLICES = 7;
constexpr int ROWS = 16;                        // complex rows per stage: K = 32 bytes
constexpr int FSTAGES = 6;                      // FP64 ring depth
constexpr int FBYTES = ROWS * 64 * 16;          // 16 KB: 16 rows x 64 columns
constexpr int BTILE = SLICES * 64 * 32;         // B: 7 x 64 rows x 32 bytes
constexpr int SBUFS = 2;
constexpr int TMEM_COLS = 512;
constexpr int A_COL = 448;                      // A slice t at tensor memory column A_COL + 8 t
constexpr int EPOCH_STAGES = 8192 / ROWS;       // int32 headroom: 7 x 2^14 x 2 x 8192 < 2^31
constexpr int HEADROOM = 2;                     // spare exponent bits above the maximum that set a scale
constexpr int E_UNSET = -4000;                  // column seen only zeros so far
constexpr int SLICERS = 512;                    // sixteen warps
constexpr int THREADS = SLICERS + 64;
// 2^52 + 2^51 + 0x80808080808: the FMA addend that leaves x_int + B + 2^51
// in the mantissa of a double whose high word starts with 0x433.
constexpr long long MAGIC_BITS = 0x4338080808080808ll;

constexpr size_t OFF_F = 0;
constexpr size_t OFF_B = OFF_F + (size_t)FSTAGES * FBYTES;
constexpr size_t OFF_MAX = OFF_B + (size_t)SBUFS * BTILE;   // uint32 [4][64] column maxima
constexpr size_t OFF_BAR = OFF_MAX + 4 * 64 * 4;            // mbarriers
constexpr size_t OFF_MISC = OFF_BAR + 32 * 8;
constexpr size_t MISC_BYTES = 512;                          // flags, TMEM slot, column exponents
constexpr size_t SMEM_BYTES = OFF_MISC + MISC_BYTES + 1024;  // + alignment slack

struct Flags {
    int timeout;
    int nonfinite;
    int drains;      // epochs drained, all CTAs together (a statistic)
    int rescales;    // of them, drains forced by a column outgrowing its scale
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

// The seven slice words of four FMA results (bit patterns, each shifted
// left by 4): word t holds slice t of each, low to high. Bytes 6..0 of the
// four values are transposed with byte permutes and the bias bit of every
// digit flipped back.
__device__ __forceinline__ void slice_words(const uint64_t (&y)[4], uint32_t (&w)[SLICES]) {
    const uint32_t l0 = (uint32_t)y[0], l1 = (uint32_t)y[1], l2 = (uint32_t)y[2], l3 = (uint32_t)y[3];
    const uint32_t h0 = (uint32_t)(y[0] >> 32), h1 = (uint32_t)(y[1] >> 32);
    const uint32_t h2 = (uint32_t)(y[2] >> 32), h3 = (uint32_t)(y[3] >> 32);
    const uint32_t a01 = __byte_perm(l0, l1, 0x5140), b01 = __byte_perm(l0, l1, 0x7362);
    const uint32_t a23 = __byte_perm(l2, l3, 0x5140), b23 = __byte_perm(l2, l3, 0x7362);
    const uint32_t c01 = __byte_perm(h0, h1, 0x5140), d01 = __byte_perm(h0, h1, 0x7362);
    const uint32_t c23 = __byte_perm(h2, h3, 0x5140), d23 = __byte_perm(h2, h3, 0x7362);
    w[0] = __byte_perm(d01, d23, 0x5410) ^ 0x80808080u;  // byte 6
    w[1] = __byte_perm(c01, c23, 0x7632) ^ 0x80808080u;  // byte 5
    w[2] = __byte_perm(c01, c23, 0x5410) ^ 0x80808080u;  // byte 4
    w[3] = __byte_perm(b01, b23, 0x7632) ^ 0x80808080u;  // byte 3
    w[4] = __byte_perm(b01, b23, 0x5410) ^ 0x80808080u;  // byte 2
    w[5] = __byte_perm(a01, a23, 0x7632) ^ 0x80808080u;  // byte 1
    w[6] = __byte_perm(a01, a23, 0x5410) ^ 0x80808080u;  // byte 0
}

// Adds the accumulators of the epoch that ended with last_stage into P: row
// prow, columns 16c..16c+15 of the 128 x 64 partial, read from tensor memory
// at tcol (this thread's lane, column 16c of group 0). False if the MMAs
// never finished. Kept out of line: it runs a few times per CTA and would
// otherwise hold registers across the slicing loop.
__device__ __noinline__ bool drain_epoch(uint64_t* sl_empty, int last_stage, uint32_t tcol, const int* Es, int prow,
                                         int c, double* P, bool initialized) {
    // Every MMA up to last_stage has finished once its commit arrived.
    if (!mbar_wait(&sl_empty[last_stage % SBUFS], (last_stage / SBUFS) & 1)) return false;
    umma::fence_after_sync();
    const int Em = Es[prow & 63];
    double acc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = 0.0;
#pragma unroll 1
    for (int g = 0; g < SLICES; ++g) {
        uint32_t r[16];
        umma::tmem_ld16(tcol + 64 * g, r);
        umma::tmem_wait_ld();
        const double w = pow2(-8 * (g + 2));
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] = fma((double)(int)r[i], w, acc[i]);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = 16 * c + i;
        const int En = Es[n];
        double v = 0.0;
        if (Em != E_UNSET && En != E_UNSET) v = acc[i] * pow2(Em + En + 2);
        double* dst = P + (size_t)n * 128 + prow;
        *dst = initialized ? *dst + v : v;
    }
    umma::fence_before_sync();
    return true;
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
    uint32_t* colmax = reinterpret_cast<uint32_t*>(smem + OFF_MAX);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = (int64_t)blockIdx.x * chunk_rows;
    const int64_t row_end = min(rows, row0 + chunk_rows);
    const int nstages = (int)((row_end - row0 + ROWS - 1) / ROWS);
    double* P = partial + (size_t)blockIdx.x * (128 * 64);

    if (threadIdx.x == 0) {
        for (int b = 0; b < FSTAGES; ++b) {
            mbar_init(&fp_full[b], 1);
            mbar_init(&fp_empty[b], SLICERS);
        }
        for (int b = 0; b < SBUFS; ++b) {
            mbar_init(&sl_full[b], SLICERS);
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

    if (warp == SLICERS / 32 + 1) {
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
    } else if (warp == SLICERS / 32) {
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
                const uint32_t bbase = smem_u32(smem + OFF_B + (size_t)b * BTILE);
#pragma unroll
                for (int t = 0; t < SLICES; ++t) {
                    const int ntot = 64 * (SLICES - t);
#pragma unroll
                    for (int off = 0; off < ntot; off += 256) {
                        const int n = ntot - off < 256 ? ntot - off : 256;
                        umma::mma_s8_tmem_a(taddr + 64 * t + off, taddr + A_COL + 8 * t, desc_sw32(bbase + off * 32),
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
        // ---- slicers and drains: warps 0..15 ----
        const int tid = threadIdx.x;
        const int q = warp & 3, kq = warp >> 2;
        const bool jw = lane >= 16;
        const int j = 16 * q + (lane & 15);                  // this thread's column
        const int prow = (jw ? 64 : 0) + j;                  // its row of the 128 x 64 partial
        const uint32_t lane_base = (uint32_t)(32 * q) << 16;
        int E = E_UNSET;            // scale exponent of column j
        int epoch_start = 0;
        bool initialized = false;   // P written at least once
        bool bad = false;

        // A CTA-uniform OR over the slicer threads; also a barrier.
        auto any = [](bool p) -> bool {
            uint32_t qq;
            asm volatile(
                "{\n\t.reg .pred a, b;\n\t"
                "setp.ne.u32 a, %1, 0;\n\t"
                "barrier.cta.red.or.pred b, 1, %2, a;\n\t"
                "selp.u32 %0, 1, 0, b;\n\t}"
                : "=r"(qq)
                : "r"((uint32_t)p), "n"(SLICERS)
                : "memory");
            return qq != 0;
        };
        auto fail = [&]() {
            atomicExch(&flags->timeout, 1);
            *abort_flag = 1;
        };
        auto drain = [&](int last_stage) -> bool {
            const bool ok = drain_epoch(sl_empty, last_stage, taddr + lane_base + 16 * kq, Es, prow, kq, P, initialized);
            initialized = true;
            return ok;
        };
        // Complex rows 4 (kq & 1) .. + 3 of column j in box kq / 2 of stage st.
        auto load = [&](int st, double (&vv)[8]) -> bool {
            const int fb = st % FSTAGES;
            if (!mbar_wait(&fp_full[fb], (st / FSTAGES) & 1)) return false;
            const unsigned char* box = smem + OFF_F + (size_t)fb * FBYTES + (size_t)(kq >> 1) * (FBYTES / 2) + j * 128;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int rr = 4 * (kq & 1) + r;
                const double2 z = *reinterpret_cast<const double2*>(box + ((rr ^ (j & 7)) << 4));
                vv[2 * r] = z.x;
                vv[2 * r + 1] = z.y;
            }
            mbar_arrive(&fp_empty[fb]);
            return true;
        };

        // Every decision that can end the loop is taken by all slicer threads
        // together (any), so none of them is ever left waiting at a barrier:
        // one barrier per stage in the common case. A failed wait elsewhere
        // is recorded and stops the loop at the next stage's barrier.
        const double magic = __longlong_as_double(MAGIC_BITS);
        bool timed_out = false;
        int s = 0;
        for (; s < nstages; ++s) {
            const int sb = s % SBUFS;
            double v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = 0.0;
            const bool landed = load(s, v);
            // Scale and split: W rows take re0 im0 re1 im1 .., JW rows
            // im0 -re0 im1 -re1 .., four K values to a word. A result whose
            // high word does not start 0x433 was out of range.
            double sc = (E == E_UNSET || bad) ? 0.0 : pow2(51 - E);
            uint64_t t[8];
            uint32_t range = 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double first = jw ? v[2 * c + 1] : v[2 * c];
                const double second = jw ? v[2 * c] : v[2 * c + 1];
                t[2 * c] = (uint64_t)__double_as_longlong(fma(first, sc, magic));
                t[2 * c + 1] = (uint64_t)__double_as_longlong(fma(second, jw ? -sc : sc, magic));
                range |= ((uint32_t)(t[2 * c] >> 32) ^ 0x43300000u) | ((uint32_t)(t[2 * c + 1] >> 32) ^ 0x43300000u);
            }
            bool out_of_range = (range & 0xFFF00000u) != 0;
            if (E == E_UNSET) {
                uint32_t nz = 0;
#pragma unroll
                for (int i = 0; i < 8; ++i) nz |= (uint32_t)(__double_as_longlong(v[i]) >> 32) & 0x7FF00000u;
                out_of_range = nz != 0;
            }
            const bool epoch_full = s - epoch_start >= EPOCH_STAGES;
            const bool stop = !landed || timed_out || *abort_flag;
            bool fresh = s == 0;
            if (any(stop || out_of_range || epoch_full)) {
                if (any(stop)) { fail(); break; }
                // The column maxima: the high word of |x| orders magnitudes
                // by exponent, and Inf and NaN above every finite value.
                uint32_t mx = 0;
#pragma unroll
                for (int i = 0; i < 8; ++i) mx = max(mx, (uint32_t)(__double_as_longlong(v[i]) >> 32) & 0x7FFFFFFFu);
                if (!jw) colmax[kq * 64 + j] = mx;
                asm volatile("bar.sync 1, %0;" ::"n"(SLICERS) : "memory");
                const uint32_t cm = max(max(colmax[j], colmax[64 + j]), max(colmax[128 + j], colmax[192 + j]));
                if (cm >= 0x7FF00000u) bad = true;
                // A column outgrows its scale when its maximum is no longer
                // below 2^(E - 1); the new scale leaves HEADROOM bits above it.
                const int need = cm >= 0x00100000u ? (int)(cm >> 20) - 1023 + 2 + HEADROOM : E_UNSET;
                const bool over = need != E_UNSET && (E == E_UNSET || (int)(cm >> 20) - 1023 >= E - 1);
                const bool any_over = any(over);
                if (any_over || epoch_full) {
                    const bool drained = s > epoch_start ? drain(s - 1) : true;
                    if (tid == 0 && s > epoch_start) {
                        atomicAdd(&flags->drains, 1);
                        if (any_over) atomicAdd(&flags->rescales, 1);
                    }
                    if (any(!drained)) { fail(); break; }
                    if (over) E = E == E_UNSET ? need : max(E, need);
                    if (kq == 0 && !jw) Es[j] = E;
                    epoch_start = s;
                    fresh = true;
                    if (any_over) {
                        sc = (E == E_UNSET || bad) ? 0.0 : pow2(51 - E);
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const double first = jw ? v[2 * c + 1] : v[2 * c];
                            const double second = jw ? v[2 * c] : v[2 * c + 1];
                            t[2 * c] = (uint64_t)__double_as_longlong(fma(first, sc, magic));
                            t[2 * c + 1] = (uint64_t)__double_as_longlong(fma(second, jw ? -sc : sc, magic));
                        }
                    }
                }
            }
            uint32_t w0[SLICES], w1[SLICES];
            {
                const uint64_t y0[4] = {t[0] << 4, t[1] << 4, t[2] << 4, t[3] << 4};
                const uint64_t y1[4] = {t[4] << 4, t[5] << 4, t[6] << 4, t[7] << 4};
                slice_words(y0, w0);
                slice_words(y1, w1);
            }
            // The MMAs of stage s - 1 still read A and, two stages back, B:
            // wait for them, then write this stage's slices.
            if (s >= 1 && !mbar_wait(&sl_empty[(s - 1) % SBUFS], ((s - 1) / SBUFS) & 1)) timed_out = true;
            umma::fence_after_sync();
            unsigned char* bbuf = smem + OFF_B + (size_t)sb * BTILE;
            const uint32_t boff = sw32_offset(j, kq >> 1) + (kq & 1) * 8;
#pragma unroll
            for (int tt = 0; tt < SLICES; ++tt) {
                umma::tmem_st2(taddr + lane_base + A_COL + 8 * tt + 2 * kq, w0[tt], w1[tt]);
                if (!jw) *reinterpret_cast<uint2*>(bbuf + boff + tt * (64 * 32)) = make_uint2(w0[tt], w1[tt]);
            }
            umma::tmem_wait_st();
            umma::fence_smem_to_async();
            umma::fence_before_sync();
            if (tid == 0) fresh_flag[sb] = fresh ? 1 : 0;
            mbar_arrive(&sl_full[sb]);
        }
        if (s == nstages && nstages > 0) {
            if (any(!drain(nstages - 1))) fail();
            if (tid == 0) atomicAdd(&flags->drains, 1);
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
