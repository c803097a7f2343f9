// gram_accumulate! (src/kernels.jl:22-55): C <- alpha A^H B + beta C for tall
// skinny A (rows x kA) and B (rows x kB), ComplexF64, FP64 throughout.
//
// Layout of the work. C is cut into tiles of at most 64 x 64 columns. A CTA
// owns one tile and one chunk of rows, which it streams through shared memory
// in stages of 32 rows: one producer warp issues TMA loads (boxes of 8 rows x
// the tile's columns, 128-byte swizzled, zero-filled past the last row and
// column, so ragged views need no special code) into a ring of stages guarded
// by mbarriers, and the consumer warps multiply. The products run on the FP64
// tensor cores (mma m8n8k4): with W the real matrix whose rows are the real
// and imaginary parts of Y's rows, Re(A^H B) = W_A^T W_B and
// Im(A^H B) = (J W_A)^T W_B, J taking each (re, im) pair to (-im, re). So
// an 8 x 8 block of C costs two MMAs per two complex rows, and the J costs
// only a register select: the A fragment's 16-byte load holds both parts, and
// a warp loads it once for all its blocks in the same block row.
// Every consumer warp owns whole 8 x 8 blocks of the tile for the whole
// chunk, so nothing is reduced across warps. A warp's blocks accumulate in
// registers; at the end the CTA's partial tile goes to the workspace, and a
// second kernel adds the chunks in a fixed order and applies alpha and beta.
// Nothing depends on timing, so the bits of the result depend only on
// (rows, kA, kB) and the device.
//
// When A and B are the same view the tile grid is folded: only tiles on or
// above the diagonal run and, inside a diagonal tile, only 8 x 8 blocks on or
// above the diagonal (36 of 64 at k = 64). The lower triangle is written as
// the conjugate of the upper one and the diagonal is made real.
//
// Swizzle: a TMA box is 8 rows (128 bytes per column) by the tile's columns,
// and 128-byte swizzling stores the 16-byte element of row r in column c at
// chunk r ^ (c % 8) of that column's 128-byte line. The eight lanes that read
// eight consecutive columns of one row therefore hit eight different banks.
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "fb_common.cuh"
#include "fb_tma.cuh"

namespace fb {

constexpr int GS_ROWS = 32;             // complex rows per stage
constexpr int GS_BOX_ROWS = 8;          // complex rows per TMA box (128 bytes)
constexpr int GS_BOXES = GS_ROWS / GS_BOX_ROWS;
constexpr int G_TILE = 64;              // columns per output tile side, at most
constexpr int G_MAX_WARPS = 17;         // 16 consumers + the producer

struct GramShape {
    int tw_a, tw_b;      // tile widths in columns (multiples of 8, at most 64)
    int nt_a, nt_b;      // tiles along the columns of A and of B
    int hermitian;
    int sdiag;           // diagonal 8 x 8 blocks of folded tiles hold S = Re + Im
    int ntiles;          // tiles in the partial buffer
    int64_t chunk_rows;  // a multiple of GS_ROWS
    int nchunks;
};

struct GramLaunch {
    int diag;            // folded diagonal tiles (hermitian mode)
    int ntiles;          // CTAs along x
    int nb_a, nb_b;      // 8-column blocks per tile side
    int npairs;          // 8 x 8 blocks of the tile that are computed
    int ppw;             // blocks per consumer warp
    int consumers;       // consumer warps
    int stages;
    int stage_bytes;
    int sdiag;           // slot 0 of warps 0..nb-1 holds diagonal block (w, w), S-coded
    size_t smem;
    // Block (I, J) of every consumer slot (warp * ppw + i); -1 for an empty
    // slot. Built on the host so that the SM's four sub-partitions get equal
    // MMA counts (a block on the diagonal costs one MMA per k-step, the others
    // two).
    signed char pi[64], pj[64];
};

__host__ __device__ inline int off_tile_index(int nt, int ti, int tj) {
    // Off-diagonal tile (ti < tj) in row-major order over the strict upper
    // triangle, after the nt diagonal tiles.
    return nt + ti * (2 * nt - ti - 1) / 2 + (tj - ti - 1);
}

// Consumer warps per block count: at most 16 with two or four blocks a warp,
// 12 with three, 8 with eight. Fewer warps leave each more registers.
template <int PPW>
__global__ void __launch_bounds__(PPW >= 8 ? 9 * 32 : PPW == 3 ? 13 * 32 : G_MAX_WARPS * 32, 1)
gram_dmma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 int64_t rows, GramShape sh, GramLaunch ln, z64* __restrict__ partial,
                 const ChainStatus* st, int gate, int chunk0) {
    if (gated_off(st, gate)) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // Aligned for the 128-byte swizzle by pointer arithmetic on the shared
    // array itself, so the compiler keeps seeing a shared-memory pointer and
    // emits 32-bit shared loads (an integer round trip would make every
    // fragment load generic, with 64-bit address arithmetic).
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);

    // Which tile this CTA owns.
    int ti, tj, tile_index;
    if (ln.diag) {
        ti = tj = blockIdx.x;
        tile_index = blockIdx.x;
    } else if (sh.hermitian) {
        int t = blockIdx.x;
        ti = 0;
        while (t >= sh.nt_a - 1 - ti) { t -= sh.nt_a - 1 - ti; ++ti; }
        tj = ti + 1 + t;
        tile_index = off_tile_index(sh.nt_a, ti, tj);
    } else {
        ti = blockIdx.x / sh.nt_b;
        tj = blockIdx.x % sh.nt_b;
        tile_index = blockIdx.x;
    }
    const int chunk = chunk0 + (int)blockIdx.y;
    const int64_t row0 = (int64_t)chunk * sh.chunk_rows;
    const int64_t row_end = min(rows, row0 + sh.chunk_rows);
    const int64_t nstages = (row_end - row0 + GS_ROWS - 1) / GS_ROWS;
    const int box_a = sh.tw_a * 128, box_b = ln.diag ? box_a : sh.tw_b * 128;
    const int stages = ln.stages;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)stages * ln.stage_bytes);
    uint64_t* empty = full + stages;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int b = 0; b < stages; ++b) {
            mbar_init(&full[b], 1);
            mbar_init(&empty[b], ln.consumers);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == ln.consumers) {
        // Producer: one lane keeps the ring full.
        if (lane == 0) {
            tma_prefetch_map(&tmA);
            if (!ln.diag) tma_prefetch_map(&tmB);
            // Ring slot and phase advance incrementally: a 64-bit division per
            // stage would run on the slow XU pipe and starve the MMAs.
            int b = 0;
            uint32_t phase = 0;
            for (int64_t s = 0; s < nstages; ++s) {
                if (s >= stages && !mbar_wait(&empty[b], phase ^ 1u)) break;
                mbar_arrive_expect_tx(&full[b], (uint32_t)ln.stage_bytes);
                unsigned char* dst = smem + (size_t)b * ln.stage_bytes;
                const int64_t r = row0 + s * GS_ROWS;
                for (int g = 0; g < GS_BOXES; ++g)
                    tma_load_2d(dst + g * box_a, &tmA, (int)(2 * (r + g * GS_BOX_ROWS)), ti * sh.tw_a, &full[b]);
                if (!ln.diag) {
                    unsigned char* dstb = dst + GS_BOXES * box_a;
                    for (int g = 0; g < GS_BOXES; ++g)
                        tma_load_2d(dstb + g * box_b, &tmB, (int)(2 * (r + g * GS_BOX_ROWS)), tj * sh.tw_b, &full[b]);
                }
                if (++b == stages) { b = 0; phase ^= 1u; }
            }
        }
        return;
    }

    // Consumers: this warp's 8 x 8 blocks. A warp past the last block
    // computes a copy of block 0 and never writes it, so the inner loop has no
    // branch on it.
    int bi[PPW], bj[PPW];
    bool valid[PPW], dpair[PPW];
#pragma unroll
    for (int i = 0; i < PPW; ++i) {
        const int slot = warp * PPW + i;
        if constexpr (PPW == 4) {
            // A full 64 x 64 tile: warp w owns half of block row w / 2. The
            // offsets below are then one base plus constants, which keeps the
            // 16-warp kernel inside its register budget.
            valid[i] = true;
            bi[i] = warp >> 1;
            bj[i] = 4 * (warp & 1) + i;
            dpair[i] = false;
            continue;
        }
        valid[i] = ln.pi[slot] >= 0;
        bi[i] = valid[i] ? ln.pi[slot] : ln.pi[0];
        bj[i] = valid[i] ? ln.pj[slot] : ln.pj[0];
        // A diagonal block of a folded tile: Re there is symmetric and Im
        // antisymmetric, so one product S = (W + J W)^T W = Re + Im carries
        // both, and the reduction recovers them as (S + S^T)/2, (S - S^T)/2.
        // Such a block only ever sits in slot 0.
        dpair[i] = (i == 0) && ln.sdiag && valid[i] && bi[i] == bj[i];
    }

    // Lane roles in the m8n8k4 fragments: col8 = column within the 8-block,
    // t = which of the k-step's two complex rows, part = re or im. A k-step
    // takes rows q and q + 4 of a box, so the swizzled chunks of the two rows
    // (q ^ c and (q + 4) ^ c) never share a bank within a half warp.
    const int col8 = lane >> 2;
    const int t = (lane >> 1) & 1;
    const int part = lane & 1;
    int swz[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) swz[q] = ((q + 4 * t) ^ col8) << 4;
    // Byte offsets within a box: the lane's own part of A and of B, and the
    // other part of A, whose sign flip turns W_A into (J W_A) for the
    // imaginary product (J takes (re, im) to (-im, re)).
    int offA[PPW], offAo[PPW], offB[PPW];
    bool newA[PPW];
#pragma unroll
    for (int i = 0; i < PPW; ++i) {
        offA[i] = (bi[i] * 8 + col8) * 128 + part * 8;
        offAo[i] = (bi[i] * 8 + col8) * 128 + (part ^ 1) * 8;
        offB[i] = (bj[i] * 8 + col8) * 128 + part * 8;
        newA[i] = (i == 0) || (bi[i] != bi[i > 0 ? i - 1 : 0]);
    }
    const unsigned long long flip = part ? 0ull : 0x8000000000000000ull;

    // NACC interleaved accumulator sets (alternate k-steps) double the
    // independent MMA chains per warp.
    constexpr int NACC = PPW == 2 ? 2 : 1;
    double acc[NACC][PPW][2][2];
#pragma unroll
    for (int h = 0; h < NACC; ++h)
#pragma unroll
        for (int i = 0; i < PPW; ++i)
            acc[h][i][0][0] = acc[h][i][0][1] = acc[h][i][1][0] = acc[h][i][1][1] = 0.0;

    // The stage loop, compiled twice: with slot 0 a diagonal S block (one MMA
    // a k-step) and without. The choice is per warp and made once, here, so
    // no MMA in the loop is predicated (a predicated-off MMA still occupies
    // the tensor pipe).
    bool ok = true;
    auto run = [&](auto s0_tag) {
        constexpr bool S0 = decltype(s0_tag)::value;
        int b = 0;
        uint32_t phase = 0;
        for (int64_t s = 0; s < nstages; ++s) {
            if (!mbar_wait(&full[b], phase)) { ok = false; break; }
            const unsigned char* sa = smem + (size_t)b * ln.stage_bytes;
            const unsigned char* sbb = ln.diag ? sa : sa + GS_BOXES * box_a;
#pragma unroll 1
            for (int g = 0; g < GS_BOXES; ++g) {
                const unsigned char* ba = sa + g * box_a;
                const unsigned char* bb = sbb + g * box_b;
                constexpr int Q_UNROLL = PPW >= 8 ? 1 : 4;
#pragma unroll Q_UNROLL
                for (int q = 0; q < 4; ++q) {
                    const int h = q % NACC;
                    double are = 0.0, aim = 0.0;
#pragma unroll
                    for (int i = 0; i < PPW; ++i) {
                        if (newA[i]) {
                            are = *reinterpret_cast<const double*>(ba + offA[i] + swz[q]);
                            aim = __longlong_as_double(
                                __double_as_longlong(*reinterpret_cast<const double*>(ba + offAo[i] + swz[q])) ^ flip);
                        }
                        const double bw = *reinterpret_cast<const double*>(bb + offB[i] + swz[q]);
                        if constexpr (S0) {
                            if (i == 0) {
                                dmma_884(acc[h][i][0][0], acc[h][i][0][1], are + aim, bw);
                                continue;
                            }
                        }
                        dmma_884(acc[h][i][0][0], acc[h][i][0][1], are, bw);
                        dmma_884(acc[h][i][1][0], acc[h][i][1][1], aim, bw);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[b]);
            if (++b == stages) { b = 0; phase ^= 1u; }
        }
    };
    if constexpr (PPW >= 8) {
        run(std::false_type{});   // eight blocks a warp: full tiles only, no diagonal block
    } else {
        if (dpair[0]) run(std::true_type{});
        else run(std::false_type{});
    }
    if (!ok) {
        // A stage never arrived: poison this CTA's share of the result so the
        // failure reaches the caller as NaN instead of a silent wrong answer.
#pragma unroll
        for (int i = 0; i < PPW; ++i)
            acc[0][i][0][0] = acc[0][i][0][1] = acc[0][i][1][0] = acc[0][i][1][1] = __longlong_as_double(0x7ff8000000000000ll);
    }
#pragma unroll
    for (int h = 1; h < NACC; ++h)
#pragma unroll
        for (int i = 0; i < PPW; ++i)
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                acc[0][i][x][0] += acc[h][i][x][0];
                acc[0][i][x][1] += acc[h][i][x][1];
            }

    // A partial tile holds tw_a x tw_b entries, column-major: narrow tiles
    // take only the scratch they fill.
    z64* out = partial + ((size_t)tile_index * sh.nchunks + chunk) * (size_t)(sh.tw_a * sh.tw_b);
#pragma unroll
    for (int i = 0; i < PPW; ++i) {
        if (!valid[i]) continue;
        const int li = bi[i] * 8 + (lane >> 2);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int lj = bj[i] * 8 + 2 * (lane & 3) + c;
            out[lj * sh.tw_a + li] = zmake(acc[0][i][0][c], dpair[i] ? 0.0 : acc[0][i][1][c]);
        }
    }
}

// One warp per entry of C: lane l adds chunks l, l+32, ... in order, then a
// fixed shuffle tree adds the lanes.
__global__ void gram_reduce_kernel(z64* __restrict__ C, int64_t ldc, int kA, int kB, GramShape sh,
                                   const z64* __restrict__ partial, z64 alpha, z64 beta,
                                   const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    const int lane = threadIdx.x & 31;
    const int64_t entry = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (entry >= (int64_t)kA * kB) return;
    const int i = (int)(entry % kA), j = (int)(entry / kA);
    int si = i, sj = j;
    bool mirror = false;
    if (sh.hermitian && i > j) { si = j; sj = i; mirror = true; }
    const int ti = si / sh.tw_a, tj = sj / sh.tw_b;
    const int li = si - ti * sh.tw_a, lj = sj - tj * sh.tw_b;
    int tile;
    if (sh.hermitian) tile = (ti == tj) ? ti : off_tile_index(sh.nt_a, ti, tj);
    else tile = ti * sh.nt_b + tj;
    const size_t tile_entries = (size_t)(sh.tw_a * sh.tw_b);
    const z64* src = partial + (size_t)tile * sh.nchunks * tile_entries + lj * sh.tw_a + li;
    // A diagonal 8 x 8 block of a folded tile holds S = Re + Im: Re and Im
    // come back as the symmetric and antisymmetric parts of S. Folded tiles
    // are square (tw_a == tw_b).
    const bool sblock = sh.sdiag && ti == tj && (li >> 3) == (lj >> 3);
    const z64* srcT = partial + (size_t)tile * sh.nchunks * tile_entries + li * sh.tw_a + lj;
    z64 s = zmake(0.0, 0.0);
    for (int c = lane; c < sh.nchunks; c += 32) {
        z64 v = src[(size_t)c * tile_entries];
        if (sblock) v.y = srcT[(size_t)c * tile_entries].x;
        s.x += v.x;
        s.y += v.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s.x += __shfl_down_sync(0xffffffffu, s.x, off);
        s.y += __shfl_down_sync(0xffffffffu, s.y, off);
    }
    if (lane != 0) return;
    if (sblock) s = (li == lj) ? zmake(s.x, 0.0) : zmake(0.5 * (s.x + s.y), 0.5 * (s.x - s.y));
    if (mirror) s.y = -s.y;
    if (sh.hermitian && i == j) s.y = 0.0;
    z64 out = zmul(alpha, s);
    z64* dst = C + i + (int64_t)j * ldc;
    if (beta.x != 0.0 || beta.y != 0.0) zmac(out, beta, *dst);
    *dst = out;
}

// The autotuner's table: for a shape class (floor(log2 rows), max(kA, kB)), a
// shift of the row-chunk count. 0 (untuned) is one wave of CTAs; s > 0
// divides the chunk count by 2^s (longer chunks, fewer partial tiles),
// s < 0 multiplies it (shorter chunks, more CTAs). The chunk count sets the
// order of the reduction, so a shape's bits follow its table entry.
static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, int> g_tune_gram;

static int shape_class(int64_t rows) {
    int c = 0;
    while (c < 62 && ((int64_t)1 << (c + 1)) <= rows) ++c;
    return c;
}

static int tuned_gram_shift(int64_t rows, int kA, int kB) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_gram.find({shape_class(rows), kA > kB ? kA : kB});
    return it == g_tune_gram.end() ? 0 : it->second;
}

static GramShape gram_shape(int64_t rows, int kA, int kB, int hermitian, int ctas_per_sm) {
    GramShape sh{};
    auto tile_width = [](int k) { int w = k < G_TILE ? k : G_TILE; return (w + 7) / 8 * 8; };
    sh.tw_a = tile_width(kA);
    sh.tw_b = tile_width(kB);
    sh.nt_a = (kA + sh.tw_a - 1) / sh.tw_a;
    sh.nt_b = (kB + sh.tw_b - 1) / sh.tw_b;
    sh.hermitian = hermitian;
    sh.ntiles = hermitian ? sh.nt_a * (sh.nt_a + 1) / 2 : sh.nt_a * sh.nt_b;
    // Chunks along the rows: enough for the launch with fewer tiles to fill
    // the GPU by itself (the other then runs in whole or near-whole waves).
    // A Hermitian Gram of two tile columns has two diagonal tiles but one
    // off-diagonal tile; sizing for the larger launch would leave half the
    // SMs idle in the smaller.
    int smallest_launch = sh.ntiles;
    if (hermitian && sh.nt_a > 1) {
        const int off = sh.nt_a * (sh.nt_a - 1) / 2;
        smallest_launch = off < sh.nt_a ? off : sh.nt_a;
    }
    const int64_t stages = (rows + GS_ROWS - 1) / GS_ROWS;
    int64_t target = (int64_t)sm_count() * ctas_per_sm / smallest_launch;
    const int shift = tuned_gram_shift(rows, kA, kB);
    if (shift > 0) target >>= shift;
    else if (shift < 0) target <<= -shift;
    if (target < 1) target = 1;
    if (target > stages) target = stages;
    if (target < 1) target = 1;
    int64_t chunk_stages = stages > 0 ? (stages + target - 1) / target : 1;
    sh.chunk_rows = chunk_stages * GS_ROWS;
    sh.nchunks = rows > 0 ? (int)((rows + sh.chunk_rows - 1) / sh.chunk_rows) : 0;
    return sh;
}

// The consumer slots' blocks. Full tiles: row-major. Folded diagonal tiles
// with at least as many warps as block rows: warp w < nb takes the diagonal
// block (w, w) in slot 0 (one MMA a k-step, S-coded) and then blocks of its
// own block row (sharing the A fragment); the rest fill the free slots in
// order. At k = 64 (eight block rows, three blocks a warp, twelve warps) this
// gives warps 0-7 one diagonal and two off-diagonal blocks and warps 8-11
// three off-diagonal ones, so each sub-partition (warps w, w + 4, w + 8)
// issues 5 + 5 + 6 = 16 MMAs a k-step. Smaller tiles without that many warps
// compute their diagonal blocks like any other.
static void build_pair_table(GramLaunch& ln) {
    for (int i = 0; i < 64; ++i) ln.pi[i] = ln.pj[i] = -1;
    ln.sdiag = 0;
    std::vector<std::pair<int, int>> order;
    if (ln.diag) {
        for (int I = 0; I < ln.nb_a; ++I)
            for (int J = I; J < ln.nb_a; ++J) order.push_back({I, J});
    } else {
        for (int I = 0; I < ln.nb_a; ++I)
            for (int J = 0; J < ln.nb_b; ++J) order.push_back({I, J});
    }
    if (ln.diag && ln.consumers >= ln.nb_a) {
        ln.sdiag = 1;
        std::vector<std::vector<std::pair<int, int>>> warps(ln.consumers);
        std::vector<std::pair<int, int>> off;
        for (auto& p : order)
            if (p.first != p.second) off.push_back(p);
        std::vector<bool> used(off.size(), false);
        for (int w = 0; w < ln.nb_a; ++w) {
            warps[w].push_back({w, w});
            for (size_t q = 0; q < off.size() && (int)warps[w].size() < ln.ppw; ++q)
                if (!used[q] && off[q].first == w) { warps[w].push_back(off[q]); used[q] = true; }
        }
        for (int w = 0; w < ln.consumers; ++w)
            for (size_t q = 0; q < off.size() && (int)warps[w].size() < ln.ppw; ++q)
                if (!used[q]) { warps[w].push_back(off[q]); used[q] = true; }
        for (int w = 0; w < ln.consumers; ++w)
            for (size_t i = 0; i < warps[w].size(); ++i) {
                ln.pi[w * ln.ppw + i] = (signed char)warps[w][i].first;
                ln.pj[w * ln.ppw + i] = (signed char)warps[w][i].second;
            }
        return;
    }
    for (size_t q = 0; q < order.size() && q < 64; ++q) {
        ln.pi[q] = (signed char)order[q].first;
        ln.pj[q] = (signed char)order[q].second;
    }
}

static GramLaunch gram_launch(const GramShape& sh, bool diag) {
    GramLaunch ln{};
    ln.diag = diag;
    ln.nb_a = sh.tw_a / 8;
    ln.nb_b = diag ? ln.nb_a : sh.tw_b / 8;
    if (diag) {
        ln.ntiles = sh.nt_a;
        ln.npairs = ln.nb_a * (ln.nb_a + 1) / 2;
    } else {
        ln.ntiles = sh.hermitian ? sh.nt_a * (sh.nt_a - 1) / 2 : sh.nt_a * sh.nt_b;
        ln.npairs = ln.nb_a * ln.nb_b;
    }
    // Blocks per warp: three (at most 12 consumer warps), two (at most 16),
    // four (a full 64 x 64 tile: 16 warps, each half a block row) or eight
    // (at most 8), whichever leaves no warp with a block to spare.
    if (ln.npairs % 3 == 0 && ln.npairs <= 36) ln.ppw = 3;
    else if (ln.npairs <= 32) ln.ppw = 2;
    else if (ln.npairs == 64) ln.ppw = 4;
    else ln.ppw = 8;
    ln.consumers = (ln.npairs + ln.ppw - 1) / ln.ppw;
    build_pair_table(ln);
    ln.stage_bytes = GS_BOXES * (sh.tw_a * 128 + (diag ? 0 : sh.tw_b * 128));
    ln.stages = diag ? 6 : 3;
    while (ln.stages > 2 && (size_t)ln.stages * ln.stage_bytes > 200 * 1024) --ln.stages;
    ln.smem = (size_t)ln.stages * ln.stage_bytes + 2 * ln.stages * sizeof(uint64_t) + 1024;
    return ln;
}

template <int PPW>
static int set_gram_attr(size_t smem) {
    FB_CUDA(cudaFuncSetAttribute(gram_dmma_kernel<PPW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "cudaFuncSetAttribute(gram_dmma_kernel)");
    return FB_OK;
}

// CTAs of the larger launch that fit on one SM at once: the chunk count is
// chosen from it so that one wave covers the GPU.
static int gram_ctas_per_sm(int64_t rows, int kA, int kB, bool hermitian) {
    GramShape sh = gram_shape(rows, kA, kB, hermitian ? 1 : 0, 1);
    // The larger of the two launches sets the pace: the diagonal tile when
    // there is only one, the off-diagonal tiles otherwise.
    GramLaunch ln = gram_launch(sh, hermitian && sh.nt_a == 1);
    int threads = (ln.consumers + 1) * 32;
    int by_smem = (int)((227 * 1024) / (ln.smem + 1024));
    int by_threads = 2048 / threads;
    int by_regs = 65536 / (threads * 128);  // the consumers' register count, from ptxas
    int n = by_smem;
    if (by_threads < n) n = by_threads;
    if (by_regs < n) n = by_regs;
    return n < 1 ? 1 : n;
}

template <int PPW>
static int launch_gram_dmma(const CUtensorMap& ma, const CUtensorMap& mb, int64_t rows, const GramShape& sh,
                            const GramLaunch& ln, z64* partial, cudaStream_t stream, const ChainStatus* st, int gate,
                            int chunk0, int chunk1) {
    FB_TRY(set_gram_attr<PPW>(ln.smem));
    dim3 grid(ln.ntiles, chunk1 - chunk0);
    gram_dmma_kernel<PPW><<<grid, (ln.consumers + 1) * 32, ln.smem, stream>>>(ma, mb, rows, sh, ln, partial, st, gate,
                                                                              chunk0);
    FB_LAUNCHED("gram_dmma_kernel");
    return FB_OK;
}

static size_t gram_workspace_bytes(const GramShape& sh) {
    return (size_t)sh.ntiles * (size_t)(sh.nchunks > 0 ? sh.nchunks : 1) * (size_t)(sh.tw_a * sh.tw_b) * sizeof(z64);
}

static GramShape gram_plan(int64_t rows, int kA, int kB, bool hermitian) {
    return gram_shape(rows, kA, kB, hermitian ? 1 : 0, gram_ctas_per_sm(rows, kA, kB, hermitian));
}

// The row chunks of a Gram: chunk c covers rows [c chunk_rows, (c + 1)
// chunk_rows). Each chunk's partial tiles depend on its rows alone, so the
// partials of a chunk range can be computed as soon as those rows are in
// place (a pipelined upload), with the same bits as one launch over all.
void gram_chunks(int64_t rows, int kA, int kB, bool hermitian, int64_t* chunk_rows, int* nchunks) {
    const GramShape sh = gram_plan(rows, kA, kB, hermitian);
    *chunk_rows = sh.chunk_rows;
    *nchunks = sh.nchunks;
}

// The partial tiles of chunks [chunk0, chunk1).
int gram_partials_enqueue(const z64* A, int64_t lda, const z64* B, int64_t ldb, int64_t rows, int kA, int kB,
                          bool hermitian, void* workspace, size_t workspace_bytes, cudaStream_t stream,
                          const ChainStatus* st, int gate, int chunk0, int chunk1) {
    GramShape sh = gram_plan(rows, kA, kB, hermitian);
    size_t need = gram_workspace_bytes(sh);
    if (workspace_bytes < need || workspace == nullptr) {
        set_error(FB_ENOMEM, "gram: workspace of %zu bytes is smaller than the %zu bytes this shape needs",
                  workspace_bytes, need);
        return FB_ENOMEM;
    }
    if (chunk0 < 0) chunk0 = 0;
    if (chunk1 > sh.nchunks) chunk1 = sh.nchunks;
    if (chunk0 >= chunk1) return FB_OK;
    z64* partial = static_cast<z64*>(workspace);
    CUtensorMap ma, mb;
    FB_TRY(encode_panel_map(&ma, A, rows, kA, lda, sh.tw_a));
    FB_TRY(encode_panel_map(&mb, B, rows, kB, ldb, sh.tw_b));
    if (hermitian) sh.sdiag = gram_launch(sh, true).sdiag;
    const bool launches[2] = {hermitian, !hermitian || sh.nt_a > 1};
    for (int d = 0; d < 2; ++d) {
        if (!launches[d]) continue;
        GramLaunch ln = gram_launch(sh, d == 0);
        if (ln.ntiles == 0) continue;
        int status;
        switch (ln.ppw) {
            case 2: status = launch_gram_dmma<2>(ma, mb, rows, sh, ln, partial, stream, st, gate, chunk0, chunk1); break;
            case 3: status = launch_gram_dmma<3>(ma, mb, rows, sh, ln, partial, stream, st, gate, chunk0, chunk1); break;
            case 4: status = launch_gram_dmma<4>(ma, mb, rows, sh, ln, partial, stream, st, gate, chunk0, chunk1); break;
            default: status = launch_gram_dmma<8>(ma, mb, rows, sh, ln, partial, stream, st, gate, chunk0, chunk1); break;
        }
        FB_TRY(status);
    }
    return FB_OK;
}

// C <- alpha (sum of the partial tiles of every chunk) + beta C.
int gram_reduce_enqueue(z64* C, int64_t ldc, int64_t rows, int kA, int kB, bool hermitian, z64 alpha, z64 beta,
                        void* workspace, cudaStream_t stream, const ChainStatus* st, int gate) {
    GramShape sh = gram_plan(rows, kA, kB, hermitian);
    if (hermitian && sh.nchunks > 0) sh.sdiag = gram_launch(sh, true).sdiag;
    z64* partial = static_cast<z64*>(workspace);
    int64_t entries = (int64_t)kA * kB;
    int64_t threads = entries * 32;
    int block = 256;
    int64_t grid = (threads + block - 1) / block;
    gram_reduce_kernel<<<(unsigned)grid, block, 0, stream>>>(C, ldc, kA, kB, sh, partial, alpha, beta, st, gate);
    FB_LAUNCHED("gram_reduce_kernel");
    return FB_OK;
}

// Shared by fb_zgram and the orthonormalization chain.
int gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, const z64* B, int64_t ldb,
                 int64_t rows, int kA, int kB, z64 alpha, z64 beta, bool hermitian,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream,
                 const ChainStatus* st, int gate) {
    const GramShape sh = gram_plan(rows, kA, kB, hermitian);
    const size_t need = gram_workspace_bytes(sh);
    if (workspace_bytes < need || workspace == nullptr) {
        set_error(FB_ENOMEM, "gram: workspace of %zu bytes is smaller than the %zu bytes this shape needs",
                  workspace_bytes, need);
        return FB_ENOMEM;
    }
    FB_TRY(gram_partials_enqueue(A, lda, B, ldb, rows, kA, kB, hermitian, workspace, workspace_bytes, stream, st,
                                 gate, 0, sh.nchunks));
    return gram_reduce_enqueue(C, ldc, rows, kA, kB, hermitian, alpha, beta, workspace, stream, st, gate);
}

size_t gram_workspace_size(int64_t rows, int kA, int kB, bool hermitian) {
    return gram_workspace_bytes(gram_plan(rows, kA, kB, hermitian));
}

// Scratch for fb_zgram_static, the entry point for callers that cannot
// allocate device memory. It is an ordinary global of this module, so every
// GPU that loads the library holds these bytes until the process exits. The
// partial tiles it holds are written by each call before that call reads
// them, so nothing in it has to start at zero.
constexpr size_t GRAM_STATIC_SCRATCH_BYTES = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_gram_static_scratch[GRAM_STATIC_SCRATCH_BYTES];

// The device address of g_gram_static_scratch on the current device. Host
// code sees the symbol's name only as a host-side stand-in, so the address is
// asked of the runtime once per device (with that device current) and cached.
static int gram_static_scratch(void** out) {
    static std::mutex mu;
    static std::vector<void*> addresses;
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    if ((int)addresses.size() <= dev) addresses.resize(dev + 1, nullptr);
    if (addresses[dev] == nullptr) {
        void* p = nullptr;
        FB_CUDA(cudaGetSymbolAddress(&p, g_gram_static_scratch), "cudaGetSymbolAddress(g_gram_static_scratch)");
        addresses[dev] = p;
    }
    *out = addresses[dev];
    return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zgram_workspace_size(int64_t rows, int kA, int kB, int hermitian, size_t* bytes) {
    if (!bytes) { set_error(FB_EINVAL, "fb_zgram_workspace_size: bytes is NULL"); return FB_EINVAL; }
    if (rows < 0 || kA < 0 || kB < 0) { set_error(FB_EINVAL, "fb_zgram_workspace_size: negative size"); return FB_EINVAL; }
    if (hermitian && kA != kB) { set_error(FB_EDIM, "fb_zgram_workspace_size: a Hermitian Gram is square"); return FB_EDIM; }
    *bytes = (kA == 0 || kB == 0) ? 0 : gram_workspace_size(rows, kA, kB, hermitian != 0);
    return FB_OK;
}

int fb_zgram(fb_z128* C, int64_t ldc, const fb_z128* A, int64_t lda, const fb_z128* B, int64_t ldb,
             int64_t rows, int kA, int kB, fb_z128 alpha, fb_z128 beta,
             void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (rows < 0 || kA < 0 || kB < 0) {
        set_error(FB_EDIM, "cannot accumulate a product with negative sizes (rows=%lld, kA=%d, kB=%d)",
                  (long long)rows, kA, kB);
        return FB_EDIM;
    }
    if (kA == 0 || kB == 0) return FB_OK;
    if (!C || (rows > 0 && (!A || !B))) { set_error(FB_EINVAL, "fb_zgram: NULL matrix"); return FB_EINVAL; }
    if (ldc < kA || (rows > 0 && (lda < rows || ldb < rows))) {
        set_error(FB_EDIM, "fb_zgram: a leading dimension is smaller than the column it holds (ldc=%lld for %d rows, lda=%lld, ldb=%lld for %lld rows)",
                  (long long)ldc, kA, (long long)lda, (long long)ldb, (long long)rows);
        return FB_EDIM;
    }
    if (((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15) {
        set_error(FB_EINVAL, "fb_zgram: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    bool hermitian = (A == B) && (lda == ldb) && (kA == kB);
    z64 a = zmake(alpha.re, alpha.im), b = zmake(beta.re, beta.im);
    return gram_enqueue(reinterpret_cast<z64*>(C), ldc, reinterpret_cast<const z64*>(A), lda,
                        reinterpret_cast<const z64*>(B), ldb, rows, kA, kB, a, b, hermitian,
                        workspace, workspace_bytes, stream_of(queue), nullptr, GATE_ALWAYS);
}

int fb_zgram_static(fb_z128* C, int64_t ldc, const fb_z128* A, int64_t lda, const fb_z128* B, int64_t ldb,
                    int64_t rows, int kA, int kB, fb_z128 alpha, fb_z128 beta, fb_queue_t queue) {
    if (rows < 0 || kA < 0 || kB < 0) {
        set_error(FB_EDIM, "cannot accumulate a product with negative sizes (rows=%lld, kA=%d, kB=%d)",
                  (long long)rows, kA, kB);
        return FB_EDIM;
    }
    if (kA == 0 || kB == 0) return FB_OK;
    if (!C || (rows > 0 && (!A || !B))) { set_error(FB_EINVAL, "fb_zgram_static: NULL matrix"); return FB_EINVAL; }
    if (ldc < kA || (rows > 0 && (lda < rows || ldb < rows))) {
        set_error(FB_EDIM, "fb_zgram_static: a leading dimension is smaller than the column it holds (ldc=%lld for %d rows, lda=%lld, ldb=%lld for %lld rows)",
                  (long long)ldc, kA, (long long)lda, (long long)ldb, (long long)rows);
        return FB_EDIM;
    }
    if (((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15) {
        set_error(FB_EINVAL, "fb_zgram_static: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    const bool hermitian = (A == B) && (lda == ldb) && (kA == kB);
    const size_t need = gram_workspace_size(rows, kA, kB, hermitian);
    if (need > GRAM_STATIC_SCRATCH_BYTES) {
        set_error(FB_ENOMEM,
                  "fb_zgram_static: a %d x %d Gram over %lld rows needs %zu bytes of scratch, more than the %zu bytes "
                  "this entry point holds; use fb_zgram with a workspace of fb_zgram_workspace_size bytes",
                  kA, kB, (long long)rows, need, GRAM_STATIC_SCRATCH_BYTES);
        return FB_ENOMEM;
    }
    void* scratch = nullptr;
    FB_TRY(gram_static_scratch(&scratch));
    z64 a = zmake(alpha.re, alpha.im), b = zmake(beta.re, beta.im);
    return gram_enqueue(reinterpret_cast<z64*>(C), ldc, reinterpret_cast<const z64*>(A), lda,
                        reinterpret_cast<const z64*>(B), ldb, rows, kA, kB, a, b, hermitian,
                        scratch, GRAM_STATIC_SCRATCH_BYTES, stream_of(queue), nullptr, GATE_ALWAYS);
}

int fb_tune_set_gram_chunks(int64_t rows, int k, int shift) {
    if (rows < 1 || k < 1 || shift < -3 || shift > 8) {
        set_error(FB_EINVAL, "fb_tune_set_gram_chunks: rows %lld, k %d, shift %d (shift in [-3, 8])", (long long)rows, k,
                  shift);
        return FB_EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_tune_mu);
    if (shift == 0) g_tune_gram.erase({shape_class(rows), k});
    else g_tune_gram[{shape_class(rows), k}] = shift;
    return FB_OK;
}

int fb_tune_get_gram_chunks(int64_t rows, int k, int* shift) {
    if (rows < 1 || k < 1 || !shift) { set_error(FB_EINVAL, "fb_tune_get_gram_chunks: bad argument"); return FB_EINVAL; }
    *shift = tuned_gram_shift(rows, k, k);
    return FB_OK;
}

int fb_tune_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_gram.clear();
    return FB_OK;
}

}  // extern "C"
