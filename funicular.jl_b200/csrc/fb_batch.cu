// cholqr2! (src/panelblas.jl:130-139) of many independent tall-skinny
// instances of uneven N and k <= 64 in one persistent kernel launch: the
// batched range finder's orthonormalizations, with every pass of every
// instance (Gram, Cholesky with the shifted retry, solve plan, triangular
// solve, the optional third pass) run by one grid of CTAs, one per SM, that
// take jobs from a ticket counter until none are left.
//
// Jobs. Each instance's rows are cut into chunks (at most 64, each holding at
// least 4 MB of Y). Tickets run through six phases: the Gram chunks of pass 1
// of every instance, then the solve chunks of pass 1, the Gram chunks of pass
// 2, the solves of pass 2, and the Gram and solve chunks of a third pass
// (which return at once unless the instance needs one). Within a phase the
// instances come largest first. A Gram job writes its chunk's partial Gram
// matrix; the CTA that finishes the last Gram chunk of an instance's pass
// (an arrival counter) adds the partials in chunk order, factors, multiplies
// R, builds the solve plan and releases the instance's "factor ready" flag. A
// solve job waits for that flag; the Gram job of the next pass waits for the
// solve of its own chunk (a per-chunk flag). Every wait is on a job with a
// smaller ticket, which a running CTA holds, so every wait ends; each still
// gives up after 2 s, marks the instance's status and stops the kernel.
//
// Gram job: a copy warp streams the chunk through shared memory in stages of
// about 33 KB (32 rows at k = 64 up to 256 rows at k <= 8) with bulk copies
// (cp.async.bulk, one per column and stage, no tensor map, so an instance
// needs no host-encoded descriptor), into a ring of four or more stages
// guarded by mbarriers (135 KB; 190 KB at k <= 32, whose fragments are
// small). Twelve warps multiply on the FP64 tensor cores (mma m8n8k4 on the
// real form of the complex product, as the chain's Gram kernel): the
// upper triangle of 8 x 8 blocks is split into sets of block rows
// {g, nb-1-g}, which carry equal MMA counts, each set owned by 12, 6, 4 or 3
// warps that deal out the chunk's k-steps among them; a diagonal block costs
// one MMA a k-step (S = Re + Im), the others two. The warps of a set add their
// sums in a fixed order, so the bits of an instance depend only on its shape.
// A CTA has sixteen warps (four per SM sub-partition, 128 registers each):
// twelve multiply, one copies, three wait out the Gram jobs.
//
// Solve jobs: the product by inv(R), the blocked solve or substitution, as
// the plan says (the chain's paths, restated for a chunk of rows and the
// CTA's sixteen warps). Up to k = 32 the product by inv(R) reads its rows
// through the same ring (15 warps multiply), which keeps up to 190 KB in
// flight where one warp's own loads would not; wider panels load straight
// into registers. Data another CTA wrote during the launch is read through
// L2 (ld.global.cg), never from a possibly stale L1 line.
#include <algorithm>
#include <memory>
#include <vector>

#include "fb_factor.cuh"
#include "fb_tma.cuh"

namespace fb {

constexpr int PB_WARPS = 16;                         // warps of a CTA: four on each SM sub-partition
constexpr int PB_THREADS = PB_WARPS * 32;
constexpr int PB_GRAM_WARPS = 12;                    // multiply in a Gram job; warp 12 issues its copies
constexpr int PB_COPY_WARP = PB_GRAM_WARPS;
constexpr int PB_SR_MAX = 256;                       // rows per Gram stage at k <= 8; chunks are multiples
constexpr int PB_RING = 4 * 64 * (32 * 16 + 16);     // ring bytes: four stages of 32 rows at k = 64
constexpr int PB_MAX_STAGES = 16;
constexpr int PB_MAX_CHUNKS = 64;
constexpr int PB_MAX_INST = 384;                     // instances per launch (kernel parameter space)
constexpr int PB_PHASES = 6;
constexpr int64_t PB_CHUNK_BYTES = 4 << 20;          // a chunk holds at least this much of Y
constexpr int PB_STAGED_SOLVE_KMAX = 32;             // the product by inv(R) reads its rows through the ring up to here
constexpr int PB_REGION = TR_KMAX * TR_PREP_LD * 16; // one k x k matrix of the factor step, padded
// Dynamic shared memory: the solve's B fragments, then the ring (which the
// blocked solve's transpose buffers use when no copies run). The factor step
// overlays both with its two k x k regions. Gram jobs leave the fragments in
// place, so a CTA reuses them across its jobs until it runs a factor step.
constexpr int PB_RING_OFF = TR_FRAG_DOUBLES * 8;
constexpr int PB_SMEM = PB_RING_OFF + PB_RING;
// At k <= 32 the fragments take at most 18 KB, so the ring of that width's
// Gram and solve jobs starts right after them and takes the rest: five or
// more slots instead of three or four, which is what their HBM-bound sweeps
// need in flight. Such a job overwrites the fragment area of wider panels,
// which the caller then forgets.
constexpr int PB_SMALL_FRAG_BYTES = 32 * 8 * 9 * 8;
constexpr int PB_SMALL_RING = PB_SMEM - PB_SMALL_FRAG_BYTES;
static_assert(2 * PB_REGION <= PB_SMEM, "factor regions exceed shared memory");
static_assert(PB_WARPS * TR_BUF * 16 <= PB_RING, "transpose buffers exceed the ring");

// Per instance, in the zeroed counter block (ints): arrivals of Gram chunks
// by pass, factor-ready flags by pass, the last solved pass of each chunk.
constexpr int PB_ARRIVE = 0, PB_READY = 4, PB_SOLVED = 8;
constexpr int PB_COUNTER_INTS = 128;
static_assert(PB_SOLVED + PB_MAX_CHUNKS <= PB_COUNTER_INTS, "counter block");

struct PbInst {
    z64* Y;
    z64* R;
    char* scratch;
    int* counters;
    ChainStatus* st;
    int64_t ldy, ldr, N;
    int k, nchunks, chunk_rows, first_job;
};

struct PbArgs {
    unsigned* ticket;      // ticket counter, then the stop word
    int count, jobs;       // instances of this launch, jobs per phase
    int zero, pad;
    PbInst inst[PB_MAX_INST];
};
static_assert(sizeof(PbArgs) <= 32764, "kernel parameters past the 32764-byte limit");

__host__ __device__ inline size_t pb_align(size_t n) { return (n + 255) / 256 * 256; }
__host__ __device__ inline int pb_kp(int k) { return (k + 7) / 8 * 8; }
__host__ __device__ inline int pb_npairs(int k) { const int nb = pb_kp(k) / 8; return nb * (nb + 1) / 2; }

// Rows of a Gram stage at nb 8-column blocks: about 33 KB of Y a stage at any
// width (32 rows at k = 64, 256 at k <= 8), so narrow panels pay the ring's
// barrier handshakes per as many bytes as wide ones. A column of a Gram stage
// takes its rows plus 16 bytes of padding: with a k-step's two rows 4 apart
// (rows r and r + 4 of a group of 8), the half warp's eight columns and two
// rows land in eight different 16-byte bank groups.
__host__ __device__ constexpr int pb_stage_rows(int nb) { return 32 * (8 / nb); }
__host__ __device__ constexpr int pb_col_bytes(int nb) { return pb_stage_rows(nb) * 16 + 16; }
// Solve stages pad a column by 64 bytes instead: a quarter warp's A-fragment
// load takes 4 rows of two adjacent columns, which this puts in the two
// halves of the bank space.
__host__ __device__ constexpr int pb_solve_col_bytes(int nb) { return pb_stage_rows(nb) * 16 + 64; }

// An instance's scratch: solve plan, B fragments, U, Ra (R1), Rb (R2 R1), and
// the chunks' partial Gram matrices (8 x 8 blocks of the upper triangle,
// row-major, 64 entries each).
struct PbLayout {
    size_t plan, frag, U, Ra, Rb, partial, total;
};

__host__ __device__ inline PbLayout pb_layout(int k, int nchunks) {
    PbLayout L{};
    const size_t kk = (size_t)pb_kp(k) * pb_kp(k) * 16;
    size_t off = 0;
    L.plan = off; off += pb_align(TR_PLAN_BYTES);
    L.frag = off; off += pb_align((size_t)TR_FRAG_DOUBLES * 8);
    L.U = off; off += pb_align(kk);
    L.Ra = off; off += pb_align(kk);
    L.Rb = off; off += pb_align(kk);
    L.partial = off; off += pb_align((size_t)nchunks * pb_npairs(k) * 64 * 16);
    L.total = off;
    return L;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until *flag >= want; false after WAIT_LIMIT_NS.
__device__ bool wait_flag(const int* flag, int want) {
    if (ld_acquire(flag) >= want) return true;
    const uint64_t t0 = globaltimer_ns();
    while (ld_acquire(flag) < want) {
        __nanosleep(200);
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) return false;
    }
    return true;
}

// One contiguous run of bytes global -> shared, completion counted on bar.
// No multicast: the bytes go to this CTA alone.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Orders this thread's generic-proxy accesses before later async-proxy
// (bulk copy) accesses, in shared and in global memory.
__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }

// Named barrier over a Gram job's multiplying warps.
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, %0;" ::"n"(PB_GRAM_WARPS * 32) : "memory"); }

// Where a wait gave up, as the status records it.
enum PbWaitSite : int {
    WAIT_GRAM_STAGE = 1, WAIT_GRAM_SLOT = 2, WAIT_SOLVE_STAGE = 3, WAIT_SOLVE_SLOT = 4,
    WAIT_READY = 5, WAIT_SOLVED = 6,
};

// Marks a wait that gave up: the instance's status says where, and the
// kernel stops taking jobs.
__device__ void pb_timeout(const PbArgs& a, ChainStatus* st, int site) {
    atomicCAS(&st->timeout, 0, site);
    atomicExch(a.ticket + 1, 1u);
}

// ---- Gram jobs ---------------------------------------------------------------

// The blocks of the upper triangle that the set of block rows {G0, NB-1-G0}
// owns: row R0 from its diagonal block on, then row R1 likewise. Both rows
// together carry 2 NB MMAs a k-step (NB for a lone middle row).
template <int NB, int G0>
struct GramSet {
    static constexpr int R0 = G0, R1 = NB - 1 - G0;
    static constexpr bool TWO = R1 > R0;
    static constexpr int NO = NB - R0;              // column blocks R0..NB-1: own parts a k-step loads
    static constexpr int OFF0 = NB - 1 - R0;        // off-diagonal blocks of row R0
    static constexpr int OFF1 = TWO ? NB - 1 - R1 : 0;
    static constexpr int B1 = 2 + 4 * OFF0;         // where row R1's sums start
    static constexpr int NACC = B1 + (TWO ? 2 + 4 * OFF1 : 0);
};

// One k-step (two complex rows, 4 apart) of the set's blocks. p: this lane's
// own part of column block 0 in the stage, at the k-step's rows; odelta: from there to
// the lane's other part; flip: the sign bit that turns the other part into
// the J W entry. Sums: a diagonal block S (2 doubles: D[li][lj], lj = 2 (lane
// & 3) + 0/1), an off-diagonal block Re then Im (4 doubles).
template <int NB, int G0>
__device__ __forceinline__ void gram_kstep(const unsigned char* p, int odelta, unsigned long long flip,
                                           double (&acc)[GramSet<NB, G0>::NACC]) {
    using S = GramSet<NB, G0>;
    constexpr int BLK = 8 * pb_col_bytes(NB);   // bytes from one 8-column block to the next
    double own[S::NO];
#pragma unroll
    for (int b = 0; b < S::NO; ++b) own[b] = *reinterpret_cast<const double*>(p + (S::R0 + b) * BLK);
    const double aim0 = __longlong_as_double(
        __double_as_longlong(*reinterpret_cast<const double*>(p + S::R0 * BLK + odelta)) ^ flip);
    dmma_884(acc[0], acc[1], own[0] + aim0, own[0]);
#pragma unroll
    for (int j = 0; j < S::OFF0; ++j) {
        dmma_884(acc[2 + 4 * j], acc[3 + 4 * j], own[0], own[1 + j]);
        dmma_884(acc[4 + 4 * j], acc[5 + 4 * j], aim0, own[1 + j]);
    }
    if constexpr (S::TWO) {
        constexpr int D1 = S::R1 - S::R0;
        const double are1 = own[D1];
        const double aim1 = __longlong_as_double(
            __double_as_longlong(*reinterpret_cast<const double*>(p + S::R1 * BLK + odelta)) ^ flip);
        dmma_884(acc[S::B1], acc[S::B1 + 1], are1 + aim1, are1);
#pragma unroll
        for (int j = 0; j < S::OFF1; ++j) {
            dmma_884(acc[S::B1 + 2 + 4 * j], acc[S::B1 + 3 + 4 * j], are1, own[D1 + 1 + j]);
            dmma_884(acc[S::B1 + 4 + 4 * j], acc[S::B1 + 5 + 4 * j], aim1, own[D1 + 1 + j]);
        }
    }
}

// What the warps of a Gram job share.
struct GramCtx {
    unsigned char* ring;
    uint64_t* full;
    uint64_t* empty;
    int stage_bytes, nslots, kp, sr, col_bytes;   // sr: rows a stage
    int64_t row0, row1;
    z64* out;           // this chunk's partial: npairs blocks of 64 entries
    bool ok;            // every stage arrived
    int bad_site;       // the wait that gave up, if one did
};

// Waits for each stage of the chunk in turn, lets `work` multiply it, and
// hands the slot back. The k-steps of the chunk (SR / 2 a stage) are dealt to the
// WPG warps of a set in turn, h, h + WPG, ..., across stage boundaries; work
// gets the stage and its first k-step for this warp. A stage whose wait gave
// up is skipped (ok = false), but the loop still runs to the end so every
// multiplying warp passes the same named barriers. A short last stage whose
// row count is not a multiple of 8 gets zero rows up to the next multiple,
// so the k-steps across them add nothing.
template <int WPG, int SR, class Work>
__device__ __forceinline__ void gram_stages(GramCtx& c, uint32_t& full_par, int h, Work work) {
    const int lane = threadIdx.x & 31, ctid = threadIdx.x;
    const int64_t nst = (c.row1 - c.row0 + SR - 1) / SR;
    int slot = 0, q0 = h;
    for (int64_t s = 0; s < nst; ++s) {
        const bool got = c.ok && mbar_wait(&c.full[slot], (full_par >> slot) & 1u);
        full_par ^= 1u << slot;
        if (!got && c.ok) {
            c.ok = false;
            c.bad_site = WAIT_GRAM_STAGE;
        }
        const int valid = (int)min((int64_t)SR, c.row1 - (c.row0 + s * SR));
        unsigned char* base = c.ring + (size_t)slot * c.stage_bytes;
        if (valid & 7) {
            const int pad = 8 - (valid & 7);
            for (int e = ctid; e < c.kp * pad; e += PB_GRAM_WARPS * 32)
                *reinterpret_cast<z64*>(base + (e / pad) * c.col_bytes + (valid + e % pad) * 16) = zmake(0.0, 0.0);
            fence_proxy_async_all();
            compute_sync();
        }
        if (got) work(base, q0, (valid + 7) / 8 * 4);
        __syncwarp();
        if (lane == 0) mbar_arrive(&c.empty[slot]);
        if (++slot == c.nslots) slot = 0;
        q0 = (q0 + SR / 2 * WPG - SR / 2) % WPG;
    }
}

// A multiplying warp of set G0 (one of WPG that split the k-steps): its sums
// over the chunk, then the set's sums added in warp order and stored.
template <int NB, int G0, int WPG>
__device__ void gram_warp(GramCtx& c, uint32_t& full_par) {
    using S = GramSet<NB, G0>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = warp % WPG;
    const int col8 = lane >> 2, t = (lane >> 1) & 1, part = lane & 1;
    constexpr int SR = pb_stage_rows(NB);
    const int lane_off = col8 * pb_col_bytes(NB) + t * 64 + part * 8;
    const int odelta = part ? -8 : 8;
    const unsigned long long flip = part ? 0ull : 0x8000000000000000ull;
    double acc[S::NACC];
#pragma unroll
    for (int i = 0; i < S::NACC; ++i) acc[i] = 0.0;
    gram_stages<WPG, SR>(c, full_par, h, [&](const unsigned char* base, int q0, int nq) {
        const unsigned char* p = base + lane_off;
#pragma unroll (NB <= 4 ? 4 : 2)
        for (int q = q0; q < nq; q += WPG) gram_kstep<NB, G0>(p + (q >> 2) * 128 + (q & 3) * 16, odelta, flip, acc);
    });
    // The ring is free once every multiplying warp is past its last stage.
    double* comb = reinterpret_cast<double*>(c.ring);
    compute_sync();
    if (h > 0) {
#pragma unroll
        for (int i = 0; i < S::NACC; ++i) comb[(warp * 32 + i) * 32 + lane] = acc[i];
    }
    compute_sync();
    if (h != 0) return;
#pragma unroll 1
    for (int o = 1; o < WPG; ++o)
#pragma unroll
        for (int i = 0; i < S::NACC; ++i) acc[i] += comb[((warp + o) * 32 + i) * 32 + lane];
    if (!c.ok) {
#pragma unroll
        for (int i = 0; i < S::NACC; ++i) acc[i] = __longlong_as_double(0x7ff8000000000000ll);
    }
    const int e = (lane >> 2) * 8 + 2 * (lane & 3);
    auto block = [&](int bi, int bj) { return c.out + (bi * NB - bi * (bi - 1) / 2 + (bj - bi)) * 64 + e; };
    auto store2 = [&](z64* dst, z64 v0, z64 v1) {
        __stcg(dst, v0);
        __stcg(dst + 1, v1);
    };
    store2(block(S::R0, S::R0), zmake(acc[0], 0.0), zmake(acc[1], 0.0));
#pragma unroll
    for (int j = 0; j < S::OFF0; ++j)
        store2(block(S::R0, S::R0 + 1 + j), zmake(acc[2 + 4 * j], acc[4 + 4 * j]), zmake(acc[3 + 4 * j], acc[5 + 4 * j]));
    if constexpr (S::TWO) {
        store2(block(S::R1, S::R1), zmake(acc[S::B1], 0.0), zmake(acc[S::B1 + 1], 0.0));
#pragma unroll
        for (int j = 0; j < S::OFF1; ++j)
            store2(block(S::R1, S::R1 + 1 + j), zmake(acc[S::B1 + 2 + 4 * j], acc[S::B1 + 4 + 4 * j]),
                   zmake(acc[S::B1 + 3 + 4 * j], acc[S::B1 + 5 + 4 * j]));
    }
}

// The multiplying warps' share of a Gram job at nb = NB column blocks: sets
// of block rows {g, NB-1-g}, 12 / (number of sets) warps a set.
template <int NB>
__device__ void gram_compute(GramCtx& c, uint32_t& full_par) {
    constexpr int G = (NB + 1) / 2;
    constexpr int WPG = PB_GRAM_WARPS / G;
    static_assert(WPG * G == PB_GRAM_WARPS, "sets must share the warps evenly");
    const int g = (threadIdx.x >> 5) / WPG;
    if (g == 0) {
        gram_warp<NB, 0, WPG>(c, full_par);
    } else if (g == 1) {
        if constexpr (G > 1) gram_warp<NB, 1, WPG>(c, full_par);
    } else if (g == 2) {
        if constexpr (G > 2) gram_warp<NB, 2, WPG>(c, full_par);
    } else {
        if constexpr (G > 3) gram_warp<NB, 3, WPG>(c, full_par);
    }
}

// The copy warp: for every stage, waits for its slot to come back, announces
// the bytes on the slot's full barrier and copies each column's rows with one
// bulk copy per lane and column. ok = false if a wait gave up (no more copies
// are then issued; the multiplying warps' own waits give up too).
__device__ void gram_produce(const z64* Y, int64_t ldy, int k, GramCtx& c, uint32_t& empty_par, uint32_t& used,
                             int copy_site) {
    const int lane = threadIdx.x & 31;
    const int64_t nst = (c.row1 - c.row0 + c.sr - 1) / c.sr;
    int slot = 0;
    for (int64_t s = 0; s < nst; ++s) {
        const int64_t r = c.row0 + s * c.sr;
        const int valid = (int)min((int64_t)c.sr, c.row1 - r);
        const bool reuse = (used >> slot) & 1u;
        int good = 1;
        if (lane == 0 && c.ok) {
            if (reuse) good = mbar_wait(&c.empty[slot], (empty_par >> slot) & 1u);
            if (good) mbar_arrive_expect_tx(&c.full[slot], (uint32_t)(k * valid * 16));
        }
        good = __shfl_sync(0xffffffffu, good, 0) && c.ok;
        if (reuse) empty_par ^= 1u << slot;
        used |= 1u << slot;
        if (!good) {
            if (c.ok) c.bad_site = copy_site;
            c.ok = false;
        } else {
            __syncwarp();
            unsigned char* dst = c.ring + (size_t)slot * c.stage_bytes;
            for (int col = lane; col < k; col += 32)
                bulk_load(dst + col * c.col_bytes, Y + r + (int64_t)col * ldy, (uint32_t)valid * 16, &c.full[slot]);
        }
        if (++slot == c.nslots) slot = 0;
    }
}

// ---- the factor step ------------------------------------------------------------

// Run by the CTA whose Gram chunk arrived last for (instance, pass): adds the
// chunks' partials in chunk order, recovers the diagonal blocks' Re and Im
// from S, factors with the shifted retry, writes U, R (R1, R2 R1, or the
// caller's R on the last pass) and the solve plan, then releases the
// instance's ready flag for the pass. A pass that does not run (an earlier
// one failed, or a third pass nobody needs) only releases the flag.
__device__ void factor_step(const PbInst& I, int pass, unsigned char* smem, double* red) {
    __shared__ int s_run;
    ChainStatus* st = I.st;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int k = I.k, kp = pb_kp(k), nb = kp / 8, np = pb_npairs(k);
    const PbLayout L = pb_layout(k, I.nchunks);
    char* sc = I.scratch;
    if (tid == 0) {
        int run = __ldcg(&st->failed) == 0 && __ldcg(&st->timeout) == 0;
        if (pass == 3) run = run && (__ldcg(&st->shifted[1]) | __ldcg(&st->shifted[2]));
        s_run = run;
    }
    __syncthreads();
    if (s_run) {
        z64* Gs = reinterpret_cast<z64*>(smem);                  // kp x kp, row-major
        z64* W = reinterpret_cast<z64*>(smem + PB_REGION);       // k x k, row-major
        const z64* part = reinterpret_cast<const z64*>(sc + L.partial);
        const int entries = np * 64;
        constexpr int M = 8;   // entries a thread sums at once
        for (int e0 = tid; e0 < entries; e0 += nt * M) {
            z64 acc[M];
#pragma unroll
            for (int m = 0; m < M; ++m) acc[m] = zmake(0.0, 0.0);
            for (int c = 0; c < I.nchunks; ++c) {
                const z64* src = part + (size_t)c * entries;
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const int e = e0 + m * nt;
                    if (e < entries) {
                        const z64 v = __ldcg(src + e);
                        acc[m].x += v.x;
                        acc[m].y += v.y;
                    }
                }
            }
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const int e = e0 + m * nt;
                if (e >= entries) continue;
                int P = e >> 6, bi = 0;
                while (P >= nb - bi) { P -= nb - bi; ++bi; }
                const int bj = bi + P, li = (e >> 3) & 7, lj = e & 7;
                Gs[(bi * 8 + li) * kp + bj * 8 + lj] = acc[m];
            }
        }
        __syncthreads();
        // Diagonal blocks: Re and Im are the symmetric and antisymmetric parts of S.
        for (int e = tid; e < nb * 64; e += nt) {
            const int b = e >> 6, li = (e >> 3) & 7, lj = e & 7;
            if (li > lj) continue;
            const int i = b * 8 + li, j = b * 8 + lj;
            const double sij = Gs[i * kp + j].x, sji = Gs[j * kp + i].x;
            Gs[i * kp + j] = (li == lj) ? zmake(sij, 0.0) : zmake(0.5 * (sij + sji), 0.5 * (sij - sji));
        }
        __syncthreads();
        auto g = [&](int i, int j) { return Gs[i * kp + j]; };
        const double gnorm = hermitian_fro(g, k, red);
        bool shifted = false;
        double shift = 0.0;
        const bool ok = factor_shifted(g, k, I.N, gnorm, 0.0, W, shifted, shift);
        if (tid == 0) {
            st->shifted[pass] = shifted ? 1 : 0;
            st->shift[pass] = shift;
            st->norm[pass] = gnorm;
            if (!ok) st->failed = pass;
        }
        if (ok) {
            const bool third = pass == 2 && (shifted || __ldcg(&st->shifted[1]) != 0);
            const bool last = pass == 3 || (pass == 2 && !third);
            z64* U = reinterpret_cast<z64*>(sc + L.U);
            z64* Ra = reinterpret_cast<z64*>(sc + L.Ra);
            z64* Rb = reinterpret_cast<z64*>(sc + L.Rb);
            const z64* Rin = pass == 1 ? nullptr : (pass == 2 ? Ra : Rb);
            z64* Rout = last ? I.R : (pass == 1 ? Ra : Rb);
            const int64_t ldo = last ? I.ldr : k;
            for (int e = tid; e < k * k; e += nt) {
                const int j = e / k, i = e - j * k;
                z64 acc = zmake(0.0, 0.0);
                if (i <= j) {
                    if (Rin) {
                        for (int m = i; m <= j; ++m) zmac(acc, W[i * k + m], __ldcg(Rin + m + (int64_t)j * k));
                    } else {
                        acc = W[i * k + j];
                    }
                }
                Rout[i + j * ldo] = acc;
                U[i + (int64_t)j * k] = (i <= j) ? W[i * k + j] : zmake(0.0, 0.0);
            }
            // The solve plan of U: Rs over Gs, then inv(U) over W.
            constexpr int LD = TR_PREP_LD;
            z64* Rs = Gs;
            z64* Xs = W;
            for (int e = tid; e < kp * kp; e += nt) {
                const int i = e / kp, j = e - i * kp;
                z64 v = zmake(i == j ? 1.0 : 0.0, 0.0);
                if (i < k && j < k && i <= j) v = W[i * k + j];
                Rs[i * LD + j] = v;
            }
            __syncthreads();
            for (int e = tid; e < kp * kp; e += nt) {
                const int i = e / kp, j = e - i * kp;
                Xs[i * LD + j] = zmake(0.0, 0.0);
            }
            __syncthreads();
            solve_plan(Rs, Xs, k, reinterpret_cast<TrsmPlan*>(sc + L.plan), reinterpret_cast<double*>(sc + L.frag));
        }
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        st_release(I.counters + PB_READY + pass, 1);
    }
}

// ---- solve jobs ------------------------------------------------------------------

// Y inv(R) for the rows of a chunk that the copy warp streams through the
// ring (stages of c.sr rows, c.sr / 8 units of 8 rows a stage), so up to
// 135 KB of Y is in flight per SM whatever k is. The fifteen other warps
// pass every stage in order, as a Gram job's warps do: wait for it, load the
// rows of their own units (unit u belongs to warp u mod 15) in the MMA A
// layout, hand the slot back (fifteen hand-backs free it), then multiply as
// the chain's product by the inverse does: n-tile t needs k-steps 0..2t+1
// only, and the fragment loads of tile t wait for the result of tile t - 2.
// Since no slot is refilled before every warp has passed it, a warp always
// waits on the phase right after the one it saw last.
template <int NT>
__device__ void pb_solve_inverse(GramCtx& c, uint32_t& full_par, z64* Y, int64_t ldy, int64_t rows, int k,
                                 const double* frag, int zero) {
    constexpr int NS = 2 * NT;
    constexpr int NSW = PB_WARPS - 1;   // solving warps: all but the copy warp
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sw = warp < PB_COPY_WARP ? warp : warp - 1;
    const int cq = lane & 3, acol = cq >> 1, apart = lane & 1, rr = lane >> 2;
    const int ups = c.sr / 8;
    const int64_t nunits = (c.row1 - c.row0 + 7) / 8;
    const int64_t nst = (c.row1 - c.row0 + c.sr - 1) / c.sr;
    int slot = 0;
    for (int64_t st = 0; st < nst; ++st) {
        const bool got = c.ok && mbar_wait(&c.full[slot], (full_par >> slot) & 1u);
        full_par ^= 1u << slot;
        if (!got && c.ok) {
            c.ok = false;
            c.bad_site = WAIT_SOLVE_STAGE;
        }
        const unsigned char* stage = c.ring + (size_t)slot * c.stage_bytes;
        const int64_t first = st * ups, end = min(nunits, first + ups);
        // This warp's first unit in the stage: the least u >= first with u = sw (mod 15).
        int64_t u = first + ((sw - first % NSW) % NSW + NSW) % NSW;
        if (u >= end) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&c.empty[slot]);
        }
        for (; u < end; u += NSW) {
            const unsigned char* base = stage + ((int)(u - first) * 8 + rr) * 16 + apart * 8;
            double a[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int col = 2 * s + acol;
                a[s] = (got && col < k) ? *reinterpret_cast<const double*>(base + col * c.col_bytes) : 0.0;
            }
            if (u + NSW >= end) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&c.empty[slot]);
            }
            const int64_t row = c.row0 + u * 8 + rr;
            const bool live = row < rows;
            z64* yrow = Y + (live ? row : 0);
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
                if (live && col < k) __stcg(yrow + (int64_t)col * ldy, x);
                done2 = done1;
                done1 = x.x;
            }
        }
        if (++slot == c.nslots) slot = 0;
    }
}

// Y inv(R) with each warp loading its own units' rows straight into
// registers (a unit of 8 rows at a time, all sixteen warps): for wide panels
// (k > 32), where a unit's 4k loads already keep enough bytes in flight and
// its products are long, so the ring's stage-by-stage hand-backs only hold
// the warps back. Per unit as pb_solve_inverse.
template <int NT>
__device__ void pb_solve_inverse_direct(z64* Y, int64_t ldy, int64_t rows, int k, int64_t u0, int64_t u1,
                                        const double* frag, int zero) {
    constexpr int NS = 2 * NT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cq = lane & 3, acol = cq >> 1, apart = lane & 1, rr = lane >> 2;
    for (int64_t u = u0 + warp; u < u1; u += PB_WARPS) {
        const int64_t row = u * 8 + rr;
        const bool live = row < rows;
        z64* yrow = Y + (live ? row : 0);
        const double* y = reinterpret_cast<const double*>(yrow) + apart;
        double a[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int col = 2 * s + acol;
            a[s] = (live && col < k) ? __ldcg(y + 2 * (int64_t)col * ldy) : 0.0;
        }
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
            if (live && col < k) __stcg(yrow + (int64_t)col * ldy, x);
            done2 = done1;
            done1 = x.x;
        }
    }
}

// The blocked solve for the units [u0, u1), one unit a warp at a time:
// X_b = (Y_b - sum_{c<b} X_c R_cb) inv(R_bb), the solved blocks kept in the
// MMA A layout, results through the warp's transpose buffer, the Y blocks of
// the next two steps always in flight (slots swapped after each unit when
// the block count is odd).
template <int NBLK>
__device__ void pb_solve_blocked(z64* Y, int64_t ldy, int64_t rows, int k, int64_t u0, int64_t u1,
                                 const double* frag, z64* tbuf) {
    constexpr int NW = PB_WARPS;
    constexpr int NCH = 4;   // accumulator chains per n-tile
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    z64* buf = tbuf + warp * TR_BUF;
    const int rr = lane >> 2, cq = lane & 3, acol = cq >> 1, apart = lane & 1;
    auto load_y = [&](int64_t unit, int b, z64 (&v)[2]) {
        const int64_t row = unit * 8 + rr;
        const bool ok_row = unit < u1 && row < rows;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int col = TR_NB * b + 4 * t + cq;
            v[t] = (ok_row && col < k) ? __ldcg(Y + row + (int64_t)col * ldy) : zmake(0.0, 0.0);
        }
    };
    int64_t u = u0 + warp;
    z64 yq[2][2];
    load_y(u, 0, yq[0]);
    load_y(u + (1 / NBLK) * NW, 1 % NBLK, yq[1]);
    for (; u < u1; u += NW) {
        const int64_t row = u * 8 + rr;
        const bool live = row < rows;
        z64* yrow = Y + (live ? row : 0);
        double xa[NBLK][4];
#pragma unroll
        for (int b = 0; b < NBLK; ++b) {
            double acc[NCH][2][2];
            const int slot = b & 1;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                acc[0][t][0] = yq[slot][t].x;
                acc[0][t][1] = yq[slot][t].y;
#pragma unroll
                for (int h = 1; h < NCH; ++h) acc[h][t][0] = acc[h][t][1] = 0.0;
            }
            load_y(u + ((b + 2) / NBLK) * NW, (b + 2) % NBLK, yq[slot]);
#pragma unroll
            for (int c = 0; c < b; ++c) {
                const double* fp = frag + pair_index(c, b) * TR_FRAG + lane;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int h = (c * 4 + s) % NCH;
#pragma unroll
                    for (int t = 0; t < 2; ++t)
                        dmma_884(acc[h][t][0], acc[h][t][1], xa[c][s], fp[(s * 2 + t) * 32]);
                }
            }
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                double re = acc[0][t][0], im = acc[0][t][1];
#pragma unroll
                for (int h = 1; h < NCH; ++h) {
                    re += acc[h][t][0];
                    im += acc[h][t][1];
                }
                buf[tbuf_index(rr, 4 * t + cq)] = zmake(re, im);
            }
            __syncwarp();
            double ta[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) ta[s] = reinterpret_cast<const double*>(&buf[tbuf_index(rr, 2 * s + acol)])[apart];
            __syncwarp();
            double xb[2][2][2] = {};
            const double* fd = frag + pair_index(b, b) * TR_FRAG + lane;
#pragma unroll
            for (int s = 0; s < 4; ++s)
#pragma unroll
                for (int t = 0; t < 2; ++t)
                    if (2 * s <= 4 * t + 3) dmma_884(xb[s & 1][t][0], xb[s & 1][t][1], ta[s], fd[(s * 2 + t) * 32]);
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const z64 x = zmake(xb[0][t][0] + xb[1][t][0], xb[0][t][1] + xb[1][t][1]);
                const int col = TR_NB * b + 4 * t + cq;
                if (live && col < k) __stcg(yrow + (int64_t)col * ldy, x);
                if (b + 1 < NBLK) buf[tbuf_index(rr, 4 * t + cq)] = x;
            }
            if (b + 1 < NBLK) {
                __syncwarp();
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    xa[b][s] = reinterpret_cast<const double*>(&buf[tbuf_index(rr, 2 * s + acol)])[apart];
                __syncwarp();
            }
        }
        if (NBLK & 1) {
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const z64 tmp = yq[0][t];
                yq[0][t] = yq[1][t];
                yq[1][t] = tmp;
            }
        }
    }
}

// Plain substitution for the rows [row0, row1), a thread a row (the
// reference's ztrsm arithmetic), for a factor whose diagonal blocks are too
// ill-conditioned to invert. U: column-major k x k.
__device__ void pb_solve_substitute(z64* Y, int64_t ldy, int64_t row0, int64_t row1, int k, const z64* U) {
    for (int64_t r = row0 + threadIdx.x; r < row1; r += blockDim.x) {
        z64* row = Y + r;
        for (int j = 0; j < k; ++j) {
            z64 acc = __ldcg(row + (int64_t)j * ldy);
            for (int i = 0; i < j; ++i) zmsub(acc, __ldcg(row + (int64_t)i * ldy), __ldcg(U + i + (int64_t)j * k));
            __stcg(row + (int64_t)j * ldy, zmul(acc, zrecip_d(__ldcg(U + j + (int64_t)j * k))));
        }
    }
}

// ---- jobs and the kernel -------------------------------------------------------------

// The ring's barriers as one kind of job uses them: Gram jobs and solve jobs
// have a set each (their empty barriers count 12 and 15 hand-backs a stage),
// initialized once. Every waiting warp passes every stage of every job of its
// kind, so the per-slot phase parities below, kept across jobs, stay the same
// in every thread of the CTA whatever the slot count of a job is.
struct PbRing {
    uint64_t* full;
    uint64_t* empty;
    uint32_t full_par, empty_par, used;   // per slot: phase parities, and whether it was ever filled
};

// The ring of a job over the rows of `chunk` (stage height and slot count by
// the instance's width).
__device__ GramCtx ring_ctx(const PbInst& I, int chunk, unsigned char* smem, const PbRing& ring, bool solve) {
    const int kp = pb_kp(I.k);
    const bool small = I.k <= PB_STAGED_SOLVE_KMAX;
    GramCtx c;
    c.ring = smem + (small ? PB_SMALL_FRAG_BYTES : PB_RING_OFF);
    c.full = ring.full;
    c.empty = ring.empty;
    c.sr = pb_stage_rows(kp / 8);
    c.col_bytes = solve ? pb_solve_col_bytes(kp / 8) : pb_col_bytes(kp / 8);
    c.stage_bytes = kp * c.col_bytes;
    c.nslots = min(PB_MAX_STAGES, (small ? PB_SMALL_RING : PB_RING) / c.stage_bytes);
    c.kp = kp;
    c.row0 = (int64_t)chunk * I.chunk_rows;
    c.row1 = min(I.N, c.row0 + I.chunk_rows);
    c.out = nullptr;
    c.ok = true;
    c.bad_site = 0;
    return c;
}

// The Gram chunk `chunk` of pass `pass`: waits (pass >= 2) for the chunk's
// solve of the previous pass, multiplies unless the instance stopped, adds
// the arrival, and runs the factor step if it was the last chunk to arrive.
// Returns whether it overwrote cached fragments (a factor step, or a narrow
// job's ring).
__device__ bool gram_job(const PbArgs& a, const PbInst& I, int pass, int chunk, unsigned char* smem, PbRing& ring,
                         double* red) {
    __shared__ int s_skip, s_bad, s_last;
    const int tid = threadIdx.x, warp = tid >> 5;
    ChainStatus* st = I.st;
    if (tid == 0) {
        int skip = 0;
        if (pass >= 2) {
            if (!wait_flag(I.counters + PB_SOLVED + chunk, pass - 1)) {
                pb_timeout(a, st, WAIT_SOLVED);
                skip = 1;
            } else {
                skip = __ldcg(&st->failed) != 0 || __ldcg(&st->timeout) != 0;
                if (pass == 3) skip = skip || !(__ldcg(&st->shifted[1]) | __ldcg(&st->shifted[2]));
            }
        }
        s_skip = skip;
        s_bad = 0;
    }
    __syncthreads();
    if (!s_skip) {
        const int k = I.k;
        GramCtx c = ring_ctx(I, chunk, smem, ring, false);
        c.out = reinterpret_cast<z64*>(I.scratch + pb_layout(k, I.nchunks).partial) + (size_t)chunk * pb_npairs(k) * 64;
        // Padding columns past k read as zero: no copy writes them.
        if (k < c.kp) {
            for (int e = tid; e < c.nslots * (c.kp - k) * c.sr; e += blockDim.x) {
                const int slot = e / ((c.kp - k) * c.sr), rem = e - slot * (c.kp - k) * c.sr;
                const int col = k + rem / c.sr, row = rem % c.sr;
                *reinterpret_cast<z64*>(c.ring + (size_t)slot * c.stage_bytes + col * c.col_bytes + row * 16) =
                    zmake(0.0, 0.0);
            }
        }
        // Whatever this CTA last wrote into the ring through generic stores is
        // ordered before the bulk copies that now refill it.
        fence_proxy_async_all();
        __syncthreads();
        if (warp == PB_COPY_WARP) {
            gram_produce(I.Y, I.ldy, k, c, ring.empty_par, ring.used, WAIT_GRAM_SLOT);
        } else if (warp < PB_GRAM_WARPS) {
            switch (c.kp / 8) {
#define FB_PB_GRAM(n) case n: gram_compute<n>(c, ring.full_par); break;
                FB_PB_GRAM(1) FB_PB_GRAM(2) FB_PB_GRAM(3) FB_PB_GRAM(4)
                FB_PB_GRAM(5) FB_PB_GRAM(6) FB_PB_GRAM(7) FB_PB_GRAM(8)
#undef FB_PB_GRAM
            }
        }
        if (!c.ok) s_bad = c.bad_site;
    }
    __syncthreads();
    if (tid == 0) {
        if (s_bad) pb_timeout(a, st, s_bad);
        __threadfence();
        const int before = atomicAdd(I.counters + PB_ARRIVE + pass, 1);
        s_last = before == I.nchunks - 1;
    }
    __syncthreads();
    if (!s_last) return I.k <= PB_STAGED_SOLVE_KMAX;
    __threadfence();
    factor_step(I, pass, smem, red);
    return true;
}

// The solve chunk `chunk` of pass `pass`: waits for the pass's factor, solves
// the chunk's rows by the plan's path (unless the instance stopped), and
// marks the chunk solved for this pass. `cached` names the fragments already
// in shared memory (instance slot * 4 + pass, -1 for none).
__device__ void solve_job(const PbArgs& a, const PbInst& I, int slot, int pass, int chunk, unsigned char* smem,
                          PbRing& ring, int& cached) {
    // ring: the solve jobs' barrier set.
    __shared__ int s_skip, s_path, s_bad;
    const int tid = threadIdx.x, warp = tid >> 5;
    ChainStatus* st = I.st;
    const int k = I.k;
    const PbLayout L = pb_layout(k, I.nchunks);
    if (tid == 0) {
        int skip = 0;
        if (!wait_flag(I.counters + PB_READY + pass, 1)) {
            pb_timeout(a, st, WAIT_READY);
            skip = 1;
        } else {
            skip = __ldcg(&st->failed) != 0 || __ldcg(&st->timeout) != 0;
            if (pass == 3) skip = skip || !(__ldcg(&st->shifted[1]) | __ldcg(&st->shifted[2]));
        }
        s_skip = skip;
        s_bad = 0;
        s_path = skip ? PATH_SUBSTITUTE : __ldcg(&reinterpret_cast<const TrsmPlan*>(I.scratch + L.plan)->path);
    }
    __syncthreads();
    if (!s_skip) {
        const int path = s_path;
        double* frag = reinterpret_cast<double*>(smem);
        const int key = slot * 4 + pass;
        if (cached != key) {
            const int n = path == PATH_INVERSE ? inverse_frag_doubles(k)
                          : path == PATH_BLOCKED ? blocked_frag_doubles(k) : 0;
            const double2* src = reinterpret_cast<const double2*>(I.scratch + L.frag);
            for (int e = tid; e < n / 2; e += blockDim.x) reinterpret_cast<double2*>(frag)[e] = __ldcg(src + e);
            cached = key;
        }
        GramCtx c = ring_ctx(I, chunk, smem, ring, true);
        if (path == PATH_INVERSE && k <= PB_STAGED_SOLVE_KMAX) {
            fence_proxy_async_all();
            __syncthreads();
            if (warp == PB_COPY_WARP) {
                gram_produce(I.Y, I.ldy, k, c, ring.empty_par, ring.used, WAIT_SOLVE_SLOT);
            } else {
                switch ((k + 3) / 4) {
#define FB_PB_INV(n) case n: pb_solve_inverse<n>(c, ring.full_par, I.Y, I.ldy, I.N, k, frag, a.zero); break;
                    FB_PB_INV(1) FB_PB_INV(2) FB_PB_INV(3) FB_PB_INV(4)
                    FB_PB_INV(5) FB_PB_INV(6) FB_PB_INV(7) FB_PB_INV(8)
#undef FB_PB_INV
                }
            }
            if (!c.ok) s_bad = c.bad_site;
        } else {
            __syncthreads();
            const int64_t u0 = c.row0 / 8, u1 = (c.row1 + 7) / 8;
            if (path == PATH_INVERSE) {
                switch ((k + 3) / 4) {
#define FB_PB_INV(n) case n: pb_solve_inverse_direct<n>(I.Y, I.ldy, I.N, k, u0, u1, frag, a.zero); break;
                    FB_PB_INV(9) FB_PB_INV(10) FB_PB_INV(11) FB_PB_INV(12)
                    FB_PB_INV(13) FB_PB_INV(14) FB_PB_INV(15) FB_PB_INV(16)
#undef FB_PB_INV
                }
            } else if (path == PATH_BLOCKED) {
                z64* tbuf = reinterpret_cast<z64*>(smem + PB_RING_OFF);
                switch (pb_kp(k) / 8) {
#define FB_PB_BLK(n) case n: pb_solve_blocked<n>(I.Y, I.ldy, I.N, k, u0, u1, frag, tbuf); break;
                    FB_PB_BLK(1) FB_PB_BLK(2) FB_PB_BLK(3) FB_PB_BLK(4)
                    FB_PB_BLK(5) FB_PB_BLK(6) FB_PB_BLK(7) FB_PB_BLK(8)
#undef FB_PB_BLK
                }
            } else {
                pb_solve_substitute(I.Y, I.ldy, c.row0, c.row1, k, reinterpret_cast<const z64*>(I.scratch + L.U));
            }
        }
        // The next pass's Gram reads these rows with bulk copies.
        fence_proxy_async_all();
    }
    __syncthreads();
    if (tid == 0) {
        if (s_bad) pb_timeout(a, st, s_bad);
        __threadfence();
        st_release(I.counters + PB_SOLVED + chunk, pass);
    }
}

__global__ void __launch_bounds__(PB_THREADS, 1) batch_chain_kernel(const __grid_constant__ PbArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t gfull[PB_MAX_STAGES], gempty[PB_MAX_STAGES];
    __shared__ uint64_t sfull[PB_MAX_STAGES], sempty[PB_MAX_STAGES];
    __shared__ double red[33];
    __shared__ int s_job;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int b = 0; b < PB_MAX_STAGES; ++b) {
            mbar_init(&gfull[b], 1);
            mbar_init(&gempty[b], PB_GRAM_WARPS);
            mbar_init(&sfull[b], 1);
            mbar_init(&sempty[b], PB_WARPS - 1);
        }
        mbar_fence_init();
    }
    __syncthreads();
    PbRing gring{gfull, gempty, 0u, 0u, 0u};
    PbRing sring{sfull, sempty, 0u, 0u, 0u};
    int cached = -1;
    const int total = PB_PHASES * a.jobs;
    for (;;) {
        if (tid == 0) {
            int job = (int)atomicAdd(a.ticket, 1u);
            if (__ldcg(a.ticket + 1) != 0u) job = total;
            s_job = job;
        }
        __syncthreads();
        const int job = s_job;
        if (job >= total) break;
        const int phase = job / a.jobs, j = job - phase * a.jobs;
        int lo = 0, hi = a.count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.inst[mid].first_job <= j) lo = mid;
            else hi = mid - 1;
        }
        const PbInst& I = a.inst[lo];
        const int pass = phase / 2 + 1, chunk = j - I.first_job;
        if ((phase & 1) == 0) {
            if (gram_job(a, I, pass, chunk, smem, gring, red)) cached = -1;
        } else {
            solve_job(a, I, lo, pass, chunk, smem, sring, cached);
        }
        __syncthreads();
    }
}

}  // namespace fb

using namespace fb;

namespace {

// Rows a chunk of an N x k instance holds: at least PB_CHUNK_BYTES of Y, at
// most 64 chunks, a multiple of every stage height.
void pb_chunking(int64_t N, int k, int& chunk_rows, int& nchunks) {
    int64_t rows = PB_CHUNK_BYTES / (16 * (int64_t)k);
    const int64_t spread = (N + PB_MAX_CHUNKS - 1) / PB_MAX_CHUNKS;
    if (rows < spread) rows = spread;
    rows = (rows + PB_SR_MAX - 1) / PB_SR_MAX * PB_SR_MAX;
    const int64_t whole = (N + PB_SR_MAX - 1) / PB_SR_MAX * PB_SR_MAX;
    if (rows > whole) rows = whole;
    chunk_rows = (int)rows;
    nchunks = (int)((N + rows - 1) / rows);
}

// The workspace: status blocks (one per instance, as fb_zcholqr2_batched's),
// ticket words (one 256-byte block per launch), counter blocks, all zeroed by
// each call; then the instances' scratch.
struct PbWorkspace {
    size_t tickets, counters, scratch, total;
    int launches;
};

int pb_workspace(const int64_t* N, const int* k, int count, PbWorkspace& W, std::vector<size_t>* offsets) {
    W.launches = (count + PB_MAX_INST - 1) / PB_MAX_INST;
    W.tickets = align_up((size_t)count * sizeof(ChainStatus), 256);
    W.counters = W.tickets + (size_t)W.launches * 256;
    W.scratch = W.counters + align_up((size_t)count * PB_COUNTER_INTS * sizeof(int), 256);
    size_t off = W.scratch;
    if (offsets) offsets->resize(count);
    for (int i = 0; i < count; ++i) {
        if (N[i] < 1 || k[i] < 1) {
            set_error(FB_EINVAL, "cholqr2! batch: instance %d has N=%lld, k=%d", i, (long long)N[i], k[i]);
            return FB_EINVAL;
        }
        if (k[i] > TR_KMAX) {
            set_error(FB_ENOTSUP, "the persistent cholqr2! batch handles k <= %d, instance %d has k=%d (the lane "
                      "schedule, fb_zcholqr2_batched, takes any k)", TR_KMAX, i, k[i]);
            return FB_ENOTSUP;
        }
        int rows = 0, nch = 0;
        pb_chunking(N[i], k[i], rows, nch);
        if (offsets) (*offsets)[i] = off;
        off += pb_layout(k[i], nch).total;
    }
    W.total = off;
    return FB_OK;
}

}  // namespace

extern "C" {

int fb_zcholqr2_batched_persistent_workspace_size(const int64_t* N, const int* k, int count, size_t* bytes) {
    if (!bytes || count < 0 || (count > 0 && (!N || !k))) {
        set_error(FB_EINVAL, "fb_zcholqr2_batched_persistent_workspace_size: bad argument");
        return FB_EINVAL;
    }
    PbWorkspace W{};
    FB_TRY(pb_workspace(N, k, count, W, nullptr));
    *bytes = W.total;
    return FB_OK;
}

int fb_zcholqr2_batched_persistent(fb_z128* const* Y, const int64_t* ldy, const int64_t* N, const int* k,
                                   fb_z128* const* R, const int64_t* ldr, int count, void* workspace,
                                   size_t workspace_bytes, fb_queue_t queue) {
    if (count < 0 || (count > 0 && (!Y || !ldy || !N || !k || !R || !ldr))) {
        set_error(FB_EINVAL, "fb_zcholqr2_batched_persistent: NULL argument array");
        return FB_EINVAL;
    }
    if (count == 0) return FB_OK;
    PbWorkspace W{};
    std::vector<size_t> offsets;
    FB_TRY(pb_workspace(N, k, count, W, &offsets));
    if (!workspace || workspace_bytes < W.total || ((uintptr_t)workspace & 255)) {
        set_error(FB_ENOMEM, "fb_zcholqr2_batched_persistent: workspace must be 256-byte aligned and hold %zu bytes "
                  "(got %zu)", W.total, workspace_bytes);
        return FB_ENOMEM;
    }
    for (int i = 0; i < count; ++i) {
        if (!Y[i] || !R[i]) {
            set_error(FB_EINVAL, "cholqr2! batch: instance %d has a NULL matrix", i);
            return FB_EINVAL;
        }
        if (ldy[i] < N[i] || ldr[i] < k[i]) {
            set_error(FB_EDIM, "cholqr2! batch: instance %d has a leading dimension smaller than its rows", i);
            return FB_EDIM;
        }
        if (((uintptr_t)Y[i] | (uintptr_t)R[i]) & 15) {
            set_error(FB_EINVAL, "cholqr2! batch: instance %d: device pointers must be 16-byte aligned", i);
            return FB_EINVAL;
        }
    }
    cudaStream_t stream = stream_of(queue);
    char* ws = static_cast<char*>(workspace);
    FB_CUDA(cudaMemsetAsync(ws, 0, W.scratch, stream), "cudaMemsetAsync");
    FB_CUDA(cudaFuncSetAttribute(batch_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PB_SMEM),
            "cudaFuncSetAttribute(batch_chain_kernel)");
    // Largest first (work ~ N k^2), so that the long chunks start early and
    // the small instances fill the end of every phase.
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (double)N[x] * k[x] * k[x] > (double)N[y] * k[y] * k[y];
    });
    std::unique_ptr<PbArgs> args(new PbArgs());
    ChainStatus* status = reinterpret_cast<ChainStatus*>(ws);
    int* counters = reinterpret_cast<int*>(ws + W.counters);
    for (int l = 0; l < W.launches; ++l) {
        PbArgs& a = *args;
        a.ticket = reinterpret_cast<unsigned*>(ws + W.tickets + (size_t)l * 256);
        a.count = std::min(PB_MAX_INST, count - l * PB_MAX_INST);
        a.zero = 0;
        a.pad = 0;
        int jobs = 0;
        for (int s = 0; s < a.count; ++s) {
            const int i = order[l * PB_MAX_INST + s];
            PbInst& p = a.inst[s];
            p.Y = reinterpret_cast<z64*>(Y[i]);
            p.R = reinterpret_cast<z64*>(R[i]);
            p.scratch = ws + offsets[i];
            p.counters = counters + (size_t)i * PB_COUNTER_INTS;
            p.st = status + i;
            p.ldy = ldy[i];
            p.ldr = ldr[i];
            p.N = N[i];
            p.k = k[i];
            pb_chunking(N[i], k[i], p.chunk_rows, p.nchunks);
            p.first_job = jobs;
            jobs += p.nchunks;
        }
        a.jobs = jobs;
        const int grid = std::max(1, std::min(sm_count(), PB_PHASES * jobs));
        batch_chain_kernel<<<grid, PB_THREADS, PB_SMEM, stream>>>(a);
        FB_LAUNCHED("batch_chain_kernel");
    }
    return FB_OK;
}

}  // extern "C"
