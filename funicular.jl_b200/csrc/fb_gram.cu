// gram_accumulate! (src/kernels.jl:22-55): C <- alpha A^H B + beta C for tall
// skinny A (rows x kA) and B (rows x kB), ComplexF64, FP64 throughout.
//
// Layout of the work. C is cut into tiles of at most 64 x 64 columns. A CTA
// owns one tile and one chunk of rows. It streams its rows through shared
// memory in stages of 32 rows (cp.async, zero-filled past the last row and
// the last column, so ragged views need no special case), and every thread
// accumulates a 4 x 4 block of the tile in registers over the whole chunk.
// The threads of a CTA form several row groups that cover the tile each, so
// the thread count is a whole number of warps for every tile shape. At the
// end the row groups are summed in a fixed order and the CTA's partial tile
// goes to the workspace; a second kernel adds the chunks, again in a fixed
// order, and applies alpha and beta. Nothing depends on timing, so the bits
// of the result depend only on (rows, kA, kB) and the device's SM count.
//
// When A and B are the same view the tile grid is folded: only tiles on or
// above the diagonal run, and inside a diagonal tile only the 4 x 4 blocks on
// or above the diagonal. The lower triangle is written as the conjugate of the
// upper one and the diagonal is made real.
//
// Shared memory holds each stage row-major (one row of the tile contiguous)
// with the columns permuted, column 4*m + c stored at c*nm + m, so that the
// threads of a warp, which read four columns 4*m..4*m+3 for different m,
// touch consecutive 16-byte words and never share a bank.
#include <mutex>
#include <vector>

#include "fb_common.cuh"

namespace fb {

constexpr int GS_ROWS = 32;
constexpr int GS_STAGES = 3;
constexpr int G_TILE = 64;
constexpr int G_MAX_THREADS = 576;

struct GramShape {
    int tw_a, tw_b;      // tile widths in columns (multiples of 4, at most 64)
    int nt_a, nt_b;      // tiles along the columns of A and of B
    int hermitian;
    int ntiles;          // tiles in the partial buffer
    int64_t chunk_rows;
    int nchunks;
};

struct GramLaunch {
    int diag;            // folded diagonal tiles (hermitian mode)
    int ntiles;          // CTAs along x
    int nm_a, nm_b;      // 4-column micro blocks per tile side
    int micro;           // micro blocks a row group covers
    int groups;          // row groups
    int threads;
    size_t smem;
};

__host__ __device__ inline int off_tile_index(int nt, int ti, int tj) {
    // Off-diagonal tile (ti < tj) in row-major order over the strict upper
    // triangle, after the nt diagonal tiles.
    return nt + ti * (2 * nt - ti - 1) / 2 + (tj - ti - 1);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int src_size = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_size));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__global__ void __launch_bounds__(G_MAX_THREADS, 1)
gram_partial_kernel(const z64* __restrict__ A, int64_t lda, const z64* __restrict__ B, int64_t ldb,
                    int64_t rows, int kA, int kB, GramShape sh, GramLaunch ln,
                    z64* __restrict__ partial, const ChainStatus* st, int gate) {
    if (gated_off(st, gate)) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    z64* smem = reinterpret_cast<z64*>(smem_raw);

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
    const int chunk = blockIdx.y;
    const int64_t row0 = (int64_t)chunk * sh.chunk_rows;
    const int64_t row_end = min(rows, row0 + sh.chunk_rows);
    const int col_a0 = ti * sh.tw_a, col_b0 = tj * sh.tw_b;
    const bool same = ln.diag != 0;  // B tile is the A tile
    const int tw_a = sh.tw_a, tw_b = sh.tw_b;
    const int stride_a = tw_a + 1, stride_b = tw_b + 1;
    const int stage_a = GS_ROWS * stride_a, stage_b = same ? 0 : GS_ROWS * stride_b;
    const int stage_elems = stage_a + stage_b;

    // This thread's 4 x 4 block and row group.
    const int tid = threadIdx.x;
    const int g = tid / ln.micro;
    const int m = tid - g * ln.micro;
    const bool computes = g < ln.groups;
    int mi = 0, mj = 0;
    if (computes) {
        if (ln.diag) {
            int r = m;
            while (r >= ln.nm_a - mi) { r -= ln.nm_a - mi; ++mi; }
            mj = mi + r;
        } else {
            mi = m / ln.nm_b;
            mj = m - mi * ln.nm_b;
        }
    }
    const int rows_per_group = GS_ROWS / ln.groups;

    z64 acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = zmake(0.0, 0.0);

    const int64_t nstages = (row_end > row0) ? (row_end - row0 + GS_ROWS - 1) / GS_ROWS : 0;

    auto load_stage = [&](int64_t s, int buf) {
        z64* sa = smem + buf * stage_elems;
        z64* sb = same ? sa : sa + stage_a;
        const int64_t r0 = row0 + s * GS_ROWS;
        const int total_a = GS_ROWS * tw_a;
        for (int e = tid; e < total_a; e += blockDim.x) {
            int l = e & (GS_ROWS - 1), c = e >> 5;
            int64_t r = r0 + l;
            int col = col_a0 + c;
            bool valid = (r < row_end) && (col < kA);
            const z64* src = valid ? (A + r + (int64_t)col * lda) : A;
            int phys = (c & 3) * ln.nm_a + (c >> 2);
            cp_async16(sa + l * stride_a + phys, src, valid);
        }
        if (!same) {
            const int total_b = GS_ROWS * tw_b;
            for (int e = tid; e < total_b; e += blockDim.x) {
                int l = e & (GS_ROWS - 1), c = e >> 5;
                int64_t r = r0 + l;
                int col = col_b0 + c;
                bool valid = (r < row_end) && (col < kB);
                const z64* src = valid ? (B + r + (int64_t)col * ldb) : B;
                int phys = (c & 3) * ln.nm_b + (c >> 2);
                cp_async16(sb + l * stride_b + phys, src, valid);
            }
        }
    };

    // Prologue: fill GS_STAGES - 1 stages.
#pragma unroll
    for (int s = 0; s < GS_STAGES - 1; ++s) {
        if (s < nstages) load_stage(s, s);
        cp_async_commit();
    }

    for (int64_t s = 0; s < nstages; ++s) {
        cp_async_wait<GS_STAGES - 2>();
        __syncthreads();
        // Refill the buffer the previous iteration finished with.
        {
            int64_t nxt = s + GS_STAGES - 1;
            if (nxt < nstages) load_stage(nxt, (int)(nxt % GS_STAGES));
            cp_async_commit();
        }
        if (computes) {
            const z64* sa = smem + (int)(s % GS_STAGES) * stage_elems;
            const z64* sb = same ? sa : sa + stage_a;
            const int l0 = g * rows_per_group;
#pragma unroll 1
            for (int l = l0; l < l0 + rows_per_group; ++l) {
                z64 a[4], b[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) a[c] = sa[l * stride_a + c * ln.nm_a + mi];
#pragma unroll
                for (int c = 0; c < 4; ++c) b[c] = sb[l * stride_b + c * ln.nm_b + mj];
#pragma unroll
                for (int x = 0; x < 4; ++x)
#pragma unroll
                    for (int y = 0; y < 4; ++y) zmac_conj(acc[x][y], a[x], b[y]);
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();

    // Sum the row groups into group 0, in group order, through shared memory.
    z64* red = smem;
    for (int r = 1; r < ln.groups; ++r) {
        if (computes && g == r) {
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) red[(x * 4 + y) * ln.micro + m] = acc[x][y];
        }
        __syncthreads();
        if (computes && g == 0) {
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) {
                    z64 v = red[(x * 4 + y) * ln.micro + m];
                    acc[x][y].x += v.x;
                    acc[x][y].y += v.y;
                }
        }
        __syncthreads();
    }

    if (computes && g == 0) {
        z64* out = partial + ((size_t)tile_index * sh.nchunks + chunk) * (G_TILE * G_TILE);
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                int li = 4 * mi + x, lj = 4 * mj + y;
                out[lj * G_TILE + li] = acc[x][y];
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
    const z64* src = partial + (size_t)tile * sh.nchunks * (G_TILE * G_TILE) + lj * G_TILE + li;
    z64 s = zmake(0.0, 0.0);
    for (int c = lane; c < sh.nchunks; c += 32) {
        z64 v = src[(size_t)c * (G_TILE * G_TILE)];
        s.x += v.x;
        s.y += v.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s.x += __shfl_down_sync(0xffffffffu, s.x, off);
        s.y += __shfl_down_sync(0xffffffffu, s.y, off);
    }
    if (lane != 0) return;
    if (mirror) s.y = -s.y;
    if (sh.hermitian && i == j) s.y = 0.0;
    z64 out = zmul(alpha, s);
    z64* dst = C + i + (int64_t)j * ldc;
    if (beta.x != 0.0 || beta.y != 0.0) zmac(out, beta, *dst);
    *dst = out;
}

static int pick_groups(int micro) {
    int best = 1;
    for (int g = 1; g <= 32; g <<= 1) {
        if (micro * g > G_MAX_THREADS) break;
        best = g;
    }
    // Prefer a whole number of warps when a smaller group count gives one.
    for (int g = best; g >= 1; g >>= 1)
        if ((micro * g) % 32 == 0) return g;
    return best;
}

static GramShape gram_shape(int64_t rows, int kA, int kB, int hermitian) {
    GramShape sh{};
    auto tile_width = [](int k) { int w = k < G_TILE ? k : G_TILE; return (w + 3) / 4 * 4; };
    sh.tw_a = tile_width(kA);
    sh.tw_b = tile_width(kB);
    sh.nt_a = (kA + sh.tw_a - 1) / sh.tw_a;
    sh.nt_b = (kB + sh.tw_b - 1) / sh.tw_b;
    sh.hermitian = hermitian;
    sh.ntiles = hermitian ? sh.nt_a * (sh.nt_a + 1) / 2 : sh.nt_a * sh.nt_b;
    int largest_launch = hermitian ? (sh.nt_a > 1 ? sh.nt_a * (sh.nt_a - 1) / 2 : 1) : sh.ntiles;
    if (hermitian && sh.nt_a > largest_launch) largest_launch = sh.nt_a;
    const int64_t stages = (rows + GS_ROWS - 1) / GS_ROWS;
    int64_t target = (int64_t)sm_count() / largest_launch;
    if (target < 1) target = 1;
    if (target > stages) target = stages;
    if (target < 1) target = 1;
    int64_t chunk_stages = stages > 0 ? (stages + target - 1) / target : 1;
    sh.chunk_rows = chunk_stages * GS_ROWS;
    sh.nchunks = rows > 0 ? (int)((rows + sh.chunk_rows - 1) / sh.chunk_rows) : 0;
    return sh;
}

static GramLaunch gram_launch(const GramShape& sh, bool diag) {
    GramLaunch ln{};
    ln.diag = diag;
    ln.nm_a = sh.tw_a / 4;
    ln.nm_b = diag ? ln.nm_a : sh.tw_b / 4;
    if (diag) {
        ln.ntiles = sh.nt_a;
        ln.micro = ln.nm_a * (ln.nm_a + 1) / 2;
    } else {
        ln.ntiles = sh.hermitian ? sh.nt_a * (sh.nt_a - 1) / 2 : sh.nt_a * sh.nt_b;
        ln.micro = ln.nm_a * ln.nm_b;
    }
    ln.groups = pick_groups(ln.micro);
    ln.threads = (ln.micro * ln.groups + 31) / 32 * 32;
    int stage = GS_ROWS * (sh.tw_a + 1) + (diag ? 0 : GS_ROWS * (sh.tw_b + 1));
    size_t stages_bytes = (size_t)GS_STAGES * stage * sizeof(z64);
    size_t red_bytes = (size_t)16 * ln.micro * sizeof(z64);
    ln.smem = stages_bytes > red_bytes ? stages_bytes : red_bytes;
    return ln;
}

static size_t gram_workspace_bytes(const GramShape& sh) {
    return (size_t)sh.ntiles * (size_t)(sh.nchunks > 0 ? sh.nchunks : 1) * G_TILE * G_TILE * sizeof(z64);
}

// Shared by fb_zgram and the orthonormalization chain.
int gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, const z64* B, int64_t ldb,
                 int64_t rows, int kA, int kB, z64 alpha, z64 beta, bool hermitian,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream,
                 const ChainStatus* st, int gate) {
    GramShape sh = gram_shape(rows, kA, kB, hermitian ? 1 : 0);
    size_t need = gram_workspace_bytes(sh);
    if (workspace_bytes < need || workspace == nullptr) {
        set_error(FB_ENOMEM, "gram: workspace of %zu bytes is smaller than the %zu bytes this shape needs",
                  workspace_bytes, need);
        return FB_ENOMEM;
    }
    z64* partial = static_cast<z64*>(workspace);
    if (sh.nchunks > 0) {
        const bool launches[2] = {hermitian, !hermitian || sh.nt_a > 1};
        for (int d = 0; d < 2; ++d) {
            if (!launches[d]) continue;
            bool diag = (d == 0);
            GramLaunch ln = gram_launch(sh, diag);
            if (ln.ntiles == 0) continue;
            static bool attr_set = false;
            if (!attr_set) {
                FB_CUDA(cudaFuncSetAttribute(gram_partial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             227 * 1024),
                        "cudaFuncSetAttribute(gram_partial_kernel)");
                attr_set = true;
            }
            dim3 grid(ln.ntiles, sh.nchunks);
            gram_partial_kernel<<<grid, ln.threads, ln.smem, stream>>>(A, lda, B, ldb, rows, kA, kB, sh, ln,
                                                                       partial, st, gate);
            FB_LAUNCHED("gram_partial_kernel");
        }
    }
    int64_t entries = (int64_t)kA * kB;
    int64_t threads = entries * 32;
    int block = 256;
    int64_t grid = (threads + block - 1) / block;
    gram_reduce_kernel<<<(unsigned)grid, block, 0, stream>>>(C, ldc, kA, kB, sh, partial, alpha, beta, st, gate);
    FB_LAUNCHED("gram_reduce_kernel");
    return FB_OK;
}

size_t gram_workspace_size(int64_t rows, int kA, int kB, bool hermitian) {
    return gram_workspace_bytes(gram_shape(rows, kA, kB, hermitian ? 1 : 0));
}

// Scratch for fb_zgram_static, the entry point for callers that cannot
// allocate device memory. It is an ordinary global of this module, so every
// GPU that loads the library holds these bytes until the process exits. The
// partial tiles it holds are written by each call before that call reads
// them, so nothing in it has to start at zero.
constexpr size_t GRAM_STATIC_SCRATCH_BYTES = (size_t)16 << 20;
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

}  // extern "C"
