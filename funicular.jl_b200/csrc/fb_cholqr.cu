// cholqr2! (src/panelblas.jl:130-146) on a matrix resident in device memory.
//
// The reference runs each pass as gram -> host Cholesky -> rdiv_rows!, with
// the k x k matrices crossing to the host and back twice per pass. Here the
// whole chain is one fixed sequence of launches on one queue: every pass is
// Gram (folded, Hermitian) -> single-CTA Cholesky with the shifted retry ->
// row-parallel triangular solve, and the factors never leave the device. The
// decisions the reference takes on the host are taken on the device through
// a status block in the workspace: a pass whose Cholesky fails stops every
// later kernel (Y keeps what the finished passes made of it, as when the
// reference throws before its rdiv_rows!), and the third pass runs only if a
// shift fired in pass 1 or 2.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "fb_common.cuh"

namespace fb {

int gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, const z64* B, int64_t ldb,
                 int64_t rows, int kA, int kB, z64 alpha, z64 beta, bool hermitian,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream,
                 const ChainStatus* st, int gate);
size_t gram_workspace_size(int64_t rows, int kA, int kB, bool hermitian);
void gram_chunks(int64_t rows, int kA, int kB, bool hermitian, int64_t* chunk_rows, int* nchunks);
int gram_partials_enqueue(const z64* A, int64_t lda, const z64* B, int64_t ldb, int64_t rows, int kA, int kB,
                          bool hermitian, void* workspace, size_t workspace_bytes, cudaStream_t stream,
                          const ChainStatus* st, int gate, int chunk0, int chunk1);
int gram_reduce_enqueue(z64* C, int64_t ldc, int64_t rows, int kA, int kB, bool hermitian, z64 alpha, z64 beta,
                        void* workspace, cudaStream_t stream, const ChainStatus* st, int gate);
int trsm_enqueue(z64* Y, int64_t ldy, int64_t rows, int k, const z64* R, int64_t ldr, void* workspace,
                 size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st, int gate);
size_t trsm_workspace_bytes(int k);
size_t potrf_gwork_bytes(int k);
size_t ozaki_gram_workspace_size(int64_t rows);
int ozaki_gram_enqueue(z64* C, int64_t ldc, const z64* A, int64_t lda, int64_t rows, int k, z64 alpha, z64 beta,
                       void* workspace, size_t workspace_bytes, cudaStream_t stream, const ChainStatus* st,
                       int gate);
int potrf_enqueue(const z64* G, int64_t ldg, int k, int64_t N, z64* U, int64_t ldu,
                  const z64* Rin, int64_t ldrin, z64* Rout, int64_t ldrout, z64* gwork,
                  ChainStatus* st, int pass, int gate, cudaStream_t stream, double forced_u);

struct CholqrLayout {
    size_t status, G, U, Ra, Rb, gwork, trsm, gram, total;
};

static CholqrLayout cholqr_layout(int64_t N, int k) {
    CholqrLayout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t at = off; off += align_up(bytes > 0 ? bytes : 1, 256); return at; };
    const size_t kk = (size_t)k * k * sizeof(z64);
    L.status = take(sizeof(ChainStatus));
    L.G = take(kk);
    L.U = take(kk);
    L.Ra = take(kk);
    L.Rb = take(kk);
    L.gwork = take(potrf_gwork_bytes(k));
    L.trsm = take(trsm_workspace_bytes(k));
    // One workspace serves both forms: the Gram scratch is the larger of the
    // FP64 and the tensor-core kernels' needs.
    const size_t g64 = gram_workspace_size(N, k, k, true);
    const size_t gtc = k <= 64 ? ozaki_gram_workspace_size(N) : 0;
    L.gram = take(g64 > gtc ? g64 : gtc);
    L.total = off;
    return L;
}

// Copies R of the last pass that ran into the caller's R.
__global__ void select_r_kernel(z64* __restrict__ R, int64_t ldr, const z64* __restrict__ Ra,
                                const z64* __restrict__ Rb, int k, const ChainStatus* st) {
    if (st->failed) return;
    const bool third = (st->shifted[1] | st->shifted[2]) != 0;
    const z64* src = third ? Ra : Rb;
    const int64_t kk = (int64_t)k * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < kk; e += (int64_t)gridDim.x * blockDim.x) {
        int j = (int)(e / k), i = (int)(e - (int64_t)j * k);
        R[i + (int64_t)j * ldr] = src[e];
    }
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_zcholqr2_workspace_size(int64_t N, int k, size_t* bytes) {
    if (!bytes || N < 0 || k < 0) { set_error(FB_EINVAL, "fb_zcholqr2_workspace_size: bad argument"); return FB_EINVAL; }
    *bytes = cholqr_layout(N, k).total;
    return FB_OK;
}

// The chain of one instance. status, when given, replaces the workspace's own
// status block (a batch keeps one status per instance and shares the rest).
static int cholqr2_chain(fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr, int* info,
                         int* passes, void* workspace, size_t workspace_bytes, fb_queue_t queue, bool tensor,
                         ChainStatus* status = nullptr, double forced_u = 0.0) {
    if (N < 1 || k < 1) {
        set_error(FB_EINVAL, "cholqr2!: N and k must be positive, got N=%lld, k=%d", (long long)N, k);
        return FB_EINVAL;
    }
    if (!Y || !R) { set_error(FB_EINVAL, "fb_zcholqr2: NULL matrix"); return FB_EINVAL; }
    if (ldy < N || ldr < k) { set_error(FB_EDIM, "fb_zcholqr2: leading dimension too small"); return FB_EDIM; }
    if (((uintptr_t)Y | (uintptr_t)R) & 15) {
        set_error(FB_EINVAL, "fb_zcholqr2: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    CholqrLayout L = cholqr_layout(N, k);
    if (!workspace || workspace_bytes < L.total || ((uintptr_t)workspace & 255)) {
        set_error(FB_ENOMEM, "fb_zcholqr2: workspace must be 256-byte aligned and hold %zu bytes (got %zu)",
                  L.total, workspace_bytes);
        return FB_ENOMEM;
    }
    char* ws = static_cast<char*>(workspace);
    ChainStatus* st = status ? status : reinterpret_cast<ChainStatus*>(ws + L.status);
    z64* G = reinterpret_cast<z64*>(ws + L.G);
    z64* U = reinterpret_cast<z64*>(ws + L.U);
    z64* Ra = reinterpret_cast<z64*>(ws + L.Ra);
    z64* Rb = reinterpret_cast<z64*>(ws + L.Rb);
    z64* gwork = reinterpret_cast<z64*>(ws + L.gwork);
    void* gram_ws = ws + L.gram;
    void* trsm_ws = ws + L.trsm;
    const size_t trsm_bytes = L.gram - L.trsm;
    const size_t gram_bytes = L.total - L.gram;
    cudaStream_t stream = stream_of(queue);
    z64* Yz = reinterpret_cast<z64*>(Y);
    const z64 one = zmake(1.0, 0.0), zero = zmake(0.0, 0.0);

    FB_CUDA(cudaMemsetAsync(st, 0, sizeof(ChainStatus), stream), "cudaMemsetAsync");
    // R accumulates as Ra = R1, Rb = R2 R1, Ra = R3 R2 R1.
    const z64* rin[4] = {nullptr, nullptr, Ra, Rb};
    z64* rout[4] = {nullptr, Ra, Rb, Ra};
    for (int pass = 1; pass <= 3; ++pass) {
        const int gate = pass == 3 ? GATE_THIRD : GATE_HEALTHY;
        if (tensor)
            FB_TRY(ozaki_gram_enqueue(G, k, Yz, ldy, N, k, one, zero, gram_ws, gram_bytes, stream, st, gate));
        else
            FB_TRY(gram_enqueue(G, k, Yz, ldy, Yz, ldy, N, k, k, one, zero, true, gram_ws, gram_bytes, stream, st,
                                gate));
        // The shifted CholeskyQR3 shifts pass 1 unconditionally; that marks
        // the pass as shifted, so the third pass runs and R = R3 R2 R1.
        FB_TRY(potrf_enqueue(G, k, k, N, U, k, rin[pass], k, rout[pass], k, gwork, st, pass, gate, stream,
                             pass == 1 ? forced_u : 0.0));
        FB_TRY(trsm_enqueue(Yz, ldy, N, k, U, k, trsm_ws, trsm_bytes, stream, st, gate));
    }
    int blocks = (int)((int64_t)k * k + 255) / 256;
    select_r_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<z64*>(R), ldr, Ra, Rb, k, st);
    FB_LAUNCHED("select_r_kernel");

    if (info) {
        FB_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        return fb_zcholqr2_query(st, info, passes, nullptr);
    }
    return FB_OK;
}

// A batch runs on up to 8 (tunable to 1..16) library-owned streams ("lanes") forked
// from the caller's queue and joined back into it with events, so the
// one-CTA kernels of one instance (the Cholesky, the solve's prep) run beside
// the full-GPU kernels of others instead of leaving the GPU idle. Each
// instance's chain is the same launch sequence as a single call, on one lane:
// its bits do not depend on the batch. The workspace holds one status block
// per instance, then one scratch area per lane sized for the largest
// instance. Fork and join are plain event records and waits, so a captured
// batch is one graph with the lanes as parallel branches.
constexpr int BATCH_LANES = 16;        // most lanes a batch can use
constexpr int STAGED_BLOCKS = 8;       // row blocks of the host-staged cholqr2!
static std::atomic<int> g_batch_lanes{8};  // lanes a batch uses: the autotuner's entry, 8 untuned
static size_t batch_status_bytes(int count) { return align_up((size_t)count * sizeof(ChainStatus), 256); }
static int batch_lanes(int count) {
    const int lanes = g_batch_lanes.load();
    return count < lanes ? count : lanes;
}

// The lane streams of the current device, created once.
static int lane_streams(cudaStream_t* out, int n) {
    static std::mutex mu;
    static cudaStream_t lanes[64][BATCH_LANES] = {};
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) { set_error(FB_ENOTSUP, "cholqr2! batch: device %d", dev); return FB_ENOTSUP; }
    std::lock_guard<std::mutex> lock(mu);
    for (int l = 0; l < n; ++l) {
        if (!lanes[dev][l])
            FB_CUDA(cudaStreamCreateWithFlags(&lanes[dev][l], cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
        out[l] = lanes[dev][l];
    }
    return FB_OK;
}

int fb_zcholqr2(fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr, int* info, int* passes,
                void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    return cholqr2_chain(Y, ldy, N, k, R, ldr, info, passes, workspace, workspace_bytes, queue, false);
}

int fb_zcholqr3_shifted(fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr, double unit_roundoff,
                        int* info, int* passes, void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (!(unit_roundoff > 0.0 && unit_roundoff < 1.0)) {
        set_error(FB_EINVAL, "fb_zcholqr3_shifted: the unit roundoff must lie in (0, 1), got %g", unit_roundoff);
        return FB_EINVAL;
    }
    return cholqr2_chain(Y, ldy, N, k, R, ldr, info, passes, workspace, workspace_bytes, queue, false, nullptr,
                         unit_roundoff);
}

int fb_zcholqr2_tc(fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr, int* info, int* passes,
                   void* workspace, size_t workspace_bytes, fb_queue_t queue) {
    if (k > 64) {
        set_error(FB_ENOTSUP, "the tensor-core form of cholqr2! handles k <= 64, got k = %d", k);
        return FB_ENOTSUP;
    }
    return cholqr2_chain(Y, ldy, N, k, R, ldr, info, passes, workspace, workspace_bytes, queue, true);
}

int fb_zcholqr2_batched_workspace_size(const int64_t* N, const int* k, int count, size_t* bytes) {
    if (!bytes || count < 0 || (count > 0 && (!N || !k))) {
        set_error(FB_EINVAL, "fb_zcholqr2_batched_workspace_size: bad argument");
        return FB_EINVAL;
    }
    size_t scratch = 0;
    for (int i = 0; i < count; ++i) {
        if (N[i] < 1 || k[i] < 1) {
            set_error(FB_EINVAL, "cholqr2! batch: instance %d has N=%lld, k=%d", i, (long long)N[i], k[i]);
            return FB_EINVAL;
        }
        const size_t t = cholqr_layout(N[i], k[i]).total;
        if (t > scratch) scratch = t;
    }
    *bytes = batch_status_bytes(count) + (size_t)batch_lanes(count) * align_up(scratch, 256);
    return FB_OK;
}

int fb_zcholqr2_batched(fb_z128* const* Y, const int64_t* ldy, const int64_t* N, const int* k, fb_z128* const* R,
                        const int64_t* ldr, int count, int tensor_form, void* workspace, size_t workspace_bytes,
                        fb_queue_t queue) {
    if (count < 0 || (count > 0 && (!Y || !ldy || !N || !k || !R || !ldr))) {
        set_error(FB_EINVAL, "fb_zcholqr2_batched: NULL argument array");
        return FB_EINVAL;
    }
    if (count == 0) return FB_OK;
    size_t need = 0;
    FB_TRY(fb_zcholqr2_batched_workspace_size(N, k, count, &need));
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255)) {
        set_error(FB_ENOMEM, "fb_zcholqr2_batched: workspace must be 256-byte aligned and hold %zu bytes (got %zu)",
                  need, workspace_bytes);
        return FB_ENOMEM;
    }
    for (int i = 0; i < count; ++i)
        if (tensor_form && k[i] > 64) {
            set_error(FB_ENOTSUP, "cholqr2! batch: the tensor-core form handles k <= 64, instance %d has k=%d", i, k[i]);
            return FB_ENOTSUP;
        }
    ChainStatus* status = static_cast<ChainStatus*>(workspace);
    const int L = batch_lanes(count);
    const size_t lane_bytes = (workspace_bytes - batch_status_bytes(count)) / L / 256 * 256;
    char* scratch = static_cast<char*>(workspace) + batch_status_bytes(count);
    cudaStream_t lanes[BATCH_LANES];
    FB_TRY(lane_streams(lanes, L));
    // Longest first, each to the lane with the least work so far (work ~ N k^2).
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)N[a] * k[a] * k[a] > (double)N[b] * k[b] * k[b];
    });
    std::vector<double> load(L, 0.0);
    std::vector<int> lane_of(count);
    for (int i : order) {
        int best = 0;
        for (int l = 1; l < L; ++l)
            if (load[l] < load[best]) best = l;
        lane_of[i] = best;
        load[best] += (double)N[i] * k[i] * k[i];
    }
    cudaStream_t origin = stream_of(queue);
    cudaEvent_t fork = nullptr, join[BATCH_LANES] = {};
    auto release = [&]() {
        if (fork) cudaEventDestroy(fork);
        for (int l = 0; l < L; ++l)
            if (join[l]) cudaEventDestroy(join[l]);
    };
    auto cu = [](cudaError_t err, const char* what) { return err == cudaSuccess ? FB_OK : cuda_status(err, what); };
    int rc = FB_OK;
    do {
        if ((rc = cu(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreateWithFlags")))
            break;
        if ((rc = cu(cudaEventRecord(fork, origin), "cudaEventRecord"))) break;
        for (int l = 0; l < L && !rc; ++l)
            rc = cu(cudaStreamWaitEvent(lanes[l], fork, 0), "cudaStreamWaitEvent");
        for (int i : order) {
            if (rc) break;
            const int l = lane_of[i];
            rc = cholqr2_chain(Y[i], ldy[i], N[i], k[i], R[i], ldr[i], nullptr, nullptr, scratch + l * lane_bytes,
                               lane_bytes, reinterpret_cast<fb_queue_t>(lanes[l]), tensor_form != 0, status + i);
        }
        // Join every lane back into the caller's queue, also after a failure,
        // so nothing the lanes hold outlives the call unordered.
        for (int l = 0; l < L; ++l) {
            int j = cu(cudaEventCreateWithFlags(&join[l], cudaEventDisableTiming), "cudaEventCreateWithFlags");
            if (!j) j = cu(cudaEventRecord(join[l], lanes[l]), "cudaEventRecord");
            if (!j) j = cu(cudaStreamWaitEvent(origin, join[l], 0), "cudaStreamWaitEvent");
            if (!rc) rc = j;
        }
    } while (false);
    release();
    return rc;
}

int fb_zcholqr2_batched_query(const void* workspace, int count, int* info, int* passes) {
    if (!workspace || count < 0) { set_error(FB_EINVAL, "fb_zcholqr2_batched_query: bad argument"); return FB_EINVAL; }
    int first_failed = -1;
    for (int i = 0; i < count; ++i) {
        int inf = 0, pas = 0;
        const int st = fb_zcholqr2_query(static_cast<const ChainStatus*>(workspace) + i, &inf, &pas, nullptr);
        if (st != FB_OK && st != FB_ENOTSPD) return st;
        if (info) info[i] = inf;
        if (passes) passes[i] = pas;
        if (inf && first_failed < 0) first_failed = i;
    }
    if (first_failed >= 0) {
        set_error(FB_ENOTSPD, "cholqr2! batch: the Gram matrix of instance %d is not positive definite even after "
                  "the shift", first_failed);
        return FB_ENOTSPD;
    }
    return FB_OK;
}

int fb_zcholqr2_query(const void* workspace, int* info, int* passes, double* shifts) {
    if (!workspace) { set_error(FB_EINVAL, "fb_zcholqr2_query: NULL workspace"); return FB_EINVAL; }
    ChainStatus host{};
    FB_CUDA(cudaMemcpy(&host, workspace, sizeof host, cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (host.timeout) {
        static const char* const sites[] = {"?", "a Gram stage", "a Gram copy slot", "a solve stage",
                                            "a solve copy slot", "a factor-ready flag", "a chunk-solved flag"};
        const int site = host.timeout >= 1 && host.timeout <= 6 ? host.timeout : 0;
        set_error(FB_ECUDA, "cholqr2! batch: a device-side wait of the persistent kernel (on %s) gave up after its "
                  "2 s limit, so the results are not valid", sites[site]);
        return FB_ECUDA;
    }
    if (info) *info = host.failed;
    if (passes) *passes = (host.shifted[1] | host.shifted[2]) ? 3 : 2;
    if (shifts)
        for (int p = 0; p < 3; ++p) shifts[p] = host.shift[p + 1];
    if (host.failed) {
        set_error(FB_ENOTSPD,
                  "the Gram matrix of pass %d is not positive definite even after a shift of %.17g, so the "
                  "columns are numerically dependent: a zero column, a duplicated one, or a condition number "
                  "past 4.5e15. Drop the dependent columns before orthonormalizing",
                  host.failed, host.shift[host.failed]);
        return FB_ENOTSPD;
    }
    return FB_OK;
}

int fb_tune_set_batch_lanes(int lanes) {
    if (lanes < 1 || lanes > BATCH_LANES) {
        set_error(FB_EINVAL, "fb_tune_set_batch_lanes: lanes must lie in [1, %d], got %d", BATCH_LANES, lanes);
        return FB_EINVAL;
    }
    g_batch_lanes.store(lanes);
    return FB_OK;
}

int fb_tune_get_batch_lanes(int* lanes) {
    if (!lanes) { set_error(FB_EINVAL, "fb_tune_get_batch_lanes: NULL"); return FB_EINVAL; }
    *lanes = g_batch_lanes.load();
    return FB_OK;
}

// ---- cholqr2! of a matrix held in page-locked host panels -----------------
//
// The end-to-end form: the panels go up in row blocks on one stream while the
// first pass's Gram consumes the blocks that have landed (the Gram's row
// chunks are grouped into the blocks, so its partial tiles, and with them its
// bits, are those of one launch over the whole matrix); the chain runs on the
// device; the last triangular solve runs block by block and each finished
// block goes down on a second stream while the next is solved. Every result
// equals fb_zcholqr2's on the same matrix to the bit.

// The up and down streams of the current device, created once.
static int staging_streams(cudaStream_t* up, cudaStream_t* down) {
    static std::mutex mu;
    static cudaStream_t streams[64][2] = {};
    int dev = 0;
    FB_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) { set_error(FB_ENOTSUP, "cholqr2! staged: device %d", dev); return FB_ENOTSUP; }
    std::lock_guard<std::mutex> lock(mu);
    for (int i = 0; i < 2; ++i)
        if (!streams[dev][i])
            FB_CUDA(cudaStreamCreateWithFlags(&streams[dev][i], cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    *up = streams[dev][0];
    *down = streams[dev][1];
    return FB_OK;
}

namespace {
// Events of one staged call, destroyed when it returns.
struct EventSet {
    std::vector<cudaEvent_t> ev;
    ~EventSet() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    int make(cudaEvent_t* out) {
        cudaEvent_t e;
        FB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreateWithFlags");
        ev.push_back(e);
        *out = e;
        return FB_OK;
    }
};
}  // namespace

// Row blocks of a staged call: whole Gram chunks, at most STAGED_BLOCKS.
struct StagedBlocks {
    int64_t chunk_rows = 0;
    int nchunks = 0, nb = 0;
    std::vector<int> c0;
    int64_t max_rows = 0;
    void rows(int b, int64_t N, int64_t* r0, int64_t* r1) const {
        *r0 = (int64_t)c0[b] * chunk_rows;
        *r1 = std::min<int64_t>(N, (int64_t)c0[b + 1] * chunk_rows);
    }
};

static StagedBlocks staged_blocks(int64_t N, int k) {
    StagedBlocks B;
    gram_chunks(N, k, k, true, &B.chunk_rows, &B.nchunks);
    B.nb = B.nchunks < STAGED_BLOCKS ? B.nchunks : STAGED_BLOCKS;
    B.c0.resize(B.nb + 1);
    for (int b = 0; b <= B.nb; ++b) B.c0[b] = (int)((int64_t)B.nchunks * b / B.nb);
    for (int b = 0; b < B.nb; ++b) {
        int64_t r0, r1;
        B.rows(b, N, &r0, &r1);
        B.max_rows = std::max(B.max_rows, r1 - r0);
    }
    return B;
}

// The chain's workspace, then (for a ComplexF32 host tier) two narrow
// staging buffers of one row block each.
static size_t staged_stage_bytes(int64_t N, int k, int host_type) {
    if (host_type != FB_C64) return 0;
    return align_up((size_t)staged_blocks(N, k).max_rows * k * 8, 256);
}

int fb_zcholqr2_staged_blocks(int64_t N, int k, int* blocks) {
    if (!blocks || N < 1 || k < 1) { set_error(FB_EINVAL, "fb_zcholqr2_staged_blocks: bad argument"); return FB_EINVAL; }
    *blocks = staged_blocks(N, k).nb;
    return FB_OK;
}

int fb_zcholqr2_staged_workspace_size(int64_t N, int k, int host_type, size_t* bytes) {
    if (!bytes || N < 1 || k < 1 || (host_type != FB_C128 && host_type != FB_C64)) {
        set_error(FB_EINVAL, "fb_zcholqr2_staged_workspace_size: bad argument");
        return FB_EINVAL;
    }
    *bytes = cholqr_layout(N, k).total + 2 * staged_stage_bytes(N, k, host_type);
    return FB_OK;
}

int fb_zcholqr2_staged(void* const* host_panels, int host_type, const int64_t* host_ld, const int* panel_cols,
                       int npanels, fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr,
                       double shift_unit_roundoff, int* info, int* passes, void* workspace, size_t workspace_bytes,
                       fb_queue_t queue) {
    if (N < 1 || k < 1) {
        set_error(FB_EINVAL, "cholqr2!: N and k must be positive, got N=%lld, k=%d", (long long)N, k);
        return FB_EINVAL;
    }
    if (!host_panels || !host_ld || !panel_cols || npanels < 1 || !Y || !R) {
        set_error(FB_EINVAL, "fb_zcholqr2_staged: NULL argument");
        return FB_EINVAL;
    }
    if (host_type != FB_C128 && host_type != FB_C64) {
        set_error(FB_EINVAL, "fb_zcholqr2_staged: host panels are ComplexF64 (FB_C128) or ComplexF32 (FB_C64), got %d",
                  host_type);
        return FB_EINVAL;
    }
    if (!(shift_unit_roundoff >= 0.0 && shift_unit_roundoff < 1.0)) {
        set_error(FB_EINVAL, "fb_zcholqr2_staged: the unit roundoff of the shift must lie in [0, 1), got %g",
                  shift_unit_roundoff);
        return FB_EINVAL;
    }
    int cols = 0;
    for (int p = 0; p < npanels; ++p) {
        if (!host_panels[p] || panel_cols[p] < 1 || host_ld[p] < N) {
            set_error(FB_EDIM, "fb_zcholqr2_staged: panel %d is NULL, empty or has a leading dimension below N", p);
            return FB_EDIM;
        }
        cols += panel_cols[p];
    }
    if (cols != k) {
        set_error(FB_EDIM, "fb_zcholqr2_staged: the panels hold %d columns, the matrix %d", cols, k);
        return FB_EDIM;
    }
    if (ldy < N || ldr < k) { set_error(FB_EDIM, "fb_zcholqr2_staged: leading dimension too small"); return FB_EDIM; }
    if (((uintptr_t)Y | (uintptr_t)R) & 15) {
        set_error(FB_EINVAL, "fb_zcholqr2_staged: device pointers must be 16-byte aligned");
        return FB_EINVAL;
    }
    CholqrLayout L = cholqr_layout(N, k);
    const size_t stage_bytes = staged_stage_bytes(N, k, host_type);
    const size_t total = L.total + 2 * stage_bytes;
    if (!workspace || workspace_bytes < total || ((uintptr_t)workspace & 255)) {
        set_error(FB_ENOMEM, "fb_zcholqr2_staged: workspace must be 256-byte aligned and hold %zu bytes (got %zu)",
                  total, workspace_bytes);
        return FB_ENOMEM;
    }
    char* ws = static_cast<char*>(workspace);
    ChainStatus* st = reinterpret_cast<ChainStatus*>(ws + L.status);
    z64* G = reinterpret_cast<z64*>(ws + L.G);
    z64* U = reinterpret_cast<z64*>(ws + L.U);
    z64* Ra = reinterpret_cast<z64*>(ws + L.Ra);
    z64* Rb = reinterpret_cast<z64*>(ws + L.Rb);
    z64* gwork = reinterpret_cast<z64*>(ws + L.gwork);
    void* gram_ws = ws + L.gram;
    void* trsm_ws = ws + L.trsm;
    const size_t trsm_bytes = L.gram - L.trsm;
    const size_t gram_bytes = L.total - L.gram;
    char* stage[2] = {ws + L.total, ws + L.total + stage_bytes};
    cudaStream_t stream = stream_of(queue);
    z64* Yz = reinterpret_cast<z64*>(Y);
    const z64 one = zmake(1.0, 0.0), zero = zmake(0.0, 0.0);
    const bool narrow = host_type == FB_C64;
    const size_t hsize = narrow ? 8 : 16;
    cudaStream_t up, down;
    FB_TRY(staging_streams(&up, &down));
    const StagedBlocks B = staged_blocks(N, k);
    const int nb = B.nb;
    const int64_t sld = B.max_rows;   // leading dimension of a narrow staging block

    // One 2-D copy per panel of row block b, between host panel p (column
    // major, leading dimension host_ld[p]) and its columns of `dev` (Y
    // itself, or a narrow staging block whose rows start at r0).
    auto copy_block = [&](int b, bool to_device, cudaStream_t s) -> int {
        int64_t r0, r1;
        B.rows(b, N, &r0, &r1);
        if (r1 <= r0) return FB_OK;
        int col = 0;
        for (int p = 0; p < npanels; ++p) {
            char* dev = narrow ? stage[b & 1] + (size_t)col * sld * hsize
                               : reinterpret_cast<char*>(Yz + r0 + (int64_t)col * ldy);
            const size_t dpitch = narrow ? (size_t)sld * hsize : (size_t)ldy * sizeof(z64);
            char* host = static_cast<char*>(host_panels[p]) + (size_t)r0 * hsize;
            const size_t hpitch = (size_t)host_ld[p] * hsize;
            const size_t width = (size_t)(r1 - r0) * hsize;
            if (to_device)
                FB_CUDA(cudaMemcpy2DAsync(dev, dpitch, host, hpitch, width, panel_cols[p], cudaMemcpyHostToDevice, s),
                        "cudaMemcpy2DAsync");
            else
                FB_CUDA(cudaMemcpy2DAsync(host, hpitch, dev, dpitch, width, panel_cols[p], cudaMemcpyDeviceToHost, s),
                        "cudaMemcpy2DAsync");
            col += panel_cols[p];
        }
        return FB_OK;
    };

    EventSet events;
    std::vector<cudaEvent_t> widened(nb), sent(nb);
    cudaEvent_t start;
    FB_TRY(events.make(&start));
    FB_CUDA(cudaMemsetAsync(st, 0, sizeof(ChainStatus), stream), "cudaMemsetAsync");
    FB_CUDA(cudaEventRecord(start, stream), "cudaEventRecord");
    FB_CUDA(cudaStreamWaitEvent(up, start, 0), "cudaStreamWaitEvent");
    // Pass 1's Gram, block by block as the rows land (widened first when the
    // panels are narrow; a staging block is reused once its widening ran).
    for (int b = 0; b < nb; ++b) {
        if (narrow && b >= 2) FB_CUDA(cudaStreamWaitEvent(up, widened[b - 2], 0), "cudaStreamWaitEvent");
        FB_TRY(copy_block(b, true, up));
        cudaEvent_t landed;
        FB_TRY(events.make(&landed));
        FB_CUDA(cudaEventRecord(landed, up), "cudaEventRecord");
        FB_CUDA(cudaStreamWaitEvent(stream, landed, 0), "cudaStreamWaitEvent");
        if (narrow) {
            int64_t r0, r1;
            B.rows(b, N, &r0, &r1);
            FB_TRY(fb_convert_copy(Yz + r0, FB_C128, ldy, stage[b & 1], FB_C64, sld, r1 - r0, k, queue));
            FB_TRY(events.make(&widened[b]));
            FB_CUDA(cudaEventRecord(widened[b], stream), "cudaEventRecord");
        }
        FB_TRY(gram_partials_enqueue(Yz, ldy, Yz, ldy, N, k, k, true, gram_ws, gram_bytes, stream, st, GATE_HEALTHY,
                                     B.c0[b], B.c0[b + 1]));
    }
    FB_TRY(gram_reduce_enqueue(G, k, N, k, k, true, one, zero, gram_ws, stream, st, GATE_HEALTHY));
    FB_TRY(potrf_enqueue(G, k, k, N, U, k, nullptr, k, Ra, k, gwork, st, 1, GATE_HEALTHY, stream,
                         shift_unit_roundoff));
    FB_TRY(trsm_enqueue(Yz, ldy, N, k, U, k, trsm_ws, trsm_bytes, stream, st, GATE_HEALTHY));
    FB_TRY(gram_enqueue(G, k, Yz, ldy, Yz, ldy, N, k, k, one, zero, true, gram_ws, gram_bytes, stream, st,
                        GATE_HEALTHY));
    FB_TRY(potrf_enqueue(G, k, k, N, U, k, Ra, k, Rb, k, gwork, st, 2, GATE_HEALTHY, stream, 0.0));
    // Whether a third pass runs (or the chain stopped) decides which solve is
    // the last: read the status once here.
    ChainStatus hs;
    FB_CUDA(cudaMemcpyAsync(&hs, st, sizeof(ChainStatus), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
    FB_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const bool third = !hs.failed && (hs.shifted[1] | hs.shifted[2]);
    if (third) {
        FB_TRY(trsm_enqueue(Yz, ldy, N, k, U, k, trsm_ws, trsm_bytes, stream, st, GATE_HEALTHY));
        FB_TRY(gram_enqueue(G, k, Yz, ldy, Yz, ldy, N, k, k, one, zero, true, gram_ws, gram_bytes, stream, st,
                            GATE_HEALTHY));
        FB_TRY(potrf_enqueue(G, k, k, N, U, k, Rb, k, Ra, k, gwork, st, 3, GATE_HEALTHY, stream, 0.0));
        FB_CUDA(cudaMemcpyAsync(&hs, st, sizeof(ChainStatus), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
        FB_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    }
    if (!hs.failed) {
        // The last solve, block by block, each block going down once solved
        // (narrowed first when the panels are narrow, into a staging block
        // whose previous contents have gone down). A failed chain writes
        // nothing back: the panels keep Y.
        for (int b = 0; b < nb; ++b) {
            int64_t r0, r1;
            B.rows(b, N, &r0, &r1);
            FB_TRY(trsm_enqueue(Yz + r0, ldy, r1 - r0, k, U, k, trsm_ws, trsm_bytes, stream, st, GATE_HEALTHY));
            if (narrow) {
                if (b >= 2) FB_CUDA(cudaStreamWaitEvent(stream, sent[b - 2], 0), "cudaStreamWaitEvent");
                FB_TRY(fb_convert_copy(stage[b & 1], FB_C64, sld, Yz + r0, FB_C128, ldy, r1 - r0, k, queue));
            }
            cudaEvent_t solved;
            FB_TRY(events.make(&solved));
            FB_CUDA(cudaEventRecord(solved, stream), "cudaEventRecord");
            FB_CUDA(cudaStreamWaitEvent(down, solved, 0), "cudaStreamWaitEvent");
            FB_TRY(copy_block(b, false, down));
            FB_TRY(events.make(&sent[b]));
            FB_CUDA(cudaEventRecord(sent[b], down), "cudaEventRecord");
        }
        FB_CUDA(cudaStreamWaitEvent(stream, sent[nb - 1], 0), "cudaStreamWaitEvent");
    }
    int blocks = (int)((int64_t)k * k + 255) / 256;
    select_r_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<z64*>(R), ldr, Ra, Rb, k, st);
    FB_LAUNCHED("select_r_kernel");
    FB_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    int inf = 0;
    const int status = fb_zcholqr2_query(st, &inf, passes, nullptr);
    if (info) *info = inf;
    return status;
}

}  // extern "C"
