/*
 * libfunicular_b200 — C ABI of the B200 device backend for Funicular's panel
 * linear algebra.
 *
 * Every entry point takes plain pointers, sizes and opaque queue handles, and
 * returns an int status (FB_OK = 0). A non-zero status leaves a message that
 * fb_last_error() returns on the same host thread. The statuses map onto the
 * exceptions the reference raises:
 *   FB_EINVAL  -> ArgumentError      FB_EDIM   -> DimensionMismatch
 *   FB_ENOTSPD -> ArgumentError (the Gram matrix is not positive definite even
 *                 after the shift, src/panelblas.jl:153)
 *
 * Matrices are column major ComplexF64 (16 bytes, re then im), the first
 * dimension contiguous, with a leading dimension in elements, exactly the
 * layout Funicular's panels and staging buffers have
 * (ext/FunicularCUDAExt.jl:154-163). Device pointers must be 16-byte aligned.
 *
 * A queue is a non-blocking CUDA stream (fb_queue_t). Passing NULL as a
 * queue means "complete on return" for copies (the reference's queue=nothing)
 * and the legacy per-thread default stream for kernels. Kernels never
 * synchronize the host unless their comment says so.
 *
 * Citations name the reference function each entry point replaces, as
 * file:line within Funicular.jl.
 */
#ifndef FUNICULAR_B200_H
#define FUNICULAR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FB_ABI_VERSION 1

enum fb_status_code {
    FB_OK = 0,
    FB_EINVAL = 1,    /* bad argument: ArgumentError */
    FB_EDIM = 2,      /* shape mismatch: DimensionMismatch */
    FB_ENOMEM = 3,    /* allocation failed or workspace too small */
    FB_ENOTSPD = 4,   /* not positive definite even after the shift */
    FB_ECUDA = 5,     /* the CUDA runtime reported an error */
    FB_ENOTSUP = 6    /* shape or type this build does not handle */
};

/* Element types for fb_convert_copy (ComplexF64, ComplexF32, Float64, Float32). */
enum fb_eltype { FB_C128 = 0, FB_C64 = 1, FB_F64 = 2, FB_F32 = 3 };

typedef struct { double re, im; } fb_z128;
typedef void* fb_queue_t;
typedef void* fb_event_t;
typedef void* fb_graph_t;

/* ---- library ---------------------------------------------------------- */

int fb_abi_version(void);
/* The message of the last failing call on this host thread ("" if none). */
const char* fb_last_error(void);
/* Kernels this library has launched in this process, all devices together. */
uint64_t fb_kernel_launches(void);
/* Number of visible CUDA devices (0 on a machine without a GPU). */
int fb_device_count(int* count);
int fb_set_device(int device);

/* ---- device API: src/device_api.jl:5-138, ext/FunicularCUDAExt.jl ------ */

/* alloc_device(backend, T, dims) (src/device_api.jl:19,
 * ext/FunicularCUDAExt.jl:32-40). Complete on return. */
int fb_alloc_device(void** ptr, size_t nbytes);
int fb_free_device(void* ptr);

/* alloc_host_slab(backend, nbytes) (src/device_api.jl:28,
 * ext/FunicularCUDAExt.jl:45-49): page-locked host memory, so that copies
 * out of it are asynchronous. The pointer is at least 64-byte aligned
 * (SLAB_ALIGN, src/device_api.jl:140). */
int fb_alloc_host_slab(void** ptr, size_t nbytes);
int fb_free_host_slab(void* ptr);
/* Page-locks host memory the caller already owns (CUDA.pin in the
 * reference's CUDA backend). */
int fb_pin_host(void* ptr, size_t nbytes);
int fb_unpin_host(void* ptr);

/* make_queue(backend) (src/device_api.jl:53, ext/FunicularCUDAExt.jl:73-76):
 * a non-blocking stream, so it never serializes against the legacy default
 * stream. */
int fb_queue_create(fb_queue_t* queue);
int fb_queue_destroy(fb_queue_t queue);
/* record_event(backend, queue) (src/device_api.jl:81,
 * ext/FunicularCUDAExt.jl:91-95): a new timing-free event recorded on queue. */
int fb_event_record(fb_queue_t queue, fb_event_t* event);
int fb_event_destroy(fb_event_t event);
/* wait_event(backend, queue, event) (src/device_api.jl:88,
 * ext/FunicularCUDAExt.jl:99-102): a device-side wait, the host carries on. */
int fb_queue_wait_event(fb_queue_t queue, fb_event_t event);
/* sync_queue / sync_event / sync_all (src/device_api.jl:95,102,109). A
 * failure of earlier work on the queue surfaces here as FB_ECUDA. */
int fb_queue_sync(fb_queue_t queue);
int fb_event_sync(fb_event_t event);
/* *done = 1 once the event has been signalled. */
int fb_event_query(fb_event_t event, int* done);
int fb_sync_all(void);

/* Stream capture into a CUDA graph, for callers that replay a fixed
 * sequence of launches (a batch of cholqr2! instances, a whole sweep step).
 * No counterpart in the reference's device API. Capture begins on a queue
 * (not NULL), every library call that enqueues on that queue until
 * fb_graph_capture_end is recorded instead of run, and the instantiated graph
 * replays them with one fb_graph_launch. Pointers and sizes are baked in. */
int fb_graph_capture_begin(fb_queue_t queue);
int fb_graph_capture_end(fb_queue_t queue, fb_graph_t* graph);
int fb_graph_launch(fb_graph_t graph, fb_queue_t queue);
int fb_graph_destroy(fb_graph_t graph);

/* h2d!/d2h! and device-to-device copies (src/device_api.jl:37,45;
 * copy_region! at ext/FunicularCUDAExt.jl:138-152): a 2-D copy of `cols`
 * columns of `width_bytes` each, the columns `dpitch`/`spitch` bytes apart.
 * Covers a whole panel, a column range of a staging buffer and a row block
 * slice of a panel. queue == NULL: complete on return; otherwise enqueued. */
int fb_copy2d(void* dst, size_t dpitch, const void* src, size_t spitch,
              size_t width_bytes, size_t cols, fb_queue_t queue);

/* ---- kernels: src/kernels.jl ----------------------------------------- */

/* convert_copy!(backend, dst, src) (src/kernels.jl:14): elementwise
 * conversion between two rows x cols device views with leading dimensions
 * ldd and lds (in elements of their own type). Complex to real is refused. */
int fb_convert_copy(void* dst, int dst_type, int64_t ldd,
                    const void* src, int src_type, int64_t lds,
                    int64_t rows, int64_t cols, fb_queue_t queue);

/* gram_accumulate!(backend, C, A, B, alpha, beta) (src/kernels.jl:40):
 * C <- alpha * A^H B + beta * C with A rows x kA, B rows x kB, C kA x kB.
 * beta == 0 overwrites C without reading it (a pooled buffer may hold NaN,
 * src/kernels.jl:29-30). When A and B are the same view (same pointer, ld and
 * width) only the upper triangle is computed and the lower one is its
 * conjugate mirror, so the result is Hermitian to the bit. The reduction
 * order depends only on rows, kA, kB and the device, never on the caller's
 * pipelining, so repeated calls give identical bits.
 * workspace must hold fb_zgram_workspace_size bytes of device memory. */
int fb_zgram_workspace_size(int64_t rows, int kA, int kB, int hermitian, size_t* bytes);
int fb_zgram(fb_z128* C, int64_t ldc,
             const fb_z128* A, int64_t lda, const fb_z128* B, int64_t ldb,
             int64_t rows, int kA, int kB, fb_z128 alpha, fb_z128 beta,
             void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* gram_accumulate! for callers that cannot allocate device memory. No
 * counterpart in the reference. fb_zgram needs a workspace from its caller;
 * some callers have none to give: a host whose allocator has promised every
 * device byte to a budgeted pool (a Funicular plan checks each buffer against
 * device_budget, and its sweep loop must not allocate at all), or a host that
 * cannot afford cudaMalloc's implicit device synchronization in the middle of
 * a pipelined sweep. This entry point computes the same thing as fb_zgram,
 * with the same bits, but keeps its partial tiles in a scratch array built
 * into the library: 32 MiB, held on every GPU that loads the library until
 * the process exits. Shapes whose scratch would not fit in it
 * (fb_zgram_workspace_size above 32 MiB, which takes many 64 x 64 output
 * tiles: on a 148-SM B200 every Gram of at most 128 columns a side fits,
 * whatever the row count) are refused with FB_ENOMEM before anything is
 * enqueued. The first call on each device looks up the array's device
 * address and keeps it for the life of the process; make that call before any
 * stream capture begins, and do not use this entry point across a
 * cudaDeviceReset, after which the kept address is stale. All calls share the
 * one array: two calls whose work can overlap on the GPU (different queues
 * with no event ordering them) race on it, while calls on one queue are safe.
 * Each call writes every part of the array it reads, so nothing has to be
 * cleared between calls. The call allocates nothing. */
int fb_zgram_static(fb_z128* C, int64_t ldc,
                    const fb_z128* A, int64_t lda, const fb_z128* B, int64_t ldb,
                    int64_t rows, int kA, int kB, fb_z128 alpha, fb_z128 beta, fb_queue_t queue);

/* rdiv_upper!(backend, Y, R) (src/kernels.jl:108): Y <- Y R^-1 in place for
 * an upper triangular, non-unit k x k R; Y is rows x k with leading
 * dimension ldy (a row block view of a staging buffer is fine). For k <= 64
 * the solve runs on the FP64 tensor cores and needs a workspace of
 * fb_ztrsm_workspace_size bytes (72 KB at k = 64, 0 past 64): a product by
 * inv(R) when cond_1(R) <= 16, a blocked solve with inverted 8 x 8 diagonal
 * blocks when those are well conditioned, plain substitution otherwise; the
 * choice is made on the device. */
int fb_ztrsm_workspace_size(int k, size_t* bytes);
int fb_ztrsm_right_upper(fb_z128* Y, int64_t ldy, int64_t rows, int k,
                         const fb_z128* R, int64_t ldr, void* workspace, size_t workspace_bytes,
                         fb_queue_t queue);

/* rightmul_gemm!(backend, dst, A, C) (src/kernels.jl:73): dst <- A C with A
 * rows x s, C s x r, dst rows x r. dst must not overlap A. */
int fb_zgemm_right(fb_z128* dst, int64_t ldd, const fb_z128* A, int64_t lda,
                   int64_t rows, int s, const fb_z128* C, int64_t ldc, int r,
                   fb_queue_t queue);

/* cholesky_upper(G, N, k) (src/panelblas.jl:148-155) on the device: U upper
 * with U^H U = G, reading G's upper triangle. When G is not positive
 * definite it factors G + s I with s = 11 N k eps(Float64) ||G||_F instead.
 * If Rin is non-NULL, Rout <- U * Rin (the R2 * R product of
 * src/panelblas.jl:133,136); Rout must not alias Rin. U and Rout are written
 * in full, zeros below the diagonal. Synchronizes `queue` and reports:
 * *shifted = 1 if the shift was taken, *shift = s. Returns FB_ENOTSPD when
 * even G + s I fails. workspace: fb_zpotrf_workspace_size bytes. */
int fb_zpotrf_workspace_size(int k, size_t* bytes);
int fb_zpotrf_shifted(fb_z128* U, int64_t ldu, const fb_z128* G, int64_t ldg,
                      int k, int64_t N, const fb_z128* Rin, int64_t ldrin,
                      fb_z128* Rout, int64_t ldrout,
                      int* shifted, double* shift,
                      void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* cholqr2!(Y) (src/panelblas.jl:130-146) on a device-resident matrix: two
 * passes of gram -> cholesky_upper -> rdiv_rows!, a third pass when either
 * shifted, R = R3 R2 R1 written to R (k x k, zeros below the diagonal).
 * Every step runs on `queue`; the branch to the third pass and the stop after
 * a failed factorization are taken on the device, so the call enqueues a
 * fixed sequence of launches. With info != NULL the call synchronizes and
 * sets *info = 0, or the 1-based pass whose Gram was not positive definite
 * (returning FB_ENOTSPD); *passes = 2 or 3 if non-NULL. With info == NULL it
 * returns at once and fb_zcholqr2_query reads the outcome after the queue
 * has drained. workspace: fb_zcholqr2_workspace_size bytes, 256-byte
 * aligned; the same workspace must not be used by two calls in flight. */
int fb_zcholqr2_workspace_size(int64_t N, int k, size_t* bytes);
int fb_zcholqr2(fb_z128* Y, int64_t ldy, int64_t N, int k,
                fb_z128* R, int64_t ldr, int* info, int* passes,
                void* workspace, size_t workspace_bytes, fb_queue_t queue);
int fb_zcholqr2_query(const void* workspace, int* info, int* passes,
                      double* shifts /* 3 entries, or NULL */);

/* cholqr2!(Y) (src/panelblas.jl:130-146) end to end for a matrix held in
 * page-locked host panels (the resident path of a PanelMatrix whose panels
 * live on the host tier, src/panels.jl:365-458, narrowed tiers included,
 * src/panels.jl:94-122): panel p holds panel_cols[p] consecutive columns,
 * column major with leading dimension host_ld[p] >= N, of element type
 * host_type (FB_C128, or FB_C64 for a ComplexF32 tier); the panels together
 * hold the k columns in order. Y (device, N x k ComplexF64, leading dimension
 * ldy) is the staging copy. The panels go up in row blocks on a library-owned
 * stream while pass 1's Gram consumes the blocks already landed (narrow
 * blocks widened on the device first); the last triangular solve runs block
 * by block, each solved block going back into the panels (narrowed on the
 * device) on a second stream while the next is solved. All arithmetic is
 * FP64. shift_unit_roundoff = 0 runs cholqr2!; u in (0, 1) runs the shifted
 * CholeskyQR3 of fb_zcholqr3_shifted with that unit roundoff. Q replaces Y in
 * the panels and R (device) is as in fb_zcholqr2; for ComplexF64 panels both
 * equal fb_zcholqr2's (fb_zcholqr3_shifted's) on the same matrix to the bit.
 * Synchronizes: it reads the chain's status once after pass 2 (and after
 * pass 3) and returns when Q is in the panels. A chain that stops on a Gram
 * that is not positive definite writes nothing back (the panels keep Y) and
 * returns FB_ENOTSPD with *info set. Workspace:
 * fb_zcholqr2_staged_workspace_size bytes, 256-byte aligned (the chain's, plus
 * two narrow staging blocks for FB_C64). fb_zcholqr2_staged_blocks gives the
 * number of row blocks. */
int fb_zcholqr2_staged_blocks(int64_t N, int k, int* blocks);
int fb_zcholqr2_staged_workspace_size(int64_t N, int k, int host_type, size_t* bytes);
int fb_zcholqr2_staged(void* const* host_panels, int host_type, const int64_t* host_ld, const int* panel_cols,
                       int npanels, fb_z128* Y, int64_t ldy, int64_t N, int k, fb_z128* R, int64_t ldr,
                       double shift_unit_roundoff, int* info, int* passes, void* workspace, size_t workspace_bytes,
                       fb_queue_t queue);

/* The shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Zhang, Yamamoto,
 * SIAM J. Sci. Comput. 2020), the orthonormalization the north-star backend
 * adds for a ComplexF32 storage tier (no counterpart in the reference, whose
 * cholqr2! shifts only a pass whose factorization failed,
 * src/panelblas.jl:148-155): pass 1 factors G + s I unconditionally with
 * s = 11 (N k + k (k+1)) u ||G||_F, passes 2 and 3 are plain, R = R3 R2 R1.
 * unit_roundoff = u, in (0, 1): 2^-53 when Y holds FP64 values throughout,
 * 2^-24 when it is rounded to ComplexF32 between passes. Same workspace,
 * status and query as fb_zcholqr2; *passes = 3 on success. */
int fb_zcholqr3_shifted(fb_z128* Y, int64_t ldy, int64_t N, int k,
                        fb_z128* R, int64_t ldr, double unit_roundoff, int* info, int* passes,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* The first factorization of the shifted CholeskyQR3 for a caller that runs
 * the passes itself (the streamed form): as fb_zpotrf_shifted, but G + s I is
 * factored at once with s = 11 (N k + k (k+1)) u ||G||_F and not retried;
 * *shift = s. Synchronizes `queue`; FB_ENOTSPD when even G + s I fails. */
int fb_zpotrf_forced_shift(fb_z128* U, int64_t ldu, const fb_z128* G, int64_t ldg,
                           int k, int64_t N, const fb_z128* Rin, int64_t ldrin,
                           fb_z128* Rout, int64_t ldrout, double unit_roundoff, double* shift,
                           void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* ---- operators: src/operator.jl ------------------------------------- */

/* The matrix-free operator of the streamed range finder: Y[:, c] <-
 * (-Lap_7 + shift I) X[:, c] for c < cols on an nx x ny x nz grid, grid point
 * (x, y, z) at row x + nx (y + ny z), unit spacing, zero outside the grid:
 * (G v)_p = (6 + shift) v_p - (sum of the six neighbours of p). The
 * panel-capable mul! that apply_operator! (src/operator.jl:80-87) hands a
 * resident panel to. Y and X must not overlap. */
int fb_zlaplace7_apply(fb_z128* Y, int64_t ldy, const fb_z128* X, int64_t ldx,
                       int nx, int ny, int nz, int cols, fb_z128 shift, fb_queue_t queue);

/* ---- tensor-core form ------------------------------------------------- */

/* gram_accumulate!(backend, C, A, A, alpha, beta) (src/kernels.jl:40) with
 * A === B, on the integer tensor cores: C <- alpha A^H A + beta C for a
 * rows x k device matrix A (1 <= k <= 64, rows <= 2^30, 16-byte aligned).
 * Every FP64 entry is split into seven 8-bit slices against a power-of-two
 * scale of its column (55 bits kept); the 28 slice products that reach FP64
 * accuracy are exact in 32-bit integer accumulators and recovered to FP64
 * with power-of-two weights. The result is exactly Hermitian and
 * deterministic; its error is of the order of FP64 rounding relative to the
 * product of the column maxima. A non-finite entry makes the whole result
 * NaN. workspace: at least fb_zgram_tc_workspace_size bytes, 256-byte
 * aligned. */
int fb_zgram_tc_workspace_size(int64_t rows, int k, size_t* bytes);
int fb_zgram_tc(fb_z128* C, int64_t ldc, const fb_z128* A, int64_t lda,
                int64_t rows, int k, fb_z128 alpha, fb_z128 beta,
                void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* cholqr2!(Y) in the tensor-core form: as fb_zcholqr2, with every Gram of
 * the chain computed by fb_zgram_tc (k <= 64); the Cholesky factorizations,
 * the shift and the triangular solves stay in FP64. Same workspace
 * (fb_zcholqr2_workspace_size), same status and query. */
int fb_zcholqr2_tc(fb_z128* Y, int64_t ldy, int64_t N, int k,
                   fb_z128* R, int64_t ldr, int* info, int* passes,
                   void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* Many independent cholqr2! instances of uneven N and k (the batched range
 * finder; no counterpart in the reference, which orthonormalizes one
 * PanelMatrix per call): instance i is Y[i] (N[i] x k[i], leading dimension
 * ldy[i]) with its R in R[i] (ldr[i]). The instances' chains run on up to
 * eight (fb_tune_set_batch_lanes) library-owned streams forked from `queue`
 * and joined back into it
 * (each chain on one stream, in the same launch sequence as a single call,
 * so each instance's bits equal its own fb_zcholqr2's); each keeps its own
 * status block, read by fb_zcholqr2_batched_query after the queue drained
 * (info[i] = the failing pass or 0, passes[i] = 2 or 3). tensor_form != 0
 * runs every Gram on the integer tensor cores (all k[i] <= 64). Nothing
 * synchronizes, so the whole batch can be captured into one CUDA graph
 * (fb_graph_capture_begin) and replayed with one launch. workspace:
 * fb_zcholqr2_batched_workspace_size bytes, 256-byte aligned. */
int fb_zcholqr2_batched_workspace_size(const int64_t* N, const int* k, int count, size_t* bytes);
int fb_zcholqr2_batched(fb_z128* const* Y, const int64_t* ldy, const int64_t* N, const int* k,
                        fb_z128* const* R, const int64_t* ldr, int count, int tensor_form,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue);
int fb_zcholqr2_batched_query(const void* workspace, int count, int* info, int* passes);

/* The same batch (the same arguments, status blocks and query) as ONE
 * persistent kernel launch: a grid of one CTA per SM takes jobs from a ticket
 * counter (the Gram chunks, factors and solve chunks of every pass of every
 * instance), with device-side arrival counters and ready flags between them,
 * so a batch is a memset and one launch (one more launch per 384 instances)
 * and captures into a graph of those nodes. FP64 form, every k[i] <= 64
 * (FB_ENOTSUP otherwise: fb_zcholqr2_batched takes any k). Each instance's
 * bits depend only on its own (N, k), not on the rest of the batch, but its
 * Gram chunking differs from fb_zcholqr2's, so they are not those of a single
 * call. A device-side wait that gives up (2 s; it cannot happen unless the
 * kernel is broken) stops the kernel and makes the query return FB_ECUDA.
 * workspace: fb_zcholqr2_batched_persistent_workspace_size bytes, 256-byte
 * aligned; read by fb_zcholqr2_batched_query after the queue drained. */
int fb_zcholqr2_batched_persistent_workspace_size(const int64_t* N, const int* k, int count, size_t* bytes);
int fb_zcholqr2_batched_persistent(fb_z128* const* Y, const int64_t* ldy, const int64_t* N, const int* k,
                                   fb_z128* const* R, const int64_t* ldr, int count,
                                   void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* ---- differentiation: the adjoints behind the rrules ------------------
 * The reference has no rrule (Project.toml:6-9 has no ChainRulesCore); these
 * are the kernels a ChainRulesCore.rrule for cholqr2! (src/panelblas.jl:130)
 * and project (src/panelblas.jl:268) calls in its pullback. */

/* The pullback of (Q, R) = cholqr2!(Y): Ybar <- (Qbar + Q H) R^-H with
 * H = copyltu(R Rbar^H - Qbar^H Q) (the Hermitian matrix with the strictly
 * lower triangle of its argument, that triangle's conjugate transpose above
 * the diagonal and the real part of the diagonal on it). Y is the ORIGINAL
 * input (N x k) and R the factor cholqr2! returned: Q is recomputed as
 * Y R^-1 inside the products, never stored. Qbar (N x k) and Rbar (k x k) may
 * each be NULL for a zero cotangent; only Rbar's upper triangle and the real
 * part of its diagonal matter. Ybar may be Qbar itself (same pointer and
 * leading dimension) and must not overlap Y. Runs on the FP64 tensor cores
 * for k <= 64 (DMMA), on the FP64 pipes past that. workspace:
 * fb_zcholqr2_adjoint_workspace_size bytes, 256-byte aligned. Enqueues only. */
int fb_zcholqr2_adjoint_workspace_size(int64_t N, int k, size_t* bytes);
int fb_zcholqr2_adjoint(fb_z128* Ybar, int64_t ldyb, const fb_z128* Y, int64_t ldy,
                        const fb_z128* R, int64_t ldr, const fb_z128* Qbar, int64_t ldqb,
                        const fb_z128* Rbar, int64_t ldrb, int64_t N, int k,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* The pullback of S = project(Q, G) = Q^H (G Q) with respect to Q:
 * Qbar <- [Qbar +] (G Q) Sbar^H + (G^H Q) Sbar, with GQ = G Q and GhQ =
 * G^H Q the operator images the caller computed (N x k). GhQ == NULL means G
 * is Hermitian: then Qbar gets (G Q)(Sbar + Sbar^H) in one product.
 * accumulate != 0 adds to Qbar, 0 overwrites it (NaN in it included). Qbar
 * must not overlap GQ or GhQ. workspace: fb_zproject_adjoint_workspace_size
 * bytes, 256-byte aligned. Enqueues only. */
int fb_zproject_adjoint_workspace_size(int k, size_t* bytes);
int fb_zproject_adjoint(fb_z128* Qbar, int64_t ldqb, const fb_z128* GQ, int64_t ldgq,
                        const fb_z128* GhQ, int64_t ldghq, const fb_z128* Sbar, int64_t ldsb,
                        int64_t N, int k, int accumulate,
                        void* workspace, size_t workspace_bytes, fb_queue_t queue);

/* A Hermitian band operator (the G of the differentiation workload; no
 * counterpart in the reference, whose operators are user callables behind
 * apply_operator!, src/operator.jl:80-87): Y[:, c] <- G X[:, c] for c < cols,
 * G N x N Hermitian with kd superdiagonals, stored by diagonals: Dg is
 * N x (kd + 1), leading dimension lddg, Dg[i + d lddg] = G[i, i + d]
 * (entries with i + d >= N are ignored, as is the imaginary part of the main
 * diagonal). Y and X must not overlap. */
int fb_zhband_apply(fb_z128* Y, int64_t ldy, const fb_z128* X, int64_t ldx,
                    const fb_z128* Dg, int64_t lddg, int64_t N, int kd, int cols,
                    fb_queue_t queue);

/* ---- autotuning -------------------------------------------------------
 * No counterpart in the reference. The library keeps a table of tile-shape
 * choices per shape class (floor(log2 rows), columns) that its kernels read
 * when they lay out a launch; an autotuner (funicular_b200.autotune) times
 * candidates on the device and fills it. Untuned shapes keep the built-in
 * choice. For the Gram, the entry is a shift of its row-chunk count: 0 is
 * one wave of CTAs over the GPU, s > 0 divides the count by 2^s (longer
 * chunks), s < 0 multiplies it (shorter ones); shift in [-3, 8]. The chunk
 * count fixes the reduction order, so a shape's results are reproducible to
 * the bit for a fixed table, and fb_zgram_workspace_size follows the table:
 * tune before sizing workspaces. */
int fb_tune_set_gram_chunks(int64_t rows, int k, int shift);
int fb_tune_get_gram_chunks(int64_t rows, int k, int* shift);
/* Clears the Gram entries (the batch's lane count is kept). */
int fb_tune_clear(void);
/* The number of stream lanes fb_zcholqr2_batched spreads a batch over, in
 * [1, 16], 8 untuned; fb_zcholqr2_batched_workspace_size follows it. */
int fb_tune_set_batch_lanes(int lanes);
int fb_tune_get_batch_lanes(int* lanes);

/* ---- ghost panels: src/ghosts.jl ------------------------------------- */

/* The device fill behind GhostPanels(T, N, k; seed) (replaces the host
 * generation of generate_panel! / stage_host!(panel, ::GhostTier, plan) at
 * src/ghosts.jl:97-122 followed by materialize! of the staged panel, and
 * materialize!(dst, panel, rows, ...) for a row block, src/panels.jl:427-431).
 * Writes the rows x cols block whose top left entry is (row0, col0) of the
 * ghost matrix (0-based, col0 the column in the full matrix) into dst,
 * leading dimension ld, element type dst_type. Entry (r, c) is a function of
 * (seed, r, c) only: Philox4x32-10 with counter (r, c) and key seed gives two
 * uniforms, Box-Muller turns them into standard normals (for a complex
 * eltype, real and imaginary parts of variance 1/2 each). value_type rounds
 * the values to that precision before they are stored (FB_C64/FB_F32: what
 * a narrowed host tier holds); it must be complex exactly when dst_type is.
 * The stream differs from the reference's Julia Xoshiro stream, which is
 * itself defined only within one Julia version (src/ghosts.jl:34-38). */
int fb_ghost_fill(void* dst, int dst_type, int64_t ld, int64_t rows, int64_t cols,
                  int64_t row0, int64_t col0, uint64_t seed, int value_type,
                  fb_queue_t queue);

#ifdef __cplusplus
}
#endif

#endif /* FUNICULAR_B200_H */
