// Shared definitions for libfunicular_b200: status handling, complex arithmetic
// on ComplexF64 stored as interleaved (re, im) doubles, and launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#include "funicular_b200.h"

namespace fb {

// The message behind the last non-zero status returned on this host thread.
void set_error(int status, const char* fmt, ...);
int cuda_status(cudaError_t err, const char* what);
int sm_count();
// Every kernel launch of this library goes through FB_LAUNCHED, which counts it.
void count_launch();

#define FB_TRY(expr)                       \
    do {                                   \
        int fb_try_status_ = (expr);       \
        if (fb_try_status_ != FB_OK)       \
            return fb_try_status_;         \
    } while (0)

#define FB_CUDA(expr, what)                                  \
    do {                                                     \
        cudaError_t fb_cuda_err_ = (expr);                   \
        if (fb_cuda_err_ != cudaSuccess)                     \
            return ::fb::cuda_status(fb_cuda_err_, what);    \
    } while (0)

// Checks the launch that was just issued. Only the launch configuration is
// checked here: errors raised while the kernel runs surface at the next
// synchronizing call on the queue.
#define FB_LAUNCHED(what)                  \
    do {                                   \
        ::fb::count_launch();              \
        FB_CUDA(cudaGetLastError(), what); \
    } while (0)

inline cudaStream_t stream_of(fb_queue_t q) { return reinterpret_cast<cudaStream_t>(q); }

// ComplexF64 as the device sees it: 16 bytes, re then im, 16-byte aligned so
// that one element moves with one 128-bit load or store.
using z64 = double2;

__host__ __device__ inline z64 zmake(double re, double im) { return make_double2(re, im); }

// acc += conj(a) * b, each real operation a fused multiply-add.
__device__ __forceinline__ void zmac_conj(z64& acc, z64 a, z64 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

// acc -= a * b
__device__ __forceinline__ void zmsub(z64& acc, z64 a, z64 b) {
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}

// acc += a * b
__device__ __forceinline__ void zmac(z64& acc, z64 a, z64 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

__device__ __forceinline__ z64 zmul(z64 a, z64 b) {
    return zmake(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// Status words that chain the kernels of one orthonormalization on the
// device: a failed Cholesky stops every later kernel of the chain, and the
// optional third pass runs only when a shift fired in the first two.
struct ChainStatus {
    int failed;        // 0, or the pass (1-based) whose Gram was not positive definite
    int shifted[4];    // shifted[p] = 1 when pass p factored G + sI
    int timeout;       // where a device-side wait of the batch kernel gave up (0: none)
    int pad[2];
    double shift[4];   // the shift s of pass p, when one was taken
    double norm[4];    // ||G||_F of pass p
};

enum Gate : int {
    GATE_ALWAYS = 0,    // run unconditionally
    GATE_HEALTHY = 1,   // run unless an earlier pass failed
    GATE_THIRD = 2,     // run only if healthy and a shift fired in pass 1 or 2
};

__device__ __forceinline__ bool gated_off(const ChainStatus* st, int gate) {
    if (st == nullptr || gate == GATE_ALWAYS) return false;
    if (st->failed != 0) return true;
    if (gate == GATE_THIRD) return !(st->shifted[1] | st->shifted[2]);
    return false;
}

inline size_t align_up(size_t n, size_t a) { return (n + a - 1) / a * a; }

// Makes a pointer opaque to the optimizer at this point, so loads through it
// inside a loop body are issued in that body rather than hoisted out of the
// loop into registers (which, for a k x k factor, is more registers than a
// thread has).
template <typename T>
__device__ __forceinline__ const T* opaque(const T* p) {
    asm volatile("" : "+l"(p));
    return p;
}

// p, but only once v is known: `zero` is a kernel argument that is always 0,
// which the compiler cannot see, so the address really depends on v. A long
// unrolled sweep of loads threaded through this issues its loads a group at a
// time instead of hoisting all of them (and spilling).
template <typename T>
__device__ __forceinline__ const T* hold(const T* p, double v, int zero) {
    return p + (zero & (int)__double_as_longlong(v));
}

// A 16-byte shared memory load the compiler keeps in program order with the
// other loads of this kind, so a long unrolled sweep over a factor does not
// turn into hundreds of loads issued ahead of their use.
__device__ __forceinline__ z64 lds_ordered(const z64* p) {
    z64 v;
    unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}

}  // namespace fb
