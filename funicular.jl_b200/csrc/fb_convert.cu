// convert_copy! (src/kernels.jl:7-20): elementwise conversion between two
// device views, used to widen a narrowed host tier's panels after the narrow
// bytes have crossed the bus and to narrow them on the way back
// (convert_staged!, src/panels.jl:365-371). Rounding is IEEE round to
// nearest, as Julia's convert(ComplexF32, x) does it.
#include "fb_common.cuh"

namespace fb {

template <typename D, typename S>
__device__ __forceinline__ D convert_elem(S s);

template <> __device__ __forceinline__ double2 convert_elem<double2, double2>(double2 s) { return s; }
template <> __device__ __forceinline__ double2 convert_elem<double2, float2>(float2 s) { return make_double2(s.x, s.y); }
template <> __device__ __forceinline__ float2 convert_elem<float2, double2>(double2 s) { return make_float2(__double2float_rn(s.x), __double2float_rn(s.y)); }
template <> __device__ __forceinline__ float2 convert_elem<float2, float2>(float2 s) { return s; }
template <> __device__ __forceinline__ double2 convert_elem<double2, double>(double s) { return make_double2(s, 0.0); }
template <> __device__ __forceinline__ double2 convert_elem<double2, float>(float s) { return make_double2(s, 0.0); }
template <> __device__ __forceinline__ float2 convert_elem<float2, double>(double s) { return make_float2(__double2float_rn(s), 0.f); }
template <> __device__ __forceinline__ float2 convert_elem<float2, float>(float s) { return make_float2(s, 0.f); }
template <> __device__ __forceinline__ double convert_elem<double, double>(double s) { return s; }
template <> __device__ __forceinline__ double convert_elem<double, float>(float s) { return (double)s; }
template <> __device__ __forceinline__ float convert_elem<float, double>(double s) { return __double2float_rn(s); }
template <> __device__ __forceinline__ float convert_elem<float, float>(float s) { return s; }

// Columns along y, rows along x (grid-strided), so no thread divides.
template <typename D, typename S>
__global__ void convert_kernel(D* __restrict__ dst, int64_t ldd, const S* __restrict__ src, int64_t lds,
                               int64_t rows, int64_t cols) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = blockIdx.y; j < cols; j += gridDim.y) {
        D* dcol = dst + j * ldd;
        const S* scol = src + j * lds;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride)
            dcol[i] = convert_elem<D, S>(scol[i]);
    }
}

template <typename D, typename S>
static int launch_convert(void* dst, int64_t ldd, const void* src, int64_t lds, int64_t rows, int64_t cols,
                          cudaStream_t stream) {
    const int64_t gy = cols < 65535 ? cols : 65535;
    int64_t gx = (rows + 255) / 256;
    const int64_t want = (int64_t)sm_count() * 16;
    const int64_t cap_x = (want + gy - 1) / gy;
    if (gx > cap_x) gx = cap_x;
    if (gx < 1) gx = 1;
    convert_kernel<D, S><<<dim3((unsigned)gx, (unsigned)gy), 256, 0, stream>>>(
        static_cast<D*>(dst), ldd, static_cast<const S*>(src), lds, rows, cols);
    FB_LAUNCHED("convert_kernel");
    return FB_OK;
}

static size_t elsize(int t) {
    switch (t) {
        case FB_C128: return 16;
        case FB_C64: return 8;
        case FB_F64: return 8;
        case FB_F32: return 4;
        default: return 0;
    }
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_convert_copy(void* dst, int dst_type, int64_t ldd, const void* src, int src_type, int64_t lds,
                    int64_t rows, int64_t cols, fb_queue_t queue) {
    if (elsize(dst_type) == 0 || elsize(src_type) == 0) {
        set_error(FB_EINVAL, "fb_convert_copy: unknown element type (%d, %d)", dst_type, src_type);
        return FB_EINVAL;
    }
    if (rows < 0 || cols < 0) { set_error(FB_EDIM, "fb_convert_copy: negative size"); return FB_EDIM; }
    if (rows == 0 || cols == 0) return FB_OK;
    if (!dst || !src) { set_error(FB_EINVAL, "fb_convert_copy: NULL pointer"); return FB_EINVAL; }
    if (ldd < rows || lds < rows) { set_error(FB_EDIM, "fb_convert_copy: leading dimension smaller than rows"); return FB_EDIM; }
    const bool dst_complex = dst_type == FB_C128 || dst_type == FB_C64;
    const bool src_complex = src_type == FB_C128 || src_type == FB_C64;
    if (src_complex && !dst_complex) {
        set_error(FB_EINVAL, "fb_convert_copy: a real destination cannot hold a complex source");
        return FB_EINVAL;
    }
    if ((((uintptr_t)dst) % elsize(dst_type)) || (((uintptr_t)src) % elsize(src_type))) {
        set_error(FB_EINVAL, "fb_convert_copy: misaligned pointer");
        return FB_EINVAL;
    }
    cudaStream_t s = stream_of(queue);
#define FB_CONV(DT, DTy, ST, STy) \
    if (dst_type == DT && src_type == ST) return launch_convert<DTy, STy>(dst, ldd, src, lds, rows, cols, s);
    FB_CONV(FB_C128, double2, FB_C128, double2)
    FB_CONV(FB_C128, double2, FB_C64, float2)
    FB_CONV(FB_C64, float2, FB_C128, double2)
    FB_CONV(FB_C64, float2, FB_C64, float2)
    FB_CONV(FB_C128, double2, FB_F64, double)
    FB_CONV(FB_C128, double2, FB_F32, float)
    FB_CONV(FB_C64, float2, FB_F64, double)
    FB_CONV(FB_C64, float2, FB_F32, float)
    FB_CONV(FB_F64, double, FB_F64, double)
    FB_CONV(FB_F64, double, FB_F32, float)
    FB_CONV(FB_F32, float, FB_F64, double)
    FB_CONV(FB_F32, float, FB_F32, float)
#undef FB_CONV
    set_error(FB_ENOTSUP, "fb_convert_copy: conversion %d <- %d not handled", dst_type, src_type);
    return FB_ENOTSUP;
}

}  // extern "C"
