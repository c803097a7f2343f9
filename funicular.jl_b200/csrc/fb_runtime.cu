// The device API half of the backend: memory, page-locked slabs, queues,
// events and pitched copies. Mirrors the contract of src/device_api.jl:5-138
// as the reference's CUDA extension implements it
// (ext/FunicularCUDAExt.jl:29-182), without any per-array stream bookkeeping:
// ordering between queues is the caller's events alone.
#include <atomic>
#include <cstdarg>
#include <mutex>
#include <vector>

#include "fb_common.cuh"
#include "fb_tma.cuh"

namespace fb {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    (void)status;
    g_last_error = buf;
}

int cuda_status(cudaError_t err, const char* what) {
    set_error(FB_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(err), cudaGetErrorName(err));
    return FB_ECUDA;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> counts;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)counts.size() <= dev) counts.resize(dev + 1, 0);
    if (counts[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        counts[dev] = n;
    }
    return counts[dev];
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

int encode_panel_map(CUtensorMap* map, const void* base, int64_t rows, int64_t cols, int64_t ld, int box_cols) {
    auto encode = tensor_map_encoder();
    if (!encode) {
        set_error(FB_ECUDA, "the driver does not provide cuTensorMapEncodeTiled");
        return FB_ECUDA;
    }
    if (rows < 1) rows = 1;
    if (cols < 1) cols = 1;
    cuuint64_t dims[2] = {(cuuint64_t)(2 * rows), (cuuint64_t)cols};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 16)};
    cuuint32_t box[2] = {16u, (cuuint32_t)box_cols};
    cuuint32_t elem[2] = {1u, 1u};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error(FB_ECUDA, "cuTensorMapEncodeTiled failed (%d) for a %lld x %lld panel, ld %lld, box %d columns",
                  (int)r, (long long)rows, (long long)cols, (long long)ld, box_cols);
        return FB_ECUDA;
    }
    return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_abi_version(void) { return FB_ABI_VERSION; }

const char* fb_last_error(void) { return g_last_error.c_str(); }

uint64_t fb_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int fb_device_count(int* count) {
    if (!count) { set_error(FB_EINVAL, "fb_device_count: count is NULL"); return FB_EINVAL; }
    int n = 0;
    cudaError_t err = cudaGetDeviceCount(&n);
    if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) {
        cudaGetLastError();
        *count = 0;
        return FB_OK;
    }
    FB_CUDA(err, "cudaGetDeviceCount");
    *count = n;
    return FB_OK;
}

int fb_set_device(int device) {
    FB_CUDA(cudaSetDevice(device), "cudaSetDevice");
    return FB_OK;
}

int fb_alloc_device(void** ptr, size_t nbytes) {
    if (!ptr) { set_error(FB_EINVAL, "fb_alloc_device: ptr is NULL"); return FB_EINVAL; }
    *ptr = nullptr;
    if (nbytes == 0) return FB_OK;
    cudaError_t err = cudaMalloc(ptr, nbytes);
    if (err == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        set_error(FB_ENOMEM, "fb_alloc_device: out of device memory allocating %zu bytes", nbytes);
        return FB_ENOMEM;
    }
    FB_CUDA(err, "cudaMalloc");
    // cudaMalloc is synchronous with respect to the device, so the buffer is
    // ready for any stream on return, which is what alloc_device promises.
    return FB_OK;
}

int fb_free_device(void* ptr) {
    if (!ptr) return FB_OK;
    FB_CUDA(cudaFree(ptr), "cudaFree");
    return FB_OK;
}

int fb_alloc_host_slab(void** ptr, size_t nbytes) {
    if (!ptr) { set_error(FB_EINVAL, "fb_alloc_host_slab: ptr is NULL"); return FB_EINVAL; }
    *ptr = nullptr;
    if (nbytes == 0) nbytes = 64;
    cudaError_t err = cudaHostAlloc(ptr, nbytes, cudaHostAllocPortable);
    if (err == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        set_error(FB_ENOMEM, "fb_alloc_host_slab: cannot page-lock %zu bytes of host memory", nbytes);
        return FB_ENOMEM;
    }
    FB_CUDA(err, "cudaHostAlloc");
    return FB_OK;
}

int fb_free_host_slab(void* ptr) {
    if (!ptr) return FB_OK;
    FB_CUDA(cudaFreeHost(ptr), "cudaFreeHost");
    return FB_OK;
}

int fb_pin_host(void* ptr, size_t nbytes) {
    if (!ptr || nbytes == 0) { set_error(FB_EINVAL, "fb_pin_host: empty range"); return FB_EINVAL; }
    FB_CUDA(cudaHostRegister(ptr, nbytes, cudaHostRegisterPortable), "cudaHostRegister");
    return FB_OK;
}

int fb_unpin_host(void* ptr) {
    if (!ptr) return FB_OK;
    FB_CUDA(cudaHostUnregister(ptr), "cudaHostUnregister");
    return FB_OK;
}

int fb_queue_create(fb_queue_t* queue) {
    if (!queue) { set_error(FB_EINVAL, "fb_queue_create: queue is NULL"); return FB_EINVAL; }
    cudaStream_t s = nullptr;
    FB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    *queue = reinterpret_cast<fb_queue_t>(s);
    return FB_OK;
}

int fb_queue_destroy(fb_queue_t queue) {
    if (!queue) return FB_OK;
    FB_CUDA(cudaStreamDestroy(stream_of(queue)), "cudaStreamDestroy");
    return FB_OK;
}

int fb_event_record(fb_queue_t queue, fb_event_t* event) {
    if (!event) { set_error(FB_EINVAL, "fb_event_record: event is NULL"); return FB_EINVAL; }
    cudaEvent_t e = nullptr;
    FB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreateWithFlags");
    cudaError_t err = cudaEventRecord(e, stream_of(queue));
    if (err != cudaSuccess) {
        cudaEventDestroy(e);
        return cuda_status(err, "cudaEventRecord");
    }
    *event = reinterpret_cast<fb_event_t>(e);
    return FB_OK;
}

int fb_event_destroy(fb_event_t event) {
    if (!event) return FB_OK;
    FB_CUDA(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(event)), "cudaEventDestroy");
    return FB_OK;
}

int fb_queue_wait_event(fb_queue_t queue, fb_event_t event) {
    if (!event) return FB_OK;
    FB_CUDA(cudaStreamWaitEvent(stream_of(queue), reinterpret_cast<cudaEvent_t>(event), 0),
            "cudaStreamWaitEvent");
    return FB_OK;
}

int fb_queue_sync(fb_queue_t queue) {
    FB_CUDA(cudaStreamSynchronize(stream_of(queue)), "cudaStreamSynchronize");
    return FB_OK;
}

int fb_event_sync(fb_event_t event) {
    if (!event) return FB_OK;
    FB_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(event)), "cudaEventSynchronize");
    return FB_OK;
}

int fb_event_query(fb_event_t event, int* done) {
    if (!done) { set_error(FB_EINVAL, "fb_event_query: done is NULL"); return FB_EINVAL; }
    if (!event) { *done = 1; return FB_OK; }
    cudaError_t err = cudaEventQuery(reinterpret_cast<cudaEvent_t>(event));
    if (err == cudaErrorNotReady) {
        cudaGetLastError();
        *done = 0;
        return FB_OK;
    }
    FB_CUDA(err, "cudaEventQuery");
    *done = 1;
    return FB_OK;
}

int fb_sync_all(void) {
    FB_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    return FB_OK;
}

int fb_graph_capture_begin(fb_queue_t queue) {
    if (!queue) { set_error(FB_EINVAL, "fb_graph_capture_begin: the default stream cannot be captured"); return FB_EINVAL; }
    FB_CUDA(cudaStreamBeginCapture(static_cast<cudaStream_t>(queue), cudaStreamCaptureModeThreadLocal),
            "cudaStreamBeginCapture");
    return FB_OK;
}

int fb_graph_capture_end(fb_queue_t queue, fb_graph_t* graph) {
    if (!queue || !graph) { set_error(FB_EINVAL, "fb_graph_capture_end: NULL argument"); return FB_EINVAL; }
    cudaGraph_t g = nullptr;
    FB_CUDA(cudaStreamEndCapture(static_cast<cudaStream_t>(queue), &g), "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t err = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    FB_CUDA(err, "cudaGraphInstantiate");
    *graph = exec;
    return FB_OK;
}

int fb_graph_launch(fb_graph_t graph, fb_queue_t queue) {
    if (!graph) { set_error(FB_EINVAL, "fb_graph_launch: NULL graph"); return FB_EINVAL; }
    FB_CUDA(cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph), static_cast<cudaStream_t>(queue)), "cudaGraphLaunch");
    return FB_OK;
}

int fb_graph_destroy(fb_graph_t graph) {
    if (graph) FB_CUDA(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph)), "cudaGraphExecDestroy");
    return FB_OK;
}

int fb_copy2d(void* dst, size_t dpitch, const void* src, size_t spitch,
              size_t width_bytes, size_t cols, fb_queue_t queue) {
    if (width_bytes == 0 || cols == 0) return FB_OK;
    if (!dst || !src) { set_error(FB_EINVAL, "fb_copy2d: NULL pointer"); return FB_EINVAL; }
    if (dpitch < width_bytes || spitch < width_bytes) {
        set_error(FB_EINVAL, "fb_copy2d: a pitch (%zu, %zu) is narrower than a column of %zu bytes",
                  dpitch, spitch, width_bytes);
        return FB_EINVAL;
    }
    if (queue == nullptr) {
        FB_CUDA(cudaMemcpy2D(dst, dpitch, src, spitch, width_bytes, cols, cudaMemcpyDefault), "cudaMemcpy2D");
        return FB_OK;
    }
    FB_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width_bytes, cols, cudaMemcpyDefault, stream_of(queue)),
            "cudaMemcpy2DAsync");
    return FB_OK;
}

}  // extern "C"
