// runtime.cu -- controls, memory, copies and error reporting of the C ABI.
//
// Replaces the reference's Controls (src/core/controls.hpp:12-28: one
// device, an in-order queue and an out-of-order queue) and
// create_controls/show_devices (src/common/env.cpp:7-54) with one CUDA
// device, one stream and a stream-ordered memory pool.  There is no JIT
// kernel cache (src/core/kernel_cache.hpp): every kernel is compiled ahead
// of time for sm_100a.
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"

namespace clb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int status, const std::string &msg) {
    g_last_error = std::string(clb_status_string(status)) + ": " + msg;
    return status;
}

void *dev_alloc(clb_controls *ctl, size_t bytes) {
    if (bytes == 0) return nullptr;
    if (ctl->alloc) return ctl->alloc(ctl->alloc_ctx, bytes, (void *)ctl->stream);
    void *p = nullptr;
    if (cudaMallocAsync(&p, bytes, ctl->stream) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void dev_free(clb_controls *ctl, void *p) {
    if (!p) return;
    if (ctl->release) {
        ctl->release(ctl->alloc_ctx, p, (void *)ctl->stream);
        return;
    }
    cudaFreeAsync(p, ctl->stream);
}

namespace {
// Device words -> page-locked host staging, stored by the SMs over PCIe.
__global__ void stage_words_kernel(const uint32_t *__restrict__ src, uint32_t n, volatile uint32_t *dst) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    __threadfence_system();
}
}  // namespace

int read_small(clb_controls *ctl, const void *d_src, void *h_dst, size_t bytes) {
    if (bytes == 0) return CLB_SUCCESS;
    if (bytes > 64 * sizeof(uint64_t) || (bytes & 3)) return fail(CLB_INVALID_ARGUMENT, "read_small: bad size");
    stage_words_kernel<<<1, 32, 0, ctl->stream>>>(static_cast<const uint32_t *>(d_src), (uint32_t)(bytes / 4),
                                                   reinterpret_cast<volatile uint32_t *>(ctl->d_h_scalars));
    CLB_TRY_CUDA(cudaGetLastError(), CLB_RUN_KERNEL_FAILURE);
    ctl->launches += 1;
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    memcpy(h_dst, ctl->h_scalars, bytes);
    return CLB_SUCCESS;
}

int read_small_multi(clb_controls *ctl, const SmallRead *r, int n) {
    size_t at = 0;
    for (int k = 0; k < n; ++k) {
        if (r[k].bytes == 0) continue;
        if ((r[k].bytes & 3) || at + r[k].bytes > 64 * sizeof(uint64_t))
            return fail(CLB_INVALID_ARGUMENT, "read_small_multi: bad size");
        stage_words_kernel<<<1, 32, 0, ctl->stream>>>(
            static_cast<const uint32_t *>(r[k].src), (uint32_t)(r[k].bytes / 4),
            reinterpret_cast<volatile uint32_t *>(ctl->d_h_scalars) + at / 4);
        CLB_TRY_CUDA(cudaGetLastError(), CLB_RUN_KERNEL_FAILURE);
        ctl->launches += 1;
        at += r[k].bytes;
    }
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    at = 0;
    for (int k = 0; k < n; ++k) {
        memcpy(r[k].dst, reinterpret_cast<const char *>(ctl->h_scalars) + at, r[k].bytes);
        at += r[k].bytes;
    }
    return CLB_SUCCESS;
}

int read_scalars(clb_controls *ctl, const uint64_t *d_src, uint64_t *h_dst, int count) {
    return read_small(ctl, d_src, h_dst, sizeof(uint64_t) * (size_t)count);
}

int clear_status(clb_controls *ctl) {
    CLB_TRY_CUDA(cudaMemsetAsync(ctl->d_status, 0, sizeof(uint32_t), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    return CLB_SUCCESS;
}

int check_status(clb_controls *ctl, const char *op) {
    uint32_t s = 0;
    CLB_RETURN_IF(read_small(ctl, ctl->d_status, &s, sizeof(uint32_t)));
    if (s != 0) {
        char buf[160];
        snprintf(buf, sizeof(buf), "%s: device status word 0x%x", op, s);
        return fail(CLB_DEVICE_STATUS_ERROR, buf);
    }
    return CLB_SUCCESS;
}

static cudaEvent_t take_event(clb_controls *ctl) {
    if (!ctl->event_pool.empty()) {
        cudaEvent_t e = ctl->event_pool.back();
        ctl->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

ProfScope::ProfScope(clb_controls *c, const char *n) : ctl(c), name(n) {
    if (!ctl->profiling) return;
    start = take_event(ctl);
    if (start) cudaEventRecord(start, ctl->stream);
}

ProfScope::~ProfScope() {
    if (!start) return;
    cudaEvent_t stop = take_event(ctl);
    if (!stop) return;
    cudaEventRecord(stop, ctl->stream);
    ctl->prof.push_back({name, start, stop});
}

}  // namespace clb

using namespace clb;

extern "C" {

const char *clb_status_string(int s) {
    switch (s) {
        case CLB_SUCCESS: return "CLBOOL_SUCCESS";
        case CLB_NO_SUCH_PROGRAM: return "CLBOOL_NO_SUCH_PROGRAM";
        case CLB_CREATE_KERNEL_ERROR: return "CLBOOL_CREATE_KERNEL_ERROR";
        case CLB_BUILD_PROGRAM_ERROR: return "CLBOOL_BUILD_PROGRAM_ERROR";
        case CLB_INCOMPLETE_KERNEL: return "CLBOOL_INCOMPLETE_KERNEL";
        case CLB_RUN_KERNEL_FAILURE: return "CLBOOL_RUN_KERNEL_FAILURE";
        case CLB_EVENT_WAITING_ERROR: return "CLBOOL_EVENT_WAITING_ERROR";
        case CLB_CREATE_BUFFER_ERROR: return "CLBOOL_CREATE_BUFFER_ERROR";
        case CLB_COPY_BUFFER_ERROR: return "CLBOOL_COPY_BUFFER_ERROR";
        case CLB_READ_BUFFER_ERROR: return "CLBOOL_READ_BUFFER_ERROR";
        case CLB_WRITE_BUFFER_ERROR: return "CLBOOL_WRITE_BUFFER_ERROR";
        case CLB_CREATE_CONTROLS_ERROR: return "CLBOOL_CREATE_CONTROLS_ERROR";
        case CLB_INVALID_ARGUMENT: return "CLBOOL_INVALID_ARGUMENT";
        case CLB_INVALID_VALUE: return "CLBOOL_INVALID_VALUE";
        case CLB_INITIALIZATION_ERROR: return "CLBOOL_INITIALIZATION_ERROR";
        case CLB_DEVICE_STATUS_ERROR: return "CLBOOL_DEVICE_STATUS_ERROR";
        case CLB_NOT_SUPPORTED: return "CLBOOL_NOT_SUPPORTED";
        default: return "CLBOOL_UNKNOWN_STATUS";
    }
}

const char *clb_last_error(void) { return g_last_error.c_str(); }

int clb_version(void) { return 100; }

int clb_device_count(int *count) {
    if (!count) return fail(CLB_INVALID_ARGUMENT, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return CLB_SUCCESS;
}

int clb_device_info(int device, char *name, size_t name_len, int *sm_count, uint64_t *total_mem) {
    int n = 0;
    clb_device_count(&n);
    if (device < 0 || device >= n)
        return fail(CLB_CREATE_CONTROLS_ERROR, "no CUDA device with id " + std::to_string(device));
    cudaDeviceProp p;
    CLB_TRY_CUDA(cudaGetDeviceProperties(&p, device), CLB_CREATE_CONTROLS_ERROR);
    if (name && name_len) {
        strncpy(name, p.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (total_mem) *total_mem = p.totalGlobalMem;
    return CLB_SUCCESS;
}

int clb_controls_create(int device, clb_controls **out) {
    if (!out) return fail(CLB_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int n = 0;
    clb_device_count(&n);
    if (device < 0 || device >= n)
        return fail(CLB_CREATE_CONTROLS_ERROR, "no CUDA device with id " + std::to_string(device));
    int prev = -1;
    cudaGetDevice(&prev);
    CLB_TRY_CUDA(cudaSetDevice(device), CLB_CREATE_CONTROLS_ERROR);
    clb_controls *ctl = new clb_controls();
    ctl->device = device;
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e == cudaSuccess) {
        ctl->sm_count = p.multiProcessorCount;
        ctl->smem_optin = p.sharedMemPerBlockOptin;
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctl->stream, cudaStreamNonBlocking);
    ctl->own_stream = true;
    if (e == cudaSuccess) e = cudaMallocHost(&ctl->h_scalars, 64 * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&ctl->d_h_scalars, ctl->h_scalars, 0);
    if (e == cudaSuccess) e = cudaMalloc(&ctl->d_status, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(ctl->d_status, 0, sizeof(uint32_t));
    if (e == cudaSuccess) {
        // Keep freed pool memory cached: repeated calls reuse it instead of
        // returning it to the driver at every synchronisation.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        std::string msg = cudaGetErrorString(e);
        clb_controls_destroy(ctl);
        return fail(CLB_CREATE_CONTROLS_ERROR, msg);
    }
    *out = ctl;
    return CLB_SUCCESS;
}

int clb_controls_destroy(clb_controls *ctl) {
    if (!ctl) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    if (ctl->stream) cudaStreamSynchronize(ctl->stream);
    for (auto &r : ctl->prof) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    for (auto e : ctl->event_pool) cudaEventDestroy(e);
    if (ctl->own_stream && ctl->stream) cudaStreamDestroy(ctl->stream);
    if (ctl->h_scalars) cudaFreeHost(ctl->h_scalars);
    if (ctl->d_status) cudaFree(ctl->d_status);
    delete ctl;
    return CLB_SUCCESS;
}

int clb_controls_set_stream(clb_controls *ctl, void *stream) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    DeviceGuard g(ctl);
    if (ctl->own_stream && ctl->stream) {
        cudaStreamSynchronize(ctl->stream);
        cudaStreamDestroy(ctl->stream);
    }
    if (stream) {
        ctl->stream = (cudaStream_t)stream;
        ctl->own_stream = false;
    } else {
        CLB_TRY_CUDA(cudaStreamCreateWithFlags(&ctl->stream, cudaStreamNonBlocking), CLB_CREATE_CONTROLS_ERROR);
        ctl->own_stream = true;
    }
    return CLB_SUCCESS;
}

void *clb_controls_get_stream(clb_controls *ctl) { return ctl ? (void *)ctl->stream : nullptr; }

int clb_controls_device(clb_controls *ctl) { return ctl ? ctl->device : -1; }

int clb_controls_set_allocator(clb_controls *ctl, clb_alloc_fn alloc, clb_free_fn release, void *ctx) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    if ((alloc == nullptr) != (release == nullptr))
        return fail(CLB_INVALID_ARGUMENT, "allocator needs both alloc and release (or neither)");
    ctl->alloc = alloc;
    ctl->release = release;
    ctl->alloc_ctx = ctx;
    return CLB_SUCCESS;
}

int clb_controls_sync(clb_controls *ctl) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_controls_trim(clb_controls *ctl) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    cudaMemPool_t pool;
    CLB_TRY_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctl->device), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemPoolTrimTo(pool, 0), CLB_RUN_KERNEL_FAILURE);
    return CLB_SUCCESS;
}

int clb_graph_begin(clb_controls *ctl) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaStreamBeginCapture(ctl->stream, cudaStreamCaptureModeThreadLocal), CLB_RUN_KERNEL_FAILURE);
    return CLB_SUCCESS;
}

int clb_graph_end(clb_controls *ctl, void **graph) {
    if (!ctl || !graph) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    *graph = nullptr;
    cudaGraph_t gr = nullptr;
    CLB_TRY_CUDA(cudaStreamEndCapture(ctl->stream, &gr), CLB_RUN_KERNEL_FAILURE);
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(CLB_RUN_KERNEL_FAILURE, std::string("graph instantiation: ") + cudaGetErrorString(e));
    }
    *graph = ex;
    return CLB_SUCCESS;
}

int clb_graph_launch(clb_controls *ctl, void *graph) {
    if (!ctl || !graph) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph), ctl->stream), CLB_RUN_KERNEL_FAILURE);
    return CLB_SUCCESS;
}

int clb_graph_destroy(void *graph) {
    if (graph) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph));
    return CLB_SUCCESS;
}

int clb_profile_enable(clb_controls *ctl, int on) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    for (auto &r : ctl->prof) {
        ctl->event_pool.push_back(r.start);
        ctl->event_pool.push_back(r.stop);
    }
    ctl->prof.clear();
    ctl->profiling = on != 0;
    return CLB_SUCCESS;
}

int clb_profile_read(clb_controls *ctl, clb_profile_entry *out, int capacity, int *count) {
    if (!ctl || !count) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    int n = 0;
    for (auto &r : ctl->prof) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.start, r.stop);
        int k = 0;
        while (k < n && strncmp(out[k].name, r.name, sizeof(out[k].name)) != 0) ++k;
        if (k == n) {
            if (n >= capacity || !out) continue;
            memset(&out[n], 0, sizeof(out[n]));
            strncpy(out[n].name, r.name, sizeof(out[n].name) - 1);
            ++n;
        }
        out[k].launches += 1;
        out[k].ms += ms;
        ctl->event_pool.push_back(r.start);
        ctl->event_pool.push_back(r.stop);
    }
    ctl->prof.clear();
    *count = n;
    return CLB_SUCCESS;
}

int clb_malloc(clb_controls *ctl, size_t bytes, void **out) {
    if (!ctl || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    *out = nullptr;
    if (bytes == 0) return fail(CLB_CREATE_BUFFER_ERROR, "zero-size buffer");
    void *p = dev_alloc(ctl, bytes);
    if (!p) return fail(CLB_CREATE_BUFFER_ERROR, "device allocation of " + std::to_string(bytes) + " bytes failed");
    *out = p;
    return CLB_SUCCESS;
}

int clb_free(clb_controls *ctl, void *ptr) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    if (!ptr) return CLB_SUCCESS;
    DeviceGuard g(ctl);
    dev_free(ctl, ptr);
    return CLB_SUCCESS;
}

static int copy_sync(clb_controls *ctl, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, int err) {
    if (!ctl) return fail(CLB_INVALID_ARGUMENT, "controls is NULL");
    if (bytes == 0) return CLB_SUCCESS;
    if (!dst || !src) return fail(CLB_INVALID_ARGUMENT, "NULL pointer");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, ctl->stream), err);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_memcpy_h2d(clb_controls *ctl, void *dst, const void *src, size_t bytes) {
    return copy_sync(ctl, dst, src, bytes, cudaMemcpyHostToDevice, CLB_WRITE_BUFFER_ERROR);
}
int clb_memcpy_d2h(clb_controls *ctl, void *dst, const void *src, size_t bytes) {
    return copy_sync(ctl, dst, src, bytes, cudaMemcpyDeviceToHost, CLB_READ_BUFFER_ERROR);
}
int clb_memcpy_d2d(clb_controls *ctl, void *dst, const void *src, size_t bytes) {
    return copy_sync(ctl, dst, src, bytes, cudaMemcpyDeviceToDevice, CLB_COPY_BUFFER_ERROR);
}

int clb_host_alloc(size_t bytes, void **out) {
    if (!out) return fail(CLB_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (bytes == 0) return CLB_SUCCESS;
    CLB_TRY_CUDA(cudaMallocHost(out, bytes), CLB_CREATE_BUFFER_ERROR);
    return CLB_SUCCESS;
}

int clb_host_free(void *ptr) {
    if (ptr) CLB_TRY_CUDA(cudaFreeHost(ptr), CLB_RUN_KERNEL_FAILURE);
    return CLB_SUCCESS;
}

int clb_dcsr_release(clb_controls *ctl, clb_dcsr *m) {
    if (!ctl || !m) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    dev_free(ctl, m->rpt);
    dev_free(ctl, m->rows);
    dev_free(ctl, m->cols);
    m->rpt = nullptr;
    m->rows = nullptr;
    m->cols = nullptr;
    m->nnz = m->nzr = 0;
    return CLB_SUCCESS;
}

int clb_coo_release(clb_controls *ctl, clb_coo *m) {
    if (!ctl || !m) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    dev_free(ctl, m->rows);
    dev_free(ctl, m->cols);
    m->rows = m->cols = nullptr;
    m->nnz = 0;
    return CLB_SUCCESS;
}

int clb_csr_release(clb_controls *ctl, clb_csr *m) {
    if (!ctl || !m) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    dev_free(ctl, m->rpt);
    dev_free(ctl, m->cols);
    m->rpt = nullptr;
    m->cols = nullptr;
    m->nnz = 0;
    return CLB_SUCCESS;
}

}  // extern "C"
