// Allocation-free recount of a prepared query.
//
// Some callers cannot allocate device memory at the moment they want a
// count: latency-critical serving loops that must not take the implicit
// device-wide synchronisation a cudaMalloc/cudaFree can cause, and host
// processes whose device memory is owned by another runtime's pool (a
// database or JVM host that reserved the GPU's free memory up front), where
// a fresh allocation fails or steals from that pool.
// psm_run_recount_noalloc lets them re-run the enumeration kernel of a query
// that was prepared earlier (psm_run_create) without touching an allocator:
// the kernel's scratch (work-queue control block, queue slots and the
// per-query pool descriptor) lives in the file-scope device array below
// instead of the context arena.
//
// The array is PSM_NOALLOC_SCRATCH_BYTES (1 MiB) per device; every GPU that
// loads this library holds it until the process exits. The first call on a
// device looks up the array's device address (cudaGetSymbolAddress with that
// device current), so that first call should come before any stream capture
// begins. All calls share the array and it keeps the contents of the last
// call; the enumeration's init kernel rewrites every field it reads, so
// nothing stale is used, but two calls whose launches overlap on the GPU
// (different streams, or different threads on one device) race on the array
// and must not be issued.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "host.h"

#define PSM_NOALLOC_SCRATCH_BYTES (1u << 20)
#define PSM_NOALLOC_MAX_DEVICES 64

__device__ __align__(256) unsigned char g_enum_noalloc_scratch[PSM_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_mu;
void* g_scratch_addr[PSM_NOALLOC_MAX_DEVICES];  // device address per device, set once

// In host code `g_enum_noalloc_scratch` names a host-side shadow, not device
// memory: the device address of this device's copy has to be looked up with
// cudaGetSymbolAddress while the device is current.
cudaError_t scratch_for_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= PSM_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_enum_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// Resets the enumeration results of a prepared query before a recount.
__global__ void reset_counts_kernel(QState* q, u64 cap) {
    q->count = 0;
    q->calls = 0;
    q->alg_bytes = 0;
    q->stop = 0;
    q->overtime = 0;
    q->emit_rows = 0;
    q->cap = cap;
}

// Makes `dev` current for the lifetime of the guard and restores the
// caller's current device on every return path.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int psm_run_recount_noalloc(psm_run* run, uint64_t cap, double time_limit_s, uint64_t* count,
                                       uint32_t* overtime) {
    if (!run || !count) return psm_fail(PSM_ERR_ARG, "null argument");
    RunInternals ri{};
    int rc = psm_run_internals(run, &ri);
    if (rc) return rc;
    if (ri.emit) return psm_fail(PSM_ERR_ARG, "recount_noalloc: the run was prepared with emit=1");
    // A run whose preparation failed has no complete candidates or tables:
    // its enumeration would queue no work and report a count of 0.
    if (ri.prep_status == PSM_DEV_OOM)
        return psm_fail(PSM_ERR_OOM, "recount_noalloc: the run's preparation ran out of device memory");
    if (ri.prep_status == PSM_DEV_TIMEOUT)
        return psm_fail(PSM_ERR_TIMEOUT, "recount_noalloc: the run's preparation reached its time limit");
    if (ri.prep_status != PSM_DEV_OK)
        return psm_fail(PSM_ERR_INTERNAL, "recount_noalloc: the run's preparation failed");
    const size_t ctl_bytes = (psm_enum_scratch_bytes() + 255) & ~(size_t)255;
    const size_t need = ctl_bytes + psm_enum_query_bytes(1);
    if (need > PSM_NOALLOC_SCRATCH_BYTES)
        return psm_fail(PSM_ERR_ARG, "recount_noalloc: enumeration scratch exceeds the static 1 MiB maximum");
    DeviceGuard guard(ri.device);
    cudaError_t e = guard.err;
    void* scratch = nullptr;
    if (e == cudaSuccess) e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess) return psm_fail(PSM_ERR_CUDA, std::string("recount_noalloc: ") + cudaGetErrorString(e));
    const double s = time_limit_s > 0 ? time_limit_s : 60.0;
    reset_counts_kernel<<<1, 1, 0, ri.stream>>>(ri.dq, cap);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = psm_launch_enum(*ri.dev, ri.dq, 1, scratch, (char*)scratch + ctl_bytes, (u64)(s * 1e9), 0,
                            ri.enum_blocks, nullptr, nullptr, 0, ri.stream, 8u, ri.isect);
    u64 got = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&got, &ri.dq->count, sizeof(u64), cudaMemcpyDeviceToHost, ri.stream);
    u32 ov = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ov, &ri.dq->overtime, sizeof(u32), cudaMemcpyDeviceToHost, ri.stream);
    EnumStats es{};
    if (e == cudaSuccess) e = psm_enum_read_ctl(scratch, &es, ri.stream);  // synchronises the stream
    if (e != cudaSuccess) return psm_fail(PSM_ERR_CUDA, std::string("recount_noalloc: ") + cudaGetErrorString(e));
    if (es.error) return psm_fail(PSM_ERR_INTERNAL, "recount_noalloc: enumeration wait gave up");
    *count = cap && got > cap ? cap : got;
    if (overtime) *overtime = ov;
    return ov ? psm_fail(PSM_ERR_TIMEOUT, "time limit reached") : PSM_OK;
}
