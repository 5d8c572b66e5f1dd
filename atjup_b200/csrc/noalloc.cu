// Column balance of v with no device allocation (atjup_gpu_balance_column_v_noalloc).
//
// Some callers cannot call cudaMalloc at all: a host model that hands the GPU layer one
// preallocated memory pool and forbids allocations after start-up, or an embedding that must
// never fail mid-run on an out-of-memory allocation. This entry point takes the caller's device
// buffers for inputs and output and keeps its own scratch -- the per-column means of r v and the
// per-row means -- in a fixed-size file-scope device array, so it allocates nothing.
//
// Limits: jm <= ATJUP_NOALLOC_MAX_J and pitch <= ATJUP_NOALLOC_MAX_PITCH (larger sizes are
// rejected with ATJUP_ERR_ARG). The array (~1.05 MB) is resident on every GPU that loads this
// library, until the process exits. All calls share it and it keeps the last call's contents;
// every value a call reads is written earlier in that same call, so nothing needs clearing.
// Calls that overlap on the GPU (different streams, or different host threads without ordering)
// race on the array: order them on one stream.
//
// Set-up: the first call on each device, with that device current, looks up the array's device
// address with cudaGetSymbolAddress and keeps it for the rest of the process; that first call
// should come before any stream capture. A cudaDeviceReset ends the module the address belongs
// to, so the kept address is stale afterwards: a process that resets a device must not call this
// entry point on it again.
#include "ctx.cuh"

#include <atomic>
#include <cstdio>

namespace {

constexpr int MAX_J = ATJUP_NOALLOC_MAX_J;
constexpr int MAX_PITCH = ATJUP_NOALLOC_MAX_PITCH;

// scratch: column means [MAX_J * MAX_PITCH] then row means [MAX_J]
static __device__ __align__(256) double g_vbal_scratch[(size_t)MAX_J * MAX_PITCH + MAX_J];

// The array's device address, looked up once per device (the host-side name is only a
// stand-in for the symbol and must never be handed to a kernel).
constexpr int MAX_DEVICES = 64;
std::atomic<double*> g_scratch_addr[MAX_DEVICES];

int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return atjup::cuda_status(e, "balance_column_v_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= MAX_DEVICES) {
        atjup::set_error("balance_column_v_noalloc: device ordinal above 63");
        return ATJUP_ERR_ARG;
    }
    double* p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        void* a = nullptr;
        e = cudaGetSymbolAddress(&a, g_vbal_scratch);
        if (e != cudaSuccess) return atjup::cuda_status(e, "balance_column_v_noalloc: cudaGetSymbolAddress");
        p = static_cast<double*>(a);
        g_scratch_addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return ATJUP_OK;
}

}  // namespace

extern "C" int atjup_gpu_balance_column_v_noalloc(double* v, const int32_t* i_topo,
                                                  const double* rad, int32_t im, int32_t jm,
                                                  int32_t km, int32_t pitch, double dr,
                                                  int32_t zonal, void* stream) {
    if (!v || !i_topo || !rad) {
        atjup::set_error("balance_column_v_noalloc: null pointer");
        return ATJUP_ERR_ARG;
    }
    if (im < 2 || jm < 3 || km < 2 || pitch < km) {
        atjup::set_error("balance_column_v_noalloc: need im >= 2, jm >= 3, km >= 2, pitch >= km");
        return ATJUP_ERR_ARG;
    }
    if (jm > MAX_J || pitch > MAX_PITCH) {
        char msg[200];
        snprintf(msg, sizeof(msg),
                 "balance_column_v_noalloc: jm = %d, pitch = %d above the fixed scratch limits "
                 "jm <= %d, pitch <= %d", jm, pitch, MAX_J, MAX_PITCH);
        atjup::set_error(msg);
        return ATJUP_ERR_ARG;
    }
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != ATJUP_OK) return rc;
    double* dvc = scratch;
    double* dvrow = scratch + (size_t)MAX_J * MAX_PITCH;
    return atjup::launch_balance_v_buffers(v, i_topo, rad, dvc, dvrow, im, jm, km, pitch, dr,
                                           zonal, static_cast<cudaStream_t>(stream));
}
