/*
 * Fused measurement that allocates no device memory.
 *
 * Some callers cannot call cudaMalloc: a host that owns all device memory
 * through its own caching pool (as PyTorch's allocator does) and forbids
 * driver allocations outside it; a service running under a fixed device
 * memory budget that must not grow; and latency-critical loops that must not
 * risk the device-wide synchronisation that cudaMalloc and cudaFree can
 * cause.  slsf_measure_noalloc serves them: the caller passes the lattice
 * (device pointers) and receives the observables, and the only scratch the
 * reduction needs -- per-block FP64 partial sums, the final sums and the
 * last-block counter -- lives in the file-scope array below, about 75 KiB,
 * which every GPU that loads this library keeps until the process exits.
 *
 * The array is shared by every call: a call overwrites what the previous one
 * left, and calls whose kernels overlap on the GPU (different streams, or
 * different host threads, on the same device) race on it.  Serialise them.
 *
 * Every call takes the array's device address with cudaGetSymbolAddress on
 * the current device (the host-side name of a __device__ array is only a
 * stand-in, not a device address; the lookup allocates nothing).  The first
 * call on a device -- and the first after the device's context was rebuilt,
 * which moves the array -- also zeroes the last-block counter and waits for
 * that: make such a first call before any stream capture.
 */
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/slsf_gpu.h"
#include "engine.h"

namespace {

/* Partial-sum rows: one per block of the measurement grid, whose size the
 * measurement launcher bounds by the same constant. */
constexpr int kNoAllocMaxBlocks = slsf::kMeasureMaxBlocks;
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
    double partials[kNoAllocMaxBlocks * 8];
    double result[8];
    unsigned int done;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_setup_mutex;
/* The array's address on each device when its counter was last zeroed. */
NoAllocScratch* g_scratch_ptr[kNoAllocMaxDevices] = {};

}  // namespace

/* The array's device address on the current device; its counter is zeroed
 * whenever that address is new (first use, or a rebuilt context). */
static int noalloc_scratch(int device, cudaStream_t stream, NoAllocScratch** out, std::string* err) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
        *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return SLSF_ERR_CUDA;
    }
    NoAllocScratch* s = static_cast<NoAllocScratch*>(p);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[device] != s) {
        e = cudaMemsetAsync(&s->done, 0, sizeof(unsigned int), stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            *err = std::string("scratch set-up: ") + cudaGetErrorString(e);
            return SLSF_ERR_CUDA;
        }
        g_scratch_ptr[device] = s;
    }
    *out = s;
    return SLSF_OK;
}

extern "C" int slsf_measure_noalloc(const float* theta, const float* j_xy, const float* j_z, uint32_t lx,
                                    uint32_t ly, uint32_t lz, void* stream, slsf_observables* out) {
    /* Errors are reported through slsf_last_error like every other call. */
    auto fail = [](int code, const std::string& msg) { return slsf::report_error(code, msg); };
    if (!theta || !j_xy || !j_z || !out) return fail(SLSF_ERR_INVALID, "NULL argument");
    if (lx == 0) return fail(SLSF_ERR_INVALID, "L_x must be positive");
    if (ly == 0) return fail(SLSF_ERR_INVALID, "L_y must be positive");
    if (lz == 0) return fail(SLSF_ERR_INVALID, "L_z must be positive");
    const uint64_t volume = (uint64_t)lx * ly * lz;
    if (volume > SLSF_NOALLOC_MAX_SITES)
        return fail(SLSF_ERR_INVALID, "lattice volume exceeds the no-allocation measurement limit of 2^31 - 1 sites");
    /* measure_partial_blocks never exceeds kMeasureMaxBlocks, the rows of the array */
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(SLSF_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(SLSF_ERR_INVALID, "device index out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    NoAllocScratch* scratch = nullptr;
    std::string err;
    if (int rc = noalloc_scratch(device, s, &scratch, &err)) return fail(rc, err);

    slsf::TaskView v = {};
    v.theta = const_cast<float*>(theta);
    v.jxy = j_xy;
    v.jz = j_z;
    v.lx = lx;
    v.ly = ly;
    v.lz = lz;
    slsf::launch_measure(v, scratch->partials, &scratch->done, scratch->result, s);
    e = cudaGetLastError();
    double r[8];
    if (e == cudaSuccess) e = cudaMemcpyAsync(r, scratch->result, sizeof(r), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(SLSF_ERR_CUDA, std::string("measurement: ") + cudaGetErrorString(e));
    const double vol = (double)volume;
    out->energy = -(r[2] + r[3] + r[4]) / vol;
    out->magnetization_squared = (r[0] * r[0] + r[1] * r[1]) / (vol * vol);
    out->cos_x = r[2];
    out->cos_y = r[3];
    out->cos_z = r[4];
    out->sin_x = r[5];
    out->sin_y = r[6];
    out->sin_z = r[7];
    return SLSF_OK;
}
