// fv_kp07_dimsplit_substep_noalloc: one KP07_dimsplit substep that allocates
// no memory.
//
// Some callers cannot call cudaMalloc: applications that reserve the GPU's
// memory up front in their own pool and do not let plug-in solvers allocate,
// and time-stepping loops that must not pay allocation latency, or risk an
// out-of-memory failure, in the middle of a run.  They pass their own state
// buffers; the scratch this substep needs (the per-CTA CFL minima, the
// arrival counter and control block of the CTA epilogue) lives in the
// file-scope device array below, which every GPU that loads libfvgpu.so keeps
// until the process exits.
//
// Limits and behaviour:
//   * at most kMaxTiles tiles of 124 x 60 cells per call (a 4096 x 4096 grid
//     needs 2346); larger grids are rejected with FV_ERR_INVALID;
//   * every call shares the one array, so calls that overlap on the GPU (on
//     different streams, or from different host threads) race and give wrong
//     results; calls on one stream are ordered and safe;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and sets the kernel's shared-memory limit, with
//     that device current; make that first call before any stream capture;
//   * a tile load that gives up (the kernel's bounded wait) leaves a sticky
//     error flag in the array; the next call on the device reads it first
//     (waiting for its stream), clears it and returns FV_ERR_DEVICE without
//     launching, since the previous output is incomplete.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fvgpu.h"
#include "fv_stage.cuh"

namespace {

constexpr int kW = 124, kH = 60, kNT = 256;
constexpr int kMaxTiles = 8192;
constexpr size_t kCtlBytes = (sizeof(fv::SimCtl) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kCtlBytes + kMaxTiles * sizeof(float);  // about 33 KB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

}  // namespace

// Sets the message returned by fv_last_error() (defined in fv_api.cu).
void fv_internal_set_error(const char* msg);

namespace {

int noalloc_fail(int code, const char* msg) {
    fv_internal_set_error(msg);
    return code;
}

struct DeviceState {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
};
constexpr int kMaxDevices = 64;
DeviceState g_devices[kMaxDevices];
std::mutex g_devices_mu;

using KernelFn = void (*)(fv::StageArgs);
const KernelFn kKernel = fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, kW, kH, kNT>;
constexpr size_t kSmem = 3 * (size_t)(kW + 8) * (kH + 4) * sizeof(float);

PFN_cuTensorMapEncodeTiled_v12000 noalloc_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// One-time set-up per device, with that device current.
int device_setup(unsigned char** scratch) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(FV_ERR_CUDA, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_devices_mu);
    DeviceState& d = g_devices[dev];
    if (!d.ready) {
        void* addr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (e != cudaSuccess || addr == nullptr)
            return noalloc_fail(FV_ERR_CUDA, "cudaGetSymbolAddress of the static scratch array failed");
        e = cudaFuncSetAttribute(reinterpret_cast<const void*>(kKernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmem);
        if (e != cudaSuccess) return noalloc_fail(FV_ERR_CUDA, "cudaFuncSetAttribute failed");
        if (!noalloc_encode_fn()) return noalloc_fail(FV_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
        d.scratch = static_cast<unsigned char*>(addr);
        d.ready = true;
    }
    *scratch = d.scratch;
    return FV_OK;
}

// Poll limit of the kernel's tile-load wait (StageArgs::wait_limit): 0, the
// default, is the library's limit.  FVGPU_NOALLOC_WAIT_POLLS, read once per
// process, overrides it; tests set it negative so that every tile load gives
// up at once and the error report can be checked without a GPU fault.
int noalloc_wait_limit() {
    static const int limit = [] {
        const char* e = getenv("FVGPU_NOALLOC_WAIT_POLLS");
        return e ? atoi(e) : 0;
    }();
    return limit;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Whether two planes of `n` floats share any element.
bool overlaps(const float* a, const float* b, size_t n) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    const uintptr_t bytes = n * sizeof(float);
    return x < y + bytes && y < x + bytes;
}

// Wall codes the kernel implements: Dirichlet, periodic, reflective.
int check_bc(int bc) {
    if (bc & (int)0xF0F0F0F0u) return noalloc_fail(FV_ERR_INVALID, "unknown bits in the boundary-condition code");
    for (int side = 0; side < 4; ++side) {
        const int t = (bc >> (8 * side)) & 0xF;
        if (t == fv::BC_NEUMANN) return noalloc_fail(FV_ERR_UNSUPPORTED, "Neumann boundary condition not supported");
        if (t != fv::BC_DIRICHLET && t != fv::BC_PERIODIC && t != fv::BC_REFLECTIVE)
            return noalloc_fail(FV_ERR_INVALID, "boundary-condition code of a side is not 0, 1, 2 or 3");
    }
    return FV_OK;
}

}  // namespace

extern "C" {

int fv_kp07_dimsplit_substep_noalloc(const float* const* in, float* const* out, int pitch, int nx, int ny, float dx,
                                     float dy, float dt, float g, float theta, int step, int bc, float* cfl_min,
                                     void* stream) {
    if (!in || !out) return noalloc_fail(FV_ERR_INVALID, "in/out must hold 3 device pointers");
    for (int v = 0; v < 3; ++v)
        if (!in[v] || !out[v] || !aligned16(in[v]) || !aligned16(out[v]))
            return noalloc_fail(FV_ERR_INVALID, "state pointers must be non-null and 16-byte aligned");
    if (nx < 1 || ny < 1) return noalloc_fail(FV_ERR_INVALID, "grid must be at least 1 x 1");
    if (pitch % 4 != 0 || pitch < nx + 8)
        return noalloc_fail(FV_ERR_INVALID, "pitch must be a multiple of 4 floats and at least nx + 8");
    int rc = check_bc(bc);
    if (rc != FV_OK) return rc;
    const dim3 grid((nx + kW - 1) / kW, (ny + kH - 1) / kH);
    if ((long long)grid.x * grid.y > kMaxTiles) {
        char msg[160];
        snprintf(msg, sizeof(msg), "grid of %d x %d needs %lld tiles; the static scratch holds %d (124 x 60 cells each)",
                 nx, ny, (long long)grid.x * grid.y, kMaxTiles);
        return noalloc_fail(FV_ERR_INVALID, msg);
    }
    // The kernel reads halo cells of `in` that neighbouring CTAs may already
    // have written in `out`: the output planes must share no element with any
    // input plane or with each other.
    const size_t plane = (size_t)(ny + 4) * (size_t)pitch;
    for (int v = 0; v < 3; ++v)
        for (int w = 0; w < 3; ++w)
            if (overlaps(in[v], out[w], plane) || (w != v && overlaps(out[v], out[w], plane)))
                return noalloc_fail(FV_ERR_INVALID, "output planes must not overlap the input planes or each other");
    unsigned char* scratch = nullptr;
    rc = device_setup(&scratch);
    if (rc != FV_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    fv::SimCtl* ctl = reinterpret_cast<fv::SimCtl*>(scratch);
    float* block_cfl = reinterpret_cast<float*>(scratch + kCtlBytes);

    // The error flag of the previous call: a tile load of it that gave up
    // left part of its output unwritten.  Reading it waits for this stream.
    int prev_error = 0;
    if (cudaMemcpyAsync(&prev_error, &ctl->error, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return noalloc_fail(FV_ERR_CUDA, "reading the static control block's error flag failed");
    if (prev_error) {
        if (cudaMemsetAsync(&ctl->error, 0, sizeof(int), s) != cudaSuccess)
            return noalloc_fail(FV_ERR_CUDA, "clearing the static control block's error flag failed");
        return noalloc_fail(FV_ERR_DEVICE,
                            "a tile load of the previous allocation-free substep on this device gave up: its output "
                            "is incomplete (the flag is now cleared)");
    }

    alignas(64) fv::StageArgs a;
    memset(&a, 0, sizeof(a));
    auto enc = noalloc_encode_fn();
    for (int v = 0; v < 3; ++v) {
        cuuint64_t dims[2] = {(cuuint64_t)(nx + 8), (cuuint64_t)(ny + 4)};
        cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
        cuuint32_t box[2] = {(cuuint32_t)(kW + 8), (cuuint32_t)(kH + 4)};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = enc(&a.tmap[0][v], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(in[v]), dims, strides,
                         box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return noalloc_fail(FV_ERR_INVALID, "cuTensorMapEncodeTiled rejected the state layout");
        a.buf[0][v] = const_cast<float*>(in[v]);
        a.buf[1][v] = out[v];
    }
    a.ctl = ctl;
    a.block_cfl = block_cfl;
    a.block_sums = nullptr;  // want_sums == 0: never written
    a.nx = nx;
    a.ny = ny;
    a.pitch = pitch;
    a.dx = dx;
    a.dy = dy;
    a.g = g;
    a.theta = theta;
    a.dt_scale = 1.0f;
    a.bc = bc;
    a.substep = step;
    a.order = 2;
    a.is_last = 0;
    a.force_cfl = cfl_min ? 1 : 0;
    a.explicit_dt = 1;
    a.dt_step = dt;
    a.want_sums = 0;
    a.wait_limit = noalloc_wait_limit();

    // The control block must start at zero up to the error flag: buffer
    // parity 0 (read `in`, write `out`), arrival counter 0.  The error flag
    // (zero here) stays as this call's kernel leaves it, for the next call.
    static_assert(offsetof(fv::SimCtl, error) > offsetof(fv::SimCtl, arrive) &&
                      offsetof(fv::SimCtl, error) > offsetof(fv::SimCtl, cur),
                  "the cleared prefix of the control block covers the buffer parity and the arrival counter");
    if (cudaMemsetAsync(ctl, 0, offsetof(fv::SimCtl, error), s) != cudaSuccess)
        return noalloc_fail(FV_ERR_CUDA, "clearing the static control block failed");
    void* kargs[] = {&a};
    cudaError_t e = cudaLaunchKernel(reinterpret_cast<const void*>(kKernel), grid, dim3(kNT), kargs, kSmem, s);
    if (e != cudaSuccess) return noalloc_fail(FV_ERR_CUDA, cudaGetErrorString(e));
    if (cfl_min && cudaMemcpyAsync(cfl_min, &ctl->cfl_min, sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return noalloc_fail(FV_ERR_CUDA, "copying the CFL minimum failed");
    return FV_OK;
}

}  // extern "C"
