// Host runtime and C ABI of libfvgpu.so (declared in include/fvgpu.h).
//
// A simulation owns two state buffers per conserved variable (u0/u1 of the
// reference, GPUSimulators/Common.py:741-755), a device control block with t,
// nt, dt and the buffer parity, one TMA descriptor per buffer and variable,
// and CUDA graphs of 1 and 16 steps.  simulate() reproduces the reference's
// host loop (GPUSimulators/Simulator.py:176-217) with one synchronisation per
// 100-step dt interval, where the reference reads back min(cfl_data).

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/fvgpu.h"
#include "fv_stage.cuh"

using fv::SimCtl;
using fv::StageArgs;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define FV_CK(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return fail(FV_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define FV_TRY(call)              \
    do {                          \
        int r_ = (call);          \
        if (r_ != FV_OK) return r_; \
    } while (0)

int scheme_nv(int scheme) { return scheme == FV_EE2D_KP07_DIMSPLIT ? 4 : 3; }
int scheme_ghost(int scheme) { return (scheme == FV_LXF || scheme == FV_FORCE || scheme == FV_HLL) ? 1 : 2; }

using KernelFn = void (*)(StageArgs);

struct KEntry {
    int scheme;
    int W, H, NT;
    bool split;
    KernelFn fn;
};

// Tile configurations per scheme; the first entry of a scheme is its default.
const KEntry kTable[] = {
    {FV_KP07_DIMSPLIT, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 124, 60, 256>},
    {FV_KP07_DIMSPLIT, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 124, 28, 128>},
    {FV_KP07_DIMSPLIT, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 60, 28, 128>},
    {FV_KP07_DIMSPLIT, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 28, 28, 128>},
    {FV_HLL2, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::HLL2, 124, 60, 256>},
    {FV_HLL2, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 124, 28, 128>},
    {FV_HLL2, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 28, 28, 128>},
    {FV_HLL2, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 60, 28, 128>},
    {FV_WAF, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::WAF, 124, 60, 256>},
    {FV_WAF, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 124, 28, 128>},
    {FV_WAF, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 28, 28, 128>},
    {FV_WAF, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 60, 28, 128>},
    {FV_FORCE, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::FORCE, 124, 60, 256>},
    {FV_FORCE, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::FORCE, 124, 28, 128>},
    {FV_FORCE, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::FORCE, 28, 28, 128>},
    {FV_FORCE, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::FORCE, 60, 28, 128>},
    {FV_HLL, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::HLL, 124, 60, 256>},
    {FV_HLL, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL, 124, 28, 128>},
    {FV_HLL, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL, 60, 28, 128>},
    {FV_HLL, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL, 28, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 124, 28, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 124, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 124, 60, 256, true, fv::dimsplit_stage_kernel<fv::EE2D, 124, 60, 256>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 28, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 60, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 28, 28, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 28, 28, 128>},
    {FV_LXF, 120, 60, 256, false, fv::unsplit_stage_kernel<fv::LXF, 120, 60, 256>},
    {FV_LXF, 120, 28, 128, false, fv::unsplit_stage_kernel<fv::LXF, 120, 28, 128>},
    {FV_LXF, 120, 60, 128, false, fv::unsplit_stage_kernel<fv::LXF, 120, 60, 128>},
    {FV_LXF, 60, 28, 128, false, fv::unsplit_stage_kernel<fv::LXF, 60, 28, 128>},
    {FV_KP07, 120, 28, 128, false, fv::unsplit_stage_kernel<fv::KP07, 120, 28, 128>},
    {FV_KP07, 120, 60, 128, false, fv::unsplit_stage_kernel<fv::KP07, 120, 60, 128>},
    {FV_KP07, 120, 60, 256, false, fv::unsplit_stage_kernel<fv::KP07, 120, 60, 256>},
    {FV_KP07, 60, 28, 128, false, fv::unsplit_stage_kernel<fv::KP07, 60, 28, 128>},
    // two lines per thread in packed FP32 (same cells, bit for bit)
    {FV_KP07_DIMSPLIT, 124, 28, 64, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 124, 28, 64, 0, 2>},
    {FV_KP07_DIMSPLIT, 124, 60, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 124, 60, 128, 0, 2>},
    {FV_KP07_DIMSPLIT, 60, 28, 64, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 60, 28, 64, 0, 2>},
    {FV_HLL2, 124, 28, 64, true, fv::dimsplit_stage_kernel<fv::HLL2, 124, 28, 64, 0, 2>},
    {FV_HLL2, 124, 60, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 124, 60, 128, 0, 2>},
    {FV_HLL2, 60, 28, 64, true, fv::dimsplit_stage_kernel<fv::HLL2, 60, 28, 64, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 124, 28, 64, true, fv::dimsplit_stage_kernel<fv::EE2D, 124, 28, 64, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 124, 60, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 124, 60, 128, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 28, 64, true, fv::dimsplit_stage_kernel<fv::EE2D, 60, 28, 64, 0, 2>},
    {FV_WAF, 124, 28, 64, true, fv::dimsplit_stage_kernel<fv::WAF, 124, 28, 64, 0, 2>},
    {FV_WAF, 124, 60, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 124, 60, 128, 0, 2>},
    {FV_WAF, 60, 28, 64, true, fv::dimsplit_stage_kernel<fv::WAF, 60, 28, 64, 0, 2>},
    // 8-segment rows (120 wide, padded pitch 136): twice the warps of the 124-wide packed tiles
    {FV_KP07_DIMSPLIT, 120, 28, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 120, 28, 128, 0, 2>},
    {FV_KP07_DIMSPLIT, 120, 60, 256, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 120, 60, 256, 0, 2>},
    {FV_HLL2, 120, 28, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 120, 28, 128, 0, 2>},
    {FV_HLL2, 120, 60, 256, true, fv::dimsplit_stage_kernel<fv::HLL2, 120, 60, 256, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 120, 28, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 120, 28, 128, 0, 2>},
    {FV_WAF, 120, 28, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 120, 28, 128, 0, 2>},
    {FV_WAF, 120, 60, 256, true, fv::dimsplit_stage_kernel<fv::WAF, 120, 60, 256, 0, 2>},
    // 60 x 60: fewer halo rows per tile than 60 x 28 at the same warps per SM
    {FV_KP07_DIMSPLIT, 60, 60, 128, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 60, 60, 128, 0, 2>},
    {FV_KP07_DIMSPLIT, 60, 60, 256, true, fv::dimsplit_stage_kernel<fv::KP07_DIMSPLIT, 60, 60, 256, 0, 1>},
    {FV_HLL2, 60, 60, 128, true, fv::dimsplit_stage_kernel<fv::HLL2, 60, 60, 128, 0, 2>},
    {FV_HLL2, 60, 60, 256, true, fv::dimsplit_stage_kernel<fv::HLL2, 60, 60, 256, 0, 1>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 60, 128, true, fv::dimsplit_stage_kernel<fv::EE2D, 60, 60, 128, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 60, 256, true, fv::dimsplit_stage_kernel<fv::EE2D, 60, 60, 256, 0, 1>},
    {FV_WAF, 60, 60, 128, true, fv::dimsplit_stage_kernel<fv::WAF, 60, 60, 128, 0, 2>},
    {FV_WAF, 60, 60, 256, true, fv::dimsplit_stage_kernel<fv::WAF, 60, 60, 256, 0, 1>},
};
constexpr int kNumEntries = sizeof(kTable) / sizeof(kTable[0]);

// Kernels of HLL's HLLC and Godunov-centred fluxes and of WAF's other limiters
// (variant 0 is the reference's own and uses kTable), one tile configuration
// each: the variant is a template parameter, so the default kernels carry no
// switch in their cell loops.
struct VEntry {
    int variant;
    KEntry k;
};
const VEntry kVariantTable[] = {
#define FV_V(S, ES, V) {V, {S, 124, 60, 256, true, fv::dimsplit_stage_kernel<ES, 124, 60, 256, V>}}
    FV_V(FV_HLL, fv::HLL, 1), FV_V(FV_HLL, fv::HLL, 2),
    FV_V(FV_WAF, fv::WAF, 1), FV_V(FV_WAF, fv::WAF, 2), FV_V(FV_WAF, fv::WAF, 3), FV_V(FV_WAF, fv::WAF, 4),
    FV_V(FV_WAF, fv::WAF, 5), FV_V(FV_WAF, fv::WAF, 6), FV_V(FV_WAF, fv::WAF, 7), FV_V(FV_WAF, fv::WAF, 8),
#undef FV_V
};
constexpr int kNumVariants = sizeof(kVariantTable) / sizeof(kVariantTable[0]);

using BatchFn = void (*)(fv::BatchArgs);
struct BEntry {
    int scheme;
    int W, H, NT;
    BatchFn fn;
    bool persistent = false;  // resident CTAs striding over the work list (else one CTA per entry)
};
// Batched kernels; the first entry of a scheme is its default.
const BEntry kBatchTable[] = {
    {FV_LXF, 60, 28, 128, fv::batched_stage_kernel<fv::LXF, 60, 28, 128>},
    {FV_LXF, 120, 28, 128, fv::batched_stage_kernel<fv::LXF, 120, 28, 128>},
    {FV_KP07, 60, 28, 128, fv::batched_stage_kernel<fv::KP07, 60, 28, 128>},
    {FV_KP07, 120, 28, 128, fv::batched_stage_kernel<fv::KP07, 120, 28, 128>},
    {FV_KP07_DIMSPLIT, 60, 28, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 60, 28, 128>},
    {FV_KP07_DIMSPLIT, 124, 28, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 124, 28, 128>},
    {FV_KP07_DIMSPLIT, 124, 60, 256, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 124, 60, 256>},
    {FV_KP07_DIMSPLIT, 28, 28, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 28, 28, 128>},
    {FV_HLL, 60, 28, 128, fv::batched_stage_kernel<fv::HLL, 60, 28, 128>},
    {FV_HLL, 124, 28, 128, fv::batched_stage_kernel<fv::HLL, 124, 28, 128>},
    {FV_HLL, 124, 60, 256, fv::batched_stage_kernel<fv::HLL, 124, 60, 256>},
    {FV_HLL, 28, 28, 128, fv::batched_stage_kernel<fv::HLL, 28, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 28, 128, fv::batched_stage_kernel<fv::EE2D, 60, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 124, 28, 128, fv::batched_stage_kernel<fv::EE2D, 124, 28, 128>},
    {FV_EE2D_KP07_DIMSPLIT, 28, 28, 128, fv::batched_stage_kernel<fv::EE2D, 28, 28, 128>},
    {FV_HLL2, 60, 28, 128, fv::batched_stage_kernel<fv::HLL2, 60, 28, 128>},
    {FV_HLL2, 124, 28, 128, fv::batched_stage_kernel<fv::HLL2, 124, 28, 128>},
    {FV_HLL2, 28, 28, 128, fv::batched_stage_kernel<fv::HLL2, 28, 28, 128>},
    {FV_WAF, 60, 28, 128, fv::batched_stage_kernel<fv::WAF, 60, 28, 128>},
    {FV_WAF, 124, 28, 128, fv::batched_stage_kernel<fv::WAF, 124, 28, 128>},
    {FV_WAF, 28, 28, 128, fv::batched_stage_kernel<fv::WAF, 28, 28, 128>},
    {FV_FORCE, 60, 28, 128, fv::batched_stage_kernel<fv::FORCE, 60, 28, 128>},
    {FV_FORCE, 124, 28, 128, fv::batched_stage_kernel<fv::FORCE, 124, 28, 128>},
    {FV_FORCE, 28, 28, 128, fv::batched_stage_kernel<fv::FORCE, 28, 28, 128>},
    // 60 x 60, two lines per thread in packed FP32 (same cells, bit for bit)
    {FV_KP07_DIMSPLIT, 60, 60, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 60, 60, 128, 0, 2>},
    {FV_HLL2, 60, 60, 128, fv::batched_stage_kernel<fv::HLL2, 60, 60, 128, 0, 2>},
    {FV_WAF, 60, 60, 128, fv::batched_stage_kernel<fv::WAF, 60, 60, 128, 0, 2>},
    {FV_EE2D_KP07_DIMSPLIT, 60, 60, 128, fv::batched_stage_kernel<fv::EE2D, 60, 60, 128, 0, 2>},
    // persistent forms of the KP07_dimsplit tiles (timed against the one-tile-per-CTA forms)
    {FV_KP07_DIMSPLIT, 60, 60, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 60, 60, 128, 0, 2, true>, true},
    {FV_KP07_DIMSPLIT, 124, 28, 128, fv::batched_stage_kernel<fv::KP07_DIMSPLIT, 124, 28, 128, 0, 1, true>, true},
};
constexpr int kNumBatchEntries = sizeof(kBatchTable) / sizeof(kBatchTable[0]);

// Batched kernels of the variants other than 0, one tile configuration each.
struct VBEntry {
    int variant;
    BEntry b;
};
const VBEntry kBatchVariantTable[] = {
#define FV_V(S, ES, V) {V, {S, 60, 28, 128, fv::batched_stage_kernel<ES, 60, 28, 128, V>}}
    FV_V(FV_HLL, fv::HLL, 1), FV_V(FV_HLL, fv::HLL, 2),
    FV_V(FV_WAF, fv::WAF, 1), FV_V(FV_WAF, fv::WAF, 2), FV_V(FV_WAF, fv::WAF, 3), FV_V(FV_WAF, fv::WAF, 4),
    FV_V(FV_WAF, fv::WAF, 5), FV_V(FV_WAF, fv::WAF, 6), FV_V(FV_WAF, fv::WAF, 7), FV_V(FV_WAF, fv::WAF, 8),
#undef FV_V
};
constexpr int kNumBatchVariants = sizeof(kBatchVariantTable) / sizeof(kBatchVariantTable[0]);

bool scheme_split(int scheme) { return scheme != FV_LXF && scheme != FV_KP07; }

// Width of a batched kernel's TMA box, the row pitch of its shared tile.
int batch_box_w(const BEntry& e) { return scheme_split(e.scheme) ? fv::split_pitch(e.W) : e.W + 8; }

size_t batch_smem(const BEntry& e) {
    return scheme_nv(e.scheme) * (size_t)batch_box_w(e) * (e.H + 4) * sizeof(float);
}

// The batched kernel of tile configuration `cfg`, or for variant > 0 the
// variant's single kernel (cfg is then ignored).
const BEntry* find_batch_entry(int scheme, int cfg, int variant) {
    if (variant > 0) {
        for (int i = 0; i < kNumBatchVariants; ++i)
            if (kBatchVariantTable[i].b.scheme == scheme && kBatchVariantTable[i].variant == variant)
                return &kBatchVariantTable[i].b;
        return nullptr;
    }
    int k = 0;
    for (int i = 0; i < kNumBatchEntries; ++i) {
        if (kBatchTable[i].scheme != scheme) continue;
        if (k == cfg) return &kBatchTable[i];
        ++k;
    }
    return nullptr;
}


int entry_box_w(const KEntry& e) { return e.split ? fv::split_pitch(e.W) : e.W + 8; }

size_t entry_smem(const KEntry& e) {
    // row pitch of the shared tile = width of the TMA box (entry_box_w)
    const size_t tile = (size_t)entry_box_w(e) * (e.H + 4) * sizeof(float);
    return scheme_nv(e.scheme) * tile;
}

// The stage kernel of tile configuration `cfg`, or for variant > 0 the
// variant's single kernel (cfg is then ignored).
const KEntry* find_entry(int scheme, int cfg, int variant) {
    if (variant > 0) {
        for (int i = 0; i < kNumVariants; ++i)
            if (kVariantTable[i].k.scheme == scheme && kVariantTable[i].variant == variant)
                return &kVariantTable[i].k;
        return nullptr;
    }
    int k = 0;
    for (int i = 0; i < kNumEntries; ++i) {
        if (kTable[i].scheme != scheme) continue;
        if (k == cfg) return &kTable[i];
        ++k;
    }
    return nullptr;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// Host replica of the reference's initial CFL estimate, in float32 with numpy's
// NaN-propagating np.min (e.g. GPUSimulators/KP07_dimsplit.py:103-105).

// Initial CFL estimate of an uploaded state, computed on the device after the
// upload: the reference's host formula min(dx / (|hu/h| + sqrt(g h)),
// dy / (|hv/h| + sqrt(g h))) over every uploaded value (e.g.
// GPUSimulators/KP07_dimsplit.py:102-106; EE2D uses gamma and rho,
// EE2D_KP07_dimsplit.py:106-108), in IEEE FP32 with denormals kept (explicit
// round-to-nearest PTX, not the fast-math operators), i.e. exactly what the
// reference's NumPy float32 code computes.  A NaN anywhere along an axis makes
// that axis' minimum NaN (NumPy's min); the two axes then combine with
// Python's min.
__device__ __forceinline__ float ieee_div(float a, float b) {
    float d;
    asm("div.rn.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float ieee_mul(float a, float b) {
    float d;
    asm("mul.rn.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float ieee_add(float a, float b) {
    float d;
    asm("add.rn.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float ieee_sqrt(float a) {
    float d;
    asm("sqrt.rn.f32 %0, %1;" : "=f"(d) : "f"(a));
    return d;
}

__global__ void cfl0_partial_kernel(const float* __restrict__ h, const float* __restrict__ hu,
                                    const float* __restrict__ hv, int rows, int cols, int pitch, float dx, float dy,
                                    float c2, float2* __restrict__ part) {
    float mx = INFINITY, my = INFINITY;
    int nan_x = 0, nan_y = 0;
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
        const long long k = (long long)r * pitch + c;
        const float hh = h[k];
        const float cc = ieee_sqrt(ieee_mul(c2, hh));
        const float ax = ieee_div(dx, ieee_add(fabsf(ieee_div(hu[k], hh)), cc));
        const float ay = ieee_div(dy, ieee_add(fabsf(ieee_div(hv[k], hh)), cc));
        if (isnan(ax)) nan_x = 1; else if (ax < mx) mx = ax;
        if (isnan(ay)) nan_y = 1; else if (ay < my) my = ay;
    }
    __shared__ float rx[256 / 32], ry[256 / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fminf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        my = fminf(my, __shfl_xor_sync(0xffffffffu, my, o));
    }
    nan_x = __syncthreads_or(nan_x);
    nan_y = __syncthreads_or(nan_y);
    if ((threadIdx.x & 31) == 0) {
        rx[threadIdx.x >> 5] = mx;
        ry[threadIdx.x >> 5] = my;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mx = fminf(mx, rx[w]);
            my = fminf(my, ry[w]);
        }
        part[blockIdx.x] = make_float2(nan_x ? NAN : mx, nan_y ? NAN : my);
    }
}

// Combines the partial minima and seeds the control block: cfl_min = the
// estimate, dt = the estimate (a simulator before simulate(),
// EE2D_KP07_dimsplit.py:107) or dt = estimate * factor * cfl_scale (a batch
// instance, whose first step is simulate()'s step 0).
// Self-test of the stage kernels' bounded wait: one warp waits on an mbarrier
// whose expected transaction bytes no copy will ever deliver (no copy is
// issued, so nothing lands in shared memory later); out[0] = 1 when the wait
// ended by its poll limit, 0 if it completed.
__global__ void selftest_wait_kernel(uint32_t polls, int* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        fv::mbar_init(&bar, 1);
        fv::fence_barrier_init();
        fv::mbar_arrive_expect_tx(&bar, 16);
    }
    __syncthreads();
    const bool ok = fv::mbar_wait_bounded(&bar, 0, polls);
    if (threadIdx.x == 0) out[0] = ok ? 0 : 1;
}

__global__ void cfl0_final_kernel(const float2* __restrict__ part, int n, SimCtl* ctl, int scaled) {
    float mx = INFINITY, my = INFINITY;
    bool nan_x = false, nan_y = false;
    for (int i = 0; i < n; ++i) {
        const float2 p = part[i];
        if (isnan(p.x)) nan_x = true; else if (p.x < mx) mx = p.x;
        if (isnan(p.y)) nan_y = true; else if (p.y < my) my = p.y;
    }
    if (nan_x) mx = NAN;
    if (nan_y) my = NAN;
    const float cfl0 = (my < mx) ? my : mx;
    ctl->cfl_min = cfl0;
    ctl->dt = scaled ? ieee_mul(ieee_mul(cfl0, ctl->factor), ctl->cfl_scale) : cfl0;
}

// Queues the initial-CFL kernels on `st`; `scratch` holds at least
// `max_parts` float2.
int launch_initial_cfl(cudaStream_t st, const float* h, const float* hu, const float* hv, int rows, int cols,
                       int pitch, float dx, float dy, float c2, float2* scratch, int max_parts, SimCtl* ctl,
                       bool scaled) {
    const long long n = (long long)rows * cols;
    const int parts = (int)std::max<long long>(1, std::min<long long>({(n + 255) / 256, (long long)max_parts, 592}));
    cfl0_partial_kernel<<<parts, 256, 0, st>>>(h, hu, hv, rows, cols, pitch, dx, dy, c2, scratch);
    cfl0_final_kernel<<<1, 1, 0, st>>>(scratch, parts, ctl, scaled ? 1 : 0);
    FV_CK(cudaGetLastError());
    return FV_OK;
}

__global__ void sum_rows_kernel(const float* __restrict__ a, int nx, int pitch, double* __restrict__ out) {
    // one CTA per interior row, fixed reduction order
    __shared__ double red[256 / 32];
    const float* row = a + fv::cell_index(blockIdx.x, 0, pitch);
    double acc = 0.0;
    for (int i = threadIdx.x; i < nx; i += 256) acc += (double)row[i];
    const double r = fv::block_sum<256>(acc, red);
    if (threadIdx.x == 0) out[blockIdx.x] = r;
}

__global__ void sum_final_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double red[256 / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) acc += part[i];
    const double r = fv::block_sum<256>(acc, red);
    if (threadIdx.x == 0) *out = r;
}

__global__ void nan_scan_kernel(const float* __restrict__ a, long long n, int* __restrict__ flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (isnan(a[i])) atomicOr(flag, 1);
}

}  // namespace

// Shared with the other translation units of the library (not exported).
void fv_internal_set_error(const char* msg) { g_err = msg; }

// Pinned host staging for copies between pageable host arrays and the device:
// a pageable 2-D copy is staged by the driver row by row, while a pinned one is
// a single DMA.  A ring of slots serves all simulations and batches of a
// context; a copy reserves a slot (the lock covers only the reservation, so
// copies of different threads proceed in parallel), waits for the slot's
// previous copy (its event) and releases the slot when done.
struct HostStaging {
    static constexpr int kSlots = 8;
    void* ptr[kSlots] = {};
    size_t cap[kSlots] = {};
    cudaEvent_t ev[kSlots] = {};
    bool busy[kSlots] = {};
    int next = 0;
    std::mutex mu;
    std::condition_variable freed;
    ~HostStaging() {
        for (int k = 0; k < kSlots; ++k) {
            if (ev[k]) {
                cudaEventSynchronize(ev[k]);
                cudaEventDestroy(ev[k]);
            }
            if (ptr[k]) cudaFreeHost(ptr[k]);
        }
    }
};

// Pinned host mirrors of the simulations' control blocks, handed out from
// chunks of 64 so that creating and destroying a simulation pins and unpins
// no memory (cudaMallocHost/cudaFreeHost cost milliseconds each).
struct CtlSlab {
    static constexpr int kPerChunk = 64;
    std::mutex mu;
    std::vector<SimCtl*> chunks;
    std::vector<SimCtl*> free_list;
    SimCtl* acquire() {
        std::lock_guard<std::mutex> lock(mu);
        if (free_list.empty()) {
            SimCtl* c = nullptr;
            if (cudaMallocHost(&c, kPerChunk * sizeof(SimCtl)) != cudaSuccess) return nullptr;
            chunks.push_back(c);
            for (int i = kPerChunk - 1; i >= 0; --i) free_list.push_back(c + i);
        }
        SimCtl* p = free_list.back();
        free_list.pop_back();
        return p;
    }
    void release(SimCtl* p) {
        std::lock_guard<std::mutex> lock(mu);
        free_list.push_back(p);
    }
    ~CtlSlab() {
        for (SimCtl* c : chunks) cudaFreeHost(c);
    }
};

struct fv_context {
    int device = 0;
    int sm_count = 0;
    char name[256] = {0};
    HostStaging staging;
    CtlSlab ctl_slab;
};

struct fv_sim {
    fv_context* ctx = nullptr;
    int scheme = 0, nx = 0, ny = 0, pitch = 0, nv = 0, gc = 0, num_substeps = 1;
    float dx = 1, dy = 1;
    fv_params p{};
    int bc = 0;
    float dt_scale = 1.0f;
    float factor = 0.5f;
    void* mem = nullptr;      // one pool allocation: both buffers, control block, scratch
    float* buf[2][4] = {{nullptr}};
    SimCtl* ctl = nullptr;    // device
    SimCtl* ctl_h = nullptr;  // pinned host mirror (from the context's slab)
    float* block_cfl = nullptr;
    double* block_sums = nullptr;
    double* sum_part = nullptr;
    int* flag = nullptr;
    const KEntry* ke = nullptr;
    dim3 grid;
    cudaStream_t stream = nullptr;
    alignas(64) StageArgs args;
    cudaGraphExec_t graph1 = nullptr, graph16 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
};

namespace {

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host copies in progress (all contexts): copy_rows shares 8 helper threads
// among them, so that several host threads copying at once (admissions and
// returns of a served stream) do not oversubscribe the cores.
std::atomic<int> g_active_copies{0};

// rows x width bytes from src (row stride spitch) to dst (row stride dpitch),
// split across up to 8 threads (one per 512 KB) for copies of 1 MB and more,
// fewer while other copies run.
void copy_rows(char* dst, size_t dpitch, const char* src, size_t spitch, size_t width, size_t rows) {
    auto work = [=](size_t r0, size_t r1) {
        if (dpitch == width && spitch == width) {
            memcpy(dst + r0 * width, src + r0 * width, (r1 - r0) * width);
        } else {
            for (size_t r = r0; r < r1; ++r) memcpy(dst + r * dpitch, src + r * spitch, width);
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t bytes = width * rows;
    const int active = g_active_copies.fetch_add(1) + 1;
    struct Leave {
        ~Leave() { g_active_copies.fetch_sub(1); }
    } leave;
    const size_t share = std::max<size_t>(1, 8 / (size_t)active);
    const size_t nt = (bytes >= (1u << 20)) ? std::min<size_t>({share, hw, rows, bytes >> 19}) : 1;
    if (nt <= 1) {
        work(0, rows);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nt; ++t) pool.emplace_back(work, rows * t / nt, rows * (t + 1) / nt);
    work(0, rows / nt);
    for (auto& th : pool) th.join();
}

// A reserved staging slot of at least `bytes`, free of earlier copies; the
// slot is released when the object goes out of scope.
struct StagingSlot {
    HostStaging* H = nullptr;
    int k = -1;
    void* ptr = nullptr;
    cudaEvent_t ev = nullptr;
    ~StagingSlot() {
        if (k >= 0) {
            std::lock_guard<std::mutex> lock(H->mu);
            H->busy[k] = false;
            H->freed.notify_one();
        }
    }
};

int staging_slot(fv_context* ctx, size_t bytes, StagingSlot& out) {
    HostStaging& H = ctx->staging;
    int k = -1;
    {
        std::unique_lock<std::mutex> lock(H.mu);
        for (;;) {
            for (int i = 0; i < HostStaging::kSlots && k < 0; ++i) {
                const int c = (H.next + i) % HostStaging::kSlots;
                if (!H.busy[c]) k = c;
            }
            if (k >= 0) break;
            H.freed.wait(lock);
        }
        H.busy[k] = true;
        H.next = (k + 1) % HostStaging::kSlots;
    }
    out.H = &H;
    out.k = k;
    if (!H.ev[k]) {
        FV_CK(cudaEventCreateWithFlags(&H.ev[k], cudaEventDisableTiming));
    } else {
        FV_CK(cudaEventSynchronize(H.ev[k]));
    }
    if (H.cap[k] < bytes) {
        if (H.ptr[k]) cudaFreeHost(H.ptr[k]);
        H.ptr[k] = nullptr;
        H.cap[k] = 0;
        const size_t cap = std::max<size_t>(bytes, 8u << 20);
        if (cudaHostAlloc(&H.ptr[k], cap, cudaHostAllocPortable) != cudaSuccess)
            return fail(FV_ERR_NOMEM, "cannot allocate %zu bytes of pinned staging memory", cap);
        H.cap[k] = cap;
    }
    out.ptr = H.ptr[k];
    out.ev = H.ev[k];
    return FV_OK;
}

// Host (any memory) -> device 2-D copy queued on `st`; pageable sources go
// through a staging slot.  Returns once the host array may be reused.
int copy_h2d(fv_context* ctx, cudaStream_t st, float* dst, size_t dpitch, const float* src, size_t spitch,
             size_t width, size_t rows) {
    if (is_pinned(src)) {
        FV_CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyHostToDevice, st));
        return FV_OK;
    }
    StagingSlot slot;
    FV_TRY(staging_slot(ctx, width * rows, slot));
    copy_rows(static_cast<char*>(slot.ptr), width, reinterpret_cast<const char*>(src), spitch, width, rows);
    FV_CK(cudaMemcpy2DAsync(dst, dpitch, slot.ptr, width, width, rows, cudaMemcpyHostToDevice, st));
    FV_CK(cudaEventRecord(slot.ev, st));
    return FV_OK;
}

// Device -> host (any memory) 2-D copy ordered after the work queued on `st`;
// returns when the host array holds the data.
int copy_d2h(fv_context* ctx, cudaStream_t st, float* dst, size_t dpitch, const float* src, size_t spitch,
             size_t width, size_t rows) {
    if (is_pinned(dst)) {
        FV_CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost, st));
        FV_CK(cudaStreamSynchronize(st));
        return FV_OK;
    }
    StagingSlot slot;
    FV_TRY(staging_slot(ctx, width * rows, slot));
    FV_CK(cudaMemcpy2DAsync(slot.ptr, width, src, spitch, width, rows, cudaMemcpyDeviceToHost, st));
    FV_CK(cudaEventRecord(slot.ev, st));
    FV_CK(cudaEventSynchronize(slot.ev));
    copy_rows(reinterpret_cast<char*>(dst), dpitch, static_cast<const char*>(slot.ptr), width, width, rows);
    return FV_OK;
}

// Flux variants exist for HLL (3) and limiters for WAF (9); other schemes take 0.
int check_variant(int scheme, const fv_params* p) {
    const int n = (scheme == FV_HLL) ? 3 : (scheme == FV_WAF) ? 9 : 1;
    if (p->variant < 0 || p->variant >= n)
        return fail(FV_ERR_INVALID, "variant %d does not exist for scheme %d", p->variant, scheme);
    return FV_OK;
}

int read_ctl(fv_sim* s) {
    FV_CK(cudaMemcpyAsync(s->ctl_h, s->ctl, sizeof(SimCtl), cudaMemcpyDeviceToHost, s->stream));
    FV_CK(cudaStreamSynchronize(s->stream));
    if (s->ctl_h->error) return fail(FV_ERR_DEVICE, "a stage kernel gave up waiting for its tile load");
    return FV_OK;
}

int write_ctl(fv_sim* s) {
    FV_CK(cudaMemcpyAsync(s->ctl, s->ctl_h, sizeof(SimCtl), cudaMemcpyHostToDevice, s->stream));
    FV_CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

// An NVTX range over a host-side scope (stage launches, graph replays, batch
// runs and syncs), visible on a profiler's timeline; without a profiler
// attached the push and pop return at once.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Stage kernels are launched with programmatic stream serialization: the next
// substep's CTAs may launch while this one's last CTAs run, and wait in the
// kernel (grid_dependency_wait) for its completion before reading anything.
cudaError_t launch_dependent(const void* fn, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

int launch_stage(fv_sim* s, int substep, bool is_last, bool force_cfl, bool explicit_dt, float dt, bool sums,
                 int row0 = 0, int nrows = -1) {
    NvtxRange range(nrows >= 0 ? "fv stage launch (band)" : "fv stage launch");
    alignas(64) StageArgs a = s->args;
    dim3 grid = s->grid;
    if (nrows >= 0) {  // a band of tile rows of the substep
        a.tile_row0 = row0;
        a.ntiles_total = (int)(s->grid.x * s->grid.y);
        grid.y = (unsigned)nrows;
    }
    a.substep = substep;
    a.is_last = is_last ? 1 : 0;
    a.force_cfl = force_cfl ? 1 : 0;
    a.explicit_dt = explicit_dt ? 1 : 0;
    a.dt_step = dt;
    a.want_sums = sums ? 1 : 0;
    void* kargs[] = {&a};
    FV_CK(launch_dependent(reinterpret_cast<const void*>(s->ke->fn), grid, dim3(s->ke->NT), kargs,
                           entry_smem(*s->ke), s->stream));
    return FV_OK;
}

int launch_step_graphless(fv_sim* s) {
    for (int i = 0; i < s->num_substeps; ++i)
        FV_TRY(launch_stage(s, i, i == s->num_substeps - 1, false, false, 0.0f, false));
    return FV_OK;
}

int build_graph(fv_sim* s, int nsteps, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    FV_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = FV_OK;
    for (int k = 0; k < nsteps && rc == FV_OK; ++k) rc = launch_step_graphless(s);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc != FV_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(FV_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(FV_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return FV_OK;
}

int run_steps(fv_sim* s, long long k) {
    NvtxRange range("fv step graph replays");
    if (!s->graph1) FV_TRY(build_graph(s, 1, &s->graph1));
    if (!s->graph16) FV_TRY(build_graph(s, 16, &s->graph16));
    while (k >= 16) {
        FV_CK(cudaGraphLaunch(s->graph16, s->stream));
        k -= 16;
    }
    while (k > 0) {
        FV_CK(cudaGraphLaunch(s->graph1, s->stream));
        --k;
    }
    return FV_OK;
}

// dt = computeDt() * cfl_scale at steps 0, 100, 200, ... (Simulator.py:195-196).
void host_dt_update(fv_sim* s) {
    SimCtl& c = *s->ctl_h;
    if (c.update_dt && c.nt % 100 == 0) c.dt = (c.cfl_min * c.factor) * c.cfl_scale;
}

int check_sim(fv_sim* s) {
    if (!s) return fail(FV_ERR_INVALID, "null simulation");
    FV_CK(cudaSetDevice(s->ctx->device));
    return FV_OK;
}

}  // namespace

extern "C" {

int fv_version(void) { return 100; }

const char* fv_last_error(void) { return g_err.c_str(); }

int fv_context_create(int device, fv_context** out) {
    if (!out) return fail(FV_ERR_INVALID, "out is null");
    int n = 0;
    FV_CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(FV_ERR_INVALID, "device %d out of range (%d devices)", device, n);
    FV_CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    FV_CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(FV_ERR_UNSUPPORTED, "libfvgpu is built for sm_100a; device is sm_%d%d", prop.major, prop.minor);
    if (!encode_fn()) return fail(FV_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    for (int i = 0; i < kNumEntries; ++i) {
        FV_CK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kTable[i].fn),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)entry_smem(kTable[i])));
        FV_CK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kTable[i].fn),
                                   cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    }
    for (int i = 0; i < kNumVariants; ++i)
        FV_CK(cudaFuncSetAttribute(reinterpret_cast<const void*>(kVariantTable[i].k.fn),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)entry_smem(kVariantTable[i].k)));
    // Device memory of finished simulations stays in the stream-ordered pool
    // for the next ones instead of being unmapped at every synchronisation
    // (the pool is trimmed when the context is destroyed).  Memory freed on
    // one stream is reused on another only once the free has completed: an
    // admission queued on a batch's copy stream must not wait for the
    // compute stream's current chunk.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        int no = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    }
    fv_context* c = new fv_context;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    snprintf(c->name, sizeof(c->name), "%s", prop.name);
    *out = c;
    return FV_OK;
}

int fv_context_destroy(fv_context* ctx) {
    if (ctx) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    }
    delete ctx;
    return FV_OK;
}

int fv_context_device_name(fv_context* ctx, char* buf, int len) {
    if (!ctx || !buf || len <= 0) return fail(FV_ERR_INVALID, "bad argument");
    snprintf(buf, (size_t)len, "%s", ctx->name);
    return FV_OK;
}

int fv_sim_create(fv_context* ctx, int scheme, int nx, int ny, float dx, float dy, const fv_params* params, int bc,
                  const float* const* host_vars, int host_rows, int host_cols, fv_sim** out) {
    if (!ctx || !params || !host_vars || !out) return fail(FV_ERR_INVALID, "null argument");
    if (scheme < FV_LXF || scheme > FV_EE2D_KP07_DIMSPLIT) return fail(FV_ERR_INVALID, "unknown scheme %d", scheme);
    if (nx < 1 || ny < 1 || nx > (1 << 20) || ny > (1 << 20)) return fail(FV_ERR_INVALID, "bad grid %d x %d", nx, ny);
    FV_TRY(check_variant(scheme, params));
    for (int side = 0; side < 4; ++side)
        if (((bc >> (8 * side)) & 0xF) == fv::BC_NEUMANN)
            return fail(FV_ERR_UNSUPPORTED, "Neumann boundary condition not supported");
    const int nv = scheme_nv(scheme), gc = scheme_ghost(scheme);
    const bool halo = (host_rows == ny + 2 * gc && host_cols == nx + 2 * gc);
    if (!halo && !(host_rows == ny && host_cols == nx))
        return fail(FV_ERR_INVALID, "Wrong shape of data (%d, %d) vs (%d, %d) / (%d, %d)", host_rows, host_cols, ny, nx,
                    ny + 2 * gc, nx + 2 * gc);
    for (int v = 0; v < nv; ++v)
        if (!host_vars[v]) return fail(FV_ERR_INVALID, "variable %d is null", v);
    const int cfg = params->tile < 0 ? 0 : params->tile;
    const KEntry* ke = find_entry(scheme, cfg, params->variant);
    if (!ke) return fail(FV_ERR_INVALID, "tile configuration %d does not exist for scheme %d", cfg, scheme);
    FV_CK(cudaSetDevice(ctx->device));

    fv_sim* s = new fv_sim;
    s->ctx = ctx;
    s->scheme = scheme;
    s->nx = nx;
    s->ny = ny;
    s->nv = nv;
    s->gc = gc;
    s->dx = dx;
    s->dy = dy;
    s->p = *params;
    s->bc = bc;
    s->ke = ke;
    s->pitch = ((nx + 8) + 31) / 32 * 32;  // 128-byte rows; column x at x+4
    s->num_substeps = (scheme == FV_LXF || scheme == FV_FORCE || scheme == FV_HLL) ? 1
                      : (scheme == FV_KP07)                                   ? (params->order == 1 ? 1 : 2)
                                                                              : 2;
    s->dt_scale = (scheme == FV_HLL2 || scheme == FV_WAF || scheme == FV_KP07_DIMSPLIT ||
                   scheme == FV_EE2D_KP07_DIMSPLIT)
                      ? 0.5f
                      : 1.0f;
    // computeDt factors (e.g. KP07_dimsplit.py:137, FORCE.py:129, KP07.py:138)
    s->factor = (scheme == FV_FORCE) ? 1.0f : (scheme == FV_KP07 && params->order == 1) ? 1.0f : 0.5f;
    s->grid = dim3((nx + ke->W - 1) / ke->W, (ny + ke->H - 1) / ke->H);

    auto cleanup = [&](int rc) {
        fv_sim_destroy(s);
        return rc;
    };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(FV_ERR_CUDA, "stream creation failed"));
    // One stream-ordered allocation, zero-filled, holds both state buffers
    // (planes of 128-byte-aligned rows) and the small device objects; no
    // cudaMalloc/cudaFree, which synchronise the device, on create or destroy.
    const size_t plane = (size_t)(ny + 4) * s->pitch * sizeof(float);
    const size_t nblocks = (size_t)s->grid.x * s->grid.y;
    auto r256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t off_ctl = 2 * nv * plane;
    const size_t off_cfl = off_ctl + r256(sizeof(SimCtl));
    const size_t off_sums = off_cfl + r256(nblocks * sizeof(float));
    const size_t off_part = off_sums + r256(nblocks * 4 * sizeof(double));
    const size_t off_flag = off_part + r256((size_t)(ny + 1) * sizeof(double));
    const size_t total = off_flag + 256;
    if (cudaMallocAsync(&s->mem, total, s->stream) != cudaSuccess) {
        cudaGetLastError();
        s->mem = nullptr;
        return cleanup(fail(FV_ERR_NOMEM, "out of device memory"));
    }
    if (cudaMemsetAsync(s->mem, 0, total, s->stream) != cudaSuccess)
        return cleanup(fail(FV_ERR_CUDA, "memset failed"));
    char* base = static_cast<char*>(s->mem);
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < nv; ++v) s->buf[b][v] = reinterpret_cast<float*>(base + (size_t)(b * nv + v) * plane);
    s->ctl = reinterpret_cast<SimCtl*>(base + off_ctl);
    s->block_cfl = reinterpret_cast<float*>(base + off_cfl);
    s->block_sums = reinterpret_cast<double*>(base + off_sums);
    s->sum_part = reinterpret_cast<double*>(base + off_part);
    s->flag = reinterpret_cast<int*>(base + off_flag);
    s->ctl_h = ctx->ctl_slab.acquire();
    if (!s->ctl_h) return cleanup(fail(FV_ERR_NOMEM, "out of pinned host memory"));
    if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess)
        return cleanup(fail(FV_ERR_CUDA, "event creation failed"));

    // upload u0 (interior or full halo, Common.py:524-531)
    const int off = halo ? gc : 0;
    for (int v = 0; v < nv; ++v) {
        float* dst = s->buf[0][v] + fv::cell_index(-off, -off, s->pitch);
        if (copy_h2d(ctx, s->stream, dst, s->pitch * sizeof(float), host_vars[v], host_cols * sizeof(float),
                     host_cols * sizeof(float), host_rows) != FV_OK)
            return cleanup(FV_ERR_CUDA);
    }

    // control block
    SimCtl& c = *s->ctl_h;
    memset(&c, 0, sizeof(SimCtl));
    const float c2 = (scheme == FV_EE2D_KP07_DIMSPLIT) ? params->gamma : params->g;
    c.t = 0.0;
    c.t_end = 0.0;
    c.nt = 0;
    c.factor = s->factor;
    c.cfl_scale = params->cfl_scale;
    c.update_dt = 1;
    c.cur = 0;
    if (write_ctl(s) != FV_OK) return cleanup(FV_ERR_CUDA);
    // cfl_min and dt = the initial CFL estimate (dt as EE2D_KP07_dimsplit.py:107;
    // the other classes leave dt unset until simulate())
    if (launch_initial_cfl(s->stream, s->buf[0][0] + fv::cell_index(-off, -off, s->pitch),
                           s->buf[0][1] + fv::cell_index(-off, -off, s->pitch),
                           s->buf[0][2] + fv::cell_index(-off, -off, s->pitch), host_rows, host_cols, s->pitch, dx, dy,
                           c2, reinterpret_cast<float2*>(s->block_sums), (int)(nblocks * 4), s->ctl, false) != FV_OK)
        return cleanup(FV_ERR_CUDA);

    // kernel arguments and TMA descriptors
    StageArgs& a = s->args;
    memset(&a, 0, sizeof(StageArgs));
    auto enc = encode_fn();
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < nv; ++v) {
            a.buf[b][v] = s->buf[b][v];
            cuuint64_t dims[2] = {(cuuint64_t)(nx + 8), (cuuint64_t)(ny + 4)};
            cuuint64_t strides[1] = {(cuuint64_t)s->pitch * sizeof(float)};
            cuuint32_t box[2] = {(cuuint32_t)entry_box_w(*ke), (cuuint32_t)(ke->H + 4)};
            cuuint32_t estr[2] = {1, 1};
            CUresult r = enc(&a.tmap[b][v], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, s->buf[b][v], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return cleanup(fail(FV_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r));
        }
    a.ctl = s->ctl;
    a.block_cfl = s->block_cfl;
    a.block_sums = s->block_sums;
    a.nx = nx;
    a.ny = ny;
    a.pitch = s->pitch;
    a.dx = dx;
    a.dy = dy;
    a.g = params->g;
    a.gamma = params->gamma;
    a.theta = params->theta;
    a.dt_scale = s->dt_scale;
    a.bc = bc;
    a.order = params->order;
    a.variant_beta = params->variant_beta;
    *out = s;
    return FV_OK;
}

int fv_sim_destroy(fv_sim* s) {
    if (!s) return FV_OK;
    cudaSetDevice(s->ctx->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph1) cudaGraphExecDestroy(s->graph1);
    if (s->graph16) cudaGraphExecDestroy(s->graph16);
    if (s->mem) cudaFreeAsync(s->mem, s->stream);
    if (s->ctl_h) s->ctx->ctl_slab.release(s->ctl_h);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FV_OK;
}

int fv_sim_substep(fv_sim* s, float dt, int step_number) {
    FV_TRY(check_sim(s));
    if (step_number < 0 || step_number >= s->num_substeps)
        return fail(FV_ERR_INVALID, "substep %d out of range", step_number);
    return launch_stage(s, step_number, false, true, true, dt, false);
}

int fv_sim_substep_rows(fv_sim* s, float dt, int step_number, int row0, int nrows) {
    FV_TRY(check_sim(s));
    if (step_number < 0 || step_number >= s->num_substeps)
        return fail(FV_ERR_INVALID, "substep %d out of range", step_number);
    if (row0 < 0 || nrows < 1 || row0 + nrows > (int)s->grid.y)
        return fail(FV_ERR_INVALID, "tile rows [%d, %d) outside [0, %d)", row0, row0 + nrows, (int)s->grid.y);
    return launch_stage(s, step_number, false, true, true, dt, false, row0, nrows);
}

int fv_sim_tile_rows(fv_sim* s, int* rows) {
    FV_TRY(check_sim(s));
    if (!rows) return fail(FV_ERR_INVALID, "null argument");
    *rows = (int)s->grid.y;
    return FV_OK;
}

int fv_sim_step(fv_sim* s, float dt) {
    FV_TRY(check_sim(s));
    for (int i = 0; i < s->num_substeps; ++i)
        FV_TRY(launch_stage(s, i, i == s->num_substeps - 1, true, true, dt, false));
    return FV_OK;
}

int fv_sim_simulate(fv_sim* s, double t, float dt, int use_dt) {
    NvtxRange range("fv_sim_simulate");
    FV_TRY(check_sim(s));
    FV_TRY(read_ctl(s));
    SimCtl& c = *s->ctl_h;
    const double t_end = c.t + t;
    c.t_end = t_end;
    c.update_dt = use_dt ? 0 : 1;
    if (use_dt) c.dt = dt;
    for (;;) {
        if (!(c.t < t_end)) break;
        host_dt_update(s);
        FV_TRY(write_ctl(s));
        // steps until the next dt update or t_end, replaying the device arithmetic
        const long long limit = c.update_dt ? 100 - (c.nt % 100) : 1000;
        long long k = 0;
        double tt = c.t;
        while (k < limit && tt < t_end) {
            const double rem = t_end - tt;
            const double d = (double)c.dt;
            const float cur = (float)((rem < d) ? rem : d);
            if (cur <= 0.0f) break;
            tt += (double)cur;
            ++k;
        }
        if (k == 0) break;  // dt <= 0: the reference warns and stops (Simulator.py:202-204)
        FV_TRY(run_steps(s, k));
        FV_TRY(read_ctl(s));
    }
    return FV_OK;
}

int fv_sim_advance(fv_sim* s, long long n_steps) {
    FV_TRY(check_sim(s));
    if (n_steps < 0) return fail(FV_ERR_INVALID, "negative step count");
    FV_TRY(read_ctl(s));
    SimCtl& c = *s->ctl_h;
    c.t_end = INFINITY;
    c.update_dt = 1;
    host_dt_update(s);
    FV_TRY(write_ctl(s));
    if (!s->graph1) FV_TRY(build_graph(s, 1, &s->graph1));
    if (!s->graph16) FV_TRY(build_graph(s, 16, &s->graph16));
    FV_CK(cudaEventRecord(s->ev0, s->stream));
    FV_TRY(run_steps(s, n_steps));
    FV_CK(cudaEventRecord(s->ev1, s->stream));
    FV_CK(cudaEventSynchronize(s->ev1));
    float ms = 0.0f;
    FV_CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->last_ms = n_steps > 0 ? (double)ms / (double)n_steps : 0.0;
    return read_ctl(s);
}

int fv_sim_compute_dt(fv_sim* s, float* dt) {
    FV_TRY(check_sim(s));
    if (!dt) return fail(FV_ERR_INVALID, "dt is null");
    FV_TRY(read_ctl(s));
    *dt = s->ctl_h->cfl_min * s->ctl_h->factor;
    return FV_OK;
}

int fv_sim_download(fv_sim* s, int var, float* host, int host_pitch) {
    FV_TRY(check_sim(s));
    if (var < 0 || var >= s->nv || !host || host_pitch < s->nx) return fail(FV_ERR_INVALID, "bad download argument");
    FV_TRY(read_ctl(s));
    const float* src = s->buf[s->ctl_h->cur][var] + fv::cell_index(0, 0, s->pitch);
    return copy_d2h(s->ctx, s->stream, host, (size_t)host_pitch * sizeof(float), src, (size_t)s->pitch * sizeof(float),
                    (size_t)s->nx * sizeof(float), s->ny);
}

int fv_sim_upload(fv_sim* s, int var, const float* host, int host_pitch) {
    FV_TRY(check_sim(s));
    if (var < 0 || var >= s->nv || !host || host_pitch < s->nx) return fail(FV_ERR_INVALID, "bad upload argument");
    FV_TRY(read_ctl(s));
    float* dst = s->buf[s->ctl_h->cur][var] + fv::cell_index(0, 0, s->pitch);
    FV_TRY(copy_h2d(s->ctx, s->stream, dst, (size_t)s->pitch * sizeof(float), host, (size_t)host_pitch * sizeof(float),
                    (size_t)s->nx * sizeof(float), s->ny));
    FV_CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

// The region's first cell in storage coordinates, after checking that the
// region lies inside the reference's halo-inclusive array (Common.py:564-565).
int region_check(fv_sim* s, int var, int x, int y, int w, int h, const void* host, int host_pitch) {
    const int gc = s->gc;
    if (var < 0 || var >= s->nv || !host || w < 1 || h < 1 || host_pitch < w || x < 0 || y < 0 ||
        x + w > s->nx + 2 * gc || y + h > s->ny + 2 * gc)
        return fail(FV_ERR_INVALID, "region (%d, %d, %d, %d) outside the %d x %d array with ghost cells", x, y, w, h,
                    s->nx + 2 * gc, s->ny + 2 * gc);
    return FV_OK;
}

int fv_sim_download_region(fv_sim* s, int var, int x, int y, int w, int h, float* host, int host_pitch) {
    FV_TRY(check_sim(s));
    FV_TRY(region_check(s, var, x, y, w, h, host, host_pitch));
    FV_TRY(read_ctl(s));
    const float* src = s->buf[s->ctl_h->cur][var] + fv::cell_index(y - s->gc, x - s->gc, s->pitch);
    return copy_d2h(s->ctx, s->stream, host, (size_t)host_pitch * sizeof(float), src, (size_t)s->pitch * sizeof(float),
                    (size_t)w * sizeof(float), h);
}

int fv_sim_upload_region(fv_sim* s, int var, int x, int y, int w, int h, const float* host, int host_pitch) {
    FV_TRY(check_sim(s));
    FV_TRY(region_check(s, var, x, y, w, h, host, host_pitch));
    FV_TRY(read_ctl(s));
    float* dst = s->buf[s->ctl_h->cur][var] + fv::cell_index(y - s->gc, x - s->gc, s->pitch);
    FV_TRY(copy_h2d(s->ctx, s->stream, dst, (size_t)s->pitch * sizeof(float), host, (size_t)host_pitch * sizeof(float),
                    (size_t)w * sizeof(float), h));
    FV_CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_sim_time(fv_sim* s, double* t, long long* nt, float* dt) {
    FV_TRY(check_sim(s));
    FV_TRY(read_ctl(s));
    if (t) *t = s->ctl_h->t;
    if (nt) *nt = s->ctl_h->nt;
    if (dt) *dt = s->ctl_h->dt;
    return FV_OK;
}

int fv_sim_conservation(fv_sim* s, double* sums) {
    FV_TRY(check_sim(s));
    if (!sums) return fail(FV_ERR_INVALID, "sums is null");
    FV_TRY(read_ctl(s));
    double* dev_tot = s->block_sums;  // scratch: reduced before any stage kernel reuses it
    for (int v = 0; v < s->nv; ++v) {
        sum_rows_kernel<<<s->ny, 256, 0, s->stream>>>(s->buf[s->ctl_h->cur][v], s->nx, s->pitch, s->sum_part);
        sum_final_kernel<<<1, 256, 0, s->stream>>>(s->sum_part, s->ny, dev_tot + v);
        FV_CK(cudaGetLastError());
    }
    FV_CK(cudaMemcpyAsync(sums, dev_tot, s->nv * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    FV_CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_sim_check(fv_sim* s, int* has_nan) {
    FV_TRY(check_sim(s));
    if (!has_nan) return fail(FV_ERR_INVALID, "has_nan is null");
    FV_CK(cudaMemsetAsync(s->flag, 0, sizeof(int), s->stream));
    const long long n = (long long)(s->ny + 4) * s->pitch;
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < s->nv; ++v) nan_scan_kernel<<<4 * s->ctx->sm_count, 256, 0, s->stream>>>(s->buf[b][v], n, s->flag);
    FV_CK(cudaGetLastError());
    int f = 0;
    FV_CK(cudaMemcpyAsync(&f, s->flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    FV_CK(cudaStreamSynchronize(s->stream));
    *has_nan = f;
    return FV_OK;
}

int fv_sim_synchronize(fv_sim* s) {
    FV_TRY(check_sim(s));
    FV_CK(cudaStreamSynchronize(s->stream));
    return FV_OK;
}

int fv_sim_set_boundary_conditions(fv_sim* s, int bc) {
    FV_TRY(check_sim(s));
    for (int side = 0; side < 4; ++side)
        if (((bc >> (8 * side)) & 0xF) == fv::BC_NEUMANN)
            return fail(FV_ERR_UNSUPPORTED, "Neumann boundary condition not supported");
    FV_CK(cudaStreamSynchronize(s->stream));
    s->bc = bc;
    s->args.bc = bc;
    if (s->graph1) cudaGraphExecDestroy(s->graph1);
    if (s->graph16) cudaGraphExecDestroy(s->graph16);
    s->graph1 = s->graph16 = nullptr;
    return FV_OK;
}

int fv_sim_set_wait_limit(fv_sim* s, int polls) {
    FV_TRY(check_sim(s));
    FV_CK(cudaStreamSynchronize(s->stream));
    s->args.wait_limit = polls < 0 ? 0 : (polls == 0 ? -1 : polls);
    if (s->graph1) cudaGraphExecDestroy(s->graph1);
    if (s->graph16) cudaGraphExecDestroy(s->graph16);
    s->graph1 = s->graph16 = nullptr;
    return FV_OK;
}

int fv_selftest_bounded_wait(int polls, int* gave_up) {
    if (!gave_up || polls < 0) return fail(FV_ERR_INVALID, "bad argument");
    int* d = nullptr;
    FV_CK(cudaMalloc(&d, sizeof(int)));
    selftest_wait_kernel<<<1, 32>>>((uint32_t)polls, d);
    int h = -1;
    const cudaError_t e1 = cudaGetLastError();
    const cudaError_t e2 = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return fail(FV_ERR_CUDA, "self-test kernel failed");
    *gave_up = h;
    return FV_OK;
}

int fv_sim_get_control(fv_sim* s, double* t, long long* nt, float* dt, float* cfl_min) {
    FV_TRY(check_sim(s));
    FV_TRY(read_ctl(s));
    if (t) *t = s->ctl_h->t;
    if (nt) *nt = s->ctl_h->nt;
    if (dt) *dt = s->ctl_h->dt;
    if (cfl_min) *cfl_min = s->ctl_h->cfl_min;
    return FV_OK;
}

int fv_sim_set_control(fv_sim* s, double t, long long nt, float dt, float cfl_min) {
    FV_TRY(check_sim(s));
    if (nt < 0) return fail(FV_ERR_INVALID, "negative step count");
    FV_TRY(read_ctl(s));
    s->ctl_h->t = t;
    s->ctl_h->nt = nt;
    s->ctl_h->dt = dt;
    s->ctl_h->cfl_min = cfl_min;
    return write_ctl(s);
}

int fv_sim_buffers(fv_sim* s, float** ptrs, int* pitch, int* cur) {
    FV_TRY(check_sim(s));
    if (!ptrs || !pitch || !cur) return fail(FV_ERR_INVALID, "bad argument");
    FV_TRY(read_ctl(s));
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < 4; ++v) ptrs[b * 4 + v] = (v < s->nv) ? s->buf[b][v] : nullptr;
    *pitch = s->pitch;
    *cur = s->ctl_h->cur;
    return FV_OK;
}

int fv_sim_stream(fv_sim* s, void** stream) {
    FV_TRY(check_sim(s));
    if (!stream) return fail(FV_ERR_INVALID, "stream is null");
    *stream = static_cast<void*>(s->stream);
    return FV_OK;
}

int fv_sim_info(fv_sim* s, int* tile_w, int* tile_h, int* threads, int* launches_per_step) {
    if (!s) return fail(FV_ERR_INVALID, "null simulation");
    if (tile_w) *tile_w = s->ke->W;
    if (tile_h) *tile_h = s->ke->H;
    if (threads) *threads = s->ke->NT;
    if (launches_per_step) *launches_per_step = s->num_substeps;
    return FV_OK;
}

int fv_sim_last_advance_ms(fv_sim* s, double* ms) {
    if (!s || !ms) return fail(FV_ERR_INVALID, "bad argument");
    *ms = s->last_ms;
    return FV_OK;
}

int fv_host_alloc(void** ptr, size_t bytes) {
    if (!ptr) return fail(FV_ERR_INVALID, "ptr is null");
    if (cudaMallocHost(ptr, bytes) != cudaSuccess) return fail(FV_ERR_NOMEM, "pinned allocation of %zu bytes failed", bytes);
    return FV_OK;
}

int fv_host_free(void* ptr) {
    FV_CK(cudaFreeHost(ptr));
    return FV_OK;
}

}  // extern "C"

// ====================================================================== batches
//
// A batch advances many simulations of one scheme together: each launch of
// the batched kernel covers a device-resident work list of (simulation, tile)
// pairs, every simulation keeps its own control block (t, dt, t_end, buffer
// parity), and graphs of 1 and 16 steps are captured once.  Adding or
// removing a simulation rewrites the work list between graph replays and sets
// the graphs' launch grid to its new length (one CTA per entry).

struct fv_batch {
    fv_context* ctx = nullptr;
    int scheme = 0, nv = 3, gc = 2, num_substeps = 2;
    fv_params p{};
    float dt_scale = 0.5f, factor = 0.5f;
    const BEntry* be = nullptr;
    int max_inst = 0;
    cudaStream_t stream = nullptr;
    fv::BatchInstance* d_inst = nullptr;  // device, max_inst entries
    fv::BatchInstance* h_inst = nullptr;  // pinned staging
    SimCtl* d_ctl = nullptr;              // device, one control block per slot
    SimCtl* h_ctl = nullptr;              // pinned host view, refreshed by fv_batch_sync
    SimCtl* h_ctl_up = nullptr;           // pinned source of an admitted slot's first control block
    int2* d_work = nullptr;
    int2* h_work[2] = {nullptr, nullptr};  // pinned staging, alternated between publishes
    int* h_nwork[2] = {nullptr, nullptr};
    cudaEvent_t ev_work[2] = {nullptr, nullptr};
    int work_buf = 0;
    int work_cap = 0;
    int nwork = 0;
    int* d_nwork = nullptr;
    int* d_err = nullptr;
    cudaStream_t copy_stream = nullptr;  // uploads/downloads, concurrent with the kernels
    cudaEvent_t ev_up = nullptr, ev_compute = nullptr;
    std::vector<int> done_at_sync;        // slot finished as of the last fv_batch_sync
    std::vector<int> registered;          // slot fully admitted (its instance and control block are queued)
    bool dirty = false;                   // work list changed since the last publish
    std::vector<int> used;               // slot in use
    std::vector<void*> slot_mem;          // per-slot device allocation (planes + tile scratch)
    std::vector<size_t> slot_bytes;
    size_t bytes = 0;
    // Graphs of 1 and 16 steps, kept with their executables so that the grid
    // of their kernel nodes (one CTA per work-list entry) follows the list.
    cudaGraph_t g1 = nullptr, g16 = nullptr;
    cudaGraphExec_t graph1 = nullptr, graph16 = nullptr;
    int graph_grid = 0;  // grid the executables launch
    int resident_grid = 0;  // CTAs resident on the GPU at once (the persistent form's grid)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    // Guards the slot bookkeeping (used, done_at_sync, slot_mem, bytes, dirty,
    // h_inst, h_ctl reads) so that one host thread can return finished
    // simulations (status, download, remove) while another admits and runs.
    // Held only for short sections: never across copies or stream waits.
    std::mutex mu;
};

namespace {

void batch_drop_graphs(fv_batch* b) {
    if (b->graph1) cudaGraphExecDestroy(b->graph1);
    if (b->graph16) cudaGraphExecDestroy(b->graph16);
    if (b->g1) cudaGraphDestroy(b->g1);
    if (b->g16) cudaGraphDestroy(b->g16);
    b->graph1 = b->graph16 = nullptr;
    b->g1 = b->g16 = nullptr;
    b->graph_grid = 0;
}

// CTAs of one batched launch: one per entry of the published work list, or
// for the persistent form every CTA the GPU holds at once.
int batch_grid(const fv_batch* b) {
    if (b->be->persistent) return b->resident_grid;
    return b->nwork > 0 ? b->nwork : 1;
}

// 0 running, 1 reached t_end (simulate()'s stopping rule), 2 failed: a step
// left a non-finite value or a non-positive depth (density), t or dt is not a
// number, or dt is not positive before t_end.
int batch_done_state(const SimCtl& c) {
    if (c.bad || std::isnan(c.t) || std::isnan(c.dt)) return 2;
    if (c.t < c.t_end && !(c.dt > 0.0f)) return 2;  // cannot advance (simulate() would stop here)
    const double rem = c.t_end - c.t;
    const float cur = (float)((rem < (double)c.dt) ? rem : (double)c.dt);
    return (!(c.t < c.t_end) || cur <= 0.0f) ? 1 : 0;
}

int batch_launch_step(fv_batch* b) {
    for (int i = 0; i < b->num_substeps; ++i) {
        fv::BatchArgs a;
        a.inst = b->d_inst;
        a.ctl = b->d_ctl;
        a.work = b->d_work;
        a.nwork = b->d_nwork;
        a.substep = i;
        a.is_last = (i == b->num_substeps - 1) ? 1 : 0;
        a.want_sums = 0;
        a.order = b->p.order;
        a.err = b->d_err;
        void* kargs[] = {&a};
        FV_CK(launch_dependent(reinterpret_cast<const void*>(b->be->fn), dim3(batch_grid(b)), dim3(b->be->NT), kargs,
                               batch_smem(*b->be), b->stream));
    }
    return FV_OK;
}

// Captures nsteps steps into *graph and instantiates it into *out; the graph
// is kept for batch_set_graph_grid.
int batch_build_graph(fv_batch* b, int nsteps, cudaGraph_t* graph, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    FV_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = FV_OK;
    for (int k = 0; k < nsteps && rc == FV_OK; ++k) rc = batch_launch_step(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc != FV_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(FV_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(FV_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
    }
    *graph = g;
    return FV_OK;
}

// Sets the grid of every kernel node of the executable graphs to the current
// work list's length.  An update applies to later launches only; launches
// already queued keep the grid (and, by stream order, the work list) they
// were queued with.  If an update fails the graphs are dropped and rebuilt on
// the next run.
int batch_set_graph_grid(fv_batch* b) {
    const int grid = batch_grid(b);
    if (!b->graph1 || b->graph_grid == grid) return FV_OK;
    const std::pair<cudaGraph_t, cudaGraphExec_t> graphs[2] = {{b->g1, b->graph1}, {b->g16, b->graph16}};
    for (const auto& ge : graphs) {
        size_t count = 0;
        cudaError_t e = cudaGraphGetNodes(ge.first, nullptr, &count);
        std::vector<cudaGraphNode_t> nodes(count);
        if (e == cudaSuccess && count > 0) e = cudaGraphGetNodes(ge.first, nodes.data(), &count);
        for (size_t i = 0; i < count && e == cudaSuccess; ++i) {
            cudaGraphNodeType type;
            e = cudaGraphNodeGetType(nodes[i], &type);
            if (e != cudaSuccess || type != cudaGraphNodeTypeKernel) continue;
            cudaKernelNodeParams kp;
            e = cudaGraphKernelNodeGetParams(nodes[i], &kp);
            if (e != cudaSuccess) break;
            kp.gridDim = dim3(grid);
            e = cudaGraphExecKernelNodeSetParams(ge.second, nodes[i], &kp);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            batch_drop_graphs(b);
            return FV_OK;
        }
    }
    b->graph_grid = grid;
    return FV_OK;
}

// Rebuilds the work list from the slots in use and queues its upload on the
// compute stream, so the kernels enqueued before it still see the old list and
// the ones after it the new one.  The two pinned staging buffers alternate;
// a buffer is rewritten only after its previous copy has completed.
int batch_publish(fv_batch* b) {
    // Slots reserved by an fv_batch_add still in progress (on another host
    // thread) are not registered yet and stay out of the list.
    int n = 0;
    for (int s = 0; s < b->max_inst; ++s)
        if (b->used[s] && b->registered[s]) n += b->h_inst[s].ntiles;
    if (n > b->work_cap) {
        int cap = b->work_cap;
        while (cap < n) cap *= 2;
        FV_CK(cudaStreamSynchronize(b->stream));  // the old list may still be read by queued kernels
        // The new buffers are allocated before the old ones are released, so a
        // failed allocation leaves the batch with its previous, consistent list
        // (and graphs that still point at it); the next run retries the grow.
        int2* d_new = nullptr;
        int2* h_new[2] = {nullptr, nullptr};
        if (cudaMalloc(reinterpret_cast<void**>(&d_new), (size_t)cap * sizeof(int2)) != cudaSuccess ||
            cudaMallocHost(reinterpret_cast<void**>(&h_new[0]), (size_t)cap * sizeof(int2)) != cudaSuccess ||
            cudaMallocHost(reinterpret_cast<void**>(&h_new[1]), (size_t)cap * sizeof(int2)) != cudaSuccess) {
            if (d_new) cudaFree(d_new);
            for (int k = 0; k < 2; ++k)
                if (h_new[k]) cudaFreeHost(h_new[k]);
            cudaGetLastError();  // an out-of-memory error is not sticky; clear it
            return fail(FV_ERR_NOMEM, "out of memory growing the batch work list to %d tiles", cap);
        }
        cudaFree(b->d_work);
        for (int k = 0; k < 2; ++k) cudaFreeHost(b->h_work[k]);
        b->d_work = d_new;
        b->h_work[0] = h_new[0];
        b->h_work[1] = h_new[1];
        b->bytes += (size_t)(cap - b->work_cap) * sizeof(int2);
        b->work_cap = cap;
        batch_drop_graphs(b);  // the graphs captured the old work-list pointer
    }
    const int k = b->work_buf ^ 1;
    FV_CK(cudaEventSynchronize(b->ev_work[k]));
    int i = 0;
    for (int s = 0; s < b->max_inst; ++s) {
        if (!b->used[s] || !b->registered[s]) continue;
        for (int t = 0; t < b->h_inst[s].ntiles; ++t) b->h_work[k][i++] = make_int2(s, t);
    }
    *b->h_nwork[k] = n;
    if (n > 0)
        FV_CK(cudaMemcpyAsync(b->d_work, b->h_work[k], (size_t)n * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    FV_CK(cudaMemcpyAsync(b->d_nwork, b->h_nwork[k], sizeof(int), cudaMemcpyHostToDevice, b->stream));
    FV_CK(cudaEventRecord(b->ev_work[k], b->stream));
    b->work_buf = k;
    b->nwork = n;
    return FV_OK;
}

int check_batch(fv_batch* b) {
    if (!b) return fail(FV_ERR_INVALID, "null batch");
    FV_CK(cudaSetDevice(b->ctx->device));
    return FV_OK;
}

}  // namespace

extern "C" {

int fv_batch_create(fv_context* ctx, int scheme, const fv_params* params, int max_instances, fv_batch** out) {
    if (!ctx || !params || !out) return fail(FV_ERR_INVALID, "null argument");
    FV_TRY(check_variant(scheme, params));
    if (max_instances < 1 || max_instances > (1 << 20)) return fail(FV_ERR_INVALID, "bad max_instances");
    const int cfg = params->tile < 0 ? 0 : params->tile;
    const BEntry* be = find_batch_entry(scheme, cfg, params->variant);
    if (!be) return fail(FV_ERR_INVALID, "no batched kernel for scheme %d (tile %d)", scheme, cfg);
    FV_CK(cudaSetDevice(ctx->device));
    FV_CK(cudaFuncSetAttribute(reinterpret_cast<const void*>(be->fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)batch_smem(*be)));
    int per_sm = 0;
    FV_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(be->fn), be->NT,
                                                        batch_smem(*be)));
    if (per_sm < 1) return fail(FV_ERR_CUDA, "batched kernel does not fit on an SM");
    fv_batch* b = new fv_batch;
    b->ctx = ctx;
    b->scheme = scheme;
    b->nv = scheme_nv(scheme);
    b->gc = scheme_ghost(scheme);
    // substeps, kernel dt and computeDt factor as for one simulation (fv_sim_create)
    b->num_substeps = (scheme == FV_LXF || scheme == FV_FORCE || scheme == FV_HLL) ? 1
                      : (scheme == FV_KP07)                                   ? (params->order == 1 ? 1 : 2)
                                                                              : 2;
    b->dt_scale = (scheme_split(scheme) && b->num_substeps == 2) ? 0.5f : 1.0f;
    b->factor = (scheme == FV_FORCE) ? 1.0f : (scheme == FV_KP07 && params->order == 1) ? 1.0f : 0.5f;
    b->p = *params;
    b->be = be;
    b->max_inst = max_instances;
    b->resident_grid = per_sm * ctx->sm_count;
    b->used.assign(max_instances, 0);
    b->slot_mem.assign(max_instances, nullptr);
    b->slot_bytes.assign(max_instances, 0);
    auto bail = [&](int rc) {
        fv_batch_destroy(b);
        return rc;
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_up, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_compute, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_work[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_work[1], cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(FV_ERR_CUDA, "stream/event creation failed"));
    b->done_at_sync.assign(max_instances, 0);
    b->registered.assign(max_instances, 0);
    b->work_cap = 4096;
    if (cudaMalloc(&b->d_inst, (size_t)max_instances * sizeof(fv::BatchInstance)) != cudaSuccess ||
        cudaMallocHost(&b->h_inst, (size_t)max_instances * sizeof(fv::BatchInstance)) != cudaSuccess ||
        cudaMalloc(&b->d_ctl, (size_t)max_instances * sizeof(SimCtl)) != cudaSuccess ||
        cudaMallocHost(&b->h_ctl, (size_t)max_instances * sizeof(SimCtl)) != cudaSuccess ||
        cudaMallocHost(&b->h_ctl_up, (size_t)max_instances * sizeof(SimCtl)) != cudaSuccess ||
        cudaMalloc(&b->d_work, (size_t)b->work_cap * sizeof(int2)) != cudaSuccess ||
        cudaMallocHost(&b->h_work[0], (size_t)b->work_cap * sizeof(int2)) != cudaSuccess ||
        cudaMallocHost(&b->h_work[1], (size_t)b->work_cap * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&b->d_nwork, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&b->h_nwork[0], sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&b->h_nwork[1], sizeof(int)) != cudaSuccess || cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess)
        return bail(fail(FV_ERR_NOMEM, "out of memory creating the batch"));
    memset(b->h_inst, 0, (size_t)max_instances * sizeof(fv::BatchInstance));
    memset(b->h_ctl, 0, (size_t)max_instances * sizeof(SimCtl));
    memset(b->h_ctl_up, 0, (size_t)max_instances * sizeof(SimCtl));
    *b->h_nwork[0] = *b->h_nwork[1] = 0;
    if (cudaMemsetAsync(b->d_ctl, 0, (size_t)max_instances * sizeof(SimCtl), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream) != cudaSuccess ||
        cudaMemsetAsync(b->d_nwork, 0, sizeof(int), b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bail(fail(FV_ERR_CUDA, "batch initialisation failed"));
    b->bytes = (size_t)max_instances * (sizeof(fv::BatchInstance) + sizeof(SimCtl)) + b->work_cap * sizeof(int2);
    *out = b;
    return FV_OK;
}

int fv_batch_destroy(fv_batch* b) {
    if (!b) return FV_OK;
    cudaSetDevice(b->ctx->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    for (size_t s = 0; s < b->slot_mem.size(); ++s)
        if (b->slot_mem[s]) cudaFreeAsync(b->slot_mem[s], b->stream);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->d_inst) cudaFree(b->d_inst);
    if (b->h_inst) cudaFreeHost(b->h_inst);
    if (b->d_ctl) cudaFree(b->d_ctl);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->h_ctl_up) cudaFreeHost(b->h_ctl_up);
    if (b->d_work) cudaFree(b->d_work);
    if (b->d_nwork) cudaFree(b->d_nwork);
    for (int k = 0; k < 2; ++k) {
        if (b->h_work[k]) cudaFreeHost(b->h_work[k]);
        if (b->h_nwork[k]) cudaFreeHost(b->h_nwork[k]);
        if (b->ev_work[k]) cudaEventDestroy(b->ev_work[k]);
    }
    if (b->d_err) cudaFree(b->d_err);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->ev_up) cudaEventDestroy(b->ev_up);
    if (b->ev_compute) cudaEventDestroy(b->ev_compute);
    if (b->copy_stream) {
        cudaStreamSynchronize(b->copy_stream);
        cudaStreamDestroy(b->copy_stream);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FV_OK;
}

int fv_batch_add(fv_batch* b, int nx, int ny, float dx, float dy, int bc, const float* const* host_vars,
                 int host_rows, int host_cols, double t_end, int* slot) {
    FV_TRY(check_batch(b));
    if (!host_vars || !slot) return fail(FV_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1 || nx > (1 << 16) || ny > (1 << 16)) return fail(FV_ERR_INVALID, "bad grid %d x %d", nx, ny);
    for (int side = 0; side < 4; ++side)
        if (((bc >> (8 * side)) & 0xF) == fv::BC_NEUMANN)
            return fail(FV_ERR_UNSUPPORTED, "Neumann boundary condition not supported");
    const int gc = b->gc;
    const bool halo = (host_rows == ny + 2 * gc && host_cols == nx + 2 * gc);
    if (!halo && !(host_rows == ny && host_cols == nx)) return fail(FV_ERR_INVALID, "Wrong shape of data");
    for (int v = 0; v < b->nv; ++v)
        if (!host_vars[v]) return fail(FV_ERR_INVALID, "variable %d is null", v);
    int s = -1;
    {
        std::lock_guard<std::mutex> lock(b->mu);
        for (int i = 0; i < b->max_inst; ++i)
            if (!b->used[i]) {
                s = i;
                break;
            }
        if (s < 0) return fail(FV_ERR_NOMEM, "batch is full (%d simulations)", b->max_inst);
        b->used[s] = 1;  // reserved; joins the work list only when registered below
        b->done_at_sync[s] = 0;
    }
    auto release = [&](int rc) {
        std::lock_guard<std::mutex> lock(b->mu);
        b->used[s] = 0;
        return rc;
    };

    const int W = b->be->W, H = b->be->H;
    const int pitch = ((nx + 8) + 31) / 32 * 32;
    const int tiles_x = (nx + W - 1) / W, tiles_y = (ny + H - 1) / H, ntiles = tiles_x * tiles_y;
    const size_t plane = (size_t)(ny + 4) * pitch * sizeof(float);
    const size_t scratch = (size_t)ntiles * (sizeof(float) + 4 * sizeof(double));
    const size_t total = 2 * b->nv * plane + scratch + 256;
    // The new simulation's memory is prepared on the copy stream, concurrently
    // with kernels already queued for the other simulations.
    void* mem = nullptr;
    if (cudaMallocAsync(&mem, total, b->copy_stream) != cudaSuccess) {
        cudaGetLastError();
        return release(fail(FV_ERR_NOMEM, "out of device memory for a %d x %d simulation", nx, ny));
    }
    if (cudaMemsetAsync(mem, 0, total, b->copy_stream) != cudaSuccess) {
        cudaFreeAsync(mem, b->copy_stream);
        return release(fail(FV_ERR_CUDA, "memset failed"));
    }
    fv::BatchInstance& I = b->h_inst[s];
    memset(&I, 0, sizeof(I));
    char* base = static_cast<char*>(mem);
    for (int k = 0; k < 2; ++k)
        for (int v = 0; v < b->nv; ++v) I.buf[k][v] = reinterpret_cast<float*>(base + (size_t)(k * b->nv + v) * plane);
    I.block_cfl = reinterpret_cast<float*>(base + 2 * b->nv * plane);
    I.block_sums = reinterpret_cast<double*>(base + 2 * b->nv * plane + ((ntiles * sizeof(float) + 255) / 256 * 256));
    I.ctl = b->d_ctl + s;
    I.nx = nx;
    I.ny = ny;
    I.pitch = pitch;
    I.bc = bc;
    I.tiles_x = tiles_x;
    I.ntiles = ntiles;
    I.dx = dx;
    I.dy = dy;
    I.g = b->p.g;
    I.gamma = b->p.gamma;
    I.theta = b->p.theta;
    I.dt_scale = b->dt_scale;
    I.variant_beta = b->p.variant_beta;
    const int off = halo ? gc : 0;
    for (int v = 0; v < b->nv; ++v)
        if (copy_h2d(b->ctx, b->copy_stream, I.buf[0][v] + fv::cell_index(-off, -off, pitch), pitch * sizeof(float),
                     host_vars[v], host_cols * sizeof(float), host_cols * sizeof(float), host_rows) != FV_OK) {
            cudaFreeAsync(mem, b->copy_stream);
            return release(FV_ERR_CUDA);
        }
    std::lock_guard<std::mutex> lock(b->mu);
    FV_CK(cudaEventRecord(b->ev_up, b->copy_stream));
    FV_CK(cudaStreamWaitEvent(b->stream, b->ev_up, 0));  // later kernels see the uploaded state
    // The upload's source is h_ctl_up, not h_ctl: an fv_batch_sync on another
    // thread may have queued a copy of every control block into h_ctl ahead of
    // this upload, which would overwrite the new values before they are read.
    SimCtl& c = b->h_ctl_up[s];
    memset(&c, 0, sizeof(c));
    const float c2 = (b->scheme == FV_EE2D_KP07_DIMSPLIT) ? b->p.gamma : b->p.g;
    c.t_end = t_end;
    c.factor = b->factor;
    c.cfl_scale = b->p.cfl_scale;
    c.update_dt = 1;
    // From pinned staging (h_ctl_up, h_inst): asynchronous, ordered before the next kernels.
    FV_CK(cudaMemcpyAsync(b->d_ctl + s, &c, sizeof(SimCtl), cudaMemcpyHostToDevice, b->stream));
    FV_CK(cudaMemcpyAsync(b->d_inst + s, &I, sizeof(fv::BatchInstance), cudaMemcpyHostToDevice, b->stream));
    // cfl_min = the initial CFL estimate, dt = estimate * factor * cfl_scale
    // (simulate() computes dt at step 0), on the device once the upload landed
    FV_TRY(launch_initial_cfl(b->stream, I.buf[0][0] + fv::cell_index(-off, -off, pitch),
                              I.buf[0][1] + fv::cell_index(-off, -off, pitch),
                              I.buf[0][2] + fv::cell_index(-off, -off, pitch), host_rows, host_cols, pitch, dx, dy, c2,
                              reinterpret_cast<float2*>(I.block_sums), ntiles * 4, b->d_ctl + s, true));
    b->slot_mem[s] = mem;
    b->slot_bytes[s] = total;
    b->bytes += total;
    b->registered[s] = 1;
    b->dirty = true;  // joins the work list at the next fv_batch_run
    *slot = s;
    return FV_OK;
}

int fv_batch_remove(fv_batch* b, int slot) {
    FV_TRY(check_batch(b));
    std::lock_guard<std::mutex> lock(b->mu);
    if (slot < 0 || slot >= b->max_inst || !b->used[slot]) return fail(FV_ERR_INVALID, "slot %d is not in use", slot);
    b->used[slot] = 0;
    b->registered[slot] = 0;
    b->dirty = true;  // leaves the work list at the next fv_batch_run
    // Freed in stream order, after every kernel already queued that may read it.
    FV_CK(cudaFreeAsync(b->slot_mem[slot], b->stream));
    b->slot_mem[slot] = nullptr;
    b->bytes -= b->slot_bytes[slot];
    b->slot_bytes[slot] = 0;
    return FV_OK;
}

int fv_batch_run(fv_batch* b, int n_steps) {
    NvtxRange range("fv batch run (graph replays)");
    FV_TRY(check_batch(b));
    if (n_steps < 0) return fail(FV_ERR_INVALID, "negative step count");
    std::lock_guard<std::mutex> lock(b->mu);
    if (b->dirty) {
        FV_TRY(batch_publish(b));
        b->dirty = false;
    }
    FV_TRY(batch_set_graph_grid(b));
    if (!b->graph1 || !b->graph16) {
        batch_drop_graphs(b);
        FV_TRY(batch_build_graph(b, 1, &b->g1, &b->graph1));
        FV_TRY(batch_build_graph(b, 16, &b->g16, &b->graph16));
        b->graph_grid = batch_grid(b);
    }
    FV_CK(cudaEventRecord(b->ev0, b->stream));
    int k = n_steps;
    while (k >= 16) {
        FV_CK(cudaGraphLaunch(b->graph16, b->stream));
        k -= 16;
    }
    while (k > 0) {
        FV_CK(cudaGraphLaunch(b->graph1, b->stream));
        --k;
    }
    FV_CK(cudaEventRecord(b->ev1, b->stream));
    return FV_OK;
}

int fv_batch_sync(fv_batch* b) {
    NvtxRange range("fv batch sync");
    FV_TRY(check_batch(b));
    {
        std::lock_guard<std::mutex> lock(b->mu);
        FV_CK(cudaMemcpyAsync(b->h_ctl, b->d_ctl, (size_t)b->max_inst * sizeof(SimCtl), cudaMemcpyDeviceToHost,
                              b->stream));
    }
    int err = 0;
    FV_CK(cudaStreamSynchronize(b->stream));
    FV_CK(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    std::lock_guard<std::mutex> lock(b->mu);
    for (int s = 0; s < b->max_inst; ++s) {
        if (!b->used[s] || !b->registered[s]) continue;
        b->done_at_sync[s] = batch_done_state(b->h_ctl[s]);
    }
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->last_ms = ms;
    cudaGetLastError();
    if (err) return fail(FV_ERR_DEVICE, "a batched stage kernel gave up waiting for a tile load");
    return FV_OK;
}

int fv_batch_status(fv_batch* b, int slot, double* t, long long* nt, float* dt, int* done) {
    if (!b) return fail(FV_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lock(b->mu);
    if (slot < 0 || slot >= b->max_inst || !b->used[slot]) return fail(FV_ERR_INVALID, "slot not in use");
    const SimCtl& c = b->h_ctl[slot];
    if (t) *t = c.t;
    if (nt) *nt = c.nt;
    if (dt) *dt = c.dt;
    if (done) *done = batch_done_state(c);
    return FV_OK;
}

int fv_batch_download(fv_batch* b, int slot, int var, float* host, int host_pitch) {
    FV_TRY(check_batch(b));
    int nx, ny, pitch, done;
    float* bufs[2];
    {
        std::lock_guard<std::mutex> lock(b->mu);
        if (slot < 0 || slot >= b->max_inst || !b->used[slot] || var < 0 || var >= b->nv || !host)
            return fail(FV_ERR_INVALID, "bad download argument");
        const fv::BatchInstance& I = b->h_inst[slot];
        nx = I.nx;
        ny = I.ny;
        pitch = I.pitch;
        bufs[0] = I.buf[0][var];
        bufs[1] = I.buf[1][var];
        done = b->done_at_sync[slot];
    }
    if (host_pitch < nx) return fail(FV_ERR_INVALID, "host pitch too small");
    SimCtl c;
    if (!done) {
        // still running at the last sync: include every kernel queued since
        FV_CK(cudaStreamSynchronize(b->stream));
        FV_CK(cudaMemcpy(&c, b->d_ctl + slot, sizeof(SimCtl), cudaMemcpyDeviceToHost));
    } else {
        // A simulation that had reached t_end at the last sync is skipped by the
        // kernels queued since, so its state can be read while they run.
        std::lock_guard<std::mutex> lock(b->mu);
        c = b->h_ctl[slot];
    }
    return copy_d2h(b->ctx, b->copy_stream, host, (size_t)host_pitch * sizeof(float),
                    bufs[c.cur] + fv::cell_index(0, 0, pitch), (size_t)pitch * sizeof(float),
                    (size_t)nx * sizeof(float), ny);
}

int fv_batch_info(fv_batch* b, size_t* device_bytes, int* active, int* work_items, double* last_run_ms) {
    if (!b) return fail(FV_ERR_INVALID, "null batch");
    std::lock_guard<std::mutex> lock(b->mu);
    if (device_bytes) *device_bytes = b->bytes;
    if (active) {
        int n = 0;
        for (int s = 0; s < b->max_inst; ++s) n += b->used[s];
        *active = n;
    }
    if (work_items) *work_items = b->nwork;
    if (last_run_ms) *last_run_ms = b->last_ms;
    return FV_OK;
}

int fv_batch_tile(fv_batch* b, int* tile_w, int* tile_h, int* threads, int* grid) {
    if (!b) return fail(FV_ERR_INVALID, "null batch");
    if (tile_w) *tile_w = b->be->W;
    if (tile_h) *tile_h = b->be->H;
    if (threads) *threads = b->be->NT;
    if (grid) {
        std::lock_guard<std::mutex> lock(b->mu);  // nwork changes when the list is republished
        *grid = batch_grid(b);
    }
    return FV_OK;
}

}  // extern "C"
