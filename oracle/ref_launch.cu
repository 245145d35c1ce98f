// Test infrastructure only: a C-ABI launcher around ONE of the reference's
// own stage kernels, selected at compile time by -DREF_SCHEME_<name>.  The
// kernel source is #included unmodified from the reference tree (the include
// path is set by oracle/Makefile); nothing from it is copied here.
//
// The exported ref_substep() makes the launch that each reference class makes
// in its substep() (for example GPUSimulators/KP07_dimsplit.py:112-125), with
// grid = ceil(n / block) (GPUSimulators/Simulator.py:157-161).  Buffers use the
// reference's layout: one dense (ny+2g) x (nx+2g) float32 array per variable,
// row pitch in bytes.

#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>

#if defined(REF_SCHEME_LxF)
#include "SWE2D_LxF.cu"
#elif defined(REF_SCHEME_FORCE)
#include "SWE2D_FORCE.cu"
#elif defined(REF_SCHEME_HLL)
#include "SWE2D_HLL.cu"
#elif defined(REF_SCHEME_HLL2)
#include "SWE2D_HLL2.cu"
#elif defined(REF_SCHEME_WAF)
#include "SWE2D_WAF.cu"
#elif defined(REF_SCHEME_KP07)
#include "SWE2D_KP07.cu"
#elif defined(REF_SCHEME_KP07_dimsplit)
#include "SWE2D_KP07_dimsplit.cu"
#elif defined(REF_SCHEME_EE2D_KP07_dimsplit)
#include "EE2D_KP07_dimsplit.cu"
#else
#error "define REF_SCHEME_<name>"
#endif

static thread_local char g_err[256];

static int check(cudaError_t e) {
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "%s", cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

extern "C" {

const char* ref_last_error(void) { return g_err; }
int ref_block_width(void) { return BLOCK_WIDTH; }
int ref_block_height(void) { return BLOCK_HEIGHT; }

int ref_malloc(void** p, size_t bytes) { return check(cudaMalloc(p, bytes)); }
int ref_free(void* p) { return check(cudaFree(p)); }
int ref_memset(void* p, size_t bytes) { return check(cudaMemset(p, 0, bytes)); }
int ref_h2d(void* dst, const void* src, size_t bytes) { return check(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice)); }
int ref_d2h(void* dst, const void* src, size_t bytes) { return check(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost)); }
int ref_sync(void) { return check(cudaDeviceSynchronize()); }

int ref_event_create(void** ev) { return check(cudaEventCreate((cudaEvent_t*)ev)); }
int ref_event_record(void* ev) { return check(cudaEventRecord((cudaEvent_t)ev, 0)); }
int ref_event_elapsed(void* a, void* b, float* ms) {
    if (check(cudaEventSynchronize((cudaEvent_t)b))) return 1;
    return check(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b));
}
int ref_event_destroy(void* ev) { return check(cudaEventDestroy((cudaEvent_t)ev)); }

// in/out: nv device pointers; pitch in bytes; cfl: device float[grid.x*grid.y] or NULL.
int ref_substep(int nx, int ny, float dx, float dy, float dt, float g, float gamma, float theta, int step,
                int order, int bc, float* const* in, float* const* out, int pitch, float* cfl) {
    (void)cudaGetLastError();  // clear any error left by an earlier, unrelated runtime call
    const dim3 block(BLOCK_WIDTH, BLOCK_HEIGHT);
    const dim3 grid((nx + BLOCK_WIDTH - 1) / BLOCK_WIDTH, (ny + BLOCK_HEIGHT - 1) / BLOCK_HEIGHT);
    (void)gamma;
    (void)theta;
    (void)step;
    (void)order;
#if defined(REF_SCHEME_LxF)
    LxFKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, bc, in[0], pitch, in[1], pitch, in[2], pitch, out[0], pitch,
                               out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_FORCE)
    FORCEKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, bc, in[0], pitch, in[1], pitch, in[2], pitch, out[0], pitch,
                                 out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_HLL)
    HLLKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, bc, in[0], pitch, in[1], pitch, in[2], pitch, out[0], pitch,
                               out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_HLL2)
    HLL2Kernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, theta, step, bc, in[0], pitch, in[1], pitch, in[2], pitch,
                                out[0], pitch, out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_WAF)
    (void)cfl;
    WAFKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, step, bc, in[0], pitch, in[1], pitch, in[2], pitch, out[0],
                               pitch, out[1], pitch, out[2], pitch);
#elif defined(REF_SCHEME_KP07)
    // Simulator.stepOrderToCodedInt: step << 16 | order (GPUSimulators/Simulator.py:280-287)
    KP07Kernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, theta, (step << 16) | (order & 0xFFFF), bc, in[0], pitch,
                                in[1], pitch, in[2], pitch, out[0], pitch, out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_KP07_dimsplit)
    KP07DimsplitKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, theta, step, bc, in[0], pitch, in[1], pitch, in[2],
                                        pitch, out[0], pitch, out[1], pitch, out[2], pitch, cfl);
#elif defined(REF_SCHEME_EE2D_KP07_dimsplit)
    KP07DimsplitKernel<<<grid, block>>>(nx, ny, dx, dy, dt, g, gamma, theta, step, bc, in[0], pitch, in[1], pitch,
                                        in[2], pitch, in[3], pitch, out[0], pitch, out[1], pitch, out[2], pitch,
                                        out[3], pitch, cfl, 0, 0, nx, ny);
#endif
    return check(cudaGetLastError());
}

}  // extern "C"
