// Test infrastructure only: a C-ABI harness around the reference's own flux
// and limiter device functions that none of its schemes calls (HLLC_flux,
// GodC_1D_flux in GPUSimulators/cuda/SWECommon.h:248-255, :334-387; the
// limiters of GPUSimulators/cuda/limiters.h:84-118), plus HLL_flux for
// comparison.  The headers are #included unmodified from the reference tree
// (include path set by oracle/Makefile); nothing from them is copied here.
// Each entry point evaluates one function on n inputs on the GPU.

#include <cuda_runtime.h>
#include <cstdio>

#include "common.h"
#include "limiters.h"
#include "SWECommon.h"

// kind: 0 HLL_flux, 1 HLLC_flux, 2 GodC_1D_flux
__global__ void flux_kernel(int kind, int n, const float* ql, const float* qr, float g, float dx, float dt, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 l = make_float3(ql[3 * i], ql[3 * i + 1], ql[3 * i + 2]);
    const float3 r = make_float3(qr[3 * i], qr[3 * i + 1], qr[3 * i + 2]);
    float3 f;
    if (kind == 1) f = HLLC_flux(l, r, g);
    else if (kind == 2) f = GodC_1D_flux(l, r, g, dx, dt);
    else f = HLL_flux(l, r, g);
    out[3 * i] = f.x;
    out[3 * i + 1] = f.y;
    out[3 * i + 2] = f.z;
}

// id: 0 generalized_minmod(r, beta), 1 minmod, 2 superbee, 3 vanLeer, 4 vanAlbada1,
// 5 vanAlbada2, 6 monotonized_central, 7 osher(r, beta), 8 sweby(r, beta)
__global__ void limiter_kernel(int id, int n, const float* r, float beta, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = r[i];
    float y;
    switch (id) {
    case 1: y = minmod(x); break;
    case 2: y = superbee(x); break;
    case 3: y = vanLeer(x); break;
    case 4: y = vanAlbada1(x); break;
    case 5: y = vanAlbada2(x); break;
    case 6: y = monotonized_central(x); break;
    case 7: y = osher(x, beta); break;
    case 8: y = sweby(x, beta); break;
    default: y = generalized_minmod(x, beta); break;
    }
    out[i] = y;
}

static int run(const void* h_in0, const void* h_in1, size_t in_bytes, void* h_out, size_t out_bytes, int n,
               int which, int kind, float a, float b, float c) {
    float *d0 = nullptr, *d1 = nullptr, *d2 = nullptr;
    if (cudaMalloc(&d0, in_bytes) || cudaMalloc(&d1, in_bytes ? in_bytes : 4) || cudaMalloc(&d2, out_bytes)) return 1;
    cudaMemcpy(d0, h_in0, in_bytes, cudaMemcpyHostToDevice);
    if (h_in1) cudaMemcpy(d1, h_in1, in_bytes, cudaMemcpyHostToDevice);
    const int blocks = (n + 127) / 128;
    if (which == 0) flux_kernel<<<blocks, 128>>>(kind, n, d0, d1, a, b, c, d2);
    else limiter_kernel<<<blocks, 128>>>(kind, n, d0, a, d2);
    int rc = cudaDeviceSynchronize() != cudaSuccess;
    cudaMemcpy(h_out, d2, out_bytes, cudaMemcpyDeviceToHost);
    cudaFree(d0);
    cudaFree(d1);
    cudaFree(d2);
    return rc;
}

extern "C" {
int ref_flux_eval(int kind, int n, const float* ql, const float* qr, float g, float dx, float dt, float* out) {
    return run(ql, qr, (size_t)n * 3 * sizeof(float), out, (size_t)n * 3 * sizeof(float), n, 0, kind, g, dx, dt);
}
int ref_limiter_eval(int id, int n, const float* r, float beta, float* out) {
    return run(r, nullptr, (size_t)n * sizeof(float), out, (size_t)n * sizeof(float), n, 1, id, beta, 0.0f, 0.0f);
}
}
