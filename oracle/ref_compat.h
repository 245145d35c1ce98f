// Test infrastructure only: force-included ahead of each reference kernel
// source when oracle/Makefile builds oracle/_ref/.
//
// The reference's readBlock/writeBlock gained a sub-rectangle (x0, y0, x1, y1)
// for its MPI path (GPUSimulators/cuda/common.h:321-326, :360-365), but the SWE
// kernels still call the older 6- and 7-argument forms (for example
// GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:157-159, :197-199), so they do not
// compile as shipped.  These two overloads forward to the full domain
// (x0 = y0 = 0, x1 = nx, y1 = ny), for which the clamps in common.h:336, :342
// and :372-373 reduce to the whole-grid behaviour the SWE kernels were written
// for.
//
// common.h also carries an uninstantiated template, reduce_max
// (GPUSimulators/cuda/common.h:499-547), that names FLT_MIN and an undeclared
// object dt_ctx; the declarations below only let that dead code parse.  No
// kernel uses either.
#pragma once
#include <cfloat>

struct RefCompatDtCtx {
    float L[1];
};
static __device__ RefCompatDtCtx dt_ctx;

#include "common.h"

template <int w, int h, int gc_x, int gc_y, int sign_x, int sign_y>
inline __device__ void readBlock(float* ptr_, int pitch_, float Q[h + 2 * gc_y][w + 2 * gc_x], const int nx_,
                                 const int ny_, const int boundary_conditions_) {
    readBlock<w, h, gc_x, gc_y, sign_x, sign_y>(ptr_, pitch_, Q, nx_, ny_, boundary_conditions_, 0, 0, nx_, ny_);
}

template <int w, int h, int gc_x, int gc_y>
inline __device__ void writeBlock(float* ptr_, int pitch_, float shmem[h + 2 * gc_y][w + 2 * gc_x], const int nx_,
                                  const int ny_, int rk_step_, int rk_order_) {
    writeBlock<w, h, gc_x, gc_y>(ptr_, pitch_, shmem, nx_, ny_, rk_step_, rk_order_, 0, 0, nx_, ny_);
}
