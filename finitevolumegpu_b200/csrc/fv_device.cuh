// Device-side building blocks for the finite-volume stage kernels (sm_100a):
// PTX wrappers for mbarrier / TMA, and the per-face physics of the shallow-water
// and Euler schemes.
//
// The physics mirrors the reference formulas (file:line given per function),
// rearranged so that values shared by neighbouring faces are computed once per
// cell: a MUSCL-Hancock cell produces both of its predicted face states from one
// flux difference, and each face state carries its flux, velocity and wave speed.
// Arithmetic is FP32 with fast-math division and square root and flush to
// zero, as the reference compiles its kernels (--use_fast_math,
// GPUSimulators/KP07_dimsplit.py:87).  The library is built with -fmad=false
// and every fused multiply-add is written out with fmaf, so the rounding of
// each formula does not depend on how the compiler inlines it: a cell's result
// is the same whichever tile shape, kernel or batch computes it.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fv {

// ------------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barrier visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Programmatic dependent launch.  A stage kernel launched with programmatic
// stream serialization may start while the previous kernel of its stream is
// finishing: grid_launch_dependents lets the next kernel's CTAs launch into
// SMs this grid frees once all of this grid's CTAs have started, and
// grid_dependency_wait blocks until the previous kernel has completed and its
// memory is visible (a no-op for a launch without the attribute).
__device__ __forceinline__ void grid_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Bounded wait: gives up after `limit` polls (each poll may suspend the thread
// for a short hardware-defined time) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// 2-D tiled TMA load of one box into this CTA's shared memory, completing
// on `bar`.  x must be a multiple of 4 (16-byte rule for FP32).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Orders a tensor map written to global memory by earlier (host-issued) copies
// before its use by this thread's TMA operations.
__device__ __forceinline__ void fence_tmap_acquire(const void* tmap) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(tmap))
                 : "memory");
}

// 16-byte asynchronous copy global -> shared (cached in L2 only) of the first
// `src_bytes` (0..16) bytes at src; the rest of the 16 destination bytes are
// zero-filled.  With src_bytes = 0 nothing is read.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(src_bytes)
                 : "memory");
}

// Waits until this thread's asynchronous copies have landed in shared memory.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// ------------------------------------------------------------------ explicit FP32 operations

// Round-to-nearest FP32 add/sub/mul/fma (flush to zero, as in fast-math code)
// written as PTX, so each one is exactly the operation the formula states:
// the compiler can neither contract nor rewrite them (fast-math code may turn
// x * (1/y) into x / y, for instance, which costs more reciprocals).  Division
// and square root stay C operators (fast-math approximations).
__device__ __forceinline__ float fadd(float a, float b) {
    float d;
    asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fsub(float a, float b) {
    float d;
    asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fmul(float a, float b) {
    float d;
    asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float ffma(float a, float b, float c) {
    float d;
    asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// ------------------------------------------------------------------ two lanes per thread

// Two independent FP32 values, one from each of two lines a thread walks side
// by side.  Add, subtract, multiply and FMA on a pair are one packed
// round-to-nearest instruction (add/sub/mul/fma.rn.ftz.f32x2, sm_100), whose
// lanes round exactly as the scalar instructions above do, so a pair holds the
// same bits as two scalar computations.  Everything else (min/max, division,
// square root, comparisons) runs lane by lane with the scalar operations.
struct __align__(8) f2 {
    float x, y;
};

__device__ __forceinline__ uint64_t& u64(f2& a) { return reinterpret_cast<uint64_t&>(a); }
__device__ __forceinline__ const uint64_t& u64(const f2& a) { return reinterpret_cast<const uint64_t&>(a); }

// The packed multiply is an FMA with a -0.0 addend read from constant memory
// (a*b + -0 is a*b exactly, signed zeros included).  A plain packed multiply
// whose product feeds a packed add or subtract may be fused with it into one
// FMA by the assembler (round-to-nearest modifiers notwithstanding), which
// rounds once instead of twice; measured on a B200, that made two-line walkers
// differ from one-line ones in the last bits.  An FMA result cannot be fused
// further, and the addend's value is not known at compile time, so the
// multiply stays a separate, correctly rounded operation as in the scalar code.
static __constant__ float kOpaqueNegZero = -0.0f;

__device__ __forceinline__ f2 fadd(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(u64(d)) : "l"(u64(a)), "l"(u64(b)));
    return d;
}
__device__ __forceinline__ f2 fsub(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(u64(d)) : "l"(u64(a)), "l"(u64(b)));
    return d;
}
__device__ __forceinline__ f2 ffma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(u64(d)) : "l"(u64(a)), "l"(u64(b)), "l"(u64(c)));
    return d;
}
__device__ __forceinline__ f2 fmul(f2 a, f2 b) { return ffma(a, b, f2{kOpaqueNegZero, kOpaqueNegZero}); }

// A scalar constant in the number type of a computation (both lanes for f2).
template <class N> __device__ __forceinline__ N splat(float a);
template <> __device__ __forceinline__ float splat<float>(float a) { return a; }
template <> __device__ __forceinline__ f2 splat<f2>(float a) { return f2{a, a}; }

// Fast-math division, reciprocal and square root as explicit PTX: the
// approximations the reference's --use_fast_math build uses for x / y,
// 1.0f / x and sqrtf(x), written out so that the compiler cannot rewrite them
// per call site (fast math lets it turn a / b into a * (1 / b) where it
// shares a reciprocal), which would round a cell differently depending on
// the kernel that inlines the formula.
__device__ __forceinline__ float frcp_fast(float a) {
    float d;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(d) : "f"(a));
    return d;
}
// a * (1 / b) with the approximate reciprocal: bit for bit the fast-math
// quotient for divisors below 2^126 (checked on a B200), and two
// instructions, of which the multiply can be packed.
__device__ __forceinline__ float fdiv_fast(float a, float b) { return fmul(a, frcp_fast(b)); }
__device__ __forceinline__ float fsqrt_fast(float a) {
    float d;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(d) : "f"(a));
    return d;
}

// Lane-wise operations, scalar or pair.
__device__ __forceinline__ float vneg(float a) { return -a; }
__device__ __forceinline__ f2 vneg(f2 a) { return f2{-a.x, -a.y}; }
__device__ __forceinline__ float vdiv(float a, float b) { return fdiv_fast(a, b); }
__device__ __forceinline__ f2 vdiv(f2 a, f2 b) { return fmul(a, f2{frcp_fast(b.x), frcp_fast(b.y)}); }
__device__ __forceinline__ float vrcp(float a) { return frcp_fast(a); }
__device__ __forceinline__ f2 vrcp(f2 a) { return f2{frcp_fast(a.x), frcp_fast(a.y)}; }
__device__ __forceinline__ float vsqrt(float a) { return fsqrt_fast(a); }
__device__ __forceinline__ f2 vsqrt(f2 a) { return f2{fsqrt_fast(a.x), fsqrt_fast(a.y)}; }
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ f2 vmin(f2 a, f2 b) { return f2{fminf(a.x, b.x), fminf(a.y, b.y)}; }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ f2 vmax(f2 a, f2 b) { return f2{fmaxf(a.x, b.x), fmaxf(a.y, b.y)}; }

// Three-input minimum (NaN-dropping) and maximum (NaN-propagating): one
// instruction each on sm_100, and exactly min(min(a, b), c) and
// max.NaN(max.NaN(a, b), c).
__device__ __forceinline__ float vmin3(float a, float b, float c) {
    float d;
    asm("min.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float vmax3_nan(float a, float b, float c) {
    float d;
    asm("max.ftz.NaN.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float vmin3_nan(float a, float b, float c) {
    float d;
    asm("min.ftz.NaN.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float vmin_nan(float a, float b) {
    float d;
    asm("min.ftz.NaN.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float vmax3(float a, float b, float c) {
    float d;
    asm("max.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ f2 vmin3(f2 a, f2 b, f2 c) { return f2{vmin3(a.x, b.x, c.x), vmin3(a.y, b.y, c.y)}; }
__device__ __forceinline__ f2 vmax3_nan(f2 a, f2 b, f2 c) {
    return f2{vmax3_nan(a.x, b.x, c.x), vmax3_nan(a.y, b.y, c.y)};
}
__device__ __forceinline__ f2 vmax3(f2 a, f2 b, f2 c) { return f2{vmax3(a.x, b.x, c.x), vmax3(a.y, b.y, c.y)}; }

// Lane-wise selects: a > b ? t : f, and s >= 0 ? t : f, s <= 0 ? t : f.
__device__ __forceinline__ float vsel_gt(float a, float b, float t, float f) { return (a > b) ? t : f; }
__device__ __forceinline__ f2 vsel_gt(f2 a, f2 b, f2 t, f2 f) {
    return f2{(a.x > b.x) ? t.x : f.x, (a.y > b.y) ? t.y : f.y};
}
__device__ __forceinline__ float vsel_ge0(float s, float t, float f) { return (s >= 0.0f) ? t : f; }
__device__ __forceinline__ f2 vsel_ge0(f2 s, f2 t, f2 f) {
    return f2{(s.x >= 0.0f) ? t.x : f.x, (s.y >= 0.0f) ? t.y : f.y};
}
__device__ __forceinline__ float vsel_le0(float s, float t, float f) { return (s <= 0.0f) ? t : f; }
__device__ __forceinline__ f2 vsel_le0(f2 s, f2 t, f2 f) {
    return f2{(s.x <= 0.0f) ? t.x : f.x, (s.y <= 0.0f) ? t.y : f.y};
}

// ------------------------------------------------------------------ limiters

// Generalised minmod slope (GPUSimulators/cuda/limiters.h:31-41).  The
// reference's sign product 0.25*s(b)*(s(b)+s(c))*(s(c)+s(f)) is +-1 when the
// three differences share a sign and 0 otherwise, so the slope is the smallest
// magnitude with b's sign, or zero.
// minmod3 takes the scaled differences b = theta*(center - left),
// c = (right - left)/2 and f = theta*(right - center).
//
// It is computed with min/max only.  With lo and hi the smallest and largest
// of the three: all positive gives lo, all negative gives hi (the one nearest
// zero), and mixed signs give max(lo, min(hi, 0)) = 0.  NaN follows the
// reference's sign test, which reads a NaN's sign bit and drops it from the
// magnitude min: the differences come from FP32 arithmetic, so a NaN among
// them is the canonical positive NaN and acts as +infinity.  hi and the final
// max therefore propagate NaN (max.NaN; it reaches the result only when all
// three are NaN, as the reference's 0.25*...*NaN does), lo drops it (fminf).
// A zero slope may come out as -0 where the sign test gave +0, which changes
// no nonzero value.
__device__ __forceinline__ float fmax_nan(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float vmax_nan(float a, float b) { return fmax_nan(a, b); }
__device__ __forceinline__ f2 vmax_nan(f2 a, f2 b) { return f2{fmax_nan(a.x, b.x), fmax_nan(a.y, b.y)}; }

template <class N>
__device__ __forceinline__ N minmod3(N b, N c, N f) {
    const N lo = vmin3(b, c, f);
    const N hi = vmax3_nan(b, c, f);
    return vmax_nan(lo, vmin(hi, splat<N>(0.0f)));
}

__device__ __forceinline__ float minmod_slope(float left, float center, float right, float theta) {
    return minmod3(fmul(fsub(center, left), theta), fmul(fsub(right, left), 0.5f), fmul(fsub(right, center), theta));
}

// Twice minmod_slope, bit for bit, without the multiply of the central
// difference: theta2 = 2 * theta (scaling by 2 commutes with rounding).
__device__ __forceinline__ float minmod_slope2(float left, float center, float right, float theta2) {
    return minmod3(fmul(fsub(center, left), theta2), fsub(right, left), fmul(fsub(right, center), theta2));
}

// GPUSimulators/cuda/limiters.h:100-102
__device__ __forceinline__ float generalized_minmod(float r, float theta) {
    return fmaxf(0.0f, fminf(theta * r, fminf((1.0f + r) * 0.5f, theta)));
}

// Flux limiters phi(r) of GPUSimulators/cuda/limiters.h:84-118, by id:
// 0 generalized minmod with theta = 1.9 (the one WAF uses, SWECommon.h:199-201),
// 1 minmod, 2 superbee, 3 van Leer, 4 van Albada 1, 5 van Albada 2,
// 6 monotonized central, 7 Osher(beta), 8 Sweby(beta).  van Albada 2 is the
// textbook 2r/(r^2+1); the reference's spelling `r_*r_* + 1.0f` parses as
// r^2 (limiters.h:110), and no reference scheme calls it.
__device__ __forceinline__ float flux_limiter(float r, int id, float beta) {
    switch (id) {
    case 1: return fmaxf(0.0f, fminf(1.0f, r));
    case 2: return fmaxf(0.0f, fmaxf(fminf(2.0f * r, 1.0f), fminf(r, 2.0f)));
    case 3: return (r + fabsf(r)) / (1.0f + fabsf(r));
    case 4: return (r * r + r) / (r * r + 1.0f);
    case 5: return 2.0f * r / (r * r + 1.0f);
    case 6: return fmaxf(0.0f, fminf(2.0f, fminf(2.0f * r, 0.5f * (1.0f + r))));
    case 7: return fmaxf(0.0f, fminf(beta, r));
    case 8: return fmaxf(0.0f, fmaxf(fminf(r, beta), fminf(beta * r, 1.0f)));
    default: return fmaxf(0.0f, fminf(1.9f * r, fminf((1.0f + r) * 0.5f, 1.9f)));
    }
}

// GPUSimulators/cuda/common.h:81-83
__device__ __forceinline__ float desingularize(float x, float eps) {
    return copysignf(fmaxf(fabsf(x), fminf(fadd(fdiv_fast(fmul(x, x), 2.0f * eps), 0.5f * eps), eps)), x);
}

// ------------------------------------------------------------------ shallow water

// A state at a cell face together with its physical flux
// (GPUSimulators/cuda/SWECommon.h:29-37), velocity and gravity-wave speed.
// N is float, or f2 for two lines walked side by side.
template <class N>
struct SweFaceT {
    N q[3];
    N f[3];
    N u, c;
};
using SweFace = SweFaceT<float>;

template <class N>
__device__ __forceinline__ SweFaceT<N> swe_face(N h, N hu, N hv, N g, N half_g) {
    SweFaceT<N> s;
    s.q[0] = h;
    s.q[1] = hu;
    s.q[2] = hv;
    const N rh = vrcp(h);
    s.u = fmul(hu, rh);
    s.f[0] = hu;
    s.f[1] = ffma(hu, s.u, fmul(fmul(half_g, h), h));
    s.f[2] = fmul(hv, s.u);
    s.c = vsqrt(fmul(g, h));
    return s;
}

// Central-upwind flux (GPUSimulators/cuda/SWECommon.h:228-241); m is the left
// (minus) state, p the right (plus) state.
template <class N>
__device__ __forceinline__ void swe_central_upwind(const SweFaceT<N>& m, const SweFaceT<N>& p, N out[3]) {
    const N am = vmin3(fsub(m.u, m.c), fsub(p.u, p.c), splat<N>(0.0f));
    const N ap = vmax3(fadd(m.u, m.c), fadd(p.u, p.c), splat<N>(0.0f));
    const N inv = vrcp(fsub(ap, am));
    const N apam = fmul(ap, am);
    const N nam = vneg(am);
#pragma unroll
    for (int v = 0; v < 3; ++v)
        out[v] = fmul(ffma(apam, fsub(p.q[v], m.q[v]), ffma(ap, m.f[v], fmul(nam, p.f[v]))), inv);
}

// HLL flux (GPUSimulators/cuda/SWECommon.h:274-313).  The three cases (all
// waves to the right, all to the left, the star region) are lane-wise
// selects, so one formula serves scalars and pairs.
template <class N>
__device__ __forceinline__ void swe_hll(const SweFaceT<N>& l, const SweFaceT<N>& r, N out[3]) {
    const N h_l = l.q[0], h_r = r.q[0];
    const N one = splat<N>(1.0f), half = splat<N>(0.5f);
    const N hsum = fadd(h_l, h_r);
    const N h_dag = fsub(fmul(half, hsum), vdiv(fmul(fmul(splat<N>(0.25f), fsub(r.u, l.u)), hsum), fadd(l.c, r.c)));
    const N q_l = vsel_gt(h_dag, h_l, vsqrt(fmul(half, vdiv(fmul(fadd(h_dag, h_l), h_dag), fmul(h_l, h_l)))), one);
    const N q_r = vsel_gt(h_dag, h_r, vsqrt(fmul(half, vdiv(fmul(fadd(h_dag, h_r), h_dag), fmul(h_r, h_r)))), one);
    const N S_l = ffma(vneg(l.c), q_l, l.u);
    const N S_r = ffma(r.c, q_r, r.u);
    const N inv = vrcp(fsub(S_r, S_l));
    const N srsl = fmul(S_r, S_l);
    const N nsl = vneg(S_l);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const N star = fmul(ffma(srsl, fsub(r.q[v], l.q[v]), ffma(S_r, l.f[v], fmul(nsl, r.f[v]))), inv);
        out[v] = vsel_ge0(S_l, l.f[v], vsel_le0(S_r, r.f[v], star));
    }
}

// MUSCL-Hancock reconstruction of one cell for the dimensionally split SWE
// schemes (GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:38-58, SWE2D_HLL2.cu:39-59):
// minmod slope, face values Q -+ slope/2, and the half-step predictor
// Q_face + dt/(2dx) * (F(Q_west) - F(Q_east)), which is the same flux
// difference for both faces of the cell.  w/e: predicted west/east face states.
// bd holds theta2*(q0 - qm) on entry and theta2*(qp - q0) on return: a cell's
// forward difference is the backward difference of the next one, so a line
// walker computes each difference once.
//
// The slope is formed at twice its size: with theta2 = 2*theta, minmod of
// (theta2*b, qp - qm, theta2*f) is exactly 2 * minmod(theta*b, (qp - qm)/2,
// theta*f), since scaling by 2 commutes with rounding, and the face values
// q0 -+ s2/4 equal q0 -+ s/2 bit for bit.  This saves the multiply of the
// central difference.
template <class N>
__device__ __forceinline__ void swe_muscl_hancock(const N (&qm)[3], const N (&q0)[3], const N (&qp)[3], N (&bd)[3],
                                                  N theta2, N g, N half_g, N k2, SweFaceT<N>& w, SweFaceT<N>& e) {
    N W[3], E[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const N f = fmul(fsub(qp[v], q0[v]), theta2);
        const N s2 = minmod3(bd[v], fsub(qp[v], qm[v]), f);
        bd[v] = f;
        W[v] = ffma(splat<N>(-0.25f), s2, q0[v]);
        E[v] = ffma(splat<N>(0.25f), s2, q0[v]);
    }
    const N uw = vdiv(W[1], W[0]);
    const N ue = vdiv(E[1], E[0]);
    N D[3];
    D[0] = fsub(W[1], E[1]);
    D[1] = fsub(ffma(W[1], uw, fmul(fmul(half_g, W[0]), W[0])), ffma(E[1], ue, fmul(fmul(half_g, E[0]), E[0])));
    D[2] = ffma(W[2], uw, fmul(vneg(E[2]), ue));
    w = swe_face(ffma(k2, D[0], W[0]), ffma(k2, D[1], W[1]), ffma(k2, D[2], W[2]), g, half_g);
    e = swe_face(ffma(k2, D[0], E[0]), ffma(k2, D[1], E[1]), ffma(k2, D[2], E[2]), g, half_g);
}

// ------------------------------------------------------------------ Euler

template <class N>
struct EulerFaceT {
    N q[4];
    N f[4];
    N u, c;
};
using EulerFace = EulerFaceT<float>;

// Face state with pressure (GPUSimulators/cuda/EulerCommon.h:83-90), flux
// (EulerCommon.h:93-109) and sound speed sqrt(gamma*P/rho) (EulerCommon.h:130-131, :176).
// gm1 = gamma - 1.
template <class N>
__device__ __forceinline__ EulerFaceT<N> euler_face(N rho, N ru, N rv, N E, N gamma, N gm1) {
    EulerFaceT<N> s;
    s.q[0] = rho;
    s.q[1] = ru;
    s.q[2] = rv;
    s.q[3] = E;
    const N rr = vrcp(rho);
    const N P = fmul(gm1, ffma(fmul(splat<N>(-0.5f), ffma(ru, ru, fmul(rv, rv))), rr, E));
    s.u = fmul(ru, rr);
    s.f[0] = ru;
    s.f[1] = ffma(ru, s.u, P);
    s.f[2] = fmul(rv, s.u);
    s.f[3] = fmul(s.u, fadd(E, P));
    s.c = vsqrt(fmul(fmul(gamma, P), rr));
    return s;
}

// GPUSimulators/cuda/EulerCommon.h:171-187
template <class N>
__device__ __forceinline__ void euler_central_upwind(const EulerFaceT<N>& m, const EulerFaceT<N>& p, N out[4]) {
    const N am = vmin3(fsub(m.u, m.c), fsub(p.u, p.c), splat<N>(0.0f));
    const N ap = vmax3(fadd(m.u, m.c), fadd(p.u, p.c), splat<N>(0.0f));
    const N inv = vrcp(fsub(ap, am));
    const N apam = fmul(ap, am);
    const N nam = vneg(am);
#pragma unroll
    for (int v = 0; v < 4; ++v)
        out[v] = fmul(ffma(apam, fsub(p.q[v], m.q[v]), ffma(ap, m.f[v], fmul(nam, p.f[v]))), inv);
}

// GPUSimulators/cuda/EulerCommon.h:117-160; the cases are lane-wise selects
// as in swe_hll.
template <class N>
__device__ __forceinline__ void euler_hll(const EulerFaceT<N>& l, const EulerFaceT<N>& r, N out[4]) {
    const N h_l = l.q[0], h_r = r.q[0];
    const N one = splat<N>(1.0f), half = splat<N>(0.5f);
    const N hsum = fadd(h_l, h_r);
    const N h_dag = fsub(fmul(half, hsum), vdiv(fmul(fmul(splat<N>(0.25f), fsub(r.u, l.u)), hsum), fadd(l.c, r.c)));
    const N q_l = vsel_gt(h_dag, h_l, vsqrt(fmul(half, vdiv(fmul(fadd(h_dag, h_l), h_dag), fmul(h_l, h_l)))), one);
    const N q_r = vsel_gt(h_dag, h_r, vsqrt(fmul(half, vdiv(fmul(fadd(h_dag, h_r), h_dag), fmul(h_r, h_r)))), one);
    const N S_l = ffma(vneg(l.c), q_l, l.u);
    const N S_r = ffma(r.c, q_r, r.u);
    const N inv = vrcp(fsub(S_r, S_l));
    const N srsl = fmul(S_r, S_l);
    const N nsl = vneg(S_l);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const N star = fmul(ffma(srsl, fsub(r.q[v], l.q[v]), ffma(S_r, l.f[v], fmul(nsl, r.f[v]))), inv);
        out[v] = vsel_ge0(S_l, l.f[v], vsel_le0(S_r, r.f[v], star));
    }
}

// MUSCL-Hancock reconstruction for the Euler kernel
// (GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:33-58 and :78-103).  The reference's
// predictor calls F_func(Q, gamma_), whose second argument is the pressure, so
// the predictor flux uses gamma in place of P; that is reproduced here.
// bd: theta2*(q0 - qm) on entry, theta2*(qp - q0) on return, theta2 = 2*theta,
// and the slope at twice its size (as in swe_muscl_hancock).
template <class N>
__device__ __forceinline__ void euler_muscl_hancock(const N (&qm)[4], const N (&q0)[4], const N (&qp)[4], N (&bd)[4],
                                                    N theta2, N gamma, N gm1, N k2, EulerFaceT<N>& w,
                                                    EulerFaceT<N>& e) {
    N W[4], E[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const N f = fmul(fsub(qp[v], q0[v]), theta2);
        const N s2 = minmod3(bd[v], fsub(qp[v], qm[v]), f);
        bd[v] = f;
        W[v] = ffma(splat<N>(-0.25f), s2, q0[v]);
        E[v] = ffma(splat<N>(0.25f), s2, q0[v]);
    }
    const N uw = vdiv(W[1], W[0]);
    const N ue = vdiv(E[1], E[0]);
    N D[4];
    D[0] = fsub(W[1], E[1]);
    D[1] = fsub(ffma(W[1], uw, gamma), ffma(E[1], ue, gamma));
    D[2] = ffma(W[2], uw, fmul(vneg(E[2]), ue));
    D[3] = ffma(uw, fadd(W[3], gamma), fmul(vneg(ue), fadd(E[3], gamma)));
    w = euler_face(ffma(k2, D[0], W[0]), ffma(k2, D[1], W[1]), ffma(k2, D[2], W[2]), ffma(k2, D[3], W[3]), gamma, gm1);
    e = euler_face(ffma(k2, D[0], E[0]), ffma(k2, D[1], E[1]), ffma(k2, D[2], E[2]), ffma(k2, D[3], E[3]), gamma, gm1);
}

// ------------------------------------------------------------------ WAF

// Per-cell quantities of the WAF flux (GPUSimulators/cuda/SWECommon.h:131-210):
// state, velocities, wave speed and physical flux.  N is float, or f2 for two
// lines walked side by side.
template <class N>
struct WafCellT {
    N q[3];
    N f[3];
    N u, v, c;
};
using WafCell = WafCellT<float>;

template <class N>
__device__ __forceinline__ WafCellT<N> waf_cell(const N q[3], N g, N half_g) {
    WafCellT<N> s;
    s.q[0] = q[0];
    s.q[1] = q[1];
    s.q[2] = q[2];
    const N rh = vrcp(q[0]);
    s.u = fmul(q[1], rh);
    s.v = fmul(q[2], rh);
    s.c = vsqrt(fmul(g, q[0]));
    s.f[0] = q[1];
    s.f[1] = ffma(q[1], s.u, fmul(fmul(half_g, q[0]), q[0]));
    s.f[2] = fmul(q[2], s.u);
    return s;
}

// h in the star region between two cells (GPUSimulators/cuda/SWECommon.h:114-121).
template <class N>
__device__ __forceinline__ N waf_h_star(const WafCellT<N>& l, const WafCellT<N>& r, N inv_g) {
    const N t = fadd(fmul(splat<N>(0.5f), fadd(l.c, r.c)), fmul(splat<N>(0.25f), fsub(l.u, r.u)));
    return fmul(fmul(t, t), inv_g);
}

// The WAF weight of one wave (SWECommon.h:109-111, :199-201): the ratio r of
// upwind to local jumps (both desingularised) through the flux limiter,
// A = sign(c) * (1 - (1 - |c|) * limiter(r)); up: upwind jump for c > 0,
// dn: for c <= 0, loc: the local jump.
__device__ __forceinline__ float waf_weight(float c, float up, float dn, float loc, int limiter, float beta) {
    const float eps = 1.0e-6f;
    const float r = fdiv_fast(desingularize((c > 0.0f) ? up : dn, eps), desingularize(loc, eps));
    return fmul(copysignf(1.0f, c), fsub(1.0f, fmul(fsub(1.0f, fabsf(c)), flux_limiter(r, limiter, beta))));
}
__device__ __forceinline__ f2 waf_weight(f2 c, f2 up, f2 dn, f2 loc, int limiter, float beta) {
    return f2{waf_weight(c.x, up.x, dn.x, loc.x, limiter, beta), waf_weight(c.y, up.y, dn.y, loc.y, limiter, beta)};
}

// WAF flux at the face between l1 and r1 (GPUSimulators/cuda/SWECommon.h:131-210);
// hd_l, hd, hd_r are the star depths of the pairs (l2,l1), (l1,r1), (r1,r2).
template <class N>
__device__ __forceinline__ void waf_flux(const WafCellT<N>& l2, const WafCellT<N>& l1, const WafCellT<N>& r1,
                                         const WafCellT<N>& r2, N hd_l, N hd, N hd_r, N dtdx, N out[3],
                                         int limiter = 0, float beta = 0.0f) {
    const N h_l = l1.q[0], h_r = r1.q[0];
    const N one = splat<N>(1.0f), half = splat<N>(0.5f);
    const N q_l = vsel_gt(hd, h_l, vdiv(vsqrt(fmul(half, fmul(fadd(hd, h_l), hd))), h_l), one);
    const N q_r = vsel_gt(hd, h_r, vdiv(vsqrt(fmul(half, fmul(fadd(hd, h_r), hd))), h_r), one);
    const N S_l = ffma(vneg(l1.c), q_l, l1.u);
    const N S_r = ffma(r1.c, q_r, r1.u);
    const N a_r = fmul(h_r, fsub(r1.u, S_r));
    const N a_l = fmul(h_l, fsub(l1.u, S_l));
    const N S_star = vdiv(fsub(fmul(S_l, a_r), fmul(S_r, a_l)), fsub(a_r, a_l));
    const N sl = vdiv(fmul(h_l, fsub(S_l, l1.u)), fsub(S_l, S_star));
    const N sr = vdiv(fmul(h_r, fsub(S_r, r1.u)), fsub(S_r, S_star));
    const N Qsl[3] = {sl, fmul(sl, S_star), fmul(sl, l1.v)};
    const N Qsr[3] = {sr, fmul(sr, S_star), fmul(sr, r1.v)};
    const N c_1 = fmul(S_l, dtdx);
    const N c_2 = fmul(S_star, dtdx);
    const N c_3 = fmul(S_r, dtdx);
    const N A_1 = waf_weight(c_1, fsub(hd_l, l2.q[0]), fsub(hd_r, h_r), fsub(hd, h_l), limiter, beta);
    const N A_2 = waf_weight(c_2, fsub(l1.v, l2.v), fsub(r2.v, r1.v), fsub(r1.v, l1.v), limiter, beta);
    const N A_3 = waf_weight(c_3, fsub(h_l, hd_l), fsub(r2.q[0], hd_r), fsub(h_r, hd), limiter, beta);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const N F1 = l1.f[v], F4 = r1.f[v];
        const N F2 = ffma(S_l, fsub(Qsl[v], l1.q[v]), F1);
        const N F3 = ffma(S_r, fsub(Qsr[v], r1.q[v]), F4);
        const N wsum = ffma(A_3, fsub(F4, F3), ffma(A_2, fsub(F3, F2), fmul(A_1, fsub(F2, F1))));
        out[v] = ffma(splat<N>(-0.5f), wsum, fmul(half, fadd(F1, F4)));
    }
}

// ------------------------------------------------------------------ first-order fluxes

// HLLC flux (GPUSimulators/cuda/SWECommon.h:334-387): HLL's wave speeds plus
// the contact speed S*, with the star states h (S - u) / (S - S*) (1, S*, v)
// on either side of it.
__device__ __forceinline__ void swe_hllc(const SweFace& l, const SweFace& r, float out[3]) {
    const float h_l = l.q[0], h_r = r.q[0];
    const float hsum = fadd(h_l, h_r);
    const float h_dag = fsub(fmul(0.5f, hsum), fmul(fmul(0.25f, fsub(r.u, l.u)), hsum) / fadd(l.c, r.c));
    const float q_l = (h_dag > h_l) ? sqrtf(fmul(0.5f, fmul(fadd(h_dag, h_l), h_dag) / fmul(h_l, h_l))) : 1.0f;
    const float q_r = (h_dag > h_r) ? sqrtf(fmul(0.5f, fmul(fadd(h_dag, h_r), h_dag) / fmul(h_r, h_r))) : 1.0f;
    const float S_l = ffma(-l.c, q_l, l.u);
    const float S_r = ffma(r.c, q_r, r.u);
    const float a_r = fmul(h_r, fsub(r.u, S_r)), a_l = fmul(h_l, fsub(l.u, S_l));
    const float S_star = fsub(fmul(S_l, a_r), fmul(S_r, a_l)) / fsub(a_r, a_l);
    if (S_l >= 0.0f) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = l.f[v];
    } else if (S_r <= 0.0f) {
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = r.f[v];
    } else if (S_star >= 0.0f) {
        const float k = fmul(h_l, fsub(S_l, l.u)) / fsub(S_l, S_star);
        const float qs[3] = {k, fmul(k, S_star), fmul(k, l.q[2] / h_l)};
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = ffma(S_l, fsub(qs[v], l.q[v]), l.f[v]);
    } else {
        const float k = fmul(h_r, fsub(S_r, r.u)) / fsub(S_r, S_star);
        const float qs[3] = {k, fmul(k, S_star), fmul(k, r.q[2] / h_r)};
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = ffma(S_r, fsub(qs[v], r.q[v]), r.f[v]);
    }
}

// Godunov's centred flux (GPUSimulators/cuda/SWECommon.h:248-255):
// F(0.5 (Ql + Qr) + dt/dx (F(Ql) - F(Qr))); kdx = dt/dx.
__device__ __forceinline__ void swe_godc(const SweFace& l, const SweFace& r, float g, float half_g, float kdx,
                                         float out[3]) {
    float q[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) q[v] = ffma(kdx, fsub(l.f[v], r.f[v]), fmul(0.5f, fadd(l.q[v], r.q[v])));
    const SweFace c = swe_face(q[0], q[1], q[2], g, half_g);
#pragma unroll
    for (int v = 0; v < 3; ++v) out[v] = c.f[v];
}

// FORCE = (LxF + Lax-Wendroff two-step) / 2 (GPUSimulators/cuda/SWECommon.h:404-409,
// :443-450, :466-470).  kx = dx/(2dt), kw = dt/(2dx).
__device__ __forceinline__ void swe_force(const SweFace& l, const SweFace& r, float g, float half_g, float kx,
                                          float kw, float out[3]) {
    float qlw[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) qlw[v] = fmaf(kw, l.f[v] - r.f[v], 0.5f * (l.q[v] + r.q[v]));
    const SweFace w = swe_face(qlw[0], qlw[1], qlw[2], g, half_g);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const float lxf = fmaf(kx, l.q[v] - r.q[v], 0.5f * (l.f[v] + r.f[v]));
        out[v] = 0.5f * (lxf + w.f[v]);
    }
}

// Lax-Friedrichs flux with the 2-D diffusion dx/(4dt) (GPUSimulators/cuda/SWECommon.h:421-427).
__device__ __forceinline__ void swe_lxf_2d(const SweFace& l, const SweFace& r, float k4, float out[3]) {
#pragma unroll
    for (int v = 0; v < 3; ++v) out[v] = fmaf(k4, l.q[v] - r.q[v], 0.5f * (l.f[v] + r.f[v]));
}

// Per-cell CFL time step (GPUSimulators/cuda/SWECommon.h:497-504; EulerCommon.h:42-49
// with sqrt(gamma*rho)).
__device__ __forceinline__ float cell_cfl(float h, float hu, float hv, float dx, float dy, float gg) {
    const float rh = frcp_fast(h);
    const float c = fsqrt_fast(fmul(gg, h));
    const float max_u = fdiv_fast(dx, ffma(fabsf(hu), fabsf(rh), c));
    const float max_v = fdiv_fast(dy, ffma(fabsf(hv), fabsf(rh), c));
    return fminf(max_u, max_v);
}

}  // namespace fv
