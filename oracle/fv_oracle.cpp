// CPU oracle for the GPUSimulators time-step path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the CPU and in plain IEEE arithmetic, what one
// substep of each GPUSimulators scheme computes.  It exists so that tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg can check and time
// the CUDA product path; nothing in finitevolumegpu_b200/ links or calls it.
//
// Form: each scheme is written as a global operator on the whole grid
// (interior plus ghost cells), not as the reference's 16x16 shared-memory
// blocks.  The block kernels compute exactly this operator (the halo rows of a
// dimensionally split block are swept along x exactly like the ghost rows of
// the full grid), with one exception that is a reference defect: when
// nx % block_width == 1 (or ny % block_height == 1) the reference's reflective
// east (north) ghost fill for a 2-cell halo writes past its shared-memory row
// (GPUSimulators/cuda/common.h:168-171, :223-226).  The oracle implements the
// intended reflective fill.
//
// Every helper cites the reference line range it restates (paths relative to
// the reference project root).  Arithmetic order follows the reference source
// expression by expression; the library is built with -ffp-contract=off so
// that the FP32 variant is plain round-to-nearest IEEE single precision.
//
// Both FP32 and FP64 variants are exported; the FP64 one evaluates the same
// formulas in double precision (single-precision literals such as 0.5f become
// the same decimal constant in double).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Scheme {
    LXF = 0, FORCE = 1, HLL = 2, HLL2 = 3, WAF = 4, KP07 = 5, KP07_DIMSPLIT = 6, EE2D_KP07_DIMSPLIT = 7
};

// GPUSimulators/cuda/common.h:109-114
enum BC { DIRICHLET = 0, NEUMANN = 1, PERIODIC = 2, REFLECTIVE = 3 };

// GPUSimulators/cuda/common.h:116-130 (N<<24 | S<<16 | E<<8 | W)
inline int bc_north(int bc) { return (bc >> 24) & 0xF; }
inline int bc_south(int bc) { return (bc >> 16) & 0xF; }
inline int bc_east(int bc)  { return (bc >> 8) & 0xF; }
inline int bc_west(int bc)  { return bc & 0xF; }

int ghost_cells(int scheme) {
    return (scheme == LXF || scheme == FORCE || scheme == HLL) ? 1 : 2;
}
int num_vars(int scheme) { return scheme == EE2D_KP07_DIMSPLIT ? 4 : 3; }

// Math helpers.  Unqualified so that the operation-counting type below can
// supply its own overloads.
template <typename T> inline T sqrt_(T x) { return std::sqrt(x); }
template <typename T> inline T fabs_(T x) { return std::fabs(x); }
template <typename T> inline T copysign_(T a, T b) { return std::copysign(a, b); }
template <typename T> inline T fmin_(T a, T b) { return std::fmin(a, b); }
template <typename T> inline T fmax_(T a, T b) { return std::fmax(a, b); }
template <typename T> inline T sgn1(T x) { return copysign_(T(1), x); }

// ---------------------------------------------------------------- operation counting
// A double that counts the floating-point operations applied to it, used to
// measure the algorithmic cost of one substep of each scheme as the reference
// formulates it (run single-threaded).  Sign manipulation (fabs, copysign) and
// comparisons are not counted.
struct OpCounts {
    long long add, sub, mul, div, sqrt, minmax;
};
OpCounts g_ops;

struct Counted {
    double v;
    Counted() : v(0.0) {}
    Counted(double x) : v(x) {}
    explicit operator double() const { return v; }
    Counted operator-() const { return Counted(-v); }
};
inline Counted operator+(Counted a, Counted b) { ++g_ops.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_ops.sub; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_ops.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_ops.div; return Counted(a.v / b.v); }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
template <> inline Counted sqrt_(Counted x) { ++g_ops.sqrt; return Counted(std::sqrt(x.v)); }
template <> inline Counted fabs_(Counted x) { return Counted(std::fabs(x.v)); }
template <> inline Counted copysign_(Counted a, Counted b) { return Counted(std::copysign(a.v, b.v)); }
template <> inline Counted fmin_(Counted a, Counted b) { ++g_ops.minmax; return Counted(std::fmin(a.v, b.v)); }
template <> inline Counted fmax_(Counted a, Counted b) { ++g_ops.minmax; return Counted(std::fmax(a.v, b.v)); }

template <typename T, int N> struct Vec {
    T c[N];
};

// ---------------------------------------------------------------- limiters
// GPUSimulators/cuda/limiters.h:31-41
template <typename T>
inline T minmod_slope(T left, T center, T right, T theta) {
    const T backward = (center - left) * theta;
    const T central = (right - left) * T(0.5);
    const T forward = (right - center) * theta;
    return T(0.25) * sgn1(backward) * (sgn1(backward) + sgn1(central)) *
           (sgn1(central) + sgn1(forward)) *
           fmin_(fmin_(fabs_(backward), fabs_(central)), fabs_(forward));
}

// GPUSimulators/cuda/limiters.h:100-102
template <typename T> inline T generalized_minmod(T r, T theta) {
    return fmax_(T(0), fmin_(theta * r, fmin_((T(1) + r) / T(2), theta)));
}

// Flux limiters of GPUSimulators/cuda/limiters.h:84-118, by id: 0 generalized
// minmod with theta 1.9 (WAF's, SWECommon.h:199-201), 1 minmod, 2 superbee,
// 3 van Leer, 4 van Albada 1, 5 van Albada 2 (2r/(r^2+1): the reference's
// `r_*r_* + 1.0f` parses as r^2, limiters.h:110), 6 monotonized central,
// 7 Osher(beta), 8 Sweby(beta).
template <typename T> inline T flux_limiter(T r, int id, T beta) {
    switch (id) {
    case 1: return fmax_(T(0), fmin_(T(1), r));                                            // limiters.h:96-98
    case 2: return fmax_(T(0), fmax_(fmin_(T(2) * r, T(1)), fmin_(r, T(2))));              // :104-106
    case 3: return (r + fabs_(r)) / (T(1) + fabs_(r));                                     // :116-118
    case 4: return (r * r + r) / (r * r + T(1));                                           // :108-110
    case 5: return T(2) * r / (r * r + T(1));                                              // :112-114
    case 6: return fmax_(T(0), fmin_(T(2), fmin_(T(2) * r, T(0.5) * (T(1) + r))));          // :84-86
    case 7: return fmax_(T(0), fmin_(beta, r));                                            // :88-90
    case 8: return fmax_(T(0), fmax_(fmin_(r, beta), fmin_(beta * r, T(1))));               // :92-94
    default: return generalized_minmod(r, T(1.9));
    }
}

// GPUSimulators/cuda/common.h:81-83
template <typename T> inline T desingularize(T x, T eps) {
    return sgn1(x) * fmax_(fabs_(x), fmin_(x * x / (T(2) * eps) + T(0.5) * eps, eps));
}

// ---------------------------------------------------------------- shallow water
// GPUSimulators/cuda/SWECommon.h:29-37
template <typename T> inline Vec<T, 3> swe_F(const Vec<T, 3>& Q, T g) {
    Vec<T, 3> F;
    F.c[0] = Q.c[1];
    F.c[1] = Q.c[1] * Q.c[1] / Q.c[0] + T(0.5) * g * Q.c[0] * Q.c[0];
    F.c[2] = Q.c[1] * Q.c[2] / Q.c[0];
    return F;
}

// GPUSimulators/cuda/SWECommon.h:228-241
template <typename T> inline Vec<T, 3> swe_central_upwind(const Vec<T, 3>& Qm, const Vec<T, 3>& Qp, T g) {
    const Vec<T, 3> Fp = swe_F(Qp, g);
    const T up = Qp.c[1] / Qp.c[0];
    const T cp = sqrt_(g * Qp.c[0]);
    const Vec<T, 3> Fm = swe_F(Qm, g);
    const T um = Qm.c[1] / Qm.c[0];
    const T cm = sqrt_(g * Qm.c[0]);
    const T am = fmin_(fmin_(um - cm, up - cp), T(0));
    const T ap = fmax_(fmax_(um + cm, up + cp), T(0));
    const T apam = ap * am;
    const T den = ap - am;
    Vec<T, 3> r;
    for (int v = 0; v < 3; ++v) r.c[v] = ((ap * Fm.c[v] - am * Fp.c[v]) + apam * (Qp.c[v] - Qm.c[v])) / den;
    return r;
}

// GPUSimulators/cuda/SWECommon.h:274-313
template <typename T> inline Vec<T, 3> swe_hll(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g) {
    const T h_l = Ql.c[0];
    const T h_r = Qr.c[0];
    const T u_l = Ql.c[1] / h_l;
    const T u_r = Qr.c[1] / h_r;
    const T c_l = sqrt_(g * h_l);
    const T c_r = sqrt_(g * h_r);
    const T h_dag = T(0.5) * (h_l + h_r) - T(0.25) * (u_r - u_l) * (h_l + h_r) / (c_l + c_r);
    const T q_l_tmp = sqrt_(T(0.5) * ((h_dag + h_l) * h_dag / (h_l * h_l)));
    const T q_r_tmp = sqrt_(T(0.5) * ((h_dag + h_r) * h_dag / (h_r * h_r)));
    const T q_l = (h_dag > h_l) ? q_l_tmp : T(1);
    const T q_r = (h_dag > h_r) ? q_r_tmp : T(1);
    const T S_l = u_l - c_l * q_l;
    const T S_r = u_r + c_r * q_r;
    if (S_l >= T(0)) return swe_F(Ql, g);
    if (S_r <= T(0)) return swe_F(Qr, g);
    const Vec<T, 3> F_l = swe_F(Ql, g);
    const Vec<T, 3> F_r = swe_F(Qr, g);
    const T srsl = S_r * S_l;
    const T den = S_r - S_l;
    Vec<T, 3> f;
    for (int v = 0; v < 3; ++v) f.c[v] = ((S_r * F_l.c[v] - S_l * F_r.c[v]) + srsl * (Qr.c[v] - Ql.c[v])) / den;
    return f;
}

// GPUSimulators/cuda/SWECommon.h:334-387
template <typename T> inline Vec<T, 3> swe_hllc(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g) {
    const T h_l = Ql.c[0];
    const T h_r = Qr.c[0];
    const T u_l = Ql.c[1] / h_l;
    const T u_r = Qr.c[1] / h_r;
    const T c_l = sqrt_(g * h_l);
    const T c_r = sqrt_(g * h_r);
    const T h_dag = T(0.5) * (h_l + h_r) - T(0.25) * (u_r - u_l) * (h_l + h_r) / (c_l + c_r);
    const T q_l_tmp = sqrt_(T(0.5) * ((h_dag + h_l) * h_dag / (h_l * h_l)));
    const T q_r_tmp = sqrt_(T(0.5) * ((h_dag + h_r) * h_dag / (h_r * h_r)));
    const T q_l = (h_dag > h_l) ? q_l_tmp : T(1);
    const T q_r = (h_dag > h_r) ? q_r_tmp : T(1);
    const T S_l = u_l - c_l * q_l;
    const T S_r = u_r + c_r * q_r;
    const T S_star = (S_l * h_r * (u_r - S_r) - S_r * h_l * (u_l - S_l)) / (h_r * (u_r - S_r) - h_l * (u_l - S_l));
    const Vec<T, 3> F_l = swe_F(Ql, g);
    const Vec<T, 3> F_r = swe_F(Qr, g);
    if (S_l >= T(0)) return F_l;
    if (S_r <= T(0)) return F_r;
    Vec<T, 3> f;
    if (S_l <= T(0) && T(0) <= S_star) {
        const T v_l = Ql.c[2] / h_l;
        const T k = h_l * (S_l - u_l) / (S_l - S_star);
        const T qs[3] = {k * T(1), k * S_star, k * v_l};
        for (int v = 0; v < 3; ++v) f.c[v] = F_l.c[v] + S_l * (qs[v] - Ql.c[v]);
        return f;
    }
    const T v_r = Qr.c[2] / h_r;
    const T k = h_r * (S_r - u_r) / (S_r - S_star);
    const T qs[3] = {k * T(1), k * S_star, k * v_r};
    for (int v = 0; v < 3; ++v) f.c[v] = F_r.c[v] + S_r * (qs[v] - Qr.c[v]);
    return f;
}

// GPUSimulators/cuda/SWECommon.h:248-255
template <typename T> inline Vec<T, 3> swe_godc_1d(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g, T dx, T dt) {
    const Vec<T, 3> F_l = swe_F(Ql, g), F_r = swe_F(Qr, g);
    Vec<T, 3> q;
    for (int v = 0; v < 3; ++v) q.c[v] = T(0.5) * (Ql.c[v] + Qr.c[v]) + (dt / dx) * (F_l.c[v] - F_r.c[v]);
    return swe_F(q, g);
}

// GPUSimulators/cuda/SWECommon.h:109-111
template <typename T> inline T limiter_to_waf_limiter(T r, T c) { return T(1) - (T(1) - fabs_(c)) * r; }

// GPUSimulators/cuda/SWECommon.h:114-121
template <typename T> inline T compute_h_star(T h_l, T h_r, T u_l, T u_r, T c_l, T c_r, T g) {
    (void)h_l;
    (void)h_r;
    const T h_tmp = T(0.5) * (c_l + c_r) + T(0.25) * (u_l - u_r);
    return h_tmp * h_tmp / g;
}

// GPUSimulators/cuda/SWECommon.h:131-210 (interface i+1/2 from Q_{i-1}, Q_i, Q_{i+1}, Q_{i+2})
template <typename T>
inline Vec<T, 3> swe_waf(const Vec<T, 3>& Ql2, const Vec<T, 3>& Ql1, const Vec<T, 3>& Qr1, const Vec<T, 3>& Qr2,
                         T g, T dx, T dt, int limiter = 0, T beta = T(0)) {
    const T h_l = Ql1.c[0], h_r = Qr1.c[0];
    const T h_l2 = Ql2.c[0], h_r2 = Qr2.c[0];
    const T u_l = Ql1.c[1] / h_l, u_r = Qr1.c[1] / h_r;
    const T u_l2 = Ql2.c[1] / h_l2, u_r2 = Qr2.c[1] / h_r2;
    const T v_l = Ql1.c[2] / h_l, v_r = Qr1.c[2] / h_r;
    const T v_l2 = Ql2.c[2] / h_l2, v_r2 = Qr2.c[2] / h_r2;
    const T c_l = sqrt_(g * h_l), c_r = sqrt_(g * h_r);
    const T c_l2 = sqrt_(g * h_l2), c_r2 = sqrt_(g * h_r2);
    const T h_dag_l = compute_h_star(h_l2, h_l, u_l2, u_l, c_l2, c_l, g);
    const T h_dag = compute_h_star(h_l, h_r, u_l, u_r, c_l, c_r, g);
    const T h_dag_r = compute_h_star(h_r, h_r2, u_r, u_r2, c_r, c_r2, g);
    const T q_l_tmp = sqrt_(T(0.5) * ((h_dag + h_l) * h_dag)) / h_l;
    const T q_r_tmp = sqrt_(T(0.5) * ((h_dag + h_r) * h_dag)) / h_r;
    const T q_l = (h_dag > h_l) ? q_l_tmp : T(1);
    const T q_r = (h_dag > h_r) ? q_r_tmp : T(1);
    const T S_l = u_l - c_l * q_l;
    const T S_r = u_r + c_r * q_r;
    const T S_star = (S_l * h_r * (u_r - S_r) - S_r * h_l * (u_l - S_l)) / (h_r * (u_r - S_r) - h_l * (u_l - S_l));
    const T sl = h_l * (S_l - u_l) / (S_l - S_star);
    const T sr = h_r * (S_r - u_r) / (S_r - S_star);
    const Vec<T, 3> Qsl = {{sl * T(1), sl * S_star, sl * v_l}};
    const Vec<T, 3> Qsr = {{sr * T(1), sr * S_star, sr * v_r}};
    const Vec<T, 3> F_1 = swe_F(Ql1, g);
    const Vec<T, 3> F_4 = swe_F(Qr1, g);
    Vec<T, 3> F_2, F_3;
    for (int v = 0; v < 3; ++v) {
        F_2.c[v] = F_1.c[v] + S_l * (Qsl.c[v] - Ql1.c[v]);
        F_3.c[v] = F_4.c[v] + S_r * (Qsr.c[v] - Qr1.c[v]);
    }
    const T c_1 = S_l * dt / dx;
    const T c_2 = S_star * dt / dx;
    const T c_3 = S_r * dt / dx;
    const T eps = T(1.0e-6);
    const T r_1 = desingularize((c_1 > T(0)) ? (h_dag_l - h_l2) : (h_dag_r - h_r), eps) / desingularize(h_dag - h_l, eps);
    const T r_2 = desingularize((c_2 > T(0)) ? (v_l - v_l2) : (v_r2 - v_r), eps) / desingularize(v_r - v_l, eps);
    const T r_3 = desingularize((c_3 > T(0)) ? (h_l - h_dag_l) : (h_r2 - h_dag_r), eps) / desingularize(h_r - h_dag, eps);
    const T A_1 = sgn1(c_1) * limiter_to_waf_limiter(flux_limiter(r_1, limiter, beta), c_1);
    const T A_2 = sgn1(c_2) * limiter_to_waf_limiter(flux_limiter(r_2, limiter, beta), c_2);
    const T A_3 = sgn1(c_3) * limiter_to_waf_limiter(flux_limiter(r_3, limiter, beta), c_3);
    Vec<T, 3> f;
    for (int v = 0; v < 3; ++v)
        f.c[v] = T(0.5) * (F_1.c[v] + F_4.c[v]) -
                 T(0.5) * (A_1 * (F_2.c[v] - F_1.c[v]) + A_2 * (F_3.c[v] - F_2.c[v]) + A_3 * (F_4.c[v] - F_3.c[v]));
    return f;
}

// GPUSimulators/cuda/SWECommon.h:404-409
template <typename T> inline Vec<T, 3> swe_lxf_1d(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g, T dx, T dt) {
    const Vec<T, 3> F_l = swe_F(Ql, g), F_r = swe_F(Qr, g);
    const T k = dx / (T(2) * dt);
    Vec<T, 3> f;
    for (int v = 0; v < 3; ++v) f.c[v] = T(0.5) * (F_l.c[v] + F_r.c[v]) + k * (Ql.c[v] - Qr.c[v]);
    return f;
}

// GPUSimulators/cuda/SWECommon.h:421-427
template <typename T> inline Vec<T, 3> swe_lxf_2d(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g, T dx, T dt) {
    const Vec<T, 3> F_l = swe_F(Ql, g), F_r = swe_F(Qr, g);
    const T k = dx / (T(4) * dt);
    Vec<T, 3> f;
    for (int v = 0; v < 3; ++v) f.c[v] = T(0.5) * (F_l.c[v] + F_r.c[v]) + k * (Ql.c[v] - Qr.c[v]);
    return f;
}

// GPUSimulators/cuda/SWECommon.h:443-450
template <typename T> inline Vec<T, 3> swe_lxw2_1d(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g, T dx, T dt) {
    const Vec<T, 3> F_l = swe_F(Ql, g), F_r = swe_F(Qr, g);
    const T k = dt / (T(2) * dx);
    Vec<T, 3> Q;
    for (int v = 0; v < 3; ++v) Q.c[v] = T(0.5) * (Ql.c[v] + Qr.c[v]) + k * (F_l.c[v] - F_r.c[v]);
    return swe_F(Q, g);
}

// GPUSimulators/cuda/SWECommon.h:466-470
template <typename T> inline Vec<T, 3> swe_force_1d(const Vec<T, 3>& Ql, const Vec<T, 3>& Qr, T g, T dx, T dt) {
    const Vec<T, 3> a = swe_lxf_1d(Ql, Qr, g, dx, dt);
    const Vec<T, 3> b = swe_lxw2_1d(Ql, Qr, g, dx, dt);
    Vec<T, 3> f;
    for (int v = 0; v < 3; ++v) f.c[v] = T(0.5) * (a.c[v] + b.c[v]);
    return f;
}

// ---------------------------------------------------------------- Euler
// GPUSimulators/cuda/EulerCommon.h:83-90
template <typename T> inline T euler_pressure(const Vec<T, 4>& Q, T gamma) {
    return (gamma - T(1)) * (Q.c[3] - T(0.5) * (Q.c[1] * Q.c[1] + Q.c[2] * Q.c[2]) / Q.c[0]);
}

// GPUSimulators/cuda/EulerCommon.h:93-109
template <typename T> inline Vec<T, 4> euler_F(const Vec<T, 4>& Q, T P) {
    const T u = Q.c[1] / Q.c[0];
    Vec<T, 4> F;
    F.c[0] = Q.c[1];
    F.c[1] = Q.c[1] * u + P;
    F.c[2] = Q.c[2] * u;
    F.c[3] = u * (Q.c[3] + P);
    return F;
}

// GPUSimulators/cuda/EulerCommon.h:117-160
template <typename T> inline Vec<T, 4> euler_hll(const Vec<T, 4>& Ql, const Vec<T, 4>& Qr, T gamma) {
    const T h_l = Ql.c[0], h_r = Qr.c[0];
    const T u_l = Ql.c[1] / h_l, u_r = Qr.c[1] / h_r;
    const T P_l = euler_pressure(Ql, gamma), P_r = euler_pressure(Qr, gamma);
    const T c_l = sqrt_(gamma * P_l / Ql.c[0]);
    const T c_r = sqrt_(gamma * P_r / Qr.c[0]);
    const T h_dag = T(0.5) * (h_l + h_r) - T(0.25) * (u_r - u_l) * (h_l + h_r) / (c_l + c_r);
    const T q_l_tmp = sqrt_(T(0.5) * ((h_dag + h_l) * h_dag / (h_l * h_l)));
    const T q_r_tmp = sqrt_(T(0.5) * ((h_dag + h_r) * h_dag / (h_r * h_r)));
    const T q_l = (h_dag > h_l) ? q_l_tmp : T(1);
    const T q_r = (h_dag > h_r) ? q_r_tmp : T(1);
    const T S_l = u_l - c_l * q_l;
    const T S_r = u_r + c_r * q_r;
    if (S_l >= T(0)) return euler_F(Ql, P_l);
    if (S_r <= T(0)) return euler_F(Qr, P_r);
    const Vec<T, 4> F_l = euler_F(Ql, P_l), F_r = euler_F(Qr, P_r);
    const T srsl = S_r * S_l;
    const T den = S_r - S_l;
    Vec<T, 4> f;
    for (int v = 0; v < 4; ++v) f.c[v] = ((S_r * F_l.c[v] - S_l * F_r.c[v]) + srsl * (Qr.c[v] - Ql.c[v])) / den;
    return f;
}

// GPUSimulators/cuda/EulerCommon.h:171-187
template <typename T> inline Vec<T, 4> euler_central_upwind(const Vec<T, 4>& Qm, const Vec<T, 4>& Qp, T gamma) {
    const T Pp = euler_pressure(Qp, gamma);
    const Vec<T, 4> Fp = euler_F(Qp, Pp);
    const T up = Qp.c[1] / Qp.c[0];
    const T cp = sqrt_(gamma * Pp / Qp.c[0]);
    const T Pm = euler_pressure(Qm, gamma);
    const Vec<T, 4> Fm = euler_F(Qm, Pm);
    const T um = Qm.c[1] / Qm.c[0];
    const T cm = sqrt_(gamma * Pm / Qm.c[0]);
    const T am = fmin_(fmin_(um - cm, up - cp), T(0));
    const T ap = fmax_(fmax_(um + cm, up + cp), T(0));
    const T apam = ap * am;
    const T den = ap - am;
    Vec<T, 4> r;
    for (int v = 0; v < 4; ++v) r.c[v] = ((ap * Fm.c[v] - am * Fp.c[v]) + apam * (Qp.c[v] - Qm.c[v])) / den;
    return r;
}

// ---------------------------------------------------------------- grid helpers
// Extended working copy of one substep's input: (ny+2g) x (nx+2g) per variable.
template <typename T> struct Grid {
    int nx, ny, g, nv, w, h;
    std::vector<T> d[4];
    Grid(int nx_, int ny_, int g_, int nv_) : nx(nx_), ny(ny_), g(g_), nv(nv_), w(nx_ + 2 * g_), h(ny_ + 2 * g_) {
        for (int v = 0; v < nv; ++v) d[v].assign((size_t)w * h, T(0));
    }
    T& at(int v, int l, int k) { return d[v][(size_t)l * w + k]; }
    T at(int v, int l, int k) const { return d[v][(size_t)l * w + k]; }
};

// Per-variable reflective signs (sign_x, sign_y): h/rho and E keep their sign,
// the normal momentum flips (GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:157-159,
// GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:174-177).
inline int sign_x(int v) { return v == 1 ? -1 : 1; }
inline int sign_y(int v) { return v == 2 ? -1 : 1; }

// readBlock's ghost-cell semantics on the full grid: periodic index wrap per
// side (GPUSimulators/cuda/common.h:248-288, :333-347), then reflective mirror
// in the order north, south, east, west (common.h:293-315, :135-239).
// Dirichlet ghosts keep the stored values of the input buffer.
template <typename T>
void fill_ghosts(Grid<T>& E, const T* const* in, int bc) {
    const int g = E.g, nx = E.nx, ny = E.ny, w = E.w, h = E.h;
    const bool pw = bc_west(bc) == PERIODIC, pe = bc_east(bc) == PERIODIC;
    const bool ps = bc_south(bc) == PERIODIC, pn = bc_north(bc) == PERIODIC;
    for (int v = 0; v < E.nv; ++v) {
        for (int l = 0; l < h; ++l) {
            int ls = l;
            if (ls < g && ps) ls += ny;
            else if (ls >= ny + g && pn) ls -= ny;
            for (int k = 0; k < w; ++k) {
                int ks = k;
                if (ks < g && pw) ks += nx;
                else if (ks >= nx + g && pe) ks -= nx;
                E.at(v, l, k) = in[v][(size_t)ls * w + ks];
            }
        }
        const T sx = T(sign_x(v)), sy = T(sign_y(v));
        if (bc_north(bc) == REFLECTIVE)
            for (int m = 0; m < g; ++m)
                for (int k = 0; k < w; ++k) E.at(v, ny + g + m, k) = sy * E.at(v, ny + g - 1 - m, k);
        if (bc_south(bc) == REFLECTIVE)
            for (int m = 0; m < g; ++m)
                for (int k = 0; k < w; ++k) E.at(v, g - 1 - m, k) = sy * E.at(v, g + m, k);
        if (bc_east(bc) == REFLECTIVE)
            for (int l = 0; l < h; ++l)
                for (int m = 0; m < g; ++m) E.at(v, l, nx + g + m) = sx * E.at(v, l, nx + g - 1 - m);
        if (bc_west(bc) == REFLECTIVE)
            for (int l = 0; l < h; ++l)
                for (int m = 0; m < g; ++m) E.at(v, l, g - 1 - m) = sx * E.at(v, l, g + m);
    }
}

// Parameters of one substep.
template <typename T> struct Params {
    int scheme;
    T dx, dy, dt, g, gamma, theta;
    int step, order, bc;
    int variant;  // HLL: flux (0 HLL, 1 HLLC, 2 GodC); WAF: limiter id (flux_limiter)
    T beta;       // Osher / Sweby limiter parameter
};

// A line (row or column) of NV variables, accessed with a stride.  For the
// y direction the caller swaps the two momentum components, as every
// computeFluxG in the reference does (e.g. GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:81-107).
template <typename T, int NV> struct Line {
    T* p[NV];
    ptrdiff_t stride;
    Vec<T, NV> get(int k) const {
        Vec<T, NV> q;
        for (int v = 0; v < NV; ++v) q.c[v] = p[v][k * stride];
        return q;
    }
};

// MUSCL-Hancock face states for interface k+1/2 (slopes at k and k+1, half-step
// predictor): GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:38-58 (and the same
// code in SWE2D_HLL2.cu:39-59 and EE2D_KP07_dimsplit.cu:33-58).
template <typename T, int NV, typename FF>
inline void muscl_hancock(const Line<T, NV>& L, int k, T theta, T c, FF flux_fn, Vec<T, NV>& Ql_bar,
                          Vec<T, NV>& Qr_bar) {
    Vec<T, NV> Q_ll, Q_lr, Q_rl, Q_rr;
    for (int v = 0; v < NV; ++v) {
        const T qm1 = L.p[v][(k - 1) * L.stride], q0 = L.p[v][k * L.stride];
        const T q1 = L.p[v][(k + 1) * L.stride], q2 = L.p[v][(k + 2) * L.stride];
        const T sl = minmod_slope(qm1, q0, q1, theta);
        const T sr = minmod_slope(q0, q1, q2, theta);
        Q_rl.c[v] = q1 - T(0.5) * sr;
        Q_rr.c[v] = q1 + T(0.5) * sr;
        Q_ll.c[v] = q0 - T(0.5) * sl;
        Q_lr.c[v] = q0 + T(0.5) * sl;
    }
    const Vec<T, NV> F_rl = flux_fn(Q_rl), F_rr = flux_fn(Q_rr), F_ll = flux_fn(Q_ll), F_lr = flux_fn(Q_lr);
    for (int v = 0; v < NV; ++v) {
        Qr_bar.c[v] = Q_rl.c[v] + c * (F_rl.c[v] - F_rr.c[v]);
        Ql_bar.c[v] = Q_lr.c[v] + c * (F_ll.c[v] - F_lr.c[v]);
    }
}

// Numerical flux at interface k+1/2 of a line, for the dimensionally split
// schemes.  `ydir` selects the second sweep's flux where it differs (Euler).
template <typename T, int NV>
inline Vec<T, NV> face_flux(const Params<T>& P, const Line<T, NV>& L, int k, T dxx, bool ydir);

template <>
inline Vec<float, 3> face_flux<float, 3>(const Params<float>& P, const Line<float, 3>& L, int k, float dxx, bool);
template <>
inline Vec<double, 3> face_flux<double, 3>(const Params<double>& P, const Line<double, 3>& L, int k, double dxx, bool);

template <typename T>
inline Vec<T, 3> swe_face_flux(const Params<T>& P, const Line<T, 3>& L, int k, T dxx) {
    const T g = P.g;
    switch (P.scheme) {
    case FORCE:  // GPUSimulators/cuda/SWE2D_FORCE.cu:34-50
        return swe_force_1d(L.get(k), L.get(k + 1), g, dxx, P.dt);
    case HLL:  // GPUSimulators/cuda/SWE2D_HLL.cu:36-52 (variant 0)
        if (P.variant == 1) return swe_hllc(L.get(k), L.get(k + 1), g);
        if (P.variant == 2) return swe_godc_1d(L.get(k), L.get(k + 1), g, dxx, P.dt);
        return swe_hll(L.get(k), L.get(k + 1), g);
    case WAF:  // GPUSimulators/cuda/SWE2D_WAF.cu:39-53 (limiter 0)
        return swe_waf(L.get(k - 1), L.get(k), L.get(k + 1), L.get(k + 2), g, dxx, P.dt, P.variant, P.beta);
    case HLL2:
    case KP07_DIMSPLIT: {
        const T c = P.dt / (T(2) * dxx);
        Vec<T, 3> Ql_bar, Qr_bar;
        muscl_hancock<T, 3>(L, k, P.theta, c, [g](const Vec<T, 3>& q) { return swe_F(q, g); }, Ql_bar, Qr_bar);
        if (P.scheme == HLL2) return swe_hll(Ql_bar, Qr_bar, g);  // SWE2D_HLL2.cu:62
        return swe_central_upwind(Ql_bar, Qr_bar, g);           // SWE2D_KP07_dimsplit.cu:61
    }
    default:
        break;
    }
    return Vec<T, 3>{{T(NAN), T(NAN), T(NAN)}};
}

template <>
inline Vec<float, 3> face_flux<float, 3>(const Params<float>& P, const Line<float, 3>& L, int k, float dxx, bool) {
    return swe_face_flux<float>(P, L, k, dxx);
}
template <>
inline Vec<double, 3> face_flux<double, 3>(const Params<double>& P, const Line<double, 3>& L, int k, double dxx,
                                           bool) {
    return swe_face_flux<double>(P, L, k, dxx);
}

template <typename T>
inline Vec<T, 4> euler_face_flux(const Params<T>& P, const Line<T, 4>& L, int k, T dxx, bool ydir) {
    const T gamma = P.gamma;
    const T c = P.dt / (T(2) * dxx);
    Vec<T, 4> Ql_bar, Qr_bar;
    // The reference's predictor calls F_func(Q, gamma_): the pressure argument
    // receives gamma (GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:57-58, :102-103).
    muscl_hancock<T, 4>(L, k, P.theta, c, [gamma](const Vec<T, 4>& q) { return euler_F(q, gamma); }, Ql_bar, Qr_bar);
    if (!ydir) return euler_hll(Ql_bar, Qr_bar, gamma);         // EE2D_KP07_dimsplit.cu:62
    return euler_central_upwind(Ql_bar, Qr_bar, gamma);         // EE2D_KP07_dimsplit.cu:106
}
template <>
inline Vec<Counted, 3> face_flux<Counted, 3>(const Params<Counted>& P, const Line<Counted, 3>& L, int k, Counted dxx,
                                             bool) {
    return swe_face_flux<Counted>(P, L, k, dxx);
}
template <>
inline Vec<Counted, 4> face_flux<Counted, 4>(const Params<Counted>& P, const Line<Counted, 4>& L, int k, Counted dxx,
                                             bool y) {
    return euler_face_flux<Counted>(P, L, k, dxx, y);
}
template <>
inline Vec<float, 4> face_flux<float, 4>(const Params<float>& P, const Line<float, 4>& L, int k, float dxx, bool y) {
    return euler_face_flux<float>(P, L, k, dxx, y);
}
template <>
inline Vec<double, 4> face_flux<double, 4>(const Params<double>& P, const Line<double, 4>& L, int k, double dxx,
                                           bool y) {
    return euler_face_flux<double>(P, L, k, dxx, y);
}

// One 1-D sweep of a line: interior cells [g, n+g) become
// Q + (F_{k-1/2} - F_{k+1/2}) * dt / dxx (GPUSimulators/cuda/common.h:444-475).
// `src` and `dst` may not alias.
template <typename T, int NV>
void sweep_line(const Params<T>& P, const Line<T, NV>& src, const Line<T, NV>& dst, int n, int g, T dxx, bool ydir) {
    std::vector<Vec<T, NV>> F(n + 1);
    for (int f = 0; f <= n; ++f) F[f] = face_flux<T, NV>(P, src, g - 1 + f, dxx, ydir);
    for (int i = 0; i < n; ++i) {
        const int k = g + i;
        for (int v = 0; v < NV; ++v)
            dst.p[v][k * dst.stride] = src.p[v][k * src.stride] + (F[i].c[v] - F[i + 1].c[v]) * P.dt / dxx;
    }
}

template <typename T, int NV> Line<T, NV> row_line(Grid<T>& G, int l) {
    Line<T, NV> L;
    for (int v = 0; v < NV; ++v) L.p[v] = G.d[v].data() + (size_t)l * G.w;
    L.stride = 1;
    return L;
}
template <typename T, int NV> Line<T, NV> col_line(Grid<T>& G, int k) {
    Line<T, NV> L;
    for (int v = 0; v < NV; ++v) L.p[v] = G.d[v].data() + k;
    L.stride = G.w;
    std::swap(L.p[1], L.p[2]);  // transpose: the sweep sees (h, hv, hu) / (rho, rho_v, rho_u, E)
    return L;
}

// X sweep of the rows [l0, l1) of A into B (interior columns only; every other
// cell of B is left as it was).
template <typename T, int NV>
void x_sweep(const Params<T>& P, Grid<T>& A, Grid<T>& B, int l0, int l1) {
#pragma omp parallel for schedule(static)
    for (int l = l0; l < l1; ++l)
        sweep_line<T, NV>(P, row_line<T, NV>(A, l), row_line<T, NV>(B, l), A.nx, A.g, P.dx, false);
}
template <typename T, int NV>
void y_sweep(const Params<T>& P, Grid<T>& A, Grid<T>& B, int k0, int k1) {
#pragma omp parallel for schedule(static)
    for (int k = k0; k < k1; ++k)
        sweep_line<T, NV>(P, col_line<T, NV>(A, k), col_line<T, NV>(B, k), A.ny, A.g, P.dy, true);
}

// CFL of the updated state: GPUSimulators/cuda/SWECommon.h:482-532 (SWE, sqrt(g*h)) and
// GPUSimulators/cuda/EulerCommon.h:27-77 (Euler, sqrt(gamma*rho)); the block minima of
// the reference reduce to the minimum over all interior cells.  fmin ignores NaN
// exactly like the reference's fminf.
template <typename T>
T cfl_min(const Params<T>& P, const Grid<T>& Q) {
    const T gg = (P.scheme == EE2D_KP07_DIMSPLIT) ? P.gamma : P.g;
    T m = T(INFINITY);
    bool any = false;
    for (int l = Q.g; l < Q.ny + Q.g; ++l)
        for (int k = Q.g; k < Q.nx + Q.g; ++k) {
            const T h = Q.at(0, l, k);
            const T u = Q.at(1, l, k) / h;
            const T v = Q.at(2, l, k) / h;
            const T max_u = P.dx / (fabs_(u) + sqrt_(gg * h));
            const T max_v = P.dy / (fabs_(v) + sqrt_(gg * h));
            const T c = fmin_(max_u, max_v);
            m = any ? fmin_(m, c) : c;
            any = true;
        }
    return m;
}

// Dimensionally split substep (FORCE, HLL, HLL2, WAF, KP07_dimsplit, EE2D).
// step 0 sweeps x then y; step 1 sweeps y then x (e.g. SWE2D_KP07_dimsplit.cu:161-194).
// FORCE and HLL always sweep x then y with the full dt (SWE2D_FORCE.cu:120-130,
// SWE2D_HLL.cu:136-148).  The first sweep covers every line of the grid
// including ghost lines, as the reference's block sweep covers its halo lines.
template <typename T, int NV>
void dimsplit_substep(const Params<T>& P, const T* const* in, T* const* out, int nx, int ny, T* cfl) {
    const int g = ghost_cells(P.scheme);
    Grid<T> E(nx, ny, g, NV);
    fill_ghosts(E, in, P.bc);
    Grid<T> A = E;
    Grid<T> B = E;
    const bool x_first = (P.scheme == FORCE || P.scheme == HLL) ? true : (P.step == 0);
    if (x_first) {
        x_sweep<T, NV>(P, E, A, 0, E.h);
        B = A;
        y_sweep<T, NV>(P, A, B, g, nx + g);
    } else {
        y_sweep<T, NV>(P, E, A, 0, E.w);
        B = A;
        x_sweep<T, NV>(P, A, B, g, ny + g);
    }
    if (P.scheme == EE2D_KP07_DIMSPLIT && P.g > T(0)) {
        // Gravity source term: GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:197-205, :226-233
        for (int l = g; l < ny + g; ++l)
            for (int k = g; k < nx + g; ++k) {
                const T rho_v = B.at(2, l, k);
                B.at(2, l, k) = B.at(2, l, k) - P.g * B.at(0, l, k) * P.dt;
                B.at(3, l, k) = B.at(3, l, k) - P.g * rho_v * P.dt;
            }
    }
    for (int v = 0; v < NV; ++v)
        for (int l = g; l < ny + g; ++l)
            for (int k = g; k < nx + g; ++k) out[v][(size_t)l * E.w + k] = B.at(v, l, k);
    if (cfl) *cfl = cfl_min(P, B);
}

// Unsplit substep: LxF (GPUSimulators/cuda/SWE2D_LxF.cu:102-165) and KP07
// (GPUSimulators/cuda/SWE2D_KP07.cu:136-232, RK2 blend at :215-225).
template <typename T>
void unsplit_substep(const Params<T>& P, const T* const* in, T* const* out, int nx, int ny, T* cfl) {
    const int g = ghost_cells(P.scheme);
    Grid<T> E(nx, ny, g, 3);
    fill_ghosts(E, in, P.bc);
    Grid<T> B = E;
    const int w = E.w;
    const bool kp07 = (P.scheme == KP07);
    const bool blend = kp07 && P.order == 2 && P.step == 1;
#pragma omp parallel for schedule(static)
    for (int l = g; l < ny + g; ++l) {
        Line<T, 3> row = row_line<T, 3>(E, l);
        std::vector<Vec<T, 3>> F(nx + 1), G0(nx), G1(nx);
        for (int f = 0; f <= nx; ++f) {
            const int k = g - 1 + f;  // interface k+1/2
            if (!kp07) {
                F[f] = swe_lxf_2d(row.get(k), row.get(k + 1), P.g, P.dx, P.dt);  // SWE2D_LxF.cu:38-58
            } else {
                // SWE2D_KP07.cu:41-60 with slopes from SWE2D_KP07.cu:99-111
                Vec<T, 3> Qm, Qp;
                for (int v = 0; v < 3; ++v) {
                    const T sm = minmod_slope(row.p[v][k - 1], row.p[v][k], row.p[v][k + 1], P.theta);
                    const T sp = minmod_slope(row.p[v][k], row.p[v][k + 1], row.p[v][k + 2], P.theta);
                    Qp.c[v] = row.p[v][k + 1] - T(0.5) * sp;
                    Qm.c[v] = row.p[v][k] + T(0.5) * sm;
                }
                F[f] = swe_central_upwind(Qm, Qp, P.g);
            }
        }
        for (int i = 0; i < nx; ++i) {
            const int k = g + i;
            Line<T, 3> col = col_line<T, 3>(E, k);
            for (int s = 0; s < 2; ++s) {
                const int m = l - 1 + s;  // interface m+1/2 along y
                Vec<T, 3> Gs;
                if (!kp07) {
                    Gs = swe_lxf_2d(col.get(m), col.get(m + 1), P.g, P.dy, P.dt);
                } else {
                    Vec<T, 3> Qm, Qp;
                    for (int v = 0; v < 3; ++v) {
                        const ptrdiff_t st = col.stride;
                        const T* c = col.p[v];
                        const T sm = minmod_slope(c[(m - 1) * st], c[m * st], c[(m + 1) * st], P.theta);
                        const T sp = minmod_slope(c[m * st], c[(m + 1) * st], c[(m + 2) * st], P.theta);
                        Qp.c[v] = c[(m + 1) * st] - T(0.5) * sp;
                        Qm.c[v] = c[m * st] + T(0.5) * sm;
                    }
                    Gs = swe_central_upwind(Qm, Qp, P.g);
                }
                std::swap(Gs.c[1], Gs.c[2]);  // swap back to (h, hu, hv)
                (s == 0 ? G0 : G1)[i] = Gs;
            }
        }
        for (int i = 0; i < nx; ++i) {
            const int k = g + i;
            for (int v = 0; v < 3; ++v) {
                const T q = E.at(v, l, k) +
                            ((F[i].c[v] - F[i + 1].c[v]) * P.dt / P.dx + (G0[i].c[v] - G1[i].c[v]) * P.dt / P.dy);
                B.at(v, l, k) = q;
                T* o = &out[v][(size_t)l * w + k];
                *o = blend ? T(0.5) * (*o + q) : q;
            }
        }
    }
    if (cfl) *cfl = cfl_min(P, B);
}

template <typename T>
int substep_impl(int scheme, int nx, int ny, const T* const* in, T* const* out, T dx, T dy, T dt, T g, T gamma,
                 T theta, int step, int order, int bc, T* cfl, int nthreads, int variant = 0, T beta = T(0)) {
    if (scheme < 0 || scheme > 7 || nx <= 0 || ny <= 0) return 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    Params<T> P{scheme, dx, dy, dt, g, gamma, theta, step, order, bc, variant, beta};
    if (scheme == LXF || scheme == KP07) {
        unsplit_substep<T>(P, in, out, nx, ny, cfl);
    } else if (scheme == EE2D_KP07_DIMSPLIT) {
        dimsplit_substep<T, 4>(P, in, out, nx, ny, cfl);
    } else {
        dimsplit_substep<T, 3>(P, in, out, nx, ny, cfl);
    }
    return 0;
}

}  // namespace

extern "C" {

// One substep of `scheme` (0 LxF, 1 FORCE, 2 HLL, 3 HLL2, 4 WAF, 5 KP07,
// 6 KP07_dimsplit, 7 EE2D_KP07_dimsplit).  `in`/`out` hold nv dense arrays of
// (ny+2g) x (nx+2g) values including ghost cells; only interior cells of `out`
// are written (the reference never writes ghost cells, common.h:376).  `cfl`
// (nullable) receives the minimum CFL time step of the updated state.
// `variant`, `beta`: HLL's flux or WAF's limiter (see Params); 0 for the reference's.
int fvo_substep_f32(int scheme, int nx, int ny, const float* const* in, float* const* out, float dx, float dy,
                    float dt, float g, float gamma, float theta, int step, int order, int bc, float* cfl,
                    int nthreads, int variant, float beta) {
    return substep_impl<float>(scheme, nx, ny, in, out, dx, dy, dt, g, gamma, theta, step, order, bc, cfl, nthreads,
                               variant, beta);
}

int fvo_substep_f64(int scheme, int nx, int ny, const double* const* in, double* const* out, double dx, double dy,
                    double dt, double g, double gamma, double theta, int step, int order, int bc, double* cfl,
                    int nthreads, int variant, double beta) {
    return substep_impl<double>(scheme, nx, ny, in, out, dx, dy, dt, g, gamma, theta, step, order, bc, cfl,
                                nthreads, variant, beta);
}

// One face flux in FP32 for n face pairs (ql, qr: n x 3): kind 0 HLL, 1 HLLC,
// 2 Godunov centred (dx, dt used by 2 only).
int fvo_flux_eval(int kind, int n, const float* ql, const float* qr, float g, float dx, float dt, float* out) {
    for (int i = 0; i < n; ++i) {
        const Vec<float, 3> l{{ql[3 * i], ql[3 * i + 1], ql[3 * i + 2]}}, r{{qr[3 * i], qr[3 * i + 1], qr[3 * i + 2]}};
        const Vec<float, 3> f = kind == 1 ? swe_hllc(l, r, g) : kind == 2 ? swe_godc_1d(l, r, g, dx, dt)
                                                                           : swe_hll(l, r, g);
        for (int v = 0; v < 3; ++v) out[3 * i + v] = f.c[v];
    }
    return 0;
}

// A flux limiter (flux_limiter ids) in FP32 on n ratios.
int fvo_limiter_eval(int id, int n, const float* r, float beta, float* out) {
    for (int i = 0; i < n; ++i) out[i] = flux_limiter(r[i], id, beta);
    return 0;
}

// Floating-point operations of one substep as the reference formulates it:
// runs the substep single-threaded on `in` (nv arrays of (ny+2g) x (nx+2g)
// values) with the counting type and stores the counts of add, sub, mul, div,
// sqrt and min/max into counts[0..5].  The state it computes is discarded.
int fvo_count_ops(int scheme, int nx, int ny, const double* const* in, double dx, double dy, double dt, double g,
                  double gamma, double theta, int step, int order, int bc, long long* counts) {
    if (scheme < 0 || scheme > 7 || nx <= 0 || ny <= 0) return 1;
    const int gh = ghost_cells(scheme), nv = num_vars(scheme);
    const size_t n = (size_t)(nx + 2 * gh) * (ny + 2 * gh);
    std::vector<Counted> src[4], dst[4];
    const Counted* ip[4] = {nullptr, nullptr, nullptr, nullptr};
    Counted* op[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int v = 0; v < nv; ++v) {
        src[v].assign(in[v], in[v] + n);
        dst[v].assign(n, Counted(0.0));
        ip[v] = src[v].data();
        op[v] = dst[v].data();
    }
#ifdef _OPENMP
    const int threads = omp_get_max_threads();
#endif
    g_ops = OpCounts{0, 0, 0, 0, 0, 0};
    const int rc = substep_impl<Counted>(scheme, nx, ny, ip, op, Counted(dx), Counted(dy), Counted(dt), Counted(g),
                                         Counted(gamma), Counted(theta), step, order, bc, nullptr, 1);
#ifdef _OPENMP
    omp_set_num_threads(threads);
#endif
    counts[0] = g_ops.add;
    counts[1] = g_ops.sub;
    counts[2] = g_ops.mul;
    counts[3] = g_ops.div;
    counts[4] = g_ops.sqrt;
    counts[5] = g_ops.minmax;
    return rc;
}

int fvo_ghost_cells(int scheme) { return ghost_cells(scheme); }
int fvo_num_vars(int scheme) { return num_vars(scheme); }

}  // extern "C"
