// Stage kernels: one launch advances every cell of one simulation by one
// substep of its scheme (the work of one reference kernel launch, e.g.
// GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:123-205).
//
// Tile: a CTA owns W x H interior cells.  One TMA box per variable brings the
// tile plus a 4-column / 2-row halo into shared memory ((H+4) x P floats with
// row pitch P = W+8, or wider for 8-segment tiles, split_pitch; box x aligned
// to 4 floats).  Ghost cells are then completed in shared memory
// (periodic wrap from global memory, reflective mirror in the reference's
// N, S, E, W order), the sweeps run in place, and the interior is written back
// with 128-bit stores.  The CFL minimum and the FP64 conservation sums are
// reduced in the same pass; the last CTA to finish advances the simulation's
// control block (t, nt, dt, buffer parity), so a whole step sequence can be
// captured in a CUDA graph without host round trips.
//
// Sweep mapping:
//   x sweeps: a thread walks one row segment of W/4 cells (lanes = 8 rows x
//     4 segments; or W/8 cells, lanes = 4 rows x 8 segments).  With a shared
//     row pitch of 4 (8) mod 32 floats and an odd segment length the 32
//     lanes hit 32 distinct banks.
//   y sweeps: a thread walks one column segment (lanes = consecutive columns).
//   LPT = 2: a thread walks two lines side by side in packed f32x2
//     arithmetic (rows t and t + n/2, columns s and s + n/2).
// Each thread keeps a 3-cell window in registers and reconstructs every cell
// once; the halo cells of its segment are read before a barrier so that
// in-place updates by neighbouring segments cannot race with them.
#pragma once

#include <cuda.h>

#include "fv_device.cuh"

namespace fv {

enum Scheme { LXF = 0, FORCE = 1, HLL = 2, HLL2 = 3, WAF = 4, KP07 = 5, KP07_DIMSPLIT = 6, EE2D = 7 };

// Reference boundary codec (GPUSimulators/cuda/common.h:109-130).
enum BoundaryType { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_PERIODIC = 2, BC_REFLECTIVE = 3 };
__host__ __device__ inline int bc_north(int bc) { return (bc >> 24) & 0xF; }
__host__ __device__ inline int bc_south(int bc) { return (bc >> 16) & 0xF; }
__host__ __device__ inline int bc_east(int bc) { return (bc >> 8) & 0xF; }
__host__ __device__ inline int bc_west(int bc) { return bc & 0xF; }

// Control block of one simulation, resident in device memory.
struct alignas(16) SimCtl {
    double t;          // simulation time (BaseSimulator.t, FP64)
    double t_end;      // end time of the current simulate() call
    long long nt;      // completed steps (BaseSimulator.nt)
    float dt;          // CFL step in use (BaseSimulator.dt)
    float cfl_min;     // min of the last CFL field (gpuarray.min(cfl_data))
    float factor;      // the scheme's computeDt factor
    float cfl_scale;   // Courant number
    int update_dt;     // recompute dt every 100 steps (simulate(t) without dt)
    int cur;           // buffer index holding u0
    unsigned int arrive;  // CTA arrival counter for the last-CTA epilogue
    int error;         // nonzero once a bounded wait gave up
    double sums[4];    // FP64 sums of the interior of u0 after the last step that asked for them
    int bad;           // batched simulations: a step left a non-finite value or a non-positive depth
                       // (density); the simulation then stops (t_end is set to t)
};

// Launch arguments (passed as a __grid_constant__ parameter; the tensor maps
// must live in parameter, constant or global memory).
struct StageArgs {
    CUtensorMap tmap[2][4];  // [buffer][variable]
    float* buf[2][4];
    SimCtl* ctl;
    float* block_cfl;    // one float per CTA
    double* block_sums;  // 4 doubles per CTA
    int nx, ny, pitch;   // pitch in floats
    float dx, dy, g, gamma, theta;
    float dt_scale;      // kernel dt = step dt * dt_scale (0.5 for split substeps)
    int bc;
    int substep;         // sweep order (split schemes) or RK stage (KP07)
    int order;           // RK order (KP07)
    int is_last;         // this launch completes a step
    int force_cfl;       // compute the CFL field in this launch
    int explicit_dt;     // take the step dt from dt_step instead of the control block
    float dt_step;
    int want_sums;       // compute FP64 sums of the new state at the end of a step
    float variant_beta;  // parameter of the Osher and Sweby limiters (the variant itself is a kernel template)
    int wait_limit;      // tile-load wait: 0 = kWaitPolls polls (the default, also for zero-filled
                         // arguments), n > 0 = n polls, negative = give up at once (tests)
    int tile_row0;       // first tile row of this launch (a substep may be split into launches by rows)
    int ntiles_total;    // tiles of the whole substep, 0 = this launch's grid; the last of them to
                         // arrive, over all launches, finishes the substep
};

// Polls of a bounded mbarrier wait before it gives up (each poll may suspend
// the thread for a short hardware-defined time; in all about a second).
constexpr uint32_t kWaitPolls = 1u << 20;
__host__ __device__ inline uint32_t wait_polls(int wait_limit) {
    return wait_limit == 0 ? kWaitPolls : (wait_limit < 0 ? 0u : (uint32_t)wait_limit);
}

// Storage: per variable, rows y = -2 .. ny+1 and columns x = -4 .. pitch-5,
// element (y, x) at [(y + 2) * pitch + (x + 4)].
__host__ __device__ inline long long cell_index(int y, int x, int pitch) {
    return (long long)(y + 2) * pitch + (x + 4);
}

// Split-scheme tiles: x-sweep segments per tile row and the shared-memory row
// pitch (the TMA box width) of a W-wide tile.  A warp's x-sweep lanes cover
// 32/NSEG rows x NSEG segments of W/NSEG cells; they hit 32 distinct banks
// when the segment length is odd and the pitch is 4 (mod 32) for 4 segments,
// 8 (mod 32) for 8.  W + 8 (4 halo columns each side) is 4 (mod 32) for the
// 4-segment widths (124, 60, 28); 8-segment widths (120) load a box padded on
// the right to the next pitch of 8 (mod 32).
__host__ __device__ constexpr int split_nseg_x(int W) { return ((W / 4) % 2 == 1) ? 4 : 8; }
__host__ __device__ constexpr int split_pitch(int W) {
    return split_nseg_x(W) == 4 ? W + 8 : W + 8 + (((8 - (W + 8)) % 32) + 32) % 32;
}

struct StepCtl {
    float dt;      // step dt (before dt_scale)
    double t_new;  // t after this step
    int cur;
    bool active;
    bool do_cfl;
};

// dt of the current step: float32(min(dt, t_end - t)) (GPUSimulators/Simulator.py:199),
// with Python's min() tie and NaN behaviour; a step runs while t < t_end and
// dt > 0 (Simulator.py:192, :202).
//
// The control block changes only between launches, or in this launch after
// every tile of the simulation has read it (the last tile's epilogue), so its
// first 48 bytes are read with three 16-byte relaxed loads issued together: one
// L2 round trip per warp instead of one per field.
__device__ __forceinline__ int4 ld_relaxed_v4(const void* p) {
    int4 r;
    asm volatile("ld.relaxed.gpu.global.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p));
    return r;
}

// The step of a control block from its first 48 bytes (w0, w1, w2).
__device__ __forceinline__ StepCtl step_from_words(const int4& w0, const int4& w1, const int4& w2, bool explicit_dt,
                                                   float dt_step, bool force_cfl, bool is_last) {
    StepCtl s;
    s.cur = w2.w;
    const double t = __hiloint2double(w0.y, w0.x);
    const double t_end = __hiloint2double(w0.w, w0.z);
    if (explicit_dt) {
        s.dt = dt_step;
        s.active = true;
    } else {
        const double rem = t_end - t;
        const double d = (double)__int_as_float(w1.z);
        s.dt = (float)((rem < d) ? rem : d);
        s.active = (t < t_end) && !(s.dt <= 0.0f);
    }
    s.t_new = t + (double)s.dt;
    const long long nt = (long long)(((unsigned long long)(unsigned)w1.y << 32) | (unsigned)w1.x);
    const bool sched = w2.z && ((nt + 1) % 100 == 0);
    s.do_cfl = force_cfl || (is_last && !explicit_dt && (sched || !(s.t_new < t_end)));
    return s;
}

__device__ __forceinline__ StepCtl read_step(const SimCtl* ctl, bool explicit_dt, float dt_step, bool force_cfl,
                                             bool is_last) {
    static_assert(offsetof(SimCtl, t_end) == 8 && offsetof(SimCtl, nt) == 16 && offsetof(SimCtl, dt) == 24 &&
                      offsetof(SimCtl, update_dt) == 40 && offsetof(SimCtl, cur) == 44,
                  "read_step's vector loads follow SimCtl's layout");
    const int4 w0 = ld_relaxed_v4(ctl);                                          // t, t_end
    const int4 w1 = ld_relaxed_v4(reinterpret_cast<const char*>(ctl) + 16);      // nt, dt, cfl_min
    const int4 w2 = ld_relaxed_v4(reinterpret_cast<const char*>(ctl) + 32);      // factor, cfl_scale, update_dt, cur
    return step_from_words(w0, w1, w2, explicit_dt, dt_step, force_cfl, is_last);
}

__device__ __forceinline__ StepCtl read_step(const StageArgs& A) {
    return read_step(A.ctl, A.explicit_dt != 0, A.dt_step, A.force_cfl != 0, A.is_last != 0);
}

template <int NT>
__device__ __forceinline__ float block_min(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    float r = red[0];
#pragma unroll
    for (int i = 1; i < NT / 32; ++i) r = fminf(r, red[i]);
    return r;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
#pragma unroll
    for (int i = 1; i < NT / 32; ++i) r += red[i];
    return r;
}

// Tile epilogue: per-tile CFL minimum and FP64 sums, arrival count on the
// simulation's control block, and (last tile of the simulation in this launch)
// the reduction over all its tiles in fixed order plus the control-block update
// of Simulator.step / simulate (GPUSimulators/Simulator.py:195-196, :227-228).
template <int NT, int NV>
__device__ void tile_epilogue(SimCtl* ctl, float* block_cfl, double* block_sums, int tile, int ntiles, bool is_last,
                              bool explicit_dt, const StepCtl& s, float my_cfl, const double (&my_sums)[NV],
                              bool sums) {
    __shared__ float red_f[NT / 32];
    __shared__ double red_d[NT / 32];
    __shared__ int am_last;
    if (s.do_cfl) {
        const float m = block_min<NT>(my_cfl, red_f);
        if (threadIdx.x == 0) block_cfl[tile] = m;
    }
    if (sums) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double t = block_sum<NT>(my_sums[v], red_d);
            if (threadIdx.x == 0) block_sums[(size_t)tile * 4 + v] = t;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->arrive, 1u);
        am_last = (prev == (unsigned)ntiles - 1u);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    float m = __int_as_float(0x7f800000);
    if (s.do_cfl) {
        for (int i = threadIdx.x; i < ntiles; i += NT) m = fminf(m, __ldcg(&block_cfl[i]));
        m = block_min<NT>(m, red_f);
    }
    double tot[NV];
    if (sums) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            // fixed per-thread striding and tree: deterministic for a given grid
            double acc = 0.0;
            for (int i = threadIdx.x; i < ntiles; i += NT) acc += __ldcg(&block_sums[(size_t)i * 4 + v]);
            tot[v] = block_sum<NT>(acc, red_d);
        }
    }
    if (threadIdx.x == 0) {
        SimCtl* c = ctl;
        c->cur = s.cur ^ 1;
        if (s.do_cfl) c->cfl_min = m;
        if (sums) {
#pragma unroll
            for (int v = 0; v < NV; ++v) c->sums[v] = tot[v];
        }
        if (is_last) {
            c->t = s.t_new;
            c->nt = c->nt + 1;
            if (!explicit_dt && c->update_dt && (c->nt % 100 == 0)) c->dt = (c->cfl_min * c->factor) * c->cfl_scale;
            if (c->bad) c->t_end = c->t;  // a failed simulation takes no further steps
        }
        c->arrive = 0u;
        __threadfence();
    }
    __syncthreads();  // am_last and the reduction scratch are reused by the next tile of a persistent CTA
}

template <int NT, int NV>
__device__ __forceinline__ void stage_epilogue(const StageArgs& A, const StepCtl& s, float my_cfl,
                                               const double (&my_sums)[NV], bool sums) {
    // The tile is written: the next substep's CTAs may launch once every CTA
    // of this grid is here (they wait in grid_dependency_wait for its end).
    grid_launch_dependents();
    tile_epilogue<NT, NV>(A.ctl, A.block_cfl, A.block_sums, (blockIdx.y + A.tile_row0) * gridDim.x + blockIdx.x,
                          A.ntiles_total ? A.ntiles_total : gridDim.x * gridDim.y, A.is_last != 0,
                          A.explicit_dt != 0, s, my_cfl, my_sums, sums);
}

// ------------------------------------------------------------------ tile load + ghost cells

// One tile of one simulation: where its input comes from and where it goes.
struct TileJob {
    const CUtensorMap* tmap;  // NV tensor maps of the input planes (kernel parameters; unused by async loads)
    float* const* in;         // NV input planes
    float* const* out;        // NV output planes
    int nx, ny, pitch, bc;
    int x0, y0;               // first interior cell of the tile
};

// Issues the TMA loads of the tile (thread 0) and waits for them with a bounded
// wait of `polls` polls on `phase` of the mbarrier (initialised here when
// `init`).  Returns false (uniformly across the CTA) if the wait gave up; *err
// is then set, after a second bounded wait has let the copies in flight land.
template <int NV, int SP, int TR>
__device__ __forceinline__ bool load_tile(float* Qs, const CUtensorMap* tmap, int x0, int y0, uint64_t* bar,
                                          uint32_t phase, bool init, int* err, uint32_t polls = kWaitPolls) {
    constexpr int PS = SP * TR;
    // Each variable's plane is the destination of a tensor copy, which must
    // start on a 128-byte boundary: tiles whose (W+8) x (H+4) plane is not a
    // multiple of 32 floats would misalign every plane after the first.
    static_assert((PS * sizeof(float)) % 128 == 0, "variable planes in shared memory must be 128-byte aligned");
    if (threadIdx.x == 0) {
        if (init) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
        // The CTA's generic-proxy reads and writes of the previous tile in this
        // buffer (ordered before this point by the last barrier) must precede
        // the async-proxy writes of the new load.
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, NV * PS * (uint32_t)sizeof(float));
#pragma unroll
        for (int v = 0; v < NV; ++v) tma_load_2d(Qs + v * PS, tmap + v, x0, y0, bar);
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(bar, phase, polls);
    const int failed = __syncthreads_or(ok ? 0 : 1);
    if (failed) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        mbar_wait_bounded(bar, phase, kWaitPolls);  // let copies in flight land before the CTA moves on
        return false;
    }
    return true;
}

// The same tile as load_tile, brought in by the CTA's threads with 16-byte
// asynchronous copies instead of a tensor map: the box of SP x TR floats at
// storage (x0, y0) of each input plane, with the tensor maps' extents
// (nx + 8 columns, ny + 4 rows) and their zero fill beyond them, so the shared
// tile holds the same values.  The batched kernels use it: their simulations
// are only known on the device, and a tensor map in global memory needs a
// proxy fence before every use, which measured about 10 us per tile.  Storage
// rows start on 16-byte boundaries and x0 is a multiple of 4, so every chunk
// is aligned; a chunk that straddles column nx + 8 copies its valid floats.
template <int NV, int SP, int TR, int NT>
__device__ __forceinline__ void load_tile_async(float* Qs, const TileJob& J) {
    constexpr int PS = SP * TR, CH = SP / 4, G = NT / CH;  // G rows of CH chunks at a time
    static_assert(SP % 4 == 0 && G >= 1, "shared rows of whole 16-byte chunks, one chunk per thread");
    // thread k copies chunk c = k % CH of tile rows g, g + G, g + 2G, ... (g = k / CH)
    const int c = threadIdx.x % CH, g = threadIdx.x / CH;
    if (g < G) {
        const float* in[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) in[v] = J.in[v];
        const int col = J.x0 + 4 * c;
        const uint32_t bytes = 4u * (uint32_t)max(0, min(4, J.nx + 8 - col));  // the tensor maps' nx + 8 columns
        const int rows = J.ny + 4 - J.y0;                                       // and ny + 4 rows
        long long gi = (long long)(J.y0 + g) * J.pitch + col;
        const long long gstep = (long long)G * J.pitch;
        float* dst = Qs + g * SP + 4 * c;
        for (int t = g; t < TR; t += G, gi += gstep, dst += G * SP) {
            const bool in_rows = t < rows;
#pragma unroll
            for (int v = 0; v < NV; ++v) cp_async16(dst + v * PS, in[v] + (in_rows ? gi : 0), in_rows ? bytes : 0u);
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

__device__ __forceinline__ float sign_x(int v) { return v == 1 ? -1.0f : 1.0f; }
__device__ __forceinline__ float sign_y(int v) { return v == 2 ? -1.0f : 1.0f; }

// Ghost cells of a tile that reaches the domain boundary, with readBlock's
// semantics (GPUSimulators/cuda/common.h:248-351): periodic sides read the
// wrapped cell from global memory, then reflective sides mirror interior cells
// with the normal momentum negated, north, south, east, west in turn.
// Dirichlet ghosts keep the stored values the TMA load brought in.
template <int NV, int W, int H, int NT, int SP = W + 8>
__device__ void apply_boundary(float* Qs, const TileJob& J) {
    constexpr int TR = H + 4, PS = SP * TR;
    const int nx = J.nx, ny = J.ny, bc = J.bc, x0 = J.x0, y0 = J.y0;
    const bool pw = bc_west(bc) == BC_PERIODIC, pe = bc_east(bc) == BC_PERIODIC;
    const bool ps = bc_south(bc) == BC_PERIODIC, pn = bc_north(bc) == BC_PERIODIC;
    if (pw || pe || ps || pn) {
        for (int i = threadIdx.x; i < TR * SP; i += NT) {
            const int t = i / SP, s = i - t * SP;
            const int x = x0 - 4 + s, y = y0 - 2 + t;
            if (x < -2 || x >= nx + 2 || y < -2 || y >= ny + 2) continue;
            int xs = x, ys = y;
            if (x < 0 && pw) xs = x + nx;
            else if (x >= nx && pe) xs = x - nx;
            if (y < 0 && ps) ys = y + ny;
            else if (y >= ny && pn) ys = y - ny;
            if (xs == x && ys == y) continue;
            const long long gi = cell_index(ys, xs, J.pitch);
#pragma unroll
            for (int v = 0; v < NV; ++v) Qs[v * PS + i] = __ldg(J.in[v] + gi);
        }
        __syncthreads();
    }
    // Tile row of domain row y: t = y - y0 + 2; tile column of x: s = x - x0 + 4.
    if (bc_north(bc) == BC_REFLECTIVE && y0 + H + 2 > ny) {
        for (int i = threadIdx.x; i < 2 * SP; i += NT) {
            const int m = i / SP, s = i - m * SP;
            const int t = ny + m - y0 + 2, ts = ny - 1 - m - y0 + 2;
            if (t < TR) {
#pragma unroll
                for (int v = 0; v < NV; ++v) Qs[v * PS + t * SP + s] = sign_y(v) * Qs[v * PS + ts * SP + s];
            }
        }
        __syncthreads();
    }
    if (bc_south(bc) == BC_REFLECTIVE && y0 == 0) {
        for (int i = threadIdx.x; i < 2 * SP; i += NT) {
            const int m = i / SP, s = i - m * SP;
            const int t = -1 - m + 2, ts = m + 2;
            if (ts < TR) {
#pragma unroll
                for (int v = 0; v < NV; ++v) Qs[v * PS + t * SP + s] = sign_y(v) * Qs[v * PS + ts * SP + s];
            }
        }
        __syncthreads();
    }
    if (bc_east(bc) == BC_REFLECTIVE && x0 + W + 2 > nx) {
        for (int i = threadIdx.x; i < 2 * TR; i += NT) {
            const int m = i / TR, t = i - m * TR;
            const int s = nx + m - x0 + 4, ss = nx - 1 - m - x0 + 4;
            if (s < SP) {
#pragma unroll
                for (int v = 0; v < NV; ++v) Qs[v * PS + t * SP + s] = sign_x(v) * Qs[v * PS + t * SP + ss];
            }
        }
        __syncthreads();
    }
    if (bc_west(bc) == BC_REFLECTIVE && x0 == 0) {
        for (int i = threadIdx.x; i < 2 * TR; i += NT) {
            const int m = i / TR, t = i - m * TR;
            const int s = -1 - m + 4, ss = m + 4;
            if (ss < SP) {
#pragma unroll
                for (int v = 0; v < NV; ++v) Qs[v * PS + t * SP + s] = sign_x(v) * Qs[v * PS + t * SP + ss];
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ line walkers

// Variable slot of logical component v along a line: y lines see (h, hv, hu)
// ("transposing" the domain, GPUSimulators/cuda/SWE2D_KP07_dimsplit.cu:81-107).
template <bool SWAP> __device__ __forceinline__ constexpr int vslot(int v) {
    return SWAP ? (v == 1 ? 2 : (v == 2 ? 1 : v)) : v;
}

template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void ld_cell(const float* line, int k, int step, float (&q)[NV]) {
    const float* p = line + k * step;
#pragma unroll
    for (int v = 0; v < NV; ++v) q[v] = p[vslot<SWAP>(v) * PS];
}

template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void st_cell(float* line, int k, int step, const float (&q)[NV]) {
    float* p = line + k * step;
#pragma unroll
    for (int v = 0; v < NV; ++v) p[vslot<SWAP>(v) * PS] = q[v];
}

// Two lines walked side by side: the second line starts d2 floats after the
// first; lane x of a pair is the first line, lane y the second.
template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void ld_cell(const float* line, int k, int step, int d2, f2 (&q)[NV]) {
    const float* p = line + k * step;
#pragma unroll
    for (int v = 0; v < NV; ++v) q[v] = f2{p[vslot<SWAP>(v) * PS], p[vslot<SWAP>(v) * PS + d2]};
}

template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void st_cell(float* line, int k, int step, int d2, const f2 (&q)[NV]) {
    float* p = line + k * step;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        p[vslot<SWAP>(v) * PS] = q[v].x;
        p[vslot<SWAP>(v) * PS + d2] = q[v].y;
    }
}

template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void ld_cell(const float* line, int k, int step, int, float (&q)[NV]) {
    ld_cell<NV, SWAP, PS>(line, k, step, q);
}

template <int NV, bool SWAP, int PS>
__device__ __forceinline__ void st_cell(float* line, int k, int step, int, const float (&q)[NV]) {
    st_cell<NV, SWAP, PS>(line, k, step, q);
}

// Physics policies for the MUSCL-Hancock walker; N is float (one line per
// thread) or f2 (two lines per thread).
template <class N>
struct SwePhys {
    static constexpr int NV = 3;
    using Num = N;
    using Face = SweFaceT<N>;
    N theta2, g, half_g, k2;  // theta2 = 2 * theta (swe_muscl_hancock)
    __device__ __forceinline__ void recon(const N (&qm)[3], const N (&q0)[3], const N (&qp)[3], N (&bd)[3], Face& w,
                                          Face& e) const {
        swe_muscl_hancock(qm, q0, qp, bd, theta2, g, half_g, k2, w, e);
    }
    template <bool HLLF> __device__ __forceinline__ static void flux(const Face& l, const Face& r, N (&F)[3]) {
        if (HLLF) swe_hll(l, r, F);
        else swe_central_upwind(l, r, F);
    }
};

template <class N>
struct EulerPhys {
    static constexpr int NV = 4;
    using Num = N;
    using Face = EulerFaceT<N>;
    N theta2, gamma, gm1, k2;  // theta2 = 2 * theta, gm1 = gamma - 1
    __device__ __forceinline__ void recon(const N (&qm)[4], const N (&q0)[4], const N (&qp)[4], N (&bd)[4], Face& w,
                                          Face& e) const {
        euler_muscl_hancock(qm, q0, qp, bd, theta2, gamma, gm1, k2, w, e);
    }
    template <bool HLLF> __device__ __forceinline__ static void flux(const Face& l, const Face& r, N (&F)[4]) {
        if (HLLF) euler_hll(l, r, F);
        else euler_central_upwind(l, r, F);
    }
};

// One MUSCL-Hancock window step at cell c: shift in Q[c+1], reconstruct c,
// flux at c-1/2, update cell c-1 (GPUSimulators/cuda/common.h:444-475).
template <class Phys, bool HLLF, bool SWAP, int PS, class N = typename Phys::Num>
__device__ __forceinline__ void mh_step(float* line, int step, int d2, int c, N (&qm)[Phys::NV], N (&q0)[Phys::NV],
                                        N (&qp)[Phys::NV], const N (&qn)[Phys::NV], N (&bd)[Phys::NV],
                                        typename Phys::Face& eL, N (&Fprev)[Phys::NV], const Phys& P, N kdx,
                                        bool update) {
    constexpr int NV = Phys::NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        qm[v] = q0[v];
        q0[v] = qp[v];
        qp[v] = qn[v];
    }
    typename Phys::Face w, e;
    P.recon(qm, q0, qp, bd, w, e);
    N F[NV];
    Phys::template flux<HLLF>(eL, w, F);
    if (update) {
        N out[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v] = ffma(fsub(Fprev[v], F[v]), kdx, qm[v]);
        st_cell<NV, SWAP, PS>(line, c - 1, step, d2, out);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) Fprev[v] = F[v];
    eL = e;
}

// Updates cells [a, b) of a line (of two lines, d2 floats apart, for f2) in
// place.  pre holds Q[a-2], Q[a-1], Q[b], Q[b+1].
template <class Phys, bool HLLF, bool SWAP, int PS, class N = typename Phys::Num>
__device__ __forceinline__ void walk_mh(float* line, int step, int d2, int a, int b, const N (&pre)[4][Phys::NV],
                                        const Phys& P, N kdx) {
    constexpr int NV = Phys::NV;
    N qm[NV], q0[NV], qp[NV], qn[NV], Fprev[NV], bd[NV];
    typename Phys::Face eL;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        q0[v] = pre[0][v];
        qp[v] = pre[1][v];
        Fprev[v] = splat<N>(0.0f);
    }
    // c = a-1: reconstruct only
    ld_cell<NV, SWAP, PS>(line, a, step, d2, qn);
    {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            qm[v] = q0[v];
            q0[v] = qp[v];
            qp[v] = qn[v];
            bd[v] = fmul(fsub(q0[v], qm[v]), P.theta2);
        }
        typename Phys::Face w;
        P.recon(qm, q0, qp, bd, w, eL);
    }
    // c = a: first face, no update
    ld_cell<NV, SWAP, PS>(line, a + 1, step, d2, qn);
    mh_step<Phys, HLLF, SWAP, PS>(line, step, d2, a, qm, q0, qp, qn, bd, eL, Fprev, P, kdx, false);
    // unrolled by the window's length, so the rotation of the three-cell
    // window becomes register renaming instead of moves
#pragma unroll 3
    for (int c = a + 1; c < b - 1; ++c) {
        ld_cell<NV, SWAP, PS>(line, c + 1, step, d2, qn);
        mh_step<Phys, HLLF, SWAP, PS>(line, step, d2, c, qm, q0, qp, qn, bd, eL, Fprev, P, kdx, true);
    }
    mh_step<Phys, HLLF, SWAP, PS>(line, step, d2, b - 1, qm, q0, qp, pre[2], bd, eL, Fprev, P, kdx, true);
    mh_step<Phys, HLLF, SWAP, PS>(line, step, d2, b, qm, q0, qp, pre[3], bd, eL, Fprev, P, kdx, true);
}

// Two-point flux walker (FORCE, HLL: GPUSimulators/cuda/SWE2D_FORCE.cu:29-81,
// SWE2D_HLL.cu:32-86).  pre holds Q[a-1] (slot 1) and Q[b] (slot 2).
// For HLL, VAR picks the flux: 0 HLL, 1 HLLC, 2 Godunov centred.
template <int SCHEME, bool SWAP, int PS, int VAR>
__device__ __forceinline__ void walk_2pt(float* line, int step, int a, int b, const float (&pre)[4][3], float g,
                                         float half_g, float kx, float kw, float kdx) {
    auto face_flux = [&](const SweFace& l, const SweFace& r, float (&F)[3]) {
        if constexpr (SCHEME == FORCE) swe_force(l, r, g, half_g, kx, kw, F);
        else if constexpr (VAR == 1) swe_hllc(l, r, F);
        else if constexpr (VAR == 2) swe_godc(l, r, g, half_g, kdx, F);
        else swe_hll(l, r, F);
    };
    SweFace sL = swe_face(pre[1][0], pre[1][1], pre[1][2], g, half_g);
    float qa[3];
    ld_cell<3, SWAP, PS>(line, a, step, qa);
    SweFace s = swe_face(qa[0], qa[1], qa[2], g, half_g);
    float Fprev[3];
    face_flux(sL, s, Fprev);
    float qprev[3] = {qa[0], qa[1], qa[2]};
    sL = s;
#pragma unroll 2
    for (int c = a + 1; c <= b; ++c) {
        float q[3];
        if (c < b) {
            ld_cell<3, SWAP, PS>(line, c, step, q);
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v) q[v] = pre[2][v];
        }
        s = swe_face(q[0], q[1], q[2], g, half_g);
        float F[3];
        face_flux(sL, s, F);
        float out[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = fmaf(Fprev[v] - F[v], kdx, qprev[v]);
        st_cell<3, SWAP, PS>(line, c - 1, step, out);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            Fprev[v] = F[v];
            qprev[v] = q[v];
        }
        sL = s;
    }
}

// WAF walker (GPUSimulators/cuda/SWE2D_WAF.cu:35-87): the flux at c-1/2 uses
// cells c-2 .. c+1; per-cell quantities and the star depths of neighbouring
// pairs are carried along the window.  N = f2 walks two lines d2 floats apart.
template <bool SWAP, int PS, int LIM, class N>
__device__ __forceinline__ void walk_waf(float* line, int step, int d2, int a, int b, const N (&pre)[4][3], N g,
                                         N half_g, N inv_g, N dtdx, N kdx, float beta) {
    constexpr int limiter = LIM;
    WafCellT<N> C0 = waf_cell(pre[0], g, half_g);
    WafCellT<N> C1 = waf_cell(pre[1], g, half_g);
    N q[3];
    ld_cell<3, SWAP, PS>(line, a, step, d2, q);
    WafCellT<N> C2 = waf_cell(q, g, half_g);
    ld_cell<3, SWAP, PS>(line, a + 1, step, d2, q);
    WafCellT<N> C3 = waf_cell(q, g, half_g);
    N hs01 = waf_h_star(C0, C1, inv_g), hs12 = waf_h_star(C1, C2, inv_g), hs23 = waf_h_star(C2, C3, inv_g);
    N Fprev[3];
    waf_flux(C0, C1, C2, C3, hs01, hs12, hs23, dtdx, Fprev, limiter, beta);  // face a-1/2
#pragma unroll 4
    for (int c = a + 1; c <= b; ++c) {
        if (c + 1 < b) {
            ld_cell<3, SWAP, PS>(line, c + 1, step, d2, q);
        } else {
            // a select, not pre[k]: a run-time index would put pre in local memory
            const bool first = (c + 1 == b);
#pragma unroll
            for (int v = 0; v < 3; ++v) q[v] = first ? pre[2][v] : pre[3][v];
        }
        C0 = C1;
        C1 = C2;
        C2 = C3;
        C3 = waf_cell(q, g, half_g);
        hs01 = hs12;
        hs12 = hs23;
        hs23 = waf_h_star(C2, C3, inv_g);
        N F[3];
        waf_flux(C0, C1, C2, C3, hs01, hs12, hs23, dtdx, F, limiter, beta);  // face c-1/2
        N out[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) out[v] = ffma(fsub(Fprev[v], F[v]), kdx, C1.q[v]);
        st_cell<3, SWAP, PS>(line, c - 1, step, d2, out);
#pragma unroll
        for (int v = 0; v < 3; ++v) Fprev[v] = F[v];
    }
}

// Per-scheme parameters of one sweep direction.  The ratios of the time step
// to the cell size are formed once per sweep, here, for every walker (one
// line or two lines per thread), so each tile configuration uses the same
// bits.
struct SweepPar {
    float theta, g, half_g, inv_g, gamma;
    float kdt;   // kernel dt
    float dxx;   // cell size along the sweep
    float kdx;   // kdt / dxx
    float k2;    // kdt / (2 dxx)
    float beta;   // parameter of the Osher and Sweby limiters
    __device__ __forceinline__ void set_direction(float cell) {
        dxx = cell;
        kdx = fdiv_fast(kdt, cell);
        k2 = fmul(kdx, 0.5f);
    }
};

// VAR: HLL's flux variant or WAF's limiter (walk_2pt, flux_limiter); 0 is the
// reference's.  It is a template parameter so that each kernel inlines one.
template <int SCHEME, bool SWAP, int PS, int VAR>
__device__ __forceinline__ void walk_line(float* line, int step, int a, int b, const float (&pre)[4][(SCHEME == EE2D) ? 4 : 3],
                                          const SweepPar& p) {
    const float kdx = p.kdx;
    if constexpr (SCHEME == KP07_DIMSPLIT || SCHEME == HLL2) {
        const SwePhys<float> P{2.0f * p.theta, p.g, p.half_g, p.k2};
        walk_mh<SwePhys<float>, SCHEME == HLL2, SWAP, PS>(line, step, 0, a, b, pre, P, kdx);
    } else if constexpr (SCHEME == EE2D) {
        const EulerPhys<float> P{2.0f * p.theta, p.gamma, fsub(p.gamma, 1.0f), p.k2};
        // x sweeps use HLL, y sweeps central-upwind (GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:62, :106)
        walk_mh<EulerPhys<float>, !SWAP, SWAP, PS>(line, step, 0, a, b, pre, P, kdx);
    } else if constexpr (SCHEME == WAF) {
        walk_waf<SWAP, PS, VAR>(line, step, 0, a, b, pre, p.g, p.half_g, p.inv_g, kdx, kdx, p.beta);
    } else {
        walk_2pt<SCHEME, SWAP, PS, VAR>(line, step, a, b, pre, p.g, p.half_g, fdiv_fast(p.dxx, fmul(2.0f, p.kdt)),
                                        p.k2, kdx);
    }
}

// Two lines, d2 floats apart, walked side by side in packed arithmetic
// (the MUSCL-Hancock schemes).  Each cell gets the same bits as walk_line.
template <int SCHEME, bool SWAP, int PS, int VAR>
__device__ __forceinline__ void walk_line2(float* line, int step, int d2, int a, int b,
                                           const f2 (&pre)[4][(SCHEME == EE2D) ? 4 : 3], const SweepPar& p) {
    static_assert(SCHEME == KP07_DIMSPLIT || SCHEME == HLL2 || SCHEME == EE2D || SCHEME == WAF,
                  "packed walkers: MUSCL-Hancock schemes and WAF");
    const f2 kdx = splat<f2>(p.kdx);
    if constexpr (SCHEME == WAF) {
        walk_waf<SWAP, PS, VAR>(line, step, d2, a, b, pre, splat<f2>(p.g), splat<f2>(p.half_g), splat<f2>(p.inv_g),
                                kdx, kdx, p.beta);
    } else if constexpr (SCHEME == EE2D) {
        const EulerPhys<f2> P{splat<f2>(2.0f * p.theta), splat<f2>(p.gamma), splat<f2>(fsub(p.gamma, 1.0f)),
                              splat<f2>(p.k2)};
        walk_mh<EulerPhys<f2>, !SWAP, SWAP, PS>(line, step, d2, a, b, pre, P, kdx);
    } else {
        const SwePhys<f2> P{splat<f2>(2.0f * p.theta), splat<f2>(p.g), splat<f2>(p.half_g), splat<f2>(p.k2)};
        walk_mh<SwePhys<f2>, SCHEME == HLL2, SWAP, PS>(line, step, d2, a, b, pre, P, kdx);
    }
}

// x sweep over tile rows [t0, t1): interior columns updated in place.
// LPT = 2: a thread walks rows t and t + (t1 - t0)/2 side by side.
template <int SCHEME, int NV, int W, int H, int NT, int VAR, int LPT>
__device__ __forceinline__ void sweep_x(float* Qs, int t0, int t1, const SweepPar& p) {
    constexpr int SP = split_pitch(W), PS = SP * (H + 4), NSEG = split_nseg_x(W), R = W / NSEG;
    const int item = threadIdx.x;
    const int nlines = (t1 - t0) / LPT;
    const bool has = item < nlines * NSEG;
    const int t = t0 + item / NSEG, seg = item % NSEG;
    const int a = 4 + seg * R, b = a + R;
    float* line = Qs + t * SP;
    if constexpr (LPT == 1) {
        float pre[4][NV];
        if (has) {
            ld_cell<NV, false, PS>(line, a - 2, 1, pre[0]);
            ld_cell<NV, false, PS>(line, a - 1, 1, pre[1]);
            ld_cell<NV, false, PS>(line, b, 1, pre[2]);
            ld_cell<NV, false, PS>(line, b + 1, 1, pre[3]);
        }
        __syncthreads();
        if (has) walk_line<SCHEME, false, PS, VAR>(line, 1, a, b, pre, p);
    } else {
        const int d2 = nlines * SP;
        f2 pre[4][NV];
        if (has) {
            ld_cell<NV, false, PS>(line, a - 2, 1, d2, pre[0]);
            ld_cell<NV, false, PS>(line, a - 1, 1, d2, pre[1]);
            ld_cell<NV, false, PS>(line, b, 1, d2, pre[2]);
            ld_cell<NV, false, PS>(line, b + 1, 1, d2, pre[3]);
        }
        __syncthreads();
        if (has) walk_line2<SCHEME, false, PS, VAR>(line, 1, d2, a, b, pre, p);
    }
    __syncthreads();
}

// y sweep over tile columns [s0, s1): interior rows updated in place.
// LPT = 2: a thread walks columns s and s + (s1 - s0)/2 side by side.
template <int SCHEME, int NV, int W, int H, int NT, int VAR, int LPT>
__device__ __forceinline__ void sweep_y(float* Qs, int s0, int s1, const SweepPar& p) {
    constexpr int SP = split_pitch(W), PS = SP * (H + 4);
    constexpr int NSEG = NT * LPT / (W + 4), R = H / NSEG;
    const int ncols = (s1 - s0) / LPT;
    const int item = threadIdx.x;
    const bool has = item < ncols * NSEG;
    const int s = s0 + item % ncols, seg = item / ncols;
    const int a = 2 + seg * R, b = a + R;
    float* line = Qs + s;
    if constexpr (LPT == 1) {
        float pre[4][NV];
        if (has) {
            ld_cell<NV, true, PS>(line, a - 2, SP, pre[0]);
            ld_cell<NV, true, PS>(line, a - 1, SP, pre[1]);
            ld_cell<NV, true, PS>(line, b, SP, pre[2]);
            ld_cell<NV, true, PS>(line, b + 1, SP, pre[3]);
        }
        __syncthreads();
        if (has) walk_line<SCHEME, true, PS, VAR>(line, SP, a, b, pre, p);
    } else {
        const int d2 = ncols;
        f2 pre[4][NV];
        if (has) {
            ld_cell<NV, true, PS>(line, a - 2, SP, d2, pre[0]);
            ld_cell<NV, true, PS>(line, a - 1, SP, d2, pre[1]);
            ld_cell<NV, true, PS>(line, b, SP, d2, pre[2]);
            ld_cell<NV, true, PS>(line, b + 1, SP, d2, pre[3]);
        }
        __syncthreads();
        if (has) walk_line2<SCHEME, true, PS, VAR>(line, SP, d2, a, b, pre, p);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ split-scheme stage kernel

// Scheme constants of a split-scheme tile.
struct SplitPar {
    float dx, dy, g, gamma, theta;
    float kdt;  // kernel dt of this substep
    int substep;
    float beta;  // parameter of the Osher and Sweby limiters
};

// Load, ghost cells, both sweeps and copy-out of one tile of a split scheme
// (FORCE, HLL, HLL2, WAF, KP07_dimsplit, EE2D).  Accumulates the tile's CFL
// minimum and FP64 sums into the per-thread values.  Returns false if the tile
// load gave up (nothing was written).
// ASYNC_LOAD (batched kernels): the tile comes in through load_tile_async
// instead of the TMA (bar, phase, init_bar, err and polls are then unused).
// HEALTH (batched kernels): with `health` set, *unhealthy becomes true if any
// written cell holds a non-finite value or a non-positive depth (density).
template <int SCHEME, int W, int H, int NT, bool ASYNC_LOAD = false, int VAR = 0, int LPT = 1, bool HEALTH = false>
__device__ bool process_tile_dimsplit(float* Qs, uint64_t* bar, uint32_t phase, bool init_bar, const TileJob& J,
                                      const SplitPar& P, bool do_cfl, bool sums, int* err, float& my_cfl,
                                      double (&my_sums)[(SCHEME == EE2D) ? 4 : 3], uint32_t polls = kWaitPolls,
                                      bool health = false, bool* unhealthy = nullptr) {
    constexpr int NV = (SCHEME == EE2D) ? 4 : 3;
    constexpr int G = (SCHEME == FORCE || SCHEME == HLL) ? 1 : 2;
    constexpr int SP = split_pitch(W), TR = H + 4, PS = SP * TR, NSEG_X = split_nseg_x(W);
    static_assert(W % NSEG_X == 0 && (W / NSEG_X) % 2 == 1 && SP % 32 == (NSEG_X == 4 ? 4 : 8),
                  "row segments must be odd and the pitch 4 (8) mod 32 for conflict-free x sweeps");
    static_assert(TR * NSEG_X <= NT * LPT, "one x-sweep segment (LPT lines) per thread");
    static_assert((NT * LPT) / (W + 4) >= 1 && H % ((NT * LPT) / (W + 4)) == 0, "y-sweep segments must tile the block");
    static_assert(LPT == 1 || (LPT == 2 && H % 2 == 0 &&
                               (SCHEME == KP07_DIMSPLIT || SCHEME == HLL2 || SCHEME == EE2D || SCHEME == WAF)),
                  "two lines per thread: MUSCL-Hancock schemes and WAF, with an even number of tile rows");
    if constexpr (ASYNC_LOAD) {
        load_tile_async<NV, SP, TR, NT>(Qs, J);
    } else {
        if (!load_tile<NV, SP, TR>(Qs, J.tmap, J.x0, J.y0, bar, phase, init_bar, err, polls)) return false;
    }
    const int x0 = J.x0, y0 = J.y0;
    if (x0 == 0 || x0 + W + 2 > J.nx || y0 == 0 || y0 + H + 2 > J.ny) apply_boundary<NV, W, H, NT, SP>(Qs, J);

    SweepPar p;
    p.theta = P.theta;
    p.g = P.g;
    p.half_g = fmul(0.5f, P.g);
    p.inv_g = frcp_fast(P.g);
    p.gamma = P.gamma;
    p.kdt = P.kdt;
    p.beta = P.beta;
    const bool x_first = (SCHEME == FORCE || SCHEME == HLL) ? true : (P.substep == 0);
    if (x_first) {
        p.set_direction(P.dx);
        sweep_x<SCHEME, NV, W, H, NT, VAR, LPT>(Qs, 2 - G, H + 2 + G, p);
        p.set_direction(P.dy);
        sweep_y<SCHEME, NV, W, H, NT, VAR, LPT>(Qs, 4, W + 4, p);
    } else {
        p.set_direction(P.dy);
        sweep_y<SCHEME, NV, W, H, NT, VAR, LPT>(Qs, 4 - G, W + 4 + G, p);
        p.set_direction(P.dx);
        sweep_x<SCHEME, NV, W, H, NT, VAR, LPT>(Qs, 2, H + 2, p);
    }

    // copy-out of the interior (+ gravity source, CFL, sums); the output plane
    // pointers are read once (for batched kernels they live in global memory,
    // where a store through a float pointer could otherwise force a reload)
    constexpr int QW = W / 4;
    const float gg = (SCHEME == EE2D) ? P.gamma : P.g;
    float* outp[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) outp[v] = J.out[v];
    for (int i = threadIdx.x; i < H * QW; i += NT) {
        const int r = i / QW, q = i - r * QW;
        const int y = y0 + r, x = x0 + 4 * q;
        if (y >= J.ny || x >= J.nx) continue;
        float4 val[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) val[v] = *reinterpret_cast<const float4*>(Qs + v * PS + (r + 2) * SP + 4 + 4 * q);
        if (SCHEME == EE2D) {
            if (P.g > 0.0f) {
                // gravity source (GPUSimulators/cuda/EE2D_KP07_dimsplit.cu:197-205)
                const float gsrc = P.g;
                float* r0 = &val[0].x;
                float* r2 = &val[2].x;
                float* r3 = &val[3].x;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float rho_v = r2[j];
                    r2[j] = r2[j] - gsrc * r0[j] * P.kdt;
                    r3[j] = r3[j] - gsrc * rho_v * P.kdt;
                }
            }
        }
        const long long gi = cell_index(y, x, J.pitch);
        const int nvalid = min(4, J.nx - x);
        if (nvalid == 4) {
#pragma unroll
            for (int v = 0; v < NV; ++v) *reinterpret_cast<float4*>(outp[v] + gi) = val[v];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const float* e = &val[v].x;
                for (int j = 0; j < nvalid; ++j) outp[v][gi + j] = e[j];
            }
        }
        if constexpr (HEALTH) {
            if (health) {
                bool bad = false;
                if (nvalid == 4) {
                    // NaN-propagating minimum of the depths (densities) and
                    // maximum of the other variables' magnitudes: the same
                    // verdict as the per-value tests below, in fewer instructions
                    const float hmin = vmin_nan(vmin3_nan(val[0].x, val[0].y, val[0].z), val[0].w);
                    float qmax = 0.0f;
#pragma unroll
                    for (int v = 1; v < NV; ++v)
                        qmax = vmax3_nan(qmax, vmax3_nan(fabsf(val[v].x), fabsf(val[v].y), fabsf(val[v].z)),
                                         fabsf(val[v].w));
                    bad = !(hmin > 0.0f) || !(qmax < __int_as_float(0x7f800000));
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (j < nvalid) {
                            bad |= !((&val[0].x)[j] > 0.0f);
#pragma unroll
                            for (int v = 1; v < NV; ++v)
                                bad |= !(fabsf((&val[v].x)[j]) < __int_as_float(0x7f800000));
                        }
                    }
                }
                if (bad) *unhealthy = true;
            }
        }
        if (do_cfl || sums) {
            const float* h = &val[0].x;
            const float* hu = &val[1].x;
            const float* hv = &val[2].x;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j < nvalid) {
                    if (do_cfl) my_cfl = fminf(my_cfl, cell_cfl(h[j], hu[j], hv[j], P.dx, P.dy, gg));
                    if (sums) {
#pragma unroll
                        for (int v = 0; v < NV; ++v) my_sums[v] += (double)(&val[v].x)[j];
                    }
                }
            }
        }
    }
    return true;
}

template <int SCHEME, int W, int H, int NT, int VAR = 0, int LPT = 1>
__global__ void __launch_bounds__(NT) dimsplit_stage_kernel(const __grid_constant__ StageArgs A) {
    constexpr int NV = (SCHEME == EE2D) ? 4 : 3;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* Qs = reinterpret_cast<float*>(smem_raw);
    __shared__ __align__(8) uint64_t bar;

    grid_dependency_wait();  // the previous substep's state and control block
    StepCtl sc = read_step(A);
    if (!sc.active) return;
    if (SCHEME == WAF) sc.do_cfl = false;  // WAFKernel has no CFL output (GPUSimulators/cuda/SWE2D_WAF.cu:103-119)
    float my_cfl = __int_as_float(0x7f800000);
    double my_sums[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) my_sums[v] = 0.0;
    const bool sums = A.want_sums && A.is_last;

    TileJob J;
    J.tmap = &A.tmap[sc.cur][0];
    J.in = A.buf[sc.cur];
    J.out = A.buf[sc.cur ^ 1];
    J.nx = A.nx;
    J.ny = A.ny;
    J.pitch = A.pitch;
    J.bc = A.bc;
    J.x0 = blockIdx.x * W;
    J.y0 = (blockIdx.y + A.tile_row0) * H;
    SplitPar P{A.dx, A.dy, A.g, A.gamma, A.theta, sc.dt * A.dt_scale, A.substep, A.variant_beta};
    process_tile_dimsplit<SCHEME, W, H, NT, false, VAR, LPT>(Qs, &bar, 0, true, J, P, sc.do_cfl, sums, &A.ctl->error,
                                                             my_cfl, my_sums, wait_polls(A.wait_limit));
    stage_epilogue<NT, NV>(A, sc, my_cfl, my_sums, sums);
}

// ------------------------------------------------------------------ unsplit stage kernel (LxF, KP07)

__device__ __forceinline__ SweFace shfl_up_face(const SweFace& f, int d) {
    SweFace r;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        r.q[v] = __shfl_up_sync(0xffffffffu, f.q[v], d);
        r.f[v] = __shfl_up_sync(0xffffffffu, f.f[v], d);
    }
    r.u = __shfl_up_sync(0xffffffffu, f.u, d);
    r.c = __shfl_up_sync(0xffffffffu, f.c, d);
    return r;
}

// Scheme constants of an unsplit tile.
struct UnsplitPar {
    float dx, dy, g, theta;
    float kdt;    // kernel dt of this stage
    int substep;  // RK stage (KP07)
    int order;    // RK order (KP07)
};

// Load, ghost cells, the one-pass update and the stores of one tile of an
// unsplit scheme (LxF, KP07); the per-thread CFL minimum and FP64 sums are
// accumulated.  Returns false if the tile load gave up (nothing was written).
// ASYNC_LOAD (batched kernels): the tile comes in through load_tile_async.
// HEALTH (batched kernels): with `health` set, *unhealthy becomes true if a
// written cell holds a non-finite value or a non-positive depth.
template <int SCHEME, int W, int H, int NT, bool ASYNC_LOAD = false, bool HEALTH = false>
__device__ bool process_tile_unsplit(float* Qs, uint64_t* bar, uint32_t phase, bool init_bar, const TileJob& J,
                                     const UnsplitPar& P, bool do_cfl, bool sums, int* err, float& my_cfl,
                                     double (&my_sums)[3], uint32_t polls = kWaitPolls, bool health = false,
                                     bool* unhealthy = nullptr) {
    constexpr int SP = W + 8, TR = H + 4, PS = SP * TR;
    constexpr int WX = W / 30, NSEG = NT / (32 * WX), R = H / NSEG;
    static_assert(W % 30 == 0 && NT % (32 * WX) == 0 && NSEG >= 1 && H % NSEG == 0,
                  "warps of 30 updated columns must tile the block");
    const int x0 = J.x0, y0 = J.y0;
    bool bad = false;
    if constexpr (ASYNC_LOAD) {
        load_tile_async<3, SP, TR, NT>(Qs, J);
    } else {
        if (!load_tile<3, SP, TR>(Qs, J.tmap, x0, y0, bar, phase, init_bar, err, polls)) return false;
    }
    {
        if (x0 == 0 || x0 + W + 2 > J.nx || y0 == 0 || y0 + H + 2 > J.ny) apply_boundary<3, W, H, NT>(Qs, J);
        const float kdt = P.kdt;
        const float g = P.g, half_g = fmul(0.5f, g), theta2 = fmul(2.0f, P.theta);
        const float k4x = fdiv_fast(P.dx, fmul(4.0f, kdt)), k4y = fdiv_fast(P.dy, fmul(4.0f, kdt));
        const float kdx = fdiv_fast(kdt, P.dx), kdy = fdiv_fast(kdt, P.dy);
        const bool blend = (SCHEME == KP07) && P.order == 2 && P.substep == 1;

        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int wx = warp % WX, seg = warp / WX;
        const int s = 3 + 30 * wx + lane;  // tile column of this lane
        const int x = x0 + s - 4;          // domain column
        const bool owner = lane >= 1 && lane <= 30;
        const int a = 2 + seg * R, b = a + R;  // tile rows updated by this segment

        // q of tile cell (t, c), components in (h, hu, hv) order
        auto qat = [&](int t, int c, float (&q)[3]) {
#pragma unroll
            for (int v = 0; v < 3; ++v) q[v] = Qs[v * PS + t * SP + c];
        };
        // y-face states of row t (south, north) from rows t-1, t, t+1 of this
        // column, components swapped to (h, hv, hu) as computeFluxG does
        // (GPUSimulators/cuda/SWE2D_KP07.cu:117-131).  The slope is formed at
        // twice its size (minmod_slope2); bd carries theta2*(q0 - qm) in and
        // theta2*(qp - q0) out, in q's component order, since a row's forward
        // difference is the next row's backward one.
        auto ystates = [&](const float (&qm)[3], const float (&q0)[3], const float (&qp)[3], float (&bd)[3],
                           SweFace& sf, SweFace& nf) {
            float sv[3], nv[3];
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const int k = (v == 0) ? 0 : 3 - v;  // (h, hv, hu)
                if (SCHEME == LXF) {
                    sv[v] = nv[v] = q0[k];
                } else {
                    const float f = fmul(fsub(qp[k], q0[k]), theta2);
                    const float sl2 = minmod3(bd[k], fsub(qp[k], qm[k]), f);
                    bd[k] = f;
                    sv[v] = fmaf(-0.25f, sl2, q0[k]);
                    nv[v] = fmaf(0.25f, sl2, q0[k]);
                }
            }
            sf = swe_face(sv[0], sv[1], sv[2], g, half_g);
            nf = (SCHEME == LXF) ? sf : swe_face(nv[0], nv[1], nv[2], g, half_g);
        };
        auto yflux = [&](const SweFace& l, const SweFace& r, float (&G)[3]) {
            float tmp[3];
            if (SCHEME == LXF) swe_lxf_2d(l, r, k4y, tmp);
            else swe_central_upwind(l, r, tmp);
            G[0] = tmp[0];  // back to (h, hu, hv)
            G[1] = tmp[2];
            G[2] = tmp[1];
        };

        // window: rows a-1, a, a+1 of this column
        float qm[3], q0[3], qp[3];
        qat(a - 1, s, qm);
        qat(a, s, q0);
        qat(a + 1, s, qp);
        SweFace s_cur, n_cur, n_prev;
        float bdy[3];
        {
            float qmm[3];
            qat(a - 2, s, qmm);
#pragma unroll
            for (int v = 0; v < 3; ++v) bdy[v] = fmul(fsub(qm[v], qmm[v]), theta2);
            SweFace sd;
            ystates(qmm, qm, q0, bdy, sd, n_prev);  // row a-1
        }
        ystates(qm, q0, qp, bdy, s_cur, n_cur);  // row a
        float Gs[3];
        yflux(n_prev, s_cur, Gs);  // south face of row a
        float* outp[3];  // read once (batched kernels keep them in global memory)
#pragma unroll
        for (int v = 0; v < 3; ++v) outp[v] = J.out[v];
        // unrolled by the row window's length: its rotation becomes renaming
#pragma unroll 3
        for (int t = a; t < b; ++t) {
            const int y = y0 + t - 2;
            const bool store = owner && x < J.nx && y < J.ny;
            const long long gi = cell_index(y, x, J.pitch);
            float old[3] = {0.0f, 0.0f, 0.0f};
            if (blend && store) {
#pragma unroll
                for (int v = 0; v < 3; ++v) old[v] = outp[v][gi];
            }
            // x faces of (t, s): west and east states
            SweFace fw, fe;
            if (SCHEME == LXF) {
                fw = fe = swe_face(q0[0], q0[1], q0[2], g, half_g);
            } else {
                float ql[3], qr[3], wv[3], ev[3];
                qat(t, s - 1, ql);
                qat(t, s + 1, qr);
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const float sl2 = minmod_slope2(ql[v], q0[v], qr[v], theta2);
                    wv[v] = fmaf(-0.25f, sl2, q0[v]);
                    ev[v] = fmaf(0.25f, sl2, q0[v]);
                }
                fw = swe_face(wv[0], wv[1], wv[2], g, half_g);
                fe = swe_face(ev[0], ev[1], ev[2], g, half_g);
            }
            const SweFace le = shfl_up_face(fe, 1);  // east state of the column to the left
            float Fw[3], Fe[3];
            if (SCHEME == LXF) swe_lxf_2d(le, fw, k4x, Fw);
            else swe_central_upwind(le, fw, Fw);
#pragma unroll
            for (int v = 0; v < 3; ++v) Fe[v] = __shfl_down_sync(0xffffffffu, Fw[v], 1);
            // y: states of row t+1, flux at the north face of row t
            float qn2[3];
            qat(t + 2, s, qn2);
            SweFace s_nxt, n_nxt;
            ystates(q0, qp, qn2, bdy, s_nxt, n_nxt);
            float Gn[3];
            yflux(n_cur, s_nxt, Gn);
            if (store) {
                float qn[3];
#pragma unroll
                for (int v = 0; v < 3; ++v) qn[v] = q0[v] + fmaf(Fw[v] - Fe[v], kdx, (Gs[v] - Gn[v]) * kdy);
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const float o = blend ? 0.5f * (old[v] + qn[v]) : qn[v];
                    outp[v][gi] = o;
                    if (sums) my_sums[v] += (double)o;
                    if constexpr (HEALTH) {
                        if (health) bad |= (v == 0) ? !(o > 0.0f) : !(fabsf(o) < __int_as_float(0x7f800000));
                    }
                }
                if (do_cfl) my_cfl = fminf(my_cfl, cell_cfl(qn[0], qn[1], qn[2], P.dx, P.dy, g));
            }
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                Gs[v] = Gn[v];
                qm[v] = q0[v];
                q0[v] = qp[v];
                qp[v] = qn2[v];
            }
            s_cur = s_nxt;
            n_cur = n_nxt;
        }
    }
    if constexpr (HEALTH) {
        if (bad) *unhealthy = true;
    }
    return true;
}

// One pass over the tile, as column walkers (GPUSimulators/cuda/SWE2D_LxF.cu:102-165,
// SWE2D_KP07.cu:136-232).  Lanes run along x: warp column wx of a row segment
// covers tile columns 3+30wx .. 34+30wx; lanes 1..30 update interior columns
// 30wx .. 30wx+29, lanes 0 and 31 supply the states of the columns beside
// them.  At each row a lane builds the west and east face states of its cell;
// the flux at its west face takes the east state of the lane to its left
// (warp shuffle), and its east-face flux is the west-face flux of the lane
// to its right, so each x face is computed once.  Along y each lane keeps a
// sliding window: the north face state of the row above and the flux at the
// south face carry over from the previous row.  The updated cells (KP07
// stage 2 blended with the old output) go straight to global memory.
template <int SCHEME, int W, int H, int NT>
__global__ void __launch_bounds__(NT) unsplit_stage_kernel(const __grid_constant__ StageArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* Qs = reinterpret_cast<float*>(smem_raw);
    __shared__ __align__(8) uint64_t bar;

    grid_dependency_wait();  // the previous stage's state and control block
    const StepCtl sc = read_step(A);
    if (!sc.active) return;
    float my_cfl = __int_as_float(0x7f800000);
    double my_sums[3] = {0.0, 0.0, 0.0};
    const bool sums = A.want_sums && A.is_last;

    TileJob J;
    J.tmap = &A.tmap[sc.cur][0];
    J.in = A.buf[sc.cur];
    J.out = A.buf[sc.cur ^ 1];
    J.nx = A.nx;
    J.ny = A.ny;
    J.pitch = A.pitch;
    J.bc = A.bc;
    J.x0 = blockIdx.x * W;
    J.y0 = (blockIdx.y + A.tile_row0) * H;
    const UnsplitPar P{A.dx, A.dy, A.g, A.theta, sc.dt * A.dt_scale, A.substep, A.order};
    process_tile_unsplit<SCHEME, W, H, NT>(Qs, &bar, 0, true, J, P, sc.do_cfl, sums, &A.ctl->error, my_cfl, my_sums,
                                           wait_polls(A.wait_limit));
    stage_epilogue<NT, 3>(A, sc, my_cfl, my_sums, sums);
}

// ------------------------------------------------------------------ batched persistent stage kernel

// One simulation of a batch, resident in device memory.  Its tiles are loaded
// with load_tile_async, so it carries no tensor maps.
struct alignas(64) BatchInstance {
    float* buf[2][4];
    SimCtl* ctl;
    float* block_cfl;    // one float per tile of this simulation
    double* block_sums;  // 4 doubles per tile
    int nx, ny, pitch, bc;
    int tiles_x, ntiles;
    float dx, dy, g, gamma, theta, dt_scale;
    float variant_beta;  // parameter of the Osher and Sweby limiters
};

struct BatchArgs {
    const BatchInstance* inst;
    SimCtl* ctl;          // control blocks, one per instance: inst[i].ctl == ctl + i
    const int2* work;     // (instance, tile within instance) per work item
    const int* nwork;     // number of work items (device scalar, updated between graph replays)
    int substep;
    int is_last;
    int want_sums;
    int order;  // RK order (KP07)
    int* err;
};

// The part of a work item's records a batched tile reads before its load: the
// first 48 bytes of the simulation's control block (read_step's words) and
// the instance record up to its last field, copied into shared memory by the
// CTA's first threads (BatchTileMeta).
constexpr int kInstPrefix = 144;
static_assert(offsetof(BatchInstance, variant_beta) + sizeof(float) <= kInstPrefix &&
                  kInstPrefix % 16 == 0 && sizeof(BatchInstance) >= kInstPrefix && sizeof(SimCtl) % 16 == 0,
              "the prefetched instance prefix holds every field, in whole 16-byte chunks");
struct alignas(64) BatchTileMeta {
    unsigned char inst[kInstPrefix];  // read as a BatchInstance (same alignment)
    int4 ctl[3];
};

// Issues (threads 0..11) the asynchronous copies of `job`'s metadata into m.
__device__ __forceinline__ void prefetch_tile_meta(BatchTileMeta& m, const BatchInstance* inst, const SimCtl* ctl,
                                                   int2 job) {
    constexpr int NI = kInstPrefix / 16;
    const int i = threadIdx.x;
    if (i < NI) {
        cp_async16(m.inst + 16 * i, reinterpret_cast<const char*>(inst + job.x) + 16 * i, 16);
    } else if (i < NI + 3) {
        cp_async16(&m.ctl[i - NI], reinterpret_cast<const char*>(ctl + job.x) + 16 * (i - NI), 16);
    }
}

// One tile of a batched launch: work item `job` (simulation, tile within it),
// whose control-block words and instance fields are in shared memory (M).
// Simulations that reached t_end are skipped (uniformly across the CTA).
template <int SCHEME, int W, int H, int NT, int VAR, int LPT>
__device__ __forceinline__ void batched_tile(float* Qs, uint64_t* bar, const BatchTileMeta& M, int2 job,
                                             const BatchArgs& B) {
    constexpr int NV = (SCHEME == EE2D) ? 4 : 3;
    const BatchInstance& I = *reinterpret_cast<const BatchInstance*>(M.inst);
    SimCtl* const ctl = B.ctl + job.x;
    StepCtl sc = step_from_words(M.ctl[0], M.ctl[1], M.ctl[2], false, 0.0f, false, B.is_last != 0);
    if (!sc.active) return;
    if (SCHEME == WAF) sc.do_cfl = false;
    float my_cfl = __int_as_float(0x7f800000);
    double my_sums[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) my_sums[v] = 0.0;
    const bool sums = B.want_sums && B.is_last;
    TileJob J;
    J.tmap = nullptr;
    J.in = I.buf[sc.cur];
    J.out = I.buf[sc.cur ^ 1];
    J.nx = I.nx;
    J.ny = I.ny;
    J.pitch = I.pitch;
    J.bc = I.bc;
    const int ty = job.y / I.tiles_x;
    J.x0 = (job.y - ty * I.tiles_x) * W;
    J.y0 = ty * H;
    bool unhealthy = false;
    if constexpr (SCHEME == LXF || SCHEME == KP07) {
        const UnsplitPar P{I.dx, I.dy, I.g, I.theta, sc.dt * I.dt_scale, B.substep, B.order};
        process_tile_unsplit<SCHEME, W, H, NT, true, true>(Qs, bar, 0, false, J, P, sc.do_cfl, sums, B.err, my_cfl,
                                                           my_sums, kWaitPolls, B.is_last != 0, &unhealthy);
    } else {
        const SplitPar P{I.dx, I.dy, I.g, I.gamma, I.theta, sc.dt * I.dt_scale, B.substep, I.variant_beta};
        process_tile_dimsplit<SCHEME, W, H, NT, true, VAR, LPT, true>(Qs, bar, 0, false, J, P, sc.do_cfl, sums,
                                                                      B.err, my_cfl, my_sums, kWaitPolls,
                                                                      B.is_last != 0, &unhealthy);
    }
    // ordered before this tile's arrival (tile_epilogue fences before it counts)
    if (__syncthreads_or(unhealthy) && threadIdx.x == 0) atomicOr(&ctl->bad, 1);
    tile_epilogue<NT, NV>(ctl, I.block_cfl, I.block_sums, job.y, I.ntiles, B.is_last != 0, false, sc, my_cfl,
                          my_sums, sums);
}

// Stage kernel of any scheme over a batch (one dimensional sweep of the split
// schemes, one RK stage of LxF and KP07): one launch covers the work list of
// all tiles of all simulations of the batch; each simulation keeps its own t,
// dt (its own CFL every 100 of its steps) and t_end, and its last tile
// finalises its control block exactly as the single-simulation kernel does.
// The work list and its length live in device memory, so one pair of captured
// CUDA graphs serves any batch composition.  Two forms of the walk:
//  * PERSIST = false: CTA w takes entry w; the host launches one CTA per entry
//    and sets the grid of the graphs' kernel nodes to the list's length when
//    the list changes.  The CTAs resident on an SM (four of 128 threads)
//    overlap one tile's metadata and tile loads with the others' sweeps, as
//    in the single-simulation kernels.
//  * PERSIST = true: a fixed grid of resident CTAs (occupancy x SMs) strides
//    over the list, copying the next tile's metadata into shared memory while
//    the current tile is computed.  Inside that loop the compiler keeps far
//    more registers live for the same sweeps (242 against 122 for the packed
//    60 x 60 tile, 184 against 80 for the one-line 124 x 28), so under the
//    128-register bound the packed form spills; on mixes of 128 grids with
//    sides of 64 to 1024 cells the one-tile form measured 14-49 % faster per
//    scheme, and the autotuner times both.
// At most 128 registers per thread (the launch bound), so that four 128-thread
// (two 256-thread) CTAs fit an SM as their shared tiles allow.
template <int SCHEME, int W, int H, int NT, int VAR = 0, int LPT = 1, bool PERSIST = false>
__global__ void __launch_bounds__(NT, 65536 / (NT * 128)) batched_stage_kernel(const __grid_constant__ BatchArgs B) {
    static_assert(NT >= 3 + kInstPrefix / 16, "one thread per copied 16-byte chunk");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* Qs = reinterpret_cast<float*>(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    __shared__ BatchTileMeta meta[PERSIST ? 2 : 1];
    grid_dependency_wait();  // the previous substep's states and control blocks
    const int n = *B.nwork;
    int w = blockIdx.x;
    if (w >= n) return;
    int2 job = B.work[w];
    if constexpr (!PERSIST) {
        prefetch_tile_meta(meta[0], B.inst, B.ctl, job);
        cp_async_wait_all();
        __syncthreads();
        batched_tile<SCHEME, W, H, NT, VAR, LPT>(Qs, &bar, meta[0], job, B);
    } else {
        // The work list is read two tiles ahead.  A control block read early
        // holds the values of this launch's start: it changes in this launch
        // only once every tile of its simulation has arrived, and the
        // prefetched tile has not.
        const int G = gridDim.x;
        int2 next = (w + G < n) ? B.work[w + G] : job;
        prefetch_tile_meta(meta[0], B.inst, B.ctl, job);
        cp_async_wait_all();
        __syncthreads();
        int slot = 0;
        for (; w < n; w += G) {
            const int2 next2 = (w + 2 * G < n) ? B.work[w + 2 * G] : next;
            if (w + G < n) prefetch_tile_meta(meta[slot ^ 1], B.inst, B.ctl, next);
            batched_tile<SCHEME, W, H, NT, VAR, LPT>(Qs, &bar, meta[slot], job, B);
            // the next tile's metadata has landed and every thread is done with
            // this slot, which the tile after next overwrites
            cp_async_wait_all();
            __syncthreads();
            slot ^= 1;
            job = next;
            next = next2;
        }
    }
}

}  // namespace fv
