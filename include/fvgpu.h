/*
 * fvgpu.h -- C ABI of libfvgpu.so, the B200 (sm_100a) implementation of the
 * GPUSimulators time-step path (babrodtk/FiniteVolumeGPU).
 *
 * Every entry point returns an int status (FV_OK == 0); the message of the
 * last failure on the calling thread is available from fv_last_error().
 * No C++ exception crosses this boundary.  All host arrays are float32,
 * C-ordered, row pitch given in elements.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project).
 */
#ifndef FVGPU_H
#define FVGPU_H

#include <stddef.h>

#if defined(__GNUC__)
#define FV_API __attribute__((visibility("default")))
#else
#define FV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FV_OK 0
#define FV_ERR_INVALID 1     /* bad argument: shape, size, pointer (reference: AssertionError) */
#define FV_ERR_UNSUPPORTED 2 /* e.g. Neumann boundaries (reference: NotImplementedError, Simulator.py:68-72) */
#define FV_ERR_CUDA 3        /* a CUDA runtime call failed */
#define FV_ERR_DEVICE 4      /* a kernel's bounded wait gave up; the simulation state is not trustworthy */
#define FV_ERR_NOMEM 5       /* device or pinned host allocation failed */

/* Scheme ids: the reference classes GPUSimulators/{LxF,FORCE,HLL,HLL2,WAF,KP07,
 * KP07_dimsplit,EE2D_KP07_dimsplit}.py. */
enum fv_scheme {
    FV_LXF = 0,
    FV_FORCE = 1,
    FV_HLL = 2,
    FV_HLL2 = 3,
    FV_WAF = 4,
    FV_KP07 = 5,
    FV_KP07_DIMSPLIT = 6,
    FV_EE2D_KP07_DIMSPLIT = 7
};

typedef struct fv_context fv_context;
typedef struct fv_sim fv_sim;

/* Scheme parameters (constructor keywords of the reference classes). */
typedef struct fv_params {
    float g;         /* gravitational acceleration (all classes) */
    float gamma;     /* ratio of specific heats (EE2D_KP07_dimsplit only) */
    float theta;     /* minmod parameter (HLL2, KP07, KP07_dimsplit, EE2D) */
    float cfl_scale; /* Courant number used by simulate() */
    int order;       /* Runge-Kutta order of KP07 (1 or 2) */
    int tile;        /* tile configuration index, or -1 for the scheme default */
    /* Options the reference defines but none of its schemes uses
     * (GPUSimulators/cuda/SWECommon.h:248-255, :334-387; limiters.h:84-118):
     * HLL's flux (0 HLL, 1 HLLC, 2 Godunov centred) or WAF's limiter (0 the
     * reference's generalized minmod with theta 1.9, 1 minmod, 2 superbee,
     * 3 van Leer, 4 van Albada 1, 5 van Albada 2, 6 monotonized central,
     * 7 Osher, 8 Sweby); 0 for every other scheme.  Each variant other
     * than 0 has one kernel of its own, and `tile` is then ignored. */
    int variant;
    float variant_beta; /* beta of the Osher and Sweby limiters */
} fv_params;

/* Library version (major*10000 + minor*100 + patch). */
FV_API int fv_version(void);

/* Message of the last failing call on this thread ("" if none). */
FV_API const char* fv_last_error(void);

/* Replaces CudaContext(device=...) (GPUSimulators/CudaContext.py:47-101):
 * selects the device and prepares the kernels.  No JIT: kernels are built
 * ahead of time for sm_100a. */
FV_API int fv_context_create(int device, fv_context** out);
FV_API int fv_context_destroy(fv_context* ctx);
/* Device name, e.g. "NVIDIA B200" (CudaContext.__str__, CudaContext.py:103-108). */
FV_API int fv_context_device_name(fv_context* ctx, char* buf, int len);

/* Replaces the constructors of the eight scheme classes (e.g.
 * GPUSimulators/KP07_dimsplit.py:55-106): uploads the initial state into two
 * state buffers (u0 with the data, u1 zeroed, as ArakawaA2D does,
 * GPUSimulators/Common.py:741-755) and seeds the CFL value with the host
 * estimate min(dx/(|u|+sqrt(g h)), dy/(|v|+sqrt(g h))) (KP07_dimsplit.py:102-106;
 * sqrt(gamma*rho) for Euler, EE2D_KP07_dimsplit.py:105-108).
 * host_vars: nv pointers (3, or 4 for Euler) to arrays of host_rows x host_cols
 * floats, either (ny, nx) interior data or (ny+2g, nx+2g) data with ghost cells
 * (Common.py:524-531), with g = 1 for LxF/FORCE/HLL and 2 otherwise.
 * bc: BoundaryCondition.asCodedInt() (GPUSimulators/Simulator.py:78-92). */
FV_API int fv_sim_create(fv_context* ctx, int scheme, int nx, int ny, float dx, float dy, const fv_params* params, int bc,
                  const float* const* host_vars, int host_rows, int host_cols, fv_sim** out);
FV_API int fv_sim_destroy(fv_sim* sim);

/* Replaces <Scheme>.substep(dt, step_number) (e.g. KP07_dimsplit.py:108-126):
 * one stage-kernel launch and the buffer swap.  The split schemes apply dt/2,
 * as the reference classes do.  Always writes the CFL field. */
FV_API int fv_sim_substep(fv_sim* sim, float dt, int step_number);

/* One band of tile rows [row0, row0 + nrows) of substep `step_number`, for
 * overlapping a stripe's halo exchange with its interior (the reference's
 * interior/exterior launches on two streams, MPISimulator.py:318-331,
 * EE2D_KP07_dimsplit.py:140-266).  A substep launched as bands covering every
 * tile row once, in order on the simulation's stream, equals fv_sim_substep;
 * the band that arrives last finishes it.  fv_sim_tile_rows gives the number
 * of tile rows. */
FV_API int fv_sim_substep_rows(fv_sim* sim, float dt, int step_number, int row0, int nrows);
FV_API int fv_sim_tile_rows(fv_sim* sim, int* rows);

/* Replaces BaseSimulator.step(dt) (GPUSimulators/Simulator.py:220-228). */
FV_API int fv_sim_step(fv_sim* sim, float dt);

/* Replaces BaseSimulator.simulate(t, dt=None) (GPUSimulators/Simulator.py:176-217):
 * advances until simTime() >= start + t.  use_dt == 0: dt = computeDt()*cfl_scale,
 * recomputed every 100 steps; use_dt != 0: the given dt.  The step sequence runs
 * as CUDA graphs with the time step kept on the device. */
FV_API int fv_sim_simulate(fv_sim* sim, double t, float dt, int use_dt);

/* Advances exactly n_steps steps with the simulate() dt schedule and no end
 * time (benchmark helper; same kernels and graphs as fv_sim_simulate). */
FV_API int fv_sim_advance(fv_sim* sim, long long n_steps);

/* Replaces <Scheme>.computeDt() (e.g. KP07_dimsplit.py:135-137):
 * min(cfl_data) times the scheme's factor. */
FV_API int fv_sim_compute_dt(fv_sim* sim, float* dt);

/* Replaces BaseSimulator.download(variables) / ArakawaA2D.download
 * (GPUSimulators/Common.py:757-770): copies the interior (ny x nx) of variable
 * `var` of u0 into host memory (row pitch in floats) and waits for the copy,
 * which the reference leaves unsynchronised (Common.py:769). */
FV_API int fv_sim_download(fv_sim* sim, int var, float* host, int host_pitch);

/* Uploads new interior data (ny x nx) for variable `var` of u0 (CudaArray2D.upload,
 * GPUSimulators/Common.py:587-616). */
FV_API int fv_sim_upload(fv_sim* sim, int var, const float* host, int host_pitch);

/* CudaArray2D.download/upload with an extent (GPUSimulators/Common.py:543-616):
 * the w x h region whose first cell is (x, y) in the reference's coordinates,
 * which count the ghost cells (x in [0, nx + 2g), y in [0, ny + 2g), g = 1 for
 * LxF, FORCE and HLL, 2 otherwise), of variable `var` of u0.  The download
 * waits for its copy; regions outside [0, nx + 2g) x [0, ny + 2g) are rejected. */
FV_API int fv_sim_download_region(fv_sim* sim, int var, int x, int y, int w, int h, float* host, int host_pitch);
FV_API int fv_sim_upload_region(fv_sim* sim, int var, int x, int y, int w, int h, const float* host, int host_pitch);

/* simTime(), simSteps() and the current dt (Simulator.py:236-240). */
FV_API int fv_sim_time(fv_sim* sim, double* t, long long* nt, float* dt);

/* FP64 sums of each conserved variable over the interior of u0 (no
 * counterpart in the reference; supports its conservation checks). */
FV_API int fv_sim_conservation(fv_sim* sim, double* sums);

/* Replaces check() (GPUSimulators/Common.py:772-780): *has_nan != 0 if any
 * value of u0 or u1 (ghost cells included) is NaN. */
FV_API int fv_sim_check(fv_sim* sim, int* has_nan);

/* synchronize() (Simulator.py:233-234). */
FV_API int fv_sim_synchronize(fv_sim* sim);

/* setBoundaryConditions (Simulator.py:245-247). */
FV_API int fv_sim_set_boundary_conditions(fv_sim* sim, int bc);

/* Test hooks (no counterpart in the reference): the give-up path of the
 * stage kernels' bounded waits, exercised without faulting or hanging a GPU.
 * fv_sim_set_wait_limit sets how many times a stage kernel polls for its
 * tile load before it gives up (negative: the default, about a second); 0
 * gives up at once, after which the kernel still waits, boundedly, for its
 * copies to land, writes nothing and the next synchronising call returns
 * FV_ERR_DEVICE.  fv_selftest_bounded_wait runs one warp that waits `polls`
 * times on a barrier that nothing completes; *gave_up = 1 when it gave up. */
FV_API int fv_sim_set_wait_limit(fv_sim* sim, int polls);
FV_API int fv_selftest_bounded_wait(int polls, int* gave_up);

/* Time-stepping state of a simulation: simulated time t, steps nt, the
 * current time step dt and the last CFL minimum (from which simulate()
 * derives dt every 100 steps).  get/set let a caller checkpoint a simulation
 * and resume it later with the same continuation; no reference counterpart
 * (the reference keeps t, nt and dt as Python attributes,
 * GPUSimulators/Simulator.py:139-143, and has no resume). */
FV_API int fv_sim_get_control(fv_sim* sim, double* t, long long* nt, float* dt, float* cfl_min);
FV_API int fv_sim_set_control(fv_sim* sim, double t, long long nt, float dt, float cfl_min);

/* Device state of a simulation for halo exchange between row stripes
 * (replaces the PyCUDA array access of MPISimulator.full_exchange,
 * GPUSimulators/MPISimulator.py:371-480).  ptrs[b * 4 + v] receives the base
 * of buffer b (0, 1) of variable v: storage row 0 is domain row y = -2, every
 * row holds *pitch floats and domain cell (y, x) is at [(y + 2) * pitch +
 * x + 4].  *cur is the buffer that holds the current state (this call waits
 * for the simulation's stream).  Entries for v >= number of variables are
 * null. */
FV_API int fv_sim_buffers(fv_sim* sim, float** ptrs, int* pitch, int* cur);

/* The CUDA stream (cudaStream_t) every launch and copy of the simulation is
 * ordered on, so that a caller can order its own device work (e.g. NCCL halo
 * sends and receives) with the stage kernels without host synchronisation.
 * No reference counterpart (the reference's Simulator.stream is a PyCUDA
 * stream, GPUSimulators/Simulator.py:164). */
FV_API int fv_sim_stream(fv_sim* sim, void** stream);

/* Device-side launches per step of the graph path, and the tile used
 * (introspection for benchmarks and tests). */
FV_API int fv_sim_info(fv_sim* sim, int* tile_w, int* tile_h, int* threads, int* launches_per_step);

/* Average device time of the stage kernels over the last fv_sim_advance
 * call, measured with CUDA events on the simulation's stream (0 if unknown). */
FV_API int fv_sim_last_advance_ms(fv_sim* sim, double* ms);

/* ---- Batches: many simulations of one scheme advanced together.
 * No counterpart in the reference (it runs one simulation per class instance);
 * each simulation in a batch follows exactly the reference's simulate(t_end)
 * semantics (own CFL dt every 100 of its own steps, last step shortened to
 * t_end), so its result equals a plain fv_sim_simulate of the same scenario. */
typedef struct fv_batch fv_batch;

/* Any scheme (params->order sets KP07's Runge-Kutta order for every
 * simulation of the batch); params->tile selects the batched kernel's tile shape. */
FV_API int fv_batch_create(fv_context* ctx, int scheme, const fv_params* params, int max_instances, fv_batch** out);
FV_API int fv_batch_destroy(fv_batch* batch);
/* Admits one simulation (initial state as for fv_sim_create) that runs until
 * its time reaches t_end; returns its slot, or FV_ERR_NOMEM when the device
 * has no room for it (the batch is unchanged). */
FV_API int fv_batch_add(fv_batch* batch, int nx, int ny, float dx, float dy, int bc, const float* const* host_vars,
                        int host_rows, int host_cols, double t_end, int* slot);
FV_API int fv_batch_remove(fv_batch* batch, int slot);
/* Queues n_steps steps for every simulation of the batch (CUDA graphs of the
 * batched kernel, one launch per substep over the tile work list);
 * simulations that reached t_end do nothing. Asynchronous.
 * Simulations admitted or removed since the last run join or leave the tile
 * work list first; FV_ERR_NOMEM means the list could not grow, nothing was
 * queued and the batch is unchanged (a later call retries). */
FV_API int fv_batch_run(fv_batch* batch, int n_steps);
/* Waits for queued work and refreshes the host view of every simulation. */
FV_API int fv_batch_sync(fv_batch* batch);
/* t, nt, dt and the simulation's state as of the last sync: done = 0 still
 * running, 1 reached t_end, 2 failed (a step left a non-finite value or a
 * non-positive depth or density, t or dt is not a number, e.g. from a
 * non-finite initial state, or dt is not positive before t_end): a failed
 * simulation takes no further steps and
 * its state is undefined; the other simulations of the batch are unaffected.
 * The reference's counterpart is check()'s NaN test (GPUSimulators/Common.py:772-780,
 * called from Simulator.simulate, GPUSimulators/Simulator.py:210-217). */
FV_API int fv_batch_status(fv_batch* batch, int slot, double* t, long long* nt, float* dt, int* done);
FV_API int fv_batch_download(fv_batch* batch, int slot, int var, float* host, int host_pitch);
/* Device bytes held, simulations in the batch, work-list length, device time
 * of the last fv_batch_run (ms, valid after fv_batch_sync). */
FV_API int fv_batch_info(fv_batch* batch, size_t* device_bytes, int* active, int* work_items, double* last_run_ms);
/* Tile shape, threads per CTA and CTAs per launch of the batch's kernel (one
 * per tile of the last published work list, or the resident grid of a
 * persistent tile configuration). */
FV_API int fv_batch_tile(fv_batch* batch, int* tile_w, int* tile_h, int* threads, int* grid);

/* One KP07_dimsplit substep that allocates no memory, for callers that may
 * not call cudaMalloc: applications that own all device memory through their
 * own pool, or loops that must not pay allocation latency or risk running out
 * of memory mid-run.  No counterpart in the reference.
 * in/out: 3 device pointers (h, hu, hv), each (ny+4) x pitch floats, element
 * (y, x) at [(y+2)*pitch + x+4], 16-byte aligned, pitch a multiple of 4 and
 * >= nx+8; no output plane may overlap an input plane or another output
 * plane (FV_ERR_INVALID).  dt is the kernel dt (half the step dt of a split
 * step); step selects the sweep order (0: x then y); bc is the boundary codec
 * of fv_sim_create with each side Dirichlet, periodic or reflective (Neumann:
 * FV_ERR_UNSUPPORTED, other codes FV_ERR_INVALID); cfl_min (device float*,
 * may be NULL) receives min over cells of min(dx/(|u|+sqrt(gh)),
 * dy/(|v|+sqrt(gh))).
 * Scratch is a static device array of about 33 KB per GPU, limiting a call to
 * 8192 tiles of 124 x 60 cells (FV_ERR_INVALID beyond).  Calls that overlap on
 * the GPU share that array and race.  The first call on a device performs its
 * set-up (symbol lookup, kernel attribute); make it before any stream capture.
 * Each call first waits for `stream` and reads the error flag the previous
 * call may have left: if a tile load of that call gave up, its output is
 * incomplete, and this call clears the flag and returns FV_ERR_DEVICE without
 * launching.  Otherwise asynchronous on `stream` (a cudaStream_t, or NULL).
 * Test hook: FVGPU_NOALLOC_WAIT_POLLS (read once per process) sets the tile
 * load's poll limit; a negative value makes every tile load give up at once. */
FV_API int fv_kp07_dimsplit_substep_noalloc(const float* const* in, float* const* out, int pitch, int nx, int ny,
                                            float dx, float dy, float dt, float g, float theta, int step, int bc,
                                            float* cfl_min, void* stream);

/* Pinned host memory for end-to-end transfers (CudaArray2D uses page-locked
 * buffers for downloads, Common.py:563-564). */
FV_API int fv_host_alloc(void** ptr, size_t bytes);
FV_API int fv_host_free(void* ptr);

#ifdef __cplusplus
}
#endif

#endif /* FVGPU_H */
