/*
 * flowlb.h -- C ABI of the B200 D2Q9 lattice-Boltzmann engine.
 *
 * Drop-in for the solver path of FlowLB (a 2D culvert-flow LBM with a VOF
 * free surface).  FlowLB's solver boundary is the C++ template set of
 * src/cuda/runCuda.cuh:25-38 (h_launchCudaCalculations2D and the four run
 * loops), called only from App::calculate (src/ui/app.cpp:293,310).  That
 * boundary allocates every device buffer (runCuda.cu:85, cudaInitData.cuh:90-125),
 * initialises the state on the host (initData.h:220-333), runs the time loop
 * (runCuda.cu:460-528) and copies density, velocity, fill level and flags back
 * to host vectors for the VTK writer (cudaUtils.cuh:42-53).  This header
 * splits that into handle-based calls with plain pointers and status codes:
 *
 *   flb_create / flb_reset       <- h_initDataCuda2D + initData + h_initConstantDataCuda2D
 *   flb_step                     <- the body of the run loops, n time steps
 *   flb_read_field               <- CudaUtils::copyDataFromDevice
 *   flb_destroy                  <- the cudaFree block, runCuda.cu:111-127
 *
 * Conventions.  Every function returns flb_status (never exits the process);
 * flb_last_error() gives a message.  Calls on one handle must not overlap;
 * different handles are independent.  All device work of a handle is issued
 * on one CUDA stream (the caller's, if given).  Arrays are structure-of-arrays
 * in the reference layout: cell c = x + y*nx; DDF slot s of cell c at
 * f[c + s*N]; u[c] = u_x, u[c + N] = u_y.  Cell flags use the reference's
 * uint8 encoding (src/utils.h:91-108): FLUID 0x01, GAS 0x02, INTERFACE 0x04,
 * WALL 0x08, MOVING_WALL 0x10, INLET 0x20, OUTLET 0x40, GAS_INTERFACE 0x80.
 */
#ifndef FLOWLB_H
#define FLOWLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FLB_API __attribute__((visibility("default")))
#else
#define FLB_API
#endif

typedef enum flb_status {
  FLB_OK = 0,
  FLB_ERR_INVALID_ARGUMENT = 1,
  FLB_ERR_CUDA = 2,
  FLB_ERR_OUT_OF_MEMORY = 3,
  FLB_ERR_UNSUPPORTED = 4,
  FLB_ERR_IO = 5,
  FLB_ERR_NONFINITE = 6,
  FLB_ERR_NO_DEVICE = 7
} flb_status;

/* Storage precision of the populations (OptionsCalc.txt PRECISION,
 * src/io/reader.cpp:367).  16 stores (f_i - w_i) * f16_scale in binary16 and
 * computes in float. */
enum { FLB_PRECISION_F64 = 64, FLB_PRECISION_F32 = 32, FLB_PRECISION_F16S = 16 };

/* Wall treatment.  IMPLICIT mirrors the reference: solid cells are skipped and
 * a population sent into one returns two steps later.  HALFWAY reflects it
 * into the opposite direction for the next step. */
enum { FLB_BB_IMPLICIT = 0, FLB_BB_HALFWAY = 1 };

/* Free-surface semantics.  REFERENCE mirrors lbmKernel2D.cu:14-303.
 * CONSERVATIVE weights interface mass exchange symmetrically with the stored
 * fill levels, reconstructs the populations that arrive from gas neighbours,
 * and hands excess mass only to cells that collect it; with FP64 mass and
 * HALFWAY walls it conserves total fluid mass to round-off. */
enum { FLB_FS_REFERENCE = 0, FLB_FS_CONSERVATIVE = 1 };

/* Arithmetic of the stream-collide step.  REFERENCE evaluates density,
 * velocity, equilibrium, Guo forcing and the relaxation with the reference's
 * expressions and operand order (bit-identical to FlowLB built without
 * floating-point contraction).  FUSED computes the same second-order BGK + Guo
 * update with explicit fused multiply-adds and shared subexpressions (about a
 * third of the operations); it applies to SRT without the subgrid model, and
 * TRT, the subgrid model and inlet/outlet cells keep the reference
 * expressions. */
enum { FLB_ARITH_REFERENCE = 0, FLB_ARITH_FUSED = 1 };

/* Collision operator (reference d_collisionOperator). */
enum { FLB_COLLISION_SRT = 0, FLB_COLLISION_TRT = 1 };

/* Field ids for flb_read_field / flb_write_field / flb_field_info. */
enum {
  FLB_FIELD_F = 0,       /* 9N populations, arithmetic type, reference slot layout */
  FLB_FIELD_RHO = 1,     /* N, arithmetic type */
  FLB_FIELD_U = 2,       /* 2N, arithmetic type */
  FLB_FIELD_FLAGS = 3,   /* N, uint8 */
  FLB_FIELD_MASS = 4,    /* N, mass type (free surface) */
  FLB_FIELD_EXCESS = 5,  /* N, mass type (free surface) */
  FLB_FIELD_PHI = 6      /* N, mass type (free surface): fill fraction */
};

/* Case description.  Fill with flb_case_desc_init() and override. */
typedef struct flb_case_desc {
  uint32_t nx, ny;            /* lattice size; N = nx*ny, 9N < 2^32 */
  const uint8_t* flags;       /* host geometry flags, N bytes: FLUID/GAS/WALL/INLET/OUTLET cells as
                                 the reference's geometry stage produces them (initData.h:256-317) */
  int32_t free_surface;       /* TYPE_PROBLEM: 0 MONOFLUID, 1 FREE_SURFACE */
  int32_t precision;          /* FLB_PRECISION_* */
  int32_t mass_precision;     /* 64 or 32 (32 only with precision 32) */
  int32_t collision;          /* FLB_COLLISION_* */
  int32_t subgrid;            /* Smagorinsky subgrid model */
  int32_t use_volumetric_force;
  float tau;                  /* relaxation time (> 0.5) */
  float fx, fy;               /* body force density in lattice units */
  int32_t bounce_back;        /* FLB_BB_* */
  int32_t fs_mode;            /* FLB_FS_* */
  float f16_scale;            /* power of two; 0 selects 4096 */
  int32_t device;             /* CUDA device ordinal; -1 = current */
  void* stream;               /* cudaStream_t to issue on; NULL = a stream owned by the handle */
  double inlet_ux, inlet_uy;  /* lattice velocity of INLET cells (double, as the reference's LBVelocity) */
  int32_t kernel_variant;     /* stream-collide data path: 0 auto, 1 one cell per thread, 2 vector
                                 (V cells per thread; needs nx % V == 0, V = 4 for FP32/FP16S, 2 for FP64) */
  float u_max;                /* velocity limiter, lattice units (0 = off, the reference behaviour): the
                                 force-shifted velocity used for feq and forcing is scaled down to |u| = u_max;
                                 keeps high-Mach free-surface fronts stable; mass is still conserved */
  int32_t arithmetic;         /* FLB_ARITH_* (default FUSED; REFERENCE reproduces FlowLB's rounding) */
} flb_case_desc;

typedef struct flb_engine* flb_handle;

FLB_API void flb_case_desc_init(flb_case_desc* desc);

/* Allocates the device state and builds the initial state on the device from
 * desc->flags (host): f = feq(rho=1, u) stored with the t=1 esoteric pattern,
 * and for free surface the interface layer, fill level and mass
 * (initData.h:125-206, initData.cpp:13-37).  Replaces h_launchCudaCalculations2D's
 * set-up half, runCuda.cu:34-85. */
FLB_API flb_status flb_create(const flb_case_desc* desc, flb_handle* out);

/* Rebuilds the initial state from new host geometry flags of the same size and
 * sets t = 0, reusing the device buffers. */
FLB_API flb_status flb_reset(flb_handle h, const uint8_t* host_flags);

FLB_API flb_status flb_destroy(flb_handle h);

/* Advances n time steps asynchronously on the handle's stream: per step
 * FS_1, stream-collide, FS_2..4 (free surface) or stream-collide alone.
 * Replaces the loop bodies of runCuda.cu:473-490 and :506-527. */
FLB_API flb_status flb_step(flb_handle h, uint64_t n);

/* Waits for the handle's stream.  FLB_ERR_CUDA if a grid barrier of the
 * persistent free-surface step gave up waiting (the state is then undefined
 * and flb_step is refused until flb_reset). */
FLB_API flb_status flb_sync(flb_handle h);
FLB_API flb_status flb_get_time(flb_handle h, uint64_t* t);

/* How the free-surface steps that flb_step replays from CUDA graphs run (no
 * counterpart in the reference, whose host loop launches five kernels per
 * step, runCuda.cu:506-527).  FLB_STEP_KERNELS: FS_1, stream-collide and
 * the flag pass (which lists the next step's super-tiles) as three kernels
 * per step.
 * FLB_STEP_PERSISTENT: one cooperative kernel per graph (every CTA resident,
 * one per SM) runs all its steps, the passes separated by grid barriers in
 * global memory; a barrier wait gives up after a bounded number of polls
 * (flb_set_wait_limit) and the next flb_sync or flb_read_field returns
 * FLB_ERR_CUDA.  FLB_STEP_AUTO (default): the per-pass kernels, measured
 * faster on a B200 (the persistent kernel holds 1024 threads per SM, the
 * per-pass stream-collide and flag kernels 2048).  Both give identical
 * results.
 * The persistent form needs a free-surface case without inlet/outlet cells
 * (FLB_ERR_UNSUPPORTED otherwise); single-phase cases ignore the mode.  With
 * FLB_PERSIST_SKIP_ARRIVAL=1 in the environment (failure injection for
 * tests) one CTA never arrives at the barriers, so every wait runs out. */
enum { FLB_STEP_AUTO = 0, FLB_STEP_KERNELS = 1, FLB_STEP_PERSISTENT = 2 };
FLB_API flb_status flb_set_step_mode(flb_handle h, int mode);
/* mode as set; *persistent = 1 when graph-replayed steps run persistent */
FLB_API flb_status flb_get_step_mode(flb_handle h, int* mode, int* persistent);
/* Polls a CTA of the persistent step waits at a grid barrier before the
 * launch gives up; 0 restores the default (2^22). */
FLB_API flb_status flb_set_wait_limit(flb_handle h, uint32_t polls);
FLB_API flb_status flb_set_stream(flb_handle h, void* stream);
FLB_API flb_status flb_get_stream(flb_handle h, void** stream);

/* Element size and element count of a field (0 count: not held in this mode). */
FLB_API flb_status flb_field_info(flb_handle h, int field, size_t* elem_size, size_t* count);

/* Copies a field into dst (host memory when on_device = 0, device memory of the
 * handle's GPU when 1) and waits for the copy.  Replaces copyDataFromDevice,
 * cudaUtils.cuh:42-53; on_device = 1 is the headless stand-in for the OpenGL
 * interop buffers of runCuda.cu:137-147. */
FLB_API flb_status flb_read_field(flb_handle h, int field, void* dst, int on_device);

/* Overwrites a field from src (same element type as flb_field_info). */
FLB_API flb_status flb_write_field(flb_handle h, int field, const void* src, int on_device);

/* Total fluid mass in FP64: free surface, the sum of cell masses plus the
 * excess mass its neighbours will collect next step; mono-fluid, the sum of
 * the populations the next step loads into non-solid cells. */
FLB_API flb_status flb_total_mass(flb_handle h, double* mass);

/* Allocation-free free-surface total mass; no counterpart in the reference.
 * For callers that may not allocate device memory when they need the check
 * (under a fixed audited memory budget, in a loop that cannot take the
 * implicit synchronisation of cudaMalloc/cudaFree, or holding only pointers
 * to someone else's buffers): it takes the device
 * fields directly (mass and excess in FP64, flags as the solver keeps them,
 * nx*ny cells each), launches on `stream` and writes the same FP64 sum as
 * flb_total_mass to the device pointer `out` without waiting.  Its scratch is
 * a fixed array of FLB_NOALLOC_MAX_CELLS/256 doubles (512 KiB) that every GPU
 * loading the library holds until exit; larger grids are rejected with
 * FLB_ERR_INVALID_ARGUMENT.  Nothing needs zeroing beforehand.  Calls that
 * overlap on the GPU (other streams or host threads) share that scratch and
 * race; the first call on a device looks its address up, so make it before
 * any capture. */
#define FLB_NOALLOC_MAX_CELLS 16777216u
FLB_API flb_status flb_total_mass_noalloc(const double* mass, const double* excess, const uint8_t* flags,
                                          uint32_t nx, uint32_t ny, int fs_mode, double* out, void* stream);

/* Cell-type census: counts[0..3] = fluid, interface, gas, solid(wall). */
FLB_API flb_status flb_cell_counts(flb_handle h, uint64_t counts[4]);

/* FLB_ERR_NONFINITE if any population of a non-solid cell is NaN or Inf. */
FLB_API flb_status flb_check_finite(flb_handle h);

/* Runs one pass of the step at the current t without advancing it (parity
 * testing): 0 stream-collide, 1 FS_1 (mass exchange), 2 FS_2..4 (flag and
 * mass finalisation). */
FLB_API flb_status flb_run_pass(flb_handle h, int pass);

/* Runs n time steps with a CUDA event around every pass on the handle's
 * stream (no graphs) and returns the summed device time per pass kind in
 * milliseconds: pass_ms[0] stream-collide, [1] FS_1, [2] FS_2..4.  Advances t. */
FLB_API flb_status flb_profile_steps(flb_handle h, uint64_t n, double pass_ms[3]);

/* Runs n time steps (rounded up to even, from the next even t in steady
 * state) in the persistent free-surface form with a device clock read by one
 * CTA as it leaves every grid barrier, and returns the summed time of each
 * phase in milliseconds: phase_ms[0] FS_1, [1] stream-collide, [2] FS_2..4
 * (with the next step's lists), each with the barrier that ends it.  Unlike
 * flb_profile_steps nothing is serialised: the phases sum to the step time
 * of the persistent kernel.  Advances t; FLB_ERR_UNSUPPORTED without a
 * persistent form. */
FLB_API flb_status flb_profile_phases(flb_handle h, uint64_t n, double phase_ms[3]);

/* Kernels this handle has launched so far (graph replays count each kernel). */
FLB_API flb_status flb_launch_count(flb_handle h, uint64_t* launches);

/* Binary checkpoint of the full state (populations, t, flags, mass, excess,
 * fill level, density, velocity); the reference has none. */
FLB_API flb_status flb_save_checkpoint(flb_handle h, const char* path);
FLB_API flb_status flb_load_checkpoint(flb_handle h, const char* path);

/* ---- batched ensemble (no counterpart in the reference, which runs one case
 * per call) ------------------------------------------------------------------
 * n independent single-phase FP32 cases (their own sizes, geometry, tau and
 * body force; one bounce-back, arithmetic, collision and subgrid setting for
 * all; no inlet/outlet cells) advanced together: flb_batch_step(b, k) is one
 * graph launch of one persistent kernel that runs all k steps of every case.
 * Each case ends bit-identical to k flb_step calls on its own handle.
 * A group of CTAs steps one case at a time; the steps of a case are separated
 * by a barrier among the group: a thread-block cluster of 1, 2, 4, 8 or 16
 * CTAs (FLB_BATCH_CLUSTER) or a team of any number of CTAs meeting in global
 * memory, every CTA of the launch resident at once (FLB_BATCH_TEAM, a
 * cooperative launch; a team barrier gives up after about two seconds, or
 * the limit of flb_batch_set_wait_limit, and flb_batch_sync then returns
 * FLB_ERR_CUDA).
 * The streams form (FLB_BATCH_STREAMS) is not one persistent launch: every
 * case becomes an engine handle (the single-case kernels and step graphs,
 * so the results are those of flb_step by construction), the cases spread
 * over a pool of streams longest first, and a batch step launches each
 * case's own step graphs on its stream; the cases run concurrently, which
 * hides the per-step launch latency that bounds a per-case loop on one
 * stream.  It keeps a second copy of the state (the handles') and is
 * entered at even steps only.
 * autotune: 0 uses 8-CTA clusters, one CTA per SM; 1 (100 probe steps) or a
 * probe step count > 1 times candidate modes, group sizes and counts of the
 * persistent kernel and the streams form with 8 and 16 streams on the batch
 * itself and keeps the fastest, then rebuilds the initial state.  The
 * device, and the stream if given, come from cases[0]. */
enum { FLB_BATCH_CLUSTER = 0, FLB_BATCH_TEAM = 1, FLB_BATCH_VECTOR = 4, FLB_BATCH_STREAMS = 8 };
typedef struct flb_batch_s* flb_batch;
FLB_API flb_status flb_batch_create(const flb_case_desc* cases, uint32_t n, int autotune, flb_batch* out);
FLB_API flb_status flb_batch_step(flb_batch b, uint64_t n);
FLB_API flb_status flb_batch_sync(flb_batch b);
/* back to the initial state, t = 0 */
FLB_API flb_status flb_batch_reset(flb_batch b);
/* FLB_FIELD_F, _RHO, _U or _FLAGS of case i (float, as a precision-32 handle) */
FLB_API flb_status flb_batch_read_field(flb_batch b, uint32_t i, int field, void* dst, int on_device);
/* info[0..7] = cases, cells, t, CTAs per group, groups, autotuned, threads
 * per CTA, mode (FLB_BATCH_CLUSTER or FLB_BATCH_TEAM, with FLB_BATCH_VECTOR
 * set when the vector data path runs; FLB_BATCH_STREAMS with group 1,
 * groups = streams, threads 0) */
FLB_API flb_status flb_batch_info(flb_batch b, int64_t info[8]);
/* Sets the launch shape (info[7], [3], [4], [6] of an earlier tuned batch,
 * for instance): mode, with FLB_BATCH_VECTOR or'ed in for the vector data
 * path (four cells per thread, 16-byte population accesses; the state is
 * stored with rows padded to a multiple of four cells, so every case can take
 * it); CTAs per group (1, 2, 4, 8 or 16 for a cluster, >= 1 for a team);
 * 1 <= groups <= the groups of that shape that fit on the device at once, and
 * <= the number of cases; 256, 512 or 1024 threads per CTA (256 or 512 on the
 * vector path).
 * FLB_BATCH_STREAMS with group 1 and 1..64 streams selects the streams
 * form (FLB_ERR_UNSUPPORTED at an odd step).
 * The state and t are kept (results do not depend on the shape).
 * FLB_ERR_INVALID_ARGUMENT for a shape out of range, FLB_ERR_UNSUPPORTED for
 * one that cannot launch. */
FLB_API flb_status flb_batch_set_launch(flb_batch b, int mode, int group, int groups, int threads);
/* Team mode: how many polls (about 1 us each) a CTA waits at its team's
 * barrier before the launch gives up; 0 restores the default (2^21).  After
 * a wait gave up, flb_batch_sync returns FLB_ERR_CUDA, the state and t are
 * undefined, and flb_batch_step refuses with FLB_ERR_CUDA until
 * flb_batch_reset.  With FLB_BATCH_SKIP_ARRIVAL=1 in the environment (failure
 * injection for tests, read at every flb_batch_step) one CTA of every team
 * never arrives, so every wait runs out. */
FLB_API flb_status flb_batch_set_wait_limit(flb_batch b, uint32_t polls);
/* Times the launch shapes again (probe_steps each, 0: 100) among the forms
 * given (FLB_TUNE_PERSISTENT: the persistent kernel's shapes;
 * FLB_TUNE_STREAMS: the streams form), keeps the fastest and rebuilds the
 * initial state (t = 0), as flb_batch_create with autotune does. */
enum { FLB_TUNE_PERSISTENT = 1, FLB_TUNE_STREAMS = 2 };
FLB_API flb_status flb_batch_tune(flb_batch b, uint32_t probe_steps, int forms);
FLB_API flb_status flb_batch_destroy(flb_batch b);
FLB_API const char* flb_batch_last_error(flb_batch b);

/* ---- adjoint of the Brinkman-porosity single phase (no counterpart in the
 * reference) -------------------------------------------------------------------
 * Forward model per fluid cell (pull streaming, half-way walls, x periodic):
 * rho = sum f, v = j/rho, u = (v + g/2)/(1 + s/2), F = rho (g - s u), BGK with
 * Guo forcing; s in [0,1] is a per-cell drag coefficient (0 free fluid, 1 a
 * quasi-solid).  Objective J = (1/window) * sum over the last `window` steps
 * of sum_y rho u_x in the last column.  flb_adjoint_forward runs the steps from
 * rest and keeps a checkpoint every checkpoint_every steps; flb_adjoint_backward
 * recomputes each segment from its checkpoint and runs the hand-written
 * adjoint step backwards, giving dJ/ds per cell and dJ/dg. */
typedef struct flb_adjoint_desc {
  uint32_t nx, ny;
  const uint8_t* flags;      /* N bytes: FLUID or WALL */
  const double* porosity;    /* N drag coefficients s in [0,1] */
  int32_t precision;         /* 32 or 64 (arithmetic and storage) */
  double tau;                /* relaxation time */
  double gx, gy;             /* body acceleration, lattice units */
  uint64_t steps;            /* a multiple of checkpoint_every */
  uint64_t window;           /* objective steps at the end, 1..steps */
  uint32_t checkpoint_every; /* even */
  int32_t device;
  void* stream;
} flb_adjoint_desc;
typedef struct flb_adjoint_s* flb_adjoint;
FLB_API void flb_adjoint_desc_init(flb_adjoint_desc* d);
FLB_API flb_status flb_adjoint_create(const flb_adjoint_desc* d, flb_adjoint* out);
FLB_API flb_status flb_adjoint_set_porosity(flb_adjoint a, const double* s);
FLB_API flb_status flb_adjoint_set_force(flb_adjoint a, double gx, double gy);
FLB_API flb_status flb_adjoint_forward(flb_adjoint a, double* J);
/* dJ_ds: N doubles (host, may be null); dJ_dg: {dJ/dgx, dJ/dgy} (may be null) */
FLB_API flb_status flb_adjoint_backward(flb_adjoint a, double* dJ_ds, double dJ_dg[2]);
/* device milliseconds of the last forward and backward calls */
FLB_API flb_status flb_adjoint_timing(flb_adjoint a, double ms[2]);
FLB_API flb_status flb_adjoint_destroy(flb_adjoint a);
FLB_API const char* flb_adjoint_last_error(flb_adjoint a);

/* ---- Headless visualisation (device buffers in place of the OpenGL view) -- */
/* FlowLB's OpenGL loops (runCuda.cu:130-458) fill interop surfaces from the
 * velocity and fill-level fields and shade them with GLSL.  These calls draw
 * the same pictures into plain buffers (host memory when on_device = 0, the
 * handle's GPU when 1), from the handle's current fields; no graphics API is
 * involved. */
enum { FLB_VIZ_UX = 0, FLB_VIZ_UY = 1, FLB_VIZ_MAGNITUDE = 2, FLB_VIZ_PRESSURE = 3 };

/* save2DDataToOpenGL (src/cuda/cudaUtils.cu:107-118): u as nx*ny interleaved
 * float pairs (ux, uy), row y at [2*(x + y*nx)]. */
FLB_API flb_status flb_viz_velocity(flb_handle h, float* dst, int on_device);

/* The texture*2D fragment shaders (assets/shaders/{monoFluid,freeSurface}/):
 * per node v = ux, uy or |u| (the pressure shader also shades |u|),
 * s = max((v - min_value)/(max_value - min_value), 0), colour = the n_colors
 * RGB colour map (host memory, 3 floats per entry, n_colors <= 4096) sampled at
 * s with linear filtering and mirrored-repeat wrapping as OpenGL does
 * (OpenGLTexture1D, OpenGLTexture.cpp:44-53); written as RGBA8 (alpha 255),
 * one pixel per node, rows as the lattice. */
FLB_API flb_status flb_viz_shade(flb_handle h, int quantity, const float* colormap_rgb, uint32_t n_colors,
                                 float max_value, float min_value, uint8_t* rgba, int on_device);

/* d_CreateIsoSurfaceVector2D (src/cuda/cudaIsosurface.cuh:33-199): the
 * iso-line v = iso_value of |u| (field FLB_FIELD_U) or of the fill level
 * (FLB_FIELD_PHI, free surface) over the camera window of lattice nodes
 * [b0, b1) x [b2, b3), drawn by marching squares and Bresenham lines as 255
 * into a width x height uint8 image that is cleared first.  The reference
 * draws the fill level through its two-component path (reading past the end
 * of phi); this reads phi as a scalar. */
FLB_API flb_status flb_viz_isoline(flb_handle h, int field, float iso_value, uint32_t width, uint32_t height,
                                   const uint32_t camera_bounds[4], uint8_t* image, int on_device);

/* ---- File-based set-up: Geometry.txt + OptionsCalc.txt ------------------ */
/* What App::calculate (src/ui/app.cpp:241-310) derives from the two input
 * files before the solver starts: GeometryReader::readGeometryOptions
 * (src/io/reader.cpp:1192-1217) and Mesh::init (src/geometry/mesh.cpp:11-51),
 * CalculationReader::readOptionsCalculation (reader.cpp:694-713), the unit
 * conversion (src/utils.cpp:7-82, runCuda.cu:71-79), the geometry sweep of
 * initData (src/initData.h:220-317), tau and the body force
 * (src/cuda/cudaInitData.cu:57-82) and the loop bounds (runCuda.cu:497-499).
 * Host code only: no CUDA call is made. */
typedef struct flb_setup {
  uint32_t nx, ny;              /* lattice size (Mesh::calculateNumberPointsMesh) */
  double x_min, y_min, z_min;   /* mesh origin (m) */
  double spacing;               /* SIZE (m) */
  uint8_t* flags;               /* nx*ny geometry flags, owned here (flb_setup_free) */
  flb_case_desc desc;           /* ready for flb_create, in the reference's modes (IMPLICIT walls,
                                   REFERENCE free surface and arithmetic); desc.flags == flags */
  uint64_t time_steps;          /* T: the reference loop runs t = 0..T, T+1 steps */
  uint64_t save_every;          /* tSave: results after the steps with t % tSave == 0 */
  float time_simulation, time_save;  /* TIME_SIMULATION, TIME_SAVE (s) */
  float nu_lattice;             /* kinematic viscosity in lattice units (float, as h_nu) */
  double length_to_si, time_to_si, mass_to_si, velocity_to_si, rho_to_si;  /* FLB::Units */
  int32_t graphics_api;         /* GRAPHICS_API: 0 NONE, 1 OPENGL (the engine is headless either way) */
  int32_t reference_precision;  /* PRECISION as read: 16, 32 or 64 */
  uint32_t cuda_block[3];       /* CUDA_BLOCK_SIZE as read (checked, not used) */
  char error[256];              /* the reader's message when a call fails */
} flb_setup;

/* Reads both files.  mesh_only = 0 follows App::calculate (every option read
 * and checked); mesh_only = 1 follows App::createDomain (src/ui/app.cpp:202-238,
 * reader.cpp:715-742): only TYPE_PROBLEM, the four boundaries and the initial
 * conditions are read, and only the boundaries are checked.  CSV_2D shapes are
 * read from the folder of the file that names them.  Errors: FLB_ERR_IO for a
 * file that cannot be opened, FLB_ERR_UNSUPPORTED for 3D, otherwise
 * FLB_ERR_INVALID_ARGUMENT with the reader's message in out->error. */
FLB_API flb_status flb_setup_from_files(const char* geometry_txt, const char* options_txt, int mesh_only,
                                        flb_setup* out);
FLB_API void flb_setup_free(flb_setup* s);

/* The flags after the free-surface sweep of initFreeSurfaceFlags
 * (src/initData.cpp:13-37): the content of FlowLB's mesh.vti, and of
 * FLB_FIELD_FLAGS right after flb_create.  out holds nx*ny bytes. */
FLB_API flb_status flb_setup_initial_flags(const flb_setup* s, uint8_t* out);

/* App::createDomain's mesh.vti (app.cpp:233-238): the initial flags as one
 * UInt8 field, written by the VTK writer below. */
FLB_API flb_status flb_setup_write_mesh_vti(const flb_setup* s, const char* path);

/* flb_setup_from_files (mesh_only = 0) followed by flb_create of its desc:
 * the whole set-up half of h_launchCudaCalculations2D from the two files.
 * The reader's message goes to stderr; flb_setup_from_files returns it. */
FLB_API flb_status flb_create_from_files(const char* geometry_txt, const char* options_txt, flb_handle* out);

/* ---- VTK ImageData output (src/io/writer.cpp:15-252) --------------------- */
enum { FLB_VTI_UINT8 = 0, FLB_VTI_FLOAT32 = 1, FLB_VTI_FLOAT64 = 2 };

typedef struct flb_vti_field {
  const char* name;       /* DataArray Name: "Flags", "U", "rho", "phi" */
  int32_t type;           /* FLB_VTI_*: element type of data and the DataArray type */
  int32_t components;     /* 1 scalar; 2 or 3: component k of cell i at data[i + k*N] */
  const void* data;       /* host memory, N = nx*ny cells per component */
  double to_si;           /* factor applied to every value (the writer's constantToSI) */
  int32_t flip_y;         /* nonzero: the second component is negated */
} flb_vti_field;

/* One ASCII .vti file byte-identical to FlowLB's VTIWriter for the same
 * fields: values printed as std::ostream prints a double by default,
 * origin and spacing as std::to_string does. */
FLB_API flb_status flb_write_vti(const char* path, uint32_t nx, uint32_t ny, double x0, double y0, double z0,
                                 double spacing, const flb_vti_field* fields, uint32_t n_fields);

/* <directory>/loaderFiles.vti.series listing result_0.vti .. result_<n-1>.vti
 * at times i * time_interval (Writer::createTimeSeriesFile, writer.cpp:163-182). */
FLB_API flb_status flb_write_vti_series(const char* directory, uint32_t n_files, double time_interval);

typedef struct flb_run_info {
  uint64_t steps;         /* time steps run */
  uint32_t files;         /* result_<i>.vti files written */
  char directory[512];    /* the results_<k> folder created under save_dir */
  char error[256];
} flb_run_info;

/* The headless run of FlowLB from its two input files
 * (h_runCudaMonoFluidNoGraphics2D / h_runCudaFreeSurfaceNoGraphics2D,
 * runCuda.cu:460-528): set-up as flb_create_from_files, then T+1 steps (at
 * most max_steps when nonzero), and after every step with t % tSave == 0 the
 * reference's fields written to save_dir/results_<k>/result_<i>.vti with the
 * series file rewritten; mono-fluid U and rho in SI units, free-surface
 * fields in lattice units, as the reference writes them. */
FLB_API flb_status flb_run_from_files(const char* geometry_txt, const char* options_txt, const char* save_dir,
                                      uint64_t max_steps, flb_run_info* info);

FLB_API const char* flb_last_error(flb_handle h);
FLB_API const char* flb_status_string(flb_status s);
FLB_API const char* flb_version(void);

#ifdef __cplusplus
}
#endif
#endif
