/*
 * flb_oracle.h -- CPU oracle for the D2Q9 lattice-Boltzmann solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solver step (FlowLB src/cuda/lbmKernel2D.cu, src/cuda/cellCalculations.cuh,
 * src/initData.h, src/initData.cpp, src/cuda/runCuda.cu:460-528).  It is the
 * checker for the CUDA engine in flowlb_b200/ and the timed CPU baseline of
 * bench.py; nothing in the engine links, loads or calls it.
 *
 * Parity pins (tests/): the host initialisation is compared cell by cell with
 * the reference's own initFields/initFreeSurfaceFlags/initFreeSurfaceFields
 * compiled from the reference sources (oracle/Makefile -> oracle/_ref/); the
 * per-kernel step arithmetic is compared bit for bit with the reference's own
 * CUDA kernels compiled with --fmad=false (GPU tests, oracle/_ref/).
 *
 * Deterministic semantics where the reference kernels race (see the engine
 * design notes): every cross-cell read inside one reference kernel sees the
 * value from before that kernel ("snapshot"), except the neighbour count of
 * d_FreeSurface2D_4, which sees the converted flags ("post").  The option
 * fs_count_pre makes that count read the unconverted flags instead; the
 * reference's result lies between the two.
 */
#ifndef FLB_ORACLE_H
#define FLB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Storage / arithmetic variants. */
enum {
  ORC_F64 = 0,      /* DDF f64, arithmetic f64, mass f64 (reference double build) */
  ORC_F32 = 1,      /* DDF f32, arithmetic f32, mass/excess/phi f64            */
  ORC_F16S = 2,     /* DDF stored f16 as (f - w_i) * scale, arithmetic f32, mass f64 */
  ORC_F32_M32 = 3   /* DDF f32, arithmetic f32, mass f32 (reference float build) */
};

/* Wall treatment. */
enum { ORC_BB_IMPLICIT = 0, ORC_BB_HALFWAY = 1 };

/* Free-surface semantics. */
enum { ORC_FS_REFERENCE = 0, ORC_FS_CONSERVATIVE = 1 };

/* Field ids for orc_field(). */
enum {
  ORC_FIELD_F = 0, ORC_FIELD_RHO = 1, ORC_FIELD_U = 2, ORC_FIELD_FLAGS = 3,
  ORC_FIELD_MASS = 4, ORC_FIELD_EXCESS = 5, ORC_FIELD_PHI = 6
};

/* Kernel ids for orc_kernel(). */
enum {
  ORC_K_STREAM_COLLIDE = 0, ORC_K_FS1 = 1, ORC_K_FS2 = 2, ORC_K_FS3 = 3, ORC_K_FS4 = 4
};

typedef struct {
  int32_t nx, ny;
  int32_t variant;       /* ORC_F64 ... */
  int32_t free_surface;  /* 0 mono-fluid, 1 free surface */
  int32_t bb;            /* ORC_BB_* */
  int32_t fs_mode;       /* ORC_FS_* */
  int32_t collision;     /* 0 SRT, 1 TRT */
  int32_t subgrid;       /* Smagorinsky on/off */
  int32_t use_force;     /* Guo forcing on/off */
  int32_t fs_count_pre;  /* oracle-only: FS_4 counts IG neighbours as unconverted */
  int32_t fs1_post;      /* oracle-only: FS_1 outgoing reads see neighbours' rebuilt populations */
  float tau;             /* relaxation time */
  float fx, fy;          /* body force, lattice units */
  float f16_scale;       /* power-of-two scale S of the F16S storage */
  int32_t threads;       /* OpenMP threads (<=0: default) */
  double inlet_ux, inlet_uy; /* inlet velocity, lattice units (double, as LBVelocity) */
  float u_max;           /* velocity limiter (0: off), see flb_case_desc.u_max */
  int32_t arithmetic;    /* 0 the reference's expressions, 1 the engine's fused SRT form */
} orc_params;

typedef struct orc_state orc_state;

/* Builds the initial state from geometry flags (FLUID/GAS/WALL/INLET/OUTLET as
 * the reference's geometry stage produces them, before the free-surface
 * interface layer is added).  Returns NULL on bad parameters. */
orc_state* orc_create(const orc_params* p, const uint8_t* geometry_flags);
void orc_destroy(orc_state* s);

/* Advances n time steps (FS_1, stream-collide, FS_2, FS_3, FS_4 per step in
 * free-surface mode; stream-collide alone otherwise). */
int orc_step(orc_state* s, uint64_t n);

/* Runs one reference kernel at the current time step without advancing t. */
int orc_kernel(orc_state* s, int kernel_id);

uint64_t orc_time(const orc_state* s);
void orc_set_time(orc_state* s, uint64_t t);
size_t orc_cells(const orc_state* s);

/* Pointer to an internal array (writable).  Element types: F is double (F64),
 * float (F32/F32_M32) or _Float16 storage (F16S); RHO/U are the arithmetic
 * type; MASS/EXCESS/PHI the mass type; FLAGS uint8.  *elem_size receives the
 * element size in bytes. */
void* orc_field(orc_state* s, int field, size_t* elem_size);

/* Reads the DDF in the reference slot layout f[c + s*N], decoded to double. */
void orc_read_f64(const orc_state* s, double* out);

/* Total fluid mass in FP64.  Free surface: sum of cell masses plus the excess
 * mass still to be pulled by neighbours.  Mono-fluid: sum of the populations
 * the next step loads into non-solid cells. */
double orc_total_mass(const orc_state* s);

/* Race enumeration (test support), see flb_oracle_body.inc.  fs1: up to 256
 * options of (mass, 8 rebuilt populations, rebuilt mask) for cell idx, state
 * before FS_1.  fs4: up to 9 options of (mass, excess, fill level), state
 * after FS_3.  Return the number of options (0: the kernel skips the cell). */
int orc_fs1_options(orc_state* s, size_t idx, double* masses, double* recs, uint8_t* masks);
int orc_fs4_options(const orc_state* s, size_t idx, double* out3);

#ifdef __cplusplus
}
#endif
#endif
