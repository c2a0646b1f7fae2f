/*
 * flb_oracle.c -- CPU oracle for the D2Q9 lattice-Boltzmann solver path.
 *
 * TEST INFRASTRUCTURE ONLY (see flb_oracle.h): the checker of the CUDA engine
 * and the timed CPU baseline.  Compile with -ffp-contract=off so that float
 * and double expressions round exactly as written, like the reference kernels
 * built with --fmad=false.
 *
 * Reference files restated here (paths inside the FlowLB project):
 *   src/cuda/cellCalculations.cuh:16-259   per-cell helpers
 *   src/cuda/lbmKernel2D.cu:14-121         d_FreeSurface2D_1
 *   src/cuda/lbmKernel2D.cu:124-148        d_FreeSurface2D_2
 *   src/cuda/lbmKernel2D.cu:151-190        d_FreeSurface2D_3
 *   src/cuda/lbmKernel2D.cu:193-303        d_FreeSurface2D_4
 *   src/cuda/lbmKernel2D.cu:306-519        d_StreamCollide2D
 *   src/cuda/cudaInitData.cu:25-39,57-108  cell-type masks, tau and force
 *   src/initData.h:75-206, initData.cpp:13-151  initial state
 *   src/cuda/runCuda.cu:460-528            step order of the headless loops
 */
#include "flb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Cell-type bits, src/cuda/cudaInitData.cu:25-39 and src/utils.h:91-108. */
enum {
  ORC_FLUID = 0x01, ORC_GAS = 0x02, ORC_INTERFACE = 0x04, ORC_WALL = 0x08, ORC_MWALL = 0x10,
  ORC_INLET = 0x20, ORC_OUTLET = 0x40, ORC_GI = 0x80,
  ORC_FGI = 0x07, ORC_IF = 0x05, ORC_IG = 0x06, ORC_INLET_FLUID = 0x21
};

/* Lattice velocities, src/cuda/cudaInitData.cu:76,78. */
static const int ORC_CX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
static const int ORC_CY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};

struct orc_state {
  orc_params p;
  uint32_t nx, ny;
  size_t N;
  uint64_t t;
  int nthreads;
  float inv_tau;
  /* constants of the fused SRT arithmetic (see FN(collide_fused)) */
  int fused;
  float fu_omc, fu_nk3, fu_hfx, fu_hfy, fu_fx, fu_fy, fu_g[4], fu_h[4], fu_sw[3];
  float f16_scale, f16_inv_scale;
  size_t s_size, c_size, m_size;
  void* f;
  void* rho;
  void* u;
  uint8_t* flags;
  void* mass;
  void* excess;
  void* phi;
  uint8_t* flags_tmp;
  uint8_t* flags_tmp2;
  void* recon;
  uint8_t* recon_mask;
  void* rho_snap;
  void* u_snap;
  int has_io;
};

/* calculateNeighborsIdxD2Q9, cellCalculations.cuh:82-109 (periodic wrap). */
/* FP16S stochastic rounding of the engine's fused single-phase step (its
 * lattice.cuh f16_rs_*): the cell pair (2k, 2k+1) draws a 32-bit word per time
 * step (multiplicative hash of 2k and t, xor-shift / multiply mix), population
 * i adds i*K; the low 13 bits round the even cell, bits 16..28 the odd one.
 * orc_f16_rs restates the binary32 -> binary16 conversion with 13 random bits
 * r (the engine's cvt.rs.f16x2.f32): r is added just below the last binary16
 * bit kept, then the value is truncated; on the binary16 normal range that is
 * r added to the binary32 bits, on the subnormal range r is aligned to the
 * wider discarded field.  Checked against the instruction on the GPU for
 * normal, subnormal and near-maximum values. */
static inline uint32_t orc_rs_base(uint32_t idx_even, uint32_t t) {
  uint32_t x = idx_even * 0x85EBCA6Bu + t * 0x9E3779B9u;
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  return x;
}
static inline uint32_t orc_rs_bits(uint32_t base, int i) { return base + (uint32_t)i * 0x632BE5ABu; }

/* binary32 bits -> binary16 bits, rounding toward zero (overflow gives the
 * largest finite value, as a round-toward-zero conversion does) */
static inline uint16_t orc_f16_rz(uint32_t x) {
  const uint16_t sg = (uint16_t)((x >> 16) & 0x8000u);
  const int e = (int)((x >> 23) & 0xffu);
  const uint32_t m = x & 0x7fffffu;
  if (e == 255) return (uint16_t)(sg | (m ? 0x7e00u : 0x7c00u));
  const int E = e - 127 + 15;
  if (E >= 31) return (uint16_t)(sg | 0x7bffu);
  if (E <= 0) {
    if (E < -10) return sg;
    return (uint16_t)(sg | ((m | 0x800000u) >> (14 - E)));
  }
  return (uint16_t)(sg | ((uint32_t)E << 10) | (m >> 13));
}

/* binary32 bits x -> binary16 bits, stochastic rounding with the 13 bits r */
static inline uint16_t orc_f16_rs(uint32_t x, uint32_t r) {
  const uint16_t sg = (uint16_t)((x >> 16) & 0x8000u);
  const int e = (int)((x >> 23) & 0xffu);
  const uint32_t m = x & 0x7fffffu;
  if (e == 255) return (uint16_t)(sg | (m ? 0x7e00u : 0x7c00u));
  if (e - 127 >= -14) return (uint16_t)(sg | orc_f16_rz((x & 0x7fffffffu) + r));
  const uint64_t full = e ? (uint64_t)(m | 0x800000u) : (uint64_t)m;
  const int shift = -(e ? e - 127 : -126) - 1; /* bits below the binary16 subnormal unit */
  if (shift >= 64) return sg;
  return (uint16_t)(sg | (uint16_t)((full + ((uint64_t)r << (shift - 13))) >> shift));
}

static inline void orc_nbrs(uint32_t idx, uint32_t x, uint32_t y, uint32_t nx, uint32_t ny, uint32_t* nb) {
  const uint32_t yc = y * nx;
  const uint32_t yu = ((y + 1u) % ny) * nx;
  const uint32_t yd = ((y + ny - 1u) % ny) * nx;
  const uint32_t xr = (x + 1u) % nx;
  const uint32_t xl = (x + nx - 1u) % nx;
  nb[0] = idx;
  nb[1] = xr + yc;
  nb[2] = xl + yc;
  nb[3] = x + yu;
  nb[4] = x + yd;
  nb[5] = xr + yu;
  nb[6] = xl + yd;
  nb[7] = xr + yd;
  nb[8] = xl + yu;
}

/* __saturatef: clamp to [0, 1], NaN to 0. */
static inline float orc_sat(float v) { return v > 1.0f ? 1.0f : (v > 0.0f ? v : 0.0f); }

/* d_FreeSurface2D_4 neighbour count, lbmKernel2D.cu:290-294. */
static inline int orc_counted_ref(uint8_t f) {
  const uint8_t e = f & (ORC_IF | ORC_GI);
  return e == ORC_FLUID || e == ORC_INTERFACE || e == ORC_IF || e == ORC_GI;
}
/* d_FreeSurface2D_1 pulls excess mass unless gas, wall or inlet (:26,39). */
static inline int orc_puller_ref(uint8_t f) { return !(f & (ORC_GAS | ORC_WALL | ORC_INLET)); }
/* Conservative mode: exactly the fluid/interface cells that are not walls or
 * inlets pull excess mass, and only those are counted as receivers. */
static inline int orc_puller_cons(uint8_t f) {
  const uint8_t e = f & ORC_FGI;
  return (e == ORC_FLUID || e == ORC_INTERFACE) && !(f & (ORC_WALL | ORC_MWALL | ORC_INLET));
}

/* initFreeSurfaceFlags, initData.cpp:13-37, with the bounded (non-periodic)
 * neighbour list of calculateNeighborsIndexD2Q9BBox, initData.cpp:39-124. */
static void orc_init_fs_flags(uint8_t* flags, uint32_t idx, uint32_t x, uint32_t y, uint32_t nx, uint32_t ny) {
  uint8_t* flag = &flags[idx];
  if (*flag & ~(ORC_FLUID | ORC_INLET | ORC_OUTLET)) return;
  if (*flag & ORC_INLET) *flag |= ORC_FLUID;
  else if (*flag & ORC_OUTLET) *flag |= ORC_GAS;
  for (int dy = -1; dy <= 1; dy++) {
    for (int dx = -1; dx <= 1; dx++) {
      if (!dx && !dy) continue;
      const long xx = (long)x + dx, yy = (long)y + dy;
      if (xx < 0 || yy < 0 || xx >= (long)nx || yy >= (long)ny) continue;
      uint8_t* nf = &flags[(size_t)xx + (size_t)yy * nx];
      if (*nf == ORC_GAS && (*flag & ORC_FLUID)) *nf = ORC_INTERFACE;
    }
  }
}

/* d_FreeSurface2D_2, lbmKernel2D.cu:124-148, as a gather: every writer of a
 * neighbour writes the same function of its old value. */
static void orc_fs2_flags(const orc_state* s, const uint8_t* in, uint8_t* out) {
  const uint32_t nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
  for (uint32_t y = 0; y < ny; y++) {
    for (uint32_t x = 0; x < nx; x++) {
      const size_t idx = (size_t)x + (size_t)y * nx;
      uint8_t f = in[idx];
      uint32_t nb[9];
      orc_nbrs((uint32_t)idx, x, y, nx, ny, nb);
      int any_if = 0;
      for (int i = 1; i < 9; i++) any_if |= (in[nb[i]] & ORC_IF) == ORC_IF;
      if (any_if) {
        const uint8_t e = f & ORC_IG;
        if (e == ORC_IG) f = (uint8_t)(f & ~ORC_GAS);
        else if (e == ORC_GAS) f = (uint8_t)((f & ~ORC_GAS) | ORC_GI);
      }
      out[idx] = f;
    }
  }
}

/* d_FreeSurface2D_3 flag part, lbmKernel2D.cu:178-188, as a gather. */
static void orc_fs3_flags(const orc_state* s, const uint8_t* in, uint8_t* out) {
  const uint32_t nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
  for (uint32_t y = 0; y < ny; y++) {
    for (uint32_t x = 0; x < nx; x++) {
      const size_t idx = (size_t)x + (size_t)y * nx;
      uint8_t f = in[idx];
      const uint8_t e = f & (ORC_INLET_FLUID | ORC_INTERFACE);
      if (e != ORC_INLET_FLUID && (e == ORC_FLUID || e == ORC_IF)) {
        uint32_t nb[9];
        orc_nbrs((uint32_t)idx, x, y, nx, ny, nb);
        int any_ig = 0;
        for (int i = 1; i < 9; i++) any_ig |= (in[nb[i]] & (ORC_GI | ORC_IG)) == ORC_IG;
        if (any_ig) f = (uint8_t)((f & ~ORC_IF) | ORC_INTERFACE);
      }
      out[idx] = f;
    }
  }
}

/* d_FreeSurface2D_4 flag conversions, lbmKernel2D.cu:247-267. */
static void orc_fs4_flags(const orc_state* s, const uint8_t* in, uint8_t* out) {
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
  for (size_t idx = 0; idx < s->N; idx++) {
    uint8_t f = in[idx];
    if (!(f & (ORC_WALL | ORC_MWALL | ORC_INLET))) {
      switch (f & (ORC_FGI | ORC_GI)) {
        case 5:
        case 6:
          f = (uint8_t)(f & ~ORC_INTERFACE);
          break;
        case 128:
          f = (uint8_t)((f & ~ORC_GI) | ORC_INTERFACE);
          break;
        default:
          break;
      }
    }
    out[idx] = f;
  }
}

/* ---- precision instances ------------------------------------------------ */
#define ST double
#define CT double
#define MT double
#define CT_IS_DOUBLE 1
#define ST_HALF 0
#define SFX _f64
#include "flb_oracle_body.inc"
#undef ST
#undef CT
#undef MT
#undef CT_IS_DOUBLE
#undef ST_HALF
#undef SFX

#define ST float
#define CT float
#define MT double
#define CT_IS_DOUBLE 0
#define ST_HALF 0
#define SFX _f32
#include "flb_oracle_body.inc"
#undef ST
#undef CT
#undef MT
#undef CT_IS_DOUBLE
#undef ST_HALF
#undef SFX

#define ST _Float16
#define CT float
#define MT double
#define CT_IS_DOUBLE 0
#define ST_HALF 1
#define SFX _f16s
#include "flb_oracle_body.inc"
#undef ST
#undef CT
#undef MT
#undef CT_IS_DOUBLE
#undef ST_HALF
#undef SFX

#define ST float
#define CT float
#define MT float
#define CT_IS_DOUBLE 0
#define ST_HALF 0
#define SFX _f32m32
#include "flb_oracle_body.inc"
#undef ST
#undef CT
#undef MT
#undef CT_IS_DOUBLE
#undef ST_HALF
#undef SFX

/* ---- variant dispatch --------------------------------------------------- */
typedef struct {
  void (*stream_collide)(orc_state*);
  void (*fs1)(orc_state*);
  void (*fs3_fields)(orc_state*, const uint8_t*);
  void (*fs4_fields)(orc_state*, const uint8_t*, const uint8_t*);
  void (*init)(orc_state*);
  void (*read_f64)(const orc_state*, double*);
  double (*total_mass)(const orc_state*);
  int (*fs1_options)(orc_state*, size_t, double*, double*, uint8_t*);
  int (*fs4_options)(const orc_state*, size_t, double*);
} orc_vtable;

static const orc_vtable ORC_VT[4] = {
    {stream_collide_f64, fs1_f64, fs3_fields_f64, fs4_fields_f64, init_f64, read_f64_f64, total_mass_f64,
     fs1_options_f64, fs4_options_f64},
    {stream_collide_f32, fs1_f32, fs3_fields_f32, fs4_fields_f32, init_f32, read_f64_f32, total_mass_f32,
     fs1_options_f32, fs4_options_f32},
    {stream_collide_f16s, fs1_f16s, fs3_fields_f16s, fs4_fields_f16s, init_f16s, read_f64_f16s,
     total_mass_f16s, fs1_options_f16s, fs4_options_f16s},
    {stream_collide_f32m32, fs1_f32m32, fs3_fields_f32m32, fs4_fields_f32m32, init_f32m32, read_f64_f32m32,
     total_mass_f32m32, fs1_options_f32m32, fs4_options_f32m32},
};

static void orc_free(orc_state* s) {
  if (!s) return;
  free(s->f);
  free(s->rho);
  free(s->u);
  free(s->flags);
  free(s->mass);
  free(s->excess);
  free(s->phi);
  free(s->flags_tmp);
  free(s->flags_tmp2);
  free(s->recon);
  free(s->recon_mask);
  free(s->rho_snap);
  free(s->u_snap);
  free(s);
}

orc_state* orc_create(const orc_params* p, const uint8_t* geometry_flags) {
  if (!p || !geometry_flags || p->nx < 3 || p->ny < 3) return NULL;
  if (p->variant < 0 || p->variant > 3) return NULL;
  if (!(p->tau > 0.5f)) return NULL;
  orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
  if (!s) return NULL;
  s->p = *p;
  s->nx = (uint32_t)p->nx;
  s->ny = (uint32_t)p->ny;
  s->N = (size_t)s->nx * s->ny;
  s->t = 0;
#ifdef _OPENMP
  s->nthreads = p->threads > 0 ? p->threads : omp_get_max_threads();
#else
  s->nthreads = 1;
#endif
  /* cudaInitData.cu:81-82: tau and its inverse are float */
  const float h_tau = p->tau;
  s->inv_tau = 1.0f / h_tau;
  {
    /* fused arithmetic: float constants, each operation rounded on its own */
    s->fused = p->arithmetic == 1 && p->collision == 0 && !p->subgrid;
    const float fx = p->use_force ? p->fx : 0.0f, fy = p->use_force ? p->fy : 0.0f;
    const float om = s->inv_tau;
    const float kk = 1.0f - 0.5f * om;
    const float k3 = 3.0f * kk, k9 = 9.0f * kk;
    s->fu_omc = 1.0f - om;
    s->fu_nk3 = -k3;
    s->fu_fx = fx;
    s->fu_fy = fy;
    s->fu_hfx = 0.5f * fx;
    s->fu_hfy = 0.5f * fy;
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const float a = (float)ORC_CX[i] * fx;
      const float b = (float)ORC_CY[i] * fy;
      const float cF = a + b;
      s->fu_g[q] = k3 * cF;
      s->fu_h[q] = k9 * cF;
    }
  }
  s->f16_scale = p->f16_scale > 0.0f ? p->f16_scale : 4096.0f;
  s->f16_inv_scale = 1.0f / s->f16_scale;
  s->fu_sw[0] = s->f16_scale * (4.0f / 9.0f);
  s->fu_sw[1] = s->f16_scale * (1.0f / 9.0f);
  s->fu_sw[2] = s->f16_scale * (1.0f / 36.0f);
  switch (p->variant) {
    case ORC_F64: s->s_size = 8; s->c_size = 8; s->m_size = 8; break;
    case ORC_F32: s->s_size = 4; s->c_size = 4; s->m_size = 8; break;
    case ORC_F16S: s->s_size = 2; s->c_size = 4; s->m_size = 8; break;
    default: s->s_size = 4; s->c_size = 4; s->m_size = 4; break;
  }
  const size_t N = s->N;
  s->f = calloc(9 * N, s->s_size);
  s->rho = calloc(N, s->c_size);
  s->u = calloc(2 * N, s->c_size);
  s->flags = (uint8_t*)malloc(N);
  s->mass = calloc(N, s->m_size);
  s->excess = calloc(N, s->m_size);
  s->phi = calloc(N, s->m_size);
  s->flags_tmp = (uint8_t*)malloc(N);
  s->flags_tmp2 = (uint8_t*)malloc(N);
  if (!s->f || !s->rho || !s->u || !s->flags || !s->mass || !s->excess || !s->phi || !s->flags_tmp ||
      !s->flags_tmp2) {
    orc_free(s);
    return NULL;
  }
  memcpy(s->flags, geometry_flags, N);
  for (size_t i = 0; i < N; i++) {
    if (s->flags[i] & (ORC_INLET | ORC_OUTLET)) s->has_io = 1;
    /* the inlet reads rho[idx+1] and the outlet u[idx-1] without a wrap */
    if ((s->flags[i] & ORC_INLET) && i + 1 >= N) { orc_free(s); return NULL; }
    if ((s->flags[i] & ORC_OUTLET) && i == 0) { orc_free(s); return NULL; }
  }
  if (s->has_io) {
    s->rho_snap = malloc(N * s->c_size);
    s->u_snap = malloc(2 * N * s->c_size);
    if (!s->rho_snap || !s->u_snap) { orc_free(s); return NULL; }
  }
  if (p->free_surface) {
    s->recon = malloc(8 * N * s->c_size);
    s->recon_mask = (uint8_t*)malloc(N);
    if (!s->recon || !s->recon_mask) { orc_free(s); return NULL; }
  }
  ORC_VT[p->variant].init(s);
  return s;
}

void orc_destroy(orc_state* s) { orc_free(s); }

static int orc_run(orc_state* s, int k) {
  const orc_vtable* vt = &ORC_VT[s->p.variant];
  switch (k) {
    case ORC_K_STREAM_COLLIDE:
      vt->stream_collide(s);
      return 0;
    case ORC_K_FS1:
      if (!s->p.free_surface) return -1;
      vt->fs1(s);
      return 0;
    case ORC_K_FS2:
      orc_fs2_flags(s, s->flags, s->flags_tmp);
      memcpy(s->flags, s->flags_tmp, s->N);
      return 0;
    case ORC_K_FS3:
      if (!s->p.free_surface) return -1;
      vt->fs3_fields(s, s->flags);
      orc_fs3_flags(s, s->flags, s->flags_tmp);
      memcpy(s->flags, s->flags_tmp, s->N);
      return 0;
    case ORC_K_FS4:
      if (!s->p.free_surface) return -1;
      orc_fs4_flags(s, s->flags, s->flags_tmp);
      vt->fs4_fields(s, s->flags, s->flags_tmp);
      memcpy(s->flags, s->flags_tmp, s->N);
      return 0;
    default:
      return -1;
  }
}

int orc_kernel(orc_state* s, int kernel_id) {
  if (!s) return -1;
  return orc_run(s, kernel_id);
}

/* runCuda.cu:493-528 (free surface) and :460-491 (mono-fluid). */
int orc_step(orc_state* s, uint64_t n) {
  if (!s) return -1;
  for (uint64_t k = 0; k < n; k++) {
    if (s->p.free_surface) {
      orc_run(s, ORC_K_FS1);
      orc_run(s, ORC_K_STREAM_COLLIDE);
      orc_run(s, ORC_K_FS2);
      orc_run(s, ORC_K_FS3);
      orc_run(s, ORC_K_FS4);
    } else {
      orc_run(s, ORC_K_STREAM_COLLIDE);
    }
    s->t += 1;
  }
  return 0;
}

uint64_t orc_time(const orc_state* s) { return s ? s->t : 0; }
void orc_set_time(orc_state* s, uint64_t t) {
  if (s) s->t = t;
}
size_t orc_cells(const orc_state* s) { return s ? s->N : 0; }

void* orc_field(orc_state* s, int field, size_t* elem_size) {
  if (!s) return NULL;
  size_t es = 0;
  void* ptr = NULL;
  switch (field) {
    case ORC_FIELD_F: ptr = s->f; es = s->s_size; break;
    case ORC_FIELD_RHO: ptr = s->rho; es = s->c_size; break;
    case ORC_FIELD_U: ptr = s->u; es = s->c_size; break;
    case ORC_FIELD_FLAGS: ptr = s->flags; es = 1; break;
    case ORC_FIELD_MASS: ptr = s->mass; es = s->m_size; break;
    case ORC_FIELD_EXCESS: ptr = s->excess; es = s->m_size; break;
    case ORC_FIELD_PHI: ptr = s->phi; es = s->m_size; break;
    default: break;
  }
  if (elem_size) *elem_size = es;
  return ptr;
}

void orc_read_f64(const orc_state* s, double* out) {
  if (s && out) ORC_VT[s->p.variant].read_f64(s, out);
}

int orc_fs1_options(orc_state* s, size_t idx, double* masses, double* recs, uint8_t* masks) {
  if (!s || !s->p.free_surface || idx >= s->N) return -1;
  return ORC_VT[s->p.variant].fs1_options(s, idx, masses, recs, masks);
}

int orc_fs4_options(const orc_state* s, size_t idx, double* out3) {
  if (!s || !s->p.free_surface || idx >= s->N) return -1;
  return ORC_VT[s->p.variant].fs4_options(s, idx, out3);
}

double orc_total_mass(const orc_state* s) { return s ? ORC_VT[s->p.variant].total_mass(s) : 0.0; }

/* The FP16S pair conversion as the engine issues it: binary32 bits a (upper
 * half) and b (lower half) with the random word r; for checking the
 * restatement against the instruction's recorded outputs. */
uint32_t orc_f16_rs_pair(uint32_t a, uint32_t b, uint32_t r) {
  return ((uint32_t)orc_f16_rs(a, (r >> 16) & 0x1fffu) << 16) | orc_f16_rs(b, r & 0x1fffu);
}
