// lattice.cuh -- D2Q9 constants and per-cell arithmetic of the engine.
//
// The formulas follow FlowLB src/cuda/cellCalculations.cuh with the same
// operand order and literal types, so that with --fmad=false every float and
// double operation rounds exactly as in the reference kernels.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

namespace flb {

// Cell-type bits, src/cuda/cudaInitData.cu:25-39 and src/utils.h:91-108.
enum : uint8_t {
  kFluid = 0x01,
  kGas = 0x02,
  kInterface = 0x04,
  kWall = 0x08,
  kMovingWall = 0x10,
  kInlet = 0x20,
  kOutlet = 0x40,
  kGasInterface = 0x80,
  kFGI = 0x07,
  kIF = 0x05,
  kIG = 0x06,
  kInletFluid = 0x21
};

// Directions: 0 rest, 1 +x, 2 -x, 3 +y, 4 -y, 5 +x+y, 6 -x-y, 7 +x-y, 8 -x+y
// (cudaInitData.cu:76,78); i and i+1 (odd i) are opposite.
__host__ __device__ constexpr int cx(int i) {
  return i == 1 || i == 5 || i == 7 ? 1 : (i == 2 || i == 6 || i == 8 ? -1 : 0);
}
__host__ __device__ constexpr int cy(int i) {
  return i == 3 || i == 5 || i == 8 ? 1 : (i == 4 || i == 6 || i == 7 ? -1 : 0);
}

// Weights as the reference host builds them (src/ui/app.cpp:288 float, :304 double).
template <class C>
__host__ __device__ constexpr C wgt(int i) {
  return i == 0 ? C(4) / C(9) : (i < 5 ? C(1) / C(9) : C(1) / C(36));
}

// ---- storage codecs -------------------------------------------------------
// S is the storage type of the population array, C the arithmetic type.
template <class S, class C>
struct Codec {
  __device__ __forceinline__ static C ld(const S* F, uint32_t a, int, float) { return (C)F[a]; }
  __device__ __forceinline__ static void st(S* F, uint32_t a, int, C v, float) { F[a] = (S)v; }
};

// FP16S: binary16 holds (f_i - w_i) * scale; scale is a power of two.
template <>
struct Codec<__half, float> {
  __device__ __forceinline__ static float ld(const __half* F, uint32_t a, int dir, float inv_scale) {
    // h * inv_scale is exact (power-of-two scale), so the fused form rounds once
    // like the separate multiply and add
    return __fmaf_rn(__half2float(F[a]), inv_scale, wgt<float>(dir));
  }
  __device__ __forceinline__ static void st(__half* F, uint32_t a, int dir, float v, float scale) {
    F[a] = __float2half_rn((v - wgt<float>(dir)) * scale);
  }
};

// The value population v of direction dir reads back as once it has been
// stored in the population array (S) and loaded again: v itself unless the
// storage is narrower than the arithmetic (FP16S).
template <class S, class C>
__device__ __forceinline__ C stored_value(C v, int, float, float) {
  return v;
}
template <>
__device__ __forceinline__ float stored_value<__half, float>(float v, int dir, float scale, float inv_scale) {
  __half h;
  Codec<__half, float>::st(&h, 0, dir, v, scale);
  return Codec<__half, float>::ld(&h, 0, dir, inv_scale);
}

// Raw FP16S access: the stored scaled deviation h = (f - w) * scale as a
// float, for arithmetic done in deviation units (collide_fused_dev).
// Stores round toward zero: the values arrive already rounded to binary16
// (f16_rs_one), so the store is exact.
struct RawHalf {
  __device__ __forceinline__ static float ld(const __half* F, uint32_t a, int, float) { return __half2float(F[a]); }
  __device__ __forceinline__ static void st(__half* F, uint32_t a, int, float v, float) { F[a] = __float2half_rz(v); }
};

// Stochastic rounding of the FP16S deviation units.  Rounding to nearest gives
// a value that changes slowly from step to step the same rounding error every
// step, and in near-steady flow those errors add up: on the 256x64 culvert
// channel the FP16S velocity drifts 1e-2 (relative L2) from FP64 after 10,000
// steps.  Instead every stored value rounds up with probability equal to its
// distance from the lower binary16 neighbour, deterministically: the pair of
// cells (2k, 2k+1) draws one 32-bit word per time step (a multiplicative hash
// of 2k and t, mixed by xor-shift and multiply), population i adds i*K to it,
// and cvt.rs.f16x2.f32 converts the pair with it: the low 13 bits round the
// even cell, bits 16..28 the odd one, each added below the last binary16 bit
// kept (subnormal results included) before truncation.
__host__ __device__ __forceinline__ uint32_t f16_rs_base(uint32_t idx_even, uint32_t t) {
  uint32_t x = idx_even * 0x85EBCA6Bu + t * 0x9E3779B9u;
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  return x;
}
__host__ __device__ __forceinline__ uint32_t f16_rs_bits(uint32_t base, int i) {
  return base + (uint32_t)i * 0x632BE5ABu;
}
// lo -> low half (even cell), hi -> high half (odd cell)
__device__ __forceinline__ uint32_t f2h_rs(float lo, float hi, uint32_t rbits) {
  uint32_t w;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(w) : "f"(hi), "f"(lo), "r"(rbits));
  return w;
}
// One value of cell idx rounded as in its pair, returned as the exact float of
// the binary16 result (a later round-toward-zero store keeps it).
__device__ __forceinline__ float f16_rs_one(float v, uint32_t idx, uint32_t rbits) {
  const bool odd = (idx & 1u) != 0;
  const uint32_t w = odd ? f2h_rs(0.0f, v, rbits) : f2h_rs(v, 0.0f, rbits);
  return __half2float(__ushort_as_half((unsigned short)(odd ? (w >> 16) : (w & 0xffffu))));
}

// ---- per-cell arithmetic, cellCalculations.cuh ----------------------------

// calculateDensity, cellCalculations.cuh:16-22
template <class C>
__device__ __forceinline__ C density(const C* f) {
  C rho = f[0];
#pragma unroll
  for (int i = 1; i < 9; i++) rho += f[i];
  return rho;
}

// calculateVelocityD2Q9, cellCalculations.cuh:168-174
template <class C>
__device__ __forceinline__ void velocity(const C* f, C rho, C& ux, C& uy) {
  ux = (f[1] - f[2] + f[5] - f[6] + f[7] - f[8]) / rho;
  uy = (f[3] - f[4] + f[5] - f[6] + f[8] - f[7]) / rho;
}

// calculateEquilibriumDDF2Q9, cellCalculations.cuh:32-52
template <class C>
__device__ __forceinline__ void equilibrium(C rho, C ux, C uy, C* feq) {
  const C u2 = 3.0f * (ux * ux + uy * uy);
  const C rhow14 = wgt<C>(1) * rho;
  const C rhow58 = wgt<C>(5) * rho;
  ux *= 3.0f;
  uy *= 3.0f;
  const C u0 = ux - uy;
  const C u1 = ux + uy;
  feq[0] = wgt<C>(0) * rho * (1.0f - 0.5f * u2);
  feq[1] = rhow14 * (1.0f + ux - 0.5f * u2 + 0.5f * ux * ux);
  feq[2] = rhow14 * (1.0f - ux - 0.5f * u2 + 0.5f * ux * ux);
  feq[3] = rhow14 * (1.0f + uy - 0.5f * u2 + 0.5f * uy * uy);
  feq[4] = rhow14 * (1.0f - uy - 0.5f * u2 + 0.5f * uy * uy);
  feq[5] = rhow58 * (1.0f + u1 - 0.5f * u2 + 0.5f * u1 * u1);
  feq[6] = rhow58 * (1.0f - u1 - 0.5f * u2 + 0.5f * u1 * u1);
  feq[7] = rhow58 * (1.0f + u0 - 0.5f * u2 + 0.5f * u0 * u0);
  feq[8] = rhow58 * (1.0f - u0 - 0.5f * u2 + 0.5f * u0 * u0);
}

// calculateForcingTerms2D (Guo), cellCalculations.cuh:64-73.  cF[i] is the
// cell-independent factor cx[i]*Fx + cy[i]*Fy, evaluated once in float with
// the same operations (see flb_create).
template <class C>
__device__ __forceinline__ void forcing(C* Fi, C ux, C uy, float Fx, float Fy, const float* cF) {
  const C uF = -0.33333334f * (ux * Fx + uy * Fy);
  Fi[0] = 9.0f * wgt<C>(0) * uF;
#pragma unroll
  for (int i = 1; i < 9; i++) Fi[i] = 9.0f * wgt<C>(i) * (cF[i] * (cx(i) * ux + cy(i) * uy + 0.33333334f) + uF);
}

// calculatePhi, cellCalculations.cuh:153-158: the quotient is clamped in
// float (__saturatef) whatever the precision.
template <class M, class C>
__device__ __forceinline__ M fill_level(M m, C rho) {
  if (rho > 0.0f) return (M)__saturatef((float)(m / (M)rho));
  return (M)0.5f;
}

// Optional velocity limiter (no reference counterpart; off unless u_max > 0):
// scales u down to |u| = u_max.
template <class C>
__device__ __forceinline__ void limit_u(float umax, C& ux, C& uy) {
  if (!(umax > 0.0f)) return;
  const C uu = ux * ux + uy * uy;
  if (uu > umax * umax) {
    const C sc = umax / sqrt(uu);
    ux = ux * sc;
    uy = uy * sc;
  }
}

// ---- fused arithmetic (no reference counterpart) ---------------------------
// The reference evaluates density, velocity, equilibrium, Guo forcing and the
// BGK relaxation as separate expressions (about 200 float operations per
// cell, all of them rounded separately).  The fused form below gives the same
// second-order BGK + Guo update with fused multiply-adds and shared
// subexpressions, about 80 operations:
//   f_i <- (1-w) f_i + w_i [B + g_i + cu (3A + h_i + 4.5 A cu)]
//   A = w rho,  B = A (1 - 1.5 u.u) - 3k u.F,  cu = c_i.u,
//   g_i = 3k c_i.F,  h_i = 9k c_i.F,  k = 1 - w/2,
// which expands to (1-w) f_i + w feq_i + k F_i.  Opposite directions share
// E = B + cu (h_i + 4.5 A cu) and O = g_i + 3A cu: t_i = E + O, t_opp = E - O.
// Every fused multiply-add is written out, so its rounding is fixed and a CPU
// restatement with fma()/fmaf() matches bit for bit.
__device__ __forceinline__ float fmac(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmac(double a, double b, double c) { return __fma_rn(a, b, c); }
// correctly rounded 1/x (the same value as 1/x with IEEE division)
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }

// Density, momentum and 1/rho in the fused form (pairwise sums).
template <class C>
__device__ __forceinline__ void moments_fused(const C* f, C& rho, C& jx, C& jy, C& inv) {
  const C s12 = f[1] + f[2], s34 = f[3] + f[4], s56 = f[5] + f[6], s78 = f[7] + f[8];
  const C d12 = f[1] - f[2], d34 = f[3] - f[4], d56 = f[5] - f[6], d78 = f[7] - f[8];
  rho = ((f[0] + s12) + (s34 + s56)) + s78;
  jx = (d12 + d56) + d78;
  jy = (d34 + d56) - d78;
  inv = rcp(rho);
}

// The relaxation with forcing, from the force-shifted (and limited) velocity.
template <class C>
__device__ __forceinline__ void collide_fused(C* f, C rho, C ux, C uy, float om, float omc, float nk3, float fx,
                                              float fy, const float* g, const float* h) {
  const C usq = fmac(ux, ux, uy * uy);
  const C uF = fmac(ux, (C)fx, uy * (C)fy);
  const C A = (C)om * rho;
  const C t1 = fmac(C(-1.5f), usq, C(1));
  const C B = fmac(A, t1, (C)nk3 * uF);
  const C A3 = C(3) * A, A45 = C(4.5f) * A;
  const C w = (C)omc;
  f[0] = fmac(w, f[0], wgt<C>(0) * B);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const C cu = q == 0 ? ux : (q == 1 ? uy : (q == 2 ? ux + uy : ux - uy));
    const C E = fmac(cu, fmac(A45, cu, (C)h[q]), B);
    const C O = fmac(A3, cu, (C)g[q]);
    const C wi = wgt<C>(i);
    f[i] = fmac(w, f[i], wi * (E + O));
    f[i + 1] = fmac(w, f[i + 1], wi * (E - O));
  }
}

// The fused update in FP16S deviation units (single phase): h_i = S (f_i - w_i)
// goes in and out without conversion to f.  With rho = 1 + delta,
//   h_i <- (1-w) h_i + S w_i (t_i - w),   t_i - w = Bd + g_i + cu (3A + h_i' + 4.5 A cu),
//   Bd = w (delta t1 - 1.5 u.u) - 3k u.F,  t1 = 1 - 1.5 u.u,
// the same update as collide_fused (the +-w_i of the codec cancel).
// rho, ux, uy: out; h: in/out.  LIM: apply the velocity limiter (u_max > 0);
// without it the limiter code is not in the instruction stream at all (5 % of
// the FP16S step on a B200).
struct DevOut {
  float rho, ux, uy;
};
template <bool LIM = true>
__device__ __forceinline__ DevOut collide_fused_dev(float* h, float invS, float om, float omc, float nk3, float hfx,
                                                    float hfy, float fx, float fy, float umax, const float* g,
                                                    const float* hh, const float* sw) {
  const float s12 = h[1] + h[2], s34 = h[3] + h[4], s56 = h[5] + h[6], s78 = h[7] + h[8];
  const float d12 = h[1] - h[2], d34 = h[3] - h[4], d56 = h[5] - h[6], d78 = h[7] - h[8];
  const float dS = ((h[0] + s12) + (s34 + s56)) + s78;
  const float jx = (d12 + d56) + d78, jy = (d34 + d56) - d78;
  const float delta = dS * invS;
  const float rho = fmac(dS, invS, 1.0f);
  const float inv = rcp(rho);
  const float invs = inv * invS;
  float ux = fmac(hfx, inv, jx * invs);
  float uy = fmac(hfy, inv, jy * invs);
  if (LIM) limit_u(umax, ux, uy);
  const float usq = fmac(ux, ux, uy * uy);
  const float uF = fmac(ux, fx, uy * fy);
  const float A = om * rho;
  const float t1 = fmac(-1.5f, usq, 1.0f);
  const float x = fmac(delta, t1, -1.5f * usq);
  const float Bd = fmac(om, x, nk3 * uF);
  const float A3 = 3.0f * A, A45 = 4.5f * A;
  h[0] = fmac(omc, h[0], sw[0] * Bd);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const float cu = q == 0 ? ux : (q == 1 ? uy : (q == 2 ? ux + uy : ux - uy));
    const float E = fmac(cu, fmac(A45, cu, hh[q]), Bd);
    const float O = fmac(A3, cu, g[q]);
    const float swi = sw[q < 2 ? 1 : 2];
    h[i] = fmac(omc, h[i], swi * (E + O));
    h[i + 1] = fmac(omc, h[i + 1], swi * (E - O));
  }
  return DevOut{rho, ux, uy};
}

// Neighbour cells with periodic wrap, cellCalculations.cuh:82-109.
__device__ __forceinline__ void neighbours(uint32_t x, uint32_t y, uint32_t nx, uint32_t ny, uint32_t* nb) {
  const uint32_t yc = y * nx;
  const uint32_t yu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t yd = (y == 0u ? ny - 1u : y - 1u) * nx;
  const uint32_t xr = x + 1u == nx ? 0u : x + 1u;
  const uint32_t xl = x == 0u ? nx - 1u : x - 1u;
  nb[0] = x + yc;
  nb[1] = xr + yc;
  nb[2] = xl + yc;
  nb[3] = x + yu;
  nb[4] = x + yd;
  nb[5] = xr + yu;
  nb[6] = xl + yd;
  nb[7] = xr + yd;
  nb[8] = xl + yu;
}

}  // namespace flb
