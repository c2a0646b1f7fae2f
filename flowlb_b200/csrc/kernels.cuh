// kernels.cuh -- the engine's sm_100a kernels.
//
// Layout in HBM (structure of arrays, reference layout, one population buffer):
//   f      9N  S   slot s of cell c at f[c + s*N], updated in place by the
//                  esoteric-pull pattern (loads and stores of a cell hit the
//                  same 9 addresses, so no second buffer is needed)
//   rho     N  C   density of the incoming populations of the last step
//   u      2N  C   force-shifted velocity, u_x then u_y
//   flags  2xN u8  cell types; two buffers, the flag stencil pass reads one
//                  and writes the other
//   nbmask  N  u8  bit i-1 set when neighbour i is a wall (half-way walls)
//   mass, excess, phi  N  M   free-surface cell mass, excess mass share, fill level
//   recon  8N  C   populations rebuilt by FS_1 toward gas (reference mode only)
// S/C/M: storage / arithmetic / mass types.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

#include "lattice.cuh"

namespace flb {

constexpr int kBlock = 256;

struct KParams {
  uint32_t nx, ny, N;
  void* f;
  void* rho;
  void* u;
  uint8_t* flags;      // current flags
  uint8_t* flags_out;  // flag stencil pass output
  const uint8_t* nbmask;
  void* mass;
  void* excess;
  void* phi;
  void* recon;
  uint8_t* recon_mask;
  const void* rho_snap;
  const void* u_snap;
  float inv_tau, fx, fy;
  float f16_scale, f16_inv;
  double inlet_ux, inlet_uy;
  int use_force, subgrid, collision, fs_cons, count_pre;
  // 1 when flags_out holds the previous step's post-stream-collide flags and
  // the mass fields come from the previous full step (see k_fs234)
  int trust_prev;
};

// ---- population access helpers -------------------------------------------
// Slot a = the cell's own slot holding incoming population i, slot b = the
// neighbour's slot holding incoming population i+1 (cellCalculations.cuh:185-238).

template <class S, class C>
__device__ __forceinline__ void load_incoming(const S* F, uint32_t idx, const uint32_t* nb, uint32_t N, uint32_t odd,
                                              float inv, C* f) {
  f[0] = Codec<S, C>::ld(F, idx, 0, inv);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    f[i] = Codec<S, C>::ld(F, idx + N * a, i, inv);
    f[i + 1] = Codec<S, C>::ld(F, nb[i] + N * b, i + 1, inv);
  }
}

// storef plus the half-way redirect: a population aimed at a wall neighbour is
// also written where this cell loads the opposite direction at t+1 (its
// regular slot belongs to the wall cell and is never read).
template <class S, class C, bool HW>
__device__ __forceinline__ void store_post(S* F, uint32_t idx, const uint32_t* nb, uint32_t N, uint32_t odd,
                                           uint32_t nbm, float scale, const C* f) {
  Codec<S, C>::st(F, idx, 0, f[0], scale);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    Codec<S, C>::st(F, nb[i] + N * b, i, f[i], scale);
    if (HW && ((nbm >> (i - 1)) & 1u)) Codec<S, C>::st(F, nb[i] + N * a, i, f[i], scale);
    Codec<S, C>::st(F, idx + N * a, i + 1, f[i + 1], scale);
    if (HW && ((nbm >> i) & 1u)) Codec<S, C>::st(F, idx + N * b, i + 1, f[i + 1], scale);
  }
}

// ---- initial state ----------------------------------------------------------

// Free-surface interface layer and fields (initData.cpp:13-37 with the bounded
// neighbour list of :39-124, initData.h:175-206).  The reference sweeps cells
// in index order and initialises each cell's fields right after visiting it;
// that makes the result a per-cell rule: a GAS cell next to a fluid source
// becomes INTERFACE, and gets m = phi = 0.5 only if some source precedes it in
// index order (otherwise it was initialised as gas).
__global__ void k_init_flags(const uint8_t* __restrict__ geo, uint8_t* __restrict__ flags, uint32_t nx, uint32_t ny,
                             int free_surface, void* mass_v, void* excess_v, void* phi_v, int mass_f64) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= nx) return;
  const uint32_t idx = x + y * nx;
  uint8_t g = geo[idx];
  if (!free_surface) {
    flags[idx] = g;
    return;
  }
  auto source = [](uint8_t v) -> bool {
    return !(v & ~(kFluid | kInlet | kOutlet)) && (v & (kFluid | kInlet));
  };
  uint8_t f = g;
  bool early = false, any = false;
  if (g == kGas) {
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        if (!dx && !dy) continue;
        const long xx = (long)x + dx, yy = (long)y + dy;
        if (xx < 0 || yy < 0 || xx >= (long)nx || yy >= (long)ny) continue;
        const uint32_t n = (uint32_t)xx + (uint32_t)yy * nx;
        if (source(geo[n])) {
          any = true;
          if (n < idx) early = true;
        }
      }
    if (any) f = kInterface;
  } else if (!(g & ~(kFluid | kInlet | kOutlet))) {
    if (g & kInlet) f = g | kFluid;
    else if (g & kOutlet) f = g | kGas;
  }
  flags[idx] = f;
  double m = 0.0, ph = 0.0;
  bool set = true;
  switch (f) {
    case kFluid:
    case kFluid | kInlet:
    case kFluid | kOutlet: m = 1.0; ph = 1.0; break;
    case kGas:
    case kGas | kOutlet: m = 0.0; ph = 0.0; break;
    case kInterface:
      m = early ? 0.5 : 0.0;
      ph = early ? 0.5 : 0.0;
      break;
    default: set = false; break;
  }
  if (!set) m = ph = 0.0;
  if (mass_f64) {
    ((double*)mass_v)[idx] = m;
    ((double*)phi_v)[idx] = ph;
    ((double*)excess_v)[idx] = 0.0;
  } else {
    ((float*)mass_v)[idx] = (float)m;
    ((float*)phi_v)[idx] = (float)ph;
    ((float*)excess_v)[idx] = 0.0f;
  }
}

// Solid-neighbour mask for half-way walls.
__global__ void k_nbmask(const uint8_t* __restrict__ flags, uint8_t* __restrict__ nbmask, uint32_t nx, uint32_t ny) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= nx) return;
  uint32_t nb[9];
  neighbours(x, y, nx, ny, nb);
  uint32_t m = 0;
#pragma unroll
  for (int i = 1; i < 9; i++) m |= (flags[nb[i]] & kWall) ? (1u << (i - 1)) : 0u;
  nbmask[x + y * nx] = (uint8_t)m;
}

// f = feq(rho=1, u) with the host's double arithmetic (initEquilibriumDDF2Q9,
// initData.h:75-100) stored with the t=1 pattern (initData.h:102-112, :155);
// rho = 1; u = inlet velocity on INLET cells, else 0 (initData.h:125-148).
// With half-way walls wall cells store nothing and the redirect applies.
template <class S, class C, bool HW>
__global__ void k_init_ddf(const __grid_constant__ KParams p, const uint8_t* __restrict__ geo) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t N = p.N, idx = x + y * p.nx;
  C* R = static_cast<C*>(p.rho);
  C* U = static_cast<C*>(p.u);
  const uint8_t g = geo[idx];
  C ux, uy;
  if (g & kInlet) {
    ux = (C)p.inlet_ux;
    uy = (C)p.inlet_uy;
  } else {
    ux = 0;
    uy = 0;
  }
  U[idx] = ux;
  U[idx + N] = uy;
  const double rho = 1.0;
  R[idx] = (C)rho;
  if (HW && (g & kWall)) return;
  const double u2 = 3.0 * (ux * ux + uy * uy);
  const double rhow14 = wgt<C>(1) * rho;
  const double rhow58 = wgt<C>(5) * rho;
  ux *= 3.0;
  uy *= 3.0;
  const double u0 = ux - uy;
  const double u1 = ux + uy;
  C feq[9];
  feq[0] = (C)(wgt<C>(0) * rho * (1.0 - 0.5 * u2));
  feq[1] = (C)(rhow14 * (1.0 + ux - 0.5 * u2 + 0.5 * ux * ux));
  feq[2] = (C)(rhow14 * (1.0 - ux - 0.5 * u2 + 0.5 * ux * ux));
  feq[3] = (C)(rhow14 * (1.0 + uy - 0.5 * u2 + 0.5 * uy * uy));
  feq[4] = (C)(rhow14 * (1.0 - uy - 0.5 * u2 + 0.5 * uy * uy));
  feq[5] = (C)(rhow58 * (1.0 + u1 - 0.5 * u2 + 0.5 * u1 * u1));
  feq[6] = (C)(rhow58 * (1.0 - u1 - 0.5 * u2 + 0.5 * u1 * u1));
  feq[7] = (C)(rhow58 * (1.0 + u0 - 0.5 * u2 + 0.5 * u0 * u0));
  feq[8] = (C)(rhow58 * (1.0 - u0 - 0.5 * u2 + 0.5 * u0 * u0));
  uint32_t nb[9];
  neighbours(x, y, p.nx, p.ny, nb);
  store_post<S, C, HW>(static_cast<S*>(p.f), idx, nb, N, 1u, HW ? p.nbmask[idx] : 0u, p.f16_scale, feq);
}

// ---- stream-collide: d_StreamCollide2D, lbmKernel2D.cu:306-519 -------------
// One thread per cell.  FS: free-surface build (interface marking, rebuilt
// populations); HW: half-way walls; WM: write density and velocity.
template <class S, class C, class M, bool FS, bool HW, bool WM>
__global__ void __launch_bounds__(kBlock) k_stream_collide(const __grid_constant__ KParams p, uint32_t odd) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t nx = p.nx, N = p.N;
  const uint32_t idx = x + y * nx;
  uint8_t* flags = p.flags;
  const uint8_t flag = flags[idx];
  if (flag & (kGas | kWall)) return;
  uint32_t nb[9];
  neighbours(x, y, nx, p.ny, nb);
  S* F = static_cast<S*>(p.f);
  C f[9];
  load_incoming<S, C>(F, idx, nb, N, odd, p.f16_inv, f);
  if constexpr (FS) {
    // reference mode: FS_1 left the populations it rebuilt toward gas here
    if (!p.fs_cons && (flag & (kFGI | kInlet)) == kInterface) {
      const uint32_t m = p.recon_mask[idx];
      if (m) {
        const C* rec = static_cast<const C*>(p.recon);
#pragma unroll
        for (int k = 0; k < 8; k++)
          if ((m >> k) & 1u) f[k + 1] = rec[(uint32_t)k * N + idx];
      }
    }
  }
  C rho, ux, uy;
  const uint8_t io = flag & (kInlet | kOutlet);
  if (io & kInlet) {
    const C* Rs = static_cast<const C*>(p.rho_snap);
    const C* Us = static_cast<const C*>(p.u_snap);
    rho = Rs[idx + 1];
    ux = Us[idx];
    uy = Us[idx + N];
  } else if (flag & kOutlet) {
    const C* Rs = static_cast<const C*>(p.rho_snap);
    const C* Us = static_cast<const C*>(p.u_snap);
    rho = Rs[idx];
    ux = Us[idx - 1];
    uy = Us[idx + N - 1];
  } else {
    rho = density(f);
    velocity(f, rho, ux, uy);
  }
  if constexpr (FS) {
    if ((flag & kInterface) == kInterface) {
      const M m = static_cast<const M*>(p.mass)[idx];
      bool notFluid = true, notGas = true;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        const uint8_t e = flags[nb[i]] & kFGI;
        notFluid = notFluid && (e != kFluid);
        notGas = notGas && (e != kGas);
      }
      // neighbours read these bytes concurrently; IF/IG compare unequal to
      // FLUID and GAS either way, so the outcome does not depend on timing
      if ((m > 1.001f * rho) || notGas) flags[idx] = (uint8_t)((flag & ~kFGI) | kIF);
      else if ((m < -0.001f) || notFluid) flags[idx] = (uint8_t)((flag & ~kFGI) | kIG);
    }
  }
  C Fi[9];
  const bool use_force = p.use_force != 0;
  if (use_force) {
    const C rhol2 = 0.5f / rho;
    ux = ux + rhol2 * p.fx;
    uy = uy + rhol2 * p.fy;
    forcing(Fi, ux, uy, p.fx, p.fy);
  }
  if (FS || WM) {
    C* R = static_cast<C*>(p.rho);
    C* U = static_cast<C*>(p.u);
    if (!io) {
      U[idx] = ux;
      U[idx + N] = uy;
    } else if (flag & kOutlet) {
      U[idx] = ux;
      U[idx + N] = uy;
    }
    R[idx] = rho;
  }
  C feq[9];
  equilibrium(rho, ux, uy, feq);
  float invTau = p.inv_tau;
  if (p.subgrid) {
    C Hxx = 0.0f, Hyy = 0.0f, Hxy = 0.0f;
#pragma unroll
    for (int i = 1; i < 9; i++) {
      const C fne = f[i] - feq[i];
      const C ccx = (C)cx(i), ccy = (C)cy(i);
      Hxx += ccx * ccx * fne;
      Hyy += ccy * ccy * fne;
      Hxy += ccx * ccy * fne;
    }
    const C Q = Hxx * Hxx + Hyy * Hyy + 2.0f * Hxy * Hxy;
    const float tau = 1.0f / invTau;
    invTau = 2.0f / (tau + sqrtf(tau * tau + 0.54037965f * sqrtf(Q) / rho));
  }
  if (p.collision == 0) {
    if (!io) {
      if (use_force) {
        const float taul = 1.0f - 0.5f * invTau;
#pragma unroll
        for (int i = 0; i < 9; i++) f[i] = (1.0f - invTau) * f[i] + invTau * feq[i] + taul * Fi[i];
      } else {
#pragma unroll
        for (int i = 0; i < 9; i++) f[i] = (1.0f - invTau) * f[i] + invTau * feq[i];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = feq[i];
    }
  } else {
    const float invTauPos = invTau;
    const float invTauNeg = 1.0f / (0.25f / (1.0f / invTau - 0.5f) + 0.5f);
    if (!io) {
      if (!use_force) {  // with forcing the reference leaves TRT empty (lbmKernel2D.cu:485-488)
        f[0] = f[0] - invTauPos * (f[0] - feq[0]);
#pragma unroll
        for (int i = 1; i < 9; i += 2) {
          const float fMinusFeq = f[i] - feq[i] + f[i + 1] - feq[i + 1];
          const float fAnti = f[i] - f[i + 1];
          const float feqAnti = feq[i] - feq[i + 1];
          f[i] = f[i] - 0.5f * invTauPos * fMinusFeq - 0.5f * invTauNeg * (fAnti - feqAnti);
          f[i + 1] = f[i + 1] - 0.5f * invTauPos * fMinusFeq - 0.5f * invTauNeg * (feqAnti - fAnti);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = feq[i];
    }
  }
  store_post<S, C, HW>(F, idx, nb, N, odd, HW ? p.nbmask[idx] : 0u, p.f16_scale, f);
}

// ---- FS_1: mass exchange and gas reconstruction, lbmKernel2D.cu:14-121 -----
template <class S, class C, class M, bool HW>
__global__ void __launch_bounds__(kBlock) k_fs1(const __grid_constant__ KParams p, uint32_t odd) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t nx = p.nx, N = p.N;
  const uint32_t idx = x + y * nx;
  const uint8_t* flags = p.flags;
  const uint8_t flag = flags[idx];
  if (flag & (kGas | kWall | kInlet)) return;
  const bool cons = p.fs_cons != 0;
  const uint8_t e = flag & kFGI;
  if (cons && (!(e == kFluid || e == kInterface) || (flag & kMovingWall))) return;
  uint32_t nb[9];
  neighbours(x, y, nx, p.ny, nb);
  S* F = static_cast<S*>(p.f);
  const float inv = p.f16_inv;
  C in[9], out[9];
  load_incoming<S, C>(F, idx, nb, N, odd, inv, in);
  out[0] = in[0];
  const uint32_t nbm = HW ? p.nbmask[idx] : 0u;
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    if (HW && ((nbm >> (i - 1)) & 1u)) out[i] = in[i + 1];
    else out[i] = Codec<S, C>::ld(F, nb[i] + N * a, i, inv);
    if (HW && ((nbm >> i) & 1u)) out[i + 1] = in[i];
    else out[i + 1] = Codec<S, C>::ld(F, idx + N * b, i + 1, inv);
  }
  M* Ms = static_cast<M*>(p.mass);
  const M* Ex = static_cast<const M*>(p.excess);
  const M* Ph = static_cast<const M*>(p.phi);
  M m = Ms[idx];
#pragma unroll
  for (int i = 1; i < 9; i++) m += Ex[nb[i]];
  if (e == kFluid) {
    if (!cons) {
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        m += in[i + 1] - out[i];
        m += in[i] - out[i + 1];
      }
    } else {
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        const uint8_t na = flags[nb[i]] & kFGI, nbb = flags[nb[i + 1]] & kFGI;
        if (na == kFluid || na == kInterface) m += in[i + 1] - out[i];
        if (nbb == kFluid || nbb == kInterface) m += in[i] - out[i + 1];
      }
    }
  } else if (e == kInterface) {
    C rho, ux, uy, rhoYL = 0.0f;
    if (flag & (kInlet | kOutlet)) {
      rho = static_cast<const C*>(p.rho)[idx];
      ux = static_cast<const C*>(p.u)[idx];
      uy = static_cast<const C*>(p.u)[idx + N];
    } else {
      rho = density(out);
      velocity(out, rho, ux, uy);
    }
    M phiN[9];
#pragma unroll
    for (int i = 1; i < 9; i++) phiN[i] = Ph[nb[i]];
    phiN[0] = cons ? Ph[idx] : fill_level<M, C>(m, rho);
    const C rho2 = 0.5f / rho;
    ux = ux + rho2 * p.fx;
    uy = uy + rho2 * p.fy;
    C feq[9];
    equilibrium<C>(1.0f - rhoYL, ux, uy, feq);
    uint8_t nF[9];
#pragma unroll
    for (int i = 1; i < 9; i++) nF[i] = flags[nb[i]] & kFGI;
#pragma unroll
    for (int i = 1; i < 9; i += 2) {
      uint8_t ne = nF[i];
      if (ne == kFluid) m += in[i + 1] - out[i];
      else if (ne == kInterface) m += (in[i + 1] - out[i]) * 0.5f * (phiN[i] + phiN[0]);
      ne = nF[i + 1];
      if (ne == kFluid) m += in[i] - out[i + 1];
      else if (ne == kInterface) m += (in[i] - out[i + 1]) * 0.5f * (phiN[i + 1] + phiN[0]);
    }
#pragma unroll
    for (int i = 1; i < 9; i += 2) {
      in[i] = feq[i] - out[i + 1] + feq[i + 1];
      in[i + 1] = feq[i + 1] - out[i] + feq[i];
    }
    if (!cons) {
      // reference gate (storeReconstructedGasf, cellCalculations.cuh:250-259):
      // tests the neighbour the population travels toward.  Parked in recon so
      // that neighbours reading their outgoing slots see the pre-pass values.
      C* rec = static_cast<C*>(p.recon);
      uint32_t mask = 0;
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        if (nF[i] == kGas) { mask |= 1u << (i - 1); rec[(uint32_t)(i - 1) * N + idx] = in[i]; }
        if (nF[i + 1] == kGas) { mask |= 1u << i; rec[(uint32_t)i * N + idx] = in[i + 1]; }
      }
      p.recon_mask[idx] = (uint8_t)mask;
    } else {
      // population arriving from a gas neighbour: its slot is read by no other
      // cell in this pass (the gas cell does not run), so store in place
      const float scale = p.f16_scale;
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
        if (nF[i + 1] == kGas) Codec<S, C>::st(F, idx + N * a, i, in[i], scale);
        if (nF[i] == kGas) Codec<S, C>::st(F, nb[i] + N * b, i + 1, in[i + 1], scale);
      }
    }
  }
  Ms[idx] = m;
}

// Writes the populations FS_1 parked in recon (reference mode) into their
// incoming slots, as the reference FS_1 kernel does itself.  Only the
// isolated-pass path uses it; a full step hands them to stream-collide.
template <class S, class C>
__global__ void k_apply_recon(const __grid_constant__ KParams p, uint32_t odd) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t N = p.N, idx = x + y * p.nx;
  const uint8_t flag = p.flags[idx];
  if ((flag & (kFGI | kGas | kWall | kInlet)) != kInterface) return;
  const uint32_t m = p.recon_mask[idx];
  if (!m) return;
  uint32_t nb[9];
  neighbours(x, y, p.nx, p.ny, nb);
  S* F = static_cast<S*>(p.f);
  const C* rec = static_cast<const C*>(p.recon);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    if ((m >> (i - 1)) & 1u) Codec<S, C>::st(F, idx + N * a, i, rec[(uint32_t)(i - 1) * N + idx], p.f16_scale);
    if ((m >> i) & 1u) Codec<S, C>::st(F, nb[i] + N * b, i + 1, rec[(uint32_t)i * N + idx], p.f16_scale);
  }
  p.recon_mask[idx] = 0;
}

// ---- FS_2 + FS_3 + FS_4 fused: lbmKernel2D.cu:124-303 ----------------------
// The three reference passes are flag stencils of radius one, chained; a tile
// of 32x8 cells stages the flags of its 3-cell halo in shared memory and
// evaluates the chain there, so neighbour flags are never read while another
// block rewrites them.  Reads p.flags, writes p.flags_out.
constexpr int kTX = 32, kTY = 8, kHalo = 3;
constexpr int kSX = kTX + 2 * kHalo, kSY = kTY + 2 * kHalo;

__device__ __forceinline__ int wrapi(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

template <class S, class C, class M, bool HW>
__global__ void __launch_bounds__(kTX* kTY) k_fs234(const __grid_constant__ KParams p, uint32_t odd) {
  __shared__ uint8_t s0[kSY][kSX];  // after stream-collide
  __shared__ uint8_t s1[kSY][kSX];  // after FS_2
  __shared__ uint8_t s2[kSY][kSX];  // after FS_3
  __shared__ uint8_t s3[kSY][kSX];  // after FS_4 conversion
  const int nx = (int)p.nx, ny = (int)p.ny;
  const int x0 = (int)blockIdx.x * kTX - kHalo, y0 = (int)blockIdx.y * kTY - kHalo;
  const int tid = threadIdx.x + threadIdx.y * kTX;
  const uint8_t* flags = p.flags;
  for (int k = tid; k < kSX * kSY; k += kTX * kTY) {
    const int lx = k % kSX, ly = k / kSX;
    s0[ly][lx] = flags[wrapi(x0 + lx, nx) + wrapi(y0 + ly, ny) * nx];
  }
  __syncthreads();
  // FS_2: next to an IF cell, IG -> I and G -> GI
  for (int k = tid; k < kSX * kSY; k += kTX * kTY) {
    const int lx = k % kSX, ly = k / kSX;
    if (lx < 1 || ly < 1 || lx >= kSX - 1 || ly >= kSY - 1) continue;
    uint8_t f = s0[ly][lx];
    bool any_if = false;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
      for (int dx = -1; dx <= 1; dx++)
        if (dx || dy) any_if |= (s0[ly + dy][lx + dx] & kIF) == kIF;
    if (any_if) {
      const uint8_t e = f & kIG;
      if (e == kIG) f = (uint8_t)(f & ~kGas);
      else if (e == kGas) f = (uint8_t)((f & ~kGas) | kGasInterface);
    }
    s1[ly][lx] = f;
  }
  __syncthreads();
  // FS_3 flags: next to an IG cell, F / IF (not inlet) -> I
  for (int k = tid; k < kSX * kSY; k += kTX * kTY) {
    const int lx = k % kSX, ly = k / kSX;
    if (lx < 2 || ly < 2 || lx >= kSX - 2 || ly >= kSY - 2) continue;
    uint8_t f = s1[ly][lx];
    const uint8_t e = f & (kInletFluid | kInterface);
    if (e != kInletFluid && (e == kFluid || e == kIF)) {
      bool any_ig = false;
#pragma unroll
      for (int dy = -1; dy <= 1; dy++)
#pragma unroll
        for (int dx = -1; dx <= 1; dx++)
          if (dx || dy) any_ig |= (s1[ly + dy][lx + dx] & (kGasInterface | kIG)) == kIG;
      if (any_ig) f = (uint8_t)((f & ~kIF) | kInterface);
    }
    s2[ly][lx] = f;
    // FS_4 conversion
    uint8_t g = f;
    if (!(g & (kWall | kMovingWall | kInlet))) {
      const uint8_t sw = g & (kFGI | kGasInterface);
      if (sw == kIF || sw == kIG) g = (uint8_t)(g & ~kInterface);
      else if (sw == kGasInterface) g = (uint8_t)((g & ~kGasInterface) | kInterface);
    }
    s3[ly][lx] = g;
  }
  __syncthreads();
  const int lx = threadIdx.x + kHalo, ly = threadIdx.y + kHalo;
  const int gx = (int)blockIdx.x * kTX + (int)threadIdx.x, gy = (int)blockIdx.y * kTY + (int)threadIdx.y;
  if (gx >= nx || gy >= ny) return;
  const uint32_t N = p.N, idx = (uint32_t)gx + (uint32_t)gy * (uint32_t)nx;
  const uint8_t f1 = s1[ly][lx];
  const uint8_t f3 = s2[ly][lx];
  const uint8_t fin = s3[ly][lx];
  // Write skipping.  flags_out still holds this cell's flag after the previous
  // step's stream-collide ("old").  When the buffers come from consecutive
  // full steps (trust_prev), a value already in memory is not rewritten:
  //  * the flag, when old equals the new flag;
  //  * all mass fields of a cell that was gas in the previous step and stays
  //    gas: that step (or the initial state) left m = excess = phi = +0, and
  //    FS_1 does not touch gas cells, so FS_4 would write the same zeros;
  //  * the fill level of a cell that was fluid after the previous step and
  //    stays fluid: it is already 1.
  const bool trust = p.trust_prev != 0;
  const uint8_t old = p.flags_out[idx];
  if (!trust || old != fin) p.flags_out[idx] = fin;
  const C* R = static_cast<const C*>(p.rho);
  const C* U = static_cast<const C*>(p.u);
  uint32_t nb[9];
  neighbours((uint32_t)gx, (uint32_t)gy, (uint32_t)nx, (uint32_t)ny, nb);
  // FS_3 fields: a gas->interface cell starts from feq of the neighbour
  // average (calculateAverageValuesNeighbors2D, accumulating in float)
  if ((f1 & (kGasInterface | kIG)) == kGasInterface) {
    float count = 0.0f, lrho = 0.0f, lux = 0.0f, luy = 0.0f;
    const int ddx[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    const int ddy[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
#pragma unroll
    for (int i = 1; i < 9; i++) {
      if (s1[ly + ddy[i]][lx + ddx[i]] & kIF) {
        count += 1.0f;
        lrho += R[nb[i]];
        lux += U[nb[i]];
        luy += U[nb[i] + N];
      }
    }
    C rho = count > 0.0f ? lrho / count : 0.0f;
    C ux = count > 0.0f ? lux / count : 0.0f;
    C uy = count > 0.0f ? luy / count : 0.0f;
    C feq[9];
    const C rho2 = 0.5f / rho;
    ux = ux + rho2 * p.fx;
    uy = uy + rho2 * p.fy;
    equilibrium(rho, ux, uy, feq);
    store_post<S, C, HW>(static_cast<S*>(p.f), idx, nb, N, odd, HW ? p.nbmask[idx] : 0u, p.f16_scale, feq);
  }
  // FS_4 fields
  if (f3 & (kWall | kMovingWall | kInlet)) return;
  const uint8_t sw4 = f3 & (kFGI | kGasInterface);
  if (trust && sw4 == kGas && (old & (kFGI | kGasInterface)) == kGas) return;
  const bool keep_phi = trust && sw4 == kFluid && (s0[ly][lx] & (kFGI | kGasInterface)) == kFluid;
  M* Ms = static_cast<M*>(p.mass);
  const C rho = R[idx];
  M m = Ms[idx];
  M ex = 0.0f, ph = 0.0f;
  switch (f3 & (kFGI | kGasInterface)) {
    case 1:
    case 5:
      ex = m - rho;
      m = rho;
      ph = 1.0f;
      break;
    case 2:
    case 6:
      ex = m;
      m = 0.0f;
      ph = 0.0f;
      break;
    case 4:
    case 128:
      if (m > rho) {
        ex = m - rho;
        m = rho;
      } else if (m < 0.0f) {
        ex = m;
        m = 0.0f;
      } else {
        ex = 0.0f;
      }
      ph = fill_level<M, C>(m, rho);
      break;
    default:
      break;
  }
  int cont = 0;
  const bool cons = p.fs_cons != 0;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
#pragma unroll
    for (int dx = -1; dx <= 1; dx++) {
      if (!dx && !dy) continue;
      const uint8_t v = p.count_pre ? s2[ly + dy][lx + dx] : s3[ly + dy][lx + dx];
      if (cons) {
        const uint8_t ev = v & kFGI;
        cont += (ev == kFluid || ev == kInterface) && !(v & (kWall | kMovingWall | kInlet));
      } else {
        const uint8_t ev = v & (kIF | kGasInterface);
        cont += ev == kFluid || ev == kInterface || ev == kIF || ev == kGasInterface;
      }
    }
  m += cont > 0 ? 0.0f : ex;
  ex = cont > 0 ? ex / (float)cont : 0.0f;
  Ms[idx] = m;
  static_cast<M*>(p.excess)[idx] = ex;
  if (!keep_phi) static_cast<M*>(p.phi)[idx] = ph;
}

// ---- reductions and codecs --------------------------------------------------

// Per-block FP64 partial sums of the total fluid mass (see flb_total_mass).
template <class S, class C, class M>
__global__ void __launch_bounds__(kBlock) k_mass_partial(const __grid_constant__ KParams p, uint32_t odd, int fs,
                                                         double* __restrict__ partial) {
  __shared__ double red[kBlock];
  const uint32_t tid = threadIdx.x;
  const uint32_t cell = blockIdx.x * kBlock + tid;
  double v = 0.0;
  if (cell < p.N) {
    const uint32_t x = cell % p.nx, y = cell / p.nx;
    uint32_t nb[9];
    neighbours(x, y, p.nx, p.ny, nb);
    const uint8_t* flags = p.flags;
    const uint8_t flag = flags[cell];
    if (fs) {
      const M* Ms = static_cast<const M*>(p.mass);
      const M* Ex = static_cast<const M*>(p.excess);
      int pullers = 0;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        const uint8_t nf = flags[nb[i]];
        if (p.fs_cons) {
          const uint8_t e = nf & kFGI;
          pullers += (e == kFluid || e == kInterface) && !(nf & (kWall | kMovingWall | kInlet));
        } else {
          pullers += !(nf & (kGas | kWall | kInlet));
        }
      }
      if (!(flag & (kWall | kMovingWall))) v += (double)Ms[cell];
      v += (double)Ex[cell] * (double)pullers;
    } else if (!(flag & (kGas | kWall))) {
      C f[9];
      load_incoming<S, C>(static_cast<const S*>(p.f), cell, nb, p.N, odd, p.f16_inv, f);
#pragma unroll
      for (int i = 0; i < 9; i++) v += (double)f[i];
    }
  }
  red[tid] = v;
  __syncthreads();
  for (uint32_t s = kBlock / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  if (tid == 0) partial[blockIdx.x] = red[0];
}

// Sums n partials in a fixed order with one block (deterministic).
__global__ void k_sum_partials(const double* __restrict__ partial, uint32_t n, double* __restrict__ out) {
  __shared__ double red[kBlock];
  double v = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += kBlock) v += partial[i];
  red[threadIdx.x] = v;
  __syncthreads();
  for (uint32_t s = kBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Census of cell types and non-finite populations: counts[0..4] = fluid,
// interface, gas, wall, non-finite.
template <class S, class C>
__global__ void __launch_bounds__(kBlock) k_census(const __grid_constant__ KParams p, uint32_t odd,
                                                   unsigned long long* __restrict__ counts) {
  const uint32_t cell = blockIdx.x * kBlock + threadIdx.x;
  uint32_t c[5] = {0, 0, 0, 0, 0};
  if (cell < p.N) {
    const uint8_t flag = p.flags[cell];
    const uint8_t e = flag & kFGI;
    if (flag & kWall) c[3] = 1;
    else if (e == kFluid) c[0] = 1;
    else if (e == kInterface) c[1] = 1;
    else if (e == kGas) c[2] = 1;
    if (!(flag & (kGas | kWall))) {
      const uint32_t x = cell % p.nx, y = cell / p.nx;
      uint32_t nb[9];
      neighbours(x, y, p.nx, p.ny, nb);
      C f[9];
      load_incoming<S, C>(static_cast<const S*>(p.f), cell, nb, p.N, odd, p.f16_inv, f);
      bool bad = false;
#pragma unroll
      for (int i = 0; i < 9; i++) bad |= !isfinite((double)f[i]);
      c[4] = bad;
    }
  }
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const uint32_t s = __reduce_add_sync(0xffffffffu, c[k]);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&counts[k], (unsigned long long)s);
  }
}

// Storage -> arithmetic type (read-back) and back (write).
template <class S, class C>
__global__ void k_decode(const S* __restrict__ F, C* __restrict__ out, uint32_t N, float inv) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= 9u * N) return;
  out[k] = Codec<S, C>::ld(F, k, (int)(k / N), inv);
}
template <class S, class C>
__global__ void k_encode(S* __restrict__ F, const C* __restrict__ in, uint32_t N, float scale) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= 9u * N) return;
  Codec<S, C>::st(F, k, (int)(k / N), in[k], scale);
}

}  // namespace flb
