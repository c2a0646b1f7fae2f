// sc_cell.cuh -- the stream-collide update of one cell (load, collide,
// store), shared by the single-case kernels (k_sc.cu) and the batched
// ensemble kernel (batch.cu).
#pragma once

#include <type_traits>

#include "common.cuh"

namespace flb {

// Everything between the load and the store of d_StreamCollide2D for one
// updated cell: density and velocity (or the inlet/outlet values), interface
// marking, Guo forcing, the optional velocity limiter, density/velocity
// write-back, equilibrium, Smagorinsky, SRT/TRT.  f: incoming -> post.
// FU: the fused SRT arithmetic (collide_fused) for cells that are neither inlet
// nor outlet; the host selects it only for SRT without the subgrid model.
// DEV: f holds FP16S deviations h = (f - w) * scale (single phase with FU).
// tnow: the time step (DEV only, for the stochastic rounding).  S: the
// storage type of the populations (a parked population is used as the
// value it would read back as from the population array).
template <class C, class M, bool FS, bool WM, bool FU, bool DEV = false, class S = C>
__device__ __forceinline__ void collide_cell(const KParams& p, uint32_t idx, uint32_t x, uint32_t y, uint8_t flag,
                                             uint32_t nbm, C* f, uint32_t tnow = 0u) {
  const uint32_t N = p.N;
  if constexpr (DEV) {
    if (flag & (kInlet | kOutlet)) {
      // inlet / outlet: the reference expressions on the decoded populations
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = fmac(f[i], p.f16_inv, wgt<C>(i));
      collide_cell<C, M, FS, WM, false, false>(p, idx, x, y, flag, nbm, f);
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = (f[i] - wgt<C>(i)) * p.f16_scale;
    } else {
      const DevOut o = collide_fused_dev(f, p.f16_inv, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx,
                                         p.fu_fy, p.u_max, p.fu_g, p.fu_h, p.fu_sw);
      if (WM) {
        static_cast<C*>(p.u)[idx] = o.ux;
        static_cast<C*>(p.u)[idx + N] = o.uy;
        static_cast<C*>(p.rho)[idx] = o.rho;
      }
    }
    const uint32_t base = f16_rs_base(idx & ~1u, tnow);
#pragma unroll
    for (int i = 0; i < 9; i++) f[i] = f16_rs_one(f[i], idx, f16_rs_bits(base, i));
    return;
  }
  if constexpr (FS) {
    // reference mode: FS_1 left the populations it rebuilt toward gas here.
    // FS_1 wrote them to their regular slots; where a half-way wall reflects
    // the population instead (its source is a wall), that slot is not read.
    // Each is taken at the value its slot would hold (rounded to the
    // storage), as if FS_1 had stored it and this step had loaded it.
    if (!p.fs_cons && (flag & (kFGI | kInlet)) == kInterface) {
      uint32_t wallsrc = 0;  // bit k: the source of incoming population k+1 is a wall
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        wallsrc |= ((nbm >> i) & 1u) << (i - 1);        // f_i comes from neighbour i+1
        wallsrc |= ((nbm >> (i - 1)) & 1u) << i;        // f_{i+1} comes from neighbour i
      }
      const uint32_t m = p.recon_mask[idx] & ~wallsrc;
      if (m) {
        const C* rec = static_cast<const C*>(p.recon);
#pragma unroll
        for (int k = 0; k < 8; k++)
          if ((m >> k) & 1u) f[k + 1] = stored_value<S, C>(rec[(uint32_t)k * N + idx], k + 1, p.f16_scale, p.f16_inv);
      }
    }
  }
  C rho, ux, uy, inv = C(0);
  const uint8_t io = flag & (kInlet | kOutlet);
  if (FU && !io) {
    C jx, jy;
    moments_fused(f, rho, jx, jy, inv);
    ux = jx * inv;
    uy = jy * inv;
  } else if (io & kInlet) {
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
      uint32_t nb[9];
      neighbours(x, y, p.nx, p.ny, nb);
      const M m = static_cast<const M*>(p.mass)[idx];
      bool notFluid = true, notGas = true;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        const uint8_t e = p.flags[nb[i]] & kFGI;
        notFluid = notFluid && (e != kFluid);
        notGas = notGas && (e != kGas);
      }
      // neighbours read these bytes concurrently; IF/IG compare unequal to
      // FLUID and GAS either way, so the outcome does not depend on timing
      if ((m > 1.001f * rho) || notGas) p.flags[idx] = (uint8_t)((flag & ~kFGI) | kIF);
      else if ((m < -0.001f) || notFluid) p.flags[idx] = (uint8_t)((flag & ~kFGI) | kIG);
    }
  }
  if (FU && !io) {
    ux = fmac((C)p.fu_hfx, inv, ux);
    uy = fmac((C)p.fu_hfy, inv, uy);
    limit_u(p.u_max, ux, uy);
    if (FS || WM) {
      static_cast<C*>(p.u)[idx] = ux;
      static_cast<C*>(p.u)[idx + N] = uy;
      static_cast<C*>(p.rho)[idx] = rho;
    }
    collide_fused(f, rho, ux, uy, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_fx, p.fu_fy, p.fu_g, p.fu_h);
    return;
  }
  C Fi[9];
  const bool use_force = p.use_force != 0;
  if (use_force) {
    const C rhol2 = 0.5f / rho;
    ux = ux + rhol2 * p.fx;
    uy = uy + rhol2 * p.fy;
  }
  limit_u(p.u_max, ux, uy);
  if (use_force) forcing(Fi, ux, uy, p.fx, p.fy, p.cF);
  if (FS || WM) {
    C* R = static_cast<C*>(p.rho);
    C* U = static_cast<C*>(p.u);
    if (!io || (flag & kOutlet)) {
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
}

// ---- one cell per thread -----------------------------------------------------
// FP16S single phase with the fused arithmetic works in deviation units
template <class S, bool FS, bool FU>
constexpr bool kDev = FU && !FS && std::is_same<S, __half>::value;

template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__device__ __forceinline__ void sc_cell(const KParams& p, uint32_t x, uint32_t y) {
  constexpr bool DEV = kDev<S, FS, FU>;
  using K = typename std::conditional<DEV, RawHalf, Codec<S, C>>::type;
  const uint32_t idx = x + y * p.nx;
  uint32_t nb[9];
  neighbours(x, y, p.nx, p.ny, nb);
  C f[9];
  uint8_t flag;
  uint32_t nbm = 0;
  if constexpr (!FS) {
    // single phase: nearly every cell is updated, so load with the flag
    flag = p.flags[idx];
    if (HW) nbm = p.nbmask[idx];
    load_in<S, C, HW, ODD, K>(p, idx, nb, nbm, f);
    if (flag & (kGas | kWall)) return;
  } else {
    // the wall mask and the populations are loaded with the flag (one round
    // trip, not two): the populations as if no neighbour were a wall, and a
    // cell next to a wall then reloads the ones a wall reflects
    flag = p.flags[idx];
    if (HW) nbm = p.nbmask[idx];
    load_in<S, C, false, ODD, K>(p, idx, nb, 0u, f);
    if (flag & (kGas | kWall)) return;
    if (HW && nbm) reload_reflected<S, C, ODD, K>(p, idx, nb, nbm, f);
  }
  collide_cell<C, M, FS, WM, FU, DEV, S>(p, idx, x, y, flag, nbm, f, DEV ? p.tstep[ODD] : 0u);
  store_post<S, C, ODD, K>(p, idx, nb, f);
}

}  // namespace flb
