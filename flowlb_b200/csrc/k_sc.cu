// k_sc.cu -- stream-collide: d_StreamCollide2D, lbmKernel2D.cu:306-519.
//
// Two data paths with the same per-cell arithmetic (collide_cell):
//  * k_sc_scalar: one cell per thread;
//  * k_sc_vec: V consecutive cells of a row per thread (V = 4 for FP32 and
//    FP16S, 2 for FP64), every population slot moved with one aligned V-wide
//    access (16 bytes for FP32/FP64, 8 for FP16S).  Own-cell slots and the
//    (x, y+1) slot are aligned as they are; the three slots at the x+1
//    neighbour ((x+1,y), (x+1,y+1), (x+1,y-1)) are loaded aligned at x0 and
//    shifted one cell with a warp shuffle (the cell past the warp, or the
//    row's periodic wrap, is a scalar), and stored the other way: an aligned
//    store at x0 whose first element comes from the previous lane, lane 0
//    writing its first V-1 elements as scalars and the warp's last lane the
//    element past the warp.  A cell that is not updated (wall, gas) writes
//    back the raw values it loaded: no other thread writes a slot that
//    cell owns during this pass.
// Both are templated on the step parity (slot indices become constants) and,
// for the single-phase build, issue the population loads together with the
// flag load instead of after it.
#include <type_traits>

#include "launch.h"

// occupancy targets (resident blocks per SM) of the two data paths
// (measured on a B200, 8192x2048 single phase: one cell per thread is fastest
// at full occupancy, 8 blocks of 256 threads, even with a few spilled values)
#ifndef FLB_SC_MIN_BLOCKS
#define FLB_SC_MIN_BLOCKS 8
#endif
#ifndef FLB_VEC_MIN_BLOCKS
#define FLB_VEC_MIN_BLOCKS 3
#endif
#ifndef FLB_F16_V
#define FLB_F16_V 4  // FP16S cells per thread of the vector path (4 or 2)
#endif
#ifndef FLB_VEC_MIN_BLOCKS_FUSED
#define FLB_VEC_MIN_BLOCKS_FUSED 4
#endif
#ifndef FLB_F16_MIN_BLOCKS
#define FLB_F16_MIN_BLOCKS 4
#endif

namespace flb {

// Everything between the load and the store of d_StreamCollide2D for one
// updated cell: density and velocity (or the inlet/outlet values), interface
// marking, Guo forcing, the optional velocity limiter, density/velocity
// write-back, equilibrium, Smagorinsky, SRT/TRT.  f: incoming -> post.
// FU: the fused SRT arithmetic (collide_fused) for cells that are neither inlet
// nor outlet; the host selects it only for SRT without the subgrid model.
// DEV: f holds FP16S deviations h = (f - w) * scale (single phase with FU).
template <class C, class M, bool FS, bool WM, bool FU, bool DEV = false>
__device__ __forceinline__ void collide_cell(const KParams& p, uint32_t idx, uint32_t x, uint32_t y, uint8_t flag,
                                             uint32_t nbm, C* f) {
  const uint32_t N = p.N;
  if constexpr (DEV) {
    if (flag & (kInlet | kOutlet)) {
      // inlet / outlet: the reference expressions on the decoded populations
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = fmac(f[i], p.f16_inv, wgt<C>(i));
      collide_cell<C, M, FS, WM, false, false>(p, idx, x, y, flag, nbm, f);
#pragma unroll
      for (int i = 0; i < 9; i++) f[i] = (f[i] - wgt<C>(i)) * p.f16_scale;
      return;
    }
    const DevOut o = collide_fused_dev(f, p.f16_inv, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx,
                                       p.fu_fy, p.u_max, p.fu_g, p.fu_h, p.fu_sw);
    if (WM) {
      static_cast<C*>(p.u)[idx] = o.ux;
      static_cast<C*>(p.u)[idx + N] = o.uy;
      static_cast<C*>(p.rho)[idx] = o.rho;
    }
    return;
  }
  if constexpr (FS) {
    // reference mode: FS_1 left the populations it rebuilt toward gas here.
    // FS_1 wrote them to their regular slots; where a half-way wall reflects
    // the population instead (its source is a wall), that slot is not read.
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
          if ((m >> k) & 1u) f[k + 1] = rec[(uint32_t)k * N + idx];
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
    flag = p.flags[idx];
    if (flag & (kGas | kWall)) return;
    if (HW) nbm = p.nbmask[idx];
    load_in<S, C, HW, ODD, K>(p, idx, nb, nbm, f);
  }
  collide_cell<C, M, FS, WM, FU, DEV>(p, idx, x, y, flag, nbm, f);
  store_post<S, C, ODD, K>(p, idx, nb, f);
}

template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__global__ void __launch_bounds__(kBlock, FLB_SC_MIN_BLOCKS) k_sc_scalar(const __grid_constant__ KParams p) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  sc_cell<S, C, M, FS, HW, WM, ODD, FU>(p, x, y);
}

// Free surface: the listed super-tiles, one row of a super-tile per warp.
template <class S, class C, class M, bool HW, bool ODD, bool FU>
__global__ void __launch_bounds__(kBlock, FLB_SC_MIN_BLOCKS) k_sc_list(const __grid_constant__ KParams p,
                                                                       const TileList tl) {
  const uint32_t n = tile_count(tl);
  const uint32_t lane = threadIdx.x & 31u, row = threadIdx.x >> 5;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t t = tile_at(tl, i);
    const uint32_t y = (t / tl.nsx) * kSTH + row;
    if (y >= p.ny) continue;
    const uint32_t xb = (t % tl.nsx) * kSTW + lane;
#pragma unroll 1
    for (uint32_t j = 0; j < kSTW; j += 32)
      if (xb + j < p.nx) sc_cell<S, C, M, true, HW, true, ODD, FU>(p, xb + j, y);
  }
}

// ---- V cells per thread ----------------------------------------------------------
template <class S, int V>
struct VecT;
template <>
struct VecT<float, 4> { using T = float4; };
template <>
struct VecT<double, 2> { using T = double2; };
template <>
struct VecT<__half, 4> { using T = uint2; };
template <>
struct VecT<__half, 2> { using T = unsigned int; };

template <class S>
struct Lanes;
template <>
struct Lanes<float> { static constexpr int V = 4; };
template <>
struct Lanes<double> { static constexpr int V = 2; };
template <>
struct Lanes<__half> { static constexpr int V = FLB_F16_V; };

template <class S, int V>
__device__ __forceinline__ void vload(const S* ptr, S (&r)[V]) {
  using T = typename VecT<S, V>::T;
  const T v = *reinterpret_cast<const T*>(ptr);
  memcpy(r, &v, sizeof(T));
}
template <class S, int V>
__device__ __forceinline__ void vstore(S* ptr, const S (&r)[V]) {
  using T = typename VecT<S, V>::T;
  T v;
  memcpy(&v, r, sizeof(T));
  *reinterpret_cast<T*>(ptr) = v;
}

__device__ __forceinline__ float shfl_dn(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_dn(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ __half shfl_dn(__half v) {
  return __ushort_as_half((unsigned short)__shfl_down_sync(0xffffffffu, (int)__half_as_ushort(v), 1));
}
__device__ __forceinline__ float shfl_up1(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_up1(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ __half shfl_up1(__half v) {
  return __ushort_as_half((unsigned short)__shfl_up_sync(0xffffffffu, (int)__half_as_ushort(v), 1));
}

template <int V>
__device__ __forceinline__ void load_bytes(const uint8_t* ptr, uint8_t (&f)[V]) {
  if constexpr (V == 4) {
    const uchar4 v = *reinterpret_cast<const uchar4*>(ptr);
    f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
  } else {
    const uchar2 v = *reinterpret_cast<const uchar2*>(ptr);
    f[0] = v.x; f[1] = v.y;
  }
}

constexpr int kVecBlock = 256;

template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__global__ void __launch_bounds__(kVecBlock, FU ? (std::is_same<S, __half>::value ? FLB_F16_MIN_BLOCKS
                                                                                     : FLB_VEC_MIN_BLOCKS_FUSED)
                                                    : FLB_VEC_MIN_BLOCKS)
    k_sc_vec(const __grid_constant__ KParams p) {
  constexpr int V = Lanes<S>::V;
  constexpr bool DEV = kDev<S, FS, FU>;
  using K = typename std::conditional<DEV, RawHalf, Codec<S, C>>::type;
  const uint32_t nx = p.nx, ny = p.ny;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t x0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  const uint32_t y = blockIdx.y;
  const bool inrow = x0 < nx;
  const uint32_t row = y * nx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * nx;
  const bool tail = (lane == 31u) || (x0 + V >= nx);  // the cell past this lane is not the next lane's
  const uint32_t xn = (x0 + V >= nx) ? 0u : x0 + V;   // position past this lane (periodic wrap)

  uint8_t fl[V];
  bool act[V];
  bool any = false;
  S raw0[V], own[4][V], nbr[4][V], tmp[4][V];
  if (inrow) load_bytes<V>(p.flags + row + x0, fl);
  if constexpr (!FS) {
    // single phase: load the populations with the flags
    if (inrow) {
      vload<S, V>(slotp<S>(p, 0) + row + x0, raw0);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
        vload<S, V>(slotp<S>(p, slot_a<ODD>(i)) + row + x0, own[q]);
        vload<S, V>(slotp<S>(p, slot_b<ODD>(i)) + r + x0, tmp[q]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < V; k++) {
    act[k] = inrow && !(fl[k] & (kGas | kWall));
    any |= act[k];
  }
  // a warp with no cell to update leaves memory untouched
  if (!__any_sync(0xffffffffu, any)) return;
  if constexpr (FS) {
    if (inrow) {
      vload<S, V>(slotp<S>(p, 0) + row + x0, raw0);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
        vload<S, V>(slotp<S>(p, slot_a<ODD>(i)) + row + x0, own[q]);
        vload<S, V>(slotp<S>(p, slot_b<ODD>(i)) + r + x0, tmp[q]);
      }
    }
  }
  // realign the x+1 slots
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (i == 3) {
#pragma unroll
      for (int k = 0; k < V; k++) nbr[q][k] = tmp[q][k];
    } else {
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      const S from_next = shfl_dn(tmp[q][0]);
#pragma unroll
      for (int k = 0; k < V - 1; k++) nbr[q][k] = tmp[q][k + 1];
      nbr[q][V - 1] = (tail && inrow) ? slotp<S>(p, slot_b<ODD>(i))[r + xn] : from_next;
    }
  }
  uint8_t nbmv[V];
#pragma unroll
  for (int k = 0; k < V; k++) nbmv[k] = 0;
  if (HW && inrow) load_bytes<V>(p.nbmask + row + x0, nbmv);

  // ---- per-cell collision; cells not updated keep their raw values ---------
#pragma unroll
  for (int k = 0; k < V; k++) {
    if (!act[k]) continue;
    const uint32_t x = x0 + k;
    const uint32_t idx = row + x;
    C f[9];
    f[0] = K::ld(raw0, k, 0, p.f16_inv);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      f[i] = K::ld(own[q], k, i, p.f16_inv);
      f[i + 1] = K::ld(nbr[q], k, i + 1, p.f16_inv);
    }
    const uint32_t nbm = nbmv[k];
    if (HW && nbm) {
      // half-way walls: reflected populations, scalar (wall-adjacent cells only)
      uint32_t nb[9];
      neighbours(x, y, nx, ny, nb);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        if ((nbm >> i) & 1u) f[i] = K::ld(slotp<S>(p, slot_b<ODD>(i)), idx, i, p.f16_inv);
        if ((nbm >> (i - 1)) & 1u) f[i + 1] = K::ld(slotp<S>(p, slot_a<ODD>(i)), nb[i], i + 1, p.f16_inv);
      }
    }
    collide_cell<C, M, FS, WM, FU, DEV>(p, idx, x, y, fl[k], nbm, f);
    K::st(raw0, k, 0, f[0], p.f16_scale);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      K::st(nbr[q], k, i, f[i], p.f16_scale);      // post f_i -> neighbour slot b
      K::st(own[q], k, i + 1, f[i + 1], p.f16_scale);  // post f_{i+1} -> own slot a
    }
  }

  // ---- stores ------------------------------------------------------------------
  if (inrow) vstore<S, V>(slotp<S>(p, 0) + row + x0, raw0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (inrow) vstore<S, V>(slotp<S>(p, slot_a<ODD>(i)) + row + x0, own[q]);
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    S* dst = slotp<S>(p, slot_b<ODD>(i)) + r;
    if (i == 3) {
      if (inrow) vstore<S, V>(dst + x0, nbr[q]);
    } else {
      const S from_prev = shfl_up1(nbr[q][V - 1]);
      if (inrow) {
        if (lane != 0u) {
          S v[V];
          v[0] = from_prev;
#pragma unroll
          for (int k = 1; k < V; k++) v[k] = nbr[q][k - 1];
          vstore<S, V>(dst + x0, v);
        } else {
#pragma unroll
          for (int k = 0; k < V - 1; k++) dst[x0 + 1 + k] = nbr[q][k];
        }
        if (tail) dst[xn] = nbr[q][V - 1];
      }
    }
  }
}

// ---- FP16S single phase, fused deviation arithmetic, binary16 pairs --------
// The vector data path of k_sc_vec (4 cells per thread, one 8-byte access per
// population slot) specialised for FP16S storage with collide_fused_dev: the
// four halves of a slot stay packed in two 32-bit words, two cells are
// converted per instruction pair (__half22float2) and packed back with one
// conversion per two values, and the one-cell shift of the x+1 slots is a byte
// permutation of the packed words.  Cells that are not updated (wall, gas)
// keep their loaded halves through a per-half mask.  Used when the case has
// no inlet or outlet cells (those need the reference expressions).
__device__ __forceinline__ float2 h2f(uint32_t w) {
  __half2 h;
  memcpy(&h, &w, 4);
  return __half22float2(h);
}
__device__ __forceinline__ uint32_t f2h(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  uint32_t w;
  memcpy(&w, &h, 4);
  return w;
}
// words (a, b) = halves [a0 a1 b0 b1] -> [a1 b0]
__device__ __forceinline__ uint32_t mid(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x5432); }
__device__ __forceinline__ uint2 ldw(const __half* base, uint32_t at) {
  return *reinterpret_cast<const uint2*>(base + at);
}
__device__ __forceinline__ void stw(__half* base, uint32_t at, uint2 v) { *reinterpret_cast<uint2*>(base + at) = v; }

template <bool HW, bool WM, bool ODD>
__global__ void __launch_bounds__(kVecBlock, FLB_F16_MIN_BLOCKS) k_sc_h16(const __grid_constant__ KParams p) {
  const uint32_t nx = p.nx, ny = p.ny;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t x0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4u;
  const uint32_t y = blockIdx.y;
  const bool inrow = x0 < nx;
  const uint32_t row = y * nx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * nx;
  const bool tail = (lane == 31u) || (x0 + 4u >= nx);
  const uint32_t xn = (x0 + 4u >= nx) ? 0u : x0 + 4u;

  uint32_t fl = 0, nbw = 0;
  uint2 w0 = make_uint2(0u, 0u), own[4], tmp[4], nbr[4];
#pragma unroll
  for (int q = 0; q < 4; q++) own[q] = tmp[q] = make_uint2(0u, 0u);
  if (inrow) {
    fl = *reinterpret_cast<const uint32_t*>(p.flags + row + x0);
    w0 = ldw(slotp<__half>(p, 0), row + x0);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      own[q] = ldw(slotp<__half>(p, slot_a<ODD>(i)), row + x0);
      tmp[q] = ldw(slotp<__half>(p, slot_b<ODD>(i)), r + x0);
    }
    if (HW) nbw = *reinterpret_cast<const uint32_t*>(p.nbmask + row + x0);
  }
  bool act[4];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    act[k] = inrow && !((fl >> (8 * k)) & (kGas | kWall));
    any |= act[k];
  }
  if (!__any_sync(0xffffffffu, any)) return;
  // realign the x+1 slots: element k of nbr is cell x0+k+1
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (i == 3) {
      nbr[q] = tmp[q];
    } else {
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      uint32_t nxt = __shfl_down_sync(0xffffffffu, tmp[q].x, 1);
      if (tail && inrow) nxt = (uint32_t)__half_as_ushort(slotp<__half>(p, slot_b<ODD>(i))[r + xn]);
      nbr[q].x = mid(tmp[q].x, tmp[q].y);
      nbr[q].y = mid(tmp[q].y, nxt);
    }
  }
  const float invS = p.f16_inv;
  // two cells (2P, 2P+1) per pass: the low and high halves of word P
#pragma unroll
  for (int P = 0; P < 2; P++) {
    float ha[9], hb[9];
    {
      const float2 v = h2f(P ? w0.y : w0.x);
      ha[0] = v.x;
      hb[0] = v.y;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const float2 vo = h2f(P ? own[q].y : own[q].x);
      const float2 vn = h2f(P ? nbr[q].y : nbr[q].x);
      ha[i] = vo.x;
      hb[i] = vo.y;
      ha[i + 1] = vn.x;
      hb[i + 1] = vn.y;
    }
    if (HW) {
      // half-way walls: reflected populations, scalar (wall-adjacent cells only)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int k = 2 * P + c;
        const uint32_t nbm = (nbw >> (8 * k)) & 0xffu;
        if (act[k] && nbm) {
          float* h = c ? hb : ha;
          const uint32_t x = x0 + k, idx = row + x;
          uint32_t nb[9];
          neighbours(x, y, nx, ny, nb);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int i = 2 * q + 1;
            if ((nbm >> i) & 1u) h[i] = RawHalf::ld(slotp<__half>(p, slot_b<ODD>(i)), idx, i, invS);
            if ((nbm >> (i - 1)) & 1u) h[i + 1] = RawHalf::ld(slotp<__half>(p, slot_a<ODD>(i)), nb[i], i + 1, invS);
          }
        }
      }
    }
    const DevOut oa = collide_fused_dev(ha, invS, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx, p.fu_fy,
                                        p.u_max, p.fu_g, p.fu_h, p.fu_sw);
    const DevOut ob = collide_fused_dev(hb, invS, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx, p.fu_fy,
                                        p.u_max, p.fu_g, p.fu_h, p.fu_sw);
    if (WM) {
      float* R = static_cast<float*>(p.rho);
      float* U = static_cast<float*>(p.u);
      const uint32_t idx = row + x0 + 2 * P;
      if (act[2 * P]) {
        R[idx] = oa.rho;
        U[idx] = oa.ux;
        U[idx + p.N] = oa.uy;
      }
      if (act[2 * P + 1]) {
        R[idx + 1] = ob.rho;
        U[idx + 1] = ob.ux;
        U[idx + 1 + p.N] = ob.uy;
      }
    }
    // computed halves where the cell is updated, loaded ones elsewhere
    const uint32_t m = (act[2 * P] ? 0x0000ffffu : 0u) | (act[2 * P + 1] ? 0xffff0000u : 0u);
    auto put = [m](uint32_t& w, uint32_t v) { w = (v & m) | (w & ~m); };
    if (P) put(w0.y, f2h(ha[0], hb[0]));
    else put(w0.x, f2h(ha[0], hb[0]));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      // post f_i -> neighbour slot b (nbr), post f_{i+1} -> own slot a (own)
      if (P) {
        put(nbr[q].y, f2h(ha[i], hb[i]));
        put(own[q].y, f2h(ha[i + 1], hb[i + 1]));
      } else {
        put(nbr[q].x, f2h(ha[i], hb[i]));
        put(own[q].x, f2h(ha[i + 1], hb[i + 1]));
      }
    }
  }

  // ---- stores ------------------------------------------------------------------
  if (inrow) stw(slotp<__half>(p, 0), row + x0, w0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (inrow) stw(slotp<__half>(p, slot_a<ODD>(i)), row + x0, own[q]);
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    __half* dst = slotp<__half>(p, slot_b<ODD>(i)) + r;
    if (i == 3) {
      if (inrow) stw(dst, x0, nbr[q]);
    } else {
      const uint32_t prev = __shfl_up_sync(0xffffffffu, nbr[q].y, 1);
      if (inrow) {
        if (lane != 0u) {
          stw(dst, x0, make_uint2(mid(prev, nbr[q].x), mid(nbr[q].x, nbr[q].y)));
        } else {
          // x0 belongs to the previous warp's last lane
          dst[x0 + 1] = __ushort_as_half((unsigned short)(nbr[q].x & 0xffffu));
          *reinterpret_cast<uint32_t*>(dst + x0 + 2) = mid(nbr[q].x, nbr[q].y);
        }
        if (tail) dst[xn] = __ushort_as_half((unsigned short)(nbr[q].y >> 16));
      }
    }
  }
}

// ---- launchers -------------------------------------------------------------------
template <class S, class C, class M, bool FS, bool HW, bool WM, bool FU>
static void launch_sc_t(const KParams& kp, cudaStream_t st, uint32_t odd, bool vec) {
  if constexpr (kDev<S, FS, FU>) {
    if (vec && !kp.has_io) {
      const uint32_t per_row = kp.nx / 4u;
      const uint32_t block = per_row >= (uint32_t)kVecBlock ? (uint32_t)kVecBlock : ((per_row + 31u) / 32u) * 32u;
      const dim3 g((per_row + block - 1) / block, kp.ny);
      if (odd) k_sc_h16<HW, WM, true><<<g, block, 0, st>>>(kp);
      else k_sc_h16<HW, WM, false><<<g, block, 0, st>>>(kp);
      return;
    }
  }
  if (vec) {
    constexpr int V = Lanes<S>::V;
    const uint32_t per_row = kp.nx / V;
    const uint32_t block = per_row >= (uint32_t)kVecBlock ? (uint32_t)kVecBlock : ((per_row + 31u) / 32u) * 32u;
    const dim3 g((per_row + block - 1) / block, kp.ny);
    if (odd) k_sc_vec<S, C, M, FS, HW, WM, true, FU><<<g, block, 0, st>>>(kp);
    else k_sc_vec<S, C, M, FS, HW, WM, false, FU><<<g, block, 0, st>>>(kp);
  } else {
    const dim3 g((kp.nx + kBlock - 1) / kBlock, kp.ny);
    if (odd) k_sc_scalar<S, C, M, FS, HW, WM, true, FU><<<g, kBlock, 0, st>>>(kp);
    else k_sc_scalar<S, C, M, FS, HW, WM, false, FU><<<g, kBlock, 0, st>>>(kp);
  }
}

template <class S, class C, class M, bool FU>
static void launch_sc_f(const KParams& kp, cudaStream_t st, uint32_t odd, bool fs, bool hw, bool wm, bool vec) {
  if (fs) {
    if (hw) launch_sc_t<S, C, M, true, true, true, FU>(kp, st, odd, vec);
    else launch_sc_t<S, C, M, true, false, true, FU>(kp, st, odd, vec);
  } else if (wm) {
    if (hw) launch_sc_t<S, C, M, false, true, true, FU>(kp, st, odd, vec);
    else launch_sc_t<S, C, M, false, false, true, FU>(kp, st, odd, vec);
  } else {
    if (hw) launch_sc_t<S, C, M, false, true, false, FU>(kp, st, odd, vec);
    else launch_sc_t<S, C, M, false, false, false, FU>(kp, st, odd, vec);
  }
}

template <class S, class C, class M>
void launch_sc(const KParams& kp, cudaStream_t st, uint32_t odd, bool fs, bool hw, bool wm, bool vec, bool fu) {
  if (fu) launch_sc_f<S, C, M, true>(kp, st, odd, fs, hw, wm, vec);
  else launch_sc_f<S, C, M, false>(kp, st, odd, fs, hw, wm, vec);
}

int vec_width(int precision) {
  return precision == 64 ? Lanes<double>::V : (precision == 16 ? Lanes<__half>::V : Lanes<float>::V);
}

template <class S, class C, class M, bool FU>
static void launch_sc_list_f(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl,
                             uint32_t grid) {
  if (hw) {
    if (odd) k_sc_list<S, C, M, true, true, FU><<<grid, kBlock, 0, st>>>(kp, tl);
    else k_sc_list<S, C, M, true, false, FU><<<grid, kBlock, 0, st>>>(kp, tl);
  } else {
    if (odd) k_sc_list<S, C, M, false, true, FU><<<grid, kBlock, 0, st>>>(kp, tl);
    else k_sc_list<S, C, M, false, false, FU><<<grid, kBlock, 0, st>>>(kp, tl);
  }
}

template <class S, class C, class M>
void launch_sc_list(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid,
                    bool fu) {
  if (fu) launch_sc_list_f<S, C, M, true>(kp, st, odd, hw, tl, grid);
  else launch_sc_list_f<S, C, M, false>(kp, st, odd, hw, tl, grid);
}

template <class S, class C, class M>
int sc_list_blocks_per_sm() {
  int n = 0, m = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sc_list<S, C, M, true, false, false>, kBlock, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_sc_list<S, C, M, true, false, true>, kBlock, 0);
  n = n < m ? n : m;
  return n > 0 ? n : 1;
}

#define FLB_INSTANTIATE(S, C, M)                                                                               \
  template void launch_sc<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, bool, bool, bool, bool);     \
  template void launch_sc_list<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, const TileList&, uint32_t,  \
                                        bool);                                                                  \
  template int sc_list_blocks_per_sm<S, C, M>();
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
