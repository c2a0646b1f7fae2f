// sc_vec.cuh -- vectorised stream-collide: V consecutive cells per thread.
//
// Same arithmetic as k_stream_collide (lattice.cuh), different data movement.
// A warp owns 32*V consecutive cells of one row.  Every population slot is
// moved with one aligned V-wide access per thread (16 bytes for FP32 and FP64,
// 8 bytes for FP16S):
//   * own-cell slots and the (x, y+1) neighbour slot are aligned as they are;
//   * the three slots that live at the x+1 neighbour ((x+1,y), (x+1,y+1),
//     (x+1,y-1)) are loaded aligned at x0 and shifted by one cell with a warp
//     shuffle; the cell past the warp (or the row's periodic wrap) is a scalar;
//   * their stores go the other way: an aligned store at x0 whose first
//     element comes from the previous lane, lane 0 writing its first V-1
//     elements as scalars and the warp's last lane writing the element past
//     the warp as a scalar.
// Only elements of updated cells are written: skipped (wall/gas) cells own
// slots that half-way redirects of their neighbours write, so a vector whose
// elements are not all from updated cells is stored element by element.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

#include "kernels.cuh"

namespace flb {

template <class S, int V>
struct VecT;
template <>
struct VecT<float, 4> { using T = float4; };
template <>
struct VecT<double, 2> { using T = double2; };
template <>
struct VecT<__half, 4> { using T = uint2; };

template <class S>
struct Lanes;  // the native vector width per storage type
template <>
struct Lanes<float> { static constexpr int V = 4; };
template <>
struct Lanes<double> { static constexpr int V = 2; };
template <>
struct Lanes<__half> { static constexpr int V = 4; };

template <class S, int V>
__device__ __forceinline__ void vload(const S* p, S (&r)[V]) {
  using T = typename VecT<S, V>::T;
  const T v = *reinterpret_cast<const T*>(p);
  memcpy(r, &v, sizeof(T));
}
template <class S, int V>
__device__ __forceinline__ void vstore(S* p, const S (&r)[V]) {
  using T = typename VecT<S, V>::T;
  T v;
  memcpy(&v, r, sizeof(T));
  *reinterpret_cast<T*>(p) = v;
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

// Stores vals to dst[0..V) where valid; one vector store when all are valid.
template <class S, int V>
__device__ __forceinline__ void store_masked(S* dst, const S (&vals)[V], const bool (&valid)[V]) {
  bool all = true;
#pragma unroll
  for (int e = 0; e < V; e++) all &= valid[e];
  if (all) {
    vstore<S, V>(dst, vals);
  } else {
#pragma unroll
    for (int e = 0; e < V; e++)
      if (valid[e]) dst[e] = vals[e];
  }
}

template <int V>
__device__ __forceinline__ void load_flags(const uint8_t* p, uint8_t (&f)[V]) {
  if constexpr (V == 4) {
    const uchar4 v = *reinterpret_cast<const uchar4*>(p);
    f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
  } else {
    const uchar2 v = *reinterpret_cast<const uchar2*>(p);
    f[0] = v.x; f[1] = v.y;
  }
}

constexpr int kVecBlock = 256;

template <class S, class C, class M, bool FS, bool HW, bool WM>
__global__ void __launch_bounds__(kVecBlock, 2) k_sc_vec(const __grid_constant__ KParams p, uint32_t odd) {
  constexpr int V = Lanes<S>::V;
  using K = Codec<S, C>;
  const uint32_t nx = p.nx, ny = p.ny, N = p.N;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t x0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
  const uint32_t y = blockIdx.y;
  const bool inrow = x0 < nx;
  const uint32_t row = y * nx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * nx;
  uint8_t* flags = p.flags;
  uint8_t fl[V];
  bool act[V];
  bool any = false;
  if (inrow) load_flags<V>(flags + row + x0, fl);
#pragma unroll
  for (int k = 0; k < V; k++) {
    act[k] = inrow && !(fl[k] & (kGas | kWall));
    any |= act[k];
  }
  // a warp with no cell to update leaves memory untouched
  if (!__any_sync(0xffffffffu, any)) return;

  S* F = static_cast<S*>(p.f);
  const bool tail = (lane == 31u) || (x0 + V >= nx);  // the next cell is not the next lane's
  const uint32_t xn = (x0 + V >= nx) ? 0u : x0 + V;   // position past this lane (row wrap)

  // the previous lane's last cell reads this lane's first x+1 slot
  const bool prev_last = __shfl_up_sync(0xffffffffu, (int)act[V - 1], 1) != 0 && lane != 0u;
  const bool mine = inrow && any;

  // ---- loads ---------------------------------------------------------------
  S raw0[V], own[4][V], nbr[4][V];
  if (mine) vload<S, V>(F + row + x0, raw0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    if (mine) vload<S, V>(F + N * a + row + x0, own[q]);
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    S tmp[V];
    if (mine) vload<S, V>(F + N * b + r + x0, tmp);
    if (i == 3) {
#pragma unroll
      for (int k = 0; k < V; k++) nbr[q][k] = tmp[k];
    } else {
      if (!mine && inrow && prev_last) tmp[0] = F[N * b + r + x0];
      const S from_next = shfl_dn(tmp[0]);
#pragma unroll
      for (int k = 0; k < V - 1; k++) nbr[q][k] = tmp[k + 1];
      nbr[q][V - 1] = (tail && act[V - 1]) ? F[N * b + r + xn] : from_next;
    }
  }

  // ---- per-cell collision ----------------------------------------------------
  S out0[V], outa[4][V], outb[4][V];  // outa: own slot a; outb: neighbour slot b
  uint8_t nbmv[V];
#pragma unroll
  for (int k = 0; k < V; k++) nbmv[k] = 0;
  if (HW && inrow) load_flags<V>(p.nbmask + row + x0, nbmv);
#pragma unroll
  for (int k = 0; k < V; k++) {
    out0[k] = raw0[k];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      outa[q][k] = own[q][k];
      outb[q][k] = nbr[q][k];
    }
    if (!act[k]) continue;
    const uint32_t x = x0 + k;
    const uint32_t idx = row + x;
    const uint8_t flag = fl[k];
    C f[9];
    f[0] = K::ld(raw0, k, 0, p.f16_inv);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      f[i] = K::ld(own[q], k, i, p.f16_inv);
      f[i + 1] = K::ld(nbr[q], k, i + 1, p.f16_inv);
    }
    if constexpr (FS) {
      if (!p.fs_cons && (flag & (kFGI | kInlet)) == kInterface) {
        const uint32_t m = p.recon_mask[idx];
        if (m) {
          const C* rec = static_cast<const C*>(p.recon);
#pragma unroll
          for (int j = 0; j < 8; j++)
            if ((m >> j) & 1u) f[j + 1] = rec[(uint32_t)j * N + idx];
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
        uint32_t nb[9];
        neighbours(x, y, nx, ny, nb);
        const M m = static_cast<const M*>(p.mass)[idx];
        bool notFluid = true, notGas = true;
#pragma unroll
        for (int i = 1; i < 9; i++) {
          const uint8_t e = flags[nb[i]] & kFGI;
          notFluid = notFluid && (e != kFluid);
          notGas = notGas && (e != kGas);
        }
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
        if (!use_force) {
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
    K::st(out0, k, 0, f[0], p.f16_scale);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      K::st(outb[q], k, i, f[i], p.f16_scale);          // post f_i -> neighbour slot b
      K::st(outa[q], k, i + 1, f[i + 1], p.f16_scale);  // post f_{i+1} -> own slot a
    }
    if (HW) {
      // half-way redirect, scalar: f_i toward a wall also to the wall's slot a,
      // f_{i+1} toward a wall also to the own slot b
      const uint32_t nbm = nbmv[k];
      if (nbm) {
        uint32_t nb[9];
        neighbours(x, y, nx, ny, nb);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int i = 2 * q + 1;
          const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
          if ((nbm >> (i - 1)) & 1u) F[nb[i] + N * a] = outb[q][k];
          if ((nbm >> i) & 1u) F[idx + N * b] = outa[q][k];
        }
      }
    }
  }

  // ---- stores ----------------------------------------------------------------
  // shifted stores: element e of the vector at x0 comes from cell x0+e-1
  bool sh_valid[V];
  sh_valid[0] = prev_last;
#pragma unroll
  for (int e = 1; e < V; e++) sh_valid[e] = act[e - 1];
  if (inrow) store_masked<S, V>(F + row + x0, out0, act);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const uint32_t a = odd ? i : i + 1, b = odd ? i + 1 : i;
    if (inrow) store_masked<S, V>(F + N * a + row + x0, outa[q], act);
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    S* dst = F + N * b + r;
    if (i == 3) {
      if (inrow) store_masked<S, V>(dst + x0, outb[q], act);
    } else {
      const S from_prev = shfl_up1(outb[q][V - 1]);
      if (inrow) {
        S v[V];
        v[0] = from_prev;
#pragma unroll
        for (int k = 1; k < V; k++) v[k] = outb[q][k - 1];
        store_masked<S, V>(dst + x0, v, sh_valid);
        if (tail && act[V - 1]) dst[xn] = outb[q][V - 1];
      }
    }
  }
}

}  // namespace flb
