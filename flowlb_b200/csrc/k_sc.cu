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
#include "sc_cell.cuh"

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

template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__global__ void __launch_bounds__(kBlock, FLB_SC_MIN_BLOCKS) k_sc_scalar(const __grid_constant__ KParams p) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (kDev<S, FS, FU> && x == 0 && y == 0) p.tstep[!ODD] = p.tstep[ODD] + 1u;
  if (x >= p.nx) return;
  sc_cell<S, C, M, FS, HW, WM, ODD, FU>(p, x, y);
}

// Free surface: the listed super-tiles, one row of a super-tile per warp.
template <class S, class C, class M, bool HW, bool ODD, bool FU>
__global__ void __launch_bounds__(kListBlock, 2048 / kListBlock) k_sc_list(const __grid_constant__ KParams p,
                                                                           const TileList tl) {
  // the list was built two kernels back (FS_1 waited for it), so it is read
  // before waiting for FS_1, whose writes the cell updates need
  const uint32_t n = tile_count(tl);
  pdl_wait();
  pdl_trigger();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = warp % kSTH, chunk = warp / kSTH, cpr = (blockDim.x >> 5) / kSTH;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t t = tile_at(tl, i);
    const uint32_t y = (t / tl.nsx) * kSTH + row;
    if (y >= p.ny) continue;
    const uint32_t xb = (t % tl.nsx) * kSTW + lane;
#pragma unroll 1
    for (uint32_t j = chunk * 32u; j < kSTW; j += 32u * cpr)
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

// V consecutive cells x0 .. x0+V-1 of row y per thread (x0 a multiple of V;
// the 32 lanes of the warp take consecutive groups of one row, every lane of
// the warp must call it).  Used over whole rows (k_sc_vec) and over the rows
// of listed super-tiles (k_sc_list_vec).
template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__device__ __forceinline__ void sc_vec_cells(const KParams& p, uint32_t x0, uint32_t y, uint32_t lane) {
  constexpr int V = Lanes<S>::V;
  constexpr bool DEV = kDev<S, FS, FU>;
  using K = typename std::conditional<DEV, RawHalf, Codec<S, C>>::type;
  const uint32_t nx = p.nx, ny = p.ny;
  const bool inrow = x0 < nx;
  const uint32_t row = y * nx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * nx;
  const bool tail = (lane == 31u) || (x0 + V >= nx);  // the cell past this lane is not the next lane's
  const uint32_t xn = (x0 + V >= nx) ? 0u : x0 + V;   // position past this lane (periodic wrap)
  if (DEV && x0 == 0 && y == 0) p.tstep[!ODD] = p.tstep[ODD] + 1u;

  uint8_t fl[V];
  bool act[V];
  bool any = false;
  S raw0[V], own[4][V], nbr[4][V], tmp[4][V];
  bool plain = false;  // single phase: all V cells plain fluid, flag and mask bytes not read
  if constexpr (!FS && V == 4) plain = inrow && p.plain && plain_cells<1>(p.plain, row + x0);
  if (plain) {
#pragma unroll
    for (int k = 0; k < V; k++) fl[k] = kFluid;
  } else if (inrow) {
    load_bytes<V>(p.flags + row + x0, fl);
  }
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
  if (HW && inrow && !plain) load_bytes<V>(p.nbmask + row + x0, nbmv);

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
    collide_cell<C, M, FS, WM, FU, DEV, S>(p, idx, x, y, fl[k], nbm, f, DEV ? p.tstep[ODD] : 0u);
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

template <class S, class C, class M, bool FS, bool HW, bool WM, bool ODD, bool FU>
__global__ void __launch_bounds__(kVecBlock, FU ? (std::is_same<S, __half>::value ? FLB_F16_MIN_BLOCKS
                                                                                     : FLB_VEC_MIN_BLOCKS_FUSED)
                                                    : FLB_VEC_MIN_BLOCKS)
    k_sc_vec(const __grid_constant__ KParams p) {
  constexpr int V = Lanes<S>::V;
  sc_vec_cells<S, C, M, FS, HW, WM, ODD, FU>(p, (blockIdx.x * blockDim.x + threadIdx.x) * V, blockIdx.y,
                                             threadIdx.x & 31u);
}

// Free surface, vector data path: the listed super-tiles, each row of a
// super-tile taken by kSTW / (32 V) warps (one warp for FP32 and FP16S).
template <class S>
__host__ __device__ constexpr int list_vec_block() {
  return (int)kSTH * (int)(kSTW / (32u * (uint32_t)Lanes<S>::V)) * 32;
}
template <class S, class C, class M, bool HW, bool ODD, bool FU>
__global__ void __launch_bounds__(list_vec_block<S>(), 1024 / list_vec_block<S>())
    k_sc_list_vec(const __grid_constant__ KParams p, const TileList tl) {
  constexpr uint32_t V = (uint32_t)Lanes<S>::V, wpr = kSTW / (32u * V);
  // the list was built two kernels back (FS_1 waited for it), so it is read
  // before waiting for FS_1, whose writes the cell updates need
  const uint32_t n = tile_count(tl);
  pdl_wait();
  pdl_trigger();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = warp / wpr, chunk = warp % wpr;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t t = tile_at(tl, i);
    const uint32_t y = (t / tl.nsx) * kSTH + row;
    if (y >= p.ny) continue;  // warp-uniform
    const uint32_t x0 = (t % tl.nsx) * kSTW + (chunk * 32u + lane) * V;
    sc_vec_cells<S, C, M, true, HW, true, ODD, FU>(p, x0, y, lane);
  }
}

// ---- FP16S single phase, fused deviation arithmetic, binary16 pairs --------
// The vector data path of k_sc_vec specialised for FP16S storage with
// collide_fused_dev: 2W cells per thread, the 2W halves of a population slot
// moved with one 4W-byte access and kept packed in W 32-bit words; two cells
// are converted per instruction pair (__half22float2) and packed back with one
// conversion per two values, and the one-cell shift of the x+1 slots is a
// byte permutation of the packed words.  Cells that are not updated (wall,
// gas) keep their loaded halves through a per-half mask.  Used when the case
// has no inlet or outlet cells (those need the reference expressions).
#ifndef FLB_H16_WORDS
#define FLB_H16_WORDS 4  // 32-bit words (cell pairs) per thread and slot: 8 cells
#endif
// measured on a B200 (8192x2048): 128-thread blocks, 6 per SM (80 registers),
// 157 GLUPS; 256 x 3: 149; 64 x 12: 157; 512 x 1: 116; a persistent
// grid-stride loop over row chunks: 135; evict-first cache hints on the slot
// accesses: -9 %; the slots staged in shared memory by bulk async copies
// (cp.async.bulk, two stages, 2 blocks per SM): 135
#ifndef FLB_H16_BLOCK
#define FLB_H16_BLOCK 128
#endif
#ifndef FLB_H16_MIN_BLOCKS
#define FLB_H16_MIN_BLOCKS 6
#endif
__device__ __forceinline__ float2 h2f(uint32_t w) {
  __half2 h;
  memcpy(&h, &w, 4);
  return __half22float2(h);
}
// words (a, b) = halves [a0 a1 b0 b1] -> [a1 b0]
__device__ __forceinline__ uint32_t mid(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x5432); }

template <int W>
struct Words {
  uint32_t w[W];
};
template <int W>
__device__ __forceinline__ Words<W> ldw(const void* base, uint32_t at_bytes) {
  Words<W> r;
  const char* q = static_cast<const char*>(base) + at_bytes;
  if constexpr (W == 1) {
    r.w[0] = *reinterpret_cast<const uint32_t*>(q);
  } else if constexpr (W == 2) {
    const uint2 v = *reinterpret_cast<const uint2*>(q);
    r.w[0] = v.x; r.w[1] = v.y;
  } else {
    const uint4 v = *reinterpret_cast<const uint4*>(q);
    r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
  }
  return r;
}
template <int W>
__device__ __forceinline__ void stw(void* base, uint32_t at_bytes, const Words<W>& r) {
  char* q = static_cast<char*>(base) + at_bytes;
  if constexpr (W == 2) *reinterpret_cast<uint2*>(q) = make_uint2(r.w[0], r.w[1]);
  else *reinterpret_cast<uint4*>(q) = make_uint4(r.w[0], r.w[1], r.w[2], r.w[3]);
}

// V = 2W cells from (x0, y); every lane of the warp calls it with the same y.
// LIM: the velocity limiter is on.
template <bool HW, bool WM, bool ODD, bool LIM>
__device__ __forceinline__ void h16_cells(const KParams& p, const uint32_t x0, const uint32_t y) {
  constexpr int W = FLB_H16_WORDS, V = 2 * W;
  const uint32_t nx = p.nx, ny = p.ny;
  const uint32_t lane = threadIdx.x & 31u;
  const bool inrow = x0 < nx;
  const uint32_t row = y * nx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * nx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * nx;
  const bool tail = (lane == 31u) || (x0 + V >= nx);
  const uint32_t xn = (x0 + V >= nx) ? 0u : x0 + V;
  const uint32_t at = (row + x0) * 2u;  // byte offset of this thread's cells in a slot

  Words<W / 2> flw{}, nbmw{};  // V flag / neighbour-mask bytes
  Words<W> w0{}, own[4], tmp[4], nbr[4];
#pragma unroll
  for (int q = 0; q < 4; q++) own[q] = tmp[q] = Words<W>{};
  bool plain = false;  // all V cells plain fluid: flag and mask bytes not read
  if (inrow) {
    // the population loads first: the chunk-map word must not delay them
    w0 = ldw<W>(p.slot[0], at);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      own[q] = ldw<W>(p.slot[slot_a<ODD>(i)], at);
      tmp[q] = ldw<W>(p.slot[slot_b<ODD>(i)], (r + x0) * 2u);
    }
    plain = p.plain && plain_cells<V / 4>(p.plain, row + x0);
    if (plain) {
#pragma unroll
      for (int j = 0; j < W / 2; j++) flw.w[j] = 0x01010101u;
    } else {
      flw = ldw<W / 2>(p.flags, row + x0);
    }
    if (HW && !plain) nbmw = ldw<W / 2>(p.nbmask, row + x0);
  }
  // per-half masks of the updated cells (0xffff: not gas, not wall), pair P
  // in word P; a lane past the row end updates nothing
  uint32_t upd[W];
  bool any = false;
#pragma unroll
  for (int P = 0; P < W; P++) {
    const uint32_t two = __byte_perm(flw.w[P >> 1], 0u, (P & 1) ? 0x3322u : 0x1100u);  // bytes k, k, k+1, k+1
    upd[P] = inrow ? __vcmpeq4(two & 0x0a0a0a0au, 0u) : 0u;
    any |= upd[P] != 0u;
  }
  if (!__any_sync(0xffffffffu, any)) return;
  bool walls = false;  // some cell of this thread has a wall neighbour
  if (HW) {
#pragma unroll
    for (int j = 0; j < W / 2; j++) walls |= nbmw.w[j] != 0u;
  }
  // realign the x+1 slots: element k of nbr is cell x0+k+1
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (i == 3) {
      nbr[q] = tmp[q];
    } else {
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      uint32_t nxt = __shfl_down_sync(0xffffffffu, tmp[q].w[0], 1);
      if (tail && inrow) nxt = (uint32_t)__half_as_ushort(slotp<__half>(p, slot_b<ODD>(i))[r + xn]);
#pragma unroll
      for (int j = 0; j < W - 1; j++) nbr[q].w[j] = mid(tmp[q].w[j], tmp[q].w[j + 1]);
      nbr[q].w[W - 1] = mid(tmp[q].w[W - 1], nxt);
    }
  }
  const float invS = p.f16_inv;
  const uint32_t tnow = p.tstep[ODD];
  // two cells (2P, 2P+1) per pass: the low and high halves of word P
#pragma unroll
  for (int P = 0; P < W; P++) {
    float ha[9], hb[9];
    {
      const float2 v = h2f(w0.w[P]);
      ha[0] = v.x;
      hb[0] = v.y;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const float2 vo = h2f(own[q].w[P]);
      const float2 vn = h2f(nbr[q].w[P]);
      ha[i] = vo.x;
      hb[i] = vo.y;
      ha[i + 1] = vn.x;
      hb[i + 1] = vn.y;
    }
    if (HW && walls) {
      // half-way walls: reflected populations, scalar (wall-adjacent cells only)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int k = 2 * P + c;
        const uint32_t nbm = (nbmw.w[k >> 2] >> (8 * (k & 3))) & 0xffu;
        if (((upd[P] >> (16 * c)) & 1u) && nbm) {
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
    const DevOut oa = collide_fused_dev<LIM>(ha, invS, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx,
                                             p.fu_fy, p.u_max, p.fu_g, p.fu_h, p.fu_sw);
    const DevOut ob = collide_fused_dev<LIM>(hb, invS, p.inv_tau, p.fu_omc, p.fu_nk3, p.fu_hfx, p.fu_hfy, p.fu_fx,
                                             p.fu_fy, p.u_max, p.fu_g, p.fu_h, p.fu_sw);
    const uint32_t idx = row + x0 + 2 * P;
    if (WM) {
      float* R = static_cast<float*>(p.rho);
      float* U = static_cast<float*>(p.u);
      if (upd[P] & 1u) {
        R[idx] = oa.rho;
        U[idx] = oa.ux;
        U[idx + p.N] = oa.uy;
      }
      if (upd[P] >> 16) {
        R[idx + 1] = ob.rho;
        U[idx + 1] = ob.ux;
        U[idx + 1 + p.N] = ob.uy;
      }
    }
    // stochastic rounding of the pair (idx is even: row and x0 are)
    const uint32_t base = f16_rs_base(idx, tnow);
    // computed halves where the cell is updated, loaded ones elsewhere
    const uint32_t m = upd[P];
    auto put = [m](uint32_t& w, uint32_t v) { w = (v & m) | (w & ~m); };
    put(w0.w[P], f2h_rs(ha[0], hb[0], f16_rs_bits(base, 0)));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      put(nbr[q].w[P], f2h_rs(ha[i], hb[i], f16_rs_bits(base, i)));              // post f_i -> neighbour slot b
      put(own[q].w[P], f2h_rs(ha[i + 1], hb[i + 1], f16_rs_bits(base, i + 1)));  // post f_{i+1} -> own slot a
    }
  }

  // ---- stores ------------------------------------------------------------------
  if (inrow) stw<W>(p.slot[0], at, w0);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (inrow) stw<W>(p.slot[slot_a<ODD>(i)], at, own[q]);
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    __half* dst = slotp<__half>(p, slot_b<ODD>(i)) + r;
    if (i == 3) {
      if (inrow) stw<W>(dst, x0 * 2u, nbr[q]);
    } else {
      const uint32_t prev = __shfl_up_sync(0xffffffffu, nbr[q].w[W - 1], 1);
      if (inrow) {
        if (lane != 0u) {
          Words<W> o;
          o.w[0] = mid(prev, nbr[q].w[0]);
#pragma unroll
          for (int j = 1; j < W; j++) o.w[j] = mid(nbr[q].w[j - 1], nbr[q].w[j]);
          stw<W>(dst, x0 * 2u, o);
        } else {
          // x0 belongs to the previous warp's last lane
          dst[x0 + 1] = __ushort_as_half((unsigned short)(nbr[q].w[0] & 0xffffu));
#pragma unroll
          for (int j = 1; j < W; j++)
            *reinterpret_cast<uint32_t*>(dst + x0 + 2 * j) = mid(nbr[q].w[j - 1], nbr[q].w[j]);
        }
        if (tail) dst[xn] = __ushort_as_half((unsigned short)(nbr[q].w[W - 1] >> 16));
      }
    }
  }
}

// One row chunk of blockDim.x * V cells per block.
template <bool HW, bool WM, bool ODD, bool LIM>
__global__ void __launch_bounds__(FLB_H16_BLOCK, FLB_H16_MIN_BLOCKS) k_sc_h16(const __grid_constant__ KParams p) {
  constexpr uint32_t V = 2 * FLB_H16_WORDS;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) p.tstep[!ODD] = p.tstep[ODD] + 1u;
  h16_cells<HW, WM, ODD, LIM>(p, (blockIdx.x * blockDim.x + threadIdx.x) * V, blockIdx.y);
}

// ---- launchers -------------------------------------------------------------------
template <class S, class C, class M, bool FS, bool HW, bool WM, bool FU>
static void launch_sc_t(const KParams& kp, cudaStream_t st, uint32_t odd, bool vec) {
  if constexpr (kDev<S, FS, FU>) {
    constexpr uint32_t V = 2u * FLB_H16_WORDS;
    if (vec && !kp.has_io && kp.nx % V == 0) {
      const uint32_t per_row = kp.nx / V;
      const uint32_t bmax = FLB_H16_BLOCK;
      const uint32_t block = per_row >= bmax ? bmax : ((per_row + 31u) / 32u) * 32u;
      const dim3 g((per_row + block - 1) / block, kp.ny);
      const bool lim = kp.u_max > 0.0f;
      if (odd) {
        if (lim) k_sc_h16<HW, WM, true, true><<<g, block, 0, st>>>(kp);
        else k_sc_h16<HW, WM, true, false><<<g, block, 0, st>>>(kp);
      } else {
        if (lim) k_sc_h16<HW, WM, false, true><<<g, block, 0, st>>>(kp);
        else k_sc_h16<HW, WM, false, false><<<g, block, 0, st>>>(kp);
      }
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
                             uint32_t grid, bool vec) {
  if (vec) {
    constexpr int B = list_vec_block<S>();
    if (hw) {
      if (odd) launch_pdl(k_sc_list_vec<S, C, M, true, true, FU>, grid, B, st, kp, tl);
      else launch_pdl(k_sc_list_vec<S, C, M, true, false, FU>, grid, B, st, kp, tl);
    } else {
      if (odd) launch_pdl(k_sc_list_vec<S, C, M, false, true, FU>, grid, B, st, kp, tl);
      else launch_pdl(k_sc_list_vec<S, C, M, false, false, FU>, grid, B, st, kp, tl);
    }
    return;
  }
  if (hw) {
    if (odd) launch_pdl(k_sc_list<S, C, M, true, true, FU>, grid, kListBlock, st, kp, tl);
    else launch_pdl(k_sc_list<S, C, M, true, false, FU>, grid, kListBlock, st, kp, tl);
  } else {
    if (odd) launch_pdl(k_sc_list<S, C, M, false, true, FU>, grid, kListBlock, st, kp, tl);
    else launch_pdl(k_sc_list<S, C, M, false, false, FU>, grid, kListBlock, st, kp, tl);
  }
}

template <class S, class C, class M>
void launch_sc_list(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid,
                    bool fu, bool vec) {
  if (fu) launch_sc_list_f<S, C, M, true>(kp, st, odd, hw, tl, grid, vec);
  else launch_sc_list_f<S, C, M, false>(kp, st, odd, hw, tl, grid, vec);
}

template <class S, class C, class M>
int sc_list_blocks_per_sm(bool vec) {
  int n = 0, m = 0;
  if (vec) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sc_list_vec<S, C, M, true, false, false>,
                                                  list_vec_block<S>(), 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_sc_list_vec<S, C, M, true, false, true>,
                                                  list_vec_block<S>(), 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sc_list<S, C, M, true, false, false>, kListBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_sc_list<S, C, M, true, false, true>, kListBlock, 0);
  }
  n = n < m ? n : m;
  return n > 0 ? n : 1;
}

#define FLB_INSTANTIATE(S, C, M)                                                                               \
  template void launch_sc<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, bool, bool, bool, bool);     \
  template void launch_sc_list<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, const TileList&, uint32_t,  \
                                        bool, bool);                                                            \
  template int sc_list_blocks_per_sm<S, C, M>(bool);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
