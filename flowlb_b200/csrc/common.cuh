// common.cuh -- kernel parameters and population access shared by all passes.
//
// Layout in HBM (structure of arrays, the reference layout, one population
// buffer):
//   f      9N  S   slot s of cell c at f[c + s*N] (slot[s] below points at
//                  f + s*N); updated in place by the esoteric-pull pattern:
//                  a cell loads and stores the same 9 addresses, so no second
//                  buffer is needed
//   rho     N  C   density of the incoming populations of the last step
//   u      2N  C   force-shifted velocity, u_x then u_y
//   flags  2xN u8  cell types; two buffers, the flag-stencil pass reads one
//                  and writes the other
//   nbmask  N  u8  bit k-1 set when neighbour k is a wall (half-way walls)
//   mass, excess, phi  N  M   free-surface cell mass, excess share, fill level
//   recon  8N  C   populations rebuilt by FS_1 toward gas (reference mode only)
// S/C/M: storage / arithmetic / mass types.
#pragma once

#include <utility>

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lattice.cuh"

namespace flb {

constexpr int kBlock = 256;

struct KParams {
  uint32_t nx, ny, N;
  void* f;
  void* slot[9];  // f + s*N, typed by the kernel
  void* rho;
  void* u;
  uint8_t* flags;      // current flags
  uint8_t* flags_out;  // flag-stencil pass output
  const uint8_t* nbmask;
  void* mass;
  void* excess;
  void* phi;
  void* recon;
  uint8_t* recon_mask;
  const void* rho_snap;
  const void* u_snap;
  float inv_tau, fx, fy;
  float cF[9];  // cx[i]*Fx + cy[i]*Fy, computed on the host in float as the reference does per cell
  float f16_scale, f16_inv;
  double inlet_ux, inlet_uy;
  int use_force, subgrid, collision, fs_cons;
  // 1 when flags_out holds the previous step's post-stream-collide flags and
  // the mass fields come from the previous full step (see k_fs234)
  int trust_prev;
  float u_max;  // velocity limiter, 0 = off
  // fused SRT arithmetic (collide_fused), float constants computed on the host:
  // 1-w, -3k, F/2, F (zero without forcing), and per direction pair q (odd
  // direction 2q+1) 3k c.F and 9k c.F, with k = 1 - w/2
  float fu_omc, fu_nk3, fu_hfx, fu_hfy, fu_fx, fu_fy;
  float fu_g[4], fu_h[4];
  float fu_sw[3];  // FP16S deviation form: f16_scale * w for directions 0, 1..4, 5..8
  int has_io;      // the case has inlet or outlet cells
  // time step of the FP16S stochastic rounding: the step with parity q reads
  // tstep[q] and writes tstep[q ^ 1] = t + 1 (graph replays see the current t)
  uint32_t* tstep;
  // single phase: chunk map of plain fluid cells, 4 cells per bit (k_plain_chunks); null otherwise
  const uint32_t* plain;
};

// Whether the n*4 cells from cell c (a multiple of 4n, n = 1 or 2) are all
// plain fluid cells with no wall neighbour.
template <int n>
__device__ __forceinline__ bool plain_cells(const uint32_t* plain, uint32_t c) {
  const uint32_t word = plain[c >> 7], bit = (c >> 2) & 31u;
  constexpr uint32_t m = (1u << n) - 1u;
  return ((word >> bit) & m) == m;
}

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}
__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }

// Free-surface steps work on super-tiles of kSTW x kSTH cells.  Only the
// super-tiles a pass can change are visited: the flag pass, as it finishes a
// super-tile, appends to the next step's lists the super-tiles that step must
// visit (NextLists), and the next step's passes loop over the lists in a
// persistent grid.  all = 1 visits every super-tile (first step after the
// state was set from outside).
constexpr uint32_t kSTW = 128, kSTH = 8;
// threads per block of the listed stream-collide and FS_1 kernels: 1024 take
// a super-tile in one pass (one cell per thread), 256 in four (row chunks)
#ifndef FLB_LIST_BLOCK
#define FLB_LIST_BLOCK 1024
#endif
constexpr int kListBlock = FLB_LIST_BLOCK;

struct TileList {
  const uint32_t* list;
  const uint32_t* count;
  uint32_t ntiles, nsx;
  int all;
};

// Programmatic dependent launch.  The free-surface step kernels are launched
// with launch_pdl, so the next kernel on the stream (also inside a CUDA graph)
// may be scheduled while this one drains.  Each such kernel calls pdl_wait()
// before its first read of anything the previous kernel wrote (it returns once
// that kernel has completed and its writes are visible; it returns at once
// when the kernel was launched without the attribute), then pdl_trigger() to
// let its own successor be scheduled.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Where the flag pass of the step at t appends the super-tiles of step t+1:
// FS_1 and stream-collide visit those holding fluid or interface cells
// (list_sc); the flag pass also visits a neighbour of such a super-tile when
// one of those cells lies within the stencil chain's reach of their shared
// edge or corner, and, once more, those that held such cells a step earlier
// (list_fs; bits marks the super-tiles already in it, so each is listed once).
// The lengths and the marks start at zero: FS_1 of the same step clears them
// (ListClear), after the previous step's passes have finished reading that
// parity's lists.
struct NextLists {
  uint32_t* list_sc;
  uint32_t* list_fs;
  uint32_t* counts;  // [2]: lengths of list_sc and list_fs
  uint32_t* bits;    // (ntiles + 31) / 32 words
  uint32_t nsx, nsy;
};
struct ListClear {
  uint32_t* counts;  // [2]
  uint32_t* bits;
  uint32_t nwords;
};

// FS_1's first block clears the lengths and marks the flag pass of the same
// step appends to (called after pdl_wait).
__device__ __forceinline__ void clear_next_lists(const ListClear& lc) {
  if (blockIdx.x != 0 || !lc.counts) return;
  if (threadIdx.x < 2) lc.counts[threadIdx.x] = 0u;
  for (uint32_t i = threadIdx.x; i < lc.nwords; i += blockDim.x) lc.bits[i] = 0u;
}

// What the persistent free-surface step (k_fsp.cu) needs besides the step
// parameters: the lists and their lengths of both parities (read by the step
// of that parity, built by the step before), the activity words, and its
// grid barrier.
struct FspArgs {
  uint32_t* list[2][2];  // [parity][0: FS_1 and stream-collide, 1: flag pass]
  uint32_t* lcount;      // [parity][2] list lengths
  uint32_t* lbits;       // [parity][nwords] marks of the flag-pass lists
  uint32_t nwords;
  uint32_t* nz;
  uint32_t nsx, nsy;
  int fs_all;            // the flag pass visits every super-tile (thin last super-tiles)
  uint32_t* bar;         // grid barrier arrivals, zeroed before each launch
  uint32_t* err;         // set when a barrier wait gave up
  uint32_t steps;        // even: the run starts at an even t with flag buffer 0 current
  uint32_t wait_limit;   // polls before a barrier wait gives up
  uint32_t skip_cta;     // failure injection: this CTA never arrives (0xffffffff: none)
  uint64_t* trace;       // null, or 3*steps+1 slots: CTA 0's exit time of each barrier (ns)
};

// A list holds at most ntiles entries; the length is clamped so that no state
// (a launch that gave up part-way, for instance) can make a pass read past it.
__device__ __forceinline__ uint32_t tile_count(const TileList& tl) {
  return tl.all ? tl.ntiles : min(__ldcg(tl.count), tl.ntiles);
}
__device__ __forceinline__ uint32_t tile_at(const TileList& tl, uint32_t i) { return tl.all ? i : tl.list[i]; }

// ---- L2 prefetch of a super-tile ------------------------------------------------
// Bulk L2 prefetch (a hint with no reply) of `bytes` bytes from `p`, rounded
// inward to 16-byte boundaries so that it never leaves the range given.
__device__ __forceinline__ void l2_prefetch_inward(const char* p, uint32_t bytes) {
  const uintptr_t a = ((uintptr_t)p + 15u) & ~(uintptr_t)15u, e = ((uintptr_t)p + bytes) & ~(uintptr_t)15u;
  if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// The rows a listed pass reads for super-tile t, prefetched into L2 while the
// block works on its current super-tile: the nine population slots (pop
// bytes per value) of rows y0-1 .. y0+8, the flags of the same rows, and
// (with_mass) the mass of rows y0 .. y0+7 and the excess of rows y0-1 ..
// y0+8 (FP64 or FP32, m bytes), each row over the super-tile's columns.
// Rows outside the grid are left out (their periodic images are read
// normally).  Thread k of the block issues task k; the block needs at least
// 9 * 10 + 10 (+ 8 + 10) threads.  FS_1 uses it (8192x2048 dam break: 83 ->
// 80 us per step); in the listed stream-collide it measured slower (76.5 ->
// 85.4 us), so that pass does without.
__device__ __forceinline__ void prefetch_super_tile(const KParams& p, uint32_t t, uint32_t nsx, uint32_t pop,
                                                   bool with_mass, uint32_t m) {
  const uint32_t k = threadIdx.x;
  const uint32_t x0 = (t % nsx) * kSTW, y0 = (t / nsx) * kSTH;
  const uint32_t w = min(kSTW, p.nx - x0);
  int row = -1;
  const char* base = nullptr;
  uint32_t elem = 0;
  if (k < 90u) {  // populations: slot k / 10, row y0 - 1 + k % 10
    row = (int)y0 - 1 + (int)(k % 10u);
    base = static_cast<const char*>(p.slot[k / 10u]);
    elem = pop;
  } else if (k < 100u) {  // flags
    row = (int)y0 - 1 + (int)(k - 90u);
    base = reinterpret_cast<const char*>(p.flags);
    elem = 1;
  } else if (with_mass && k < 108u) {  // mass
    row = (int)y0 + (int)(k - 100u);
    base = static_cast<const char*>(p.mass);
    elem = m;
  } else if (with_mass && k < 118u) {  // excess
    row = (int)y0 - 1 + (int)(k - 108u);
    base = static_cast<const char*>(p.excess);
    elem = m;
  }
  if (row < 0 || row >= (int)p.ny) return;
  l2_prefetch_inward(base + ((size_t)row * p.nx + x0) * elem, w * elem);
}

template <class S>
__device__ __forceinline__ S* slotp(const KParams& p, int s) {
  return static_cast<S*>(p.slot[s]);
}

// Slot holding incoming population i of a cell (i odd: own cell, slot a;
// i+1: neighbour i's cell, slot b), cellCalculations.cuh:185-196.
template <bool ODD>
__device__ __forceinline__ constexpr int slot_a(int i) { return ODD ? i : i + 1; }
template <bool ODD>
__device__ __forceinline__ constexpr int slot_b(int i) { return ODD ? i + 1 : i; }

// loadf plus the half-way wall: a population that would arrive from a wall
// neighbour is read from where this cell stored the opposite population last
// step, i.e. it comes back reflected after one step.  nbm bit k-1 = neighbour
// k is a wall.
template <class S, class C, bool HW, bool ODD, class K = Codec<S, C>>
__device__ __forceinline__ void load_in(const KParams& p, uint32_t idx, const uint32_t* nb, uint32_t nbm, C* f) {
  const float inv = p.f16_inv;
  f[0] = K::ld(slotp<S>(p, 0), idx, 0, inv);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const int a = slot_a<ODD>(i), b = slot_b<ODD>(i);
    if (HW && ((nbm >> i) & 1u)) f[i] = K::ld(slotp<S>(p, b), idx, i, inv);
    else f[i] = K::ld(slotp<S>(p, a), idx, i, inv);
    if (HW && ((nbm >> (i - 1)) & 1u)) f[i + 1] = K::ld(slotp<S>(p, a), nb[i], i + 1, inv);
    else f[i + 1] = K::ld(slotp<S>(p, b), nb[i], i + 1, inv);
  }
}

// The half-way wall part of load_in alone: f holds what load_in reads when
// no neighbour is a wall, and the populations that arrive from a wall
// neighbour (nbm) are replaced by their reflections.
template <class S, class C, bool ODD, class K = Codec<S, C>>
__device__ __forceinline__ void reload_reflected(const KParams& p, uint32_t idx, const uint32_t* nb, uint32_t nbm,
                                                 C* f) {
  const float inv = p.f16_inv;
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const int a = slot_a<ODD>(i), b = slot_b<ODD>(i);
    if ((nbm >> i) & 1u) f[i] = K::ld(slotp<S>(p, b), idx, i, inv);
    if ((nbm >> (i - 1)) & 1u) f[i + 1] = K::ld(slotp<S>(p, a), nb[i], i + 1, inv);
  }
}

// loadOutgoingf, cellCalculations.cuh:207-217.
template <class S, class C, bool ODD>
__device__ __forceinline__ void load_out(const KParams& p, uint32_t idx, const uint32_t* nb, C* out) {
  const float inv = p.f16_inv;
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    out[i] = Codec<S, C>::ld(slotp<S>(p, slot_a<ODD>(i)), nb[i], i, inv);
    out[i + 1] = Codec<S, C>::ld(slotp<S>(p, slot_b<ODD>(i)), idx, i + 1, inv);
  }
}

// storef, cellCalculations.cuh:228-238.
template <class S, class C, bool ODD, class K = Codec<S, C>>
__device__ __forceinline__ void store_post(const KParams& p, uint32_t idx, const uint32_t* nb, const C* f) {
  const float sc = p.f16_scale;
  K::st(slotp<S>(p, 0), idx, 0, f[0], sc);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    K::st(slotp<S>(p, slot_b<ODD>(i)), nb[i], i, f[i], sc);
    K::st(slotp<S>(p, slot_a<ODD>(i)), idx, i + 1, f[i + 1], sc);
  }
}

// Runtime-parity wrappers for passes that are not on the step's hot path.
template <class S, class C, bool HW>
__device__ __forceinline__ void load_in_rt(const KParams& p, uint32_t odd, uint32_t idx, const uint32_t* nb,
                                           uint32_t nbm, C* f) {
  if (odd) load_in<S, C, HW, true>(p, idx, nb, nbm, f);
  else load_in<S, C, HW, false>(p, idx, nb, nbm, f);
}

}  // namespace flb
