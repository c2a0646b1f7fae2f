// batch.cu -- a batch of independent single-phase cases advanced together.
//
// FlowLB runs one case per call (runCuda.cu:30-128).  An ensemble of small
// cases (the culvert parameter sweep: 512 grids of 128..1024 x 64..256 cells)
// run that way is bound by launch latency: every step of a case is one small
// kernel.  Here one persistent kernel runs all the steps of all the cases:
//  * the grid is made of thread-block clusters; a cluster owns a list of
//    cases (longest-processing-time assignment on the host) and runs each to
//    the end before the next, the steps separated by a cluster barrier
//    (barrier.cluster arrive.release / wait.acquire, which also orders the
//    global-memory exchange of populations between the cluster's CTAs);
//  * the warps of a cluster share a case step by 32-cell row segments;
//  * a case's parameters sit in shared memory for the duration of the case;
//  * the cells are updated with the loads, collision (collide_cell) and
//    stores of the single-case kernels, so every case ends bit-identical to
//    flb_step on its own handle.
// With few clusters only a few cases are active at a time, so their
// populations stay in the 126 MB L2 while they are stepped.  The cluster size
// and the number of clusters are chosen by a short timed search at creation
// (flb_batch_create with autotune).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "launch.h"
#include "sc_cell.cuh"

namespace cg = cooperative_groups;

namespace flb {
namespace {

constexpr int kBatchMaxThreads = 1024;  // CTA sizes 256, 512 or 1024 (autotuned)
constexpr int kMaxStreams = 64;         // streams of the streams form
#ifndef FLB_BATCH_MIN_BLOCKS
#define FLB_BATCH_MIN_BLOCKS 2  // two 1024-thread CTAs per SM: at most 32 registers
#endif
// the vector data path: CTAs of at most 512 threads, FLB_BATCH_VEC_MIN_BLOCKS
// per SM (two: 64 registers)
constexpr int kBatchVecMaxThreads = 512;
#ifndef FLB_BATCH_VEC_MIN_BLOCKS
#define FLB_BATCH_VEC_MIN_BLOCKS 2
#endif
constexpr uint32_t kVecCells = 4;  // cells per thread on the vector path

// A case of the batch.  Its rows are stored kVecCells-aligned: row y starts at
// cell y * sx, sx = nx rounded up to a multiple of 4, and the cells x >= nx of
// a row are padding (flagged solid, never updated; their population slots are
// scratch).  kp.N = sx * ny is the padded cell count (slot s at s * N).
struct BatchCase {
  KParams kp;
  uint32_t sx;  // row stride
  // set on the device for the launch shape: row segments per row (32 cells,
  // or 128 on the vector path), and a warp's walk over them advances dy rows
  // and ds segments per item
  uint32_t nseg, dy, ds;
};

// Neighbour cells of (x, y) in a case stored with row stride sx (periodic).
__device__ __forceinline__ void neighbours_sx(uint32_t x, uint32_t y, uint32_t nx, uint32_t ny, uint32_t sx,
                                              uint32_t* nb) {
  const uint32_t yc = y * sx;
  const uint32_t yu = (y + 1u == ny ? 0u : y + 1u) * sx;
  const uint32_t yd = (y == 0u ? ny - 1u : y - 1u) * sx;
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

// sc_cell for a batch case (single phase, FP32): the same loads, collision
// and stores, with slot s addressed as s*N cells past the case's first
// population instead of through the slot pointer table, which here sits in
// shared memory and would cost a 64-bit shared load per population.
template <bool HW, bool FU, bool ODD, bool WM>
__device__ __forceinline__ void batch_cell(const KParams& p, uint32_t sx, uint32_t x, uint32_t y) {
  const uint32_t N = p.N, idx = x + y * sx;
  float* __restrict__ F = static_cast<float*>(p.f);
  uint32_t nb[9];
  neighbours_sx(x, y, p.nx, p.ny, sx, nb);
  const uint8_t flag = p.flags[idx];
  const uint32_t nbm = HW ? (uint32_t)p.nbmask[idx] : 0u;
  // populations through L2 only: other CTAs wrote them last step, and no
  // location is read twice in a step
  float f[9];
  f[0] = __ldcg(F + idx);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const uint32_t a = (uint32_t)slot_a<ODD>(i) * N, b = (uint32_t)slot_b<ODD>(i) * N;
    f[i] = __ldcg(F + ((HW && ((nbm >> i) & 1u)) ? b : a) + idx);
    f[i + 1] = __ldcg(F + ((HW && ((nbm >> (i - 1)) & 1u)) ? a : b) + nb[i]);
  }
  if (flag & (kGas | kWall)) return;
  collide_cell<float, double, false, WM, FU>(p, idx, x, y, flag, nbm, f);
  // the addresses again, from shared memory and (x, y): cheaper than keeping
  // them live through the collision under the 32-register budget
  asm volatile("" ::: "memory");
  float* G = static_cast<float*>(p.f);
  const uint32_t M = p.N, ids = x + y * sx;
  neighbours_sx(x, y, p.nx, p.ny, sx, nb);
  G[ids] = f[0];
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    G[(uint32_t)slot_b<ODD>(i) * M + nb[i]] = f[i];
    G[(uint32_t)slot_a<ODD>(i) * M + ids] = f[i + 1];
  }
}

// The vector data path: kVecCells consecutive cells per thread (x0 .. x0+3 of
// row y; x0 a multiple of 4), each population slot moved with one 16-byte
// access (the padded row stride keeps them aligned), the slots of the x+1
// neighbours shifted between lanes by shuffles, as the single-case vector
// kernel (k_sc_vec) does.  The 32 lanes of a warp cover a 128-cell row
// segment.  The group holding the row's last cell (x = nx - 1) takes that
// cell's x+1 neighbour from x = 0 (periodic) and writes its outgoing
// population there; padding cells are never updated.  Same loads, collision
// and stores per cell as batch_cell, so the results are the same bit for bit.
template <bool HW, bool FU, bool ODD, bool WM>
__device__ __forceinline__ void batch_vec(const KParams& p, uint32_t sx, uint32_t x0, uint32_t y, uint32_t lane) {
  constexpr int V = (int)kVecCells;
  const uint32_t nx = p.nx, ny = p.ny, N = p.N;
  float* F = static_cast<float*>(p.f);
  const bool inrow = x0 < nx;
  const uint32_t row = y * sx;
  const uint32_t rowu = (y + 1u == ny ? 0u : y + 1u) * sx;
  const uint32_t rowd = (y == 0u ? ny - 1u : y - 1u) * sx;
  const bool last = inrow && x0 + (uint32_t)V >= nx;       // the group holding the row's last cell
  const uint32_t kl = last ? nx - 1u - x0 : (uint32_t)V - 1u;  // that cell's position in the group
  const bool tail = inrow && (lane == 31u || last);        // its x+1 neighbour is not in the next lane
  const uint32_t xn = last ? 0u : x0 + (uint32_t)V;         // where that neighbour is
  uint8_t fl[V] = {kWall, kWall, kWall, kWall};
  uint8_t nbmv[V] = {0, 0, 0, 0};
  float raw0[V], own[4][V], nbr[4][V], tmp[4][V];
  if (inrow) {
    const uchar4 fv = *reinterpret_cast<const uchar4*>(p.flags + row + x0);
    fl[0] = fv.x; fl[1] = fv.y; fl[2] = fv.z; fl[3] = fv.w;
    if (HW) {
      const uchar4 mv = *reinterpret_cast<const uchar4*>(p.nbmask + row + x0);
      nbmv[0] = mv.x; nbmv[1] = mv.y; nbmv[2] = mv.z; nbmv[3] = mv.w;
    }
    // populations through L2 only (other CTAs wrote them last step)
    const float4 r0 = __ldcg(reinterpret_cast<const float4*>(F + row + x0));
    raw0[0] = r0.x; raw0[1] = r0.y; raw0[2] = r0.z; raw0[3] = r0.w;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      const float4 a = __ldcg(reinterpret_cast<const float4*>(F + (uint32_t)slot_a<ODD>(i) * N + row + x0));
      const float4 b = __ldcg(reinterpret_cast<const float4*>(F + (uint32_t)slot_b<ODD>(i) * N + r + x0));
      own[q][0] = a.x; own[q][1] = a.y; own[q][2] = a.z; own[q][3] = a.w;
      tmp[q][0] = b.x; tmp[q][1] = b.y; tmp[q][2] = b.z; tmp[q][3] = b.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < V; k++) {
      raw0[k] = 0.0f;
#pragma unroll
      for (int q = 0; q < 4; q++) own[q][k] = tmp[q][k] = 0.0f;
    }
  }
  bool act[V];
  bool any = false;
#pragma unroll
  for (int k = 0; k < V; k++) {
    act[k] = !(fl[k] & (kGas | kWall));
    any |= act[k];
  }
  // a warp with no cell to update leaves memory untouched
  if (!__any_sync(0xffffffffu, any)) return;
  // realign the x+1 slots (direction 3, +y, has no x shift)
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    if (i == 3) {
#pragma unroll
      for (int k = 0; k < V; k++) nbr[q][k] = tmp[q][k];
    } else {
      const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
      const float from_next = __shfl_down_sync(0xffffffffu, tmp[q][0], 1);
#pragma unroll
      for (int k = 0; k < V - 1; k++) nbr[q][k] = tmp[q][k + 1];
      nbr[q][V - 1] = from_next;
      if (tail) {
        const float w = __ldcg(F + (uint32_t)slot_b<ODD>(i) * N + r + xn);
#pragma unroll
        for (int k = 0; k < V; k++)
          if ((uint32_t)k == kl) nbr[q][k] = w;
      }
    }
  }
  // per-cell collision; cells not updated keep their loaded values
#pragma unroll
  for (int k = 0; k < V; k++) {
    if (!act[k]) continue;
    const uint32_t x = x0 + (uint32_t)k, idx = row + x;
    float f[9];
    f[0] = raw0[k];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      f[2 * q + 1] = own[q][k];
      f[2 * q + 2] = nbr[q][k];
    }
    const uint32_t nbm = nbmv[k];
    if (HW && nbm) {
      // half-way walls: reflected populations, scalar (wall-adjacent cells only)
      uint32_t nb[9];
      neighbours_sx(x, y, nx, ny, sx, nb);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        if ((nbm >> i) & 1u) f[i] = __ldcg(F + (uint32_t)slot_b<ODD>(i) * N + idx);
        if ((nbm >> (i - 1)) & 1u) f[i + 1] = __ldcg(F + (uint32_t)slot_a<ODD>(i) * N + nb[i]);
      }
    }
    collide_cell<float, double, false, WM, FU>(p, idx, x, y, fl[k], nbm, f);
    raw0[k] = f[0];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      nbr[q][k] = f[2 * q + 1];  // post f_i -> the x+1 (or +y) neighbour's slot b
      own[q][k] = f[2 * q + 2];  // post f_{i+1} -> own slot a
    }
  }
  // stores
  if (inrow) {
    *reinterpret_cast<float4*>(F + row + x0) = make_float4(raw0[0], raw0[1], raw0[2], raw0[3]);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = 2 * q + 1;
      *reinterpret_cast<float4*>(F + (uint32_t)slot_a<ODD>(i) * N + row + x0) =
          make_float4(own[q][0], own[q][1], own[q][2], own[q][3]);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const uint32_t r = (i == 1) ? row : (i == 7 ? rowd : rowu);
    float* dst = F + (uint32_t)slot_b<ODD>(i) * N + r;
    if (i == 3) {
      if (inrow) *reinterpret_cast<float4*>(dst + x0) = make_float4(nbr[q][0], nbr[q][1], nbr[q][2], nbr[q][3]);
    } else {
      const float from_prev = __shfl_up_sync(0xffffffffu, nbr[q][V - 1], 1);
      if (inrow) {
        // position x0 belongs to the previous lane's last cell (or, for lane 0,
        // to the previous segment, which writes it itself)
        if (lane != 0u) {
          *reinterpret_cast<float4*>(dst + x0) = make_float4(from_prev, nbr[q][0], nbr[q][1], nbr[q][2]);
        } else {
#pragma unroll
          for (int k = 0; k < V - 1; k++) dst[x0 + 1 + k] = nbr[q][k];
        }
        if (tail) {
          float w = nbr[q][V - 1];
#pragma unroll
          for (int k = 0; k < V; k++)
            if ((uint32_t)k == kl) w = nbr[q][k];
          dst[xn] = w;
        }
      }
    }
  }
}

// One step of one case: the warps of the group take row segments (32 cells;
// 128 on the vector path), warp k the segments k, k + nw, k + 2 nw, ... (nw
// warps in the group); a warp starts at row y, segment s.  The case (in
// shared memory) is re-read per item rather than held in registers.
template <bool HW, bool FU, bool ODD, bool WM>
__device__ __noinline__ void batch_step_cells(const BatchCase& c, uint32_t y, uint32_t s, uint32_t lane) {
  while (y < c.kp.ny) {
    const uint32_t x = s * 32u + lane;
    if (x < c.kp.nx) batch_cell<HW, FU, ODD, WM>(c.kp, c.sx, x, y);
    s += c.ds;
    y += c.dy;
    if (s >= c.nseg) {
      s -= c.nseg;
      y++;
    }
  }
}
template <bool HW, bool FU, bool ODD, bool WM>
__device__ __noinline__ void batch_step_vec(const BatchCase& c, uint32_t y, uint32_t s, uint32_t lane) {
  while (y < c.kp.ny) {
    batch_vec<HW, FU, ODD, WM>(c.kp, c.sx, s * (32u * kVecCells) + lane * kVecCells, y, lane);
    s += c.ds;
    y += c.dy;
    if (s >= c.nseg) {
      s -= c.nseg;
      y++;
    }
  }
}
template <bool HW, bool FU, bool ODD, bool WM, bool VEC>
__device__ __forceinline__ void batch_step(const BatchCase& c, uint32_t y, uint32_t s, uint32_t lane) {
  if constexpr (VEC) batch_step_vec<HW, FU, ODD, WM>(c, y, s, lane);
  else batch_step_cells<HW, FU, ODD, WM>(c, y, s, lane);
}

// Team barrier (FLB_BATCH_TEAM): the CTAs of a team meet in global memory on
// an arrival count, one per team, 128 bytes apart.  The counts are zeroed
// before every launch and only grow: the r-th barrier of a team in a launch
// is passed once its count reaches r times the team's size, so an arrival is
// a single reduction with no reply and no reset is needed between rounds.
struct TeamSync {
  uint32_t count, pad[31];
};
// polls (about 1 us each) before a wait gives up, unless flb_batch_set_wait_limit set another
constexpr uint32_t kTeamSpinLimit = 1u << 21;
// no CTA skips its arrival (see k_batch's skip_rank)
constexpr uint32_t kNoSkip = 0xffffffffu;

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* a) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(uint32_t* a, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

// All CTAs of the team have finished the step (and their writes are visible)
// when this returns true: the team's count has reached `target` arrivals.
// Thread 0 arrives for the CTA (fence, then a release reduction) and polls
// with acquire loads.  A wait longer than `limit` polls sets *err; a CTA that
// sees *err set (checked every 64 polls) stops waiting too; either returns
// false and the caller leaves the kernel.  arrive = false (failure injection
// only) makes this CTA wait without arriving, so the round never completes
// and every wait of the team runs out.
__device__ __forceinline__ bool team_sync(TeamSync* ts, uint32_t target, uint32_t* err, int& ok, uint32_t limit,
                                          bool arrive) {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool good = true;
    __threadfence();
    if (arrive) red_release_add(&ts->count, 1u);
    uint32_t it = 0;
    while (ld_acquire(&ts->count) < target) {
      if (++it >= limit) {
        good = false;
        atomicOr(err, 1u);
        break;
      }
      if ((it & 63u) == 0u && ld_acquire(err) != 0u) {
        good = false;
        break;
      }
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// *tdev: time step of the first step (its parity selects the slot pattern);
// steps >= 1; wm_last: write density and velocity in the last step.  A group
// of `group` consecutive CTAs steps one case at a time: a thread-block cluster
// (TEAM false; cluster barrier between steps) or a team of co-resident CTAs of
// a cooperative launch (TEAM true; team_sync between steps, each wait bounded
// by wait_limit polls).  skip_rank: in team mode, the CTA of each team with
// this rank never arrives at its team's barriers (failure injection; kNoSkip
// in normal operation); unused in cluster mode.
// VEC: the vector data path (kVecCells cells per thread, at most
// kBatchVecMaxThreads threads per CTA).
template <bool HW, bool FU, bool TEAM, bool VEC>
__global__ void __launch_bounds__(VEC ? kBatchVecMaxThreads : kBatchMaxThreads,
                                  VEC ? FLB_BATCH_VEC_MIN_BLOCKS : FLB_BATCH_MIN_BLOCKS)
    k_batch(const BatchCase* __restrict__ cases, const uint32_t* __restrict__ order, const uint32_t* __restrict__ start,
            const uint32_t* __restrict__ tdev, uint32_t steps, int wm_last, uint32_t group, TeamSync* sync,
            uint32_t* err, uint32_t wait_limit, uint32_t skip_rank) {
  __shared__ BatchCase sc;
  __shared__ int ok;
  const uint32_t t0 = *tdev;
  const uint32_t cid = blockIdx.x / group, rank = blockIdx.x % group;
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t wid = rank * warps + (threadIdx.x >> 5), nw = group * warps;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t round = 0;  // team barriers passed in this launch
  for (uint32_t k = start[cid]; k < start[cid + 1]; k++) {
    __syncthreads();  // the previous case's parameters are no longer read
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&cases[order[k]]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sc);
      for (uint32_t i = threadIdx.x; i < offsetof(BatchCase, nseg) / 4; i += blockDim.x) dst[i] = src[i];
      if (threadIdx.x == 0) {
        const uint32_t seg = VEC ? 32u * kVecCells : 32u;
        const uint32_t n = (cases[order[k]].kp.nx + seg - 1u) / seg;
        sc.nseg = n;
        sc.dy = nw / n;
        sc.ds = nw % n;
      }
    }
    __syncthreads();
    const uint32_t nsegx = sc.nseg, y0 = wid / nsegx, s0 = wid % nsegx;
    for (uint32_t s = 0; s < steps; s++) {
      const bool odd = ((t0 + s) & 1u) != 0;
      const bool wm = wm_last && s + 1 == steps;
      if (odd) {
        if (wm) batch_step<HW, FU, true, true, VEC>(sc, y0, s0, lane);
        else batch_step<HW, FU, true, false, VEC>(sc, y0, s0, lane);
      } else {
        if (wm) batch_step<HW, FU, false, true, VEC>(sc, y0, s0, lane);
        else batch_step<HW, FU, false, false, VEC>(sc, y0, s0, lane);
      }
      if constexpr (TEAM) {
        if (!team_sync(&sync[cid], ++round * group, err, ok, wait_limit, rank != skip_rank)) return;
      } else {
        cg::this_cluster().sync();
      }
    }
  }
}

// advances the device time-step counter after a batch launch
__global__ void k_tadd(uint32_t* t, uint32_t n) { *t += n; }

using BatchKernel = void (*)(const BatchCase*, const uint32_t*, const uint32_t*, const uint32_t*, uint32_t, int,
                             uint32_t, TeamSync*, uint32_t*, uint32_t, uint32_t);

template <bool VEC>
BatchKernel pick_kernel_v(bool hw, bool fu, bool team) {
  if (team) {
    if (hw) return fu ? k_batch<true, true, true, VEC> : k_batch<true, false, true, VEC>;
    return fu ? k_batch<false, true, true, VEC> : k_batch<false, false, true, VEC>;
  }
  if (hw) return fu ? k_batch<true, true, false, VEC> : k_batch<true, false, false, VEC>;
  return fu ? k_batch<false, true, false, VEC> : k_batch<false, false, false, VEC>;
}
BatchKernel pick_kernel(bool hw, bool fu, bool team, bool vec) {
  return vec ? pick_kernel_v<true>(hw, fu, team) : pick_kernel_v<false>(hw, fu, team);
}

}  // namespace
}  // namespace flb

using namespace flb;

struct flb_batch_s {
  uint32_t n = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool hw = false, fu = false;
  uint64_t t = 0;
  std::vector<uint32_t> nx, ny;
  std::vector<size_t> off;   // first cell of each case in the concatenated geometry (nx * ny cells each)
  std::vector<size_t> poff;  // first cell of each case in the padded state arrays (sx * ny cells each)
  std::vector<uint32_t> sx;  // padded row stride of each case (nx rounded up to a multiple of 4)
  size_t cells = 0, pcells = 0, max_cells = 0;
  // initialisation scratch for one case in the compact layout
  float *d_sf = nullptr, *d_srho = nullptr, *d_su = nullptr;
  uint8_t *d_sflags = nullptr, *d_snb = nullptr;
  float* d_f = nullptr;
  float* d_rho = nullptr;
  float* d_u = nullptr;
  uint8_t* d_flags = nullptr;
  uint8_t* d_geo = nullptr;
  uint8_t* d_nbmask = nullptr;
  uint32_t* d_tstep = nullptr;
  BatchCase* d_cases = nullptr;
  uint32_t* d_order = nullptr;
  uint32_t* d_start = nullptr;
  TeamSync* d_sync = nullptr;  // one per team (FLB_BATCH_TEAM)
  uint32_t* d_err = nullptr;   // set when a team barrier gave up waiting
  uint32_t wait_limit = kTeamSpinLimit;  // polls before a team barrier wait gives up
  // a team barrier gave up: populations and t no longer describe a finished
  // step, so stepping is refused until flb_batch_reset
  bool broken = false;
  std::vector<BatchCase> hcases;
  // launch configuration: `clusters` groups of `cluster` CTAs of `threads`
  // threads, each group a thread-block cluster or (team) a team
  int cluster = 8, clusters = 0, threads = 512, tuned = 0;
  bool team = false;
  bool vec = false;  // the vector data path (kVecCells cells per thread)
  // FLB_BATCH_STREAMS: every case an engine handle (the single-case kernels
  // and step graphs) on one of `nstreams` streams, longest cases first, so
  // that the cases' step sequences run concurrently; while the form is on,
  // the handles hold the state
  bool streams_mode = false;
  int nstreams = 0;
  std::vector<flb_case_desc> descs;  // the cases (flags point into hgeo)
  std::vector<uint8_t> hgeo;         // host copy of every case's geometry flags
  std::vector<flb_handle> handles;
  std::vector<uint32_t> stream_of;   // the pool stream of each case
  std::vector<uint32_t> sorder;      // the cases longest first
  std::vector<cudaStream_t> pool;
  std::vector<cudaEvent_t> pool_ev;
  cudaEvent_t start_ev = nullptr;
  uint64_t launches = 0;
  // the step graph (batch kernel + counter update) for one step count
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint32_t g_steps = 0, g_limit = 0, g_skip = 0;
  int g_wm = -1, g_cluster = 0, g_clusters = 0, g_threads = 0;
  bool g_team = false, g_vec = false;
  std::string err;
};

namespace {

flb_status bfail(flb_batch b, flb_status s, const std::string& m) {
  if (b) b->err = m;
  return s;
}
flb_status bcuda(flb_batch b, cudaError_t e, const char* what) {
  return bfail(b, e == cudaErrorMemoryAllocation ? FLB_ERR_OUT_OF_MEMORY : FLB_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}
#define FLB_BCUDA(b, call)                            \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return bcuda((b), e_, #call); \
  } while (0)

struct BDevice {
  int prev = -1;
  explicit BDevice(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~BDevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

void bdrop_graph(flb_batch b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  b->g_steps = 0;
}

void bfree(flb_batch b) {
  bdrop_graph(b);
  for (flb_handle h : b->handles)
    if (h) flb_destroy(h);
  b->handles.clear();
  for (cudaStream_t st : b->pool) cudaStreamDestroy(st);
  for (cudaEvent_t ev : b->pool_ev) cudaEventDestroy(ev);
  b->pool.clear();
  b->pool_ev.clear();
  if (b->start_ev) cudaEventDestroy(b->start_ev);
  b->start_ev = nullptr;
  void* bufs[] = {b->d_sf,    b->d_srho,  b->d_su,    b->d_sflags, b->d_snb,
                  b->d_f,     b->d_rho,   b->d_u,     b->d_flags, b->d_geo, b->d_nbmask,
                  b->d_tstep, b->d_cases, b->d_order, b->d_start, b->d_sync, b->d_err};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

// Copies `rows` rows of `width` bytes between the compact layout (pitch =
// width) and a padded one (pitch = stride bytes).
cudaError_t copy_rows(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows,
                      cudaMemcpyKind kind, cudaStream_t st) {
  return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, st);
}

// Initial state of every case: the single-case initialisation in the compact
// layout (scratch), copied row by row into the padded state; padding cells
// are solid, with zero populations and no wall neighbours.
flb_status binit(flb_batch b) {
  BDevice g(b->device);
  const size_t P = b->pcells;
  FLB_BCUDA(b, cudaMemsetAsync(b->d_f, 0, 9 * P * sizeof(float), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_rho, 0, P * sizeof(float), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_u, 0, 2 * P * sizeof(float), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_flags, kWall, P, b->stream));
  if (b->hw) FLB_BCUDA(b, cudaMemsetAsync(b->d_nbmask, 0, P, b->stream));
  for (uint32_t c = 0; c < b->n; c++) {
    const size_t o = b->off[c], po = b->poff[c];
    const uint32_t nx = b->nx[c], ny = b->ny[c], sx = b->sx[c];
    const size_t N = (size_t)nx * ny;
    KParams kp = b->hcases[c].kp;  // constants of the case, compact scratch pointers
    kp.N = (uint32_t)N;
    kp.f = b->d_sf;
    for (int q = 0; q < 9; q++) kp.slot[q] = b->d_sf + (size_t)q * N;
    kp.rho = b->d_srho;
    kp.u = b->d_su;
    FLB_BCUDA(b, cudaMemsetAsync(b->d_sf, 0, 9 * N * sizeof(float), b->stream));
    launch_init_flags(b->d_geo + o, b->d_sflags, nx, ny, 0, nullptr, nullptr, nullptr, 1, b->stream);
    if (b->hw) launch_nbmask(b->d_geo + o, b->d_snb, nx, ny, b->stream);
    launch_init_ddf<float, float, double>(kp, b->stream, b->d_geo + o, b->hw);
    const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
    FLB_BCUDA(b, copy_rows(b->d_f + 9 * po, sx * 4, b->d_sf, nx * 4, nx * 4, 9 * (size_t)ny, dd, b->stream));
    FLB_BCUDA(b, copy_rows(b->d_rho + po, sx * 4, b->d_srho, nx * 4, nx * 4, ny, dd, b->stream));
    FLB_BCUDA(b, copy_rows(b->d_u + 2 * po, sx * 4, b->d_su, nx * 4, nx * 4, 2 * (size_t)ny, dd, b->stream));
    FLB_BCUDA(b, copy_rows(b->d_flags + po, sx, b->d_sflags, nx, nx, ny, dd, b->stream));
    if (b->hw) FLB_BCUDA(b, copy_rows(b->d_nbmask + po, sx, b->d_snb, nx, nx, ny, dd, b->stream));
  }
  FLB_BCUDA(b, cudaMemsetAsync(b->d_tstep, 0, 2 * sizeof(uint32_t), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_sync, 0, b->n * sizeof(TeamSync), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), b->stream));
  FLB_BCUDA(b, cudaGetLastError());
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  b->t = 0;
  b->broken = false;
  return FLB_OK;
}

// Longest-processing-time assignment of the cases to `clusters` clusters.
flb_status bassign(flb_batch b, int clusters) {
  std::vector<uint32_t> idx(b->n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t c) {
    return (uint64_t)b->nx[a] * b->ny[a] > (uint64_t)b->nx[c] * b->ny[c];
  });
  std::vector<uint64_t> load(clusters, 0);
  std::vector<std::vector<uint32_t>> lists(clusters);
  for (uint32_t c : idx) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lists[k].push_back(c);
    load[k] += (uint64_t)b->nx[c] * b->ny[c];
  }
  std::vector<uint32_t> order, start(1, 0u);
  for (auto& l : lists) {
    order.insert(order.end(), l.begin(), l.end());
    start.push_back((uint32_t)order.size());
  }
  // the new arrays are complete before the old ones go, so a failure leaves
  // the previous assignment in place
  uint32_t* d_start = nullptr;
  FLB_BCUDA(b, cudaMalloc(&d_start, start.size() * sizeof(uint32_t)));
  // stream-ordered copies (the batch's stream is non-blocking, and a plain
  // cudaMemcpy from pageable memory may return before its data land), waited
  // for before the host arrays go out of scope
  cudaError_t e = cudaMemcpyAsync(d_start, start.data(), start.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                  b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    cudaFree(d_start);
    return bcuda(b, e, "cudaMemcpy");
  }
  bdrop_graph(b);  // the captured launch refers to the old arrays
  FLB_BCUDA(b, cudaMemcpyAsync(b->d_order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  if (b->d_start) cudaFree(b->d_start);
  b->d_start = d_start;
  b->clusters = clusters;
  return FLB_OK;
}

// Failure injection for tests, read at every launch: with
// FLB_BATCH_SKIP_ARRIVAL=1 in the environment the last CTA of every team never
// arrives at its team's barriers, so each wait runs out after the wait limit
// and the launch reports FLB_ERR_CUDA (team mode only; a hardware cluster
// barrier has no bounded wait and is never skipped).
uint32_t skip_rank_for(flb_batch b) {
  const char* v = std::getenv("FLB_BATCH_SKIP_ARRIVAL");
  if (!b->team || !v || std::strcmp(v, "1") != 0) return kNoSkip;
  return (uint32_t)b->cluster - 1u;
}

// One launch of the batch kernel for n steps on the stream (captured or not).
flb_status bissue(flb_batch b, uint32_t n, int wm_last, uint32_t skip) {
  BatchKernel kern = pick_kernel(b->hw, b->fu, b->team, b->vec);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(b->clusters * b->cluster));
  cfg.blockDim = dim3((unsigned)b->threads);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  if (b->team) {
    // every CTA resident at once: the team barriers wait for one another
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
  } else {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)b->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
  }
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // the team arrival counts start every launch at zero
  if (b->team) FLB_BCUDA(b, cudaMemsetAsync(b->d_sync, 0, (size_t)b->clusters * sizeof(TeamSync), b->stream));
  FLB_BCUDA(b, cudaLaunchKernelEx(&cfg, kern, (const BatchCase*)b->d_cases, (const uint32_t*)b->d_order,
                                  (const uint32_t*)b->d_start, (const uint32_t*)b->d_tstep, n, wm_last,
                                  (uint32_t)b->cluster, b->d_sync, b->d_err, b->wait_limit, skip));
  k_tadd<<<1, 1, 0, b->stream>>>(b->d_tstep, n);
  FLB_BCUDA(b, cudaGetLastError());
  return FLB_OK;
}

// n steps as one graph launch (the graph is kept for the next call with the
// same step count and configuration).
flb_status blaunch(flb_batch b, uint64_t steps, int wm_last) {
  uint64_t done = 0;
  const uint32_t skip = skip_rank_for(b);
  while (done < steps) {  // at most 2^31 steps per launch
    const uint32_t n = (uint32_t)std::min<uint64_t>(steps - done, 1u << 31);
    const int wm = wm_last && done + n == steps;
    if (!b->gexec || b->g_steps != n || b->g_wm != wm || b->g_cluster != b->cluster ||
        b->g_clusters != b->clusters || b->g_threads != b->threads || b->g_team != b->team || b->g_vec != b->vec ||
        b->g_limit != b->wait_limit || b->g_skip != skip) {
      bdrop_graph(b);
      FLB_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      flb_status s = bissue(b, n, wm, skip);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (s != FLB_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
      }
      if (e != cudaSuccess) return bcuda(b, e, "cudaStreamEndCapture");
      b->graph = g;
      FLB_BCUDA(b, cudaGraphInstantiate(&b->gexec, g, 0));
      b->g_steps = n;
      b->g_wm = wm;
      b->g_cluster = b->cluster;
      b->g_clusters = b->clusters;
      b->g_threads = b->threads;
      b->g_team = b->team;
      b->g_vec = b->vec;
      b->g_limit = b->wait_limit;
      b->g_skip = skip;
    }
    FLB_BCUDA(b, cudaGraphLaunch(b->gexec, b->stream));
    b->launches += 2;
    done += n;
  }
  b->t += steps;
  return FLB_OK;
}

// Resident clusters of the given size (0 when the size cannot launch).
int max_clusters(flb_batch b, int cs, int threads, bool vec) {
  if (vec && threads > kBatchVecMaxThreads) return 0;
  BatchKernel kern = pick_kernel(b->hw, b->fu, false, vec);
  if (cs > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cs);
  cfg.blockDim = dim3((unsigned)threads);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// CTAs of the team kernel resident on the device at once (0 on failure).
int max_team_ctas(flb_batch b, int threads, bool vec) {
  if (vec && threads > kBatchVecMaxThreads) return 0;
  int nsm = 0, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick_kernel(b->hw, b->fu, true, vec), threads, 0) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nsm * per_sm;
}

// Groups of `group` CTAs that fit on the device at once for the mode.
int max_groups(flb_batch b, bool team, int group, int threads, bool vec) {
  return team ? max_team_ctas(b, threads, vec) / group : max_clusters(b, group, threads, vec);
}

// Reads and clears the team barriers' error flag: FLB_ERR_CUDA when a wait
// gave up.  The populations of the cases then hold an unfinished step and t
// (advanced when the launch was issued) no longer matches them, so the batch
// refuses to step until flb_batch_reset.
flb_status bcheck(flb_batch b) {
  uint32_t e = 0;
  FLB_BCUDA(b, cudaMemcpyAsync(&e, b->d_err, sizeof(e), cudaMemcpyDeviceToHost, b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  if (!e) return FLB_OK;
  b->broken = true;
  FLB_BCUDA(b, cudaMemsetAsync(b->d_sync, 0, b->n * sizeof(TeamSync), b->stream));
  FLB_BCUDA(b, cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return bfail(b, FLB_ERR_CUDA, "a team barrier gave up waiting; the batch state is undefined until reset");
}

// ---- the streams form (FLB_BATCH_STREAMS) -----------------------------------
void streams_free(flb_batch b) {
  for (flb_handle h : b->handles)
    if (h) flb_destroy(h);
  b->handles.clear();
  b->streams_mode = false;
}

// The pool of nstreams streams, the cases longest first, and every case's
// handle bound to its stream (rank k of that order on stream k % nstreams);
// the handles are created on first use, from the cases' descriptors.
flb_status streams_setup(flb_batch b, int nstreams) {
  while ((int)b->pool.size() < nstreams) {
    cudaStream_t st = nullptr;
    FLB_BCUDA(b, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->pool.push_back(st);
    cudaEvent_t ev = nullptr;
    FLB_BCUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->pool_ev.push_back(ev);
  }
  if (!b->start_ev) FLB_BCUDA(b, cudaEventCreateWithFlags(&b->start_ev, cudaEventDisableTiming));
  b->sorder.resize(b->n);
  std::iota(b->sorder.begin(), b->sorder.end(), 0u);
  std::stable_sort(b->sorder.begin(), b->sorder.end(), [&](uint32_t a, uint32_t c) {
    return (uint64_t)b->nx[a] * b->ny[a] > (uint64_t)b->nx[c] * b->ny[c];
  });
  b->stream_of.assign(b->n, 0u);
  for (uint32_t k = 0; k < b->n; k++) b->stream_of[b->sorder[k]] = k % (uint32_t)nstreams;
  if (b->handles.empty()) {
    b->handles.assign(b->n, nullptr);
    for (uint32_t c = 0; c < b->n; c++) {
      flb_case_desc d = b->descs[c];
      d.device = b->device;
      d.stream = b->pool[b->stream_of[c]];
      const flb_status s = flb_create(&d, &b->handles[c]);
      if (s != FLB_OK) {
        streams_free(b);
        return bfail(b, s, "the streams form could not create the handle of case " + std::to_string(c));
      }
    }
  } else {
    for (uint32_t c = 0; c < b->n; c++) {
      const flb_status s = flb_set_stream(b->handles[c], b->pool[b->stream_of[c]]);
      if (s != FLB_OK) return bfail(b, s, flb_last_error(b->handles[c]));
    }
  }
  b->nstreams = nstreams;
  return FLB_OK;
}

// Populations, density and velocity of case c between the batch's arrays
// (rows padded to sx) and its handle (compact rows), through the scratch.
flb_status case_state_copy(flb_batch b, uint32_t c, bool to_handle) {
  const size_t po = b->poff[c], nx = b->nx[c], ny = b->ny[c], sx = b->sx[c];
  const struct {
    int field;
    float* arr;
    size_t rows;
  } fs[] = {{FLB_FIELD_F, b->d_f + 9 * po, 9 * ny}, {FLB_FIELD_RHO, b->d_rho + po, ny},
            {FLB_FIELD_U, b->d_u + 2 * po, 2 * ny}};
  const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
  for (const auto& f : fs) {
    if (to_handle) {
      FLB_BCUDA(b, copy_rows(b->d_sf, nx * 4, f.arr, sx * 4, nx * 4, f.rows, dd, b->stream));
      FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
      const flb_status s = flb_write_field(b->handles[c], f.field, b->d_sf, 1);  // ends with a stream sync
      if (s != FLB_OK) return bfail(b, s, flb_last_error(b->handles[c]));
    } else {
      const flb_status s = flb_read_field(b->handles[c], f.field, b->d_sf, 1);  // ends with a stream sync
      if (s != FLB_OK) return bfail(b, s, flb_last_error(b->handles[c]));
      FLB_BCUDA(b, copy_rows(f.arr, sx * 4, b->d_sf, nx * 4, nx * 4, f.rows, dd, b->stream));
      FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    }
  }
  return FLB_OK;
}

// Into the streams form with nstreams streams: the state moves into the
// handles.  At an even step only (a handle starts at t = 0, and the slot
// pattern follows the step's parity).
flb_status streams_enter(flb_batch b, int nstreams) {
  if (b->t & 1u) return bfail(b, FLB_ERR_UNSUPPORTED, "the streams form is entered at an even step");
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  const bool was = b->streams_mode;
  flb_status s = streams_setup(b, nstreams);
  if (s != FLB_OK || was) return s;
  // each handle back to t = 0 (its slot pattern then follows the batch's
  // even step), then the batch's state copied in
  for (uint32_t c = 0; c < b->n && s == FLB_OK; c++) {
    s = flb_reset(b->handles[c], b->hgeo.data() + b->off[c]);
    if (s != FLB_OK) bfail(b, s, flb_last_error(b->handles[c]));
    else s = case_state_copy(b, c, true);
  }
  if (s == FLB_OK) b->streams_mode = true;
  return s;
}

// Out of the streams form: the state moves back into the batch's arrays.
flb_status streams_leave(flb_batch b) {
  if (!b->streams_mode) return FLB_OK;
  flb_status s = FLB_OK;
  for (uint32_t c = 0; c < b->n && s == FLB_OK; c++) s = case_state_copy(b, c, false);
  if (s != FLB_OK) return s;
  // the persistent kernel takes the step's parity from the device counter,
  // which the streams form's steps did not advance
  const uint32_t t32 = (uint32_t)b->t;
  FLB_BCUDA(b, cudaMemcpyAsync(b->d_tstep, &t32, sizeof(t32), cudaMemcpyHostToDevice, b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  b->streams_mode = false;
  return FLB_OK;
}

// n steps in the streams form: every case's own step graphs on its stream,
// after the work already on the batch's stream; the batch's stream then
// waits for every stream of the pool.
flb_status streams_step(flb_batch b, uint64_t n) {
  FLB_BCUDA(b, cudaEventRecord(b->start_ev, b->stream));
  for (int k = 0; k < b->nstreams; k++) FLB_BCUDA(b, cudaStreamWaitEvent(b->pool[k], b->start_ev, 0));
  for (uint32_t c : b->sorder) {
    const flb_status s = flb_step(b->handles[c], n);
    if (s != FLB_OK) return bfail(b, s, flb_last_error(b->handles[c]));
  }
  for (int k = 0; k < b->nstreams; k++) {
    FLB_BCUDA(b, cudaEventRecord(b->pool_ev[k], b->pool[k]));
    FLB_BCUDA(b, cudaStreamWaitEvent(b->stream, b->pool_ev[k], 0));
  }
  b->t += n;
  return FLB_OK;
}

// Timed search over launch shapes: probe steps of the whole batch from the
// initial state for every candidate; the fastest wins.  Each group of CTAs
// holds one case at a time, so the number of groups sets how many bytes of
// cases are active at once: counts sized so that they fit in about half of
// the L2 let a case be stepped from L2 after its first step (the probe, 100
// steps by default, is long enough for that reuse to show).  Hardware
// clusters give the cheapest barrier but pack into the GPCs unevenly at 8 or
// 16 CTAs; teams take any number of CTAs and fill every SM.
// forms: FLB_TUNE_PERSISTENT (the persistent kernel's shapes) and / or
// FLB_TUNE_STREAMS (the streams form with 8 and 16 streams).
flb_status btune(flb_batch b, uint32_t probe_steps, int forms) {
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  int l2 = 0;
  cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, b->device);
  // bytes a case touches per step: 9 FP32 populations, flags, wall mask
  const double case_bytes = (double)b->cells / b->n * (9.0 * 4.0 + 2.0);
  const int l2_fit = std::max(1, (int)(0.5 * (double)l2 / std::max(1.0, case_bytes)));
  struct Cand {
    bool team, vec;
    int cs, clusters, threads;
    int streams;  // > 0: the streams form with that many streams
  };
  std::vector<Cand> cands;
  auto add = [&](bool team, bool vec, int cs, int k, int mx, int threads) {
    if (!(forms & FLB_TUNE_PERSISTENT)) return;
    const int cl = std::min(std::max(k, 1), std::min(mx, (int)b->n));
    for (auto& c : cands)
      if (c.team == team && c.vec == vec && c.cs == cs && c.clusters == cl && c.threads == threads) return;
    cands.push_back({team, vec, cs, cl, threads, 0});
  };
  // teams: every resident CTA, split into l2_fit/2 .. 2 l2_fit teams (on a
  // B200 the ensemble runs fastest with its active cases near l2_fit)
  auto add_teams = [&](bool vec, int threads) {
    const int R = max_team_ctas(b, threads, vec);
    for (int teams : {l2_fit / 2, (3 * l2_fit) / 4, l2_fit, (5 * l2_fit) / 4, (3 * l2_fit) / 2, 2 * l2_fit}) {
      teams = std::min(std::max(teams, 1), std::min(R, (int)b->n));
      if (R <= 0 || teams <= 0) continue;
      add(true, vec, R / teams, teams, teams, threads);
    }
  };
  for (int threads : {512, 1024}) {
    for (int cs : {1, 4, 8, 16}) {
      const int mx = max_clusters(b, cs, threads, false);
      if (mx <= 0) continue;
      const int per_sm = std::max(1, nsm / cs);
      for (int k : {l2_fit, per_sm, mx}) add(false, false, cs, k, mx, threads);
    }
    add_teams(false, threads);
  }
  // the vector data path: teams, one-CTA groups (every case of the batch at
  // once), and 8- and 16-CTA clusters at the L2-sized count
  for (int threads : {256, 512}) {
    for (int cs : {1, 8, 16}) {
      const int mx = max_clusters(b, cs, threads, true);
      if (mx <= 0) continue;
      add(false, true, cs, l2_fit, mx, threads);
      if (cs == 1) add(false, true, cs, mx, mx, threads);
    }
    add_teams(true, threads);
  }
  // the streams form: the cases' own step graphs on 8 or 16 concurrent
  // streams (more streams than hardware queues measured slower on a B200)
  if (forms & FLB_TUNE_STREAMS)
    for (int st : {8, 16}) cands.push_back({false, false, 1, 1, 0, std::min(st, kMaxStreams)});
  if (cands.empty()) return bfail(b, FLB_ERR_UNSUPPORTED, "no launch shape can run the batch");
  if (b->streams_mode) {
    flb_status s = streams_leave(b);
    if (s != FLB_OK) return s;
  }
  cudaEvent_t e0, e1;
  FLB_BCUDA(b, cudaEventCreate(&e0));
  FLB_BCUDA(b, cudaEventCreate(&e1));
  float best = 1e30f;
  Cand win = cands[0];
  flb_status s = FLB_OK;
  for (const Cand& c : cands) {
    b->streams_mode = false;
    if (c.streams > 0) {
      s = binit(b);
      if (s == FLB_OK) s = streams_enter(b, c.streams);
      if (s == FLB_OK) s = streams_step(b, 2);  // warm-up: the handles capture their graphs
      if (s == FLB_OK) {
        cudaEventRecord(e0, b->stream);
        s = streams_step(b, probe_steps);
        cudaEventRecord(e1, b->stream);
      }
      if (s == FLB_OK) FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
      b->streams_mode = false;  // the next candidate starts from the initial state again
    } else {
    b->team = c.team;
    b->vec = c.vec;
    b->cluster = c.cs;
    b->threads = c.threads;
    s = bassign(b, c.clusters);
    if (s == FLB_OK) s = binit(b);
    if (s == FLB_OK) s = blaunch(b, 2, 0);  // warm-up
    if (s == FLB_OK) {
      cudaEventRecord(e0, b->stream);
      s = blaunch(b, probe_steps, 0);
      cudaEventRecord(e1, b->stream);
    }
    }
    if (s != FLB_OK) {
      // a shape that does not launch is skipped; an error that outlives the
      // call ends the search
      cudaGetLastError();
      if (cudaStreamSynchronize(b->stream) != cudaSuccess) break;
      s = FLB_OK;
      continue;
    }
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (bcheck(b) != FLB_OK) continue;  // a barrier that gave up: not a candidate
    if (ms < best) {
      best = ms;
      win = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != FLB_OK) return s;
  FLB_BCUDA(b, cudaGetLastError());
  if (best == 1e30f) return bfail(b, FLB_ERR_CUDA, "no launch shape completed the probe steps");
  b->tuned = 1;
  if (win.streams > 0) {
    s = binit(b);
    if (s == FLB_OK) s = streams_enter(b, win.streams);  // the handles start from the initial state too
    return s;
  }
  streams_free(b);  // not chosen: the handles' memory goes back
  b->team = win.team;
  b->vec = win.vec;
  b->cluster = win.cs;
  b->threads = win.threads;
  s = bassign(b, win.clusters);
  if (s != FLB_OK) return s;
  return binit(b);
}

}  // namespace

extern "C" {

FLB_API flb_status flb_batch_create(const flb_case_desc* cases, uint32_t n, int autotune, flb_batch* out) {
  if (!out || !cases || n == 0) return FLB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::string msg;
  for (uint32_t c = 0; c < n; c++) {
    flb_status s = validate_desc(&cases[c], msg);
    if (s != FLB_OK) {
      std::fprintf(stderr, "flb_batch_create: case %u: %s\n", c, msg.c_str());
      return s;
    }
    const flb_case_desc& d = cases[c];
    if (d.free_surface || d.precision != 32 || d.bounce_back != cases[0].bounce_back ||
        d.arithmetic != cases[0].arithmetic || d.collision != cases[0].collision || d.subgrid != cases[0].subgrid) {
      std::fprintf(stderr,
                   "flb_batch_create: case %u: the batch takes single-phase FP32 cases sharing bounce-back, "
                   "arithmetic, collision and subgrid settings\n",
                   c);
      return FLB_ERR_UNSUPPORTED;
    }
    const uint64_t N = (uint64_t)d.nx * d.ny;
    for (uint64_t i = 0; i < N; i++)
      if (d.flags[i] & (kInlet | kOutlet)) {
        std::fprintf(stderr, "flb_batch_create: case %u: inlet/outlet cells are not supported in a batch\n", c);
        return FLB_ERR_UNSUPPORTED;
      }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FLB_ERR_NO_DEVICE;
  flb_batch b = new flb_batch_s();
  b->n = n;
  if (cases[0].device >= 0) b->device = cases[0].device;
  else cudaGetDevice(&b->device);
  if (b->device >= ndev) {
    delete b;
    return FLB_ERR_INVALID_ARGUMENT;
  }
  BDevice guard(b->device);
  b->hw = cases[0].bounce_back == FLB_BB_HALFWAY;
  b->fu = cases[0].arithmetic == FLB_ARITH_FUSED && cases[0].collision == FLB_COLLISION_SRT && !cases[0].subgrid;
  b->nx.resize(n);
  b->ny.resize(n);
  b->off.resize(n);
  b->poff.resize(n);
  b->sx.resize(n);
  for (uint32_t c = 0; c < n; c++) {
    b->nx[c] = cases[c].nx;
    b->ny[c] = cases[c].ny;
    b->sx[c] = (cases[c].nx + kVecCells - 1u) / kVecCells * kVecCells;
    b->off[c] = b->cells;
    b->poff[c] = b->pcells;
    b->cells += (size_t)cases[c].nx * cases[c].ny;
    b->pcells += (size_t)b->sx[c] * cases[c].ny;
    b->max_cells = std::max(b->max_cells, (size_t)cases[c].nx * cases[c].ny);
  }
  // the cases as given, for the handles of the streams form
  b->hgeo.resize(b->cells);
  b->descs.assign(cases, cases + n);
  for (uint32_t c = 0; c < n; c++) {
    std::memcpy(b->hgeo.data() + b->off[c], cases[c].flags, (size_t)cases[c].nx * cases[c].ny);
    b->descs[c].flags = b->hgeo.data() + b->off[c];
  }
  auto bail = [&](flb_status s) {
    std::fprintf(stderr, "flb_batch_create: %s\n", b->err.c_str());
    bfree(b);
    delete b;
    return s;
  };
  if (cases[0].stream) {
    b->stream = static_cast<cudaStream_t>(cases[0].stream);
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaStreamCreate"));
    b->own_stream = true;
  }
  const size_t M = b->cells, P = b->pcells, S = b->max_cells;
  struct A {
    void** p;
    size_t bytes;
    bool need;
  } allocs[] = {
      {(void**)&b->d_f, 9 * P * sizeof(float), true},         {(void**)&b->d_rho, P * sizeof(float), true},
      {(void**)&b->d_u, 2 * P * sizeof(float), true},         {(void**)&b->d_flags, P, true},
      {(void**)&b->d_geo, M, true},                           {(void**)&b->d_nbmask, P, b->hw},
      {(void**)&b->d_sf, 9 * S * sizeof(float), true},        {(void**)&b->d_srho, S * sizeof(float), true},
      {(void**)&b->d_su, 2 * S * sizeof(float), true},        {(void**)&b->d_sflags, S, true},
      {(void**)&b->d_snb, S, b->hw},
      {(void**)&b->d_tstep, 2 * sizeof(uint32_t), true},      {(void**)&b->d_cases, n * sizeof(BatchCase), true},
      {(void**)&b->d_order, n * sizeof(uint32_t), true},
      {(void**)&b->d_sync, n * sizeof(TeamSync), true},       {(void**)&b->d_err, sizeof(uint32_t), true},
  };
  for (A& a : allocs) {
    if (!a.need) continue;
    cudaError_t e = cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMalloc"));
  }
  b->hcases.resize(n);
  for (uint32_t c = 0; c < n; c++) {
    const size_t o = b->off[c], po = b->poff[c], N = (size_t)b->nx[c] * b->ny[c];
    const size_t NP = (size_t)b->sx[c] * b->ny[c];
    KParams& k = b->hcases[c].kp;
    fill_case_constants(&cases[c], k);
    k.nx = b->nx[c];
    k.ny = b->ny[c];
    k.N = (uint32_t)NP;
    k.f = b->d_f + 9 * po;
    for (int q = 0; q < 9; q++) k.slot[q] = b->d_f + 9 * po + (size_t)q * NP;
    k.rho = b->d_rho + po;
    k.u = b->d_u + 2 * po;
    k.flags = b->d_flags + po;
    k.flags_out = b->d_flags + po;
    k.nbmask = b->hw ? b->d_nbmask + po : nullptr;
    k.tstep = b->d_tstep;
    b->hcases[c].sx = b->sx[c];
    cudaError_t e = cudaMemcpyAsync(b->d_geo + o, cases[c].flags, N, cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMemcpyAsync"));
  }
  cudaError_t e = cudaMemcpyAsync(b->d_cases, b->hcases.data(), n * sizeof(BatchCase), cudaMemcpyHostToDevice,
                                  b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMemcpy"));
  flb_status s = FLB_OK;
  if (autotune) {
    s = btune(b, autotune > 1 ? (uint32_t)autotune : 100u, FLB_TUNE_PERSISTENT | FLB_TUNE_STREAMS);
  } else {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    b->cluster = 8;
    s = bassign(b, std::max(1, std::min<int>(nsm / 8, (int)n)));
    if (s == FLB_OK) s = binit(b);
  }
  if (s != FLB_OK) return bail(s);
  *out = b;
  return FLB_OK;
}

FLB_API flb_status flb_batch_step(flb_batch b, uint64_t n) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  if (b->broken)
    return bfail(b, FLB_ERR_CUDA, "a team barrier gave up waiting in an earlier launch; call flb_batch_reset");
  if (n == 0) return FLB_OK;
  BDevice g(b->device);
  if (b->streams_mode) return streams_step(b, n);
  return blaunch(b, n, 1);
}

FLB_API flb_status flb_batch_sync(flb_batch b) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return bcheck(b);
}

FLB_API flb_status flb_batch_reset(flb_batch b) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  flb_status s = binit(b);
  if (s == FLB_OK && b->streams_mode)
    for (uint32_t c = 0; c < b->n && s == FLB_OK; c++) {
      s = flb_reset(b->handles[c], b->hgeo.data() + b->off[c]);
      if (s != FLB_OK) bfail(b, s, flb_last_error(b->handles[c]));
    }
  return s;
}

FLB_API flb_status flb_batch_read_field(flb_batch b, uint32_t i, int field, void* dst, int on_device) {
  if (!b || !dst || i >= b->n) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  if (b->streams_mode) {
    if (field != FLB_FIELD_F && field != FLB_FIELD_RHO && field != FLB_FIELD_U && field != FLB_FIELD_FLAGS)
      return bfail(b, FLB_ERR_INVALID_ARGUMENT, "the batch holds populations, density, velocity and flags");
    FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
    const flb_status s = flb_read_field(b->handles[i], field, dst, on_device);
    return s == FLB_OK ? s : bfail(b, s, flb_last_error(b->handles[i]));
  }
  // the state is stored with padded rows; the copy drops the padding
  const size_t po = b->poff[i], nx = b->nx[i], ny = b->ny[i], sx = b->sx[i];
  const void* src = nullptr;
  size_t es = 4, rows = 0;
  switch (field) {
    case FLB_FIELD_F: src = b->d_f + 9 * po; rows = 9 * ny; break;
    case FLB_FIELD_RHO: src = b->d_rho + po; rows = ny; break;
    case FLB_FIELD_U: src = b->d_u + 2 * po; rows = 2 * ny; break;
    case FLB_FIELD_FLAGS: src = b->d_flags + po; rows = ny; es = 1; break;
    default: return bfail(b, FLB_ERR_INVALID_ARGUMENT, "the batch holds populations, density, velocity and flags");
  }
  FLB_BCUDA(b, copy_rows(dst, nx * es, src, sx * es, nx * es, rows,
                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return FLB_OK;
}

FLB_API flb_status flb_batch_info(flb_batch b, int64_t info[8]) {
  if (!b || !info) return FLB_ERR_INVALID_ARGUMENT;
  info[0] = b->n;
  info[1] = (int64_t)b->cells;
  info[2] = (int64_t)b->t;
  info[3] = b->cluster;
  info[4] = b->clusters;
  info[5] = b->tuned;
  info[6] = b->threads;
  info[7] = (b->team ? FLB_BATCH_TEAM : FLB_BATCH_CLUSTER) | (b->vec ? FLB_BATCH_VECTOR : 0);
  if (b->streams_mode) {
    info[3] = 1;
    info[4] = b->nstreams;
    info[6] = 0;
    info[7] = FLB_BATCH_STREAMS;
  }
  return FLB_OK;
}

FLB_API flb_status flb_batch_set_launch(flb_batch b, int mode, int group, int groups, int threads) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  if (mode == FLB_BATCH_STREAMS) {
    if (group != 1 || groups < 1 || groups > kMaxStreams)
      return bfail(b, FLB_ERR_INVALID_ARGUMENT,
                   "the streams form takes group 1 and 1 to " + std::to_string(kMaxStreams) + " streams");
    BDevice g(b->device);
    return streams_enter(b, groups);
  }
  const bool vec = (mode & FLB_BATCH_VECTOR) != 0;
  mode &= ~FLB_BATCH_VECTOR;
  if (mode != FLB_BATCH_CLUSTER && mode != FLB_BATCH_TEAM)
    return bfail(b, FLB_ERR_INVALID_ARGUMENT,
                 "mode must be FLB_BATCH_CLUSTER or FLB_BATCH_TEAM, optionally with FLB_BATCH_VECTOR, or "
                 "FLB_BATCH_STREAMS");
  const bool team = mode == FLB_BATCH_TEAM;
  if (!team && group != 1 && group != 2 && group != 4 && group != 8 && group != 16)
    return bfail(b, FLB_ERR_INVALID_ARGUMENT, "a cluster has 1, 2, 4, 8 or 16 CTAs");
  if (team && group < 1) return bfail(b, FLB_ERR_INVALID_ARGUMENT, "a team has at least one CTA");
  if (threads != 256 && threads != 512 && threads != 1024)
    return bfail(b, FLB_ERR_INVALID_ARGUMENT, "threads per CTA must be 256, 512 or 1024");
  if (vec && threads > kBatchVecMaxThreads)
    return bfail(b, FLB_ERR_INVALID_ARGUMENT, "the vector data path takes 256 or 512 threads per CTA");
  if (groups < 1 || (uint32_t)groups > b->n)
    return bfail(b, FLB_ERR_INVALID_ARGUMENT, "groups must be between 1 and the number of cases");
  BDevice g(b->device);
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));  // a running launch reads the assignment
  const int mx = max_groups(b, team, group, threads, vec);
  if (groups > mx)
    return bfail(b, FLB_ERR_UNSUPPORTED,
                 "at most " + std::to_string(mx) + " groups of this shape fit on the device at once");
  if (b->streams_mode) {
    const flb_status s = streams_leave(b);
    if (s != FLB_OK) return s;
  }
  const int pc = b->cluster, pt = b->threads;
  const bool pm = b->team, pv = b->vec;
  b->team = team;
  b->vec = vec;
  b->cluster = group;
  b->threads = threads;
  flb_status s = bassign(b, groups);
  if (s != FLB_OK) {
    b->team = pm;
    b->vec = pv;
    b->cluster = pc;
    b->threads = pt;
  }
  return s;
}

FLB_API flb_status flb_batch_tune(flb_batch b, uint32_t probe_steps, int forms) {
  if (!b || !(forms & (FLB_TUNE_PERSISTENT | FLB_TUNE_STREAMS))) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return btune(b, probe_steps ? probe_steps : 100u, forms);
}

FLB_API flb_status flb_batch_set_wait_limit(flb_batch b, uint32_t polls) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  b->wait_limit = polls == 0 ? kTeamSpinLimit : polls;
  return FLB_OK;
}

FLB_API flb_status flb_batch_destroy(flb_batch b) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  {
    BDevice g(b->device);
    cudaStreamSynchronize(b->stream);
    bfree(b);
  }
  delete b;
  return FLB_OK;
}

FLB_API const char* flb_batch_last_error(flb_batch b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
