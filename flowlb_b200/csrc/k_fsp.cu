// k_fsp.cu -- the free-surface step as one persistent kernel per run of steps.
//
// The per-pass step (k_fs.cu, k_sc.cu) launches three kernels per time step:
// FS_1, stream-collide and the flag pass (which lists the next step's
// super-tiles).  On grids whose
// live super-tiles fill the GPU about once (a few hundred on the 2048x512 dam
// break) every pass is a single round of latency-bound work, and the launch,
// ramp-up and drain of each kernel are a large part of the step.  Here one
// cooperative launch runs an even number of steps: every CTA stays resident
// (one per SM, 1024 threads, one cell per thread of a 128x8 super-tile), and
// the three passes of each step are separated by grid barriers in global
// memory instead of kernel boundaries.  The passes themselves are the same
// device code as the per-pass kernels (fs1_cell, sc_cell, fs234_super_tile),
// so both paths give identical results.
//
// The reference runs five full-grid kernels per step with a host loop around
// them (src/cuda/runCuda.cu:506-527); nothing there corresponds to the
// barriers or the lists.
#include "fs_cells.cuh"
#include "launch.h"
#include "sc_cell.cuh"

namespace flb {
namespace {

constexpr int kPBlock = 1024;

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* a) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

// Barrier of all CTAs of the grid.  *count is zero when the kernel starts and
// only grows: the k-th barrier (k = 1, 2, ...) is passed once it holds
// k * gridDim.x arrivals, so no reset is needed between barriers.  Writes of
// every CTA before the barrier are visible to every CTA after it (fence,
// arrival, acquire poll, fence, block barrier).  A wait longer than `limit`
// polls sets *err; a CTA that sees *err set (checked every 64 polls) stops
// waiting too.  Returns false on either, and the caller leaves the kernel.
// arrive = false (failure injection only) makes this CTA wait without
// arriving, so the barrier never completes and every wait runs out.
__device__ __forceinline__ bool grid_barrier(uint32_t* count, uint32_t target, uint32_t* err, uint32_t limit,
                                             bool arrive, int& ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool good = true;
    __threadfence();
    if (arrive) atomicAdd(count, 1u);
    uint32_t it = 0;
    while (ld_acquire_gpu(count) < target) {
      if (++it >= limit) {
        good = false;
        atomicOr(err, 1u);
        break;
      }
      if ((it & 63u) == 0u && ld_acquire_gpu(err) != 0u) {
        good = false;
        break;
      }
    }
    __threadfence();
    ok = good ? 1 : 0;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The next grid barrier of the launch; with a.trace set, CTA 0 records the
// time it leaves the barrier (a.trace[k] for the k-th barrier, a.trace[0] the
// start of the launch), so the phases of the production kernel can be timed.
__device__ __forceinline__ bool next_barrier(const FspArgs& a, uint32_t& nbar, int& ok) {
  ++nbar;
  const bool good = grid_barrier(a.bar, nbar * gridDim.x, a.err, a.wait_limit, blockIdx.x != a.skip_cta, ok);
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0) a.trace[nbar] = global_ns();
  return good;
}

// One time step with parity ODD (p: the step's parameters, its flag buffers
// in the order of that parity).  Returns false when a barrier gave up.
template <class S, class C, class M, bool HW, bool FU, bool ODD>
__device__ __forceinline__ bool fsp_step(const KParams& p, const FspArgs& a, FlagMasks<128>& sm, uint32_t* wact_sm,
                                         uint32_t& nbar, int& ok) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t row = warp % kSTH, xo = (warp / kSTH) * 32u + lane;  // this thread's cell of a super-tile
  const uint32_t G = gridDim.x;
  const uint32_t* lsc = a.list[ODD][0];
  const uint32_t* lfs = a.list[ODD][1];
  // lengths of this step's lists (built by the previous step)
  const uint32_t T = a.nsx * a.nsy;
  const uint32_t nsc = min(__ldcg(a.lcount + 2 * ODD), T);
  const uint32_t nfs = a.fs_all ? T : min(__ldcg(a.lcount + 2 * ODD + 1), T);
  // the next step's list lengths and marks, which this step's flag pass
  // appends to (the previous step's passes have finished reading them)
  clear_next_lists(ListClear{a.lcount + 2 * (ODD ^ 1), a.lbits + (ODD ^ 1) * a.nwords, a.nwords});
  // FS_1: mass exchange and gas reconstruction
  for (uint32_t i = blockIdx.x; i < nsc; i += G) {
    const uint32_t t = __ldcg(lsc + i);
    const uint32_t y = (t / a.nsx) * kSTH + row, x = (t % a.nsx) * kSTW + xo;
    if (y < p.ny && x < p.nx) fs1_cell<S, C, M, HW, ODD>(p, x, y);
  }
  if (!next_barrier(a, nbar, ok)) return false;
  // stream-collide
  for (uint32_t i = blockIdx.x; i < nsc; i += G) {
    const uint32_t t = __ldcg(lsc + i);
    const uint32_t y = (t / a.nsx) * kSTH + row, x = (t % a.nsx) * kSTW + xo;
    if (y < p.ny && x < p.nx) sc_cell<S, C, M, true, HW, true, ODD, FU>(p, x, y);
  }
  if (!next_barrier(a, nbar, ok)) return false;
  // FS_2..4: flag stencil, mass / excess / fill level, activity words and the
  // next step's lists
  const NextLists nl{a.list[ODD ^ 1][0], a.list[ODD ^ 1][1], a.lcount + 2 * (ODD ^ 1), a.lbits + (ODD ^ 1) * a.nwords,
                     a.nsx, a.nsy};
  for (uint32_t i = blockIdx.x; i < nfs; i += G)
    fs234_super_tile<S, C, M, ODD, 128>(p, a.fs_all ? i : __ldcg(lfs + i), a.nsx, a.nz, nl, sm, wact_sm);
  return next_barrier(a, nbar, ok);
}

// a.steps steps (even) from an even t with flag buffer 0 current: p0 holds the
// parameters of the even steps (flags = buffer 0, flags_out = buffer 1), p1
// those of the odd steps (swapped).
template <class S, class C, class M, bool HW, bool FU>
__global__ void __launch_bounds__(kPBlock, 1) k_fs_persist(const __grid_constant__ KParams p0,
                                                          const __grid_constant__ KParams p1,
                                                          const __grid_constant__ FspArgs a) {
  __shared__ FlagMasks<128> sm;
  __shared__ uint32_t wact_sm[kPBlock / 32];
  __shared__ int ok;
  // a barrier of an earlier launch gave up: the state is undefined until the
  // host resets it, so nothing runs
  if (threadIdx.x == 0) ok = __ldcg(a.err) == 0u ? 1 : 0;
  __syncthreads();
  if (!ok) return;
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0) a.trace[0] = global_ns();
  uint32_t nbar = 0;
  for (uint32_t s = 0; s < a.steps; s += 2) {
    if (!fsp_step<S, C, M, HW, FU, false>(p0, a, sm, wact_sm, nbar, ok)) return;
    if (!fsp_step<S, C, M, HW, FU, true>(p1, a, sm, wact_sm, nbar, ok)) return;
  }
}

template <class S, class C, class M>
using FspKernel = void (*)(const KParams, const KParams, const FspArgs);

template <class S, class C, class M>
FspKernel<S, C, M> pick_fsp(bool hw, bool fu) {
  if (hw) return fu ? k_fs_persist<S, C, M, true, true> : k_fs_persist<S, C, M, true, false>;
  return fu ? k_fs_persist<S, C, M, false, true> : k_fs_persist<S, C, M, false, false>;
}

}  // namespace

template <class S, class C, class M>
cudaError_t launch_fs_persist(const KParams& p0, const KParams& p1, const FspArgs& a, uint32_t grid, bool hw, bool fu,
                              cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kPBlock);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  // every CTA resident at once: the grid barriers wait for one another
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, pick_fsp<S, C, M>(hw, fu), p0, p1, a);
}

template <class S, class C, class M>
int fs_persist_blocks_per_sm(bool hw, bool fu) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pick_fsp<S, C, M>(hw, fu), kPBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

#define FLB_INSTANTIATE(S, C, M)                                                                          \
  template cudaError_t launch_fs_persist<S, C, M>(const KParams&, const KParams&, const FspArgs&, uint32_t, \
                                                  bool, bool, cudaStream_t);                              \
  template int fs_persist_blocks_per_sm<S, C, M>(bool, bool);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
