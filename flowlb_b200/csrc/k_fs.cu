// k_fs.cu -- the free-surface passes as separate kernels: FS_1
// (lbmKernel2D.cu:14-121), FS_2, FS_3, FS_4 fused into one shared-memory
// flag-stencil kernel (lbmKernel2D.cu:124-303), and the list build.  The
// per-cell and per-tile code is in fs_cells.cuh.  Templated on the step parity.
#include "fs_cells.cuh"
#include "launch.h"

namespace flb {

// FS_1 on the listed super-tiles, one row of a super-tile per warp.
// FS_1 blocks: 512 threads, two per SM at 64 registers, so that a step's
// listed super-tiles (a few hundred on a 2048x512 dam break) run in one wave.
constexpr int kFs1Block = 512;
template <class S, class C, class M, bool HW, bool ODD>
__global__ void __launch_bounds__(kFs1Block, 2) k_fs1(const __grid_constant__ KParams p,
                                                                       const TileList tl) {
  pdl_wait();
  pdl_trigger();
  const uint32_t n = tile_count(tl);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = warp % kSTH, chunk = warp / kSTH, cpr = (blockDim.x >> 5) / kSTH;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t t = tile_at(tl, i);
    const uint32_t y = (t / tl.nsx) * kSTH + row;
    if (y >= p.ny) continue;
    const uint32_t xb = (t % tl.nsx) * kSTW + lane;
#pragma unroll 1
    for (uint32_t j = chunk * 32u; j < kSTW; j += 32u * cpr)
      if (xb + j < p.nx) fs1_cell<S, C, M, HW, ODD>(p, xb + j, y);
  }
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
  const C* rec = static_cast<const C*>(p.recon);
#pragma unroll
  for (int i = 1; i < 9; i += 2) {
    const int a = odd ? i : i + 1, b = odd ? i + 1 : i;
    if ((m >> (i - 1)) & 1u) Codec<S, C>::st(slotp<S>(p, a), idx, i, rec[(uint32_t)(i - 1) * N + idx], p.f16_scale);
    if ((m >> i) & 1u) Codec<S, C>::st(slotp<S>(p, b), nb[i], i + 1, rec[(uint32_t)i * N + idx], p.f16_scale);
  }
  p.recon_mask[idx] = 0;
}

// The listed super-tiles: each block runs the flag pass on a super-tile and
// records its activity word in nz.
template <class S, class C, class M, bool ODD, int TW>
__global__ void __launch_bounds__(TW* kTY, TW == 128 ? FLB_FS_WIDE_MIN_BLOCKS : 6)
    k_fs234(const __grid_constant__ KParams p, const TileList tl, uint32_t* __restrict__ nz) {
  __shared__ FlagMasks<TW> sm;
  __shared__ uint32_t wact_sm[TW * kTY / 32];
  // the list was built by the previous step (FS_1 waited for it), so it is
  // read before waiting for stream-collide, whose flags the pass needs
  const uint32_t n = tile_count(tl);
  pdl_wait();
  pdl_trigger();
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
    fs234_super_tile<S, C, M, ODD, TW>(p, tile_at(tl, i), tl.nsx, nz, sm, wact_sm);
}

// Compacts the super-tiles for the next step: FS_1 and stream-collide visit
// super-tiles holding fluid or interface cells; the flag pass also visits a
// neighbour of such a super-tile when one of those cells lies within the
// chain's reach (3 cells) of their shared edge or corner, and, once more,
// super-tiles that held such cells a step earlier (their converted gas cells
// still clear excess mass and the flag buffers re-synchronise).  Appends with
// one atomic per warp; list order does not affect results.
// The lengths it appends to (counts) start at zero: each build zeroes the
// other parity's lengths (other_counts), which this step's passes have
// finished reading and the next step's build appends to.
__global__ void k_build_lists(const uint32_t* __restrict__ nz, uint32_t* __restrict__ nz_prev, uint32_t nsx,
                              uint32_t nsy, int prev_unknown, uint32_t* __restrict__ list_sc,
                              uint32_t* __restrict__ list_fs, uint32_t* __restrict__ counts,
                              uint32_t* __restrict__ other_counts) {
  pdl_wait();
  pdl_trigger();
  const uint32_t T = nsx * nsy;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    other_counts[0] = 0;
    other_counts[1] = 0;
  }
  bool sc = false, fs = false;
  if (t < T) list_flags(nz, nz_prev, nsx, nsy, prev_unknown, t, sc, fs);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t bsc = __ballot_sync(0xffffffffu, sc), bfs = __ballot_sync(0xffffffffu, fs);
  uint32_t base_sc = 0, base_fs = 0;
  if (lane == 0) {
    if (bsc) base_sc = atomicAdd(&counts[0], (uint32_t)__popc(bsc));
    if (bfs) base_fs = atomicAdd(&counts[1], (uint32_t)__popc(bfs));
  }
  base_sc = __shfl_sync(0xffffffffu, base_sc, 0);
  base_fs = __shfl_sync(0xffffffffu, base_fs, 0);
  const uint32_t below = (1u << lane) - 1u;
  // a list holds at most T entries (the lengths start at zero; the bound only
  // matters after a launch that gave up part-way)
  const uint32_t ksc = base_sc + __popc(bsc & below), kfs = base_fs + __popc(bfs & below);
  if (sc && ksc < T) list_sc[ksc] = t;
  if (fs && kfs < T) list_fs[kfs] = t;
}

// ---- launchers -------------------------------------------------------------------
template <class S, class C, class M>
void launch_fs1(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid) {
  if (hw) {
    if (odd) launch_pdl(k_fs1<S, C, M, true, true>, grid, kFs1Block, st, kp, tl);
    else launch_pdl(k_fs1<S, C, M, true, false>, grid, kFs1Block, st, kp, tl);
  } else {
    if (odd) launch_pdl(k_fs1<S, C, M, false, true>, grid, kFs1Block, st, kp, tl);
    else launch_pdl(k_fs1<S, C, M, false, false>, grid, kFs1Block, st, kp, tl);
  }
}

template <class S, class C, class M>
void launch_apply_recon(const KParams& kp, cudaStream_t st, uint32_t odd) {
  k_apply_recon<S, C><<<dim3((kp.nx + kBlock - 1) / kBlock, kp.ny), kBlock, 0, st>>>(kp, odd);
}

// The flag pass and the list build of the next step.  On grids of up to
// kWideTiles super-tiles both are launched so that each may start while its
// predecessor drains (measured on the 2048x512 dam break: 28.4 instead of 30.2
// us per step with the build in the flag pass's last block); above, with
// ordinary launches (measured faster on the 8192x2048 one).  Returns the
// number of kernels launched.
template <class S, class C, class M>
int launch_fs234(const KParams& kp, cudaStream_t st, uint32_t odd, const TileList& tl, uint32_t grid, uint32_t* nz,
                 const ListBuild& lb) {
  const uint32_t T = lb.nsx * lb.nsy;
  if (tl.ntiles <= kWideTiles) {
    if (odd) launch_pdl(k_fs234<S, C, M, true, 128>, grid, 128 * kTY, st, kp, tl, nz);
    else launch_pdl(k_fs234<S, C, M, false, 128>, grid, 128 * kTY, st, kp, tl, nz);
    launch_pdl(k_build_lists, dim3((T + kBlock - 1) / kBlock), dim3(kBlock), st, (const uint32_t*)nz, lb.nz_prev,
               lb.nsx, lb.nsy, lb.prev_unknown, lb.list_sc, lb.list_fs, lb.counts, lb.other_counts);
    return 2;
  }
  if (odd) k_fs234<S, C, M, true, 32><<<grid, 32 * kTY, 0, st>>>(kp, tl, nz);
  else k_fs234<S, C, M, false, 32><<<grid, 32 * kTY, 0, st>>>(kp, tl, nz);
  k_build_lists<<<(T + kBlock - 1) / kBlock, kBlock, 0, st>>>(nz, lb.nz_prev, lb.nsx, lb.nsy, lb.prev_unknown,
                                                              lb.list_sc, lb.list_fs, lb.counts, lb.other_counts);
  return 2;
}

template <class S, class C, class M>
int fs_blocks_per_sm(int which) {
  int n = 0;
  if (which == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fs1<S, C, M, true, false>, kFs1Block, 0);
  else if (which == 1)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fs234<S, C, M, false, 128>, 128 * kTY, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fs234<S, C, M, false, 32>, 32 * kTY, 0);
  return n > 0 ? n : 1;
}

#define FLB_INSTANTIATE(S, C, M)                                                                                  \
  template void launch_fs1<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, const TileList&, uint32_t);     \
  template void launch_apply_recon<S, C, M>(const KParams&, cudaStream_t, uint32_t);                             \
  template int launch_fs234<S, C, M>(const KParams&, cudaStream_t, uint32_t, const TileList&, uint32_t, uint32_t*,   \
                                     const ListBuild&);                                                          \
  template int fs_blocks_per_sm<S, C, M>(int);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
