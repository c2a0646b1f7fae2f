// k_fs.cu -- the free-surface passes as separate kernels: FS_1
// (lbmKernel2D.cu:14-121) and FS_2, FS_3, FS_4 fused into one shared-memory
// flag-stencil kernel (lbmKernel2D.cu:124-303) that also lists the next
// step's super-tiles.  The per-cell and per-tile code is in fs_cells.cuh.
// Templated on the step parity.
#include "fs_cells.cuh"
#include "launch.h"

namespace flb {

// FS_1 on the listed super-tiles, one row of a super-tile per warp.
// FS_1 blocks: kFs1Block threads (512: two cells per thread and super-tile,
// x and x + 64 of a row; 1024: one cell per thread), FLB_FS1_MIN_BLOCKS per
// SM.  Measured on a B200 (dam break, step time at 2048x512 / FS_1 time at
// 8192x2048): 512 threads, two blocks per SM (64 registers) 28.4 / 83 us;
// 1024 threads at 32 registers 33.3 / 103 us and at 64 registers 29.8 /
// 93 us; 512 threads at 40 registers 33.1 / 90 us (the spills cost more than
// the added warps gain).
#ifndef FLB_FS1_BLOCK
#define FLB_FS1_BLOCK 512
#endif
#ifndef FLB_FS1_MIN_BLOCKS
#define FLB_FS1_MIN_BLOCKS 2
#endif
constexpr int kFs1Block = FLB_FS1_BLOCK;
// lc: the next step's list lengths and marks, cleared here for this step's
// flag pass.
template <class S, class C, class M, bool HW, bool ODD>
__global__ void __launch_bounds__(kFs1Block, FLB_FS1_MIN_BLOCKS) k_fs1(const __grid_constant__ KParams p,
                                                                       const TileList tl, const ListClear lc) {
  pdl_wait();
  pdl_trigger();
  clear_next_lists(lc);
  constexpr uint32_t kCpr = kFs1Block / 32 / kSTH;     // warps per row of a super-tile
  constexpr uint32_t kCells = kSTW / (32u * kCpr);     // cells per thread and super-tile
  static_assert(kCells * 32u * kCpr == kSTW && kCells <= 2u, "FS_1: one or two cells per thread and super-tile");
  static_assert(kFs1Block >= 118, "FS_1: prefetch_super_tile needs 118 threads");
  const uint32_t n = tile_count(tl);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t row = warp % kSTH, chunk = warp / kSTH;
  const uint32_t nx = p.nx;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t t = tile_at(tl, i);
    // the block's next super-tile into L2 while this one is worked on
    if (i + gridDim.x < n) prefetch_super_tile(p, tile_at(tl, i + gridDim.x), tl.nsx, sizeof(S), true, sizeof(M));
    const uint32_t y = (t / tl.nsx) * kSTH + row;
    if (y >= p.ny) continue;
    const uint32_t xa = (t % tl.nsx) * kSTW + chunk * 32u + lane, xc = xa + 32u * kCpr;
    // the cells' flags and wall masks first: one round trip for both
    uint8_t fa = kGas, fc = kGas;
    uint32_t ma = 0, mc = 0;
    if (xa < nx) {
      fa = p.flags[xa + y * nx];
      if (HW) ma = p.nbmask[xa + y * nx];
    }
    if (kCells == 2u && xc < nx) {
      fc = p.flags[xc + y * nx];
      if (HW) mc = p.nbmask[xc + y * nx];
    }
    if (xa < nx) fs1_cell<S, C, M, HW, ODD>(p, xa, y, fa, ma);
    if (kCells == 2u && xc < nx) fs1_cell<S, C, M, HW, ODD>(p, xc, y, fc, mc);
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

// The listed super-tiles: each block runs the flag pass on a super-tile,
// records its activity word in nz and appends to the next step's lists.
// TW x 8 tiles, CPT cells per thread.
template <int TW, int CPT>
constexpr int fs234_min_blocks() {
  return TW == 128  ? (CPT == 1 ? FLB_FS_WIDE_MIN_BLOCKS : CPT == 2 ? FLB_FS_HALF_MIN_BLOCKS : FLB_FS_QUARTER_MIN_BLOCKS)
         : TW == 64 ? (CPT == 1 ? FLB_FS_W64_MIN_BLOCKS : FLB_FS_W64X2_MIN_BLOCKS)
                    : 6;
}
template <class S, class C, class M, bool ODD, int TW, int CPT>
__global__ void __launch_bounds__(TW* kTY / CPT, fs234_min_blocks<TW, CPT>())
    k_fs234(const __grid_constant__ KParams p, const TileList tl, uint32_t* __restrict__ nz, const NextLists nl) {
  __shared__ FlagMasks<TW> sm;
  __shared__ uint32_t wact_sm[TW * kTY / CPT / 32];
  // the list was built by the previous step (FS_1 waited for it), so it is
  // read before waiting for stream-collide, whose flags the pass needs
  const uint32_t n = tile_count(tl);
  pdl_wait();
  pdl_trigger();
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
    fs234_super_tile<S, C, M, ODD, TW, CPT>(p, tile_at(tl, i), tl.nsx, nz, nl, sm, wact_sm);
}

// ---- launchers -------------------------------------------------------------------
template <class S, class C, class M>
void launch_fs1(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid,
                const ListClear& lc) {
  if (hw) {
    if (odd) launch_pdl(k_fs1<S, C, M, true, true>, grid, kFs1Block, st, kp, tl, lc);
    else launch_pdl(k_fs1<S, C, M, true, false>, grid, kFs1Block, st, kp, tl, lc);
  } else {
    if (odd) launch_pdl(k_fs1<S, C, M, false, true>, grid, kFs1Block, st, kp, tl, lc);
    else launch_pdl(k_fs1<S, C, M, false, false>, grid, kFs1Block, st, kp, tl, lc);
  }
}

template <class S, class C, class M>
void launch_apply_recon(const KParams& kp, cudaStream_t st, uint32_t odd) {
  k_apply_recon<S, C><<<dim3((kp.nx + kBlock - 1) / kBlock, kp.ny), kBlock, 0, st>>>(kp, odd);
}

// The flag pass, which also lists the next step's super-tiles, in one of its
// launch forms (FsForm: tile width and cells per thread).  On grids of up to
// kWideTiles super-tiles it is launched so that it may start while
// stream-collide drains (programmatic dependent launch); above, with an
// ordinary launch (measured faster on the 8192x2048 dam break).  Returns the
// number of kernels launched.
template <class S, class C, class M, int TW, int CPT>
void launch_fs234_form(const KParams& kp, cudaStream_t st, uint32_t odd, const TileList& tl, uint32_t grid,
                       uint32_t* nz, const NextLists& nl) {
  constexpr int threads = TW * kTY / CPT;
  if (tl.ntiles <= kWideTiles) {
    if (odd) launch_pdl(k_fs234<S, C, M, true, TW, CPT>, grid, threads, st, kp, tl, nz, nl);
    else launch_pdl(k_fs234<S, C, M, false, TW, CPT>, grid, threads, st, kp, tl, nz, nl);
  } else {
    if (odd) k_fs234<S, C, M, true, TW, CPT><<<grid, threads, 0, st>>>(kp, tl, nz, nl);
    else k_fs234<S, C, M, false, TW, CPT><<<grid, threads, 0, st>>>(kp, tl, nz, nl);
  }
}

template <class S, class C, class M>
int launch_fs234(const KParams& kp, cudaStream_t st, uint32_t odd, const TileList& tl, uint32_t grid, uint32_t* nz,
                 const NextLists& nl, int form) {
  switch (form) {
    case FS_FORM_W32: launch_fs234_form<S, C, M, 32, 1>(kp, st, odd, tl, grid, nz, nl); break;
    case FS_FORM_W128X2: launch_fs234_form<S, C, M, 128, 2>(kp, st, odd, tl, grid, nz, nl); break;
    case FS_FORM_W128X4: launch_fs234_form<S, C, M, 128, 4>(kp, st, odd, tl, grid, nz, nl); break;
    case FS_FORM_W64X1: launch_fs234_form<S, C, M, 64, 1>(kp, st, odd, tl, grid, nz, nl); break;
    case FS_FORM_W64X2: launch_fs234_form<S, C, M, 64, 2>(kp, st, odd, tl, grid, nz, nl); break;
    default: launch_fs234_form<S, C, M, 128, 1>(kp, st, odd, tl, grid, nz, nl); break;
  }
  return 1;
}

// Resident blocks per SM of FS_1 (which 0) or of the flag pass in the given
// form (which 1).
template <class S, class C, class M, int TW, int CPT>
int fs234_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fs234<S, C, M, false, TW, CPT>, TW * kTY / CPT, 0);
  return n;
}
template <class S, class C, class M>
int fs_blocks_per_sm(int which, int form) {
  int n = 0;
  if (which == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fs1<S, C, M, true, false>, kFs1Block, 0);
  else if (form == FS_FORM_W32) n = fs234_blocks_per_sm<S, C, M, 32, 1>();
  else if (form == FS_FORM_W128X2) n = fs234_blocks_per_sm<S, C, M, 128, 2>();
  else if (form == FS_FORM_W128X4) n = fs234_blocks_per_sm<S, C, M, 128, 4>();
  else if (form == FS_FORM_W64X1) n = fs234_blocks_per_sm<S, C, M, 64, 1>();
  else if (form == FS_FORM_W64X2) n = fs234_blocks_per_sm<S, C, M, 64, 2>();
  else n = fs234_blocks_per_sm<S, C, M, 128, 1>();
  return n > 0 ? n : 1;
}

#define FLB_INSTANTIATE(S, C, M)                                                                                  \
  template void launch_fs1<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, const TileList&, uint32_t,       \
                                    const ListClear&);                                                          \
  template void launch_apply_recon<S, C, M>(const KParams&, cudaStream_t, uint32_t);                             \
  template int launch_fs234<S, C, M>(const KParams&, cudaStream_t, uint32_t, const TileList&, uint32_t, uint32_t*,   \
                                     const NextLists&, int);                                                     \
  template int fs_blocks_per_sm<S, C, M>(int, int);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
