// launch.h -- host launchers of the engine's kernels (one translation unit
// per pass family: k_init.cu, k_sc.cu, k_fs.cu, k_reduce.cu).  Each is
// instantiated for the four storage variants below.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/flowlb.h"
#include "common.cuh"

// (storage, arithmetic, mass) type triples
#define FLB_FOR_EACH_VARIANT(X) \
  X(double, double, double)     \
  X(float, float, double)       \
  X(__half, float, double)      \
  X(float, float, float)

namespace flb {

// engine.cu: descriptor checks and per-case constants shared with the batch
flb_status validate_desc(const flb_case_desc* d, std::string& msg);
void fill_case_constants(const flb_case_desc* desc, KParams& k);

// stream-collide; vec selects the V-cells-per-thread data path, fu the fused
// SRT arithmetic
template <class S, class C, class M>
void launch_sc(const KParams& kp, cudaStream_t st, uint32_t odd, bool fs, bool hw, bool wm, bool vec, bool fu);
int vec_width(int precision);
// free surface: the listed super-tiles in a persistent grid of `grid` blocks;
// vec: the vector data path (needs nx divisible by the vector width)
template <class S, class C, class M>
void launch_sc_list(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid,
                    bool fu, bool vec);
template <class S, class C, class M>
int sc_list_blocks_per_sm(bool vec);

// FS_1 (clears the next step's list lengths), its reference-mode apply, and
// FS_2..4 on listed super-tiles (appends the next step's lists)
template <class S, class C, class M>
void launch_fs1(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, const TileList& tl, uint32_t grid,
                const ListClear& lc);
template <class S, class C, class M>
void launch_apply_recon(const KParams& kp, cudaStream_t st, uint32_t odd);
template <class S, class C, class M>
int launch_fs234(const KParams& kp, cudaStream_t st, uint32_t odd, const TileList& tl, uint32_t grid, uint32_t* nz,
                 const NextLists& nl, int form);
// launch forms of the flag pass: tile width x cells per thread (threads per
// block = width * 8 / cells per thread)
enum FsForm { FS_FORM_W128X1 = 0, FS_FORM_W32 = 1, FS_FORM_W128X2 = 2, FS_FORM_W128X4 = 4, FS_FORM_W64X1 = 5,
              FS_FORM_W64X2 = 6 };
// resident blocks per SM of FS_1 (which 0) or of the flag pass in `form` (which 1)
template <class S, class C, class M>
int fs_blocks_per_sm(int which, int form);

// the free-surface step as one persistent cooperative kernel (k_fsp.cu):
// a.steps steps per launch, `grid` CTAs of 1024 threads all resident at once
template <class S, class C, class M>
cudaError_t launch_fs_persist(const KParams& p0, const KParams& p1, const FspArgs& a, uint32_t grid, bool hw, bool fu,
                              cudaStream_t st);
template <class S, class C, class M>
int fs_persist_blocks_per_sm(bool hw, bool fu);

// headless visualisation (k_viz.cu), T = the arithmetic type of u / the mass type of phi
template <class T>
void launch_viz_uv(const void* u, float* out, uint32_t N, cudaStream_t st);
template <class T>
void launch_viz_shade(const void* u, uint32_t N, int quantity, const float* cmap, uint32_t n, float vmax, float vmin,
                      uint8_t* rgba, cudaStream_t st);
template <class T>
void launch_viz_isoline(const void* f, bool vec, uint32_t nx, uint32_t ny, float iso, uint32_t width, uint32_t height,
                        const uint32_t bounds[4], uint8_t* img, cudaStream_t st);

// initial state
void launch_init_flags(const uint8_t* geo, uint8_t* flags, uint32_t nx, uint32_t ny, int free_surface, void* mass,
                       void* excess, void* phi, int mass_f64, cudaStream_t st);
void launch_nbmask(const uint8_t* geo, uint8_t* nbmask, uint32_t nx, uint32_t ny, cudaStream_t st);
void launch_plain_chunks(const uint8_t* flags, const uint8_t* nbmask, uint32_t N, uint32_t* plain, cudaStream_t st);
template <class S, class C, class M>
void launch_init_ddf(const KParams& kp, cudaStream_t st, const uint8_t* geo, bool hw);

// reductions and codecs
template <class S, class C, class M>
void launch_mass_partial(const KParams& kp, cudaStream_t st, uint32_t odd, int fs, bool hw, double* partial);
void launch_sum_partials(const double* partial, uint32_t n, double* out, cudaStream_t st);
template <class S, class C, class M>
void launch_census(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, unsigned long long* counts);
template <class S, class C, class M>
void launch_decode(const KParams& kp, cudaStream_t st, void* out);
template <class S, class C, class M>
void launch_encode(const KParams& kp, cudaStream_t st, const void* in);

}  // namespace flb
