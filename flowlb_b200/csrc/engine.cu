// engine.cu -- host side of the engine behind the C ABI of include/flowlb.h.
//
// Owns the device state of one case, issues the step passes on one stream and
// replays steady runs of steps from captured CUDA graphs.  The reference's
// counterpart is src/cuda/runCuda.cu (h_launchCudaCalculations2D and the
// headless loops :460-528) plus src/cuda/cudaInitData.* (constants and
// buffers).  Differences by design: parameters travel by value in the kernel
// argument block instead of mutable __constant__ symbols, errors come back as
// status codes instead of exit(), and there is no per-step host sync.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/flowlb.h"
#include "launch.h"

using namespace flb;

namespace {

enum Variant { V_F64 = 0, V_F32 = 1, V_F16S = 2, V_F32M32 = 3 };

constexpr int kGraphPairs = 16;  // steps per large graph = 2 * kGraphPairs
// FLB_STEP_AUTO runs the free-surface step as one persistent kernel on grids of
// up to this many super-tiles.  Measured on a B200 (2048x512 dam break, 1024
// super-tiles): 34.8 us per step persistent against 29.3 us for the PDL-chained
// per-pass kernels.  FS_1 needs 64 registers, so the persistent kernel keeps
// 1024 threads per SM where the per-pass stream-collide and flag kernels keep
// 2048, and each of its four grid barriers per step costs about 1.5 us; AUTO
// therefore runs the per-pass kernels everywhere (0 super-tiles).
constexpr uint32_t kPersistAutoTiles = 0;
constexpr uint32_t kPersistWaitLimit = 1u << 22;  // barrier polls before the persistent step gives up

struct GraphSlot {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;
};

}  // namespace

struct flb_engine {
  flb_case_desc desc{};
  Variant variant = V_F32;
  uint32_t nx = 0, ny = 0, N = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t s_size = 4, c_size = 4, m_size = 8;
  bool fs = false, hw = false, has_io = false;
  bool use_vec = false;       // vectorised stream-collide (single phase)
  bool use_vec_list = false;  // vectorised listed stream-collide (free surface)
  int fs_form = FS_FORM_W128X1;  // launch form of the flag pass (FsForm)
  bool fused = false;    // fused SRT arithmetic in stream-collide
  uint64_t t = 0;
  uint64_t launches = 0;
  int cur = 0;  // index of the current flag buffer (free surface)
  // the other flag buffer holds the previous step's post-stream-collide flags
  // and the mass fields follow from full steps (enables write skipping)
  bool trust = false;
  // free surface: super-tile activity bitmaps and the lists of the next step
  uint32_t nsx = 0, nsy = 0, ntiles = 0;
  uint32_t* d_nz = nullptr;       // super-tile activity words of the last flag pass that visited each
  uint32_t* d_lbits = nullptr;    // [step parity][nwords]: marks of the flag-pass lists
  uint32_t nwords = 0;
  uint32_t* d_list[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [step parity][0 FS_1/SC, 1 flag pass]
  uint32_t* d_lcount = nullptr;   // [step parity][2] list lengths
  bool lists_valid = false;       // lists of the current parity were built by the previous step
  // the previous step visited every super-tile: this step's flag pass must
  // too (the activity words of two steps back are unknown)
  bool fs_all_next = false;
  bool thin_tiles = false;        // a last super-tile column or row narrower than the flag pass's reach
  uint32_t grid_sc = 0, grid_fs1 = 0, grid_fs234 = 0;
  // persistent free-surface step (k_fsp.cu): requested mode, resolved path,
  // resident grid, barrier count and error word
  int step_mode = FLB_STEP_AUTO;
  bool persist = false;
  uint32_t grid_persist = 0;
  uint32_t wait_limit = kPersistWaitLimit;
  uint32_t g_skip = 0xffffffffu;  // failure injection the captured graphs were built with
  uint32_t* d_bar = nullptr;
  uint32_t* d_perr = nullptr;
  // a barrier of the persistent step gave up: the state is undefined and
  // stepping is refused until flb_reset
  bool broken = false;
  KParams kp{};
  // device buffers
  void* d_f = nullptr;
  void* d_rho = nullptr;
  void* d_u = nullptr;
  uint8_t* d_flags[2] = {nullptr, nullptr};
  uint8_t* d_geo = nullptr;
  uint8_t* d_nbmask = nullptr;
  void* d_mass = nullptr;
  void* d_excess = nullptr;
  void* d_phi = nullptr;
  void* d_recon = nullptr;
  uint8_t* d_recon_mask = nullptr;
  void* d_rho_snap = nullptr;
  void* d_u_snap = nullptr;
  double* d_partial = nullptr;
  double* d_scalar = nullptr;
  unsigned long long* d_counts = nullptr;
  uint32_t* d_tstep = nullptr;  // [2] time step by parity (FP16S stochastic rounding)
  uint32_t* d_plain = nullptr;  // single phase: plain-fluid chunk map (k_plain_chunks)
  GraphSlot g_pair, g_big;
  std::string err;
};

namespace {

const char* kStatusText[] = {"ok",          "invalid argument", "CUDA error", "out of memory",
                             "unsupported", "I/O error",        "non-finite populations", "no CUDA device"};

flb_status fail(flb_handle h, flb_status s, const std::string& msg) {
  if (h) h->err = msg;
  return s;
}

flb_status cuda_fail(flb_handle h, cudaError_t e, const char* what) {
  const flb_status s = e == cudaErrorMemoryAllocation ? FLB_ERR_OUT_OF_MEMORY : FLB_ERR_CUDA;
  return fail(h, s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FLB_CUDA(h, call)                                          \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call);       \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int now = -1;
    cudaGetDevice(&now);
    if (prev >= 0 && now != prev) cudaSetDevice(prev);
  }
};


// ---- per-variant launchers ------------------------------------------------
template <class S, class C, class M>
struct Ops {
  static void sc(flb_engine* h, uint32_t odd, bool wm) {
    launch_sc<S, C, M>(h->kp, h->stream, odd, h->fs, h->hw, wm, h->use_vec, h->fused);
  }
  static void sc_list(flb_engine* h, uint32_t odd, const TileList& tl) {
    launch_sc_list<S, C, M>(h->kp, h->stream, odd, h->hw, tl, h->grid_sc, h->fused, h->use_vec_list);
  }
  static void fs1(flb_engine* h, uint32_t odd, const TileList& tl, const ListClear& lc) {
    launch_fs1<S, C, M>(h->kp, h->stream, odd, h->hw, tl, h->grid_fs1, lc);
  }
  static int fs234(flb_engine* h, uint32_t odd, const TileList& tl, const NextLists& nl) {
    return launch_fs234<S, C, M>(h->kp, h->stream, odd, tl, h->grid_fs234, h->d_nz, nl, h->fs_form);
  }
  static void grids(flb_engine* h, int nsm) {
    h->grid_sc = (uint32_t)(nsm * sc_list_blocks_per_sm<S, C, M>(h->use_vec_list));
    h->grid_fs1 = (uint32_t)(nsm * fs_blocks_per_sm<S, C, M>(0, 0));
    h->grid_fs234 = (uint32_t)(nsm * fs_blocks_per_sm<S, C, M>(1, h->fs_form));
  }
  static void apply_recon(flb_engine* h, uint32_t odd) { launch_apply_recon<S, C, M>(h->kp, h->stream, odd); }
  static cudaError_t persist(flb_engine* h, const KParams& p0, const KParams& p1, const FspArgs& a) {
    return launch_fs_persist<S, C, M>(p0, p1, a, h->grid_persist, h->hw, h->fused, h->stream);
  }
  static int persist_blocks(flb_engine* h) { return fs_persist_blocks_per_sm<S, C, M>(h->hw, h->fused); }
  static void init_ddf(flb_engine* h) { launch_init_ddf<S, C, M>(h->kp, h->stream, h->d_geo, h->hw); }
  static void mass_partial(flb_engine* h, uint32_t odd) {
    launch_mass_partial<S, C, M>(h->kp, h->stream, odd, h->fs ? 1 : 0, h->hw, h->d_partial);
  }
  static void census(flb_engine* h, uint32_t odd) {
    launch_census<S, C, M>(h->kp, h->stream, odd, h->hw, h->d_counts);
  }
  static void decode(flb_engine* h, void* out) { launch_decode<S, C, M>(h->kp, h->stream, out); }
  static void encode(flb_engine* h, const void* in) { launch_encode<S, C, M>(h->kp, h->stream, in); }
};

template <class Fn>
void dispatch(flb_engine* h, Fn&& fn) {
  switch (h->variant) {
    case V_F64: fn(Ops<double, double, double>{}); break;
    case V_F32: fn(Ops<float, float, double>{}); break;
    case V_F16S: fn(Ops<__half, float, double>{}); break;
    case V_F32M32: fn(Ops<float, float, float>{}); break;
  }
}

void refresh_params(flb_engine* h) {
  KParams& k = h->kp;
  k.nx = h->nx;
  k.ny = h->ny;
  k.N = h->N;
  k.f = h->d_f;
  for (int q = 0; q < 9; q++) k.slot[q] = static_cast<char*>(h->d_f) + (size_t)q * h->N * h->s_size;
  k.rho = h->d_rho;
  k.u = h->d_u;
  k.flags = h->d_flags[h->cur];
  k.flags_out = h->d_flags[h->cur ^ 1];
  k.nbmask = h->d_nbmask;
  k.mass = h->d_mass;
  k.excess = h->d_excess;
  k.phi = h->d_phi;
  k.recon = h->d_recon;
  k.recon_mask = h->d_recon_mask;
  k.rho_snap = h->d_rho_snap;
  k.u_snap = h->d_u_snap;
  k.has_io = h->has_io ? 1 : 0;
  k.tstep = h->d_tstep;
  k.plain = h->d_plain;
}

// Rebuilds the single-phase plain-fluid chunk map from the current flags.
void refresh_plain(flb_engine* h) {
  if (h->fs || !h->d_plain) return;
  launch_plain_chunks(h->d_flags[h->cur], h->hw ? h->d_nbmask : nullptr, h->N, h->d_plain, h->stream);
  h->launches++;
}

// Sets the device time-step counter to t (its parity slot).
flb_status set_tstep(flb_engine* h) {
  const uint32_t t32 = (uint32_t)h->t;
  FLB_CUDA(h, cudaMemcpyAsync(h->d_tstep + (h->t & 1u), &t32, sizeof(t32), cudaMemcpyHostToDevice, h->stream));
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

// Super-tile lists consumed by the step at t (built by the step before) and the
// buffers the step fills for t+1.  Without valid lists every super-tile is visited.
struct FsLists {
  TileList sc, fs;
  uint32_t* next_count;
  bool all;
};

// A live cell can reach past a super-tile narrower than 3 cells into the one
// beyond it; such grids visit every super-tile in the flag pass.
FsLists fs_lists(flb_engine* h, uint64_t t) {
  const int lp = (int)(t & 1u);
  FsLists L;
  L.all = !h->lists_valid;
  const bool fs_all = L.all || h->fs_all_next || h->thin_tiles;
  L.sc = TileList{h->d_list[lp][0], h->d_lcount + 2 * lp, h->ntiles, h->nsx, L.all ? 1 : 0};
  L.fs = TileList{h->d_list[lp][1], h->d_lcount + 2 * lp + 1, h->ntiles, h->nsx, fs_all ? 1 : 0};
  L.next_count = h->d_lcount + 2 * (lp ^ 1);
  return L;
}

// The next step's lists, which the flag pass of the step at t appends to
// and FS_1 of that step clears.
NextLists next_lists(flb_engine* h, uint64_t t) {
  const int np = (int)((t + 1) & 1u);
  return NextLists{h->d_list[np][0], h->d_list[np][1], h->d_lcount + 2 * np, h->d_lbits + (size_t)np * h->nwords,
                   h->nsx, h->nsy};
}
ListClear list_clear(flb_engine* h, uint64_t t) {
  const NextLists nl = next_lists(h, t);
  return ListClear{nl.counts, nl.bits, h->nwords};
}

// Issues the passes of one time step at t on the stream.
uint64_t issue_step(flb_engine* h, uint64_t t, bool write_macro) {
  const uint32_t odd = (uint32_t)(t & 1u);
  uint64_t k = 0;
  refresh_params(h);
  if (h->has_io) {
    cudaMemcpyAsync(h->d_rho_snap, h->d_rho, (size_t)h->N * h->c_size, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(h->d_u_snap, h->d_u, 2ull * h->N * h->c_size, cudaMemcpyDeviceToDevice, h->stream);
  }
  if (h->fs) {
    h->kp.trust_prev = h->trust ? 1 : 0;
    const FsLists L = fs_lists(h, t);
    dispatch(h, [&](auto ops) {
      ops.fs1(h, odd, L.sc, list_clear(h, t));
      ops.sc_list(h, odd, L.sc);
      k = 2 + (uint64_t)ops.fs234(h, odd, L.fs, next_lists(h, t));
    });
    h->cur ^= 1;
    h->trust = true;
    h->fs_all_next = L.all;
    h->lists_valid = true;
    refresh_params(h);
  } else {
    dispatch(h, [&](auto ops) { ops.sc(h, odd, write_macro || h->has_io); });
    k = 1;
  }
  return k;
}

// Failure injection for tests, read when the step graphs are built: with
// FLB_PERSIST_SKIP_ARRIVAL=1 in the environment the last CTA of the persistent
// step never arrives at its grid barriers, so each wait runs out after the
// wait limit and the launch reports FLB_ERR_CUDA at the next flb_sync.
uint32_t persist_skip_cta(flb_engine* h) {
  const char* v = std::getenv("FLB_PERSIST_SKIP_ARRIVAL");
  if (!v || std::strcmp(v, "1") != 0 || h->grid_persist == 0) return 0xffffffffu;
  return h->grid_persist - 1u;
}

// Issues 2*pairs free-surface steps from an even t (flag buffer 0 current) as
// one persistent launch (trace: see FspArgs).
flb_status issue_persist(flb_engine* h, int pairs, uint64_t* trace = nullptr) {
  const int saved = h->cur;
  h->cur = 0;
  refresh_params(h);
  KParams p0 = h->kp;
  h->cur = 1;
  refresh_params(h);
  KParams p1 = h->kp;
  h->cur = saved;
  refresh_params(h);
  p0.trust_prev = 1;
  p1.trust_prev = 1;
  FspArgs a{};
  for (int q = 0; q < 2; q++)
    for (int k = 0; k < 2; k++) a.list[q][k] = h->d_list[q][k];
  a.lcount = h->d_lcount;
  a.lbits = h->d_lbits;
  a.nwords = h->nwords;
  a.nz = h->d_nz;
  a.nsx = h->nsx;
  a.nsy = h->nsy;
  a.fs_all = h->thin_tiles ? 1 : 0;
  a.bar = h->d_bar;
  a.err = h->d_perr;
  a.steps = 2u * (uint32_t)pairs;
  a.wait_limit = h->wait_limit;
  a.skip_cta = h->g_skip;
  a.trace = trace;
  cudaError_t e = cudaSuccess;
  dispatch(h, [&](auto ops) { e = ops.persist(h, p0, p1, a); });
  if (e != cudaSuccess) return cuda_fail(h, e, "persistent free-surface step launch");
  return FLB_OK;
}

void destroy_graph(GraphSlot& g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g = GraphSlot{};
}

// Captures 2*pairs steps starting at an even t with flag buffer 0 current:
// the passes of every step, or one persistent launch (free surface, h->persist).
flb_status capture(flb_engine* h, GraphSlot& g, int pairs) {
  if (g.exec) return FLB_OK;
  const int saved_cur = h->cur;
  FLB_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  uint64_t kernels = 0;
  flb_status ps = FLB_OK;
  if (h->fs && h->persist) {
    ps = issue_persist(h, pairs);
    kernels = 1;
  } else {
    for (int s = 0; s < 2 * pairs; s++) kernels += issue_step(h, (uint64_t)s, false);
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
  if (ps != FLB_OK) {
    if (graph) cudaGraphDestroy(graph);
    h->cur = saved_cur;
    refresh_params(h);
    return ps;
  }
  h->cur = saved_cur;
  refresh_params(h);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_fail(h, e, "cudaGraphInstantiate");
  }
  g.graph = graph;
  g.exec = exec;
  g.kernels = kernels;
  return FLB_OK;
}

// Whether the free-surface steps replayed from graphs run as one persistent
// launch (k_fsp.cu) or as four kernels per step.
void resolve_persist(flb_engine* h) {
  const bool can = h->fs && h->grid_persist > 0;
  h->persist = can && (h->step_mode == FLB_STEP_PERSISTENT ||
                       (h->step_mode == FLB_STEP_AUTO && h->ntiles <= kPersistAutoTiles));
}

// Reads (and clears) the persistent step's error word after the stream has
// drained: a grid barrier that gave up leaves the state undefined.
flb_status check_persist(flb_engine* h) {
  if (!h->fs || !h->d_perr) return FLB_OK;
  uint32_t e = 0;
  FLB_CUDA(h, cudaMemcpyAsync(&e, h->d_perr, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!e) return FLB_OK;
  h->broken = true;
  FLB_CUDA(h, cudaMemsetAsync(h->d_perr, 0, sizeof(uint32_t), h->stream));
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return fail(h, FLB_ERR_CUDA,
              "a grid barrier of the persistent free-surface step gave up waiting; the state is undefined until "
              "flb_reset");
}

void free_all(flb_engine* h) {
  destroy_graph(h->g_pair);
  destroy_graph(h->g_big);
  void* bufs[] = {h->d_f,          h->d_rho,         h->d_u,           h->d_flags[0],    h->d_flags[1],
                  h->d_geo,        h->d_nbmask,      h->d_mass,        h->d_excess,      h->d_phi,
                  h->d_recon,      h->d_recon_mask,  h->d_rho_snap,    h->d_u_snap,      h->d_partial,
                  h->d_scalar,     h->d_counts,      h->d_nz,          h->d_lbits,       h->d_list[0][0],
                  h->d_list[0][1], h->d_list[1][0],  h->d_list[1][1],  h->d_lcount,     h->d_tstep,
                  h->d_plain,      h->d_bar,         h->d_perr};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

flb_status validate(const flb_case_desc* d, std::string& msg) {
  if (!d) return msg = "null descriptor", FLB_ERR_INVALID_ARGUMENT;
  if (!d->flags) return msg = "flags is null", FLB_ERR_INVALID_ARGUMENT;
  if (d->nx < 3 || d->ny < 3) return msg = "nx and ny must be at least 3", FLB_ERR_INVALID_ARGUMENT;
  const uint64_t N = (uint64_t)d->nx * d->ny;
  if (9ull * N >= (1ull << 32)) return msg = "9*nx*ny must stay below 2^32", FLB_ERR_INVALID_ARGUMENT;
  if (!(d->tau > 0.5f) || !std::isfinite(d->tau)) return msg = "tau must be finite and > 0.5", FLB_ERR_INVALID_ARGUMENT;
  if (d->precision != 64 && d->precision != 32 && d->precision != 16)
    return msg = "precision must be 64, 32 or 16", FLB_ERR_INVALID_ARGUMENT;
  if (d->mass_precision != 64 && d->mass_precision != 32)
    return msg = "mass_precision must be 64 or 32", FLB_ERR_INVALID_ARGUMENT;
  if (d->mass_precision == 32 && d->precision != 32)
    return msg = "mass_precision 32 requires precision 32", FLB_ERR_UNSUPPORTED;
  if (d->collision != 0 && d->collision != 1) return msg = "collision must be SRT or TRT", FLB_ERR_INVALID_ARGUMENT;
  if (d->bounce_back != FLB_BB_IMPLICIT && d->bounce_back != FLB_BB_HALFWAY)
    return msg = "bounce_back must be IMPLICIT or HALFWAY", FLB_ERR_INVALID_ARGUMENT;
  if (d->fs_mode != FLB_FS_REFERENCE && d->fs_mode != FLB_FS_CONSERVATIVE)
    return msg = "fs_mode must be REFERENCE or CONSERVATIVE", FLB_ERR_INVALID_ARGUMENT;
  if (!(d->u_max >= 0.0f) || !std::isfinite(d->u_max)) return msg = "u_max must be finite and >= 0", FLB_ERR_INVALID_ARGUMENT;
  if (d->arithmetic != FLB_ARITH_REFERENCE && d->arithmetic != FLB_ARITH_FUSED)
    return msg = "arithmetic must be REFERENCE or FUSED", FLB_ERR_INVALID_ARGUMENT;
  if (d->kernel_variant < 0 || d->kernel_variant > 2) return msg = "kernel_variant must be 0, 1 or 2", FLB_ERR_INVALID_ARGUMENT;
  if (d->kernel_variant == 2 && d->nx % (uint32_t)vec_width(d->precision) != 0)
    return msg = "the vector stream-collide needs nx divisible by its vector width", FLB_ERR_UNSUPPORTED;
  if (d->precision == 16) {
    const float s = d->f16_scale == 0.0f ? 4096.0f : d->f16_scale;
    int e = 0;
    if (!(s > 0.0f) || std::frexp(s, &e) != 0.5f) return msg = "f16_scale must be a power of two", FLB_ERR_INVALID_ARGUMENT;
  }
  return FLB_OK;
}

flb_status check_io(flb_engine* h, const uint8_t* flags) {
  // one OR over all the bytes (a loop the compiler vectorises: it runs on
  // every reset), then the two cells an inlet or outlet may not occupy, in
  // the order a cell-by-cell scan meets them
  const uint64_t N = h->N;
  uint8_t any = 0;
  for (uint64_t i = 0; i < N; i++) any = (uint8_t)(any | flags[i]);
  h->has_io = (any & (kInlet | kOutlet)) != 0;
  if (N == 1 && (flags[0] & kInlet)) return fail(h, FLB_ERR_INVALID_ARGUMENT, "inlet in the last cell");
  if (N > 0 && (flags[0] & kOutlet)) return fail(h, FLB_ERR_INVALID_ARGUMENT, "outlet in the first cell");
  if (N > 0 && (flags[N - 1] & kInlet)) return fail(h, FLB_ERR_INVALID_ARGUMENT, "inlet in the last cell");
  return FLB_OK;
}

// Builds the initial state from the geometry flags in d_geo.
flb_status initialise(flb_engine* h) {
  FLB_CUDA(h, cudaMemsetAsync(h->d_f, 0, 9ull * h->N * h->s_size, h->stream));
  h->cur = 0;
  h->t = 0;
  if (h->fs)
    launch_init_flags(h->d_geo, h->d_flags[0], h->nx, h->ny, 1, h->d_mass, h->d_excess, h->d_phi, h->m_size == 8,
                      h->stream);
  else
    launch_init_flags(h->d_geo, h->d_flags[0], h->nx, h->ny, 0, nullptr, nullptr, nullptr, 1, h->stream);
  h->launches++;
  if (h->hw) {
    launch_nbmask(h->d_geo, h->d_nbmask, h->nx, h->ny, h->stream);
    h->launches++;
  }
  refresh_params(h);
  dispatch(h, [&](auto ops) { ops.init_ddf(h); });
  h->launches++;
  if (h->fs) FLB_CUDA(h, cudaMemcpyAsync(h->d_flags[1], h->d_flags[0], h->N, cudaMemcpyDeviceToDevice, h->stream));
  if (h->d_recon_mask) FLB_CUDA(h, cudaMemsetAsync(h->d_recon_mask, 0, h->N, h->stream));
  FLB_CUDA(h, cudaMemsetAsync(h->d_tstep, 0, 2 * sizeof(uint32_t), h->stream));
  refresh_plain(h);
  h->trust = true;  // flags[1] = flags[0] and the initial fields satisfy the skip invariants
  h->lists_valid = false;
  h->fs_all_next = false;
  h->broken = false;
  FLB_CUDA(h, cudaGetLastError());
  return FLB_OK;
}

// Runs a visualisation launch into dst (device) or through a temporary (host).
template <class Launch>
flb_status viz_run(flb_handle h, size_t bytes, void* dst, int on_device, Launch&& launch) {
  uint8_t* out = static_cast<uint8_t*>(dst);
  if (!on_device) FLB_CUDA(h, cudaMallocAsync((void**)&out, bytes, h->stream));
  launch(out);
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(dst, out, bytes, cudaMemcpyDeviceToHost, h->stream);
  if (!on_device) cudaFreeAsync(out, h->stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "visualisation kernel");
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

}  // namespace

namespace flb {
// The per-case constants of KParams (relaxation, forcing, codec, fused-
// arithmetic factors) from a validated descriptor; pointers are left null.
void fill_case_constants(const flb_case_desc* desc, KParams& k) {
  std::memset(&k, 0, sizeof(k));
  const float tau = desc->tau;  // float, as cudaInitData.cu:81-82
  k.inv_tau = 1.0f / tau;
  k.use_force = desc->use_volumetric_force ? 1 : 0;
  k.fx = desc->use_volumetric_force ? desc->fx : 0.0f;
  k.fy = desc->use_volumetric_force ? desc->fy : 0.0f;
  k.subgrid = desc->subgrid ? 1 : 0;
  k.collision = desc->collision;
  k.f16_scale = desc->f16_scale == 0.0f ? 4096.0f : desc->f16_scale;
  k.f16_inv = 1.0f / k.f16_scale;
  k.inlet_ux = desc->inlet_ux;
  k.inlet_uy = desc->inlet_uy;
  k.fs_cons = desc->fs_mode == FLB_FS_CONSERVATIVE ? 1 : 0;
  k.u_max = desc->u_max > 0.0f ? desc->u_max : 0.0f;
  {
    // cx[i]*Fx + cy[i]*Fy in float, the same IEEE operations the reference
    // kernel evaluates per cell (cellCalculations.cuh:71); volatile keeps the
    // host compiler from contracting or folding them
    const int cxs[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1}, cys[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
    for (int i = 0; i < 9; i++) {
      volatile float a = (float)cxs[i] * k.fx;
      volatile float b = (float)cys[i] * k.fy;
      k.cF[i] = a + b;
    }
    // constants of the fused arithmetic, float, uncontracted (the oracle
    // computes the same ones)
    volatile float om = k.inv_tau;
    volatile float omc = 1.0f - om;
    volatile float half = 0.5f * om;
    volatile float kk = 1.0f - half;
    volatile float k3 = 3.0f * kk;
    volatile float k9 = 9.0f * kk;
    k.fu_omc = omc;
    k.fu_nk3 = -k3;
    k.fu_fx = k.fx;
    k.fu_fy = k.fy;
    volatile float hx = 0.5f * k.fx, hy = 0.5f * k.fy;
    k.fu_hfx = hx;
    k.fu_hfy = hy;
    k.fu_sw[0] = k.f16_scale * wgt<float>(0);  // exact: power-of-two scale
    k.fu_sw[1] = k.f16_scale * wgt<float>(1);
    k.fu_sw[2] = k.f16_scale * wgt<float>(5);
    for (int q = 0; q < 4; q++) {
      volatile float g = k3 * k.cF[2 * q + 1];
      volatile float hh = k9 * k.cF[2 * q + 1];
      k.fu_g[q] = g;
      k.fu_h[q] = hh;
    }
  }
}

flb_status validate_desc(const flb_case_desc* d, std::string& msg) { return validate(d, msg); }

}  // namespace flb

// =============================================================================
extern "C" {

FLB_API void flb_case_desc_init(flb_case_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->precision = 32;
  d->mass_precision = 64;
  d->collision = FLB_COLLISION_SRT;
  d->use_volumetric_force = 1;
  d->tau = 0.6f;
  d->bounce_back = FLB_BB_HALFWAY;
  d->fs_mode = FLB_FS_CONSERVATIVE;
  d->device = -1;
  d->arithmetic = FLB_ARITH_FUSED;
}

FLB_API flb_status flb_create(const flb_case_desc* desc, flb_handle* out) {
  if (!out) return FLB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::string msg;
  flb_status s = validate(desc, msg);
  if (s != FLB_OK) {
    std::fprintf(stderr, "flb_create: %s\n", msg.c_str());
    return s;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FLB_ERR_NO_DEVICE;
  flb_engine* h = new flb_engine();
  h->desc = *desc;
  h->desc.flags = nullptr;
  h->nx = desc->nx;
  h->ny = desc->ny;
  h->N = desc->nx * desc->ny;
  h->fs = desc->free_surface != 0;
  h->hw = desc->bounce_back == FLB_BB_HALFWAY;
  h->fused = desc->arithmetic == FLB_ARITH_FUSED && desc->collision == FLB_COLLISION_SRT && !desc->subgrid;
  if (desc->device >= 0) h->device = desc->device;
  else cudaGetDevice(&h->device);
  if (h->device >= ndev) {
    delete h;
    return FLB_ERR_INVALID_ARGUMENT;
  }
  DeviceGuard guard(h->device);
  if (desc->precision == 64) {
    h->variant = V_F64;
    h->s_size = 8; h->c_size = 8; h->m_size = 8;
  } else if (desc->precision == 16) {
    h->variant = V_F16S;
    h->s_size = 2; h->c_size = 4; h->m_size = 8;
  } else if (desc->mass_precision == 32) {
    h->variant = V_F32M32;
    h->s_size = 4; h->c_size = 4; h->m_size = 4;
  } else {
    h->variant = V_F32;
    h->s_size = 4; h->c_size = 4; h->m_size = 8;
  }
  {
    const uint32_t V = (uint32_t)vec_width(desc->precision);
    // measured on a B200 (8192x2048 single phase): the vector path is faster
    // for FP16S, and for FP32 with the fused arithmetic (89 vs 82 GLUPS); with
    // the reference arithmetic FP32 runs faster one cell per thread (full
    // occupancy), and so does FP64
    const bool fused = desc->arithmetic == FLB_ARITH_FUSED && desc->collision == FLB_COLLISION_SRT && !desc->subgrid;
    h->use_vec = desc->kernel_variant == 2 ||
                 (desc->kernel_variant == 0 && desc->nx % V == 0 &&
                  (desc->precision == 16 || (desc->precision == 32 && fused)));
    // free surface, the listed stream-collide: measured on a B200, the vector
    // path is slower for FP32 (2048x512 dam break 33.3 against 29.4 us per
    // step; 8192x2048 53.4 against 54.8 GLUPS) and faster for FP16S on large
    // grids (8192x2048: 57.5 against 54.7 GLUPS), so it runs there, or when
    // asked for
    const uint64_t tiles = (uint64_t)((desc->nx + kSTW - 1) / kSTW) * ((desc->ny + kSTH - 1) / kSTH);
    h->use_vec_list = desc->kernel_variant == 2 ||
                      (desc->kernel_variant == 0 && desc->nx % V == 0 && desc->precision == 16 && fused &&
                       tiles > 4096u);
    // flag pass: 128-wide tiles with two cells per thread (512-thread
    // blocks, two per SM) on grids of up to 4096 super-tiles, 64-wide tiles
    // with two cells per thread (256-thread blocks, five per SM at 48
    // registers) above.  Measured on a B200 (quiet tiles counting their
    // neighbours from the flags): 2048x512 dam break 25.9 us per step with
    // 128x2 against 28.0 with 128x1, 28.0 with 64x1, 33.4 with 64x2 and 33.5
    // with 128x4; 8192x2048 224.5 with 64x2 against 226.9 with 128x2, 232.1
    // with 64x1 and 242.0 with 128x1.  Earlier builds (before the quiet-tile
    // path): 2048x512 one cell per thread 29.2, two 30.1, four 34.6;
    // 8192x2048 flag pass 110 us per step with two cells per thread at two
    // blocks per SM (114 at three, 119 at four), one cell per thread 124,
    // four 131, 32-wide tiles 158.  FLB_FS_FLAG_FORM (32, 64x1, 64x2, 128x1,
    // 128x2 or 128x4: tile width x cells per thread) selects another form,
    // with the same results.
    h->fs_form = tiles <= 4096u ? FS_FORM_W128X2 : FS_FORM_W64X2;
    if (const char* v = std::getenv("FLB_FS_FLAG_FORM")) {
      if (!std::strcmp(v, "32")) h->fs_form = FS_FORM_W32;
      else if (!std::strcmp(v, "128x1")) h->fs_form = FS_FORM_W128X1;
      else if (!std::strcmp(v, "128x2")) h->fs_form = FS_FORM_W128X2;
      else if (!std::strcmp(v, "128x4")) h->fs_form = FS_FORM_W128X4;
      else if (!std::strcmp(v, "64x1")) h->fs_form = FS_FORM_W64X1;
      else if (!std::strcmp(v, "64x2")) h->fs_form = FS_FORM_W64X2;
    }
  }
  s = check_io(h, desc->flags);
  if (s != FLB_OK) {
    std::fprintf(stderr, "flb_create: %s\n", h->err.c_str());
    delete h;
    return s;
  }
  auto bail = [&](flb_status st) {
    std::fprintf(stderr, "flb_create: %s\n", h->err.c_str());
    free_all(h);
    delete h;
    return st;
  };
  if (desc->stream) {
    h->stream = static_cast<cudaStream_t>(desc->stream);
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaStreamCreate"));
    h->own_stream = true;
  }
  const uint64_t N = h->N;
  struct Alloc { void** p; size_t bytes; bool need; };
  const uint64_t blocks = (N + kBlock - 1) / kBlock;
  h->nsx = (h->nx + kSTW - 1) / kSTW;
  h->nsy = (h->ny + kSTH - 1) / kSTH;
  h->thin_tiles = (h->nx % kSTW != 0 && h->nx % kSTW < 3) || (h->ny % kSTH != 0 && h->ny % kSTH < 3);
  h->ntiles = h->nsx * h->nsy;
  h->nwords = (h->ntiles + 31u) / 32u;
  const uint64_t tiles = h->ntiles;
  Alloc allocs[] = {
      {&h->d_f, 9 * N * h->s_size, true},
      {&h->d_rho, N * h->c_size, true},
      {&h->d_u, 2 * N * h->c_size, true},
      {(void**)&h->d_flags[0], N, true},
      {(void**)&h->d_flags[1], N, h->fs},
      {(void**)&h->d_geo, N, true},
      {(void**)&h->d_nbmask, N, h->hw},
      {&h->d_mass, N * h->m_size, h->fs},
      {&h->d_excess, N * h->m_size, h->fs},
      {&h->d_phi, N * h->m_size, h->fs},
      {&h->d_recon, 8 * N * h->c_size, h->fs && desc->fs_mode == FLB_FS_REFERENCE},
      {(void**)&h->d_recon_mask, N, h->fs && desc->fs_mode == FLB_FS_REFERENCE},
      {&h->d_rho_snap, N * h->c_size, h->has_io},
      {&h->d_u_snap, 2 * N * h->c_size, h->has_io},
      {(void**)&h->d_partial, blocks * sizeof(double), true},
      {(void**)&h->d_scalar, sizeof(double), true},
      {(void**)&h->d_counts, 8 * sizeof(unsigned long long), true},
      {(void**)&h->d_tstep, 2 * sizeof(uint32_t), true},
      {(void**)&h->d_plain, (((size_t)N + 3) / 4 + 31) / 32 * sizeof(uint32_t), !h->fs},
      {(void**)&h->d_nz, tiles * sizeof(uint32_t), h->fs},
      {(void**)&h->d_lbits, 2 * (size_t)((tiles + 31) / 32) * sizeof(uint32_t), h->fs},
      {(void**)&h->d_list[0][0], tiles * sizeof(uint32_t), h->fs},
      {(void**)&h->d_list[0][1], tiles * sizeof(uint32_t), h->fs},
      {(void**)&h->d_list[1][0], tiles * sizeof(uint32_t), h->fs},
      {(void**)&h->d_list[1][1], tiles * sizeof(uint32_t), h->fs},
      {(void**)&h->d_lcount, 4 * sizeof(uint32_t), h->fs},
      {(void**)&h->d_bar, sizeof(uint32_t), h->fs},
      {(void**)&h->d_perr, sizeof(uint32_t), h->fs},
  };
  // Failure injection on the host: with FLB_FAIL_ALLOC_AT=k in the
  // environment the k-th device allocation of this creation fails as
  // cudaMalloc does when memory runs out (nothing is allocated for it), so the
  // clean-up path can be exercised without exhausting a GPU.
  long fail_at = 0;
  if (const char* v = std::getenv("FLB_FAIL_ALLOC_AT")) fail_at = std::strtol(v, nullptr, 10);
  long nalloc = 0;
  for (Alloc& a : allocs) {
    if (!a.need) continue;
    cudaError_t e = ++nalloc == fail_at ? cudaErrorMemoryAllocation : cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc"));
  }
  if (h->fs) {
    // list lengths start at zero
    cudaError_t e0 = cudaMemsetAsync(h->d_lcount, 0, 4 * sizeof(uint32_t), h->stream);
    if (e0 != cudaSuccess) return bail(cuda_fail(h, e0, "cudaMemsetAsync"));
    e0 = cudaMemsetAsync(h->d_perr, 0, sizeof(uint32_t), h->stream);
    if (e0 != cudaSuccess) return bail(cuda_fail(h, e0, "cudaMemsetAsync"));
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    dispatch(h, [&](auto ops) { ops.grids(h, nsm > 0 ? nsm : 1); });
    // the persistent step needs every CTA resident at once (inlet/outlet cells
    // need a density/velocity snapshot before each stream-collide: per-pass only)
    int per_sm = 0;
    dispatch(h, [&](auto ops) { per_sm = ops.persist_blocks(h); });
    h->grid_persist = h->has_io || per_sm <= 0 ? 0u : (uint32_t)(nsm * per_sm);
    resolve_persist(h);
  }
  fill_case_constants(desc, h->kp);
  cudaError_t e = cudaMemcpyAsync(h->d_geo, desc->flags, N, cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaMemcpyAsync"));
  s = initialise(h);
  if (s != FLB_OK) return bail(s);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaStreamSynchronize"));
  *out = h;
  return FLB_OK;
}

FLB_API flb_status flb_reset(flb_handle h, const uint8_t* host_flags) {
  if (!h || !host_flags) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  const bool had_io = h->has_io;
  flb_status s = check_io(h, host_flags);
  if (s != FLB_OK) {
    h->has_io = had_io;  // the handle keeps its state
    return s;
  }
  if (h->has_io && !had_io) {
    h->has_io = false;
    return fail(h, FLB_ERR_UNSUPPORTED, "reset adds inlet/outlet cells to a case created without them");
  }
  if (had_io != h->has_io) {
    destroy_graph(h->g_pair);
    destroy_graph(h->g_big);
  }
  FLB_CUDA(h, cudaMemcpyAsync(h->d_geo, host_flags, h->N, cudaMemcpyHostToDevice, h->stream));
  return initialise(h);
}

FLB_API flb_status flb_destroy(flb_handle h) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  {
    DeviceGuard guard(h->device);
    cudaStreamSynchronize(h->stream);
    free_all(h);
  }
  delete h;
  return FLB_OK;
}

FLB_API flb_status flb_step(flb_handle h, uint64_t n) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  if (h->broken)
    return fail(h, FLB_ERR_CUDA, "a grid barrier of the persistent step gave up in an earlier launch; call flb_reset");
  if (n == 0) return FLB_OK;
  DeviceGuard guard(h->device);
  if (h->fs && h->persist) {
    const uint32_t skip = persist_skip_cta(h);
    if (skip != h->g_skip) {  // graphs carry the injection setting they were built with
      destroy_graph(h->g_pair);
      destroy_graph(h->g_big);
      h->g_skip = skip;
    }
  }
  nvtxRangePushA("flb_step");
  uint64_t remaining = n;
  flb_status s = FLB_OK;
  while (remaining > 0 && s == FLB_OK) {
    // graphs cover pairs of steps from an even t; the last step of the call
    // runs on its own so that it writes density and velocity
    // (free surface: every stream-collide writes density and velocity, so
    // the graphs run to the end of the call)
    const uint64_t big = 2ull * kGraphPairs;
    const uint64_t tail = h->fs ? 0u : 1u;
    if (h->fs && (!h->trust || !h->lists_valid || h->fs_all_next)) {
      // first step after the state was written from outside: no write skipping
      h->launches += issue_step(h, h->t, remaining == 1);
      h->t += 1;
      remaining -= 1;
    } else if ((h->t & 1u) == 0 && remaining >= big + tail) {
      s = capture(h, h->g_big, kGraphPairs);
      if (s != FLB_OK) break;
      cudaError_t e = cudaGraphLaunch(h->g_big.exec, h->stream);
      if (e != cudaSuccess) { s = cuda_fail(h, e, "cudaGraphLaunch"); break; }
      h->launches += h->g_big.kernels;
      h->t += big;
      remaining -= big;
    } else if ((h->t & 1u) == 0 && remaining >= 2 + tail) {
      s = capture(h, h->g_pair, 1);
      if (s != FLB_OK) break;
      cudaError_t e = cudaGraphLaunch(h->g_pair.exec, h->stream);
      if (e != cudaSuccess) { s = cuda_fail(h, e, "cudaGraphLaunch"); break; }
      h->launches += h->g_pair.kernels;
      h->t += 2;
      remaining -= 2;
    } else {
      h->launches += issue_step(h, h->t, remaining == 1);
      h->t += 1;
      remaining -= 1;
    }
  }
  nvtxRangePop();
  if (s != FLB_OK) return s;
  FLB_CUDA(h, cudaGetLastError());
  return FLB_OK;
}

FLB_API flb_status flb_sync(flb_handle h) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return check_persist(h);
}

FLB_API flb_status flb_set_step_mode(flb_handle h, int mode) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  if (mode != FLB_STEP_AUTO && mode != FLB_STEP_KERNELS && mode != FLB_STEP_PERSISTENT)
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "mode must be FLB_STEP_AUTO, FLB_STEP_KERNELS or FLB_STEP_PERSISTENT");
  if (mode == FLB_STEP_PERSISTENT && !(h->fs && h->grid_persist > 0))
    return fail(h, FLB_ERR_UNSUPPORTED,
                "the persistent step needs a free-surface case without inlet/outlet cells that can keep every CTA "
                "resident");
  DeviceGuard guard(h->device);
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));  // a running graph may be the one replaced
  const bool before = h->persist;
  h->step_mode = mode;
  resolve_persist(h);
  if (before != h->persist) {
    destroy_graph(h->g_pair);
    destroy_graph(h->g_big);
  }
  return FLB_OK;
}

FLB_API flb_status flb_get_step_mode(flb_handle h, int* mode, int* persistent) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  if (mode) *mode = h->step_mode;
  if (persistent) *persistent = h->persist ? 1 : 0;
  return FLB_OK;
}

FLB_API flb_status flb_set_wait_limit(flb_handle h, uint32_t polls) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  const uint32_t v = polls == 0 ? kPersistWaitLimit : polls;
  if (v != h->wait_limit) {
    h->wait_limit = v;
    destroy_graph(h->g_pair);
    destroy_graph(h->g_big);
  }
  return FLB_OK;
}

FLB_API flb_status flb_get_time(flb_handle h, uint64_t* t) {
  if (!h || !t) return FLB_ERR_INVALID_ARGUMENT;
  *t = h->t;
  return FLB_OK;
}

FLB_API flb_status flb_set_stream(flb_handle h, void* stream) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  if (stream) {
    h->stream = static_cast<cudaStream_t>(stream);
    h->own_stream = false;
  } else {
    FLB_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return FLB_OK;
}

FLB_API flb_status flb_get_stream(flb_handle h, void** stream) {
  if (!h || !stream) return FLB_ERR_INVALID_ARGUMENT;
  *stream = h->stream;
  return FLB_OK;
}

FLB_API flb_status flb_field_info(flb_handle h, int field, size_t* elem_size, size_t* count) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  size_t es = 0, n = 0;
  switch (field) {
    case FLB_FIELD_F: es = h->c_size; n = 9ull * h->N; break;
    case FLB_FIELD_RHO: es = h->c_size; n = h->N; break;
    case FLB_FIELD_U: es = h->c_size; n = 2ull * h->N; break;
    case FLB_FIELD_FLAGS: es = 1; n = h->N; break;
    case FLB_FIELD_MASS:
    case FLB_FIELD_EXCESS:
    case FLB_FIELD_PHI: es = h->m_size; n = h->fs ? h->N : 0; break;
    default: return fail(h, FLB_ERR_INVALID_ARGUMENT, "unknown field");
  }
  if (elem_size) *elem_size = es;
  if (count) *count = n;
  return FLB_OK;
}

static flb_status field_ptr(flb_handle h, int field, void** ptr, size_t* bytes) {
  size_t es = 0, n = 0;
  flb_status s = flb_field_info(h, field, &es, &n);
  if (s != FLB_OK) return s;
  if (n == 0) return fail(h, FLB_ERR_UNSUPPORTED, "field not held in mono-fluid mode");
  *bytes = es * n;
  switch (field) {
    case FLB_FIELD_F: *ptr = h->d_f; break;
    case FLB_FIELD_RHO: *ptr = h->d_rho; break;
    case FLB_FIELD_U: *ptr = h->d_u; break;
    case FLB_FIELD_FLAGS: *ptr = h->d_flags[h->cur]; break;
    case FLB_FIELD_MASS: *ptr = h->d_mass; break;
    case FLB_FIELD_EXCESS: *ptr = h->d_excess; break;
    case FLB_FIELD_PHI: *ptr = h->d_phi; break;
  }
  return FLB_OK;
}

FLB_API flb_status flb_read_field(flb_handle h, int field, void* dst, int on_device) {
  if (!h || !dst) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  void* src = nullptr;
  size_t bytes = 0;
  flb_status s = field_ptr(h, field, &src, &bytes);
  if (s != FLB_OK) return s;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (field == FLB_FIELD_F && h->variant == V_F16S) {
    void* tmp = nullptr;
    FLB_CUDA(h, cudaMallocAsync(&tmp, bytes, h->stream));
    refresh_params(h);
    dispatch(h, [&](auto ops) { ops.decode(h, tmp); });
    h->launches++;
    cudaError_t e = cudaMemcpyAsync(dst, tmp, bytes, kind, h->stream);
    cudaFreeAsync(tmp, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemcpyAsync");
  } else {
    FLB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
  }
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return check_persist(h);
}

FLB_API flb_status flb_write_field(flb_handle h, int field, const void* src, int on_device) {
  if (!h || !src) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  void* dst = nullptr;
  size_t bytes = 0;
  flb_status s = field_ptr(h, field, &dst, &bytes);
  if (s != FLB_OK) return s;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (field == FLB_FIELD_F && h->variant == V_F16S) {
    void* tmp = nullptr;
    FLB_CUDA(h, cudaMallocAsync(&tmp, bytes, h->stream));
    cudaError_t e = cudaMemcpyAsync(tmp, src, bytes, kind, h->stream);
    if (e == cudaSuccess) {
      refresh_params(h);
      dispatch(h, [&](auto ops) { ops.encode(h, tmp); });
      h->launches++;
    }
    cudaFreeAsync(tmp, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMemcpyAsync");
  } else {
    FLB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
  }
  if (field == FLB_FIELD_FLAGS) refresh_plain(h);
  h->trust = false;
  h->lists_valid = false;
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

// ---- headless visualisation (k_viz.cu) --------------------------------------
// Output goes straight to dst when it is device memory, else through a
// stream-ordered temporary that is copied to the host.

FLB_API flb_status flb_viz_velocity(flb_handle h, float* dst, int on_device) {
  if (!h || !dst) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  const bool dbl = h->c_size == 8;
  return viz_run(h, 2 * sizeof(float) * (size_t)h->N, dst, on_device, [&](uint8_t* out) {
    if (dbl) flb::launch_viz_uv<double>(h->d_u, (float*)out, h->N, h->stream);
    else flb::launch_viz_uv<float>(h->d_u, (float*)out, h->N, h->stream);
  });
}

FLB_API flb_status flb_viz_shade(flb_handle h, int quantity, const float* colormap_rgb, uint32_t n_colors,
                                 float max_value, float min_value, uint8_t* rgba, int on_device) {
  if (!h || !rgba || !colormap_rgb) return FLB_ERR_INVALID_ARGUMENT;
  if (quantity < FLB_VIZ_UX || quantity > FLB_VIZ_PRESSURE)
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "quantity must be FLB_VIZ_UX, _UY, _MAGNITUDE or _PRESSURE");
  if (n_colors == 0 || n_colors > 4096) return fail(h, FLB_ERR_INVALID_ARGUMENT, "n_colors must be 1..4096");
  DeviceGuard guard(h->device);
  float* cmap = nullptr;
  const size_t cbytes = 3 * sizeof(float) * (size_t)n_colors;
  FLB_CUDA(h, cudaMallocAsync((void**)&cmap, cbytes, h->stream));
  cudaError_t e = cudaMemcpyAsync(cmap, colormap_rgb, cbytes, cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(cmap, h->stream);
    return cuda_fail(h, e, "cudaMemcpyAsync");
  }
  const bool dbl = h->c_size == 8;
  flb_status s = viz_run(h, 4 * (size_t)h->N, rgba, on_device, [&](uint8_t* out) {
    if (dbl) flb::launch_viz_shade<double>(h->d_u, h->N, quantity, cmap, n_colors, max_value, min_value, out, h->stream);
    else flb::launch_viz_shade<float>(h->d_u, h->N, quantity, cmap, n_colors, max_value, min_value, out, h->stream);
  });
  cudaFreeAsync(cmap, h->stream);
  return s;
}

FLB_API flb_status flb_viz_isoline(flb_handle h, int field, float iso_value, uint32_t width, uint32_t height,
                                   const uint32_t camera_bounds[4], uint8_t* image, int on_device) {
  if (!h || !image || !camera_bounds) return FLB_ERR_INVALID_ARGUMENT;
  if (field != FLB_FIELD_U && !(field == FLB_FIELD_PHI && h->fs))
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "field must be FLB_FIELD_U, or FLB_FIELD_PHI with a free surface");
  if (width == 0 || height == 0 || width > 32768 || height > 32768)
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "image size must be 1..32768 in each direction");
  const uint32_t* b = camera_bounds;
  if (!(b[0] < b[1] && b[1] <= h->nx && b[2] < b[3] && b[3] <= h->ny))
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "camera bounds must satisfy b0 < b1 <= nx and b2 < b3 <= ny");
  DeviceGuard guard(h->device);
  const size_t bytes = (size_t)width * height;
  const bool vec = field == FLB_FIELD_U;
  const bool dbl = vec ? h->c_size == 8 : h->m_size == 8;
  const void* src = vec ? h->d_u : h->d_phi;
  return viz_run(h, bytes, image, on_device, [&](uint8_t* out) {
    cudaMemsetAsync(out, 0, bytes, h->stream);
    if (dbl) flb::launch_viz_isoline<double>(src, vec, h->nx, h->ny, iso_value, width, height, b, out, h->stream);
    else flb::launch_viz_isoline<float>(src, vec, h->nx, h->ny, iso_value, width, height, b, out, h->stream);
  });
}

FLB_API flb_status flb_total_mass(flb_handle h, double* mass) {
  if (!h || !mass) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  refresh_params(h);
  const uint32_t odd = (uint32_t)(h->t & 1u);
  dispatch(h, [&](auto ops) { ops.mass_partial(h, odd); });
  const uint32_t blocks = (h->N + kBlock - 1) / kBlock;
  launch_sum_partials(h->d_partial, blocks, h->d_scalar, h->stream);
  h->launches += 2;
  FLB_CUDA(h, cudaGetLastError());
  FLB_CUDA(h, cudaMemcpyAsync(mass, h->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

static flb_status census(flb_handle h, unsigned long long out[5]) {
  DeviceGuard guard(h->device);
  refresh_params(h);
  FLB_CUDA(h, cudaMemsetAsync(h->d_counts, 0, 8 * sizeof(unsigned long long), h->stream));
  const uint32_t odd = (uint32_t)(h->t & 1u);
  dispatch(h, [&](auto ops) { ops.census(h, odd); });
  h->launches++;
  FLB_CUDA(h, cudaGetLastError());
  FLB_CUDA(h, cudaMemcpyAsync(out, h->d_counts, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

FLB_API flb_status flb_cell_counts(flb_handle h, uint64_t counts[4]) {
  if (!h || !counts) return FLB_ERR_INVALID_ARGUMENT;
  unsigned long long c[5];
  flb_status s = census(h, c);
  if (s != FLB_OK) return s;
  for (int k = 0; k < 4; k++) counts[k] = c[k];
  return FLB_OK;
}

FLB_API flb_status flb_check_finite(flb_handle h) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  unsigned long long c[5];
  flb_status s = census(h, c);
  if (s != FLB_OK) return s;
  if (c[4]) return fail(h, FLB_ERR_NONFINITE, std::to_string(c[4]) + " cells hold non-finite populations");
  return FLB_OK;
}

FLB_API flb_status flb_run_pass(flb_handle h, int pass) {
  if (!h) return FLB_ERR_INVALID_ARGUMENT;
  if (pass < 0 || pass > 2) return fail(h, FLB_ERR_INVALID_ARGUMENT, "pass must be 0, 1 or 2");
  if (!h->fs && pass != 0) return fail(h, FLB_ERR_UNSUPPORTED, "free-surface pass on a mono-fluid case");
  DeviceGuard guard(h->device);
  refresh_params(h);
  const uint32_t odd = (uint32_t)(h->t & 1u);
  if (h->has_io && pass == 0) {
    FLB_CUDA(h, cudaMemcpyAsync(h->d_rho_snap, h->d_rho, (size_t)h->N * h->c_size, cudaMemcpyDeviceToDevice,
                                h->stream));
    FLB_CUDA(h, cudaMemcpyAsync(h->d_u_snap, h->d_u, 2ull * h->N * h->c_size, cudaMemcpyDeviceToDevice, h->stream));
  }
  const bool recon = h->fs && h->d_recon_mask;
  h->trust = false;
  h->lists_valid = false;
  h->kp.trust_prev = 0;
  const TileList all{nullptr, nullptr, h->ntiles, h->nsx, 1};
  // alone, stream-collide sees no parked populations, and FS_1 writes its
  // rebuilt populations into the population array like the reference kernel
  if (pass == 0 && recon) FLB_CUDA(h, cudaMemsetAsync(h->d_recon_mask, 0, h->N, h->stream));
  uint64_t k = (pass == 1 && recon) ? 2 : 1;
  dispatch(h, [&](auto ops) {
    if (pass == 0) {
      if (h->fs) ops.sc_list(h, odd, all);
      else ops.sc(h, odd, true);
    } else if (pass == 1) {
      ops.fs1(h, odd, all, list_clear(h, h->t));
    } else {
      // the lists it appends to go unused: lists_valid is false
      k = (uint64_t)ops.fs234(h, odd, all, next_lists(h, h->t));
    }
    if (pass == 1 && recon) ops.apply_recon(h, odd);
  });
  h->launches += k;
  if (pass == 2)  // keep the current buffer index tied to t
    FLB_CUDA(h, cudaMemcpyAsync(h->d_flags[h->cur], h->d_flags[h->cur ^ 1], h->N, cudaMemcpyDeviceToDevice,
                                h->stream));
  FLB_CUDA(h, cudaGetLastError());
  FLB_CUDA(h, cudaStreamSynchronize(h->stream));
  return FLB_OK;
}

FLB_API flb_status flb_profile_steps(flb_handle h, uint64_t n, double pass_ms[3]) {
  if (!h || !pass_ms) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  pass_ms[0] = pass_ms[1] = pass_ms[2] = 0.0;
  cudaEvent_t ev[4];
  for (auto& e : ev) FLB_CUDA(h, cudaEventCreate(&e));
  flb_status st = FLB_OK;
  for (uint64_t k = 0; k < n && st == FLB_OK; k++) {
    const uint32_t odd = (uint32_t)(h->t & 1u);
    refresh_params(h);
    if (h->has_io) {
      cudaMemcpyAsync(h->d_rho_snap, h->d_rho, (size_t)h->N * h->c_size, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(h->d_u_snap, h->d_u, 2ull * h->N * h->c_size, cudaMemcpyDeviceToDevice, h->stream);
    }
    cudaEventRecord(ev[0], h->stream);
    if (h->fs) {
      h->kp.trust_prev = h->trust ? 1 : 0;
      const FsLists L = fs_lists(h, h->t);
      cudaEventRecord(ev[0], h->stream);
      dispatch(h, [&](auto ops) { ops.fs1(h, odd, L.sc, list_clear(h, h->t)); });
      cudaEventRecord(ev[1], h->stream);
      dispatch(h, [&](auto ops) { ops.sc_list(h, odd, L.sc); });
      cudaEventRecord(ev[2], h->stream);
      int kf = 0;
      dispatch(h, [&](auto ops) { kf = ops.fs234(h, odd, L.fs, next_lists(h, h->t)); });
      cudaEventRecord(ev[3], h->stream);
      h->launches += 2 + (uint64_t)kf;
      h->cur ^= 1;
      h->trust = true;
      h->fs_all_next = L.all;
      h->lists_valid = true;
    } else {
      cudaEventRecord(ev[1], h->stream);
      dispatch(h, [&](auto ops) { ops.sc(h, odd, k + 1 == n || h->has_io); });
      cudaEventRecord(ev[2], h->stream);
      cudaEventRecord(ev[3], h->stream);
      h->launches += 1;
    }
    h->t += 1;
    cudaError_t e = cudaEventSynchronize(ev[3]);
    if (e != cudaSuccess) {
      st = cuda_fail(h, e, "cudaEventSynchronize");
      break;
    }
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[1], ev[2]);
    cudaEventElapsedTime(&c, ev[2], ev[3]);
    pass_ms[1] += a;
    pass_ms[0] += b;
    pass_ms[2] += c;
  }
  refresh_params(h);
  for (auto& e : ev) cudaEventDestroy(e);
  return st;
}

FLB_API flb_status flb_profile_phases(flb_handle h, uint64_t n, double phase_ms[3]) {
  if (!h || !phase_ms) return FLB_ERR_INVALID_ARGUMENT;
  if (!h->fs || h->grid_persist == 0)
    return fail(h, FLB_ERR_UNSUPPORTED, "phase timing needs the persistent free-surface step");
  if (h->broken) return fail(h, FLB_ERR_CUDA, "call flb_reset first");
  DeviceGuard guard(h->device);
  for (int k = 0; k < 3; k++) phase_ms[k] = 0.0;
  // steady state from an even t: per-pass steps until then
  while (!h->trust || !h->lists_valid || h->fs_all_next || (h->t & 1u)) {
    h->launches += issue_step(h, h->t, false);
    h->t += 1;
  }
  const uint64_t pairs_total = (n + 1) / 2;
  const int per = kGraphPairs;
  uint64_t* d_trace = nullptr;
  const size_t slots = 6u * per + 1u;
  FLB_CUDA(h, cudaMallocAsync((void**)&d_trace, slots * sizeof(uint64_t), h->stream));
  std::vector<uint64_t> tr(slots);
  flb_status st = FLB_OK;
  for (uint64_t done = 0; done < pairs_total && st == FLB_OK; done += per) {
    const int pairs = (int)std::min<uint64_t>((uint64_t)per, pairs_total - done);
    st = issue_persist(h, pairs, d_trace);
    if (st != FLB_OK) break;
    h->launches += 1;
    h->t += 2u * (uint64_t)pairs;
    cudaError_t e = cudaMemcpyAsync(tr.data(), d_trace, (6u * pairs + 1u) * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      st = cuda_fail(h, e, "phase trace read-back");
      break;
    }
    st = check_persist(h);
    for (int b = 1; b <= 6 * pairs && st == FLB_OK; b++) phase_ms[(b - 1) % 3] += (double)(tr[b] - tr[b - 1]) * 1e-6;
  }
  cudaFreeAsync(d_trace, h->stream);
  cudaStreamSynchronize(h->stream);
  return st;
}

FLB_API flb_status flb_launch_count(flb_handle h, uint64_t* launches) {
  if (!h || !launches) return FLB_ERR_INVALID_ARGUMENT;
  *launches = h->launches;
  return FLB_OK;
}

// ---- checkpoint ------------------------------------------------------------
namespace {
struct CkptHeader {
  char magic[8];
  uint32_t version, nx, ny, precision, mass_precision, free_surface, bounce_back, fs_mode;
  uint64_t t;
};
}  // namespace

FLB_API flb_status flb_save_checkpoint(flb_handle h, const char* path) {
  if (!h || !path) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  CkptHeader hd{};
  std::memcpy(hd.magic, "FLBCKPT1", 8);
  hd.version = 1;
  hd.nx = h->nx;
  hd.ny = h->ny;
  hd.precision = (uint32_t)h->desc.precision;
  hd.mass_precision = (uint32_t)h->desc.mass_precision;
  hd.free_surface = h->fs;
  hd.bounce_back = (uint32_t)h->desc.bounce_back;
  hd.fs_mode = (uint32_t)h->desc.fs_mode;
  hd.t = h->t;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(h, FLB_ERR_IO, std::string("cannot open ") + path);
  std::fwrite(&hd, sizeof(hd), 1, fp);
  struct Part { void* d; size_t bytes; };
  std::vector<Part> parts = {{h->d_f, 9ull * h->N * h->s_size}, {h->d_rho, (size_t)h->N * h->c_size},
                             {h->d_u, 2ull * h->N * h->c_size}, {h->d_flags[h->cur], h->N}};
  if (h->fs) {
    parts.push_back({h->d_mass, (size_t)h->N * h->m_size});
    parts.push_back({h->d_excess, (size_t)h->N * h->m_size});
    parts.push_back({h->d_phi, (size_t)h->N * h->m_size});
  }
  std::vector<char> buf;
  for (const Part& p : parts) {
    buf.resize(p.bytes);
    cudaError_t e = cudaMemcpyAsync(buf.data(), p.d, p.bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      std::fclose(fp);
      return cuda_fail(h, e, "checkpoint read-back");
    }
    if (std::fwrite(buf.data(), 1, p.bytes, fp) != p.bytes) {
      std::fclose(fp);
      return fail(h, FLB_ERR_IO, "short write");
    }
  }
  std::fclose(fp);
  return FLB_OK;
}

FLB_API flb_status flb_load_checkpoint(flb_handle h, const char* path) {
  if (!h || !path) return FLB_ERR_INVALID_ARGUMENT;
  DeviceGuard guard(h->device);
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(h, FLB_ERR_IO, std::string("cannot open ") + path);
  CkptHeader hd{};
  if (std::fread(&hd, sizeof(hd), 1, fp) != 1 || std::memcmp(hd.magic, "FLBCKPT1", 8) != 0) {
    std::fclose(fp);
    return fail(h, FLB_ERR_IO, "not a checkpoint file");
  }
  if (hd.nx != h->nx || hd.ny != h->ny || hd.precision != (uint32_t)h->desc.precision ||
      hd.mass_precision != (uint32_t)h->desc.mass_precision || hd.free_surface != (uint32_t)h->fs ||
      hd.bounce_back != (uint32_t)h->desc.bounce_back || hd.fs_mode != (uint32_t)h->desc.fs_mode) {
    std::fclose(fp);
    return fail(h, FLB_ERR_INVALID_ARGUMENT, "checkpoint was written by a different case configuration");
  }
  const int cur = (int)(hd.t & 1u) & (h->fs ? 1 : 0);
  struct Part { void* d; size_t bytes; };
  std::vector<Part> parts = {{h->d_f, 9ull * h->N * h->s_size}, {h->d_rho, (size_t)h->N * h->c_size},
                             {h->d_u, 2ull * h->N * h->c_size}, {h->d_flags[cur], h->N}};
  if (h->fs) {
    parts.push_back({h->d_mass, (size_t)h->N * h->m_size});
    parts.push_back({h->d_excess, (size_t)h->N * h->m_size});
    parts.push_back({h->d_phi, (size_t)h->N * h->m_size});
  }
  std::vector<char> buf;
  for (const Part& p : parts) {
    buf.resize(p.bytes);
    if (std::fread(buf.data(), 1, p.bytes, fp) != p.bytes) {
      std::fclose(fp);
      return fail(h, FLB_ERR_IO, "truncated checkpoint");
    }
    cudaError_t e = cudaMemcpyAsync(p.d, buf.data(), p.bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      std::fclose(fp);
      return cuda_fail(h, e, "checkpoint upload");
    }
  }
  std::fclose(fp);
  h->t = hd.t;
  h->cur = cur;
  h->trust = false;
  h->lists_valid = false;
  refresh_params(h);
  refresh_plain(h);
  return set_tstep(h);
}

FLB_API const char* flb_last_error(flb_handle h) { return h ? h->err.c_str() : "null handle"; }

FLB_API const char* flb_status_string(flb_status s) {
  const int i = (int)s;
  return (i >= 0 && i < (int)(sizeof(kStatusText) / sizeof(kStatusText[0]))) ? kStatusText[i] : "unknown status";
}

FLB_API const char* flb_version(void) { return "flowlb-b200 0.1 (sm_100a)"; }

}  // extern "C"
