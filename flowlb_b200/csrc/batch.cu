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
//  * the cells are updated by the same sc_cell as the single-case kernels, so
//    every case ends bit-identical to flb_step on its own handle.
// With few clusters only a few cases are active at a time, so their
// populations stay in the 126 MB L2 while they are stepped.  The cluster size
// and the number of clusters are chosen by a short timed search at creation
// (flb_batch_create with autotune).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
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
#ifndef FLB_BATCH_MIN_BLOCKS
#define FLB_BATCH_MIN_BLOCKS 2  // two 1024-thread CTAs per SM: at most 32 registers
#endif

struct BatchCase {
  KParams kp;
  uint32_t nsegx;  // 32-cell row segments
};

// One step of one case: the warps of the cluster take 32-cell row segments.
template <bool HW, bool FU, bool ODD, bool WM>
__device__ __noinline__ void batch_step(const KParams& p, uint32_t items, uint32_t nsegx, uint32_t wid, uint32_t nw,
                                        uint32_t lane) {
  for (uint32_t it = wid; it < items; it += nw) {
    const uint32_t y = it / nsegx;
    const uint32_t x = (it - y * nsegx) * 32u + lane;
    if (x < p.nx) sc_cell<float, float, double, false, HW, WM, ODD, FU>(p, x, y);
  }
}

// *tdev: time step of the first step (its parity selects the slot pattern);
// steps >= 1; wm_last: write density and velocity in the last step.
template <bool HW, bool FU>
__global__ void __launch_bounds__(kBatchMaxThreads, FLB_BATCH_MIN_BLOCKS) k_batch(const BatchCase* __restrict__ cases,
                                                         const uint32_t* __restrict__ order,
                                                         const uint32_t* __restrict__ start,
                                                         const uint32_t* __restrict__ tdev, uint32_t steps,
                                                         int wm_last) {
  __shared__ BatchCase sc;
  const uint32_t t0 = *tdev;
  cg::cluster_group cl = cg::this_cluster();
  const uint32_t cs = cl.num_blocks();
  const uint32_t cid = blockIdx.x / cs;
  const uint32_t rank = cl.block_rank();
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t wid = rank * warps + (threadIdx.x >> 5), nw = cs * warps;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t k = start[cid]; k < start[cid + 1]; k++) {
    __syncthreads();  // the previous case's parameters are no longer read
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&cases[order[k]]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sc);
      for (uint32_t i = threadIdx.x; i < sizeof(BatchCase) / 4; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const KParams& p = sc.kp;
    const uint32_t nsegx = sc.nsegx, items = p.ny * nsegx;
    for (uint32_t s = 0; s < steps; s++) {
      const bool odd = ((t0 + s) & 1u) != 0;
      const bool wm = wm_last && s + 1 == steps;
      if (odd) {
        if (wm) batch_step<HW, FU, true, true>(p, items, nsegx, wid, nw, lane);
        else batch_step<HW, FU, true, false>(p, items, nsegx, wid, nw, lane);
      } else {
        if (wm) batch_step<HW, FU, false, true>(p, items, nsegx, wid, nw, lane);
        else batch_step<HW, FU, false, false>(p, items, nsegx, wid, nw, lane);
      }
      cl.sync();
    }
  }
}

// advances the device time-step counter after a batch launch
__global__ void k_tadd(uint32_t* t, uint32_t n) { *t += n; }

using BatchKernel = void (*)(const BatchCase*, const uint32_t*, const uint32_t*, const uint32_t*, uint32_t, int);

BatchKernel pick_kernel(bool hw, bool fu) {
  if (hw) return fu ? k_batch<true, true> : k_batch<true, false>;
  return fu ? k_batch<false, true> : k_batch<false, false>;
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
  std::vector<size_t> off;  // first cell of each case in the concatenated cell arrays
  size_t cells = 0;
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
  std::vector<BatchCase> hcases;
  // launch configuration
  int cluster = 8, clusters = 0, threads = 512, tuned = 0;
  uint64_t launches = 0;
  // the step graph (batch kernel + counter update) for one step count
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint32_t g_steps = 0;
  int g_wm = -1, g_cluster = 0, g_clusters = 0, g_threads = 0;
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
  void* bufs[] = {b->d_f, b->d_rho, b->d_u, b->d_flags, b->d_geo, b->d_nbmask, b->d_tstep, b->d_cases, b->d_order,
                  b->d_start};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

// Initial state of every case (the single-case initialisation, per case).
flb_status binit(flb_batch b) {
  BDevice g(b->device);
  for (uint32_t c = 0; c < b->n; c++) {
    const size_t o = b->off[c];
    launch_init_flags(b->d_geo + o, b->d_flags + o, b->nx[c], b->ny[c], 0, nullptr, nullptr, nullptr, 1, b->stream);
    if (b->hw) launch_nbmask(b->d_geo + o, b->d_nbmask + o, b->nx[c], b->ny[c], b->stream);
    launch_init_ddf<float, float, double>(b->hcases[c].kp, b->stream, b->d_geo + o, b->hw);
  }
  FLB_BCUDA(b, cudaMemsetAsync(b->d_tstep, 0, 2 * sizeof(uint32_t), b->stream));
  FLB_BCUDA(b, cudaGetLastError());
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  b->t = 0;
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
  bdrop_graph(b);  // the captured launch refers to the old arrays
  if (b->d_start) cudaFree(b->d_start);
  b->d_start = nullptr;
  FLB_BCUDA(b, cudaMalloc(&b->d_start, start.size() * sizeof(uint32_t)));
  FLB_BCUDA(b, cudaMemcpy(b->d_order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  FLB_BCUDA(b, cudaMemcpy(b->d_start, start.data(), start.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  b->clusters = clusters;
  return FLB_OK;
}

// One launch of the batch kernel for n steps on the stream (captured or not).
flb_status bissue(flb_batch b, uint32_t n, int wm_last) {
  BatchKernel kern = pick_kernel(b->hw, b->fu);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(b->clusters * b->cluster));
  cfg.blockDim = dim3((unsigned)b->threads);
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)b->cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  FLB_BCUDA(b, cudaLaunchKernelEx(&cfg, kern, (const BatchCase*)b->d_cases, (const uint32_t*)b->d_order,
                                  (const uint32_t*)b->d_start, (const uint32_t*)b->d_tstep, n, wm_last));
  k_tadd<<<1, 1, 0, b->stream>>>(b->d_tstep, n);
  FLB_BCUDA(b, cudaGetLastError());
  return FLB_OK;
}

// n steps as one graph launch (the graph is kept for the next call with the
// same step count and configuration).
flb_status blaunch(flb_batch b, uint64_t steps, int wm_last) {
  uint64_t done = 0;
  while (done < steps) {  // at most 2^31 steps per launch
    const uint32_t n = (uint32_t)std::min<uint64_t>(steps - done, 1u << 31);
    const int wm = wm_last && done + n == steps;
    if (!b->gexec || b->g_steps != n || b->g_wm != wm || b->g_cluster != b->cluster ||
        b->g_clusters != b->clusters || b->g_threads != b->threads) {
      bdrop_graph(b);
      FLB_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      flb_status s = bissue(b, n, wm);
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
    }
    FLB_BCUDA(b, cudaGraphLaunch(b->gexec, b->stream));
    b->launches += 2;
    done += n;
  }
  b->t += steps;
  return FLB_OK;
}

// Resident clusters of the given size (0 when the size cannot launch).
int max_clusters(flb_batch b, int cs, int threads) {
  BatchKernel kern = pick_kernel(b->hw, b->fu);
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

// Timed search over cluster sizes and cluster counts: probe steps of the whole
// batch from the initial state for every candidate; the fastest wins.  The
// counts include one sized so that the cases active at a time fit in about
// half of the L2 (each cluster holds one case at a time): over thousands of
// steps such a case is stepped from L2 after its first step.  The probe is long
// enough (100 steps by default) for that reuse to show.
flb_status btune(flb_batch b, uint32_t probe_steps) {
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
  int l2 = 0;
  cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, b->device);
  // bytes a case touches per step: 9 FP32 populations, flags, wall mask
  const double case_bytes = (double)b->cells / b->n * (9.0 * 4.0 + 2.0);
  const int l2_fit = std::max(1, (int)(0.5 * (double)l2 / std::max(1.0, case_bytes)));
  struct Cand {
    int cs, clusters, threads;
  };
  std::vector<Cand> cands;
  for (int threads : {512, 1024}) {
    for (int cs : {1, 2, 4, 8, 16}) {
      const int mx = max_clusters(b, cs, threads);
      if (mx <= 0) continue;
      const int per_sm = std::max(1, nsm / cs);
      for (int k : {l2_fit, per_sm / 2, per_sm, 2 * per_sm, mx}) {
        const int cl = std::min(std::max(k, 1), std::min(mx, (int)b->n));
        bool seen = false;
        for (auto& c : cands) seen |= c.cs == cs && c.clusters == cl && c.threads == threads;
        if (!seen) cands.push_back({cs, cl, threads});
      }
    }
  }
  if (cands.empty()) return bfail(b, FLB_ERR_UNSUPPORTED, "no thread-block cluster size can launch");
  cudaEvent_t e0, e1;
  FLB_BCUDA(b, cudaEventCreate(&e0));
  FLB_BCUDA(b, cudaEventCreate(&e1));
  float best = 1e30f;
  Cand win = cands[0];
  for (const Cand& c : cands) {
    b->cluster = c.cs;
    b->threads = c.threads;
    flb_status s = bassign(b, c.clusters);
    if (s == FLB_OK) s = binit(b);
    if (s == FLB_OK) s = blaunch(b, 2, 0);  // warm-up
    if (s != FLB_OK) break;
    cudaEventRecord(e0, b->stream);
    s = blaunch(b, probe_steps, 0);
    cudaEventRecord(e1, b->stream);
    if (s != FLB_OK) break;
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      win = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  FLB_BCUDA(b, cudaGetLastError());
  b->cluster = win.cs;
  b->threads = win.threads;
  flb_status s = bassign(b, win.clusters);
  if (s != FLB_OK) return s;
  b->tuned = 1;
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
  for (uint32_t c = 0; c < n; c++) {
    b->nx[c] = cases[c].nx;
    b->ny[c] = cases[c].ny;
    b->off[c] = b->cells;
    b->cells += (size_t)cases[c].nx * cases[c].ny;
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
  const size_t M = b->cells;
  struct A {
    void** p;
    size_t bytes;
    bool need;
  } allocs[] = {
      {(void**)&b->d_f, 9 * M * sizeof(float), true},         {(void**)&b->d_rho, M * sizeof(float), true},
      {(void**)&b->d_u, 2 * M * sizeof(float), true},         {(void**)&b->d_flags, M, true},
      {(void**)&b->d_geo, M, true},                           {(void**)&b->d_nbmask, M, b->hw},
      {(void**)&b->d_tstep, 2 * sizeof(uint32_t), true},      {(void**)&b->d_cases, n * sizeof(BatchCase), true},
      {(void**)&b->d_order, n * sizeof(uint32_t), true},
  };
  for (A& a : allocs) {
    if (!a.need) continue;
    cudaError_t e = cudaMalloc(a.p, a.bytes);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMalloc"));
  }
  b->hcases.resize(n);
  for (uint32_t c = 0; c < n; c++) {
    const size_t o = b->off[c], N = (size_t)b->nx[c] * b->ny[c];
    KParams& k = b->hcases[c].kp;
    fill_case_constants(&cases[c], k);
    k.nx = b->nx[c];
    k.ny = b->ny[c];
    k.N = (uint32_t)N;
    k.f = b->d_f + 9 * o;
    for (int q = 0; q < 9; q++) k.slot[q] = b->d_f + 9 * o + (size_t)q * N;
    k.rho = b->d_rho + o;
    k.u = b->d_u + 2 * o;
    k.flags = b->d_flags + o;
    k.flags_out = b->d_flags + o;
    k.nbmask = b->hw ? b->d_nbmask + o : nullptr;
    k.tstep = b->d_tstep;
    b->hcases[c].nsegx = (b->nx[c] + 31u) / 32u;
    cudaError_t e = cudaMemcpyAsync(b->d_geo + o, cases[c].flags, N, cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMemcpyAsync"));
  }
  cudaError_t e = cudaMemcpy(b->d_cases, b->hcases.data(), n * sizeof(BatchCase), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return bail(bcuda(b, e, "cudaMemcpy"));
  flb_status s = FLB_OK;
  if (autotune) {
    s = btune(b, autotune > 1 ? (uint32_t)autotune : 100u);
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
  if (n == 0) return FLB_OK;
  BDevice g(b->device);
  return blaunch(b, n, 1);
}

FLB_API flb_status flb_batch_sync(flb_batch b) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return FLB_OK;
}

FLB_API flb_status flb_batch_reset(flb_batch b) {
  if (!b) return FLB_ERR_INVALID_ARGUMENT;
  return binit(b);
}

FLB_API flb_status flb_batch_read_field(flb_batch b, uint32_t i, int field, void* dst, int on_device) {
  if (!b || !dst || i >= b->n) return FLB_ERR_INVALID_ARGUMENT;
  BDevice g(b->device);
  const size_t o = b->off[i], N = (size_t)b->nx[i] * b->ny[i];
  const void* src = nullptr;
  size_t bytes = 0;
  switch (field) {
    case FLB_FIELD_F: src = b->d_f + 9 * o; bytes = 9 * N * sizeof(float); break;
    case FLB_FIELD_RHO: src = b->d_rho + o; bytes = N * sizeof(float); break;
    case FLB_FIELD_U: src = b->d_u + 2 * o; bytes = 2 * N * sizeof(float); break;
    case FLB_FIELD_FLAGS: src = b->d_flags + o; bytes = N; break;
    default: return bfail(b, FLB_ERR_INVALID_ARGUMENT, "the batch holds populations, density, velocity and flags");
  }
  FLB_BCUDA(b, cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               b->stream));
  FLB_BCUDA(b, cudaStreamSynchronize(b->stream));
  return FLB_OK;
}

FLB_API flb_status flb_batch_info(flb_batch b, int64_t info[7]) {
  if (!b || !info) return FLB_ERR_INVALID_ARGUMENT;
  info[0] = b->n;
  info[1] = (int64_t)b->cells;
  info[2] = (int64_t)b->t;
  info[3] = b->cluster;
  info[4] = b->clusters;
  info[5] = b->tuned;
  info[6] = b->threads;
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
