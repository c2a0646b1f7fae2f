// k_noalloc.cu -- free-surface total mass for callers that cannot allocate.
//
// Some callers may not allocate device memory at the moment they need the
// mass check: a real-time loop whose device memory budget is fixed up front
// and audited, a loop that cannot afford the implicit device synchronisation
// of cudaMalloc/cudaFree between steps, or a plug-in that only ever receives
// pointers to buffers owned by someone else.
// flb_total_mass needs a handle, whose creation allocates; this entry point
// takes plain device pointers instead and keeps its scratch (one FP64 partial
// sum per block of 256 cells) in a file-scope __device__ array of fixed size,
// which every GPU that loads the library holds until the process exits.
//
// The arithmetic and the reduction order are those of k_mass_partial /
// k_sum_partials (k_reduce.cu), so the result equals flb_total_mass bit for
// bit on the same fields.
#include <cstdio>

#include "../../include/flowlb.h"
#include "common.cuh"

namespace flb {
namespace {

constexpr uint32_t kNoAllocMaxBlocks = FLB_NOALLOC_MAX_CELLS / kBlock;

// Shared by every call on a device; holds the previous call's partial sums.
// Every slot a call reads was written earlier in the same call, so nothing
// needs clearing.  Calls that overlap on the GPU (different streams, or
// different host threads) race on it.
static __device__ __align__(256) double g_partial[kNoAllocMaxBlocks];

// Device address of g_partial in the current device's context.  In host code
// the name g_partial is only a host-side stand-in for the symbol, not a device
// address; passing it to a kernel would fault (or, where the GPU can reach
// host memory, silently use the wrong memory).  Looked up on every call: the
// lookup is a host-side query (no stream work), and an address kept from an
// earlier call would be stale after the context was reset (cudaDeviceReset
// reloads the module and its __device__ arrays).
cudaError_t scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_partial);
  if (e != cudaSuccess) return e;
  *out = static_cast<double*>(p);
  return cudaSuccess;
}

__global__ void __launch_bounds__(kBlock) k_mass_partial_noalloc(const double* __restrict__ mass,
                                                                 const double* __restrict__ excess,
                                                                 const uint8_t* __restrict__ flags, uint32_t nx,
                                                                 uint32_t ny, int cons, double* __restrict__ partial) {
  __shared__ double red[kBlock];
  const uint32_t tid = threadIdx.x;
  const uint32_t N = nx * ny;
  const uint32_t cell = blockIdx.x * kBlock + tid;
  double v = 0.0;
  if (cell < N) {
    uint32_t nb[9];
    neighbours(cell % nx, cell / nx, nx, ny, nb);
    const uint8_t flag = flags[cell];
    int pullers = 0;
#pragma unroll
    for (int i = 1; i < 9; i++) {
      const uint8_t nf = flags[nb[i]];
      if (cons) {
        const uint8_t e = nf & kFGI;
        pullers += (e == kFluid || e == kInterface) && !(nf & (kWall | kMovingWall | kInlet));
      } else {
        pullers += !(nf & (kGas | kWall | kInlet));
      }
    }
    if (!(flag & (kWall | kMovingWall))) v += mass[cell];
    v += excess[cell] * (double)pullers;
  }
  red[tid] = v;
  __syncthreads();
  for (uint32_t s = kBlock / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  if (tid == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_sum_noalloc(const double* __restrict__ partial, uint32_t n, double* __restrict__ out) {
  __shared__ double red[kBlock];
  double v = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += kBlock) v += partial[i];
  red[threadIdx.x] = v;
  __syncthreads();
  for (uint32_t s = kBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

}  // namespace
}  // namespace flb

extern "C" FLB_API flb_status flb_total_mass_noalloc(const double* mass, const double* excess,
                                                     const uint8_t* flags, uint32_t nx, uint32_t ny, int fs_mode,
                                                     double* out, void* stream) {
  using namespace flb;
  if (!mass || !excess || !flags || !out || nx < 3 || ny < 3) return FLB_ERR_INVALID_ARGUMENT;
  if (fs_mode != FLB_FS_REFERENCE && fs_mode != FLB_FS_CONSERVATIVE) return FLB_ERR_INVALID_ARGUMENT;
  const uint64_t N = (uint64_t)nx * ny;
  if (N > (uint64_t)FLB_NOALLOC_MAX_CELLS) {
    std::fprintf(stderr,
                 "flb_total_mass_noalloc: %llu cells exceed the fixed scratch of this entry point "
                 "(at most %u cells); use flb_total_mass\n",
                 (unsigned long long)N, (unsigned)FLB_NOALLOC_MAX_CELLS);
    return FLB_ERR_INVALID_ARGUMENT;
  }
  double* partial = nullptr;
  cudaError_t e = scratch_address(&partial);
  if (e != cudaSuccess) return FLB_ERR_CUDA;
  const uint32_t blocks = (uint32_t)((N + kBlock - 1) / kBlock);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_mass_partial_noalloc<<<blocks, kBlock, 0, st>>>(mass, excess, flags, nx, ny,
                                                    fs_mode == FLB_FS_CONSERVATIVE ? 1 : 0, partial);
  k_sum_noalloc<<<1, kBlock, 0, st>>>(partial, blocks, out);
  e = cudaGetLastError();
  return e == cudaSuccess ? FLB_OK : FLB_ERR_CUDA;
}
