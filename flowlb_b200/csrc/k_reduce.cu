// k_reduce.cu -- FP64 mass reduction, cell census, storage codecs.
#include "launch.h"

namespace flb {

// ---- reductions and codecs --------------------------------------------------

// Per-block FP64 partial sums of the total fluid mass (see flb_total_mass).
template <class S, class C, class M, bool HW>
__global__ void __launch_bounds__(kBlock) k_mass_partial(const __grid_constant__ KParams p, uint32_t odd, int fs,
                                                         double* __restrict__ partial) {
  __shared__ double red[kBlock];
  const uint32_t tid = threadIdx.x;
  const uint32_t cell = blockIdx.x * kBlock + tid;
  double v = 0.0;
  if (cell < p.N) {
    const uint32_t x = cell % p.nx, y = cell / p.nx;
    uint32_t nb[9];
    neighbours(x, y, p.nx, p.ny, nb);
    const uint8_t* flags = p.flags;
    const uint8_t flag = flags[cell];
    if (fs) {
      const M* Ms = static_cast<const M*>(p.mass);
      const M* Ex = static_cast<const M*>(p.excess);
      int pullers = 0;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        const uint8_t nf = flags[nb[i]];
        if (p.fs_cons) {
          const uint8_t e = nf & kFGI;
          pullers += (e == kFluid || e == kInterface) && !(nf & (kWall | kMovingWall | kInlet));
        } else {
          pullers += !(nf & (kGas | kWall | kInlet));
        }
      }
      if (!(flag & (kWall | kMovingWall))) v += (double)Ms[cell];
      v += (double)Ex[cell] * (double)pullers;
    } else if (!(flag & (kGas | kWall))) {
      C f[9];
      load_in_rt<S, C, HW>(p, odd, cell, nb, HW ? p.nbmask[cell] : 0u, f);
#pragma unroll
      for (int i = 0; i < 9; i++) v += (double)f[i];
    }
  }
  red[tid] = v;
  __syncthreads();
  for (uint32_t s = kBlock / 2; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  if (tid == 0) partial[blockIdx.x] = red[0];
}

// Sums n partials in a fixed order with one block (deterministic).
__global__ void k_sum_partials(const double* __restrict__ partial, uint32_t n, double* __restrict__ out) {
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

// Census of cell types and non-finite populations: counts[0..4] = fluid,
// interface, gas, wall, non-finite.
template <class S, class C, bool HW>
__global__ void __launch_bounds__(kBlock) k_census(const __grid_constant__ KParams p, uint32_t odd,
                                                   unsigned long long* __restrict__ counts) {
  const uint32_t cell = blockIdx.x * kBlock + threadIdx.x;
  uint32_t c[5] = {0, 0, 0, 0, 0};
  if (cell < p.N) {
    const uint8_t flag = p.flags[cell];
    const uint8_t e = flag & kFGI;
    if (flag & kWall) c[3] = 1;
    else if (e == kFluid) c[0] = 1;
    else if (e == kInterface) c[1] = 1;
    else if (e == kGas) c[2] = 1;
    if (!(flag & (kGas | kWall))) {
      const uint32_t x = cell % p.nx, y = cell / p.nx;
      uint32_t nb[9];
      neighbours(x, y, p.nx, p.ny, nb);
      C f[9];
      load_in_rt<S, C, HW>(p, odd, cell, nb, HW ? p.nbmask[cell] : 0u, f);
      bool bad = false;
#pragma unroll
      for (int i = 0; i < 9; i++) bad |= !isfinite((double)f[i]);
      c[4] = bad;
    }
  }
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const uint32_t s = __reduce_add_sync(0xffffffffu, c[k]);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&counts[k], (unsigned long long)s);
  }
}

// Storage -> arithmetic type (read-back) and back (write).
template <class S, class C>
__global__ void k_decode(const S* __restrict__ F, C* __restrict__ out, uint32_t N, float inv) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= 9u * N) return;
  out[k] = Codec<S, C>::ld(F, k, (int)(k / N), inv);
}
template <class S, class C>
__global__ void k_encode(S* __restrict__ F, const C* __restrict__ in, uint32_t N, float scale) {
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;
  if (k >= 9u * N) return;
  Codec<S, C>::st(F, k, (int)(k / N), in[k], scale);
}


template <class S, class C, class M>
void launch_mass_partial(const KParams& kp, cudaStream_t st, uint32_t odd, int fs, bool hw, double* partial) {
  const dim3 g((kp.N + kBlock - 1) / kBlock);
  if (hw) k_mass_partial<S, C, M, true><<<g, kBlock, 0, st>>>(kp, odd, fs, partial);
  else k_mass_partial<S, C, M, false><<<g, kBlock, 0, st>>>(kp, odd, fs, partial);
}

void launch_sum_partials(const double* partial, uint32_t n, double* out, cudaStream_t st) {
  k_sum_partials<<<1, kBlock, 0, st>>>(partial, n, out);
}

template <class S, class C, class M>
void launch_census(const KParams& kp, cudaStream_t st, uint32_t odd, bool hw, unsigned long long* counts) {
  const dim3 g((kp.N + kBlock - 1) / kBlock);
  if (hw) k_census<S, C, true><<<g, kBlock, 0, st>>>(kp, odd, counts);
  else k_census<S, C, false><<<g, kBlock, 0, st>>>(kp, odd, counts);
}

template <class S, class C, class M>
void launch_decode(const KParams& kp, cudaStream_t st, void* out) {
  const uint64_t n = 9ull * kp.N;
  k_decode<S, C><<<dim3((unsigned)((n + kBlock - 1) / kBlock)), kBlock, 0, st>>>(static_cast<const S*>(kp.f),
                                                                                 static_cast<C*>(out), kp.N, kp.f16_inv);
}

template <class S, class C, class M>
void launch_encode(const KParams& kp, cudaStream_t st, const void* in) {
  const uint64_t n = 9ull * kp.N;
  k_encode<S, C><<<dim3((unsigned)((n + kBlock - 1) / kBlock)), kBlock, 0, st>>>(static_cast<S*>(kp.f),
                                                                                 static_cast<const C*>(in), kp.N,
                                                                                 kp.f16_scale);
}

#define FLB_INSTANTIATE(S, C, M)                                                                                 \
  template void launch_mass_partial<S, C, M>(const KParams&, cudaStream_t, uint32_t, int, bool, double*);       \
  template void launch_census<S, C, M>(const KParams&, cudaStream_t, uint32_t, bool, unsigned long long*);     \
  template void launch_decode<S, C, M>(const KParams&, cudaStream_t, void*);                                    \
  template void launch_encode<S, C, M>(const KParams&, cudaStream_t, const void*);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
