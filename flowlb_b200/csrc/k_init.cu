// k_init.cu -- the initial state, built on the device from geometry flags.
#include "launch.h"

namespace flb {

// ---- initial state ----------------------------------------------------------

// Free-surface interface layer and fields (initData.cpp:13-37 with the bounded
// neighbour list of :39-124, initData.h:175-206).  The reference sweeps cells
// in index order and initialises each cell's fields right after visiting it;
// that makes the result a per-cell rule: a GAS cell next to a fluid source
// becomes INTERFACE, and gets m = phi = 0.5 only if some source precedes it in
// index order (otherwise it was initialised as gas).
__global__ void k_init_flags(const uint8_t* __restrict__ geo, uint8_t* __restrict__ flags, uint32_t nx, uint32_t ny,
                             int free_surface, void* mass_v, void* excess_v, void* phi_v, int mass_f64) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= nx) return;
  const uint32_t idx = x + y * nx;
  uint8_t g = geo[idx];
  if (!free_surface) {
    flags[idx] = g;
    return;
  }
  auto source = [](uint8_t v) -> bool {
    return !(v & ~(kFluid | kInlet | kOutlet)) && (v & (kFluid | kInlet));
  };
  uint8_t f = g;
  bool early = false, any = false;
  if (g == kGas) {
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        if (!dx && !dy) continue;
        const long xx = (long)x + dx, yy = (long)y + dy;
        if (xx < 0 || yy < 0 || xx >= (long)nx || yy >= (long)ny) continue;
        const uint32_t n = (uint32_t)xx + (uint32_t)yy * nx;
        if (source(geo[n])) {
          any = true;
          if (n < idx) early = true;
        }
      }
    if (any) f = kInterface;
  } else if (!(g & ~(kFluid | kInlet | kOutlet))) {
    if (g & kInlet) f = g | kFluid;
    else if (g & kOutlet) f = g | kGas;
  }
  flags[idx] = f;
  double m = 0.0, ph = 0.0;
  bool set = true;
  switch (f) {
    case kFluid:
    case kFluid | kInlet:
    case kFluid | kOutlet: m = 1.0; ph = 1.0; break;
    case kGas:
    case kGas | kOutlet: m = 0.0; ph = 0.0; break;
    case kInterface:
      m = early ? 0.5 : 0.0;
      ph = early ? 0.5 : 0.0;
      break;
    default: set = false; break;
  }
  if (!set) m = ph = 0.0;
  if (mass_f64) {
    ((double*)mass_v)[idx] = m;
    ((double*)phi_v)[idx] = ph;
    ((double*)excess_v)[idx] = 0.0;
  } else {
    ((float*)mass_v)[idx] = (float)m;
    ((float*)phi_v)[idx] = (float)ph;
    ((float*)excess_v)[idx] = 0.0f;
  }
}

// Solid-neighbour mask for half-way walls.
__global__ void k_nbmask(const uint8_t* __restrict__ flags, uint8_t* __restrict__ nbmask, uint32_t nx, uint32_t ny) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= nx) return;
  uint32_t nb[9];
  neighbours(x, y, nx, ny, nb);
  uint32_t m = 0;
#pragma unroll
  for (int i = 1; i < 9; i++) m |= (flags[nb[i]] & kWall) ? (1u << (i - 1)) : 0u;
  nbmask[x + y * nx] = (uint8_t)m;
}

// Single-phase chunk map: bit c % 32 of plain[c / 32] is set when the four
// cells 4c..4c+3 are all plain FLUID (no inlet, outlet, wall or gas) with no
// wall neighbour, so that the vector stream-collide can skip reading their
// flag and neighbour-mask bytes.  nbmask may be null (no half-way walls).
__global__ void k_plain_chunks(const uint8_t* __restrict__ flags, const uint8_t* __restrict__ nbmask, uint32_t N,
                               uint32_t* __restrict__ plain) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nchunk = (N + 3u) / 4u;
  bool pl = c < nchunk;
  if (pl) {
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      const uint32_t cell = 4u * c + k;
      pl = pl && cell < N && flags[cell] == kFluid && (!nbmask || nbmask[cell] == 0);
    }
  }
  const uint32_t b = __ballot_sync(0xffffffffu, pl);
  if ((threadIdx.x & 31u) == 0u && c < nchunk) plain[c >> 5] = b;
}

void launch_plain_chunks(const uint8_t* flags, const uint8_t* nbmask, uint32_t N, uint32_t* plain, cudaStream_t st) {
  const uint32_t nchunk = (N + 3u) / 4u;
  k_plain_chunks<<<(nchunk + kBlock - 1) / kBlock, kBlock, 0, st>>>(flags, nbmask, N, plain);
}

// f = feq(rho=1, u) with the host's double arithmetic (initEquilibriumDDF2Q9,
// initData.h:75-100) stored with the t=1 pattern (initData.h:102-112, :155);
// rho = 1; u = inlet velocity on INLET cells, else 0 (initData.h:125-148).
// With half-way walls wall cells store nothing.
template <class S, class C, bool HW>
__global__ void k_init_ddf(const __grid_constant__ KParams p, const uint8_t* __restrict__ geo) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t N = p.N, idx = x + y * p.nx;
  C* R = static_cast<C*>(p.rho);
  C* U = static_cast<C*>(p.u);
  const uint8_t g = geo[idx];
  C ux, uy;
  if (g & kInlet) {
    ux = (C)p.inlet_ux;
    uy = (C)p.inlet_uy;
  } else {
    ux = 0;
    uy = 0;
  }
  U[idx] = ux;
  U[idx + N] = uy;
  const double rho = 1.0;
  R[idx] = (C)rho;
  if (HW && (g & kWall)) return;
  const double u2 = 3.0 * (ux * ux + uy * uy);
  const double rhow14 = wgt<C>(1) * rho;
  const double rhow58 = wgt<C>(5) * rho;
  ux *= 3.0;
  uy *= 3.0;
  const double u0 = ux - uy;
  const double u1 = ux + uy;
  C feq[9];
  feq[0] = (C)(wgt<C>(0) * rho * (1.0 - 0.5 * u2));
  feq[1] = (C)(rhow14 * (1.0 + ux - 0.5 * u2 + 0.5 * ux * ux));
  feq[2] = (C)(rhow14 * (1.0 - ux - 0.5 * u2 + 0.5 * ux * ux));
  feq[3] = (C)(rhow14 * (1.0 + uy - 0.5 * u2 + 0.5 * uy * uy));
  feq[4] = (C)(rhow14 * (1.0 - uy - 0.5 * u2 + 0.5 * uy * uy));
  feq[5] = (C)(rhow58 * (1.0 + u1 - 0.5 * u2 + 0.5 * u1 * u1));
  feq[6] = (C)(rhow58 * (1.0 - u1 - 0.5 * u2 + 0.5 * u1 * u1));
  feq[7] = (C)(rhow58 * (1.0 + u0 - 0.5 * u2 + 0.5 * u0 * u0));
  feq[8] = (C)(rhow58 * (1.0 - u0 - 0.5 * u2 + 0.5 * u0 * u0));
  uint32_t nb[9];
  neighbours(x, y, p.nx, p.ny, nb);
  store_post<S, C, true>(p, idx, nb, feq);
}


void launch_init_flags(const uint8_t* geo, uint8_t* flags, uint32_t nx, uint32_t ny, int free_surface, void* mass,
                       void* excess, void* phi, int mass_f64, cudaStream_t st) {
  k_init_flags<<<dim3((nx + kBlock - 1) / kBlock, ny), kBlock, 0, st>>>(geo, flags, nx, ny, free_surface, mass, excess,
                                                                        phi, mass_f64);
}

void launch_nbmask(const uint8_t* geo, uint8_t* nbmask, uint32_t nx, uint32_t ny, cudaStream_t st) {
  k_nbmask<<<dim3((nx + kBlock - 1) / kBlock, ny), kBlock, 0, st>>>(geo, nbmask, nx, ny);
}

template <class S, class C, class M>
void launch_init_ddf(const KParams& kp, cudaStream_t st, const uint8_t* geo, bool hw) {
  const dim3 g((kp.nx + kBlock - 1) / kBlock, kp.ny);
  if (hw) k_init_ddf<S, C, true><<<g, kBlock, 0, st>>>(kp, geo);
  else k_init_ddf<S, C, false><<<g, kBlock, 0, st>>>(kp, geo);
}

#define FLB_INSTANTIATE(S, C, M) \
  template void launch_init_ddf<S, C, M>(const KParams&, cudaStream_t, const uint8_t*, bool);
FLB_FOR_EACH_VARIANT(FLB_INSTANTIATE)
#undef FLB_INSTANTIATE

}  // namespace flb
