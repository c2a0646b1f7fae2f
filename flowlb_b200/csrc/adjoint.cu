// adjoint.cu -- discrete adjoint of the single-phase step with a Brinkman
// porosity field (no counterpart in the reference).
//
// Forward model, per fluid cell and step (state: post-collision populations;
// pull streaming with half-way walls; x periodic):
//   f_i   = gathered f[i] from x - c_i (f[opp i] of the cell itself when that
//           neighbour is a wall)
//   rho   = sum f_i,  j = sum c_i f_i,  v = j (1 / rho)
//   u     = (v + g/2) (1 / (1 + s/2))            (Guo, F = rho (g - s u))
//   F     = rho (g - s u)
//   feq_i = w_i rho (1 + 3 cu + 4.5 cu^2 - 1.5 u.u),    cu = c_i.u
//   F_i   = w_i (3 (c_i.F - u.F) + 9 cu c_i.F)
//   out_i = (1 - w) f_i + w feq_i + (1 - w/2) F_i
// s in [0,1] is a drag coefficient per step: s = 0 free fluid, s = 1 removes
// about two thirds of the momentum every step (a quasi-solid culvert).
// Objective: J = (1/W) sum over the last W steps of sum_y rho u_x in the last
// column x = nx - 1.
//
// The backward step is the hand-derived reverse mode of that cell update:
// with mu_i = dJ/d out_i it forms dJ/d f_i and scatters it to the gathered
// source slot (each source slot is gathered by exactly one cell, so no
// atomics), and accumulates dJ/ds per cell (FP64) and dJ/dg per block (FP64,
// fixed-order tree, so the result is deterministic).
//
// Checkpointing: the forward pass keeps the state every K steps; the backward
// pass recomputes each K-step segment from its checkpoint, keeping rho and v
// of every step (all the backward step needs), and walks it backwards.  Each segment (forward or backward) is one
// CUDA graph replayed with its time offset and checkpoint slot read from a
// small device descriptor.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "launch.h"

namespace flb {
namespace {

constexpr int kAdjBlock = 256;
// resident blocks per SM the reverse step is compiled for: four (at most 64
// registers a thread; the FP64 step spills 44 bytes) measured faster than the
// 92-register build's two on a B200 (FP64 backward of the 1024x256 case 68.1
// -> 62.7 ms; three blocks, 80 registers: 67.4 ms)
constexpr int kAdjBwdBlocks = 4;
// opposite direction (directions of lattice.cuh: i and i+1 opposite for odd i)
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

template <class T>
struct AdjParams {
  uint32_t nx, ny, N;
  const uint8_t* flags;   // FLUID / WALL
  const uint8_t* srcw;    // bit i-1: the source x - c_i of population i >= 1 is a wall
  const T* s;             // drag coefficient per cell
  const T* id;            // 1 / (1 + s/2) per cell (k_por_inv_d, whenever s is set)
  T om, omc, kk;          // w, 1 - w, 1 - w/2
  T gx, gy;
  T winv;                 // 1 / W
  uint64_t steps, window;
};

struct SegDesc {
  uint64_t t0;  // time step of the segment's first step
  void* ckpt;   // checkpoint slot of the segment
};

template <class T>
__device__ __forceinline__ T wq(int i) {
  return i == 0 ? T(4) / T(9) : (i < 5 ? T(1) / T(9) : T(1) / T(36));
}

// Source cells x - c_i of a cell: columns xm = x-1, xp = x+1, rows ym, yp
// (periodic).
struct Nb {
  uint32_t src[9];
};
__device__ __forceinline__ Nb sources(uint32_t x, uint32_t y, uint32_t nx, uint32_t ny) {
  const uint32_t xm = x == 0 ? nx - 1 : x - 1, xp = x + 1 == nx ? 0 : x + 1;
  const uint32_t rm = (y == 0 ? ny - 1 : y - 1) * nx, r0 = y * nx, rp = (y + 1 == ny ? 0 : y + 1) * nx;
  Nb n;
  n.src[0] = x + r0;
  n.src[1] = xm + r0;  // population 1 (+x) comes from x - 1
  n.src[2] = xp + r0;
  n.src[3] = x + rm;
  n.src[4] = x + rp;
  n.src[5] = xm + rm;
  n.src[6] = xp + rp;
  n.src[7] = xm + rp;  // population 7 (+x, -y) comes from (x - 1, y + 1)
  n.src[8] = xp + rm;
  return n;
}

// Gathers the 9 inputs of a cell from the state fin.
template <class T>
__device__ __forceinline__ void gather(const AdjParams<T>& p, const T* __restrict__ fin, uint32_t idx, uint32_t sw,
                                       const Nb& nb, T* f) {
  const uint32_t N = p.N;
  f[0] = fin[idx];
#pragma unroll
  for (int i = 1; i < 9; i++) f[i] = ((sw >> (i - 1)) & 1u) ? fin[(uint32_t)opp(i) * N + idx] : fin[(uint32_t)i * N + nb.src[i]];
}

// Forward intermediates of one cell.  The two divisions of the update are
// taken once as reciprocals (ir = 1 / rho, id = 1 / d) and multiplied in, in
// the forward and in the reverse step alike (an FP64 division is a long
// instruction sequence; the reverse step would otherwise need ten).
template <class T>
struct Cell {
  T rho, ir, vx, vy, id, ux, uy, Fx, Fy, usq, uF;
};

// the rest of the intermediates from rho, v, s and id = 1 / (1 + s/2), the
// latter computed once per porosity field by k_por_inv_d with the same
// operations
template <class T>
__device__ __forceinline__ void cell_rest(const AdjParams<T>& p, Cell<T>& c, T s, T id) {
  c.id = id;
  c.ux = (c.vx + T(0.5) * p.gx) * c.id;
  c.uy = (c.vy + T(0.5) * p.gy) * c.id;
  c.Fx = c.rho * (p.gx - s * c.ux);
  c.Fy = c.rho * (p.gy - s * c.uy);
  c.usq = c.ux * c.ux + c.uy * c.uy;
  c.uF = c.ux * c.Fx + c.uy * c.Fy;
}

template <class T>
__device__ __forceinline__ Cell<T> cell_state(const AdjParams<T>& p, const T* f, T s, T id) {
  Cell<T> c;
  c.rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const T jx = f[1] - f[2] + f[5] - f[6] + f[7] - f[8];
  const T jy = f[3] - f[4] + f[5] - f[6] - f[7] + f[8];
  c.ir = T(1) / c.rho;
  c.vx = jx * c.ir;
  c.vy = jy * c.ir;
  cell_rest(p, c, s, id);
  return c;
}


// One forward step fin -> fout.  obj: add rho u_x of the last column to jrow.
// ckpt (segment's first step only): the input state is also copied there.
template <class T>
__global__ void __launch_bounds__(kAdjBlock) k_por_fwd(const AdjParams<T> p, const T* __restrict__ fin,
                                                       T* __restrict__ fout, double* __restrict__ jrow,
                                                       const SegDesc* __restrict__ seg, uint32_t j, int copy_ckpt,
                                                       T* __restrict__ mac) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= p.nx) return;
  const uint32_t idx = x + y * p.nx, N = p.N;
  if (copy_ckpt) {
    T* ck = static_cast<T*>(seg->ckpt);
#pragma unroll
    for (int i = 0; i < 9; i++) ck[(uint32_t)i * N + idx] = fin[(uint32_t)i * N + idx];
  }
  if (p.flags[idx] & kWall) return;
  const Nb nb = sources(x, y, p.nx, p.ny);
  T f[9];
  gather(p, fin, idx, p.srcw[idx], nb, f);
  const T s = p.s[idx];
  const Cell<T> c = cell_state(p, f, s, p.id[idx]);
  if (mac) {  // the backward step's inputs: rho and v = j / rho
    mac[idx] = c.rho;
    mac[N + idx] = c.vx;
    mac[2 * N + idx] = c.vy;
  }
  // opposite directions i, i+1 share the even part E and flip the odd part O:
  // feq_i = w rho (base + 4.5 cu^2) + w rho 3 cu,  F_i = w (9 cu cF - 3 uF) + w 3 cF
  const T base = T(1) - T(1.5) * c.usq;
  fout[idx] = p.omc * f[0] + p.om * (wq<T>(0) * c.rho * base) + p.kk * (wq<T>(0) * (T(-3) * c.uF));
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int i = 2 * q + 1;
    const T cu = q == 0 ? c.ux : (q == 1 ? c.uy : (q == 2 ? c.ux + c.uy : c.ux - c.uy));
    const T cF = q == 0 ? c.Fx : (q == 1 ? c.Fy : (q == 2 ? c.Fx + c.Fy : c.Fx - c.Fy));
    const T w = wq<T>(i);
    const T wr = w * c.rho;
    const T E = p.om * (wr * (base + T(4.5) * cu * cu)) + p.kk * (w * (T(9) * cu * cF - T(3) * c.uF));
    const T O = p.om * (wr * (T(3) * cu)) + p.kk * (w * (T(3) * cF));
    fout[(uint32_t)i * N + idx] = p.omc * f[i] + E + O;
    fout[(uint32_t)(i + 1) * N + idx] = p.omc * f[i + 1] + E - O;
  }
  if (jrow && x + 1 == p.nx) {
    const uint64_t t = seg->t0 + j;
    if (t + p.window >= p.steps) jrow[y] += (double)(c.rho * c.ux);
  }
}

// One backward step: mac holds rho, v_x, v_y of step t (written by its forward
// recomputation), lam_next = dJ/d(output of step t), lam = dJ/d(input of step
// t) (scattered).  sbar: dJ/ds per cell; gpart: dJ/dg per block (2 doubles per
// block).  The update's derivative needs no population itself, only rho and v.
template <class T>
__global__ void __launch_bounds__(kAdjBlock, kAdjBwdBlocks) k_por_bwd(const AdjParams<T> p, const T* __restrict__ mac,
                                                       const T* __restrict__ lam_next, T* __restrict__ lam,
                                                       double* __restrict__ sbar, double* __restrict__ gpart,
                                                       const SegDesc* __restrict__ seg, uint32_t j) {
  __shared__ double red[2][kAdjBlock / 32];
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  double gxb_d = 0.0, gyb_d = 0.0;
  if (x < p.nx) {
    const uint32_t idx = x + y * p.nx, N = p.N;
    if (!(p.flags[idx] & kWall)) {
      const uint32_t sw = p.srcw[idx];
      const Nb nb = sources(x, y, p.nx, p.ny);
      const T s = p.s[idx];
      Cell<T> c;
      c.rho = mac[idx];
      c.ir = T(1) / c.rho;
      c.vx = mac[N + idx];
      c.vy = mac[2 * N + idx];
      cell_rest(p, c, s, p.id[idx]);
      const T base = T(1) - T(1.5) * c.usq;
      T fb[9];
      const T m0 = lam_next[idx];
      fb[0] = p.omc * m0;
      T rhob = p.om * m0 * wq<T>(0) * base;
      T usqb = p.om * m0 * wq<T>(0) * c.rho * T(-1.5);
      T uFb = p.kk * m0 * wq<T>(0) * T(-3);
      T uxb = 0, uyb = 0, Fxb = 0, Fyb = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        const T mi = lam_next[(uint32_t)i * N + idx], mo = lam_next[(uint32_t)(i + 1) * N + idx];
        fb[i] = p.omc * mi;
        fb[i + 1] = p.omc * mo;
        const T Sb = mi + mo, Db = mi - mo;  // adjoints of E and O
        const T cu = q == 0 ? c.ux : (q == 1 ? c.uy : (q == 2 ? c.ux + c.uy : c.ux - c.uy));
        const T cF = q == 0 ? c.Fx : (q == 1 ? c.Fy : (q == 2 ? c.Fx + c.Fy : c.Fx - c.Fy));
        const T w = wq<T>(i);
        const T wr = w * c.rho;
        rhob += Sb * p.om * w * (base + T(4.5) * cu * cu) + Db * p.om * w * (T(3) * cu);
        usqb += Sb * p.om * wr * T(-1.5);
        uFb += Sb * p.kk * w * T(-3);
        const T cub = Sb * p.om * wr * T(9) * cu + Sb * p.kk * w * T(9) * cF + Db * p.om * wr * T(3);
        const T cFb = Sb * p.kk * w * T(9) * cu + Db * p.kk * w * T(3);
        // cu = cx ux + cy uy, cF = cx Fx + cy Fy for the odd direction i
        if (q == 0) {
          uxb += cub;
          Fxb += cFb;
        } else if (q == 1) {
          uyb += cub;
          Fyb += cFb;
        } else if (q == 2) {
          uxb += cub;
          uyb += cub;
          Fxb += cFb;
          Fyb += cFb;
        } else {
          uxb += cub;
          uyb -= cub;
          Fxb += cFb;
          Fyb -= cFb;
        }
      }
      // usq = ux ux + uy uy, uF = ux Fx + uy Fy
      uxb += usqb * T(2) * c.ux + uFb * c.Fx;
      uyb += usqb * T(2) * c.uy + uFb * c.Fy;
      Fxb += uFb * c.ux;
      Fyb += uFb * c.uy;
      if (x + 1 == p.nx) {
        const uint64_t t = seg->t0 + j;
        if (t + p.window >= p.steps) {
          rhob += c.ux * p.winv;
          uxb += c.rho * p.winv;
        }
      }
      // F = rho (g - s u)
      rhob += Fxb * (p.gx - s * c.ux) + Fyb * (p.gy - s * c.uy);
      uxb += -s * c.rho * Fxb;
      uyb += -s * c.rho * Fyb;
      T sb = -c.rho * (Fxb * c.ux + Fyb * c.uy);
      T gxb = c.rho * Fxb, gyb = c.rho * Fyb;
      // u = (v + g/2) id, id = 1 / d, d = 1 + s/2
      const T vxb = uxb * c.id, vyb = uyb * c.id;
      sb += T(-0.5) * (uxb * c.ux + uyb * c.uy) * c.id;
      gxb += T(0.5) * uxb * c.id;
      gyb += T(0.5) * uyb * c.id;
      // v = j ir, ir = 1 / rho
      const T jxb = vxb * c.ir, jyb = vyb * c.ir;
      rhob += -(vxb * c.vx + vyb * c.vy) * c.ir;
      lam[idx] = fb[0] + rhob;
#pragma unroll
      for (int i = 1; i < 9; i++) {
        const T v = fb[i] + rhob + jxb * (T)cx(i) + jyb * (T)cy(i);
        if ((sw >> (i - 1)) & 1u) lam[(uint32_t)opp(i) * N + idx] = v;
        else lam[(uint32_t)i * N + nb.src[i]] = v;
      }
      sbar[idx] += (double)sb;
      gxb_d = (double)gxb;
      gyb_d = (double)gyb;
    }
  }
  // fixed-order tree: within each warp by shuffles, then over the warps
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    gxb_d += __shfl_down_sync(0xffffffffu, gxb_d, o);
    gyb_d += __shfl_down_sync(0xffffffffu, gyb_d, o);
  }
  if (lane == 0) {
    red[0][warp] = gxb_d;
    red[1][warp] = gyb_d;
  }
  __syncthreads();
  if (warp == 0) {
    constexpr int kWarps = kAdjBlock / 32;
    double a0 = lane < (uint32_t)kWarps ? red[0][lane] : 0.0, a1 = lane < (uint32_t)kWarps ? red[1][lane] : 0.0;
#pragma unroll
    for (int o = kWarps / 2; o > 0; o >>= 1) {
      a0 += __shfl_down_sync(0xffffffffu, a0, o);
      a1 += __shfl_down_sync(0xffffffffu, a1, o);
    }
    if (lane == 0) {
      const uint32_t b = blockIdx.x + blockIdx.y * gridDim.x;
      gpart[2 * b] += a0;
      gpart[2 * b + 1] += a1;
    }
  }
}

// id = 1 / (1 + s/2) per cell
template <class T>
__global__ void k_por_inv_d(const T* __restrict__ s, T* __restrict__ id, uint32_t N) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) id[k] = T(1) / (T(1) + T(0.5) * s[k]);
}

// state = w_i (rest), also used to reset the adjoint to zero (zero = 1)
template <class T>
__global__ void k_por_fill(T* f, uint32_t N, int zero) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < 9 * N) f[k] = zero ? T(0) : wq<T>((int)(k / N));
}

// tape[0] = checkpoint of the segment
template <class T>
__global__ void k_por_load(T* dst, const SegDesc* __restrict__ seg, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[k] = static_cast<const T*>(seg->ckpt)[k];
}

__global__ void k_srcw(const uint8_t* __restrict__ flags, uint8_t* __restrict__ srcw, uint32_t nx, uint32_t ny) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= nx) return;
  uint32_t m = 0;
#pragma unroll
  for (int i = 1; i < 9; i++) {
    const uint32_t xs = cx(i) > 0 ? (x == 0 ? nx - 1 : x - 1) : (cx(i) < 0 ? (x + 1 == nx ? 0 : x + 1) : x);
    const uint32_t ys = cy(i) > 0 ? (y == 0 ? ny - 1 : y - 1) : (cy(i) < 0 ? (y + 1 == ny ? 0 : y + 1) : y);
    if (flags[xs + ys * nx] & kWall) m |= 1u << (i - 1);
  }
  srcw[x + y * nx] = (uint8_t)m;
}

}  // namespace
}  // namespace flb

using namespace flb;

struct flb_adjoint_s {
  flb_adjoint_desc d{};
  uint32_t nx = 0, ny = 0, N = 0, K = 0, nseg = 0;
  size_t ts = 4;  // bytes of the arithmetic type
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint8_t *d_flags = nullptr, *d_srcw = nullptr;
  void* d_s = nullptr;
  void* d_id = nullptr;
  void* d_state[2] = {nullptr, nullptr};
  void* d_ckpt = nullptr;  // nseg states
  void* d_tape = nullptr;  // 2 x K x (rho, v_x, v_y)
  void* d_rstate[2] = {nullptr, nullptr};  // states of the recomputation
  void* d_lam[2] = {nullptr, nullptr};
  double* d_sbar = nullptr;
  double* d_gpart = nullptr;
  double* d_jrow = nullptr;
  SegDesc* d_seg = nullptr;   // [0] segment stepped, [1] segment recomputed
  SegDesc* h_seg = nullptr;   // pinned copy
  uint32_t gx_blocks = 0, nblocks = 0;
  double gx = 0, gy = 0;
  bool forward_done = false;
  cudaGraphExec_t g_fwd = nullptr, g_back = nullptr, g_rec_b[2] = {nullptr, nullptr}, g_pipe[2] = {nullptr, nullptr};
  cudaStream_t side = nullptr;  // second branch of the pipelined backward graphs
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  double ms_fwd = 0, ms_bwd = 0;
  std::string err;
};

namespace {

flb_status afail(flb_adjoint a, flb_status s, const std::string& m) {
  if (a) a->err = m;
  return s;
}
#define FLB_ACUDA(a, call)                                                                              \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return afail((a), e_ == cudaErrorMemoryAllocation ? FLB_ERR_OUT_OF_MEMORY : FLB_ERR_CUDA,          \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                                 \
  } while (0)

struct ADevice {
  int prev = -1;
  explicit ADevice(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~ADevice() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <class T>
AdjParams<T> params(flb_adjoint a) {
  AdjParams<T> p;
  p.nx = a->nx;
  p.ny = a->ny;
  p.N = a->N;
  p.flags = a->d_flags;
  p.srcw = a->d_srcw;
  p.s = static_cast<const T*>(a->d_s);
  p.id = static_cast<const T*>(a->d_id);
  const T tau = (T)a->d.tau;
  p.om = T(1) / tau;
  p.omc = T(1) - p.om;
  p.kk = T(1) - T(0.5) * p.om;
  p.gx = (T)a->gx;
  p.gy = (T)a->gy;
  p.winv = T(1) / (T)a->d.window;
  p.steps = a->d.steps;
  p.window = a->d.window;
  return p;
}

void adrop_graphs(flb_adjoint a) {
  cudaGraphExec_t* gs[] = {&a->g_fwd, &a->g_back, &a->g_rec_b[0], &a->g_rec_b[1], &a->g_pipe[0], &a->g_pipe[1]};
  for (cudaGraphExec_t* g : gs) {
    if (*g) cudaGraphExecDestroy(*g);
    *g = nullptr;
  }
}

void afree(flb_adjoint a) {
  adrop_graphs(a);
  void* bufs[] = {a->d_flags, a->d_srcw,   a->d_s,    a->d_id,       a->d_state[0], a->d_state[1], a->d_ckpt, a->d_tape,
                  a->d_lam[0], a->d_lam[1], a->d_sbar, a->d_gpart,    a->d_jrow,     a->d_seg,
                  a->d_rstate[0], a->d_rstate[1]};
  for (void* p : bufs)
    if (p) cudaFree(p);
  if (a->h_seg) cudaFreeHost(a->h_seg);
  if (a->ev_fork) cudaEventDestroy(a->ev_fork);
  if (a->ev_join) cudaEventDestroy(a->ev_join);
  if (a->side) cudaStreamDestroy(a->side);
  if (a->own_stream && a->stream) cudaStreamDestroy(a->stream);
}

template <class T>
void* slot_state(void* base, uint32_t k, uint32_t N) {
  return static_cast<T*>(base) + (size_t)k * 9 * N;
}

// Captures the segment graphs:
//  fwd:   K steps state[0] -> state[1] -> ... (K even: ends in state[0]), the
//         first step also copying its input to the segment's checkpoint
//         (descriptor d_seg[0]);
//  rec:   the recomputation of one segment from its checkpoint (descriptor
//         d_seg[1]) through the spare state buffers, keeping rho and v of each
//         step in tape[b];
//  back:  the K backward steps of one segment (descriptor d_seg[0]) from
//         tape[b], lam[0] -> lam[1] -> ... (ends in lam[0]);
//  pipe[b]: back from tape[b] and, on a second branch running at the same
//         time, rec of the segment before it into tape[b ^ 1].
template <class T>
flb_status capture(flb_adjoint a) {
  adrop_graphs(a);
  const AdjParams<T> p = params<T>(a);
  const dim3 grid(a->gx_blocks, a->ny), block(kAdjBlock);
  const uint32_t N = a->N, K = a->K, n9 = 9 * N, n3 = 3 * N;
  T* st[2] = {static_cast<T*>(a->d_state[0]), static_cast<T*>(a->d_state[1])};
  T* rs[2] = {static_cast<T*>(a->d_rstate[0]), static_cast<T*>(a->d_rstate[1])};
  T* lam[2] = {static_cast<T*>(a->d_lam[0]), static_cast<T*>(a->d_lam[1])};
  T* tape[2] = {static_cast<T*>(a->d_tape), static_cast<T*>(a->d_tape) + (size_t)K * n3};
  auto emit_rec = [&](cudaStream_t sm, int b) {
    k_por_load<T><<<(n9 + 255) / 256, 256, 0, sm>>>(rs[0], a->d_seg + 1, n9);
    for (uint32_t j = 0; j < K; j++)
      k_por_fwd<T><<<grid, block, 0, sm>>>(p, rs[j & 1], rs[(j + 1) & 1], nullptr, a->d_seg + 1, j, 0,
                                          tape[b] + (size_t)j * n3);
  };
  auto emit_back = [&](cudaStream_t sm, int b) {
    for (uint32_t q = 0; q < K; q++) {
      const uint32_t j = K - 1 - q;
      k_por_bwd<T><<<grid, block, 0, sm>>>(p, tape[b] + (size_t)j * n3, lam[q & 1], lam[(q + 1) & 1], a->d_sbar,
                                          a->d_gpart, a->d_seg, j);
    }
  };
  auto finish = [&](cudaGraphExec_t* out) -> flb_status {
    cudaGraph_t g = nullptr;
    FLB_ACUDA(a, cudaStreamEndCapture(a->stream, &g));
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    FLB_ACUDA(a, e);
    return FLB_OK;
  };
  flb_status s;
  FLB_ACUDA(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
  for (uint32_t j = 0; j < K; j++)
    k_por_fwd<T><<<grid, block, 0, a->stream>>>(p, st[j & 1], st[(j + 1) & 1], a->d_jrow, a->d_seg, j, j == 0,
                                                nullptr);
  if ((s = finish(&a->g_fwd)) != FLB_OK) return s;
  for (int b = 0; b < 2; b++) {
    FLB_ACUDA(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
    emit_rec(a->stream, b);
    if ((s = finish(&a->g_rec_b[b])) != FLB_OK) return s;
  }
  FLB_ACUDA(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
  emit_back(a->stream, 0);
  if ((s = finish(&a->g_back)) != FLB_OK) return s;
  for (int b = 0; b < 2; b++) {
    FLB_ACUDA(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
    FLB_ACUDA(a, cudaEventRecord(a->ev_fork, a->stream));
    FLB_ACUDA(a, cudaStreamWaitEvent(a->side, a->ev_fork, 0));
    emit_rec(a->side, b ^ 1);
    emit_back(a->stream, b);
    FLB_ACUDA(a, cudaEventRecord(a->ev_join, a->side));
    FLB_ACUDA(a, cudaStreamWaitEvent(a->stream, a->ev_join, 0));
    if ((s = finish(&a->g_pipe[b])) != FLB_OK) return s;
  }
  return FLB_OK;
}

// Descriptors: d_seg[0] for the segment being stepped forward or backward,
// d_seg[1] for the segment being recomputed.
flb_status set_seg(flb_adjoint a, int slot, uint32_t k) {
  FLB_ACUDA(a, cudaMemcpyAsync(a->d_seg + slot, a->h_seg + k, sizeof(SegDesc), cudaMemcpyHostToDevice, a->stream));
  return FLB_OK;
}

template <class T>
flb_status forward(flb_adjoint a, double* J) {
  const uint32_t N = a->N;
  k_por_fill<T><<<(9 * N + 255) / 256, 256, 0, a->stream>>>(static_cast<T*>(a->d_state[0]), N, 0);
  FLB_ACUDA(a, cudaMemsetAsync(a->d_jrow, 0, a->ny * sizeof(double), a->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, a->stream);
  for (uint32_t k = 0; k < a->nseg; k++) {
    flb_status s = set_seg(a, 0, k);
    if (s != FLB_OK) return s;
    FLB_ACUDA(a, cudaGraphLaunch(a->g_fwd, a->stream));
  }
  cudaEventRecord(e1, a->stream);
  std::vector<double> jrow(a->ny);
  FLB_ACUDA(a, cudaMemcpyAsync(jrow.data(), a->d_jrow, a->ny * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
  FLB_ACUDA(a, cudaStreamSynchronize(a->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  a->ms_fwd = ms;
  double sum = 0;
  for (double v : jrow) sum += v;
  *J = sum / (double)a->d.window;
  a->forward_done = true;
  return FLB_OK;
}

template <class T>
flb_status backward(flb_adjoint a, double* dJds, double* dJdg) {
  const uint32_t N = a->N;
  k_por_fill<T><<<(9 * N + 255) / 256, 256, 0, a->stream>>>(static_cast<T*>(a->d_lam[0]), N, 1);
  FLB_ACUDA(a, cudaMemsetAsync(a->d_sbar, 0, N * sizeof(double), a->stream));
  FLB_ACUDA(a, cudaMemsetAsync(a->d_gpart, 0, 2 * a->nblocks * sizeof(double), a->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, a->stream);
  // the last segment's recomputation, then each segment's backward steps with
  // the recomputation of the one before it alongside, then segment 0's
  // backward steps (tape[k & 1] holds segment k)
  const uint32_t last = a->nseg - 1;
  flb_status s = set_seg(a, 1, last);
  if (s != FLB_OK) return s;
  FLB_ACUDA(a, cudaGraphLaunch(a->g_rec_b[last & 1], a->stream));
  for (uint32_t k = last; k >= 1; k--) {
    if ((s = set_seg(a, 0, k)) != FLB_OK || (s = set_seg(a, 1, k - 1)) != FLB_OK) return s;
    FLB_ACUDA(a, cudaGraphLaunch(a->g_pipe[k & 1], a->stream));
  }
  if ((s = set_seg(a, 0, 0)) != FLB_OK) return s;
  FLB_ACUDA(a, cudaGraphLaunch(a->g_back, a->stream));
  cudaEventRecord(e1, a->stream);
  std::vector<double> gp(2 * a->nblocks);
  if (dJds)
    FLB_ACUDA(a, cudaMemcpyAsync(dJds, a->d_sbar, N * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
  FLB_ACUDA(a, cudaMemcpyAsync(gp.data(), a->d_gpart, gp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               a->stream));
  FLB_ACUDA(a, cudaStreamSynchronize(a->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  a->ms_bwd = ms;
  if (dJdg) {
    double sx = 0, sy = 0;
    for (uint32_t b = 0; b < a->nblocks; b++) {
      sx += gp[2 * b];
      sy += gp[2 * b + 1];
    }
    dJdg[0] = sx;
    dJdg[1] = sy;
  }
  return FLB_OK;
}

template <class T>
flb_status upload_s(flb_adjoint a, const double* s) {
  std::vector<T> v(a->N);
  for (uint32_t k = 0; k < a->N; k++) v[k] = (T)s[k];
  // on the handle's stream: a plain cudaMemcpy from pageable memory may return
  // before its data reach the device, and the handle's non-blocking stream is
  // not ordered after it
  FLB_ACUDA(a, cudaMemcpyAsync(a->d_s, v.data(), a->N * sizeof(T), cudaMemcpyHostToDevice, a->stream));
  k_por_inv_d<T><<<(a->N + 255) / 256, 256, 0, a->stream>>>(static_cast<const T*>(a->d_s), static_cast<T*>(a->d_id),
                                                            a->N);
  FLB_ACUDA(a, cudaGetLastError());
  FLB_ACUDA(a, cudaStreamSynchronize(a->stream));
  return FLB_OK;
}

}  // namespace

extern "C" {

FLB_API void flb_adjoint_desc_init(flb_adjoint_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->precision = 32;
  d->tau = 0.6;
  d->steps = 4096;
  d->window = 512;
  d->checkpoint_every = 64;
  d->device = -1;
}

FLB_API flb_status flb_adjoint_create(const flb_adjoint_desc* d, flb_adjoint* out) {
  if (!d || !out || !d->flags || !d->porosity) return FLB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const uint64_t N = (uint64_t)d->nx * d->ny;
  const char* why = nullptr;
  if (d->nx < 3 || d->ny < 3 || 9 * N >= (1ull << 32)) why = "grid size";
  else if (d->precision != 32 && d->precision != 64) why = "precision must be 32 or 64";
  else if (!(d->tau > 0.5)) why = "tau must be > 0.5";
  else if (d->checkpoint_every < 2 || d->checkpoint_every % 2 || d->steps == 0 || d->steps % d->checkpoint_every)
    why = "steps must be a positive multiple of an even checkpoint_every";
  else if (d->window == 0 || d->window > d->steps) why = "window must be in [1, steps]";
  if (why) {
    std::fprintf(stderr, "flb_adjoint_create: %s\n", why);
    return FLB_ERR_INVALID_ARGUMENT;
  }
  for (uint64_t k = 0; k < N; k++)
    if ((d->flags[k] != kFluid && d->flags[k] != kWall) || !(d->porosity[k] >= 0.0 && d->porosity[k] <= 1.0)) {
      std::fprintf(stderr, "flb_adjoint_create: cells must be FLUID or WALL with porosity in [0,1]\n");
      return FLB_ERR_INVALID_ARGUMENT;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FLB_ERR_NO_DEVICE;
  flb_adjoint a = new flb_adjoint_s();
  a->d = *d;
  a->d.flags = nullptr;
  a->d.porosity = nullptr;
  a->nx = d->nx;
  a->ny = d->ny;
  a->N = (uint32_t)N;
  a->K = d->checkpoint_every;
  a->nseg = (uint32_t)(d->steps / d->checkpoint_every);
  a->ts = d->precision == 64 ? 8 : 4;
  a->gx = d->gx;
  a->gy = d->gy;
  a->gx_blocks = (a->nx + kAdjBlock - 1) / kAdjBlock;
  a->nblocks = a->gx_blocks * a->ny;
  a->device = d->device >= 0 ? d->device : 0;
  if (d->device < 0) cudaGetDevice(&a->device);
  ADevice guard(a->device);
  auto bail = [&](flb_status s) {
    std::fprintf(stderr, "flb_adjoint_create: %s\n", a->err.c_str());
    afree(a);
    delete a;
    return s;
  };
  if (d->stream) {
    a->stream = static_cast<cudaStream_t>(d->stream);
  } else {
    if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess)
      return bail(afail(a, FLB_ERR_CUDA, "cudaStreamCreate"));
    a->own_stream = true;
  }
  const size_t st = 9 * N * a->ts;
  struct Al {
    void** p;
    size_t bytes;
  } allocs[] = {{(void**)&a->d_flags, N},           {(void**)&a->d_srcw, N},
                {&a->d_s, N * a->ts},               {&a->d_id, N * a->ts},
                {&a->d_state[0], st},
                {&a->d_state[1], st},               {&a->d_ckpt, st * a->nseg},
                {&a->d_tape, 2 * 3 * N * a->ts * a->K},
                {&a->d_rstate[0], st},              {&a->d_rstate[1], st},            {&a->d_lam[0], st},
                {&a->d_lam[1], st},                 {(void**)&a->d_sbar, N * sizeof(double)},
                {(void**)&a->d_gpart, 2 * (size_t)a->nblocks * sizeof(double)},
                {(void**)&a->d_jrow, a->ny * sizeof(double)}, {(void**)&a->d_seg, 2 * sizeof(SegDesc)}};
  for (Al& x : allocs) {
    cudaError_t e = cudaMalloc(x.p, x.bytes);
    if (e != cudaSuccess) return bail(afail(a, FLB_ERR_OUT_OF_MEMORY, "cudaMalloc"));
  }
  if (cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return bail(afail(a, FLB_ERR_CUDA, "stream/event creation"));
  if (cudaMallocHost(&a->h_seg, a->nseg * sizeof(SegDesc)) != cudaSuccess)
    return bail(afail(a, FLB_ERR_OUT_OF_MEMORY, "cudaMallocHost"));
  for (uint32_t k = 0; k < a->nseg; k++) {
    a->h_seg[k].t0 = (uint64_t)k * a->K;
    a->h_seg[k].ckpt = static_cast<char*>(a->d_ckpt) + (size_t)k * st;
  }
  if (cudaMemcpyAsync(a->d_flags, d->flags, N, cudaMemcpyHostToDevice, a->stream) != cudaSuccess)
    return bail(afail(a, FLB_ERR_CUDA, "cudaMemcpy"));
  k_srcw<<<dim3(a->gx_blocks, a->ny), kAdjBlock, 0, a->stream>>>(a->d_flags, a->d_srcw, a->nx, a->ny);
  flb_status s = a->ts == 8 ? upload_s<double>(a, d->porosity) : upload_s<float>(a, d->porosity);
  if (s == FLB_OK) s = a->ts == 8 ? capture<double>(a) : capture<float>(a);
  if (s != FLB_OK) return bail(s);
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return bail(afail(a, FLB_ERR_CUDA, "set-up"));
  *out = a;
  return FLB_OK;
}

FLB_API flb_status flb_adjoint_set_porosity(flb_adjoint a, const double* s) {
  if (!a || !s) return FLB_ERR_INVALID_ARGUMENT;
  ADevice g(a->device);
  for (uint32_t k = 0; k < a->N; k++)
    if (!(s[k] >= 0.0 && s[k] <= 1.0)) return afail(a, FLB_ERR_INVALID_ARGUMENT, "porosity outside [0,1]");
  a->forward_done = false;
  return a->ts == 8 ? upload_s<double>(a, s) : upload_s<float>(a, s);
}

FLB_API flb_status flb_adjoint_set_force(flb_adjoint a, double gx, double gy) {
  if (!a) return FLB_ERR_INVALID_ARGUMENT;
  ADevice g(a->device);
  a->gx = gx;
  a->gy = gy;
  a->forward_done = false;
  return a->ts == 8 ? capture<double>(a) : capture<float>(a);  // the force is a kernel argument
}

FLB_API flb_status flb_adjoint_forward(flb_adjoint a, double* J) {
  if (!a || !J) return FLB_ERR_INVALID_ARGUMENT;
  ADevice g(a->device);
  return a->ts == 8 ? forward<double>(a, J) : forward<float>(a, J);
}

FLB_API flb_status flb_adjoint_backward(flb_adjoint a, double* dJ_ds, double dJ_dg[2]) {
  if (!a) return FLB_ERR_INVALID_ARGUMENT;
  if (!a->forward_done) return afail(a, FLB_ERR_INVALID_ARGUMENT, "flb_adjoint_forward must run first");
  ADevice g(a->device);
  return a->ts == 8 ? backward<double>(a, dJ_ds, dJ_dg) : backward<float>(a, dJ_ds, dJ_dg);
}

FLB_API flb_status flb_adjoint_timing(flb_adjoint a, double ms[2]) {
  if (!a || !ms) return FLB_ERR_INVALID_ARGUMENT;
  ms[0] = a->ms_fwd;
  ms[1] = a->ms_bwd;
  return FLB_OK;
}

FLB_API flb_status flb_adjoint_destroy(flb_adjoint a) {
  if (!a) return FLB_ERR_INVALID_ARGUMENT;
  {
    ADevice g(a->device);
    cudaStreamSynchronize(a->stream);
    afree(a);
  }
  delete a;
  return FLB_OK;
}

FLB_API const char* flb_adjoint_last_error(flb_adjoint a) { return a ? a->err.c_str() : "null adjoint"; }

}  // extern "C"
