// fs_cells.cuh -- per-cell and per-tile device code of the free-surface
// passes: FS_1 (lbmKernel2D.cu:14-121) and FS_2, FS_3, FS_4 fused into one
// shared-memory flag stencil (lbmKernel2D.cu:124-303), plus the super-tile
// activity words the list build reads.  Shared by the per-pass kernels
// (k_fs.cu) and the persistent free-surface step (k_fsp.cu).
#pragma once

#include "common.cuh"

namespace flb {

// ---- FS_1: mass exchange and gas reconstruction, lbmKernel2D.cu:14-121 -----
// flag, nbm: the cell's flag and wall mask (0 without half-way walls),
// loaded by the caller.
template <class S, class C, class M, bool HW, bool ODD>
__device__ __forceinline__ void fs1_cell(const KParams& p, uint32_t x, uint32_t y, uint8_t flag, uint32_t nbm) {
  const uint32_t nx = p.nx, N = p.N;
  const uint32_t idx = x + y * nx;
  const uint8_t* flags = p.flags;
  // the populations, the mass and the neighbours' excess are loaded before
  // the flag is tested (a caller that has just loaded the flag then waits
  // one round trip, not two), the populations as if no neighbour were a
  // wall; a cell next to a wall reloads the ones a wall reflects
  uint32_t nb[9];
  neighbours(x, y, nx, p.ny, nb);
  C in[9], out[9];
  load_in<S, C, false, ODD>(p, idx, nb, 0u, in);
  load_out<S, C, ODD>(p, idx, nb, out);
  M* Ms = static_cast<M*>(p.mass);
  const M* Ex = static_cast<const M*>(p.excess);
  const M* Ph = static_cast<const M*>(p.phi);
  M m = Ms[idx];
  M exn[9];
#pragma unroll
  for (int i = 1; i < 9; i++) exn[i] = Ex[nb[i]];
  if (flag & (kGas | kWall | kInlet)) return;
  const bool cons = p.fs_cons != 0;
  const uint8_t e = flag & kFGI;
  if (cons && (!(e == kFluid || e == kInterface) || (flag & kMovingWall))) return;
  if (HW && nbm) reload_reflected<S, C, ODD>(p, idx, nb, nbm, in);
  out[0] = in[0];
#pragma unroll
  for (int i = 1; i < 9; i++) m += exn[i];
  if (e == kFluid) {
    if (!cons) {
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        m += in[i + 1] - out[i];
        m += in[i] - out[i + 1];
      }
    } else {
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        const uint8_t na = flags[nb[i]] & kFGI, nbb = flags[nb[i + 1]] & kFGI;
        if (na == kFluid || na == kInterface) m += in[i + 1] - out[i];
        if (nbb == kFluid || nbb == kInterface) m += in[i] - out[i + 1];
      }
    }
  } else if (e == kInterface) {
    C rho, ux, uy, rhoYL = 0.0f;
    if (flag & (kInlet | kOutlet)) {
      rho = static_cast<const C*>(p.rho)[idx];
      ux = static_cast<const C*>(p.u)[idx];
      uy = static_cast<const C*>(p.u)[idx + N];
    } else {
      rho = density(out);
      velocity(out, rho, ux, uy);
    }
    M phiN[9];
#pragma unroll
    for (int i = 1; i < 9; i++) phiN[i] = Ph[nb[i]];
    phiN[0] = cons ? Ph[idx] : fill_level<M, C>(m, rho);
    const C rho2 = 0.5f / rho;
    ux = ux + rho2 * p.fx;
    uy = uy + rho2 * p.fy;
    limit_u(p.u_max, ux, uy);
    C feq[9];
    equilibrium<C>(1.0f - rhoYL, ux, uy, feq);
    uint8_t nF[9];
#pragma unroll
    for (int i = 1; i < 9; i++) nF[i] = flags[nb[i]] & kFGI;
#pragma unroll
    for (int i = 1; i < 9; i += 2) {
      uint8_t ne = nF[i];
      if (ne == kFluid) m += in[i + 1] - out[i];
      else if (ne == kInterface) m += (in[i + 1] - out[i]) * 0.5f * (phiN[i] + phiN[0]);
      ne = nF[i + 1];
      if (ne == kFluid) m += in[i] - out[i + 1];
      else if (ne == kInterface) m += (in[i] - out[i + 1]) * 0.5f * (phiN[i + 1] + phiN[0]);
    }
#pragma unroll
    for (int i = 1; i < 9; i += 2) {
      in[i] = feq[i] - out[i + 1] + feq[i + 1];
      in[i + 1] = feq[i + 1] - out[i] + feq[i];
    }
    if (!cons) {
      // reference gate (storeReconstructedGasf, cellCalculations.cuh:250-259):
      // tests the neighbour the population travels toward.  Parked in recon so
      // that neighbours reading their outgoing slots see the pre-pass values.
      C* rec = static_cast<C*>(p.recon);
      uint32_t mask = 0;
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        if (nF[i] == kGas) { mask |= 1u << (i - 1); rec[(uint32_t)(i - 1) * N + idx] = in[i]; }
        if (nF[i + 1] == kGas) { mask |= 1u << i; rec[(uint32_t)i * N + idx] = in[i + 1]; }
      }
      p.recon_mask[idx] = (uint8_t)mask;
    } else {
      // population arriving from a gas neighbour: its slot is read by no other
      // cell in this pass (the gas cell does not run), so store in place
      const float scale = p.f16_scale;
#pragma unroll
      for (int i = 1; i < 9; i += 2) {
        if (nF[i + 1] == kGas) Codec<S, C>::st(slotp<S>(p, slot_a<ODD>(i)), idx, i, in[i], scale);
        if (nF[i] == kGas) Codec<S, C>::st(slotp<S>(p, slot_b<ODD>(i)), nb[i], i + 1, in[i + 1], scale);
      }
    }
  }
  Ms[idx] = m;
}

// The cell's flag and wall mask in one round trip, then the cell.
template <class S, class C, class M, bool HW, bool ODD>
__device__ __forceinline__ void fs1_cell(const KParams& p, uint32_t x, uint32_t y) {
  const uint32_t idx = x + y * p.nx;
  const uint8_t flag = p.flags[idx];
  const uint32_t nbm = HW ? p.nbmask[idx] : 0u;
  fs1_cell<S, C, M, HW, ODD>(p, x, y, flag, nbm);
}

// ---- FS_2 + FS_3 + FS_4 fused: lbmKernel2D.cu:124-303 ----------------------
// The three reference passes are flag stencils of radius one, chained; a tile
// of kTX x 8 cells stages the flags of its 3-cell halo in shared memory and
// evaluates the chain there, so neighbour flags are never read while another
// block rewrites them.  Reads p.flags, writes p.flags_out.
// Tiles of the flag pass: 128 x 8 (a whole super-tile) or 32 x 8 (a quarter,
// the super-tile's four quarters in turn), with one, two or four cells per
// thread (FsForm; the host picks by the grid's super-tile count).  On grids
// of up to kWideTiles super-tiles the pass is launched with programmatic
// dependent launch.
constexpr int kTY = 8, kHalo = 3;
#ifndef FLB_FS_PDL_TILES
#define FLB_FS_PDL_TILES 4096
#endif
constexpr uint32_t kWideTiles = FLB_FS_PDL_TILES;
#ifndef FLB_FS_WIDE_MIN_BLOCKS
#define FLB_FS_WIDE_MIN_BLOCKS 2
#endif
#ifndef FLB_FS_HALF_MIN_BLOCKS
#define FLB_FS_HALF_MIN_BLOCKS 2
#endif
#ifndef FLB_FS_W64_MIN_BLOCKS
#define FLB_FS_W64_MIN_BLOCKS 3
#endif
#ifndef FLB_FS_W64X2_MIN_BLOCKS
#define FLB_FS_W64X2_MIN_BLOCKS 5
#endif
#ifndef FLB_FS_QUARTER_MIN_BLOCKS
#define FLB_FS_QUARTER_MIN_BLOCKS 4
#endif
// periodic index; halos of in-range tiles need one add or subtract, the
// modulo is only reached on grids narrower than a tile
__device__ __forceinline__ int wrapi(int v, int n) {
  if (v < 0) v += n;
  else if (v >= n) v -= n;
  if ((unsigned)v >= (unsigned)n) v = ((v % n) + n) % n;
  return v;
}

// ex / cont for a neighbour count of 1..8.  Counts 1, 2, 4 and 8 scale by an
// exact power of two, which rounds exactly as the division does; only 3, 5, 6
// and 7 divide (a double division is a long instruction sequence, and deep
// fluid cells all have 8 neighbours).
template <class M>
__device__ __forceinline__ M div_count(M ex, int cont) {
  if ((cont & (cont - 1)) == 0) return ex * (M)(1.0f / (float)cont);
  return ex / (M)(float)cont;
}

// Bit-plane form of the stencil chain.  For each row of the tile and of its
// 3-row halo, and each 32-cell word of the tile plus one word on either side,
// a warp ballot turns 32 flag bytes into predicate masks (bit i = cell i of the
// word).  FS_2's and FS_3's "any neighbour with property P" is then an 8-way
// dilation of a mask (shifts and ORs across neighbouring words and rows), the
// flag rewrites are bitwise logic on whole words, and FS_4's neighbour count
// is a popcount of a 3x3 window; each cell finally reads its own bits.  The
// words at the outer ends of a row lack a neighbour word, so their outermost
// bits are wrong after each dilation; the three stages reach at most the third
// bit from either end, and only the innermost 3 bits of those words (the halo)
// are read.
template <int TW>
struct FlagMasks {
  static constexpr int kW = TW / 32 + 2;      // words per row
  static constexpr int kR = kTY + 2 * kHalo;  // rows
  // from the flags after stream-collide (s0)
  uint32_t a[kR][kW];      // (f & 5) == 5   IF
  uint32_t gas[kR][kW];    // f & GAS
  uint32_t gonly[kR][kW];  // (f & 6) == 2   gas, not interface
  uint32_t gi[kR][kW];     // f & GAS_INTERFACE
  uint32_t fl[kR][kW];     // FLUID set, INLET clear
  uint32_t it[kR][kW];     // f & INTERFACE
  uint32_t fb[kR][kW];     // f & FLUID
  uint32_t sk[kR][kW];     // f & (WALL | MOVING_WALL | INLET)
  // derived
  uint32_t anyif[kR][kW];  // FS_2: a neighbour is IF
  uint32_t ig1[kR][kW];    // after FS_2: (f & (GI | IG)) == IG
  uint32_t p1[kR][kW];     // after FS_2: GAS bit
  uint32_t p7[kR][kW];     // after FS_2: GAS_INTERFACE bit
  uint32_t anyig[kR][kW];  // FS_3: a neighbour is IG (after FS_2)
  uint32_t cnt[kR][kW];    // after FS_4's conversion: counted by FS_4's neighbour count
};

// 8-neighbourhood of bit i of word c, row r, of mask m (missing words read 0).
template <int TW>
__device__ __forceinline__ uint32_t dilate8(const uint32_t (&m)[FlagMasks<TW>::kR][FlagMasks<TW>::kW], int r,
                                            int c) {
  constexpr int kW = FlagMasks<TW>::kW;
  uint32_t out = 0;
#pragma unroll
  for (int dr = -1; dr <= 1; dr++) {
    const uint32_t w = m[r + dr][c];
    const uint32_t l = c > 0 ? m[r + dr][c - 1] : 0u;
    const uint32_t rt = c < kW - 1 ? m[r + dr][c + 1] : 0u;
    const uint32_t sh = (w << 1) | (l >> 31) | (w >> 1) | (rt << 31);  // left and right neighbours
    out |= dr ? (sh | w) : sh;
  }
  return out;
}

// Bits i-1, i, i+1 of row r around word c (c has words on both sides).
template <int TW>
__device__ __forceinline__ uint32_t window3(const uint32_t (&m)[FlagMasks<TW>::kR][FlagMasks<TW>::kW], int r, int c,
                                            int i) {
  const uint64_t v = ((uint64_t)m[r][c + 1] << 33) | ((uint64_t)m[r][c] << 1) | (uint64_t)(m[r][c - 1] >> 31);
  return (uint32_t)(v >> i) & 7u;
}

template <int TW>
__device__ __forceinline__ bool bit_at(const uint32_t (&m)[FlagMasks<TW>::kR][FlagMasks<TW>::kW], int r, int c,
                                       int i) {
  if (i < 0) {
    c--;
    i += 32;
  } else if (i >= 32) {
    c++;
    i -= 32;
  }
  return (m[r][c] >> i) & 1u;
}

// Per super-tile activity word written by the flag pass: bit 0 = it holds a
// fluid or interface cell; bits 1..8 = it holds one within kReach cells of
// the edge or corner facing the neighbour in direction (dx, dy) (edge_bit).
// The stencil chain of the flag pass reaches kReach = 3 cells, so a neighbour
// needs the pass next step only if such a cell faces it.
constexpr int kReach = 3;
__host__ __device__ constexpr int edge_bit(int dx, int dy) {
  return dy == 0 ? (dx > 0 ? 1 : 2) : dx == 0 ? (dy > 0 ? 3 : 4) : dy > 0 ? (dx > 0 ? 5 : 6) : (dx > 0 ? 7 : 8);
}

// Activity word of a live cell at (lx, ly) in a super-tile of wact x hact cells.
__device__ __forceinline__ uint32_t activity(int lx, int ly, int wact, int hact) {
  const bool r = lx >= wact - kReach, l = lx < kReach, u = ly >= hact - kReach, d = ly < kReach;
  return 1u | ((uint32_t)r << edge_bit(1, 0)) | ((uint32_t)l << edge_bit(-1, 0)) | ((uint32_t)u << edge_bit(0, 1)) |
         ((uint32_t)d << edge_bit(0, -1)) | ((uint32_t)(u && r) << edge_bit(1, 1)) |
         ((uint32_t)(u && l) << edge_bit(-1, 1)) | ((uint32_t)(d && r) << edge_bit(1, -1)) |
         ((uint32_t)(d && l) << edge_bit(-1, -1));
}

// This cell's values after stream-collide that the flag pass reads and
// rewrites; loaded before the stencil stages so that their latency overlaps.
template <class C, class M>
struct Fs4Own {
  uint8_t f0, old;
  M m, ex;
  C rho;
};

template <class C, class M>
__device__ __forceinline__ void fs4_own_load(const KParams& p, uint32_t idx, Fs4Own<C, M>& o) {
  o.f0 = p.flags[idx];
  o.old = p.flags_out[idx];
  o.m = static_cast<const M*>(p.mass)[idx];
  o.rho = static_cast<const C*>(p.rho)[idx];
  // the old excess is compared only by a gas cell that stays gas (write
  // skipping), so only a cell with the gas bit reads it
  o.ex = (o.f0 & kGas) ? static_cast<const M*>(p.excess)[idx] : M(0);
}

// The per-cell end of the flag pass: the byte chain of FS_2, FS_3 and FS_4 for
// cell (gx, gy) at (lx, ly) in the tile, from the masks the stencil stages
// left in sm, and the FS_3 / FS_4 field updates.  Returns whether the cell is
// fluid or interface after the pass.  Q: the cell lies in a quiet tile (no
// gas, interface or gas-interface cell within reach), where the byte chain
// leaves the flag as it is and no cell turns from gas to interface.
template <class S, class C, class M, bool ODD, int TW, bool Q>
__device__ __forceinline__ bool fs234_cell(const KParams& p, const FlagMasks<TW>& sm, int gx, int gy, int lx, int ly,
                                           const Fs4Own<C, M>& own) {
  const int nx = (int)p.nx, ny = (int)p.ny;
  const int r = kHalo + ly, c = 1 + lx / 32, i = lx % 32;
  const uint32_t idx = (uint32_t)gx + (uint32_t)gy * (uint32_t)nx;
  const uint8_t f0 = own.f0, old = own.old;
  const M m_old = own.m, ex_old = own.ex;
  const C rho_own = own.rho;
  M* Ms = static_cast<M*>(p.mass);
  M* Exs = static_cast<M*>(p.excess);
  const C* R = static_cast<const C*>(p.rho);
  // (a quiet tile has no IF or IG cell near: the stages that set these bits did not run)
  const bool any_if = !Q && ((sm.anyif[r][c] >> i) & 1u), any_ig = !Q && ((sm.anyig[r][c] >> i) & 1u);
  // the byte chain of the reference passes, for this cell
  uint8_t f1 = f0;
  if (any_if) {
    const uint8_t e = f1 & kIG;
    if (e == kIG) f1 = (uint8_t)(f1 & ~kGas);
    else if (e == kGas) f1 = (uint8_t)((f1 & ~kGas) | kGasInterface);
  }
  uint8_t f3 = f1;
  {
    const uint8_t e = f3 & (kInletFluid | kInterface);
    if (e != kInletFluid && (e == kFluid || e == kIF) && any_ig) f3 = (uint8_t)((f3 & ~kIF) | kInterface);
  }
  uint8_t fin = f3;
  if (!Q && !(fin & (kWall | kMovingWall | kInlet))) {
    const uint8_t sw = fin & (kFGI | kGasInterface);
    if (sw == kIF || sw == kIG) fin = (uint8_t)(fin & ~kInterface);
    else if (sw == kGasInterface) fin = (uint8_t)((fin & ~kGasInterface) | kInterface);
  }
  const uint32_t N = p.N;
  const bool live = (fin & (kWall | kMovingWall)) == 0 && ((fin & kFGI) == kFluid || (fin & kFGI) == kInterface);
  // Write skipping.  flags_out still holds this cell's flag after the previous
  // step's stream-collide ("old").  When the buffers come from consecutive
  // full steps (trust_prev), values already in memory are not rewritten:
  //  * the flag, when old equals the new flag;
  //  * the fill level of a cell that is fluid (gas) both before and after this
  //    pass: it was fluid (gas) after the previous step too, whose FS_4 left
  //    phi = 1 (0);
  //  * mass and excess of a gas cell when they do not change (deep gas holds
  //    zeros; a gas cell with no fluid or interface neighbour keeps its mass,
  //    lbmKernel2D.cu:296, so nothing else is assumed about them).
  const bool trust = p.trust_prev != 0;
  if (!trust || old != fin) p.flags_out[idx] = fin;
  const C* U = static_cast<const C*>(p.u);
  // FS_3 fields: a gas->interface cell starts from feq of the neighbour
  // average (calculateAverageValuesNeighbors2D, accumulating in float)
  if (!Q && (f1 & (kGasInterface | kIG)) == kGasInterface) {
    uint32_t nb[9];
    neighbours((uint32_t)gx, (uint32_t)gy, (uint32_t)nx, (uint32_t)ny, nb);
    float count = 0.0f, lrho = 0.0f, lux = 0.0f, luy = 0.0f;
    const int ddx[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    const int ddy[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
#pragma unroll
    for (int k = 1; k < 9; k++) {
      // FLUID or INTERFACE set after FS_2 (FS_2 changes neither bit)
      if (bit_at<TW>(sm.fb, r + ddy[k], c, i + ddx[k]) || bit_at<TW>(sm.it, r + ddy[k], c, i + ddx[k])) {
        count += 1.0f;
        lrho += R[nb[k]];
        lux += U[nb[k]];
        luy += U[nb[k] + N];
      }
    }
    C rho = count > 0.0f ? lrho / count : 0.0f;
    C ux = count > 0.0f ? lux / count : 0.0f;
    C uy = count > 0.0f ? luy / count : 0.0f;
    C feq[9];
    const C rho2 = 0.5f / rho;
    ux = ux + rho2 * p.fx;
    uy = uy + rho2 * p.fy;
    limit_u(p.u_max, ux, uy);
    equilibrium(rho, ux, uy, feq);
    store_post<S, C, ODD>(p, idx, nb, feq);
  }
  // FS_4 fields
  if (f3 & (kWall | kMovingWall | kInlet)) return live;
  const uint8_t sw4 = f3 & (kFGI | kGasInterface);
  const uint8_t sw0 = f0 & (kFGI | kGasInterface);
  const bool gas_stays = trust && sw4 == kGas && sw0 == kGas;
  const bool keep_phi = gas_stays || (trust && sw4 == kFluid && sw0 == kFluid);
  const C rho = sw4 == kGas ? C(0) : rho_own;  // the gas case does not use the density
  M m = m_old;
  M ex = 0.0f, ph = 0.0f;
  switch (f3 & (kFGI | kGasInterface)) {
    case 1:
    case 5:
      ex = m - rho;
      m = rho;
      ph = 1.0f;
      break;
    case 2:
    case 6:
      ex = m;
      m = 0.0f;
      ph = 0.0f;
      break;
    case 4:
    case 128:
      if (m > rho) {
        ex = m - rho;
        m = rho;
      } else if (m < 0.0f) {
        ex = m;
        m = 0.0f;
      } else {
        ex = 0.0f;
      }
      ph = fill_level<M, C>(m, rho);
      break;
    default:
      break;
  }
  // FS_4's count of fluid / interface neighbours after the conversion
  int cont = 0;
  if constexpr (Q) {
    // a quiet tile converts no cell: the count comes straight from the
    // neighbours' flags (which the window's loads left in L1): fluid cells
    // that are not solid or inlet (conservative mode), all fluid cells in the
    // reference mode
    uint32_t nb[9];
    neighbours((uint32_t)gx, (uint32_t)gy, (uint32_t)nx, (uint32_t)ny, nb);
    const bool cons = p.fs_cons != 0;
#pragma unroll
    for (int k = 1; k < 9; k++) {
      const uint8_t f = p.flags[nb[k]];
      cont += ((f & kFluid) && !(cons && (f & (kWall | kMovingWall | kInlet)))) ? 1 : 0;
    }
  } else {
    cont = __popc(window3<TW>(sm.cnt, r - 1, c, i)) + __popc(window3<TW>(sm.cnt, r, c, i) & 5u) +
           __popc(window3<TW>(sm.cnt, r + 1, c, i));
  }
  m += cont > 0 ? 0.0f : ex;
  ex = cont > 0 ? div_count(ex, cont) : M(0);
  if (gas_stays) {
    if (!same_bits(m, m_old)) Ms[idx] = m;
    if (!same_bits(ex, ex_old)) Exs[idx] = ex;
  } else {
    Ms[idx] = m;
    Exs[idx] = ex;
  }
  if (!keep_phi) static_cast<M*>(p.phi)[idx] = ph;
  return live;
}

// The general stencil stages of the flag pass on a tile (every thread of the
// block calls it): the masks of the flags after stream-collide (from the flag
// bytes fv each warp loaded), FS_2 and FS_3 as dilations and word logic, and
// FS_4's conversion and neighbour-count mask.
template <int TW, int kWarps, int kIters>
__device__ __forceinline__ void fs234_stages(const KParams& p, FlagMasks<TW>& sm, const uint8_t (&fv)[kIters],
                                             int tid) {
  constexpr int kW = FlagMasks<TW>::kW, kR = FlagMasks<TW>::kR, kRW = kR * kW;
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int k = 0; k < kIters; k++) {
    const int rw = warp + k * kWarps;  // the same for the whole warp
    if (rw >= kRW) break;
    const int r = rw / kW, c = rw % kW;
    const uint8_t f = fv[k];
    // ballots of the flag bits; the masks a row needs are formed from them:
    // the outer halo rows only feed FS_2's IF dilation, the next rows also
    // FS_2's rewrite, the inner ten rows everything (warp-uniform branches)
    const uint32_t bF = __ballot_sync(0xffffffffu, (f & kFluid) != 0);
    const uint32_t bI = __ballot_sync(0xffffffffu, (f & kInterface) != 0);
    if (lane == 0) sm.a[r][c] = bF & bI;
    if (r == 0 || r == kR - 1) continue;
    const uint32_t bG = __ballot_sync(0xffffffffu, (f & kGas) != 0);
    const uint32_t bGI = __ballot_sync(0xffffffffu, (f & kGasInterface) != 0);
    if (lane == 0) {
      sm.gas[r][c] = bG;
      sm.gonly[r][c] = bG & ~bI;
      sm.gi[r][c] = bGI;
      sm.it[r][c] = bI;
    }
    if (r == 1 || r == kR - 2) continue;
    const uint32_t bIn = __ballot_sync(0xffffffffu, (f & kInlet) != 0);
    const uint32_t bSk = __ballot_sync(0xffffffffu, (f & (kWall | kMovingWall | kInlet)) != 0);
    if (lane == 0) {
      sm.fl[r][c] = bF & ~bIn;
      sm.fb[r][c] = bF;
      sm.sk[r][c] = bSk;
    }
  }
  __syncthreads();
  // FS_2 on rows 1 .. kR-2: next to an IF cell, IG -> I and G -> GI
  if (tid < (kR - 2) * kW) {
    const int r = 1 + tid / kW, c = tid % kW;
    const uint32_t any_if = dilate8<TW>(sm.a, r, c);
    const uint32_t p1 = sm.gas[r][c] & ~any_if;
    const uint32_t p7 = sm.gi[r][c] | (any_if & sm.gonly[r][c]);
    sm.anyif[r][c] = any_if;
    sm.p1[r][c] = p1;
    sm.p7[r][c] = p7;
    sm.ig1[r][c] = p1 & sm.it[r][c] & ~p7;
  }
  __syncthreads();
  // FS_3 on rows 2 .. kR-3: next to an IG cell, F / IF (not inlet) -> I; then
  // FS_4's conversion and the mask of the neighbours FS_4 counts
  if (tid < (kR - 4) * kW) {
    const int r = 2 + tid / kW, c = tid % kW;
    const uint32_t any_ig = dilate8<TW>(sm.ig1, r, c);
    const uint32_t conv = sm.fl[r][c] & any_ig;
    const uint32_t P0 = sm.fb[r][c] & ~conv, P1 = sm.p1[r][c], P2 = sm.it[r][c] | conv, P7 = sm.p7[r][c];
    const uint32_t go = ~sm.sk[r][c];
    const uint32_t to_plain = go & ((P0 & ~P1 & P2 & ~P7) | (~P0 & P1 & P2 & ~P7));  // IF, IG lose the I bit
    const uint32_t from_gi = go & (~P0 & ~P1 & ~P2 & P7);                          // GI -> I
    const uint32_t P2f = (P2 & ~to_plain) | from_gi, P7f = P7 & ~from_gi;
    sm.anyig[r][c] = any_ig;
    sm.cnt[r][c] = p.fs_cons ? ((P0 ^ P2f) & ~P1 & go) : ((P0 | P2f) ^ P7f);
  }
  __syncthreads();
}

// The flag bytes of a TW x 8 tile's window (the tile, its kHalo-row halo and
// one 32-cell word on either side: all that the three stencils reach), one
// byte per lane and row-word, with the kWarps warps of the block; a window
// inside the grid is addressed directly, one that crosses an edge wraps
// (periodic).  Returns whether one of this lane's bytes has a gas,
// interface or gas-interface bit.
template <int TW, int kWarps, int kIters>
__device__ __forceinline__ bool load_window(const KParams& p, int tx, int ty, int tid, uint8_t (&fv)[kIters]) {
  constexpr int kTX = TW, kW = FlagMasks<TW>::kW, kR = FlagMasks<TW>::kR, kRW = kR * kW;
  static_assert(kIters * kWarps >= kRW, "window: too few loads");
  const int nx = (int)p.nx, ny = (int)p.ny;
  const uint8_t* flags = p.flags;
  const int lane = tid & 31, warp = tid >> 5;
  const int xw = tx * kTX - 32 + lane;  // word 0 starts one word left of the tile
  const int wx0 = tx * kTX - 32, wy0 = ty * kTY - kHalo;
  const bool inner = wx0 >= 0 && wx0 + 32 * kW <= nx && wy0 >= 0 && wy0 + kR <= ny;
  const uint8_t* wbase = flags + (inner ? xw + wy0 * nx : 0);
  bool nq = false;
#pragma unroll
  for (int k = 0; k < kIters; k++) {
    const int rw = warp + k * kWarps;
    const int r = rw / kW, c = rw % kW;
    fv[k] = rw >= kRW ? 0
            : inner   ? wbase[r * nx + 32 * c]
                      : flags[wrapi(xw + 32 * c, nx) + wrapi(wy0 + r, ny) * nx];
  }
#pragma unroll
  for (int k = 0; k < kIters; k++) nq |= (fv[k] & (kGas | kInterface | kGasInterface)) != 0;
  return nq;
}

// One TW x 8 tile (tile coordinates tx, ty) with the TW*8/CPT threads of the
// block, CPT cells per thread (rows ly and ly + 8/CPT, ...); every thread of
// the block must call it.  Returns the activity bits (activity, above) of
// this thread's cells that are fluid or interface after the pass, with the
// tile at column xoff of a super-tile of wact x hact cells.
template <class S, class C, class M, bool ODD, int TW, int CPT>
__device__ __forceinline__ uint32_t fs234_tile(const KParams& p, int tx, int ty, int tid, FlagMasks<TW>& sm,
                                               int xoff, int wact, int hact) {
  constexpr int kTX = TW, kW = FlagMasks<TW>::kW, kR = FlagMasks<TW>::kR;
  constexpr int kThreads = TW * kTY / CPT, kWarps = kThreads / 32, kRowStep = kTY / CPT;
  static_assert(kTY % CPT == 0 && kThreads >= (kR - 2) * kW, "flag pass: block too small for the stencil stages");
  const int nx = (int)p.nx, ny = (int)p.ny;
  // this thread's cells: their own values are loaded now, so that their
  // latency overlaps the mask building and the stencil stages
  const int lx = tid % kTX, ly0 = tid / kTX;
  const int gx = tx * kTX + lx;
  Fs4Own<C, M> own[CPT];
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    const int gy = ty * kTY + ly0 + k * kRowStep;
    own[k] = Fs4Own<C, M>{0, 0, M(0), M(0), C(0)};
    if (gx < nx && gy < ny) fs4_own_load<C, M>(p, (uint32_t)gx + (uint32_t)gy * (uint32_t)nx, own[k]);
  }
  // masks of the flags after stream-collide: every flag byte a lane needs is
  // loaded first, so the loads of all its row-words are in flight together
  constexpr int kRW = kR * kW, kIters = (kRW + kWarps - 1) / kWarps;
  uint8_t fv[kIters];
  const bool nq = load_window<TW, kWarps, kIters>(p, tx, ty, tid, fv);
  // a quiet tile (no gas, interface or gas-interface cell in the window)
  // needs none of the masks: FS_2 and FS_3 change no flag there and FS_4
  // converts none, and each cell counts its neighbours itself
  const bool quiet = __syncthreads_or(nq) == 0;
  if (!quiet) fs234_stages<TW, kWarps, kIters>(p, sm, fv, tid);
  uint32_t act = 0;
#pragma unroll
  for (int k = 0; k < CPT; k++) {
    const int ly = ly0 + k * kRowStep, gy = ty * kTY + ly;
    if (gx < nx && gy < ny &&
        (quiet ? fs234_cell<S, C, M, ODD, TW, true>(p, sm, gx, gy, lx, ly, own[k])
               : fs234_cell<S, C, M, ODD, TW, false>(p, sm, gx, gy, lx, ly, own[k])))
      act |= activity(xoff + lx, ly, wact, hact);
  }
  return act;
}

// Appends super-tile t to the next step's lists (NextLists), with warp 0 of
// the block (every lane calls it): t itself when it holds fluid or interface
// cells now (m bit 0: both lists) or held some after the previous step (old
// bit 0: the flag-pass list), and the neighbour in the direction of every set
// edge bit of m (the flag-pass list).  A super-tile is added to the flag-pass
// list once (the first to set its mark adds it).  The lengths never pass the
// super-tile count, whatever the state of the marks.
__device__ __forceinline__ void append_next(const NextLists& nl, uint32_t t, uint32_t m, uint32_t old,
                                            uint32_t lane) {
  constexpr uint32_t kNone = 0xffffffffu;
  const uint32_t T = nl.nsx * nl.nsy;
  uint32_t cand = kNone;
  if (lane == 0) {
    if ((m | old) & 1u) cand = t;
  } else if (lane <= 8u && ((m >> lane) & 1u)) {
    // edge_bit: 1 +x, 2 -x, 3 +y, 4 -y, 5 +x+y, 6 -x+y, 7 +x-y, 8 -x-y
    const int dx = (lane == 1 || lane == 5 || lane == 7) ? 1 : (lane == 2 || lane == 6 || lane == 8) ? -1 : 0;
    const int dy = (lane == 3 || lane == 5 || lane == 6) ? 1 : (lane == 4 || lane == 7 || lane == 8) ? -1 : 0;
    const uint32_t sx = t % nl.nsx, sy = t / nl.nsx;
    const uint32_t xx = dx > 0 ? (sx + 1u == nl.nsx ? 0u : sx + 1u) : dx < 0 ? (sx == 0u ? nl.nsx - 1u : sx - 1u) : sx;
    const uint32_t yy = dy > 0 ? (sy + 1u == nl.nsy ? 0u : sy + 1u) : dy < 0 ? (sy == 0u ? nl.nsy - 1u : sy - 1u) : sy;
    cand = xx + yy * nl.nsx;
  }
  // the stream-collide slot is taken beside the marks (independent atomics,
  // so their round trips overlap)
  const bool add_sc = lane == 0 && (m & 1u);
  uint32_t base_fs = 0, base_sc = 0;
  if (add_sc) base_sc = atomicAdd(nl.counts, 1u);
  bool add_fs = false;
  if (cand != kNone) {
    const uint32_t bit = 1u << (cand & 31u);
    add_fs = (atomicOr(nl.bits + (cand >> 5), bit) & bit) == 0u;
  }
  const uint32_t bfs = __ballot_sync(0xffffffffu, add_fs);
  if (lane == 0 && bfs) base_fs = atomicAdd(nl.counts + 1, (uint32_t)__popc(bfs));
  base_fs = __shfl_sync(0xffffffffu, base_fs, 0);
  if (add_fs) {
    const uint32_t k = base_fs + __popc(bfs & ((1u << lane) - 1u));
    if (k < T) nl.list_fs[k] = cand;
  }
  if (add_sc && base_sc < T) nl.list_sc[base_sc] = t;
}

// The flag pass over one super-tile t (its kSTW / TW tiles in turn) with the
// TW*kTY/CPT threads of the block; every thread of the block must call it.
// Records the super-tile's activity word in nz[t] (whose previous value, the
// word of the last step, it reads first) and appends to the next step's
// lists.  wact_sm: one word per warp of the block.
template <class S, class C, class M, bool ODD, int TW, int CPT = 1>
__device__ __forceinline__ void fs234_super_tile(const KParams& p, uint32_t t, uint32_t nsx, uint32_t* nz,
                                                 const NextLists& nl, FlagMasks<TW>& sm, uint32_t* wact_sm) {
  constexpr int kTX = TW, kWarps = TW * kTY / CPT / 32;
  const int tid = threadIdx.x;
  const int sx = (int)(t % nsx), sy = (int)(t / nsx);
  const int wact = min((int)kSTW, (int)p.nx - sx * (int)kSTW), hact = min((int)kSTH, (int)p.ny - sy * (int)kSTH);
  uint32_t act = 0;
  // the word of the last step, read now so that its latency overlaps the
  // tile (only this block writes nz[t] during the pass, at the end)
  const uint32_t word = tid < 32 ? __ldcg(nz + t) : 0u;
  // (no barrier between tiles: a tile's first write to sm comes after its
  // __syncthreads_or, which no thread passes before every thread has
  // finished reading the previous tile's masks)
#pragma unroll 1
  for (int j = 0; j < (int)(kSTW / kTX); j++) {
    const int tx = sx * (int)(kSTW / kTX) + j;
    if (tx * kTX < (int)p.nx) act |= fs234_tile<S, C, M, ODD, TW, CPT>(p, tx, sy, tid, sm, j * kTX, wact, hact);
  }
  act = __reduce_or_sync(0xffffffffu, act);
  if ((tid & 31) == 0) wact_sm[tid >> 5] = act;
  __syncthreads();
  if (tid < 32) {
    uint32_t m = 0;
    for (int w = 0; w < kWarps; w++) m |= wact_sm[w];
    if (tid == 0) nz[t] = m;
    append_next(nl, t, m, word, (uint32_t)tid);
  }
}

}  // namespace flb
