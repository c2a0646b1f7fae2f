/*
 * flb_adjoint_oracle.c -- FP64 CPU tape adjoint of the Brinkman-porosity
 * single-phase step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the engine's adjoint
 * (flowlb_b200/csrc/adjoint.cu).  There is no reference counterpart (FlowLB
 * has no porosity model and no adjoint); this file states the engine's own
 * forward model independently, keeps every state of the run (a full tape, so
 * small cases only), and runs the reverse mode step by step.  Every per-cell
 * expression has the same operand order as the engine's FP64 kernels, so with
 * floating-point contraction off J and dJ/ds agree bit for bit.
 *
 * Model per fluid cell: pull streaming with half-way walls (x and y periodic,
 * walls given by flags), rho = sum f, v = j (1 / rho), u = (v + g/2) (1 / d)
 * with d = 1 + s/2 (each reciprocal taken once and multiplied in),
 * F = rho (g - s u), out_i = (1 - w) f_i + w feq_i + (1 - w/2) F_i with the
 * second-order feq and Guo's F_i.  J = (1/W) sum over the last W steps of
 * sum_y rho u_x at x = nx - 1.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const int ACX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
static const int ACY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
static int aopp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
static double aw(int i) { return i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0); }

typedef struct {
  uint32_t nx, ny, N;
  const uint8_t* flags;
  const double* s;
  double om, omc, kk, gx, gy, winv;
  uint64_t steps, window;
} adj_p;

/* source cell of population i of (x, y), or the cell itself with flag 1 when
 * that source is a wall (half-way reflection) */
static size_t asrc(const adj_p* p, uint32_t x, uint32_t y, int i, int* bounce) {
  const uint32_t xs = ACX[i] > 0 ? (x == 0 ? p->nx - 1 : x - 1) : (ACX[i] < 0 ? (x + 1 == p->nx ? 0 : x + 1) : x);
  const uint32_t ys = ACY[i] > 0 ? (y == 0 ? p->ny - 1 : y - 1) : (ACY[i] < 0 ? (y + 1 == p->ny ? 0 : y + 1) : y);
  const size_t c = (size_t)xs + (size_t)ys * p->nx;
  *bounce = (p->flags[c] & 0x08) != 0;
  return *bounce ? (size_t)x + (size_t)y * p->nx : c;
}

static void agather(const adj_p* p, const double* fin, uint32_t x, uint32_t y, double* f) {
  for (int i = 0; i < 9; i++) {
    int b;
    const size_t c = asrc(p, x, y, i, &b);
    f[i] = b ? fin[(size_t)aopp(i) * p->N + c] : fin[(size_t)i * p->N + c];
  }
}

typedef struct {
  double rho, ir, vx, vy, d, id, ux, uy, Fx, Fy, usq, uF;
} acell;

static acell astate(const adj_p* p, const double* f, double s) {
  acell c;
  c.rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const double jx = f[1] - f[2] + f[5] - f[6] + f[7] - f[8];
  const double jy = f[3] - f[4] + f[5] - f[6] - f[7] + f[8];
  c.ir = 1.0 / c.rho;
  c.vx = jx * c.ir;
  c.vy = jy * c.ir;
  c.d = 1.0 + 0.5 * s;
  c.id = 1.0 / c.d;
  c.ux = (c.vx + 0.5 * p->gx) * c.id;
  c.uy = (c.vy + 0.5 * p->gy) * c.id;
  c.Fx = c.rho * (p->gx - s * c.ux);
  c.Fy = c.rho * (p->gy - s * c.uy);
  c.usq = c.ux * c.ux + c.uy * c.uy;
  c.uF = c.ux * c.Fx + c.uy * c.Fy;
  return c;
}

static void astep(const adj_p* p, const double* fin, double* fout, double* jrow, uint64_t t) {
  for (uint32_t y = 0; y < p->ny; y++)
    for (uint32_t x = 0; x < p->nx; x++) {
      const size_t idx = (size_t)x + (size_t)y * p->nx;
      if (p->flags[idx] & 0x08) continue;
      double f[9];
      agather(p, fin, x, y, f);
      const double s = p->s[idx];
      const acell c = astate(p, f, s);
      /* opposite directions share the even part E and flip the odd part O */
      const double base = 1.0 - 1.5 * c.usq;
      fout[idx] = p->omc * f[0] + p->om * (aw(0) * c.rho * base) + p->kk * (aw(0) * (-3.0 * c.uF));
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        const double cu = q == 0 ? c.ux : (q == 1 ? c.uy : (q == 2 ? c.ux + c.uy : c.ux - c.uy));
        const double cF = q == 0 ? c.Fx : (q == 1 ? c.Fy : (q == 2 ? c.Fx + c.Fy : c.Fx - c.Fy));
        const double w = aw(i);
        const double wr = w * c.rho;
        const double E = p->om * (wr * (base + 4.5 * cu * cu)) + p->kk * (w * (9.0 * cu * cF - 3.0 * c.uF));
        const double O = p->om * (wr * (3.0 * cu)) + p->kk * (w * (3.0 * cF));
        fout[(size_t)i * p->N + idx] = p->omc * f[i] + E + O;
        fout[(size_t)(i + 1) * p->N + idx] = p->omc * f[i + 1] + E - O;
      }
      if (jrow && x + 1 == p->nx && t + p->window >= p->steps) jrow[y] += c.rho * c.ux;
    }
}

static void abackstep(const adj_p* p, const double* fin, const double* lam_next, double* lam, double* sbar,
                      double* gb, uint64_t t) {
  for (uint32_t y = 0; y < p->ny; y++)
    for (uint32_t x = 0; x < p->nx; x++) {
      const size_t idx = (size_t)x + (size_t)y * p->nx;
      if (p->flags[idx] & 0x08) continue;
      double f[9], fb[9];
      agather(p, fin, x, y, f);
      const double s = p->s[idx];
      const acell c = astate(p, f, s);
      const double base = 1.0 - 1.5 * c.usq;
      const double m0 = lam_next[idx];
      fb[0] = p->omc * m0;
      double rhob = p->om * m0 * aw(0) * base;
      double usqb = p->om * m0 * aw(0) * c.rho * -1.5;
      double uFb = p->kk * m0 * aw(0) * -3.0;
      double uxb = 0, uyb = 0, Fxb = 0, Fyb = 0;
      for (int q = 0; q < 4; q++) {
        const int i = 2 * q + 1;
        const double mi = lam_next[(size_t)i * p->N + idx], mo = lam_next[(size_t)(i + 1) * p->N + idx];
        fb[i] = p->omc * mi;
        fb[i + 1] = p->omc * mo;
        const double Sb = mi + mo, Db = mi - mo;
        const double cu = q == 0 ? c.ux : (q == 1 ? c.uy : (q == 2 ? c.ux + c.uy : c.ux - c.uy));
        const double cF = q == 0 ? c.Fx : (q == 1 ? c.Fy : (q == 2 ? c.Fx + c.Fy : c.Fx - c.Fy));
        const double w = aw(i);
        const double wr = w * c.rho;
        rhob += Sb * p->om * w * (base + 4.5 * cu * cu) + Db * p->om * w * (3.0 * cu);
        usqb += Sb * p->om * wr * -1.5;
        uFb += Sb * p->kk * w * -3.0;
        const double cub = Sb * p->om * wr * 9.0 * cu + Sb * p->kk * w * 9.0 * cF + Db * p->om * wr * 3.0;
        const double cFb = Sb * p->kk * w * 9.0 * cu + Db * p->kk * w * 3.0;
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
      uxb += usqb * 2.0 * c.ux + uFb * c.Fx;
      uyb += usqb * 2.0 * c.uy + uFb * c.Fy;
      Fxb += uFb * c.ux;
      Fyb += uFb * c.uy;
      if (x + 1 == p->nx && t + p->window >= p->steps) {
        rhob += c.ux * p->winv;
        uxb += c.rho * p->winv;
      }
      rhob += Fxb * (p->gx - s * c.ux) + Fyb * (p->gy - s * c.uy);
      uxb += -s * c.rho * Fxb;
      uyb += -s * c.rho * Fyb;
      double sb = -c.rho * (Fxb * c.ux + Fyb * c.uy);
      double gxb = c.rho * Fxb, gyb = c.rho * Fyb;
      const double vxb = uxb * c.id, vyb = uyb * c.id;
      sb += -0.5 * (uxb * c.ux + uyb * c.uy) * c.id;
      gxb += 0.5 * uxb * c.id;
      gyb += 0.5 * uyb * c.id;
      const double jxb = vxb * c.ir, jyb = vyb * c.ir;
      rhob += -(vxb * c.vx + vyb * c.vy) * c.ir;
      for (int i = 0; i < 9; i++) {
        const double v = fb[i] + rhob + jxb * (double)ACX[i] + jyb * (double)ACY[i];
        int b;
        const size_t src = asrc(p, x, y, i, &b);
        if (b) lam[(size_t)aopp(i) * p->N + idx] = v;
        else lam[(size_t)i * p->N + src] = v;
      }
      sbar[idx] += sb;
      gb[0] += gxb;
      gb[1] += gyb;
    }
}

/* Runs `steps` steps from rest (f = w) and returns J; with dJds (N) or dJdg (2)
 * non-null also runs the tape adjoint.  Returns 0, or -1 when out of memory. */
int orc_adj_run(uint32_t nx, uint32_t ny, const uint8_t* flags, const double* s, double tau, double gx, double gy,
                uint64_t steps, uint64_t window, double* J, double* dJds, double* dJdg) {
  adj_p p;
  p.nx = nx;
  p.ny = ny;
  p.N = nx * ny;
  p.flags = flags;
  p.s = s;
  p.om = 1.0 / tau;
  p.omc = 1.0 - p.om;
  p.kk = 1.0 - 0.5 * p.om;
  p.gx = gx;
  p.gy = gy;
  p.winv = 1.0 / (double)window;
  p.steps = steps;
  p.window = window;
  const size_t n9 = (size_t)9 * p.N;
  const int grad = dJds || dJdg;
  double* tape = (double*)calloc((grad ? steps + 1 : 2) * n9, sizeof(double));
  double* jrow = (double*)calloc(ny, sizeof(double));
  if (!tape || !jrow) {
    free(tape);
    free(jrow);
    return -1;
  }
  for (size_t k = 0; k < n9; k++) tape[k] = aw((int)(k / p.N));
  for (uint64_t t = 0; t < steps; t++) {
    const double* fin = grad ? tape + t * n9 : tape + (t & 1) * n9;
    double* fout = grad ? tape + (t + 1) * n9 : tape + ((t + 1) & 1) * n9;
    memcpy(fout, fin, n9 * sizeof(double)); /* wall slots keep their values */
    astep(&p, fin, fout, jrow, t);
  }
  double sum = 0;
  for (uint32_t y = 0; y < ny; y++) sum += jrow[y];
  *J = sum / (double)window;
  if (grad) {
    double* lam = (double*)calloc(2 * n9, sizeof(double));
    double* sbar = (double*)calloc(p.N, sizeof(double));
    double gb[2] = {0, 0};
    if (!lam || !sbar) {
      free(lam);
      free(sbar);
      free(tape);
      free(jrow);
      return -1;
    }
    for (uint64_t q = 0; q < steps; q++) {
      const uint64_t t = steps - 1 - q;
      abackstep(&p, tape + t * n9, lam + (q & 1) * n9, lam + ((q + 1) & 1) * n9, sbar, gb, t);
    }
    if (dJds) memcpy(dJds, sbar, p.N * sizeof(double));
    if (dJdg) {
      dJdg[0] = gb[0];
      dJdg[1] = gb[1];
    }
    free(lam);
    free(sbar);
  }
  free(tape);
  free(jrow);
  return 0;
}
