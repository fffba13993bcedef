/* Oracle: plain-C FP64 restatement of the reference's viscous KT step.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each routine cites the
 * reference lines it restates (paths relative to the reference project).
 *
 * Arithmetic order follows the reference where it is cheap to do so, so
 * that the oracle and the compiled reference agree to a few ulps; the
 * Israel-Stewart source is our own covariant derivation (the reference
 * evaluates machine-generated polynomials of the same expression).
 *
 * The cell loops run on OpenMP threads (OMP_NUM_THREADS): every cell is
 * written by one thread and nothing is summed across cells in floating
 * point, so the results do not depend on the number of threads.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NG 3 /* ghost layers, NEWEST5/maindef.h:369-371 BORDER */

struct vho_grid {
  vho_config c;
  int gx, gy, gz;       /* ghost-inclusive extents */
  int il, ir, jl, jr, kl, kr;
  size_t n;             /* gx*gy*gz */
  double* f[VHO_NF];    /* canonical state */
  /* work */
  double *var, *var0, *var1, *lrk, *res, *src, *du, *flux, *spd;
  double* eos_buf;
  long long iters;
};

static inline size_t IX(const vho_grid* g, int i, int j, int k) {
  return ((size_t)k * g->gy + j) * g->gx + i;
}

/* ------------------------------------------------------------------ EOS */

/* bracket e in the log-spaced table: the returned row i satisfies
 * eos_e[i] <= e < eos_e[i+1] (clamped to [0, n-2]) */
static int eos_row(const vho_config* c, double e) {
  int n = c->eos_n;
  double l0 = log(c->eos_e[0]);
  double dl = (log(c->eos_e[n - 1]) - l0) / (n - 1);
  int i = (int)((log(e) - l0) / dl);
  if (i < 0) i = 0;
  if (i > n - 2) i = n - 2;
  while (i > 0 && e < c->eos_e[i]) i--;
  while (i < n - 2 && e >= c->eos_e[i + 1]) i++;
  return i;
}

/* P, cs2, T of the synthetic table: linear in e between log-spaced rows;
 * below the first row P = cs2_0 e, T ~ e^(1/4); above the last row P grows
 * with the last cs2 and T ~ e^(1/4) */
static void eos_table(const vho_config* c, double e, double* P, double* cs2, double* T) {
  int n = c->eos_n;
  if (e <= c->eos_e[0]) {
    *cs2 = c->eos_cs2[0];
    *P = c->eos_cs2[0] * e;
    *T = c->eos_t[0] * sqrt(sqrt(e / c->eos_e[0]));
    return;
  }
  if (e >= c->eos_e[n - 1]) {
    *cs2 = c->eos_cs2[n - 1];
    *P = c->eos_p[n - 1] + c->eos_cs2[n - 1] * (e - c->eos_e[n - 1]);
    *T = c->eos_t[n - 1] * sqrt(sqrt(e / c->eos_e[n - 1]));
    return;
  }
  int i = eos_row(c, e);
  double w = (e - c->eos_e[i]) / (c->eos_e[i + 1] - c->eos_e[i]);
  *P = c->eos_p[i] + w * (c->eos_p[i + 1] - c->eos_p[i]);
  *cs2 = c->eos_cs2[i] + w * (c->eos_cs2[i + 1] - c->eos_cs2[i]);
  *T = c->eos_t[i] + w * (c->eos_t[i + 1] - c->eos_t[i]);
}

static inline double eos_P(const vho_config* c, double e) {
  if (c->eos_kind == 0) return e / 3.0; /* NEWEST5/maindef.h:332 */
  double P, cs2, T;
  eos_table(c, e, &P, &cs2, &T);
  return P;
}
static inline double eos_cs2(const vho_config* c, double e) {
  if (c->eos_kind == 0) return 1.0 / 3.0;
  double P, cs2, T;
  eos_table(c, e, &P, &cs2, &T);
  return cs2;
}
static inline double eos_T(const vho_config* c, double e) {
  if (c->eos_kind == 0) return pow(e / c->eos_a, 0.25); /* NEWEST5/maindef.h:335 */
  double P, cs2, T;
  eos_table(c, e, &P, &cs2, &T);
  return T;
}

/* eta and tau_pi (NEWEST5/maindef.h:337-339, 277-286) */
static inline void transport(const vho_config* c, double e, double P, double* eta, double* taupi) {
  double T = eos_T(c, e);
  double s = (e + P) / T;
  double tg = T * c->hbarc - c->etas_tc;
  double etas = c->etas0 + c->etas1 * (tg > 0 ? tg : 0.0);
  *eta = etas * s;
  *taupi = (c->taupi_kind == 1) ? 5.0 * (*eta) / (e + P) : c->taupi_kind == 2 ? c->taupi_const : 1.5 * ((*eta) / P);
}

void vho_eos(const vho_grid* g, double e, double* out) {
  const vho_config* c = &g->c;
  double P = eos_P(c, e), eta, tp;
  transport(c, e, P, &eta, &tp);
  double T = eos_T(c, e);
  out[0] = P; out[1] = eos_cs2(c, e); out[2] = T; out[3] = (e + P) / T; out[4] = eta; out[5] = tp;
}

/* ------------------------------------------------ pi closure (A1..A5) */

/* Full pi^{mu nu} from the five evolved components by transversality
 * u_mu pi^{mu nu} = 0 and tracelessness in g = diag(1,-1,-1,-t2)
 * (NEWEST5/maindef.h:497-501; t2 = tau^2, or 1 in Cartesian). */
static void pi_full(const double* u, const double* p, double t2, double pi[4][4]) {
  double u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
  double p1 = p[0], p2 = p[1], p3 = p[2], p4 = p[3], p5 = p[4];
  double D = u0 * u0 - t2 * u3 * u3;
  double Q = u1 * u1 * p1 + 2 * u1 * u2 * p3 + u2 * u2 * p2 + 2 * t2 * u3 * (u1 * p4 + u2 * p5);
  double ptt = (Q - t2 * u3 * u3 * (p1 + p2)) / D;
  double pee = (Q - u0 * u0 * (p1 + p2)) / (t2 * D);
  double ptx = (p1 * u1 + p3 * u2 + p4 * u3 * t2) / u0;
  double pty = (p3 * u1 + p2 * u2 + p5 * u3 * t2) / u0;
  double pte = (u1 * p4 + u2 * p5 + t2 * u3 * pee) / u0;
  pi[0][0] = ptt; pi[0][1] = pi[1][0] = ptx; pi[0][2] = pi[2][0] = pty; pi[0][3] = pi[3][0] = pte;
  pi[1][1] = p1; pi[2][2] = p2; pi[1][2] = pi[2][1] = p3;
  pi[1][3] = pi[3][1] = p4; pi[2][3] = pi[3][2] = p5; pi[3][3] = pee;
}

/* ------------------------------------------------------------- WENO5 */

/* smoothness indicators of the three 3-point substencils (NEWEST5/utils.h:111-114) */
static inline void weno_beta(double qm2, double qm1, double qc, double qp1, double qp2, double b[3]) {
  double a;
  a = qc - 2 * qp1 + qp2; double c0 = 3 * qc - 4 * qp1 + qp2;
  b[0] = (13. / 12.) * (a * a) + 0.25 * (c0 * c0);
  a = qm1 - 2 * qc + qp1; double c1 = qm1 - qp1;
  b[1] = (13. / 12.) * (a * a) + 0.25 * (c1 * c1);
  a = qm2 - 2 * qm1 + qc; double c2 = qm2 - 4 * qm1 + 3 * qc;
  b[2] = (13. / 12.) * (a * a) + 0.25 * (c2 * c2);
}
#define WENO_EPS 1e-6
/* value at the right face i+1/2 from the stencil centred on i (utils.h:132-160) */
static inline double weno_left(double qm2, double qm1, double qc, double qp1, double qp2) {
  double b[3]; weno_beta(qm2, qm1, qc, qp1, qp2, b);
  double q0 = (2 * qc + 5 * qp1 - 1 * qp2) / 6.0;
  double q1 = (-1 * qm1 + 5 * qc + 2 * qp1) / 6.0;
  double q2 = (2 * qm2 - 7 * qm1 + 11 * qc) / 6.0;
  double e0 = WENO_EPS + b[0], e1 = WENO_EPS + b[1], e2 = WENO_EPS + b[2];
  double a0 = 0.3 / (e0 * e0), a1 = 0.6 / (e1 * e1), a2 = 0.1 / (e2 * e2);
  double s = 0; s += a0; s += a1; s += a2;
  double r = 0; r += (a0 / s) * q0; r += (a1 / s) * q1; r += (a2 / s) * q2;
  return r;
}
/* value at the left face i-1/2 from the stencil centred on i (utils.h:102-131) */
static inline double weno_right(double qm2, double qm1, double qc, double qp1, double qp2) {
  double b[3]; weno_beta(qm2, qm1, qc, qp1, qp2, b);
  double q0 = (11 * qc - 7 * qp1 + 2 * qp2) / 6.0;
  double q1 = (2 * qm1 + 5 * qc - 1 * qp1) / 6.0;
  double q2 = (-1 * qm2 + 5 * qm1 + 2 * qc) / 6.0;
  double e0 = WENO_EPS + b[0], e1 = WENO_EPS + b[1], e2 = WENO_EPS + b[2];
  double a0 = 0.1 / (e0 * e0), a1 = 0.6 / (e1 * e1), a2 = 0.3 / (e2 * e2);
  double s = 0; s += a0; s += a1; s += a2;
  double r = 0; r += (a0 / s) * q0; r += (a1 / s) * q1; r += (a2 / s) * q2;
  return r;
}
/* derivative (L - R)/dx on one stencil (utils.h:57-98) */
static inline double weno_der(const double* q, double dx) {
  return (weno_left(q[0], q[1], q[2], q[3], q[4]) - weno_right(q[0], q[1], q[2], q[3], q[4])) / dx;
}

/* generalized minmod slope with theta (utils.h:33-55) */
static inline double mm3(double a, double b, double c) {
  if (a * b > 0 && b * c > 0) {
    double m = fmin(fmin(fabs(a), fabs(b)), fabs(c));
    return a < 0 ? -m : m;
  }
  return 0;
}
/* piecewise-linear face values with the generalized minmod slope:
 * left state at i+1/2 and right state at i-1/2 of cell i (unit spacing) */
static inline double mm_left(const vho_config* c, double qm1, double qc, double qp1) {
  return qc + 0.5 * mm3(c->minmod_theta * (qc - qm1), 0.5 * (qp1 - qm1), c->minmod_theta * (qp1 - qc));
}
static inline double mm_right(const vho_config* c, double qm1, double qc, double qp1) {
  return qc - 0.5 * mm3(c->minmod_theta * (qc - qm1), 0.5 * (qp1 - qm1), c->minmod_theta * (qp1 - qc));
}

/* ---------------------------------------------------------- lifecycle */

vho_grid* vho_create(const vho_config* cfg) {
  vho_grid* g = (vho_grid*)calloc(1, sizeof(vho_grid));
  g->c = *cfg;
  if (cfg->eos_kind == 1) {
    int n = cfg->eos_n;
    g->eos_buf = (double*)malloc(sizeof(double) * 4 * n);
    memcpy(g->eos_buf, cfg->eos_e, sizeof(double) * n);
    memcpy(g->eos_buf + n, cfg->eos_p, sizeof(double) * n);
    memcpy(g->eos_buf + 2 * n, cfg->eos_cs2, sizeof(double) * n);
    memcpy(g->eos_buf + 3 * n, cfg->eos_t, sizeof(double) * n);
    g->c.eos_e = g->eos_buf; g->c.eos_p = g->eos_buf + n;
    g->c.eos_cs2 = g->eos_buf + 2 * n; g->c.eos_t = g->eos_buf + 3 * n;
  }
  g->gx = cfg->nx + 2 * NG;
  g->gy = cfg->ny + 2 * NG;
  g->gz = cfg->boost_invariant ? 1 : cfg->nz + 2 * NG;
  g->il = NG; g->ir = NG + cfg->nx;
  g->jl = NG; g->jr = NG + cfg->ny;
  if (cfg->boost_invariant) { g->kl = 0; g->kr = 1; }
  else { g->kl = NG; g->kr = NG + cfg->nz; }
  g->n = (size_t)g->gx * g->gy * g->gz;
  for (int q = 0; q < VHO_NF; q++) g->f[q] = (double*)calloc(g->n, sizeof(double));
  g->var = (double*)calloc(9 * g->n, sizeof(double));
  g->var0 = (double*)calloc(9 * g->n, sizeof(double));
  g->var1 = (double*)calloc(9 * g->n, sizeof(double));
  g->lrk = (double*)calloc(9 * g->n, sizeof(double));
  g->res = (double*)calloc(9 * g->n, sizeof(double));
  g->src = (double*)calloc(9 * g->n, sizeof(double));
  g->du = (double*)calloc(16 * g->n, sizeof(double));
  g->flux = (double*)calloc(27 * g->n, sizeof(double));
  g->spd = (double*)calloc(3 * g->n, sizeof(double));
  return g;
}

void vho_destroy(vho_grid* g) {
  if (!g) return;
  for (int q = 0; q < VHO_NF; q++) free(g->f[q]);
  free(g->var); free(g->var0); free(g->var1); free(g->lrk); free(g->res); free(g->src);
  free(g->du); free(g->flux); free(g->spd); free(g->eos_buf);
  free(g);
}

void vho_dims(const vho_grid* g, int* gx, int* gy, int* gz) { *gx = g->gx; *gy = g->gy; *gz = g->gz; }

void vho_set_state(vho_grid* g, const double* f) {
  for (int q = 0; q < VHO_NF; q++) memcpy(g->f[q], f + q * g->n, sizeof(double) * g->n);
}
void vho_get_state(const vho_grid* g, double* f) {
  for (int q = 0; q < VHO_NF; q++) memcpy(f + q * g->n, g->f[q], sizeof(double) * g->n);
}
long long vho_last_iterations(const vho_grid* g) { return g->iters; }

enum { F_E = 0, F_U0 = 1, F_PI = 5, F_T = 10, F_PU = 14 };

static inline void load_cell(const vho_grid* g, size_t c, double* e, double u[4], double p[5]) {
  *e = g->f[F_E][c];
  for (int l = 0; l < 4; l++) u[l] = g->f[F_U0 + l][c];
  for (int l = 0; l < 5; l++) p[l] = g->f[F_PI + l][c];
}

/* ------------------------------------------------- centre fluxes, Var */

/* F^x, F^y, F^eta of the 9 evolved quantities at one cell
 * (NEWEST5/hydroKT.h:16-83; Cartesian TXYZ5/hydroKT.h:16-64) */
static void centre_flux(const vho_grid* g, size_t c, double tau, double* fx, double* fy, double* fz) {
  const int cart = g->c.cartesian;
  double e, u[4], p[5], pi[4][4];
  load_cell(g, c, &e, u, p);
  double P = eos_P(&g->c, e);
  double t2 = cart ? 1.0 : tau * tau;
  double tf = cart ? 1.0 : tau;
  pi_full(u, p, t2, pi);
  double u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
  double ep = e + P;
  fx[0] = tf * (pi[0][1] + u1 * u0 * ep);
  fx[1] = tf * (p[0] + P + u1 * u1 * ep);
  fx[2] = tf * (p[2] + u1 * u2 * ep);
  fx[3] = tf * (p[3] + u1 * u3 * ep);
  fy[0] = tf * (pi[0][2] + u2 * u0 * ep);
  fy[1] = tf * (p[2] + u2 * u1 * ep);
  fy[2] = tf * (p[1] + P + u2 * u2 * ep);
  fy[3] = tf * (p[4] + u2 * u3 * ep);
  fz[0] = tf * (pi[0][3] + u3 * u0 * ep);
  fz[1] = tf * (p[3] + u3 * u1 * ep);
  fz[2] = tf * (p[4] + u3 * u2 * ep);
  fz[3] = cart ? (pi[3][3] + P + u3 * u3 * ep) : tf * (pi[3][3] + P / t2 + u3 * u3 * ep);
  for (int l = 0; l < 5; l++) {
    fx[4 + l] = (p[l] * u1) / u0;
    fy[4 + l] = (p[l] * u2) / u0;
    /* the eta flux of pi carries a factor tau (NEWEST5/hydroKT.h:76-81) */
    fz[4 + l] = cart ? (p[l] * u3) / u0 : tau * (p[l] * u3) / u0;
  }
}

/* Var = tau T^{tau mu} and pi on every cell (NEWEST5/hydroKT.h:349-367) */
static void fill_var(vho_grid* g, double tau) {
  const double tf = g->c.cartesian ? 1.0 : tau;
#pragma omp parallel for schedule(static)
  for (size_t c = 0; c < g->n; c++) {
    for (int l = 0; l < 4; l++) g->var[l * g->n + c] = g->c.cartesian ? g->f[F_T + l][c] : tf * g->f[F_T + l][c];
    for (int l = 0; l < 5; l++) g->var[(4 + l) * g->n + c] = g->f[F_PI + l][c];
  }
}

/* ------------------------------------------------------------ KT operator */

/* one direction of the KT flux divergence into g->res (accumulated):
 * faces i+1/2 for i in [lo-1, hi-1] along the axis, interior rows across it
 * (NEWEST5/hydroKT.h:88-156 reconstruction, 265-314 max speed, 429-491
 * fluxes).  The face at lo-1/2 has zero dissipation: its max speed lives in
 * a ghost cell the reference never sets. */
static void kt_direction(vho_grid* g, int dir, double tau) {
  const vho_config* C = &g->c;
  int stride, n_along, lo, hi;
  int o1lo, o1hi, o2lo, o2hi;
  size_t s1, s2;
  double h;
  if (dir == 0) { stride = 1; lo = g->il; hi = g->ir; n_along = g->gx; h = C->dx;
    o1lo = g->jl; o1hi = g->jr; s1 = g->gx; o2lo = g->kl; o2hi = g->kr; s2 = (size_t)g->gx * g->gy; }
  else if (dir == 1) { stride = g->gx; lo = g->jl; hi = g->jr; n_along = g->gy; h = C->dy;
    o1lo = g->il; o1hi = g->ir; s1 = 1; o2lo = g->kl; o2hi = g->kr; s2 = (size_t)g->gx * g->gy; }
  else { stride = g->gx * g->gy; lo = g->kl; hi = g->kr; n_along = g->gz; h = C->dz;
    o1lo = g->il; o1hi = g->ir; s1 = 1; o2lo = g->jl; o2hi = g->jr; s2 = g->gx; }
  (void)n_along;
  const double* F = g->flux + (size_t)dir * 9 * g->n;
  const double* A = g->spd + (size_t)dir * g->n;
#pragma omp parallel
  {
  double* H = (double*)malloc(sizeof(double) * 9 * (hi - lo + 1));
#pragma omp for collapse(2) schedule(static)
  for (int b = o2lo; b < o2hi; b++)
    for (int a = o1lo; a < o1hi; a++) {
      size_t base = (size_t)a * s1 + (size_t)b * s2;
      for (int i = lo - 1; i < hi; i++) {
        size_t ci = base + (size_t)i * stride;
        double amax = 0.0;
        if (i >= lo) {
          double sl, sr;
          if (C->recon == 0) {
            sl = weno_left(A[ci - 2 * stride], A[ci - stride], A[ci], A[ci + stride], A[ci + 2 * stride]);
            sr = weno_right(A[ci - stride], A[ci], A[ci + stride], A[ci + 2 * stride], A[ci + 3 * stride]);
          } else {
            sl = mm_left(C, A[ci - stride], A[ci], A[ci + stride]);
            sr = mm_right(C, A[ci], A[ci + stride], A[ci + 2 * stride]);
          }
          amax = fmax(fabs(sl), fabs(sr));
        }
        for (int l = 0; l < 9; l++) {
          const double* q = F + (size_t)l * g->n;
          const double* v = g->var + (size_t)l * g->n;
          double fl, fr, vl, vr;
          if (C->recon == 0) {
            fl = weno_left(q[ci - 2 * stride], q[ci - stride], q[ci], q[ci + stride], q[ci + 2 * stride]);
            fr = weno_right(q[ci - stride], q[ci], q[ci + stride], q[ci + 2 * stride], q[ci + 3 * stride]);
            vl = weno_left(v[ci - 2 * stride], v[ci - stride], v[ci], v[ci + stride], v[ci + 2 * stride]);
            vr = weno_right(v[ci - stride], v[ci], v[ci + stride], v[ci + 2 * stride], v[ci + 3 * stride]);
          } else {
            fl = mm_left(C, q[ci - stride], q[ci], q[ci + stride]);
            fr = mm_right(C, q[ci], q[ci + stride], q[ci + 2 * stride]);
            vl = mm_left(C, v[ci - stride], v[ci], v[ci + stride]);
            vr = mm_right(C, v[ci], v[ci + stride], v[ci + 2 * stride]);
          }
          H[(size_t)(i - lo + 1) * 9 + l] = 0.5 * (fl + fr) - 0.5 * amax * (vr - vl);
        }
      }
      for (int i = lo; i < hi; i++) {
        size_t ci = base + (size_t)i * stride;
        for (int l = 0; l < 9; l++)
          g->res[(size_t)l * g->n + ci] += -(1.0 / h) * (H[(size_t)(i - lo + 1) * 9 + l] - H[(size_t)(i - lo) * 9 + l]);
      }
    }
  free(H);
  }
}

/* centre fluxes on every cell, speeds on the interior only, Var, and the
 * flux divergence summed over the directions (NEWEST5/hydroKT.h:391-421) */
static void hydro_explicit(vho_grid* g, double tau) {
  const int cart = g->c.cartesian;
#pragma omp parallel for schedule(static)
  for (size_t c = 0; c < g->n; c++) {
    double fx[9], fy[9], fz[9];
    centre_flux(g, c, tau, fx, fy, fz);
    for (int l = 0; l < 9; l++) {
      g->flux[(size_t)l * g->n + c] = fx[l];
      g->flux[(size_t)(9 + l) * g->n + c] = fy[l];
      g->flux[(size_t)(18 + l) * g->n + c] = fz[l];
    }
  }
  memset(g->spd, 0, sizeof(double) * 3 * g->n);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        double u0 = g->f[F_U0][c];
        g->spd[c] = g->f[F_U0 + 1][c] / u0;
        g->spd[g->n + c] = g->f[F_U0 + 2][c] / u0;
        g->spd[2 * g->n + c] = cart ? g->f[F_U0 + 3][c] / u0 : tau * g->f[F_U0 + 3][c] / u0;
      }
  fill_var(g, tau);
  memset(g->res, 0, sizeof(double) * 9 * g->n);
  kt_direction(g, 0, tau);
  kt_direction(g, 1, tau);
  if (!g->c.boost_invariant) kt_direction(g, 2, tau);
}

/* --------------------------------------------------------- derivatives */

/* du[l][m] = d_m u^l where the reference computes it (NEWEST5/Source.h:3-101):
 * time derivative on the interior; x derivative for i in [2, gx-3] on
 * interior (j,k); y likewise; eta derivative for every k on interior (i,j)
 * with the edge stencils clamped.  Elsewhere du keeps its previous value,
 * which is zero unless set by an earlier call. */
static void calc_du(vho_grid* g, double ts) {
  const size_t n = g->n;
#pragma omp parallel for collapse(3) schedule(static)
  for (int l = 0; l < 4; l++)
    for (int k = g->kl; k < g->kr; k++)
      for (int j = g->jl; j < g->jr; j++)
        for (int i = g->il; i < g->ir; i++) {
          size_t c = IX(g, i, j, k);
          g->du[(size_t)(l * 4 + 0) * n + c] = (g->f[F_U0 + l][c] - g->f[F_PU + l][c]) / ts;
        }
  for (int l = 0; l < 4; l++) {
    const double* u = g->f[F_U0 + l];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = g->kl; k < g->kr; k++)
      for (int j = g->jl; j < g->jr; j++)
        for (int i = 2; i < g->gx - 2; i++) {
          size_t c = IX(g, i, j, k);
          double q[5] = {u[c - 2], u[c - 1], u[c], u[c + 1], u[c + 2]};
          g->du[(size_t)(l * 4 + 1) * n + c] = weno_der(q, g->c.dx);
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = g->kl; k < g->kr; k++)
      for (int i = g->il; i < g->ir; i++)
        for (int j = 2; j < g->gy - 2; j++) {
          size_t c = IX(g, i, j, k);
          size_t s = g->gx;
          double q[5] = {u[c - 2 * s], u[c - s], u[c], u[c + s], u[c + 2 * s]};
          g->du[(size_t)(l * 4 + 2) * n + c] = weno_der(q, g->c.dy);
        }
    if (!g->c.boost_invariant) {
      size_t s = (size_t)g->gx * g->gy;
      int Z = g->gz;
#pragma omp parallel for collapse(2) schedule(static)
      for (int i = g->il; i < g->ir; i++)
        for (int j = g->jl; j < g->jr; j++)
          for (int k = 0; k < Z; k++) {
            size_t c = IX(g, i, j, k);
            double qc = u[c], qm2, qm1, qp1, qp2;
            if (k > 1 && k < Z - 2) { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
            else if (k == 0) { qm2 = qm1 = qc; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
            else if (k == 1) { qm2 = qm1 = u[c - s]; qp1 = u[c + s]; qp2 = u[c + 2 * s]; }
            else if (k == Z - 2) { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp2 = qp1 = u[c + s]; }
            else { qm1 = u[c - s]; qm2 = u[c - 2 * s]; qp2 = qp1 = qc; }
            double q[5] = {qm2, qm1, qc, qp1, qp2};
            g->du[(size_t)(l * 4 + 3) * n + c] = weno_der(q, g->c.dz);
          }
    }
  }
}

/* ---------------------------------------------------------- IS source */

/* Shared tensor algebra of the Israel-Stewart equation at one cell.
 * Writes the shear tensor sigma^{mu nu}, the expansion theta and the
 * acceleration a_mu (lower index).  Conventions: du[l*4+m] = d_m u^l,
 * metric g = diag(1,-1,-1,-t2), Christoffels (Milne) Gamma^tau_{ee} = tau,
 * Gamma^e_{tau e} = Gamma^e_{e tau} = 1/tau; none in Cartesian.
 *   nabla_a u^l = d_a u^l + Gamma^l_{a r} u^r
 *   theta = nabla_a u^a
 *   sigma^{mu nu} = Delta^{mu a} Delta^{nu b} (nabla_a u_b + nabla_b u_a)/2
 *                   - Delta^{mu nu} (Delta^{ab} nabla_a u_b) / 3
 *   a_b = g_bb u^a nabla_a u^b
 * (the reference evaluates the fully projected sigma, NEWEST5/Source.h:317-370) */
static void is_kinematics(int cart, double tau, const double* u, const double* du,
                          double sig[4][4], double* theta, double acc[4]) {
  double t2 = cart ? 1.0 : tau * tau;
  double g[4] = {1.0, -1.0, -1.0, -t2};
  double gi[4] = {1.0, -1.0, -1.0, -1.0 / t2};
  double Dm[4][4]; /* Dm[l][a] = nabla_a u^l */
  for (int l = 0; l < 4; l++)
    for (int a = 0; a < 4; a++) Dm[l][a] = du[l * 4 + a];
  if (!cart) {
    Dm[0][3] += tau * u[3];
    Dm[3][0] += u[3] / tau;
    Dm[3][3] += u[0] / tau;
  }
  double Dl[4][4]; /* Dl[a][b] = nabla_a u_b */
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dl[a][b] = g[b] * Dm[b][a];
  *theta = Dm[0][0] + Dm[1][1] + Dm[2][2] + Dm[3][3];
  double Dt[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dt[a][b] = (a == b ? gi[a] : 0.0) - u[a] * u[b];
  double tr = 0;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) tr += Dt[a][b] * Dl[a][b];
  double S[4][4], M[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) S[a][b] = 0.5 * (Dl[a][b] + Dl[b][a]);
  for (int m = 0; m < 4; m++)
    for (int b = 0; b < 4; b++) {
      double s = 0;
      for (int a = 0; a < 4; a++) s += Dt[m][a] * S[a][b];
      M[m][b] = s;
    }
  for (int m = 0; m < 4; m++)
    for (int v = 0; v < 4; v++) {
      double s = 0;
      for (int b = 0; b < 4; b++) s += M[m][b] * Dt[v][b];
      sig[m][v] = s - Dt[m][v] * tr / 3.0;
    }
  for (int v = 0; v < 4; v++) {
    double s = 0;
    for (int a = 0; a < 4; a++) s += u[a] * Dm[v][a];
    acc[v] = g[v] * s;
  }
}

/* Source of the five evolved pi components in the flux form
 *   d_tau pi + d_i (v^i pi) = S,  v^i = u^i/u^tau:
 *   S^{mu nu} = [ -(pi - 2 eta sigma)/taupi - (4/3) pi theta
 *                 - (u^mu pi^{nu b} + u^nu pi^{mu b}) a_b
 *                 - u^a (Gamma^mu_{a l} pi^{l nu} + Gamma^nu_{a l} pi^{mu l}) ] / u^tau
 *               + pi^{mu nu} d_i v^i
 * (NEWEST5/Source.h:317-370; TXYZ5/Source.h:291-335 without Christoffels). */
static void is_source_cell(const vho_config* C, double tau, double e, const double* u, const double* p5,
                           const double* du, double* out) {
  const int cart = C->cartesian;
  double t2 = cart ? 1.0 : tau * tau;
  double P = eos_P(C, e), eta, tp;
  transport(C, e, P, &eta, &tp);
  double pi[4][4], sig[4][4], th, acc[4];
  pi_full(u, p5, t2, pi);
  is_kinematics(cart, tau, u, du, sig, &th, acc);
  double pa[4];
  for (int v = 0; v < 4; v++) pa[v] = pi[v][0] * acc[0] + pi[v][1] * acc[1] + pi[v][2] * acc[2] + pi[v][3] * acc[3];
  double divv = 0;
  for (int i = 1; i < 4; i++) divv += du[i * 4 + i] / u[0] - u[i] * du[i] / (u[0] * u[0]);
  static const int MU[5] = {1, 2, 1, 1, 2}, NU[5] = {1, 2, 2, 3, 3};
  for (int q = 0; q < 5; q++) {
    int m = MU[q], v = NU[q];
    /* COLDPLASMA (NEWEST5/Source.h:371-410) drops the relaxation -pi/tau_pi */
    double relax = C->cold_plasma ? 0.0 : pi[m][v];
    double rhs = -(relax - 2.0 * eta * sig[m][v]) / tp - (4.0 / 3.0) * pi[m][v] * th - (u[m] * pa[v] + u[v] * pa[m]);
    double chr = 0;
    if (!cart) {
      /* Gamma^tau_{ee} = tau, Gamma^e_{tau e} = Gamma^e_{e tau} = 1/tau */
      for (int w = 0; w < 2; w++) {
        int A = w ? v : m, B = w ? m : v; /* Gamma^A_{a l} pi^{l B} */
        if (A == 0) chr += u[3] * tau * pi[3][B];
        if (A == 3) chr += (u[0] * pi[3][B] + u[3] * pi[0][B]) / tau;
      }
    }
    out[q] = (rhs - chr) / u[0] + pi[m][v] * divv;
  }
}

void vho_is_source(const vho_grid* g, double e, const double* u, const double* pi5, const double* du16, double tau, double* out) {
  is_source_cell(&g->c, tau, e, u, pi5, du16, out);
}

/* geometric sources of tau T^{tau tau} and tau T^{tau eta}, then the IS
 * sources (NEWEST5/Source.h:165-191, 311-433) */
static void calc_source(vho_grid* g, double tau, double ts) {
  const vho_config* C = &g->c;
  const size_t n = g->n;
  calc_du(g, ts);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        double e, u[4], p[5], pi[4][4], du[16], s5[5];
        load_cell(g, c, &e, u, p);
        double P = eos_P(C, e);
        if (C->cartesian) {
          for (int l = 0; l < 4; l++) g->src[l * n + c] = 0.0;
        } else {
          double t2 = tau * tau;
          pi_full(u, p, t2, pi);
          double ep = e + P;
          g->src[0 * n + c] = -P - t2 * (pi[3][3] + ep * u[3] * u[3]);
          g->src[1 * n + c] = 0.0;
          g->src[2 * n + c] = 0.0;
          g->src[3 * n + c] = -2.0 * (pi[0][3] + ep * u[0] * u[3]);
        }
        for (int a = 0; a < 16; a++) du[a] = g->du[(size_t)a * n + c];
        is_source_cell(C, tau, e, u, p, du, s5);
        /* TXYZ5/Source.h:268-270 loops k over [0, ZCMA) instead of the
         * interior [kl, kr): the last three interior z layers keep a zero
         * shear source in the Cartesian 3+1D step */
        if (C->cartesian && !C->boost_invariant && k >= C->nz)
          for (int q = 0; q < 5; q++) s5[q] = 0.0;
        for (int q = 0; q < 5; q++) g->src[(4 + q) * n + c] = s5[q];
      }
}

/* ------------------------------------------------------------- con2prim */

/* Residuals of T^{tau nu} u_nu = e u^tau (Landau frame) for
 * x = (e, u^x, u^y, u^eta), with u^tau = sqrt(1 + u1^2 + u2^2 + t2 u3^2),
 * and their Jacobian (NEWEST5/multiroot.h:202-319).  The eta row uses the
 * tracelessness of pi to eliminate pi^{eta eta}. */
static void c2p_fj(const vho_config* C, const double* Tt, const double* p, double t2, const double* x, double* y, double J[4][4]) {
  double e = x[0];
  double u1 = x[1], u2 = x[2], u3 = x[3];
  if (e <= 0) e = 1e-6; /* NEWEST5/multiroot.h:225-226 */
  double P = eos_P(C, e);
  double W = Tt[0], X = Tt[1], Y = Tt[2], Z = Tt[3];
  double p1 = p[0], p2 = p[1], p3 = p[2], p4 = p[3], p5 = p[4];
  double S = 1 + u1 * u1 + u2 * u2 + t2 * u3 * u3;
  double u0 = sqrt(S);
  double ep = e + P;
  y[0] = (W - e) * u0 - X * u1 - Y * u2 - t2 * Z * u3;
  y[1] = X * u0 - e * u1 - u1 * (P + p1 + ep * u1 * u1) - u2 * (p3 + ep * u1 * u2) - t2 * u3 * (p4 + ep * u1 * u3);
  y[2] = Y * u0 - e * u2 - u1 * (p3 + ep * u1 * u2) - u2 * (P + p2 + ep * u2 * u2) - t2 * u3 * (p5 + ep * u2 * u3);
  y[3] = Z * u0 - p4 * u1 - p5 * u2 - u3 * (P + W - p1 - p2);
  if (!J) return;
  double a = eos_cs2(C, e);
  double iu = 1.0 / u0;
  J[0][0] = -u0;
  J[0][1] = (W - e) * u1 * iu - X;
  J[0][2] = (W - e) * u2 * iu - Y;
  J[0][3] = t2 * ((W - e) * u3 * iu - Z);
  J[1][0] = -(1 + a) * u1 * S;
  J[1][1] = X * u1 * iu - p1 - ep * (1 + 3 * u1 * u1 + u2 * u2 + t2 * u3 * u3);
  J[1][2] = X * u2 * iu - p3 - 2 * ep * u1 * u2;
  J[1][3] = t2 * (X * u3 * iu - p4 - 2 * ep * u1 * u3);
  J[2][0] = -(1 + a) * u2 * S;
  J[2][1] = Y * u1 * iu - p3 - 2 * ep * u1 * u2;
  J[2][2] = Y * u2 * iu - p2 - ep * (1 + u1 * u1 + 3 * u2 * u2 + t2 * u3 * u3);
  J[2][3] = t2 * (Y * u3 * iu - p5 - 2 * ep * u2 * u3);
  J[3][0] = -a * u3;
  J[3][1] = Z * u1 * iu - p4;
  J[3][2] = Z * u2 * iu - p5;
  J[3][3] = t2 * Z * u3 * iu - (P + W - p1 - p2);
}

static int solve4(double A[4][4], double b[4]) {
  for (int c = 0; c < 4; c++) {
    int p = c;
    for (int r = c + 1; r < 4; r++) if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
    if (A[p][c] == 0.0) return -1;
    if (p != c) {
      for (int k = 0; k < 4; k++) { double t = A[c][k]; A[c][k] = A[p][k]; A[p][k] = t; }
      double t = b[c]; b[c] = b[p]; b[p] = t;
    }
    for (int r = c + 1; r < 4; r++) {
      double m = A[r][c] / A[c][c];
      for (int k = c; k < 4; k++) A[r][k] -= m * A[c][k];
      b[r] -= m * b[c];
    }
  }
  for (int c = 3; c >= 0; c--) {
    double s = b[c];
    for (int k = c + 1; k < 4; k++) s -= A[c][k] * b[k];
    b[c] = s / A[c][c];
  }
  return 0;
}

/* residuals and Jacobian of the conserved-to-primitive system (test hook) */
void vho_residual(const vho_grid* g, const double* x, const double* prm, double* y, double* J16) {
  /* prm = {T00, T10, T20, T30, pi1..pi5, Pi (ignored, 0), tau} */
  double J[4][4];
  double t2 = g->c.cartesian ? 1.0 : prm[10] * prm[10];
  c2p_fj(&g->c, prm, prm + 4, t2, x, y, J);
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) J16[a * 4 + b] = J[a][b];
}

/* Globally convergent Newton with the reference's stopping rule
 * (|dx_i| < 1e-16 |x_i| or dx_i == 0 for all i, at most 100 iterations,
 * NEWEST5/multiroot.h:389-422).  Step control restates GSL's documented
 * gnewton: a step that raises |f| is shortened by
 * t = (sqrt(1 + 6 r) - 1)/(3 r), r = |f_new|^2/|f_old|^2. */
int vho_con2prim(const vho_grid* g, const double* Tt, const double* p, double tau, double* x) {
  const vho_config* C = &g->c;
  double t2 = C->cartesian ? 1.0 : tau * tau;
  double y[4], J[4][4];
  c2p_fj(C, Tt, p, t2, x, y, J);
  double phi = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
  int it = 0;
  while (it < 100) {
    it++;
    double A[4][4], st[4];
    memcpy(A, J, sizeof(A));
    for (int i = 0; i < 4; i++) st[i] = -y[i];
    if (solve4(A, st) != 0) return -1;
    double t = 1.0, xt[4], yt[4], phi1 = 0;
    int ok = 0;
    for (int tries = 0; tries < 64; tries++) {
      for (int i = 0; i < 4; i++) xt[i] = x[i] + t * st[i];
      c2p_fj(C, Tt, p, t2, xt, yt, NULL);
      for (int i = 0; i < 4; i++) if (!isfinite(yt[i])) return -1;
      phi1 = sqrt(yt[0] * yt[0] + yt[1] * yt[1] + yt[2] * yt[2] + yt[3] * yt[3]);
      if (phi1 <= phi || phi == 0.0) { ok = 1; break; }
      double r = (phi1 * phi1) / (phi * phi);
      t *= (sqrt(1.0 + 6.0 * r) - 1.0) / (3.0 * r);
    }
    if (!ok) return -1;
    double dx[4];
    for (int i = 0; i < 4; i++) { dx[i] = xt[i] - x[i]; x[i] = xt[i]; y[i] = yt[i]; }
    phi = phi1;
    c2p_fj(C, Tt, p, t2, x, y, J);
    int conv = 1;
    for (int i = 0; i < 4; i++)
      if (!(fabs(dx[i]) < 1e-16 * fabs(x[i]) || dx[i] == 0.0)) { conv = 0; break; }
    if (conv) break;
  }
  /* an iterate that is not a root counts as a failure (the reference keeps
   * it silently after 100 iterations): residual above 1e-8 of |T^{tau mu}| */
  double scale = fabs(Tt[0]) + fabs(Tt[1]) + fabs(Tt[2]) + fabs(Tt[3]);
  if (!(phi <= 1e-8 * scale)) return -1;
  return it;
}

/* per-cell root-find over the interior, then u^tau and the causality /
 * positive-energy check (NEWEST5/multiroot.h:331-493) */
static int root_find(vho_grid* g, double tau) {
  const vho_config* C = &g->c;
  double t2 = C->cartesian ? 1.0 : tau * tau;
  int status = 0;
  long long iters = 0;
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(|:status) reduction(+:iters)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        double Tt[4], p[5], x[4];
        for (int l = 0; l < 4; l++) Tt[l] = g->f[F_T + l][c];
        for (int l = 0; l < 5; l++) p[l] = g->f[F_PI + l][c];
        x[0] = g->f[F_E][c]; x[1] = g->f[F_U0 + 1][c]; x[2] = g->f[F_U0 + 2][c]; x[3] = g->f[F_U0 + 3][c];
        int it = vho_con2prim(g, Tt, p, tau, x);
        if (it < 0) { status |= 1; continue; }
        iters += it;
        double u1 = x[1], u2 = x[2], u3 = x[3];
        double u0 = sqrt(1 + u1 * u1 + u2 * u2 + u3 * u3 * (C->cartesian ? 1.0 : tau) * (C->cartesian ? 1.0 : tau));
        g->f[F_E][c] = x[0];
        g->f[F_U0][c] = u0; g->f[F_U0 + 1][c] = u1; g->f[F_U0 + 2][c] = u2; g->f[F_U0 + 3][c] = u3;
        double vx = u1 / u0, vy = u2 / u0, ve = u3 / u0;
        if (sqrt(vx * vx + vy * vy + t2 * ve * ve) >= 1 || x[0] <= 0) status |= 2;
      }
  g->iters += iters;
  return status;
}

/* ------------------------------------------------------------- boundary */

static void copy_cell(vho_grid* g, size_t dst, size_t src) {
  for (int q = 0; q < VHO_NF; q++) g->f[q][dst] = g->f[q][src];
}

/* face ghosts only (corners untouched); zero-gradient copy of every field,
 * with u^x,u^y mirrored across the face in the Gubser test
 * (NEWEST5/boundary.h:1-276) */
void vho_boundary(vho_grid* g) {
  const int mir = g->c.gubser_mirror;
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int m = 0; m < NG; m++) {
        size_t gl = IX(g, m, j, k), gr = IX(g, g->ir + m, j, k);
        copy_cell(g, gl, IX(g, g->il, j, k));
        copy_cell(g, gr, IX(g, g->ir - 1, j, k));
        if (mir) {
          size_t ml = IX(g, g->il + NG - m - 1, j, k), mr = IX(g, g->ir - m - 1, j, k);
          g->f[F_U0 + 1][gl] = g->f[F_U0 + 1][ml]; g->f[F_U0 + 2][gl] = g->f[F_U0 + 2][ml];
          g->f[F_U0 + 1][gr] = g->f[F_U0 + 1][mr]; g->f[F_U0 + 2][gr] = g->f[F_U0 + 2][mr];
        }
      }
  for (int k = g->kl; k < g->kr; k++)
    for (int i = g->il; i < g->ir; i++)
      for (int m = 0; m < NG; m++) {
        size_t gl = IX(g, i, m, k), gr = IX(g, i, g->jr + m, k);
        copy_cell(g, gl, IX(g, i, g->jl, k));
        copy_cell(g, gr, IX(g, i, g->jr - 1, k));
        if (mir) {
          size_t ml = IX(g, i, g->jl + NG - m - 1, k), mr = IX(g, i, g->jr - m - 1, k);
          g->f[F_U0 + 1][gl] = g->f[F_U0 + 1][ml]; g->f[F_U0 + 2][gl] = g->f[F_U0 + 2][ml];
          g->f[F_U0 + 1][gr] = g->f[F_U0 + 1][mr]; g->f[F_U0 + 2][gr] = g->f[F_U0 + 2][mr];
        }
      }
  if (!g->c.boost_invariant)
    for (int i = g->il; i < g->ir; i++)
      for (int j = g->jl; j < g->jr; j++)
        for (int m = 0; m < NG; m++) {
          copy_cell(g, IX(g, i, j, m), IX(g, i, j, g->kl));
          copy_cell(g, IX(g, i, j, g->kr + m), IX(g, i, j, g->kr - 1));
        }
}

/* ------------------------------------------------------------ the step */

static void stage_rhs(vho_grid* g, double tau, double ts) {
  calc_source(g, tau, ts);
  hydro_explicit(g, tau);
}

static void unpack_var(vho_grid* g, const double* v, double tau) {
  const size_t n = g->n;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        for (int l = 0; l < 4; l++) g->f[F_T + l][c] = g->c.cartesian ? v[l * n + c] : v[l * n + c] / tau;
        for (int l = 0; l < 5; l++) g->f[F_PI + l][c] = v[(4 + l) * n + c];
      }
}

/* TVDRK2 (NEWEST5/time.h:333-387): Var1 = Var0 + ts L0 at stage 1,
 * Var2 = Var0/2 + Var1/2 + ts L1/2 at stage 2, both unpacked at tau + ts. */
int vho_step(vho_grid* g, double tau, double ts) {
  const size_t n = g->n;
  int status = 0;
  g->iters = 0;
  double t1 = tau + ts;
  stage_rhs(g, tau, ts);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        for (int l = 0; l < 9; l++) {
          size_t q = (size_t)l * n + c;
          double L0 = g->res[q] + g->src[q];
          g->var0[q] = g->var[q];
          g->var1[q] = g->var0[q] + ts * L0;
        }
      }
  unpack_var(g, g->var1, t1);
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        for (int l = 0; l < 4; l++) g->f[F_PU + l][c] = g->f[F_U0 + l][c];
      }
  status |= root_find(g, t1);
  vho_boundary(g);
  stage_rhs(g, t1, ts);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        size_t c = IX(g, i, j, k);
        for (int l = 0; l < 9; l++) {
          size_t q = (size_t)l * n + c;
          double L1 = g->res[q] + g->src[q];
          g->lrk[q] = 0.5 * g->var0[q] + 0.5 * g->var1[q] + 0.5 * ts * L1;
        }
      }
  unpack_var(g, g->lrk, t1);
  status |= root_find(g, t1);
  vho_boundary(g);
  return status;
}

void vho_stage_terms(vho_grid* g, double tau, double ts, double* src, double* res, double* du) {
  const size_t n = g->n;
  stage_rhs(g, tau, ts);
  if (src) {
    memset(src, 0, sizeof(double) * 10 * n);
    memcpy(src, g->src, sizeof(double) * 9 * n);
  }
  if (res) {
    memset(res, 0, sizeof(double) * 10 * n);
    memcpy(res, g->res, sizeof(double) * 9 * n);
  }
  if (du) memcpy(du, g->du, sizeof(double) * 16 * n);
}

/* T^{tau mu} = (e+P) u^tau u^mu - P g^{tau mu} + pi^{tau mu} on every cell
 * (NEWEST5/init.h:539-549, NEWEST5/Source.h:618-626) */
void vho_fill_tmunu(vho_grid* g, double tau) {
  const vho_config* C = &g->c;
  double t2 = C->cartesian ? 1.0 : tau * tau;
  for (size_t c = 0; c < g->n; c++) {
    double e, u[4], p[5], pi[4][4];
    load_cell(g, c, &e, u, p);
    double P = eos_P(C, e), ep = e + P;
    pi_full(u, p, t2, pi);
    g->f[F_T][c] = -P + ep * (u[0] * u[0]) + pi[0][0];
    g->f[F_T + 1][c] = ep * u[0] * u[1] + pi[0][1];
    g->f[F_T + 2][c] = ep * u[0] * u[2] + pi[0][2];
    g->f[F_T + 3][c] = ep * u[0] * u[3] + pi[0][3];
  }
}

/* Navier-Stokes initialisation (NEWEST5/Source.h:535-630): du as the
 * reference computes it at this moment, pi = 2 eta sigma on every cell
 * (ghosts included, with whatever du those cells have), then T^{tau mu}. */
void vho_ns_init(vho_grid* g, double tau, double ts) {
  const vho_config* C = &g->c;
  const size_t n = g->n;
  calc_du(g, ts);
  for (size_t c = 0; c < n; c++) {
    double e, u[4], p[5], du[16], sig[4][4], th, acc[4];
    load_cell(g, c, &e, u, p);
    for (int a = 0; a < 16; a++) du[a] = g->du[(size_t)a * n + c];
    double P = eos_P(C, e), eta, tp;
    transport(C, e, P, &eta, &tp);
    is_kinematics(C->cartesian, tau, u, du, sig, &th, acc);
    g->f[F_PI][c] = 2.0 * eta * sig[1][1];
    g->f[F_PI + 1][c] = 2.0 * eta * sig[2][2];
    g->f[F_PI + 2][c] = 2.0 * eta * sig[1][2];
    g->f[F_PI + 3][c] = 2.0 * eta * sig[1][3];
    g->f[F_PI + 4][c] = 2.0 * eta * sig[2][3];
  }
  vho_fill_tmunu(g, tau);
}

/* Navier-Stokes shear 2 eta sigma^{mu nu}, all ten components in the order
 * tt, tx, ty, t-eta, xx, xy, x-eta, yy, y-eta, eta-eta, for one cell from
 * (e, u, du, tau).  NEWEST10/Source.h:643-753 (CalcNS) writes the same
 * tensor as expanded polynomials in u and du; here it is the projector form
 * of is_kinematics. */
void vho_ns_pi10_cell(const vho_grid* g, double tau, double e, const double* u, const double* du, double* out10) {
  static const int MU[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, NU[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
  double sig[4][4], th, acc[4], eta, tp;
  transport(&g->c, e, eos_P(&g->c, e), &eta, &tp);
  is_kinematics(g->c.cartesian, tau, u, du, sig, &th, acc);
  for (int q = 0; q < 10; q++) out10[q] = 2.0 * eta * sig[MU[q]][NU[q]];
}

/* The same on every cell with the velocity derivatives the step would use
 * at this moment (d_tau u from prevu over ts): out[10*G]. */
void vho_ns_pi10(vho_grid* g, double tau, double ts, double* out) {
  const size_t n = g->n;
  calc_du(g, ts);
  for (size_t c = 0; c < n; c++) {
    double e, u[4], p[5], du[16], o[10];
    load_cell(g, c, &e, u, p);
    for (int a = 0; a < 16; a++) du[a] = g->du[(size_t)a * n + c];
    vho_ns_pi10_cell(g, tau, e, u, du, o);
    for (int q = 0; q < 10; q++) out[(size_t)q * n + c] = o[q];
  }
}

double vho_max_temp_gev(const vho_grid* g) {
  double tmax = 0;
  for (int k = g->kl; k < g->kr; k++)
    for (int j = g->jl; j < g->jr; j++)
      for (int i = g->il; i < g->ir; i++) {
        double t = g->c.hbarc * eos_T(&g->c, g->f[F_E][IX(g, i, j, k)]);
        if (t > tmax) tmax = t;
      }
  return tmax;
}
