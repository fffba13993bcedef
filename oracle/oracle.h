/* Oracle for the viscous Kurganov-Tadmor step: a plain-C, FP64, CPU
 * restatement of the reference's hot path (rjfries/VIRAL, NEWEST5/ for
 * Milne, TXYZ5/ for Cartesian).  TEST INFRASTRUCTURE ONLY: tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it as the
 * checker; the product never links or calls it.
 *
 * Pinning: oracle/ref_harness.cpp compiles the reference's own headers
 * into oracle/_ref/; tests/golden/ holds fixtures made from those builds
 * (tests/golden/make_golden.py), and the CPU tests check this oracle against
 * them (stage terms, NS initialisation, full TVDRK2 steps).
 *
 * Canonical state layout (shared with the reference harness and the GPU
 * C-ABI): structure of arrays over the ghost-inclusive grid
 * GX x GY x GZ (GX = nx + 6, GY = ny + 6, GZ = nz + 6, or 1 when boost
 * invariant), index (k*GY + j)*GX + i, 18 fields:
 *   0 e, 1..4 u^tau,u^x,u^y,u^eta, 5..9 pi^{xx},pi^{yy},pi^{xy},pi^{x eta},
 *   pi^{y eta}, 10..13 T^{tau tau},T^{tau x},T^{tau y},T^{tau eta},
 *   14..17 prevu^tau..prevu^eta.
 * Units: fm^-4 for e and T^{mu nu}, fm^-1 for temperature.
 */
#ifndef VH_ORACLE_H
#define VH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { VHO_NF = 18 };

typedef struct {
  int nx, ny, nz;       /* interior cells; nz is 1 when boost invariant */
  int boost_invariant;  /* 1: no eta direction (reference LBI) */
  int cartesian;        /* 0: Milne (tau,x,y,eta); 1: Cartesian (t,x,y,z) */
  double dx, dy, dz;
  /* EOS: 0 conformal P = e/3, T = (e/a)^(1/4); 1 table */
  int eos_kind;
  double eos_a;
  int eos_n;            /* table rows, log-spaced in e */
  const double* eos_e;  /* [eos_n] energy density (fm^-4), increasing */
  const double* eos_p;  /* [eos_n] pressure */
  const double* eos_cs2;/* [eos_n] dP/de */
  const double* eos_t;  /* [eos_n] temperature (fm^-1) */
  /* shear viscosity: eta = s * (etas0 + etas1 * max(T*hbarc - etas_tc, 0)),
   * s = (e + P)/T; T in GeV inside the bracket */
  double etas0, etas1, etas_tc, hbarc;
  /* relaxation time: 0 -> 1.5 eta / P (NEWEST5/maindef.h:69);
   *                  1 -> 5 eta / (e + P) (NEWEST5/maindef.h:339);
   *                  2 -> taupi_const (NEWEST5/maindef.h:228, Bjorken) */
  int taupi_kind;
  int gubser_mirror;    /* ghost u^x,u^y mirrored (NEWEST5/boundary.h:32-37) */
  int recon;            /* 0: WENO5 (reference); 1: generalized minmod */
  double minmod_theta;  /* generalized minmod theta (NEWEST5/maindef.h:370) */
  double taupi_const;   /* taupi_kind 2: constant tau_pi (NEWEST5/maindef.h:228) */
  int cold_plasma;      /* shear source without -pi/tau_pi (NEWEST5/Source.h:371-410) */
} vho_config;

typedef struct vho_grid vho_grid;

vho_grid* vho_create(const vho_config* cfg);
void vho_destroy(vho_grid* g);
void vho_dims(const vho_grid* g, int* gx, int* gy, int* gz);
void vho_set_state(vho_grid* g, const double* f);
void vho_get_state(const vho_grid* g, double* f);

/* EOS and transport at e: out = {P, cs2, T, s, eta, taupi} */
void vho_eos(const vho_grid* g, double e, double* out);

/* one TVDRK2 step from tau to tau + ts (NEWEST5/time.h:333-387).
 * Returns 0, or a nonzero status if a cell failed the root-find or the
 * causality / positive-energy check (the reference exits there). */
int vho_step(vho_grid* g, double tau, double ts);

/* stage-1 terms on the current state without advancing it:
 * src[10*G], res[10*G] (flux divergence), du[16*G] */
void vho_stage_terms(vho_grid* g, double tau, double ts, double* src, double* res, double* du);

/* Navier-Stokes pi and T^{tau mu} on every cell (NEWEST5/Source.h:535-630) */
void vho_ns_init(vho_grid* g, double tau, double ts);

/* Navier-Stokes shear 2 eta sigma^{mu nu}, ten components (tt, tx, ty,
 * t-eta, xx, xy, x-eta, yy, y-eta, eta-eta) as NEWEST10/Source.h:643-753:
 * for one cell from du16 (du[l*4+m] = d_m u^l), or on every cell with the
 * step's velocity derivatives (out[10*G]) */
void vho_ns_pi10_cell(const vho_grid* g, double tau, double e, const double* u, const double* du16, double* out10);
void vho_ns_pi10(vho_grid* g, double tau, double ts, double* out);

/* zero-gradient (or Gubser-mirror) ghost copy (NEWEST5/boundary.h) */
void vho_boundary(vho_grid* g);

/* T^{tau mu} from (e,u,pi) on every cell (NEWEST5/init.h:539-549) */
void vho_fill_tmunu(vho_grid* g, double tau);

/* max temperature over the interior in GeV (NEWEST5/utils.h:263) */
double vho_max_temp_gev(const vho_grid* g);

/* Newton iterations used by the last step, summed over cells */
long long vho_last_iterations(const vho_grid* g);

/* conserved-to-primitive for one cell: inputs T[4], pi[5], tau, guess
 * x[4] = (e,u1,u2,u3); on return x holds the root; returns iterations or -1 */
int vho_con2prim(const vho_grid* g, const double* T, const double* pi, double tau, double* x);

/* residuals y[4] and Jacobian J16 (row-major) of the conserved-to-primitive
 * system at x = (e,u1,u2,u3); prm = {T00,T10,T20,T30,pi1..pi5,0,tau} */
void vho_residual(const vho_grid* g, const double* x, const double* prm, double* y, double* J16);

/* Israel-Stewart source for one cell from (e,u,pi,du,tau): out[5] */
void vho_is_source(const vho_grid* g, double e, const double* u, const double* pi5,
                   const double* du16, double tau, double* out);

#ifdef __cplusplus
}
#endif
#endif
