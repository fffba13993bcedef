/* Reference harness: compiles the reference's own hot-path headers where they
 * lie (NEWEST5/ or TXYZ5/ under the reference tree, passed with -I) into a
 * shared library with a small extern "C" surface, so that tests can run the
 * reference's arithmetic on inputs we choose and pin the oracle against it.
 *
 * What is the reference's code here: maindef.h (cell, EOS hooks, the
 * A1..A5 closure), utils.h (WENO), boundary.h, Source.h (sources, NS init),
 * multiroot.h (residuals, Jacobian and the per-cell solver loop), hydroKT.h
 * (KT operator) and time.h (TVDRK2 / TVDRK3 orchestration).
 * What is ours: the single-rank MPI declarations and the GSL gnewton
 * restatement (ref_shim/), the globals and neighbour macros that init.h
 * would declare (init.h itself opens MPI files), a no-op pack() (with one
 * rank every neighbour is BOUNDARY, NEWEST5/pack.h:689-775 moves nothing),
 * a no-op DebugMSG() (NEWEST5/debug.h:3 prints diagnostics only), and the
 * state import/export below.  For TXYZ5 the A1..A5 macros, which that
 * variant uses but never defines, are supplied as the tau = 1 form of
 * NEWEST5/maindef.h:497-501.
 *
 * The scenario (grid, dx, EOS, transport) is the reference's compile-time
 * block selected by -D flags; ZCM/ZCMA, which NEWEST5's default block leaves
 * undefined, are passed on the command line.  With -DGINIT -DVH_REF_EOS_TABLE
 * the GINIT block (30 x 30 cells of 0.1 fm per rank, eta = s/4pi,
 * tau_pi = 1.5 eta/P) runs on a tabulated EOS set at run time
 * (ref_shim/eos_table_s95p.h): the windows of the benchmark workloads.
 *
 * Canonical state layout shared with the oracle: structure of arrays over
 * the ghost-inclusive grid, index (k*YCM + j)*XCM + i (x fastest).
 * Field order: 0 En, 1..4 u^0..u^3, 5..9 pi^{xx,yy,xy,x eta,y eta},
 * 10..13 T^{tau tau},T^{tau x},T^{tau y},T^{tau eta}, 14..17 prevu^0..3.
 */
#include <mpi.h>
#include "gsl_multiroot_shim.h"

#include <iostream>
#include <fstream>
#include <iomanip>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#include <float.h>

#define GEVFM 0.1973
#define PIE 3.141592653589793

using namespace std;

#ifdef VH_REF_TXYZ5
#include "maindef.h"
#elif defined(VH_REF_EOS_TABLE)
/* the GINIT block's EOS hooks on a run-time table instead of s95p */
#include "eos_table_s95p.h"
#include "maindef.h"
#else
#include "s95p.h"
#include "maindef.h"
#endif

/* ---- what init.h would declare (NEWEST5/init.h:1-20) ---- */
void NSInit(GRID HydroGrid, double tau, double ts);
void ZeroInit(GRID HydroGrid, double tau, double ts);
void CheckRoot(GRID HydroGrid, double tau);
double DebugMSG(GRID HydroGrid, double tau);
double MaxTempGev(GRID HydroGrid);
int k0;
int rank = 0, size = 1, root = 0;
int xcord = 0, ycord = 0, zcord = 0;
MPI_Comm mpi_grid = 0;
int il, jl, kl, ir, jr, kr;
int debug = 0;
#define BOUNDARY -1
#define MYXLEFT BOUNDARY
#define MYXRIGHT BOUNDARY
#define MYYLEFT BOUNDARY
#define MYYRIGHT BOUNDARY
#define MYZLEFT BOUNDARY
#define MYZRIGHT BOUNDARY

#ifdef VH_REF_TXYZ5
/* tau = 1 form of NEWEST5/maindef.h:497-501 (the Cartesian metric) */
#define A1 (-((2*p3*u1*u2 + p1*pow(u1,2) + p2*pow(u2,2) + (2*(p4*u1 + p5*u2)*u3 - (p1 + p2)*pow(u3,2)))*pow(-pow(u0,2) + pow(u3,2),-1)))
#define A2 ((p1*u1 + p3*u2 + p4*u3)*pow(u0,-1))
#define A3 ((p3*u1 + p2*u2 + p5*u3)*pow(u0,-1))
#define A4 (pow(u0,-1)*(2*p3*u1*u2*u3 + (p4*u1 + p5*u2 - (p1 + p2)*u3)*pow(u0,2) + p1*u3*pow(u1,2) + p2*u3*pow(u2,2) + p4*u1*pow(u3,2) + p5*u2*pow(u3,2))*pow(pow(u0,2) - pow(u3,2),-1))
#define A5 (-((2*p3*u1*u2 + 2*(p4*u1 + p5*u2)*u3 - (p1 + p2)*pow(u0,2) + p1*pow(u1,2) + p2*pow(u2,2))*pow(-pow(u0,2) + pow(u3,2),-1)))
#endif

#include "utils.h"

/* one rank: nothing to exchange */
void pack(GRID) {}

#include "boundary.h"

double DebugMSG(GRID, double) { return 0.0; }
double DebugMSG(GRID) { return 0.0; }  /* TXYZ5/debug.h:2 signature */

#include "Source.h"
#include "multiroot.h"
#include "hydroKT.h"
#include "time.h"

/* ---------------------------------------------------------------------- */
static inline size_t cidx(int i, int j, int k) { return ((size_t)k * YCM + j) * XCM + i; }
static const size_t NCELL = (size_t)XCM * YCM * ZCM;

extern "C" {

int ref_dims(int* out) {
  out[0] = XCM; out[1] = YCM; out[2] = ZCM;
  out[3] = il; out[4] = ir; out[5] = jl; out[6] = jr; out[7] = kl; out[8] = kr;
#ifdef LBI
  out[9] = 1;
#else
  out[9] = 0;
#endif
  return 10;
}

int ref_consts(double* out) {
  out[0] = XS; out[1] = YS; out[2] = ZS; out[3] = FACTOR; out[4] = GEVFM;
  return 5;
}

/* EOS / transport hooks of the compiled scenario, evaluated at e */
void ref_eos(double e, double* out) {
  double P = EOS(e);
  double T = FT(e);
  double s = FS(e, P, T);
  double eta = Feta(s, e);
  out[0] = P; out[1] = DPDE(e); out[2] = T; out[3] = s; out[4] = eta; out[5] = Ftaupi(eta, P, e);
}

/* allocate the grid and set interior bounds and coordinates
 * (NEWEST5/alloc.h:33-36, NEWEST5/init.h:565-589 with one rank) */
void ref_init_grid(void) {
  if (!HydroGrid) HydroGrid = new cell[XCM][YCM][ZCM]();
  il = jl = BORDER;
  ir = il + XCMA;
  jr = jl + YCMA;
#ifndef LBI
  kl = BORDER;
  kr = kl + ZCMA;
#else
  kl = 0;
  kr = 1;
#endif
  const double xstart = -((double)((1 * XCMA) / 2) * XS);
  const double ystart = -((double)((1 * YCMA) / 2) * YS);
#ifdef LBI
  const double zstart = 0.0;
#else
  const double zstart = -((double)(ZCMA / 2) * ZS);
#endif
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        cell& c = HydroGrid[i][j][k];
        c.X = xstart + (i - BORDER) * XS;
        c.Y = ystart + (j - BORDER) * YS;
#ifdef LBI
        c.eta = zstart;
#else
        c.eta = zstart + (k - BORDER) * ZS;
#endif
        c.r = sqrt(c.X * c.X + c.Y * c.Y);
      }
#ifdef LBI
  k0 = 0;
#else
  k0 = (ZCM - 1) / 2;
#endif
}

void ref_coords(double* x, double* y, double* eta) {
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        size_t c = cidx(i, j, k);
        x[c] = HydroGrid[i][j][k].X; y[c] = HydroGrid[i][j][k].Y; eta[c] = HydroGrid[i][j][k].eta;
      }
}

/* import the canonical SoA state (18 fields) into every cell, clearing the
 * work buffers as a fresh `new cell[]()` would */
void ref_set_state(const double* f) {
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        size_t c = cidx(i, j, k);
        cell& h = HydroGrid[i][j][k];
        h.En = f[0 * NCELL + c];
        for (int l = 0; l < 4; l++) h.u[l] = f[(1 + l) * NCELL + c];
        for (int l = 0; l < 5; l++) h.pi[l] = f[(5 + l) * NCELL + c];
        h.T00 = f[10 * NCELL + c]; h.T10 = f[11 * NCELL + c];
        h.T20 = f[12 * NCELL + c]; h.T30 = f[13 * NCELL + c];
        for (int l = 0; l < 4; l++) h.prevu[l] = f[(14 + l) * NCELL + c];
        h.PI = 0;
        h.P = EOS(h.En);
        h.Temp = FT(h.En);
        h.Vx = h.u[1] / h.u[0]; h.Vy = h.u[2] / h.u[0]; h.Ve = h.u[3] / h.u[0];
      }
}

void ref_get_state(double* f) {
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        size_t c = cidx(i, j, k);
        cell& h = HydroGrid[i][j][k];
        f[0 * NCELL + c] = h.En;
        for (int l = 0; l < 4; l++) f[(1 + l) * NCELL + c] = h.u[l];
        for (int l = 0; l < 5; l++) f[(5 + l) * NCELL + c] = h.pi[l];
        f[10 * NCELL + c] = h.T00; f[11 * NCELL + c] = h.T10;
        f[12 * NCELL + c] = h.T20; f[13 * NCELL + c] = h.T30;
        for (int l = 0; l < 4; l++) f[(14 + l) * NCELL + c] = h.prevu[l];
      }
}

/* full time step: the reference's own TVDRK2 (NEWEST5/time.h:333) */
void ref_tvdrk2(double tau, double ts) { TVDRK2(HydroGrid, tau, ts); }
void ref_tvdrk3(double tau, double ts) { TVDRK3(HydroGrid, tau, ts); }

/* stage-1 pieces on the current state, dumped per interior-inclusive cell:
 * src[10*NCELL] = Source, res[10*NCELL] = Result (flux divergence),
 * du[16*NCELL] = du[mu][nu] */
void ref_stage_terms(double tau, double ts, double* src, double* res, double* du) {
  CalcSource(HydroGrid, tau, ts);
  CalcCentreFlux(HydroGrid, tau);
  hydroExplicit(HydroGrid, tau, ts / 2);
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        size_t c = cidx(i, j, k);
        cell& h = HydroGrid[i][j][k];
        for (int l = 0; l < 10; l++) { src[l * NCELL + c] = h.Source[l]; res[l * NCELL + c] = h.Result[l]; }
        for (int a = 0; a < 4; a++)
          for (int b = 0; b < 4; b++) du[(a * 4 + b) * NCELL + c] = h.du[a][b];
      }
}

/* Navier-Stokes initialisation of pi and T^{tau mu} (NEWEST5/Source.h:607) */
#ifndef VH_REF_TXYZ5
void ref_ns_init(double tau, double ts) { NSInit(HydroGrid, tau, ts); }
#else
/* TXYZ5 declares NSInit but does not define it */
void ref_ns_init(double, double) { abort(); }
#endif

/* zero-gradient ghost copy (NEWEST5/boundary.h:266) */
void ref_boundary(void) { boundary(HydroGrid); }

/* residuals y0..y3 of the conserved-to-primitive system at x = (e,u1,u2,u3)
 * (NEWEST5/multiroot.h:202-242); p = {T00,T10,T20,T30,pi1..pi5,PI,tau} */
void ref_residual(const double* x, const double* p, double* y, double* J) {
  struct rparams rp = {p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], 0.0};
  gsl_vector xv = {4, (double*)x};
  gsl_vector yv = {4, y};
  gsl_matrix Jm = {4, 4, J};
  conservation_f(&xv, &rp, &yv);
  conservation_df(&xv, &rp, &Jm);
}

/* maximum temperature in GeV over the interior (NEWEST5/utils.h:263) */
double ref_max_temp_gev(void) { return MaxTempGev(HydroGrid); }

}  /* extern "C" */
