/* Reference harness for the Glasma (optical-Glauber CGC) initialisation:
 * compiles NEWEST5's own ginit.h where it lies, with its GINIT scenario
 * block (maindef.h:240-295: s95p EOS, tau0 = 0.1 fm/c, dtau = 0.002, 30 x 30
 * cells of 0.1 fm per rank out of 10 x 10 ranks, nuclei at x = -/+3 fm), so
 * that tests can compare our generator and Landau matching with the
 * reference's ginit() on one rank's window of the global 300 x 300 grid.
 * Test infrastructure only.
 *
 * What is the reference's code here: maindef.h, s95p.h, utils.h (WENO
 * derivative), ginit.h (thickness, derivatives, T^{mu nu}, FindVar, the pi
 * and T^{tau mu} of the state) and the step's headers (boundary.h,
 * Source.h, multiroot.h, hydroKT.h, time.h), so that the window's state can
 * also be evolved.  What is ours: the single-rank MPI declarations and the
 * GSL stand-ins (ref_shim/), the globals and coordinate functions that
 * init.h would declare (NEWEST5/init.h:18-80, restated for the chosen rank
 * coordinates), no-op MPI file output for ginit's WriteXY, a no-op pack()
 * and DebugMSG() as in ref_harness.cpp, the grid allocation and the state
 * export below.
 *
 * Canonical state layout as the oracle's: structure of arrays over the
 * ghost-inclusive grid, index (k*YCM + j)*XCM + i; fields 0 En, 1..4 u,
 * 5..9 pi, 10..13 T^{tau mu}, 14..17 prevu.
 */
#include <mpi.h>
#include "gsl_multiroot_shim.h"
#include "gsl_ginit_shim.h"

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
/* ginit.h's unqualified `rank` would clash with C++11's std::rank under the
 * using-directive: the rank number gets another name here */
#define rank vh_ref_rank

/* MPI file output and finalisation: ginit's WriteXY dumps T^{mu nu} planes
 * into init/; nothing is written here */
static inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File* f) { *f = 0; return 0; }
static inline int MPI_File_seek(MPI_File, MPI_Offset, int) { return 0; }
static inline int MPI_File_write(MPI_File, const void*, int, MPI_Datatype, MPI_Status*) { return 0; }
static inline int MPI_File_close(MPI_File*) { return 0; }
static inline int MPI_Finalize() { return 0; }

#include "s95p.h"
#include "maindef.h"

/* ---- what init.h would declare (NEWEST5/init.h:1-80), one rank at the
 * chosen rank coordinates of the reference's NPX x NPY layout ---- */
int k0;
int rank = 0, size = 1, root = 0;
int xcord = 4, ycord = 4, zcord = 0;
MPI_Comm mpi_grid = 0;
int il, jl, kl, ir, jr, kr;
int debug = 0;
#define GRIDXPOINTS (NPX * XCMA)
#define GRIDYPOINTS (NPY * YCMA)
#define GRIDXMAX ((GRIDXPOINTS / 2) * XS)
#define GRIDYMAX ((GRIDYPOINTS / 2) * YS)
#define XSTART (-GRIDXMAX + xcord * (XL))
#define YSTART (-GRIDYMAX + ycord * (YL))
#define iSTART (xcord * (XCMA))
#define jSTART (ycord * (YCMA))
inline int MYGLOBALiWB(int i) { return (iSTART + (i - BORDER)); }
inline int MYGLOBALjWB(int j) { return (jSTART + (j - BORDER)); }
inline double XCORDWB(int i) { return (XSTART + (i - BORDER) * XS); }
inline double YCORDWB(int j) { return (YSTART + (j - BORDER) * YS); }
#if defined LBI
inline double ZCORDWB(int) { return 0.0; }
#else
#define GRIDZMAX ((ZCMA / 2) * ZS)
inline double ZCORDWB(int k) { return (-GRIDZMAX + (k - BORDER) * ZS); }
#endif

void NSInit(GRID HydroGrid, double tau, double ts);
void ZeroInit(GRID HydroGrid, double tau, double ts);
void CheckRoot(GRID HydroGrid, double tau);
double DebugMSG(GRID HydroGrid, double tau);
double MaxTempGev(GRID HydroGrid);
#define BOUNDARY -1
#define MYXLEFT BOUNDARY
#define MYXRIGHT BOUNDARY
#define MYYLEFT BOUNDARY
#define MYYRIGHT BOUNDARY
#define MYZLEFT BOUNDARY
#define MYZRIGHT BOUNDARY

#include "utils.h"

/* one rank: nothing to exchange (every neighbour is BOUNDARY) */
void pack(GRID) {}

#include "boundary.h"

double DebugMSG(GRID, double) { return 0.0; }

#include "Source.h"
#include "multiroot.h"
#include "hydroKT.h"
#include "time.h"
#include "ginit.h"

static const size_t NCELL = (size_t)XCM * YCM * ZCM;
static inline size_t cidx(int i, int j, int k) { return ((size_t)k * YCM + j) * XCM + i; }

extern "C" {

/* allocate the grid for rank (xc, yc) of the layout and set coordinates;
 * dims: XCM, YCM, ZCM, il, ir, jl, jr, kl, kr, LBI; consts: XS, YS, ZS,
 * TAUSTART, TS, XPOSNUCLEI, FLAT, GEVFM */
int ref_ginit_init(int xc, int yc, int* dims, double* consts) {
  xcord = xc;
  ycord = yc;
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
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        cell& q = HydroGrid[i][j][k];
        q.X = XCORDWB(i);
        q.Y = YCORDWB(j);
        q.eta = ZCORDWB(k);
        q.r = sqrt(q.X * q.X + q.Y * q.Y);
      }
  dims[0] = XCM; dims[1] = YCM; dims[2] = ZCM;
  dims[3] = il; dims[4] = ir; dims[5] = jl; dims[6] = jr; dims[7] = kl; dims[8] = kr;
#ifdef LBI
  dims[9] = 1;
#else
  dims[9] = 0;
#endif
  consts[0] = XS; consts[1] = YS; consts[2] = ZS; consts[3] = TAUSTART; consts[4] = TS;
  consts[5] = XPOSNUCLEI; consts[6] = FLAT; consts[7] = GEVFM;
  return 10;
}

void ref_ginit_set_eig(vh_shim_eig_fn fn) { vh_shim_eig = fn; }

/* the reference's initialisation sequence (NEWEST5/init.h:658-662): ginit
 * at tau - ts (prevu), then at tau = TAUSTART (the state) */
void ref_ginit_run(double tau, double ts) {
  ginit(HydroGrid, tau - ts);
  ginit(HydroGrid, tau);
}

/* one TVDRK2 step of the reference from tau (NEWEST5/time.h:333-387), with
 * this rank's window treated as the whole grid (outflow ghosts) */
void ref_ginit_step(double tau, double ts) { TVDRK2(HydroGrid, tau, ts); }

/* the canonical 18 fields of every cell, and X, Y, eta */
void ref_ginit_state(double* f, double* x, double* y, double* eta) {
  for (int k = 0; k < ZCM; k++)
    for (int j = 0; j < YCM; j++)
      for (int i = 0; i < XCM; i++) {
        const size_t c = cidx(i, j, k);
        const cell& q = HydroGrid[i][j][k];
        f[c] = q.En;
        for (int l = 0; l < 4; l++) f[(1 + l) * NCELL + c] = q.u[l];
        for (int l = 0; l < 5; l++) f[(5 + l) * NCELL + c] = q.pi[l];
        f[10 * NCELL + c] = q.T00;
        f[11 * NCELL + c] = q.T10;
        f[12 * NCELL + c] = q.T20;
        f[13 * NCELL + c] = q.T30;
        for (int l = 0; l < 4; l++) f[(14 + l) * NCELL + c] = q.prevu[l];
        x[c] = q.X;
        y[c] = q.Y;
        eta[c] = q.eta;
      }
}

/* EOS hooks of the block at e: P, dP/de, T, s */
void ref_ginit_eos(double e, double* out) {
  const double P = EOS(e), T = FT(e);
  out[0] = P; out[1] = DPDE(e); out[2] = T; out[3] = FS(e, P, T);
}

/* T = 0.4 GeV at 0.6 fm/c as ginit finds it (NEWEST5/ginit.h:723-734):
 * the energy density from s95p by Newton's method */
double ref_ginit_e_at_0p4gev(void) {
  const double Tmax = 0.4 / GEVFM;
  double E = FEnFromTemp(Tmax), e0;
  while (fabs(s95p_T(E) - Tmax) > 1e-10) {
    e0 = E;
    E = e0 - (s95p_T(e0) - Tmax) / (6.608681233 * pow(e0, -0.25));
  }
  return E;
}

}  /* extern "C" */
