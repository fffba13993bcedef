/* Reference harness for the snapshot writers: compiles the reference's
 * write.h where it lies (NEWEST5/write.h: WriteResultsXY and WriteResults,
 * 12 doubles per cell; with -DVH_REF_N10, NEWEST10/write.h: the 17-variable
 * WriteResultsXY and WriteNSXY) with its maindef.h scenario block, so that
 * tests can compare the files it writes with vh_write's byte for byte.
 * Test infrastructure only.
 *
 * What is ours: the globals and grid macros that init.h would declare for
 * one rank (NEWEST5/init.h:15-70: GRIDXPOINTS, jSTART, MYGLOBALiWB, ...),
 * every neighbour BOUNDARY, MPI-IO through ref_shim/mpi.h's stdio streams,
 * and the state import below.  The cell's derived fields are set as the
 * reference's root-find sets them (NEWEST5/multiroot.h:428-429, 485-492):
 * Temp = FT(En), P = EOS(En), V = u^i/u^tau; PI = 0.  The writers open
 * res/tau%2.3ffm.bin (and res/NStau...) relative to the working directory.
 */
#include <mpi.h>

#include <iostream>
#include <fstream>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#include <stdio.h>

#define GEVFM 0.1973
#define PIE 3.141592653589793

using namespace std;

#ifndef VH_REF_N10
#include "s95p.h"
#endif
#include "maindef.h"

/* ---- what init.h would declare, one rank (NEWEST5/init.h:15-70) ---- */
int k0;
int rank = 0, size = 1, root = 0;
int xcord = 0, ycord = 0, zcord = 0;
MPI_Comm mpi_grid = 0;
int il, jl, kl, ir, jr, kr;
#define BOUNDARY -1
#define MYXLEFT BOUNDARY
#define MYXRIGHT BOUNDARY
#define MYYLEFT BOUNDARY
#define MYYRIGHT BOUNDARY
#define GRIDXPOINTS (NPX * XCMA)
#define GRIDYPOINTS (NPY * YCMA)
#define iSTART (xcord * (XCMA))
#define jSTART (ycord * (YCMA))
#define iSTARTWB (iSTART)
#define jSTARTWB (jSTART)
inline int MYGLOBALi(int i) { return (iSTARTWB + i); }
inline int MYGLOBALj(int j) { return (jSTARTWB + j); }
inline int MYGLOBALiWB(int i) { return (iSTART + (i - BORDER)); }
inline int MYGLOBALjWB(int j) { return (jSTART + (j - BORDER)); }
#ifdef LBI
#define GRIDZPOINTS (1)
#else
#define GRIDZPOINTS (ZCMA)
#endif

#include "write.h"

static const size_t NCELL = (size_t)XCM * YCM * ZCM;
static inline size_t cidx(int i, int j, int k) { return ((size_t)k * YCM + j) * XCM + i; }

extern "C" {

/* XCM, YCM, ZCM, XCMA, YCMA, ZCMA, FREQ, FREQZ, LBI; consts XS, YS, ZS, FACTOR */
int refw_init(int* dims, double* consts) {
  if (!HydroGrid) HydroGrid = new cell[XCM][YCM][ZCM]();
  il = jl = BORDER;
  ir = il + XCMA;
  jr = jl + YCMA;
#ifdef LBI
  kl = 0; kr = 1; k0 = 0;
  dims[8] = 1;
#else
  kl = BORDER; kr = kl + ZCMA; k0 = (ZCM - 1) / 2;
  dims[8] = 0;
#endif
  dims[0] = XCM; dims[1] = YCM; dims[2] = ZCM; dims[3] = XCMA; dims[4] = YCMA; dims[5] = ZCMA;
  dims[6] = FREQ; dims[7] = FREQZ;
  consts[0] = XS; consts[1] = YS; consts[2] = ZS; consts[3] = FACTOR;
  return 9;
}

/* the canonical 18 fields (En, u^mu, pi^{xx,yy,xy,x eta,y eta}, ...) on
 * every cell; pi10 (10 x cells, NEWEST10's ten components) and nspi
 * (11 x cells: ten components and the bulk part) when not NULL */
void refw_set_state(const double* f, const double* pi10, const double* nspi) {
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        const size_t c = cidx(i, j, k);
        cell& h = HydroGrid[i][j][k];
        h.En = f[c];
        for (int l = 0; l < 4; l++) h.u[l] = f[(1 + l) * NCELL + c];
#ifdef VH_REF_N10
        for (int l = 0; l < 10; l++) h.pi[l] = pi10 ? pi10[l * NCELL + c] : 0.0;
        if (nspi) {
          for (int l = 0; l < 10; l++) h.nspi[l] = nspi[l * NCELL + c];
          h.nsPI = nspi[10 * NCELL + c];
        }
#else
        (void)pi10; (void)nspi;
        for (int l = 0; l < 5; l++) h.pi[l] = f[(5 + l) * NCELL + c];
#endif
        h.PI = 0;
        h.Temp = FT(h.En);
        h.P = EOS(h.En);
        h.Vx = h.u[1] / h.u[0];
        h.Vy = h.u[2] / h.u[0];
        h.Ve = h.u[3] / h.u[0];
      }
}

void refw_write_xy(double tau) { WriteResultsXY(tau, HydroGrid); }
#ifdef VH_REF_N10
void refw_write_ns_xy(double tau) { WriteNSXY(tau, HydroGrid); }
#else
void refw_write_full(double tau) { WriteResults(tau, HydroGrid); }
#endif

}  /* extern "C" */
