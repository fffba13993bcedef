/* Reference harness for NEWEST10's Navier-Stokes shear tensor: compiles the
 * reference's NEWEST10 headers where they lie (maindef.h, utils.h,
 * Source.h under the reference tree, passed with -iquote) into a shared
 * library, so that tests can evaluate the reference's CalcNS
 * (NEWEST10/Source.h:643-753), all ten components of pi^{mu nu}_NS and the
 * bulk nsPI, on a state we choose.  Test infrastructure only.
 *
 * The scenario is NEWEST10's default compile-time block (maindef.h:36-87:
 * conformal EOS e = FACTOR T^4, eta = s/(4 pi), dx = dy = 0.1, 40 x 40
 * interior cells) with LBI (one eta cell).  In that build CalcDer4Vel
 * (Source.h:3-95) computes d_tau u^l and the x, y derivatives but leaves
 * du[l][3] alone, so the caller supplies du[l][3]: with u^eta and d_eta u
 * set freely every term of the ten polynomials is exercised.
 *
 * What is ours: the globals that NEWEST10/init.h would declare, the grid
 * allocation and the state import/export below.  Canonical state layout
 * as the oracle's: structure of arrays over the ghost-inclusive grid, index
 * (k*YCM + j)*XCM + i; fields 0 En, 1..4 u^0..u^3, 14..17 prevu^0..3 of 18.
 */
#include <mpi.h>

#include <iostream>
#include <fstream>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#include <float.h>

#define GEVFM 0.1973
#define PIE 3.141592653589793

using namespace std;

#include "maindef.h"

/* ---- what NEWEST10/init.h would declare, one rank ---- */
int k0;
int rank = 0, size = 1, root = 0;
MPI_Comm mpi_grid = 0;
int il, jl, kl, ir, jr, kr;

#include "utils.h"
#include "Source.h"

static const size_t NCELL = (size_t)XCM * YCM * ZCM;
static inline size_t cidx(int i, int j, int k) { return ((size_t)k * YCM + j) * XCM + i; }

extern "C" {

/* allocate the grid and set the interior bounds (one rank) */
int ref10_init(int* dims, double* consts) {
  if (!HydroGrid) HydroGrid = new cell[XCM][YCM][ZCM]();
  il = jl = BORDER;
  ir = il + XCMA;
  jr = jl + YCMA;
  kl = 0;
  kr = 1;
  dims[0] = XCM; dims[1] = YCM; dims[2] = ZCM;
  dims[3] = il; dims[4] = ir; dims[5] = jl; dims[6] = jr; dims[7] = kl; dims[8] = kr;
  consts[0] = XS; consts[1] = YS; consts[2] = FACTOR;
  return 9;
}

/* f: 18 x NCELL canonical state (En, u, prevu used); du3: 4 x NCELL values
 * of du[l][3].  Runs CalcNS(HydroGrid, tau, ts) and returns nspi[0..9] and
 * nsPI (11 x NCELL) and the du[l][m] it used (16 x NCELL, l*4+m). */
void ref10_calc_ns(const double* f, const double* du3, double tau, double ts, double* ns, double* du) {
  for (int k = 0; k < ZCM; k++)
    for (int j = 0; j < YCM; j++)
      for (int i = 0; i < XCM; i++) {
        const size_t c = cidx(i, j, k);
        cell& q = HydroGrid[i][j][k];
        q.En = f[c];
        q.P = EOS(q.En);
        q.PI = 0;
        q.Temp = FT(q.En);
        for (int l = 0; l < 4; l++) {
          q.u[l] = f[(1 + l) * NCELL + c];
          q.prevu[l] = f[(14 + l) * NCELL + c];
          for (int m = 0; m < 4; m++) q.du[l][m] = 0;
          q.du[l][3] = du3[l * NCELL + c];
        }
        for (int l = 0; l < Npi; l++) q.pi[l] = 0;
      }
  CalcNS(HydroGrid, tau, ts);
  for (int k = 0; k < ZCM; k++)
    for (int j = 0; j < YCM; j++)
      for (int i = 0; i < XCM; i++) {
        const size_t c = cidx(i, j, k);
        const cell& q = HydroGrid[i][j][k];
        for (int l = 0; l < Npi; l++) ns[l * NCELL + c] = q.nspi[l];
        ns[10 * NCELL + c] = q.nsPI;
        for (int l = 0; l < 4; l++)
          for (int m = 0; m < 4; m++) du[(l * 4 + m) * NCELL + c] = q.du[l][m];
      }
}

}  /* extern "C" */
