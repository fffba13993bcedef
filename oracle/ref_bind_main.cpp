/* The binding a maintainer adds to the reference (the
 * vh_bind.h block, extracted into _ref/vh_bind.h by oracle/Makefile) in a
 * program of the reference's main-loop shape (NEWEST5/main.cpp:90-223):
 * the reference's maindef.h scenario block and cell type, the cells loaded
 * the way init() would leave them, then TVDRK2 / tau += ts / MaxTempGev /
 * the snapshot writes of main.cpp:132-206, with the binding's TVDRK2,
 * MaxTempGev and WriteResults[XY] in place of time.h, utils.h and write.h.
 * After the steps vh_unpack fills the cells, which are written out in the
 * canonical layout.  Test infrastructure: it checks the documented binding.
 *
 *   vh_bind_run_3d STATE_IN STATE_OUT STEPS TAU0 TS
 * STATE_IN/OUT: 18 x XCM*YCM*ZCM doubles (En, u^mu, pi^{xx,yy,xy,x eta,y eta},
 * T^{tau mu}, prevu^mu; index (k*YCM + j)*XCM + i).  Snapshots go to res/.
 * What is ours: the state import/export and the argument handling; the
 * globals init.h would declare for one rank.
 */
#include <mpi.h>

#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <math.h>
#include <vector>

#define GEVFM 0.1973
#define PIE 3.141592653589793

using namespace std;

#include "s95p.h"
#include "maindef.h"

int k0;
int rank = 0, size = 1, root = 0;
MPI_Comm mpi_grid = 0;
int il, jl, kl, ir, jr, kr;

#include "vh_bind.h"

static const size_t NCELL = (size_t)XCM * YCM * ZCM;
static inline size_t cidx(int i, int j, int k) { return ((size_t)k * YCM + j) * XCM + i; }

int main(int argc, char** argv) {
  if (argc < 6) { fprintf(stderr, "usage: %s STATE_IN STATE_OUT STEPS TAU0 TS\n", argv[0]); return 2; }
  const int steps = atoi(argv[3]);
  double tau = atof(argv[4]), ts = atof(argv[5]);
  std::vector<double> f(18 * NCELL);
  FILE* fi = fopen(argv[1], "rb");
  if (!fi || fread(f.data(), sizeof(double), f.size(), fi) != f.size()) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
  fclose(fi);
  // the grid and the cells as init() leaves them (NEWEST5/alloc.h:33-36, init.h:539-549)
  HydroGrid = new cell[XCM][YCM][ZCM]();
  il = jl = BORDER; ir = il + XCMA; jr = jl + YCMA;
#ifdef LBI
  kl = 0; kr = 1; k0 = 0;
#else
  kl = BORDER; kr = kl + ZCMA; k0 = (ZCM - 1) / 2;
#endif
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        const size_t c = cidx(i, j, k);
        cell& h = HydroGrid[i][j][k];
        h.En = f[c];
        for (int l = 0; l < 4; l++) { h.u[l] = f[(1 + l) * NCELL + c]; h.prevu[l] = f[(14 + l) * NCELL + c]; }
        for (int l = 0; l < 5; l++) h.pi[l] = f[(5 + l) * NCELL + c];
        h.T00 = f[10 * NCELL + c]; h.T10 = f[11 * NCELL + c]; h.T20 = f[12 * NCELL + c]; h.T30 = f[13 * NCELL + c];
        h.P = EOS(h.En); h.Temp = FT(h.En);
      }
  const double tau0 = tau;
  // NEWEST5/main.cpp:118-206, with the step count as the break
#ifdef LBI
  WriteResultsXY(tau, HydroGrid);
#else
  WriteResults(tau, HydroGrid);
#endif
  for (int l = 1; l <= steps; l++) {
    TVDRK2(HydroGrid, tau, ts);
    tau += ts;
    const double tmaxMev = 1000 * MaxTempGev(HydroGrid);
    cout << "Time Step is " << ts << " @ " << std::fixed << std::setprecision(4) << " TempMax is " << tmaxMev
         << " MeV at TAU -->" << tau << " This is tau step no. " << l << endl;
#ifdef LBI
    if (fabs(tau - (tau0 + ts)) < 1e-6) WriteResultsXY(tau, HydroGrid);
#else
    if (fabs(tau - (tau0 + ts)) < 1e-6) WriteResults(tau, HydroGrid);
#endif
  }
  vh_unpack(HydroGrid);
  for (int i = 0; i < XCM; i++)
    for (int j = 0; j < YCM; j++)
      for (int k = 0; k < ZCM; k++) {
        const size_t c = cidx(i, j, k);
        const cell& h = HydroGrid[i][j][k];
        f[c] = h.En;
        for (int l = 0; l < 4; l++) { f[(1 + l) * NCELL + c] = h.u[l]; f[(14 + l) * NCELL + c] = h.prevu[l]; }
        for (int l = 0; l < 5; l++) f[(5 + l) * NCELL + c] = h.pi[l];
        f[10 * NCELL + c] = h.T00; f[11 * NCELL + c] = h.T10; f[12 * NCELL + c] = h.T20; f[13 * NCELL + c] = h.T30;
        // the derived fields vh_unpack set, checked here against their definitions
        if (h.P != EOS(h.En) || h.Temp != FT(h.En) || h.Vx != h.u[1] / h.u[0]) { fprintf(stderr, "derived fields\n"); return 3; }
      }
  FILE* fo = fopen(argv[2], "wb");
  if (!fo || fwrite(f.data(), sizeof(double), f.size(), fo) != f.size()) { fprintf(stderr, "cannot write %s\n", argv[2]); return 2; }
  fclose(fo);
  return 0;
}
