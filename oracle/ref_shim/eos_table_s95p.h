/* Stand-in for the reference's s95p.h in the table-EOS builds of the
 * reference harness (ref_harness.cpp with -DGINIT -DVH_REF_EOS_TABLE).
 *
 * The reference's GINIT scenario block (NEWEST5/maindef.h:240-295) is the one
 * whose EOS hooks call out to functions (s95p_p, s95p_a, s95p_T, s95p_s)
 * instead of being written inline, so defining those four here gives the
 * reference's step any tabulated EOS: the synthetic table of the benchmark
 * workloads, set at run time by ref_set_eos_table().  The lookup is the one
 * the oracle and the GPU use: linear in e between rows e_i <= e < e_{i+1};
 * below the first row P = cs2_0 e, T ~ e^(1/4); above the last row P grows
 * with the last cs2 and T ~ e^(1/4).  Entropy density s = (e + P)/T, which
 * the block's eta = s/(4 pi) uses.  Units: the table's (fm^-4, fm^-1).
 * Test infrastructure for the oracle only. */
#ifndef VH_REF_SHIM_EOS_TABLE_S95P_H
#define VH_REF_SHIM_EOS_TABLE_S95P_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int vh_tab_n = 0;
static double* vh_tab = 0; /* [4][n]: e, P, cs2, T */

static void vh_tab_eval(double e, double* P, double* cs2, double* T) {
  const int n = vh_tab_n;
  const double *te = vh_tab, *tp = vh_tab + n, *tc = vh_tab + 2 * n, *tt = vh_tab + 3 * n;
  if (e <= te[0]) {
    *cs2 = tc[0]; *P = tc[0] * e; *T = tt[0] * sqrt(sqrt(e / te[0]));
    return;
  }
  if (e >= te[n - 1]) {
    *cs2 = tc[n - 1]; *P = tp[n - 1] + tc[n - 1] * (e - te[n - 1]); *T = tt[n - 1] * sqrt(sqrt(e / te[n - 1]));
    return;
  }
  const double l0 = log(te[0]);
  const double dl = (log(te[n - 1]) - l0) / (n - 1);
  int i = (int)((log(e) - l0) / dl);
  if (i < 0) i = 0;
  if (i > n - 2) i = n - 2;
  while (i > 0 && e < te[i]) i--;
  while (i < n - 2 && e >= te[i + 1]) i++;
  const double w = (e - te[i]) / (te[i + 1] - te[i]);
  *P = tp[i] + w * (tp[i + 1] - tp[i]);
  *cs2 = tc[i] + w * (tc[i + 1] - tc[i]);
  *T = tt[i] + w * (tt[i + 1] - tt[i]);
}

double s95p_p(double e) { double P, c, T; vh_tab_eval(e, &P, &c, &T); return P; }
double s95p_a(double e) { double P, c, T; vh_tab_eval(e, &P, &c, &T); return c; }
double s95p_T(double e) { double P, c, T; vh_tab_eval(e, &P, &c, &T); return T; }
double s95p_s(double e) { double P, c, T; vh_tab_eval(e, &P, &c, &T); return (e + P) / T; }

extern "C" int ref_set_eos_table(int n, const double* t) {
  if (n < 2 || !t) return -1;
  double* c = (double*)malloc(sizeof(double) * 4 * (size_t)n);
  if (!c) return -1;
  memcpy(c, t, sizeof(double) * 4 * (size_t)n);
  free(vh_tab);
  vh_tab = c;
  vh_tab_n = n;
  return 0;
}

#endif
