// Reverse-mode (vector-Jacobian) building blocks of the discrete adjoint of
// the boost-invariant Milne step.  Each function recomputes the forward
// values it needs from the same inputs as the forward kernels (so branch
// choices -- max-speed selection, EOS table row, the eta/s(T) kink -- are the
// forward pass's) and propagates adjoints by hand.  Host+device so that each
// piece can be checked against finite differences on the CPU.
//
// Boost invariance: u^eta, pi^{x eta}, pi^{y eta}, T^{tau eta} and every eta
// derivative are identically zero at all times (their sources vanish), so
// their adjoints are never needed and are not propagated.
//
// Flux quantities of one direction (13): F^0,F^1,F^2 (tau T^{d mu}, mu =
// tau,x,y), F^4..F^6 (pi^{xx,yy,xy} v^d), V^0..V^2 (tau T^{tau mu}),
// V^4..V^6 (pi), and the signal speed s.
#pragma once

#include "vh_device.cuh"

namespace vh {

constexpr int NQ = 13;  // flux quantities per direction in 2+1D

// P, dP/de, T, dT/de of the EOS interpolant (the derivative of what the
// forward evaluates, not the tabulated c_s^2)
template <class R>
VH_HD inline void eos_d(const DevCfg& C, R e, R& P, R& dP, R& T, R& dT) {
  if (C.eos_kind == 0) {
    P = e / (R)3;
    dP = (R)1 / (R)3;
    T = conf_T(e / (R)C.eos_a);
    dT = T / ((R)4 * e);
    return;
  }
  const R* t = eos_tab<R>(C);
  const int n = C.eos_n;
  const R *te = t, *tp = t + n, *tc = t + 2 * n, *tt = t + 3 * n;
  if (e <= te[0]) {
    P = tc[0] * e; dP = tc[0];
    T = tt[0] * d_sqrt(d_sqrt(e / te[0])); dT = T / ((R)4 * e);
    return;
  }
  if (e >= te[n - 1]) {
    P = tp[n - 1] + tc[n - 1] * (e - te[n - 1]); dP = tc[n - 1];
    T = tt[n - 1] * d_sqrt(d_sqrt(e / te[n - 1])); dT = T / ((R)4 * e);
    return;
  }
  const int i = eos_row<R>(C, te, e);
  const R de = te[i + 1] - te[i];
  const R w = (e - te[i]) / de;
  P = tp[i] + w * (tp[i + 1] - tp[i]);
  T = tt[i] + w * (tt[i + 1] - tt[i]);
  dP = (tp[i + 1] - tp[i]) / de;
  dT = (tt[i + 1] - tt[i]) / de;
}

// ------------------------------------------------------------------ WENO

// the weights' adjoint in the normalised form (alpha_k = d_k / E_k): five
// reciprocals, but no product of E's, so its range is that of FP32 as well
template <class R>
VH_HD inline void weno_wvjp(const R* E, const R* e, const R* ql, const R* qr, R Lbar, R Rbar, R* qlb, R* qrb,
                            R* eb) {
  const R dl[3] = {(R)0.3, (R)0.6, (R)0.1}, dr[3] = {(R)0.1, (R)0.6, (R)0.3};
  // five reciprocals instead of a division per use
  const R iE[3] = {(R)1 / E[0], (R)1 / E[1], (R)1 / E[2]};
  R al[3], ar[3], sl = 0, sr = 0;
  for (int k = 0; k < 3; k++) { al[k] = dl[k] * iE[k]; ar[k] = dr[k] * iE[k]; sl += al[k]; sr += ar[k]; }
  const R isl = (R)1 / sl, isr = (R)1 / sr;
  R wl[3], wr[3];
  for (int k = 0; k < 3; k++) { wl[k] = al[k] * isl; wr[k] = ar[k] * isr; }
  // candidates
  const R L6 = Lbar * ((R)1 / (R)6), R6 = Rbar * ((R)1 / (R)6);
  R wlb[3], wrb[3];
  for (int k = 0; k < 3; k++) {
    qlb[k] = wl[k] * L6; qrb[k] = wr[k] * R6;
    wlb[k] = ql[k] * L6; wrb[k] = qr[k] * R6;
  }
  R swl = 0, swr = 0;
  for (int k = 0; k < 3; k++) { swl += wl[k] * wlb[k]; swr += wr[k] * wrb[k]; }
  for (int k = 0; k < 3; k++) {
    const R alb = (wlb[k] - swl) * isl, arb = (wrb[k] - swr) * isr;
    const R Eb = -(alb * al[k] + arb * ar[k]) * iE[k];
    eb[k] = Eb * (R)2 * e[k];  // d(e^2) and e = eps + beta: betabar = Ebar 2 e
  }
}

// q = (q_{i-2}..q_{i+2}); adjoints Lbar of the face value at i+1/2 and Rbar
// of the face value at i-1/2 are pulled back into qbar (accumulated)
template <class R>
VH_HD inline void weno_lr_vjp(const R* q, R Lbar, R Rbar, R* qbar) {
  const R c13 = (R)(13. / 12.), eps = (R)1e-6;
  const R a0 = q[2] - (R)2 * q[3] + q[4], g0 = (R)3 * q[2] - (R)4 * q[3] + q[4];
  const R a1 = q[1] - (R)2 * q[2] + q[3], g1 = q[1] - q[3];
  const R a2 = q[0] - (R)2 * q[1] + q[2], g2 = q[0] - (R)4 * q[1] + (R)3 * q[2];
  const R e[3] = {eps + c13 * a0 * a0 + (R)0.25 * g0 * g0, eps + c13 * a1 * a1 + (R)0.25 * g1 * g1,
                  eps + c13 * a2 * a2 + (R)0.25 * g2 * g2};
  const R E[3] = {e[0] * e[0], e[1] * e[1], e[2] * e[2]};
  const R ql[3] = {(R)2 * q[2] + (R)5 * q[3] - q[4], -q[1] + (R)5 * q[2] + (R)2 * q[3],
                   (R)2 * q[0] - (R)7 * q[1] + (R)11 * q[2]};
  const R qr[3] = {(R)11 * q[2] - (R)7 * q[3] + (R)2 * q[4], (R)2 * q[1] + (R)5 * q[2] - q[3],
                   -q[0] + (R)5 * q[1] + (R)2 * q[2]};
  R qlb[3], qrb[3], eb[3];
  if constexpr (sizeof(R) == 8) {
    // the forward's product form (weights proportional to d_k prod_{j != k}
    // E_j, both faces' normalisations through one reciprocal): one FP64
    // reciprocal instead of five; the products stay far inside double range
    const R P12 = E[1] * E[2], P02 = E[0] * E[2], P01 = E[0] * E[1];
    const R nl[3] = {(R)0.3 * P12, (R)0.6 * P02, (R)0.1 * P01}, nr[3] = {(R)0.1 * P12, (R)0.6 * P02, (R)0.3 * P01};
    const R numl = nl[0] * ql[0] + nl[1] * ql[1] + nl[2] * ql[2], denl = (R)6 * (nl[0] + nl[1] + nl[2]);
    const R numr = nr[0] * qr[0] + nr[1] * qr[1] + nr[2] * qr[2], denr = (R)6 * (nr[0] + nr[1] + nr[2]);
    const R inv = (R)1 / (denl * denr), idl = denr * inv, idr = denl * inv;
    const R numlb = Lbar * idl, denlb = -Lbar * numl * idl * idl;
    const R numrb = Rbar * idr, denrb = -Rbar * numr * idr * idr;
    R nlb[3], nrb[3];
    for (int k = 0; k < 3; k++) {
      qlb[k] = nl[k] * numlb;
      qrb[k] = nr[k] * numrb;
      nlb[k] = ql[k] * numlb + (R)6 * denlb;
      nrb[k] = qr[k] * numrb + (R)6 * denrb;
    }
    const R P12b = (R)0.3 * nlb[0] + (R)0.1 * nrb[0], P02b = (R)0.6 * (nlb[1] + nrb[1]),
            P01b = (R)0.1 * nlb[2] + (R)0.3 * nrb[2];
    const R Eb[3] = {P02b * E[2] + P01b * E[1], P12b * E[2] + P01b * E[0], P12b * E[1] + P02b * E[0]};
    for (int k = 0; k < 3; k++) eb[k] = Eb[k] * (R)2 * e[k];
  } else {
    weno_wvjp<R>(E, e, ql, qr, Lbar, Rbar, qlb, qrb, eb);
  }
  const R a0b = eb[0] * (R)2 * c13 * a0, g0b = eb[0] * (R)0.5 * g0;
  const R a1b = eb[1] * (R)2 * c13 * a1, g1b = eb[1] * (R)0.5 * g1;
  const R a2b = eb[2] * (R)2 * c13 * a2, g2b = eb[2] * (R)0.5 * g2;
  qbar[0] += (R)2 * qlb[2] - qrb[2] + a2b + g2b;
  qbar[1] += -qlb[1] - (R)7 * qlb[2] + (R)2 * qrb[1] + (R)5 * qrb[2] + a1b + g1b - (R)2 * a2b - (R)4 * g2b;
  qbar[2] += (R)2 * qlb[0] + (R)5 * qlb[1] + (R)11 * qlb[2] + (R)11 * qrb[0] + (R)5 * qrb[1] + (R)2 * qrb[2] + a0b +
             (R)3 * g0b - (R)2 * a1b + a2b + (R)3 * g2b;
  qbar[3] += (R)5 * qlb[0] + (R)2 * qlb[1] - (R)7 * qrb[0] - qrb[1] - (R)2 * a0b - (R)4 * g0b + a1b - g1b;
  qbar[4] += -qlb[0] + (R)2 * qrb[0] + a0b + g0b;
}

// ---------------------------------------------------------- flux quantities

// Forward flux quantities of one cell, 2+1D (u3 = p4 = p5 = T3 = 0):
// x = (e, u0, u1, u2, p1, p2, p3, T0, T1, T2)
template <class R, int DIR>
VH_HD inline void cell_q(const DevCfg& C, R tau, const R* x, bool interior, R* q) {
  const R e = x[0], u0 = x[1], u1 = x[2], u2 = x[3], p1 = x[4], p2 = x[5], p3 = x[6];
  const R P = eos_P<R>(C, e), ep = e + P, iu0 = (R)1 / u0;
  if (DIR == 0) {
    const R pt = (p1 * u1 + p3 * u2) * iu0;
    q[0] = tau * (pt + u1 * u0 * ep);
    q[1] = tau * (p1 + P + u1 * u1 * ep);
    q[2] = tau * (p3 + u1 * u2 * ep);
    q[3] = p1 * u1 * iu0; q[4] = p2 * u1 * iu0; q[5] = p3 * u1 * iu0;
    q[12] = interior ? u1 * iu0 : (R)0;
  } else {
    const R pt = (p3 * u1 + p2 * u2) * iu0;
    q[0] = tau * (pt + u2 * u0 * ep);
    q[1] = tau * (p3 + u2 * u1 * ep);
    q[2] = tau * (p2 + P + u2 * u2 * ep);
    q[3] = p1 * u2 * iu0; q[4] = p2 * u2 * iu0; q[5] = p3 * u2 * iu0;
    q[12] = interior ? u2 * iu0 : (R)0;
  }
  q[6] = tau * x[7]; q[7] = tau * x[8]; q[8] = tau * x[9];
  q[9] = p1; q[10] = p2; q[11] = p3;
}

// xbar += (d q / d x)^T qbar
template <class R, int DIR>
VH_HD inline void cell_q_vjp(const DevCfg& C, R tau, const R* x, bool interior, const R* qb, R* xb) {
  const R e = x[0], u0 = x[1], u1 = x[2], u2 = x[3], p1 = x[4], p2 = x[5], p3 = x[6];
  R P, dP, T, dT;
  eos_d<R>(C, e, P, dP, T, dT);
  const R ep = e + P, iu0 = (R)1 / u0;
  R eb = 0, u0b = 0, u1b = 0, u2b = 0, p1b = 0, p2b = 0, p3b = 0, epb = 0, Pb = 0;
  const R v = DIR == 0 ? u1 : u2;  // velocity along the direction
  R vb = 0;
  // pi^{tau d}
  const R pt = DIR == 0 ? (p1 * u1 + p3 * u2) * iu0 : (p3 * u1 + p2 * u2) * iu0;
  const R ptb = tau * qb[0];
  vb += tau * qb[0] * u0 * ep;
  u0b += tau * qb[0] * v * ep;
  epb += tau * qb[0] * v * u0;
  if (DIR == 0) {
    p1b += ptb * u1 * iu0; p3b += ptb * u2 * iu0; u1b += ptb * p1 * iu0; u2b += ptb * p3 * iu0;
    // q1 = tau (p1 + P + u1 u1 ep), q2 = tau (p3 + u1 u2 ep)
    p1b += tau * qb[1]; Pb += tau * qb[1]; vb += tau * qb[1] * (R)2 * u1 * ep; epb += tau * qb[1] * u1 * u1;
    p3b += tau * qb[2]; vb += tau * qb[2] * u2 * ep; u2b += tau * qb[2] * u1 * ep; epb += tau * qb[2] * u1 * u2;
  } else {
    p3b += ptb * u1 * iu0; p2b += ptb * u2 * iu0; u1b += ptb * p3 * iu0; u2b += ptb * p2 * iu0;
    // q1 = tau (p3 + u2 u1 ep), q2 = tau (p2 + P + u2 u2 ep)
    p3b += tau * qb[1]; vb += tau * qb[1] * u1 * ep; u1b += tau * qb[1] * u2 * ep; epb += tau * qb[1] * u2 * u1;
    p2b += tau * qb[2]; Pb += tau * qb[2]; vb += tau * qb[2] * (R)2 * u2 * ep; epb += tau * qb[2] * u2 * u2;
  }
  u0b -= ptb * pt * iu0;
  // q3..q5 = p v / u0
  p1b += qb[3] * v * iu0; p2b += qb[4] * v * iu0; p3b += qb[5] * v * iu0;
  vb += (qb[3] * p1 + qb[4] * p2 + qb[5] * p3) * iu0;
  u0b -= (qb[3] * p1 + qb[4] * p2 + qb[5] * p3) * v * iu0 * iu0;
  // speed
  if (interior) { vb += qb[12] * iu0; u0b -= qb[12] * v * iu0 * iu0; }
  // Var
  xb[7] += tau * qb[6]; xb[8] += tau * qb[7]; xb[9] += tau * qb[8];
  p1b += qb[9]; p2b += qb[10]; p3b += qb[11];
  // e + P
  eb += epb; Pb += epb;
  eb += Pb * dP;
  if (DIR == 0) u1b += vb; else u2b += vb;
  xb[0] += eb; xb[1] += u0b; xb[2] += u1b; xb[3] += u2b;
  xb[4] += p1b; xb[5] += p2b; xb[6] += p3b;
}

// ---------------------------------------------------------------- source

// Forward 2+1D source of (tau T^{tau tau}, pi^xx, pi^yy, pi^xy) at one cell:
// out = {S0, Sxx, Syy, Sxy}; du is 3x3 (l, m in tau,x,y); c0, c1 of eta/s(T)
template <class R>
VH_HD inline void src2d(const DevCfg& C, R tau, R e, const R* u3v, const R* p3v, const R* du9, R* out) {
  const R u[4] = {u3v[0], u3v[1], u3v[2], (R)0};
  const R p[5] = {p3v[0], p3v[1], p3v[2], (R)0, (R)0};
  R du[4][4];
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) du[l][m] = (l < 3 && m < 3) ? du9[l * 3 + m] : (R)0;
  const R t2 = tau * tau;
  const R P = eos_P<R>(C, e);
  PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  out[0] = -P - t2 * (d.ee + (e + P) * u[3] * u[3]);
  R s5[5];
  is_source<R>(C, tau, e, u, p, du, s5);
  out[1] = s5[0]; out[2] = s5[1]; out[3] = s5[2];
}

// Adjoint of src2d, accumulated: ob[4] -> eb, ub3 (u0,u1,u2), pb[3], dub[9],
// cb[2] (c0, c1)
template <class R>
VH_HD inline void src2d_vjp(const DevCfg& C, R tau, R e, const R* u3v, const R* p3v, const R* du9, const R* ob,
                            R& eb, R* ub3, R* pb, R* dub, R* cb) {
  const R u[4] = {u3v[0], u3v[1], u3v[2], (R)0};
  const R t2 = tau * tau, itau = (R)1 / tau;
  const R g[4] = {(R)1, (R)-1, (R)-1, -t2};
  const R gi[4] = {(R)1, (R)-1, (R)-1, (R)-1 / t2};
  // ---- forward recompute
  R P, dP, T, dT;
  eos_d<R>(C, e, P, dP, T, dT);
  const R iT = (R)1 / T, iep = (R)1 / (e + P), iP = (R)1 / P;
  const R s = (e + P) * iT;
  const R tg = T * (R)C.hbarc - (R)C.etas_tc;
  const bool kink = tg > (R)0;
  const R etas = (R)C.etas0 + (R)C.etas1 * (kink ? tg : (R)0);
  const R eta = etas * s;
  const R tp = C.taupi_kind == 1 ? (R)5 * eta * iep : C.taupi_kind == 2 ? (R)C.taupi_c : (R)1.5 * (eta * iP);
  const R itp = (R)1 / tp;
  const R u0 = u[0], u1 = u[1], u2 = u[2];
  const R iu0 = (R)1 / u0, iD = iu0 * iu0, it2 = (R)1 / t2;
  const R p1 = p3v[0], p2 = p3v[1], p3 = p3v[2];
  const R D = u0 * u0;
  const R Q = u1 * u1 * p1 + (R)2 * u1 * u2 * p3 + u2 * u2 * p2;
  const R ptt = Q * iD, pee = (Q - D * (p1 + p2)) * it2 * iD;
  const R ptx = (p1 * u1 + p3 * u2) * iu0, pty = (p3 * u1 + p2 * u2) * iu0;
  R pi[4][4] = {{ptt, ptx, pty, 0}, {ptx, p1, p3, 0}, {pty, p3, p2, 0}, {0, 0, 0, pee}};
  R Dm[4][4];
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) Dm[l][m] = (l < 3 && m < 3) ? du9[l * 3 + m] : (R)0;
  Dm[3][3] += u0 * itau;
  R Dl[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dl[a][b] = g[b] * Dm[b][a];
  const R th = Dm[0][0] + Dm[1][1] + Dm[2][2] + Dm[3][3];
  R Dt[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dt[a][b] = (a == b ? gi[a] : (R)0) - u[a] * u[b];
  R tr = 0;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) tr += Dt[a][b] * Dl[a][b];
  const R tr3 = tr / (R)3;
  R S[4][4], M[3][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) S[a][b] = (R)0.5 * (Dl[a][b] + Dl[b][a]);
  for (int m = 1; m < 3; m++)
    for (int b = 0; b < 4; b++) {
      R acc = 0;
      for (int a = 0; a < 4; a++) acc += Dt[m][a] * S[a][b];
      M[m][b] = acc;
    }
  R sig[3][3];
  for (int m = 1; m < 3; m++)
    for (int v = 1; v < 3; v++) {
      R acc = 0;
      for (int b = 0; b < 4; b++) acc += M[m][b] * Dt[v][b];
      sig[m][v] = acc - Dt[m][v] * tr3;
    }
  R acc4[4];
  for (int v = 0; v < 4; v++) {
    R a = 0;
    for (int b = 0; b < 4; b++) a += u[b] * Dm[v][b];
    acc4[v] = g[v] * a;
  }
  R pa[4];
  for (int v = 0; v < 4; v++) pa[v] = pi[v][0] * acc4[0] + pi[v][1] * acc4[1] + pi[v][2] * acc4[2] + pi[v][3] * acc4[3];
  R divv = 0;
  for (int i = 1; i < 3; i++) divv += du9[i * 3 + i] * iu0 - u[i] * du9[i] * iD;

  // ---- reverse
  R u0b = 0, u1b = 0, u2b = 0, p1b = 0, p2b = 0, p3b = 0, Pb = 0, etab = 0, tpb = 0, thb = 0, divvb = 0;
  R pib[4][4] = {}, sigb[3][3] = {}, pab[4] = {}, accb[4] = {}, Dmb[4][4] = {};
  R ub[4] = {0, 0, 0, 0};
  // geometric: out0 = -P - t2 * pee (u3 = 0)
  Pb -= ob[0];
  pib[3][3] -= t2 * ob[0];
  const int MU[3] = {1, 2, 1}, NU[3] = {1, 2, 2};
  for (int q = 0; q < 3; q++) {
    const R o = ob[1 + q];
    if (o == (R)0) continue;
    const int m = MU[q], v = NU[q];
    const R rhs = -(pi[m][v] - (R)2 * eta * sig[m][v]) * itp - ((R)4 / (R)3) * pi[m][v] * th - (u[m] * pa[v] + u[v] * pa[m]);
    const R rb = o * iu0;
    u0b -= o * rhs * iD;
    pib[m][v] += o * divv;
    divvb += o * pi[m][v];
    pib[m][v] += -rb * itp - ((R)4 / (R)3) * th * rb;
    sigb[m][v] += (R)2 * eta * rb * itp;
    etab += (R)2 * sig[m][v] * rb * itp;
    tpb += (pi[m][v] - (R)2 * eta * sig[m][v]) * rb * (itp * itp);
    thb += -((R)4 / (R)3) * pi[m][v] * rb;
    ub[m] -= pa[v] * rb; pab[v] -= u[m] * rb;
    ub[v] -= pa[m] * rb; pab[m] -= u[v] * rb;
  }
  // divv = sum_i du[i][i]/u0 - u_i du[0][i]/u0^2
  for (int i = 1; i < 3; i++) {
    dub[i * 3 + i] += divvb * iu0;
    u0b += divvb * (-du9[i * 3 + i] * iD + (R)2 * u[i] * du9[i] * iD * iu0);
    ub[i] -= divvb * du9[i] * iD;
    dub[i] -= divvb * u[i] * iD;
  }
  // pa[v] = sum_b pi[v][b] acc[b]
  for (int v = 0; v < 4; v++)
    for (int b = 0; b < 4; b++) { pib[v][b] += pab[v] * acc4[b]; accb[b] += pab[v] * pi[v][b]; }
  // acc[v] = g[v] sum_b u[b] Dm[v][b]
  for (int v = 0; v < 4; v++)
    for (int b = 0; b < 4; b++) { ub[b] += accb[v] * g[v] * Dm[v][b]; Dmb[v][b] += accb[v] * g[v] * u[b]; }
  // sig[m][v] = sum_b M[m][b] Dt[v][b] - Dt[m][v] tr3
  R Mb[3][4] = {}, Dtb[4][4] = {}, Sb[4][4] = {}, Dlb[4][4] = {};
  R tr3b = 0;
  for (int m = 1; m < 3; m++)
    for (int v = 1; v < 3; v++) {
      const R sb = sigb[m][v];
      if (sb == (R)0) continue;
      for (int b = 0; b < 4; b++) { Mb[m][b] += sb * Dt[v][b]; Dtb[v][b] += sb * M[m][b]; }
      Dtb[m][v] -= sb * tr3;
      tr3b -= sb * Dt[m][v];
    }
  // M[m][b] = sum_a Dt[m][a] S[a][b]
  for (int m = 1; m < 3; m++)
    for (int b = 0; b < 4; b++)
      for (int a = 0; a < 4; a++) { Dtb[m][a] += Mb[m][b] * S[a][b]; Sb[a][b] += Mb[m][b] * Dt[m][a]; }
  // S = (Dl + Dl^T)/2
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { Dlb[a][b] += (R)0.5 * Sb[a][b]; Dlb[b][a] += (R)0.5 * Sb[a][b]; }
  // tr = sum Dt Dl
  const R trb = tr3b / (R)3;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { Dtb[a][b] += trb * Dl[a][b]; Dlb[a][b] += trb * Dt[a][b]; }
  // Dt[a][b] = gi delta - u_a u_b
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { ub[a] -= Dtb[a][b] * u[b]; ub[b] -= Dtb[a][b] * u[a]; }
  // th = trace Dm
  for (int l = 0; l < 4; l++) Dmb[l][l] += thb;
  // Dl[a][b] = g[b] Dm[b][a]
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dmb[b][a] += Dlb[a][b] * g[b];
  // Christoffel term Dm[3][3] += u0 / tau
  ub[0] += Dmb[3][3] * itau;
  for (int l = 0; l < 3; l++)
    for (int m = 0; m < 3; m++) dub[l * 3 + m] += Dmb[l][m];
  // closure: symmetric pi entries share one variable
  const R pttb = pib[0][0], ptxb = pib[0][1] + pib[1][0], ptyb = pib[0][2] + pib[2][0];
  p1b += pib[1][1]; p2b += pib[2][2]; p3b += pib[1][2] + pib[2][1];
  const R peeb = pib[3][3];
  // ptt = Q/D, pee = (Q - D (p1+p2))/(t2 D), D = u0^2
  const R Qb = pttb * iD + peeb * it2 * iD;
  const R Db = -pttb * ptt * iD + peeb * (-(p1 + p2) * it2 * iD - pee * iD);
  p1b -= peeb * it2; p2b -= peeb * it2;
  ub[0] += (R)2 * u0 * Db;
  p1b += Qb * u1 * u1; p2b += Qb * u2 * u2; p3b += Qb * (R)2 * u1 * u2;
  ub[1] += Qb * ((R)2 * u1 * p1 + (R)2 * u2 * p3);
  ub[2] += Qb * ((R)2 * u1 * p3 + (R)2 * u2 * p2);
  // ptx = (p1 u1 + p3 u2)/u0, pty = (p3 u1 + p2 u2)/u0
  p1b += ptxb * u1 * iu0; p3b += ptxb * u2 * iu0; ub[1] += ptxb * p1 * iu0; ub[2] += ptxb * p3 * iu0; ub[0] -= ptxb * ptx * iu0;
  p3b += ptyb * u1 * iu0; p2b += ptyb * u2 * iu0; ub[1] += ptyb * p3 * iu0; ub[2] += ptyb * p2 * iu0; ub[0] -= ptyb * pty * iu0;
  // transport: eta = etas s, s = (e+P)/T, etas = c0 + c1 max(T hbarc - tc, 0), tp
  R eb_ = 0, Tb = 0;
  if (C.taupi_kind == 1) {
    etab += tpb * (R)5 * iep;
    const R eppb = -tpb * (R)5 * eta * (iep * iep);
    eb_ += eppb; Pb += eppb;
  } else if (C.taupi_kind == 0) {
    etab += tpb * (R)1.5 * iP;
    Pb -= tpb * (R)1.5 * eta * (iP * iP);
  }
  const R etasb = etab * s, sb = etab * etas;
  cb[0] += etasb;
  cb[1] += etasb * (kink ? tg : (R)0);
  if (kink) Tb += etasb * (R)C.etas1 * (R)C.hbarc;
  eb_ += sb * iT; Pb += sb * iT; Tb -= sb * s * iT;
  eb_ += Pb * dP + Tb * dT;
  eb += eb_;
  ub3[0] += ub[0] + u0b;
  ub3[1] += ub[1] + u1b;
  ub3[2] += ub[2] + u2b;
  pb[0] += p1b; pb[1] += p2b; pb[2] += p3b;
}

// ------------------------------------------------------------- con2prim
// Adjoint of the root x = (e, u^x, u^y) of the conserved-to-primitive system
// (u^eta = 0) with respect to theta = (T^{tau tau}, T^{tau x}, T^{tau y},
// pi^xx, pi^yy, pi^xy), by the implicit-function theorem: R(x, theta) = 0
// gives dx/dtheta = -J_x^{-1} J_theta, so thetabar = -J_theta^T lambda with
// J_x^T lambda = xbar.  J_x is the derivative of the residuals of
// NEWEST5/multiroot.h:202-243 at the root, with dP/de of the EOS interpolant
// (the Newton iteration uses the tabulated c_s^2 instead, which only changes
// its convergence, not the root); J_theta is read off the same residuals.
// Returns false when J_x is singular.
VH_HD inline bool c2p_ift_vjp(const DevCfg& C, const double* Tt, const double* p, double tau, const double* x3,
                              const double* xb3, double* Tb3, double* pb3) {
  const double t2 = C.cart ? 1.0 : tau * tau;
  (void)t2;  // u^eta = 0: the metric factor drops out of every 2+1D residual
  const double W = Tt[0], X = Tt[1], Y = Tt[2], p1 = p[0], p2 = p[1], p3 = p[2];
  const double e = x3[0], u1 = x3[1], u2 = x3[2];
  double P, dP, T, dT;
  eos_d<double>(C, e, P, dP, T, dT);
  const double S = 1 + u1 * u1 + u2 * u2, u0 = sqrt(S), iu = 1.0 / u0, ep = e + P;
  double J[3][3];
  J[0][0] = -u0;
  J[0][1] = (W - e) * u1 * iu - X;
  J[0][2] = (W - e) * u2 * iu - Y;
  J[1][0] = -(1 + dP) * u1 * S;
  J[1][1] = X * u1 * iu - p1 - ep * (1 + 3 * u1 * u1 + u2 * u2);
  J[1][2] = X * u2 * iu - p3 - 2 * ep * u1 * u2;
  J[2][0] = -(1 + dP) * u2 * S;
  J[2][1] = Y * u1 * iu - p3 - 2 * ep * u1 * u2;
  J[2][2] = Y * u2 * iu - p2 - ep * (1 + u1 * u1 + 3 * u2 * u2);
  // solve J^T lambda = xbar by Gaussian elimination with partial pivoting
  double A[3][3], b[3] = {xb3[0], xb3[1], xb3[2]};
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) A[r][c] = J[c][r];
  for (int c = 0; c < 3; c++) {
    int pv = c;
    for (int r = c + 1; r < 3; r++)
      if (fabs(A[r][c]) > fabs(A[pv][c])) pv = r;
    if (A[pv][c] == 0.0) return false;
    if (pv != c) {
      for (int k = 0; k < 3; k++) { const double t = A[c][k]; A[c][k] = A[pv][k]; A[pv][k] = t; }
      const double t = b[c]; b[c] = b[pv]; b[pv] = t;
    }
    for (int r = c + 1; r < 3; r++) {
      const double m = A[r][c] / A[c][c];
      for (int k = c; k < 3; k++) A[r][k] -= m * A[c][k];
      b[r] -= m * b[c];
    }
  }
  for (int c = 2; c >= 0; c--) {
    double s = b[c];
    for (int k = c + 1; k < 3; k++) s -= A[c][k] * b[k];
    b[c] = s / A[c][c];
  }
  const double l0 = b[0], l1 = b[1], l2 = b[2];
  Tb3[0] += -l0 * u0;
  Tb3[1] += l0 * u1 - l1 * u0;
  Tb3[2] += l0 * u2 - l2 * u0;
  pb3[0] += l1 * u1;
  pb3[1] += l2 * u2;
  pb3[2] += l1 * u2 + l2 * u1;
  return true;
}

// ------------------------------------------------------------- observable
// momentum anisotropy eps_p = sum(T^xx - T^yy) / sum(T^xx + T^yy) over the
// interior; per-cell T^xx - T^yy and T^xx + T^yy
template <class R>
VH_HD inline void obs_cell(const DevCfg& C, R e, R u1, R u2, R p1, R p2, double& num, double& den) {
  const R P = eos_P<R>(C, e), ep = e + P;
  const double txx = (double)(ep * u1 * u1 + P + p1), tyy = (double)(ep * u2 * u2 + P + p2);
  num = txx - tyy;
  den = txx + tyy;
}
// adjoint of eps_p = N/D at one cell: returns eb, u1b, u2b, p1b, p2b
template <class R>
VH_HD inline void obs_cell_vjp(const DevCfg& C, R e, R u1, R u2, double N, double D, R& eb, R& u1b, R& u2b, R& p1b,
                               R& p2b) {
  R P, dP, T, dT;
  eos_d<R>(C, e, P, dP, T, dT);
  const R ep = e + P;
  const R txxb = (R)(1.0 / D - N / (D * D)), tyyb = (R)(-1.0 / D - N / (D * D));
  eb = (txxb * u1 * u1 + tyyb * u2 * u2) * ((R)1 + dP) + (txxb + tyyb) * dP;
  u1b = txxb * (R)2 * ep * u1;
  u2b = tyyb * (R)2 * ep * u2;
  p1b = txxb;
  p2b = tyyb;
}

}  // namespace vh
