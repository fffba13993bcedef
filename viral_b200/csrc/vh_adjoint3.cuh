// Reverse-mode (vector-Jacobian) building blocks of the discrete adjoint of
// the 3+1D Milne step: every evolved field, the eta direction and its
// Christoffel terms.  As in the boost-invariant pieces (vh_adjoint.cuh), each
// function recomputes the forward values it needs from the same inputs as the
// forward kernels (so branch choices are the forward pass's) and propagates
// adjoints by hand; host+device, so that each piece is checked against finite
// differences on the CPU.
//
// Per-cell variables (14): x = (e, u^tau, u^x, u^y, u^eta, pi^xx, pi^yy,
// pi^xy, pi^{x eta}, pi^{y eta}, T^{tau tau}, T^{tau x}, T^{tau y},
// T^{tau eta}).  Flux quantities of one direction (19): F^0..F^3 (tau T^{d mu}),
// F^4..F^8 (the five pi components times v^d, tau v^eta along eta), V^0..V^3
// (tau T^{tau mu}), V^4..V^8 (pi) and the signal speed.
#pragma once

#include "vh_adjoint.cuh"

namespace vh {

constexpr int NX3 = 14;   // per-cell variables
constexpr int NQ3 = 19;   // flux quantities per direction
enum : int { X3E = 0, X3U = 1, X3P = 5, X3T = 10 };

// ------------------------------------------------------------- pi closure
// adjoint of pi_dep (the dependent components tt, tx, ty, te, ee of pi from
// the five evolved ones): db -> ub[4], pb[5], accumulated
template <class R>
VH_HD inline void pi_dep_vjp(R u0, R u1, R u2, R u3, const R* p, R t2, const PiDep<R>& db, R* ub, R* pb) {
  const PiDep<R> d = pi_dep<R>(u0, u1, u2, u3, p, t2);
  const R iu0 = (R)1 / u0;
  const R Dn = u0 * u0 - t2 * u3 * u3, iD = (R)1 / Dn;
  const R s = p[0] + p[1];
  R eeb = db.ee;
  // te = (u1 p3 + u2 p4 + t2 u3 ee) / u0
  eeb += db.te * t2 * u3 * iu0;
  ub[1] += db.te * p[3] * iu0;
  pb[3] += db.te * u1 * iu0;
  ub[2] += db.te * p[4] * iu0;
  pb[4] += db.te * u2 * iu0;
  ub[3] += db.te * t2 * d.ee * iu0;
  ub[0] -= db.te * d.te * iu0;
  // tx = (p0 u1 + p2 u2 + p3 u3 t2) / u0
  pb[0] += db.tx * u1 * iu0; ub[1] += db.tx * p[0] * iu0;
  pb[2] += db.tx * u2 * iu0; ub[2] += db.tx * p[2] * iu0;
  pb[3] += db.tx * u3 * t2 * iu0; ub[3] += db.tx * p[3] * t2 * iu0;
  ub[0] -= db.tx * d.tx * iu0;
  // ty = (p2 u1 + p1 u2 + p4 u3 t2) / u0
  pb[2] += db.ty * u1 * iu0; ub[1] += db.ty * p[2] * iu0;
  pb[1] += db.ty * u2 * iu0; ub[2] += db.ty * p[1] * iu0;
  pb[4] += db.ty * u3 * t2 * iu0; ub[3] += db.ty * p[4] * t2 * iu0;
  ub[0] -= db.ty * d.ty * iu0;
  // ee = (Q - u0^2 s) / (t2 Dn);  tt = (Q - t2 u3^2 s) / Dn
  const R it2 = (R)1 / t2;
  R Qb = eeb * it2 * iD + db.tt * iD;
  R sb = -eeb * u0 * u0 * it2 * iD - db.tt * t2 * u3 * u3 * iD;
  R Dnb = -eeb * d.ee * iD - db.tt * d.tt * iD;
  ub[0] += -eeb * (R)2 * u0 * s * it2 * iD + Dnb * (R)2 * u0;
  ub[3] += -db.tt * (R)2 * t2 * u3 * s * iD - Dnb * (R)2 * t2 * u3;
  pb[0] += sb;
  pb[1] += sb;
  // Q = u1^2 p0 + 2 u1 u2 p2 + u2^2 p1 + 2 t2 u3 (u1 p3 + u2 p4)
  pb[0] += Qb * u1 * u1;
  pb[1] += Qb * u2 * u2;
  pb[2] += Qb * (R)2 * u1 * u2;
  pb[3] += Qb * (R)2 * t2 * u3 * u1;
  pb[4] += Qb * (R)2 * t2 * u3 * u2;
  ub[1] += Qb * ((R)2 * u1 * p[0] + (R)2 * u2 * p[2] + (R)2 * t2 * u3 * p[3]);
  ub[2] += Qb * ((R)2 * u2 * p[1] + (R)2 * u1 * p[2] + (R)2 * t2 * u3 * p[4]);
  ub[3] += Qb * (R)2 * t2 * (u1 * p[3] + u2 * p[4]);
}

// the full pi^{mu nu} from the five evolved components and the closure
template <class R>
VH_HD inline void pi_full(const PiDep<R>& d, const R* p, R pi[4][4]) {
  pi[0][0] = d.tt; pi[0][1] = d.tx; pi[0][2] = d.ty; pi[0][3] = d.te;
  pi[1][0] = d.tx; pi[1][1] = p[0]; pi[1][2] = p[2]; pi[1][3] = p[3];
  pi[2][0] = d.ty; pi[2][1] = p[2]; pi[2][2] = p[1]; pi[2][3] = p[4];
  pi[3][0] = d.te; pi[3][1] = p[3]; pi[3][2] = p[4]; pi[3][3] = d.ee;
}
// the adjoint of a full pi^{mu nu} onto the evolved five (pb) and the
// dependent components (db), accumulated
template <class R>
VH_HD inline void pi_full_bar(const R pib[4][4], R* pb, PiDep<R>& db) {
  db.tt += pib[0][0];
  db.tx += pib[0][1] + pib[1][0];
  db.ty += pib[0][2] + pib[2][0];
  db.te += pib[0][3] + pib[3][0];
  db.ee += pib[3][3];
  pb[0] += pib[1][1];
  pb[1] += pib[2][2];
  pb[2] += pib[1][2] + pib[2][1];
  pb[3] += pib[1][3] + pib[3][1];
  pb[4] += pib[2][3] + pib[3][2];
}

// ---------------------------------------------------------- flux quantities
// The flux quantities of one cell along DIR, as k_dir's cell_terms forms them
// (NEWEST5/hydroKT.h:16-83, 161-245): with a = DIR + 1,
//   F^mu = tau (pi^{a mu} + P g^{a mu}-part + u^a u^mu (e + P)), mu = 0..3
//   F^{4+l} = f_a pi_l u^a / u^tau,  speed = f_a u^a / u^tau (interior only)
// where f_a = tau along eta (1 otherwise) and the pressure enters F^a with
// |g^{aa}| (1, or 1/tau^2 along eta).
template <class R, int DIR>
VH_HD inline void cell_q3(const DevCfg& C, R tau, const R* x, bool interior, R* q) {
  constexpr int a = DIR + 1;
  const R e = x[0], u[4] = {x[1], x[2], x[3], x[4]};
  const R* p = x + X3P;
  const R t2 = tau * tau;
  const R P = eos_P<R>(C, e), ep = e + P, iu0 = (R)1 / u[0];
  const PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  R pi[4][4];
  pi_full<R>(d, p, pi);
  const R ga = a == 3 ? (R)1 / t2 : (R)1, fa = a == 3 ? tau : (R)1;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) q[mu] = tau * (pi[a][mu] + (mu == a ? P * ga : (R)0) + u[a] * u[mu] * ep);
#pragma unroll
  for (int l = 0; l < 5; l++) q[4 + l] = fa * p[l] * u[a] * iu0;
#pragma unroll
  for (int l = 0; l < 4; l++) q[9 + l] = tau * x[X3T + l];
#pragma unroll
  for (int l = 0; l < 5; l++) q[13 + l] = p[l];
  q[18] = interior ? fa * u[a] * iu0 : (R)0;
}

// xb += (d q / d x)^T qb
template <class R, int DIR>
VH_HD inline void cell_q3_vjp(const DevCfg& C, R tau, const R* x, bool interior, const R* qb, R* xb) {
  constexpr int a = DIR + 1;
  const R e = x[0], u[4] = {x[1], x[2], x[3], x[4]};
  const R* p = x + X3P;
  const R t2 = tau * tau;
  R P, dP, T, dT;
  eos_d<R>(C, e, P, dP, T, dT);
  const R ep = e + P, iu0 = (R)1 / u[0];
  const R ga = a == 3 ? (R)1 / t2 : (R)1, fa = a == 3 ? tau : (R)1;
  R ub[4] = {0, 0, 0, 0}, pb[5] = {0, 0, 0, 0, 0}, pib[4][4] = {}, Pb = 0, epb = 0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const R fb = tau * qb[mu];
    pib[a][mu] += fb;
    if (mu == a) Pb += fb * ga;
    ub[a] += fb * u[mu] * ep;
    ub[mu] += fb * u[a] * ep;
    epb += fb * u[a] * u[mu];
  }
#pragma unroll
  for (int l = 0; l < 5; l++) {
    const R g = qb[4 + l] * fa;
    pb[l] += g * u[a] * iu0;
    ub[a] += g * p[l] * iu0;
    ub[0] -= g * p[l] * u[a] * iu0 * iu0;
  }
  if (interior) {
    ub[a] += qb[18] * fa * iu0;
    ub[0] -= qb[18] * fa * u[a] * iu0 * iu0;
  }
#pragma unroll
  for (int l = 0; l < 4; l++) xb[X3T + l] += tau * qb[9 + l];
#pragma unroll
  for (int l = 0; l < 5; l++) pb[l] += qb[13 + l];
  PiDep<R> db{0, 0, 0, 0, 0};
  pi_full_bar<R>(pib, pb, db);
  pi_dep_vjp<R>(u[0], u[1], u[2], u[3], p, t2, db, ub, pb);
  Pb += epb;
  xb[0] += epb + Pb * dP;
#pragma unroll
  for (int l = 0; l < 4; l++) xb[X3U + l] += ub[l];
#pragma unroll
  for (int l = 0; l < 5; l++) xb[X3P + l] += pb[l];
}

// ---------------------------------------------------------------- source
// The Milne sources of one cell as k_update forms them (NEWEST5/Source.h:
// 165-191 geometric, 311-433 shear): out[0] (tau T^{tau tau}) =
// -P - tau^2 (pi^{eta eta} + (e+P) u^eta u^eta), out[3] (tau T^{tau eta}) =
// -2 (pi^{tau eta} + (e+P) u^tau u^eta), out[4..8] the shear source of the
// five evolved pi components; out[1], out[2] are zero.  du[l][m] = d_m u^l.
template <class R>
VH_HD inline void src3(const DevCfg& C, R tau, R e, const R* u, const R* p, const R du[4][4], R* out) {
  R P, cs2, T;
  eos_all<R>(C, e, P, cs2, T);
  const R t2 = tau * tau;
  const PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  const R ep = e + P;
  out[0] = -P - t2 * (d.ee + ep * u[3] * u[3]);
  out[1] = 0;
  out[2] = 0;
  out[3] = -(R)2 * (d.te + ep * u[0] * u[3]);
  is_source_PT<R>(C, tau, e, P, T, u, p, du, out + 4);
}

// Adjoint of src3, accumulated: ob[9] -> eb, ub[4], pb[5], dub[4][4], cb[2]
// (the eta/s(T) parameters c0, c1).  Milne, not the cold-plasma limit.
template <class R>
VH_HD inline void src3_vjp(const DevCfg& C, R tau, R e, const R* u, const R* p, const R du[4][4], const R* ob,
                           R& eb, R* ub, R* pb, R dub[4][4], R* cb) {
  const R t2 = tau * tau, itau = (R)1 / tau;
  const R g[4] = {(R)1, (R)-1, (R)-1, -t2};
  const R gi[4] = {(R)1, (R)-1, (R)-1, (R)-1 / t2};
  // ---- forward recompute
  R P, dP, T, dT;
  eos_d<R>(C, e, P, dP, T, dT);
  const R ep = e + P;
  const R iT = (R)1 / T, iep = (R)1 / ep, iP = (R)1 / P;
  const R s = ep * iT;
  const R tg = T * (R)C.hbarc - (R)C.etas_tc;
  const bool kink = tg > (R)0;
  const R etas = (R)C.etas0 + (R)C.etas1 * (kink ? tg : (R)0);
  const R eta = etas * s;
  const R tp = C.taupi_kind == 1 ? (R)5 * eta * iep : C.taupi_kind == 2 ? (R)C.taupi_c : (R)1.5 * (eta * iP);
  const R itp = (R)1 / tp;
  const R iu0 = (R)1 / u[0], iD = iu0 * iu0;
  const PiDep<R> d = pi_dep<R>(u[0], u[1], u[2], u[3], p, t2);
  R pi[4][4];
  pi_full<R>(d, p, pi);
  R Dm[4][4];
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) Dm[l][m] = du[l][m];
  Dm[0][3] += tau * u[3];
  Dm[3][0] += u[3] * itau;
  Dm[3][3] += u[0] * itau;
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
  R S[4][4], M[4][4] = {}, sig[4][4] = {};
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) S[a][b] = (R)0.5 * (Dl[a][b] + Dl[b][a]);
  for (int m = 1; m < 3; m++)
    for (int b = 0; b < 4; b++) {
      R acc = 0;
      for (int a = 0; a < 4; a++) acc += Dt[m][a] * S[a][b];
      M[m][b] = acc;
    }
  for (int m = 1; m < 3; m++)
    for (int v = 1; v < 4; v++) {
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
  for (int i = 1; i < 4; i++) divv += du[i][i] * iu0 - u[i] * du[0][i] * iD;

  // ---- reverse
  R ubl[4] = {0, 0, 0, 0}, Pb = 0, epb = 0, etab = 0, tpb = 0, thb = 0, divvb = 0;
  R pib[4][4] = {}, sigb[4][4] = {}, pab[4] = {}, accb[4] = {}, Dmb[4][4] = {};
  // geometric sources
  Pb -= ob[0];
  pib[3][3] -= t2 * ob[0];
  epb -= t2 * u[3] * u[3] * ob[0];
  ubl[3] -= (R)2 * t2 * ep * u[3] * ob[0];
  pib[0][3] -= (R)2 * ob[3];
  epb -= (R)2 * u[0] * u[3] * ob[3];
  ubl[0] -= (R)2 * ep * u[3] * ob[3];
  ubl[3] -= (R)2 * ep * u[0] * ob[3];
  // shear source of (xx, yy, xy, x eta, y eta)
  const int MU[5] = {1, 2, 1, 1, 2}, NU[5] = {1, 2, 2, 3, 3};
  for (int q = 0; q < 5; q++) {
    const R o = ob[4 + q];
    if (o == (R)0) continue;
    const int m = MU[q], v = NU[q];
    const R rhs = -(pi[m][v] - (R)2 * eta * sig[m][v]) * itp - ((R)4 / (R)3) * pi[m][v] * th -
                  (u[m] * pa[v] + u[v] * pa[m]);
    const R chr = v == 3 ? (u[0] * pi[3][m] + u[3] * pi[0][m]) * itau : (R)0;
    const R rb = o * iu0;
    ubl[0] -= o * (rhs - chr) * iD;
    pib[m][v] += o * divv;
    divvb += o * pi[m][v];
    pib[m][v] += -rb * itp - ((R)4 / (R)3) * th * rb;
    sigb[m][v] += (R)2 * eta * rb * itp;
    etab += (R)2 * sig[m][v] * rb * itp;
    tpb += (pi[m][v] - (R)2 * eta * sig[m][v]) * rb * (itp * itp);
    thb += -((R)4 / (R)3) * pi[m][v] * rb;
    ubl[m] -= pa[v] * rb; pab[v] -= u[m] * rb;
    ubl[v] -= pa[m] * rb; pab[m] -= u[v] * rb;
    if (v == 3) {
      ubl[0] -= rb * pi[3][m] * itau;
      pib[3][m] -= rb * u[0] * itau;
      ubl[3] -= rb * pi[0][m] * itau;
      pib[0][m] -= rb * u[3] * itau;
    }
  }
  // divv = sum_i du[i][i] / u0 - u_i du[0][i] / u0^2
  for (int i = 1; i < 4; i++) {
    dub[i][i] += divvb * iu0;
    ubl[0] += divvb * (-du[i][i] * iD + (R)2 * u[i] * du[0][i] * iD * iu0);
    ubl[i] -= divvb * du[0][i] * iD;
    dub[0][i] -= divvb * u[i] * iD;
  }
  // pa[v] = sum_b pi[v][b] acc[b]
  for (int v = 0; v < 4; v++)
    for (int b = 0; b < 4; b++) { pib[v][b] += pab[v] * acc4[b]; accb[b] += pab[v] * pi[v][b]; }
  // acc[v] = g[v] sum_b u[b] Dm[v][b]
  for (int v = 0; v < 4; v++)
    for (int b = 0; b < 4; b++) { ubl[b] += accb[v] * g[v] * Dm[v][b]; Dmb[v][b] += accb[v] * g[v] * u[b]; }
  // sig[m][v] = sum_b M[m][b] Dt[v][b] - Dt[m][v] tr3
  R Mb[4][4] = {}, Dtb[4][4] = {}, Sb[4][4] = {}, Dlb[4][4] = {};
  R tr3b = 0;
  for (int m = 1; m < 3; m++)
    for (int v = 1; v < 4; v++) {
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
  // S = (Dl + Dl^T) / 2
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { Dlb[a][b] += (R)0.5 * Sb[a][b]; Dlb[b][a] += (R)0.5 * Sb[a][b]; }
  // tr = sum Dt Dl
  const R trb = tr3b / (R)3;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { Dtb[a][b] += trb * Dl[a][b]; Dlb[a][b] += trb * Dt[a][b]; }
  // Dt[a][b] = gi delta - u_a u_b
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) { ubl[a] -= Dtb[a][b] * u[b]; ubl[b] -= Dtb[a][b] * u[a]; }
  // theta = trace Dm
  for (int l = 0; l < 4; l++) Dmb[l][l] += thb;
  // Dl[a][b] = g[b] Dm[b][a]
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) Dmb[b][a] += Dlb[a][b] * g[b];
  // Christoffel terms of Dm
  ubl[3] += Dmb[0][3] * tau + Dmb[3][0] * itau;
  ubl[0] += Dmb[3][3] * itau;
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) dub[l][m] += Dmb[l][m];
  // pi^{mu nu} -> the evolved five and the closure
  R pbl[5] = {0, 0, 0, 0, 0};
  PiDep<R> db{0, 0, 0, 0, 0};
  pi_full_bar<R>(pib, pbl, db);
  pi_dep_vjp<R>(u[0], u[1], u[2], u[3], p, t2, db, ubl, pbl);
  // transport: eta = etas s, s = (e+P)/T, etas = c0 + c1 max(T hbarc - tc, 0), tau_pi
  R eb_ = 0, Tb = 0;
  if (C.taupi_kind == 1) {
    etab += tpb * (R)5 * iep;
    epb -= tpb * (R)5 * eta * (iep * iep);
  } else if (C.taupi_kind == 0) {
    etab += tpb * (R)1.5 * iP;
    Pb -= tpb * (R)1.5 * eta * (iP * iP);
  }
  const R etasb = etab * s, sb = etab * etas;
  cb[0] += etasb;
  cb[1] += etasb * (kink ? tg : (R)0);
  if (kink) Tb += etasb * (R)C.etas1 * (R)C.hbarc;
  epb += sb * iT;
  Tb -= sb * s * iT;
  eb_ += epb;
  Pb += epb;
  eb_ += Pb * dP + Tb * dT;
  eb += eb_;
  for (int l = 0; l < 4; l++) ub[l] += ubl[l];
  for (int l = 0; l < 5; l++) pb[l] += pbl[l];
}

// ------------------------------------------------------------- con2prim
// Adjoint of the root x = (e, u^x, u^y, u^eta) of the conserved-to-primitive
// system with respect to theta = (T^{tau mu}, pi^xx, pi^yy, pi^xy,
// pi^{x eta}, pi^{y eta}), by the implicit-function theorem:
// thetabar = -J_theta^T lambda with J_x^T lambda = xbar.  J_x is c2p_fj's
// Jacobian (NEWEST5/multiroot.h:202-319) at the root with dP/de of the EOS
// interpolant in place of the tabulated c_s^2; J_theta is read off the same
// residuals.  Returns false when J_x is singular.
VH_HD inline bool c2p_ift_vjp4(const DevCfg& C, const double* Tt, const double* p, double tau, const double* x4,
                               const double* xb4, double* Tb4, double* pb5) {
  const double t2 = tau * tau;
  const double W = Tt[0], X = Tt[1], Y = Tt[2], Z = Tt[3];
  const double p1 = p[0], p2 = p[1], p3 = p[2], p4 = p[3], p5 = p[4];
  const double e = x4[0], u1 = x4[1], u2 = x4[2], u3 = x4[3];
  double P, dP, T, dT;
  eos_d<double>(C, e, P, dP, T, dT);
  const double S = 1 + u1 * u1 + u2 * u2 + t2 * u3 * u3, u0 = sqrt(S), iu = 1.0 / u0, ep = e + P;
  double A[4][4], b[4] = {xb4[0], xb4[1], xb4[2], xb4[3]};
  double J[4][4];
  J[0][0] = -u0;
  J[0][1] = (W - e) * u1 * iu - X;
  J[0][2] = (W - e) * u2 * iu - Y;
  J[0][3] = t2 * ((W - e) * u3 * iu - Z);
  J[1][0] = -(1 + dP) * u1 * S;
  J[1][1] = X * u1 * iu - p1 - ep * (1 + 3 * u1 * u1 + u2 * u2 + t2 * u3 * u3);
  J[1][2] = X * u2 * iu - p3 - 2 * ep * u1 * u2;
  J[1][3] = t2 * (X * u3 * iu - p4 - 2 * ep * u1 * u3);
  J[2][0] = -(1 + dP) * u2 * S;
  J[2][1] = Y * u1 * iu - p3 - 2 * ep * u1 * u2;
  J[2][2] = Y * u2 * iu - p2 - ep * (1 + u1 * u1 + 3 * u2 * u2 + t2 * u3 * u3);
  J[2][3] = t2 * (Y * u3 * iu - p5 - 2 * ep * u2 * u3);
  J[3][0] = -dP * u3;
  J[3][1] = Z * u1 * iu - p4;
  J[3][2] = Z * u2 * iu - p5;
  J[3][3] = t2 * Z * u3 * iu - (P + W - p1 - p2);
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) A[r][c] = J[c][r];
  if (!solve4(A, b)) return false;
  const double l0 = b[0], l1 = b[1], l2 = b[2], l3 = b[3];
  Tb4[0] += -l0 * u0 + l3 * u3;
  Tb4[1] += l0 * u1 - l1 * u0;
  Tb4[2] += l0 * u2 - l2 * u0;
  Tb4[3] += l0 * t2 * u3 - l3 * u0;
  pb5[0] += l1 * u1 - l3 * u3;
  pb5[1] += l2 * u2 - l3 * u3;
  pb5[2] += l1 * u2 + l2 * u1;
  pb5[3] += l1 * t2 * u3 + l3 * u1;
  pb5[4] += l2 * t2 * u3 + l3 * u2;
  return true;
}

}  // namespace vh
