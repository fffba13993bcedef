// Host-side entry points onto the device arithmetic of the step and of its
// adjoint (the same __host__ __device__ functions the kernels use), for the
// CPU tests: finite-difference checks of every local adjoint.  Test hooks
// only: not part of the C ABI in include/vh.h, built as libvh_check.so.
#include <cmath>
#include <vector>

#include "vh.h"
#include "vh_adjoint.cuh"
#include "vh_adjoint3.cuh"
#include "vh_aux.cuh"
#include "vh_freezeout.cuh"

using namespace vh;

namespace {
struct HostCfg {
  DevCfg C{};
  std::vector<double> td;
  std::vector<float> tf;
};
HostCfg make_cfg(const vh_config* c) {
  HostCfg h;
  DevCfg& C = h.C;
  C.cart = c->coords == VH_COORD_CARTESIAN;
  C.bi = c->boost_invariant;
  C.recon = c->recon;
  C.eos_kind = c->eos_kind;
  C.eos_a = c->eos_a;
  C.etas0 = c->etas0; C.etas1 = c->etas1; C.etas_tc = c->etas_tc; C.hbarc = c->hbarc;
  C.taupi_kind = c->taupi_kind;
  C.taupi_c = c->taupi_const;
  C.cold = c->cold_plasma != 0;
  C.dx = c->dx; C.dy = c->dy; C.dz = c->dz;
  if (c->eos_kind == VH_EOS_TABLE) {
    const int n = c->eos_n;
    h.td.resize(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
      h.td[i] = c->eos_e[i]; h.td[n + i] = c->eos_p[i]; h.td[2 * n + i] = c->eos_cs2[i]; h.td[3 * n + i] = c->eos_t[i];
    }
    h.tf.assign(h.td.begin(), h.td.end());
    C.eos_n = n;
    C.eos_l0 = std::log(c->eos_e[0]);
    C.eos_idl = (n - 1) / (std::log(c->eos_e[n - 1]) - C.eos_l0);
    C.eos_d = h.td.data();
    C.eos_f = h.tf.data();
  }
  return h;
}
}  // namespace

extern "C" {

void vhc_weno_lr(const double* q, double* L, double* R) { weno_lr<double>(q[0], q[1], q[2], q[3], q[4], *L, *R); }
void vhc_weno_lr_vjp(const double* q, double Lb, double Rb, double* qb) { weno_lr_vjp<double>(q, Lb, Rb, qb); }

void vhc_cell_q(const vh_config* c, int dir, double tau, const double* x, int interior, double* q) {
  HostCfg h = make_cfg(c);
  if (dir == 0) cell_q<double, 0>(h.C, tau, x, interior, q);
  else cell_q<double, 1>(h.C, tau, x, interior, q);
}
void vhc_cell_q_vjp(const vh_config* c, int dir, double tau, const double* x, int interior, const double* qb,
                    double* xb) {
  HostCfg h = make_cfg(c);
  if (dir == 0) cell_q_vjp<double, 0>(h.C, tau, x, interior, qb, xb);
  else cell_q_vjp<double, 1>(h.C, tau, x, interior, qb, xb);
}
void vhc_src2d(const vh_config* c, double tau, double e, const double* u3, const double* p3, const double* du9,
               double* out4) {
  HostCfg h = make_cfg(c);
  src2d<double>(h.C, tau, e, u3, p3, du9, out4);
}
void vhc_src2d_vjp(const vh_config* c, double tau, double e, const double* u3, const double* p3, const double* du9,
                   const double* ob4, double* eb, double* ub3, double* pb3, double* dub9, double* cb2) {
  HostCfg h = make_cfg(c);
  src2d_vjp<double>(h.C, tau, e, u3, p3, du9, ob4, *eb, ub3, pb3, dub9, cb2);
}
int vhc_con2prim(const vh_config* c, const double* T3, const double* p3, double tau, double* x3) {
  HostCfg h = make_cfg(c);
  const double T[4] = {T3[0], T3[1], T3[2], 0.0}, p[5] = {p3[0], p3[1], p3[2], 0.0, 0.0};
  double x[4] = {x3[0], x3[1], x3[2], 0.0};
  const int it = con2prim(h.C, T, p, tau, x);
  x3[0] = x[0]; x3[1] = x[1]; x3[2] = x[2];
  return it;
}
int vhc_c2p_ift_vjp(const vh_config* c, const double* T3, const double* p3, double tau, const double* x3,
                    const double* xb3, double* Tb3, double* pb3) {
  HostCfg h = make_cfg(c);
  return c2p_ift_vjp(h.C, T3, p3, tau, x3, xb3, Tb3, pb3) ? 0 : 1;
}
void vhc_obs_cell(const vh_config* c, double e, double u1, double u2, double p1, double p2, double* nd) {
  HostCfg h = make_cfg(c);
  obs_cell<double>(h.C, e, u1, u2, p1, p2, nd[0], nd[1]);
}
void vhc_obs_cell_vjp(const vh_config* c, double e, double u1, double u2, double N, double D, double* g5) {
  HostCfg h = make_cfg(c);
  obs_cell_vjp<double>(h.C, e, u1, u2, N, D, g5[0], g5[1], g5[2], g5[3], g5[4]);
}
// 3+1D pieces: x[14] = (e, u^mu, pi 5, T^{tau mu}); du16[l*4 + m] = d_m u^l
void vhc_pi_dep(const double* u4, const double* p5, double t2, double* d5) {
  const PiDep<double> d = pi_dep<double>(u4[0], u4[1], u4[2], u4[3], p5, t2);
  d5[0] = d.tt; d5[1] = d.tx; d5[2] = d.ty; d5[3] = d.te; d5[4] = d.ee;
}
void vhc_pi_dep_vjp(const double* u4, const double* p5, double t2, const double* db5, double* ub4, double* pb5) {
  const PiDep<double> db{db5[0], db5[1], db5[2], db5[3], db5[4]};
  pi_dep_vjp<double>(u4[0], u4[1], u4[2], u4[3], p5, t2, db, ub4, pb5);
}
void vhc_cell_q3(const vh_config* c, int dir, double tau, const double* x, int interior, double* q) {
  HostCfg h = make_cfg(c);
  if (dir == 0) cell_q3<double, 0>(h.C, tau, x, interior, q);
  else if (dir == 1) cell_q3<double, 1>(h.C, tau, x, interior, q);
  else cell_q3<double, 2>(h.C, tau, x, interior, q);
}
void vhc_cell_q3_vjp(const vh_config* c, int dir, double tau, const double* x, int interior, const double* qb,
                     double* xb) {
  HostCfg h = make_cfg(c);
  if (dir == 0) cell_q3_vjp<double, 0>(h.C, tau, x, interior, qb, xb);
  else if (dir == 1) cell_q3_vjp<double, 1>(h.C, tau, x, interior, qb, xb);
  else cell_q3_vjp<double, 2>(h.C, tau, x, interior, qb, xb);
}
void vhc_src3(const vh_config* c, double tau, double e, const double* u4, const double* p5, const double* du16,
              double* out9) {
  HostCfg h = make_cfg(c);
  double du[4][4];
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) du[l][m] = du16[l * 4 + m];
  src3<double>(h.C, tau, e, u4, p5, du, out9);
}
void vhc_src3_vjp(const vh_config* c, double tau, double e, const double* u4, const double* p5, const double* du16,
                  const double* ob9, double* eb, double* ub4, double* pb5, double* dub16, double* cb2) {
  HostCfg h = make_cfg(c);
  double du[4][4], dub[4][4];
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) { du[l][m] = du16[l * 4 + m]; dub[l][m] = dub16[l * 4 + m]; }
  src3_vjp<double>(h.C, tau, e, u4, p5, du, ob9, *eb, ub4, pb5, dub, cb2);
  for (int l = 0; l < 4; l++)
    for (int m = 0; m < 4; m++) dub16[l * 4 + m] = dub[l][m];
}
int vhc_con2prim4(const vh_config* c, const double* T4, const double* p5, double tau, double* x4) {
  HostCfg h = make_cfg(c);
  return con2prim(h.C, T4, p5, tau, x4);
}
int vhc_c2p_ift_vjp4(const vh_config* c, const double* T4, const double* p5, double tau, const double* x4,
                     const double* xb4, double* Tb4, double* pb5) {
  HostCfg h = make_cfg(c);
  return c2p_ift_vjp4(h.C, T4, p5, tau, x4, xb4, Tb4, pb5) ? 0 : 1;
}
int vhc_landau(const double* T10, double tau, int cart, double* e, double* u4) {
  return landau_cell(T10, tau, cart != 0, *e, u4) ? 1 : 0;
}
void vhc_eos_d(const vh_config* c, double e, double* out4) {
  HostCfg h = make_cfg(c);
  eos_d<double>(h.C, e, out4[0], out4[1], out4[2], out4[3]);
}

// The algorithm of vh_freezeout_{2d,3d}_device run on the host with the same
// per-cube functions: every cube's count, their exclusive scan, then each
// cube's elements written from its offset, the cubes visited in the order
// perm (a permutation of the cube indices: the device's threads keep no
// order).  D = 3 (boost invariant) or 4.  Returns the element total, or -1
// when some cube emits other than its count of elements.
long long vhc_fo_emulate(int D, int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1,
                         const double* t0, const double* t1, const double* u0, const double* u1, double t_fo,
                         const long long* perm, double* out, long long cap) {
  const vh_fo::Geo g = vh_fo::make_geo(nx, ny, nz, dx, dy, dz, tau0, tau1, t_fo, D == 3);
  const long long nc = vh_fo::cubes(g, D);
  std::vector<long long> counts(nc), offs(nc);
  for (long long c = 0; c < nc; c++) {
    int i, j, k;
    vh_fo::cube_ijk(g, c, &i, &j, &k);
    counts[c] = D == 3 ? vh_fo::count<3>(g, i, j, k, t0, t1) : vh_fo::count<4>(g, i, j, k, t0, t1);
  }
  long long total = 0;
  for (long long c = 0; c < nc; c++) {
    offs[c] = total;
    total += counts[c];
  }
  for (long long q = 0; q < nc; q++) {
    const long long c = perm[q];
    if (counts[c] == 0) continue;
    int i, j, k;
    vh_fo::cube_ijk(g, c, &i, &j, &k);
    vh_fo::Sink s{out, offs[c], cap};
    if (D == 3) vh_fo::cube2(g, i, j, t0, t1, u0, u1, s);
    else vh_fo::cube3(g, i, j, k, t0, t1, u0, u1, s);
    if (s.at - offs[c] != counts[c]) return -1;
  }
  return total;
}
void vhc_bessel_k01e(double z, double* out2) { vh_fo::bessel_k01e(z, &out2[0], &out2[1]); }
double vhc_cf2_term(const double* el, double mt, double px, double py, double t_fo) {
  return vh_fo::cf2_term(el, mt, px, py, t_fo);
}
double vhc_cf3_term(const double* el, double mt, double px, double py, double y, double t_fo) {
  return vh_fo::cf3_term(el, mt, px, py, y, t_fo);
}
void vhc_kuhn_simplex(int s, int m, int* v) { vh_fo::kuhn_simplex(s, m, v); }
}
