// Snapshot writer in the reference's binary layout (NEWEST5/write.h).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vh.h"
#include "vh_internal.h"

namespace {

// host evaluation of T(e), the same formulas as the device EOS
struct HostEos {
  int kind = 0;
  double a = 1;
  std::vector<double> e, p, c, t;
  double T(double x) const {
    if (kind == VH_EOS_CONFORMAL) return std::pow(x / a, 0.25);
    const int n = (int)e.size();
    if (x <= e[0]) return t[0] * std::sqrt(std::sqrt(x / e[0]));
    if (x >= e[n - 1]) return t[n - 1] * std::sqrt(std::sqrt(x / e[n - 1]));
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) { int m = (lo + hi) / 2; if (x >= e[m]) lo = m; else hi = m; }
    const double w = (x - e[lo]) / (e[lo + 1] - e[lo]);
    return t[lo] + w * (t[lo + 1] - t[lo]);
  }
  double P(double x) const {
    if (kind == VH_EOS_CONFORMAL) return x / 3.0;
    const int n = (int)e.size();
    if (x <= e[0]) return c[0] * x;
    if (x >= e[n - 1]) return p[n - 1] + c[n - 1] * (x - e[n - 1]);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) { int m = (lo + hi) / 2; if (x >= e[m]) lo = m; else hi = m; }
    const double w = (x - e[lo]) / (e[lo + 1] - e[lo]);
    return p[lo] + w * (p[lo + 1] - p[lo]);
  }
};

}  // namespace

extern "C" int vh_write(vh_handle* h, const char* path, int layout, int every) {
  if (!h || !path || every < 1 || layout < VH_WRITE_XY || layout > VH_WRITE_NS_XY) return VH_E_ARG;
  const bool v17 = layout == VH_WRITE_XY17 || layout == VH_WRITE_FULL17;
  const bool nsw = layout == VH_WRITE_NS_XY;
  const int NV = nsw ? 11 : (v17 ? 17 : 12);
  if (v17) layout = layout == VH_WRITE_XY17 ? VH_WRITE_XY : VH_WRITE_FULL;
  if (nsw) layout = VH_WRITE_XY;
  vh_config cfg;
  std::vector<double> tab;
  int r = vh_internal_config(h, &cfg, &tab);
  if (r) return r;
  int gx, gy, gz;
  vh_dims(h, &gx, &gy, &gz);
  const long long n = (long long)gx * gy * gz;
  std::vector<double> f(18 * (size_t)n);
  if ((r = vh_get_state(h, f.data()))) return r;
  // the 17-variable records take the full pi^{mu nu} from the device (the
  // closure of the five stored components); T and P, as in every record,
  // come from the EOS at e on the host, as the reference's FT and EOS give
  // them (NEWEST5/multiroot.h:428-429)
  std::vector<double> pi10;
  if (v17) {
    pi10.resize(10 * (size_t)n);
    if ((r = vh_get_primitive(h, nullptr, nullptr, nullptr, nullptr, pi10.data()))) return r;
  }
  // NEWEST10/write.h:123-170 (WriteNSXY): the ten Navier-Stokes pi^{mu nu}
  // and the (zero) bulk part per cell
  std::vector<double> nspi;
  if (nsw) {
    nspi.resize(10 * (size_t)n);
    if ((r = vh_get_ns_pi(h, nspi.data()))) return r;
  }
  HostEos eos;
  eos.kind = cfg.eos_kind;
  eos.a = cfg.eos_a;
  if (eos.kind == VH_EOS_TABLE) {
    const size_t m = tab.size() / 4;
    eos.e.assign(tab.begin(), tab.begin() + m);
    eos.p.assign(tab.begin() + m, tab.begin() + 2 * m);
    eos.c.assign(tab.begin() + 2 * m, tab.begin() + 3 * m);
    eos.t.assign(tab.begin() + 3 * m, tab.end());
  }
  const int nx = cfg.nx, ny = cfg.ny, bi = cfg.boost_invariant;
  const int nzi = bi ? 1 : cfg.nz, kl = bi ? 0 : 3;
  auto rec = [&](int i, int j, int k, double* o) {
    const long long c = ((long long)k * gy + j) * gx + i;
    if (nsw) {
      for (int l = 0; l < 10; l++) o[l] = nspi[(size_t)l * n + c];
      o[10] = 0.0;  // no bulk viscosity
      return;
    }
    const double e = f[c], u0 = f[n + c];
    o[0] = e;
    o[1] = eos.T(e);
    o[2] = eos.P(e);
    o[3] = f[2 * n + c] / u0;
    o[4] = f[3 * n + c] / u0;
    o[5] = f[4 * n + c] / u0;
    if (v17) {
      for (int l = 0; l < 10; l++) o[6 + l] = pi10[(size_t)l * n + c];
      o[16] = 0.0;  // bulk pressure is not evolved
      return;
    }
    for (int l = 0; l < 5; l++) o[6 + l] = f[(5 + l) * n + c];
    o[11] = 0.0;  // bulk pressure is not evolved
  };
  const size_t R = NV * sizeof(double);
  std::vector<unsigned char> file;
  auto put = [&](size_t off, const double* src, size_t ndouble) {
    const size_t bytes = ndouble * sizeof(double);
    if (file.size() < off + bytes) file.resize(off + bytes, 0);
    std::memcpy(file.data() + off, src, bytes);
  };
  if (layout == VH_WRITE_XY) {
    // NEWEST5/write.h:51-115: per x row a chunk of (12*ny)/FREQ doubles at
    // offset (gi/FREQ * (ny/FREQ)) records, central eta slice k0
    const int k0 = bi ? 0 : (gz - 1) / 2;
    const int ypts = ny / every;
    const size_t chunk = (size_t)(NV * ny) / every;
    std::vector<double> buf(NV * (size_t)(ny / every + 2), 0.0);
    for (int i = 3; i < 3 + nx; i += every) {
      const int gi = i - 3;
      for (int j = 3, jj = 0; j < 3 + ny; j += every, jj++) rec(i, j, k0, &buf[NV * (size_t)jj]);
      put((size_t)(gi / every) * ypts * R, buf.data(), chunk);
    }
  } else {
    // NEWEST5/write.h:204-290: per (x,y) column the eta records, at offset
    // (gi/FREQ * ypts * zpts + gj/FREQ * zpts) records
    const int ypts = ny / every, zpts = nzi;
    std::vector<double> buf(NV * (size_t)nzi);
    for (int i = 3; i < 3 + nx; i += every)
      for (int j = 3; j < 3 + ny; j += every) {
        for (int k = kl, kk = 0; k < kl + nzi; k++, kk++) rec(i, j, k, &buf[NV * (size_t)kk]);
        put(((size_t)((i - 3) / every) * ypts * zpts + (size_t)((j - 3) / every) * zpts) * R, buf.data(), buf.size());
      }
  }
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return VH_E_ARG;
  const size_t w = std::fwrite(file.data(), 1, file.size(), fp);
  const bool closed = std::fclose(fp) == 0;  // a delayed write error shows here
  return w == file.size() && closed ? VH_OK : VH_E_ARG;
}

// NEWideal/init.h:296-345: interior values read row by row (x fastest),
// v -> u, and the floor applied over the whole grid.
extern "C" int vh_read_ideal_profile(const char* eps_path, const char* vx_path, const char* vy_path, int nx, int ny,
                                     double* e, double* ux, double* uy, double* min_out) {
  if (!eps_path || !vx_path || !vy_path || !e || !ux || !uy || nx < 1 || ny < 1) return VH_E_ARG;
  FILE* fe = std::fopen(eps_path, "r");
  FILE* fx = std::fopen(vx_path, "r");
  FILE* fy = std::fopen(vy_path, "r");
  auto close_all = [&]() {
    if (fe) std::fclose(fe);
    if (fx) std::fclose(fx);
    if (fy) std::fclose(fy);
  };
  if (!fe || !fx || !fy) { close_all(); return VH_E_ARG; }
  const int gx = nx + 6, gy = ny + 6;
  const size_t n = (size_t)gx * gy;
  std::vector<double> vx(n, 0.0), vy(n, 0.0);
  for (size_t c = 0; c < n; c++) e[c] = 0.0;
  double mn = 100;
  for (int j = 3; j < 3 + ny; j++)
    for (int i = 3; i < 3 + nx; i++) {
      const size_t c = (size_t)j * gx + i;
      if (std::fscanf(fe, "%lf", &e[c]) != 1 || std::fscanf(fx, "%lf", &vx[c]) != 1 ||
          std::fscanf(fy, "%lf", &vy[c]) != 1) {
        close_all();
        return VH_E_ARG;
      }
      if (e[c] < mn && std::fabs(e[c]) > 1e-5) mn = e[c];
    }
  close_all();
  for (size_t c = 0; c < n; c++) {
    if (e[c] < 0.01) e[c] = mn / 10;
    const double g = 1.0 / std::sqrt(1.0 - vx[c] * vx[c] - vy[c] * vy[c]);
    ux[c] = g * vx[c];
    uy[c] = g * vy[c];
  }
  if (min_out) *min_out = mn;
  return VH_OK;
}

// Restart files: an 8-byte tag, the grid (coords, precision, nx, ny, nz,
// boost invariance as int32), dx, dy, dz, dtau and tau as doubles, then the
// 18 canonical fields over the ghost-inclusive grid.  The reference keeps no
// restart state; these hold everything a step reads (prevu included), so a
// run resumed from one continues bit for bit.
namespace {
const char kCkptTag[8] = {'V', 'H', 'C', 'K', 'P', 'T', '0', '1'};
struct CkptHead {
  char tag[8];
  int32_t coords, precision, nx, ny, nz, boost_invariant;
  double dx, dy, dz, dtau, tau;
};
}  // namespace

extern "C" int vh_save_checkpoint(vh_handle* h, const char* path) {
  if (!h || !path) return VH_E_ARG;
  vh_config cfg;
  int r = vh_internal_config(h, &cfg, nullptr);
  if (r) return r;
  int gx, gy, gz;
  vh_dims(h, &gx, &gy, &gz);
  const size_t n = (size_t)gx * gy * gz;
  std::vector<double> f(18 * n);
  if ((r = vh_get_state(h, f.data()))) return r;
  CkptHead hd{};
  std::memcpy(hd.tag, kCkptTag, 8);
  hd.coords = cfg.coords;
  hd.precision = cfg.precision;
  hd.nx = cfg.nx;
  hd.ny = cfg.ny;
  hd.nz = cfg.nz;
  hd.boost_invariant = cfg.boost_invariant;
  hd.dx = cfg.dx;
  hd.dy = cfg.dy;
  hd.dz = cfg.dz;
  hd.dtau = cfg.dtau;
  vh_get_time(h, &hd.tau);
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return vh_internal_error(h, VH_E_ARG, "vh_save_checkpoint: cannot open the file for writing");
  const bool ok = std::fwrite(&hd, sizeof(hd), 1, fp) == 1 && std::fwrite(f.data(), sizeof(double), f.size(), fp) == f.size();
  const bool closed = std::fclose(fp) == 0;
  return ok && closed ? VH_OK : vh_internal_error(h, VH_E_ARG, "vh_save_checkpoint: short write");
}

extern "C" int vh_load_checkpoint(vh_handle* h, const char* path, double* tau_out) {
  if (!h || !path) return VH_E_ARG;
  vh_config cfg;
  int r = vh_internal_config(h, &cfg, nullptr);
  if (r) return r;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return vh_internal_error(h, VH_E_ARG, "vh_load_checkpoint: cannot open the file");
  CkptHead hd{};
  if (std::fread(&hd, sizeof(hd), 1, fp) != 1 || std::memcmp(hd.tag, kCkptTag, 8) != 0) {
    std::fclose(fp);
    return vh_internal_error(h, VH_E_ARG, "vh_load_checkpoint: not a restart file");
  }
  const bool same_grid = hd.coords == cfg.coords && hd.nx == cfg.nx && hd.ny == cfg.ny && hd.nz == cfg.nz &&
                         hd.boost_invariant == cfg.boost_invariant && hd.dx == cfg.dx && hd.dy == cfg.dy &&
                         hd.dz == cfg.dz;
  if (!same_grid) {
    std::fclose(fp);
    return vh_internal_error(h, VH_E_ARG, "vh_load_checkpoint: the file's grid differs from the handle's");
  }
  int gx, gy, gz;
  vh_dims(h, &gx, &gy, &gz);
  const size_t n = (size_t)gx * gy * gz;
  std::vector<double> f(18 * n);
  const bool ok = std::fread(f.data(), sizeof(double), f.size(), fp) == f.size();
  std::fclose(fp);
  if (!ok) return vh_internal_error(h, VH_E_ARG, "vh_load_checkpoint: the file is truncated");
  if ((r = vh_set_state(h, f.data(), hd.tau))) return r;
  if (tau_out) *tau_out = hd.tau;
  return VH_OK;
}
