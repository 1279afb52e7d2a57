// oracle.cpp -- FP64 CPU restatement of feram's MD step (TEST INFRASTRUCTURE).
//
// Nothing in the product (feram_b200/) uses this file.  It is the parity
// checker and the timed CPU baseline.  Each function restates the Fortran
// routine cited beside it, on the reference's padded column-major layout
// (coord_module.F:91-93), with OpenMP loops over z-planes like the reference.
// Reductions are summed per z-plane and then in plane order, so results do
// not depend on the thread count.
#include "oracle.h"
#include "oracle_fft.hpp"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using oracle::cd;
using oracle::FFT3D;
using oracle::Layout;

namespace {

// define.h:21-35
const double kPi = 3.14159265358979323846;
const double k2Pi = 6.28318530717958647693;
const double k2SqrtPi = 1.12837916709551257390;
const double kHartreeBohr = 14.399644;

// ---------------------------------------------------------------- uni64 ----
// marsaglia_tsang_uni64_module.f:112-168.  Fortran default integers are 32
// bit and the seed products overflow; gfortran wraps them (two's complement),
// and MOD takes the sign of the dividend like C's %.
struct Uni64 {
  int i = 97, j = 33;
  double c = 0.0, times = 0.0;
  double u[97];
  static int32_t wrap_mul(int32_t a, int32_t b) {
    return (int32_t)((uint32_t)a * (uint32_t)b);
  }
  void fillu(int seed1, int seed2) {
    int32_t x = seed1, y = seed2;
    for (int ii = 0; ii < 97; ++ii) {
      double s = 0.0, t = 0.5;
      for (int jj = 0; jj < 53; ++jj) {
        x = wrap_mul(6969, x) % 65543;
        y = wrap_mul(8888, y) % 65579;
        if (((x ^ y) & 32) > 0) s = s + t;
        t = 0.5 * t;
      }
      u[ii] = s;
    }
  }
  double seed(int s1, int s2) {
    fillu(s1, s2);
    i = 97;
    j = 33;
    c = 0.0;
    times = times + 1.0;
    return times;
  }
  double next() {
    const double r = 9007199254740881.0 / 9007199254740992.0;
    const double d = 362436069876.0 / 9007199254740992.0;
    double x = u[i - 1] - u[j - 1];
    if (x < 0.0) x = x + 1.0;
    u[i - 1] = x;
    i = i - 1;
    if (i == 0) i = 97;
    j = j - 1;
    if (j == 0) j = 97;
    c = c - d;
    if (c < 0.0) c = c + r;
    x = x - c;
    if (x < 0.0) return x + 1.0;
    return x;
  }
};

struct NormalDist {  // marsaglia_tsang_uni64_module.f:179-202
  bool sw = true;
  double t = 0.0, u = 0.0;
};

Uni64 g_uni64;
NormalDist g_normal;

double normal_dist(double mu, double sigma) {
  double n01;
  if (g_normal.sw) {
    g_normal.sw = false;
    g_normal.t = std::sqrt(-2.0 * std::log(1.0 - g_uni64.next()));
    g_normal.u = k2Pi * g_uni64.next();
    n01 = g_normal.t * std::cos(g_normal.u);
  } else {
    g_normal.sw = true;
    n01 = g_normal.t * std::sin(g_normal.u);
  }
  return n01 * sigma + mu;
}

// ----------------------------------------------------------------- wave ----
// wave_module.F:162-221
void wave(int type, int i_step, int n_thermalize, int period, const double a[3], double out[3]) {
  if (a[0] == 0.0 && a[1] == 0.0 && a[2] == 0.0) {
    out[0] = a[0]; out[1] = a[1]; out[2] = a[2];
    return;
  }
  switch (type) {
    case FG_WAVE_TRIANGULAR_COS:
    case FG_WAVE_TRIANGULAR_SIN: {
      int i = i_step - n_thermalize;
      if (i < 0) i = 0;
      int itmp;
      if (type == FG_WAVE_TRIANGULAR_COS) itmp = std::abs(i % period - period / 2) - period / 4;
      else itmp = std::abs((i + 3 * period / 4) % period - period / 2) - period / 4;
      double tmp = (double)itmp;
      float q = (float)period / 4.0f;  // period/4.0 is default (single) real
      for (int k = 0; k < 3; ++k) out[k] = a[k] * tmp / (double)q;
      return;
    }
    case FG_WAVE_RAMPING_ON:
      if (i_step < period) {
        for (int k = 0; k < 3; ++k) out[k] = a[k] * i_step / period;
      } else {
        for (int k = 0; k < 3; ++k) out[k] = a[k];
      }
      return;
    case FG_WAVE_RAMPING_OFF:
      if (i_step < period) {
        for (int k = 0; k < 3; ++k) out[k] = a[k] * (period - i_step) / period;
      } else {
        for (int k = 0; k < 3; ++k) out[k] = 0.0;
      }
      return;
    default:
      for (int k = 0; k < 3; ++k) out[k] = a[k];
      return;
  }
}

// decay_function_module.f:13-33 (derfc = libm erfc)
double B_decay(double r, double rr, double kappa) {
  return std::erfc(kappa * r) / (r * rr) + k2SqrtPi * kappa * std::exp(-kappa * kappa * rr) / rr;
}
double C_decay(double r, double rr, double kappa) {
  double Crr = 3 * std::erfc(kappa * r) / (r * rr) +
               k2SqrtPi * kappa * std::exp(-kappa * kappa * rr) * (2 * kappa * kappa + 3 / rr);
  return Crr / rr;
}

}  // namespace

// -------------------------------------------------------------- context ----
struct oracle_ctx {
  fg_params p;
  Layout L;
  FFT3D fft;
  // real fields (comp, 0:NXP-1, 0:NYP-1, 0:Lz-1)
  std::vector<double> dipoR, dipoP, dVddi, dVddi_long, Z_u_R, didiR, acouR, acouP;
  std::vector<double> E_field, E_field_local, dipoRavg, inhoR, dVdacR;
  // scalar fields (0:NXP-1, 0:NYP-1, 0:Lz-1)
  std::vector<double> mass_dipo_inv, mass_acou_inv, Z_starR, modulation_R;
  std::vector<int> relaxor;
  std::vector<char> sum_p;
  // complex fields (comp, 0:Lx/2, 0:NYP-1, 0:Lz-1)
  std::vector<cd> dipoK, Z_u_K, dipoT, didiK, acouK, c_k_modulation_k, inhoK, dVdacK, modulation_k;
  // tables
  std::vector<double> short_range, long_range;       // (3,3,k)
  std::vector<double> inhomo_K, inhomo_K_G, inhomo_coup2_K;  // (3,3,k) (3,4,k) (3,6,k)
  double strain[6];
  double H[6][6], HG[6][6], HG_inv[6], HC2[6][6];   // homogeneous, _G, _G_inv, _coupling_2
  double s_Nose = 1.0, pi_Nose = 0.0, H0 = 0.0;
  int n_sum_p = 0;
  double E_add[3] = {0.0, 0.0, 0.0};  // last uniform field added to E_field_local
  std::vector<int> n_sum_layer;
  std::vector<double> e_layer_dipo, e_layer_acou;
  bool modulation_present = false;

  int nk() const { return L.NKX * L.NYP * L.Lz; }
  size_t t33(int a, int b, int kx, int ky, int kz) const {  // (3,3,k)
    return (size_t)a + 3 * (size_t)b + 9 * ((size_t)kx + (size_t)L.NKX * ((size_t)ky + (size_t)L.NYP * kz));
  }
  size_t t34(int a, int b, int kx, int ky, int kz) const {
    return (size_t)a + 3 * (size_t)b + 12 * ((size_t)kx + (size_t)L.NKX * ((size_t)ky + (size_t)L.NYP * kz));
  }
  size_t t36(int a, int i, int kx, int ky, int kz) const {
    return (size_t)a + 3 * (size_t)i + 18 * ((size_t)kx + (size_t)L.NKX * ((size_t)ky + (size_t)L.NYP * kz));
  }
  bool film() const { return p.bulk_or_film == FG_FILM || p.bulk_or_film == FG_EPIT; }
};

namespace {

// k vectors of elastic.F:81-87 and dVddi_inho_coupling.F:93-99
inline double kvec_x(const oracle_ctx* o, int ix) { return (double)ix / o->p.Lx * k2Pi / o->p.a0; }
inline double kvec_w(int i, int L, double a0) {
  double k = (double)i / L;
  if (k > 0.5) k = k - 1.0;
  return k * k2Pi / a0;
}

// alloc_Coord (coord_module.F:67-432): allocate and initialise.
void alloc_coord(oracle_ctx* o) {
  const Layout& L = o->L;
  auto rz = [&](std::vector<double>& v, int nc) { v.assign(L.nreal(nc), 0.0); };
  auto cz = [&](std::vector<cd>& v, int nc) { v.assign(L.ncplx(nc), cd(0.0, 0.0)); };
  rz(o->mass_dipo_inv, 1); rz(o->mass_acou_inv, 1); rz(o->Z_starR, 1); rz(o->modulation_R, 1);
  rz(o->dipoR, 3); rz(o->dipoP, 3); rz(o->dVddi, 3); rz(o->dVddi_long, 3); rz(o->Z_u_R, 3);
  rz(o->didiR, 6); rz(o->acouR, 3); rz(o->acouP, 3); rz(o->E_field, 3); rz(o->E_field_local, 3);
  rz(o->dipoRavg, 3); rz(o->inhoR, 6); rz(o->dVdacR, 3);
  cz(o->dipoK, 3); cz(o->Z_u_K, 3); cz(o->dipoT, 3); cz(o->didiK, 6); cz(o->acouK, 3);
  cz(o->c_k_modulation_k, 3); cz(o->inhoK, 6); cz(o->dVdacK, 3); cz(o->modulation_k, 1);
  o->relaxor.assign(L.nreal(1), 1);
  o->sum_p.assign(L.nreal(1), 0);
  const double mdi = 1.0 / o->p.mass_dipo[0];
  const double mai = 1.0 / o->p.mass_acou[0];
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) {
        o->mass_dipo_inv[L.s(x, y, z)] = mdi;
        o->mass_acou_inv[L.s(x, y, z)] = mai;
        o->Z_starR[L.s(x, y, z)] = o->p.Z_star[0];
      }
  const size_t nk = (size_t)o->nk();
  o->short_range.assign(9 * nk, 0.0);
  o->long_range.assign(9 * nk, 0.0);
  o->inhomo_K.assign(9 * nk, 0.0);
  o->inhomo_K_G.assign(12 * nk, 0.0);
  o->inhomo_coup2_K.assign(18 * nk, 0.0);
  o->n_sum_layer.assign(L.Lz, L.Lx * L.Ly);
  o->e_layer_dipo.assign(L.Lz, 0.0);
  o->e_layer_acou.assign(L.Lz, 0.0);
}

// fft_3d_3x3upper_r2c (fft_3d_3x3upper_r2c.F:9-36): FFT of each upper-
// triangle component of an unpadded (Lx,Ly,Lz,3,3) real array; only the
// real parts are kept by the callers, and Re conj(c) = Re c.
void fft_3x3upper_real(const oracle_ctx* o, const std::vector<double>& TMP /*(x,y,z,3,3)*/,
                       std::vector<double>& table /*(3,3,k)*/) {
  const Layout& L = o->L;
  const size_t nsite = (size_t)L.Lx * L.Ly * L.Lz;
  std::vector<double> in(L.nreal(6), 0.0);
  std::vector<cd> out(L.ncplx(6));
  int pair[6][2], ip = 0;
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a <= b; ++a) { pair[ip][0] = a; pair[ip][1] = b; ++ip; }
  for (int c = 0; c < 6; ++c) {
    const int a = pair[c][0], b = pair[c][1];
    for (int z = 0; z < L.Lz; ++z)
      for (int y = 0; y < L.Ly; ++y)
        for (int x = 0; x < L.Lx; ++x)
          in[L.r(c, 6, x, y, z)] = TMP[(size_t)x + (size_t)L.Lx * (y + (size_t)L.Ly * z) + nsite * (a + 3 * b)];
  }
  o->fft.r2c(in.data(), out.data(), 6);
  for (int c = 0; c < 6; ++c) {
    const int a = pair[c][0], b = pair[c][1];
    for (int kz = 0; kz < L.Lz; ++kz)
      for (int ky = 0; ky < L.Ly; ++ky)
        for (int kx = 0; kx < L.NKX; ++kx) {
          double v = out[L.k(c, 6, kx, ky, kz)].real();
          table[o->t33(a, b, kx, ky, kz)] = v;
          table[o->t33(b, a, kx, ky, kz)] = v;
        }
  }
}

// dipole_dipole_long_range (dipole-dipole-long-range.F:14-152)
void dipole_dipole_long_range(oracle_ctx* o) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  const double four_pi_over_v = 4 * kPi / (p.a0 * p.a0 * p.a0);
  const double two_pi_over_a = 2 * kPi / p.a0;
  const double four_kappa2 = 4 * p.kappa * p.kappa;
  const double Lx_a0 = p.Lx * p.a0, Ly_a0 = p.Ly * p.a0, Lz_a0 = p.Lz * p.a0;
  const int max_x = 24 / p.Lx, max_y = 24 / p.Ly, max_z = 24 / p.Lz;
  const size_t nsite = (size_t)L.Lx * L.Ly * L.Lz;
  std::vector<double> TMP(nsite * 9, 0.0);
  for (int a = 0; a < 3; ++a) TMP[nsite * (a + 3 * a)] = -2 * k2SqrtPi * p.kappa * p.kappa * p.kappa / 3;
  // Real-space sum.  Per element the image order (jz, jy, jx) and the
  // B-then-C update order of the reference are kept; B and C are evaluated
  // once per (image, site) since they do not depend on (alpha, beta).
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < L.Lz; ++iz)
    for (int iy = 0; iy < L.Ly; ++iy)
      for (int ix = 0; ix < L.Lx; ++ix) {
        const size_t site = (size_t)ix + (size_t)L.Lx * (iy + (size_t)L.Ly * iz);
        double acc[9];
        for (int e = 0; e < 9; ++e) acc[e] = TMP[site + nsite * e];
        for (int jz = -1 - max_z; jz <= max_z; ++jz)
          for (int jy = -1 - max_y; jy <= max_y; ++jy)
            for (int jx = -1 - max_x; jx <= max_x; ++jx) {
              if (jx == 0 && jy == 0 && jz == 0 && ix == 0 && iy == 0 && iz == 0) continue;
              double rn[3] = {ix * p.a0 + jx * Lx_a0, iy * p.a0 + jy * Ly_a0, iz * p.a0 + jz * Lz_a0};
              double rnrn = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
              double rn_norm = std::sqrt(rnrn);
              double B = B_decay(rn_norm, rnrn, p.kappa);
              double C = C_decay(rn_norm, rnrn, p.kappa);
              for (int b = 0; b < 3; ++b)
                for (int a = 0; a < 3; ++a) {
                  double& t = acc[a + 3 * b];
                  if (a == b) t = t + B;
                  t = t - rn[a] * rn[b] * C;
                }
            }
        for (int e = 0; e < 9; ++e) TMP[site + nsite * e] = acc[e];
      }
  fft_3x3upper_real(o, TMP, o->long_range);
  // Reciprocal-space sum
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < L.Lz; ++iz) {
    double k[3];
    k[2] = (double)iz / p.Lz;
    if (k[2] > 0.5) k[2] = k[2] - 1.0;
    for (int iy = 0; iy < L.Ly; ++iy) {
      k[1] = (double)iy / p.Ly;
      if (k[1] > 0.5) k[1] = k[1] - 1.0;
      for (int ix = 0; ix <= p.Lx / 2; ++ix) {
        k[0] = (double)ix / p.Lx;
        for (int b = 0; b < 3; ++b)
          for (int a = 0; a < 3; ++a) {
            double& t = o->long_range[o->t33(a, b, ix, iy, iz)];
            for (int nz = -max_z; nz <= max_z; ++nz) {
              double kG2 = two_pi_over_a * (k[2] + nz);
              for (int ny = -max_y; ny <= max_y; ++ny) {
                double kG1 = two_pi_over_a * (k[1] + ny);
                for (int nx = -max_x; nx <= max_x; ++nx) {
                  if (ix == 0 && iy == 0 && iz == 0 && nx == 0 && ny == 0 && nz == 0) continue;
                  double kG0 = two_pi_over_a * (k[0] + nx);
                  double kG[3] = {kG0, kG1, kG2};
                  double kGkG = kG0 * kG0 + kG1 * kG1 + kG2 * kG2;
                  t = t + four_pi_over_v * kG[a] * kG[b] * std::exp(-kGkG / four_kappa2) / kGkG;
                }
              }
            }
          }
      }
    }
  }
  const double scale = kHartreeBohr / p.epsilon_inf;
  for (auto& v : o->long_range) v = v * scale;
}

// dipole_dipole_short_range (dipole-dipole-short-range.F:10-135)
void dipole_dipole_short_range(oracle_ctx* o) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  const size_t nsite = (size_t)L.Lx * L.Ly * L.Lz;
  std::vector<double> TMP(nsite * 9, 0.0);
  auto at = [&](int x, int y, int z, int a, int b) -> double& {
    return TMP[(size_t)x + (size_t)L.Lx * (y + (size_t)L.Ly * z) + nsite * (a + 3 * b)];
  };
  for (int a = 0; a < 3; ++a) at(0, 0, 0, a, a) = p.P_kappa2[0] * 2;
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a)
      for (int iz = -1; iz <= 1; ++iz)
        for (int iy = -1; iy <= 1; ++iy)
          for (int ix = -1; ix <= 1; ++ix) {
            int i[3] = {ix, iy, iz};
            int indx[3] = {ix >= 0 ? ix : p.Lx + ix, iy >= 0 ? iy : p.Ly + iy, iz >= 0 ? iz : p.Lz + iz};
            int ii = ix * ix + iy * iy + iz * iz;
            double& t = at(indx[0], indx[1], indx[2], a, b);
            if (ii == 1) {
              if (a == b) t = (i[a] == 0) ? p.j[0] : p.j[1];
            } else if (ii == 2) {
              if (a == b) t = (i[a] == 0) ? p.j[3] : p.j[2];
              else t = p.j[4] * i[a] * i[b];
            } else if (ii == 3) {
              if (a == b) t = p.j[5];
              else t = p.j[6] * i[a] * i[b];
            }
          }
  fft_3x3upper_real(o, TMP, o->short_range);
}

// elastic (elastic.F:7-237), without the .modulation file (see
// oracle_set_modulation_R for that branch).
void elastic(oracle_ctx* o) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  double(*H)[6] = o->H;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) { H[i][j] = 0.0; o->HG[i][j] = 0.0; o->HC2[i][j] = 0.0; }
  for (int i = 0; i < 3; ++i) H[i][i] = p.B11 * p.N;
  for (int i = 3; i < 6; ++i) H[i][i] = p.B44 * p.N;
  H[0][1] = H[0][2] = H[1][2] = H[1][0] = H[2][0] = H[2][1] = p.B12 * p.N;
  for (int j = 0; j < 6; ++j) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) s += o->HG[j][k] * o->HG[j][k];
    o->HG[j][j] = std::sqrt(H[j][j] - s);
    o->HG_inv[j] = 1.0 / o->HG[j][j];
    for (int i = j + 1; i < 6; ++i) {
      double t = 0.0;
      for (int k = 0; k < j; ++k) t += o->HG[i][k] * o->HG[j][k];
      o->HG[i][j] = (H[i][j] - t) * o->HG_inv[j];
    }
  }
  for (int i = 0; i < 3; ++i) o->HC2[i][i] = p.B1xx / 2;
  for (int i = 3; i < 6; ++i) o->HC2[i][i] = p.B4yz;
  o->HC2[0][1] = o->HC2[0][2] = o->HC2[1][2] = o->HC2[1][0] = o->HC2[2][0] = o->HC2[2][1] = p.B1yy / 2;
  // inhomo_K, its Cholesky factor, inhomo_coup2_K
  static const int ki[3][3] = {{0, 3, 2}, {3, 0, 1}, {2, 1, 0}};  // elastic.F:17 (1-based axes, 0 = none)
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < L.Lz; ++iz) {
    double k[4];
    k[0] = 0.0;
    k[3] = kvec_w(iz, p.Lz, p.a0);
    for (int iy = 0; iy < L.Ly; ++iy) {
      k[2] = kvec_w(iy, p.Ly, p.a0);
      for (int ix = 0; ix <= p.Lx / 2; ++ix) {
        k[1] = kvec_x(o, ix);
        for (int b = 1; b <= 3; ++b) {
          int other1 = (b + 1) % 3 + 1;
          int other2 = b % 3 + 1;
          for (int a = 1; a <= 3; ++a) {
            double v;
            if (a == b) v = p.B11 * k[a] * k[a] + p.B44 * k[other1] * k[other1] + p.B44 * k[other2] * k[other2];
            else v = p.B12 * k[a] * k[b] + p.B44 * k[a] * k[b];
            o->inhomo_K[o->t33(a - 1, b - 1, ix, iy, iz)] = v;
          }
        }
        if (ix != 0 || iy != 0 || iz != 0) {
          for (int b = 0; b < 3; ++b) {
            double s = 0.0;
            for (int q = 0; q < b; ++q) s += o->inhomo_K_G[o->t34(b, q, ix, iy, iz)] * o->inhomo_K_G[o->t34(b, q, ix, iy, iz)];
            double g = std::sqrt(o->inhomo_K[o->t33(b, b, ix, iy, iz)] - s);
            o->inhomo_K_G[o->t34(b, b, ix, iy, iz)] = g;
            o->inhomo_K_G[o->t34(b, 3, ix, iy, iz)] = 1.0 / g;
            for (int a = b + 1; a < 3; ++a) {
              double t = 0.0;
              for (int q = 0; q < b; ++q) t += o->inhomo_K_G[o->t34(a, q, ix, iy, iz)] * o->inhomo_K_G[o->t34(b, q, ix, iy, iz)];
              o->inhomo_K_G[o->t34(a, b, ix, iy, iz)] = (o->inhomo_K[o->t33(a, b, ix, iy, iz)] - t) * o->inhomo_K_G[o->t34(b, 3, ix, iy, iz)];
            }
          }
        }
        for (int i = 1; i <= 6; ++i)
          for (int a = 1; a <= 3; ++a) {
            double v;
            if (i <= 3) v = (i == a) ? k[a] * p.B1xx / 2 : k[a] * p.B1yy / 2;
            else v = k[ki[a - 1][i - 4]] * p.B4yz;
            o->inhomo_coup2_K[o->t36(a - 1, i - 1, ix, iy, iz)] = v;
          }
      }
    }
  }
}

// mirror (mirror.F:9-36) on a 3-component field
void mirror(const oracle_ctx* o, std::vector<double>& f) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  auto copy_layer = [&](int src, int dst) {
    for (int y = 0; y < L.NYP; ++y)
      for (int x = 0; x < L.NXP; ++x) {
        f[L.r(0, 3, x, y, dst)] = -f[L.r(0, 3, x, y, src)];
        f[L.r(1, 3, x, y, dst)] = -f[L.r(1, 3, x, y, src)];
        f[L.r(2, 3, x, y, dst)] = f[L.r(2, 3, x, y, src)];
      }
  };
  if (p.gap_id == 0) {
    for (int iz = 0; iz <= p.Lz / 2 - 1; ++iz) copy_layer(iz, p.Lz - 1 - iz);
  } else {
    for (int iz = 1; iz <= (p.Lz + 1) / 2 - 1; ++iz) copy_layer(iz, p.Lz - iz);
  }
}

// Sum over physical sites of f(x,y,z) with per-plane partials summed in order.
template <class F>
double site_sum(const oracle_ctx* o, F f) {
  const Layout& L = o->L;
  std::vector<double> part(L.Lz, 0.0);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z) {
    double acc = 0.0;
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) acc += f(x, y, z);
    part[z] = acc;
  }
  double s = 0.0;
  for (int z = 0; z < L.Lz; ++z) s += part[z];
  return s;
}

// dipoFFT (dipoFFT.F:9-47)
void dipoFFT(oracle_ctx* o) {
  const Layout& L = o->L;
  o->fft.r2c(o->dipoR.data(), o->dipoK.data(), 3);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) {
        const double* u = &o->dipoR[L.r(0, 3, x, y, z)];
        double* d = &o->didiR[L.r(0, 6, x, y, z)];
        d[0] = u[0] * u[0]; d[1] = u[1] * u[1]; d[2] = u[2] * u[2];
        d[3] = u[1] * u[2]; d[4] = u[2] * u[0]; d[5] = u[0] * u[1];
      }
  o->fft.r2c(o->didiR.data(), o->didiK.data(), 6);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a)
          o->Z_u_R[L.r(a, 3, x, y, z)] = o->Z_starR[L.s(x, y, z)] * o->dipoR[L.r(a, 3, x, y, z)];
  o->fft.r2c(o->Z_u_R.data(), o->Z_u_K.data(), 3);
}

// acouFFT (acouFFT.F:9-26)
void acouFFT(oracle_ctx* o) {
  o->fft.r2c(o->acouR.data(), o->acouK.data(), 3);
  for (auto& v : o->acouK) v = cd(0.0, 1.0) * v;
}

// dVddi_dipole_dipole (dVddi-dipole-dipole.F:8-103)
void dVddi_dipole_dipole(oracle_ctx* o, fg_energy* e) {
  const Layout& L = o->L;
  const double Ninv = o->p.Ninv;
  auto kmul = [&](const std::vector<double>& tab, const std::vector<cd>& src) {
#pragma omp parallel for schedule(static)
    for (int kz = 0; kz < L.Lz; ++kz)
      for (int ky = 0; ky < L.Ly; ++ky)
        for (int kx = 0; kx <= L.Lx / 2; ++kx)
          for (int a = 0; a < 3; ++a) {
            cd acc = 0.0;
            for (int b = 0; b < 3; ++b) acc += tab[o->t33(a, b, kx, ky, kz)] * src[L.k(b, 3, kx, ky, kz)];
            o->dipoT[L.k(a, 3, kx, ky, kz)] = acc;
          }
  };
  kmul(o->short_range, o->dipoK);
  o->fft.c2r(o->dipoT.data(), o->dVddi.data(), 3);
  for (auto& v : o->dVddi) v = v * Ninv;
  kmul(o->long_range, o->Z_u_K);
  o->fft.c2r(o->dipoT.data(), o->dVddi_long.data(), 3);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a) {
          double& v = o->dVddi_long[L.r(a, 3, x, y, z)];
          v = o->Z_starR[L.s(x, y, z)] * v * Ninv;
        }
  double es = site_sum(o, [&](int x, int y, int z) {
    const double* u = &o->dipoR[L.r(0, 3, x, y, z)];
    const double* f = &o->dVddi[L.r(0, 3, x, y, z)];
    return u[0] * f[0] + u[1] * f[1] + u[2] * f[2];
  });
  e->short_range = es / 2;
  double el = site_sum(o, [&](int x, int y, int z) {
    const double* u = &o->dipoR[L.r(0, 3, x, y, z)];
    const double* f = &o->dVddi_long[L.r(0, 3, x, y, z)];
    return u[0] * f[0] + u[1] * f[1] + u[2] * f[2];
  });
  e->long_range = el / 2;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a) o->dVddi[L.r(a, 3, x, y, z)] += o->dVddi_long[L.r(a, 3, x, y, z)];
}

// dVddi_unharmonic (dVddi-unharmonic.F:6-101)
void dVddi_unharmonic(oracle_ctx* o, fg_energy* e) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  double fa2g[3], tg[3], sk[3], tk2[3], fk[3];
  for (int s = 0; s < 3; ++s) {
    fa2g[s] = 4 * p.P_alpha[s] + 2 * p.P_gamma[s];
    tg[s] = 2 * p.P_gamma[s];
    sk[s] = 6 * p.P_k1[s] + 2 * p.P_k2[s];
    tk2[s] = 2 * p.P_k2[s];
    fk[s] = 4 * p.P_k2[s] - 2 * p.P_k3[s];
  }
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) {
        const int s = o->relaxor[L.s(x, y, z)] - 1;
        const double* u = &o->dipoR[L.r(0, 3, x, y, z)];
        const double* d = &o->didiR[L.r(0, 6, x, y, z)];
        double* f = &o->dVddi[L.r(0, 3, x, y, z)];
        for (int a = 0; a < 3; ++a) {
          f[a] = f[a] + u[a] * 2 * (p.P_kappa2[s] - p.P_kappa2[0]);
          f[a] = f[a] + u[a] * (fa2g[s] * (d[0] + d[1] + d[2]) - tg[s] * d[a]);
          int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
          double uu = d[0] + d[1] + d[2];
          f[a] = f[a] + u[a] * (sk[s] * (uu * uu) + 8 * p.P_k4[s] * (uu * uu * uu) - tk2[s] * (d[a] * d[a]) -
                                fk[s] * d[a1] * d[a2]);
        }
      }
  e->unharmonic = site_sum(o, [&](int x, int y, int z) {
    const int s = o->relaxor[L.s(x, y, z)] - 1;
    const double* d = &o->didiR[L.r(0, 6, x, y, z)];
    double uu = d[0] + d[1] + d[2];
    return (p.P_kappa2[s] - p.P_kappa2[0]) * uu + p.P_alpha[s] * (uu * uu) +
           p.P_gamma[s] * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]) + p.P_k1[s] * (uu * uu * uu) +
           p.P_k2[s] * ((d[0] * d[0]) * (d[1] + d[2]) + (d[1] * d[1]) * (d[2] + d[0]) + (d[2] * d[2]) * (d[0] + d[1])) +
           p.P_k3[s] * d[0] * d[1] * d[2] + p.P_k4[s] * (uu * uu * uu * uu);
  });
}

// optimize_homo_strain (optimize-homo-strain.F:8-89)
void optimize_homo_strain(oracle_ctx* o, fg_energy* e) {
  const fg_params& p = o->p;
  double hc2uu[6];
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += o->HC2[i][j] * o->didiK[o->L.k(j, 6, 0, 0, 0)].real();
    hc2uu[i] = s;
  }
  for (int i = 0; i < 3; ++i) hc2uu[i] = hc2uu[i] + p.pNa03[i];
  double* st = o->strain;
  if (p.bulk_or_film == FG_EPIT) {
    st[0] = p.epi_strain;
    st[1] = p.epi_strain;
    st[2] = (-(o->H[2][0] + o->H[2][1]) * p.epi_strain - hc2uu[2]) / o->H[2][2];
    st[3] = -hc2uu[3] / o->H[3][3];
    st[4] = -hc2uu[4] / o->H[4][4];
    st[5] = 0.0;
  } else if (p.bulk_or_film == FG_E110) {
    st[2] = p.epi_strain;
    st[3] = 0.0;
    st[4] = 0.0;
    double numerator = -(o->H[0][0] + o->H[1][1] + 2 * o->H[1][1]) * p.epi_strain -
                       (o->H[2][0] + o->H[2][1]) * st[2] - hc2uu[0] - hc2uu[1] + 2 * hc2uu[5];
    double denominator = o->H[0][0] + o->H[1][1] + 2 * o->H[1][0] + 4 * o->H[5][5];
    double delta = numerator / denominator;
    st[0] = p.epi_strain + delta;
    st[1] = p.epi_strain + delta;
    st[5] = -2 * delta;
  } else {
    for (int i = 0; i < 6; ++i) st[i] = -hc2uu[i];
    for (int i = 0; i < 6; ++i) {
      double tmp = 0.0;
      for (int j = 0; j < i; ++j) tmp = tmp + o->HG[i][j] * st[j];
      st[i] = (st[i] - tmp) * o->HG_inv[i];
    }
    for (int i = 5; i >= 0; --i) {
      double tmp = 0.0;
      for (int j = i + 1; j < 6; ++j) tmp = tmp + st[j] * o->HG[j][i];
      st[i] = (st[i] - tmp) * o->HG_inv[i];
    }
  }
  double hs = 0.0;
  for (int i = 0; i < 6; ++i) {
    double d = 0.0;
    for (int j = 0; j < 6; ++j) d += o->H[i][j] * st[j];
    hs = hs + st[i] * d;
  }
  e->homo_strain = hs / 2;
  double hc = 0.0;
  for (int i = 0; i < 6; ++i) hc += st[i] * hc2uu[i];
  e->homo_coupling = hc;
}

// The 3-component stencil shared by dVddi-homo-coupling.F:219-233 and
// dVddi_inho_coupling.F:127-138.
inline void strain_coupling_add(const double* w, const double* u, double* f) {
  f[0] = f[0] + 2 * w[0] * u[0] + w[4] * u[2] + w[5] * u[1];
  f[1] = f[1] + 2 * w[1] * u[1] + w[3] * u[2] + w[5] * u[0];
  f[2] = f[2] + 2 * w[2] * u[2] + w[3] * u[1] + w[4] * u[0];
}

// dVddi_homo_coupling (dVddi-homo-coupling.F:6-49)
void dVddi_homo_coupling(oracle_ctx* o) {
  const Layout& L = o->L;
  double w[6] = {0, 0, 0, 0, 0, 0};
  for (int j = 0; j < 6; ++j)
    for (int i = 0; i < 6; ++i) w[j] = w[j] + o->strain[i] * o->HC2[i][j];
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        strain_coupling_add(w, &o->dipoR[L.r(0, 3, x, y, z)], &o->dVddi[L.r(0, 3, x, y, z)]);
}

// optimize_inho_strain (optimize-inho-strain.F:10-60)
void optimize_inho_strain(oracle_ctx* o) {
  const Layout& L = o->L;
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < L.Lz; ++kz)
    for (int ky = 0; ky < L.Ly; ++ky)
      for (int kx = 0; kx <= L.Lx / 2; ++kx) {
        cd a[3];
        for (int al = 0; al < 3; ++al) {
          cd d = 0.0;
          for (int i = 0; i < 6; ++i) d += o->inhomo_coup2_K[o->t36(al, i, kx, ky, kz)] * o->didiK[L.k(i, 6, kx, ky, kz)];
          a[al] = -o->c_k_modulation_k[L.k(al, 3, kx, ky, kz)] - d;
        }
        for (int al = 0; al < 3; ++al) {
          cd tmp = 0.0;
          for (int be = 0; be < al; ++be) tmp = tmp + o->inhomo_K_G[o->t34(al, be, kx, ky, kz)] * a[be];
          a[al] = (a[al] - tmp) * o->inhomo_K_G[o->t34(al, 3, kx, ky, kz)];
        }
        for (int al = 2; al >= 0; --al) {
          cd tmp = 0.0;
          for (int be = al + 1; be < 3; ++be) tmp = tmp + a[be] * o->inhomo_K_G[o->t34(be, al, kx, ky, kz)];
          a[al] = (a[al] - tmp) * o->inhomo_K_G[o->t34(al, 3, kx, ky, kz)];
        }
        for (int al = 0; al < 3; ++al) o->acouK[L.k(al, 3, kx, ky, kz)] = a[al];
      }
}

// dVdac (dVdac.F:11-63)
void dVdac(oracle_ctx* o) {
  const Layout& L = o->L;
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < L.Lz; ++kz)
    for (int ky = 0; ky < L.NYP; ++ky)
      for (int kx = 0; kx <= L.Lx / 2; ++kx)
        for (int a = 0; a < 3; ++a) o->dVdacK[L.k(a, 3, kx, ky, kz)] = 0.0;
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < L.Lz; ++kz)
    for (int ky = 0; ky < L.Ly; ++ky)
      for (int kx = 0; kx <= L.Lx / 2; ++kx)
        for (int a = 0; a < 3; ++a) {
          cd m1 = 0.0, m2 = 0.0;
          for (int i = 0; i < 6; ++i) m1 += o->inhomo_coup2_K[o->t36(a, i, kx, ky, kz)] * o->didiK[L.k(i, 6, kx, ky, kz)];
          for (int b = 0; b < 3; ++b) m2 += o->inhomo_K[o->t33(a, b, kx, ky, kz)] * o->acouK[L.k(b, 3, kx, ky, kz)];
          cd v = o->dVdacK[L.k(a, 3, kx, ky, kz)] + o->c_k_modulation_k[L.k(a, 3, kx, ky, kz)] + m1 + m2;
          o->dVdacK[L.k(a, 3, kx, ky, kz)] = cd(0.0, -1.0) * v;
        }
  o->fft.c2r(o->dVdacK.data(), o->dVdacR.data(), 3);
  for (auto& v : o->dVdacR) v = v * o->p.Ninv;
}

// Half-spectrum weighted sum of energy_module.F:150-240: weight 1/2 at
// kx = 0 and kx = Lx/2, 1 between.
template <class F>
double half_sum(const oracle_ctx* o, F f) {
  const Layout& L = o->L;
  std::vector<double> part(L.Lz, 0.0);
  const int m = L.Lx / 2;
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < L.Lz; ++kz) {
    double acc = 0.0;
    for (int ky = 0; ky < L.Ly; ++ky) {
      double t1 = f(0, ky, kz) / 2;
      double t2 = 0.0;
      for (int kx = 1; kx <= m - 1; ++kx) t2 += f(kx, ky, kz);
      double t3 = f(m, ky, kz) / 2;
      acc += t1 + t2 + t3;
    }
    part[kz] = acc;
  }
  double s = 0.0;
  for (int kz = 0; kz < L.Lz; ++kz) s += part[kz];
  return s;
}

void inhomogeneous_energies(oracle_ctx* o, fg_energy* e) {
  const Layout& L = o->L;
  const double Ninv = o->p.Ninv;
  e->inho_strain = half_sum(o, [&](int kx, int ky, int kz) {
                     double s = 0.0;
                     for (int a = 0; a < 3; ++a)
                       for (int b = 0; b < 3; ++b)
                         s += (std::conj(o->acouK[L.k(a, 3, kx, ky, kz)]) * o->inhomo_K[o->t33(a, b, kx, ky, kz)] *
                               o->acouK[L.k(b, 3, kx, ky, kz)]).real();
                     return s;
                   }) * Ninv;
  e->inho_coupling = half_sum(o, [&](int kx, int ky, int kz) {
                       double s = 0.0;
                       for (int i = 0; i < 6; ++i)
                         for (int a = 0; a < 3; ++a)
                           s += (std::conj(o->acouK[L.k(a, 3, kx, ky, kz)]) * o->inhomo_coup2_K[o->t36(a, i, kx, ky, kz)] *
                                 o->didiK[L.k(i, 6, kx, ky, kz)]).real();
                       return s;
                     }) * 2 * Ninv;
  if (o->p.modulation_constant == 0.0) {
    e->inho_modulation = 0.0;
  } else {
    e->inho_modulation = half_sum(o, [&](int kx, int ky, int kz) {
                           double s = 0.0;
                           for (int a = 0; a < 3; ++a)
                             s += (std::conj(o->acouK[L.k(a, 3, kx, ky, kz)]) * o->c_k_modulation_k[L.k(a, 3, kx, ky, kz)]).real();
                           return s;
                         }) * 2 * Ninv;
  }
}

// dVddi_inho_coupling (dVddi_inho_coupling.F:9-84)
void dVddi_inho_coupling(oracle_ctx* o) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < L.Lz; ++iz) {
    double k[3];
    k[2] = kvec_w(iz, p.Lz, p.a0);
    for (int iy = 0; iy < L.Ly; ++iy) {
      k[1] = kvec_w(iy, p.Ly, p.a0);
      for (int ix = 0; ix <= p.Lx / 2; ++ix) {
        k[0] = (double)ix / p.Lx * k2Pi / p.a0;
        const cd a0 = o->acouK[L.k(0, 3, ix, iy, iz)], a1 = o->acouK[L.k(1, 3, ix, iy, iz)],
                 a2 = o->acouK[L.k(2, 3, ix, iy, iz)];
        cd* h = &o->inhoK[L.k(0, 6, ix, iy, iz)];
        h[0] = k[0] * a0;
        h[1] = k[1] * a1;
        h[2] = k[2] * a2;
        h[3] = k[2] * a1 + k[1] * a2;
        h[4] = k[0] * a2 + k[2] * a0;
        h[5] = k[1] * a0 + k[0] * a1;
      }
    }
  }
  o->fft.c2r(o->inhoK.data(), o->inhoR.data(), 6);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) {
        const double* r = &o->inhoR[L.r(0, 6, x, y, z)];
        double w[6];
        for (int i = 0; i < 6; ++i) {
          w[i] = r[0] * p.Ninv * o->HC2[0][i] + r[1] * p.Ninv * o->HC2[1][i] + r[2] * p.Ninv * o->HC2[2][i] +
                 r[3] * p.Ninv * o->HC2[3][i] + r[4] * p.Ninv * o->HC2[4][i] + r[5] * p.Ninv * o->HC2[5][i];
        }
        strain_coupling_add(w, &o->dipoR[L.r(0, 3, x, y, z)], &o->dVddi[L.r(0, 3, x, y, z)]);
      }
}

// mirror_force_mirror (mirror_force_mirror.F:6-89).  Writes the potential
// members of e only.
void mirror_force_mirror(oracle_ctx* o, fg_energy* e) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  if (o->film()) mirror(o, o->dipoR);
  dipoFFT(o);
  if (p.mass_acou[0] > 0.0) acouFFT(o);
  dVddi_dipole_dipole(o, e);
  dVddi_unharmonic(o, e);
  if (p.E_field_always_zero) {
    e->dipole_E_field = 0.0;
  } else {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < L.Lz; ++z)
      for (int y = 0; y < L.Ly; ++y)
        for (int x = 0; x < L.Lx; ++x)
          for (int a = 0; a < 3; ++a)
            o->dVddi[L.r(a, 3, x, y, z)] = o->dVddi[L.r(a, 3, x, y, z)] - o->Z_starR[L.s(x, y, z)] * o->E_field[L.r(a, 3, x, y, z)];
    double t = site_sum(o, [&](int x, int y, int z) {
      const double* u = &o->dipoR[L.r(0, 3, x, y, z)];
      const double* E = &o->E_field[L.r(0, 3, x, y, z)];
      return o->Z_starR[L.s(x, y, z)] * (u[0] * E[0] + u[1] * E[1] + u[2] * E[2]);
    });
    e->dipole_E_field = -t;
  }
  optimize_homo_strain(o, e);
  dVddi_homo_coupling(o);
  if (p.mass_acou[0] > 0.0) dVdac(o);
  else optimize_inho_strain(o);
  inhomogeneous_energies(o, e);
  dVddi_inho_coupling(o);
  if (o->film()) mirror(o, o->dVddi);
}

double kinetic_energy_dipo(const oracle_ctx* o) {  // kinetic_energy_dipo.F:1-29
  const Layout& L = o->L;
  double t = site_sum(o, [&](int x, int y, int z) {
    if (!o->sum_p[L.s(x, y, z)]) return 0.0;
    const double* q = &o->dipoP[L.r(0, 3, x, y, z)];
    const double mi = o->mass_dipo_inv[L.s(x, y, z)];
    return q[0] * q[0] * mi + q[1] * q[1] * mi + q[2] * q[2] * mi;
  });
  return t / o->n_sum_p * o->p.N / 2;
}

double kinetic_energy_acou(const oracle_ctx* o) {  // kinetic_energy_acou.F:1-28
  const Layout& L = o->L;
  double t = site_sum(o, [&](int x, int y, int z) {
    const double* q = &o->acouP[L.r(0, 3, x, y, z)];
    const double mi = o->mass_acou_inv[L.s(x, y, z)];
    return q[0] * q[0] * mi + q[1] * q[1] * mi + q[2] * q[2] * mi;
  });
  return t / 2;
}

double sum_potential(const fg_energy* e) {  // energy_module.F:73-87
  return e->short_range + e->long_range + e->dipole_E_field + e->unharmonic + e->homo_strain + e->homo_coupling +
         e->inho_strain + e->inho_coupling + e->inho_modulation;
}

void np_hamiltonian(const oracle_ctx* o, fg_energy* e) {  // energy_module.F:128-148
  const fg_params& p = o->p;
  double h = e->dipo_kinetic / (o->s_Nose * o->s_Nose) + sum_potential(e) + o->pi_Nose * o->pi_Nose / 2 / p.Q_Nose +
             3 * p.N * p.temperature_eV * std::log(o->s_Nose) - o->H0;
  e->H_Nose_Poincare = h * o->s_Nose;
}

// p <- p - f * F on every padded element, as the reference's whole-array
// statements (nose-poincare.F:25-28,66-71; leapfrog.F:134-138).
void kick_all(std::vector<double>& P, const std::vector<double>& F, double f, int Lz, size_t plane) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < Lz; ++z)
    for (size_t i = (size_t)z * plane; i < (size_t)(z + 1) * plane; ++i) P[i] = P[i] - f * F[i];
}

void nose_poincare(oracle_ctx* o, fg_energy* e) {  // nose-poincare.F:10-78
  const fg_params& p = o->p;
  const Layout& L = o->L;
  const size_t plane = (size_t)3 * L.NXP * L.NYP;
  double dt2s = p.dt_2 * o->s_Nose;
  kick_all(o->dipoP, o->dVddi, dt2s, L.Lz, plane);  // (35a)
  e->dipo_kinetic = kinetic_energy_dipo(o);
  double CB = p.n_freedom * p.temperature_eV * (1.0 + std::log(o->s_Nose)) - e->dipo_kinetic / (o->s_Nose * o->s_Nose) +
              sum_potential(e) - o->H0;
  CB = p.dt_2 * CB - o->pi_Nose;
  o->pi_Nose = -2 * CB / (1.0 + std::sqrt(1.0 - CB * p.dt / p.Q_Nose));  // (38)
  double s_old = o->s_Nose;
  o->s_Nose = o->s_Nose * (1.0 + p.dt_2 * o->pi_Nose / p.Q_Nose) / (1.0 - p.dt_2 * o->pi_Nose / p.Q_Nose);  // (35c)
  double dt2_s_s = p.dt_2 * (1 / o->s_Nose + 1 / s_old);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a)
          o->dipoR[L.r(a, 3, x, y, z)] = o->dipoR[L.r(a, 3, x, y, z)] +
                                         dt2_s_s * o->dipoP[L.r(a, 3, x, y, z)] * o->mass_dipo_inv[L.s(x, y, z)];  // (35d)
  mirror_force_mirror(o, e);
  np_hamiltonian(o, e);
  double delta_H = e->H_Nose_Poincare / o->s_Nose;
  o->pi_Nose = o->pi_Nose + p.dt_2 * (2 * e->dipo_kinetic / (o->s_Nose * o->s_Nose) - p.n_freedom * p.temperature_eV) -
               p.dt_2 * delta_H;  // (35e)
  dt2s = p.dt_2 * o->s_Nose;
  kick_all(o->dipoP, o->dVddi, dt2s, L.Lz, plane);  // (35f)
  e->dipo_kinetic = kinetic_energy_dipo(o);
  np_hamiltonian(o, e);
}

void leapfrog(oracle_ctx* o, fg_energy* e, int i_step) {  // leapfrog.F:9-157
  const fg_params& p = o->p;
  const Layout& L = o->L;
  const size_t plane = (size_t)3 * L.NXP * L.NYP;
  const bool acou = p.mass_acou[0] > 0.0;
  if (p.delta_e != 0.0 || p.delta_e_acou != 0.0) {
    for (int iz = 0; iz < L.Lz; ++iz) {
      double s = 0.0;
      for (int y = 0; y < L.Ly; ++y)
        for (int x = 0; x < L.Lx; ++x)
          for (int a = 0; a < 3; ++a) {
            double q = o->dipoP[L.r(a, 3, x, y, iz)];
            s = s + q * q * o->mass_dipo_inv[L.s(x, y, iz)];
          }
      o->e_layer_dipo[iz] = s / 2 * p.Lx * p.Ly / o->n_sum_layer[iz];
    }
    if (acou) {
      for (int iz = 0; iz < L.Lz; ++iz) {
        double s = 0.0;
        for (int y = 0; y < L.Ly; ++y)
          for (int x = 0; x < L.Lx; ++x)
            for (int a = 0; a < 3; ++a) {
              double q = o->acouP[L.r(a, 3, x, y, iz)];
              s = s + q * q * o->mass_acou_inv[L.s(x, y, iz)];
            }
        o->e_layer_acou[iz] = s / 2;
      }
    } else {
      std::fill(o->e_layer_acou.begin(), o->e_layer_acou.end(), 0.0);
    }
  }
  const double LxLyde = p.Lx * p.Ly * p.delta_e, LxLydea = p.Lx * p.Ly * p.delta_e_acou;
  const int z14 = p.Lz / 4, z34 = z14 * 3;
  auto scale_layer = [&](std::vector<double>& P, int iz, double f) {
    for (int y = 0; y < L.NYP; ++y)
      for (int x = 0; x < L.NXP; ++x)
        for (int a = 0; a < 3; ++a) P[L.r(a, 3, x, y, iz)] *= f;
  };
  if (p.delta_e != 0.0) {
    scale_layer(o->dipoP, z14, std::sqrt((o->e_layer_dipo[z14] + LxLyde) / o->e_layer_dipo[z14]));
    scale_layer(o->dipoP, z34, std::sqrt((o->e_layer_dipo[z34] - LxLyde) / o->e_layer_dipo[z34]));
  }
  if (p.delta_e_acou != 0.0) {
    scale_layer(o->acouP, z14, std::sqrt((o->e_layer_acou[z14] + LxLydea) / o->e_layer_acou[z14]));
    scale_layer(o->acouP, z34, std::sqrt((o->e_layer_acou[z34] - LxLydea) / o->e_layer_acou[z34]));
  }
  if (i_step == 0) {
    mirror_force_mirror(o, e);
    kick_all(o->dipoP, o->dVddi, p.dt_2, L.Lz, plane);
    if (acou) kick_all(o->acouP, o->dVdacR, p.dt_2, L.Lz, plane);
  } else {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < L.Lz; ++z)
      for (int y = 0; y < L.Ly; ++y)
        for (int x = 0; x < L.Lx; ++x)
          for (int a = 0; a < 3; ++a)
            o->dipoR[L.r(a, 3, x, y, z)] =
                o->dipoR[L.r(a, 3, x, y, z)] + p.dt * o->dipoP[L.r(a, 3, x, y, z)] * o->mass_dipo_inv[L.s(x, y, z)];
    if (acou) {
#pragma omp parallel for schedule(static)
      for (int z = 0; z < L.Lz; ++z)
        for (int y = 0; y < L.Ly; ++y)
          for (int x = 0; x < L.Lx; ++x)
            for (int a = 0; a < 3; ++a)
              o->acouR[L.r(a, 3, x, y, z)] =
                  o->acouR[L.r(a, 3, x, y, z)] + p.dt * o->acouP[L.r(a, 3, x, y, z)] * o->mass_acou_inv[L.s(x, y, z)];
    }
    mirror_force_mirror(o, e);
    kick_all(o->dipoP, o->dVddi, p.dt, L.Lz, plane);
    if (acou) kick_all(o->acouP, o->dVdacR, p.dt, L.Lz, plane);
  }
  e->dipo_kinetic = kinetic_energy_dipo(o);
  if (acou) e->acou_kinetic = kinetic_energy_acou(o);
}

void velocity_scaling(oracle_ctx* o, fg_energy* e) {  // velocity_scaling.F:9-103
  const fg_params& p = o->p;
  const Layout& L = o->L;
  const bool acou = p.mass_acou[0] > 0.0;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a) {
          o->dipoR[L.r(a, 3, x, y, z)] =
              o->dipoR[L.r(a, 3, x, y, z)] + p.dt * o->dipoP[L.r(a, 3, x, y, z)] * o->mass_dipo_inv[L.s(x, y, z)];
          if (acou)
            o->acouR[L.r(a, 3, x, y, z)] =
                o->acouR[L.r(a, 3, x, y, z)] + p.dt * o->acouP[L.r(a, 3, x, y, z)] * o->mass_acou_inv[L.s(x, y, z)];
        }
  mirror_force_mirror(o, e);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a) {
          double& q = o->dipoP[L.r(a, 3, x, y, z)];
          q = o->sum_p[L.s(x, y, z)] ? q - p.dt * o->dVddi[L.r(a, 3, x, y, z)] : 0.0;
        }
  e->dipo_kinetic = kinetic_energy_dipo(o);
  double scale = std::sqrt(p.target_kinetic_energy / e->dipo_kinetic);
  for (double& q : o->dipoP) q = q * scale;
  if (acou) {
    const size_t plane = (size_t)3 * L.NXP * L.NYP;
    kick_all(o->acouP, o->dVdacR, p.dt, L.Lz, plane);
    e->acou_kinetic = kinetic_energy_acou(o);
    scale = std::sqrt(p.target_kinetic_energy / e->acou_kinetic);
    for (double& q : o->acouP) q = q * scale;
  }
}

// read_defects_u (read_defects_u.F:8-80) without a .defects file
void read_defects_u(oracle_ctx* o) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) o->sum_p[L.s(x, y, z)] = 1;
  if (o->film()) {
    for (int z = (p.Lz + 1) / 2; z < p.Lz; ++z)
      for (int y = 0; y < L.NYP; ++y)
        for (int x = 0; x < L.NXP; ++x) o->sum_p[L.s(x, y, z)] = 0;
  }
  auto gap_layer = [&](int z) {
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) {
        for (int a = 0; a < 3; ++a) o->dipoR[L.r(a, 3, x, y, z)] = p.gap_dipole_u[a];
        o->mass_dipo_inv[L.s(x, y, z)] = 0.0;
        o->sum_p[L.s(x, y, z)] = 0;
      }
  };
  if (p.gap_id > 0) {
    gap_layer(0);
    if (p.gap_id == 2) gap_layer(p.Lz / 2);
  }
  int n = 0;
  for (int z = 0; z < L.Lz; ++z) {
    int nl = 0;
    for (int y = 0; y < L.NYP; ++y)
      for (int x = 0; x < L.NXP; ++x) nl += o->sum_p[L.s(x, y, z)] ? 1 : 0;
    o->n_sum_layer[z] = nl;
    n += nl;
  }
  o->n_sum_p = n;
}

void add_to_average(const oracle_ctx* o, const fg_energy* e, fg_average* avg) {  // average_module.F:57-128
  const Layout& L = o->L;
  double* ae = &avg->energy.acou_kinetic;
  const double* ee = &e->acou_kinetic;
  for (int i = 0; i < 13; ++i) ae[i] += ee[i];
  avg->e2 += e->total * e->total;
  avg->dipo_kinetic_true += e->dipo_kinetic / (o->s_Nose * o->s_Nose);
  for (int i = 0; i < 6; ++i) avg->strain[i] += o->strain[i];
  double ut[3] = {0, 0, 0}, pt[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    ut[a] = site_sum(o, [&](int x, int y, int z) { return o->sum_p[L.s(x, y, z)] ? o->dipoR[L.r(a, 3, x, y, z)] : 0.0; });
    pt[a] = site_sum(o, [&](int x, int y, int z) { return o->sum_p[L.s(x, y, z)] ? o->Z_u_R[L.r(a, 3, x, y, z)] : 0.0; });
  }
  for (int a = 0; a < 3; ++a) { avg->u[a] += ut[a]; avg->p[a] += pt[a]; }
  avg->uu[0] += ut[0] * ut[0]; avg->uu[1] += ut[1] * ut[1]; avg->uu[2] += ut[2] * ut[2];
  avg->uu[3] += ut[1] * ut[2]; avg->uu[4] += ut[2] * ut[0]; avg->uu[5] += ut[0] * ut[1];
  avg->pp[0] += pt[0] * pt[0]; avg->pp[1] += pt[1] * pt[1]; avg->pp[2] += pt[2] * pt[2];
  avg->pp[3] += pt[1] * pt[2]; avg->pp[4] += pt[2] * pt[0]; avg->pp[5] += pt[0] * pt[1];
  avg->n_steps += 1;
}

void set_E_field(oracle_ctx* o, const double Eadd[3]) {
  const Layout& L = o->L;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int a = 0; a < 3; ++a)
          o->E_field[L.r(a, 3, x, y, z)] = o->E_field_local[L.r(a, 3, x, y, z)] + Eadd[a];
}

void copy_in(const oracle_ctx* o, std::vector<double>& dst, const double* src, int nc) {
  const Layout& L = o->L;
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int c = 0; c < nc; ++c) dst[L.r(c, nc, x, y, z)] = src[L.r(c, nc, x, y, z)];
}
void copy_out(const oracle_ctx* o, const std::vector<double>& src, double* dst, int nc) {
  const Layout& L = o->L;
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x)
        for (int c = 0; c < nc; ++c) dst[L.r(c, nc, x, y, z)] = src[L.r(c, nc, x, y, z)];
}
void copy_out_c(const oracle_ctx* o, const std::vector<cd>& src, double* dst, int nc) {
  const Layout& L = o->L;
  for (int kz = 0; kz < L.Lz; ++kz)
    for (int ky = 0; ky < L.Ly; ++ky)
      for (int kx = 0; kx < L.NKX; ++kx)
        for (int c = 0; c < nc; ++c) {
          size_t i = L.k(c, nc, kx, ky, kz);
          dst[2 * i] = src[i].real();
          dst[2 * i + 1] = src[i].imag();
        }
}

void set_err(char* errbuf, int errlen, const std::string& s) {
  if (errbuf && errlen > 0) {
    std::snprintf(errbuf, (size_t)errlen, "%s", s.c_str());
  }
}

}  // namespace

// ================================================================ C API ====
extern "C" {

oracle_ctx* oracle_create(const fg_params* p, char* errbuf, int errlen) {
  if (!p || p->Lx < 1 || p->Ly < 1 || p->Lz < 1 || p->N != p->Lx * p->Ly * p->Lz) {
    set_err(errbuf, errlen, "oracle_create: parameters not made (call fg_make_param)");
    return nullptr;
  }
  if (p->Lx % 2 != 0) {
    set_err(errbuf, errlen, "oracle_create: Lx must be even");
    return nullptr;
  }
  oracle_ctx* o = new oracle_ctx();
  o->p = *p;
  o->L.set(p->Lx, p->Ly, p->Lz, p->padding_y);
  o->fft.init(o->L);
  alloc_coord(o);
  dipole_dipole_long_range(o);
  dipole_dipole_short_range(o);
  elastic(o);
  for (int i = 0; i < 6; ++i) o->strain[i] = 0.0;
  // sum_p/mass masks as read_defects_u leaves them without a .defects file
  read_defects_u(o);
  return o;
}

void oracle_destroy(oracle_ctx* o) { delete o; }

int oracle_get_tables(oracle_ctx* o, double* sr, double* lr) {
  if (sr) std::memcpy(sr, o->short_range.data(), sizeof(double) * o->short_range.size());
  if (lr) std::memcpy(lr, o->long_range.data(), sizeof(double) * o->long_range.size());
  return 0;
}

int oracle_get_inhomo_tables(oracle_ctx* o, double* K, double* KG, double* C2) {
  if (K) std::memcpy(K, o->inhomo_K.data(), sizeof(double) * o->inhomo_K.size());
  if (KG) std::memcpy(KG, o->inhomo_K_G.data(), sizeof(double) * o->inhomo_K_G.size());
  if (C2) std::memcpy(C2, o->inhomo_coup2_K.data(), sizeof(double) * o->inhomo_coup2_K.size());
  return 0;
}

// elastic.F:183-226: modulation_k = r2c(modulation_R); c_k = const * k * modulation_k
int oracle_set_modulation_R(oracle_ctx* o, const double* modR) {
  const Layout& L = o->L;
  const fg_params& p = o->p;
  for (int z = 0; z < L.Lz; ++z)
    for (int y = 0; y < L.Ly; ++y)
      for (int x = 0; x < L.Lx; ++x) o->modulation_R[L.s(x, y, z)] = modR[L.s(x, y, z)];
  o->fft.r2c(o->modulation_R.data(), o->modulation_k.data(), 1);
  for (int iz = 0; iz < L.Lz; ++iz) {
    double kz = kvec_w(iz, p.Lz, p.a0);
    for (int iy = 0; iy < L.Ly; ++iy) {
      double ky = kvec_w(iy, p.Ly, p.a0);
      for (int ix = 0; ix <= p.Lx / 2; ++ix) {
        double kx = kvec_x(o, ix);
        double k[3] = {kx, ky, kz};
        cd m = o->modulation_k[L.k(0, 1, ix, iy, iz)];
        for (int a = 0; a < 3; ++a) o->c_k_modulation_k[L.k(a, 3, ix, iy, iz)] = p.modulation_constant * k[a] * m;
      }
    }
  }
  o->modulation_present = true;
  return 0;
}

int oracle_get_modulation(oracle_ctx* o, double* c) {
  copy_out_c(o, o->c_k_modulation_k, c, 3);
  return 0;
}

int oracle_set_state(oracle_ctx* o, const double* dipoR, const double* dipoP, double s, double pi, double H0) {
  if (dipoR) copy_in(o, o->dipoR, dipoR, 3);
  if (dipoP) copy_in(o, o->dipoP, dipoP, 3);
  o->s_Nose = s;
  o->pi_Nose = pi;
  o->H0 = H0;
  return 0;
}

int oracle_get_state(oracle_ctx* o, double* dipoR, double* dipoP, double* dVddi, double* strain6, double* s,
                     double* pi, double* H0) {
  if (dipoR) copy_out(o, o->dipoR, dipoR, 3);
  if (dipoP) copy_out(o, o->dipoP, dipoP, 3);
  if (dVddi) copy_out(o, o->dVddi, dVddi, 3);
  if (strain6) std::memcpy(strain6, o->strain, sizeof(double) * 6);
  if (s) *s = o->s_Nose;
  if (pi) *pi = o->pi_Nose;
  if (H0) *H0 = o->H0;
  return 0;
}

int oracle_set_acou(oracle_ctx* o, const double* acouR, const double* acouP) {
  if (acouR) copy_in(o, o->acouR, acouR, 3);
  if (acouP) copy_in(o, o->acouP, acouP, 3);
  return 0;
}

int oracle_get_acou(oracle_ctx* o, double* acouR, double* acouP, double* dVdacR) {
  if (acouR) copy_out(o, o->acouR, acouR, 3);
  if (acouP) copy_out(o, o->acouP, acouP, 3);
  if (dVdacR) copy_out(o, o->dVdacR, dVdacR, 3);
  return 0;
}

int oracle_get_acouK(oracle_ctx* o, double* acouK) {
  copy_out_c(o, o->acouK, acouK, 3);
  return 0;
}

int oracle_acouR_for_coord(oracle_ctx* o, double* acouR) {
  if (o->p.mass_acou[0] <= 0.0) {
    std::vector<cd> tmp(o->acouK.size());
    for (size_t i = 0; i < tmp.size(); ++i) tmp[i] = cd(0.0, -1.0) * o->acouK[i];
    std::vector<double> r(o->L.nreal(3), 0.0);
    o->fft.c2r(tmp.data(), r.data(), 3);
    for (auto& v : r) v = v * o->p.Ninv;
    copy_out(o, r, acouR, 3);
  } else {
    copy_out(o, o->acouR, acouR, 3);
  }
  return 0;
}

// Per-site arrays as read_relaxor (read_relaxor.F), read_defects_u
// (read_defects_u.F) and initialize_E_field (initialize_E_field.F:14-45) set
// them; padded layouts; NULL keeps the current values.
int oracle_set_sites(oracle_ctx* o, const double* Z_starR, const double* mass_dipo_inv, const double* mass_acou_inv,
                     const int* relaxor, const int* sum_p, const double* E_field_local) {
  const Layout& L = o->L;
  const size_t n1 = L.nreal(1);
  for (size_t i = 0; i < n1; ++i) {
    if (Z_starR) o->Z_starR[i] = Z_starR[i];
    if (mass_dipo_inv) o->mass_dipo_inv[i] = mass_dipo_inv[i];
    if (mass_acou_inv) o->mass_acou_inv[i] = mass_acou_inv[i];
    if (relaxor) o->relaxor[i] = relaxor[i];
  }
  if (sum_p) {
    int n = 0;
    for (int z = 0; z < L.Lz; ++z) {
      int nl = 0;
      for (int y = 0; y < L.Ly; ++y)
        for (int x = 0; x < L.Lx; ++x) {
          o->sum_p[L.s(x, y, z)] = sum_p[L.s(x, y, z)] ? 1 : 0;
          nl += o->sum_p[L.s(x, y, z)];
        }
      o->n_sum_layer[z] = nl;
      n += nl;
    }
    o->n_sum_p = n;
  }
  if (E_field_local) {
    copy_in(o, o->E_field_local, E_field_local, 3);
    o->p.E_field_always_zero = 0;
    set_E_field(o, o->E_add);
    if (o->film()) mirror(o, o->E_field);
  }
  return 0;
}

int oracle_set_uniform_E(oracle_ctx* o, const double E[3]) {
  for (int a = 0; a < 3; ++a) o->E_add[a] = E[a];
  set_E_field(o, E);
  if (o->film()) mirror(o, o->E_field);
  return 0;
}

int oracle_force(oracle_ctx* o, fg_energy* e) {
  mirror_force_mirror(o, e);
  return 0;
}

int oracle_nose_poincare(oracle_ctx* o, fg_energy* e) {
  nose_poincare(o, e);
  return 0;
}

int oracle_velocity_scaling(oracle_ctx* o, fg_energy* e) {
  velocity_scaling(o, e);
  return 0;
}

int oracle_leapfrog(oracle_ctx* o, fg_energy* e, int i_step) {
  leapfrog(o, e, i_step);
  return 0;
}

double oracle_kinetic_energy_dipo(oracle_ctx* o) { return kinetic_energy_dipo(o); }

double oracle_nose_poincare_hamiltonian(oracle_ctx* o, fg_energy* e) {
  np_hamiltonian(o, e);
  return e->H_Nose_Poincare;
}

// initialize_E_field (initialize_E_field.F:6-74) + initialize_dipoR
// (initialize-dipoR.F:8-71), without sidecar files.
int oracle_initialize(oracle_ctx* o, fg_energy* e) {
  const fg_params& p = o->p;
  const Layout& L = o->L;
  double E0[3];
  wave(p.E_wave_type, 0, p.n_thermalize, p.n_E_wave_period, p.external_E_field, E0);
  oracle_set_uniform_E(o, E0);
  g_normal.sw = true;
  g_uni64.seed(p.seed[0], p.seed[1]);
  for (int a = 0; a < 3; ++a)
    for (int iz = 0; iz < L.Lz; ++iz)
      for (int iy = 0; iy < L.Ly; ++iy)
        for (int ix = 0; ix < L.Lx; ++ix) {
          double v = normal_dist(p.init_dipo_avg[a], p.init_dipo_dev[a]);
          if (std::cos(k2Pi * (p.k_stripe[0] * ix + p.k_stripe[1] * iy + p.k_stripe[2] * iz + 1.0e-4)) < 0.0) v = -v;
          o->dipoR[L.r(a, 3, ix, iy, iz)] = v;
        }
  std::fill(o->dipoP.begin(), o->dipoP.end(), 0.0);
  std::fill(o->acouR.begin(), o->acouR.end(), 0.0);
  read_defects_u(o);
  mirror_force_mirror(o, e);
  o->s_Nose = 1.0;
  o->pi_Nose = 0.0;
  e->acou_kinetic = kinetic_energy_acou(o);
  e->dipo_kinetic = kinetic_energy_dipo(o);
  e->H_Nose_Poincare = 0.0;
  return 0;
}

int oracle_md(oracle_ctx* o, int i_first, int i_last, int set_H0, fg_energy* e, fg_average* avg) {
  const fg_params& p = o->p;
  if (set_H0) {
    e->total = e->dipo_kinetic / (o->s_Nose * o->s_Nose) + e->acou_kinetic + sum_potential(e);
    o->H0 = 0.0;
    np_hamiltonian(o, e);
    o->H0 = e->H_Nose_Poincare / o->s_Nose;
    np_hamiltonian(o, e);
  }
  for (int i_step = i_first; i_step <= i_last; ++i_step) {
    if (p.E_wave_type != FG_WAVE_NONE) {
      double Eadd[3];
      wave(p.E_wave_type, i_step, p.n_thermalize, p.n_E_wave_period, p.external_E_field, Eadd);
      set_E_field(o, Eadd);
    }
    switch (p.method) {
      case FG_METHOD_MD: nose_poincare(o, e); break;
      case FG_METHOD_LF: leapfrog(o, e, i_step); break;
      case FG_METHOD_VS: velocity_scaling(o, e); break;
      default: return FG_ERR_UNSUPPORTED;
    }
    e->total = e->dipo_kinetic / (o->s_Nose * o->s_Nose) + e->acou_kinetic + sum_potential(e);
    if (i_step <= p.n_thermalize) continue;
    if (avg) add_to_average(o, e, avg);
  }
  return 0;
}

int oracle_average_accumulate(oracle_ctx* o, const fg_energy* e, fg_average* avg) {
  add_to_average(o, e, avg);
  return 0;
}

double oracle_uni64_seed(int s1, int s2) { return g_uni64.seed(s1, s2); }
double oracle_uni64(void) { return g_uni64.next(); }
double oracle_normal_dist_seed(int s1, int s2) {
  g_normal.sw = true;
  return g_uni64.seed(s1, s2);
}
double oracle_normal_dist(double mu, double sigma) { return normal_dist(mu, sigma); }

void oracle_wave(int type, int i_step, int n_thermalize, int period, const double a[3], double out[3]) {
  wave(type, i_step, n_thermalize, period, a, out);
}

int oracle_r2c(int Lx, int Ly, int Lz, int pad, int nc, const double* in, double* out) {
  Layout L;
  L.set(Lx, Ly, Lz, pad);
  FFT3D f;
  f.init(L);
  f.r2c(in, reinterpret_cast<cd*>(out), nc);
  return 0;
}

int oracle_c2r(int Lx, int Ly, int Lz, int pad, int nc, double* in, double* out) {
  Layout L;
  L.set(Lx, Ly, Lz, pad);
  FFT3D f;
  f.init(L);
  f.c2r(reinterpret_cast<cd*>(in), out, nc);
  return 0;
}

// Defaults of read_Param (param_module.F:129-194), for inputs built without
// a .feram file.  Strings are empty ("" = current directory).
void oracle_default_param(fg_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->method = FG_METHOD_MD;
  for (int i = 0; i < FG_RELAXOR_MAX; ++i) {
    p->mass_dipo[i] = 100.0 / 9648.53377163899;
    p->mass_acou[i] = -100.0;
  }
  p->Q_Nose = 0.1;
  p->bulk_or_film = FG_BULK;
  p->Lx = p->Ly = p->Lz = 32;
  p->padding_y = 1;
  p->a0 = 4.0;
  p->n_thermalize = 10000;
  p->n_average = 100000;
  p->n_coord_freq = 2147483647;  // huge(1)
  p->n_hl_freq = 10000;
  p->n_hysteresis_loop_continue = 1;
  p->E_wave_type = FG_WAVE_NONE;
  p->seed[0] = 123456789;
  p->seed[1] = 987654321;
  for (int a = 0; a < 3; ++a) p->init_dipo_dev[a] = 0.05;
  p->verbose = 1;
  p->E_field_always_zero = 1;
}

// make_Param (param_module.F:452-480), plus temperature_eV = kelvin /
// KELVIN_EV, which read_Param sets with the kelvin tag (param_module.F:226).
// Constants of define.h:21,34,35.
int oracle_make_param(fg_params* p) {
  const double kPiRef = 3.14159265358979323846, kKelvinEV = 11604.45, kElem = 1.60217653;
  if (p->Lx < 1 || p->Ly < 1 || p->Lz < 1) return FG_ERR_ARG;
  p->N = p->Lx * p->Ly * p->Lz;
  p->Ninv = 1.0 / p->N;
  p->dt_2 = p->dt / 2;
  p->n_freedom = 3 * p->N;
  if (p->kappa <= 0.0) p->kappa = std::sqrt(kPiRef) / p->a0 / std::pow((double)p->N, 1.0 / 6);
  p->unit_cell_volume = p->a0 * p->a0 * p->a0;
  for (int i = 0; i < 3; ++i) p->pNa03[i] = p->GPa[i] * 0.01 / kElem * p->N * p->unit_cell_volume;
  p->target_kinetic_energy = p->kelvin * 1.5 * p->N / kKelvinEV;
  p->temperature_eV = p->kelvin / kKelvinEV;
  if (p->bulk_or_film == FG_BULK) {
    if (p->gap_id != 0) return FG_ERR_ARG;
  } else if (p->Lz % 2 != p->gap_id % 2) {
    return FG_ERR_ARG;
  }
  return 0;
}

// initialize_dipoR without a .restart file (initialize-dipoR.F:41-56): the
// seeded Gaussian u in the reference's draw order, stripe sign flips, p = 0.
// Padded layout; dipoP may be NULL.
int oracle_init_dipoR(const fg_params* p, double* dipoR, double* dipoP) {
  if (!p || !dipoR) return FG_ERR_ARG;
  Layout L;
  L.set(p->Lx, p->Ly, p->Lz, p->padding_y);
  std::fill(dipoR, dipoR + L.nreal(3), 0.0);
  if (dipoP) std::fill(dipoP, dipoP + L.nreal(3), 0.0);
  g_normal.sw = true;
  g_uni64.seed(p->seed[0], p->seed[1]);
  for (int a = 0; a < 3; ++a)
    for (int iz = 0; iz < L.Lz; ++iz)
      for (int iy = 0; iy < L.Ly; ++iy)
        for (int ix = 0; ix < L.Lx; ++ix) {
          double v = normal_dist(p->init_dipo_avg[a], p->init_dipo_dev[a]);
          if (std::cos(k2Pi * (p->k_stripe[0] * ix + p->k_stripe[1] * iy + p->k_stripe[2] * iz + 1.0e-4)) < 0.0) v = -v;
          dipoR[L.r(a, 3, ix, iy, iz)] = v;
        }
  return 0;
}

void oracle_set_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
