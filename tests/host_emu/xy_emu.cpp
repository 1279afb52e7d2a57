// Host emulation of the xy passes of the MD step (k_xy_fwd in its SRC_U9
// form and k_xy_inv, feram_b200/csrc/fg_kernels.cuh) on small supercells:
// the kernels themselves, run block by block with one OS thread per CUDA
// thread (kernel_emu.h), against a direct 2D DFT in long double.
//
// The forward pass must give, for each z plane and each of the 9 components
// (u_x, u_y, u_z, u_x^2, u_y^2, u_z^2, u_y u_z, u_z u_x, u_x u_y; dipoFFT.F:
// 19-44), the half spectrum X(kx, ky), kx = 0..Lx/2, with ky in the
// digit-reversed slot orders of the plans: x slot s < Lx/2 holds kx =
// rev_x(s) and slot Lx/2 holds kx = Lx/2, y slot s holds ky = posm[m + s];
// the inverse pass must return Lx*Ly times each real plane.
//
// Output: one line per case, "<case> <max fwd error> <max inverse error>",
// relative to the largest |X| and to Lx*Ly times the largest |f|.
#include "kernel_emu.h"
#include "feram_gpu.h"
#include "fg_kernels.cuh"

#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

using namespace fg;
using cld = std::complex<long double>;

// The library's plan rules (fg_api.cu make_plan / digit_reversal), restated:
// the compile-time plans where fft_smem.cuh has them, otherwise radices 8,
// 4, 2, 3, 5 largest first.
bool plan_of(int n, FftPlan* P) {
  P->n = n;
  P->nst = 0;
  if (ct_supported(n)) {
    P->nst = ct_nst(n);
    for (int st = 0; st < P->nst; ++st) P->r[st] = ct_radix(n, st);
    return true;
  }
  int m = n;
  for (int r : {8, 4, 2, 3, 5})
    while (m % r == 0) {
      if (P->nst >= FFT_MAX_STAGES) return false;
      P->r[P->nst++] = r;
      m /= r;
    }
  return m == 1;
}

std::vector<int> slot_to_freq(const FftPlan& P) {
  std::vector<int> rev((size_t)P.n);
  for (int p = 0; p < P.n; ++p) {
    int q = p, k = 0, mult = 1, span = P.n;
    for (int st = 0; st < P.nst; ++st) {
      span /= P.r[st];
      const int s = q / span;
      q -= s * span;
      k += s * mult;
      mult *= P.r[st];
    }
    rev[(size_t)p] = k;
  }
  return rev;
}

template <typename T>
std::vector<cplx<T>> twiddles(int n) {
  std::vector<cplx<T>> w((size_t)n);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < n; ++k) {
    const long double a = -2.0L * pi * (long double)k / (long double)n;
    w[(size_t)k] = mk<cplx<T>>((T)std::cos(a), (T)std::sin(a));
  }
  return w;
}

std::vector<cld> unit_roots(int n) {
  std::vector<cld> w((size_t)n);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < n; ++k) w[(size_t)k] = std::polar(1.0L, -2.0L * pi * (long double)k / (long double)n);
  return w;
}

// component c of the SRC_U9 fields at site i
template <typename T>
long double field(const std::vector<T>& u, long long ns, int c, long long i) {
  const long double x = u[(size_t)i], y = u[(size_t)(ns + i)], z = u[(size_t)(2 * ns + i)];
  switch (c) {
    case 0: return x;
    case 1: return y;
    case 2: return z;
    case 3: return x * x;
    case 4: return y * y;
    case 5: return z * z;
    case 6: return y * z;
    case 7: return z * x;
    default: return x * y;
  }
}

// extra: 0 the 9 components; 1 acoustic MD (components 9..11 are src
// components 3..5, the acoustic displacement stored after u); 2 per-site Z*
// (components 9..11 are Z*(R) u, dipoFFT.F:36-44)
template <typename T, int MC, int LYC>
void xy_case(int Lx, int Ly, int Lz, int extra = 0) {
  Geom g{};
  g.Lx = Lx;
  g.Ly = Ly;
  g.Lz = Lz;
  g.m = Lx / 2;
  g.NKX = g.m + 1;
  g.KXP = (g.NKX + 15) / 16 * 16;
  g.plane_r = (long long)Lx * Ly;
  g.plane_c = (long long)Ly * g.KXP;
  g.nsite = (long long)Lx * Ly * Lz;
  g.ncplx = (long long)Lz * g.plane_c;
  g.nkpos = (long long)Ly * Lz * g.KXP;
  FftPlan px{}, py{};
  if (!plan_of(g.m, &px) || !plan_of(Ly, &py)) {
    std::printf("xy_noplan_%dx%dx%d nan nan\n", Lx, Ly, Lz);
    return;
  }
  const std::vector<int> revm = slot_to_freq(px), revy = slot_to_freq(py);
  std::vector<int> posm((size_t)(g.m + 2 * Ly));
  for (int s = 0; s < g.m; ++s) posm[(size_t)revm[(size_t)s]] = s;
  for (int s = 0; s < Ly; ++s) {
    posm[(size_t)(g.m + s)] = revy[(size_t)s];
    posm[(size_t)(g.m + Ly + revy[(size_t)s])] = s;
  }
  const std::vector<cplx<T>> twx = twiddles<T>(Lx), twm = twiddles<T>(g.m), twy = twiddles<T>(Ly);

  const long long ns = g.nsite;
  const int nc = extra ? 12 : 9, zu0 = extra == 2 ? 9 : 0;
  std::vector<T> u((size_t)((extra == 1 ? 6 : 3) * ns)), zs;
  std::mt19937_64 gen(77u + (unsigned)(Lx * 1000 + Ly * 10 + Lz + extra));
  std::uniform_real_distribution<double> dist(-0.2, 0.2), zdist(0.5, 1.5);
  for (auto& v : u) v = (T)dist(gen);
  if (extra == 2) {
    zs.resize((size_t)ns);
    for (auto& v : zs) v = (T)zdist(gen);
  }
  auto fld = [&](int c, long long i) -> long double {
    if (c < 9) return field(u, ns, c, i);
    if (extra == 1) return u[(size_t)((c - 6) * ns + i)];
    return (long double)zs[(size_t)i] * u[(size_t)((c - 9) * ns + i)];
  };
  const T nan = std::nan("");
  std::vector<cplx<T>> spec((size_t)(nc * g.ncplx), mk<cplx<T>>(nan, nan));
  const size_t smem = sizeof(cplx<T>) * (size_t)Ly * (size_t)(g.m + 1);

  emu::launch(k_xy_fwd<T, SRC_U9, MC, LYC>, dim3((unsigned)Lz, (unsigned)nc), dim3(512), smem, (const T*)u.data(),
              spec.data(), g, px, py, (const cplx<T>*)twx.data(), (const cplx<T>*)twm.data(),
              (const cplx<T>*)twy.data(), (const int*)posm.data(), 0, (const T*)(extra == 2 ? zs.data() : nullptr), zu0,
              (const RepArgs*)nullptr);

  // direct transform: along x for kx = 0..m, then along y
  const std::vector<cld> wx = unit_roots(Lx), wy = unit_roots(Ly);
  double ef = 0, xmax = 0, fmax = 0;
  std::vector<cld> rowx((size_t)Ly * (g.m + 1));
  for (int c = 0; c < nc; ++c)
    for (int z = 0; z < Lz; ++z) {
      for (int y = 0; y < Ly; ++y)
        for (int kx = 0; kx <= g.m; ++kx) {
          cld s = 0;
          for (int x = 0; x < Lx; ++x) {
            const long double f = fld(c, (long long)z * g.plane_r + (long long)y * Lx + x);
            fmax = std::max(fmax, (double)std::fabs(f));
            s += f * wx[(size_t)((kx * x) % Lx)];
          }
          rowx[(size_t)y * (g.m + 1) + kx] = s;
        }
      for (int slot = 0; slot < Ly; ++slot) {
        const int ky = posm[(size_t)(g.m + slot)];
        for (int xs = 0; xs <= g.m; ++xs) {
          const int kx = xs < g.m ? revm[(size_t)xs] : g.m;  // x slot -> kx (kx = Lx/2 in slot m)
          cld s = 0;
          for (int y = 0; y < Ly; ++y) s += rowx[(size_t)y * (g.m + 1) + kx] * wy[(size_t)((ky * y) % Ly)];
          const cplx<T> v = spec[(size_t)(c * g.ncplx + z * g.plane_c + (long long)slot * g.KXP + xs)];
          const double d = (double)std::abs(cld(v.x, v.y) - s);
          ef = std::max(ef, std::isfinite(d) ? d : 1e300);
          xmax = std::max(xmax, (double)std::abs(s));
        }
      }
    }

  std::vector<T> out((size_t)(nc * ns), nan);
  emu::launch(k_xy_inv<T, MC, LYC>, dim3((unsigned)Lz, (unsigned)nc), dim3(512), smem, (const cplx<T>*)spec.data(), out.data(),
              g, px, py, (const cplx<T>*)twx.data(), (const cplx<T>*)twm.data(), (const cplx<T>*)twy.data(),
              (const int*)posm.data(), 0, (const Phys*)nullptr, (DevScalars*)nullptr, (const double*)nullptr, 0,
              (const RepArgs*)nullptr);
  double eb = 0;
  const long double scale = (long double)Lx * Ly;
  for (int c = 0; c < nc; ++c)
    for (long long i = 0; i < ns; ++i) {
      const double d = (double)std::fabs((long double)out[(size_t)(c * ns + i)] - scale * fld(c, i));
      eb = std::max(eb, std::isfinite(d) ? d : 1e300);
    }
  std::printf("xy_%s_%s_%dx%dx%d%s %.3e %.3e\n", sizeof(T) == 4 ? "f32" : "f64", MC > 0 ? "ct" : "rt", Lx, Ly, Lz,
              extra == 1 ? "_acou" : extra == 2 ? "_zstar" : "", ef / xmax, eb / ((double)scale * fmax));
  std::fflush(stdout);
}

// The 3-component r2c / c2r of fg_fft_r2c3 / fg_fft_c2r3: k_xy_fwd
// (SRC_FIELD) then k_z_pass forward, against a direct 3D DFT in the slot
// orders of the three plans; then k_z_pass inverse and k_xy_inv, which must
// return Lx*Ly*Lz times the fields.  LZC, CWC: the z pass instance of the
// library's dispatch (0: the runtime one).
template <typename T, int MC, int LYC, int LZC, int CWC>
void fft3_case(int Lx, int Ly, int Lz) {
  Geom g{};
  g.Lx = Lx;
  g.Ly = Ly;
  g.Lz = Lz;
  g.m = Lx / 2;
  g.NKX = g.m + 1;
  g.KXP = (g.NKX + 15) / 16 * 16;
  g.plane_r = (long long)Lx * Ly;
  g.plane_c = (long long)Ly * g.KXP;
  g.nsite = (long long)Lx * Ly * Lz;
  g.ncplx = (long long)Lz * g.plane_c;
  g.nkpos = (long long)Ly * Lz * g.KXP;
  FftPlan px{}, py{}, pz{};
  if (!plan_of(g.m, &px) || !plan_of(Ly, &py) || !plan_of(Lz, &pz)) {
    std::printf("fft3_noplan_%dx%dx%d nan nan\n", Lx, Ly, Lz);
    return;
  }
  const std::vector<int> revm = slot_to_freq(px), revy = slot_to_freq(py), revz = slot_to_freq(pz);
  std::vector<int> posm((size_t)(g.m + 2 * Ly));
  for (int s = 0; s < g.m; ++s) posm[(size_t)revm[(size_t)s]] = s;
  for (int s = 0; s < Ly; ++s) {
    posm[(size_t)(g.m + s)] = revy[(size_t)s];
    posm[(size_t)(g.m + Ly + revy[(size_t)s])] = s;
  }
  const std::vector<cplx<T>> twx = twiddles<T>(Lx), twm = twiddles<T>(g.m), twy = twiddles<T>(Ly),
                             twz = twiddles<T>(Lz);
  // z tiles as the library plans them (z_tiles in fg_api.cu): the widest
  // power-of-two width up to the cap that divides Lx/2
  ZTiles zt{};
  int cw = CWC > 0 ? CWC : (sizeof(T) == 4 ? 8 : 4);
  while (cw > 1 && g.m % cw != 0) cw /= 2;
  zt.CW = cw;
  zt.ntx = g.m / cw;
  zt.nreg = zt.ntx * Ly;
  zt.nnyq = (Ly + cw - 1) / cw;

  const long long ns = g.nsite;
  std::vector<T> f((size_t)(3 * ns));
  std::mt19937_64 gen(91u + (unsigned)(Lx * 1000 + Ly * 10 + Lz));
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  for (auto& v : f) v = (T)dist(gen);
  const T nan = std::nan("");
  std::vector<cplx<T>> spec((size_t)(3 * g.ncplx), mk<cplx<T>>(nan, nan));
  const size_t smem_xy = sizeof(cplx<T>) * (size_t)Ly * (size_t)(g.m + 1);
  const size_t smem_z = 3 * sizeof(cplx<T>) * (size_t)Lz * (size_t)cw;

  emu::launch(k_xy_fwd<T, SRC_FIELD, MC, LYC>, dim3((unsigned)Lz, 3), dim3(512), smem_xy, (const T*)f.data(),
              spec.data(), g, px, py, (const cplx<T>*)twx.data(), (const cplx<T>*)twm.data(),
              (const cplx<T>*)twy.data(), (const int*)posm.data(), 0, (const T*)nullptr, 0, (const RepArgs*)nullptr);
  emu::launch(k_z_pass<T, false, LZC, CWC, (LZC > 0 ? 3 : 0)>, dim3((unsigned)(zt.nreg + zt.nnyq)), dim3(256), smem_z,
              spec.data(), g, pz, (const cplx<T>*)twz.data(), 3, zt);

  // direct transform, separable: x (kx = 0..m), y, z
  const std::vector<cld> wx = unit_roots(Lx), wy = unit_roots(Ly), wz = unit_roots(Lz);
  const int nk = g.m + 1;
  double ef = 0, xmax = 0, fmax = 0;
  std::vector<cld> a((size_t)Lz * Ly * nk), b((size_t)Lz * Ly * nk);
  for (int c = 0; c < 3; ++c) {
    for (int z = 0; z < Lz; ++z)
      for (int y = 0; y < Ly; ++y)
        for (int kx = 0; kx < nk; ++kx) {
          cld s = 0;
          for (int x = 0; x < Lx; ++x) {
            const long double v = f[(size_t)(c * ns + (long long)z * g.plane_r + (long long)y * Lx + x)];
            fmax = std::max(fmax, (double)std::fabs(v));
            s += v * wx[(size_t)((kx * x) % Lx)];
          }
          a[((size_t)z * Ly + y) * nk + kx] = s;
        }
    for (int z = 0; z < Lz; ++z)
      for (int ky = 0; ky < Ly; ++ky)
        for (int kx = 0; kx < nk; ++kx) {
          cld s = 0;
          for (int y = 0; y < Ly; ++y) s += a[((size_t)z * Ly + y) * nk + kx] * wy[(size_t)((ky * y) % Ly)];
          b[((size_t)z * Ly + ky) * nk + kx] = s;
        }
    for (int zs = 0; zs < Lz; ++zs)
      for (int ys = 0; ys < Ly; ++ys)
        for (int xs = 0; xs < nk; ++xs) {
          const int kz = revz[(size_t)zs], ky = revy[(size_t)ys], kx = xs < g.m ? revm[(size_t)xs] : g.m;
          cld s = 0;
          for (int z = 0; z < Lz; ++z) s += b[((size_t)z * Ly + ky) * nk + kx] * wz[(size_t)((kz * z) % Lz)];
          const cplx<T> v = spec[(size_t)(c * g.ncplx + (long long)zs * g.plane_c + (long long)ys * g.KXP + xs)];
          const double d = (double)std::abs(cld(v.x, v.y) - s);
          ef = std::max(ef, std::isfinite(d) ? d : 1e300);
          xmax = std::max(xmax, (double)std::abs(s));
        }
  }

  emu::launch(k_z_pass<T, true, LZC, CWC, (LZC > 0 ? 3 : 0)>, dim3((unsigned)(zt.nreg + zt.nnyq)), dim3(256), smem_z,
              spec.data(), g, pz, (const cplx<T>*)twz.data(), 3, zt);
  std::vector<T> out((size_t)(3 * ns), nan);
  emu::launch(k_xy_inv<T, MC, LYC>, dim3((unsigned)Lz, 3), dim3(512), smem_xy, (const cplx<T>*)spec.data(), out.data(),
              g, px, py, (const cplx<T>*)twx.data(), (const cplx<T>*)twm.data(), (const cplx<T>*)twy.data(),
              (const int*)posm.data(), 0, (const Phys*)nullptr, (DevScalars*)nullptr, (const double*)nullptr, 0,
              (const RepArgs*)nullptr);
  double eb = 0;
  const long double scale = (long double)ns;
  for (long long i = 0; i < 3 * ns; ++i) {
    const double d = (double)std::fabs((long double)out[(size_t)i] - scale * (long double)f[(size_t)i]);
    eb = std::max(eb, std::isfinite(d) ? d : 1e300);
  }
  std::printf("fft3_%s_%s_%dx%dx%d %.3e %.3e\n", sizeof(T) == 4 ? "f32" : "f64", LZC > 0 ? "ct" : "rt", Lx, Ly, Lz,
              ef / xmax, eb / ((double)scale * fmax));
  std::fflush(stdout);
}

template <typename T>
void all_cases() {
  // compile-time instances of the library's dispatch (m = Lx/2, Ly)
  xy_case<T, 8, 16>(16, 16, 3);
  xy_case<T, 12, 24>(24, 24, 2);
  xy_case<T, 16, 32>(32, 32, 2);
  xy_case<T, 24, 48>(48, 48, 1);
  xy_case<T, 32, 64>(64, 64, 1);
  xy_case<T, 64, 128>(128, 128, 1);
  // runtime plans (odd m, radix 3 and 5, non-square planes)
  xy_case<T, 0, 0>(10, 6, 2);
  xy_case<T, 0, 0>(12, 10, 3);
  xy_case<T, 0, 0>(20, 12, 2);
  xy_case<T, 0, 0>(30, 18, 1);
  xy_case<T, 0, 0>(16, 16, 2);
  xy_case<T, 8, 16>(16, 16, 2, 1);
  xy_case<T, 8, 16>(16, 16, 2, 2);
  xy_case<T, 0, 0>(12, 10, 2, 1);
  xy_case<T, 0, 0>(12, 10, 2, 2);
  // 3D transforms with the z pass instances of the library's dispatch
  constexpr int C = sizeof(T) == 4 ? 8 : 4;
  fft3_case<T, 8, 16, 16, C>(16, 16, 16);
  fft3_case<T, 16, 32, 32, C>(32, 32, 32);
  fft3_case<T, 8, 16, 64, C>(16, 16, 64);
  fft3_case<T, 8, 16, 128, C>(16, 16, 128);
  fft3_case<T, 12, 24, 24, 4>(24, 24, 24);
  fft3_case<T, 8, 16, 48, C>(16, 16, 48);
  fft3_case<T, 0, 0, 0, 0>(12, 10, 6);
  fft3_case<T, 0, 0, 0, 0>(20, 6, 15);
}

int main() {
  all_cases<double>();
  all_cases<float>();
  return 0;
}
