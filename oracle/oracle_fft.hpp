// oracle_fft.hpp -- FP64 FFT of the oracle (test infrastructure only).
//
// The reference executes its transforms with FFTW3 (third-party, not vendored;
// version unpinned, INSTALL:125-127 mention fftw-3.3.4/3.3.5) through
// fftw_plan_many_dft_r2c / _c2r with rank 3, dims (Lz,Ly,Lx), interleaved
// components (stride = howmany, dist = 1) and padded embeds
// (Lz, Ly+padding_y, 2(Lx/2+1)) / (Lz, Ly+padding_y, Lx/2+1)
// (coord_module.F:91-93,155-157,281-283,310-312,357-359,375-377).
// This file restates the published DFT those calls compute:
//   forward r2c  X(k) = sum_R x(R) exp(-2 pi i k.R/L)       (unnormalised)
//   backward c2r x(R) = sum_{kx<=Lx/2} w(kx) Re(X(k) exp(+2 pi i k.R/L))
// with w = 1 at kx = 0 and kx = Lx/2 and 2 otherwise, i.e. complex inverse
// transforms along z and y first, then a half-complex-to-real transform along
// x that ignores the imaginary parts of the kx = 0 and kx = Lx/2 bins (the
// FFTW rdft2 convention).  The 1D kernel is a mixed-radix Stockham FFT.
#pragma once
#include <complex>
#include <vector>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace oracle {

using cd = std::complex<double>;

// One-dimensional complex DFT of length n, any n (radices 2,3,4,5, generic).
class FFT1D {
 public:
  int n = 0;
  std::vector<int> radix;
  std::vector<cd> w_fwd;  // exp(-2 pi i k / n), k = 0..n-1
  explicit FFT1D(int n_ = 1) { init(n_); }
  void init(int n_) {
    n = n_;
    radix.clear();
    int m = n;
    while (m % 4 == 0) { radix.push_back(4); m /= 4; }
    while (m % 2 == 0) { radix.push_back(2); m /= 2; }
    while (m % 3 == 0) { radix.push_back(3); m /= 3; }
    while (m % 5 == 0) { radix.push_back(5); m /= 5; }
    for (int f = 7; m > 1; f += 2) {
      while (m % f == 0) { radix.push_back(f); m /= f; }
    }
    w_fwd.resize(n);
    for (int k = 0; k < n; ++k) {
      // angle reduced exactly in integers before the libm call
      double a = -2.0 * M_PI * (double)k / (double)n;
      w_fwd[k] = cd(std::cos(a), std::sin(a));
    }
  }
  // sign = -1 forward, +1 backward (unnormalised).  data has n elements;
  // work is scratch of n elements.
  void exec(cd* data, cd* work, int sign) const {
    if (n == 1) return;
    cd* src = data;
    cd* dst = work;
    int Ns = 1;
    cd v[64];
    for (int R : radix) {
      const int nR = n / R;
      const int tstep = n / (Ns * R);
      for (int j = 0; j < nR; ++j) {
        const int k = j % Ns;
        for (int r = 0; r < R; ++r) {
          cd x = src[j + r * nR];
          int ti = (int)(((long long)r * k * tstep) % n);
          cd t = w_fwd[ti];
          if (sign > 0) t = std::conj(t);
          v[r] = x * t;
        }
        dft_small(v, R, sign);
        const int base = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
      }
      Ns *= R;
      std::swap(src, dst);
    }
    if (src != data) std::memcpy(data, src, sizeof(cd) * n);
  }

 private:
  void dft_small(cd* v, int R, int sign) const {
    if (R == 2) {
      cd a = v[0], b = v[1];
      v[0] = a + b;
      v[1] = a - b;
      return;
    }
    if (R == 4) {
      cd a0 = v[0] + v[2], a1 = v[0] - v[2];
      cd b0 = v[1] + v[3], b1 = v[1] - v[3];
      // multiply b1 by -i (forward) or +i (backward)
      cd jb1 = (sign < 0) ? cd(b1.imag(), -b1.real()) : cd(-b1.imag(), b1.real());
      v[0] = a0 + b0;
      v[2] = a0 - b0;
      v[1] = a1 + jb1;
      v[3] = a1 - jb1;
      return;
    }
    cd out[64];
    for (int s = 0; s < R; ++s) {
      cd acc = 0.0;
      for (int q = 0; q < R; ++q) {
        int idx = (int)(((long long)q * s) % R) * (n / R);
        cd t = w_fwd[idx];
        if (sign > 0) t = std::conj(t);
        acc += v[q] * t;
      }
      out[s] = acc;
    }
    for (int s = 0; s < R; ++s) v[s] = out[s];
  }
};

// Geometry of the reference's padded arrays (coord_module.F:91-93).
struct Layout {
  int Lx = 0, Ly = 0, Lz = 0, pad = 0;
  int NXP = 0;  // 2*(Lx/2+1): padded real x extent
  int NKX = 0;  // Lx/2+1: complex x extent
  int NYP = 0;  // Ly+padding_y
  void set(int lx, int ly, int lz, int p) {
    Lx = lx; Ly = ly; Lz = lz; pad = p;
    NXP = 2 * (Lx / 2 + 1);
    NKX = Lx / 2 + 1;
    NYP = Ly + pad;
  }
  size_t r(int c, int nc, int x, int y, int z) const {
    return (size_t)c + (size_t)nc * ((size_t)x + (size_t)NXP * ((size_t)y + (size_t)NYP * z));
  }
  size_t s(int x, int y, int z) const { return (size_t)x + (size_t)NXP * ((size_t)y + (size_t)NYP * z); }
  size_t k(int c, int nc, int kx, int ky, int kz) const {
    return (size_t)c + (size_t)nc * ((size_t)kx + (size_t)NKX * ((size_t)ky + (size_t)NYP * kz));
  }
  size_t nreal(int nc) const { return (size_t)nc * NXP * NYP * Lz; }
  size_t ncplx(int nc) const { return (size_t)nc * NKX * NYP * Lz; }
};

// Batched 3D transforms on the padded interleaved layout (plan_many with
// stride = howmany = nc, dist = 1).
class FFT3D {
 public:
  Layout L;
  FFT1D fx, fy, fz;
  void init(const Layout& lay) {
    L = lay;
    fx.init(L.Lx);
    fy.init(L.Ly);
    fz.init(L.Lz);
  }
  // out(c,kx,ky,kz) = sum_R in(c,R) e^{-ik.R}
  void r2c(const double* in, cd* out, int nc) const {
    const int Lx = L.Lx, Ly = L.Ly, Lz = L.Lz, m = Lx / 2;
#pragma omp parallel
    {
      std::vector<cd> row(Lx), work(Lx);
#pragma omp for collapse(2) schedule(static)
      for (int z = 0; z < Lz; ++z)
        for (int y = 0; y < Ly; ++y)
          for (int c = 0; c < nc; ++c) {
            for (int x = 0; x < Lx; ++x) row[x] = cd(in[L.r(c, nc, x, y, z)], 0.0);
            fx.exec(row.data(), work.data(), -1);
            for (int kx = 0; kx <= m; ++kx) out[L.k(c, nc, kx, y, z)] = row[kx];
          }
    }
    axis_y(out, nc, -1);
    axis_z(out, nc, -1);
  }
  // out(c,R) = sum_half w(kx) Re(in(c,k) e^{+ik.R}); in is destroyed.
  void c2r(cd* in, double* out, int nc) const {
    const int Lx = L.Lx, Ly = L.Ly, Lz = L.Lz, m = Lx / 2;
    axis_z(in, nc, +1);
    axis_y(in, nc, +1);
#pragma omp parallel
    {
      std::vector<cd> row(Lx), work(Lx);
#pragma omp for collapse(2) schedule(static)
      for (int z = 0; z < Lz; ++z)
        for (int y = 0; y < Ly; ++y)
          for (int c = 0; c < nc; ++c) {
            for (int kx = 0; kx <= m; ++kx) row[kx] = in[L.k(c, nc, kx, y, z)];
            row[0] = cd(row[0].real(), 0.0);
            if (Lx % 2 == 0) row[m] = cd(row[m].real(), 0.0);
            for (int kx = m + 1; kx < Lx; ++kx) row[kx] = std::conj(row[Lx - kx]);
            fx.exec(row.data(), work.data(), +1);
            for (int x = 0; x < Lx; ++x) out[L.r(c, nc, x, y, z)] = row[x].real();
          }
    }
  }

 private:
  void axis_y(cd* a, int nc, int sign) const {
    const int Ly = L.Ly, Lz = L.Lz;
    const int ncol = nc * L.NKX;  // consecutive in memory for fixed (y,z)
    const int B = 16;
#pragma omp parallel
    {
      std::vector<cd> buf((size_t)B * Ly), work(Ly);
#pragma omp for collapse(2) schedule(static)
      for (int z = 0; z < Lz; ++z)
        for (int c0 = 0; c0 < ncol; c0 += B) {
          int nb = std::min(B, ncol - c0);
          for (int y = 0; y < Ly; ++y) {
            const cd* src = a + (size_t)ncol * ((size_t)y + (size_t)L.NYP * z) + c0;
            for (int b = 0; b < nb; ++b) buf[(size_t)b * Ly + y] = src[b];
          }
          for (int b = 0; b < nb; ++b) fy.exec(&buf[(size_t)b * Ly], work.data(), sign);
          for (int y = 0; y < Ly; ++y) {
            cd* dst = a + (size_t)ncol * ((size_t)y + (size_t)L.NYP * z) + c0;
            for (int b = 0; b < nb; ++b) dst[b] = buf[(size_t)b * Ly + y];
          }
        }
    }
  }
  void axis_z(cd* a, int nc, int sign) const {
    const int Ly = L.Ly, Lz = L.Lz;
    const int ncol = nc * L.NKX;
    const int B = 16;
#pragma omp parallel
    {
      std::vector<cd> buf((size_t)B * Lz), work(Lz);
#pragma omp for collapse(2) schedule(static)
      for (int y = 0; y < Ly; ++y)
        for (int c0 = 0; c0 < ncol; c0 += B) {
          int nb = std::min(B, ncol - c0);
          for (int z = 0; z < Lz; ++z) {
            const cd* src = a + (size_t)ncol * ((size_t)y + (size_t)L.NYP * z) + c0;
            for (int b = 0; b < nb; ++b) buf[(size_t)b * Lz + z] = src[b];
          }
          for (int b = 0; b < nb; ++b) fz.exec(&buf[(size_t)b * Lz], work.data(), sign);
          for (int z = 0; z < Lz; ++z) {
            cd* dst = a + (size_t)ncol * ((size_t)y + (size_t)L.NYP * z) + c0;
            for (int b = 0; b < nb; ++b) dst[b] = buf[(size_t)b * Lz + z];
          }
        }
    }
  }
};

}  // namespace oracle
