// Host emulation of the shared-memory FFT stages of feram_b200/csrc/fft_smem.cuh.
//
// The stage functions are written so that any thread may take any butterfly
// of a stage and the only ordering is a barrier between stages.  Running
// every "thread" of a stage one after another on the host, then the next
// stage, is therefore the same computation as the device's, and checks the
// index arithmetic, the stage plans (ct_radix / ct_ls / ct_nst), the radix
// kernels and the twiddle indexing of the product source itself against an
// exact DFT (long double), with no GPU.
//
// Output: one line per case, "<case> <max fwd error> <max inverse error>",
// errors relative to the largest |X(k)| (forward) and to N max|x| (inverse).
#include "emu_shim.h"
#include "fft_smem.cuh"

#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

uint3 threadIdx, blockIdx;
dim3 blockDim, gridDim;

using namespace fg;
using cld = std::complex<long double>;

template <typename T>
std::vector<cplx<T>> twiddle_table(int n) {
  std::vector<cplx<T>> w((size_t)n);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < n; ++k) {
    const long double a = -2.0L * pi * (long double)k / (long double)n;
    w[(size_t)k] = mk<cplx<T>>((T)std::cos(a), (T)std::sin(a));
  }
  return w;
}

// Slot of frequency k after a DIF with stage radices r[i..]: the stage
// leaves frequencies k = s (mod r) in the s-th sub-block of length n / r.
int slot_of(int k, const std::vector<int>& r, size_t i, int n) {
  if (i == r.size() || n == 1) return 0;
  const int R = r[i], S = n / R;
  return (k % R) * S + slot_of(k / R, r, i + 1, S);
}

std::vector<cld> exact_dft(const std::vector<cld>& x) {
  const int n = (int)x.size();
  const long double pi = 3.14159265358979323846264338327950288L;
  std::vector<cld> X((size_t)n);
  for (int k = 0; k < n; ++k) {
    cld s = 0;
    for (int j = 0; j < n; ++j) {
      const long double a = -2.0L * pi * (long double)(((long long)j * k) % n) / (long double)n;
      s += x[(size_t)j] * cld(std::cos(a), std::sin(a));
    }
    X[(size_t)k] = s;
  }
  return X;
}

// Emulated launch of one stage: every thread of the block in turn.
template <class F>
void all_threads(int nt, F&& f) {
  blockDim = dim3((unsigned)nt, 1, 1);
  for (int t = 0; t < nt; ++t) {
    threadIdx = make_uint3((unsigned)t, 0, 0);
    f();
  }
}

struct Layout {
  int count, inner, istr, outer, es, len;
};

// Compare a batch after forward stages with the exact DFT of its input, then
// after the inverse stages with n times the input.
template <typename T>
void check(const char* name, int n, const std::vector<int>& radices, const Layout& L,
           const std::vector<cplx<T>>& in, const std::vector<cplx<T>>& fwd, const std::vector<cplx<T>>& back) {
  double ef = 0, eb = 0, xmax = 0, fmax = 0;
  for (int t = 0; t < L.count; ++t) {
    const int base = (t / L.inner) * L.outer + (t % L.inner) * L.istr;
    std::vector<cld> x((size_t)n);
    for (int e = 0; e < n; ++e) {
      const cplx<T> v = in[(size_t)(base + e * L.es)];
      x[(size_t)e] = cld(v.x, v.y);
      xmax = std::max(xmax, (double)std::abs(x[(size_t)e]));
    }
    const std::vector<cld> X = exact_dft(x);
    for (int k = 0; k < n; ++k) {
      const cplx<T> v = fwd[(size_t)(base + slot_of(k, radices, 0, n) * L.es)];
      ef = std::max(ef, (double)std::abs(cld(v.x, v.y) - X[(size_t)k]));
      fmax = std::max(fmax, (double)std::abs(X[(size_t)k]));
      const cplx<T> b = back[(size_t)(base + k * L.es)];
      eb = std::max(eb, (double)std::abs(cld(b.x, b.y) - (long double)n * x[(size_t)k]));
    }
  }
  std::printf("%s %.3e %.3e\n", name, ef / fmax, eb / (n * xmax));
}

template <typename T>
std::vector<cplx<T>> random_batch(const Layout& L, unsigned seed) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<cplx<T>> v((size_t)L.len, mk<cplx<T>>((T)0, (T)0));
  for (auto& c : v) c = mk<cplx<T>>((T)u(g), (T)u(g));
  return v;
}

// ---- compile-time stages (ct_stage, as the xy and z kernels run them) ----

template <typename T, int N, int ST, int NT, class B>
void ct_fwd_stages(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST < ct_nst(N)) {
    all_threads(NT, [&] { ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), false, NT, B>(buf, tws); });
    ct_fwd_stages<T, N, ST + 1, NT, B>(buf, tws);
  }
}
// Inverse stages ST down to END + 1.
template <typename T, int N, int ST, int END, int NT, class B>
void ct_inv_stages(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST > END) {
    all_threads(NT, [&] { ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), true, NT, B>(buf, tws); });
    ct_inv_stages<T, N, ST - 1, END, NT, B>(buf, tws);
  }
}

template <int N>
std::vector<int> ct_plan() {
  std::vector<int> r;
  for (int st = 0; st < ct_nst(N); ++st) r.push_back(ct_radix(N, st));
  return r;
}

template <typename T, int N, int NT, int COUNT, int INNER, int ISTR, int OUTER, int ES>
void ct_case(const char* tag) {
  using B = BatchCT<COUNT, INNER, ISTR, OUTER, ES>;
  const Layout L{COUNT, INNER, ISTR, OUTER, ES,
                 (COUNT - 1) / INNER * OUTER + (COUNT - 1) % INNER * ISTR + (N - 1) * ES + 1};
  const std::vector<cplx<T>> tw = twiddle_table<T>(N);
  const std::vector<cplx<T>> in = random_batch<T>(L, 1000u + N);
  std::vector<cplx<T>> buf = in;
  ct_fwd_stages<T, N, 0, NT, B>(buf.data(), tw.data());
  const std::vector<cplx<T>> fwd = buf;
  ct_inv_stages<T, N, ct_nst(N) - 1, -1, NT, B>(buf.data(), tw.data());
  const std::string name = std::string("ct_") + (sizeof(T) == 4 ? "f32_" : "f64_") + tag + "_n" + std::to_string(N);
  check<T>(name.c_str(), N, ct_plan<N>(), L, in, fwd, buf);
}

// First stage read through ld() from a separate source array and last
// inverse stage written through st() (ct_stage_io, the fused global loads
// and stores of the kernels), the other stages in place.
template <typename T, int N, int NT, int COUNT, bool JFAST>
void ct_io_case() {
  constexpr int P = N + 1;  // row pitch of the shared-memory copy
  using B = BatchCT<COUNT, 1, 0, P, 1>;
  const Layout Lg{COUNT, 1, 0, N, 1, COUNT * N};  // the source: contiguous rows
  const Layout Ls{COUNT, 1, 0, P, 1, COUNT * P};
  const std::vector<cplx<T>> tw = twiddle_table<T>(N);
  const std::vector<cplx<T>> src = random_batch<T>(Lg, 2000u + N);
  std::vector<cplx<T>> buf((size_t)Ls.len, mk<cplx<T>>((T)0, (T)0)), out((size_t)Lg.len, mk<cplx<T>>((T)0, (T)0));
  auto ld = [&](int t, int e) { return src[(size_t)(t * N + e)]; };
  auto st = [&](int t, int e, const cplx<T>& v) { buf[(size_t)(t * P + e)] = v; };
  all_threads(NT, [&] { ct_stage_io<T, N, 0, false, NT, COUNT, JFAST>(ld, st, tw.data()); });
  ct_fwd_stages<T, N, 1, NT, B>(buf.data(), tw.data());
  std::vector<cplx<T>> fwd((size_t)Lg.len);
  for (int t = 0; t < COUNT; ++t)
    for (int e = 0; e < N; ++e) fwd[(size_t)(t * N + e)] = buf[(size_t)(t * P + e)];
  ct_inv_stages<T, N, ct_nst(N) - 1, 0, NT, B>(buf.data(), tw.data());  // stages down to 1 in place
  auto ld2 = [&](int t, int e) { return buf[(size_t)(t * P + e)]; };
  auto st2 = [&](int t, int e, const cplx<T>& v) { out[(size_t)(t * N + e)] = v; };
  all_threads(NT, [&] { ct_stage_io<T, N, 0, true, NT, COUNT, JFAST>(ld2, st2, tw.data()); });
  const std::string name = std::string("io_") + (sizeof(T) == 4 ? "f32_" : "f64_") + (JFAST ? "jfast" : "tfast") +
                           "_n" + std::to_string(N);
  check<T>(name.c_str(), N, ct_plan<N>(), Lg, src, fwd, out);
}

// ---- runtime-plan stages (fft_stage, any lengths of radices 2-5, 8, 16) ----

template <typename T>
void rt_stage(int R, bool inv, cplx<T>* buf, const Batch& B, int n, int Ls, const cplx<T>* tw, int len) {
  all_threads((int)blockDim.x, [&] {
    if (inv) fft_stage_rt<T, true>(R, buf, B, n, Ls, tw, len);
    else fft_stage_rt<T, false>(R, buf, B, n, Ls, tw, len);
  });
}

// radices of n, largest first (desc) or smallest first
std::vector<int> rt_plan(int n, bool desc) {
  static const int rs[] = {16, 8, 5, 4, 3, 2};
  std::vector<int> r;
  for (int k : rs)
    while (n % k == 0 && (k != 16 || n >= 16)) {
      r.push_back(k);
      n /= k;
    }
  if (!desc) std::reverse(r.begin(), r.end());
  return n == 1 ? r : std::vector<int>();
}

template <typename T>
void rt_case(int n, bool desc, bool tfast, int nt) {
  const std::vector<int> r = rt_plan(n, desc);
  if (r.empty()) return;
  const int count = 7;
  // tfast: transforms interleaved (element stride count + 1); else rows
  const Layout L = tfast ? Layout{count, count, 1, 0, count + 1, (n - 1) * (count + 1) + count}
                         : Layout{count, 1, 0, n + 3, 1, (count - 1) * (n + 3) + n};
  const Batch B{count, L.inner, L.istr, L.outer, L.es, tfast};
  const std::vector<cplx<T>> tw = twiddle_table<T>(n);
  const std::vector<cplx<T>> in = random_batch<T>(L, 3000u + (unsigned)n);
  std::vector<cplx<T>> buf = in;
  blockDim = dim3((unsigned)nt, 1, 1);
  int Ls = n;
  for (int R : r) {
    rt_stage<T>(R, false, buf.data(), B, n, Ls, tw.data(), L.len);
    Ls /= R;
  }
  const std::vector<cplx<T>> fwd = buf;
  Ls = 1;
  for (int st = (int)r.size() - 1; st >= 0; --st) {
    Ls *= r[(size_t)st];
    rt_stage<T>(r[(size_t)st], true, buf.data(), B, n, Ls, tw.data(), L.len);
  }
  std::string name = std::string("rt_") + (sizeof(T) == 4 ? "f32_" : "f64_") + (tfast ? "tfast_" : "rows_") +
                     (desc ? "desc" : "asc") + "_n" + std::to_string(n);
  check<T>(name.c_str(), n, r, L, in, fwd, buf);
}

template <typename T>
void all_cases() {
  // compile-time lengths: rows (the xy kernels' x pass: LY rows of MC + 1
  // pitch) and interleaved columns (the y pass and the z tiles)
  ct_case<T, 4, 512, 8, 1, 0, 5, 1>("rows");
  ct_case<T, 8, 512, 16, 1, 0, 9, 1>("rows");
  ct_case<T, 16, 512, 16, 1, 0, 17, 1>("rows");
  ct_case<T, 32, 512, 32, 1, 0, 33, 1>("rows");
  ct_case<T, 64, 512, 128, 1, 0, 65, 1>("rows");
  ct_case<T, 128, 512, 64, 1, 0, 129, 1>("rows");
  ct_case<T, 256, 512, 16, 1, 0, 257, 1>("rows");
  ct_case<T, 512, 256, 8, 1, 0, 513, 1>("rows");
  ct_case<T, 12, 512, 24, 1, 0, 13, 1>("rows");
  ct_case<T, 24, 512, 12, 1, 0, 25, 1>("rows");
  ct_case<T, 48, 512, 24, 1, 0, 49, 1>("rows");
  ct_case<T, 16, 512, 8, 8, 1, 0, 9>("cols");
  ct_case<T, 32, 512, 16, 16, 1, 0, 17>("cols");
  ct_case<T, 64, 256, 32, 32, 1, 0, 33>("cols");
  ct_case<T, 128, 512, 64, 64, 1, 0, 65>("cols");
  ct_case<T, 128, 256, 72, 8, 1, 128 * 8 + 8, 8>("ztile");  // 9 components x 8 columns, padded component stride
  ct_case<T, 24, 512, 12, 12, 1, 0, 13>("cols");
  ct_case<T, 48, 256, 24, 24, 1, 0, 25>("cols");
  ct_io_case<T, 64, 512, 128, true>();
  ct_io_case<T, 128, 512, 64, false>();
  ct_io_case<T, 24, 512, 12, true>();
  ct_io_case<T, 48, 512, 24, false>();
  for (int n : {6, 10, 12, 15, 20, 24, 30, 36, 40, 45, 48, 50, 60, 72, 80, 96, 100, 120, 160, 240})
    for (bool desc : {true, false})
      for (bool tfast : {true, false}) rt_case<T>(n, desc, tfast, 128);
}

int main() {
  all_cases<double>();
  all_cases<float>();
  return 0;
}
