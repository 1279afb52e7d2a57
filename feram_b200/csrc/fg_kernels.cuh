// fg_kernels.cuh -- device kernels of one feram MD step on B200.
//
// Device layout (chosen for the GPU, converted at the C-ABI boundary):
//   real fields  u, p, F, work : [comp][z][y][x]            (x contiguous)
//   spectra      spec          : [comp][z][ky_slot][kx_slot], row pitch KXP
//   k tables     dtab, ckmod   : [ky_slot][kz_slot][kx_slot][entries]
// Slots are the digit-reversed positions left by the in-place DIF FFT
// stages (fft_smem.cuh); rev{x,y,z} give the true wavenumber of a slot.
//
// One force evaluation (mirror_force_mirror.F:6-89) is four passes:
//   k_xy_fwd     per (z-plane, component): r2c along x + DIF along y of
//                u and u (x) u (dipoFFT.F:19-44) -> spec
//   k_z_kspace   per (kx tile, ky): DIF along z, every k-space operation
//                (dipole-dipole multiply, inhomogeneous strain solve,
//                energies), DIT along z
//   k_xy_inv     per (z-plane, component): DIT along y + c2r along x
//   k_assemble   per site: dipole-dipole + anharmonic + field + homogeneous
//                and inhomogeneous strain coupling forces
#pragma once
#include "fft_smem.cuh"

namespace fg {

// energy slots, fg_energy member order (energy_module.F:7-23)
enum {
  E_ACOU = 0, E_DIPO, E_SHORT, E_LONG, E_DIPE, E_UNH, E_HS, E_HC, E_IS, E_IC, E_IM, E_TOT, E_HNP, E_COUNT
};
constexpr int NQ_K = 5;   // k-space partial sums per block
constexpr int NQ_R = 2;   // real-space partial sums per block
constexpr int RED_THREADS = 256;

struct Geom {
  int Lx, Ly, Lz, m, NKX, KXP;
  long long plane_r;  // Lx*Ly
  long long plane_c;  // Ly*KXP
  long long nsite;    // Lx*Ly*Lz
  long long ncplx;    // Lz*Ly*KXP
  long long nkpos;    // Ly*Lz*KXP
};

// Constants of the Hamiltonian and integrators, resident on the device.
struct Phys {
  double N, Ninv;
  double j[7], kap2x2;                       // short range (dipole-dipole-short-range.F)
  double P_alpha, P_gamma, P_k1, P_k2, P_k3, P_k4;
  double fa2g, tg, sk, tk2, fk;              // dVddi-unharmonic.F:28-32
  double B11, B12, B44;
  double HC2[6][6];                          // homogeneous_coupling_2 (elastic.F:60-75)
  double H[6][6], HG[6][6], HG_inv[6];       // homogeneous, Cholesky (elastic.F:26-52)
  double pNa03[3], epi_strain;
  int bulk_or_film;
  double Zstar;
  double dt, dt_2, Q, nf_kT, threeN_kT;
  double Qinv;       // 1 / Q
  double ke_scale;   // N / (2 n_sum_p): kinetic energy per masked sum p^2/m
  double target_ke;  // target_kinetic_energy (param_module.F:468), velocity scaling
  // per-species on-site constants for .relaxor runs (dVddi-unharmonic.F:
  // 28-32,40,73): force combinations, energy coefficients, kappa2(s)-kappa2(1)
  struct Species {
    double fa2g, tg, sk, tk2, fk, k4x8, Pa, Pg, P1, P2, P3, P4, dk2;
  } sp[3];
  double n_sum_p;
  int E_on;
  int modulation_on;
  // per-step field of molecular-dynamics.F:66-76 evaluated on the device
  // (fg_set_wave): wave(E_wave_type, i_step, n_thermalize, n_E_wave_period,
  // external_E_field) of wave_module.F:8-67
  int wave_type, wave_n_thermalize, wave_period, wave_pad;
  double wave_amp[3];
};

struct DevScalars {
  double s, pi, H0, s_old;
  double kick_coef;   // p <- p - kick_coef * F
  double drift_coef;  // u <- u + drift_coef * p * m^-1
  double lf_dt, lf_dt_2;
  double e[E_COUNT];
  double strain[6];
  double w_hom[6];    // sum_i strain_i * HC2(i, j)
  double didiK0[6];   // Re didiK(k = 0)
  double E[3];        // uniform external field
  double ke_sum;      // last masked sum p^2/m
  // Nose-Poincare half step (35a), (38), (35c) of the next step, prepared by
  // the closing tail of the previous one (or by np_prepare) and committed by
  // block 0 of the next closing kick: masked sum p^2/m and KE at the half
  // step, pi_{n+1/2}, s_{n+1}, the drift coefficient and the (35f) kick
  // coefficient dt/2 s_{n+1}.
  double pend_ke_sum, pend_ke, pend_pi, pend_s, pend_drift, pend_kick_f;
  double vs_scale;       // velocity scaling factor of the last vs step
  double vs_scale_acou;  // the same for the acoustic momenta
  long long i_step;      // step counter of the device-side field schedule
  int status;
  int pad;
};

// Per-replica buffers of a grouped launch: replicas of one supercell size,
// precision and material (the points of a sweep) stepped by one launch per
// kernel, the replica index being the grid's last dimension.  Each kernel
// that takes a RepArgs table replaces its per-replica pointer arguments by
// its replica's entry; null = a launch for one context.
struct RepArgs {
  void* u;
  void* p;
  void* F;
  void* spec;
  void* rwork;
  const void* dtab;
  const Phys* ph;
  DevScalars* sc;
  double* part_k;
  double* part_r;
  double* part_ke;
  unsigned int* done_as;  // k_assemble's last-block ticket
  const double* layer_minv;
  const unsigned char* layer_sump;
};

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NQ values; thread 0 writes part[blockid*NQ + q].
// Fixed reduction order, so results are reproducible run to run.
template <int NQ>
__device__ void block_partials(double* v, double* part, long long blockid) {
  __shared__ double red[32][NQ];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double s = warp_sum(v[q]);
    if (lane == 0) red[wid][q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int q = 0; q < NQ; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[w][q];
      part[blockid * NQ + q] = s;
    }
  }
  __syncthreads();
}

// Sum of part[b*NQ + q] over b in fixed order by one RED_THREADS block.
__device__ double reduce_partials(const double* part, int nblk, int NQ, int q) {
  __shared__ double red[RED_THREADS];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += __ldcg(&part[(long long)b * NQ + q]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

// The same sums for all NQ columns in one pass: each thread adds its
// blocks in a fixed order, warps combine with shuffles, warps in order.
// Every thread receives the NQ totals.
template <int NQ>
__device__ void reduce_partials_all(const double* __restrict__ part, int nblk, double (&out)[NQ]) {
  __shared__ double red[32][NQ];
  double s[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) s[q] = 0.0;
#pragma unroll 4
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) s[q] += __ldcg(&part[(long long)b * NQ + q]);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double t = warp_sum(s[q]);
    if (lane == 0) red[wid][q] = t;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w][q];
    out[q] = t;
  }
  __syncthreads();
}

// Scalar work of a tail: thread 0 runs body on shared-memory copies of the
// constants and scalars, loaded and stored back by the whole block in one
// round trip each (instead of a chain of dependent global loads and stores
// by one thread).
static_assert(sizeof(DevScalars) % 8 == 0, "DevScalars is copied as doubles");
static_assert(sizeof(Phys) % 8 == 0, "Phys is copied as doubles");
template <class F>
__device__ __forceinline__ void scalar_tail(const Phys* __restrict__ ph, DevScalars* sc, F&& body) {
  __shared__ Phys sph;
  __shared__ DevScalars ssc;
  constexpr int NP = (int)(sizeof(Phys) / 8), NS = (int)(sizeof(DevScalars) / 8);
  for (int i = threadIdx.x; i < NP; i += blockDim.x)
    reinterpret_cast<double*>(&sph)[i] = __ldg(reinterpret_cast<const double*>(ph) + i);
  for (int i = threadIdx.x; i < NS; i += blockDim.x)
    reinterpret_cast<double*>(&ssc)[i] = __ldcg(reinterpret_cast<const double*>(sc) + i);
  __syncthreads();
  if (threadIdx.x == 0) body(static_cast<const Phys*>(&sph), &ssc);
  __syncthreads();
  for (int i = threadIdx.x; i < NS; i += blockDim.x)
    reinterpret_cast<double*>(sc)[i] = reinterpret_cast<const double*>(&ssc)[i];
}

// Last-block-done: thread 0 of every block fences the block's partials and
// takes a ticket; the block drawing the last ticket sees all of them and
// finishes the grid-wide work (classic threadfence reduction, no waiting).
// The counter is reset for the next launch by that block.  Only thread 0
// fences: the tails read nothing but the partials thread 0 wrote (and values
// whose writers fence themselves), so the other threads retire without
// waiting for their bulk stores to drain.
__device__ __forceinline__ bool is_last_block(unsigned int* counter) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
    if (last) *counter = 0u;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// ------------------------------------------------------- analytic short range
// S(k) of the 27-point stencil of dipole-dipole-short-range.F:35-83 (2 kappa2
// on site, j1..j7 on the first three neighbour shells), evaluated from the
// cosines and sines of theta_a = 2 pi k_a / L_a.  Valid for L_a >= 3.
// Order: xx, yy, zz, yz, zx, xy.
__host__ __device__ inline void short_range_k(const double* j, double kap2x2, const double c[3], const double s[3],
                                              double S[6]) {
  for (int a = 0; a < 3; ++a) {
    const int b = (a + 1) % 3, g = (a + 2) % 3;
    S[a] = kap2x2 + 2 * j[1] * c[a] + 2 * j[0] * (c[b] + c[g]) + 4 * j[3] * c[b] * c[g] +
           4 * j[2] * c[a] * (c[b] + c[g]) + 8 * j[5] * c[0] * c[1] * c[2];
  }
  // off-diagonal (a, b) with third axis g: -4 j5 s_a s_b - 8 j7 s_a s_b c_g
  S[3] = -4 * j[4] * s[1] * s[2] - 8 * j[6] * s[1] * s[2] * c[0];  // yz
  S[4] = -4 * j[4] * s[2] * s[0] - 8 * j[6] * s[2] * s[0] * c[1];  // zx
  S[5] = -4 * j[4] * s[0] * s[1] - 8 * j[6] * s[0] * s[1] * c[2];  // xy
}

__device__ __noinline__ void homo_strain_tail(const Phys* __restrict__ ph, DevScalars* sc,
                                              const double* __restrict__ part_k, int nblk);

// ------------------------------------------------------------------ k_xy_fwd
enum { SRC_U9 = 0, SRC_FIELD = 1 };

// Per (z-plane, component): load a real plane, DIF along x on Lx/2 complex
// pairs, unpack to the Lx/2+1 bins of the real transform, DIF along y.
// SRC_U9: component c of (u_x, u_y, u_z, u_x^2, u_y^2, u_z^2, u_y u_z,
// u_z u_x, u_x u_y) from u (dipoFFT.F:19-44); components 9..11 are src
// components 3..5 (the acoustic displacement stored after u); with a per-site
// Z* (zstar != null) components zu0..zu0+2 are Z*(R) u (Z_u_R, dipoFFT.F:
// 36-44).  SRC_FIELD: component c of src.
// MC, LYC > 0 select the compile-time transforms for m = Lx/2 = MC and
// Ly = LYC (launched with exactly kXYThreads threads); 0 = runtime plans.
// The compile-time kernels run the y transforms on MC columns, not MC + 1:
// the kx = 0 and kx = Lx/2 columns are real before the y pass (transforms of
// real rows), so X(0) + i X(Lx/2) travels as one complex column and is split
// by Hermitian symmetry after the pass (y_split); the inverse joins them the
// same way before its y pass (y_join).  posm + m and posm + m + Ly hold the
// y slot maps (slot -> ky, ky -> slot) that pair ky with -ky.
constexpr int kXYThreads = 512;

// Column kx = 0 after the forward y pass holds C = Y0 + i Ym, Y0 and Ym the
// y spectra of the real kx = 0 and kx = Lx/2 columns: Y0(k) = (C(k) +
// conj C(-k)) / 2, Ym(k) = (C(k) - conj C(-k)) / 2i.  a = C(k), b = C(-k).
template <typename C>
__device__ __forceinline__ void y_split(C a, C b, C& y0, C& ym) {
  using R = decltype(a.x);
  y0 = mk<C>((R)0.5 * (a.x + b.x), (R)0.5 * (a.y - b.y));
  ym = mk<C>((R)0.5 * (a.y + b.y), (R)0.5 * (b.x - a.x));
}
// Inverse: C(k) = H0(k) + i Hm(k) with H(k) = (Y(k) + conj Y(-k)) / 2, the
// Hermitian part, whose inverse transform is the real part of Y's (the
// imaginary parts of the kx = 0 and kx = Lx/2 bins are dropped, as FFTW's
// c2r does).  a0 = Y0(k), b0 = Y0(-k), am = Ym(k), bm = Ym(-k).
template <typename C>
__device__ __forceinline__ C y_join(C a0, C b0, C am, C bm) {
  using R = decltype(a0.x);
  const R h0x = (R)0.5 * (a0.x + b0.x), h0y = (R)0.5 * (a0.y - b0.y);
  const R hmx = (R)0.5 * (am.x + bm.x), hmy = (R)0.5 * (am.y - bm.y);
  return mk<C>(h0x - hmy, h0y + hmx);
}

template <typename T, int MC, int LYC>
__device__ __forceinline__ void xy_twiddles_to_smem(cplx<T>* tm, cplx<T>* ty, cplx<T>* tx, const cplx<T>* twm,
                                                    const cplx<T>* twy, const cplx<T>* twx) {
  if constexpr (MC > 0) {
    for (int i = threadIdx.x; i < MC; i += blockDim.x) tm[i] = twm[i];
    for (int i = threadIdx.x; i < LYC; i += blockDim.x) ty[i] = twy[i];
    for (int i = threadIdx.x; i <= MC; i += blockDim.x) tx[i] = twx[i];
  }
}

template <typename T, int MODE, int MC = 0, int LYC = 0>
__global__ void __launch_bounds__(512, sizeof(T) == 4 ? 2 : 1) k_xy_fwd(const T* __restrict__ src, cplx<T>* __restrict__ spec, Geom g,
                                                FftPlan px, FftPlan py, const cplx<T>* __restrict__ twx,
                                                const cplx<T>* __restrict__ twm, const cplx<T>* __restrict__ twy,
                                                const int* __restrict__ posm, int out_comp0,
                                                const T* __restrict__ zstar = nullptr, int zu0 = 0,
                                                const RepArgs* __restrict__ grp = nullptr) {
  pdl_enter();
  if (grp) {
    src = (const T*)grp[blockIdx.z].u;
    spec = (cplx<T>*)grp[blockIdx.z].spec;
  }
  FG_DYN_SMEM(smem_raw);
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  __shared__ cplx<T> tws_m[MC > 0 ? MC : 1], tws_y[LYC > 0 ? LYC : 1], tws_x[MC > 0 ? MC + 1 : 1];
  using T2 = typename RT2<T>::type;
  const int z = blockIdx.x, c = blockIdx.y;
  const int m = MC > 0 ? MC : g.m, Ly = LYC > 0 ? LYC : g.Ly;
  const int RS = m + 1, Lx = 2 * m;
  const int buf_len = Ly * RS;
  xy_twiddles_to_smem<T, MC, LYC>(tws_m, tws_y, tws_x, twm, twy, twx);
  const cplx<T>* twx_u = MC > 0 ? tws_x : twx;
  const long long plane_off = (long long)z * g.plane_r;
  const int total = Ly * m;
  const bool zu = MODE == SRC_U9 && zstar != nullptr && c >= zu0;  // Z*(R) u_(c - zu0)
  if constexpr (MC > 0) {
    // First x stage straight from the real rows (packed (x even, x odd)
    // pairs, products formed on load), then the rest of the x pass.
    const bool plain = !zu && (MODE == SRC_FIELD || c < 3 || c >= 9);
    const int ca = zu ? c - zu0
                      : plain ? (c >= 9 && MODE == SRC_U9 ? c - 6 : c) : (c == 3 || c == 8) ? 0 : (c == 4 || c == 6) ? 1 : 2;
    const int cb = plain || zu ? -1 : (c == 3) ? 0 : (c == 4) ? 1 : (c == 5) ? 2 : (c == 6) ? 2 : (c == 7) ? 0 : 1;
    const T* pa = src + (long long)ca * g.nsite + plane_off;
    const T* pb = zu ? zstar + plane_off : src + (long long)(cb < 0 ? ca : cb) * g.nsite + plane_off;
    auto st = [&](int y, int e, const cplx<T>& v) { buf[y * (MC + 1) + e] = v; };
    if (plain) {
      auto ld = [&](int y, int e) {
        const T2 a = *reinterpret_cast<const T2*>(pa + (long long)y * (2 * MC) + 2 * e);
        return mk<cplx<T>>(a.x, a.y);
      };
      ct_stage_io<T, MC, 0, false, kXYThreads, LYC, true>(ld, st, twm);
    } else {
      auto ld = [&](int y, int e) {
        const long long o = (long long)y * (2 * MC) + 2 * e;
        const T2 a = *reinterpret_cast<const T2*>(pa + o), b = *reinterpret_cast<const T2*>(pb + o);
        return mk<cplx<T>>(a.x * b.x, a.y * b.y);
      };
      ct_stage_io<T, MC, 0, false, kXYThreads, LYC, true>(ld, st, twm);
    }
    __syncthreads();
    ct_forward_range<T, MC, 1, ct_nst(MC), kXYThreads, BatchCT<LYC, 1, 0, MC + 1, 1>>(buf, tws_m);
  } else if (!zu && (MODE == SRC_FIELD || c < 3 || c >= 9)) {
    // plain component: asynchronous copies of packed (x even, x odd) pairs
    const T* sp = src + (long long)(c >= 9 && MODE == SRC_U9 ? c - 6 : c) * g.nsite + plane_off;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int y = idx / m, jx = idx - y * m;
      cp_async<(int)sizeof(cplx<T>)>(&buf[y * RS + jx], sp + (long long)y * Lx + 2 * jx);
    }
    cp_async_wait();
  } else {
    // products: kLB independent loads in flight per thread, then compute
    constexpr int kLB = 4;
    for (int base = threadIdx.x; base < total; base += kLB * blockDim.x) {
      T2 va[kLB], vb[kLB];
#pragma unroll
      for (int r = 0; r < kLB; ++r) {
        const int idx = base + r * blockDim.x;
        if (idx < total) {
          const int y = idx / m, jx = idx - y * m;
          const long long o = plane_off + (long long)y * Lx + 2 * jx;
          const int ca = zu ? c - zu0 : (c == 3 || c == 8) ? 0 : (c == 4 || c == 6) ? 1 : 2;
          const int cb = (c == 3) ? 0 : (c == 4) ? 1 : (c == 5) ? 2 : (c == 6) ? 2 : (c == 7) ? 0 : 1;
          va[r] = *reinterpret_cast<const T2*>(src + (long long)ca * g.nsite + o);
          vb[r] = *reinterpret_cast<const T2*>(zu ? zstar + o : src + (long long)cb * g.nsite + o);
        }
      }
#pragma unroll
      for (int r = 0; r < kLB; ++r) {
        const int idx = base + r * blockDim.x;
        if (idx < total) {
          const int y = idx / m, jx = idx - y * m;
          buf[y * RS + jx] = mk<cplx<T>>(va[r].x * vb[r].x, va[r].y * vb[r].y);
        }
      }
    }
  }
  // X pass; row stride RS = m+1 keeps the row-interleaved mapping bank-conflict free
  if constexpr (MC == 0) {
    __syncthreads();
    Batch B{Ly, 1, 0, RS, 1, true};
    fft_forward<T>(buf, B, px, twm, buf_len);
  }
  // unpack: slot posm[k] holds Z(k) of the packed row; X(k) = E(k) + w^k O(k)
  const int half = m / 2 + 1;
  // lanes run along y (same k): conflict-free rows, uniform posm and twiddle
  for (int idx = threadIdx.x; idx < Ly * half; idx += blockDim.x) {
    const int k = idx / Ly, y = idx - k * Ly;
    cplx<T>* row = buf + y * RS;
    if (k == 0) {
      const cplx<T> z0 = row[0];
      if constexpr (MC > 0) {
        row[0] = mk<cplx<T>>(z0.x + z0.y, z0.x - z0.y);  // X(0) + i X(m)
      } else {
        row[0] = mk<cplx<T>>(z0.x + z0.y, (T)0);
        row[m] = mk<cplx<T>>(z0.x - z0.y, (T)0);
      }
    } else {
      const int k2 = m - k;
      const int s1 = __ldg(&posm[k]), s2 = __ldg(&posm[k2]);
      const cplx<T> a = row[s1], b = row[s2];
      const cplx<T> w1 = twx_u[k], w2 = twx_u[k2];
      // X(k) = 1/2 (a + conj b) - i/2 w1 (a - conj b)
      const cplx<T> e1 = mk<cplx<T>>(a.x + b.x, a.y - b.y), d1 = mk<cplx<T>>(a.x - b.x, a.y + b.y);
      const cplx<T> wd1 = cmul(w1, d1);
      const cplx<T> X1 = mk<cplx<T>>((T)0.5 * (e1.x + wd1.y), (T)0.5 * (e1.y - wd1.x));
      const cplx<T> e2 = mk<cplx<T>>(b.x + a.x, b.y - a.y), d2 = mk<cplx<T>>(b.x - a.x, b.y + a.y);
      const cplx<T> wd2 = cmul(w2, d2);
      const cplx<T> X2 = mk<cplx<T>>((T)0.5 * (e2.x + wd2.y), (T)0.5 * (e2.y - wd2.x));
      row[s1] = X1;
      if (s2 != s1) row[s2] = X2;
    }
  }
  __syncthreads();
  cplx<T>* dst = spec + (long long)(out_comp0 + c) * g.ncplx + (long long)z * g.plane_c;
  if constexpr (MC > 0) {
    // y pass over the MC columns (kx = Lx/2 rides in column 0); its last
    // stage writes the spectrum rows directly, except column 0, which stays
    // in shared memory for the Hermitian split
    constexpr int NSY = ct_nst(LYC);
    ct_forward_range<T, LYC, 0, NSY - 1, kXYThreads, BatchCT<MC, MC, 1, 0, MC + 1>>(buf, tws_y);
    const long long kxp = g.KXP;
    auto ld = [&](int col, int e) { return buf[col + e * (MC + 1)]; };
    auto st = [&](int col, int e, const cplx<T>& v) {
      if (col == 0) buf[e * (MC + 1)] = v;
      else dst[(long long)e * kxp + col] = v;
    };
    ct_stage_io<T, LYC, NSY - 1, false, kXYThreads, MC, false>(ld, st, tws_y);
    __syncthreads();
    const int* revy = posm + MC;
    const int* posy = posm + MC + LYC;
    for (int sl = threadIdx.x; sl < LYC; sl += kXYThreads) {
      const int ky = __ldg(&revy[sl]);
      const int sp = __ldg(&posy[(LYC - ky) % LYC]);
      cplx<T> y0, ym;
      y_split(buf[sl * (MC + 1)], buf[sp * (MC + 1)], y0, ym);
      dst[(long long)sl * kxp] = y0;
      dst[(long long)sl * kxp + MC] = ym;
    }
  } else {
    Batch B{RS, RS, 1, 0, RS, true};
    fft_forward<T>(buf, B, py, twy, buf_len);
    for (int idx = threadIdx.x; idx < Ly * RS; idx += blockDim.x) {
      const int y = idx / RS, col = idx - y * RS;
      dst[(long long)y * g.KXP + col] = buf[idx];
    }
  }
}

// ------------------------------------------------------------------ k_xy_inv
// Per (z-plane, component): DIT along y, repack the Lx/2+1 bins into Lx/2
// complex pairs (imaginary parts of the kx = 0 and kx = Lx/2 bins dropped,
// the half-complex convention of the reference's c2r), DIT along x, store
// the real plane.  Output is unnormalised (Lx*Ly*Lz times the IDFT).
template <typename T, int MC = 0, int LYC = 0>
__global__ void __launch_bounds__(512, sizeof(T) == 4 ? 2 : 1) k_xy_inv(const cplx<T>* __restrict__ spec, T* __restrict__ out, Geom g,
                                                FftPlan px, FftPlan py, const cplx<T>* __restrict__ twx,
                                                const cplx<T>* __restrict__ twm, const cplx<T>* __restrict__ twy,
                                                const int* __restrict__ posm, int in_comp0,
                                                const Phys* __restrict__ ph, DevScalars* sc,
                                                const double* __restrict__ part_k, int nblk_k,
                                                const RepArgs* __restrict__ grp = nullptr) {
  pdl_enter();
  if (grp) {
    const RepArgs& a = grp[blockIdx.z];
    spec = (const cplx<T>*)a.spec;
    out = (T*)a.rwork;
    if (ph != nullptr) ph = a.ph;
    sc = a.sc;
    part_k = a.part_k;
  }
  // Block (0, 0) first finishes the k-space pass that wrote spec: its
  // energies and the homogeneous strain, from k_z_kspace's block partials
  // (nothing in this kernel needs them; k_assemble does).
  if (ph != nullptr && blockIdx.x == 0 && blockIdx.y == 0) homo_strain_tail(ph, sc, part_k, nblk_k);
  FG_DYN_SMEM(smem_raw);
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  __shared__ cplx<T> tws_m[MC > 0 ? MC : 1], tws_y[LYC > 0 ? LYC : 1], tws_x[MC > 0 ? MC + 1 : 1];
  using T2 = typename RT2<T>::type;
  const int z = blockIdx.x, c = blockIdx.y;
  const int m = MC > 0 ? MC : g.m, Ly = LYC > 0 ? LYC : g.Ly;
  const int RS = m + 1, Lx = 2 * m;
  const int buf_len = Ly * RS;
  xy_twiddles_to_smem<T, MC, LYC>(tws_m, tws_y, tws_x, twm, twy, twx);
  const cplx<T>* twx_u = MC > 0 ? tws_x : twx;
  const cplx<T>* srcp = spec + (long long)(in_comp0 + c) * g.ncplx + (long long)z * g.plane_c;
  if constexpr (MC > 0) {
    // y pass; its first stage (the last forward one, no twiddles) reads the
    // spectrum rows directly
    constexpr int NSY = ct_nst(LYC);
    const long long kxp = g.KXP;
    // the spectrum is consumed here (evict_first)
    const unsigned long long pol = l2_evict_first();
    auto ld = [&](int col, int e) {
      const cplx<T>* a = srcp + (long long)e * kxp + col;
      if constexpr (sizeof(T) == 4) {
        const float2 v = ld_first(reinterpret_cast<const float2*>(a), pol);
        return mk<cplx<T>>(v.x, v.y);
      } else if constexpr (FG_L2_HINT_FP64) {
        const double2 v = ld_first(reinterpret_cast<const double2*>(a), pol);
        return mk<cplx<T>>(v.x, v.y);
      } else {
        return *a;
      }
    };
    // column 0 carries the kx = 0 and kx = Lx/2 columns joined (y_join),
    // formed by LYC threads into shared memory while all threads run the
    // first stage of columns 1 .. MC-1 straight from the spectrum (the join's
    // loads overlap that stage); column 0's first stage then runs on the
    // joined column in place
    const int* revy = posm + MC;
    const int* posy = posm + MC + LYC;
    for (int sl = threadIdx.x; sl < LYC; sl += kXYThreads) {
      const int sp = __ldg(&posy[(LYC - __ldg(&revy[sl])) % LYC]);
      buf[sl * (MC + 1)] = y_join(ld(0, sl), ld(0, sp), ld(MC, sl), ld(MC, sp));
    }
    auto st = [&](int col, int e, const cplx<T>& v) { buf[col + e * (MC + 1)] = v; };
    auto ld1 = [&](int t, int e) { return ld(t + 1, e); };
    auto st1 = [&](int t, int e, const cplx<T>& v) { st(t + 1, e, v); };
    ct_stage_io<T, LYC, NSY - 1, true, kXYThreads, MC - 1, false>(ld1, st1, tws_y);
    __syncthreads();
    auto ld0 = [&](int, int e) { return buf[e * (MC + 1)]; };
    auto st0 = [&](int, int e, const cplx<T>& v) { st(0, e, v); };
    ct_stage_io<T, LYC, NSY - 1, true, kXYThreads, 1, false>(ld0, st0, tws_y);
    __syncthreads();
    ct_inverse_range<T, LYC, NSY - 2, -1, kXYThreads, BatchCT<MC, MC, 1, 0, MC + 1>>(buf, tws_y);
  } else {
    for (int idx = threadIdx.x; idx < Ly * RS; idx += blockDim.x) {
      const int y = idx / RS, col = idx - y * RS;
      cp_async<(int)sizeof(cplx<T>)>(&buf[idx], srcp + (long long)y * g.KXP + col);
    }
    cp_async_wait();
    __syncthreads();
    Batch B{RS, RS, 1, 0, RS, true};
    fft_inverse<T>(buf, B, py, twy, buf_len);
  }
  const int half = m / 2 + 1;
  // lanes run along y (same k): conflict-free rows, uniform posm and twiddle
  for (int idx = threadIdx.x; idx < Ly * half; idx += blockDim.x) {
    const int k = idx / Ly, y = idx - k * Ly;
    cplx<T>* row = buf + y * RS;
    if (k == 0) {
      // compile-time kernels: x(kx = Lx/2) came back as the imaginary part
      const T X0 = row[0].x, Xm = MC > 0 ? row[0].y : row[m].x;
      row[0] = mk<cplx<T>>(X0 + Xm, X0 - Xm);
    } else {
      const int k2 = m - k;
      const int s1 = __ldg(&posm[k]), s2 = __ldg(&posm[k2]);
      const cplx<T> a = row[s1], b = row[s2];
      const cplx<T> w1 = twx_u[k], w2 = twx_u[k2];
      // Z(k) = (a + conj b) + i conj(w1) (a - conj b)
      const cplx<T> e1 = mk<cplx<T>>(a.x + b.x, a.y - b.y), d1 = mk<cplx<T>>(a.x - b.x, a.y + b.y);
      const cplx<T> wd1 = cmulc(d1, w1);
      const cplx<T> Z1 = mk<cplx<T>>(e1.x - wd1.y, e1.y + wd1.x);
      const cplx<T> e2 = mk<cplx<T>>(b.x + a.x, b.y - a.y), d2 = mk<cplx<T>>(b.x - a.x, b.y + a.y);
      const cplx<T> wd2 = cmulc(d2, w2);
      const cplx<T> Z2 = mk<cplx<T>>(e2.x - wd2.y, e2.y + wd2.x);
      row[s1] = Z1;
      if (s2 != s1) row[s2] = Z2;
    }
  }
  __syncthreads();
  T* dst = out + (long long)c * g.nsite + (long long)z * g.plane_r;
  if constexpr (MC > 0) {
    // x pass; its last stage (stage 0, DIT) writes the real rows directly
    ct_inverse_range<T, MC, ct_nst(MC) - 1, 0, kXYThreads, BatchCT<LYC, 1, 0, MC + 1, 1>>(buf, tws_m);
    auto ld = [&](int y, int e) { return buf[y * (MC + 1) + e]; };
    auto st = [&](int y, int e, const cplx<T>& v) {
      T2 w;
      w.x = v.x;
      w.y = v.y;
      *reinterpret_cast<T2*>(dst + (long long)y * (2 * MC) + 2 * e) = w;
    };
    ct_stage_io<T, MC, 0, true, kXYThreads, LYC, true>(ld, st, tws_m);
  } else {
    Batch B{Ly, 1, 0, RS, 1, true};
    fft_inverse<T>(buf, B, px, twm, buf_len);
    for (int idx = threadIdx.x; idx < Ly * m; idx += blockDim.x) {
      const int y = idx / m, jx = idx - y * m;
      const cplx<T> v = buf[y * RS + jx];
      T2 w;
      w.x = v.x;
      w.y = v.y;
      *reinterpret_cast<T2*>(dst + (long long)y * Lx + 2 * jx) = w;
    }
  }
}

// ------------------------------------------------- z tiles (shared helpers)
// A z tile is CW pencils (kx slot, ky slot) with all z, nc components, held
// in shared memory as buf[c][z][cw].  Blocks [0, nreg) take CW consecutive kx
// slots of one ky slot (CW divides Lx/2); blocks [nreg, nreg + nnyq) take
// the Nyquist slot kx = Lx/2 of CW consecutive ky slots.
struct ZTiles {
  int CW;
  int ntx;   // regular tiles per ky slot (= (Lx/2) / CW)
  int nreg;  // ntx * Ly
  int nnyq;  // ceil(Ly / CW)
};

// Blocks 0 .. nnyq-1 take the Nyquist tiles (kx = Lx/2 batched across ky,
// one uncoalesced 8-byte access per element), the rest the regular tiles:
// the slow tiles start first instead of trailing the grid.
__device__ __forceinline__ bool tile_pencil(const ZTiles& zt, const Geom& g, int cw, int* col, int* yslot) {
  const int b = blockIdx.x;
  if (b >= zt.nnyq) {
    const int r = b - zt.nnyq;
    *yslot = r / zt.ntx;
    *col = (r - *yslot * zt.ntx) * zt.CW + cw;
    return true;
  }
  *col = g.m;
  *yslot = b * zt.CW + cw;
  return *yslot < g.Ly;
}

// Threads own a fixed pencil cw = threadIdx.x % CW (blockDim is a multiple
// of CW) and walk the tile rows r = c * Lz + z, so the pencil decode runs
// once per thread and a row step is an add.  buf[r * CW + cw].
template <typename T, int LZC = 0, int CWC = 0>
__device__ __forceinline__ void z_tile_load(cplx<T>* buf, const cplx<T>* __restrict__ spec, const Geom& g,
                                            const ZTiles& zt, int nc) {
  const int Lz = LZC > 0 ? LZC : g.Lz, CW = CWC > 0 ? CWC : zt.CW;
  const int cw = threadIdx.x % CW, rstep = blockDim.x / CW;
  int col, yslot;
  const bool valid = tile_pencil(zt, g, cw, &col, &yslot);
  const cplx<T>* base = spec + (valid ? (long long)yslot * g.KXP + col : 0);
  for (int r = threadIdx.x / CW; r < nc * Lz; r += rstep) {
    const int c = r / Lz, z = r - c * Lz;
    cplx<T>* dst = &buf[r * CW + cw];
    if (valid) cp_async<(int)sizeof(cplx<T>)>(dst, base + (long long)c * g.ncplx + (long long)z * g.plane_c);
    else *dst = mk<cplx<T>>((T)0, (T)0);
  }
  cp_async_wait();
  __syncthreads();
}

template <typename T, int LZC = 0, int CWC = 0>
__device__ __forceinline__ void z_tile_store(const cplx<T>* buf, cplx<T>* __restrict__ spec, const Geom& g,
                                             const ZTiles& zt, int nc) {
  const int Lz = LZC > 0 ? LZC : g.Lz, CW = CWC > 0 ? CWC : zt.CW;
  const int cw = threadIdx.x % CW, rstep = blockDim.x / CW;
  int col, yslot;
  if (!tile_pencil(zt, g, cw, &col, &yslot)) return;
  cplx<T>* base = spec + (long long)yslot * g.KXP + col;
  for (int r = threadIdx.x / CW; r < nc * Lz; r += rstep) {
    const int c = r / Lz, z = r - c * Lz;
    base[(long long)c * g.ncplx + (long long)z * g.plane_c] = buf[r * CW + cw];
  }
}

// ------------------------------------------------------------ scalar kernels
// Grid-wide scalar steps; each runs either as a single-block kernel or in the
// last block of the kernel whose partial sums it reduces (tail).
enum { TAIL_NONE = 0, TAIL_ENERGIES = 1, TAIL_LF_FINAL = 3, TAIL_VS = 4, TAIL_ACOU = 5, TAIL_VS_ACOU = 6 };

__device__ __forceinline__ double sum_potential(const double* e) {
  return e[E_SHORT] + e[E_LONG] + e[E_DIPE] + e[E_UNH] + e[E_HS] + e[E_HC] + e[E_IS] + e[E_IC] + e[E_IM];
}

// energy_module.F:128-148 with 1/s^2 and log(s) of the current s given
__device__ __forceinline__ void np_hamiltonian(const Phys* ph, DevScalars* sc, double inv_s2, double log_s) {
  double* e = sc->e;
  double h = e[E_DIPO] * inv_s2 + sum_potential(e) + sc->pi * sc->pi * 0.5 * ph->Qinv + ph->threeN_kT * log_s - sc->H0;
  e[E_HNP] = h * sc->s;
}
__device__ __forceinline__ void np_hamiltonian(const Phys* ph, DevScalars* sc) {
  const double inv_s = 1.0 / sc->s;
  np_hamiltonian(ph, sc, inv_s * inv_s, log(sc->s));
}

__device__ __forceinline__ void check_finite(DevScalars* sc, const double* v, int n) {
  for (int i = 0; i < n; ++i)
    if (!isfinite(v[i])) sc->status = 3;  // FG_ERR_NAN
}

// After the k-space pass: k-space energies, homogeneous strain
// (optimize-homo-strain.F:27-186) and w_hom for k_assemble.
__device__ __noinline__ void homo_strain_tail(const Phys* __restrict__ ph, DevScalars* sc,
                                              const double* __restrict__ part_k, int nblk) {
  double v[NQ_K];
  reduce_partials_all<NQ_K>(part_k, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    double* e = S->e;
    const double es = v[0] * P->Ninv / 2;  // (1/2N) sum w' Re(uK* S uK)
    const double edd = v[1] / 2;           // (1/2)  sum w' Re(uK* D uK), D = (S + Z*^2 L)/N
    e[E_SHORT] = es;
    e[E_LONG] = edd - es;
    e[E_IS] = v[2] * P->Ninv;
    e[E_IC] = v[3] * 2 * P->Ninv;
    e[E_IM] = P->modulation_on ? v[4] * 2 * P->Ninv : 0.0;
    double hc2uu[6];
    for (int i = 0; i < 6; ++i) {
      double t = 0.0;
      for (int jj = 0; jj < 6; ++jj) t += P->HC2[i][jj] * S->didiK0[jj];
      hc2uu[i] = t;
    }
    for (int i = 0; i < 3; ++i) hc2uu[i] = hc2uu[i] + P->pNa03[i];
    double* st = S->strain;
    const double(*H)[6] = P->H;
    if (P->bulk_or_film == 2) {  // epit
      st[0] = P->epi_strain;
      st[1] = P->epi_strain;
      st[2] = (-(H[2][0] + H[2][1]) * P->epi_strain - hc2uu[2]) / H[2][2];
      st[3] = -hc2uu[3] / H[3][3];
      st[4] = -hc2uu[4] / H[4][4];
      st[5] = 0.0;
    } else if (P->bulk_or_film == 3) {  // e110
      st[2] = P->epi_strain;
      st[3] = 0.0;
      st[4] = 0.0;
      double num = -(H[0][0] + H[1][1] + 2 * H[1][1]) * P->epi_strain - (H[2][0] + H[2][1]) * st[2] - hc2uu[0] -
                   hc2uu[1] + 2 * hc2uu[5];
      double den = H[0][0] + H[1][1] + 2 * H[1][0] + 4 * H[5][5];
      double delta = num / den;
      st[0] = P->epi_strain + delta;
      st[1] = P->epi_strain + delta;
      st[5] = -2 * delta;
    } else {
      for (int i = 0; i < 6; ++i) st[i] = -hc2uu[i];
      for (int i = 0; i < 6; ++i) {
        double t = 0.0;
        for (int jj = 0; jj < i; ++jj) t = t + P->HG[i][jj] * st[jj];
        st[i] = (st[i] - t) * P->HG_inv[i];
      }
      for (int i = 5; i >= 0; --i) {
        double t = 0.0;
        for (int jj = i + 1; jj < 6; ++jj) t = t + st[jj] * P->HG[jj][i];
        st[i] = (st[i] - t) * P->HG_inv[i];
      }
    }
    double hs = 0.0;
    for (int i = 0; i < 6; ++i) {
      double d = 0.0;
      for (int jj = 0; jj < 6; ++jj) d += H[i][jj] * st[jj];
      hs = hs + st[i] * d;
    }
    e[E_HS] = hs / 2;
    double hc = 0.0;
    for (int i = 0; i < 6; ++i) hc += st[i] * hc2uu[i];
    e[E_HC] = hc;
    for (int jj = 0; jj < 6; ++jj) {
      double w = 0.0;
      for (int i = 0; i < 6; ++i) w = w + st[i] * P->HC2[i][jj];
      S->w_hom[jj] = w;
    }
  });
}

// kinetic_energy_dipo.F:106 from the kick partials
__device__ __forceinline__ double ke_from(const Phys* ph, double sum) { return sum * ph->ke_scale; }

// Nose-Poincare after the force (nose-poincare.F:60-66): H_NP, (35e).
// Thread 0 only.
__device__ void np_post_body(const Phys* __restrict__ ph, DevScalars* sc) {
  const double inv_s = 1.0 / sc->s, inv_s2 = inv_s * inv_s;
  np_hamiltonian(ph, sc, inv_s2, log(sc->s));
  const double delta_H = sc->e[E_HNP] * inv_s;
  sc->pi = sc->pi + ph->dt_2 * (2 * sc->e[E_DIPO] * inv_s2 - ph->nf_kT) - ph->dt_2 * delta_H;
}

// After k_assemble: real-space energies.  With np_close also the commit of
// the prepared half step ((38), (35c): s, pi, KE at the half step) and the
// (35e) update of pi, as the closing kick of a Nose-Poincare step needs.
__device__ __noinline__ void force_energies_tail(const Phys* __restrict__ ph, DevScalars* sc,
                                                 const double* __restrict__ part_r, int nblk, bool np_close) {
  double v[NQ_R];
  reduce_partials_all<NQ_R>(part_r, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    S->e[E_UNH] = v[0];
    S->e[E_DIPE] = P->E_on ? -v[1] : 0.0;
    check_finite(S, S->e + E_SHORT, 9);
    if (np_close) {
      S->s_old = S->s;
      S->s = S->pend_s;
      S->pi = S->pend_pi;
      S->ke_sum = S->pend_ke_sum;
      S->e[E_DIPO] = S->pend_ke;
      S->drift_coef = S->pend_drift;
      np_post_body(P, S);
    }
  });
}

// Closing tail of a Nose-Poincare step.  part holds per block the masked
// sums of p^2/m, p.F/m and F^2/m after the closing kick (35f).
//  - step_done: KE, H_NP and total of the finished step (nose-poincare.F:
//    74-75, molecular-dynamics.F:293);
//  - always: the first half of the next step (nose-poincare.F:24-41) as far
//    as it is scalar: its kick (35a) p - c F with c = dt/2 s has the kinetic
//    sum  sum p^2/m - 2 c sum p.F/m + c^2 sum F^2/m,  which gives (38) pi,
//    s_{n+1} and the drift coefficient of (35c) before any site is touched.
//    They are kept pending (s and pi still report the finished step).
__device__ __noinline__ void np_close_tail(const Phys* __restrict__ ph, DevScalars* sc,
                                           const double* __restrict__ part, int nblk, bool step_done) {
  double v[3];
  reduce_partials_all<3>(part, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    // one thread's serial FP64 chain: one log, four divisions, one sqrt
    const double s = S->s;
    const double inv_s = 1.0 / s, inv_s2 = inv_s * inv_s, log_s = log(s);
    const double epot = sum_potential(S->e);
    if (step_done) {
      S->ke_sum = v[0];
      S->e[E_DIPO] = ke_from(P, v[0]);
      np_hamiltonian(P, S, inv_s2, log_s);
      S->e[E_TOT] = S->e[E_DIPO] * inv_s2 + S->e[E_ACOU] + epot;
      check_finite(S, S->e, E_COUNT);
    }
    const double ca = P->dt_2 * s;
    const double kh = v[0] - 2 * ca * v[1] + ca * ca * v[2];
    const double ke = ke_from(P, kh);
    double CB = P->nf_kT * (1.0 + log_s) - ke * inv_s2 + epot - S->H0;
    CB = P->dt_2 * CB - S->pi;
    const double r = CB * P->dt * P->Qinv;
    if (1.0 - r < 0.0) S->status = 10;  // (38) has no real root: Q_Nose too small
    const double pih = -2 * CB / (1.0 + sqrt(1.0 - r));
    const double a = P->dt_2 * pih * P->Qinv;
    const double sn = s * (1.0 + a) / (1.0 - a);
    S->kick_coef = ca;
    S->pend_ke_sum = kh;
    S->pend_ke = ke;
    S->pend_pi = pih;
    S->pend_s = sn;
    S->pend_drift = P->dt_2 * (1.0 / sn + inv_s);
    S->pend_kick_f = P->dt_2 * sn;
  });
}

// Velocity scaling (velocity_scaling.F:74-83): kinetic energy of the kicked
// momenta, the factor sqrt(target / KE) for k_scale, total.  The reported
// dipo_kinetic is the value before rescaling, as in the reference.
__device__ void vs_tail(const Phys* __restrict__ ph, DevScalars* sc, const double* __restrict__ part, int nblk) {
  double v[1];
  reduce_partials_all<1>(part, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    S->ke_sum = v[0];
    S->e[E_DIPO] = ke_from(P, v[0]);
    S->vs_scale = sqrt(P->target_ke / S->e[E_DIPO]);
    S->e[E_TOT] = S->e[E_DIPO] / (S->s * S->s) + S->e[E_ACOU] + sum_potential(S->e);
    check_finite(S, S->e, E_COUNT);
    if (!isfinite(S->vs_scale)) S->status = 3;
  });
}

// Acoustic kinetic energy sum acouP^2 / m / 2 (kinetic_energy_acou.F:15-27);
// with vs also the rescale factor (velocity_scaling.F:86-98) and the total.
__device__ void acou_tail(const Phys* __restrict__ ph, DevScalars* sc, const double* __restrict__ part, int nblk,
                          bool vs) {
  double v[1];
  reduce_partials_all<1>(part, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    S->e[E_ACOU] = v[0] / 2;
    if (vs) {
      S->vs_scale_acou = sqrt(P->target_ke / S->e[E_ACOU]);
      if (!isfinite(S->vs_scale_acou)) S->status = 3;
      S->e[E_TOT] = S->e[E_DIPO] / (S->s * S->s) + S->e[E_ACOU] + sum_potential(S->e);
    }
  });
}

// Leapfrog closing reduction (leapfrog.F:151) and total.
__device__ void lf_final_tail(const Phys* __restrict__ ph, DevScalars* sc, const double* __restrict__ part, int nblk) {
  double v[1];
  reduce_partials_all<1>(part, nblk, v);
  scalar_tail(ph, sc, [&](const Phys* P, DevScalars* S) {
    S->ke_sum = v[0];
    S->e[E_DIPO] = ke_from(P, v[0]);
    S->e[E_TOT] = S->e[E_DIPO] / (S->s * S->s) + S->e[E_ACOU] + sum_potential(S->e);
    check_finite(S, S->e, E_COUNT);
  });
}

// Wavevectors, trig tables and slot maps shared by the k-space kernels.
struct KMaps {
  const int* revx;     // kx slot -> kx
  const int* revy;     // ky slot -> ky
  const int* revz;     // kz slot -> kz
  const double* kvx;   // k(1) of elastic.F:87 per kx
  const double* kvy;   // k(2) per ky (wrapped to (-1/2, 1/2])
  const double* kvz;   // k(3) per kz
  const double2* trx;  // (cos, sin)(2 pi kx / Lx)
  const double2* try_;
  const double2* trz;
  const double2* trz_s;  // trz and kvz in kz-slot order (no revz lookup first)
  const double* kvz_s;
};

// Plain z pass of nc spectra in place: DIF (INV = false) or DIT (INV = true).
// LZC, CWC, NCC > 0: compile-time transforms for Lz = LZC, tile width CWC
// and NCC components (launched with exactly kZThreads threads); 0 = runtime.
template <typename T, bool INV, int LZC = 0, int CWC = 0, int NCC = 0>
__global__ void __launch_bounds__(256) k_z_pass(cplx<T>* __restrict__ spec, Geom g, FftPlan pz,
                                                const cplx<T>* __restrict__ twz, int nc, ZTiles zt) {
  FG_DYN_SMEM(smem_raw);
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  if constexpr (LZC > 0) {
    __shared__ cplx<T> tws[LZC];
    for (int i = threadIdx.x; i < LZC; i += blockDim.x) tws[i] = twz[i];
    z_tile_load<T, LZC, CWC>(buf, spec, g, zt, NCC);
    using B = BatchCT<NCC * CWC, CWC, 1, LZC * CWC, CWC>;
    if (INV) ct_inverse<T, LZC, 256, B>(buf, tws);
    else ct_forward<T, LZC, 256, B>(buf, tws);
    z_tile_store<T, LZC, CWC>(buf, spec, g, zt, NCC);
  } else {
    const int CW = zt.CW;
    z_tile_load<T>(buf, spec, g, zt, nc);
    Batch B{nc * CW, CW, 1, g.Lz * CW, CW, true};
    if (INV) fft_inverse<T>(buf, B, pz, twz, nc * g.Lz * CW);
    else fft_forward<T>(buf, B, pz, twz, nc * g.Lz * CW);
    z_tile_store<T>(buf, spec, g, zt, nc);
  }
}

// ------------------------------------------------------------------ k_z_kspace
// Per (kx tile, ky slot): DIF along z of the nine spectra, then for every k
//   F(k)     = D(k) uK(k),  D = (S + Z*^2 L)/N   (dVddi-dipole-dipole.F:20-36)
//   acouK(k) = -K(k)^-1 (c_k_mod + coup2(k) didiK(k))  (optimize-inho-strain.F:28-58)
//   inhoK(k) = k (x) acouK / N                        (dVddi_inho_coupling.F:91-108)
// with K, its Cholesky factor and coup2 evaluated analytically
// (elastic.F:79-180), and the half-spectrum energy sums of
// dVddi-dipole-dipole.F:226-250 (by Parseval) and energy_module.F:150-240;
// then DIT along z.  Slots 0..2 return F(k), slots 3..8 inhoK(k).
// ZSC (per-site Z*, dVddi-dipole-dipole.F:20-60): slots Z0..Z0+2 carry
// FFT(Z*(R) u) in and the long-range part (L/N) FFT(Z* u) out, while slots
// 0..2 return the short-range part (S/N) uK alone; L/N comes from ltab.
// LZC, CWC > 0 select the compile-time z transforms (launched with exactly
// kZThreads threads); 0 = runtime plan and tile width.
constexpr int kZThreads = 256;
// Resident CTAs per SM the z kernel is compiled for: FP32 tiles of 4 kx
// columns (37 KB at Lz = 128) leave room for three CTAs, whose 85-register
// budget the compiler then meets; wider tiles fit two.
template <typename T>
constexpr int kZMinBlocks(int cwc) { return (sizeof(T) == 4 && cwc == 4) ? 3 : 2; }
// Component padding of the compile-time z tile, in complex values (64 bytes).
template <typename T>
constexpr int kZPad = 64 / (int)sizeof(cplx<T>);

template <typename T, int LZC = 0, int CWC = 0, bool ACOU = false, bool ZSC = false>
__global__ void __launch_bounds__(256, kZMinBlocks<T>(CWC)) k_z_kspace(cplx<T>* __restrict__ spec, const T* __restrict__ dtab,
                                                     const cplx<T>* __restrict__ ckmod, cplx<T>* __restrict__ acouK_out,
                                                     Geom g, FftPlan pz, const cplx<T>* __restrict__ twz, KMaps km,
                                                     const Phys* __restrict__ ph, double* __restrict__ part,
                                                     DevScalars* sc, ZTiles zt, unsigned int* done,
                                                     const T* __restrict__ ltab, const RepArgs* __restrict__ grp = nullptr) {
  pdl_enter();
  if (grp) {
    const RepArgs& a = grp[blockIdx.y];
    spec = (cplx<T>*)a.spec;
    dtab = (const T*)a.dtab;
    ph = a.ph;
    part = a.part_k;
    sc = a.sc;
  }
  FG_DYN_SMEM(smem_raw);
  cplx<T>* buf = reinterpret_cast<cplx<T>*>(smem_raw);
  __shared__ cplx<T> tws_z[LZC > 0 ? LZC : 1];
  const int Lz = LZC > 0 ? LZC : g.Lz, CW = CWC > 0 ? CWC : zt.CW;
  // ACOU: acoustic-displacement MD, three more components in and out
  // (FFT(acouR) in, dVdacK out; acouFFT.F:9-26, dVdac.F:11-63)
  constexpr int Z0 = ACOU ? 12 : 9;  // first Z* u slot (ZSC)
  constexpr int NC = Z0 + (ZSC ? 3 : 0);
  const int buf_len = NC * Lz * CW;
  // component stride of the tile; the compile-time path pads it by 64 bytes
  // so that the 4 components a warp spans fall on different banks
  const int ZS = LZC > 0 ? LZC * CWC + kZPad<T> : Lz * CW;
  // this thread's pencil: every butterfly it takes belongs to pencil
  // threadIdx.x % CW (the batch and the block size are multiples of CW)
  const int cwp = threadIdx.x % CW;
  int colp = 0, ysp = 0;
  const bool okp = tile_pencil(zt, g, cwp, &colp, &ysp);
  cplx<T>* gp = spec + (okp ? (long long)ysp * g.KXP + colp : 0);
  using BZ = BatchCT<NC * (CWC > 0 ? CWC : 1), (CWC > 0 ? CWC : 1), 1,
                     (LZC > 0 ? LZC : 1) * (CWC > 0 ? CWC : 1) + kZPad<T>, (CWC > 0 ? CWC : 1)>;
  if constexpr (LZC > 0) {
    for (int i = threadIdx.x; i < LZC; i += blockDim.x) tws_z[i] = twz[i];
    // first z stage straight from the spectrum (zeros for the pencils past
    // Ly of the last Nyquist tile)
    // (an evict_first policy on these FP64 loads measured slower: 156 against 140 us)
    auto ld = [&](int t, int e) {
      return okp ? gp[(long long)(t / CWC) * g.ncplx + (long long)e * g.plane_c] : mk<cplx<T>>((T)0, (T)0);
    };
    auto st = [&](int t, int e, const cplx<T>& v) { buf[(t / CWC) * ZS + (t % CWC) + e * CWC] = v; };
    if constexpr (sizeof(T) == 4) {
      // FP32: the whole tile by cp.async first (every copy in flight at
      // once; regular tiles in 16-byte pencil pairs), then all stages
      if (blockIdx.x >= zt.nnyq) {
        int col0 = 0, ys0 = 0;
        tile_pencil(zt, g, 0, &col0, &ys0);
        const cplx<T>* base = spec + (long long)ys0 * g.KXP + col0;
        constexpr int PP = 16 / (int)sizeof(cplx<T>);
        const unsigned long long pol = l2_evict_first();  // the input spectrum is consumed
        for (int r = threadIdx.x; r < NC * LZC * (CWC / PP); r += kZThreads) {
          const int pp = r % (CWC / PP), rz = r / (CWC / PP);
          const int c = rz / LZC, z = rz - c * LZC;
          cp_async16_first(&buf[c * ZS + z * CWC + pp * PP],
                           base + (long long)c * g.ncplx + (long long)z * g.plane_c + pp * PP, pol);
        }
      } else {
        for (int r = threadIdx.x; r < NC * LZC * CWC; r += kZThreads) {
          const int cw = r % CWC, rz = r / CWC;
          const int c = rz / LZC, z = rz - c * LZC;
          int col = 0, ys = 0;
          cplx<T>* d = &buf[c * ZS + z * CWC + cw];
          if (tile_pencil(zt, g, cw, &col, &ys))
            cp_async<(int)sizeof(cplx<T>)>(
                d, spec + (long long)ys * g.KXP + col + (long long)c * g.ncplx + (long long)z * g.plane_c);
          else
            *d = mk<cplx<T>>((T)0, (T)0);
        }
      }
      cp_async_wait();
      __syncthreads();
      ct_forward_range<T, LZC, 0, ct_nst(LZC), kZThreads, BZ>(buf, tws_z);
    } else {
      ct_stage_io<T, LZC, 0, false, kZThreads, NC * CWC, false>(ld, st, twz);
      __syncthreads();
      ct_forward_range<T, LZC, 1, ct_nst(LZC), kZThreads, BZ>(buf, tws_z);
    }
  } else {
    z_tile_load<T, LZC, CWC>(buf, spec, g, zt, NC);
    Batch B{NC * CW, CW, 1, Lz * CW, CW, true};
    fft_forward<T>(buf, B, pz, twz, buf_len);
  }
  const double Ninv = ph->Ninv;
  // Energy sums: the per-k products in T (FP32 in the mixed path, whose
  // spectra are FP32), accumulated per thread in FP64
  double acc[NQ_K] = {0, 0, 0, 0, 0};
  // this thread's pencil (fixed cw), decoded once
  const int cw = cwp, col = colp, yslot = ysp;
  const bool pencil_ok = okp;
  const int ky = pencil_ok ? __ldg(&km.revy[yslot]) : 0;
  const int kx = pencil_ok ? __ldg(&km.revx[col]) : 0;
  const double kv2 = __ldg(&km.kvy[ky]);
  const double2 ty = __ldg(&km.try_[ky]);
  const double2 tx = __ldg(&km.trx[kx]);
  const double kv1 = __ldg(&km.kvx[kx]);
  // S(k) of short_range_k along this pencil: with c = cos, s = sin of the
  // x, y and z phases, S_aa = A_a + B_a cz, S_yz = C_3 sz, S_zx = C_4 sz,
  // S_xy = A_5 + B_5 cz (the x-y parts fixed per pencil, FP64)
  double sA[6], sB[6];
  {
    const double* j = ph->j;
    const double kap = ph->kap2x2, c0 = tx.x, c1 = ty.x, s0 = tx.y, s1 = ty.y;
    sA[0] = kap + 2 * j[1] * c0 + 2 * j[0] * c1 + 4 * j[2] * c0 * c1;
    sB[0] = 2 * j[0] + 4 * j[3] * c1 + 4 * j[2] * c0 + 8 * j[5] * c0 * c1;
    sA[1] = kap + 2 * j[1] * c1 + 2 * j[0] * c0 + 4 * j[2] * c1 * c0;
    sB[1] = 2 * j[0] + 4 * j[3] * c0 + 4 * j[2] * c1 + 8 * j[5] * c0 * c1;
    sA[2] = kap + 2 * j[0] * (c0 + c1) + 4 * j[3] * c0 * c1;
    sB[2] = 2 * j[1] + 4 * j[2] * (c0 + c1) + 8 * j[5] * c0 * c1;
    sA[3] = 0.0;
    sB[3] = -4 * j[4] * s1 - 8 * j[6] * s1 * c0;  // times sz
    sA[4] = 0.0;
    sB[4] = -4 * j[4] * s0 - 8 * j[6] * s0 * c1;  // times sz
    sA[5] = -4 * j[4] * s0 * s1;
    sB[5] = -8 * j[6] * s0 * s1;
  }
  const T w1 = (kx == 0 || kx == g.m) ? (T)1 : (T)2;  // full-spectrum multiplicity
  const long long tpos0 = (long long)yslot * Lz * g.KXP + col;
  for (int zs = threadIdx.x / CW; pencil_ok && zs < Lz; zs += blockDim.x / CW) {
    cplx<T> u[3], d[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) u[a] = buf[a * ZS + zs * CW + cw];
#pragma unroll
    for (int i = 0; i < 6; ++i) d[i] = buf[(3 + i) * ZS + zs * CW + cw];
    const bool k0 = kx == 0 && ky == 0 && zs == 0;  // slot 0 holds kz = 0
    if (k0) {
#pragma unroll
      for (int i = 0; i < 6; ++i) sc->didiK0[i] = (double)d[i].x;
      __threadfence();  // read by homo_strain_tail in another block
    }
    // ---- dipole-dipole
    const long long tpos = tpos0 + (long long)zs * g.KXP;
    using T2 = typename RT2<T>::type;
    const T2* Dp = reinterpret_cast<const T2*>((ZSC ? ltab : dtab) + tpos * 6);  // 6 T per k: 2 T-aligned pairs
    T D[6];  // D = (S + Z*^2 L)/N; ZSC: L/N
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const T2 v = __ldg(&Dp[q]);
      D[2 * q] = v.x;
      D[2 * q + 1] = v.y;
    }
    T qv[6];  // Re(conj(u_a) u_b): xx, yy, zz, yz, zx, xy
    qv[0] = u[0].x * u[0].x + u[0].y * u[0].y;
    qv[1] = u[1].x * u[1].x + u[1].y * u[1].y;
    qv[2] = u[2].x * u[2].x + u[2].y * u[2].y;
    qv[3] = u[1].x * u[2].x + u[1].y * u[2].y;
    qv[4] = u[2].x * u[0].x + u[2].y * u[0].y;
    qv[5] = u[0].x * u[1].x + u[0].y * u[1].y;
    {
      // short- and total dipole energies in FP64 from the same qv, so that
      // their difference (the long-range energy) keeps its digits
      const double2 tz = __ldg(&km.trz_s[zs]);
      double S[6];
      S[0] = sA[0] + sB[0] * tz.x;
      S[1] = sA[1] + sB[1] * tz.x;
      S[2] = sA[2] + sB[2] * tz.x;
      S[3] = sB[3] * tz.y;
      S[4] = sB[4] * tz.y;
      S[5] = sA[5] + sB[5] * tz.x;
      double qd[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) qd[q] = (double)qv[q];
      const double es = (double)w1 * (S[0] * qd[0] + S[1] * qd[1] + S[2] * qd[2] + 2.0 * (S[3] * qd[3] + S[4] * qd[4] + S[5] * qd[5]));
      acc[0] += es;
      if constexpr (ZSC) {
        // short range on uK, long range on FFT(Z* u): Fl = (L/N) ZuK,
        // energy (1/2N) sum w' Re(ZuK* L ZuK) by Parseval
        cplx<T> zu[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) zu[a] = buf[(Z0 + a) * ZS + zs * CW + cw];
        T qz[6];
        qz[0] = zu[0].x * zu[0].x + zu[0].y * zu[0].y;
        qz[1] = zu[1].x * zu[1].x + zu[1].y * zu[1].y;
        qz[2] = zu[2].x * zu[2].x + zu[2].y * zu[2].y;
        qz[3] = zu[1].x * zu[2].x + zu[1].y * zu[2].y;
        qz[4] = zu[2].x * zu[0].x + zu[2].y * zu[0].y;
        qz[5] = zu[0].x * zu[1].x + zu[0].y * zu[1].y;
        acc[1] += es * Ninv + (double)w1 * ((double)D[0] * qz[0] + (double)D[1] * qz[1] + (double)D[2] * qz[2] +
                                            2.0 * ((double)D[3] * qz[3] + (double)D[4] * qz[4] + (double)D[5] * qz[5]));
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int b = (a + 1) % 3, c3 = (a + 2) % 3;  // off-diagonal slots: yz 3, zx 4, xy 5
          const T dab = D[a == 0 ? 5 : a == 1 ? 3 : 4], dac = D[a == 0 ? 4 : a == 1 ? 5 : 3];
          buf[(Z0 + a) * ZS + zs * CW + cw] =
              mk<cplx<T>>(D[a] * zu[a].x + dab * zu[b].x + dac * zu[c3].x, D[a] * zu[a].y + dab * zu[b].y + dac * zu[c3].y);
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) D[q] = (T)(S[q] * Ninv);
      } else {
        acc[1] += (double)w1 * ((double)D[0] * qd[0] + (double)D[1] * qd[1] + (double)D[2] * qd[2] +
                                2.0 * ((double)D[3] * qd[3] + (double)D[4] * qd[4] + (double)D[5] * qd[5]));
      }
    }
    cplx<T> F[3];
    F[0] = mk<cplx<T>>(D[0] * u[0].x + D[5] * u[1].x + D[4] * u[2].x, D[0] * u[0].y + D[5] * u[1].y + D[4] * u[2].y);
    F[1] = mk<cplx<T>>(D[5] * u[0].x + D[1] * u[1].x + D[3] * u[2].x, D[5] * u[0].y + D[1] * u[1].y + D[3] * u[2].y);
    F[2] = mk<cplx<T>>(D[4] * u[0].x + D[3] * u[1].x + D[2] * u[2].x, D[4] * u[0].y + D[3] * u[1].y + D[2] * u[2].y);
    // ---- inhomogeneous strain
    const T k1 = (T)kv1, k2 = (T)kv2, k3 = (T)__ldg(&km.kvz_s[zs]);
    const T kk[4] = {(T)0, k1, k2, k3};
    const T B11 = (T)ph->B11, B12 = (T)ph->B12, B44 = (T)ph->B44;
    T K[3][3];
#pragma unroll
    for (int b = 1; b <= 3; ++b) {
      const int o1 = (b + 1) % 3 + 1, o2 = b % 3 + 1;
#pragma unroll
      for (int a = 1; a <= 3; ++a) {
        if (a == b) K[a - 1][b - 1] = B11 * kk[a] * kk[a] + B44 * kk[o1] * kk[o1] + B44 * kk[o2] * kk[o2];
        else K[a - 1][b - 1] = B12 * kk[a] * kk[b] + B44 * kk[a] * kk[b];
      }
    }
    // coup2 . didiK with coup2(a, i) of elastic.F:156-180: k_a B1xx/2 on
    // i = a, k_a B1yy/2 on the other two diagonal entries, k_c B4yz on the
    // shear entries (yz: b = y, c = z ...) that involve a, zero on the third
    const T hx = (T)(ph->HC2[0][0]), hy = (T)(ph->HC2[0][1]), h4 = (T)(ph->HC2[3][3]);
    cplx<T> ck[3] = {mk<cplx<T>>((T)0, (T)0), mk<cplx<T>>((T)0, (T)0), mk<cplx<T>>((T)0, (T)0)};
    if (ph->modulation_on) {
#pragma unroll
      for (int a = 0; a < 3; ++a) ck[a] = ckmod[tpos * 3 + a];
    }
    // rhs = -(c_k_mod + coup2 . didiK)  (optimize-inho-strain.F:28-45)
    cplx<T> cs[3], acou[3];
    {
      auto comb = [&](T ka, int ia, int ib, int ic, T kb, int sb, T kc, int sc_) {
        // ka (hx d_ia + hy (d_ib + d_ic)) + h4 (kb d_sb + kc d_sc)
        return mk<cplx<T>>(ka * (hx * d[ia].x + hy * (d[ib].x + d[ic].x)) + h4 * (kb * d[sb].x + kc * d[sc_].x),
                           ka * (hx * d[ia].y + hy * (d[ib].y + d[ic].y)) + h4 * (kb * d[sb].y + kc * d[sc_].y));
      };
      cs[0] = comb(k1, 0, 1, 2, k3, 4, k2, 5);
      cs[1] = comb(k2, 1, 0, 2, k3, 3, k1, 5);
      cs[2] = comb(k3, 2, 0, 1, k2, 3, k1, 4);
    }
    if constexpr (ACOU) {
      // dynamic acoustic field: acouK = i FFT(acouR) (acouFFT.F:22);
      // dVdacK = -i (c_k + coup2 didiK + K acouK) / N (dVdac.F:30-60);
      // energies with the K acouK of this field (energy_module.F:150-240)
      cplx<T> KA[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const cplx<T> X = buf[(9 + a) * ZS + zs * CW + cw];
        acou[a] = mk<cplx<T>>(-X.y, X.x);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
        KA[a] = mk<cplx<T>>(K[a][0] * acou[0].x + K[a][1] * acou[1].x + K[a][2] * acou[2].x,
                            K[a][0] * acou[0].y + K[a][1] * acou[1].y + K[a][2] * acou[2].y);
      const T w2 = (T)0.5 * w1;
      T es = 0, ec = 0, em = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        es += acou[a].x * KA[a].x + acou[a].y * KA[a].y;
        ec += acou[a].x * cs[a].x + acou[a].y * cs[a].y;
        em += acou[a].x * ck[a].x + acou[a].y * ck[a].y;
      }
      acc[2] += (double)(w2 * es);
      acc[3] += (double)(w2 * ec);
      acc[4] += (double)(w2 * em);
      const T ni = (T)Ninv;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const cplx<T> v = mk<cplx<T>>(ck[a].x + cs[a].x + KA[a].x, ck[a].y + cs[a].y + KA[a].y);
        buf[(9 + a) * ZS + zs * CW + cw] = mk<cplx<T>>(v.y * ni, -v.x * ni);
      }
    } else if (k0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) acou[a] = mk<cplx<T>>((T)0, (T)0);  // inhomo_K_G(:,:,0,0,0) = 0
    } else {
      // K acou = rhs with K symmetric positive definite: adjugate over the
      // determinant (the reference factorises K by Cholesky, elastic.F:
      // 110-125; the solution is the same up to rounding)
      const T c00 = K[1][1] * K[2][2] - K[1][2] * K[1][2], c11 = K[0][0] * K[2][2] - K[0][2] * K[0][2];
      const T c22 = K[0][0] * K[1][1] - K[0][1] * K[0][1], c01 = K[0][2] * K[1][2] - K[0][1] * K[2][2];
      const T c02 = K[0][1] * K[1][2] - K[0][2] * K[1][1], c12 = K[0][1] * K[0][2] - K[0][0] * K[1][2];
      const T inv = (T)1 / (K[0][0] * c00 + K[0][1] * c01 + K[0][2] * c02);
      cplx<T> r[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) r[a] = mk<cplx<T>>((-ck[a].x - cs[a].x) * inv, (-ck[a].y - cs[a].y) * inv);
      acou[0] = mk<cplx<T>>(c00 * r[0].x + c01 * r[1].x + c02 * r[2].x, c00 * r[0].y + c01 * r[1].y + c02 * r[2].y);
      acou[1] = mk<cplx<T>>(c01 * r[0].x + c11 * r[1].x + c12 * r[2].x, c01 * r[0].y + c11 * r[1].y + c12 * r[2].y);
      acou[2] = mk<cplx<T>>(c02 * r[0].x + c12 * r[1].x + c22 * r[2].x, c02 * r[0].y + c12 * r[1].y + c22 * r[2].y);
    }
    if constexpr (!ACOU) {
      // coupling Re(acou* . coup2 didiK), modulation Re(acou* . c_k); the
      // strain energy Re(acou* K acou) = -(coupling + modulation) because
      // K acou = -(c_k + coup2 didiK)
      const T w2 = (T)0.5 * w1;  // energy_module.F weights: 1/2 at kx = 0, Lx/2
      T ec = 0, em = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        ec += acou[a].x * cs[a].x + acou[a].y * cs[a].y;
        em += acou[a].x * ck[a].x + acou[a].y * ck[a].y;
      }
      acc[2] -= (double)(w2 * (ec + em));
      acc[3] += (double)(w2 * ec);
      acc[4] += (double)(w2 * em);
    }
    if (acouK_out) {
#pragma unroll
      for (int a = 0; a < 3; ++a) acouK_out[tpos * 3 + a] = acou[a];
    }
    const T ni = (T)Ninv;
    d[0] = mk<cplx<T>>(k1 * acou[0].x * ni, k1 * acou[0].y * ni);
    d[1] = mk<cplx<T>>(k2 * acou[1].x * ni, k2 * acou[1].y * ni);
    d[2] = mk<cplx<T>>(k3 * acou[2].x * ni, k3 * acou[2].y * ni);
    d[3] = mk<cplx<T>>((k3 * acou[1].x + k2 * acou[2].x) * ni, (k3 * acou[1].y + k2 * acou[2].y) * ni);
    d[4] = mk<cplx<T>>((k1 * acou[2].x + k3 * acou[0].x) * ni, (k1 * acou[2].y + k3 * acou[0].y) * ni);
    d[5] = mk<cplx<T>>((k2 * acou[0].x + k1 * acou[1].x) * ni, (k2 * acou[0].y + k1 * acou[1].y) * ni);
#pragma unroll
    for (int a = 0; a < 3; ++a) buf[a * ZS + zs * CW + cw] = F[a];
#pragma unroll
    for (int i = 0; i < 6; ++i) buf[(3 + i) * ZS + zs * CW + cw] = d[i];
  }
  __syncthreads();
  if constexpr (LZC > 0) {
    ct_inverse_range<T, LZC, ct_nst(LZC) - 1, 0, kZThreads, BZ>(buf, tws_z);
    // last z stage straight to the spectrum
    auto ld = [&](int t, int e) { return buf[(t / CWC) * ZS + (t % CWC) + e * CWC]; };
    auto st = [&](int t, int e, const cplx<T>& v) {
      if (okp) gp[(long long)(t / CWC) * g.ncplx + (long long)e * g.plane_c] = v;
    };
    ct_stage_io<T, LZC, 0, true, kZThreads, NC * CWC, false>(ld, st, tws_z);
  } else {
    Batch B{NC * CW, CW, 1, Lz * CW, CW, true};
    fft_inverse<T>(buf, B, pz, twz, buf_len);
    z_tile_store<T, LZC, CWC>(buf, spec, g, zt, NC);
  }
  block_partials<NQ_K>(acc, part, blockIdx.x);
  if (done != nullptr && is_last_block(done)) homo_strain_tail(ph, sc, part, gridDim.x);
}

// ------------------------------------------------------------------ k_assemble
// Real-space force (dVddi) on every site:
//   F = F_dd                                      (c2r of k_z_kspace slots 0..2)
//     + anharmonic polynomial force               (dVddi-unharmonic.F:34-65)
//     - Z* E                                      (mirror_force_mirror.F:42-50)
//     + homogeneous strain coupling, w = strain B2 (dVddi-homo-coupling.F:209-237)
//     + inhomogeneous strain coupling, w(R) = eta(R) B2 (dVddi_inho_coupling.F:114-142)
// and the per-block sums of the anharmonic energy (:67-99) and Z* u.E.
// 16-byte vectors of consecutive sites of one component (4 floats or 2
// doubles); used when a vector never straddles a z layer (plane % width == 0).
template <typename T>
struct alignas(16) V16 {
  static constexpr int n = 16 / (int)sizeof(T);
  T v[16 / sizeof(T)];
};
template <typename T>
__device__ __forceinline__ V16<T> ldv(const T* p) { return *reinterpret_cast<const V16<T>*>(p); }
// ldv with the evict_first L2 policy (FP64: when FG_L2_HINT_FP64)
template <typename T>
__device__ __forceinline__ V16<T> ldv_first(const T* p, unsigned long long pol) {
  V16<T> r;
  if constexpr (sizeof(T) == 4) {
    const float4 v = ld_first(reinterpret_cast<const float4*>(p), pol);
    r.v[0] = v.x; r.v[1] = v.y; r.v[2] = v.z; r.v[3] = v.w;
  } else if constexpr (FG_L2_HINT_FP64) {
    const double2 v = ld_first(reinterpret_cast<const double2*>(p), pol);
    r.v[0] = v.x; r.v[1] = v.y;
  } else {
    r = ldv(p);
  }
  return r;
}
template <typename T>
__device__ __forceinline__ void stv(T* p, const V16<T>& a) { *reinterpret_cast<V16<T>*>(p) = a; }

// Constants of the site force, in FP64 for both precisions: the mixed path
// reads FP32 u, the FP32 dipole-dipole force and the FP32 eta, and sums the
// on-site polynomial, the field and both strain couplings in FP64.  Those
// local terms carry the largest forces (|F| up to ~30x the rms force on the
// tail sites of a sigma = 0.1 A configuration), so evaluating them in FP32
// would put their rounding (~1e-6 of the rms force) on exactly those sites.
// On-site polynomial of one species: force combinations and energy
// coefficients (dVddi-unharmonic.F:28-32,67-99)
struct Poly {
  double fa2g, tg, sk, tk2, fk, k4x8;
  double Pa, Pg, P1, P2, P3, P4;
};
struct AsmConst {
  Poly pl;                             // species 1 (the bulk sweeps)
  double hx, hy, h4;                   // homogeneous_coupling_2: B1xx/2, B1yy/2, B4yz
  double Zs;
  int E_on;
  int pad;
};
// Per-step values of the site force, read from DevScalars: strain . B2 and
// the uniform field.
struct AsmDyn {
  double wh[6];
  double E0, E1, E2;
};

// Force on one site from F_dd, u and eta (see k_assemble); acc += energies.
__device__ __forceinline__ void assemble_site(const Poly& pl, const AsmConst& k, double Zs, const AsmDyn& dy,
                                              double ux, double uy, double uz, double f0, double f1, double f2,
                                              const double* eta, double& o0, double& o1, double& o2, double* acc) {
  const double d0 = ux * ux, d1 = uy * uy, d2 = uz * uz;
  const double uu = d0 + d1 + d2;
  // 4th order
  f0 = f0 + ux * (pl.fa2g * uu - pl.tg * d0);
  f1 = f1 + uy * (pl.fa2g * uu - pl.tg * d1);
  f2 = f2 + uz * (pl.fa2g * uu - pl.tg * d2);
  // 6th and 8th order
  const double uu2 = uu * uu, uu3 = uu2 * uu;
  f0 = f0 + ux * (pl.sk * uu2 + pl.k4x8 * uu3 - pl.tk2 * (d0 * d0) - pl.fk * d1 * d2);
  f1 = f1 + uy * (pl.sk * uu2 + pl.k4x8 * uu3 - pl.tk2 * (d1 * d1) - pl.fk * d2 * d0);
  f2 = f2 + uz * (pl.sk * uu2 + pl.k4x8 * uu3 - pl.tk2 * (d2 * d2) - pl.fk * d0 * d1);
  acc[0] += pl.Pa * uu2 + pl.Pg * (d0 * d1 + d1 * d2 + d2 * d0) + pl.P1 * uu3 +
            pl.P2 * ((d0 * d0) * (d1 + d2) + (d1 * d1) * (d2 + d0) + (d2 * d2) * (d0 + d1)) + pl.P3 * d0 * d1 * d2 +
            pl.P4 * (uu2 * uu2);
  if (k.E_on) {
    f0 = f0 - Zs * dy.E0;
    f1 = f1 - Zs * dy.E1;
    f2 = f2 - Zs * dy.E2;
    acc[1] += Zs * (ux * dy.E0 + uy * dy.E1 + uz * dy.E2);
  }
  // homogeneous strain coupling
  f0 = f0 + 2 * dy.wh[0] * ux + dy.wh[4] * uz + dy.wh[5] * uy;
  f1 = f1 + 2 * dy.wh[1] * uy + dy.wh[3] * uz + dy.wh[5] * ux;
  f2 = f2 + 2 * dy.wh[2] * uz + dy.wh[3] * uy + dy.wh[4] * ux;
  // inhomogeneous strain coupling, w_q = sum_j eta_j B2(j, q) with the
  // sparsity of homogeneous_coupling_2 (eta already carries 1/N)
  const double w0 = k.hx * eta[0] + k.hy * (eta[1] + eta[2]);
  const double w1 = k.hx * eta[1] + k.hy * (eta[0] + eta[2]);
  const double w2 = k.hx * eta[2] + k.hy * (eta[0] + eta[1]);
  const double w3 = k.h4 * eta[3], w4 = k.h4 * eta[4], w5 = k.h4 * eta[5];
  o0 = f0 + 2 * w0 * ux + w4 * uz + w5 * uy;
  o1 = f1 + 2 * w1 * uy + w3 * uz + w5 * ux;
  o2 = f2 + 2 * w2 * uz + w3 * uy + w4 * ux;
}

// The force of one site in the field type T.  The mixed path (T = float)
// rounds the FP64 sum once; with lo != null it also stores the rounding
// residual, so that hi + lo carries the FP64 force to ~2^-48 for a caller
// that reads dVddi, while the integrators consume hi.
template <typename T>
__device__ __forceinline__ T force_hi(double o) { return (T)o; }
template <typename T>
__device__ __forceinline__ T force_lo(double o, T hi) { return sizeof(T) == 4 ? (T)(o - (double)hi) : (T)0; }

// Masked kinetic sums of the closing kick (35f) of one site: p <- p - c F
// and p^2/m, p.F/m, F^2/m in T, added to ke (FP64) when the site counts.
template <typename T>
__device__ __forceinline__ void close_site(T* __restrict__ p, long long ns, long long i, T c, T o0, T o1, T o2,
                                           bool counted, double mi, double* ke) {
  const T q0 = p[i] - c * o0, q1 = p[ns + i] - c * o1, q2 = p[2 * ns + i] - c * o2;
  p[i] = q0;
  p[ns + i] = q1;
  p[2 * ns + i] = q2;
  if (counted) {
    ke[0] += (double)(q0 * q0 + q1 * q1 + q2 * q2) * mi;
    ke[1] += (double)(q0 * o0 + q1 * o1 + q2 * o2) * mi;
    ke[2] += (double)(o0 * o0 + o1 * o1 + o2 * o2) * mi;
  }
}

// CLOSE (the force of a Nose-Poincare step, nose-poincare.F:55-71): after the
// force, the closing kick (35f) p <- p - dt/2 s_{n+1} F with the masked sums
// p^2/m, p.F/m, F^2/m of the new p in part_ke; the last block finishes the
// force (energies, commit of the prepared half step, (35e)) and the step
// (np_close_tail: KE, H_NP and (38) of the next step).
// Flo (mixed path, may be null): the FP32 residual of each force component,
// F + Flo = the FP64 site sum.
template <typename T, bool CLOSE = false, bool SITES = false>
__global__ void __launch_bounds__(256, 2)
    k_assemble(const T* __restrict__ rw, const T* __restrict__ u, T* __restrict__ F, Geom g,
               const Phys* __restrict__ ph, DevScalars* sc, double* __restrict__ part, int tail, unsigned int* done,
               const unsigned char* __restrict__ site_species, const T* __restrict__ site_zstar,
               const T* __restrict__ site_E, int zl0, T* __restrict__ p, const double* __restrict__ layer_minv,
               const unsigned char* __restrict__ layer_sump, const T* __restrict__ site_minv,
               const unsigned char* __restrict__ site_sump, double* __restrict__ part_ke, T* __restrict__ Flo,
               const AsmConst k, const RepArgs* __restrict__ grp = nullptr) {
  pdl_enter();
  if (grp) {
    const RepArgs& a = grp[blockIdx.y];
    rw = (const T*)a.rwork;
    u = (const T*)a.u;
    F = (T*)a.F;
    ph = a.ph;
    sc = a.sc;
    part = a.part_r;
    done = a.done_as;
    p = (T*)a.p;
    layer_minv = a.layer_minv;
    layer_sump = a.layer_sump;
    part_ke = a.part_ke;
  }
  // site_*: per-site species (.relaxor), Z* and local field (.localfield);
  // they take the scalar loop.  zl0 > 0: rw components zl0..zl0+2 hold the
  // long-range dipole field of Z* u, which acts on the site times its Z*
  // (dVddi-dipole-dipole.F:52-60); components 0..2 the short-range part.
  const long long ns = g.nsite;
  // pend_kick_f: prepared by the previous step's tail, not changed by this
  // step's commit
  const T cf = CLOSE ? (T)__ldcg(&sc->pend_kick_f) : (T)0;
  double ke[3] = {0.0, 0.0, 0.0};
  const unsigned long long pol_rw = l2_evict_first();
  // k: the static constants (kernel parameter, built by asm_const on the
  // host); dy: this step's strain coupling and field
  // (in shared memory: read at each use instead of held in nine FP64
  // register pairs through the loop)
  __shared__ AsmDyn dy;
  if (threadIdx.x < 6) dy.wh[threadIdx.x] = sc->w_hom[threadIdx.x];
  if (threadIdx.x == 6) dy.E0 = sc->E[0];
  if (threadIdx.x == 7) dy.E1 = sc->E[1];
  if (threadIdx.x == 8) dy.E2 = sc->E[2];
  __syncthreads();
  double acc[NQ_R] = {0.0, 0.0};
  constexpr int NV = V16<T>::n;
  using AV = V16<T>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  // SITES: the per-site loop (any of the site arrays present, chosen on the
  // host); otherwise the bulk loops, compiled without it so that its FP64
  // species polynomial does not set their register budget
  if constexpr (SITES) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      AsmDyn dys = dy;
      double dk2 = 0.0;
      Poly pl;  // this site's species (read_relaxor.F)
      if (site_species) {
        const Phys::Species* q = &ph->sp[site_species[i]];
        pl = Poly{q->fa2g, q->tg, q->sk, q->tk2, q->fk, q->k4x8, q->Pa, q->Pg, q->P1, q->P2, q->P3, q->P4};
        dk2 = q->dk2;
      } else {
        pl = k.pl;
      }
      const double Zs = site_zstar ? (double)site_zstar[i] : k.Zs;
      if (site_E) {
        dys.E0 = dy.E0 + (double)site_E[i];
        dys.E1 = dy.E1 + (double)site_E[ns + i];
        dys.E2 = dy.E2 + (double)site_E[2 * ns + i];
      }
      double eta[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) eta[q] = (double)rw[(3 + q) * ns + i];
      const double ux = u[i], uy = u[ns + i], uz = u[2 * ns + i];
      double f0 = rw[i], f1 = rw[ns + i], f2 = rw[2 * ns + i];
      if (zl0 > 0) {
        f0 = f0 + Zs * (double)rw[(zl0 + 0) * ns + i];
        f1 = f1 + Zs * (double)rw[(zl0 + 1) * ns + i];
        f2 = f2 + Zs * (double)rw[(zl0 + 2) * ns + i];
      }
      double o0, o1, o2;
      assemble_site(pl, k, Zs, dys, ux, uy, uz, f0, f1, f2, eta, o0, o1, o2, acc);
      if (dk2 != 0.0) {  // kappa2(s) - kappa2(1) (dVddi-unharmonic.F:40,73)
        const double t = 2 * dk2;
        o0 = o0 + t * ux;
        o1 = o1 + t * uy;
        o2 = o2 + t * uz;
        acc[0] += dk2 * (ux * ux + uy * uy + uz * uz);
      }
      const T h0 = force_hi<T>(o0), h1 = force_hi<T>(o1), h2 = force_hi<T>(o2);
      F[i] = h0;
      F[ns + i] = h1;
      F[2 * ns + i] = h2;
      if (Flo) {
        Flo[i] = force_lo<T>(o0, h0);
        Flo[ns + i] = force_lo<T>(o1, h1);
        Flo[2 * ns + i] = force_lo<T>(o2, h2);
      }
      if constexpr (CLOSE) {
        const int z = (int)(i / g.plane_r);
        close_site(p, ns, i, cf, h0, h1, h2, site_sump ? site_sump[i] != 0 : layer_sump[z] != 0,
                   site_minv ? (double)site_minv[i] : layer_minv[z], ke);
      }
    }
  } else if (g.plane_r % NV == 0) {
    for (long long iv = (long long)blockIdx.x * blockDim.x + threadIdx.x; iv < ns / NV; iv += stride) {
      const long long i = iv * NV;
      const AV ux = ldv(u + i), uy = ldv(u + ns + i), uz = ldv(u + 2 * ns + i);
      // rw is consumed here: evict_first keeps u, p and F in L2
      const AV a0 = ldv_first(rw + i, pol_rw), a1 = ldv_first(rw + ns + i, pol_rw),
               a2 = ldv_first(rw + 2 * ns + i, pol_rw);
      AV e[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) e[q] = ldv_first(rw + (3 + q) * ns + i, pol_rw);
      AV o0, o1, o2, l0, l1, l2;
#pragma unroll
      for (int l = 0; l < NV; ++l) {
        const double eta[6] = {e[0].v[l], e[1].v[l], e[2].v[l], e[3].v[l], e[4].v[l], e[5].v[l]};
        double d0, d1, d2;
        assemble_site(k.pl, k, k.Zs, dy, ux.v[l], uy.v[l], uz.v[l], a0.v[l], a1.v[l], a2.v[l], eta, d0, d1, d2, acc);
        o0.v[l] = force_hi<T>(d0);
        o1.v[l] = force_hi<T>(d1);
        o2.v[l] = force_hi<T>(d2);
        l0.v[l] = force_lo<T>(d0, o0.v[l]);
        l1.v[l] = force_lo<T>(d1, o1.v[l]);
        l2.v[l] = force_lo<T>(d2, o2.v[l]);
      }
      stv(F + i, o0);
      stv(F + ns + i, o1);
      stv(F + 2 * ns + i, o2);
      if (Flo) {
        stv(Flo + i, l0);
        stv(Flo + ns + i, l1);
        stv(Flo + 2 * ns + i, l2);
      }
      if constexpr (CLOSE) {
        const int z = (int)(i / g.plane_r);
        AV q[3] = {ldv(p + i), ldv(p + ns + i), ldv(p + 2 * ns + i)};
        T pp = 0, pf = 0, ff = 0;
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const T f3[3] = {o0.v[l], o1.v[l], o2.v[l]};
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            q[a].v[l] = q[a].v[l] - cf * f3[a];
            pp += q[a].v[l] * q[a].v[l];
            pf += q[a].v[l] * f3[a];
            ff += f3[a] * f3[a];
          }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) stv(p + a * ns + i, q[a]);
        if (layer_sump[z]) {
          const double mi = layer_minv[z];
          ke[0] += (double)pp * mi;
          ke[1] += (double)pf * mi;
          ke[2] += (double)ff * mi;
        }
      }
    }
  } else {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      double eta[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) eta[q] = (double)rw[(3 + q) * ns + i];
      double o0, o1, o2;
      assemble_site(k.pl, k, k.Zs, dy, u[i], u[ns + i], u[2 * ns + i], rw[i], rw[ns + i], rw[2 * ns + i], eta, o0, o1, o2, acc);
      const T h0 = force_hi<T>(o0), h1 = force_hi<T>(o1), h2 = force_hi<T>(o2);
      F[i] = h0;
      F[ns + i] = h1;
      F[2 * ns + i] = h2;
      if (Flo) {
        Flo[i] = force_lo<T>(o0, h0);
        Flo[ns + i] = force_lo<T>(o1, h1);
        Flo[2 * ns + i] = force_lo<T>(o2, h2);
      }
      if constexpr (CLOSE) {
        const int z = (int)(i / g.plane_r);
        close_site(p, ns, i, cf, h0, h1, h2, layer_sump[z] != 0, layer_minv[z], ke);
      }
    }
  }
  block_partials<NQ_R>(acc, part, blockIdx.x);
  if constexpr (CLOSE) {
    block_partials<3>(ke, part_ke, blockIdx.x);
    if (is_last_block(done)) {
      force_energies_tail(ph, sc, part, gridDim.x, true);
      np_close_tail(ph, sc, part_ke, gridDim.x, true);
    }
  } else if (tail == TAIL_ENERGIES && is_last_block(done)) {
    force_energies_tail(ph, sc, part, gridDim.x, false);
  }
}

// --------------------------------------------------------------- integrators
// p <- p - coef * F on every site (leapfrog.F:134-138) and the masked sum
// p^2 m^-1 of kinetic_energy_dipo.F:92-105.  Per-layer masses and sum_p
// masks (film halves, dead layers).
template <typename T>
__global__ void __launch_bounds__(256) k_kick(T* __restrict__ p, const T* __restrict__ F, const double* coef, Geom g,
                                              const double* __restrict__ layer_minv,
                                              const unsigned char* __restrict__ layer_sump, double* __restrict__ part,
                                              int tail, unsigned int* done, const Phys* __restrict__ ph,
                                              DevScalars* sc, int zero_unmasked, const T* __restrict__ site_minv = nullptr,
                                              const unsigned char* __restrict__ site_sump = nullptr) {
  // zero_unmasked: p = 0 outside sum_p (velocity_scaling.F:61-71).
  // site_minv / site_sump: per-site masses and masks (.relaxor, .defects)
  // instead of the per-layer tables; they take the scalar loop.
  const long long ns = g.nsite;
  const T c = (T)(*coef);
  double acc[1] = {0.0};
  constexpr int NV = V16<T>::n;
  using AV = V16<T>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (g.plane_r % NV == 0 && site_minv == nullptr && site_sump == nullptr) {
    for (long long iv = (long long)blockIdx.x * blockDim.x + threadIdx.x; iv < ns / NV; iv += stride) {
      const long long i = iv * NV;
      const int z = (int)(i / g.plane_r);
      V16<T> q0 = ldv(p + i), q1 = ldv(p + ns + i), q2 = ldv(p + 2 * ns + i);
      const V16<T> f0 = ldv(F + i), f1 = ldv(F + ns + i), f2 = ldv(F + 2 * ns + i);
      const T keep = (zero_unmasked && !layer_sump[z]) ? (T)0 : (T)1;
      double ke = 0.0;
#pragma unroll
      for (int l = 0; l < NV; ++l) {
        q0.v[l] = keep * (q0.v[l] - c * f0.v[l]);
        q1.v[l] = keep * (q1.v[l] - c * f1.v[l]);
        q2.v[l] = keep * (q2.v[l] - c * f2.v[l]);
        ke += (double)q0.v[l] * q0.v[l] + (double)q1.v[l] * q1.v[l] + (double)q2.v[l] * q2.v[l];
      }
      stv(p + i, q0);
      stv(p + ns + i, q1);
      stv(p + 2 * ns + i, q2);
      if (layer_sump[z]) acc[0] += ke * layer_minv[z];
    }
  } else {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      const int z = (int)(i / g.plane_r);
      const bool counted = site_sump ? site_sump[i] != 0 : layer_sump[z] != 0;
      const T keep = (zero_unmasked && !counted) ? (T)0 : (T)1;
      const T p0 = keep * (p[i] - c * F[i]);
      const T p1 = keep * (p[ns + i] - c * F[ns + i]);
      const T p2 = keep * (p[2 * ns + i] - c * F[2 * ns + i]);
      p[i] = p0;
      p[ns + i] = p1;
      p[2 * ns + i] = p2;
      if (counted) {
        const double mi = site_minv ? (double)site_minv[i] : layer_minv[z];
        acc[0] += (double)p0 * p0 * mi + (double)p1 * p1 * mi + (double)p2 * p2 * mi;
      }
    }
  }
  block_partials<1>(acc, part, blockIdx.x);
  if (tail != TAIL_NONE && is_last_block(done)) {
    if (tail == TAIL_LF_FINAL) lf_final_tail(ph, sc, part, gridDim.x);
    else if (tail == TAIL_VS) vs_tail(ph, sc, part, gridDim.x);
    else if (tail == TAIL_ACOU || tail == TAIL_VS_ACOU) acou_tail(ph, sc, part, gridDim.x, tail == TAIL_VS_ACOU);
  }
}

// Sum of v over the block, returned to every thread.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// Heat pump of leapfrog.F:44-87: block 0 scales layer Lz/4 up by delta_e
// per site, block 1 layer 3 (Lz/4) down, the dipole momenta by
// sqrt((e_layer +- Lx Ly delta_e) / e_layer) with e_layer the layer's kinetic
// energy (sum p^2/m / 2 times Lx Ly / counted sites), and likewise the
// acoustic momenta with delta_e_acou (sum acouP^2/m / 2).
template <typename T>
__global__ void __launch_bounds__(256) k_layer_pump(T* __restrict__ p, T* __restrict__ pa, Geom g,
                                                    const double* __restrict__ layer_minv,
                                                    const double* __restrict__ layer_macou,
                                                    const unsigned char* __restrict__ layer_sump, double de,
                                                    double dea, const T* __restrict__ site_minv = nullptr,
                                                    const T* __restrict__ site_macou = nullptr,
                                                    const double* __restrict__ layer_nsum = nullptr) {
  const int z = blockIdx.x == 0 ? g.Lz / 4 : (g.Lz / 4) * 3;
  const double sgn = blockIdx.x == 0 ? 1.0 : -1.0;
  const long long ns = g.nsite, pr = g.plane_r, base = (long long)z * pr;
  const double LxLy = (double)pr;
  if (de != 0.0) {
    double s = 0.0;
    for (long long i = threadIdx.x; i < 3 * pr; i += blockDim.x) {
      const long long j = base + i % pr;
      const T q = p[(i / pr) * ns + j];
      s += (double)q * q * (site_minv ? (double)site_minv[j] : layer_minv[z]);
    }
    const double n_layer = layer_nsum ? layer_nsum[z] : (layer_sump[z] ? LxLy : 0.0);
    const double e = block_sum(s) / 2 * LxLy / n_layer;
    const T f = (T)sqrt((e + sgn * LxLy * de) / e);
    for (long long i = threadIdx.x; i < 3 * pr; i += blockDim.x) p[(i / pr) * ns + base + i % pr] *= f;
  }
  if (dea != 0.0 && pa != nullptr) {
    double s = 0.0;
    for (long long i = threadIdx.x; i < 3 * pr; i += blockDim.x) {
      const long long j = base + i % pr;
      const T q = pa[(i / pr) * ns + j];
      s += (double)q * q * (site_macou ? (double)site_macou[j] : layer_macou[z]);
    }
    const double e = block_sum(s) / 2;
    const T f = (T)sqrt((e + sgn * LxLy * dea) / e);
    for (long long i = threadIdx.x; i < 3 * pr; i += blockDim.x) pa[(i / pr) * ns + base + i % pr] *= f;
  }
}

// p <- scale p on every site (velocity_scaling.F:79-83)
template <typename T>
__global__ void __launch_bounds__(256) k_scale(T* __restrict__ p, const double* scale, long long n) {
  const T f = (T)(*scale);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = f * p[i];
}

// Opening half of a Nose-Poincare step in one sweep: the kick (35a)
// p <- p - kick_coef F and the drift (35c) u <- u + drift p m^-1
// (nose-poincare.F:24-53).  Both coefficients come from the previous closing
// tail, which already solved (38) with the kinetic energy of the kicked p.
// wave (wave_module.F:8-67): the field added at step i_step.  The
// triangular waves divide by period/4.0, a default-kind (single precision)
// real in the reference, so the quarter period is rounded to float.
__host__ __device__ inline void wave_field(int type, long long i_step, int n_thermalize, int period,
                                           const double a[3], double out[3]) {
  if (a[0] == 0.0 && a[1] == 0.0 && a[2] == 0.0) {
    for (int k = 0; k < 3; ++k) out[k] = a[k];
    return;
  }
  if (type == 1 || type == 2) {  // triangular_cos, triangular_sin
    long long i = i_step - n_thermalize;
    if (i < 0) i = 0;
    const long long P = period;
    const long long it = (type == 1) ? llabs(i % P - P / 2) - P / 4 : llabs((i + 3 * P / 4) % P - P / 2) - P / 4;
    const double tmp = (double)it;
    const float quarter = (float)period / 4.0f;
    for (int k = 0; k < 3; ++k) out[k] = a[k] * tmp / (double)quarter;
  } else if (type == 3 || type == 4) {  // ramping_on, ramping_off
    for (int k = 0; k < 3; ++k) {
      if (type == 3) out[k] = (i_step < period) ? a[k] * (double)i_step / period : a[k];
      else out[k] = (i_step < period) ? a[k] * (double)(period - i_step) / period : 0.0;
    }
  } else {
    for (int k = 0; k < 3; ++k) out[k] = a[k];
  }
}

// Start of a step under the device-side field schedule: the step counter
// advances and the uniform field becomes that step's wave value
// (molecular-dynamics.F:66-76, before the step's force evaluation).
__global__ void k_wave_step(const Phys* __restrict__ ph, DevScalars* sc) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const long long i = sc->i_step + 1;
  sc->i_step = i;
  double E[3];
  wave_field(ph->wave_type, i, ph->wave_n_thermalize, ph->wave_period, ph->wave_amp, E);
  for (int k = 0; k < 3; ++k) sc->E[k] = E[k];
}

template <typename T>
__global__ void __launch_bounds__(256) k_kick_drift(T* __restrict__ p, T* __restrict__ u, const T* __restrict__ F,
                                                    const DevScalars* __restrict__ sc, Geom g,
                                                    const double* __restrict__ layer_minv,
                                                    const T* __restrict__ site_minv = nullptr,
                                                    const RepArgs* __restrict__ grp = nullptr) {
  pdl_enter();
  if (grp) {
    const RepArgs& a = grp[blockIdx.y];
    p = (T*)a.p;
    u = (T*)a.u;
    F = (const T*)a.F;
    sc = a.sc;
    layer_minv = a.layer_minv;
  }
  const long long ns = g.nsite;
  const T ck = (T)sc->kick_coef;
  const double cd = sc->pend_drift;
  constexpr int NV = V16<T>::n;
  using AV = V16<T>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (g.plane_r % NV == 0 && site_minv == nullptr) {
    for (long long iv = (long long)blockIdx.x * blockDim.x + threadIdx.x; iv < ns / NV; iv += stride) {
      const long long i = iv * NV;
      const T f = (T)(cd * layer_minv[(int)(i / g.plane_r)]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        V16<T> q = ldv(p + a * ns + i), x = ldv(u + a * ns + i);
        const V16<T> y = ldv(F + a * ns + i);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          q.v[l] = q.v[l] - ck * y.v[l];
          x.v[l] = x.v[l] + f * q.v[l];
        }
        stv(p + a * ns + i, q);
        stv(u + a * ns + i, x);
      }
    }
  } else {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      const T f = (T)(cd * (site_minv ? (double)site_minv[i] : layer_minv[(int)(i / g.plane_r)]));
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const T q = p[a * ns + i] - ck * F[a * ns + i];
        p[a * ns + i] = q;
        u[a * ns + i] = u[a * ns + i] + f * q;
      }
    }
  }
}

// Closing kick of a Nose-Poincare step (35f), p <- p - dt/2 s_{n+1} F
// (nose-poincare.F:66-71), with per-block masked sums of p^2/m, p.F/m and
// F^2/m of the new p for np_close_tail.  Block 0 first finishes the force
// evaluation of this step (energies from k_assemble's partials, commit of the
// prepared half step, (35e)); the last block to arrive, after block 0, runs
// np_close_tail.  PREP: no kick and no prologue; the sums of the current
// state prepare the first step after the state or the thermostat was set.
template <typename T, bool PREP>
__global__ void __launch_bounds__(256) k_kick_close(T* __restrict__ p, const T* __restrict__ F, Geom g,
                                                    const double* __restrict__ layer_minv,
                                                    const unsigned char* __restrict__ layer_sump,
                                                    double* __restrict__ part, unsigned int* done,
                                                    const Phys* __restrict__ ph, DevScalars* sc,
                                                    const double* __restrict__ part_r, int nblk_r,
                                                    const T* __restrict__ site_minv = nullptr,
                                                    const unsigned char* __restrict__ site_sump = nullptr) {
  pdl_enter();
  if (!PREP && blockIdx.x == 0) force_energies_tail(ph, sc, part_r, nblk_r, true);
  const long long ns = g.nsite;
  // pend_kick_f is not changed by block 0's commit
  const T c = PREP ? (T)0 : (T)__ldcg(&sc->pend_kick_f);
  double acc[3] = {0.0, 0.0, 0.0};
  constexpr int NV = V16<T>::n;
  using AV = V16<T>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (g.plane_r % NV == 0 && site_minv == nullptr && site_sump == nullptr) {
    for (long long iv = (long long)blockIdx.x * blockDim.x + threadIdx.x; iv < ns / NV; iv += stride) {
      const long long i = iv * NV;
      const int z = (int)(i / g.plane_r);
      // the vector's 3 NV products summed in T, then accumulated in FP64
      T pp = 0, pf = 0, ff = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        V16<T> q = ldv(p + a * ns + i);
        const V16<T> y = ldv(F + a * ns + i);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          if (!PREP) q.v[l] = q.v[l] - c * y.v[l];
          pp += q.v[l] * q.v[l];
          pf += q.v[l] * y.v[l];
          ff += y.v[l] * y.v[l];
        }
        if (!PREP) stv(p + a * ns + i, q);
      }
      if (layer_sump[z]) {
        const double mi = layer_minv[z];
        acc[0] += (double)pp * mi;
        acc[1] += (double)pf * mi;
        acc[2] += (double)ff * mi;
      }
    }
  } else {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      const int z = (int)(i / g.plane_r);
      double pp = 0.0, pf = 0.0, ff = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        T q = p[a * ns + i];
        const T y = F[a * ns + i];
        if (!PREP) {
          q = q - c * y;
          p[a * ns + i] = q;
        }
        pp += (double)q * q;
        pf += (double)q * y;
        ff += (double)y * y;
      }
      if (site_sump ? site_sump[i] != 0 : layer_sump[z] != 0) {
        const double mi = site_minv ? (double)site_minv[i] : layer_minv[z];
        acc[0] += pp * mi;
        acc[1] += pf * mi;
        acc[2] += ff * mi;
      }
    }
  }
  block_partials<3>(acc, part, blockIdx.x);
  if (is_last_block(done)) np_close_tail(ph, sc, part, gridDim.x, !PREP);
}

// u <- u + coef * p * m^-1 (nose-poincare.F:41-53, leapfrog.F:104-114)
template <typename T>
__global__ void __launch_bounds__(256) k_drift(T* __restrict__ u, const T* __restrict__ p, const double* coef, Geom g,
                                               const double* __restrict__ layer_minv,
                                               const T* __restrict__ site_minv = nullptr) {
  const long long ns = g.nsite;
  const double c = *coef;
  constexpr int NV = V16<T>::n;
  using AV = V16<T>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (g.plane_r % NV == 0 && site_minv == nullptr) {
    for (long long iv = (long long)blockIdx.x * blockDim.x + threadIdx.x; iv < ns / NV; iv += stride) {
      const long long i = iv * NV;
      const T f = (T)(c * layer_minv[(int)(i / g.plane_r)]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        V16<T> x = ldv(u + a * ns + i);
        const V16<T> q = ldv(p + a * ns + i);
#pragma unroll
        for (int l = 0; l < NV; ++l) x.v[l] = x.v[l] + f * q.v[l];
        stv(u + a * ns + i, x);
      }
    }
  } else {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
      const int z = (int)(i / g.plane_r);
      const T f = (T)(c * (site_minv ? (double)site_minv[i] : layer_minv[z]));
      u[i] = u[i] + f * p[i];
      u[ns + i] = u[ns + i] + f * p[ns + i];
      u[2 * ns + i] = u[2 * ns + i] + f * p[2 * ns + i];
    }
  }
}

// Film mirror (mirror.F:9-36): layer z' = Lz-1-z (gap_id = 0) or Lz-z gets
// (-f_x, -f_y, f_z) of layer z.
template <typename T>
__global__ void k_mirror(T* __restrict__ f, Geom g, int gap_id) {
  const long long ns = g.nsite;
  const int z0 = (gap_id == 0) ? 0 : 1;
  const int z1 = (gap_id == 0) ? g.Lz / 2 : (g.Lz + 1) / 2;  // exclusive
  const long long n = (long long)(z1 - z0) * g.plane_r;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int z = z0 + (int)(i / g.plane_r);
    const long long r = i % g.plane_r;
    const int zd = (gap_id == 0) ? g.Lz - 1 - z : g.Lz - z;
    const long long s = (long long)z * g.plane_r + r, d = (long long)zd * g.plane_r + r;
    f[d] = -f[s];
    f[ns + d] = -f[ns + s];
    f[2 * ns + d] = f[2 * ns + s];
  }
}

// KE of the current momenta without changing them.
template <typename T>
__global__ void __launch_bounds__(256) k_ke_only(const T* __restrict__ p, Geom g, const double* __restrict__ layer_minv,
                                                 const unsigned char* __restrict__ layer_sump, double* __restrict__ part,
                                                 const T* __restrict__ site_minv = nullptr,
                                                 const unsigned char* __restrict__ site_sump = nullptr) {
  const long long ns = g.nsite;
  double acc[1] = {0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(i / g.plane_r);
    if (site_sump ? site_sump[i] != 0 : layer_sump[z] != 0) {
      const double mi = site_minv ? (double)site_minv[i] : layer_minv[z];
      const double p0 = p[i], p1 = p[ns + i], p2 = p[2 * ns + i];
      acc[0] += p0 * p0 * mi + p1 * p1 * mi + p2 * p2 * mi;
    }
  }
  block_partials<1>(acc, part, blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) k_ke_finish(const Phys* __restrict__ ph, DevScalars* sc,
                                                           const double* __restrict__ part, int nblk) {
  double v = reduce_partials(part, nblk, 1, 0);
  if (threadIdx.x != 0) return;
  sc->ke_sum = v;
  sc->e[E_DIPO] = ke_from(ph, v);
}

// add_to_Average reductions (average_module.F:86-121): masked sum of u and of
// Z* u per component.  part[b*6 + q]: q = 0..2 sum u, 3..5 sum Z* u.
template <typename T>
__global__ void __launch_bounds__(256) k_avg_sums(const T* __restrict__ u, Geom g, double Zs,
                                                  const unsigned char* __restrict__ layer_sump, double* __restrict__ part,
                                                  const unsigned char* __restrict__ site_sump = nullptr,
                                                  const T* __restrict__ site_zstar = nullptr) {
  const long long ns = g.nsite;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(i / g.plane_r);
    if (site_sump ? !site_sump[i] : !layer_sump[z]) continue;
    if (site_zstar) Zs = site_zstar[i];
    const double a = u[i], b = u[ns + i], c = u[2 * ns + i];
    acc[0] += a;
    acc[1] += b;
    acc[2] += c;
    acc[3] += Zs * a;
    acc[4] += Zs * b;
    acc[5] += Zs * c;
  }
  block_partials<6>(acc, part, blockIdx.x);
}

__global__ void __launch_bounds__(RED_THREADS) k_avg_finish(double* out6, const double* __restrict__ part, int nblk) {
  for (int q = 0; q < 6; ++q) {
    double v = reduce_partials(part, nblk, 6, q);
    if (threadIdx.x == 0) out6[q] = v;
  }
}

// One row of a context's sample series (fg_sample): the six masked sums of
// k_avg_sums (sum u, sum Z* u), then, from the scalars of the last step, the
// potential energy, the true kinetic energy KE / s^2, s, pi and the six
// homogeneous strains: the per-step quantities add_to_Average accumulates
// (average_module.F:75-128), kept as a series so that their block errors
// can be taken afterwards.
constexpr int kSampleCols = FG_SAMPLE_COLS;
constexpr int kSampleCap = FG_SAMPLE_CAP;  // rows a context holds between reads
__global__ void __launch_bounds__(RED_THREADS) k_sample_row(double* __restrict__ row, const double* __restrict__ part,
                                                            int nblk, const DevScalars* __restrict__ sc) {
  for (int q = 0; q < 6; ++q) {
    double v = reduce_partials(part, nblk, 6, q);
    if (threadIdx.x == 0) row[q] = v;
  }
  if (threadIdx.x == 0) {
    const double s = sc->s;
    row[6] = sum_potential(sc->e);
    row[7] = sc->e[E_DIPO] / (s * s);
    row[8] = s;
    row[9] = sc->pi;
    for (int i = 0; i < 6; ++i) row[10 + i] = sc->strain[i];
  }
}

template <typename T>
__global__ void k_accumulate(double* __restrict__ acc, const T* __restrict__ u, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc[i] += (double)u[i];
}

// ------------------------------------------------------- layout conversion
// Padded column-major (nc, 0:NXP-1, 0:NYP-1, 0:Lz-1) FP64 <-> [nc][z][y][x] T.
template <typename T>
__global__ void k_fortran_to_soa(T* __restrict__ dst, const double* __restrict__ src, Geom g, int nc, int NXP, int NYP) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.nsite; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.Lx);
    const long long r = i / g.Lx;
    const int y = (int)(r % g.Ly), z = (int)(r / g.Ly);
    const long long s = (long long)nc * ((long long)x + (long long)NXP * ((long long)y + (long long)NYP * z));
    for (int c = 0; c < nc; ++c) dst[(long long)c * g.nsite + i] = (T)src[s + c];
  }
}

template <typename T>
__global__ void k_soa_to_fortran(double* __restrict__ dst, const T* __restrict__ src, Geom g, int nc, int NXP, int NYP) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.nsite; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.Lx);
    const long long r = i / g.Lx;
    const int y = (int)(r % g.Ly), z = (int)(r / g.Ly);
    const long long s = (long long)nc * ((long long)x + (long long)NXP * ((long long)y + (long long)NYP * z));
    for (int c = 0; c < nc; ++c) dst[s + c] = (double)src[(long long)c * g.nsite + i];
  }
}

// The same for a field held as a hi/lo pair (the mixed path's force after a
// force evaluation that kept its FP32 residual): dst = hi + lo in FP64.
template <typename T>
__global__ void k_soa2_to_fortran(double* __restrict__ dst, const T* __restrict__ hi, const T* __restrict__ lo, Geom g,
                                  int nc, int NXP, int NYP) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.nsite; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.Lx);
    const long long r = i / g.Lx;
    const int y = (int)(r % g.Ly), z = (int)(r / g.Ly);
    const long long s = (long long)nc * ((long long)x + (long long)NXP * ((long long)y + (long long)NYP * z));
    for (int c = 0; c < nc; ++c) dst[s + c] = (double)hi[(long long)c * g.nsite + i] + (double)lo[(long long)c * g.nsite + i];
  }
}

// ------------------------------------------------------- table construction
// Real-space Ewald sum of dipole-dipole-long-range.F:106-149 per site:
// self term at R = 0, images jz, jy, jx in -1-max..max, per element +B on
// the diagonal then -rn_a rn_b C.  Output [6][z][y][x]: xx, yy, zz, yz, zx, xy.
__global__ void k_ewald_real(double* __restrict__ out, Geom g, double a0, double kappa, int max_x, int max_y, int max_z) {
  const double two_over_sqrtpi = 1.12837916709551257390;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.nsite; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % g.Lx);
    const long long r = i / g.Lx;
    const int iy = (int)(r % g.Ly), iz = (int)(r / g.Ly);
    double t[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (i == 0) {
      const double self = -2 * two_over_sqrtpi * kappa * kappa * kappa / 3;
      t[0][0] = t[1][1] = t[2][2] = self;
    }
    for (int jz = -1 - max_z; jz <= max_z; ++jz)
      for (int jy = -1 - max_y; jy <= max_y; ++jy)
        for (int jx = -1 - max_x; jx <= max_x; ++jx) {
          if (jx == 0 && jy == 0 && jz == 0 && i == 0) continue;
          const double rn[3] = {ix * a0 + jx * (g.Lx * a0), iy * a0 + jy * (g.Ly * a0), iz * a0 + jz * (g.Lz * a0)};
          const double rr = rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2];
          const double rnorm = sqrt(rr);
          const double ec = erfc(kappa * rnorm), ex = exp(-kappa * kappa * rr);
          const double B = ec / (rnorm * rr) + two_over_sqrtpi * kappa * ex / rr;
          const double C = (3 * ec / (rnorm * rr) + two_over_sqrtpi * kappa * ex * (2 * kappa * kappa + 3 / rr)) / rr;
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              if (a == b) t[a][b] = t[a][b] + B;
              t[a][b] = t[a][b] - rn[a] * rn[b] * C;
            }
        }
    out[i] = t[0][0];
    out[g.nsite + i] = t[1][1];
    out[2 * g.nsite + i] = t[2][2];
    out[3 * g.nsite + i] = t[1][2];
    out[4 * g.nsite + i] = t[2][0];
    out[5 * g.nsite + i] = t[0][1];
  }
}

// Per (kx tile, ky slot) of the six forward-transformed real-space sums:
// DIF along z, then L = (Re FFT + reciprocal sum) * Hartree*Bohr/eps_inf
// (dipole-dipole-long-range.F:151-206), D = (S + Z*^2 L)/N in the table
// layout, and L in FP64 for inspection.
template <typename T>
__global__ void __launch_bounds__(256) k_z_ewald_pack(const cplx<double>* __restrict__ spec, T* __restrict__ dtab,
                                                      double* __restrict__ L64, Geom g, FftPlan pz,
                                                      const cplx<double>* __restrict__ twz, KMaps km,
                                                      const Phys* __restrict__ ph, double a0, double kappa,
                                                      double eps_inf, int max_x, int max_y, int max_z, ZTiles zt) {
  FG_DYN_SMEM(smem_raw);
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem_raw);
  const int Lz = g.Lz, CW = zt.CW;
  z_tile_load<double>(buf, spec, g, zt, 6);
  {
    Batch B{6 * CW, CW, 1, Lz * CW, CW, true};
    fft_forward<double>(buf, B, pz, twz, 6 * Lz * CW);
  }
  const double pi = 3.14159265358979323846;
  const double four_pi_over_v = 4 * pi / (a0 * a0 * a0);
  const double two_pi_over_a = 2 * pi / a0;
  const double four_kappa2 = 4 * kappa * kappa;
  const double scale = 14.399644 / eps_inf;  // HARTREE_BOHR (define.h:32)
  for (int idx = threadIdx.x; idx < Lz * CW; idx += blockDim.x) {
    const int zs = idx / CW, cw = idx - zs * CW;
    int col, yslot;
    if (!tile_pencil(zt, g, cw, &col, &yslot)) continue;
    const int ky = km.revy[yslot];
    const int kx = km.revx[col], kz = km.revz[zs];
    double k[3];
    k[2] = (double)kz / g.Lz;
    if (k[2] > 0.5) k[2] = k[2] - 1.0;
    k[1] = (double)ky / g.Ly;
    if (k[1] > 0.5) k[1] = k[1] - 1.0;
    k[0] = (double)kx / g.Lx;
    double Lt[6];
    for (int q = 0; q < 6; ++q) Lt[q] = buf[(q * Lz + zs) * CW + cw].x;
    const int qa[6] = {0, 1, 2, 1, 2, 0}, qb[6] = {0, 1, 2, 2, 0, 1};
    for (int q = 0; q < 6; ++q) {
      double t = Lt[q];
      for (int nz = -max_z; nz <= max_z; ++nz) {
        const double kG2 = two_pi_over_a * (k[2] + nz);
        for (int ny = -max_y; ny <= max_y; ++ny) {
          const double kG1 = two_pi_over_a * (k[1] + ny);
          for (int nx = -max_x; nx <= max_x; ++nx) {
            if (kx == 0 && ky == 0 && kz == 0 && nx == 0 && ny == 0 && nz == 0) continue;
            const double kG0 = two_pi_over_a * (k[0] + nx);
            const double kG[3] = {kG0, kG1, kG2};
            const double kGkG = kG0 * kG0 + kG1 * kG1 + kG2 * kG2;
            t = t + four_pi_over_v * kG[qa[q]] * kG[qb[q]] * exp(-kGkG / four_kappa2) / kGkG;
          }
        }
      }
      Lt[q] = t * scale;
    }
    const double2 tx = km.trx[kx], ty = km.try_[ky], tz = km.trz[kz];
    const double cc[3] = {tx.x, ty.x, tz.x}, ss[3] = {tx.y, ty.y, tz.y};
    double S[6];
    short_range_k(ph->j, ph->kap2x2, cc, ss, S);
    const long long tpos = ((long long)yslot * Lz + zs) * g.KXP + col;
    const double z2 = ph->Zstar * ph->Zstar;
    for (int q = 0; q < 6; ++q) {
      dtab[tpos * 6 + q] = (T)((S[q] + z2 * Lt[q]) * ph->Ninv);
      if (L64) L64[tpos * 6 + q] = Lt[q];
    }
  }
}

// dst = (T)(src * scale): the L/N table of the per-site Z* path
template <typename T>
__global__ void __launch_bounds__(256) k_table_scale(T* __restrict__ dst, const double* __restrict__ src, double scale,
                                                     long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (T)(src[i] * scale);
}

// c_k_modulation_k = modulation_constant * k * r2c(modulation_R) (elastic.F:212-225)
template <typename T>
__global__ void __launch_bounds__(256) k_z_modulation_pack(const cplx<double>* __restrict__ spec, cplx<T>* __restrict__ ck,
                                                           Geom g, FftPlan pz, const cplx<double>* __restrict__ twz,
                                                           KMaps km, double mod_const, ZTiles zt) {
  FG_DYN_SMEM(smem_raw);
  cplx<double>* buf = reinterpret_cast<cplx<double>*>(smem_raw);
  const int Lz = g.Lz, CW = zt.CW;
  z_tile_load<double>(buf, spec, g, zt, 1);
  {
    Batch B{CW, CW, 1, Lz * CW, CW, true};
    fft_forward<double>(buf, B, pz, twz, Lz * CW);
  }
  for (int idx = threadIdx.x; idx < Lz * CW; idx += blockDim.x) {
    const int zs = idx / CW, cw = idx - zs * CW;
    int col, yslot;
    if (!tile_pencil(zt, g, cw, &col, &yslot)) continue;
    const int ky = km.revy[yslot];
    const int kx = km.revx[col], kz = km.revz[zs];
    const double kv[3] = {km.kvx[kx], km.kvy[ky], km.kvz[kz]};
    const cplx<double> mk_ = buf[zs * CW + cw];
    const long long tpos = ((long long)yslot * Lz + zs) * g.KXP + col;
    for (int a = 0; a < 3; ++a)
      ck[tpos * 3 + a] = mk<cplx<T>>((T)(mod_const * kv[a] * mk_.x), (T)(mod_const * kv[a] * mk_.y));
  }
}

}  // namespace fg
