// ws_net.cu -- the learned warm start: a small periodic 3D convolutional
// network that proposes a thermalised local-mode field u(R) for a new
// (T, E, pressure) point of a sweep, so that the thermalisation segment of
// the MD can be cut short.  No counterpart in the reference, whose sweeps
// start each point from the previous one (.restart chaining, the fallback
// here: fg_chain_point).
//
// Network: input channels (3 seeded N(0,1) noise fields, T, E_x, E_y, E_z,
// pressure; zero-padded to 16), four 3x3x3 periodic convolutions
// 16 -> 32 -> 32 -> 32 -> 16 (the first 3 output channels are u / 0.1 A),
// SiLU between them.  Weights are BF16 (FP32 master copies for Adam), every
// contraction runs on the tensor cores (tcgen05.mma kind::f16, BF16 x BF16
// with FP32 accumulation in TMEM): the forward convolution and the
// backward-data convolution as implicit GEMMs over 128-site tiles, the weight
// gradient as a GEMM over (tap, input channel) rows with the sites as K.
//
// Training target (moment matching): for every training configuration u_j
// generated by the MD itself at condition c_j, the statistics
//   S = (m.e, |m|, (sum_a m_a^4)^(1/4), <|u|^2>, <sum_a u_a^4>,
//        <sum_a u_a(R) u_a(R + a)>, <sum_a sum_b!=a u_a(R) u_a(R + b)>)
// (m = <u> the mean dipole, e = E / 0.001 V/A, <> site averages) are the
// regression targets of the generated field at c_j; their conditional means
// are what the generator learns.  All statistics are invariant under the
// cubic point group (with the field), so the generator may choose the polar
// axis of an ordered state.
//
// Activations are channels-last: act[s][c], s = sample * nsite + x + Lx (y +
// Ly z); a batch of B samples is one long site axis and the neighbour map
// stays inside each sample.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/feram_gpu.h"
#include "ws_umma.cuh"

using bf16 = __nv_bfloat16;

namespace ws {

constexpr int kTile = 128;        // sites (GEMM rows) per CTA
constexpr int kThreads = 128;     // 4 warps: one TMEM lane quarter each
constexpr int kTaps = 27;
constexpr int kNS = 7;            // statistics per sample
constexpr int kWgradSites = 2048; // sites per weight-gradient CTA (one split)
constexpr long long kWaitIter = 1LL << 22;  // bounded mbarrier waits (~0.3 s)
constexpr double kEps2 = 1e-8, kEps4 = 1e-16;  // floors of |m|^2 and sum m_a^4

struct Geo {
  int Lx, Ly, Lz, nsite;  // one sample
  int B;                  // samples
};

// Site of the periodic neighbour at tap t ((dz, dy, dx) = (t/9, t/3%3, t%3)
// - 1), or at the opposite offset when flip.
__device__ __forceinline__ int nb_site(const Geo& g, int s, int t, bool flip) {
  const int b = s / g.nsite, r = s - b * g.nsite;
  const int x = r % g.Lx, y = (r / g.Lx) % g.Ly, z = r / (g.Lx * g.Ly);
  int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
  if (flip) {
    dx = -dx;
    dy = -dy;
    dz = -dz;
  }
  const int xx = (x + dx + g.Lx) % g.Lx, yy = (y + dy + g.Ly) % g.Ly, zz = (z + dz + g.Lz) % g.Lz;
  return b * g.nsite + xx + g.Lx * (yy + g.Ly * zz);
}

__device__ __forceinline__ float silu(float x) { return x / (1.0f + __expf(-x)); }
__device__ __forceinline__ float dsilu(float x) {
  const float sg = 1.0f / (1.0f + __expf(-x));
  return sg * (1.0f + x * (1.0f - sg));
}

// byte offset of element (row, k) in the canonical no-swizzle K-major tile
__device__ __forceinline__ uint32_t kmaj(int row, int k, uint32_t sbo) {
  return (uint32_t)((row & 7) * 16 + (row >> 3) * sbo + (k >> 3) * 128 + (k & 7) * 2);
}

enum { EPI_HIDDEN = 0, EPI_LAST = 1, EPI_BWD = 2 };

// Implicit-GEMM convolution over one 128-site tile, NC output columns:
//   acc[s][n] = sum_t sum_k act[nb(s, t)][k] * w[n][t][k]     (KC = K per tap)
// forward (flip = false, w = W[cout][t][cin]) or backward-data (flip = true,
// act = dL/dpre of the layer, w = W^T[cin][t][cout]).  Epilogues:
//   EPI_HIDDEN: pre = acc + bias -> pre (FP32), silu(pre) -> out (BF16)
//   EPI_LAST:   pre = acc + bias -> pre (FP32)
//   EPI_BWD:    g = acc * silu'(pre_prev) -> gout (FP32) and gout16 (BF16)
// err: set to 1 when a bounded wait gave up (the tile's results are then
// not written).
template <int KC, int NC, int EPI>
__global__ void __launch_bounds__(kThreads) k_conv_umma(const bf16* __restrict__ act, const bf16* __restrict__ w,
                                                        const float* __restrict__ bias, Geo g, bool flip,
                                                        float* __restrict__ pre, bf16* __restrict__ out,
                                                        const float* __restrict__ pre_prev, int* err) {
  static_assert(KC % 16 == 0 && NC % 16 == 0 && NC <= 32, "K and N multiples of 16, N <= 32");
  constexpr uint32_t SBO = (KC / 8) * 128;  // bytes between 8-row groups
  __shared__ __align__(128) unsigned char sA[kTile * KC * 2];
  __shared__ __align__(128) unsigned char sB[NC * KC * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s0 = blockIdx.x * kTile;
  if (warp == 0) tmem_alloc(&tmem_base, 32);
  if (tid == 0) {
    mbar_init(&bar, 1);
    failed = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base;
  constexpr uint32_t IDESC = idesc_bf16_f32(kTile, NC);
  bool ok = true;
  for (int t = 0; t < kTaps && ok; ++t) {
    // A: this thread's site row, KC channels of the neighbour (16-byte pieces)
    {
      const int src = nb_site(g, s0 + tid, t, flip);
      const uint4* p = reinterpret_cast<const uint4*>(act + (size_t)src * KC);
#pragma unroll
      for (int c = 0; c < KC / 8; ++c)
        *reinterpret_cast<uint4*>(sA + (tid & 7) * 16 + (tid >> 3) * SBO + c * 128) = __ldg(p + c);
    }
    // B: NC rows of KC weights for tap t
    for (int i = tid; i < NC * (KC / 8); i += kThreads) {
      const int n = i / (KC / 8), c = i % (KC / 8);
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(w + ((size_t)n * kTaps + t) * KC) + c);
      *reinterpret_cast<uint4*>(sB + (n & 7) * 16 + (n >> 3) * SBO + c * 128) = v;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int j = 0; j < KC / 16; ++j)
        mma_bf16(tbase, smem_desc(a0 + j * 256, 128, SBO), smem_desc(b0 + j * 256, 128, SBO), IDESC,
                 (t > 0 || j > 0) ? 1u : 0u);
      mma_commit(&bar);
    }
    // every thread waits for this tap's MMAs before the tiles are rewritten
    if (!mbar_wait_bounded(&bar, (uint32_t)(t & 1), kWaitIter)) atomicOr(&failed, 1);
    __syncthreads();
    ok = failed == 0;
  }
  tc_fence_after();
  if (ok) {
    const int row = warp * 32 + lane, s = s0 + row;
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = c0 + i;
        if (EPI == EPI_BWD) {
          const float gv = v[i] * dsilu(pre_prev[(size_t)s * NC + n]);
          pre[(size_t)s * NC + n] = gv;
          out[(size_t)s * NC + n] = __float2bfloat16_rn(gv);
        } else {
          const float x = v[i] + bias[n];
          pre[(size_t)s * NC + n] = x;
          if (EPI == EPI_HIDDEN) out[(size_t)s * NC + n] = __float2bfloat16_rn(silu(x));
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
    mbar_wait_bounded(&bar, 0u, kWaitIter);  // let any MMA still in flight finish
    mbar_wait_bounded(&bar, 1u, kWaitIter);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, 32);
}

// Weight gradient of the sites [blockIdx.y * KS, + KS):
// part[blockIdx.y][n][t][k] = sum_s gout[s][n] act[nb(s, t)][k]; rows
// R = t * KC + k (27 KC of them, tile blockIdx.x), N = NC output channels,
// K = sites in chunks of 64.  Each split writes its own slice (no atomics);
// k_ws_sum_splits adds the slices in a fixed order, so the gradient is the
// same bit for bit from run to run.
template <int KC, int NC>
__global__ void __launch_bounds__(kThreads) k_wgrad_umma(const bf16* __restrict__ act, const bf16* __restrict__ gout,
                                                         Geo g, int KS, float* __restrict__ part, int* err) {
  constexpr size_t kNW = (size_t)NC * kTaps * KC;  // one split's slice
  constexpr int KCH = 64;                   // sites per staged chunk
  constexpr uint32_t SBO = (KCH / 8) * 128;  // 1024 bytes
  __shared__ __align__(128) unsigned char sA[kTile * KCH * 2];
  __shared__ __align__(128) unsigned char sB[NC * KCH * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int R0 = blockIdx.x * kTile, nrows = kTaps * KC;
  const int total = g.B * g.nsite;
  const int k_begin = blockIdx.y * KS, k_end = min(total, k_begin + KS);
  if (warp == 0) tmem_alloc(&tmem_base, 32);
  if (tid == 0) {
    mbar_init(&bar, 1);
    failed = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base;
  constexpr uint32_t IDESC = idesc_bf16_f32(kTile, NC);
  bool ok = true;
  int it = 0;
  for (int kc = k_begin; kc < k_end && ok; kc += KCH, ++it) {
    // A: (row group of 8 channels of one tap) x site; one 16-byte load each
    for (int i = tid; i < (kTile / 8) * KCH; i += kThreads) {
      const int k = i % KCH, rg = i / KCH;
      const int R = R0 + rg * 8;
      const int s = kc + k;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (R < nrows && s < k_end) {
        const int t = R / KC, c = R % KC;
        v = __ldg(reinterpret_cast<const uint4*>(act + (size_t)nb_site(g, s, t, false) * KC + c));
      }
      const unsigned short* h = reinterpret_cast<const unsigned short*>(&v);
#pragma unroll
      for (int q = 0; q < 8; ++q) *reinterpret_cast<unsigned short*>(sA + kmaj(rg * 8 + q, k, SBO)) = h[q];
    }
    // B: output channels x site
    for (int i = tid; i < (NC / 8) * KCH; i += kThreads) {
      const int k = i % KCH, ng = i / KCH;
      const int s = kc + k;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (s < k_end) v = __ldg(reinterpret_cast<const uint4*>(gout + (size_t)s * NC + ng * 8));
      const unsigned short* h = reinterpret_cast<const unsigned short*>(&v);
#pragma unroll
      for (int q = 0; q < 8; ++q) *reinterpret_cast<unsigned short*>(sB + kmaj(ng * 8 + q, k, SBO)) = h[q];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
      for (int j = 0; j < KCH / 16; ++j)
        mma_bf16(tbase, smem_desc(a0 + j * 256, 128, SBO), smem_desc(b0 + j * 256, 128, SBO), IDESC,
                 (it > 0 || j > 0) ? 1u : 0u);
      mma_commit(&bar);
    }
    if (!mbar_wait_bounded(&bar, (uint32_t)(it & 1), kWaitIter)) atomicOr(&failed, 1);
    __syncthreads();
    ok = failed == 0;
  }
  tc_fence_after();
  if (ok && it > 0) {
    const int R = R0 + warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (R < nrows) {
        const int t = R / KC, c = R % KC;
#pragma unroll
        for (int i = 0; i < 16; ++i) part[(size_t)blockIdx.y * kNW + ((size_t)(c0 + i) * kTaps + t) * KC + c] = v[i];
      }
    }
  } else if (!ok && tid == 0) {
    atomicExch(err, 1);
    mbar_wait_bounded(&bar, 0u, kWaitIter);
    mbar_wait_bounded(&bar, 1u, kWaitIter);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, 32);
}

// dW[i] += sum over the nsplit slices of part (fixed order)
__global__ void k_ws_sum_splits(const float* __restrict__ part, int nsplit, int nw, float* __restrict__ dW) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    float acc = 0.0f;
    for (int sp = 0; sp < nsplit; ++sp) acc += part[(size_t)sp * nw + i];
    dW[i] += acc;
  }
}

// --------------------------------------------------------------- elementwise
// Counter-based N(0,1) draws: splitmix64 of (seed, index) -> two uniforms ->
// Box-Muller.  Deterministic for a seed, independent of launch shape.
__device__ __forceinline__ unsigned long long splitmix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ float normal01(unsigned long long seed, unsigned long long i) {
  const unsigned long long h = splitmix(seed * 0x632BE59BD9B4E019ull + i);
  const float u1 = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = (float)((h >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);
  return sqrtf(-2.0f * __logf(u1)) * __cosf(6.2831853f * u2);
}

// Layer-1 input: channels 0..2 noise (seed of the sample), 3 T / 450 K,
// 4..6 E / 0.001 V/A, 7 GPa / 5, 8..15 zero.  cond[b] = (T, Ex, Ey, Ez, GPa).
__global__ void k_ws_input(bf16* __restrict__ in, Geo g, const float* __restrict__ cond,
                           const unsigned long long* __restrict__ seeds) {
  const int total = g.B * g.nsite;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
    const int b = s / g.nsite, r = s - b * g.nsite;
    const float* c = cond + 5 * b;
    float v[16];
    for (int a = 0; a < 3; ++a) v[a] = normal01(seeds[b], 3ull * r + a);
    v[3] = c[0] / 450.0f;
    v[4] = c[1] / 0.001f;
    v[5] = c[2] / 0.001f;
    v[6] = c[3] / 0.001f;
    v[7] = c[4] / 5.0f;
    for (int a = 8; a < 16; ++a) v[a] = 0.0f;
    for (int a = 0; a < 16; ++a) in[(size_t)s * 16 + a] = __float2bfloat16_rn(v[a]);
  }
}

constexpr float kUScale = 0.1f;  // u = 0.1 A x output channel

// Per-sample statistics S of u = kUScale * pre[s][0..2] (channels-last, 16
// wide) into part[block][b][kNS + 3] (the mean u as well), block partials.
__device__ __forceinline__ float uval(const float* pre, int s, int a) { return kUScale * pre[(size_t)s * 16 + a]; }

__global__ void k_ws_stats(const float* __restrict__ pre, Geo g, const float* __restrict__ cond,
                           double* __restrict__ part) {
  // grid (blocks per sample, B); accumulators: m(3), |u|^2, sum u^4, C1, C2
  const int b = blockIdx.y;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < g.nsite; r += gridDim.x * blockDim.x) {
    const int s = b * g.nsite + r;
    float u[3];
    for (int a = 0; a < 3; ++a) u[a] = uval(pre, s, a);
    for (int a = 0; a < 3; ++a) acc[a] += u[a];
    acc[3] += u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    acc[4] += u[0] * u[0] * u[0] * u[0] + u[1] * u[1] * u[1] * u[1] + u[2] * u[2] * u[2] * u[2];
    const int tp[3] = {14, 16, 22};  // +x, +y, +z taps
    for (int d = 0; d < 3; ++d) {
      const int n = nb_site(g, s, tp[d], false);
      for (int a = 0; a < 3; ++a) {
        const float p = u[a] * uval(pre, n, a);
        if (a == d) acc[5] += p;
        else acc[6] += p;
      }
    }
  }
  __shared__ double red[7][256];
  for (int q = 0; q < 7; ++q) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int wdt = blockDim.x / 2; wdt > 0; wdt >>= 1) {
    if (threadIdx.x < wdt)
      for (int q = 0; q < 7; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + wdt];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 7; ++q) part[((size_t)b * gridDim.x + blockIdx.x) * 7 + q] = red[q][0];
}

// S of each sample from the partials; also dL/dS_k = 2 w_k (S_k - target_k)
// in coef[b][k] and the sample's mean u in mean[b][3].  loss[b] = sum w dS^2.
__global__ void k_ws_stats_finish(const double* __restrict__ part, int nblk, Geo g, const float* __restrict__ cond,
                                  const float* __restrict__ target, const float* __restrict__ wts,
                                  float* __restrict__ S, float* __restrict__ coef, float* __restrict__ mean,
                                  float* __restrict__ loss) {
  const int b = blockIdx.x;
  if (threadIdx.x != 0) return;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < nblk; ++k)
    for (int q = 0; q < 7; ++q) v[q] += part[((size_t)b * nblk + k) * 7 + q];
  const double N = g.nsite;
  const double m[3] = {v[0] / N, v[1] / N, v[2] / N};
  const float* c = cond + 5 * b;
  const double e[3] = {c[1] / 0.001, c[2] / 0.001, c[3] / 0.001};
  // |m| and (sum m_a^4)^(1/4) rather than their powers: both scale with the
  // polarisation, so the paraelectric and the ordered points weigh alike
  const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const double m4 = m[0] * m[0] * m[0] * m[0] + m[1] * m[1] * m[1] * m[1] + m[2] * m[2] * m[2] * m[2];
  double st[kNS], dsd[kNS];  // statistic, and its derivative by the raw moment it comes from
  st[0] = m[0] * e[0] + m[1] * e[1] + m[2] * e[2];
  st[1] = sqrt(m2 + kEps2);
  st[2] = sqrt(sqrt(m4 + kEps4));
  st[3] = v[3] / N;
  st[4] = v[4] / N;
  st[5] = v[5] / N;
  st[6] = v[6] / N;
  for (int k = 0; k < kNS; ++k) dsd[k] = 1.0;
  dsd[1] = 0.5 / st[1];
  dsd[2] = 0.25 / (st[2] * st[2] * st[2]);
  double L = 0.0;
  for (int k = 0; k < kNS; ++k) {
    S[b * kNS + k] = (float)st[k];
    if (target) {
      const double d = st[k] - (double)target[b * kNS + k];
      coef[b * kNS + k] = (float)(2.0 * wts[k] * d * dsd[k]);  // dL / d(raw moment)
      L += wts[k] * d * d;
    }
  }
  for (int a = 0; a < 3; ++a) mean[b * 3 + a] = (float)m[a];
  if (target) loss[b] = (float)L;
}

// dL/dpre of the last layer (channels 0..2 carry u / kUScale; 3..15 zero):
// the chain rule through S(u) at every site.
__global__ void k_ws_loss_grad(const float* __restrict__ pre, Geo g, const float* __restrict__ cond,
                               const float* __restrict__ coef, const float* __restrict__ mean, float inv_batch,
                               const float* __restrict__ extra, float* __restrict__ gpre, bf16* __restrict__ gpre16) {
  const int total = g.B * g.nsite;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
    const int b = s / g.nsite;
    const float* cf = coef + b * kNS;
    const float* m = mean + b * 3;
    const float* c = cond + 5 * b;
    const float e[3] = {c[1] / 0.001f, c[2] / 0.001f, c[3] / 0.001f};
    const float invN = 1.0f / (float)g.nsite;
    const int tp[3] = {14, 16, 22}, tm[3] = {12, 10, 4};  // +x,+y,+z and -x,-y,-z
    for (int a = 0; a < 16; ++a) {
      float gv = 0.0f;
      if (a < 3) {
        const float u = uval(pre, s, a);
        float d = cf[0] * e[a] + cf[1] * 2.0f * m[a] + cf[2] * 4.0f * m[a] * m[a] * m[a] + cf[3] * 2.0f * u +
                  cf[4] * 4.0f * u * u * u;
        for (int dd = 0; dd < 3; ++dd) {
          const float nsum = uval(pre, nb_site(g, s, tp[dd], false), a) + uval(pre, nb_site(g, s, tm[dd], false), a);
          d += (dd == a ? cf[5] : cf[6]) * nsum;
        }
        gv = d * invN * kUScale * inv_batch;
        // a gradient on u from outside the statistics (an energy term
        // evaluated by the MD force: dL/du given per site), chained
        // through u = kUScale * pre
        if (extra) gv += extra[(size_t)s * 3 + a] * kUScale;
      }
      gpre[(size_t)s * 16 + a] = gv;
      gpre16[(size_t)s * 16 + a] = __float2bfloat16_rn(gv);
    }
  }
}

// dL/dbias[n] = sum_s g[s][n] (one block per n, fixed order)
__global__ void k_ws_bias_grad(const float* __restrict__ gpre, int total, int NC, float* __restrict__ db) {
  const int n = blockIdx.x;
  double acc = 0.0;
  for (int s = threadIdx.x; s < total; s += blockDim.x) acc += gpre[(size_t)s * NC + n];
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int wdt = blockDim.x / 2; wdt > 0; wdt >>= 1) {
    if (threadIdx.x < wdt) red[threadIdx.x] += red[threadIdx.x + wdt];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[n] += (float)red[0];
}

// Adam (Kingma & Ba 2015) on the FP32 master weights, then their BF16 copy
// W[n][t][k] and its transpose Wt[k][t][n] for the backward-data pass.
__global__ void k_ws_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                          const float* __restrict__ gr, int n, float lr, float b1, float b2, float eps, float bc1,
                          float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g, vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

__global__ void k_ws_cast(const float* __restrict__ w, int NC, int KC, bf16* __restrict__ w16, bf16* __restrict__ wt16) {
  const int n = NC * kTaps * KC;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % KC, t = (i / KC) % kTaps, o = i / (KC * kTaps);
    const bf16 h = __float2bfloat16_rn(w[i]);
    w16[i] = h;
    wt16[((size_t)c * kTaps + t) * NC + o] = h;
  }
}

// u (SoA [3][nsite], T) of sample b from the last layer
template <typename T>
__global__ void k_ws_to_field(const float* __restrict__ pre, int nsite, int b, T* __restrict__ u) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nsite; r += gridDim.x * blockDim.x)
    for (int a = 0; a < 3; ++a) u[(size_t)a * nsite + r] = (T)(kUScale * pre[((size_t)b * nsite + r) * 16 + a]);
}

}  // namespace ws

// ================================================================ host side
namespace {

struct Layer {
  int cin, cout;  // padded channel counts
  float* w = nullptr;       // FP32 master [cout][27][cin]
  float* b = nullptr;       // [cout]
  float* mw = nullptr;      // Adam moments
  float* vw = nullptr;
  float* mb = nullptr;
  float* vb = nullptr;
  float* dw = nullptr;      // gradients
  float* db = nullptr;
  bf16* w16 = nullptr;      // [cout][27][cin]
  bf16* wt16 = nullptr;     // [cin][27][cout]
  float* pre = nullptr;     // [site][cout] pre-activation
  bf16* act = nullptr;      // [site][cout] silu(pre) (hidden layers)
  size_t nw() const { return (size_t)cout * ws::kTaps * cin; }
};

}  // namespace

struct fg_ws {
  ws::Geo g{};
  unsigned long long seed = 0;
  int step = 0;
  Layer L[4];
  bf16* in16 = nullptr;     // layer-1 input [site][16]
  float* gA = nullptr;      // dL/dpre scratch [site][32] (FP32)
  float* gB = nullptr;
  bf16* gA16 = nullptr;     // BF16 copies for the tensor cores
  bf16* gB16 = nullptr;
  float* cond = nullptr;    // [B][5]
  unsigned long long* seeds = nullptr;
  double* part = nullptr;   // stats partials
  int nblk = 0;
  float* S = nullptr;       // [B][7]
  float* target = nullptr;
  float* wts = nullptr;
  float* coef = nullptr;
  float* mean = nullptr;
  float* loss = nullptr;    // [B]
  float* extra = nullptr;   // caller's dL/du [B][nsite][3] (fg_ws_backward_du), allocated on first use
  float* wpart = nullptr;   // weight-gradient slices [split][largest layer]
  int* err = nullptr;
  cudaStream_t stream = nullptr;
  std::string msg;
};

namespace {

int ws_fail(fg_ws* n, int rc, const std::string& m) {
  if (n) n->msg = m;
  return rc;
}
#define WCK(call)                                                                            \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) return ws_fail(n, FG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
int walloc(fg_ws* n, T** p, size_t count) {
  WCK(cudaMalloc((void**)p, count * sizeof(T)));
  // zeroed on the net's own stream: a plain cudaMemset runs on the legacy
  // default stream, which the net's non-blocking stream does not wait for
  WCK(cudaMemsetAsync(*p, 0, count * sizeof(T), n->stream));
  return FG_OK;
}

int total_sites(const fg_ws* n) { return n->g.B * n->g.nsite; }

// BF16 copies of layer l's weights
int cast_layer(fg_ws* n, int l) {
  Layer& y = n->L[l];
  ws::k_ws_cast<<<64, 256, 0, n->stream>>>(y.w, y.cout, y.cin, y.w16, y.wt16);
  WCK(cudaGetLastError());
  return FG_OK;
}

// forward launches of layer l: input act (BF16 [site][cin])
int conv_fwd(fg_ws* n, int l, const bf16* in) {
  Layer& y = n->L[l];
  const int grid = total_sites(n) / ws::kTile;
  if (l == 0) ws::k_conv_umma<16, 32, ws::EPI_HIDDEN><<<grid, ws::kThreads, 0, n->stream>>>(in, y.w16, y.b, n->g, false, y.pre, y.act, nullptr, n->err);
  else if (l < 3) ws::k_conv_umma<32, 32, ws::EPI_HIDDEN><<<grid, ws::kThreads, 0, n->stream>>>(in, y.w16, y.b, n->g, false, y.pre, y.act, nullptr, n->err);
  else ws::k_conv_umma<32, 16, ws::EPI_LAST><<<grid, ws::kThreads, 0, n->stream>>>(in, y.w16, y.b, n->g, false, y.pre, nullptr, nullptr, n->err);
  WCK(cudaGetLastError());
  return FG_OK;
}

int forward(fg_ws* n) {
  const int tot = total_sites(n);
  ws::k_ws_input<<<(tot + 255) / 256, 256, 0, n->stream>>>(n->in16, n->g, n->cond, n->seeds);
  WCK(cudaGetLastError());
  int rc;
  if ((rc = conv_fwd(n, 0, n->in16))) return rc;
  if ((rc = conv_fwd(n, 1, n->L[0].act))) return rc;
  if ((rc = conv_fwd(n, 2, n->L[1].act))) return rc;
  return conv_fwd(n, 3, n->L[2].act);
}

int stats(fg_ws* n, bool with_target) {
  ws::k_ws_stats<<<dim3(n->nblk, n->g.B), 256, 0, n->stream>>>(n->L[3].pre, n->g, n->cond, n->part);
  WCK(cudaGetLastError());
  ws::k_ws_stats_finish<<<n->g.B, 32, 0, n->stream>>>(n->part, n->nblk, n->g, n->cond, with_target ? n->target : nullptr,
                                                      n->wts, n->S, n->coef, n->mean, n->loss);
  WCK(cudaGetLastError());
  return FG_OK;
}

// Backward through the four layers into each layer's dw, db (accumulated).
int backward(fg_ws* n, const float* extra) {
  const int tot = total_sites(n);
  ws::k_ws_loss_grad<<<(tot + 255) / 256, 256, 0, n->stream>>>(n->L[3].pre, n->g, n->cond, n->coef, n->mean,
                                                                1.0f / n->g.B, extra, n->gA, n->gA16);
  WCK(cudaGetLastError());
  const int grid = tot / ws::kTile;
  const int KS = ws::kWgradSites;
  const int nsplit = (tot + KS - 1) / KS;
  float* g = n->gA;
  bf16* g16 = n->gA16;
  float* gn = n->gB;
  bf16* gn16 = n->gB16;
  for (int l = 3; l >= 0; --l) {
    Layer& y = n->L[l];
    const bf16* act_in = l == 0 ? n->in16 : n->L[l - 1].act;
    ws::k_ws_bias_grad<<<y.cout, 256, 0, n->stream>>>(g, tot, y.cout, y.db);
    WCK(cudaGetLastError());
    const int mt = (ws::kTaps * y.cin + ws::kTile - 1) / ws::kTile;
    if (l == 0) ws::k_wgrad_umma<16, 32><<<dim3(mt, nsplit), ws::kThreads, 0, n->stream>>>(act_in, g16, n->g, KS, n->wpart, n->err);
    else if (l < 3) ws::k_wgrad_umma<32, 32><<<dim3(mt, nsplit), ws::kThreads, 0, n->stream>>>(act_in, g16, n->g, KS, n->wpart, n->err);
    else ws::k_wgrad_umma<32, 16><<<dim3(mt, nsplit), ws::kThreads, 0, n->stream>>>(act_in, g16, n->g, KS, n->wpart, n->err);
    WCK(cudaGetLastError());
    ws::k_ws_sum_splits<<<(int)((y.nw() + 255) / 256), 256, 0, n->stream>>>(n->wpart, nsplit, (int)y.nw(), y.dw);
    WCK(cudaGetLastError());
    if (l == 0) break;
    // dL/dpre of layer l-1 = (W^T * g) * silu'(pre_{l-1})
    const Layer& p = n->L[l - 1];
    if (l == 3) ws::k_conv_umma<16, 32, ws::EPI_BWD><<<grid, ws::kThreads, 0, n->stream>>>(g16, y.wt16, nullptr, n->g, true, gn, gn16, p.pre, n->err);
    else ws::k_conv_umma<32, 32, ws::EPI_BWD><<<grid, ws::kThreads, 0, n->stream>>>(g16, y.wt16, nullptr, n->g, true, gn, gn16, p.pre, n->err);
    WCK(cudaGetLastError());
    std::swap(g, gn);
    std::swap(g16, gn16);
  }
  return FG_OK;
}

int check_err(fg_ws* n) {
  int e = 0;
  WCK(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
  WCK(cudaStreamSynchronize(n->stream));
  if (e) return ws_fail(n, FG_ERR_TIMEOUT, "a tensor-core wait ran out (mbarrier)");
  return FG_OK;
}

int upload_inputs(fg_ws* n, const float* cond, const unsigned long long* seeds) {
  WCK(cudaMemcpyAsync(n->cond, cond, sizeof(float) * 5 * n->g.B, cudaMemcpyHostToDevice, n->stream));
  WCK(cudaMemcpyAsync(n->seeds, seeds, sizeof(unsigned long long) * n->g.B, cudaMemcpyHostToDevice, n->stream));
  return FG_OK;
}

void zero_grads(fg_ws* n) {
  for (Layer& y : n->L) {
    cudaMemsetAsync(y.dw, 0, y.nw() * sizeof(float), n->stream);
    cudaMemsetAsync(y.db, 0, y.cout * sizeof(float), n->stream);
  }
}

}  // namespace

extern "C" {

int fg_ws_create(int Lx, int Ly, int Lz, int batch, unsigned long long seed, fg_ws** out) {
  if (!out) return FG_ERR_ARG;
  *out = nullptr;
  fg_ws* n = new fg_ws();
  *out = n;
  if (Lx < 3 || Ly < 3 || Lz < 3 || batch < 1) return ws_fail(n, FG_ERR_ARG, "fg_ws_create: L >= 3 and batch >= 1");
  const long long tot = (long long)Lx * Ly * Lz * batch;
  if (tot % ws::kTile != 0 || tot > (1LL << 30))
    return ws_fail(n, FG_ERR_UNSUPPORTED, "fg_ws_create: Lx Ly Lz batch must be a multiple of 128 sites");
  n->g = ws::Geo{Lx, Ly, Lz, Lx * Ly * Lz, batch};
  n->seed = seed;
  WCK(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
  const int cin[4] = {16, 32, 32, 32}, cout[4] = {32, 32, 32, 16};
  int rc;
  // initial weights: uniform in +-sqrt(6 / fan_in) * gain (He et al. 2015),
  // from a seeded splitmix64 stream on the host; padded input channels zero
  unsigned long long st = seed ^ 0xD1B54A32D192ED03ull;
  auto next_u = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    unsigned long long z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < 4; ++l) {
    Layer& y = n->L[l];
    y.cin = cin[l];
    y.cout = cout[l];
    const size_t nw = y.nw();
    const int real_in = l == 0 ? 8 : 32, real_out = l == 3 ? 3 : 32;
    std::vector<float> w(nw, 0.0f);
    const double lim = std::sqrt(6.0 / (27.0 * real_in)) * (l == 3 ? 0.5 : 1.0);
    for (int o = 0; o < real_out; ++o)
      for (int t = 0; t < ws::kTaps; ++t)
        for (int c = 0; c < real_in; ++c) w[((size_t)o * ws::kTaps + t) * y.cin + c] = (float)((2.0 * next_u() - 1.0) * lim);
    if ((rc = walloc(n, &y.w, nw)) || (rc = walloc(n, &y.mw, nw)) || (rc = walloc(n, &y.vw, nw)) ||
        (rc = walloc(n, &y.dw, nw)) || (rc = walloc(n, &y.b, y.cout)) || (rc = walloc(n, &y.mb, y.cout)) ||
        (rc = walloc(n, &y.vb, y.cout)) || (rc = walloc(n, &y.db, y.cout)) || (rc = walloc(n, &y.w16, nw)) ||
        (rc = walloc(n, &y.wt16, nw)) || (rc = walloc(n, &y.pre, (size_t)tot * y.cout)))
      return rc;
    if (l < 3 && (rc = walloc(n, &y.act, (size_t)tot * y.cout))) return rc;
    // after its zeroing, in the net's stream order
    WCK(cudaMemcpyAsync(y.w, w.data(), nw * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    if ((rc = cast_layer(n, l))) return rc;
  }
  n->nblk = std::max(1, std::min(64, n->g.nsite / 1024));
  if ((rc = walloc(n, &n->in16, (size_t)tot * 16)) || (rc = walloc(n, &n->gA, (size_t)tot * 32)) ||
      (rc = walloc(n, &n->gB, (size_t)tot * 32)) || (rc = walloc(n, &n->gA16, (size_t)tot * 32)) ||
      (rc = walloc(n, &n->gB16, (size_t)tot * 32)) || (rc = walloc(n, &n->cond, (size_t)5 * batch)) ||
      (rc = walloc(n, &n->seeds, (size_t)batch)) || (rc = walloc(n, &n->part, (size_t)7 * n->nblk * batch)) ||
      (rc = walloc(n, &n->S, (size_t)ws::kNS * batch)) || (rc = walloc(n, &n->target, (size_t)ws::kNS * batch)) ||
      (rc = walloc(n, &n->wts, (size_t)ws::kNS)) || (rc = walloc(n, &n->coef, (size_t)ws::kNS * batch)) ||
      (rc = walloc(n, &n->mean, (size_t)3 * batch)) || (rc = walloc(n, &n->loss, (size_t)batch)) ||
      (rc = walloc(n, &n->err, 1)))
    return rc;
  {
    size_t maxnw = 0;
    for (const Layer& y : n->L) maxnw = std::max(maxnw, y.nw());
    const size_t nsplit = ((size_t)tot + ws::kWgradSites - 1) / ws::kWgradSites;
    if ((rc = walloc(n, &n->wpart, nsplit * maxnw))) return rc;
  }
  WCK(cudaStreamSynchronize(n->stream));
  return FG_OK;
}

void fg_ws_destroy(fg_ws* n) {
  if (!n) return;
  if (n->stream) cudaStreamSynchronize(n->stream);
  for (Layer& y : n->L)
    for (void* p : {(void*)y.w, (void*)y.b, (void*)y.mw, (void*)y.vw, (void*)y.mb, (void*)y.vb, (void*)y.dw,
                    (void*)y.db, (void*)y.w16, (void*)y.wt16, (void*)y.pre, (void*)y.act})
      if (p) cudaFree(p);
  for (void* p : {(void*)n->in16, (void*)n->gA, (void*)n->gB, (void*)n->gA16, (void*)n->gB16, (void*)n->cond,
                  (void*)n->seeds, (void*)n->part, (void*)n->S, (void*)n->target, (void*)n->wts, (void*)n->coef,
                  (void*)n->mean, (void*)n->loss, (void*)n->extra, (void*)n->wpart, (void*)n->err})
    if (p) cudaFree(p);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
}

const char* fg_ws_last_error(const fg_ws* n) { return n ? n->msg.c_str() : "null network"; }

int fg_ws_forward(fg_ws* n, const float* cond, const unsigned long long* seeds, float* S) {
  if (!n || !cond || !seeds) return FG_ERR_ARG;
  int rc;
  if ((rc = upload_inputs(n, cond, seeds)) || (rc = forward(n)) || (rc = stats(n, false))) return rc;
  if (S) WCK(cudaMemcpyAsync(S, n->S, sizeof(float) * ws::kNS * n->g.B, cudaMemcpyDeviceToHost, n->stream));
  return check_err(n);
}

int fg_ws_backward_du(fg_ws* n, const float* cond, const unsigned long long* seeds, const float* target,
                      const float* weights, const float* dLdu, float* loss) {
  if (!n || !cond || !seeds || !target || !weights) return FG_ERR_ARG;
  int rc;
  if ((rc = upload_inputs(n, cond, seeds))) return rc;
  WCK(cudaMemcpyAsync(n->target, target, sizeof(float) * ws::kNS * n->g.B, cudaMemcpyHostToDevice, n->stream));
  WCK(cudaMemcpyAsync(n->wts, weights, sizeof(float) * ws::kNS, cudaMemcpyHostToDevice, n->stream));
  if (dLdu) {
    const size_t ne = (size_t)total_sites(n) * 3;
    if (!n->extra && (rc = walloc(n, &n->extra, ne))) return rc;
    WCK(cudaMemcpyAsync(n->extra, dLdu, sizeof(float) * ne, cudaMemcpyHostToDevice, n->stream));
  }
  zero_grads(n);
  if ((rc = forward(n)) || (rc = stats(n, true)) || (rc = backward(n, dLdu ? n->extra : nullptr))) return rc;
  if (loss) {
    std::vector<float> lb(n->g.B);
    WCK(cudaMemcpyAsync(lb.data(), n->loss, sizeof(float) * n->g.B, cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    double s = 0.0;
    for (float v : lb) s += v;
    *loss = (float)(s / n->g.B);
  }
  return check_err(n);
}

int fg_ws_backward(fg_ws* n, const float* cond, const unsigned long long* seeds, const float* target,
                   const float* weights, float* loss) {
  return fg_ws_backward_du(n, cond, seeds, target, weights, nullptr, loss);
}

int fg_ws_adam(fg_ws* n, float lr) {
  if (!n) return FG_ERR_ARG;
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float bc1 = 1.0f - std::pow(b1, (float)n->step), bc2 = 1.0f - std::pow(b2, (float)n->step);
  for (int l = 0; l < 4; ++l) {
    Layer& y = n->L[l];
    ws::k_ws_adam<<<64, 256, 0, n->stream>>>(y.w, y.mw, y.vw, y.dw, (int)y.nw(), lr, b1, b2, eps, bc1, bc2);
    ws::k_ws_adam<<<1, 64, 0, n->stream>>>(y.b, y.mb, y.vb, y.db, y.cout, lr, b1, b2, eps, bc1, bc2);
    WCK(cudaGetLastError());
    int rc = cast_layer(n, l);
    if (rc) return rc;
  }
  WCK(cudaStreamSynchronize(n->stream));
  return FG_OK;
}

int fg_ws_layer_shape(const fg_ws* n, int l, int* cout, int* cin) {
  if (!n || l < 0 || l > 3) return FG_ERR_ARG;
  if (cout) *cout = n->L[l].cout;
  if (cin) *cin = n->L[l].cin;
  return FG_OK;
}

int fg_ws_get_layer(fg_ws* n, int l, float* w, float* b, float* dw, float* db) {
  if (!n || l < 0 || l > 3) return FG_ERR_ARG;
  const Layer& y = n->L[l];
  if (w) WCK(cudaMemcpyAsync(w, y.w, y.nw() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  if (b) WCK(cudaMemcpyAsync(b, y.b, y.cout * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  if (dw) WCK(cudaMemcpyAsync(dw, y.dw, y.nw() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  if (db) WCK(cudaMemcpyAsync(db, y.db, y.cout * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  WCK(cudaStreamSynchronize(n->stream));
  return FG_OK;
}

int fg_ws_set_layer(fg_ws* n, int l, const float* w, const float* b) {
  if (!n || l < 0 || l > 3) return FG_ERR_ARG;
  Layer& y = n->L[l];
  if (w) WCK(cudaMemcpyAsync(y.w, w, y.nw() * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  if (b) WCK(cudaMemcpyAsync(y.b, b, y.cout * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  int rc = cast_layer(n, l);
  if (rc) return rc;
  WCK(cudaStreamSynchronize(n->stream));
  return FG_OK;
}

// The layer-1 input of the last forward (FP32 copy of the BF16 values), the
// generated u of every sample ([B][nsite][3]) and the last statistics.
int fg_ws_get_io(fg_ws* n, float* input, float* u) {
  if (!n) return FG_ERR_ARG;
  const size_t tot = (size_t)total_sites(n);
  if (input) {
    std::vector<bf16> h(tot * 16);
    WCK(cudaMemcpyAsync(h.data(), n->in16, h.size() * sizeof(bf16), cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    for (size_t i = 0; i < h.size(); ++i) input[i] = __bfloat162float(h[i]);
  }
  if (u) {
    std::vector<float> h(tot * 16);
    WCK(cudaMemcpyAsync(h.data(), n->L[3].pre, h.size() * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    WCK(cudaStreamSynchronize(n->stream));
    for (size_t s = 0; s < tot; ++s)
      for (int a = 0; a < 3; ++a) u[s * 3 + a] = ws::kUScale * h[s * 16 + a];
  }
  return FG_OK;
}

// Sample b of the last forward as dipoR in the reference's padded layout
// (coord_module.F:91-93), for fg_set_state.
int fg_ws_field(fg_ws* n, int b, int padding_y, double* dipoR) {
  if (!n || !dipoR || b < 0 || b >= n->g.B) return FG_ERR_ARG;
  const ws::Geo& g = n->g;
  std::vector<float> h((size_t)g.nsite * 16);
  WCK(cudaMemcpyAsync(h.data(), n->L[3].pre + (size_t)b * g.nsite * 16, h.size() * sizeof(float),
                      cudaMemcpyDeviceToHost, n->stream));
  WCK(cudaStreamSynchronize(n->stream));
  const int NXP = 2 * (g.Lx / 2 + 1), NYP = g.Ly + padding_y;
  std::memset(dipoR, 0, sizeof(double) * 3 * (size_t)NXP * NYP * g.Lz);
  for (int z = 0; z < g.Lz; ++z)
    for (int y = 0; y < g.Ly; ++y)
      for (int x = 0; x < g.Lx; ++x) {
        const size_t s = (size_t)x + (size_t)g.Lx * (y + (size_t)g.Ly * z);
        const size_t o = 3 * ((size_t)x + (size_t)NXP * ((size_t)y + (size_t)NYP * z));
        for (int a = 0; a < 3; ++a) dipoR[o + a] = (double)(ws::kUScale * h[s * 16 + a]);
      }
  return FG_OK;
}

}  // extern "C"
