// fft_smem.cuh -- batched in-place mixed-radix FFT stages on shared memory.
//
// Forward transforms are Sande-Tukey decimation in frequency (DIF): natural
// order in, digit-reversed order out.  Inverse transforms run the DIF stages
// backwards as decimation in time (DIT) with conjugate twiddles: digit-
// reversed order in, natural order out, unnormalised (n * IDFT).  Every
// stage reads and writes the same R slots of a butterfly, so a stage is
// in place and any thread can take any number of butterflies; the only
// barrier is one __syncthreads() between stages.  Because the k-space work
// between the forward and inverse transforms is pointwise, the spectrum is
// never permuted back to natural order: kernels map a slot to its true
// wavenumber through the digit-reversal tables built on the host.
//
// Stage st (radix R = r[st]) acts on sub-transforms of length
// Ls = n / (r[0]*...*r[st-1]) with span S = Ls / R.  Butterfly (blk, b)
// takes slots e0 + q*S, e0 = blk*Ls + b, q = 0..R-1, computes
// y_s = sum_q x_q w_R^{qs} and stores y_s * w_Ls^{b s} in slot e0 + s*S.
#pragma once
#include "fg_common.cuh"

namespace fg {

constexpr int FFT_MAX_STAGES = 12;

struct FftPlan {
  int n;
  int nst;
  int r[FFT_MAX_STAGES];
};

// Transform t of a batch starts at base(t) = (t / inner) * outer + (t % inner) * istr
// and its element e lives at base(t) + e * es.  tfast selects the thread
// mapping: consecutive threads take consecutive transforms (tfast = true,
// for transforms interleaved in memory) or consecutive butterflies of one
// transform (tfast = false, for contiguous transforms).
struct Batch {
  int count;
  int inner;
  int istr;
  int outer;
  int es;
  bool tfast;
};

template <typename T, int R, bool INV>
struct Dft;

template <typename T, bool INV>
struct Dft<T, 2, INV> {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    cplx<T> a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <typename T, bool INV>
struct Dft<T, 4, INV> {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    cplx<T> t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    cplx<T> t2 = cadd(v[1], v[3]), t3 = mul_mi<cplx<T>, INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <typename T, bool INV>
struct Dft<T, 8, INV> {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    // radix-2 split into even/odd outputs, then two DFT-4
    const T h = (T)0.70710678118654752440;  // 1/sqrt(2)
    cplx<T> a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a[q] = cadd(v[q], v[q + 4]);
      b[q] = csub(v[q], v[q + 4]);
    }
    // b[q] *= w8^q ; w8 = exp(-i pi/4) forward, conjugate inverse
    b[1] = INV ? mk<cplx<T>>(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
               : mk<cplx<T>>(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
    b[2] = mul_mi<cplx<T>, INV>(b[2]);
    b[3] = INV ? mk<cplx<T>>(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
               : mk<cplx<T>>(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
    Dft<T, 4, INV>::run(a);
    Dft<T, 4, INV>::run(b);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      v[2 * s] = a[s];
      v[2 * s + 1] = b[s];
    }
  }
};

template <typename T, bool INV>
struct Dft<T, 16, INV> {
  // 16 = 4 x 4: DFT-4 over q2 of x[q1 + 4 q2], twiddle w16^(q1 s2), DFT-4 over
  // q1, result X[s2 + 4 s1].
  static __device__ __forceinline__ void run(cplx<T>* v) {
    const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, h = (T)0.70710678118654752440;
    const T sg = INV ? (T)1 : (T)-1;  // sign of the imaginary part of w16^k
    cplx<T> a[4][4];
#pragma unroll
    for (int q1 = 0; q1 < 4; ++q1) {
#pragma unroll
      for (int q2 = 0; q2 < 4; ++q2) a[q1][q2] = v[q1 + 4 * q2];
      Dft<T, 4, INV>::run(a[q1]);
    }
    auto tw = [](cplx<T> x, T cr, T ci) { return mk<cplx<T>>(x.x * cr - x.y * ci, x.x * ci + x.y * cr); };
    a[1][1] = tw(a[1][1], c1, sg * s1);   // w^1
    a[1][2] = tw(a[1][2], h, sg * h);     // w^2
    a[1][3] = tw(a[1][3], s1, sg * c1);   // w^3
    a[2][1] = tw(a[2][1], h, sg * h);     // w^2
    a[2][2] = mul_mi<cplx<T>, INV>(a[2][2]);  // w^4
    a[2][3] = tw(a[2][3], -h, sg * h);    // w^6
    a[3][1] = tw(a[3][1], s1, sg * c1);   // w^3
    a[3][2] = tw(a[3][2], -h, sg * h);    // w^6
    a[3][3] = tw(a[3][3], -c1, -sg * s1); // w^9
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) {
      cplx<T> b[4] = {a[0][s2], a[1][s2], a[2][s2], a[3][s2]};
      Dft<T, 4, INV>::run(b);
#pragma unroll
      for (int s1i = 0; s1i < 4; ++s1i) v[s2 + 4 * s1i] = b[s1i];
    }
  }
};

template <typename T, bool INV>
struct Dft<T, 3, INV> {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    const T s3 = (T)0.86602540378443864676;  // sin(2 pi / 3)
    cplx<T> t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    cplx<T> m = mk<cplx<T>>(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
    // forward: y1 = m - i s3 t2, y2 = m + i s3 t2
    cplx<T> it = mk<cplx<T>>(-s3 * t2.y, s3 * t2.x);  // i*s3*t2
    v[0] = cadd(v[0], t1);
    if (INV) {
      v[1] = cadd(m, it);
      v[2] = csub(m, it);
    } else {
      v[1] = csub(m, it);
      v[2] = cadd(m, it);
    }
  }
};

template <typename T, bool INV>
struct Dft<T, 5, INV> {
  static __device__ __forceinline__ void run(cplx<T>* v) {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    cplx<T> t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    cplx<T> t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    cplx<T> a1 = mk<cplx<T>>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    cplx<T> a2 = mk<cplx<T>>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    cplx<T> b1 = mk<cplx<T>>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    cplx<T> b2 = mk<cplx<T>>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    // i*b
    cplx<T> ib1 = mk<cplx<T>>(-b1.y, b1.x), ib2 = mk<cplx<T>>(-b2.y, b2.x);
    v[0] = cadd(v[0], cadd(t1, t2));
    if (INV) {
      v[1] = cadd(a1, ib1);
      v[4] = csub(a1, ib1);
      v[2] = cadd(a2, ib2);
      v[3] = csub(a2, ib2);
    } else {
      v[1] = csub(a1, ib1);
      v[4] = cadd(a1, ib1);
      v[2] = csub(a2, ib2);
      v[3] = cadd(a2, ib2);
    }
  }
};

template <typename T, int R, bool INV>
__device__ __forceinline__ void fft_stage(cplx<T>* __restrict__ buf, const Batch& B, int n, int Ls,
                                          const cplx<T>* __restrict__ tw, int buf_len) {
  const int S = Ls / R;
  const int nb = n / R;
  const int total = B.count * nb;
  const int twstep = n / Ls;
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    int t, j;
    if (B.tfast) {
      t = w % B.count;
      j = w / B.count;
    } else {
      j = w % nb;
      t = w / nb;
    }
    const int blk = j / S, b = j - blk * S;
    const int base = (t / B.inner) * B.outer + (t % B.inner) * B.istr + (blk * Ls + b) * B.es;
    const int step = S * B.es;
#if FG_BOUNDS_CHECK
    if (base < 0 || base + (R - 1) * step >= buf_len) {
      fg_record_error(1, base);
      continue;
    }
#endif
    cplx<T> v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = buf[base + q * step];
    if (!INV) {
      Dft<T, R, false>::run(v);
#pragma unroll
      for (int s = 1; s < R; ++s) v[s] = cmul(v[s], __ldg(&tw[b * s * twstep]));
    } else {
#pragma unroll
      for (int s = 1; s < R; ++s) v[s] = cmulc(v[s], __ldg(&tw[b * s * twstep]));
      Dft<T, R, true>::run(v);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) buf[base + q * step] = v[q];
  }
}

template <typename T, bool INV>
__device__ __forceinline__ void fft_stage_rt(int R, cplx<T>* buf, const Batch& B, int n, int Ls,
                                             const cplx<T>* tw, int buf_len) {
  switch (R) {
    case 2: fft_stage<T, 2, INV>(buf, B, n, Ls, tw, buf_len); break;
    case 3: fft_stage<T, 3, INV>(buf, B, n, Ls, tw, buf_len); break;
    case 4: fft_stage<T, 4, INV>(buf, B, n, Ls, tw, buf_len); break;
    case 5: fft_stage<T, 5, INV>(buf, B, n, Ls, tw, buf_len); break;
    case 8: fft_stage<T, 8, INV>(buf, B, n, Ls, tw, buf_len); break;
    case 16: fft_stage<T, 16, INV>(buf, B, n, Ls, tw, buf_len); break;
    default: break;
  }
}

// Full forward (DIF) transform of a batch; ends with __syncthreads().
template <typename T>
__device__ __forceinline__ void fft_forward(cplx<T>* buf, const Batch& B, const FftPlan& P, const cplx<T>* tw, int buf_len) {
  int Ls = P.n;
  for (int st = 0; st < P.nst; ++st) {
    fft_stage_rt<T, false>(P.r[st], buf, B, P.n, Ls, tw, buf_len);
    Ls /= P.r[st];
    __syncthreads();
  }
}

// Full inverse (DIT) transform, digit-reversed in, natural out, unnormalised.
template <typename T>
__device__ __forceinline__ void fft_inverse(cplx<T>* buf, const Batch& B, const FftPlan& P, const cplx<T>* tw, int buf_len) {
  int Ls = 1;
  for (int st = P.nst - 1; st >= 0; --st) {
    Ls *= P.r[st];
    fft_stage_rt<T, true>(P.r[st], buf, B, P.n, Ls, tw, buf_len);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Compile-time transforms for power-of-two lengths and for 12, 24 and 48.
// Same DIF/DIT algorithm and slot order as above (the host builds its
// digit-reversal tables from ct_radix), but every index is a compile-time
// expression, the radices are 16 and 8 (two shared-memory stages for
// n <= 256; 12, 24, 48 add a radix-3 stage), and twiddles come from a
// shared-memory copy of the table.  Stage plans: 4:[4] 8:[8] 16:[16] 32:[8,4]
// 64:[4,16] 128:[16,8] 256:[16,16] 512:[16,8,4] 12:[4,3] 24:[8,3] 48:[16,3].
// 64 starts with radix 4 so
// that its first stage (16 butterflies per transform, elements 16 apart) can
// read a 64-point row straight from global memory in 128-byte runs.
__host__ __device__ constexpr bool ct_supported(int n) {
  return n == 4 || n == 8 || n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512 || n == 12 ||
         n == 24 || n == 48;
}
// 12, 24, 48 (the 24^3 and 48^3 supercells of the batched sweeps): a
// power-of-two stage, then a radix-3 one (the runtime plan's order for 12
// and 24)
__host__ __device__ constexpr int ct_nst(int n) {
  return (n == 12 || n == 24 || n == 48) ? 2 : (n <= 16 ? 1 : (n <= 256 ? 2 : 3));
}
__host__ __device__ constexpr int ct_radix(int n, int st) {
  return n == 12 ? (st == 0 ? 4 : 3)
       : n == 24 ? (st == 0 ? 8 : 3)
       : n == 48 ? (st == 0 ? 16 : 3)
       : n <= 16 ? n
       : n == 32 ? (st == 0 ? 8 : 4)
       : n == 64 ? (st == 0 ? 4 : 16)
       : n == 128 ? (st == 0 ? 16 : 8)
       : n == 256 ? 16
       : (st == 0 ? 16 : (st == 1 ? 8 : 4));
}
__host__ __device__ constexpr int ct_ls(int n, int st) {  // sub-transform length at stage st
  return st == 0 ? n : ct_ls(n, st - 1) / ct_radix(n, st - 1);
}

// Compile-time batch layout (see Batch); consecutive threads take
// consecutive transforms.
template <int COUNT, int INNER, int ISTR, int OUTER, int ES>
struct BatchCT {
  static constexpr int count = COUNT, inner = INNER, istr = ISTR, outer = OUTER, es = ES;
};

template <typename T, int N, int LS, int R, bool INV, int NT, class B>
__device__ __forceinline__ void ct_stage(cplx<T>* __restrict__ buf, const cplx<T>* __restrict__ tws) {
  constexpr int S = LS / R, NB = N / R, TOTAL = B::count * NB, TWS = N / LS;
  constexpr int STEP = S * B::es;
  constexpr int U = (R <= 8 || (sizeof(T) == 4 && NT <= 256)) ? 2 : 1;  // butterflies in flight per thread
#pragma unroll U
  for (int w = threadIdx.x; w < TOTAL; w += NT) {
    const int t = w % B::count, j = w / B::count;
    const int blk = j / S, b = j - blk * S;
    const int base = (t / B::inner) * B::outer + (t % B::inner) * B::istr + (blk * LS + b) * B::es;
    cplx<T> v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = buf[base + q * STEP];
    if (!INV) {
      Dft<T, R, false>::run(v);
      if (S > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tws[b * q * TWS]);
      }
    } else {
      if (S > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tws[b * q * TWS]);
      }
      Dft<T, R, true>::run(v);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) buf[base + q * STEP] = v[q];
  }
}

template <typename T, int N, int ST, int NT, class B>
__device__ __forceinline__ void ct_forward_from(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST < ct_nst(N)) {
    ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), false, NT, B>(buf, tws);
    __syncthreads();
    ct_forward_from<T, N, ST + 1, NT, B>(buf, tws);
  }
}
template <typename T, int N, int ST, int NT, class B>
__device__ __forceinline__ void ct_inverse_from(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST >= 0) {
    ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), true, NT, B>(buf, tws);
    __syncthreads();
    ct_inverse_from<T, N, ST - 1, NT, B>(buf, tws);
  }
}
// Stages ST .. END-1 (forward) or ST down to END+1 (inverse), each followed
// by __syncthreads().
template <typename T, int N, int ST, int END, int NT, class B>
__device__ __forceinline__ void ct_forward_range(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST < END) {
    ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), false, NT, B>(buf, tws);
    __syncthreads();
    ct_forward_range<T, N, ST + 1, END, NT, B>(buf, tws);
  }
}
template <typename T, int N, int ST, int END, int NT, class B>
__device__ __forceinline__ void ct_inverse_range(cplx<T>* buf, const cplx<T>* tws) {
  if constexpr (ST > END) {
    ct_stage<T, N, ct_ls(N, ST), ct_radix(N, ST), true, NT, B>(buf, tws);
    __syncthreads();
    ct_inverse_range<T, N, ST - 1, END, NT, B>(buf, tws);
  }
}

// One compile-time stage of a batch of COUNT transforms whose elements are
// read through ld(t, e) and written through st(t, e, v) (t = transform,
// e = element): the first or last stage of a pass fused with its global load
// or store.  JFAST: consecutive threads take consecutive butterflies of one
// transform (global rows whose butterflies run along the contiguous
// direction); otherwise consecutive transforms, as ct_stage.  No barrier.
template <typename T, int N, int ST, bool INV, int NT, int COUNT, bool JFAST, class LD, class SV>
__device__ __forceinline__ void ct_stage_io(const LD& ld, const SV& st, const cplx<T>* __restrict__ tws) {
  constexpr int LS = ct_ls(N, ST), R = ct_radix(N, ST);
  constexpr int S = LS / R, NB = N / R, TOTAL = COUNT * NB, TWS = N / LS;
  constexpr int U = 1;  // butterflies in flight per thread
#pragma unroll U
  for (int w = threadIdx.x; w < TOTAL; w += NT) {
    const int t = JFAST ? w / NB : w % COUNT;
    const int j = JFAST ? w - t * NB : w / COUNT;
    const int blk = j / S, b = j - blk * S;
    const int e0 = blk * LS + b;
    cplx<T> v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = ld(t, e0 + q * S);
    if (!INV) {
      Dft<T, R, false>::run(v);
      if (S > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tws[b * q * TWS]);
      }
    } else {
      if (S > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tws[b * q * TWS]);
      }
      Dft<T, R, true>::run(v);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) st(t, e0 + q * S, v[q]);
  }
}

// Forward DIF / inverse DIT of a batch; both end with __syncthreads().
template <typename T, int N, int NT, class B>
__device__ __forceinline__ void ct_forward(cplx<T>* buf, const cplx<T>* tws) {
  ct_forward_from<T, N, 0, NT, B>(buf, tws);
}
template <typename T, int N, int NT, class B>
__device__ __forceinline__ void ct_inverse(cplx<T>* buf, const cplx<T>* tws) {
  ct_inverse_from<T, N, ct_nst(N) - 1, NT, B>(buf, tws);
}

}  // namespace fg
