// fg_api.cu -- the C-ABI of include/feram_gpu.h on one B200.
//
// One fg_ctx owns the device state of one supercell (coord_module.F's
// Coord_type), the k-space tables, the FFT plans and a CUDA stream.  Each
// MD step is a CUDA graph of ~12 kernels whose scalars (Nose-Poincare s, pi,
// H0, strain, energies) live in device memory, so a step never waits on the
// host; the host reads the 13 energies back once per call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/feram_gpu.h"
#include "fg_kernels.cuh"

using namespace fg;

namespace {

constexpr int kThreadsFFT = 512;
constexpr int kThreadsZ = 256;
constexpr int kThreadsElem = 256;

int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// DIF stage radices: the compile-time plans of fft_smem.cuh for powers of
// two, otherwise largest first (8, 4, 2, then 3 and 5).
bool make_plan(int n, FftPlan* P) {
  P->n = n;
  P->nst = 0;
  if (ct_supported(n)) {
    P->nst = ct_nst(n);
    for (int st = 0; st < P->nst; ++st) P->r[st] = ct_radix(n, st);
    return true;
  }
  int m = n;
  while (m % 8 == 0) { P->r[P->nst++] = 8; m /= 8; }
  while (m % 4 == 0) { P->r[P->nst++] = 4; m /= 4; }
  while (m % 2 == 0) { P->r[P->nst++] = 2; m /= 2; }
  while (m % 3 == 0) { if (P->nst >= FFT_MAX_STAGES) return false; P->r[P->nst++] = 3; m /= 3; }
  while (m % 5 == 0) { if (P->nst >= FFT_MAX_STAGES) return false; P->r[P->nst++] = 5; m /= 5; }
  return m == 1 && P->nst <= FFT_MAX_STAGES;
}

// slot -> frequency of the DIF output (digit reversal)
std::vector<int> digit_reversal(const FftPlan& P) {
  std::vector<int> rev(P.n);
  for (int p = 0; p < P.n; ++p) {
    int q = p, k = 0, mult = 1, span = P.n;
    for (int st = 0; st < P.nst; ++st) {
      span /= P.r[st];
      int s = q / span;
      q -= s * span;
      k += s * mult;
      mult *= P.r[st];
    }
    rev[p] = k;
  }
  return rev;
}

// exp(-2 pi i k / n), k = 0..n-1, from long-double sin/cos of the reduced angle
template <typename T>
std::vector<cplx<T>> twiddles(int n) {
  std::vector<cplx<T>> w(n);
  for (int k = 0; k < n; ++k) {
    long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
    w[k] = mk<cplx<T>>((T)std::cos(a), (T)std::sin(a));
  }
  return w;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
};

}  // namespace

struct fg_ctx {
  fg_params P;
  int prec = FG_PREC_FP64;
  std::string err;
  Geom g{};
  FftPlan px{}, py{}, pz{};
  ZTiles zt{}, zt6{}, zt1{};  // z tiles: MD k-space (9 comps, T), table build (6, FP64), modulation (1, FP64)
  int smem_xy = 0, smem_xy64 = 0, smem_z = 0, smem_z3 = 0, smem_z6 = 0, smem_z1 = 0;
  int grid_elem = 1;
  // one resident wave of the step's streaming kernels (grid-stride loops):
  // k_kick_drift, k_kick_close, k_assemble; <= grid_elem
  int grid_kd = 1, grid_kc = 1, grid_as = 1, grid_asc = 1;  // grid_asc: k_assemble<T, true>
  cudaStream_t stream = nullptr;
  // fields (T = float or double)
  void* u = nullptr;
  void* p = nullptr;
  void* F = nullptr;
  // mixed path: FP32 residual of F (F + Flo = the FP64 site sum), written by
  // the force-only evaluation (fg_mirror_force_mirror); flo_valid while F
  // has not been rewritten by a step since
  void* Flo = nullptr;
  bool flo_valid = false;
  void* spec = nullptr;   // 9 complex spectra
  void* rwork = nullptr;  // 9 real fields
  void* dtab = nullptr;   // 6 per table slot
  void* ckmod = nullptr;  // 3 complex per table slot
  void* acouK = nullptr;  // 3 complex per table slot
  void* twx = nullptr;
  void* twm = nullptr;
  void* twy = nullptr;
  void* twz = nullptr;
  // FP64 twiddles for table construction
  cplx<double>* twx64 = nullptr;
  cplx<double>* twm64 = nullptr;
  cplx<double>* twy64 = nullptr;
  cplx<double>* twz64 = nullptr;
  double* L64 = nullptr;  // long-range table (FP64, table slots)
  void* ltab = nullptr;   // L/N in T (table slots), per-site Z* only
  bool ltab_ready = false;
  bool zsite = false;     // per-site Z* differs: Z* u transformed on its own
  int* revx = nullptr;
  int* revy = nullptr;
  int* revz = nullptr;
  int* posm = nullptr;
  double* kvx = nullptr;
  double* kvy = nullptr;
  double* kvz = nullptr;
  double2* trx = nullptr;
  double2* try_ = nullptr;
  double2* trz = nullptr;
  double2* trz_s = nullptr;  // trz and kvz in kz-slot order
  double* kvz_s = nullptr;
  double* layer_minv = nullptr;
  unsigned char* layer_sump = nullptr;
  // acoustic-displacement MD (acoustic mass > 0): u, p and F hold three more
  // components (acouR, acouP, unused), the passes transform 12 components and
  // rwork's components 9..11 hold dVdacR after a force evaluation
  bool acou = false;
  int ncx = 9;
  double* layer_macou = nullptr;       // 1 / mass_acou per layer
  unsigned char* layer_all = nullptr;  // all layers counted
  // per-site tables (fg_upload_site_arrays: .relaxor, .defects, .localfield);
  // null: the per-layer tables hold
  void* site_minv = nullptr;             // T, 1 / mass_dipo
  void* site_macou = nullptr;            // T, 1 / mass_acou
  unsigned char* site_sump = nullptr;    // sum_p
  unsigned char* site_species = nullptr; // relaxor index - 1
  void* site_zstar = nullptr;            // T, Z*
  void* site_E = nullptr;                // T, local field, 3 components
  double* layer_nsum = nullptr;          // counted sites per layer
  Phys* ph = nullptr;
  Phys ph_host{};
  DevScalars* sc = nullptr;
  DevScalars* sc_host = nullptr;  // pinned
  double* E_host = nullptr;       // pinned staging of fg_set_uniform_E
  double* part_k = nullptr;
  double* part_r = nullptr;
  double* part_ke = nullptr;
  double* part_avg = nullptr;
  unsigned int* done = nullptr;   // last-block tickets: [0] kicks, [1] z k-space, [2] assemble
  double* avg6 = nullptr;
  double* staging = nullptr;      // padded Fortran-layout FP64 (3 components)
  size_t staging_n = 0;
  double* dipoRavg = nullptr;     // FP64 accumulator [3][nsite]
  std::vector<int> h_revx, h_revy, h_revz;
  cudaGraphExec_t g_np = nullptr, g_lf = nullptr, g_force = nullptr, g_vs = nullptr;
  cudaGraphExec_t g_np_multi = nullptr;  // kNpGraphSteps Nose-Poincare steps
  bool tables_ready = false;
  bool force_fresh = false;
  bool np_ready = false;  // DevScalars' pending half step matches the state
  bool pdl = false;       // launch the step kernels as programmatic dependents
  unsigned gen = 0;       // bumped when buffers that graphs hold are replaced
  bool broken = false;    // a reallocation failed half way: refuse further work
  bool store_acouK = false;
  bool wave_dev = false;  // the step graphs start with k_wave_step (fg_set_wave)
  double n_sum_p = 0;
  int NXP = 0, NYP = 0;
  bool bulk_or_film_mirror() const { return P.bulk_or_film == FG_FILM || P.bulk_or_film == FG_EPIT; }
  size_t real_bytes = 0;
  // launch plan (fg_tune, fg_wisdom_import): the z-tile width asked for
  // (0: the widest that fits) and the resident waves of the streaming
  // kernels (0: one block per 256 sites, up to grid_elem)
  int plan_zcw = 0, plan_waves = 1;
  // launch priority of the kernels this context enqueues while use_prio is
  // set (a replica batch's capture: small supercells ahead of large ones)
  bool use_prio = false;
  int launch_prio = 0;
  // sample series (fg_sample): kSampleCols doubles per row, on the device
  double* samples = nullptr;
  int n_samples = 0;
};

namespace {

// wisdom entries: plans of a context stepped alone, of a replica in a batch
enum { PLAN_SOLO = 0, PLAN_BATCH = 1 };
int apply_wisdom(fg_ctx* ctx, int mode);

int fail(fg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(ctx, FG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

#define CKL()                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = cudaGetLastError();                                                          \
    if (e_ != cudaSuccess)                                                                        \
      return fail(ctx, FG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_));     \
  } while (0)

template <typename T>
KMaps kmaps(const fg_ctx* c) {
  return KMaps{c->revx, c->revy, c->revz, c->kvx, c->kvy, c->kvz, c->trx, c->try_, c->trz, c->trz_s, c->kvz_s};
}

int check_device_error(fg_ctx* ctx) {
#if FG_BOUNDS_CHECK
  DevError de{};
  CK(cudaMemcpyFromSymbol(&de, fg::g_fg_err, sizeof(de)));
  if (de.code != 0) {
    char b[128];
    std::snprintf(b, sizeof(b), "device bounds check %d failed at index %lld", de.code, de.idx);
    return fail(ctx, FG_ERR_CUDA, b);
  }
#else
  (void)ctx;
#endif
  return FG_OK;
}

// ------------------------------------------------ FFT kernel dispatch
// Compile-time instances for the cubic supercells 16^3..128^3 of powers of
// two and 24^3, 48^3 (the sizes of the batched sweeps): (m = Lx/2, Ly) =
// (8,16) .. (64,128), (12,24), (24,48) and Lz = 16..128, 24, 48; the
// runtime-plan kernels take every other size.
template <typename T, int MODE, class F>
void with_xy_fwd(int m, int Ly, F f) {
  if (m == 64 && Ly == 128) f(k_xy_fwd<T, MODE, 64, 128>);
  else if (m == 32 && Ly == 64) f(k_xy_fwd<T, MODE, 32, 64>);
  else if (m == 16 && Ly == 32) f(k_xy_fwd<T, MODE, 16, 32>);
  else if (m == 8 && Ly == 16) f(k_xy_fwd<T, MODE, 8, 16>);
  else if (m == 24 && Ly == 48) f(k_xy_fwd<T, MODE, 24, 48>);
  else if (m == 12 && Ly == 24) f(k_xy_fwd<T, MODE, 12, 24>);
  else f(k_xy_fwd<T, MODE, 0, 0>);
}
template <typename T, class F>
void with_xy_inv(int m, int Ly, F f) {
  if (m == 64 && Ly == 128) f(k_xy_inv<T, 64, 128>);
  else if (m == 32 && Ly == 64) f(k_xy_inv<T, 32, 64>);
  else if (m == 16 && Ly == 32) f(k_xy_inv<T, 16, 32>);
  else if (m == 8 && Ly == 16) f(k_xy_inv<T, 8, 16>);
  else if (m == 24 && Ly == 48) f(k_xy_inv<T, 24, 48>);
  else if (m == 12 && Ly == 24) f(k_xy_inv<T, 12, 24>);
  else f(k_xy_inv<T, 0, 0>);
}
template <typename T>
constexpr int z_cw_cap() { return sizeof(T) == 4 ? 8 : 4; }
template <typename T, class F>
void with_z_kspace(int Lz, int cw, bool acou, bool zsite, F f) {
  constexpr int C = z_cw_cap<T>();
  if (zsite) {  // per-site Z*: runtime transforms
    if (acou) f(k_z_kspace<T, 0, 0, true, true>);
    else f(k_z_kspace<T, 0, 0, false, true>);
  } else if (acou) {
    if (cw == C && Lz == 128) f(k_z_kspace<T, 128, C, true>);
    else if (cw == C && Lz == 64) f(k_z_kspace<T, 64, C, true>);
    else if (cw == C && Lz == 32) f(k_z_kspace<T, 32, C, true>);
    else if (cw == C && Lz == 16) f(k_z_kspace<T, 16, C, true>);
    else if (cw == C && Lz == 48) f(k_z_kspace<T, 48, C, true>);
    else if (cw == 4 && Lz == 24) f(k_z_kspace<T, 24, 4, true>);
    else f(k_z_kspace<T, 0, 0, true>);
  } else if (cw == C && Lz == 128) f(k_z_kspace<T, 128, C>);
  else if (sizeof(T) == 4 && cw == 4 && Lz == 128) f(k_z_kspace<T, 128, 4>);
  else if (cw == C && Lz == 64) f(k_z_kspace<T, 64, C>);
  else if (cw == C && Lz == 32) f(k_z_kspace<T, 32, C>);
  else if (cw == C && Lz == 16) f(k_z_kspace<T, 16, C>);
  else if (cw == C && Lz == 48) f(k_z_kspace<T, 48, C>);
  else if (cw == 4 && Lz == 24) f(k_z_kspace<T, 24, 4>);
  else f(k_z_kspace<T, 0, 0>);
}

// The standalone z pass of the 3-component FFT entry points (fg_fft_r2c3,
// fg_fft_c2r3, fg_time_fft): compile-time transforms where the step's own
// z tiles have them, else runtime plans.
template <typename T, bool INV, class F>
void with_z_pass(int Lz, int cw, F f) {
  constexpr int C = z_cw_cap<T>();
  if (cw == C && Lz == 128) f(k_z_pass<T, INV, 128, C, 3>);
  else if (cw == C && Lz == 64) f(k_z_pass<T, INV, 64, C, 3>);
  else if (cw == C && Lz == 32) f(k_z_pass<T, INV, 32, C, 3>);
  else if (cw == C && Lz == 16) f(k_z_pass<T, INV, 16, C, 3>);
  else if (cw == C && Lz == 48) f(k_z_pass<T, INV, 48, C, 3>);
  else if (cw == 4 && Lz == 24) f(k_z_pass<T, INV, 24, 4, 3>);
  else f(k_z_pass<T, INV>);
}

// First component of Z*(R) u in the spectrum and of the long-range dipole
// field in rwork (per-site Z*): after u, u u and the acoustic displacement.
inline int zu_comp(const fg_ctx* ctx) { return ctx->acou ? 12 : 9; }

// Kernel launch that, while ctx->pdl is set, lets the kernel be scheduled
// before its predecessor on the stream has finished (programmatic stream
// serialization).  Only kernels that start with pdl_enter() go through it.
template <typename... KArgs, typename... Args>
void launch_dep(fg_ctx* ctx, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[2];
  unsigned n = 0;
  if (ctx->pdl) {
    at[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  if (ctx->use_prio) {
    at[n].id = cudaLaunchAttributePriority;
    at[n].val.priority = ctx->launch_prio;
    ++n;
  }
  cfg.attrs = at;
  cfg.numAttrs = n;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// zstar: per-site Z*, transformed times u in components zu0..zu0+2
template <typename T, int MODE>
int launch_xy_fwd(fg_ctx* ctx, const T* src, cplx<T>* spec, int ncomp, int smem, const cplx<T>* twx,
                  const cplx<T>* twm, const cplx<T>* twy, const T* zstar = nullptr, int zu0 = 0) {
  const Geom& g = ctx->g;
  with_xy_fwd<T, MODE>(g.m, g.Ly, [&](auto kern) {
    launch_dep(ctx, kern, dim3(g.Lz, ncomp), kThreadsFFT, smem, src, spec, g, ctx->px, ctx->py, twx, twm, twy,
               ctx->posm, 0, zstar, zu0, (const RepArgs*)nullptr);
  });
  CKL();
  return FG_OK;
}

// strain_prologue: block (0, 0) also runs the k-space energies and the
// homogeneous strain from the partials of the preceding k_z_kspace.
template <typename T>
int launch_xy_inv(fg_ctx* ctx, const cplx<T>* spec, T* out, int ncomp, bool strain_prologue = false) {
  const Geom& g = ctx->g;
  with_xy_inv<T>(g.m, g.Ly, [&](auto kern) {
    launch_dep(ctx, kern, dim3(g.Lz, ncomp), kThreadsFFT, ctx->smem_xy,
        spec, out, g, ctx->px, ctx->py, (const cplx<T>*)ctx->twx, (const cplx<T>*)ctx->twm, (const cplx<T>*)ctx->twy,
        ctx->posm, 0, strain_prologue ? ctx->ph : nullptr, ctx->sc, ctx->part_k, ctx->zt.nreg + ctx->zt.nnyq,
        (const RepArgs*)nullptr);
  });
  CKL();
  return FG_OK;
}

// The k-space partials are finished by the next k_xy_inv (strain prologue).
template <typename T>
int launch_z_kspace(fg_ctx* ctx, cplx<T>* acouK_out) {
  const Geom& g = ctx->g;
  with_z_kspace<T>(g.Lz, ctx->zt.CW, ctx->acou, ctx->zsite, [&](auto kern) {
    launch_dep(ctx, kern, ctx->zt.nreg + ctx->zt.nnyq, kThreadsZ, ctx->smem_z,
        (cplx<T>*)ctx->spec, (const T*)ctx->dtab, (const cplx<T>*)ctx->ckmod, acouK_out, g, ctx->pz,
        (const cplx<T>*)ctx->twz, kmaps<T>(ctx), ctx->ph, ctx->part_k, ctx->sc, ctx->zt, nullptr,
        (const T*)ctx->ltab, (const RepArgs*)nullptr);
  });
  CKL();
  return FG_OK;
}

// ----------------------------------------------------------- force pipeline
// k_assemble on the context's arrays; CLOSE: with the closing kick of a
// Nose-Poincare step and the step's tails
// Static constants of the site force (dVddi-unharmonic.F:28-32,67-99,
// elastic.F:60-75) from the context's Phys, passed to k_assemble by value.
AsmConst asm_const(const fg_ctx* ctx) {
  const Phys& h = ctx->ph_host;
  AsmConst k{};
  k.pl = Poly{h.fa2g, h.tg, h.sk, h.tk2, h.fk, 8 * h.P_k4, h.P_alpha, h.P_gamma, h.P_k1, h.P_k2, h.P_k3, h.P_k4};
  k.hx = h.HC2[0][0]; k.hy = h.HC2[0][1]; k.h4 = h.HC2[3][3];
  k.Zs = h.Zstar;
  k.E_on = h.E_on;
  return k;
}

// flo: also store the FP32 residual of the force (mixed path)
template <typename T, bool CLOSE>
void launch_assemble(fg_ctx* ctx, int tail, bool flo = false) {
  const bool sites = ctx->site_species || ctx->site_zstar || ctx->site_E ||
                     (CLOSE && (ctx->site_minv || ctx->site_sump));
  launch_dep(ctx, sites ? k_assemble<T, CLOSE, true> : k_assemble<T, CLOSE, false>,
             CLOSE ? ctx->grid_asc : ctx->grid_as, kThreadsElem, 0, (const T*)ctx->rwork, (const T*)ctx->u, (T*)ctx->F, ctx->g, ctx->ph, ctx->sc, ctx->part_r, tail,
             ctx->done + 2, ctx->site_species, (const T*)ctx->site_zstar, (const T*)ctx->site_E,
             ctx->zsite ? zu_comp(ctx) : 0, (T*)ctx->p, ctx->layer_minv, ctx->layer_sump, (const T*)ctx->site_minv,
             ctx->site_sump, ctx->part_ke, (flo && sizeof(T) == 4) ? (T*)ctx->Flo : (T*)nullptr, asm_const(ctx),
             (const RepArgs*)nullptr);
}

// Force modes: FORCE_PLAIN finishes the energies in k_assemble's tail;
// FORCE_NP_POST leaves them to a following closing kick (k_kick_close);
// FORCE_NP_CLOSE runs the closing kick and the step's tails in k_assemble.
enum { FORCE_PLAIN = 0, FORCE_NP_POST = 1, FORCE_NP_CLOSE = 2 };

// flo: the force-only evaluation of fg_mirror_force_mirror, which keeps the
// FP32 residual of the mixed path's force for fg_get_state
template <typename T>
int enqueue_force(fg_ctx* ctx, int mode = FORCE_PLAIN, bool flo = false) {
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  T* u = (T*)ctx->u;
  if (ctx->P.bulk_or_film == FG_FILM || ctx->P.bulk_or_film == FG_EPIT) {
    k_mirror<T><<<ctx->grid_elem, kThreadsElem, 0, st>>>(u, g, ctx->P.gap_id);
    CKL();
  }
  int rc;
  if ((rc = launch_xy_fwd<T, SRC_U9>(ctx, u, (cplx<T>*)ctx->spec, ctx->ncx, ctx->smem_xy, (const cplx<T>*)ctx->twx,
                                     (const cplx<T>*)ctx->twm, (const cplx<T>*)ctx->twy,
                                     ctx->zsite ? (const T*)ctx->site_zstar : nullptr, zu_comp(ctx))))
    return rc;
  if ((rc = launch_z_kspace<T>(ctx, ctx->store_acouK ? (cplx<T>*)ctx->acouK : nullptr))) return rc;
  if ((rc = launch_xy_inv<T>(ctx, (const cplx<T>*)ctx->spec, (T*)ctx->rwork, ctx->ncx, true))) return rc;
  if (mode == FORCE_NP_CLOSE) launch_assemble<T, true>(ctx, TAIL_NONE);
  else launch_assemble<T, false>(ctx, mode == FORCE_NP_POST ? TAIL_NONE : TAIL_ENERGIES, flo);
  CKL();
  if (ctx->P.bulk_or_film == FG_FILM || ctx->P.bulk_or_film == FG_EPIT) {
    k_mirror<T><<<ctx->grid_elem, kThreadsElem, 0, st>>>((T*)ctx->F, g, ctx->P.gap_id);
    CKL();
    if (flo && sizeof(T) == 4) {
      k_mirror<T><<<ctx->grid_elem, kThreadsElem, 0, st>>>((T*)ctx->Flo, g, ctx->P.gap_id);
      CKL();
    }
  }
  return FG_OK;
}

template <typename T>
int enqueue_kick(fg_ctx* ctx, const double* coef, int tail = TAIL_NONE, int zero_unmasked = 0) {
  k_kick<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
      (T*)ctx->p, (const T*)ctx->F, coef, ctx->g, ctx->layer_minv, ctx->layer_sump, ctx->part_ke, tail, ctx->done,
      ctx->ph, ctx->sc, zero_unmasked, (const T*)ctx->site_minv, ctx->site_sump);
  CKL();
  return FG_OK;
}

template <typename T>
int enqueue_drift(fg_ctx* ctx, const double* coef) {
  k_drift<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((T*)ctx->u, (const T*)ctx->p, coef, ctx->g,
                                                                ctx->layer_minv, (const T*)ctx->site_minv);
  CKL();
  return FG_OK;
}

// Acoustic momenta and displacements (acouP, acouR: components 3..5 of p and
// u): kick by dVdacR (rwork components 9..11), no sum_p mask, uniform mass.
template <typename T>
int enqueue_kick_acou(fg_ctx* ctx, const double* coef, int tail) {
  const long long ns = ctx->g.nsite;
  k_kick<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
      (T*)ctx->p + 3 * ns, (const T*)ctx->rwork + 9 * ns, coef, ctx->g, ctx->layer_macou, ctx->layer_all,
      ctx->part_ke, tail, ctx->done, ctx->ph, ctx->sc, 0, (const T*)ctx->site_macou, nullptr);
  CKL();
  return FG_OK;
}

template <typename T>
int enqueue_drift_acou(fg_ctx* ctx, const double* coef) {
  const long long ns = ctx->g.nsite;
  k_drift<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((T*)ctx->u + 3 * ns, (const T*)ctx->p + 3 * ns, coef,
                                                                ctx->g, ctx->layer_macou, (const T*)ctx->site_macou);
  CKL();
  return FG_OK;
}

// leapfrog.F:44-87 heat pump, when delta_e or delta_e_acou is set
template <typename T>
int enqueue_pump(fg_ctx* ctx) {
  const fg_params& P = ctx->P;
  if (P.delta_e == 0.0 && P.delta_e_acou == 0.0) return FG_OK;
  const long long ns = ctx->g.nsite;
  k_layer_pump<T><<<2, kThreadsElem, 0, ctx->stream>>>((T*)ctx->p, ctx->acou ? (T*)ctx->p + 3 * ns : nullptr, ctx->g,
                                                        ctx->layer_minv, ctx->layer_macou, ctx->layer_sump, P.delta_e,
                                                        P.delta_e_acou, (const T*)ctx->site_minv,
                                                        (const T*)ctx->site_macou, ctx->layer_nsum);
  CKL();
  return FG_OK;
}

// The device-side field schedule at the start of a step (fg_set_wave).
int enqueue_wave(fg_ctx* ctx) {
  if (!ctx->wave_dev) return FG_OK;
  k_wave_step<<<1, 32, 0, ctx->stream>>>(ctx->ph, ctx->sc);
  CKL();
  return FG_OK;
}

template <typename T>
int enqueue_kick_drift(fg_ctx* ctx) {
  launch_dep(ctx, k_kick_drift<T>, ctx->grid_kd, kThreadsElem, 0, (T*)ctx->p, (T*)ctx->u, (const T*)ctx->F,
             ctx->sc, ctx->g, ctx->layer_minv, (const T*)ctx->site_minv, (const RepArgs*)nullptr);
  CKL();
  return FG_OK;
}

// prep: sums of the current state only (np_prepare)
template <typename T, bool PREP>
int enqueue_kick_close(fg_ctx* ctx) {
  launch_dep(ctx, k_kick_close<T, PREP>, ctx->grid_kc, kThreadsElem, 0,
      (T*)ctx->p, (const T*)ctx->F, ctx->g, ctx->layer_minv, ctx->layer_sump, ctx->part_ke, ctx->done, ctx->ph,
      ctx->sc, ctx->part_r, ctx->grid_as, (const T*)ctx->site_minv, ctx->site_sump);
  CKL();
  return FG_OK;
}

// nose_poincare (nose-poincare.F:24-75) as one graph of six kernels:
//   k_kick_drift       (35a) + (35c) with the coefficients prepared by the
//                      previous closing tail ((38) solved there)
//   force              xy_fwd, z_kspace, xy_inv (+ homogeneous strain),
//                      k_assemble (partials only)
//   k_kick_close       block 0: energies, commit of the half step, (35e);
//                      all: (35f) and the three kinetic sums; last block:
//                      KE, H_NP of this step and the scalars of the next.
//
// Each kernel after the first starts while its predecessor drains
// (programmatic dependent launch); follows_step: the step continues a graph
// of several steps, and its first kernel does the same after the previous
// step's closing kick.
template <typename T>
int enqueue_np(fg_ctx* ctx, bool follows_step = false) {
  const bool pdl = !ctx->bulk_or_film_mirror();
  int rc = enqueue_wave(ctx);
  if (rc) return rc;
  ctx->pdl = pdl && follows_step && !ctx->wave_dev;
  rc = enqueue_kick_drift<T>(ctx);
  ctx->pdl = pdl;
  // bulk: the closing kick runs inside k_assemble; films mirror the force
  // first, so the kick is a kernel of its own
  const bool fused = !ctx->bulk_or_film_mirror();
  if (!rc) rc = enqueue_force<T>(ctx, fused ? FORCE_NP_CLOSE : FORCE_NP_POST);
  if (!rc && !fused) rc = enqueue_kick_close<T, false>(ctx);
  ctx->pdl = false;
  return rc;
}

// Steps per graph launch of fg_run_steps / fg_time_steps (Nose-Poincare).
constexpr int kNpGraphSteps = 8;

// leapfrog (leapfrog.F:103-151), i_step != 0
template <typename T>
int enqueue_lf(fg_ctx* ctx) {
  int rc;
  if ((rc = enqueue_wave(ctx))) return rc;
  if ((rc = enqueue_pump<T>(ctx))) return rc;
  if ((rc = enqueue_drift<T>(ctx, &ctx->sc->lf_dt))) return rc;
  if (ctx->acou && (rc = enqueue_drift_acou<T>(ctx, &ctx->sc->lf_dt))) return rc;
  if ((rc = enqueue_force<T>(ctx))) return rc;
  if (ctx->acou && (rc = enqueue_kick_acou<T>(ctx, &ctx->sc->lf_dt, TAIL_ACOU))) return rc;
  if ((rc = enqueue_kick<T>(ctx, &ctx->sc->lf_dt, TAIL_LF_FINAL))) return rc;
  return FG_OK;
}

// velocity_scaling (velocity_scaling.F:9-103), acoustic mass <= 0: drift by
// dt, force, kick by dt with p = 0 outside sum_p, rescale p to the target
// kinetic energy.
template <typename T>
int enqueue_vs(fg_ctx* ctx) {
  int rc;
  if ((rc = enqueue_wave(ctx))) return rc;
  if ((rc = enqueue_drift<T>(ctx, &ctx->sc->lf_dt))) return rc;
  if (ctx->acou && (rc = enqueue_drift_acou<T>(ctx, &ctx->sc->lf_dt))) return rc;
  if ((rc = enqueue_force<T>(ctx))) return rc;
  if ((rc = enqueue_kick<T>(ctx, &ctx->sc->lf_dt, TAIL_VS, 1))) return rc;
  k_scale<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((T*)ctx->p, &ctx->sc->vs_scale, 3 * ctx->g.nsite);
  CKL();
  if (ctx->acou) {
    if ((rc = enqueue_kick_acou<T>(ctx, &ctx->sc->lf_dt, TAIL_VS_ACOU))) return rc;
    k_scale<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((T*)ctx->p + 3 * ctx->g.nsite, &ctx->sc->vs_scale_acou,
                                                                  3 * ctx->g.nsite);
    CKL();
  }
  return FG_OK;
}

// ---------------------------------------------------------- grouped steps
// A bulk Nose-Poincare step of nrep replicas of c0's size, precision and
// material as one launch per kernel (the fused five-kernel step of
// enqueue_np), each replica's buffers taken from the device table grp.
template <typename T>
int enqueue_np_group(fg_ctx* c0, const RepArgs* grp, int nrep) {
  fg_ctx* ctx = c0;  // for CKL
  const Geom& g = c0->g;
  c0->pdl = false;
  launch_dep(c0, k_kick_drift<T>, dim3(c0->grid_kd, nrep), kThreadsElem, 0, (T*)nullptr, (T*)nullptr,
             (const T*)nullptr, (const DevScalars*)nullptr, g, (const double*)nullptr, (const T*)nullptr, grp);
  CKL();
  c0->pdl = true;
  with_xy_fwd<T, SRC_U9>(g.m, g.Ly, [&](auto kern) {
    launch_dep(c0, kern, dim3(g.Lz, c0->ncx, nrep), kThreadsFFT, c0->smem_xy, (const T*)nullptr, (cplx<T>*)nullptr,
               g, c0->px, c0->py, (const cplx<T>*)c0->twx, (const cplx<T>*)c0->twm, (const cplx<T>*)c0->twy,
               c0->posm, 0, (const T*)nullptr, 0, grp);
  });
  CKL();
  with_z_kspace<T>(g.Lz, c0->zt.CW, false, false, [&](auto kern) {
    launch_dep(c0, kern, dim3(c0->zt.nreg + c0->zt.nnyq, nrep), kThreadsZ, c0->smem_z, (cplx<T>*)nullptr,
               (const T*)nullptr, (const cplx<T>*)c0->ckmod, (cplx<T>*)nullptr, g, c0->pz, (const cplx<T>*)c0->twz,
               kmaps<T>(c0), (const Phys*)nullptr, (double*)nullptr, (DevScalars*)nullptr, c0->zt,
               (unsigned int*)nullptr, (const T*)nullptr, grp);
  });
  CKL();
  with_xy_inv<T>(g.m, g.Ly, [&](auto kern) {
    launch_dep(c0, kern, dim3(g.Lz, c0->ncx, nrep), kThreadsFFT, c0->smem_xy, (const cplx<T>*)nullptr, (T*)nullptr, g,
               c0->px, c0->py, (const cplx<T>*)c0->twx, (const cplx<T>*)c0->twm, (const cplx<T>*)c0->twy, c0->posm,
               0, (const Phys*)c0->ph, (DevScalars*)nullptr, (const double*)nullptr, c0->zt.nreg + c0->zt.nnyq, grp);
  });
  CKL();
  launch_dep(c0, k_assemble<T, true>, dim3(c0->grid_asc, nrep), kThreadsElem, 0, (const T*)nullptr,
             (const T*)nullptr, (T*)nullptr, g, (const Phys*)nullptr, (DevScalars*)nullptr, (double*)nullptr,
             (int)TAIL_NONE, (unsigned int*)nullptr, (const unsigned char*)nullptr, (const T*)nullptr,
             (const T*)nullptr, 0, (T*)nullptr, (const double*)nullptr, (const unsigned char*)nullptr,
             (const T*)nullptr, (const unsigned char*)nullptr, (double*)nullptr, (T*)nullptr, asm_const(c0), grp);
  CKL();
  c0->pdl = false;
  return FG_OK;
}

// A replica that a grouped launch can step: bulk Nose-Poincare without the
// acoustic field, per-site arrays, modulation or a device field schedule.
bool groupable(const fg_ctx* c) {
  return c->P.method == FG_METHOD_MD && !c->bulk_or_film_mirror() && !c->acou && !c->zsite && !c->site_species &&
         !c->site_zstar && !c->site_E && !c->site_minv && !c->site_sump && !c->wave_dev &&
         c->ph_host.modulation_on == 0 && !c->broken;
}
// Replicas a and b step together: same size, precision and site constants.
bool same_group(const fg_ctx* a, const fg_ctx* b) {
  if (a->prec != b->prec || a->g.Lx != b->g.Lx || a->g.Ly != b->g.Ly || a->g.Lz != b->g.Lz) return false;
  // one launch covers the group with the first replica's tiles and grids
  if (a->zt.CW != b->zt.CW || a->grid_kd != b->grid_kd || a->grid_asc != b->grid_asc) return false;
  const AsmConst ka = asm_const(a), kb = asm_const(b);
  return std::memcmp(&ka, &kb, sizeof(AsmConst)) == 0;
}
RepArgs rep_args(const fg_ctx* c) {
  RepArgs a{};
  a.u = c->u;
  a.p = c->p;
  a.F = c->F;
  a.spec = c->spec;
  a.rwork = c->rwork;
  a.dtab = c->dtab;
  a.ph = c->ph;
  a.sc = c->sc;
  a.part_k = c->part_k;
  a.part_r = c->part_r;
  a.part_ke = c->part_ke;
  a.done_as = c->done + 2;
  a.layer_minv = c->layer_minv;
  a.layer_sump = c->layer_sump;
  return a;
}

// Capture fn into a CUDA graph executable (once per context).
template <typename Fn>
int capture(fg_ctx* ctx, cudaGraphExec_t* out, Fn fn) {
  if (*out) return FG_OK;
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = fn();
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return FG_OK;
}

int run_graph(fg_ctx* ctx, cudaGraphExec_t* gx, int which) {
  int rc = FG_OK;
  if (which == 0) {
    rc = capture(ctx, gx, [&] {
      return ctx->prec == FG_PREC_MIXED ? enqueue_force<float>(ctx, FORCE_PLAIN, true) : enqueue_force<double>(ctx);
    });
  } else if (which == 1) {
    rc = capture(ctx, gx, [&] { return ctx->prec == FG_PREC_MIXED ? enqueue_np<float>(ctx) : enqueue_np<double>(ctx); });
  } else if (which == 4) {
    rc = capture(ctx, gx, [&] {
      int r = FG_OK;
      for (int k = 0; k < kNpGraphSteps && r == FG_OK; ++k)
        r = ctx->prec == FG_PREC_MIXED ? enqueue_np<float>(ctx, k > 0) : enqueue_np<double>(ctx, k > 0);
      return r;
    });
  } else if (which == 2) {
    rc = capture(ctx, gx, [&] { return ctx->prec == FG_PREC_MIXED ? enqueue_lf<float>(ctx) : enqueue_lf<double>(ctx); });
  } else {
    rc = capture(ctx, gx, [&] { return ctx->prec == FG_PREC_MIXED ? enqueue_vs<float>(ctx) : enqueue_vs<double>(ctx); });
  }
  if (rc) return rc;
  CK(cudaGraphLaunch(*gx, ctx->stream));
  return FG_OK;
}

int pull_scalars(fg_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->sc_host, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int rc = check_device_error(ctx);
  if (rc) return rc;
  if (ctx->sc_host->status == 10)
    return fail(ctx, FG_ERR_NAN, "Nose-Poincare update (38): 1 - CB dt/Q < 0, Q_Nose is too small for this supercell");
  if (ctx->sc_host->status == FG_ERR_NAN) return fail(ctx, FG_ERR_NAN, "non-finite energy in a device reduction");
  return FG_OK;
}

int push_scalars(fg_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->sc, ctx->sc_host, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FG_OK;
}

void energy_out(const DevScalars* s, fg_energy* e, bool potential_only) {
  double* d = &e->acou_kinetic;
  for (int i = 0; i < E_COUNT; ++i) {
    if (potential_only && (i < E_SHORT || i > E_IM)) continue;
    d[i] = s->e[i];
  }
}

template <typename T>
void* dalloc(fg_ctx* ctx, size_t n, int* rc) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) {
    *rc = fail(ctx, FG_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return nullptr;
  }
  return p;
}

template <typename V>
int upload(fg_ctx* ctx, void** dst, const std::vector<V>& v) {
  CK(cudaMalloc(dst, v.size() * sizeof(V)));
  CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice));
  return FG_OK;
}

// host analytic k vectors and trig tables
double kvec_wrapped(int i, int L, double a0) {  // elastic.F:81-85
  double k = (double)i / L;
  if (k > 0.5) k = k - 1.0;
  return k * 6.28318530717958647693 / a0;
}

int validate(const fg_params* p, std::string* why) {
  if (p->N != p->Lx * p->Ly * p->Lz || p->N <= 0) { *why = "parameters not made (call fg_make_param)"; return FG_ERR_ARG; }
  if (p->Lx % 2 != 0 || p->Lx < 4) { *why = "Lx must be even and >= 4"; return FG_ERR_UNSUPPORTED; }
  if (p->Ly < 3 || p->Lz < 3) { *why = "Ly and Lz must be >= 3"; return FG_ERR_UNSUPPORTED; }
  if (p->method != FG_METHOD_MD && p->method != FG_METHOD_LF && p->method != FG_METHOD_VS && p->method != FG_METHOD_HL) {
    *why = "unknown method";
    return FG_ERR_UNSUPPORTED;
  }
  if (p->mass_acou[0] > 0.0 && p->method == FG_METHOD_MD) {
    *why = "acoustic_mass_amu with method 'md' (param_module.F:239-242)";
    return FG_ERR_ARG;
  }
  if ((p->delta_e != 0.0 || p->delta_e_acou != 0.0) && (p->Lz < 4 || p->method != FG_METHOD_LF)) {
    *why = "delta_e pumps heat in leapfrog runs with Lz >= 4 only";
    return FG_ERR_UNSUPPORTED;
  }
  if (p->dt <= 0.0) { *why = "dt must be positive"; return FG_ERR_ARG; }
  if (p->method == FG_METHOD_MD && p->Q_Nose <= 0.0) { *why = "Q_Nose must be positive"; return FG_ERR_ARG; }
  return FG_OK;
}

// The widest z tile the context's plan allows.
template <typename T>
int plan_cw(const fg_ctx* ctx) {
  return ctx->plan_zcw > 0 ? std::min(ctx->plan_zcw, z_cw_cap<T>()) : z_cw_cap<T>();
}

// z tiles: CW is the largest power of two <= cwmax dividing Lx/2 whose
// tile of nc components fits in shared memory
ZTiles z_tiles(const Geom& g, int nc, size_t esz, int cwmax, int smem_max) {
  ZTiles t{};
  int cw = cwmax;
  while (cw > 1 && (g.m % cw != 0 || (size_t)nc * g.Lz * cw * esz > (size_t)smem_max)) cw /= 2;
  t.CW = cw;
  t.ntx = g.m / cw;
  t.nreg = t.ntx * g.Ly;
  t.nnyq = div_up(g.Ly, cw);
  return t;
}

// Grids of the streaming kernels (grid-stride loops): `waves` resident
// waves of blocks, or (waves = 0) one block per kThreadsElem sites, never
// more than grid_elem (the size of the per-block partial-sum buffers).
template <typename T>
void plan_grids(fg_ctx* ctx, int waves, int nsm) {
  const int all = std::max(1, std::min(ctx->grid_elem, div_up(ctx->g.nsite, kThreadsElem)));
  auto grid = [&](auto kern) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kThreadsElem, 0) != cudaSuccess || nb < 1) nb = 8;
    return waves <= 0 ? all : std::max(1, std::min(all, waves * nb * nsm));
  };
  ctx->grid_kd = grid(k_kick_drift<T>);
  ctx->grid_kc = std::min(grid(k_kick_close<T, false>), grid(k_kick_close<T, true>));
  ctx->grid_as = grid(k_assemble<T, false>);
  ctx->grid_asc = grid(k_assemble<T, true>);
  ctx->plan_waves = waves;
}

template <typename T>
int create_impl(fg_ctx* ctx) {
  const fg_params& P = ctx->P;
  Geom& g = ctx->g;
  g.Lx = P.Lx;
  g.Ly = P.Ly;
  g.Lz = P.Lz;
  g.m = P.Lx / 2;
  g.NKX = g.m + 1;
  g.KXP = (g.NKX + 15) / 16 * 16;
  g.plane_r = (long long)g.Lx * g.Ly;
  g.plane_c = (long long)g.Ly * g.KXP;
  g.nsite = (long long)g.Lx * g.Ly * g.Lz;
  g.ncplx = (long long)g.Lz * g.plane_c;
  g.nkpos = (long long)g.Ly * g.Lz * g.KXP;
  ctx->NXP = 2 * (P.Lx / 2 + 1);
  ctx->NYP = P.Ly + P.padding_y;
  if (!make_plan(g.m, &ctx->px) || !make_plan(g.Ly, &ctx->py) || !make_plan(g.Lz, &ctx->pz))
    return fail(ctx, FG_ERR_UNSUPPORTED, "L/2 (x), Ly and Lz must factor into 2, 3 and 5");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  int smem_max = 0, nsm = 0;
  CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int smem_optin = smem_max;
  smem_max -= 8192;  // static shared memory: twiddles, block reductions, scalar tails
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ctx->smem_xy = (int)(sizeof(cplx<T>) * g.Ly * (g.m + 1));
  ctx->smem_xy64 = (int)(sizeof(cplx<double>) * g.Ly * (g.m + 1));
  if (ctx->smem_xy > smem_max || ctx->smem_xy64 > smem_max)
    return fail(ctx, FG_ERR_UNSUPPORTED, "an x-y plane of the supercell does not fit in shared memory");
  auto tiles = [&](int nc, size_t esz, int cwmax) { return z_tiles(g, nc, esz, cwmax, smem_max); };
  ctx->acou = P.mass_acou[0] > 0.0;
  ctx->ncx = ctx->acou ? 12 : 9;
  ctx->zt = tiles(ctx->ncx, sizeof(cplx<T>), plan_cw<T>(ctx));
  ctx->zt6 = tiles(6, sizeof(cplx<double>), 8);
  ctx->zt1 = tiles(1, sizeof(cplx<double>), 8);
  if ((size_t)ctx->ncx * g.Lz * ctx->zt.CW * sizeof(cplx<T>) > (size_t)smem_max)
    return fail(ctx, FG_ERR_UNSUPPORTED, "a z pencil of the supercell does not fit in shared memory");
  ctx->smem_z = (int)(ctx->ncx * ((size_t)g.Lz * ctx->zt.CW + kZPad<T>) * sizeof(cplx<T>));
  ctx->smem_z3 = (int)(3 * (size_t)g.Lz * ctx->zt.CW * sizeof(cplx<T>));
  ctx->smem_z6 = (int)(6 * (size_t)g.Lz * ctx->zt6.CW * sizeof(cplx<double>));
  ctx->smem_z1 = (int)(1 * (size_t)g.Lz * ctx->zt1.CW * sizeof(cplx<double>));
  ctx->grid_elem = std::max(1, std::min(div_up(g.nsite, kThreadsElem), nsm * 8));
  plan_grids<T>(ctx, ctx->plan_waves, nsm);
  {
    // The dynamic shared-memory cap is an attribute of the kernel, shared by
    // every context in the process: raise it to what the device allows next
    // to the kernel's static shared memory, never to this context's size
    // (a smaller supercell would lower it under a larger one's launches).
    cudaError_t ea = cudaSuccess;
    auto setattr = [&](auto kern, int bytes) {
      cudaFuncAttributes fa;
      cudaError_t e = cudaFuncGetAttributes(&fa, kern);
      const int cap = smem_optin - (int)fa.sharedSizeBytes;
      if (e == cudaSuccess && bytes > cap) e = cudaErrorInvalidValue;
      if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
      if (e != cudaSuccess) ea = e;
    };
    with_xy_fwd<T, SRC_U9>(g.m, g.Ly, [&](auto k) { setattr(k, ctx->smem_xy); });
    with_xy_fwd<T, SRC_FIELD>(g.m, g.Ly, [&](auto k) { setattr(k, ctx->smem_xy); });
    with_xy_fwd<double, SRC_FIELD>(g.m, g.Ly, [&](auto k) { setattr(k, ctx->smem_xy64); });
    with_xy_inv<T>(g.m, g.Ly, [&](auto k) { setattr(k, ctx->smem_xy); });
    with_z_kspace<T>(g.Lz, ctx->zt.CW, ctx->acou, false, [&](auto k) { setattr(k, ctx->smem_z); });
    with_z_pass<T, false>(g.Lz, ctx->zt.CW, [&](auto k) { setattr(k, ctx->smem_z3); });
    with_z_pass<T, true>(g.Lz, ctx->zt.CW, [&](auto k) { setattr(k, ctx->smem_z3); });
    setattr(k_z_ewald_pack<T>, ctx->smem_z6);
    setattr(k_z_modulation_pack<T>, ctx->smem_z1);
    if (ea != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  }
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));

  // slot maps
  // posm: [0, m) the slot of each packed-x frequency; then the y maps of
  // the xy kernels, [m, m + Ly) slot -> ky and [m + Ly, m + 2 Ly) ky -> slot
  std::vector<int> revm = digit_reversal(ctx->px);
  ctx->h_revx.resize(g.NKX);
  for (int s = 0; s < g.m; ++s) ctx->h_revx[s] = revm[s];
  ctx->h_revx[g.m] = g.m;
  ctx->h_revy = digit_reversal(ctx->py);
  ctx->h_revz = digit_reversal(ctx->pz);
  std::vector<int> posm(g.m + 2 * (size_t)g.Ly);
  for (int s = 0; s < g.m; ++s) posm[revm[s]] = s;
  for (int s = 0; s < g.Ly; ++s) {
    posm[g.m + s] = ctx->h_revy[s];
    posm[g.m + g.Ly + ctx->h_revy[s]] = s;
  }
  int rc;
  if ((rc = upload(ctx, (void**)&ctx->revx, ctx->h_revx))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->revy, ctx->h_revy))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->revz, ctx->h_revz))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->posm, posm))) return rc;
  // twiddles
  if ((rc = upload(ctx, &ctx->twx, twiddles<T>(g.Lx)))) return rc;
  if ((rc = upload(ctx, &ctx->twm, twiddles<T>(g.m)))) return rc;
  if ((rc = upload(ctx, &ctx->twy, twiddles<T>(g.Ly)))) return rc;
  if ((rc = upload(ctx, &ctx->twz, twiddles<T>(g.Lz)))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->twx64, twiddles<double>(g.Lx)))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->twm64, twiddles<double>(g.m)))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->twy64, twiddles<double>(g.Ly)))) return rc;
  if ((rc = upload(ctx, (void**)&ctx->twz64, twiddles<double>(g.Lz)))) return rc;
  // wavevectors and trig tables (true-k indexed)
  {
    std::vector<double> kx(g.NKX), ky(g.Ly), kz(g.Lz);
    for (int i = 0; i < g.NKX; ++i) kx[i] = (double)i / P.Lx * 6.28318530717958647693 / P.a0;  // elastic.F:87
    for (int i = 0; i < g.Ly; ++i) ky[i] = kvec_wrapped(i, P.Ly, P.a0);
    for (int i = 0; i < g.Lz; ++i) kz[i] = kvec_wrapped(i, P.Lz, P.a0);
    auto trig = [](int n, int L) {
      std::vector<double2> t(n);
      for (int i = 0; i < n; ++i) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)i / (long double)L;
        t[i] = make_double2((double)std::cos(a), (double)std::sin(a));
      }
      return t;
    };
    if ((rc = upload(ctx, (void**)&ctx->kvx, kx))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->kvy, ky))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->kvz, kz))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->trx, trig(g.NKX, P.Lx)))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->try_, trig(g.Ly, P.Ly)))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->trz, trig(g.Lz, P.Lz)))) return rc;
    {
      const std::vector<double2> tz = trig(g.Lz, P.Lz);
      std::vector<double2> tzs(g.Lz);
      std::vector<double> kzs(g.Lz);
      for (int sl = 0; sl < g.Lz; ++sl) {
        tzs[sl] = tz[ctx->h_revz[sl]];
        kzs[sl] = kz[ctx->h_revz[sl]];
      }
      if ((rc = upload(ctx, (void**)&ctx->trz_s, tzs))) return rc;
      if ((rc = upload(ctx, (void**)&ctx->kvz_s, kzs))) return rc;
    }
  }
  // per-layer masses and masks (alloc_Coord, read_defects_u.F:52-69)
  {
    std::vector<double> minv(g.Lz, 1.0 / P.mass_dipo[0]);
    std::vector<unsigned char> sump(g.Lz, 1);
    if (P.bulk_or_film == FG_FILM || P.bulk_or_film == FG_EPIT)
      for (int z = (P.Lz + 1) / 2; z < P.Lz; ++z) sump[z] = 0;
    if (P.gap_id > 0) {
      minv[0] = 0.0;
      sump[0] = 0;
      if (P.gap_id == 2) {
        minv[P.Lz / 2] = 0.0;
        sump[P.Lz / 2] = 0;
      }
    }
    double n = 0;
    for (int z = 0; z < g.Lz; ++z) n += sump[z] ? (double)g.plane_r : 0.0;
    ctx->n_sum_p = n;
    if ((rc = upload(ctx, (void**)&ctx->layer_minv, minv))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->layer_sump, sump))) return rc;
    // acoustic masses are the same on every site (alloc_Coord)
    std::vector<double> mai(g.Lz, P.mass_acou[0] > 0.0 ? 1.0 / P.mass_acou[0] : 0.0);
    std::vector<unsigned char> all(g.Lz, 1);
    if ((rc = upload(ctx, (void**)&ctx->layer_macou, mai))) return rc;
    if ((rc = upload(ctx, (void**)&ctx->layer_all, all))) return rc;
  }
  // physics constants (elastic.F:26-75, dVddi-unharmonic.F:28-32)
  {
    Phys& h = ctx->ph_host;
    std::memset(&h, 0, sizeof(h));
    h.N = P.N;
    h.Ninv = P.Ninv;
    for (int i = 0; i < 7; ++i) h.j[i] = P.j[i];
    h.kap2x2 = P.P_kappa2[0] * 2;
    h.P_alpha = P.P_alpha[0];
    h.P_gamma = P.P_gamma[0];
    h.P_k1 = P.P_k1[0];
    h.P_k2 = P.P_k2[0];
    h.P_k3 = P.P_k3[0];
    h.P_k4 = P.P_k4[0];
    h.fa2g = 4 * P.P_alpha[0] + 2 * P.P_gamma[0];
    h.tg = 2 * P.P_gamma[0];
    h.sk = 6 * P.P_k1[0] + 2 * P.P_k2[0];
    h.tk2 = 2 * P.P_k2[0];
    h.fk = 4 * P.P_k2[0] - 2 * P.P_k3[0];
    for (int sp = 0; sp < FG_RELAXOR_MAX; ++sp) {
      Phys::Species& q = h.sp[sp];
      q.fa2g = 4 * P.P_alpha[sp] + 2 * P.P_gamma[sp];
      q.tg = 2 * P.P_gamma[sp];
      q.sk = 6 * P.P_k1[sp] + 2 * P.P_k2[sp];
      q.tk2 = 2 * P.P_k2[sp];
      q.fk = 4 * P.P_k2[sp] - 2 * P.P_k3[sp];
      q.k4x8 = 8 * P.P_k4[sp];
      q.Pa = P.P_alpha[sp];
      q.Pg = P.P_gamma[sp];
      q.P1 = P.P_k1[sp];
      q.P2 = P.P_k2[sp];
      q.P3 = P.P_k3[sp];
      q.P4 = P.P_k4[sp];
      q.dk2 = P.P_kappa2[sp] - P.P_kappa2[0];
    }
    h.B11 = P.B11;
    h.B12 = P.B12;
    h.B44 = P.B44;
    for (int i = 0; i < 3; ++i) h.HC2[i][i] = P.B1xx / 2;
    for (int i = 3; i < 6; ++i) h.HC2[i][i] = P.B4yz;
    h.HC2[0][1] = h.HC2[0][2] = h.HC2[1][2] = h.HC2[1][0] = h.HC2[2][0] = h.HC2[2][1] = P.B1yy / 2;
    for (int i = 0; i < 3; ++i) h.H[i][i] = P.B11 * P.N;
    for (int i = 3; i < 6; ++i) h.H[i][i] = P.B44 * P.N;
    h.H[0][1] = h.H[0][2] = h.H[1][2] = h.H[1][0] = h.H[2][0] = h.H[2][1] = P.B12 * P.N;
    for (int jj = 0; jj < 6; ++jj) {
      double s = 0.0;
      for (int k = 0; k < jj; ++k) s += h.HG[jj][k] * h.HG[jj][k];
      h.HG[jj][jj] = std::sqrt(h.H[jj][jj] - s);
      h.HG_inv[jj] = 1.0 / h.HG[jj][jj];
      for (int i = jj + 1; i < 6; ++i) {
        double t = 0.0;
        for (int k = 0; k < jj; ++k) t += h.HG[i][k] * h.HG[jj][k];
        h.HG[i][jj] = (h.H[i][jj] - t) * h.HG_inv[jj];
      }
    }
    for (int i = 0; i < 3; ++i) h.pNa03[i] = P.pNa03[i];
    h.epi_strain = P.epi_strain;
    h.bulk_or_film = P.bulk_or_film;
    h.Zstar = P.Z_star[0];
    h.dt = P.dt;
    h.dt_2 = P.dt_2;
    h.Q = P.Q_Nose;
    h.Qinv = 1.0 / P.Q_Nose;
    h.nf_kT = (double)P.n_freedom * P.temperature_eV;
    h.threeN_kT = (double)(3 * (long long)P.N) * P.temperature_eV;
    h.target_ke = P.target_kinetic_energy;
    h.n_sum_p = ctx->n_sum_p;
    h.ke_scale = (double)P.N / (2.0 * ctx->n_sum_p);
    h.E_on = P.E_field_always_zero ? 0 : 1;
    h.modulation_on = 0;
    h.wave_type = P.E_wave_type;
    h.wave_n_thermalize = P.n_thermalize;
    h.wave_period = P.n_E_wave_period;
    for (int a = 0; a < 3; ++a) h.wave_amp[a] = P.external_E_field[a];
    CK(cudaMalloc(&ctx->ph, sizeof(Phys)));
    CK(cudaMemcpy(ctx->ph, &h, sizeof(Phys), cudaMemcpyHostToDevice));
  }
  // scalars
  CK(cudaMalloc(&ctx->sc, sizeof(DevScalars)));
  CK(cudaMallocHost(&ctx->sc_host, sizeof(DevScalars)));
  CK(cudaMallocHost(&ctx->E_host, 3 * sizeof(double)));
  std::memset(ctx->sc_host, 0, sizeof(DevScalars));
  ctx->sc_host->s = 1.0;
  ctx->sc_host->pi = 0.0;
  ctx->sc_host->H0 = 0.0;
  ctx->sc_host->lf_dt = P.dt;
  ctx->sc_host->lf_dt_2 = P.dt_2;
  ctx->sc_host->kick_coef = P.dt_2 * 1.0;
  CK(cudaMemcpy(ctx->sc, ctx->sc_host, sizeof(DevScalars), cudaMemcpyHostToDevice));
  // fields
  const size_t es = sizeof(T);
  ctx->real_bytes = es * (size_t)g.nsite;
  const size_t nfc = ctx->acou ? 6 : 3;
  CK(cudaMalloc(&ctx->u, nfc * ctx->real_bytes));
  CK(cudaMalloc(&ctx->p, nfc * ctx->real_bytes));
  CK(cudaMalloc(&ctx->F, 3 * ctx->real_bytes));
  CK(cudaMemset(ctx->u, 0, nfc * ctx->real_bytes));  // acouR = acouP = 0 (initialize-dipoR.F:56)
  CK(cudaMemset(ctx->p, 0, nfc * ctx->real_bytes));
  CK(cudaMemset(ctx->F, 0, 3 * ctx->real_bytes));
  if (sizeof(T) == 4) {
    CK(cudaMalloc(&ctx->Flo, 3 * ctx->real_bytes));
    CK(cudaMemset(ctx->Flo, 0, 3 * ctx->real_bytes));
  }
  CK(cudaMalloc(&ctx->spec, (size_t)ctx->ncx * sizeof(cplx<T>) * (size_t)g.ncplx));
  CK(cudaMemset(ctx->spec, 0, 9 * sizeof(cplx<T>) * (size_t)g.ncplx));
  CK(cudaMalloc(&ctx->rwork, (size_t)ctx->ncx * ctx->real_bytes));
  CK(cudaMalloc(&ctx->dtab, 6 * es * (size_t)g.nkpos));
  CK(cudaMemset(ctx->dtab, 0, 6 * es * (size_t)g.nkpos));
  CK(cudaMalloc(&ctx->ckmod, 3 * sizeof(cplx<T>) * (size_t)g.nkpos));
  CK(cudaMemset(ctx->ckmod, 0, 3 * sizeof(cplx<T>) * (size_t)g.nkpos));
  CK(cudaMalloc(&ctx->acouK, 3 * sizeof(cplx<T>) * (size_t)g.nkpos));
  CK(cudaMemset(ctx->acouK, 0, 3 * sizeof(cplx<T>) * (size_t)g.nkpos));
  CK(cudaMalloc(&ctx->part_k, sizeof(double) * NQ_K * (size_t)(ctx->zt.nreg + ctx->zt.nnyq)));
  CK(cudaMalloc(&ctx->part_r, sizeof(double) * NQ_R * (size_t)ctx->grid_elem));
  CK(cudaMalloc(&ctx->part_ke, sizeof(double) * 3 * (size_t)ctx->grid_elem));
  CK(cudaMalloc(&ctx->part_avg, sizeof(double) * 6 * (size_t)ctx->grid_elem));
  CK(cudaMalloc(&ctx->avg6, sizeof(double) * 6));
  CK(cudaMalloc(&ctx->done, sizeof(unsigned int) * 4));
  CK(cudaMemset(ctx->done, 0, sizeof(unsigned int) * 4));
  ctx->staging_n = (size_t)3 * ctx->NXP * ctx->NYP * P.Lz;
  CK(cudaMalloc(&ctx->staging, sizeof(double) * ctx->staging_n));
  CK(cudaMemset(ctx->staging, 0, sizeof(double) * ctx->staging_n));
  // the memsets above run on the legacy default stream, which the context's
  // non-blocking stream does not wait for: finish them before any kernel of
  // the context reads the buffers (the done tickets, the zeroed fields)
  CK(cudaStreamSynchronize(0));
  return FG_OK;
}

template <typename T>
int build_tables_impl(fg_ctx* ctx) {
  const Geom& g = ctx->g;
  const fg_params& P = ctx->P;
  double* real6 = nullptr;
  cplx<double>* spec6 = nullptr;
  CK(cudaMalloc(&real6, sizeof(double) * 6 * (size_t)g.nsite));
  CK(cudaMalloc(&spec6, sizeof(cplx<double>) * 6 * (size_t)g.ncplx));
  if (!ctx->L64) CK(cudaMalloc(&ctx->L64, sizeof(double) * 6 * (size_t)g.nkpos));
  const int max_x = 24 / P.Lx, max_y = 24 / P.Ly, max_z = 24 / P.Lz;  // dipole-dipole-long-range.F:98-100
  k_ewald_real<<<std::max(1, div_up(g.nsite, 128)), 128, 0, ctx->stream>>>(real6, g, P.a0, P.kappa, max_x, max_y, max_z);
  CKL();
  int rc0 = launch_xy_fwd<double, SRC_FIELD>(ctx, real6, spec6, 6, ctx->smem_xy64, ctx->twx64, ctx->twm64,
                                             ctx->twy64);
  if (rc0) return rc0;
  k_z_ewald_pack<T><<<ctx->zt6.nreg + ctx->zt6.nnyq, kThreadsZ, ctx->smem_z6, ctx->stream>>>(
      spec6, (T*)ctx->dtab, ctx->L64, g, ctx->pz, ctx->twz64, kmaps<T>(ctx), ctx->ph, P.a0, P.kappa, P.epsilon_inf,
      max_x, max_y, max_z, ctx->zt6);
  CKL();
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(real6);
  cudaFree(spec6);
  int rc = check_device_error(ctx);
  if (rc) return rc;
  ctx->tables_ready = true;
  ctx->ltab_ready = false;
  return FG_OK;
}

template <typename T>
int set_modulation_R_impl(fg_ctx* ctx, const double* modR) {
  const Geom& g = ctx->g;
  double* r1 = nullptr;
  cplx<double>* s1 = nullptr;
  const size_t nin = (size_t)ctx->NXP * ctx->NYP * ctx->P.Lz;
  CK(cudaMalloc(&r1, sizeof(double) * (size_t)g.nsite));
  CK(cudaMalloc(&s1, sizeof(cplx<double>) * (size_t)g.ncplx));
  CK(cudaMemcpyAsync(ctx->staging, modR, sizeof(double) * nin, cudaMemcpyHostToDevice, ctx->stream));
  k_fortran_to_soa<double><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(r1, ctx->staging, g, 1, ctx->NXP, ctx->NYP);
  CKL();
  int rc0 = launch_xy_fwd<double, SRC_FIELD>(ctx, r1, s1, 1, ctx->smem_xy64, ctx->twx64, ctx->twm64, ctx->twy64);
  if (rc0) return rc0;
  k_z_modulation_pack<T><<<ctx->zt1.nreg + ctx->zt1.nnyq, kThreadsZ, ctx->smem_z1, ctx->stream>>>(
      s1, (cplx<T>*)ctx->ckmod, g, ctx->pz, ctx->twz64, kmaps<T>(ctx), ctx->P.modulation_constant, ctx->zt1);
  CKL();
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(r1);
  cudaFree(s1);
  return check_device_error(ctx);
}

// Fortran (a,b,kx,ky,kz) index of a (3,ncol,0:Lx/2,0:NYP-1,0:Lz-1) table
inline size_t ftab(const fg_ctx* c, int ncol, int a, int b, int kx, int ky, int kz) {
  return (size_t)a + 3 * (size_t)b + (size_t)3 * ncol * ((size_t)kx + (size_t)c->g.NKX * ((size_t)ky + (size_t)c->NYP * kz));
}

// Fortran (comp, kx, ky, kz) of a complex field, in doubles (re at 2i)
inline size_t fcplx(const fg_ctx* c, int nc, int comp, int kx, int ky, int kz) {
  return (size_t)comp + (size_t)nc * ((size_t)kx + (size_t)c->g.NKX * ((size_t)ky + (size_t)c->NYP * kz));
}

template <typename T>
int upload_tables_impl(fg_ctx* ctx, const double* sr, const double* lr) {
  const Geom& g = ctx->g;
  const fg_params& P = ctx->P;
  std::vector<T> D(6 * (size_t)g.nkpos, (T)0);
  std::vector<double> L(6 * (size_t)g.nkpos, 0.0);
  const int qa[6] = {0, 1, 2, 1, 2, 0}, qb[6] = {0, 1, 2, 2, 0, 1};
  double smax = 0.0, sdiff = 0.0;
  const double z2 = P.Z_star[0] * P.Z_star[0];
  for (int ys = 0; ys < g.Ly; ++ys)
    for (int zs = 0; zs < g.Lz; ++zs)
      for (int col = 0; col < g.NKX; ++col) {
        const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
        const long double tw = 2.0L * 3.14159265358979323846264338327950288L;
        double cc[3] = {(double)std::cos(tw * kx / P.Lx), (double)std::cos(tw * ky / P.Ly), (double)std::cos(tw * kz / P.Lz)};
        double ss[3] = {(double)std::sin(tw * kx / P.Lx), (double)std::sin(tw * ky / P.Ly), (double)std::sin(tw * kz / P.Lz)};
        double S[6];
        short_range_k(P.j, P.P_kappa2[0] * 2, cc, ss, S);
        const size_t tpos = ((size_t)ys * g.Lz + zs) * g.KXP + col;
        for (int q = 0; q < 6; ++q) {
          const double s = sr[ftab(ctx, 3, qa[q], qb[q], kx, ky, kz)];
          const double l = lr[ftab(ctx, 3, qa[q], qb[q], kx, ky, kz)];
          smax = std::max(smax, std::fabs(s));
          sdiff = std::max(sdiff, std::fabs(s - S[q]));
          D[tpos * 6 + q] = (T)((s + z2 * l) * P.Ninv);
          L[tpos * 6 + q] = l;
        }
      }
  if (sdiff > 1e-9 * std::max(1.0, smax)) {
    char b[200];
    std::snprintf(b, sizeof(b), "short_range table differs from the feram stencil by %.3e (max %.3e)", sdiff, smax);
    return fail(ctx, FG_ERR_ARG, b);
  }
  CK(cudaMemcpy(ctx->dtab, D.data(), D.size() * sizeof(T), cudaMemcpyHostToDevice));
  if (!ctx->L64) CK(cudaMalloc(&ctx->L64, sizeof(double) * 6 * (size_t)g.nkpos));
  CK(cudaMemcpy(ctx->L64, L.data(), L.size() * sizeof(double), cudaMemcpyHostToDevice));
  ctx->tables_ready = true;
  ctx->ltab_ready = false;
  return FG_OK;
}

template <typename T>
int upload_modulation_impl(fg_ctx* ctx, const double* ck) {
  const Geom& g = ctx->g;
  std::vector<cplx<T>> C(3 * (size_t)g.nkpos, mk<cplx<T>>((T)0, (T)0));
  if (ck) {
    for (int ys = 0; ys < g.Ly; ++ys)
      for (int zs = 0; zs < g.Lz; ++zs)
        for (int col = 0; col < g.NKX; ++col) {
          const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
          const size_t tpos = ((size_t)ys * g.Lz + zs) * g.KXP + col;
          for (int a = 0; a < 3; ++a) {
            const size_t f = fcplx(ctx, 3, a, kx, ky, kz);
            C[tpos * 3 + a] = mk<cplx<T>>((T)ck[2 * f], (T)ck[2 * f + 1]);
          }
        }
  }
  CK(cudaMemcpy(ctx->ckmod, C.data(), C.size() * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  return FG_OK;
}

int set_modulation_flag(fg_ctx* ctx, int on) {
  ctx->ph_host.modulation_on = on;
  CK(cudaMemcpy(ctx->ph, &ctx->ph_host, sizeof(Phys), cudaMemcpyHostToDevice));
  return FG_OK;
}

template <typename T>
int set_field(fg_ctx* ctx, void* dst, const double* src) {
  const size_t nin = (size_t)3 * ctx->NXP * ctx->NYP * ctx->P.Lz;
  CK(cudaMemcpyAsync(ctx->staging, src, sizeof(double) * nin, cudaMemcpyHostToDevice, ctx->stream));
  k_fortran_to_soa<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((T*)dst, ctx->staging, ctx->g, 3, ctx->NXP,
                                                                         ctx->NYP);
  CKL();
  CK(cudaStreamSynchronize(ctx->stream));
  return FG_OK;
}

template <typename T>
int get_field(fg_ctx* ctx, double* dst, const void* src) {
  const size_t nin = (size_t)3 * ctx->NXP * ctx->NYP * ctx->P.Lz;
  k_soa_to_fortran<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(ctx->staging, (const T*)src, ctx->g, 3,
                                                                         ctx->NXP, ctx->NYP);
  CKL();
  CK(cudaMemcpyAsync(dst, ctx->staging, sizeof(double) * nin, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FG_OK;
}

// A field held as hi + lo (the mixed path's force after fg_mirror_force_mirror)
template <typename T>
int get_field2(fg_ctx* ctx, double* dst, const void* hi, const void* lo) {
  const size_t nin = (size_t)3 * ctx->NXP * ctx->NYP * ctx->P.Lz;
  k_soa2_to_fortran<T><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(ctx->staging, (const T*)hi, (const T*)lo,
                                                                          ctx->g, 3, ctx->NXP, ctx->NYP);
  CKL();
  CK(cudaMemcpyAsync(dst, ctx->staging, sizeof(double) * nin, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FG_OK;
}

template <typename T>
int get_acouK_impl(fg_ctx* ctx, double* out) {
  const Geom& g = ctx->g;
  std::vector<cplx<T>> A(3 * (size_t)g.nkpos);
  CK(cudaMemcpy(A.data(), ctx->acouK, A.size() * sizeof(cplx<T>), cudaMemcpyDeviceToHost));
  for (int ys = 0; ys < g.Ly; ++ys)
    for (int zs = 0; zs < g.Lz; ++zs)
      for (int col = 0; col < g.NKX; ++col) {
        const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
        const size_t tpos = ((size_t)ys * g.Lz + zs) * g.KXP + col;
        for (int a = 0; a < 3; ++a) {
          const size_t f = fcplx(ctx, 3, a, kx, ky, kz);
          out[2 * f] = (double)A[tpos * 3 + a].x;
          out[2 * f + 1] = (double)A[tpos * 3 + a].y;
        }
      }
  return FG_OK;
}

// 3-component r2c / c2r of the reference's plan_r2c_3_out / plan_c2r_3_out
// (coord_module.F:155-157,310-312) on the device FFT.
// z pass of the 3-component spectrum in ctx->spec
template <typename T, bool INV>
int launch_z_pass(fg_ctx* ctx) {
  with_z_pass<T, INV>(ctx->g.Lz, ctx->zt.CW, [&](auto kern) {
    kern<<<ctx->zt.nreg + ctx->zt.nnyq, kThreadsZ, ctx->smem_z3, ctx->stream>>>(
        (cplx<T>*)ctx->spec, ctx->g, ctx->pz, (const cplx<T>*)ctx->twz, 3, ctx->zt);
  });
  CKL();
  return FG_OK;
}

// The batched 3-component r2c (rwork -> spec) and c2r (spec -> rwork) of
// the FFT entry points, on the device buffers only.
template <typename T>
int enqueue_fft_r2c3(fg_ctx* ctx) {
  int rc = launch_xy_fwd<T, SRC_FIELD>(ctx, (const T*)ctx->rwork, (cplx<T>*)ctx->spec, 3, ctx->smem_xy,
                                       (const cplx<T>*)ctx->twx, (const cplx<T>*)ctx->twm, (const cplx<T>*)ctx->twy);
  if (rc) return rc;
  return launch_z_pass<T, false>(ctx);
}
template <typename T>
int enqueue_fft_c2r3(fg_ctx* ctx) {
  int rc = launch_z_pass<T, true>(ctx);
  if (rc) return rc;
  return launch_xy_inv<T>(ctx, (const cplx<T>*)ctx->spec, (T*)ctx->rwork, 3);
}

template <typename T>
int time_fft_impl(fg_ctx* ctx, int reps, double* ms) {
  cudaEvent_t ev[3];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  int rc = FG_OK;
  double t_f = 0.0, t_i = 0.0;
  for (int r = 0; r < reps + 1 && rc == FG_OK; ++r) {  // r = 0: warm-up
    if (cudaEventRecord(ev[0], ctx->stream) != cudaSuccess) rc = FG_ERR_CUDA;
    if (!rc) rc = enqueue_fft_r2c3<T>(ctx);
    if (!rc && cudaEventRecord(ev[1], ctx->stream) != cudaSuccess) rc = FG_ERR_CUDA;
    if (!rc) rc = enqueue_fft_c2r3<T>(ctx);
    if (!rc && cudaEventRecord(ev[2], ctx->stream) != cudaSuccess) rc = FG_ERR_CUDA;
    if (!rc && cudaEventSynchronize(ev[2]) != cudaSuccess) rc = FG_ERR_CUDA;
    float a = 0.0f, b = 0.0f;
    if (!rc && (cudaEventElapsedTime(&a, ev[0], ev[1]) != cudaSuccess ||
                cudaEventElapsedTime(&b, ev[1], ev[2]) != cudaSuccess))
      rc = FG_ERR_CUDA;
    if (!rc && r > 0) {
      t_f += a;
      t_i += b;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (rc == FG_ERR_CUDA && ctx->err.empty()) ctx->err = "fg_time_fft: CUDA event or launch error";
  if (rc) return rc;
  ms[0] = t_f / reps;
  ms[1] = t_i / reps;
  return check_device_error(ctx);
}

template <typename T>
int fft_r2c3_impl(fg_ctx* ctx, const double* in, double* out) {
  const Geom& g = ctx->g;
  int rc = set_field<T>(ctx, ctx->rwork, in);
  if (rc) return rc;
  if ((rc = launch_xy_fwd<T, SRC_FIELD>(ctx, (const T*)ctx->rwork, (cplx<T>*)ctx->spec, 3, ctx->smem_xy,
                                        (const cplx<T>*)ctx->twx, (const cplx<T>*)ctx->twm,
                                        (const cplx<T>*)ctx->twy)))
    return rc;
  if ((rc = launch_z_pass<T, false>(ctx))) return rc;
  std::vector<cplx<T>> S(3 * (size_t)g.ncplx);
  CK(cudaMemcpyAsync(S.data(), ctx->spec, S.size() * sizeof(cplx<T>), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((rc = check_device_error(ctx))) return rc;
  for (int c = 0; c < 3; ++c)
    for (int zs = 0; zs < g.Lz; ++zs)
      for (int ys = 0; ys < g.Ly; ++ys)
        for (int col = 0; col < g.NKX; ++col) {
          const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
          const cplx<T> v = S[(size_t)c * g.ncplx + (size_t)zs * g.plane_c + (size_t)ys * g.KXP + col];
          const size_t f = fcplx(ctx, 3, c, kx, ky, kz);
          out[2 * f] = (double)v.x;
          out[2 * f + 1] = (double)v.y;
        }
  // only the spectrum scratch changed: u, p, dVddi and the scalars stand
  return FG_OK;
}

template <typename T>
int fft_c2r3_impl(fg_ctx* ctx, const double* in, double* out) {
  const Geom& g = ctx->g;
  std::vector<cplx<T>> S(3 * (size_t)g.ncplx, mk<cplx<T>>((T)0, (T)0));
  for (int c = 0; c < 3; ++c)
    for (int zs = 0; zs < g.Lz; ++zs)
      for (int ys = 0; ys < g.Ly; ++ys)
        for (int col = 0; col < g.NKX; ++col) {
          const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
          const size_t f = fcplx(ctx, 3, c, kx, ky, kz);
          S[(size_t)c * g.ncplx + (size_t)zs * g.plane_c + (size_t)ys * g.KXP + col] = mk<cplx<T>>((T)in[2 * f], (T)in[2 * f + 1]);
        }
  CK(cudaMemcpyAsync(ctx->spec, S.data(), S.size() * sizeof(cplx<T>), cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_z_pass<T, true>(ctx);
  if (rc) return rc;
  rc = launch_xy_inv<T>(ctx, (const cplx<T>*)ctx->spec, (T*)ctx->rwork, 3);
  if (rc) return rc;
  rc = get_field<T>(ctx, out, ctx->rwork);
  if (rc) return rc;
  // only the spectrum and real-space scratch changed
  return check_device_error(ctx);
}

// fg_upload_site_arrays: per-site tables in the device's site order
// i = x + Lx (y + Ly z) from the padded Fortran arrays of alloc_Coord
// (coord_module.F:100-170) and read_relaxor / read_defects_u /
// initialize_E_field.
// Per-site Z* on or off: three more components in the force transforms
// (Z*(R) u forward, the long-range field inverse), wider spectrum and rwork,
// new z tiles, and the L/N table in T.
template <typename T>
int set_zsite(fg_ctx* ctx, bool on) {
  if (on == ctx->zsite) return FG_OK;
  const Geom& g = ctx->g;
  int dev = 0, smem_optin = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int smem_max = smem_optin - 8192;
  const int ncx = (ctx->acou ? 12 : 9) + (on ? 3 : 0);
  const ZTiles zt = z_tiles(g, ncx, sizeof(cplx<T>), plan_cw<T>(ctx), smem_max);
  if ((size_t)ncx * g.Lz * zt.CW * sizeof(cplx<T>) > (size_t)smem_max)
    return fail(ctx, FG_ERR_UNSUPPORTED, "a z pencil of the supercell does not fit in shared memory");
  const int smem_z = (int)(ncx * ((size_t)g.Lz * zt.CW + kZPad<T>) * sizeof(cplx<T>));
  cudaError_t ea = cudaSuccess;
  with_z_kspace<T>(g.Lz, zt.CW, ctx->acou, on, [&](auto kern) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    const int cap = smem_optin - (int)fa.sharedSizeBytes;
    if (e == cudaSuccess && smem_z > cap) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
    ea = e;
  });
  if (ea != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->broken = true;  // until every buffer below is allocated again
  for (void** b : {&ctx->spec, &ctx->rwork, (void**)&ctx->part_k, &ctx->ltab})
    if (*b) {
      cudaFree(*b);
      *b = nullptr;
    }
  ctx->ncx = ncx;
  ctx->zt = zt;
  ctx->smem_z = smem_z;
  ctx->smem_z3 = (int)(3 * (size_t)g.Lz * zt.CW * sizeof(cplx<T>));
  ctx->zsite = on;
  ctx->ltab_ready = false;
  CK(cudaMalloc(&ctx->spec, (size_t)ncx * sizeof(cplx<T>) * (size_t)g.ncplx));
  CK(cudaMemsetAsync(ctx->spec, 0, (size_t)ncx * sizeof(cplx<T>) * (size_t)g.ncplx, ctx->stream));
  CK(cudaMalloc(&ctx->rwork, (size_t)ncx * ctx->real_bytes));
  CK(cudaMalloc(&ctx->part_k, sizeof(double) * NQ_K * (size_t)(zt.nreg + zt.nnyq)));
  if (on) CK(cudaMalloc(&ctx->ltab, 6 * sizeof(T) * (size_t)g.nkpos));
  ctx->broken = false;
  return FG_OK;
}

template <typename T>
int upload_sites_impl(fg_ctx* ctx, const double* zstar, const double* minv, const double* macou, const int* relaxor,
                      const int* sum_p, const double* Eloc) {
  const Geom& g = ctx->g;
  const fg_params& P = ctx->P;
  const size_t ns = (size_t)g.nsite, nxp = (size_t)ctx->NXP, nyp = (size_t)ctx->NYP;
  auto fidx = [&](size_t i) {
    const size_t x = i % (size_t)g.Lx, y = (i / (size_t)g.Lx) % (size_t)g.Ly, z = i / ((size_t)g.Lx * g.Ly);
    return x + nxp * (y + nyp * z);
  };
  // The step graphs (and any batch graph, through gen) hold the current
  // table pointers as kernel arguments: drop them before the first buffer is
  // freed, so that no early return below leaves a graph pointing at freed
  // memory.  From the first replacement until the call succeeds the context
  // refuses work (ensure_ready), since its tables may be half replaced.
  CK(cudaStreamSynchronize(ctx->stream));
  ++ctx->gen;
  for (cudaGraphExec_t* gx : {&ctx->g_np, &ctx->g_np_multi, &ctx->g_lf, &ctx->g_vs, &ctx->g_force})
    if (*gx) {
      cudaGraphExecDestroy(*gx);
      *gx = nullptr;
    }
  ctx->force_fresh = false;
  ctx->np_ready = false;
  ctx->flo_valid = false;
  bool replaced = false;
  auto replace = [&](void** dst, auto vec) -> int {
    replaced = true;
    ctx->broken = true;
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    return upload(ctx, dst, vec);
  };
  int rc;
  // Z*(R): the array if given, else Z_star of each site's species when the
  // species differ in it (read_relaxor.F:35)
  std::vector<double> zs;
  if (zstar) {
    zs.resize(ns);
    for (size_t i = 0; i < ns; ++i) zs[i] = zstar[fidx(i)];
  }
  if (relaxor) {
    std::vector<unsigned char> sp(ns);
    for (size_t i = 0; i < ns; ++i) {
      const int r = relaxor[fidx(i)];
      if (r < 1 || r > FG_RELAXOR_MAX) return fail(ctx, FG_ERR_ARG, "relaxor index outside 1..3");
      sp[i] = (unsigned char)(r - 1);
    }
    bool differ = false;
    for (int r = 1; r < FG_RELAXOR_MAX; ++r) differ |= P.Z_star[r] != P.Z_star[0];
    if (!zstar && differ) {
      zs.resize(ns);
      for (size_t i = 0; i < ns; ++i) zs[i] = P.Z_star[sp[i]];
    }
    if ((rc = replace((void**)&ctx->site_species, sp))) return rc;
  }
  if (!zs.empty()) {
    std::vector<T> v(ns);
    bool differ = false;
    for (size_t i = 0; i < ns; ++i) {
      v[i] = (T)zs[i];
      differ |= zs[i] != P.Z_star[0];
    }
    if ((rc = replace(&ctx->site_zstar, v))) return rc;
    if ((rc = set_zsite<T>(ctx, differ))) return rc;
  }
  if (minv) {
    std::vector<T> v(ns);
    for (size_t i = 0; i < ns; ++i) v[i] = (T)minv[fidx(i)];
    if ((rc = replace(&ctx->site_minv, v))) return rc;
  }
  if (macou) {
    std::vector<T> v(ns);
    for (size_t i = 0; i < ns; ++i) v[i] = (T)macou[fidx(i)];
    if ((rc = replace(&ctx->site_macou, v))) return rc;
  }
  if (sum_p) {
    std::vector<unsigned char> v(ns);
    std::vector<double> nl(g.Lz, 0.0);
    double n = 0.0;
    for (size_t i = 0; i < ns; ++i) {
      v[i] = sum_p[fidx(i)] ? 1 : 0;
      nl[i / ((size_t)g.Lx * g.Ly)] += v[i];
      n += v[i];
    }
    if ((rc = replace((void**)&ctx->site_sump, v))) return rc;
    if ((rc = replace((void**)&ctx->layer_nsum, nl))) return rc;
    ctx->n_sum_p = n;
    ctx->ph_host.n_sum_p = n;
    ctx->ph_host.ke_scale = (double)P.N / (2.0 * n);
  }
  if (Eloc) {
    std::vector<T> v(3 * ns);
    for (size_t i = 0; i < ns; ++i)
      for (int a = 0; a < 3; ++a) v[(size_t)a * ns + i] = (T)Eloc[3 * fidx(i) + (size_t)a];
    if ((rc = replace(&ctx->site_E, v))) return rc;
    ctx->ph_host.E_on = 1;  // a .localfield clears E_field_always_zero (initialize_E_field.F:21)
  }
  CK(cudaMemcpy(ctx->ph, &ctx->ph_host, sizeof(Phys), cudaMemcpyHostToDevice));
  if (replaced) ctx->broken = false;
  return FG_OK;
}

int ensure_ready(fg_ctx* ctx) {
  if (!ctx) return FG_ERR_ARG;
  if (ctx->broken) return fail(ctx, FG_ERR_CUDA, "a device buffer could not be reallocated: destroy this context");
  if (!ctx->tables_ready) return fail(ctx, FG_ERR_STATE, "no k-space tables: call fg_build_tables or fg_upload_tables");
  if (ctx->zsite && !ctx->ltab_ready) {  // L/N for the per-site Z* path, from the FP64 long-range table
    const long long n = 6 * ctx->g.nkpos;
    const int grid = (int)std::min<long long>(div_up(n, 256), 4096);
    if (ctx->prec == FG_PREC_MIXED)
      k_table_scale<float><<<grid, 256, 0, ctx->stream>>>((float*)ctx->ltab, ctx->L64, ctx->P.Ninv, n);
    else
      k_table_scale<double><<<grid, 256, 0, ctx->stream>>>((double*)ctx->ltab, ctx->L64, ctx->P.Ninv, n);
    CKL();
    ctx->ltab_ready = true;
  }
  return FG_OK;
}

int force_now(fg_ctx* ctx) {
  int rc = run_graph(ctx, &ctx->g_force, 0);
  if (rc) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = ctx->prec == FG_PREC_MIXED;
  ctx->np_ready = false;
  return FG_OK;
}

// Scalars of the first half of the next Nose-Poincare step from the current
// state (after the state, the thermostat or the force changed outside a step).
int np_prepare(fg_ctx* ctx) {
  int rc = ctx->prec == FG_PREC_MIXED ? enqueue_kick_close<float, true>(ctx) : enqueue_kick_close<double, true>(ctx);
  if (rc) return rc;
  ctx->np_ready = true;
  return FG_OK;
}

// The step graph of the context's method (md, lf with i_step != 0, vs).
cudaGraphExec_t* step_graph(fg_ctx* ctx, int* which) {
  switch (ctx->P.method) {
    case FG_METHOD_MD: *which = 1; return &ctx->g_np;
    case FG_METHOD_VS: *which = 3; return &ctx->g_vs;
    default: *which = 2; return &ctx->g_lf;
  }
}

// One step of the context's method enqueued on its stream (md, vs, lf with
// i_step != 0).
int enqueue_step(fg_ctx* ctx) {
  const bool f32 = ctx->prec == FG_PREC_MIXED;
  switch (ctx->P.method) {
    case FG_METHOD_MD: return f32 ? enqueue_np<float>(ctx) : enqueue_np<double>(ctx);
    case FG_METHOD_VS:
    case FG_METHOD_HL: return f32 ? enqueue_vs<float>(ctx) : enqueue_vs<double>(ctx);
    default: return f32 ? enqueue_lf<float>(ctx) : enqueue_lf<double>(ctx);
  }
}

// Everything a Nose-Poincare graph launch needs before it starts.
int np_ready_for_step(fg_ctx* ctx) {
  int rc;
  if (!ctx->force_fresh && (rc = force_now(ctx))) return rc;
  if (!ctx->np_ready && (rc = np_prepare(ctx))) return rc;
  return FG_OK;
}

const char* kProfNames[FG_NPROF] = {"k_kick_drift(35a,35c)", "k_xy_fwd", "k_z_kspace", "k_xy_inv+homo_strain",
                                    "k_assemble+kick(35e,35f)+np_tail"};

template <typename T>
int profile_impl(fg_ctx* ctx, int reps, double* ms) {
  cudaStream_t st = ctx->stream;
  cudaEvent_t ev[FG_NPROF + 1];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  for (int k = 0; k < FG_NPROF; ++k) ms[k] = 0.0;
  T* u = (T*)ctx->u;
  int rc = FG_OK;
  for (int r = 0; r < reps && rc == FG_OK; ++r) {
    int k = 0;
    CK(cudaEventRecord(ev[k], st));
    rc |= enqueue_kick_drift<T>(ctx);
    CK(cudaEventRecord(ev[++k], st));
    rc |= launch_xy_fwd<T, SRC_U9>(ctx, u, (cplx<T>*)ctx->spec, ctx->ncx, ctx->smem_xy, (const cplx<T>*)ctx->twx,
                                   (const cplx<T>*)ctx->twm, (const cplx<T>*)ctx->twy,
                                   ctx->zsite ? (const T*)ctx->site_zstar : nullptr, zu_comp(ctx));
    CK(cudaEventRecord(ev[++k], st));
    rc |= launch_z_kspace<T>(ctx, nullptr);
    CK(cudaEventRecord(ev[++k], st));
    rc |= launch_xy_inv<T>(ctx, (const cplx<T>*)ctx->spec, (T*)ctx->rwork, ctx->ncx, true);
    CK(cudaEventRecord(ev[++k], st));
    launch_assemble<T, true>(ctx, TAIL_NONE);
    CK(cudaEventRecord(ev[++k], st));
    CKL();
    CK(cudaEventSynchronize(ev[FG_NPROF]));
    for (int i = 0; i < FG_NPROF; ++i) {
      float t = 0.0f;
      CK(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
      ms[i] += t / reps;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}

}  // namespace

// ================================================================== C-ABI ===
extern "C" {

int fg_create(const fg_params* p, int precision, fg_ctx** out) {
  if (!p || !out) return FG_ERR_ARG;
  *out = nullptr;
  std::string why;
  int rc = validate(p, &why);
  fg_ctx* ctx = new fg_ctx();
  ctx->P = *p;
  ctx->prec = precision;
  if (rc) {
    ctx->err = why;
    *out = ctx;  // returned so that fg_last_error can report; caller must destroy
    return rc;
  }
  if (precision != FG_PREC_FP64 && precision != FG_PREC_MIXED) {
    ctx->err = "unknown precision";
    *out = ctx;
    return FG_ERR_ARG;
  }
  rc = (precision == FG_PREC_MIXED) ? create_impl<float>(ctx) : create_impl<double>(ctx);
  if (rc == FG_OK) rc = apply_wisdom(ctx, PLAN_SOLO);
  *out = ctx;
  return rc;
}

void fg_destroy(fg_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->g_np) cudaGraphExecDestroy(ctx->g_np);
  if (ctx->g_np_multi) cudaGraphExecDestroy(ctx->g_np_multi);
  if (ctx->g_lf) cudaGraphExecDestroy(ctx->g_lf);
  if (ctx->g_vs) cudaGraphExecDestroy(ctx->g_vs);
  if (ctx->g_force) cudaGraphExecDestroy(ctx->g_force);
  void* bufs[] = {ctx->u, ctx->p, ctx->F, ctx->Flo, ctx->spec, ctx->rwork, ctx->dtab, ctx->ckmod, ctx->acouK, ctx->twx,
                  ctx->twm, ctx->twy, ctx->twz, ctx->twx64, ctx->twm64, ctx->twy64, ctx->twz64, ctx->L64, ctx->ltab, ctx->revx,
                  ctx->revy, ctx->revz, ctx->posm, ctx->kvx, ctx->kvy, ctx->kvz, ctx->trx, ctx->try_, ctx->trz, ctx->trz_s, ctx->kvz_s,
                  ctx->layer_minv, ctx->layer_sump, ctx->ph, ctx->sc, ctx->part_k, ctx->part_r, ctx->part_ke,
                  ctx->part_avg, ctx->avg6, ctx->staging, ctx->dipoRavg, ctx->done, ctx->layer_macou, ctx->layer_all,
                  ctx->site_minv, ctx->site_macou, ctx->site_sump, ctx->site_species, ctx->site_zstar, ctx->site_E,
                  ctx->layer_nsum, ctx->samples};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (ctx->sc_host) cudaFreeHost(ctx->sc_host);
  if (ctx->E_host) cudaFreeHost(ctx->E_host);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* fg_last_error(const fg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* fg_stream(fg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int fg_build_tables(fg_ctx* ctx) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return ctx->prec == FG_PREC_MIXED ? build_tables_impl<float>(ctx) : build_tables_impl<double>(ctx);
}

int fg_upload_tables(fg_ctx* ctx, const double* short_range, const double* long_range) {
  if (!ctx || !ctx->stream || !short_range || !long_range) return FG_ERR_ARG;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return ctx->prec == FG_PREC_MIXED ? upload_tables_impl<float>(ctx, short_range, long_range)
                                    : upload_tables_impl<double>(ctx, short_range, long_range);
}

int fg_upload_modulation(fg_ctx* ctx, const double* ck) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  int rc = ctx->prec == FG_PREC_MIXED ? upload_modulation_impl<float>(ctx, ck) : upload_modulation_impl<double>(ctx, ck);
  if (rc) return rc;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return set_modulation_flag(ctx, (ck && ctx->P.modulation_constant != 0.0) ? 1 : 0);
}

int fg_set_modulation_R(fg_ctx* ctx, const double* modR) {
  if (!ctx || !ctx->stream || !modR) return FG_ERR_ARG;
  if (ctx->P.modulation_constant == 0.0)
    return fail(ctx, FG_ERR_ARG, "There is a .modulation file, but modulation_constant is zero.");  // elastic.F:207-210
  int rc = ctx->prec == FG_PREC_MIXED ? set_modulation_R_impl<float>(ctx, modR) : set_modulation_R_impl<double>(ctx, modR);
  if (rc) return rc;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return set_modulation_flag(ctx, 1);
}

int fg_get_long_range(fg_ctx* ctx, double* lr) {
  if (!ctx || !lr) return FG_ERR_ARG;
  if (!ctx->L64) return fail(ctx, FG_ERR_STATE, "no long-range table");
  const Geom& g = ctx->g;
  std::vector<double> L(6 * (size_t)g.nkpos);
  CK(cudaMemcpy(L.data(), ctx->L64, L.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const int qa[6] = {0, 1, 2, 1, 2, 0}, qb[6] = {0, 1, 2, 2, 0, 1};
  for (int ys = 0; ys < g.Ly; ++ys)
    for (int zs = 0; zs < g.Lz; ++zs)
      for (int col = 0; col < g.NKX; ++col) {
        const int kx = ctx->h_revx[col], ky = ctx->h_revy[ys], kz = ctx->h_revz[zs];
        const size_t tpos = ((size_t)ys * g.Lz + zs) * g.KXP + col;
        for (int q = 0; q < 6; ++q) {
          lr[ftab(ctx, 3, qa[q], qb[q], kx, ky, kz)] = L[tpos * 6 + q];
          lr[ftab(ctx, 3, qb[q], qa[q], kx, ky, kz)] = L[tpos * 6 + q];
        }
      }
  return FG_OK;
}

int fg_fft_r2c3(fg_ctx* ctx, const double* in, double* out) {
  if (!ctx || !ctx->stream || !in || !out) return FG_ERR_ARG;
  if (ctx->broken) return fail(ctx, FG_ERR_CUDA, "a device buffer could not be reallocated: destroy this context");
  return ctx->prec == FG_PREC_MIXED ? fft_r2c3_impl<float>(ctx, in, out) : fft_r2c3_impl<double>(ctx, in, out);
}

int fg_fft_c2r3(fg_ctx* ctx, const double* in, double* out) {
  if (!ctx || !ctx->stream || !in || !out) return FG_ERR_ARG;
  if (ctx->broken) return fail(ctx, FG_ERR_CUDA, "a device buffer could not be reallocated: destroy this context");
  return ctx->prec == FG_PREC_MIXED ? fft_c2r3_impl<float>(ctx, in, out) : fft_c2r3_impl<double>(ctx, in, out);
}

int fg_time_fft(fg_ctx* ctx, int reps, double* ms) {
  if (!ctx || !ctx->stream || !ms || reps < 1) return FG_ERR_ARG;
  if (ctx->broken) return fail(ctx, FG_ERR_CUDA, "a device buffer could not be reallocated: destroy this context");
  ctx->err.clear();
  // only the spectrum and real-space scratch (components 0..2) change, as in
  // fg_fft_r2c3 / fg_fft_c2r3: u, p, dVddi and the scalars stand
  return ctx->prec == FG_PREC_MIXED ? time_fft_impl<float>(ctx, reps, ms) : time_fft_impl<double>(ctx, reps, ms);
}

int fg_set_state(fg_ctx* ctx, const double* dipoR, const double* dipoP, double s, double pi, double H0) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  int rc;
  if (dipoR) {
    rc = ctx->prec == FG_PREC_MIXED ? set_field<float>(ctx, ctx->u, dipoR) : set_field<double>(ctx, ctx->u, dipoR);
    if (rc) return rc;
  }
  if (dipoP) {
    rc = ctx->prec == FG_PREC_MIXED ? set_field<float>(ctx, ctx->p, dipoP) : set_field<double>(ctx, ctx->p, dipoP);
    if (rc) return rc;
  }
  if ((rc = pull_scalars(ctx))) return rc;
  ctx->sc_host->s = s;
  ctx->sc_host->pi = pi;
  ctx->sc_host->H0 = H0;
  ctx->sc_host->kick_coef = ctx->P.dt_2 * s;
  if ((rc = push_scalars(ctx))) return rc;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return FG_OK;
}

int fg_set_thermostat(fg_ctx* ctx, double s, double pi, double H0) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  int rc;
  if ((rc = pull_scalars(ctx))) return rc;
  ctx->sc_host->s = s;
  ctx->sc_host->pi = pi;
  ctx->sc_host->H0 = H0;
  ctx->sc_host->kick_coef = ctx->P.dt_2 * s;
  ctx->np_ready = false;
  return push_scalars(ctx);
}

int fg_get_params(const fg_ctx* ctx, fg_params* p) {
  if (!ctx || !p) return FG_ERR_ARG;
  *p = ctx->P;
  return FG_OK;
}

// The next point of a temperature (or field) sweep, started from the state
// on the device as the reference's sweep scripts start each point from the
// previous point's final .coord read back as .restart (cooling.sh:64-69):
// the .coord holds dipoP / s_Nose (coord_module.F:476), initialize_dipoR
// reads it (initialize-dipoR.F:22-38), evaluates the force and sets s = 1,
// pi = 0 (:62-68), and molecular_dynamics sets H0 from that state
// (molecular-dynamics.F:52-55).  Here nothing leaves the device and nothing
// is rounded to the .coord's fixed-point columns.
int fg_chain_point(fg_ctx* ctx, double kelvin, const double E[3], fg_energy* e) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (ctx->P.method != FG_METHOD_MD)
    return fail(ctx, FG_ERR_UNSUPPORTED, "fg_chain_point continues Nose-Poincare ('md') runs only");
  if (!(kelvin > 0.0)) return fail(ctx, FG_ERR_ARG, "kelvin must be positive");
  // the new point's temperature (read_Param's kelvin tag, param_module.F:226,
  // and make_Param, :468)
  fg_params q = ctx->P;
  q.kelvin = kelvin;
  char eb[128];
  if ((rc = fg_make_param(&q, eb, sizeof(eb)))) return fail(ctx, rc, eb);
  if ((rc = pull_scalars(ctx))) return rc;
  const double s_old = ctx->sc_host->s;
  // a point with a field clears E_field_always_zero (param_module.F:294-298);
  // the field term's switch is a kernel argument of the step graphs
  if (E && (E[0] != 0.0 || E[1] != 0.0 || E[2] != 0.0) && q.E_field_always_zero) {
    q.E_field_always_zero = 0;
    ctx->ph_host.E_on = 1;
    ++ctx->gen;
    for (cudaGraphExec_t* gx : {&ctx->g_np, &ctx->g_np_multi, &ctx->g_lf, &ctx->g_vs, &ctx->g_force})
      if (*gx) {
        cudaGraphExecDestroy(*gx);
        *gx = nullptr;
      }
  }
  ctx->P = q;
  Phys& h = ctx->ph_host;
  h.nf_kT = (double)q.n_freedom * q.temperature_eV;
  h.threeN_kT = (double)(3 * (long long)q.N) * q.temperature_eV;
  h.target_ke = q.target_kinetic_energy;
  CK(cudaMemcpyAsync(ctx->ph, &h, sizeof(Phys), cudaMemcpyHostToDevice, ctx->stream));
  // p <- p / s (the dipole momenta only; write_system writes acouP as is)
  ctx->sc_host->vs_scale = 1.0 / s_old;
  ctx->sc_host->s = 1.0;
  ctx->sc_host->pi = 0.0;
  ctx->sc_host->H0 = 0.0;
  ctx->sc_host->kick_coef = ctx->P.dt_2;
  if (E)
    for (int a = 0; a < 3; ++a) ctx->sc_host->E[a] = E[a];
  if ((rc = push_scalars(ctx))) return rc;
  const long long n3 = 3 * ctx->g.nsite;
  if (ctx->prec == FG_PREC_MIXED)
    k_scale<float><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((float*)ctx->p, &ctx->sc->vs_scale, n3);
  else
    k_scale<double><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>((double*)ctx->p, &ctx->sc->vs_scale, n3);
  CKL();
  // initialize_dipoR's tail: the force of the state, s = 1, pi = 0, KE
  fg_energy en{};
  if ((rc = fg_mirror_force_mirror(ctx, &en))) return rc;
  double ke = 0.0;
  if ((rc = fg_kinetic_energy_dipo(ctx, &ke))) return rc;
  en.dipo_kinetic = ke;
  en.acou_kinetic = 0.0;
  // molecular-dynamics.F:52-55 with s = 1: H0 is the total energy
  const double V = en.short_range + en.long_range + en.dipole_E_field + en.unharmonic + en.homo_strain +
                   en.homo_coupling + en.inho_strain + en.inho_coupling + en.inho_modulation;
  en.total = ke + V;
  if ((rc = fg_set_thermostat(ctx, 1.0, 0.0, en.total))) return rc;
  en.H_Nose_Poincare = 0.0;
  if (e) *e = en;
  return FG_OK;
}

int fg_get_state(fg_ctx* ctx, double* dipoR, double* dipoP, double* dVddi, double strain[6], double* s, double* pi,
                 double* H0) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  int rc;
  const bool f32 = ctx->prec == FG_PREC_MIXED;
  if (dipoR && (rc = f32 ? get_field<float>(ctx, dipoR, ctx->u) : get_field<double>(ctx, dipoR, ctx->u))) return rc;
  if (dipoP && (rc = f32 ? get_field<float>(ctx, dipoP, ctx->p) : get_field<double>(ctx, dipoP, ctx->p))) return rc;
  if (dVddi) {
    if (f32 && ctx->flo_valid) rc = get_field2<float>(ctx, dVddi, ctx->F, ctx->Flo);
    else rc = f32 ? get_field<float>(ctx, dVddi, ctx->F) : get_field<double>(ctx, dVddi, ctx->F);
    if (rc) return rc;
  }
  if ((rc = pull_scalars(ctx))) return rc;
  if (strain)
    for (int i = 0; i < 6; ++i) strain[i] = ctx->sc_host->strain[i];
  if (s) *s = ctx->sc_host->s;
  if (pi) *pi = ctx->sc_host->pi;
  if (H0) *H0 = ctx->sc_host->H0;
  return FG_OK;
}

int fg_set_acou(fg_ctx* ctx, const double* acouR, const double* acouP) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  if (!ctx->acou) return fail(ctx, FG_ERR_STATE, "the acoustic field is dynamic only with acoustic_mass_amu > 0");
  const long long ns = ctx->g.nsite;
  const bool f32 = ctx->prec == FG_PREC_MIXED;
  const size_t off = (size_t)3 * ns * (f32 ? sizeof(float) : sizeof(double));
  int rc;
  if (acouR && (rc = f32 ? set_field<float>(ctx, (char*)ctx->u + off, acouR) : set_field<double>(ctx, (char*)ctx->u + off, acouR)))
    return rc;
  if (acouP && (rc = f32 ? set_field<float>(ctx, (char*)ctx->p + off, acouP) : set_field<double>(ctx, (char*)ctx->p + off, acouP)))
    return rc;
  ctx->force_fresh = false;
  ctx->np_ready = false;
  return FG_OK;
}

int fg_get_acou(fg_ctx* ctx, double* acouR, double* acouP, double* dVdacR) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  if (!ctx->acou) return fail(ctx, FG_ERR_STATE, "the acoustic field is dynamic only with acoustic_mass_amu > 0");
  const long long ns = ctx->g.nsite;
  const bool f32 = ctx->prec == FG_PREC_MIXED;
  const size_t es = f32 ? sizeof(float) : sizeof(double);
  const char* u = (const char*)ctx->u + 3 * ns * es;
  const char* q = (const char*)ctx->p + 3 * ns * es;
  const char* d = (const char*)ctx->rwork + 9 * ns * es;
  int rc;
  if (acouR && (rc = f32 ? get_field<float>(ctx, acouR, u) : get_field<double>(ctx, acouR, u))) return rc;
  if (acouP && (rc = f32 ? get_field<float>(ctx, acouP, q) : get_field<double>(ctx, acouP, q))) return rc;
  if (dVdacR && (rc = f32 ? get_field<float>(ctx, dVdacR, d) : get_field<double>(ctx, dVdacR, d))) return rc;
  return FG_OK;
}

int fg_upload_site_arrays(fg_ctx* ctx, const double* Z_starR, const double* mass_dipo_inv, const double* mass_acou_inv,
                          const int* relaxor, const int* sum_p, const double* E_field_local) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  return ctx->prec == FG_PREC_MIXED
             ? upload_sites_impl<float>(ctx, Z_starR, mass_dipo_inv, mass_acou_inv, relaxor, sum_p, E_field_local)
             : upload_sites_impl<double>(ctx, Z_starR, mass_dipo_inv, mass_acou_inv, relaxor, sum_p, E_field_local);
}

int fg_get_acouK(fg_ctx* ctx, double* acouK) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (!acouK) return FG_ERR_ARG;
  // re-evaluate the force of the current state with the acouK store enabled
  ctx->store_acouK = true;
  rc = ctx->prec == FG_PREC_MIXED ? enqueue_force<float>(ctx) : enqueue_force<double>(ctx);
  ctx->store_acouK = false;
  if (rc) return rc;
  if ((rc = pull_scalars(ctx))) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = false;
  return ctx->prec == FG_PREC_MIXED ? get_acouK_impl<float>(ctx, acouK) : get_acouK_impl<double>(ctx, acouK);
}

int fg_set_uniform_E(fg_ctx* ctx, const double E[3]) {
  if (!ctx || !ctx->stream || !ctx->E_host || !E) return FG_ERR_ARG;
  // Staged in pinned memory and copied in stream order, without waiting:
  // every call that reads results synchronises the stream, and a second
  // fg_set_uniform_E before the copy ran only makes the later field win.
  for (int a = 0; a < 3; ++a) ctx->E_host[a] = ctx->sc_host->E[a] = E[a];  // sc_host: for push_scalars
  CK(cudaMemcpyAsync(ctx->sc->E, ctx->E_host, 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  // The stored dVddi and energies stay those of the last evaluation, as
  // c%dVddi does when molecular-dynamics.F:66-76 changes c%E_field between
  // steps: the next force evaluation sees the new field.
  return FG_OK;
}

int fg_set_wave(fg_ctx* ctx, int on, int i_step) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  const fg_params& P = ctx->P;
  if (on) {
    const int t = P.E_wave_type;
    if (t == FG_WAVE_TRIANGULAR_COS || t == FG_WAVE_TRIANGULAR_SIN) {
      if (P.n_E_wave_period <= 0) return fail(ctx, FG_ERR_ARG, "n_E_wave_period must be positive");
    } else if (t == FG_WAVE_RAMPING_ON || t == FG_WAVE_RAMPING_OFF) {
      if (P.n_E_wave_period <= 0 || P.n_E_wave_period > P.n_thermalize)
        return fail(ctx, FG_ERR_ARG, "period must be smaller than n_thermalize (wave_module.F:42-45)");
    } else {
      return fail(ctx, FG_ERR_ARG, "fg_set_wave needs an E_wave_type");
    }
    if (P.E_field_always_zero) return fail(ctx, FG_ERR_ARG, "E_field_always_zero is set: the field term is off");
  }
  int rc;
  if ((rc = pull_scalars(ctx))) return rc;
  ctx->sc_host->i_step = i_step;
  if ((rc = push_scalars(ctx))) return rc;
  if ((on != 0) != ctx->wave_dev) {
    ctx->wave_dev = on != 0;
    // the step graphs gain or lose their first kernel
    ++ctx->gen;
    for (cudaGraphExec_t* gx : {&ctx->g_np, &ctx->g_np_multi, &ctx->g_lf, &ctx->g_vs, &ctx->g_force})
      if (*gx) {
        cudaGraphExecDestroy(*gx);
        *gx = nullptr;
      }
  }
  return FG_OK;
}

int fg_mirror_force_mirror(fg_ctx* ctx, fg_energy* e) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if ((rc = force_now(ctx))) return rc;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) energy_out(ctx->sc_host, e, true);
  return FG_OK;
}

int fg_nose_poincare(fg_ctx* ctx, fg_energy* e) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if ((rc = np_ready_for_step(ctx))) return rc;
  if ((rc = run_graph(ctx, &ctx->g_np, 1))) return rc;
  ctx->np_ready = true;
  ctx->flo_valid = false;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) energy_out(ctx->sc_host, e, false);
  return FG_OK;
}

int fg_leapfrog(fg_ctx* ctx, fg_energy* e, int i_step) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (i_step == 0) {  // leapfrog.F:89-102
    const bool f32 = ctx->prec == FG_PREC_MIXED;
    if ((rc = f32 ? enqueue_pump<float>(ctx) : enqueue_pump<double>(ctx))) return rc;
    if ((rc = force_now(ctx))) return rc;
    if (ctx->acou && (rc = f32 ? enqueue_kick_acou<float>(ctx, &ctx->sc->lf_dt_2, TAIL_ACOU)
                               : enqueue_kick_acou<double>(ctx, &ctx->sc->lf_dt_2, TAIL_ACOU)))
      return rc;
    if ((rc = f32 ? enqueue_kick<float>(ctx, &ctx->sc->lf_dt_2, TAIL_LF_FINAL)
                  : enqueue_kick<double>(ctx, &ctx->sc->lf_dt_2, TAIL_LF_FINAL)))
      return rc;
  } else {
    if ((rc = run_graph(ctx, &ctx->g_lf, 2))) return rc;
  }
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = false;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) {
    e->dipo_kinetic = ctx->sc_host->e[E_DIPO];
    e->acou_kinetic = ctx->sc_host->e[E_ACOU];
    for (int i = E_SHORT; i <= E_IM; ++i) (&e->acou_kinetic)[i] = ctx->sc_host->e[i];
  }
  return FG_OK;
}

int fg_velocity_scaling(fg_ctx* ctx, fg_energy* e) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if ((rc = run_graph(ctx, &ctx->g_vs, 3))) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = false;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) energy_out(ctx->sc_host, e, false);
  return FG_OK;
}

int fg_run_steps(fg_ctx* ctx, int n_steps, fg_energy* e) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (ctx->P.method == FG_METHOD_MD && (rc = np_ready_for_step(ctx))) return rc;
  int which = 0;
  cudaGraphExec_t* gx = step_graph(ctx, &which);
  int i = 0;
  if (which == 1)
    for (; i + kNpGraphSteps <= n_steps; i += kNpGraphSteps)
      if ((rc = run_graph(ctx, &ctx->g_np_multi, 4))) return rc;
  for (; i < n_steps; ++i)
    if ((rc = run_graph(ctx, gx, which))) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = ctx->P.method == FG_METHOD_MD;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) energy_out(ctx->sc_host, e, false);
  return FG_OK;
}

int fg_time_steps(fg_ctx* ctx, int n_steps, double* ms) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (!ms || n_steps < 1) return FG_ERR_ARG;
  if (ctx->P.method == FG_METHOD_MD && (rc = np_ready_for_step(ctx))) return rc;
  // make sure the graphs exist before the timed region
  int which = 0;
  cudaGraphExec_t* gx = step_graph(ctx, &which);
  const int nmulti = which == 1 ? n_steps / kNpGraphSteps : 0;
  const int nsingle = n_steps - nmulti * kNpGraphSteps;
  if (nsingle > 0 && !*gx) {
    if ((rc = run_graph(ctx, gx, which))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if (nmulti > 0 && !ctx->g_np_multi) {
    if ((rc = run_graph(ctx, &ctx->g_np_multi, 4))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float t = 0.0f;
  cudaError_t ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(e0, ctx->stream);
  for (int i = 0; ce == cudaSuccess && i < nmulti; ++i) ce = cudaGraphLaunch(ctx->g_np_multi, ctx->stream);
  for (int i = 0; ce == cudaSuccess && i < nsingle; ++i) ce = cudaGraphLaunch(*gx, ctx->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(e1, ctx->stream);
  if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
  if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
  if (e0) cudaEventDestroy(e0);  // on every path
  if (e1) cudaEventDestroy(e1);
  if (ce != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("fg_time_steps: ") + cudaGetErrorString(ce));
  *ms = t;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = ctx->P.method == FG_METHOD_MD;
  return pull_scalars(ctx);
}

const char* fg_profile_name(int i) { return (i >= 0 && i < FG_NPROF) ? kProfNames[i] : ""; }

int fg_profile_step(fg_ctx* ctx, int reps, double* ms) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (!ms || reps < 1) return FG_ERR_ARG;
  if (ctx->bulk_or_film_mirror()) return fail(ctx, FG_ERR_UNSUPPORTED, "profile covers the bulk step only");
  if ((rc = np_ready_for_step(ctx))) return rc;
  rc = ctx->prec == FG_PREC_MIXED ? profile_impl<float>(ctx, reps, ms) : profile_impl<double>(ctx, reps, ms);
  if (rc) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = true;
  return pull_scalars(ctx);
}

int fg_kinetic_energy_dipo(fg_ctx* ctx, double* ke) {
  if (!ctx || !ctx->stream || !ke) return FG_ERR_ARG;
  if (ctx->prec == FG_PREC_MIXED)
    k_ke_only<float><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
        (const float*)ctx->p, ctx->g, ctx->layer_minv, ctx->layer_sump, ctx->part_ke, (const float*)ctx->site_minv,
        ctx->site_sump);
  else
    k_ke_only<double><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
        (const double*)ctx->p, ctx->g, ctx->layer_minv, ctx->layer_sump, ctx->part_ke, (const double*)ctx->site_minv,
        ctx->site_sump);
  CKL();
  k_ke_finish<<<1, RED_THREADS, 0, ctx->stream>>>(ctx->ph, ctx->sc, ctx->part_ke, ctx->grid_elem);
  CKL();
  int rc = pull_scalars(ctx);
  if (rc) return rc;
  *ke = ctx->sc_host->e[E_DIPO];
  return FG_OK;
}

int fg_nose_poincare_hamiltonian(fg_ctx* ctx, fg_energy* e) {
  if (!ctx || !e) return FG_ERR_ARG;
  int rc = pull_scalars(ctx);
  if (rc) return rc;
  const DevScalars* s = ctx->sc_host;
  const fg_params& P = ctx->P;
  const double V = e->short_range + e->long_range + e->dipole_E_field + e->unharmonic + e->homo_strain +
                   e->homo_coupling + e->inho_strain + e->inho_coupling + e->inho_modulation;
  double h = e->dipo_kinetic / (s->s * s->s) + V + s->pi * s->pi / 2 / P.Q_Nose +
             3 * P.N * P.temperature_eV * std::log(s->s) - s->H0;
  e->H_Nose_Poincare = h * s->s;
  return FG_OK;
}

int fg_average_accumulate(fg_ctx* ctx, const fg_energy* e, fg_average* avg) {
  if (!ctx || !ctx->stream || !e || !avg) return FG_ERR_ARG;
  if (ctx->prec == FG_PREC_MIXED)
    k_avg_sums<float><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
        (const float*)ctx->u, ctx->g, ctx->P.Z_star[0], ctx->layer_sump, ctx->part_avg, ctx->site_sump,
        (const float*)ctx->site_zstar);
  else
    k_avg_sums<double><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(
        (const double*)ctx->u, ctx->g, ctx->P.Z_star[0], ctx->layer_sump, ctx->part_avg, ctx->site_sump,
        (const double*)ctx->site_zstar);
  CKL();
  k_avg_finish<<<1, RED_THREADS, 0, ctx->stream>>>(ctx->avg6, ctx->part_avg, ctx->grid_elem);
  CKL();
  double v[6];
  CK(cudaMemcpyAsync(v, ctx->avg6, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int rc = pull_scalars(ctx);
  if (rc) return rc;
  // average_module.F:75-128
  double* ae = &avg->energy.acou_kinetic;
  const double* ee = &e->acou_kinetic;
  for (int i = 0; i < E_COUNT; ++i) ae[i] += ee[i];
  avg->e2 += e->total * e->total;
  const double s = ctx->sc_host->s;
  avg->dipo_kinetic_true += e->dipo_kinetic / (s * s);
  for (int i = 0; i < 6; ++i) avg->strain[i] += ctx->sc_host->strain[i];
  const double* ut = v;
  const double* pt = v + 3;
  for (int a = 0; a < 3; ++a) {
    avg->u[a] += ut[a];
    avg->p[a] += pt[a];
  }
  avg->uu[0] += ut[0] * ut[0]; avg->uu[1] += ut[1] * ut[1]; avg->uu[2] += ut[2] * ut[2];
  avg->uu[3] += ut[1] * ut[2]; avg->uu[4] += ut[2] * ut[0]; avg->uu[5] += ut[0] * ut[1];
  avg->pp[0] += pt[0] * pt[0]; avg->pp[1] += pt[1] * pt[1]; avg->pp[2] += pt[2] * pt[2];
  avg->pp[3] += pt[1] * pt[2]; avg->pp[4] += pt[2] * pt[0]; avg->pp[5] += pt[0] * pt[1];
  avg->n_steps += 1;
  return FG_OK;
}

int fg_dipoRavg_accumulate(fg_ctx* ctx) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  const long long n = 3 * ctx->g.nsite;
  if (!ctx->dipoRavg) {
    CK(cudaMalloc(&ctx->dipoRavg, sizeof(double) * (size_t)n));
    CK(cudaMemsetAsync(ctx->dipoRavg, 0, sizeof(double) * (size_t)n, ctx->stream));
  }
  if (ctx->prec == FG_PREC_MIXED)
    k_accumulate<float><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(ctx->dipoRavg, (const float*)ctx->u, n);
  else
    k_accumulate<double><<<ctx->grid_elem, kThreadsElem, 0, ctx->stream>>>(ctx->dipoRavg, (const double*)ctx->u, n);
  CKL();
  return FG_OK;
}

int fg_get_dipoRavg(fg_ctx* ctx, double* out) {
  if (!ctx || !out) return FG_ERR_ARG;
  if (!ctx->dipoRavg) return fail(ctx, FG_ERR_STATE, "dipoRavg was never accumulated");
  return get_field<double>(ctx, out, ctx->dipoRavg);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free kinetic energy (no counterpart in the reference).
//
// Some callers cannot allocate device memory at the point where they want the
// kinetic energy of a momentum field they already hold on the device: a
// driver that runs the MD from its own device memory pool under a fixed
// budget, or a host thread that must never enter the CUDA allocator.  This
// entry point needs no fg_ctx and calls neither cudaMalloc nor cudaFree: the
// block partial sums of k_ke_only and the per-layer mass and mask tables live
// in one file-scope device array of fixed size.  Every call on a device uses
// the same array, so two calls that overlap in time on one device (different
// streams or host threads) overwrite each other's partials; the caller orders
// them.  Nothing in the array has to start at zero: each call writes the
// tables and every partial it reads before reading them.
namespace {
constexpr int kNoAllocPartials = 4096;  // >= blocks of one k_ke_only launch
constexpr int kNoAllocMinv = kNoAllocPartials;                       // FG_NOALLOC_MAX_LZ doubles
constexpr int kNoAllocMask = kNoAllocMinv + FG_NOALLOC_MAX_LZ;       // FG_NOALLOC_MAX_LZ bytes
constexpr int kNoAllocDoubles = kNoAllocMask + FG_NOALLOC_MAX_LZ / 8;  // 5248 doubles = 41 KiB

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
  std::mutex mu;
  bool ready = false;         // set-up done on this device (a failed one is retried)
  double* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int nsm = 0;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// KE = sum p^2 m^-1 / n_sum_p * N / 2, the scaling of kinetic_energy_dipo.F:28
__global__ void __launch_bounds__(RED_THREADS) k_ke_finish_out(const double* __restrict__ part, int nblk,
                                                               double n_sum_p, double N, double* out) {
  const double v = reduce_partials(part, nblk, 1, 0);
  if (threadIdx.x == 0) *out = v / n_sum_p * N / 2;
}

int noalloc_fail(char* errbuf, int errlen, int rc, const char* msg) {
  if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", msg);
  return rc;
}
}  // namespace

extern "C" int fg_kinetic_energy_dipo_noalloc(const double* dipoP, int Lx, int Ly, int Lz,
                                              const double* layer_mass_inv, const unsigned char* layer_sum_p,
                                              void* stream, double* ke, char* errbuf, int errlen) {
  char msg[160];
  if (!dipoP || !layer_mass_inv || !layer_sum_p || !ke)
    return noalloc_fail(errbuf, errlen, FG_ERR_ARG, "fg_kinetic_energy_dipo_noalloc: null pointer argument");
  if (Lx < 1 || Ly < 1 || Lz < 1)
    return noalloc_fail(errbuf, errlen, FG_ERR_ARG, "fg_kinetic_energy_dipo_noalloc: Lx, Ly, Lz must be >= 1");
  if (Lz > FG_NOALLOC_MAX_LZ) {
    std::snprintf(msg, sizeof(msg), "fg_kinetic_energy_dipo_noalloc: Lz = %d exceeds FG_NOALLOC_MAX_LZ = %d", Lz,
                  FG_NOALLOC_MAX_LZ);
    return noalloc_fail(errbuf, errlen, FG_ERR_ARG, msg);
  }
  const long long plane = (long long)Lx * Ly;
  long long counted = 0;
  for (int z = 0; z < Lz; ++z) counted += layer_sum_p[z] ? 1 : 0;
  if (counted == 0)
    return noalloc_fail(errbuf, errlen, FG_ERR_ARG, "fg_kinetic_energy_dipo_noalloc: layer_sum_p counts no layer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, FG_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return noalloc_fail(errbuf, errlen, FG_ERR_UNSUPPORTED, "fg_kinetic_energy_dipo_noalloc: device index >= 64");
  // one-time set-up on this device (it is current): the array's device
  // address.  Only a successful set-up is kept; after a failure (a transient
  // error, or a call made while the device was not usable) the next call
  // tries again.
  NoAllocDevice& d = g_noalloc_dev[dev];
  double* scratch = nullptr;
  int nsm = 0;
  {
    std::lock_guard<std::mutex> lock(d.mu);
    if (!d.ready) {
      void* ptr = nullptr;
      cudaError_t se = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (se == cudaSuccess) se = cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev);
      if (se != cudaSuccess || ptr == nullptr) {
        std::snprintf(msg, sizeof(msg), "fg_kinetic_energy_dipo_noalloc: set-up failed: %s",
                      cudaGetErrorString(se));
        return noalloc_fail(errbuf, errlen, FG_ERR_CUDA, msg);
      }
      d.scratch = static_cast<double*>(ptr);
      d.ready = true;
    }
    scratch = d.scratch;
    nsm = d.nsm;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* part = scratch;
  double* minv = scratch + kNoAllocMinv;
  unsigned char* mask = reinterpret_cast<unsigned char*>(scratch + kNoAllocMask);
  e = cudaMemcpyAsync(minv, layer_mass_inv, sizeof(double) * (size_t)Lz, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mask, layer_sum_p, (size_t)Lz, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, FG_ERR_CUDA, cudaGetErrorString(e));
  Geom g;
  std::memset(&g, 0, sizeof(g));
  g.Lx = Lx;
  g.Ly = Ly;
  g.Lz = Lz;
  g.plane_r = plane;
  g.nsite = plane * Lz;
  const long long want = (g.nsite + kThreadsElem - 1) / kThreadsElem;
  const int grid = (int)std::max(1LL, std::min({want, (long long)std::max(nsm, 1) * 8, (long long)kNoAllocPartials}));
  k_ke_only<double><<<grid, kThreadsElem, 0, st>>>(dipoP, g, minv, mask, part);
  k_ke_finish_out<<<1, RED_THREADS, 0, st>>>(part, grid, (double)(counted * plane), (double)g.nsite, ke);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(errbuf, errlen, FG_ERR_CUDA, cudaGetErrorString(e));
  return FG_OK;
}

// ---------------------------------------------------------------------------
// Replica batches: independent supercells (temperature or field points of a
// sweep, of any sizes and methods) stepped together.  One CUDA graph holds one
// branch per replica, forked from and joined to the batch stream, so the
// kernels of small replicas run concurrently instead of one launch at a time.
struct fg_batch {
  std::vector<fg_ctx*> ctx;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t graph = nullptr;   // one step of every replica
  std::vector<unsigned> gen;         // the replicas' gen when the graphs were captured
  bool grouping = true;              // replicas of one size step as one launch per kernel
  bool priorities = true;            // branches of small supercells at a higher launch priority
  std::vector<std::vector<int>> groups;  // of the captured graph: replica indices per branch
  std::vector<RepArgs*> grp_dev;     // device tables of the grouped branches
  std::string err;
};

namespace {
int batch_fail(fg_batch* b, int rc, const std::string& msg) {
  b->err = msg;
  return rc;
}
// The batch graph of one step: a branch per replica, forked from and joined
// into the batch stream.  (Eight steps per branch, as fg_run_steps uses,
// measured no faster here: the branches already overlap.)
void free_groups(fg_batch* b) {
  for (RepArgs* p : b->grp_dev)
    if (p) cudaFree(p);
  b->grp_dev.clear();
  b->groups.clear();
}

// Branches of the batch graph: groups of replicas that one launch per kernel
// steps (enqueue_np_group), and single replicas (enqueue_step).  The device
// tables of the groups are written before the capture.
int plan_groups(fg_batch* b) {
  free_groups(b);
  std::vector<bool> used(b->ctx.size(), false);
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    if (used[i]) continue;
    std::vector<int> grp{(int)i};
    used[i] = true;
    if (b->grouping && groupable(b->ctx[i]))
      for (size_t j = i + 1; j < b->ctx.size(); ++j)
        if (!used[j] && groupable(b->ctx[j]) && same_group(b->ctx[i], b->ctx[j])) {
          grp.push_back((int)j);
          used[j] = true;
        }
    RepArgs* dev = nullptr;
    if (grp.size() > 1) {
      std::vector<RepArgs> h;
      for (int k : grp) h.push_back(rep_args(b->ctx[(size_t)k]));
      cudaError_t e = cudaMalloc(&dev, h.size() * sizeof(RepArgs));
      if (e == cudaSuccess) e = cudaMemcpy(dev, h.data(), h.size() * sizeof(RepArgs), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        if (dev) cudaFree(dev);
        return batch_fail(b, FG_ERR_CUDA, std::string("batch groups: ") + cudaGetErrorString(e));
      }
    }
    b->groups.push_back(grp);
    b->grp_dev.push_back(dev);
  }
  return FG_OK;
}

int batch_capture(fg_batch* b, cudaGraphExec_t* out) {
  if (*out) return FG_OK;
  int rc = plan_groups(b);
  if (rc) return rc;
  cudaGraph_t graph;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, cudaGetErrorString(e));
  if ((e = cudaEventRecord(b->fork, b->stream)) != cudaSuccess) rc = FG_ERR_CUDA;
  // branch priorities: the branches of the most sites at the lowest
  // priority, each smaller one a step higher (down to the device's
  // greatest), so that the short kernels of small supercells are scheduled
  // into the waves of the large ones instead of after them
  std::vector<int> prio(b->groups.size(), 0);
  if (b->priorities && b->groups.size() > 1) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    std::vector<std::pair<long long, size_t>> by_sites;
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
      long long sites = 0;
      for (int k : b->groups[gi]) sites += b->ctx[(size_t)k]->g.nsite;
      by_sites.push_back({-sites, gi});
    }
    std::sort(by_sites.begin(), by_sites.end());
    for (size_t r = 0; r < by_sites.size(); ++r) prio[by_sites[r].second] = std::max(greatest, least - (int)r);
  }
  for (size_t gi = 0; gi < b->groups.size() && rc == FG_OK; ++gi) {
    const std::vector<int>& grp = b->groups[gi];
    fg_ctx* c = b->ctx[(size_t)grp[0]];
    c->use_prio = b->priorities && b->groups.size() > 1;
    c->launch_prio = prio[gi];
    if ((e = cudaStreamWaitEvent(c->stream, b->fork, 0)) != cudaSuccess) { rc = FG_ERR_CUDA; break; }
    if (grp.size() > 1)
      rc = c->prec == FG_PREC_MIXED ? enqueue_np_group<float>(c, b->grp_dev[gi], (int)grp.size())
                                    : enqueue_np_group<double>(c, b->grp_dev[gi], (int)grp.size());
    else
      rc = enqueue_step(c);
    c->use_prio = false;
    if (rc) {
      b->err = "replica " + std::to_string(grp[0]) + ": " + c->err;
      break;
    }
    if ((e = cudaEventRecord(b->join[gi], c->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(b->stream, b->join[gi], 0)) != cudaSuccess)
      rc = FG_ERR_CUDA;
  }
  cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
  if (rc) return rc == FG_ERR_CUDA && b->err.empty() ? batch_fail(b, rc, cudaGetErrorString(e)) : rc;
  if (ee != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ee));
  e = cudaGraphInstantiateWithFlags(out, graph, b->priorities ? cudaGraphInstantiateFlagUseNodePriority : 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return FG_OK;
}
// Ready every replica for a step of the batch graph and (re)capture it:
// pending force and half step, set-up work on the replica streams finished,
// a graph whose replicas replaced buffers since its capture dropped.
int batch_prepare(fg_batch* b) {
  int rc;
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    fg_ctx* c = b->ctx[i];
    if ((rc = ensure_ready(c))) return batch_fail(b, rc, "replica " + std::to_string(i) + ": " + c->err);
    if (c->P.method == FG_METHOD_MD && (rc = np_ready_for_step(c)))
      return batch_fail(b, rc, "replica " + std::to_string(i) + ": " + c->err);
    // set-up work on the replica's own stream must finish before the batch
    // stream starts the graph
    cudaError_t ce = cudaStreamSynchronize(c->stream);
    if (ce != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, cudaGetErrorString(ce));
  }
  // a replica whose buffers were replaced (site arrays, plans) invalidates the graph
  bool stale = b->gen.size() != b->ctx.size();
  for (size_t i = 0; !stale && i < b->ctx.size(); ++i) stale = b->gen[i] != b->ctx[i]->gen;
  if (stale) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    b->gen.resize(b->ctx.size());
    for (size_t i = 0; i < b->ctx.size(); ++i) b->gen[i] = b->ctx[i]->gen;
  }
  return batch_capture(b, &b->graph);
}

// After the launches: wait for the batch stream, then every replica's
// scalars (status checked) and, with e, its energies.
int batch_finish(fg_batch* b, fg_energy* e) {
  cudaError_t ce = cudaStreamSynchronize(b->stream);
  if (ce != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, cudaGetErrorString(ce));
  int rc;
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    fg_ctx* c = b->ctx[i];
    c->force_fresh = true;
    c->flo_valid = false;
    c->np_ready = c->P.method == FG_METHOD_MD;
    if ((rc = pull_scalars(c))) return batch_fail(b, rc, "replica " + std::to_string(i) + ": " + c->err);
    if (e) energy_out(c->sc_host, &e[i], false);
  }
  return FG_OK;
}
}  // namespace

extern "C" {

void fg_batch_destroy(fg_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  free_groups(b);
  for (cudaEvent_t ev : b->join)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (fg_ctx* c : b->ctx) fg_destroy(c);
  delete b;
}

int fg_batch_create(int n, const fg_params* params, int precision, fg_batch** out, char* errbuf, int errlen) {
  auto msg = [&](const std::string& m) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
  };
  if (!out || !params || n < 1) {
    msg("fg_batch_create: n >= 1, params and out are required");
    return FG_ERR_ARG;
  }
  *out = nullptr;
  fg_batch* b = new fg_batch();
  int rc2 = FG_OK;
  for (int i = 0; i < n; ++i) {
    fg_ctx* c = nullptr;
    const int rc = fg_create(&params[i], precision, &c);
    if (rc) {
      msg("replica " + std::to_string(i) + ": " + (c ? c->err : std::string("fg_create failed")));
      if (c) fg_destroy(c);
      fg_batch_destroy(b);
      return rc;
    }
    b->ctx.push_back(c);
    if ((rc2 = apply_wisdom(c, PLAN_BATCH))) {
      msg("replica " + std::to_string(i) + ": " + c->err);
      fg_batch_destroy(b);
      return rc2;
    }
  }
  b->join.assign((size_t)n, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->join[(size_t)i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    msg(std::string("fg_batch_create: ") + cudaGetErrorString(e));
    fg_batch_destroy(b);
    return FG_ERR_CUDA;
  }
  *out = b;
  return FG_OK;
}

int fg_batch_size(const fg_batch* b) { return b ? (int)b->ctx.size() : 0; }

int fg_batch_set_grouping(fg_batch* b, int on) {
  if (!b) return FG_ERR_ARG;
  if ((on != 0) != b->grouping) {
    b->grouping = on != 0;
    if (b->graph) {
      cudaStreamSynchronize(b->stream);
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
  }
  return FG_OK;
}

int fg_batch_groups(const fg_batch* b) { return b ? (int)b->groups.size() : 0; }

int fg_batch_set_priorities(fg_batch* b, int on) {
  if (!b) return FG_ERR_ARG;
  if ((on != 0) != b->priorities) {
    b->priorities = on != 0;
    if (b->graph) {
      cudaStreamSynchronize(b->stream);
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
  }
  return FG_OK;
}

fg_ctx* fg_batch_context(fg_batch* b, int i) {
  return (b && i >= 0 && i < (int)b->ctx.size()) ? b->ctx[(size_t)i] : nullptr;
}

const char* fg_batch_last_error(const fg_batch* b) { return b ? b->err.c_str() : "null batch"; }

int fg_batch_step(fg_batch* b, int n_steps, fg_energy* e) {
  if (!b || n_steps < 0) return FG_ERR_ARG;
  int rc = batch_prepare(b);
  if (rc) return rc;
  for (int k = 0; k < n_steps; ++k) {
    cudaError_t ce = cudaGraphLaunch(b->graph, b->stream);
    if (ce != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, cudaGetErrorString(ce));
  }
  return batch_finish(b, e);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Launch plans, the autotuner and its wisdom.
//
// The reference plans each of its transforms with FFTW_MEASURE when it
// allocates the coordinates (coord_module.F:155-377), imports plans that
// were measured before from a "wisdom" file at start-up
// (feram_common.F:56-69), and ships a program that measures and exports
// them (feram_fftw_wisdom.F).  Here a plan is the z-pencil tile width (the
// kx columns one CTA of the z kernel transforms and multiplies) and the
// grid of the streaming kernels; fg_tune / fg_batch_tune time the candidates
// on the step itself and keep the fastest, and the wisdom is the table of
// the plans found, keyed by supercell, precision, components and launch kind
// (alone, or inside a replica batch), that fg_create and fg_batch_create
// consult.
namespace {

struct PlanKey {
  int mode, prec, Lx, Ly, Lz, ncx;
  bool operator<(const PlanKey& o) const {
    const int a[6] = {mode, prec, Lx, Ly, Lz, ncx}, b[6] = {o.mode, o.prec, o.Lx, o.Ly, o.Lz, o.ncx};
    return std::lexicographical_compare(a, a + 6, b, b + 6);
  }
};
struct PlanVal {
  int zcw, waves;
};
std::mutex g_wisdom_mu;
std::map<PlanKey, PlanVal> g_wisdom;

PlanKey plan_key(const fg_ctx* c, int mode) { return PlanKey{mode, c->prec, c->g.Lx, c->g.Ly, c->g.Lz, c->ncx}; }

void drop_graphs(fg_ctx* ctx) {
  for (cudaGraphExec_t* gx : {&ctx->g_np, &ctx->g_np_multi, &ctx->g_lf, &ctx->g_vs, &ctx->g_force})
    if (*gx) {
      cudaGraphExecDestroy(*gx);
      *gx = nullptr;
    }
  ++ctx->gen;  // batches holding this replica capture again
}

// Switch the context to a plan: z tiles (and their per-tile partial sums),
// the z kernels' shared-memory limit, the streaming grids; the step graphs
// are captured again at the next step.
template <typename T>
int apply_plan_t(fg_ctx* ctx, int zcw, int waves) {
  const Geom& g = ctx->g;
  int dev = 0, smem_optin = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int smem_max = smem_optin - 8192;
  const int cwmax = zcw > 0 ? std::min(zcw, z_cw_cap<T>()) : z_cw_cap<T>();
  const ZTiles zt = z_tiles(g, ctx->ncx, sizeof(cplx<T>), cwmax, smem_max);
  if ((size_t)ctx->ncx * g.Lz * zt.CW * sizeof(cplx<T>) > (size_t)smem_max)
    return fail(ctx, FG_ERR_UNSUPPORTED, "a z pencil of the supercell does not fit in shared memory");
  const int smem_z = (int)(ctx->ncx * ((size_t)g.Lz * zt.CW + kZPad<T>) * sizeof(cplx<T>));
  const int smem_z3 = (int)(3 * (size_t)g.Lz * zt.CW * sizeof(cplx<T>));
  cudaError_t ea = cudaSuccess;
  auto setattr = [&](auto kern, int bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kern);
    const int cap = smem_optin - (int)fa.sharedSizeBytes;
    if (e == cudaSuccess && bytes > cap) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
    if (e != cudaSuccess) ea = e;
  };
  with_z_kspace<T>(g.Lz, zt.CW, ctx->acou, ctx->zsite, [&](auto k) { setattr(k, smem_z); });
  with_z_pass<T, false>(g.Lz, zt.CW, [&](auto k) { setattr(k, smem_z3); });
  with_z_pass<T, true>(g.Lz, zt.CW, [&](auto k) { setattr(k, smem_z3); });
  if (ea != cudaSuccess) return fail(ctx, FG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  CK(cudaStreamSynchronize(ctx->stream));
  if (zt.nreg + zt.nnyq > ctx->zt.nreg + ctx->zt.nnyq) {
    ctx->broken = true;  // until part_k is allocated again
    cudaFree(ctx->part_k);
    ctx->part_k = nullptr;
    CK(cudaMalloc(&ctx->part_k, sizeof(double) * NQ_K * (size_t)(zt.nreg + zt.nnyq)));
    ctx->broken = false;
  }
  ctx->zt = zt;
  ctx->smem_z = smem_z;
  ctx->smem_z3 = smem_z3;
  ctx->plan_zcw = zcw;
  plan_grids<T>(ctx, waves, nsm);
  drop_graphs(ctx);
  return FG_OK;
}

int apply_plan(fg_ctx* ctx, int zcw, int waves) {
  if (ctx->broken) return fail(ctx, FG_ERR_STATE, "an earlier reallocation failed: destroy this context");
  return ctx->prec == FG_PREC_MIXED ? apply_plan_t<float>(ctx, zcw, waves) : apply_plan_t<double>(ctx, zcw, waves);
}

int apply_wisdom(fg_ctx* ctx, int mode) {
  PlanVal v{};
  {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    auto it = g_wisdom.find(plan_key(ctx, mode));
    if (it == g_wisdom.end()) return FG_OK;
    v = it->second;
  }
  if (v.zcw == ctx->plan_zcw && v.waves == ctx->plan_waves) return FG_OK;
  return apply_plan(ctx, v.zcw, v.waves);
}

void remember_plan(const fg_ctx* ctx, int mode) {
  std::lock_guard<std::mutex> lk(g_wisdom_mu);
  g_wisdom[plan_key(ctx, mode)] = PlanVal{ctx->plan_zcw, ctx->plan_waves};
}

// The candidates: z-tile widths that give distinct tiles (widest first) and
// the streaming grids (one and two resident waves, every block).
std::vector<int> zcw_candidates(const fg_ctx* ctx) {
  const int cap = ctx->prec == FG_PREC_MIXED ? z_cw_cap<float>() : z_cw_cap<double>();
  std::vector<int> out;
  int last = -1;
  for (int w = cap; w >= 1 && (int)out.size() < 3; w /= 2) {
    int cw = w;
    while (cw > 1 && ctx->g.m % cw != 0) cw /= 2;
    if (cw != last) out.push_back(w);
    last = cw;
  }
  return out;
}
const int kWaveCandidates[3] = {1, 2, 0};

// The dynamical state a tuning run overwrites: u, p (with the acoustic
// components) and the device scalars.
struct Snapshot {
  void* u = nullptr;
  void* p = nullptr;
  DevScalars sc{};
  size_t bytes = 0;
};
void snapshot_free(Snapshot* s) {
  if (s->u) cudaFree(s->u);
  if (s->p) cudaFree(s->p);
  s->u = s->p = nullptr;
}
int snapshot_take(fg_ctx* ctx, Snapshot* s) {
  int rc = pull_scalars(ctx);
  if (rc) return rc;
  s->sc = *ctx->sc_host;
  s->bytes = (ctx->acou ? 6 : 3) * ctx->real_bytes;
  CK(cudaMalloc(&s->u, s->bytes));
  CK(cudaMalloc(&s->p, s->bytes));
  CK(cudaMemcpyAsync(s->u, ctx->u, s->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(s->p, ctx->p, s->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FG_OK;
}
int snapshot_restore(fg_ctx* ctx, const Snapshot* s) {
  CK(cudaMemcpyAsync(ctx->u, s->u, s->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->p, s->p, s->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  *ctx->sc_host = s->sc;
  ctx->force_fresh = false;
  ctx->flo_valid = false;
  ctx->np_ready = false;
  return push_scalars(ctx);
}

// Fastest of `reps` timings of `steps` Nose-Poincare steps (ms per step),
// after one graph's worth of untimed steps (capture and warm-up).
int time_solo(fg_ctx* ctx, int steps, int reps, double* ms) {
  double t = 0.0, best = 1e300;
  int rc = fg_time_steps(ctx, kNpGraphSteps, &t);
  for (int r = 0; r < reps && rc == FG_OK; ++r)
    if ((rc = fg_time_steps(ctx, steps, &t)) == FG_OK) best = std::min(best, t / steps);
  *ms = best;
  return rc;
}

// Steps of every replica of the batch go on the batch stream, followed by
// one sample row of each replica.
int sample_enqueue(fg_ctx* ctx, cudaStream_t st);

}  // namespace

extern "C" {

int fg_tune(fg_ctx* ctx, int steps, int* zcw, int* waves, double* ms_per_step) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  if (steps < 1) return FG_ERR_ARG;
  if (ctx->P.method != FG_METHOD_MD) return fail(ctx, FG_ERR_UNSUPPORTED, "fg_tune times Nose-Poincare ('md') steps");
  Snapshot snap;
  if ((rc = snapshot_take(ctx, &snap))) {
    snapshot_free(&snap);
    return rc;
  }
  double best = 1e300, t = 0.0;
  int bz = ctx->plan_zcw, bw = ctx->plan_waves;
  for (int z : zcw_candidates(ctx)) {
    if ((rc = apply_plan(ctx, z, bw)) || (rc = time_solo(ctx, steps, 3, &t))) break;
    if (t < best) best = t, bz = z;
  }
  for (int w : kWaveCandidates) {
    if (rc) break;
    if (w == bw) continue;
    if ((rc = apply_plan(ctx, bz, w)) || (rc = time_solo(ctx, steps, 3, &t))) break;
    if (t < best) best = t, bw = w;
  }
  if (!rc) rc = apply_plan(ctx, bz, bw);
  if (!rc) rc = snapshot_restore(ctx, &snap);
  snapshot_free(&snap);
  if (rc) return rc;
  remember_plan(ctx, PLAN_SOLO);
  if (zcw) *zcw = ctx->zt.CW;
  if (waves) *waves = ctx->plan_waves;
  if (ms_per_step) *ms_per_step = best;
  return FG_OK;
}

int fg_set_plan(fg_ctx* ctx, int zcw, int waves) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  if (zcw < 0 || waves < 0) return fail(ctx, FG_ERR_ARG, "zcw and waves must be >= 0");
  return apply_plan(ctx, zcw, waves);
}

int fg_get_plan(const fg_ctx* ctx, int* zcw, int* waves, int* grid_kd, int* grid_asc) {
  if (!ctx) return FG_ERR_ARG;
  if (zcw) *zcw = ctx->zt.CW;
  if (waves) *waves = ctx->plan_waves;
  if (grid_kd) *grid_kd = ctx->grid_kd;
  if (grid_asc) *grid_asc = ctx->grid_asc;
  return FG_OK;
}

// Text form: a header line, then one plan per line,
// "<solo|batch> <fp64|mixed> Lx Ly Lz components zcw waves".
int fg_wisdom_export(char* buf, int len, int* needed) {
  std::string out = "feram_b200 wisdom 1\n";
  {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    for (const auto& kv : g_wisdom) {
      const PlanKey& k = kv.first;
      char line[128];
      std::snprintf(line, sizeof(line), "%s %s %d %d %d %d %d %d\n", k.mode == PLAN_BATCH ? "batch" : "solo",
                    k.prec == FG_PREC_MIXED ? "mixed" : "fp64", k.Lx, k.Ly, k.Lz, k.ncx, kv.second.zcw,
                    kv.second.waves);
      out += line;
    }
  }
  const int n = (int)out.size() + 1;
  if (needed) *needed = n;
  if (!buf) return FG_OK;
  if (len < n) return FG_ERR_ARG;
  std::memcpy(buf, out.c_str(), (size_t)n);
  return FG_OK;
}

int fg_wisdom_import(const char* text, int* n_plans) {
  if (!text) return FG_ERR_ARG;
  std::vector<std::pair<PlanKey, PlanVal>> got;
  const char* s = text;
  bool header = false;
  while (*s) {
    const char* e = std::strchr(s, '\n');
    std::string line = e ? std::string(s, (size_t)(e - s)) : std::string(s);
    s = e ? e + 1 : s + line.size();
    if (line.empty() || line[0] == '#') continue;
    if (!header) {
      if (line != "feram_b200 wisdom 1") return FG_ERR_ARG;
      header = true;
      continue;
    }
    char mode[16], prec[16];
    int Lx, Ly, Lz, ncx, zcw, waves;
    char extra;
    if (std::sscanf(line.c_str(), "%15s %15s %d %d %d %d %d %d %c", mode, prec, &Lx, &Ly, &Lz, &ncx, &zcw, &waves,
                    &extra) != 8)
      return FG_ERR_ARG;
    const std::string ms(mode), ps(prec);
    if ((ms != "solo" && ms != "batch") || (ps != "mixed" && ps != "fp64") || Lx < 1 || Ly < 1 || Lz < 1 ||
        ncx < 1 || zcw < 0 || waves < 0)
      return FG_ERR_ARG;
    got.push_back({PlanKey{ms == "batch" ? PLAN_BATCH : PLAN_SOLO, ps == "mixed" ? FG_PREC_MIXED : FG_PREC_FP64, Lx,
                           Ly, Lz, ncx},
                   PlanVal{zcw, waves}});
  }
  if (!header) return FG_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(g_wisdom_mu);
    for (const auto& kv : got) g_wisdom[kv.first] = kv.second;
  }
  if (n_plans) *n_plans = (int)got.size();
  return FG_OK;
}

void fg_wisdom_forget(void) {
  std::lock_guard<std::mutex> lk(g_wisdom_mu);
  g_wisdom.clear();
}

// The plans of one supercell measured before the runs, as the reference's
// feram_fftw_wisdom program measures FFTW plans for a supercell
// (feram_fftw_wisdom.F): a context with the run's parameters p (made by
// fg_make_param) and initialize_dipoR's seeded state, tuned over n_times
// steps; the plan goes to the wisdom (fg_wisdom_export writes it).
int fg_wisdom_measure(const fg_params* p, int n_times, int precision, char* errbuf, int errlen) {
  auto msg = [&](const std::string& m) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
  };
  if (!p || n_times < 1) {
    msg("fg_wisdom_measure: parameters and n_times >= 1 are required");
    return FG_ERR_ARG;
  }
  fg_ctx* ctx = nullptr;
  int rc = fg_create(p, precision, &ctx);
  const size_t nfield = (size_t)3 * (2 * (p->Lx / 2 + 1)) * (p->Ly + p->padding_y) * p->Lz;
  std::vector<double> u(nfield, 0.0), q(nfield, 0.0);
  if (!rc) rc = fg_build_tables(ctx);
  if (!rc && (rc = fg_init_dipoR_host(p, u.data(), q.data())) != FG_OK) msg("initialize_dipoR failed");
  if (!rc) rc = fg_set_state(ctx, u.data(), q.data(), 1.0, 0.0, 0.0);
  if (!rc) rc = fg_tune(ctx, n_times, nullptr, nullptr, nullptr);
  if (rc && ctx && !ctx->err.empty()) msg(ctx->err);
  fg_destroy(ctx);
  return rc;
}

int fg_apply_wisdom(fg_ctx* ctx) {
  if (!ctx || !ctx->stream) return FG_ERR_ARG;
  return apply_wisdom(ctx, PLAN_SOLO);
}

// ---------------------------------------------------------------------------
// Sample series and sweep points.

int fg_sample(fg_ctx* ctx) {
  int rc = ensure_ready(ctx);
  if (rc) return rc;
  return sample_enqueue(ctx, ctx->stream);
}

int fg_samples_read(fg_ctx* ctx, double* out, int max_rows, int* n_rows) {
  if (!ctx || !ctx->stream || !n_rows) return FG_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  *n_rows = ctx->n_samples;
  if (!out) return FG_OK;
  if (max_rows < ctx->n_samples) return fail(ctx, FG_ERR_ARG, "out holds fewer rows than the series");
  if (ctx->n_samples > 0)
    CK(cudaMemcpy(out, ctx->samples, sizeof(double) * kSampleCols * (size_t)ctx->n_samples, cudaMemcpyDeviceToHost));
  ctx->n_samples = 0;
  return FG_OK;
}

// One point of a temperature (field) sweep on one context: chain from the
// state on the device (fg_chain_point), n_therm steps, then n_avg steps with
// a sample row every `every` steps, as a point of the reference's cooling
// scripts runs n_thermalize and n_average steps from the previous .restart
// (cooling.sh:64-69, molecular-dynamics.F:57-110).
int fg_run_point(fg_ctx* ctx, double kelvin, const double E[3], int n_therm, int n_avg, int every, fg_energy* e) {
  if (!ctx || n_therm < 0 || n_avg < 0 || every < 1) return FG_ERR_ARG;
  if (ctx->n_samples + n_avg / every > kSampleCap)
    return fail(ctx, FG_ERR_STATE, "the sample series would overflow: read it with fg_samples_read");
  fg_energy en{};
  int rc = fg_chain_point(ctx, kelvin, E, &en);
  if (rc) return rc;
  if ((rc = np_ready_for_step(ctx))) return rc;
  int which = 0;
  cudaGraphExec_t* gx = step_graph(ctx, &which);
  auto steps = [&](int n) {
    int i = 0, r = FG_OK;
    for (; r == FG_OK && i + kNpGraphSteps <= n; i += kNpGraphSteps) r = run_graph(ctx, &ctx->g_np_multi, 4);
    for (; r == FG_OK && i < n; ++i) r = run_graph(ctx, gx, which);
    return r;
  };
  if ((rc = steps(n_therm))) return rc;
  for (int k = 0; k + every <= n_avg; k += every)
    if ((rc = steps(every)) || (rc = sample_enqueue(ctx, ctx->stream))) return rc;
  ctx->force_fresh = true;
  ctx->flo_valid = false;
  ctx->np_ready = true;
  if ((rc = pull_scalars(ctx))) return rc;
  if (e) energy_out(ctx->sc_host, e, false);
  return FG_OK;
}

}  // extern "C"

namespace {

int sample_enqueue(fg_ctx* ctx, cudaStream_t st) {
  if (!ctx->samples) CK(cudaMalloc(&ctx->samples, sizeof(double) * kSampleCols * (size_t)kSampleCap));
  if (ctx->n_samples >= kSampleCap)
    return fail(ctx, FG_ERR_STATE, "the sample series is full: read it with fg_samples_read");
  if (ctx->prec == FG_PREC_MIXED)
    k_avg_sums<float><<<ctx->grid_elem, kThreadsElem, 0, st>>>(
        (const float*)ctx->u, ctx->g, ctx->P.Z_star[0], ctx->layer_sump, ctx->part_avg, ctx->site_sump,
        (const float*)ctx->site_zstar);
  else
    k_avg_sums<double><<<ctx->grid_elem, kThreadsElem, 0, st>>>(
        (const double*)ctx->u, ctx->g, ctx->P.Z_star[0], ctx->layer_sump, ctx->part_avg, ctx->site_sump,
        (const double*)ctx->site_zstar);
  CKL();
  k_sample_row<<<1, RED_THREADS, 0, st>>>(ctx->samples + (size_t)kSampleCols * ctx->n_samples, ctx->part_avg,
                                          ctx->grid_elem, ctx->sc);
  CKL();
  ++ctx->n_samples;
  return FG_OK;
}

}  // namespace

extern "C" {

// A sweep point for every replica of the batch at once: each replica chained
// to its own temperature (kelvin[i]) and field (E[3 i .. 3 i + 2], or none),
// then n_therm and n_avg steps of the batch graph with a sample row of every
// replica each `every` steps; the host waits once, at the end.
int fg_batch_run_point(fg_batch* b, const double* kelvin, const double* E, int n_therm, int n_avg, int every) {
  if (!b || !kelvin || n_therm < 0 || n_avg < 0 || every < 1) return FG_ERR_ARG;
  int rc;
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    const fg_ctx* c = b->ctx[i];
    if (c->P.method != FG_METHOD_MD)
      return batch_fail(b, FG_ERR_UNSUPPORTED, "replica " + std::to_string(i) + ": sweep points run 'md' replicas");
    if (c->n_samples + n_avg / every > kSampleCap)
      return batch_fail(b, FG_ERR_STATE, "replica " + std::to_string(i) + ": the sample series would overflow");
  }
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    fg_ctx* c = b->ctx[i];
    fg_energy en{};
    if ((rc = fg_chain_point(c, kelvin[i], E ? E + 3 * i : nullptr, &en)))
      return batch_fail(b, rc, "replica " + std::to_string(i) + ": " + c->err);
  }
  if ((rc = batch_prepare(b))) return rc;
  auto launch = [&](int n) {
    for (int k = 0; k < n; ++k) {
      cudaError_t ce = cudaGraphLaunch(b->graph, b->stream);
      if (ce != cudaSuccess) return batch_fail(b, FG_ERR_CUDA, cudaGetErrorString(ce));
    }
    return (int)FG_OK;
  };
  if ((rc = launch(n_therm))) return rc;
  for (int k = 0; k + every <= n_avg; k += every) {
    if ((rc = launch(every))) return rc;
    for (size_t i = 0; i < b->ctx.size(); ++i)
      if ((rc = sample_enqueue(b->ctx[i], b->stream)))
        return batch_fail(b, rc, "replica " + std::to_string(i) + ": " + b->ctx[i]->err);
  }
  return batch_finish(b, nullptr);
}

// The batch autotuner: for each supercell of the batch in turn, the plan
// candidates applied to all its replicas, each timed as whole batch steps
// (the other replicas' branches run beside it, as they will), the fastest
// kept; the states are restored afterwards and the plans remembered as
// batch wisdom.
int fg_batch_tune(fg_batch* b, int steps, double* ms_before, double* ms_after) {
  if (!b || steps < 1) return FG_ERR_ARG;
  const size_t n = b->ctx.size();
  std::vector<Snapshot> snap(n);
  int rc = FG_OK;
  auto cleanup = [&](int r) {
    for (Snapshot& s : snap) snapshot_free(&s);
    return r;
  };
  for (size_t i = 0; i < n && rc == FG_OK; ++i) {
    fg_ctx* c = b->ctx[i];
    if (c->P.method != FG_METHOD_MD) rc = batch_fail(b, FG_ERR_UNSUPPORTED, "fg_batch_tune times 'md' replicas");
    else if ((rc = snapshot_take(c, &snap[i]))) rc = batch_fail(b, rc, "replica " + std::to_string(i) + ": " + c->err);
  }
  if (rc) return cleanup(rc);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto time_batch = [&](double* ms) {
    int r = batch_prepare(b);
    for (int k = 0; r == FG_OK && k < 2; ++k)
      if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) r = batch_fail(b, FG_ERR_CUDA, "graph launch");
    double best = 1e300;
    for (int rep = 0; r == FG_OK && rep < 3; ++rep) {
      cudaEventRecord(e0, b->stream);
      for (int k = 0; r == FG_OK && k < steps; ++k)
        if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) r = batch_fail(b, FG_ERR_CUDA, "graph launch");
      cudaEventRecord(e1, b->stream);
      float t = 0.0f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
        r = batch_fail(b, FG_ERR_CUDA, "batch timing events");
      best = std::min(best, (double)t / steps);
    }
    if (r == FG_OK) r = batch_finish(b, nullptr);
    *ms = best;
    return r;
  };
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = batch_fail(b, FG_ERR_CUDA, "cudaEventCreate");
  double best = 0.0, t0 = 0.0;
  if (!rc) rc = time_batch(&t0);
  best = t0;
  // one supercell (key) at a time, every replica of it on the same plan
  std::vector<bool> done(n, false);
  for (size_t i = 0; i < n && rc == FG_OK; ++i) {
    if (done[i]) continue;
    const PlanKey key = plan_key(b->ctx[i], PLAN_BATCH);
    std::vector<size_t> members;
    for (size_t j = i; j < n; ++j)
      if (!done[j] && !(plan_key(b->ctx[j], PLAN_BATCH) < key) && !(key < plan_key(b->ctx[j], PLAN_BATCH))) {
        members.push_back(j);
        done[j] = true;
      }
    int bz = b->ctx[i]->plan_zcw, bw = b->ctx[i]->plan_waves;
    auto try_plan = [&](int z, int w, bool* better) {
      *better = false;
      for (size_t j : members)
        if (int r = apply_plan(b->ctx[j], z, w)) return batch_fail(b, r, b->ctx[j]->err);
      double t = 0.0;
      int r = time_batch(&t);
      if (r == FG_OK && t < best) best = t, *better = true;
      return r;
    };
    bool better = false;
    for (int z : zcw_candidates(b->ctx[i])) {
      if (z == bz) continue;
      if ((rc = try_plan(z, bw, &better))) break;
      if (better) bz = z;
    }
    for (int w : kWaveCandidates) {
      if (rc || w == bw) continue;
      if ((rc = try_plan(bz, w, &better))) break;
      if (better) bw = w;
    }
    for (size_t j : members)
      if (!rc && (rc = apply_plan(b->ctx[j], bz, bw))) rc = batch_fail(b, rc, b->ctx[j]->err);
    if (!rc) remember_plan(b->ctx[i], PLAN_BATCH);
  }
  for (size_t i = 0; i < n && rc == FG_OK; ++i)
    if ((rc = snapshot_restore(b->ctx[i], &snap[i]))) rc = batch_fail(b, rc, b->ctx[i]->err);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc) return cleanup(rc);
  if (ms_before) *ms_before = t0;
  if (ms_after) *ms_after = best;
  return cleanup(FG_OK);
}

int fg_batch_apply_wisdom(fg_batch* b) {
  if (!b) return FG_ERR_ARG;
  for (size_t i = 0; i < b->ctx.size(); ++i)
    if (int rc = apply_wisdom(b->ctx[i], PLAN_BATCH)) return batch_fail(b, rc, b->ctx[i]->err);
  return FG_OK;
}

}  // extern "C"
