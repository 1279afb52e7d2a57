/*
 * feram_gpu.h -- C-ABI of the B200-native feram molecular-dynamics step.
 *
 * The reference (t-nissie/feram, Fortran 90 + OpenMP + FFTW) evaluates one
 * MD time step of the first-principles effective Hamiltonian through the
 * subroutines mirror_force_mirror, dVddi_*, nose_poincare and leapfrog, all
 * of which take the derived types Param_type / Coord_type / Energy_type by
 * reference.  Those types are not interoperable, so this header replaces
 * them with plain C structs and an opaque device context.  A Fortran caller
 * binds every function below with ISO_C_BINDING (see
 * fortran/feram_gpu_iface.F90); arrays cross the boundary as plain host
 * pointers in the reference's own padded, column-major layout:
 *
 *   real field  (ncomp, 0:2*(Lx/2+1)-1, 0:Ly+padding_y-1, 0:Lz-1)
 *   complex     (ncomp, 0:Lx/2,         0:Ly+padding_y-1, 0:Lz-1)
 *   k table     (3, 3,  0:Lx/2,         0:Ly+padding_y-1, 0:Lz-1)
 *
 * (coord_module.F:91-93,139-141,247,256).  Only physical points are read;
 * real fields returned by the library carry zeros in their padding, as the
 * reference's arrays do.
 *
 * Every function returns an int status (FG_OK = 0).  The library never
 * calls exit(); the text of the last error of a context is available from
 * fg_last_error().  One context per host thread; calls on one context are
 * not re-entrant; different contexts are independent.
 */
#ifndef FERAM_GPU_H
#define FERAM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define FG_RELAXOR_MAX 3
#define FG_FILENAME_LEN 300

/* status codes */
enum {
  FG_OK = 0,
  FG_ERR_ARG = 1,          /* invalid argument or parameter combination   */
  FG_ERR_CUDA = 2,         /* CUDA runtime error                           */
  FG_ERR_NAN = 3,          /* NaN or Inf found in a reduction              */
  FG_ERR_TIMEOUT = 4,      /* a bounded device-side wait ran out           */
  FG_ERR_UNSUPPORTED = 5,  /* input outside what this build implements     */
  FG_ERR_IO = 6,           /* file could not be read or parsed             */
  FG_ERR_STATE = 7         /* call order (e.g. no tables uploaded yet)     */
};

/* bulk_or_film (param_module.F:255-263) */
enum { FG_BULK = 0, FG_FILM = 1, FG_EPIT = 2, FG_E110 = 3 };
/* method (param_module.F:33) */
enum { FG_METHOD_MD = 0, FG_METHOD_VS = 1, FG_METHOD_LF = 2, FG_METHOD_HL = 3 };
/* E_wave_type (wave_module.F:180-220) */
enum {
  FG_WAVE_NONE = 0, FG_WAVE_TRIANGULAR_COS = 1, FG_WAVE_TRIANGULAR_SIN = 2,
  FG_WAVE_RAMPING_ON = 3, FG_WAVE_RAMPING_OFF = 4, FG_WAVE_OTHER = 5
};
/* arithmetic of the device path */
enum {
  FG_PREC_FP64 = 0,   /* every field, FFT and force in FP64                  */
  FG_PREC_MIXED = 1   /* FP32 fields/FFT/forces; FP64 thermostat, strain,
                         energy accumulation                                 */
};

/*
 * Param_type (param_module.F:8-111), the members the MD step reads.
 * Units as in the reference: Angstrom, eV, ps, e, V/Angstrom.
 */
typedef struct fg_params {
  /* method, temperature, masses */
  int    method;                         /* FG_METHOD_*                    */
  int    continue_run;                   /* 'continue' tag                 */
  double GPa[3];
  double kelvin;
  double mass_dipo[FG_RELAXOR_MAX];      /* eV A^-2 ps^2                   */
  double mass_acou[FG_RELAXOR_MAX];      /* <= 0: acoustic field relaxed    */
  double Q_Nose;
  /* geometry */
  int    bulk_or_film;                   /* FG_BULK ... FG_E110            */
  int    Lx, Ly, Lz;
  int    gap_id;
  int    padding_y;
  double gap_dipole_u[3];
  double a0;
  double epi_strain;
  /* time steps */
  double dt;
  int    n_thermalize, n_average, n_E_wave_period;
  int    n_coord_freq, n_hl_freq, n_hysteresis_loop_continue;
  /* external field */
  double external_E_field[3];
  int    E_wave_type;                    /* FG_WAVE_*                      */
  /* on-site polynomial, per relaxor species */
  double P_kappa2[FG_RELAXOR_MAX], P_alpha[FG_RELAXOR_MAX], P_gamma[FG_RELAXOR_MAX];
  double P_k1[FG_RELAXOR_MAX], P_k2[FG_RELAXOR_MAX], P_k3[FG_RELAXOR_MAX], P_k4[FG_RELAXOR_MAX];
  /* inter-site */
  double j[7];
  /* elastic constants and coupling */
  double B11, B12, B44, B1xx, B1yy, B4yz, modulation_constant;
  /* dipoles */
  int    seed[2];
  double init_dipo_avg[3], init_dipo_dev[3], k_stripe[3];
  double Z_star[FG_RELAXOR_MAX];
  double epsilon_inf;
  double kappa;                          /* Ewald kappa; <= 0 -> default   */
  int    plot_dispersion, output_polarization;
  double delta_e, delta_e_acou;
  int    verbose;
  /* output directories: "" (cwd) or "never" */
  char   coord_directory[FG_FILENAME_LEN];
  char   slice_directory[FG_FILENAME_LEN];
  char   distribution_directory[FG_FILENAME_LEN];
  char   filename[FG_FILENAME_LEN];      /* basename of the .feram file    */
  /* derived by fg_make_param (make_Param, param_module.F:452-480) */
  int    N;
  double Ninv, dt_2;
  int    n_freedom;
  double unit_cell_volume;
  double pNa03[3];
  double temperature_eV;
  double target_kinetic_energy;
  int    E_field_always_zero;
} fg_params;

/* Energy_type (energy_module.F:7-23), same member order; eV per supercell */
typedef struct fg_energy {
  double acou_kinetic;
  double dipo_kinetic;
  double short_range;
  double long_range;
  double dipole_E_field;
  double unharmonic;
  double homo_strain;
  double homo_coupling;
  double inho_strain;
  double inho_coupling;
  double inho_modulation;
  double total;
  double H_Nose_Poincare;
} fg_energy;

/* Running sums of add_to_Average (average_module.F:57-128) */
typedef struct fg_average {
  fg_energy energy;       /* sum of per-step energies                       */
  double e2;              /* sum of total^2                                 */
  double dipo_kinetic_true;
  double strain[6];
  double u[3], uu[6];     /* sum of (masked) sum_R u, and of (sum u)(sum u)  */
  double p[3], pp[6];     /* same for Z* u                                   */
  int    n_steps;
} fg_average;

typedef struct fg_ctx fg_ctx;

/* ---- host-side mirror of param_module.F --------------------------------- */

/* Defaults of read_Param (param_module.F:129-194). */
void fg_default_param(fg_params* p);
/* read_Param (param_module.F:114-450): parse a .feram file.  Unknown tags,
   bad bulk_or_film, acoustic_mass_amu with method 'md' and n_E_wave_period
   not divisible by 4 are errors (FG_ERR_IO), as in the reference's stops.
   errbuf (may be NULL) receives a one-line message. */
int  fg_read_param(const char* path, fg_params* p, char* errbuf, int errlen);
/* make_Param (param_module.F:452-480): derived constants and geometry checks. */
int  fg_make_param(fg_params* p, char* errbuf, int errlen);
/* wave (wave_module.F:162-221): external field added at step i_step. */
int  fg_wave(int wave_type, int i_step, int n_thermalize, int period,
             const double amplitude[3], double out[3]);
/* Marsaglia-Tsang uni64 (marsaglia_tsang_uni64_module.f:133-168) and the
   Box-Muller normal_dist (:179-202), process-global like the reference's
   SAVE variables.  fg_uni64_seed returns the running seed count (1.0, 2.0, ..). */
double fg_uni64_seed(int seed1, int seed2);
double fg_uni64(void);
double fg_normal_dist_seed(int seed1, int seed2);
double fg_normal_dist(double mu, double sigma);
/* initialize_dipoR (initialize-dipoR.F:41-56), no-.restart branch: seeded
   Gaussian u in the reference's draw order (alpha outer, z, y, x inner),
   stripe sign flips, p = 0.  Arrays in the padded Fortran layout. */
int  fg_init_dipoR_host(const fg_params* p, double* dipoR, double* dipoP);

/* ---- device context ------------------------------------------------------ */

/* Replaces alloc_Coord (coord_module.F:67-432): validates p, allocates the
   device state for one supercell on the current CUDA device. */
int  fg_create(const fg_params* p, int precision, fg_ctx** out);
void fg_destroy(fg_ctx* ctx);
const char* fg_last_error(const fg_ctx* ctx);
/* cudaStream_t of the context, as void* (for event timing by the caller). */
void* fg_stream(fg_ctx* ctx);

/* Device-built k-space tables: replaces dipole_dipole (dipole-dipole.F:6-57:
   Ewald long range + short-range stencil) and elastic (elastic.F:7-237).
   The inhomogeneous elastic tables (inhomo_K, its Cholesky factor,
   inhomo_coup2_K) are analytic in k and evaluated inside the k-space kernel. */
int  fg_build_tables(fg_ctx* ctx);
/* Tables computed by the reference's own setup (feram_common.F:82-83),
   Fortran layout (3,3,0:Lx/2,0:Ly+padding_y-1,0:Lz-1), real*8.  The short-
   range table must be the standard feram stencil (checked to 1e-9). */
int  fg_upload_tables(fg_ctx* ctx, const double* short_range, const double* long_range);
/* c_k_modulation_k (elastic.F:183-226), complex*16 (3,0:Lx/2,...); NULL clears. */
int  fg_upload_modulation(fg_ctx* ctx, const double* c_k_modulation_k);
/* .modulation real-space field modulation_R (scalar padded field); the FFT and
   c_k = modulation_constant * k * modulation_k are done on the device. */
int  fg_set_modulation_R(fg_ctx* ctx, const double* modulation_R);
/* Long-range table as built on the device, Fortran layout, eV/A^2 (testing). */
int  fg_get_long_range(fg_ctx* ctx, double* long_range);

/* fftw_execute_dft_r2c(c%plan_r2c_3_out, in, out) (dipoFFT.F:108): batched
   3D r2c of a 3-component real field into its half spectrum, unnormalised,
   on the device FFT.  in: real field layout; out: complex*16 (3, 0:Lx/2, ...). */
int  fg_fft_r2c3(fg_ctx* ctx, const double* in, double* out);
/* fftw_execute_dft_c2r(c%plan_c2r_3_out, in, out) (dVddi-dipole-dipole.F:194):
   the inverse, unnormalised; imaginary parts of the kx = 0 and kx = Lx/2
   bins are ignored as by FFTW's half-complex convention.  in is not modified. */
int  fg_fft_c2r3(fg_ctx* ctx, const double* in, double* out);

/* The same two transforms timed on the device alone (CUDA events on the
   context's stream around each, after one untimed round): ms[0] the r2c,
   ms[1] the c2r, averaged over reps round trips of whatever the context's
   scratch holds.  Only that scratch changes (u, p, dVddi and the scalars
   stand).  No counterpart in the reference (its cufft_check.F times cuFFT
   round trips the same way, cufft_check.F:188-207). */
int  fg_time_fft(fg_ctx* ctx, int reps, double* ms);

/* ---- state --------------------------------------------------------------- */

/* Coord_type members (coord_module.F:18,25,26,48,53).  dipoR/dipoP/dVddi are
   real fields with 3 components; dVddi may be NULL. */
int  fg_set_state(fg_ctx* ctx, const double* dipoR, const double* dipoP,
                  double s_Nose, double pi_Nose, double H0);
int  fg_get_state(fg_ctx* ctx, double* dipoR, double* dipoP, double* dVddi,
                  double strain[6], double* s_Nose, double* pi_Nose, double* H0);
int  fg_set_thermostat(fg_ctx* ctx, double s_Nose, double pi_Nose, double H0);
/* Per-site arrays of Coord_type (coord_module.F:100-170) as read_relaxor
   (read_relaxor.F), read_defects_u (read_defects_u.F) and initialize_E_field
   (initialize_E_field.F:14-45) fill them: Z_starR, mass_dipo_inv and
   mass_acou_inv real*8 (0:2*(Lx/2+1)-1, 0:Ly+padding_y-1, 0:Lz-1), relaxor
   integer (same shape, species 1..3), sum_p logical as int (same shape),
   E_field_local real*8 (3, same shape).  NULL keeps the default (uniform
   species 1, the film/gap masks, no local field).  Species select their own
   on-site polynomial and masses; a local field switches the E-field term on.
   Z*(R) is Z_starR when given, else Z_star of each site's species
   (read_relaxor.F:35).  When it differs from Z_star(1) anywhere, Z*(R) u is
   transformed on its own and the long-range dipole field acts on each site
   times its Z* (dipoFFT.F:36-44, dVddi-dipole-dipole.F:38-60): three more
   force components.  Call before stepping; the step graphs are rebuilt. */
int  fg_upload_site_arrays(fg_ctx* ctx, const double* Z_starR, const double* mass_dipo_inv,
                           const double* mass_acou_inv, const int* relaxor, const int* sum_p,
                           const double* E_field_local);
/* The fg_params the context runs with (after any fg_chain_point). */
int  fg_get_params(const fg_ctx* ctx, fg_params* p);
/* The next point of a Nose-Poincare temperature or field sweep, started from
   the state on the device.  The reference's sweep scripts start each point
   from the previous point's final .coord read back as .restart
   (03example-BaTiO3-bulk-phase-transition/16x16x16-40000-10000/cooling.sh:
   64-69): that file holds dipoP / s_Nose (coord_module.F:476);
   initialize_dipoR reads it (initialize-dipoR.F:22-38), evaluates the force
   and sets s = 1, pi = 0 (:62-68); molecular_dynamics sets H0 from that
   state (molecular-dynamics.F:52-55).  This call does the same on the
   device at full precision: p <- p / s, kelvin (and the derived constants
   of make_Param) of the new point, the uniform field E (NULL keeps it),
   the force, s = 1, pi = 0, H0.  e receives the energies of the new start
   (H_Nose_Poincare = 0).  Method 'md' only. */
int  fg_chain_point(fg_ctx* ctx, double kelvin, const double E[3], fg_energy* e);
/* write_system (coord_module.F:434-486): the .coord file of the current
   state (ix iy iz, dipoR, dipoP / s_Nose, dVddi, acouR, acouP per line).
   full_precision = 0: the reference's columns (i4,2i5,3f10.6,9e14.6,
   3f13.6); otherwise 17 significant digits per value, which the .restart
   readers (initialize-dipoR.F:22-38 and fg_feram_run) read back exactly. */
int  fg_write_coord(fg_ctx* ctx, const char* path, int full_precision);
/* Acoustic displacement and momentum (Coord_type acouR, acouP,
   coord_module.F:25-31) when acoustic_mass_amu > 0 (otherwise FG_ERR_STATE:
   the acoustic field is then the relaxed one of each force evaluation).
   fg_get_acou also returns dVdacR (dVdac.F:11-63) of the last force
   evaluation; any argument may be NULL.  Both start at zero. */
int  fg_set_acou(fg_ctx* ctx, const double* acouR, const double* acouP);
int  fg_get_acou(fg_ctx* ctx, double* acouR, double* acouP, double* dVdacR);
/* acouK (complex, 3 comps) of the last force evaluation, Fortran layout. */
int  fg_get_acouK(fg_ctx* ctx, double* acouK);
/* Uniform external field E(R) = E (initialize_E_field.F:139-146,
   molecular-dynamics.F:66-76 with no .localfield).  dVddi and the energies
   of the last force evaluation are kept; the next evaluation (inside the
   next nose_poincare / leapfrog step) uses E, as in the reference.  The
   copy to the device is queued on the context's stream without waiting;
   E may be reused by the caller as soon as the call returns. */
int  fg_set_uniform_E(fg_ctx* ctx, const double E[3]);

/* The per-step field of molecular-dynamics.F:66-76 on the device: with on,
   every step of this context (fg_nose_poincare, fg_leapfrog with
   i_step != 0, fg_velocity_scaling, fg_run_steps, fg_batch_step) first
   advances a device step counter and sets the uniform field to
   wave(E_wave_type, i_step, n_thermalize, n_E_wave_period,
   external_E_field) (wave_module.F:8-67), so replicas of a batch follow
   their own field waveforms inside one graph.  i_step: the counter's value
   now (the next step is i_step + 1).  on = 0 stops the schedule; the field
   keeps its last value. */
int  fg_set_wave(fg_ctx* ctx, int on, int i_step);

/* ---- the hot path -------------------------------------------------------- */

/* mirror_force_mirror (mirror_force_mirror.F:6-89): dVddi, strain, acouK and
   every potential-energy member of e (kinetic members untouched). */
int  fg_mirror_force_mirror(fg_ctx* ctx, fg_energy* e);
/* nose_poincare (nose-poincare.F:10-78): one Nose-Poincare step.  e must hold
   the energies of the previous call on entry (the reference reads them). */
int  fg_nose_poincare(fg_ctx* ctx, fg_energy* e);
/* leapfrog (leapfrog.F:9-157), with the acoustic branch when
   acoustic_mass_amu > 0 and the delta_e / delta_e_acou heat pump. */
int  fg_leapfrog(fg_ctx* ctx, fg_energy* e, int i_step);
/* velocity_scaling (velocity_scaling.F:9-103): u moves by dt p/m, the force
   is evaluated, p is kicked by dt (zero outside sum_p) and rescaled to the
   target kinetic energy 3/2 N k T, and likewise the acoustic momenta when
   acoustic_mass_amu > 0; e->dipo_kinetic and e->acou_kinetic are the kinetic
   energies before the rescale, as in the reference. */
int  fg_velocity_scaling(fg_ctx* ctx, fg_energy* e);
/* kinetic_energy_dipo (kinetic_energy_dipo.F:14-28). */
int  fg_kinetic_energy_dipo(fg_ctx* ctx, double* ke);
/* Nose_Poincare_Hamiltonian (energy_module.F:128-148), e->H_Nose_Poincare. */
int  fg_nose_poincare_hamiltonian(fg_ctx* ctx, fg_energy* e);
/* add_to_Average (average_module.F:75-128) reductions, on the device. */
int  fg_average_accumulate(fg_ctx* ctx, const fg_energy* e, fg_average* avg);
/* c%dipoRavg += c%dipoR (molecular-dynamics.F:301-305), on the device. */
int  fg_dipoRavg_accumulate(fg_ctx* ctx);
int  fg_get_dipoRavg(fg_ctx* ctx, double* dipoRavg);

/* Run n_steps of the method of p (md, lf with i_step != 0, or vs) on the
   device as CUDA graphs (md: eight steps per graph launch while eight
   remain, then one per step); the energies of the last step are returned
   in e. */
int  fg_run_steps(fg_ctx* ctx, int n_steps, fg_energy* e);

/* ---- replica batches -------------------------------------------------------
   Independent supercells (the temperature or field points of a sweep; any
   sizes and methods md / vs / hl / lf, one precision) stepped together: one
   CUDA graph with a branch per replica, so the kernels of small supercells run
   side by side.  This replaces the reference's feram_mpi task farm
   (feram_mpi.F:33-36), which runs one .feram file per MPI rank. */
typedef struct fg_batch fg_batch;
/* n contexts from params[0..n-1] (each as fg_create); errbuf names the
   failing replica. */
int  fg_batch_create(int n, const fg_params* params, int precision, fg_batch** out,
                     char* errbuf, int errlen);
void fg_batch_destroy(fg_batch* b);
int  fg_batch_size(const fg_batch* b);
/* Replica i for set-up and read-out (fg_build_tables, fg_set_state,
   fg_get_state, ...); owned by the batch, do not fg_destroy it. */
fg_ctx* fg_batch_context(fg_batch* b, int i);
const char* fg_batch_last_error(const fg_batch* b);
/* n_steps steps of every replica's method (lf: i_step != 0); e (may be NULL)
   receives each replica's energies of the last step, e[i] for replica i.
   Replicas of one supercell size, precision and set of on-site constants
   that run bulk Nose-Poincare without per-site arrays, modulation or a
   device field schedule (typically the temperature points of a sweep) are
   stepped as one group: one launch per kernel of the step for all of them,
   the replica index in the grid; the others get a graph branch each. */
int  fg_batch_step(fg_batch* b, int n_steps, fg_energy* e);
/* Grouped launches on (default) or off (a graph branch per replica); the
   results are the same bit for bit. */
int  fg_batch_set_grouping(fg_batch* b, int on);
/* Branches of the batch graph last captured (groups and single replicas). */
int  fg_batch_groups(const fg_batch* b);
/* Launch priorities for the branches of the batch graph on (default) or off:
   the branch of the most sites at the device's lowest priority, each smaller
   one a step higher, so that the short kernels of small supercells fill the
   waves of the large ones.  Scheduling only; the results are the same bit
   for bit. */
int  fg_batch_set_priorities(fg_batch* b, int on);

/* ---- sweep points and sample series -----------------------------------------
   A point of a temperature / field sweep as the reference's sweep scripts run
   it (cooling.sh:64-69: each point a feram run of n_thermalize + n_average
   steps started from the previous point's .restart; molecular-dynamics.F:57-110),
   with the state kept on the device.  Every `every` averaging steps a sample
   row of FG_SAMPLE_COLS doubles goes to a series on the device:
     0-2   sum_R u(R)       (counted sites, as average_module.F:75-128 sums)
     3-5   sum_R Z*(R) u(R)
     6     potential energy (the nine terms of the total)
     7     dipo_kinetic / s^2
     8, 9  s, pi
     10-15 homogeneous strain (xx, yy, zz, yz, zx, xy)
   so that averages, block errors and susceptibilities are taken afterwards. */
#define FG_SAMPLE_COLS 16
#define FG_SAMPLE_CAP 8192   /* rows a context holds between two reads */
/* Append one row for the present state (no host wait). */
int  fg_sample(fg_ctx* ctx);
/* Waits for the context's stream, sets *n_rows to the rows held; with out
   (room for max_rows rows) copies them and empties the series. */
int  fg_samples_read(fg_ctx* ctx, double* out, int max_rows, int* n_rows);
/* fg_chain_point(kelvin, E), n_therm steps, then n_avg steps with a row
   every `every` steps ('md' only).  e (may be NULL): energies at the end. */
int  fg_run_point(fg_ctx* ctx, double kelvin, const double E[3], int n_therm, int n_avg, int every,
                  fg_energy* e);
/* The same for every replica of a batch at once: replica i chained to
   kelvin[i] and field E[3i..3i+2] (E may be NULL), then the batch graph; the
   rows go to each replica's series (read with fg_batch_context +
   fg_samples_read).  The host waits once, at the end. */
int  fg_batch_run_point(fg_batch* b, const double* kelvin, const double* E, int n_therm, int n_avg,
                        int every);

/* ---- launch plans, the autotuner and wisdom ----------------------------------
   The reference plans its transforms with FFTW_MEASURE (coord_module.F:155-377)
   and imports saved FFTW wisdom at start-up (feram_common.F:56-69,
   feram_fftw_wisdom.F).  Here a plan is the z-pencil tile width (kx columns
   per CTA of the z kernel; the widest that divides Lx/2 and fits shared
   memory, up to 8 (mixed) / 4 (fp64)) and the grid of the streaming kernels
   (waves: 1 or 2 resident waves of blocks, 0 = one block per 256 sites).
   fg_tune times the candidates on the context's own Nose-Poincare steps and
   keeps the fastest; the state (u, p, strain, s, pi, H0) is restored after
   it.  The result goes to the process's wisdom, which fg_create (solo) and
   fg_batch_create (batch) apply to every later context of the same supercell,
   precision and component count.  Plans change the order of the energies'
   partial sums only: forces are the same bit for bit. */
int  fg_tune(fg_ctx* ctx, int steps, int* zcw, int* waves, double* ms_per_step);
/* Times the plans of each supercell of the batch as whole batch steps
   (replicas of one supercell share a plan) and keeps the fastest; states
   restored.  ms_before / ms_after: ms per batch step (may be NULL). */
int  fg_batch_tune(fg_batch* b, int steps, double* ms_before, double* ms_after);
/* A plan set by hand (zcw 0: the widest that fits). */
int  fg_set_plan(fg_ctx* ctx, int zcw, int waves);
/* The tile width in use, the waves setting and the two main grids. */
int  fg_get_plan(const fg_ctx* ctx, int* zcw, int* waves, int* grid_kd, int* grid_asc);
/* Wisdom as text: "feram_b200 wisdom 1", then one line per plan
   "<solo|batch> <fp64|mixed> Lx Ly Lz components zcw waves".  Export sets
   *needed (bytes with the NUL) and copies when len is large enough (buf may be
   NULL to ask the size); import adds the plans (all or, on a malformed line,
   none: FG_ERR_ARG). */
int  fg_wisdom_export(char* buf, int len, int* needed);
int  fg_wisdom_import(const char* text, int* n_plans);
void fg_wisdom_forget(void);
/* feram_fftw_wisdom's measurement for one supercell before the runs: a
   context with the run's parameters p (after fg_make_param) and
   initialize_dipoR's seeded state, fg_tune over n_times steps; the plan goes
   to the wisdom.  fg_feram_run imports a file "gpu_wisdom" next to the
   .feram input, if there is one, before it creates the context. */
int  fg_wisdom_measure(const fg_params* p, int n_times, int precision, char* errbuf, int errlen);
/* Apply the wisdom to a context / the replicas of a batch created before the
   import. */
int  fg_apply_wisdom(fg_ctx* ctx);
int  fg_batch_apply_wisdom(fg_batch* b);

/* ---- measurement ----------------------------------------------------------
   CUDA-event timing on the context's own stream (no host work in between). */
#define FG_NPROF 5
/* Time n_steps steps of p's method launched as fg_run_steps launches them;
   *ms = total.  A graph not yet instantiated is first captured and run once
   untimed (one step, or eight for the eight-step graph), so the state may
   advance by up to eight steps more than n_steps. */
int  fg_time_steps(fg_ctx* ctx, int n_steps, double* ms);
/* One bulk Nose-Poincare step launched kernel by kernel (the same kernels as
   the step's graph) with an event between kernels, averaged over reps steps;
   ms[i] (i < FG_NPROF) per kernel, in the order named by fg_profile_name(i).
   The steps advance the state. */
int  fg_profile_step(fg_ctx* ctx, int reps, double* ms);
const char* fg_profile_name(int i);

/* ---- host driver ----------------------------------------------------------
   feram_common + molecular_dynamics (feram_common.F:9-119,
   molecular-dynamics.F:10-160) replayed on the host through the calls above:
   reads <path>.feram, builds tables on the device, initialises u with
   uni64, runs n_thermalize + n_average steps and writes <filename>.avg and
   <filename>.log in the reference's formats.  t_sim receives the stepping
   time in seconds (the reference's t_simulation). */
int  fg_feram_run(const char* path, int precision, fg_average* avg_out,
                  double* t_sim, char* errbuf, int errlen);

/* ---- learned warm start (no counterpart in the reference) ---------------
   A periodic 3D convolutional network (3x3x3 kernels, 16 -> 32 -> 32 -> 32
   -> 16 channels, SiLU, BF16 weights, FP32 accumulation on the tensor cores)
   that maps a sweep point's condition and a seeded noise field to a proposed
   local-mode field u(R), to start that point's MD closer to equilibrium than
   the previous point's state (fg_chain_point, the reference's .restart
   chaining of cooling.sh:64-69) would.  It is trained on the site statistics
   of configurations generated by the MD: the mean dipole along the field,
   |<u>|^2, sum_a <u_a>^4, <|u|^2>, <sum_a u_a^4> and the longitudinal and
   transverse nearest-neighbour correlations (FG_WS_NSTAT values per sample).
     cond[b*5 .. +5] = (kelvin, E_x, E_y, E_z [V/A], GPa) of sample b
     seeds[b]        = the noise seed of sample b
   A net holds `batch` samples of Lx*Ly*Lz sites (a multiple of 128 sites in
   all).  Every call runs on the net's own stream and returns when done. */
#define FG_WS_NSTAT 7
typedef struct fg_ws fg_ws;
int  fg_ws_create(int Lx, int Ly, int Lz, int batch, unsigned long long seed, fg_ws** out);
void fg_ws_destroy(fg_ws* n);
const char* fg_ws_last_error(const fg_ws* n);
/* Forward pass of every sample; S (may be NULL) receives [batch][FG_WS_NSTAT]. */
int  fg_ws_forward(fg_ws* n, const float* cond, const unsigned long long* seeds, float* S);
/* Forward, the moment-matching loss sum_k w_k (S_k - target_k)^2 averaged
   over the samples (target [batch][FG_WS_NSTAT], weights [FG_WS_NSTAT]),
   and its gradients into each layer's dW, db (fg_ws_get_layer). */
int  fg_ws_backward(fg_ws* n, const float* cond, const unsigned long long* seeds, const float* target,
                    const float* weights, float* loss);
/* The same with a further gradient dL/du [batch][Lx Ly Lz][3] (sites x
   fastest) from a loss term outside the statistics, e.g. the potential
   energy of each generated field, whose gradient is the MD force dVddi
   (the loss value then covers the statistics only). */
int  fg_ws_backward_du(fg_ws* n, const float* cond, const unsigned long long* seeds, const float* target,
                       const float* weights, const float* dLdu, float* loss);
/* One Adam step (Kingma & Ba) with the gradients of the last fg_ws_backward. */
int  fg_ws_adam(fg_ws* n, float lr);
/* Layer l (0..3): [cout][27][cin] weights (tap t = 9 (dz+1) + 3 (dy+1) +
   (dx+1)), bias [cout], and their gradients; channel counts padded. */
int  fg_ws_layer_shape(const fg_ws* n, int l, int* cout, int* cin);
int  fg_ws_get_layer(fg_ws* n, int l, float* w, float* b, float* dw, float* db);
int  fg_ws_set_layer(fg_ws* n, int l, const float* w, const float* b);
/* Of the last forward: the layer-1 input [batch*nsite][16] and the generated
   u [batch*nsite][3] (sites x + Lx (y + Ly z) per sample); either may be NULL. */
int  fg_ws_get_io(fg_ws* n, float* input, float* u);
/* Sample b's generated u in the reference's padded dipoR layout, for
   fg_set_state. */
int  fg_ws_field(fg_ws* n, int b, int padding_y, double* dipoR);

/* ---- allocation-free entry point (no counterpart in the reference) -------
   kinetic_energy_dipo (kinetic_energy_dipo.F:14-28) of a momentum field the
   caller already holds in device memory, for callers that cannot allocate at
   that point: a driver running the MD from its own device memory pool under
   a fixed budget, or a host thread that must not enter the CUDA allocator.
   It needs no fg_ctx and allocates nothing: its block partials and per-layer
   tables live in one fixed device array of 5248 doubles (41 KiB) inside the
   library.
     dipoP           device, FP64, component-major [3][Lz][Ly][Lx], contiguous
     layer_mass_inv  host, Lz values of m^-1 per z-layer
     layer_sum_p     host, Lz flags of the sum_p mask (1 = layer counted)
     stream          a cudaStream_t (NULL = the legacy default stream)
     ke              device pointer; receives sum p^2 m^-1 * N / (2 n_sum_p),
                     n_sum_p = Lx*Ly*(counted layers), when the stream gets there
   Lz > FG_NOALLOC_MAX_LZ, a null pointer or a mask that counts no layer give
   FG_ERR_ARG and a message in errbuf (may be NULL).  The first call on each
   device does a one-time set-up (it looks up the array's device address) and
   should come before any stream capture; a set-up that fails is not kept,
   and the next call tries it again.  The two host tables are copied from
   ordinary (pageable) host memory, so the call may wait until the stream
   has taken them, and no call can be captured into a CUDA graph.  All calls on one device share the array: calls that
   overlap in time (different streams or host threads) race, and the caller
   must order them. */
#define FG_NOALLOC_MAX_LZ 1024
int  fg_kinetic_energy_dipo_noalloc(const double* dipoP, int Lx, int Ly, int Lz,
                                    const double* layer_mass_inv, const unsigned char* layer_sum_p,
                                    void* stream, double* ke, char* errbuf, int errlen);

#ifdef __cplusplus
}
#endif
#endif /* FERAM_GPU_H */
