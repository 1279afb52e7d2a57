/*
 * oracle.h -- FP64 CPU restatement of the reference's MD step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 path and the timed CPU baseline; nothing in feram_b200/ links, loads
 * or calls it.  Every routine follows the Fortran subroutine it names
 * (file:line citations into t-nissie/feram in oracle.cpp), on the
 * reference's own padded column-major layout, in IEEE FP64 with OpenMP.
 *
 * Parity pins: uni64 against marsaglia_tsang_uni64_check.F:11-16; wave()
 * against wave_check.f; the inhomogeneous-strain path against the numbers
 * asserted in modulation_check.sh:64-79; the Ewald long-range table against
 * the .dat files of doc/figures/BaTiO3-000-dispersion-with-ifc; the FFT against
 * numpy.fft (pocketfft), since FFTW is absent here.
 */
#ifndef FERAM_ORACLE_H
#define FERAM_ORACLE_H
#include "../include/feram_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* alloc_Coord + dipole_dipole + elastic (feram_common.F:75-83) */
oracle_ctx* oracle_create(const fg_params* p, char* errbuf, int errlen);
void   oracle_destroy(oracle_ctx* o);
int    oracle_get_tables(oracle_ctx* o, double* short_range, double* long_range);
int    oracle_get_inhomo_tables(oracle_ctx* o, double* inhomo_K, double* inhomo_K_G, double* inhomo_coup2_K);
int    oracle_set_modulation_R(oracle_ctx* o, const double* modulation_R);
int    oracle_get_modulation(oracle_ctx* o, double* c_k_modulation_k);
int    oracle_set_state(oracle_ctx* o, const double* dipoR, const double* dipoP,
                        double s_Nose, double pi_Nose, double H0);
int    oracle_get_state(oracle_ctx* o, double* dipoR, double* dipoP, double* dVddi,
                        double* strain6, double* s_Nose, double* pi_Nose, double* H0);
int    oracle_set_acou(oracle_ctx* o, const double* acouR, const double* acouP);
/* acouR, acouP and dVdacR (acoustic-displacement MD), padded layout. */
int    oracle_get_acou(oracle_ctx* o, double* acouR, double* acouP, double* dVdacR);
int    oracle_get_acouK(oracle_ctx* o, double* acouK);
/* acouR as write_system computes it for .coord (coord_module.F:457-469) */
int    oracle_acouR_for_coord(oracle_ctx* o, double* acouR);
/* Per-site arrays (read_relaxor.F, read_defects_u.F, initialize_E_field.F),
   padded layouts, NULL keeps the current values. */
int    oracle_set_sites(oracle_ctx* o, const double* Z_starR, const double* mass_dipo_inv,
                        const double* mass_acou_inv, const int* relaxor, const int* sum_p,
                        const double* E_field_local);
int    oracle_set_uniform_E(oracle_ctx* o, const double E[3]);
int    oracle_force(oracle_ctx* o, fg_energy* e);
int    oracle_nose_poincare(oracle_ctx* o, fg_energy* e);
int    oracle_leapfrog(oracle_ctx* o, fg_energy* e, int i_step);
/* velocity_scaling (velocity_scaling.F:9-103). */
int    oracle_velocity_scaling(oracle_ctx* o, fg_energy* e);
double oracle_kinetic_energy_dipo(oracle_ctx* o);
double oracle_nose_poincare_hamiltonian(oracle_ctx* o, fg_energy* e);
/* initialize_E_field + initialize_dipoR (no .restart): uni64 Gaussian u,
   masks, first force, s = 1, pi = 0, kinetic energies. */
int    oracle_initialize(oracle_ctx* o, fg_energy* e);
/* molecular_dynamics (molecular-dynamics.F:10-160) from the current state:
   steps i_first..i_last, accumulating averages for i_step > n_thermalize.
   H0 is set from the current state when set_H0 != 0 (molecular-dynamics.F:209-212). */
int    oracle_md(oracle_ctx* o, int i_first, int i_last, int set_H0,
                 fg_energy* e, fg_average* avg);
/* add_to_Average reductions of the current state */
int    oracle_average_accumulate(oracle_ctx* o, const fg_energy* e, fg_average* avg);

/* marsaglia_tsang_uni64_module.f */
double oracle_uni64_seed(int seed1, int seed2);
double oracle_uni64(void);
double oracle_normal_dist_seed(int seed1, int seed2);
double oracle_normal_dist(double mu, double sigma);
/* wave_module.F */
void   oracle_wave(int wave_type, int i_step, int n_thermalize, int period,
                   const double amplitude[3], double out[3]);
/* Batched 3D r2c / c2r on the padded interleaved layout (FFTW plan_many
   semantics); nc = howmany.  c2r destroys its input, like FFTW's. */
int    oracle_r2c(int Lx, int Ly, int Lz, int padding_y, int nc, const double* in, double* out_complex);
int    oracle_c2r(int Lx, int Ly, int Lz, int padding_y, int nc, double* in_complex, double* out);
void   oracle_set_threads(int n);
/* read_Param defaults (param_module.F:129-194), make_Param (:452-480) and the
   no-.restart branch of initialize_dipoR (initialize-dipoR.F:41-56): inputs
   built by the oracle alone, for a CPU run that loads nothing else. */
void   oracle_default_param(fg_params* p);
int    oracle_make_param(fg_params* p);
int    oracle_init_dipoR(const fg_params* p, double* dipoR, double* dipoP);

#ifdef __cplusplus
}
#endif
#endif
