// feram_driver.cpp -- the reference's per-file driver, replayed on the host
// through the public C-ABI only: feram_common (feram_common.F:9-119),
// initialize_E_field (initialize_E_field.F:6-74), initialize_dipoR
// (initialize-dipoR.F:8-71) and molecular_dynamics (molecular-dynamics.F:
// 10-160), writing .avg (average_module.F:180-261) and a .log with the
// per-step energies and the #TIMING_REPORT line.  This is what a Fortran
// caller of feram_gpu.h does; it exists because no Fortran compiler is
// available to build the reference driver against the library.
#include "../../include/feram_gpu.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

void set_msg(char* buf, int len, const std::string& s) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", s.c_str());
}

// Fortran Ew.d edit descriptor: optional sign, "0.", d digits, "E+xx".
std::string fE(double v, int w, int d) {
  char out[64];
  if (v == 0.0) {
    std::string m = "0." + std::string(d, '0') + "E+00";
    std::snprintf(out, sizeof(out), "%*s", w, m.c_str());
    return out;
  }
  double a = std::fabs(v);
  int e = (int)std::floor(std::log10(a)) + 1;
  char mant[48];
  std::snprintf(mant, sizeof(mant), "%.*f", d, a / std::pow(10.0, e));
  if (mant[0] == '1') {  // rounding carried to 1.000
    e += 1;
    std::snprintf(mant, sizeof(mant), "%.*f", d, a / std::pow(10.0, e));
  }
  char s[64];
  std::snprintf(s, sizeof(s), "%s%sE%c%02d", v < 0 ? "-" : "", mant, e < 0 ? '-' : '+', std::abs(e));
  std::snprintf(out, sizeof(out), "%*s", w, s);
  return out;
}

std::string fF(double v, int w, int d) {
  char out[64];
  std::snprintf(out, sizeof(out), "%*.*f", w, d, v);
  return out;
}

std::string dir_of(const std::string& path) {
  size_t sl = path.find_last_of('/');
  return sl == std::string::npos ? std::string() : path.substr(0, sl + 1);
}

bool file_exists(const std::string& fn) {
  std::ifstream f(fn);
  return (bool)f;
}

double potential(const fg_energy& e) {
  return e.short_range + e.long_range + e.dipole_E_field + e.unharmonic + e.homo_strain + e.homo_coupling +
         e.inho_strain + e.inho_coupling + e.inho_modulation;
}

void np_hamiltonian(const fg_params& p, double s, double pi, double H0, fg_energy* e) {  // energy_module.F:128-148
  double h = e->dipo_kinetic / (s * s) + potential(*e) + pi * pi / 2 / p.Q_Nose +
             3 * p.N * p.temperature_eV * std::log(s) - H0;
  e->H_Nose_Poincare = h * s;
}

void write_energy(std::ofstream& log, const fg_params& p, const fg_energy& e, double s, double pi) {
  auto line = [&](const char* name, double v) {
    char b[80];
    std::snprintf(b, sizeof(b), "%-15s%18.12f [eV/u.c.]", name, v);
    log << b << "\n";
  };
  line("acou_kinetic", e.acou_kinetic * p.Ninv);
  line("dipo_kinetic", e.dipo_kinetic / (s * s) * p.Ninv);
  line("short_range", e.short_range * p.Ninv);
  line("long_range", e.long_range * p.Ninv);
  line("dipole_E_field", e.dipole_E_field * p.Ninv);
  line("unharmonic", e.unharmonic * p.Ninv);
  line("homo_strain", e.homo_strain * p.Ninv);
  line("homo_coupling", e.homo_coupling * p.Ninv);
  line("inho_strain", e.inho_strain * p.Ninv);
  line("inho_coupling", e.inho_coupling * p.Ninv);
  line("inho_modulation", e.inho_modulation * p.Ninv);
  log << "--------------------------------------------\n";
  line("total_energy", e.total * p.Ninv);
  if (p.method == FG_METHOD_MD) {
    line("H_Nose_Poincare", e.H_Nose_Poincare * p.Ninv);
    char b[80];
    std::snprintf(b, sizeof(b), "s_Nose=%14.8f pi_Nose=%14.8f", s, pi);
    log << b << "\n";
  }
}

// divide_and_write_Average (average_module.F:180-261)
void write_avg(const std::string& fn, fg_params p, const fg_average& a_in, int n_sum_p) {
  fg_average a = a_in;
  if (p.n_average == 0) return;
  double* ae = &a.energy.acou_kinetic;
  for (int i = 0; i < 13; ++i) ae[i] = ae[i] / p.n_average / p.N;
  a.e2 = a.e2 / p.n_average * p.Ninv;
  a.dipo_kinetic_true = a.dipo_kinetic_true / p.n_average * p.Ninv;
  for (int i = 0; i < 6; ++i) a.strain[i] /= p.n_average;
  const bool film = p.bulk_or_film == FG_FILM || p.bulk_or_film == FG_EPIT;
  for (int i = 0; i < 3; ++i) {
    a.u[i] = film ? a.u[i] / p.n_average / n_sum_p : a.u[i] / p.n_average * p.Ninv;
    a.p[i] = film ? a.p[i] / p.n_average / n_sum_p : a.p[i] / p.n_average * p.Ninv;
  }
  for (int i = 0; i < 6; ++i) {
    a.uu[i] = film ? a.uu[i] / p.n_average / n_sum_p : a.uu[i] / p.n_average * p.Ninv;
    a.pp[i] = film ? a.pp[i] / p.n_average / n_sum_p : a.pp[i] / p.n_average * p.Ninv;
  }
  if (p.method == FG_METHOD_LF) p.kelvin = a.dipo_kinetic_true * 2 / 3 * 11604.45;
  std::ofstream f(fn);
  std::string s = fF(p.kelvin, 8, 3);
  for (int i = 0; i < 3; ++i) s += fF(p.external_E_field[i], 9, 5);
  auto grp = [&](const double* v, int n, int w0, int w, int d) {
    for (int i = 0; i < n; ++i) s += fE(v[i], i == 0 ? w0 : w, d);
  };
  grp(a.strain, 6, 15, 13, 5);
  grp(a.u, 3, 15, 13, 5);
  grp(a.uu, 6, 15, 13, 5);
  const double ev[15] = {a.energy.dipo_kinetic, a.energy.long_range, a.energy.dipole_E_field, a.energy.unharmonic,
                         a.energy.homo_strain, a.energy.homo_coupling, a.energy.inho_strain, a.energy.inho_coupling,
                         a.energy.total, a.energy.H_Nose_Poincare, a.e2, a.dipo_kinetic_true, a.energy.acou_kinetic,
                         a.energy.short_range, a.energy.inho_modulation};
  grp(ev, 15, 17, 15, 7);
  grp(a.p, 3, 15, 13, 5);
  grp(a.pp, 6, 15, 13, 5);
  f << s << "\n";
}

}  // namespace

extern "C" int fg_feram_run(const char* path, int precision, fg_average* avg_out, double* t_sim, char* errbuf,
                            int errlen) {
  fg_params p;
  int rc = fg_read_param(path, &p, errbuf, errlen);
  if (rc) return rc;
  if ((rc = fg_make_param(&p, errbuf, errlen))) return rc;
  const std::string base = dir_of(path) + p.filename;
  if (file_exists(base + ".localfield") || file_exists(base + ".defects") || file_exists(base + ".relaxor")) {
    set_msg(errbuf, errlen, "sidecar .localfield/.defects/.relaxor files are not supported by the device path");
    return FG_ERR_UNSUPPORTED;
  }
  fg_ctx* ctx = nullptr;
  rc = fg_create(&p, precision, &ctx);
  auto bail = [&](int code) {
    if (ctx) {
      set_msg(errbuf, errlen, fg_last_error(ctx));
      fg_destroy(ctx);
    }
    return code;
  };
  if (rc) return bail(rc);
  if ((rc = fg_build_tables(ctx))) return bail(rc);
  const int NXP = 2 * (p.Lx / 2 + 1), NYP = p.Ly + p.padding_y;
  const size_t nfield = (size_t)3 * NXP * NYP * p.Lz;
  // .modulation (elastic.F:184-234)
  {
    std::ifstream mf(base + ".modulation");
    if (mf) {
      std::vector<double> modR((size_t)NXP * NYP * p.Lz, 0.0);
      std::string line;
      while (std::getline(mf, line)) {
        std::istringstream is(line);
        std::string first;
        if (!(is >> first) || first[0] == '#') continue;
        std::istringstream is2(line);
        int ix, iy, iz;
        double v;
        if (!(is2 >> ix >> iy >> iz >> v)) {
          set_msg(errbuf, errlen, "there is something wrong in the .modulation file.");
          fg_destroy(ctx);
          return FG_ERR_IO;
        }
        modR[(size_t)ix + (size_t)NXP * ((size_t)iy + (size_t)NYP * iz)] = v;
      }
      if ((rc = fg_set_modulation_R(ctx, modR.data()))) return bail(rc);
    } else if (p.modulation_constant != 0.0) {
      set_msg(errbuf, errlen, "modulation_constant is non-zero, but .modulation was NOT found.");
      fg_destroy(ctx);
      return FG_ERR_IO;
    }
  }
  // initialize_E_field
  double E0[3];
  if ((rc = fg_wave(p.E_wave_type, 0, p.n_thermalize, p.n_E_wave_period, p.external_E_field, E0))) return bail(rc);
  if ((rc = fg_set_uniform_E(ctx, E0))) return bail(rc);
  // initialize_dipoR
  std::vector<double> dipoR(nfield, 0.0), dipoP(nfield, 0.0);
  {
    std::ifstream rs(base + ".restart");
    if (rs) {
      for (int iz = 0; iz < p.Lz; ++iz)
        for (int iy = 0; iy < p.Ly; ++iy)
          for (int ix = 0; ix < p.Lx; ++ix) {
            int dx, dy, dz;
            double v[15];
            if (!(rs >> dx >> dy >> dz)) {
              set_msg(errbuf, errlen, "truncated .restart file");
              fg_destroy(ctx);
              return FG_ERR_IO;
            }
            for (int k = 0; k < 15; ++k) rs >> v[k];
            const size_t o = 3 * ((size_t)ix + (size_t)NXP * ((size_t)iy + (size_t)NYP * iz));
            for (int a = 0; a < 3; ++a) {
              dipoR[o + a] = v[a];
              dipoP[o + a] = v[3 + a];
            }
          }
    } else {
      fg_init_dipoR_host(&p, dipoR.data(), dipoP.data());
    }
  }
  if ((rc = fg_set_state(ctx, dipoR.data(), dipoP.data(), 1.0, 0.0, 0.0))) return bail(rc);
  fg_energy e;
  std::memset(&e, 0, sizeof(e));
  if ((rc = fg_mirror_force_mirror(ctx, &e))) return bail(rc);
  e.acou_kinetic = 0.0;
  if ((rc = fg_kinetic_energy_dipo(ctx, &e.dipo_kinetic))) return bail(rc);
  e.H_Nose_Poincare = 0.0;
  double s = 1.0, pi = 0.0, H0 = 0.0;
  // molecular_dynamics
  std::ofstream log(base + ".log");
  e.total = e.dipo_kinetic / (s * s) + e.acou_kinetic + potential(e);
  log << "TIME_STEP        0\n";
  write_energy(log, p, e, s, pi);
  np_hamiltonian(p, s, pi, H0, &e);
  H0 = e.H_Nose_Poincare / s;
  np_hamiltonian(p, s, pi, H0, &e);
  if ((rc = fg_set_thermostat(ctx, s, pi, H0))) return bail(rc);
  fg_average avg;
  std::memset(&avg, 0, sizeof(avg));
  const int n_steps = p.n_thermalize + p.n_average;
  auto t0 = std::chrono::steady_clock::now();
  for (int i_step = 1; i_step <= n_steps; ++i_step) {
    if (p.E_wave_type != FG_WAVE_NONE) {
      double Ea[3];
      if ((rc = fg_wave(p.E_wave_type, i_step, p.n_thermalize, p.n_E_wave_period, p.external_E_field, Ea))) return bail(rc);
      if ((rc = fg_set_uniform_E(ctx, Ea))) return bail(rc);
    }
    if (p.method == FG_METHOD_MD) rc = fg_nose_poincare(ctx, &e);
    else rc = fg_leapfrog(ctx, &e, i_step);
    if (rc) return bail(rc);
    if (p.method == FG_METHOD_MD && (rc = fg_get_state(ctx, nullptr, nullptr, nullptr, nullptr, &s, &pi, nullptr)))
      return bail(rc);
    e.total = e.dipo_kinetic / (s * s) + e.acou_kinetic + potential(e);
    const bool detail = p.verbose >= 2 || i_step % p.n_coord_freq == 0 || i_step == n_steps;
    if (detail) {
      log << "TIME_STEP " << i_step << "\n";
      write_energy(log, p, e, s, pi);
    }
    if (i_step <= p.n_thermalize) continue;
    if ((rc = fg_average_accumulate(ctx, &e, &avg))) return bail(rc);
  }
  auto t1 = std::chrono::steady_clock::now();
  const double tsim = std::chrono::duration<double>(t1 - t0).count();
  int n_sum_p = p.N;
  if (p.bulk_or_film == FG_FILM || p.bulk_or_film == FG_EPIT) n_sum_p = p.Lx * p.Ly * ((p.Lz + 1) / 2);
  if (p.gap_id > 0) n_sum_p -= p.Lx * p.Ly * (p.gap_id == 2 ? 2 : 1);
  write_avg(base + ".avg", p, avg, n_sum_p);
  {
    char b[120];
    std::snprintf(b, sizeof(b), "%10.2f%15.2f%15.2f%5d     #TIMING_REPORT", 0.0, tsim, tsim, 1);
    log << "t_initialization, t_simulation,  t_total, n_threads\n" << b << "\n";
  }
  if (avg_out) *avg_out = avg;
  if (t_sim) *t_sim = tsim;
  fg_destroy(ctx);
  return FG_OK;
}
