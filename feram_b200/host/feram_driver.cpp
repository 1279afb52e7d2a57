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

// write_system (coord_module.F:434-486): one line per site, ix iy iz,
// dipoR, dipoP / s_Nose, dVddi, acouR, acouP.  full_precision = 0 writes the
// reference's edit descriptors (i4,2i5,3f10.6,9e14.6,3f13.6); otherwise every
// value gets 17 significant digits, which the .restart reader of
// initialize_dipoR (initialize-dipoR.F:22-38, list-directed) and this
// library's driver read back exactly.
extern "C" int fg_write_coord(fg_ctx* ctx, const char* path, int full_precision) {
  if (!ctx || !path) return FG_ERR_ARG;
  fg_params p;
  int r = fg_get_params(ctx, &p);
  if (r) return r;
  const int NXP = 2 * (p.Lx / 2 + 1), NYP = p.Ly + p.padding_y;
  const size_t nfield = (size_t)3 * NXP * NYP * p.Lz;
  const bool acoustic = p.mass_acou[0] > 0.0;
  std::vector<double> R(nfield), P(nfield), F(nfield), A(nfield), K(nfield), AP(nfield, 0.0);
  double ss = 1.0;
  if ((r = fg_get_state(ctx, R.data(), P.data(), F.data(), nullptr, &ss, nullptr, nullptr))) return r;
  double ascale = 1.0;
  if (acoustic) {  // the dynamic acoustic field
    if ((r = fg_get_acou(ctx, A.data(), AP.data(), nullptr))) return r;
  } else {  // the relaxed acoustic displacement: acouR = c2r(-i acouK) / N
    if ((r = fg_get_acouK(ctx, K.data()))) return r;
    for (size_t k = 0; k < K.size(); k += 2) {
      const double re = K[k], im = K[k + 1];
      K[k] = im;
      K[k + 1] = -re;
    }
    if ((r = fg_fft_c2r3(ctx, K.data(), A.data()))) return r;
    ascale = p.Ninv;
  }
  std::FILE* f = std::fopen(path, "w");
  if (!f) return FG_ERR_IO;
  auto g = [](double v) {
    char b[32];
    std::snprintf(b, sizeof(b), " %.16e", v);
    return std::string(b);
  };
  for (int iz = 0; iz < p.Lz; ++iz)
    for (int iy = 0; iy < p.Ly; ++iy)
      for (int ix = 0; ix < p.Lx; ++ix) {
        const size_t o = 3 * ((size_t)ix + (size_t)NXP * ((size_t)iy + (size_t)NYP * iz));
        std::string line;
        char b[64];
        std::snprintf(b, sizeof(b), "%4d%5d%5d", ix, iy, iz);
        line += b;
        for (int a = 0; a < 3; ++a) line += full_precision ? g(R[o + a]) : fF(R[o + a], 10, 6);
        for (int a = 0; a < 3; ++a) line += full_precision ? g(P[o + a] / ss) : fE(P[o + a] / ss, 14, 6);
        for (int a = 0; a < 3; ++a) line += full_precision ? g(F[o + a]) : fE(F[o + a], 14, 6);
        for (int a = 0; a < 3; ++a) line += full_precision ? g(A[o + a] * ascale) : fE(A[o + a] * ascale, 14, 6);
        for (int a = 0; a < 3; ++a) line += full_precision ? g(AP[o + a]) : fF(AP[o + a], 13, 6);
        std::fprintf(f, "%s\n", line.c_str());
      }
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? FG_OK : FG_ERR_IO;
}

extern "C" int fg_feram_run(const char* path, int precision, fg_average* avg_out, double* t_sim, char* errbuf,
                            int errlen) {
  fg_params p;
  int rc = fg_read_param(path, &p, errbuf, errlen);
  if (rc) return rc;
  if ((rc = fg_make_param(&p, errbuf, errlen))) return rc;
  const std::string base = dir_of(path) + p.filename;
  // saved launch plans next to the input, imported before the context is
  // made, as feram_common.F:56-69 imports FFTW wisdom at start-up (a file
  // that fails to parse is reported in the .log and the default plans hold)
  std::string wisdom_msg = "GPU_WISDOM No gpu_wisdom next to the input: default launch plans.";
  {
    std::ifstream wf(dir_of(path) + "gpu_wisdom");
    if (wf) {
      std::stringstream ss;
      ss << wf.rdbuf();
      int n = 0;
      wisdom_msg = fg_wisdom_import(ss.str().c_str(), &n) == FG_OK
                       ? "GPU_WISDOM Successfully imported " + std::to_string(n) + " plans from gpu_wisdom."
                       : "GPU_WISDOM Failed to import gpu_wisdom (malformed): default launch plans.";
    }
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
  std::vector<double> dipoR(nfield, 0.0), dipoP(nfield, 0.0), acouR(nfield, 0.0), acouP(nfield, 0.0);
  const bool acoustic = p.mass_acou[0] > 0.0;
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
              acouR[o + a] = v[9 + a];
              acouP[o + a] = v[12 + a];
            }
          }
    } else {
      fg_init_dipoR_host(&p, dipoR.data(), dipoP.data());
    }
  }
  // read_relaxor (read_relaxor.F), read_defects_u (read_defects_u.F) and the
  // .localfield of initialize_E_field (initialize_E_field.F:14-45): per-site
  // arrays, uploaded when any of the three files is present
  {
    const size_t n1 = (size_t)NXP * NYP * p.Lz;
    auto at = [&](int x, int y, int z) { return (size_t)x + (size_t)NXP * ((size_t)y + (size_t)NYP * z); };
    std::vector<int> relaxor(n1, 1), sum_p(n1, 0);
    std::vector<double> zs(n1, p.Z_star[0]), minv(n1, 1.0 / p.mass_dipo[0]),
        macou(n1, p.mass_acou[0] > 0.0 ? 1.0 / p.mass_acou[0] : 0.0), eloc(3 * n1, 0.0);
    for (int z = 0; z < p.Lz; ++z)
      for (int y = 0; y < p.Ly; ++y)
        for (int x = 0; x < p.Lx; ++x) sum_p[at(x, y, z)] = 1;
    // lines "ix iy iz v1 .. vn", '#' comments; false on a malformed line
    auto read_sites = [&](const std::string& fn, int nv, auto&& apply) -> int {
      std::ifstream f(fn);
      if (!f) return 0;
      std::string line;
      int ln = 0;
      while (std::getline(f, line)) {
        ++ln;
        std::istringstream is(line);
        std::string first;
        if (!(is >> first) || first[0] == '#') continue;
        std::istringstream is2(line);
        int x, y, z;
        double v[3] = {0.0, 0.0, 0.0};
        bool ok = (bool)(is2 >> x >> y >> z);
        for (int k = 0; k < nv && ok; ++k) ok = (bool)(is2 >> v[k]);
        if (!ok || x < 0 || x >= p.Lx || y < 0 || y >= p.Ly || z < 0 || z >= p.Lz) {
          set_msg(errbuf, errlen, "there is something wrong in line " + std::to_string(ln) + " of " + fn);
          return -1;
        }
        apply(x, y, z, v);
      }
      return 1;
    };
    const int has_rel = read_sites(base + ".relaxor", 1, [&](int x, int y, int z, const double* v) {
      const int r = (int)v[0];
      relaxor[at(x, y, z)] = r;
      if (r >= 1 && r <= FG_RELAXOR_MAX) {
        zs[at(x, y, z)] = p.Z_star[r - 1];
        minv[at(x, y, z)] = 1.0 / p.mass_dipo[r - 1];
        macou[at(x, y, z)] = p.mass_acou[r - 1] > 0.0 ? 1.0 / p.mass_acou[r - 1] : 0.0;
      }
    });
    const int has_def = read_sites(base + ".defects", 3, [&](int x, int y, int z, const double* v) {
      for (int a = 0; a < 3; ++a) dipoR[3 * at(x, y, z) + a] = v[a];
      minv[at(x, y, z)] = 0.0;  // 1/infinity
      sum_p[at(x, y, z)] = 0;
    });
    const int has_loc = read_sites(base + ".localfield", 3, [&](int x, int y, int z, const double* v) {
      for (int a = 0; a < 3; ++a) eloc[3 * at(x, y, z) + a] = v[a];
    });
    if (has_rel < 0 || has_def < 0 || has_loc < 0) {
      fg_destroy(ctx);
      return FG_ERR_IO;
    }
    if (p.bulk_or_film == FG_FILM || p.bulk_or_film == FG_EPIT)
      for (int z = (p.Lz + 1) / 2; z < p.Lz; ++z)
        for (int y = 0; y < p.Ly; ++y)
          for (int x = 0; x < p.Lx; ++x) sum_p[at(x, y, z)] = 0;
    if (p.gap_id > 0) {  // read_defects_u.F:52-66
      const int gaps[2] = {0, p.Lz / 2};
      for (int g = 0; g < (p.gap_id == 2 ? 2 : 1); ++g)
        for (int y = 0; y < p.Ly; ++y)
          for (int x = 0; x < p.Lx; ++x) {
            for (int a = 0; a < 3; ++a) dipoR[3 * at(x, y, gaps[g]) + a] = p.gap_dipole_u[a];
            minv[at(x, y, gaps[g])] = 0.0;
            sum_p[at(x, y, gaps[g])] = 0;
          }
    }
    if (has_rel || has_def || has_loc) {
      rc = fg_upload_site_arrays(ctx, has_rel ? zs.data() : nullptr, minv.data(),
                                 (has_rel && p.mass_acou[0] > 0.0) ? macou.data() : nullptr,
                                 has_rel ? relaxor.data() : nullptr, sum_p.data(), has_loc ? eloc.data() : nullptr);
      if (rc) return bail(rc);
    }
  }
  if ((rc = fg_set_state(ctx, dipoR.data(), dipoP.data(), 1.0, 0.0, 0.0))) return bail(rc);
  if (acoustic && (rc = fg_set_acou(ctx, acouR.data(), acouP.data()))) return bail(rc);
  fg_energy e;
  std::memset(&e, 0, sizeof(e));
  if ((rc = fg_mirror_force_mirror(ctx, &e))) return bail(rc);
  e.acou_kinetic = 0.0;
  if ((rc = fg_kinetic_energy_dipo(ctx, &e.dipo_kinetic))) return bail(rc);
  e.H_Nose_Poincare = 0.0;
  double s = 1.0, pi = 0.0, H0 = 0.0;
  int n_sum_p = p.N;
  if (p.bulk_or_film == FG_FILM || p.bulk_or_film == FG_EPIT) n_sum_p = p.Lx * p.Ly * ((p.Lz + 1) / 2);
  if (p.gap_id > 0) n_sum_p -= p.Lx * p.Ly * (p.gap_id == 2 ? 2 : 1);
  const bool coords = std::strcmp(p.coord_directory, "never") != 0;
  // masked average of u (molecular-dynamics.F:81-84, hysteresis_loop.F:79-82)
  auto average_u = [&](double u[3]) -> int {
    fg_average tmp;
    std::memset(&tmp, 0, sizeof(tmp));
    int r = fg_average_accumulate(ctx, &e, &tmp);
    for (int a = 0; a < 3; ++a) u[a] = tmp.u[a] / n_sum_p;
    return r;
  };
  // write_system (coord_module.F:434-486)
  auto write_system = [&](const std::string& fn) -> int {
    if (!coords) return FG_OK;
    std::string path = p.coord_directory[0] ? std::string(p.coord_directory) + "/" + fn : fn;
    if (path[0] != '/') path = dir_of(base) + path;
    return fg_write_coord(ctx, path.c_str(), 0);
  };
  char step_fn[64];
  auto numbered = [&](int i_step) {
    std::snprintf(step_fn, sizeof(step_fn), ".%010d.coord", i_step);
    return std::string(p.filename) + step_fn;
  };
  std::ofstream log(base + ".log");
  log << wisdom_msg << "\n";
  fg_average avg;
  std::memset(&avg, 0, sizeof(avg));
  const int n_steps = p.n_thermalize + p.n_average;
  std::chrono::steady_clock::time_point t0, t1;
  if (p.method == FG_METHOD_HL && p.continue_run) {
    set_msg(errbuf, errlen, "'continue' keeps the state of a previous run in the same process; every fg_feram_run starts afresh");
    fg_destroy(ctx);
    return FG_ERR_UNSUPPORTED;
  }
  if (p.method == FG_METHOD_HL) {
    // hysteresis_loop (hysteresis_loop.F:9-103): velocity scaling under a
    // field ramped from +E to -E over the averaging steps
    e.total = e.acou_kinetic + e.dipo_kinetic + potential(e);
    log << "TIME_STEP        0\n";
    write_energy(log, p, e, s, pi);
    std::ofstream hl(base + ".hl");
    double Eadd[3] = {0.0, 0.0, 0.0};
    t0 = std::chrono::steady_clock::now();
    for (int i_step = p.n_hysteresis_loop_continue; i_step <= n_steps; ++i_step) {
      if (i_step >= p.n_thermalize) {
        for (int a = 0; a < 3; ++a)
          Eadd[a] = p.external_E_field[a] - 2 * p.external_E_field[a] * (i_step - p.n_thermalize) / p.n_average;
        if ((rc = fg_set_uniform_E(ctx, Eadd))) return bail(rc);
      }
      if ((rc = fg_velocity_scaling(ctx, &e))) return bail(rc);
      e.total = e.acou_kinetic + e.dipo_kinetic + potential(e);
      if (p.verbose >= 2) {
        log << "TIME_STEP " << i_step << "\n";
        write_energy(log, p, e, s, pi);
      }
      if (i_step < p.n_thermalize) continue;
      if ((i_step - p.n_thermalize) % p.n_hl_freq == 0) {
        double u[3], strain[6];
        if ((rc = average_u(u))) return bail(rc);
        if ((rc = fg_get_state(ctx, nullptr, nullptr, nullptr, strain, nullptr, nullptr, nullptr))) return bail(rc);
        char b[32];
        std::snprintf(b, sizeof(b), "%010d", i_step);
        std::string line = b + fF(p.kelvin, 6, 1);
        for (int a = 0; a < 3; ++a) line += fF(Eadd[a], 16, 12);
        for (int a = 0; a < 6; ++a) line += fE(strain[a], 13, 5);
        for (int a = 0; a < 3; ++a) line += fE(u[a], 13, 5);
        hl << line << "\n" << std::flush;
        if ((rc = write_system(std::string(p.filename) + ".coord"))) return bail(rc);
      }
      if ((i_step - p.n_thermalize) % p.n_coord_freq == 0 && (rc = write_system(numbered(i_step)))) return bail(rc);
    }
    t1 = std::chrono::steady_clock::now();
  } else {
    // molecular_dynamics (molecular-dynamics.F:10-160)
    e.total = e.dipo_kinetic / (s * s) + e.acou_kinetic + potential(e);
    log << "TIME_STEP        0\n";
    write_energy(log, p, e, s, pi);
    np_hamiltonian(p, s, pi, H0, &e);
    H0 = e.H_Nose_Poincare / s;
    np_hamiltonian(p, s, pi, H0, &e);
    if ((rc = fg_set_thermostat(ctx, s, pi, H0))) return bail(rc);
    std::ofstream hl;
    if (p.n_E_wave_period > 0) hl.open(base + ".hl");
    const bool ramping = p.E_wave_type == FG_WAVE_RAMPING_ON || p.E_wave_type == FG_WAVE_RAMPING_OFF;
    t0 = std::chrono::steady_clock::now();
    for (int i_step = 1; i_step <= n_steps; ++i_step) {
      if (p.E_wave_type != FG_WAVE_NONE) {
        double Ea[3];
        if ((rc = fg_wave(p.E_wave_type, i_step, p.n_thermalize, p.n_E_wave_period, p.external_E_field, Ea)))
          return bail(rc);
        if ((rc = fg_set_uniform_E(ctx, Ea))) return bail(rc);
        if (hl.is_open() && (i_step >= p.n_thermalize || ramping) && (i_step - p.n_thermalize) % p.n_hl_freq == 0) {
          double u[3], strain[6];
          if ((rc = average_u(u))) return bail(rc);
          if ((rc = fg_get_state(ctx, nullptr, nullptr, nullptr, strain, nullptr, nullptr, nullptr))) return bail(rc);
          char b[32];
          std::snprintf(b, sizeof(b), "%010d", i_step);
          std::string line = b + fF(p.kelvin, 6, 1);
          for (int a = 0; a < 3; ++a) line += fF(Ea[a], 16, 12);
          for (int a = 0; a < 6; ++a) line += fE(strain[a], 13, 5);
          for (int a = 0; a < 3; ++a) line += fE(u[a], 13, 5);
          for (int a = 0; a < 6; ++a) line += fF(0.0, 4, 1);
          const double ev[15] = {e.dipo_kinetic, e.short_range, e.long_range, e.dipole_E_field, e.unharmonic,
                                 e.homo_strain, e.homo_coupling, e.inho_strain, e.inho_coupling, e.inho_modulation,
                                 e.total, e.H_Nose_Poincare, e.total * e.total, e.dipo_kinetic / (s * s),
                                 e.acou_kinetic};
          for (int a = 0; a < 15; ++a) line += fE(ev[a], a == 0 ? 15 : 13, 5);
          hl << line << "\n" << std::flush;
          if ((rc = write_system(std::string(p.filename) + ".coord"))) return bail(rc);
        }
      }
      if (p.method == FG_METHOD_MD) rc = fg_nose_poincare(ctx, &e);
      else if (p.method == FG_METHOD_VS) rc = fg_velocity_scaling(ctx, &e);
      else rc = fg_leapfrog(ctx, &e, i_step);
      if (rc) return bail(rc);
      if (p.method == FG_METHOD_MD && (rc = fg_get_state(ctx, nullptr, nullptr, nullptr, nullptr, &s, &pi, nullptr)))
        return bail(rc);
      if (i_step % p.n_coord_freq == 0 && (rc = write_system(numbered(i_step)))) return bail(rc);
      e.total = e.dipo_kinetic / (s * s) + e.acou_kinetic + potential(e);
      const bool detail = p.verbose >= 2 || i_step % p.n_coord_freq == 0 || i_step == n_steps;
      if (detail) {
        log << "TIME_STEP " << i_step << "\n";
        write_energy(log, p, e, s, pi);
      }
      if (i_step <= p.n_thermalize) continue;
      if ((rc = fg_average_accumulate(ctx, &e, &avg))) return bail(rc);
      if (coords && (rc = fg_dipoRavg_accumulate(ctx))) return bail(rc);
    }
    t1 = std::chrono::steady_clock::now();
    write_avg(base + ".avg", p, avg, n_sum_p);
    // divide_and_write_dipoRavg (coord_module.F:578-608); the reference joins
    // coord_directory and the file name without a separator
    if (coords && p.n_average > 0) {
      std::vector<double> Ravg(nfield);
      if ((rc = fg_get_dipoRavg(ctx, Ravg.data()))) return bail(rc);
      std::string fn = std::string(p.coord_directory) + p.filename + ".dipoRavg";
      if (fn[0] != '/') fn = dir_of(base) + fn;
      std::FILE* f = std::fopen(fn.c_str(), "w");
      if (!f) {
        set_msg(errbuf, errlen, "cannot write " + fn);
        fg_destroy(ctx);
        return FG_ERR_IO;
      }
      for (int iz = 0; iz < p.Lz; ++iz)
        for (int iy = 0; iy < p.Ly; ++iy)
          for (int ix = 0; ix < p.Lx; ++ix) {
            const size_t o = 3 * ((size_t)ix + (size_t)NXP * ((size_t)iy + (size_t)NYP * iz));
            std::string line;
            char b[64];
            std::snprintf(b, sizeof(b), "%4d%5d%5d", ix, iy, iz);
            line += b;
            for (int a = 0; a < 3; ++a) line += fF(Ravg[o + a] / p.n_average, 10, 6);
            std::fprintf(f, "%s\n", line.c_str());
          }
      std::fclose(f);
    }
  }
  const double tsim = std::chrono::duration<double>(t1 - t0).count();
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
