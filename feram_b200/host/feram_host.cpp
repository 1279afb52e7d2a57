// feram_host.cpp -- host-side mirror of the reference's parameter handling
// and initialisation: the .feram parser (param_module.F:114-480), the
// external-field waveform (wave_module.F:162-221) and the seeded initial
// dipole field (initialize-dipoR.F:41-56 with the Marsaglia-Tsang uni64
// generator of marsaglia_tsang_uni64_module.f:112-202).
//
// These run once per input file on the CPU, exactly where the reference
// runs them; the per-step work is on the GPU (feram_b200/csrc).
#include "../../include/feram_gpu.h"

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace {

const double kKelvinEV = 11604.45;          // define.h:34
const double kElementaryCharge = 1.60217653; // define.h:35
const double kPi = 3.14159265358979323846;   // define.h:21
const double k2Pi = 6.28318530717958647693;  // define.h:22

void set_msg(char* buf, int len, const std::string& s) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", s.c_str());
}

// Fortran list-directed tokenisation of one input line: values are separated
// by blanks or commas; a quoted string is one value; a slash ends the record.
std::vector<std::string> tokens(const std::string& line) {
  std::vector<std::string> out;
  size_t i = 0, n = line.size();
  while (i < n) {
    char c = line[i];
    if (c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n') { ++i; continue; }
    if (c == '/') break;
    if (c == '\'' || c == '"') {
      char q = c;
      size_t j = i + 1;
      std::string s;
      while (j < n && line[j] != q) s += line[j++];
      out.push_back(s);
      i = (j < n) ? j + 1 : n;
      continue;
    }
    size_t j = i;
    while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '/' && line[j] != '\r' &&
           line[j] != '\n')
      ++j;
    out.push_back(line.substr(i, j - i));
    i = j;
  }
  return out;
}

bool to_double(const std::string& t, double* v) {
  if (t.empty()) return false;
  std::string s = t;
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  double x = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') return false;
  *v = x;
  return true;
}

bool to_int(const std::string& t, int* v) {
  if (t.empty()) return false;
  char* end = nullptr;
  long x = std::strtol(t.c_str(), &end, 10);
  if (end == t.c_str() || *end != '\0') return false;
  *v = (int)x;
  return true;
}

// Fortran logical input: optional leading '.', then T or F.
bool to_logical(const std::string& t, int* v) {
  size_t i = 0;
  if (i < t.size() && t[i] == '.') ++i;
  if (i >= t.size()) return false;
  char c = (char)std::toupper((unsigned char)t[i]);
  if (c == 'T') { *v = 1; return true; }
  if (c == 'F') { *v = 0; return true; }
  return false;
}

// read n doubles from tokens[2..]; false if any is missing or malformed
bool read_doubles(const std::vector<std::string>& tk, double* out, int n) {
  if ((int)tk.size() < 2 + n) return false;
  for (int i = 0; i < n; ++i)
    if (!to_double(tk[2 + i], &out[i])) return false;
  return true;
}
bool read_ints(const std::vector<std::string>& tk, int* out, int n) {
  if ((int)tk.size() < 2 + n) return false;
  for (int i = 0; i < n; ++i)
    if (!to_int(tk[2 + i], &out[i])) return false;
  return true;
}

// Per-species tags: RELAXOR_MAX values if they all read, else one value
// replicated (param_module.F:307-316 and the like).
bool read_species(const std::vector<std::string>& tk, double* out) {
  double v[FG_RELAXOR_MAX];
  if (read_doubles(tk, v, FG_RELAXOR_MAX)) {
    for (int i = 0; i < FG_RELAXOR_MAX; ++i) out[i] = v[i];
    return true;
  }
  if (!read_doubles(tk, v, 1)) return false;
  for (int i = 0; i < FG_RELAXOR_MAX; ++i) out[i] = v[0];
  return true;
}

void copy_str(char* dst, const std::string& s) {
  std::snprintf(dst, FG_FILENAME_LEN, "%s", s.c_str());
}

int wave_code(const std::string& s) {
  if (s.empty()) return FG_WAVE_NONE;
  if (s == "triangular_cos") return FG_WAVE_TRIANGULAR_COS;
  if (s == "triangular_sin") return FG_WAVE_TRIANGULAR_SIN;
  if (s == "ramping_on") return FG_WAVE_RAMPING_ON;
  if (s == "ramping_off") return FG_WAVE_RAMPING_OFF;
  return FG_WAVE_OTHER;
}

// ---- Marsaglia-Tsang uni64, process-global like the reference's SAVE ----
struct Uni64State {
  int i = 97, j = 33;
  double c = 0.0, times = 0.0;
  double u[97] = {0};
  bool sw = true;        // normal_dist's saved switch
  double t = 0.0, phi = 0.0;
};
Uni64State g_rng;

int32_t mul_wrap(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

void fillu(int32_t x, int32_t y) {
  // fillu (marsaglia_tsang_uni64_module.f:112-131); 32-bit products wrap.
  for (int ii = 0; ii < 97; ++ii) {
    double s = 0.0, t = 0.5;
    for (int jj = 0; jj < 53; ++jj) {
      x = mul_wrap(6969, x) % 65543;
      y = mul_wrap(8888, y) % 65579;
      if (((x ^ y) & 32) > 0) s = s + t;
      t = 0.5 * t;
    }
    g_rng.u[ii] = s;
  }
}

double uni64_next() {
  const double r = 9007199254740881.0 / 9007199254740992.0;
  const double d = 362436069876.0 / 9007199254740992.0;
  double x = g_rng.u[g_rng.i - 1] - g_rng.u[g_rng.j - 1];
  if (x < 0.0) x = x + 1.0;
  g_rng.u[g_rng.i - 1] = x;
  if (--g_rng.i == 0) g_rng.i = 97;
  if (--g_rng.j == 0) g_rng.j = 97;
  g_rng.c = g_rng.c - d;
  if (g_rng.c < 0.0) g_rng.c = g_rng.c + r;
  x = x - g_rng.c;
  return (x < 0.0) ? x + 1.0 : x;
}

}  // namespace

extern "C" {

void fg_default_param(fg_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->method = FG_METHOD_MD;
  for (int i = 0; i < FG_RELAXOR_MAX; ++i) {
    p->mass_dipo[i] = 100.0 / 9648.53377163899;
    p->mass_acou[i] = -100.0;
  }
  p->Q_Nose = 0.1;
  p->bulk_or_film = FG_BULK;
  p->Lx = p->Ly = p->Lz = 32;
  p->gap_id = 0;
  p->padding_y = 1;
  p->a0 = 4.0;
  p->n_thermalize = 10000;
  p->n_average = 100000;
  p->n_E_wave_period = 0;
  p->n_coord_freq = 2147483647;  // huge(1)
  p->n_hl_freq = 10000;
  p->n_hysteresis_loop_continue = 1;
  p->E_wave_type = FG_WAVE_NONE;
  p->seed[0] = 123456789;
  p->seed[1] = 987654321;
  for (int i = 0; i < 3; ++i) p->init_dipo_dev[i] = 0.05;
  p->verbose = 1;
  p->E_field_always_zero = 1;
}

int fg_read_param(const char* path, fg_params* p, char* errbuf, int errlen) {
  fg_default_param(p);
  std::ifstream in(path);
  if (!in) {
    set_msg(errbuf, errlen, std::string(path) + ": cannot open");
    return FG_ERR_IO;
  }
  {  // filename = basename without the .feram suffix (feram_common.F:38-41)
    std::string fn(path);
    size_t sl = fn.find_last_of('/');
    if (sl != std::string::npos) fn = fn.substr(sl + 1);
    if (fn.size() > 6 && fn.substr(fn.size() - 6) == ".feram") fn = fn.substr(0, fn.size() - 6);
    copy_str(p->filename, fn);
  }
  std::string line, wave_name;
  int line_number = 0;
  while (std::getline(in, line)) {
    ++line_number;
    std::vector<std::string> tk = tokens(line);
    if (tk.empty() || tk[0][0] == '#') continue;
    const std::string& name = tk[0];
    auto fail = [&](const std::string& why) {
      set_msg(errbuf, errlen, std::string(path) + ":" + std::to_string(line_number) + ": " + line + ": " + why);
      return FG_ERR_IO;
    };
    bool ok = true;
    if (name == "method") {
      ok = tk.size() >= 3;
      if (ok) {
        const std::string& m = tk[2];
        if (m == "md") p->method = FG_METHOD_MD;
        else if (m == "vs") p->method = FG_METHOD_VS;
        else if (m == "lf") p->method = FG_METHOD_LF;
        else if (m == "hl") p->method = FG_METHOD_HL;
        else return fail("illegal or not-yet-implemented method");
        if (p->method == FG_METHOD_HL) p->E_field_always_zero = 0;
      }
    } else if (name == "E_wave_type") {
      ok = tk.size() >= 3;
      if (ok) {
        wave_name = tk[2];
        p->E_wave_type = wave_code(wave_name);
        p->E_field_always_zero = 0;
      }
    } else if (name == "GPa") {
      if (!read_doubles(tk, p->GPa, 3)) {  // hydrostatic (param_module.F:216-223)
        double g;
        ok = read_doubles(tk, &g, 1);
        p->GPa[0] = p->GPa[1] = p->GPa[2] = g;
      }
    } else if (name == "kelvin") {
      ok = read_doubles(tk, &p->kelvin, 1);
      p->temperature_eV = p->kelvin / kKelvinEV;
    } else if (name == "mass_amu") {
      double m[FG_RELAXOR_MAX];
      ok = read_species(tk, m);
      for (int i = 0; i < FG_RELAXOR_MAX; ++i) p->mass_dipo[i] = m[i] / 9648.53377163899;
    } else if (name == "acoustic_mass_amu") {
      if (p->method == FG_METHOD_MD) return fail("You cannot use method = 'md' togeter with acoustic_mass_amu.");
      double m[FG_RELAXOR_MAX];
      ok = read_species(tk, m);
      for (int i = 0; i < FG_RELAXOR_MAX; ++i) p->mass_acou[i] = m[i] / 9648.53377163899;
    } else if (name == "Q_Nose") {
      ok = read_doubles(tk, &p->Q_Nose, 1);
    } else if (name == "bulk_or_film") {
      ok = tk.size() >= 3;
      if (ok) {
        const std::string& b = tk[2];
        if (b == "bulk") p->bulk_or_film = FG_BULK;
        else if (b == "film") p->bulk_or_film = FG_FILM;
        else if (b == "epit") p->bulk_or_film = FG_EPIT;
        else if (b == "e110") p->bulk_or_film = FG_E110;
        else return fail("Input error: bulk_or_film must be bulk, film or epit.");
      }
    } else if (name == "L") {
      int v[3];
      ok = read_ints(tk, v, 3);
      if (ok) { p->Lx = v[0]; p->Ly = v[1]; p->Lz = v[2]; }
    } else if (name == "padding_y") {
      ok = read_ints(tk, &p->padding_y, 1);
    } else if (name == "gap_id") {
      ok = read_ints(tk, &p->gap_id, 1);
    } else if (name == "gap_dipole_u") {
      ok = read_doubles(tk, p->gap_dipole_u, 3);
    } else if (name == "a0") {
      ok = read_doubles(tk, &p->a0, 1);
    } else if (name == "epi_strain") {
      ok = read_doubles(tk, &p->epi_strain, 1);
    } else if (name == "dt") {
      ok = read_doubles(tk, &p->dt, 1);
    } else if (name == "n_thermalize") {
      ok = read_ints(tk, &p->n_thermalize, 1);
    } else if (name == "n_average") {
      ok = read_ints(tk, &p->n_average, 1);
    } else if (name == "n_E_wave_period") {
      ok = read_ints(tk, &p->n_E_wave_period, 1);
      if (ok && wave_name.compare(0, 7, "ramping") != 0 && p->n_E_wave_period % 4 != 0)
        return fail("Input error: n_E_wave_period must be divided by 4.");
    } else if (name == "n_coord_freq") {
      ok = read_ints(tk, &p->n_coord_freq, 1);
    } else if (name == "n_hl_freq") {
      ok = read_ints(tk, &p->n_hl_freq, 1);
    } else if (name == "external_E_field") {
      ok = read_doubles(tk, p->external_E_field, 3);
      if (ok && (p->external_E_field[0] != 0.0 || p->external_E_field[1] != 0.0 || p->external_E_field[2] != 0.0))
        p->E_field_always_zero = 0;
    } else if (name == "n_hysteresis_loop_continue") {
      ok = read_ints(tk, &p->n_hysteresis_loop_continue, 1);
    } else if (name == "coord_directory") {
      ok = tk.size() >= 3;
      if (ok) copy_str(p->coord_directory, tk[2]);
    } else if (name == "slice_directory") {
      ok = tk.size() >= 3;
      if (ok) copy_str(p->slice_directory, tk[2]);
    } else if (name == "distribution_directory") {
      ok = tk.size() >= 3;
      if (ok) copy_str(p->distribution_directory, tk[2]);
    } else if (name == "P_kappa2") {
      ok = read_species(tk, p->P_kappa2);
    } else if (name == "P_alpha") {
      ok = read_species(tk, p->P_alpha);
    } else if (name == "P_gamma") {
      ok = read_species(tk, p->P_gamma);
    } else if (name == "P_k1") {
      ok = read_species(tk, p->P_k1);
    } else if (name == "P_k2") {
      ok = read_species(tk, p->P_k2);
    } else if (name == "P_k3") {
      ok = read_species(tk, p->P_k3);
    } else if (name == "P_k4") {
      ok = read_species(tk, p->P_k4);
    } else if (name == "j") {
      ok = read_doubles(tk, p->j, 7);
    } else if (name == "B11") {
      ok = read_doubles(tk, &p->B11, 1);
    } else if (name == "B12") {
      ok = read_doubles(tk, &p->B12, 1);
    } else if (name == "B44") {
      ok = read_doubles(tk, &p->B44, 1);
    } else if (name == "B1xx") {
      ok = read_doubles(tk, &p->B1xx, 1);
    } else if (name == "B1yy") {
      ok = read_doubles(tk, &p->B1yy, 1);
    } else if (name == "B4yz") {
      ok = read_doubles(tk, &p->B4yz, 1);
    } else if (name == "modulation_constant") {
      ok = read_doubles(tk, &p->modulation_constant, 1);
    } else if (name == "seed") {
      ok = read_ints(tk, p->seed, 2);
    } else if (name == "init_dipo_avg") {
      ok = read_doubles(tk, p->init_dipo_avg, 3);
    } else if (name == "init_dipo_dev") {
      ok = read_doubles(tk, p->init_dipo_dev, 3);
    } else if (name == "k_stripe") {
      ok = read_doubles(tk, p->k_stripe, 3);
    } else if (name == "Z_star") {
      ok = read_species(tk, p->Z_star);
    } else if (name == "epsilon_inf") {
      ok = read_doubles(tk, &p->epsilon_inf, 1);
    } else if (name == "kappa") {
      ok = read_doubles(tk, &p->kappa, 1);
    } else if (name == "continue") {
      ok = tk.size() >= 3 && to_logical(tk[2], &p->continue_run);
    } else if (name == "plot_dispersion") {
      ok = tk.size() >= 3 && to_logical(tk[2], &p->plot_dispersion);
    } else if (name == "output_polarization") {
      ok = tk.size() >= 3 && to_logical(tk[2], &p->output_polarization);
    } else if (name == "delta_e") {
      ok = read_doubles(tk, &p->delta_e, 1);
    } else if (name == "delta_e_acou") {
      ok = read_doubles(tk, &p->delta_e_acou, 1);
    } else if (name == "verbose") {
      ok = read_ints(tk, &p->verbose, 1);
    } else if (name.size() == 5 && name.compare(0, 4, "DDB_") == 0 && name[4] >= 'a' && name[4] <= 'g') {
      double dummy;
      ok = read_doubles(tk, &dummy, 1);  // feram_eigenvalues2j.F only
    } else {
      return fail("Input error: No such parameter");
    }
    if (!ok) return fail("cannot read the value(s)");
  }
  return FG_OK;
}

int fg_make_param(fg_params* p, char* errbuf, int errlen) {
  if (p->Lx < 1 || p->Ly < 1 || p->Lz < 1) {
    set_msg(errbuf, errlen, "L must be positive");
    return FG_ERR_ARG;
  }
  p->N = p->Lx * p->Ly * p->Lz;
  p->Ninv = 1.0 / p->N;
  p->dt_2 = p->dt / 2;
  p->n_freedom = 3 * p->N;
  if (p->kappa <= 0.0) p->kappa = std::sqrt(kPi) / p->a0 / std::pow((double)p->N, 1.0 / 6);
  p->unit_cell_volume = p->a0 * p->a0 * p->a0;
  for (int i = 0; i < 3; ++i)
    p->pNa03[i] = p->GPa[i] * 0.01 / kElementaryCharge * p->N * p->unit_cell_volume;
  p->temperature_eV = p->kelvin / kKelvinEV;
  p->target_kinetic_energy = p->kelvin * 1.5 * p->N / kKelvinEV;
  if (p->bulk_or_film == FG_BULK) {
    if (p->gap_id != 0) {
      set_msg(errbuf, errlen, ": In the case of bulk calculation, gap_id must be 0.");
      return FG_ERR_ARG;
    }
  } else if (p->Lz % 2 != p->gap_id % 2) {
    set_msg(errbuf, errlen, ": In the case of film or epit calculation, it must be mod(Lz,2)==mod(gap_id,2).");
    return FG_ERR_ARG;
  }
  return FG_OK;
}

int fg_wave(int type, int i_step, int n_thermalize, int period, const double a[3], double out[3]) {
  if (a[0] == 0.0 && a[1] == 0.0 && a[2] == 0.0) {
    for (int k = 0; k < 3; ++k) out[k] = a[k];
    return FG_OK;
  }
  switch (type) {
    case FG_WAVE_TRIANGULAR_COS:
    case FG_WAVE_TRIANGULAR_SIN: {
      if (period <= 0) return FG_ERR_ARG;
      int i = i_step - n_thermalize;
      if (i < 0) i = 0;
      int it = (type == FG_WAVE_TRIANGULAR_COS) ? std::abs(i % period - period / 2) - period / 4
                                                : std::abs((i + 3 * period / 4) % period - period / 2) - period / 4;
      const double tmp = (double)it;
      const float quarter = (float)period / 4.0f;  // 'period/4.0' is a default-kind real
      for (int k = 0; k < 3; ++k) out[k] = a[k] * tmp / (double)quarter;
      return FG_OK;
    }
    case FG_WAVE_RAMPING_ON:
    case FG_WAVE_RAMPING_OFF:
      if (period > n_thermalize || period <= 0) return FG_ERR_ARG;  // wave_module.F:196-199,207-210
      for (int k = 0; k < 3; ++k) {
        if (type == FG_WAVE_RAMPING_ON) out[k] = (i_step < period) ? a[k] * i_step / period : a[k];
        else out[k] = (i_step < period) ? a[k] * (period - i_step) / period : 0.0;
      }
      return FG_OK;
    default:
      for (int k = 0; k < 3; ++k) out[k] = a[k];
      return FG_OK;
  }
}

double fg_uni64_seed(int seed1, int seed2) {
  fillu(seed1, seed2);
  g_rng.i = 97;
  g_rng.j = 33;
  g_rng.c = 0.0;
  g_rng.times = g_rng.times + 1.0;
  return g_rng.times;
}

double fg_uni64(void) { return uni64_next(); }

double fg_normal_dist_seed(int seed1, int seed2) {
  g_rng.sw = true;
  return fg_uni64_seed(seed1, seed2);
}

double fg_normal_dist(double mu, double sigma) {
  double n01;
  if (g_rng.sw) {
    g_rng.sw = false;
    g_rng.t = std::sqrt(-2.0 * std::log(1.0 - uni64_next()));
    g_rng.phi = k2Pi * uni64_next();
    n01 = g_rng.t * std::cos(g_rng.phi);
  } else {
    g_rng.sw = true;
    n01 = g_rng.t * std::sin(g_rng.phi);
  }
  return n01 * sigma + mu;
}

int fg_init_dipoR_host(const fg_params* p, double* dipoR, double* dipoP) {
  if (!p || !dipoR) return FG_ERR_ARG;
  const int NXP = 2 * (p->Lx / 2 + 1), NYP = p->Ly + p->padding_y;
  auto idx = [&](int a, int x, int y, int z) {
    return (size_t)a + 3 * ((size_t)x + (size_t)NXP * ((size_t)y + (size_t)NYP * z));
  };
  fg_normal_dist_seed(p->seed[0], p->seed[1]);
  for (int a = 0; a < 3; ++a)
    for (int iz = 0; iz < p->Lz; ++iz)
      for (int iy = 0; iy < p->Ly; ++iy)
        for (int ix = 0; ix < p->Lx; ++ix) {
          double v = fg_normal_dist(p->init_dipo_avg[a], p->init_dipo_dev[a]);
          if (std::cos(k2Pi * (p->k_stripe[0] * ix + p->k_stripe[1] * iy + p->k_stripe[2] * iz + 1.0e-4)) < 0.0)
            v = -v;
          dipoR[idx(a, ix, iy, iz)] = v;
        }
  if (dipoP) {
    for (int iz = 0; iz < p->Lz; ++iz)
      for (int iy = 0; iy < p->Ly; ++iy)
        for (int ix = 0; ix < p->Lx; ++ix)
          for (int a = 0; a < 3; ++a) dipoP[idx(a, ix, iy, iz)] = 0.0;
  }
  return FG_OK;
}

}  // extern "C"
