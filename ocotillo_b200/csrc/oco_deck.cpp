/*
 * oco_deck.cpp -- the reference's driver around the hot loop, with the loop on the GPU:
 * namelist input (flux_feautrier.f90:58-76, disk.f90:15-40, gas_state.f90:15-28,
 * read_athena.f90:27-62), resolution.in (a Fortran include of integer parameters, read here
 * at run time), the synthetic disk (disk.f90:42-129), the Athena reader
 * (read_athena.f90:64-291), and the writers (io.f90:31-101): diagnostics.txt with gfortran
 * Ew.d editing, the z and wavelength grids, and the per-block Fortran unformatted files.
 *
 * Host code (no kernels); the solve goes through oco_solve_block.  Input construction uses
 * the C library's exp/pow/sqrt in the reference's operation order, as the gfortran binary
 * does.
 */
#include <cerrno>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <sys/stat.h>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/oco.h"
#include "fortran_records.h"
#include "oco_ctx.h"
#include "oco_internal.h"

namespace {

thread_local std::string g_deck_err;

int derr(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_deck_err = buf;
  return code;
}

bool slurp(const std::string &path, std::string &out) {
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp) return false;
  out.clear();
  char buf[65536];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, fp)) > 0) out.append(buf, n);
  fclose(fp);
  return true;
}

std::string lower(std::string s) {
  for (auto &ch : s) ch = (char)tolower((unsigned char)ch);
  return s;
}

/* ---- namelists: &group key = value, ... / ----------------------------------------------- */
using Group = std::map<std::string, std::string>; /* lower-case key -> raw value text */

/* Reads namelist group `name` from the text of a namelist file; false if absent. */
bool namelist(const std::string &text, const std::string &name, Group &g) {
  g.clear();
  const std::string want = lower(name);
  size_t i = 0, n = text.size();
  bool found = false;
  while (i < n && !found) {
    if (text[i] == '!') {
      while (i < n && text[i] != '\n') i++;
      continue;
    }
    if (text[i] == '&') {
      size_t j = i + 1;
      while (j < n && (isalnum((unsigned char)text[j]) || text[j] == '_')) j++;
      if (lower(text.substr(i + 1, j - i - 1)) == want) {
        i = j;
        found = true;
        break;
      }
      i = j;
      continue;
    }
    i++;
  }
  if (!found) return false;
  for (;;) {
    while (i < n && (isspace((unsigned char)text[i]) || text[i] == ',')) i++;
    if (i < n && text[i] == '!') {
      while (i < n && text[i] != '\n') i++;
      continue;
    }
    if (i >= n || text[i] == '/' || text[i] == '&') break;
    size_t k0 = i;
    while (i < n && (isalnum((unsigned char)text[i]) || text[i] == '_')) i++;
    if (i == k0) break;
    std::string key = lower(text.substr(k0, i - k0));
    while (i < n && isspace((unsigned char)text[i])) i++;
    if (i >= n || text[i] != '=') break;
    i++;
    while (i < n && isspace((unsigned char)text[i])) i++;
    std::string val;
    if (i < n && (text[i] == '"' || text[i] == '\'')) {
      const char q = text[i++];
      while (i < n && text[i] != q) val += text[i++];
      if (i < n) i++;
    } else {
      while (i < n && !isspace((unsigned char)text[i]) && text[i] != ',' && text[i] != '/' && text[i] != '!')
        val += text[i++];
    }
    g[key] = val;
  }
  return true;
}

/* A Fortran real literal (d/D exponents allowed), correctly rounded. */
double fortran_real(const std::string &s) {
  std::string t = s;
  for (auto &ch : t)
    if (ch == 'd' || ch == 'D') ch = 'e';
  return strtod(t.c_str(), nullptr);
}

bool fortran_logical(const std::string &s) {
  size_t i = 0;
  while (i < s.size() && s[i] == '.') i++;
  return i < s.size() && (s[i] == 'T' || s[i] == 't');
}

void get_real(const Group &g, const char *key, double &dst) {
  auto it = g.find(lower(key));
  if (it != g.end()) dst = fortran_real(it->second);
}
void get_logical(const Group &g, const char *key, int &dst) {
  auto it = g.find(lower(key));
  if (it != g.end()) dst = fortran_logical(it->second) ? 1 : 0;
}
void get_string(const Group &g, const char *key, std::string &dst) {
  auto it = g.find(lower(key));
  if (it != g.end()) dst = it->second;
}

/* ---- resolution.in: "integer, parameter :: a=expr, b=expr" --------------------------------- */
/* Integer expression of literals and earlier names with + - * / (Fortran precedence and
 * truncating division), left to right. */
bool int_expr(const std::string &e, const std::map<std::string, long> &vars, long &out) {
  long total = 0, term = 0;
  char addop = '+', mulop = 0;
  size_t i = 0;
  for (;;) {
    while (i < e.size() && isspace((unsigned char)e[i])) i++;
    long v = 0;
    if (i < e.size() && isdigit((unsigned char)e[i])) {
      size_t j = i;
      while (j < e.size() && isdigit((unsigned char)e[j])) j++;
      v = strtol(e.substr(i, j - i).c_str(), nullptr, 10);
      i = j;
    } else if (i < e.size() && isalpha((unsigned char)e[i])) {
      size_t j = i;
      while (j < e.size() && (isalnum((unsigned char)e[j]) || e[j] == '_')) j++;
      auto it = vars.find(lower(e.substr(i, j - i)));
      if (it == vars.end()) return false;
      v = it->second;
      i = j;
    } else {
      return false;
    }
    if (mulop == 0)
      term = v;
    else if (mulop == '*')
      term *= v;
    else if (v != 0)
      term /= v;
    else
      return false;
    while (i < e.size() && isspace((unsigned char)e[i])) i++;
    if (i < e.size() && (e[i] == '*' || e[i] == '/')) {
      mulop = e[i++];
      continue;
    }
    total = addop == '+' ? total + term : total - term;
    mulop = 0;
    if (i < e.size() && (e[i] == '+' || e[i] == '-')) {
      addop = e[i++];
      continue;
    }
    break;
  }
  out = total;
  return true;
}

bool resolution(const std::string &path, std::map<std::string, long> &vars) {
  std::string text;
  if (!slurp(path, text)) return false;
  size_t pos = 0;
  while (pos <= text.size()) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    std::string line = text.substr(pos, eol - pos);
    pos = eol + 1;
    const size_t bang = line.find('!');
    if (bang != std::string::npos) line.resize(bang);
    const size_t dc = line.find("::");
    if (dc == std::string::npos) continue;
    std::string rest = line.substr(dc + 2);
    size_t s = 0;
    while (s < rest.size()) {
      size_t c = rest.find(',', s);
      if (c == std::string::npos) c = rest.size();
      const std::string as = rest.substr(s, c - s);
      s = c + 1;
      const size_t eq = as.find('=');
      if (eq == std::string::npos) continue;
      std::string name;
      for (char ch : as.substr(0, eq))
        if (!isspace((unsigned char)ch)) name += (char)tolower((unsigned char)ch);
      long v;
      if (int_expr(as.substr(eq + 1), vars, v)) vars[name] = v;
    }
    if (eol == text.size()) break;
  }
  return true;
}

long rget(const std::map<std::string, long> &v, const char *name, long dflt) {
  auto it = v.find(name);
  return it == v.end() ? dflt : it->second;
}

/* ---- writers ------------------------------------------------------------------------------- */
/* gfortran list-directed output of one INTEGER and one REAL(8): the integer right-justified in
 * 12 columns, the real with 17 significant digits in F form when 0.1 <= |x| < 1e16 (5 trailing
 * blanks in place of an exponent), else in E form with a 3-digit exponent. */
std::string list_int_real(int i, double v) {
  char ib[32], rb[64], out[128];
  snprintf(ib, sizeof ib, "%12d", i);
  const double a = std::fabs(v);
  if (v == 0.0) {
    snprintf(rb, sizeof rb, "%20s     ", "0.0000000000000000");
  } else if (a >= 0.1 && a < 1e16) {
    const int e10 = (int)std::floor(std::log10(a));
    const int dec = std::max(1, 16 - e10);
    char f[64];
    snprintf(f, sizeof f, "%.*f", dec, v);
    snprintf(rb, sizeof rb, "%20s     ", f);
  } else {
    char f[64];
    snprintf(f, sizeof f, "%.16E", v); /* d.ddddE+XX -> 3-digit exponent */
    char *e = strchr(f, 'E');
    const int ex = atoi(e + 1);
    *e = 0;
    snprintf(rb, sizeof rb, "%20s%c%03d", f, ex < 0 ? '-' : '+', std::abs(ex));
  }
  snprintf(out, sizeof out, "%s %s", ib, rb);
  return out;
}

/* A file holding one Fortran unformatted sequential record of n doubles (gfortran markers and
 * subrecords, fortran_records.h). */
bool write_record_file(const std::string &path, const double *a, size_t n) {
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) return false;
  const bool ok = oco::write_fortran_record(fp, a, n * sizeof(double));
  return (fclose(fp) == 0) && ok;
}

bool make_dirs(const std::string &path) {
  std::string cur;
  for (size_t i = 0; i <= path.size(); i++) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty() && mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) return false;
    }
    if (i < path.size()) cur += path[i];
  }
  return true;
}

/* ---- the deck -------------------------------------------------------------------------------- */
constexpr int kNg = 3;

struct Deck {
  std::string dir, snapshot;
  int nx = 0, ny = 0, nz = 0, nw = 0, nprocx = 1, nprocy = 1, nprocz = 1, nxloc = 0, nyloc = 0;
  /* &input (flux_feautrier.f90:50, 57) */
  double z0 = 0, z1 = 0, w0 = 3000, w1 = 5000, sigma_grey = 0;
  int lgrey = 0, lread_athena = 1;
  /* &temperature_input, &density_input (disk.f90:12-15) */
  double isoTemp = 0, sigma = 0, midTemp = 0, floorTemp = 0, switchTemp = 0;
  double rho0 = 0, rho_floor = 0, H = 0;
  /* &gas_state_input */
  double fully_ionized_T = 0;
  /* &athena_input (read_athena.f90:13-30) */
  std::string RunName, datadir = "./input_athena/distributed";
  double Mbh_SolarMasses = 0, r0ref_rg = 0, aspect_ratio = 0, mmw = 0, a_rho0 = 0, a_rho_floor = NAN;
  int lavoid = 1;
  double unit_density = 0, unit_length = 0, unit_temperature = 0;
  std::vector<double> wa, Tgauss;
  bool have_tgauss = false;
};

int load_deck(const char *deck_dir, const char *snapshot, Deck &d) {
  d.dir = deck_dir ? deck_dir : ".";
  d.snapshot = (snapshot && snapshot[0]) ? snapshot : "0000";
  std::map<std::string, long> rv;
  if (!resolution(d.dir + "/resolution.in", rv)) return derr(OCO_EIO, "cannot read %s/resolution.in", d.dir.c_str());
  for (const auto &kv : rv)
    if (kv.second < INT32_MIN || kv.second > INT32_MAX)
      return derr(OCO_EDIM, "resolution.in: %s = %ld is out of range", kv.first.c_str(), kv.second);
  d.nw = (int)rget(rv, "nw", 0);
  d.nx = (int)rget(rv, "nx", 0);
  d.ny = (int)rget(rv, "ny", 0);
  d.nz = (int)rget(rv, "nz", 0);
  d.nprocx = (int)rget(rv, "nprocx", 1);
  d.nprocy = (int)rget(rv, "nprocy", 1);
  d.nprocz = (int)rget(rv, "nprocz", 1);
  if (d.nprocx < 1 || d.nprocy < 1 || d.nprocz < 1)
    return derr(OCO_EDIM, "resolution.in: processor counts must be positive");
  d.nxloc = (int)rget(rv, "nxloc", d.nx / d.nprocx);
  d.nyloc = (int)rget(rv, "nyloc", d.ny / d.nprocy);
  if (d.nw < 1 || d.nz < 2 || d.nxloc < 1 || d.nyloc < 1)
    return derr(OCO_EDIM, "resolution.in: need nw >= 1, nz >= 2, nxloc, nyloc >= 1");
  if ((double)d.nxloc * d.nyloc * d.nw * (d.nz + 6.0) > 72057594037927936.0) /* the library's 2^56 limit */
    return derr(OCO_EDIM, "resolution.in: nxloc*nyloc*nw*(nz+6) exceeds 2^56 elements");
  std::string text;
  if (!slurp(d.dir + "/input.in", text)) return derr(OCO_EIO, "cannot read %s/input.in", d.dir.c_str());
  Group g;
  namelist(text, "input", g);
  get_real(g, "z0", d.z0);
  get_real(g, "z1", d.z1);
  get_real(g, "w0", d.w0);
  get_real(g, "w1", d.w1);
  get_real(g, "sigma_grey", d.sigma_grey);
  get_logical(g, "lgrey", d.lgrey);
  get_logical(g, "lread_athena", d.lread_athena);
  namelist(text, "temperature_input", g);
  get_real(g, "isoTemp", d.isoTemp);
  get_real(g, "sigma", d.sigma);
  get_real(g, "midTemp", d.midTemp);
  get_real(g, "floorTemp", d.floorTemp);
  d.switchTemp = (1.0 + 0x1p-52) * d.isoTemp; /* disk.f90:28, epsilon(1.0) of a double */
  namelist(text, "density_input", g);
  get_real(g, "rho0", d.rho0);
  get_real(g, "rho_floor", d.rho_floor);
  get_real(g, "H", d.H);
  namelist(text, "gas_state_input", g);
  get_real(g, "fully_ionized_T", d.fully_ionized_T);
  if (d.lgrey && d.nw != 1)
    return derr(OCO_EGREY, "For Grey RT use only one wavelength. Switch nw=1 in resolution.in");
  if (d.lread_athena) {
    namelist(text, "athena_input", g);
    get_string(g, "RunName", d.RunName);
    get_string(g, "datadir", d.datadir);
    get_real(g, "Mbh_SolarMasses", d.Mbh_SolarMasses);
    get_real(g, "r0ref_rg", d.r0ref_rg);
    get_real(g, "aspect_ratio", d.aspect_ratio);
    get_real(g, "mean_molecular_weight", d.mmw);
    get_real(g, "rho0", d.a_rho0);
    get_real(g, "rho_floor", d.a_rho_floor);
    get_logical(g, "lavoid_momentum_underflow", d.lavoid);
    /* read_athena_input, read_athena.f90:41-54 */
    const double G = 6.6742e-8, c_light = 2.99792458e10, SolarMass = 1.988409870698051e+33;
    const double amu = 1.66053906660e-24, k1_cgs = 1.0 / 1.380649e-16;
    const double Mbh = d.Mbh_SolarMasses * SolarMass;
    const double rg = (2.0 * (G / (c_light * c_light))) * Mbh;
    const double rr = d.r0ref_rg * rg;
    const double g0 = G * Mbh;
    const double Omega = std::sqrt(g0) * std::pow(rr, -1.5);
    d.unit_density = d.a_rho0;
    const double unit_time = 1.0 / Omega;
    d.unit_length = d.aspect_ratio * rr;
    const double unit_velocity = d.unit_length / unit_time;
    d.unit_temperature = ((d.mmw * amu) * k1_cgs) * (unit_velocity * unit_velocity);
  }
  d.wa.assign((size_t)d.nw, 0.0);
  oco_calc_wavelength(d.w1, d.w0, d.nw, d.wa.data());
  d.Tgauss.assign((size_t)d.nz, 0.0);
  return OCO_OK;
}

/* calc_temperature, disk.f90:64-109 (the Gaussian profile is fixed by the first call) */
void calc_temperature(Deck &d, double *T, const double *z, bool from_athena) {
  if (!from_athena)
    for (int i = 0; i < d.nz; i++) T[i] = d.midTemp;
  if (!d.have_tgauss) {
    for (int i = 0; i < d.nz; i++) {
      const double zz = z[kNg + i];
      d.Tgauss[(size_t)i] = d.midTemp * std::exp(-((0.5 * (zz * zz)) / (d.sigma * d.sigma)));
    }
    d.have_tgauss = true;
  }
  for (int i = 0; i < d.nz; i++)
    if (T[i] < d.switchTemp) T[i] = d.Tgauss[(size_t)i] > d.floorTemp ? d.Tgauss[(size_t)i] : d.floorTemp;
}

bool read_i32(FILE *fp, int32_t *v, size_t n) { return fread(v, 4, n, fp) == n; }
bool read_f64(FILE *fp, double *v, size_t n) { return fread(v, 8, n, fp) == n; }

/* read_from_athena + postprocess_athena_values, read_athena.f90:64-277: the block's rho and T
 * in (nz, nyloc, nxloc) order, its z grid with ghosts (mz) and dz. */
int read_athena_block(Deck &d, int iprocx, int iprocy, double *rho, double *T, double *z, double &dz) {
  const int nz = d.nz, nxl = d.nxloc, nyl = d.nyloc;
  std::vector<double> zn((size_t)nz, 0.0);
  double z0a = 0.0, dza = 0.0, gamma1 = 0.0;
  for (int iprocz = 0; iprocz < d.nprocz; iprocz++) {
    const int iproc = iprocz * d.nprocx * d.nprocy + iprocy * d.nprocx + iprocx;
    std::string head = d.dir + "/" + d.datadir + "/id" + std::to_string(iproc) + "/" + d.RunName;
    const std::string fn = iproc == 0 ? head + "." + d.snapshot + ".bin"
                                      : head + "-id" + std::to_string(iproc) + "." + d.snapshot + ".bin";
    FILE *fp = fopen(fn.c_str(), "rb");
    if (!fp) return derr(OCO_EIO, "File %s does not exist (iproc=%d)", fn.c_str(), iproc);
    int32_t coordsys, dims[3], dummies[4];
    double reals[3];
    bool ok = read_i32(fp, &coordsys, 1) && read_i32(fp, dims, 3) && read_i32(fp, dummies, 4) &&
              read_f64(fp, &gamma1, 1) && read_f64(fp, reals, 3);
    if (!ok) {
      fclose(fp);
      return derr(OCO_EIO, "%s: truncated header", fn.c_str());
    }
    if (dims[0] != nxl || dims[1] != nyl) {
      fclose(fp);
      return derr(OCO_EDIM,
                  "The Athena x/y dimensionality (%d, %d) does not match the chosen for the RT post-processing "
                  "(%d, %d). Fix.",
                  dims[0], dims[1], nxl, nyl);
    }
    const int nzl = dims[2];
    std::vector<double> coords((size_t)nxl + nyl + nzl);
    if (nzl < 1 || !read_f64(fp, coords.data(), coords.size())) {
      fclose(fp);
      return derr(OCO_EIO, "%s: truncated coordinates", fn.c_str());
    }
    const double *zloc = coords.data() + nxl + nyl;
    if (iprocz == 0) {
      z0a = zloc[0];
      dza = nzl > 1 ? zloc[1] - zloc[0] : 0.0;
    }
    const long iz0 = dza != 0.0 ? std::lround((zloc[0] - z0a) / dza) : 0; /* nint(...) + 1, 0-based */
    if (iz0 < 0 || iz0 + nzl > nz) {
      fclose(fp);
      return derr(OCO_EDIM, "%s: z block %ld..%ld outside nz=%d", fn.c_str(), iz0, iz0 + nzl - 1, nz);
    }
    for (int k = 0; k < nzl; k++) zn[(size_t)(iz0 + k)] = zloc[k];
    const size_t nc = (size_t)nxl * nyl * nzl;
    std::vector<double> tmp(nc);
    /* file arrays are (nxloc, nyloc, nzloc), x fastest; the block is (nz, nyloc, nxloc) */
    auto cell = [&](int ix, int iy, int iz) { return ((size_t)iz * nyl + iy) * nxl + ix; };
    auto dst = [&](int ix, int iy, int iz) { return ((size_t)ix * nyl + iy) * nz + (size_t)(iz0 + iz); };
    ok = read_f64(fp, tmp.data(), nc);
    for (int ix = 0; ix < nxl && ok; ix++)
      for (int iy = 0; iy < nyl; iy++)
        for (int iz = 0; iz < nzl; iz++) {
          rho[dst(ix, iy, iz)] = tmp[cell(ix, iy, iz)];
          T[dst(ix, iy, iz)] = 0.0;
        }
    for (int comp = 0; comp < 3 && ok; comp++) { /* momenta, :176-195; the underflow guard :213-228 */
      ok = read_f64(fp, tmp.data(), nc);
      for (int ix = 0; ix < nxl && ok; ix++)
        for (int iy = 0; iy < nyl; iy++)
          for (int iz = 0; iz < nzl; iz++) {
            const double pp = tmp[cell(ix, iy, iz)];
            const size_t q = dst(ix, iy, iz);
            if (!d.lavoid || std::fabs(pp) >= 0x1p-52) T[q] = T[q] + (0.5 * (pp * pp)) / rho[q];
          }
    }
    if (ok) ok = read_f64(fp, tmp.data(), nc); /* total energy, :201-202 */
    for (int ix = 0; ix < nxl && ok; ix++)
      for (int iy = 0; iy < nyl; iy++)
        for (int iz = 0; iz < nzl; iz++) {
          const size_t q = dst(ix, iy, iz);
          T[q] = (tmp[cell(ix, iy, iz)] - T[q]) / rho[q];
        }
    fclose(fp);
    if (!ok) return derr(OCO_EIO, "%s: truncated data", fn.c_str());
  }
  if (d.a_rho_floor != d.a_rho_floor)
    return derr(OCO_ENAN, "Must set `rho_floor` (cgs) value in namelist: `input.in/athena_input`.");
  const size_t n = (size_t)nxl * nyl * nz;
  for (size_t i = 0; i < n; i++) {
    rho[i] = rho[i] * d.unit_density;
    if (rho[i] < d.a_rho_floor) rho[i] = d.a_rho_floor;
    T[i] = (T[i] * gamma1) * d.unit_temperature;
  }
  for (int i = 0; i < nz; i++) zn[(size_t)i] = zn[(size_t)i] * d.unit_length;
  dz = (zn[(size_t)nz - 1] - zn[0]) / (double)(nz - 1);
  for (int i = 0; i < nz; i++) z[kNg + i] = zn[(size_t)i];
  for (int i = 1; i <= kNg; i++) {
    z[kNg - i] = z[kNg] - (double)i * dz;
    z[nz + kNg - 1 + i] = z[nz + kNg - 1] + (double)i * dz;
  }
  for (size_t c = 0; c < (size_t)nxl * nyl; c++) calc_temperature(d, T + c * nz, z, true);
  return OCO_OK;
}

/* The synthetic disk (calc_grid, calc_density, calc_temperature; disk.f90:42-129): every
 * column of the block gets the same pillar. */
void disk_block(Deck &d, double *rho, double *T, double *z, double &dz) {
  const int nz = d.nz;
  dz = (d.z1 - d.z0) / (double)(nz - 1);
  for (int i = 1; i <= nz; i++) z[kNg + i - 1] = d.z0 + (double)(i - 1) * dz;
  for (int i = 1; i <= kNg; i++) {
    z[kNg - i] = z[kNg] - (double)i * dz;
    z[nz + kNg - 1 + i] = z[nz + kNg - 1] + (double)i * dz;
  }
  for (int i = 0; i < nz; i++) {
    const double zz = z[kNg + i];
    rho[i] = d.rho0 * std::exp(-((0.5 * (zz * zz)) / (d.H * d.H)));
    if (rho[i] < d.rho_floor) rho[i] = d.rho_floor;
  }
  calc_temperature(d, T, z, false);
  for (size_t c = 1; c < (size_t)d.nxloc * d.nyloc; c++) {
    memcpy(rho + c * nz, rho, sizeof(double) * nz);
    memcpy(T + c * nz, T, sizeof(double) * nz);
  }
}

int block_inputs(Deck &d, int iprocx, int iprocy, double *rho, double *T, double *z, double &dz) {
  if (d.lread_athena) return read_athena_block(d, iprocx, iprocy, rho, T, z, dz);
  disk_block(d, rho, T, z, dz);
  return OCO_OK;
}

void fill_info(const Deck &d, double dz, oco_deck_info *info) {
  info->nx = d.nx;
  info->ny = d.ny;
  info->nz = d.nz;
  info->nw = d.nw;
  info->nprocx = d.nprocx;
  info->nprocy = d.nprocy;
  info->nprocz = d.nprocz;
  info->nxloc = d.nxloc;
  info->nyloc = d.nyloc;
  info->lgrey = d.lgrey;
  info->lread_athena = d.lread_athena;
  info->reserved = 0;
  info->dz = dz;
  info->sigma_grey = d.sigma_grey;
  info->fully_ionized_T = d.fully_ionized_T;
}

}  // namespace

extern "C" void oco_format_e(double v, int32_t w, int32_t d, char *out) {
  std::string body;
  if (v != v) {
    body = "NaN";
  } else if (std::isinf(v)) {
    body = v > 0 ? "Infinity" : "-Infinity";
  } else {
    std::string digits;
    int e10 = 0;
    if (v == 0.0 || d < 1) {
      digits.assign((size_t)std::max(d, 0), '0');
    } else {
      char buf[64];
      snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v)); /* correctly rounded d digits */
      for (const char *q = buf; *q && *q != 'e'; q++)
        if (isdigit((unsigned char)*q)) digits += *q;
      e10 = atoi(strchr(buf, 'e') + 1) + 1;
    }
    char ex[16];
    if (std::abs(e10) <= 99)
      snprintf(ex, sizeof ex, "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
    else /* gfortran drops the E for 3-digit exponents: 0.12345-100 */
      snprintf(ex, sizeof ex, "%c%03d", e10 < 0 ? '-' : '+', std::abs(e10));
    body = std::string(std::signbit(v) ? "-" : "") + "0." + digits + ex;
  }
  if ((int)body.size() > w) {
    memset(out, '*', (size_t)w);
    out[w] = 0;
    return;
  }
  const size_t pad = (size_t)w - body.size();
  memset(out, ' ', pad);
  memcpy(out + pad, body.c_str(), body.size() + 1);
}

static int deck_block_inputs(const char *deck_dir, const char *snapshot, int32_t iprocx, int32_t iprocy,
                             oco_deck_info *info, double *rho, double *T, double *wa, double *z) {
  if (!info) return derr(OCO_EINVAL, "oco_deck_block_inputs: info is NULL");
  Deck d;
  int rc = load_deck(deck_dir, snapshot, d);
  if (rc) return rc;
  if (iprocx < 0 || iprocx >= d.nprocx || iprocy < 0 || iprocy >= d.nprocy)
    return derr(OCO_EINVAL, "block (%d, %d) outside %d x %d processors", iprocx, iprocy, d.nprocx, d.nprocy);
  double dz = 0.0;
  if (rho && T) {
    std::vector<double> zz((size_t)d.nz + 2 * kNg, 0.0);
    /* the Gaussian temperature profile is fixed by the root block's grid (first call) */
    if (d.lread_athena && (iprocx || iprocy)) {
      std::vector<double> r0((size_t)d.nxloc * d.nyloc * d.nz), t0(r0.size());
      if ((rc = block_inputs(d, 0, 0, r0.data(), t0.data(), zz.data(), dz))) return rc;
    }
    if ((rc = block_inputs(d, iprocx, iprocy, rho, T, zz.data(), dz))) return rc;
    if (z) memcpy(z, zz.data(), zz.size() * sizeof(double));
  } else if (!d.lread_athena) {
    dz = (d.z1 - d.z0) / (double)(d.nz - 1);
  }
  if (wa) memcpy(wa, d.wa.data(), d.wa.size() * sizeof(double));
  fill_info(d, dz, info);
  return OCO_OK;
}

/* The Athena reader with the data into HBM: per z-block file the host reads the header and
 * coordinates (read_athena.f90:101-148, the same checks as read_athena_block) and the five raw
 * fields into pinned memory (two buffers, so that reading file k+1 overlaps the copy of file k);
 * the device reassembles the block (k_athena_zblock) and applies postprocess_athena_values and
 * calc_temperature (k_athena_post) with the host reader's operations and the host's Gaussian
 * profile, so rho and T equal read_athena_block's bit for bit. */
int read_athena_block_device(oco_ctx *c, Deck &d, int iprocx, int iprocy, double *rho, double *T, double *z,
                             double &dz, cudaStream_t s) {
  const int nz = d.nz, nxl = d.nxloc, nyl = d.nyloc;
  std::vector<double> zn((size_t)nz, 0.0);
  double z0a = 0.0, dza = 0.0, gamma1 = 0.0;
  struct Staging {
    void *host[2] = {nullptr, nullptr};
    size_t hn[2] = {0, 0};
    DevBuf dev[2], tg;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t s = nullptr;
    ~Staging() {
      if (s) cudaStreamSynchronize(s);
      for (int b = 0; b < 2; b++) {
        if (host[b]) cudaFreeHost(host[b]);
        if (ev[b]) cudaEventDestroy(ev[b]);
        dev[b].release();
      }
      tg.release();
    }
  } st;
  st.s = s;
  for (int b = 0; b < 2; b++)
    if (cudaEventCreateWithFlags(&st.ev[b], cudaEventDisableTiming) != cudaSuccess)
      return derr(OCO_ECUDA, "athena device reader: cudaEventCreate failed");
  for (int iprocz = 0; iprocz < d.nprocz; iprocz++) {
    const int iproc = iprocz * d.nprocx * d.nprocy + iprocy * d.nprocx + iprocx;
    std::string head = d.dir + "/" + d.datadir + "/id" + std::to_string(iproc) + "/" + d.RunName;
    const std::string fn = iproc == 0 ? head + "." + d.snapshot + ".bin"
                                      : head + "-id" + std::to_string(iproc) + "." + d.snapshot + ".bin";
    FILE *fp = fopen(fn.c_str(), "rb");
    if (!fp) return derr(OCO_EIO, "File %s does not exist (iproc=%d)", fn.c_str(), iproc);
    std::unique_ptr<FILE, int (*)(FILE *)> guard(fp, fclose);
    int32_t coordsys, dims[3], dummies[4];
    double reals[3];
    if (!(read_i32(fp, &coordsys, 1) && read_i32(fp, dims, 3) && read_i32(fp, dummies, 4) &&
          read_f64(fp, &gamma1, 1) && read_f64(fp, reals, 3)))
      return derr(OCO_EIO, "%s: truncated header", fn.c_str());
    if (dims[0] != nxl || dims[1] != nyl)
      return derr(OCO_EDIM,
                  "The Athena x/y dimensionality (%d, %d) does not match the chosen for the RT post-processing "
                  "(%d, %d). Fix.",
                  dims[0], dims[1], nxl, nyl);
    const int nzl = dims[2];
    std::vector<double> coords((size_t)nxl + nyl + (nzl > 0 ? nzl : 0));
    if (nzl < 1 || !read_f64(fp, coords.data(), coords.size()))
      return derr(OCO_EIO, "%s: truncated coordinates", fn.c_str());
    const double *zloc = coords.data() + nxl + nyl;
    if (iprocz == 0) {
      z0a = zloc[0];
      dza = nzl > 1 ? zloc[1] - zloc[0] : 0.0;
    }
    const long iz0 = dza != 0.0 ? std::lround((zloc[0] - z0a) / dza) : 0;
    if (iz0 < 0 || iz0 + nzl > nz)
      return derr(OCO_EDIM, "%s: z block %ld..%ld outside nz=%d", fn.c_str(), iz0, iz0 + nzl - 1, nz);
    for (int k = 0; k < nzl; k++) zn[(size_t)(iz0 + k)] = zloc[k];
    const size_t nc = (size_t)nxl * nyl * nzl, bytes = 5 * nc * sizeof(double);
    const int b = iprocz & 1;
    if (cudaEventSynchronize(st.ev[b]) != cudaSuccess) return derr(OCO_ECUDA, "athena device reader: event wait failed");
    if (st.hn[b] < bytes) {
      if (st.host[b]) cudaFreeHost(st.host[b]);
      st.host[b] = nullptr;
      st.hn[b] = 0;
      if (cudaMallocHost(&st.host[b], bytes) != cudaSuccess) return derr(OCO_ENOMEM, "athena device reader: pinned staging");
      st.hn[b] = bytes;
    }
    if (!read_f64(fp, (double *)st.host[b], 5 * nc)) return derr(OCO_EIO, "%s: truncated data", fn.c_str());
    if (st.dev[b].n < bytes) {
      cudaStreamSynchronize(s); /* the previous user of this buffer is done before it is replaced */
      if (st.dev[b].ensure(bytes) != cudaSuccess) return derr(OCO_ENOMEM, "athena device reader: device staging");
    }
    if (cudaMemcpyAsync(st.dev[b].p, st.host[b], bytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaEventRecord(st.ev[b], s) != cudaSuccess)
      return derr(OCO_ECUDA, "athena device reader: copy failed");
    oco::AthenaZBlock zb{st.dev[b].as<double>(), nxl, nyl, nzl, nz, (int)iz0, d.lavoid, rho, T};
    if (oco::launch_athena_zblock(zb, s) != cudaSuccess) return derr(OCO_ECUDA, "athena device reader: launch failed");
    c->launches += 1;
  }
  if (d.a_rho_floor != d.a_rho_floor)
    return derr(OCO_ENAN, "Must set `rho_floor` (cgs) value in namelist: `input.in/athena_input`.");
  for (int i = 0; i < nz; i++) zn[(size_t)i] = zn[(size_t)i] * d.unit_length;
  dz = (zn[(size_t)nz - 1] - zn[0]) / (double)(nz - 1);
  for (int i = 0; i < nz; i++) z[kNg + i] = zn[(size_t)i];
  for (int i = 1; i <= kNg; i++) {
    z[kNg - i] = z[kNg] - (double)i * dz;
    z[nz + kNg - 1 + i] = z[nz + kNg - 1] + (double)i * dz;
  }
  if (!d.have_tgauss) { /* calc_temperature's first call fixes the profile, as on the host */
    for (int i = 0; i < nz; i++) {
      const double zz = z[kNg + i];
      d.Tgauss[(size_t)i] = d.midTemp * std::exp(-((0.5 * (zz * zz)) / (d.sigma * d.sigma)));
    }
    d.have_tgauss = true;
  }
  if (st.tg.ensure((size_t)nz * sizeof(double)) != cudaSuccess ||
      cudaMemcpyAsync(st.tg.p, d.Tgauss.data(), (size_t)nz * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return derr(OCO_ECUDA, "athena device reader: temperature profile upload failed");
  if (oco::launch_athena_post(rho, T, (int64_t)nxl * nyl * nz, nz, d.unit_density, d.a_rho_floor, gamma1, d.unit_temperature,
                         st.tg.as<double>(), d.switchTemp, d.floorTemp, s) != cudaSuccess)
    return derr(OCO_ECUDA, "athena device reader: launch failed");
  c->launches += 1;
  if (cudaStreamSynchronize(s) != cudaSuccess) return derr(OCO_ECUDA, "athena device reader: device error");
  return OCO_OK;
}

static int deck_block_inputs_device(oco_ctx *c, const char *deck_dir, const char *snapshot, int32_t iprocx,
                                    int32_t iprocy, oco_deck_info *info, double *rho, double *T, double *wa, double *z,
                                    cudaStream_t s) {
  if (!c) return derr(OCO_EINVAL, "oco_deck_block_inputs_device: NULL context");
  if (!info || !rho || !T) return derr(OCO_EINVAL, "oco_deck_block_inputs_device: info, rho and T are required");
  Deck d;
  int rc = load_deck(deck_dir, snapshot, d);
  if (rc) return rc;
  if (iprocx < 0 || iprocx >= d.nprocx || iprocy < 0 || iprocy >= d.nprocy)
    return derr(OCO_EINVAL, "block (%d, %d) outside %d x %d processors", iprocx, iprocy, d.nprocx, d.nprocy);
  if (cudaSetDevice(c->device) != cudaSuccess) return derr(OCO_ECUDA, "oco_deck_block_inputs_device: cudaSetDevice");
  double dz = 0.0;
  std::vector<double> zz((size_t)d.nz + 2 * kNg, 0.0);
  const size_t n = (size_t)d.nxloc * d.nyloc * d.nz;
  if (d.lread_athena) {
    if (iprocx || iprocy) { /* the Gaussian temperature profile is fixed by the root block's grid (first call) */
      std::vector<double> r0(n), t0(n);
      if ((rc = block_inputs(d, 0, 0, r0.data(), t0.data(), zz.data(), dz))) return rc;
    }
    if ((rc = read_athena_block_device(c, d, iprocx, iprocy, rho, T, zz.data(), dz, s))) return rc;
  } else { /* the synthetic disk is built on the host (the C library's exp, as the reference) */
    std::vector<double> r(n), t(n);
    disk_block(d, r.data(), t.data(), zz.data(), dz);
    if (cudaMemcpyAsync(rho, r.data(), n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(T, t.data(), n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return derr(OCO_ECUDA, "oco_deck_block_inputs_device: copy failed");
  }
  if (z) memcpy(z, zz.data(), zz.size() * sizeof(double));
  if (wa) memcpy(wa, d.wa.data(), d.wa.size() * sizeof(double));
  fill_info(d, dz, info);
  return OCO_OK;
}

static int run_deck(const char *deck_dir, const char *snapshot, const char *out_dir, int32_t form, int32_t device,
                    int32_t write_binary) {
  Deck d;
  int rc = load_deck(deck_dir, snapshot, d);
  if (rc) return rc;
  if (form != OCO_FORM_PLAIN && form != OCO_FORM_STABLE && form != OCO_FORM_MIXED)
    return derr(OCO_EINVAL, "unknown form %d", form);
  if (form == OCO_FORM_MIXED && d.lgrey) return derr(OCO_EINVAL, "the mixed form has no grey variant");
  const std::string out = (out_dir && out_dir[0]) ? std::string(out_dir) : d.dir + "/output";
  if (!make_dirs(out)) return derr(OCO_EIO, "cannot create %s", out.c_str());
  oco_ctx *ctx = nullptr;
  if ((rc = oco_create(&ctx, device))) return derr(rc, "%s", oco_last_error(nullptr));
  const std::unique_ptr<oco_ctx, void (*)(oco_ctx *)> ctx_guard(ctx, oco_destroy); /* every return path */
  if (!d.lgrey && (rc = oco_set_wavelengths(ctx, d.wa.data(), d.nw))) return derr(rc, "%s", oco_last_error(ctx));
  const int nz = d.nz, nw = d.nw, mz = nz + 2 * kNg;
  const size_t ncol = (size_t)d.nxloc * d.nyloc;
  std::vector<double> rho(ncol * nz), T(ncol * nz), z((size_t)mz, 0.0);
  std::vector<double> U(ncol * mz * nw), K(ncol * nz * nw), V(write_binary ? ncol * nz * nw : 0);
  int zero_pivot_rc = OCO_OK;
  for (int ipx = 0; ipx < d.nprocx && !rc; ipx++) {
    for (int ipy = 0; ipy < d.nprocy && !rc; ipy++) {
      const bool root = ipx == 0 && ipy == 0;
      double dz = 0.0;
      if ((rc = block_inputs(d, ipx, ipy, rho.data(), T.data(), z.data(), dz))) break;
      oco_params p{};
      p.nx = d.nxloc;
      p.ny = d.nyloc;
      p.nz = nz;
      p.nw = nw;
      p.dz = dz;
      p.sigma_grey = d.sigma_grey;
      p.fully_ionized_T = d.fully_ionized_T;
      p.lgrey = d.lgrey;
      p.form = form;
      p.layout = OCO_LAYOUT_REFERENCE;
      const int src = oco_solve_block(ctx, &p, rho.data(), T.data(), U.data(), K.data(),
                                      write_binary ? V.data() : nullptr, nullptr, nullptr);
      if (src == OCO_EZEROPIVOT) {
        /* the reference stops here (auxiliary.f90:27-39); all other items are written */
        zero_pivot_rc = derr(src, "%s", oco_last_error(ctx));
      } else if (src) {
        rc = derr(src, "%s", oco_last_error(ctx));
        break;
      }
      if (root) {
        /* output_grid, io.f90:48-75 */
        FILE *fz = fopen((out + "/zgrid.txt").c_str(), "w");
        FILE *fw = fopen((out + "/wavegrid.txt").c_str(), "w");
        if (!fz || !fw) {
          if (fz) fclose(fz);
          if (fw) fclose(fw);
          rc = derr(OCO_EIO, "cannot write the grid files in %s", out.c_str());
          break;
        }
        for (int i = 1; i <= nz; i++) fprintf(fz, "%s\n", list_int_real(i, z[(size_t)(kNg + i - 1)]).c_str());
        for (int i = 1; i <= nw; i++) fprintf(fw, "%s\n", list_int_real(i, d.wa[(size_t)i - 1]).c_str());
        fclose(fz);
        fclose(fw);
        if (!write_record_file(out + "/zgrid.bin", z.data(), z.size()) ||
            !write_record_file(out + "/wavegrid.bin", d.wa.data(), d.wa.size())) {
          rc = derr(OCO_EIO, "cannot write the grid files in %s", out.c_str());
          break;
        }
        /* output_ascii of the block's last column, io.f90:31-46: "(I6, nw(2e15.5))" */
        FILE *fo = fopen((out + "/diagnostics.txt").c_str(), "w");
        if (!fo) {
          rc = derr(OCO_EIO, "cannot write %s/diagnostics.txt", out.c_str());
          break;
        }
        const size_t col = ncol - 1;
        char cell[32];
        for (int i = 0; i < nz; i++) {
          fprintf(fo, "%6d", i + 1);
          for (int iw = 0; iw < nw; iw++) {
            oco_format_e(U[((size_t)iw * ncol + col) * mz + kNg + i], 15, 5, cell);
            fputs(cell, fo);
          }
          for (int iw = 0; iw < nw; iw++) {
            oco_format_e(K[((size_t)iw * ncol + col) * nz + i], 15, 5, cell);
            fputs(cell, fo);
          }
          fputc('\n', fo);
        }
        fclose(fo);
      }
      if (write_binary) { /* output_binary, io.f90:77-101 */
        const std::string bd = out + "/procx" + std::to_string(ipx) + "_procy" + std::to_string(ipy);
        if (!make_dirs(bd) || !write_record_file(bd + "/mean_intensity_" + d.snapshot + ".bin", U.data(), U.size()) ||
            !write_record_file(bd + "/absorption_coefficients_" + d.snapshot + ".bin", K.data(), K.size()) ||
            !write_record_file(bd + "/flux_" + d.snapshot + ".bin", V.data(), V.size())) {
          rc = derr(OCO_EIO, "cannot write the binary outputs in %s", bd.c_str());
          break;
        }
      }
    }
  }
  return rc ? rc : zero_pivot_rc;
}

/* The C entry points: host allocations sized by the deck can fail, and an exception must not
 * cross the C ABI, so it becomes an error code. */
extern "C" int oco_deck_block_inputs(const char *deck_dir, const char *snapshot, int32_t iprocx, int32_t iprocy,
                                     oco_deck_info *info, double *rho, double *T, double *wa, double *z) {
  try {
    return deck_block_inputs(deck_dir, snapshot, iprocx, iprocy, info, rho, T, wa, z);
  } catch (const std::bad_alloc &) {
    return derr(OCO_ENOMEM, "oco_deck_block_inputs: out of host memory");
  } catch (const std::exception &e) {
    return derr(OCO_EINVAL, "oco_deck_block_inputs: %s", e.what());
  }
}

extern "C" int oco_deck_block_inputs_device(oco_ctx *ctx, const char *deck_dir, const char *snapshot, int32_t iprocx,
                                            int32_t iprocy, oco_deck_info *info, double *rho, double *T, double *wa,
                                            double *z, void *stream) {
  try {
    return deck_block_inputs_device(ctx, deck_dir, snapshot, iprocx, iprocy, info, rho, T, wa, z,
                                    (cudaStream_t)stream);
  } catch (const std::bad_alloc &) {
    return derr(OCO_ENOMEM, "oco_deck_block_inputs_device: out of host memory");
  } catch (const std::exception &e) {
    return derr(OCO_EINVAL, "oco_deck_block_inputs_device: %s", e.what());
  }
}

extern "C" int oco_run_deck(const char *deck_dir, const char *snapshot, const char *out_dir, int32_t form,
                            int32_t device, int32_t write_binary) {
  try {
    return run_deck(deck_dir, snapshot, out_dir, form, device, write_binary);
  } catch (const std::bad_alloc &) {
    return derr(OCO_ENOMEM, "oco_run_deck: out of host memory");
  } catch (const std::exception &e) {
    return derr(OCO_EINVAL, "oco_run_deck: %s", e.what());
  }
}

extern "C" const char *oco_deck_last_error(void) { return g_deck_err.c_str(); }
