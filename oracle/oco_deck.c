/*
 * oco_deck.c -- runs a reference sample deck through the oracle (TEST INFRASTRUCTURE ONLY).
 * Restates the driver parts around the hot loop: namelist input (flux_feautrier.f90:58-76,
 * disk.f90:15-40, gas_state.f90:15-28, read_athena.f90:27-62), the compile-time
 * resolution.in (read here as text), the synthetic disk (disk.f90:42-129), the Athena
 * reader (read_athena.f90:64-291) and output_ascii (io.f90:31-46).
 */
#include "oco_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- gfortran Ew.d editing --------------------------------------------------------- */
void oracle_format_e(double v, int w, int d, char *out) {
  char body[64];
  if (v != v) {
    snprintf(body, sizeof body, "NaN");
  } else if (isinf(v)) {
    snprintf(body, sizeof body, "%s", v > 0 ? "Infinity" : "-Infinity");
  } else {
    char buf[64];
    int e10 = 0;
    char digits[32];
    if (v == 0.0) {
      memset(digits, '0', (size_t)d);
      digits[d] = 0;
      e10 = 0;
    } else {
      snprintf(buf, sizeof buf, "%.*e", d - 1, fabs(v)); /* d.dddde+XX, correctly rounded */
      int k = 0;
      for (const char *q = buf; *q && *q != 'e'; q++)
        if (isdigit((unsigned char)*q)) digits[k++] = *q;
      digits[k] = 0;
      e10 = atoi(strchr(buf, 'e') + 1) + 1;
    }
    char ex[16];
    if (abs(e10) <= 99)
      snprintf(ex, sizeof ex, "E%c%02d", e10 < 0 ? '-' : '+', abs(e10));
    else
      snprintf(ex, sizeof ex, "%c%03d", e10 < 0 ? '-' : '+', abs(e10));
    snprintf(body, sizeof body, "%s0.%s%s", signbit(v) ? "-" : "", digits, ex);
  }
  int len = (int)strlen(body);
  if (len > w) {
    memset(out, '*', (size_t)w);
    out[w] = 0;
    return;
  }
  memset(out, ' ', (size_t)(w - len));
  memcpy(out + (w - len), body, (size_t)len + 1);
}

/* ---- namelist reading ---------------------------------------------------------------- */
static char *slurp(const char *path) {
  FILE *fp = fopen(path, "rb");
  if (!fp) return NULL;
  fseek(fp, 0, SEEK_END);
  long n = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  char *s = (char *)malloc((size_t)n + 1);
  if (s && fread(s, 1, (size_t)n, fp) != (size_t)n) {
    free(s);
    s = NULL;
  }
  if (s) s[n] = 0;
  fclose(fp);
  return s;
}

typedef struct {
  char key[64];
  char val[256];
} nml_item;

/* Parses group &name ... / into items; returns the count (or -1 if the group is absent). */
static int nml_group(const char *text, const char *name, nml_item *items, int maxitems) {
  size_t nl = strlen(name);
  const char *s = text;
  const char *g = NULL;
  while (*s) {
    if (*s == '!') { /* comment */
      while (*s && *s != '\n') s++;
      continue;
    }
    if (*s == '&' && strncasecmp(s + 1, name, nl) == 0 && !isalnum((unsigned char)s[1 + nl]) &&
        s[1 + nl] != '_') {
      g = s + 1 + nl;
      break;
    }
    s++;
  }
  if (!g) return -1;
  int n = 0;
  s = g;
  for (;;) {
    while (*s && (isspace((unsigned char)*s) || *s == ',')) s++;
    if (*s == '!') {
      while (*s && *s != '\n') s++;
      continue;
    }
    if (!*s || *s == '/' || *s == '&') break;
    const char *k0 = s;
    while (*s && (isalnum((unsigned char)*s) || *s == '_')) s++;
    if (s == k0) break;
    nml_item it;
    size_t kl = (size_t)(s - k0);
    if (kl >= sizeof it.key) kl = sizeof it.key - 1;
    memcpy(it.key, k0, kl);
    it.key[kl] = 0;
    while (*s && isspace((unsigned char)*s)) s++;
    if (*s != '=') break;
    s++;
    while (*s && isspace((unsigned char)*s)) s++;
    size_t vl = 0;
    if (*s == '"' || *s == '\'') {
      char q = *s++;
      while (*s && *s != q && vl < sizeof it.val - 1) it.val[vl++] = *s++;
      if (*s == q) s++;
    } else {
      while (*s && !isspace((unsigned char)*s) && *s != ',' && *s != '/' && *s != '!' &&
             vl < sizeof it.val - 1)
        it.val[vl++] = *s++;
    }
    it.val[vl] = 0;
    if (n < maxitems) items[n++] = it;
  }
  return n;
}

static const char *nml_get(const nml_item *items, int n, const char *key) {
  for (int i = 0; i < n; i++)
    if (strcasecmp(items[i].key, key) == 0) return items[i].val;
  return NULL;
}

/* Fortran real literal (d/D exponent) -> double, correctly rounded by strtod. */
static double fortran_real(const char *s) {
  char b[256];
  size_t i = 0;
  for (; s[i] && i < sizeof b - 1; i++) b[i] = (s[i] == 'd' || s[i] == 'D') ? 'e' : s[i];
  b[i] = 0;
  return strtod(b, NULL);
}

static int fortran_logical(const char *s) {
  while (*s == '.') s++;
  return (*s == 'T' || *s == 't');
}

static void nml_real(const nml_item *it, int n, const char *key, double *dst) {
  const char *v = nml_get(it, n, key);
  if (v) *dst = fortran_real(v);
}

/* ---- resolution.in: "integer, parameter :: a=expr, b=expr" lines -------------------- */
typedef struct {
  char name[32];
  long val;
} ivar;

static long eval_int(const char *s, const ivar *vars, int nv, int *ok) {
  /* left-to-right evaluation of terms joined by + - * / (integer arithmetic, Fortran
   * precedence: * and / before + and -) */
  long total = 0, term = 0;
  int addop = '+', mulop = 0;
  const char *p = s;
  for (;;) {
    while (*p == ' ') p++;
    long v = 0;
    if (isdigit((unsigned char)*p)) {
      v = strtol(p, (char **)&p, 10);
    } else if (isalpha((unsigned char)*p)) {
      char nm[32];
      int k = 0;
      while ((isalnum((unsigned char)*p) || *p == '_') && k < 31) nm[k++] = (char)tolower(*p++);
      nm[k] = 0;
      int found = 0;
      for (int i = 0; i < nv; i++)
        if (strcmp(vars[i].name, nm) == 0) {
          v = vars[i].val;
          found = 1;
        }
      if (!found) *ok = 0;
    } else {
      *ok = 0;
      return 0;
    }
    term = mulop == 0 ? v : (mulop == '*' ? term * v : (v ? term / v : 0));
    while (*p == ' ') p++;
    if (*p == '*' || *p == '/') {
      mulop = *p++;
      continue;
    }
    total = addop == '+' ? total + term : total - term;
    mulop = 0;
    if (*p == '+' || *p == '-') {
      addop = *p++;
      continue;
    }
    break;
  }
  return total;
}

static int read_resolution(const char *path, ivar *vars, int *nv) {
  char *t = slurp(path);
  if (!t) return -1;
  *nv = 0;
  char *save = NULL;
  for (char *line = strtok_r(t, "\n", &save); line; line = strtok_r(NULL, "\n", &save)) {
    char *bang = strchr(line, '!');
    if (bang) *bang = 0;
    char *dc = strstr(line, "::");
    if (!dc) continue;
    char *p = dc + 2;
    /* split at top-level commas */
    char *tok_save = NULL;
    for (char *as = strtok_r(p, ",", &tok_save); as; as = strtok_r(NULL, ",", &tok_save)) {
      char *eq = strchr(as, '=');
      if (!eq) continue;
      *eq = 0;
      char nm[32];
      int k = 0;
      for (char *q = as; *q && k < 31; q++)
        if (!isspace((unsigned char)*q)) nm[k++] = (char)tolower(*q);
      nm[k] = 0;
      int ok = 1;
      long v = eval_int(eq + 1, vars, *nv, &ok);
      if (ok && *nv < 32) {
        snprintf(vars[*nv].name, sizeof vars[*nv].name, "%s", nm);
        vars[*nv].val = v;
        (*nv)++;
      }
    }
  }
  free(t);
  return 0;
}

static long rget(const ivar *v, int n, const char *name, long dflt) {
  for (int i = 0; i < n; i++)
    if (strcmp(v[i].name, name) == 0) return v[i].val;
  return dflt;
}

/* ---- run a deck ------------------------------------------------------------------------- */
typedef struct {
  double isoTemp, sigma, midTemp, floorTemp, switchTemp;
  int have_tgauss;
  double *Tgauss;
} tstate;

/* calc_temperature, disk.f90:64-109 */
static void calc_temperature(double *T, const double *z, int nz, tstate *ts, int lathena) {
  if (!lathena)
    for (int i = 0; i < nz; i++) T[i] = ts->midTemp;
  if (!ts->have_tgauss) {
    for (int i = 0; i < nz; i++) {
      double zz = z[3 + i];
      ts->Tgauss[i] = ts->midTemp * exp(-((0.5 * (zz * zz)) / (ts->sigma * ts->sigma)));
    }
    ts->have_tgauss = 1;
  }
  for (int i = 0; i < nz; i++)
    if (T[i] < ts->switchTemp) T[i] = (ts->Tgauss[i] > ts->floorTemp) ? ts->Tgauss[i] : ts->floorTemp;
}

static void fail(char *msg, int len, const char *fmt, ...) {
  if (!msg || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, (size_t)len, fmt, ap);
  va_end(ap);
}

static int read_i32(FILE *fp, int32_t *v) { return fread(v, 4, 1, fp) == 1 ? 0 : -1; }
static int read_f64(FILE *fp, double *v, size_t n) { return fread(v, 8, n, fp) == n ? 0 : -1; }

int oracle_run_deck(const char *deck, const char *outdir, char *msg, int msglen) {
  char path[1024];
  int rc = 0;
  snprintf(path, sizeof path, "%s/resolution.in", deck);
  ivar rv[32];
  int nrv = 0;
  if (read_resolution(path, rv, &nrv) != 0) {
    fail(msg, msglen, "cannot read %s", path);
    return ORACLE_EIO;
  }
  const int nw = (int)rget(rv, nrv, "nw", 0), nx = (int)rget(rv, nrv, "nx", 0);
  const int ny = (int)rget(rv, nrv, "ny", 0), nz = (int)rget(rv, nrv, "nz", 0);
  const int nprocx = (int)rget(rv, nrv, "nprocx", 1), nprocy = (int)rget(rv, nrv, "nprocy", 1);
  const int nprocz = (int)rget(rv, nrv, "nprocz", 1);
  const int nxloc = (int)rget(rv, nrv, "nxloc", nx / nprocx), nyloc = (int)rget(rv, nrv, "nyloc", ny / nprocy);
  const int mz = nz + 6;
  snprintf(path, sizeof path, "%s/input.in", deck);
  char *txt = slurp(path);
  if (!txt) {
    fail(msg, msglen, "cannot read %s", path);
    return ORACLE_EIO;
  }
  nml_item it[64];
  int n;
  double z0 = 0, z1 = 0, w0 = 3000, w1 = 5000, sigma_grey = 0;
  int lgrey = 0, lread_athena = 1;
  n = nml_group(txt, "input", it, 64); /* flux_feautrier.f90:58, defaults :50, :57 */
  nml_real(it, n, "z0", &z0);
  nml_real(it, n, "z1", &z1);
  nml_real(it, n, "w0", &w0);
  nml_real(it, n, "w1", &w1);
  nml_real(it, n, "sigma_grey", &sigma_grey);
  if (nml_get(it, n, "lgrey")) lgrey = fortran_logical(nml_get(it, n, "lgrey"));
  if (nml_get(it, n, "lread_athena")) lread_athena = fortran_logical(nml_get(it, n, "lread_athena"));
  tstate ts = {0};
  n = nml_group(txt, "temperature_input", it, 64);
  nml_real(it, n, "isoTemp", &ts.isoTemp);
  nml_real(it, n, "sigma", &ts.sigma);
  nml_real(it, n, "midTemp", &ts.midTemp);
  nml_real(it, n, "floorTemp", &ts.floorTemp);
  ts.switchTemp = (1.0 + 0x1p-52) * ts.isoTemp; /* disk.f90:28 */
  double rho0 = 0, rho_floor = 0, H = 0, fully_ionized_T = 0;
  n = nml_group(txt, "density_input", it, 64);
  nml_real(it, n, "rho0", &rho0);
  nml_real(it, n, "rho_floor", &rho_floor);
  nml_real(it, n, "H", &H);
  n = nml_group(txt, "gas_state_input", it, 64);
  nml_real(it, n, "fully_ionized_T", &fully_ionized_T);
  char RunName[256] = "", datadir[512] = "./input_athena/distributed";
  double Mbh_SolarMasses = 0, r0ref_rg = 0, aspect_ratio = 0, mmw = 0, a_rho0 = 0;
  double a_rho_floor = NAN;
  int lavoid = 1;
  if (lread_athena) {
    n = nml_group(txt, "athena_input", it, 64);
    if (nml_get(it, n, "RunName")) snprintf(RunName, sizeof RunName, "%s", nml_get(it, n, "RunName"));
    if (nml_get(it, n, "datadir")) snprintf(datadir, sizeof datadir, "%s", nml_get(it, n, "datadir"));
    nml_real(it, n, "Mbh_SolarMasses", &Mbh_SolarMasses);
    nml_real(it, n, "r0ref_rg", &r0ref_rg);
    nml_real(it, n, "aspect_ratio", &aspect_ratio);
    nml_real(it, n, "mean_molecular_weight", &mmw);
    nml_real(it, n, "rho0", &a_rho0);
    nml_real(it, n, "rho_floor", &a_rho_floor);
    if (nml_get(it, n, "lavoid_momentum_underflow"))
      lavoid = fortran_logical(nml_get(it, n, "lavoid_momentum_underflow"));
  }
  free(txt);
  if (lgrey && nw != 1) {
    fail(msg, msglen, "For Grey RT use only one wavelength. Switch nw=1 in resolution.in");
    return ORACLE_EGREY;
  }
  double *wa = (double *)calloc((size_t)nw, sizeof(double));
  oracle_calc_wavelength(w1, w0, nw, wa);
  /* read_athena_input, read_athena.f90:41-54 */
  const double G = 6.6742e-8, c_light = 2.99792458e10, SolarMass = 1.988409870698051e+33;
  const double amu = 1.66053906660e-24, k1_cgs = 1.0 / 1.380649e-16;
  double unit_density = 0, unit_length = 0, unit_temperature = 0;
  if (lread_athena) {
    double Mbh = Mbh_SolarMasses * SolarMass;
    double rg = (2.0 * (G / (c_light * c_light))) * Mbh;
    double rr = r0ref_rg * rg;
    double g0 = G * Mbh;
    double Omega = sqrt(g0) * pow(rr, -1.5);
    double Hs = aspect_ratio * rr;
    unit_density = a_rho0;
    double unit_time = 1.0 / Omega;
    unit_length = Hs;
    double unit_velocity = unit_length / unit_time;
    unit_temperature = ((mmw * amu) * k1_cgs) * (unit_velocity * unit_velocity);
  }
  const size_t ncol = (size_t)nxloc * nyloc;
  double *rho3d = (double *)calloc(ncol * nz, sizeof(double));
  double *temp3d = (double *)calloc(ncol * nz, sizeof(double));
  double *U = (double *)calloc(ncol * mz * nw, sizeof(double));
  double *K = (double *)calloc(ncol * nz * nw, sizeof(double));
  double *z = (double *)calloc((size_t)mz, sizeof(double));
  double *zn = (double *)calloc((size_t)nz, sizeof(double));
  ts.Tgauss = (double *)calloc((size_t)nz, sizeof(double));
  double dz = 0;
  for (int iprocx = 0; iprocx < nprocx && rc == 0; iprocx++) {
    for (int iprocy = 0; iprocy < nprocy && rc == 0; iprocy++) {
      int lroot = (iprocx == 0 && iprocy == 0);
      if (lread_athena) {
        /* read_from_athena, read_athena.f90:98-207 */
        double z0a = 0, dza = 0, gamma1 = 0;
        for (int iprocz = 0; iprocz < nprocz && rc == 0; iprocz++) {
          int iproc = iprocz * nprocx * nprocy + iprocy * nprocx + iprocx;
          char fn[1200];
          if (iproc == 0)
            snprintf(fn, sizeof fn, "%s/%s/id%d/%s.0000.bin", deck, datadir, iproc, RunName);
          else
            snprintf(fn, sizeof fn, "%s/%s/id%d/%s-id%d.0000.bin", deck, datadir, iproc, RunName, iproc);
          FILE *fp = fopen(fn, "rb");
          if (!fp) {
            fail(msg, msglen, "File %s does not exist", fn);
            rc = ORACLE_EIO;
            break;
          }
          int32_t coordsys, nxl, nyl, nzl, dum[4];
          double dreal[3];
          if (read_i32(fp, &coordsys) || read_i32(fp, &nxl) || read_i32(fp, &nyl) || read_i32(fp, &nzl) ||
              fread(dum, 4, 4, fp) != 4 || read_f64(fp, &gamma1, 1) || read_f64(fp, dreal, 3)) {
            fclose(fp);
            rc = ORACLE_EIO;
            break;
          }
          if (nxl != nxloc || nyl != nyloc) {
            fclose(fp);
            fail(msg, msglen, "Athena dimensionality mismatch");
            rc = ORACLE_EDIM;
            break;
          }
          double *xl = (double *)malloc(sizeof(double) * (size_t)(nxl + nyl + nzl));
          size_t nc = (size_t)nxl * nyl * nzl;
          double *tmp = (double *)malloc(sizeof(double) * nc);
          if (read_f64(fp, xl, (size_t)(nxl + nyl + nzl))) rc = ORACLE_EIO;
          double *zloc = xl + nxl + nyl;
          if (iprocz == 0) {
            z0a = zloc[0];
            dza = zloc[1] - zloc[0];
          }
          int iz0 = (int)lround((zloc[0] - z0a) / dza); /* nint(...) + 1, 0-based here */
          for (int k = 0; k < nzl; k++) zn[iz0 + k] = zloc[k];
          /* tmp is (nxloc, nyloc, nzloc) with x fastest; rho(iz, iy, ix) = tmp(ix, iy, iz) */
#define CELL(ix, iy, iz) ((size_t)(iz) * nxl * nyl + (size_t)(iy) * nxl + (ix))
#define DST(ix, iy, iz) (((size_t)(ix) * nyloc + (iy)) * nz + (size_t)(iz0 + (iz)))
          if (!rc && read_f64(fp, tmp, nc)) rc = ORACLE_EIO;
          for (int ix = 0; ix < nxl && !rc; ix++)
            for (int iy = 0; iy < nyl; iy++)
              for (int iz = 0; iz < nzl; iz++) {
                rho3d[DST(ix, iy, iz)] = tmp[CELL(ix, iy, iz)];
                temp3d[DST(ix, iy, iz)] = 0.0;
              }
          for (int comp = 0; comp < 3 && !rc; comp++) { /* rux, ruy, ruz :176-195 */
            if (read_f64(fp, tmp, nc)) {
              rc = ORACLE_EIO;
              break;
            }
            for (int ix = 0; ix < nxl; ix++)
              for (int iy = 0; iy < nyl; iy++)
                for (int iz = 0; iz < nzl; iz++) {
                  double pp = tmp[CELL(ix, iy, iz)];
                  size_t dd = DST(ix, iy, iz);
                  if (!lavoid || fabs(pp) >= 0x1p-52)
                    temp3d[dd] = temp3d[dd] + (0.5 * (pp * pp)) / rho3d[dd];
                }
          }
          if (!rc && read_f64(fp, tmp, nc)) rc = ORACLE_EIO; /* eng :201-202 */
          for (int ix = 0; ix < nxl && !rc; ix++)
            for (int iy = 0; iy < nyl; iy++)
              for (int iz = 0; iz < nzl; iz++) {
                size_t dd = DST(ix, iy, iz);
                temp3d[dd] = (tmp[CELL(ix, iy, iz)] - temp3d[dd]) / rho3d[dd];
              }
#undef CELL
#undef DST
          free(tmp);
          free(xl);
          fclose(fp);
        }
        if (rc) break;
        /* postprocess_athena_values, read_athena.f90:230-277 */
        if (a_rho_floor != a_rho_floor) {
          fail(msg, msglen, "Must set rho_floor");
          rc = ORACLE_ENAN;
          break;
        }
        for (size_t i = 0; i < ncol * nz; i++) {
          rho3d[i] = rho3d[i] * unit_density;
          if (rho3d[i] < a_rho_floor) rho3d[i] = a_rho_floor;
          temp3d[i] = (temp3d[i] * gamma1) * unit_temperature;
        }
        for (int i = 0; i < nz; i++) zn[i] = zn[i] * unit_length;
        dz = (zn[nz - 1] - zn[0]) / (double)(nz - 1);
        for (int i = 0; i < nz; i++) z[3 + i] = zn[i];
        for (int i = 1; i <= 3; i++) {
          z[3 - i] = z[3] - (double)i * dz;
          z[nz + 2 + i] = z[nz + 2] + (double)i * dz;
        }
        for (size_t c = 0; c < ncol; c++) calc_temperature(temp3d + c * nz, z, nz, &ts, 1);
      } else {
        if (lroot) { /* calc_grid, disk.f90:42-62 */
          dz = (z1 - z0) / (double)(nz - 1);
          for (int i = 1; i <= nz; i++) z[3 + i - 1] = z0 + (double)(i - 1) * dz;
          for (int i = 1; i <= 3; i++) {
            z[3 - i] = z[3] - (double)i * dz;
            z[nz + 2 + i] = z[nz + 2] + (double)i * dz;
          }
        }
        double *rc0 = rho3d, *tc0 = temp3d;
        for (int i = 0; i < nz; i++) { /* calc_density, disk.f90:111-129 */
          double zz = z[3 + i];
          rc0[i] = rho0 * exp(-((0.5 * (zz * zz)) / (H * H)));
          if (rc0[i] < rho_floor) rc0[i] = rho_floor;
        }
        calc_temperature(tc0, z, nz, &ts, 0);
        for (size_t c = 1; c < ncol; c++) {
          memcpy(rho3d + c * nz, rc0, sizeof(double) * nz);
          memcpy(temp3d + c * nz, tc0, sizeof(double) * nz);
        }
      }
      oracle_params prm = {nxloc, nyloc, nz, nw, dz, lgrey, ORACLE_FORM_REFERENCE, sigma_grey, fully_ionized_T};
      int64_t bad = -1;
      int src = oracle_solve_block(&prm, wa, rho3d, temp3d, U, K, NULL, &bad);
      if (src == ORACLE_EZEROPIVOT) {
        fail(msg, msglen, "ERROR tridiag: zero pivot at item %lld", (long long)bad);
        rc = src;
        break;
      } else if (src) {
        rc = src;
        break;
      }
      if (lroot) { /* block inputs, for feeding the same bytes to the GPU engine in tests */
        snprintf(path, sizeof path, "%s/inputs_meta.txt", outdir);
        FILE *fm = fopen(path, "w");
        if (fm) {
          fprintf(fm, "%d %d %d %d %.17g %d %.17g %.17g\n", nxloc, nyloc, nz, nw, dz, lgrey, sigma_grey,
                  fully_ionized_T);
          fclose(fm);
        }
        const char *names[3] = {"inputs_rho.bin", "inputs_T.bin", "inputs_wa.bin"};
        const double *arrs[3] = {rho3d, temp3d, wa};
        size_t counts[3] = {ncol * nz, ncol * nz, (size_t)nw};
        for (int q = 0; q < 3; q++) {
          snprintf(path, sizeof path, "%s/%s", outdir, names[q]);
          FILE *fb = fopen(path, "wb");
          if (fb) {
            fwrite(arrs[q], sizeof(double), counts[q], fb);
            fclose(fb);
          }
        }
      }
      if (lroot) { /* output_ascii of the last column of the root block, io.f90:31-46 */
        snprintf(path, sizeof path, "%s/diagnostics.txt", outdir);
        FILE *fo = fopen(path, "w");
        if (!fo) {
          rc = ORACLE_EIO;
          break;
        }
        size_t col = ncol - 1;
        char cell[32];
        for (int i = 0; i < nz; i++) {
          fprintf(fo, "%6d", i + 1);
          for (int iw = 0; iw < nw; iw++) {
            oracle_format_e(U[((size_t)iw * ncol + col) * mz + 3 + i], 15, 5, cell);
            fputs(cell, fo);
          }
          for (int iw = 0; iw < nw; iw++) {
            oracle_format_e(K[((size_t)iw * ncol + col) * nz + i], 15, 5, cell);
            fputs(cell, fo);
          }
          fputc('\n', fo);
        }
        fclose(fo);
      }
    }
  }
  free(wa);
  free(rho3d);
  free(temp3d);
  free(U);
  free(K);
  free(z);
  free(zn);
  free(ts.Tgauss);
  return rc;
}
