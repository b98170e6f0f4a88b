// Host side of the `gramsci` driver (include/gramsci_host.h): the parts of
// the reference's main program (csabiu/Gramsci src/gramsci.F90) that sit
// around the hot path -- option parsing, list-directed catalogue reading,
// weight normalisation, radial bin edges and the formatted output files.
#include "../../../include/gramsci_host.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace {

// ------------------------------------------------------------ list-directed --
// A minimal model of Fortran list-directed input: a file is a sequence of
// records; one READ starts at the next record, takes values separated by
// blanks, tabs or commas, continues onto later records when the current one
// runs out, and skips the rest of its last record.  A slash ends the READ.
struct Records {
  std::vector<std::string> lines;
  size_t next = 0;
};

bool load_records(const char* path, Records& R) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::string cur;
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) {
    for (size_t i = 0; i < k; ++i) {
      if (buf[i] == '\n') {
        if (!cur.empty() && cur.back() == '\r') cur.pop_back();
        R.lines.push_back(cur);
        cur.clear();
      } else {
        cur.push_back(buf[i]);
      }
    }
  }
  if (!cur.empty()) R.lines.push_back(cur);
  std::fclose(f);
  return true;
}

void split_tokens(const std::string& s, std::vector<std::string>& out, bool& slash) {
  out.clear();
  slash = false;
  std::string t;
  for (char ch : s) {
    if (ch == '/') {
      slash = true;
      break;
    }
    if (ch == ' ' || ch == '\t' || ch == ',') {
      if (!t.empty()) out.push_back(t);
      t.clear();
    } else {
      t.push_back(ch);
    }
  }
  if (!t.empty() && !slash) out.push_back(t);
  else if (!t.empty() && slash) out.push_back(t);
}

// Fortran real: D/Q exponent letters accepted.
bool parse_real(const std::string& tok, double& v) {
  std::string s = tok;
  for (char& ch : s)
    if (ch == 'd' || ch == 'D' || ch == 'q' || ch == 'Q') ch = 'e';
  if (s.empty()) return false;
  char* end = nullptr;
  errno = 0;
  v = std::strtod(s.c_str(), &end);
  return end && *end == '\0';
}

// A real(4) item: the decimal string rounded once to single precision.
bool parse_real4(const std::string& tok, float& v) {
  std::string s = tok;
  for (char& ch : s)
    if (ch == 'd' || ch == 'D' || ch == 'q' || ch == 'Q') ch = 'e';
  if (s.empty()) return false;
  char* end = nullptr;
  v = std::strtof(s.c_str(), &end);
  return end && *end == '\0';
}

bool parse_int(const std::string& tok, long long& v) {
  if (tok.empty()) return false;
  char* end = nullptr;
  errno = 0;
  v = std::strtoll(tok.c_str(), &end, 10);
  return end && *end == '\0' && errno == 0;
}

enum ReadStatus { R_OK = 0, R_END = 1, R_ERR = 2 };

// One list-directed READ of `k` items; kind[i] = 'r' real or 'i' integer.
ReadStatus list_read(Records& R, int k, const char* kind, double* rv, long long* iv) {
  int got = 0;
  std::vector<std::string> tok;
  bool slash = false;
  while (got < k) {
    if (R.next >= R.lines.size()) return R_END;
    split_tokens(R.lines[R.next++], tok, slash);
    for (size_t t = 0; t < tok.size() && got < k; ++t) {
      bool ok = kind[got] == 'i' ? parse_int(tok[t], iv[got]) : parse_real(tok[t], rv[got]);
      if (!ok) return R_ERR;
      got++;
    }
    if (slash) return R_OK;
  }
  return R_OK;
}

// count_files_2 (src/gramsci.F90:1319-1340): one-value READs until end of
// file; a READ that fails is not counted and reading continues.
int64_t count_records(Records& R) {
  int64_t n = 0;
  R.next = 0;
  double v;
  long long iv;
  for (;;) {
    ReadStatus s = list_read(R, 1, "r", &v, &iv);
    if (s == R_END) break;
    if (s == R_OK) n++;
  }
  R.next = 0;
  return n;
}

// read_files_2 loop (src/gramsci.F90:1368-1373): READ x y z w for i = 1..n;
// on a read error the reference jumps back to its DO statement, so filling
// restarts at i = 1 with the next record; end of file stops the loop.
void read_points(Records& R, int64_t n, double* xyz, double* w) {
  R.next = 0;
  double v[4];
  long long iv[4];
  for (int64_t i = 0; i < n; ++i) {
    ReadStatus s = list_read(R, 4, "rrrr", v, iv);
    if (s == R_END) return;
    if (s == R_ERR) {
      i = -1;
      continue;
    }
    xyz[3 * i] = v[0];
    xyz[3 * i + 1] = v[1];
    xyz[3 * i + 2] = v[2];
    w[i] = v[3];
  }
}

bool opt_is(const char* opt6, const char* name) { return std::strcmp(opt6, name) == 0; }

void set_text(char* dst, size_t cap, const char* src) {
  std::snprintf(dst, cap, "%s", src ? src : "");
}

}  // namespace

extern "C" {

int grh_parse_args(int argc, const char* const* argv, grh_options* o) {
  std::memset(o, 0, sizeof(*o));
  // default_params (src/gramsci.F90:1627-1652)
  set_text(o->out, sizeof(o->out), "result.txt");
  o->nmu = 1;
  o->nbins = 0;
  o->rmin = 0.0;
  o->rmax = 0.0;
  const int n = argc - 1;
  if (n < 6) {  // :1177-1183
    o->help = 1;
    return 0;
  }
  int i = 1;
  auto arg = [&](int k) -> const char* { return k <= n ? argv[k] : ""; };
  while (i <= n) {
    // character(len=6) :: opt  -- options are compared on six characters
    char opt[7];
    std::snprintf(opt, sizeof(opt), "%s", argv[i]);
    for (int k = (int)std::strlen(opt) - 1; k >= 0 && opt[k] == ' '; --k) opt[k] = '\0';
    if (opt_is(opt, "-gal")) {
      set_text(o->gal, sizeof(o->gal), arg(i + 1));
      i += 2;
    } else if (opt_is(opt, "-ran")) {
      o->rancat = 1;
      set_text(o->ran, sizeof(o->ran), arg(i + 1));
      i += 2;
    } else if (opt_is(opt, "-out")) {
      set_text(o->out, sizeof(o->out), arg(i + 1));
      i += 2;
    } else if (opt_is(opt, "-rmin") || opt_is(opt, "-rmax")) {
      std::vector<std::string> tok;
      bool slash;
      split_tokens(arg(i + 1), tok, slash);
      double v;
      if (tok.empty() || !parse_real(tok[0], v)) {
        o->error = 2;
        std::snprintf(o->message, sizeof(o->message), "bad real number for %s: '%s'", opt, arg(i + 1));
        return 2;
      }
      if (opt[3] == 'i') o->rmin = v; else o->rmax = v;
      i += 2;
    } else if (opt_is(opt, "-nbins") || opt_is(opt, "-nmu")) {
      std::vector<std::string> tok;
      bool slash;
      split_tokens(arg(i + 1), tok, slash);
      long long v;
      if (tok.empty() || !parse_int(tok[0], v)) {
        o->error = 2;
        std::snprintf(o->message, sizeof(o->message), "bad integer for %s: '%s'", opt, arg(i + 1));
        return 2;
      }
      if (opt[2] == 'b') {
        o->nbins = (int32_t)v;
      } else {
        o->nmu = (int32_t)v;
        if (o->nmu >= 2) o->rsd = 1;  // :1216-1223
      }
      i += 2;
    } else if (opt_is(opt, "-cut")) {
      o->cut_mode = 1;
      set_text(o->cut, sizeof(o->cut), arg(i + 1));
      set_text(o->out, sizeof(o->out), arg(i + 1));  // :1224-1231 output = region file
      i += 2;
    } else if (opt_is(opt, "-mpi")) {
      o->mpi = 1;
      i += 1;
    } else if (opt_is(opt, "-log")) {
      o->logbins = 1;
      i += 1;
    } else if (opt_is(opt, "-help")) {
      o->help = 1;
      return 0;
    } else if (opt_is(opt, "-tetra")) {
      o->tetra = 1;
      i += 1;
    } else if (opt_is(opt, "-3pcf")) {
      o->three_pcf = 1;
      i += 1;
    } else if (opt_is(opt, "-4pcf")) {
      o->four_pcf = 1;
      i += 1;
    } else if (opt_is(opt, "-equi")) {
      o->equi = 1;
      i += 1;
    } else if (opt_is(opt, "-gcol")) {
      o->gcol = 1;
      i += 1;
    } else if (opt_is(opt, "-2pcf")) {
      o->two_pcf = 1;
      i += 1;
    } else {  // :1265-1267
      o->error = 1;
      std::snprintf(o->message, sizeof(o->message), "unknown option %s ignored", opt);
      return 1;
    }
  }
  return 0;
}

int grh_read_catalogue(const char* gal, const char* ran, double** xyz, double** w,
                       int64_t* n_data, int64_t* n_rand) {
  Records G, Rr;
  if (!load_records(gal, G)) return -1;
  bool have_ran = ran && ran[0];
  if (have_ran && !load_records(ran, Rr)) return -2;
  const int64_t nd = count_records(G);
  const int64_t nr = have_ran ? count_records(Rr) : 0;
  const int64_t n = nd + nr;
  double* p = static_cast<double*>(std::calloc((size_t)(3 * n + 3), sizeof(double)));
  double* q = static_cast<double*>(std::calloc((size_t)(n + 1), sizeof(double)));
  if (!p || !q) {
    std::free(p);
    std::free(q);
    return -3;
  }
  read_points(G, nd, p, q);
  if (have_ran) read_points(Rr, nr, p + 3 * nd, q + nd);
  *xyz = p;
  *w = q;
  *n_data = nd;
  *n_rand = nr;
  return 0;
}

int grh_read_region(const char* path, double** xyz, double** w, int32_t** buffer, int64_t* n) {
  Records R;
  if (!load_records(path, R)) return -1;
  const int64_t m = count_records(R);
  double* p = static_cast<double*>(std::calloc((size_t)(3 * m + 3), sizeof(double)));
  double* q = static_cast<double*>(std::calloc((size_t)(m + 1), sizeof(double)));
  int32_t* b = static_cast<int32_t*>(std::calloc((size_t)(m + 1), sizeof(int32_t)));
  if (!p || !q || !b) {
    std::free(p);
    std::free(q);
    std::free(b);
    return -3;
  }
  // read_files (src/gramsci.F90:1342-1362): x y z w buffer, stop at end
  R.next = 0;
  double v[5];
  long long iv[5];
  for (int64_t i = 0; i < m; ++i) {
    ReadStatus s = list_read(R, 5, "rrrri", v, iv);
    if (s != R_OK) break;
    p[3 * i] = v[0];
    p[3 * i + 1] = v[1];
    p[3 * i + 2] = v[2];
    q[i] = v[3];
    b[i] = (int32_t)iv[4];
  }
  *xyz = p;
  *w = q;
  *buffer = b;
  *n = m;
  return 0;
}

int grh_read_region_gal(const char* path, double** xyz, double** w, int32_t** buffer,
                        int64_t* n_data, int64_t* n_rand) {
  Records R;
  if (!load_records(path, R)) return -1;
  const int64_t m = count_records(R);
  std::vector<double> v6((size_t)m * 4);
  std::vector<long long> g((size_t)m), b((size_t)m);
  R.next = 0;
  int64_t n = 0;
  for (int64_t i = 0; i < m; ++i) {
    double v[6];
    long long iv[6];
    ReadStatus s = list_read(R, 6, "rrrrii", v, iv);
    if (s != R_OK) break;
    for (int k = 0; k < 4; ++k) v6[(size_t)n * 4 + k] = v[k];
    g[n] = iv[4];
    b[n] = iv[5];
    n++;
  }
  double* p = static_cast<double*>(std::calloc((size_t)(3 * n + 3), sizeof(double)));
  double* q = static_cast<double*>(std::calloc((size_t)(n + 1), sizeof(double)));
  int32_t* f = static_cast<int32_t*>(std::calloc((size_t)(n + 1), sizeof(int32_t)));
  if (!p || !q || !f) {
    std::free(p);
    std::free(q);
    std::free(f);
    return -3;
  }
  int64_t nd = 0, k = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int64_t i = 0; i < n; ++i) {
      if ((g[i] != 0) != (pass == 0)) continue;
      for (int c = 0; c < 3; ++c) p[3 * k + c] = v6[(size_t)i * 4 + c];
      q[k] = v6[(size_t)i * 4 + 3];
      f[k] = (int32_t)b[i];
      k++;
      if (pass == 0) nd++;
    }
  *xyz = p;
  *w = q;
  *buffer = f;
  *n_data = nd;
  *n_rand = n - nd;
  return 0;
}

void grh_free(void* p) { std::free(p); }

void grh_normalise(double* w, int64_t n_data, int64_t n_rand) {
  double sg = 0.0, sr = 0.0;
  for (int64_t i = 0; i < n_data; ++i) sg = sg + w[i];
  for (int64_t i = n_data; i < n_data + n_rand; ++i) sr = sr + w[i];
  for (int64_t i = 0; i < n_data; ++i) w[i] = w[i] / sg;
  for (int64_t i = n_data; i < n_data + n_rand; ++i) w[i] = -1.0 * w[i] / sr;
}

void grh_radial_bins(double rmin, double rmax, int32_t nbins, int32_t logbins, double* edges) {
  for (int i = 1; i <= nbins + 1; ++i) {
    const int j = i - 1;
    // float(nbins) is exact in single precision for the allowed nbins
    if (logbins)
      edges[i - 1] = std::pow(10.0, std::log10(rmin) +
                                        (double)j * (std::log10(rmax) - std::log10(rmin)) / (double)nbins);
    else
      edges[i - 1] = rmin + (double)j * (rmax - rmin) / (double)nbins;
  }
}

void grh_format_e14_7(double v, char* out) {
  char body[32];
  if (std::isnan(v)) {
    std::snprintf(out, 15, "%14s", "NaN");
    return;
  }
  if (std::isinf(v)) {
    std::snprintf(out, 15, "%14s", v < 0 ? "-Infinity" : "Infinity");
    return;
  }
  const char sign = std::signbit(v) ? '-' : ' ';
  char digits[8];
  int e10 = 0;
  if (v == 0.0) {
    std::memcpy(digits, "0000000", 8);
  } else {
    char tmp[32];
    std::snprintf(tmp, sizeof(tmp), "%.6e", std::fabs(v));  // d.dddddde+XX, correctly rounded
    digits[0] = tmp[0];
    std::memcpy(digits + 1, tmp + 2, 6);
    digits[7] = '\0';
    e10 = std::atoi(tmp + 9) + 1;  // 0.ddddddd x 10^(e+1)
  }
  if (e10 >= -99 && e10 <= 99)
    std::snprintf(body, sizeof(body), "0.%sE%c%02d", digits, e10 < 0 ? '-' : '+', e10 < 0 ? -e10 : e10);
  else
    std::snprintf(body, sizeof(body), "0.%s%c%03d", digits, e10 < 0 ? '-' : '+', e10 < 0 ? -e10 : e10);
  char line[48];
  std::snprintf(line, sizeof(line), "%c%s", sign, body);
  std::memcpy(out, line, 14);
  out[14] = '\0';
}

namespace {

// One record of an `(n(e14.7,1x))` format: values separated by one blank;
// the trailing 1x transmits nothing (no characters follow it).
void write_record(FILE* f, const double* v, int k) {
  char s[16];
  for (int i = 0; i < k; ++i) {
    grh_format_e14_7(v[i], s);
    std::fputs(s, f);
    if (i + 1 < k) std::fputc(' ', f);
  }
  std::fputc('\n', f);
}

}  // namespace

int grh_write_2pcf(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3) {
  // query_graph_2pcf writer, src/gramsci.F90:382-397
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  std::fputs(" r1 min, r1 max, r2 min, r2 max, NN, RR, 2pcf (xi)\n", f);
  const double mu_scale = (double)(0.5f * (float)nmu);
  for (int l = 1; l <= nbins; ++l)
    for (int k = 1; k <= nmu; ++k) {
      const int idx = (l - 1) + nbins * (k - 1);
      const double v[7] = {edges[l - 1], edges[l], (double)((float)k - 1.0f) / mu_scale - 1.0,
                           (double)(float)k / mu_scale - 1.0, N2[idx], N3[idx], N2[idx] / N3[idx]};
      write_record(f, v, 7);
    }
  return std::fclose(f) == 0 ? 0 : -1;
}

int grh_write_3pcf(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3) {
  // query_graph_3pcf_all writer, src/gramsci.F90:513-543
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  const bool rsd = nmu >= 2;
  if (rsd)
    std::fputs(" r1 min, r1 max, r2 min, r2 max, r3 min, r3 max, mu min, mu max, NNN, RRR, 3pcf (zeta)\n", f);
  else
    std::fputs(" r1 min, r1 max, r2 min, r2 max, r3 min, r3 max, NNN, RRR, 3pcf (zeta)\n", f);
  const double mu_scale = (double)(0.5f * (float)nmu);
  const int ncfg = nbins * (nbins + 1) * (nbins + 2) / 6;
  int cfg = 0;
  for (int i = 1; i <= nbins; ++i)
    for (int j = i; j <= nbins; ++j)
      for (int k = j; k <= nbins; ++k) {
        cfg++;
        if (rsd) {
          for (int l = 1; l <= nmu; ++l) {
            const int idx = (cfg - 1) + ncfg * (l - 1);
            const double v[11] = {edges[i - 1], edges[i], edges[j - 1], edges[j], edges[k - 1], edges[k],
                                  (double)((float)l - 1.0f) / mu_scale / 2.0,
                                  (double)(float)l / mu_scale / 2.0, N2[idx], N3[idx],
                                  N2[idx] / N3[idx]};
            write_record(f, v, 11);
          }
        } else {
          const int idx = cfg - 1;
          const double v[9] = {edges[i - 1], edges[i], edges[j - 1], edges[j], edges[k - 1], edges[k],
                               N2[idx], N3[idx], N2[idx] / N3[idx]};
          write_record(f, v, 9);
        }
      }
  return std::fclose(f) == 0 ? 0 : -1;
}

int grh_write_4pcf(const char* path, const double* edges, int32_t nbins, const double* N2,
                   const double* N3, const double* discN, const double* discR) {
  // query_4pcf_all2 writer, src/gramsci.F90:829-858
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  std::fputs(" r1 min, r1 max, r2 min, r2 max, r3 min, r3 max, r4 min, r4 max, NNNN, RRRR, 4pcf (eta)\n", f);
  const int ncfg = nbins * (nbins + 1) * (nbins + 2) * (nbins + 3) / 24;
  const int nbin = ncfg * nbins * nbins;
  int cfg = 0;
  for (int i = 1; i <= nbins; ++i)
    for (int j = i; j <= nbins; ++j)
      for (int k = j; k <= nbins; ++k)
        for (int l = k; l <= nbins; ++l) {
          cfg++;
          for (int k1 = 1; k1 <= nbins; ++k1)
            for (int k2 = 1; k2 <= nbins; ++k2) {
              const int idx = (cfg - 1) + ncfg * ((k1 - 1) + nbins * (k2 - 1));
              auto r = [&](int t) { return discN[idx + nbin * (t - 1)] / discR[idx + nbin * (t - 1)]; };
              const double v[14] = {edges[i - 1], edges[i], edges[j - 1], edges[j], edges[k - 1],
                                    edges[k], edges[l - 1], edges[l], N2[idx], N3[idx],
                                    N2[idx] / N3[idx], r(1) * r(5), r(3) * r(4), r(2) * r(6)};
              write_record(f, v, 14);
            }
        }
  return std::fclose(f) == 0 ? 0 : -1;
}

int grh_write_equi(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3) {
  // query_graph_equilateral_triangle writer, src/gramsci.F90:451-459
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  const double mu_scale = (double)(0.5f * (float)nmu);
  for (int l = 1; l <= nbins; ++l)
    for (int k = 1; k <= nmu; ++k) {
      const int idx = (l - 1) + nbins * (k - 1);
      const double v[7] = {edges[l - 1], edges[l], (double)((float)k - 1.0f) / mu_scale / 2.0,
                           (double)(float)k / mu_scale / 2.0, N2[idx], N3[idx], N2[idx] / N3[idx]};
      write_record(f, v, 7);
    }
  return std::fclose(f) == 0 ? 0 : -1;
}

int grh_write_tetra(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                    const double* N2, const double* N3, const double* discN, const double* discR) {
  // query_graph_tetrahedron writer, src/gramsci.F90:648-660: N2(l,k,3) holds
  // the counts at k = 1 only; the disconnected combination uses (l,1,1,t)
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  const double mu_scale = (double)(0.5f * (float)nmu);
  for (int l = 1; l <= nbins; ++l)
    for (int k = 1; k <= nmu; ++k) {
      const double n2 = k == 1 ? N2[l - 1] : 0.0, n3 = k == 1 ? N3[l - 1] : 0.0;
      auto r = [&](int t) { return discN[(l - 1) + nbins * (t - 1)] / discR[(l - 1) + nbins * (t - 1)]; };
      const double v[8] = {edges[l - 1], edges[l], (double)((float)k - 1.0f) / mu_scale / 2.0,
                           (double)(float)k / mu_scale / 2.0, n2, n3, n2 / n3,
                           r(1) * r(5) + r(3) * r(4) + r(2) * r(6)};
      write_record(f, v, 8);
    }
  return std::fclose(f) == 0 ? 0 : -1;
}

}  // extern "C"

// ------------------------------------------------------------ region files --
namespace {

struct RegionPoint {
  double x[3], w;
  long long gal;
  long long region;
};

// Region boxes and memberships with the arithmetic type T (float reproduces
// the reference program; double for catalogue input).
template <typename T>
int write_regions(const std::vector<RegionPoint>& P, T rmax, T grow, int digits,
                  const std::string& prefix, int32_t* nregion) {
  long long nreg = 0;
  for (const RegionPoint& p : P) nreg = p.region > nreg ? p.region : nreg;
  for (long long j = 1; j <= nreg; ++j) {
    // minval / maxval with mask=region.eq.j (+-huge for an empty region)
    T lo[3], hi[3];
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::numeric_limits<T>::max();
      hi[c] = -std::numeric_limits<T>::max();
    }
    for (const RegionPoint& p : P)
      if (p.region == j)
        for (int c = 0; c < 3; ++c) {
          const T v = (T)p.x[c];
          lo[c] = v < lo[c] ? v : lo[c];
          hi[c] = v > hi[c] ? v : hi[c];
        }
    T lo2[3], hi2[3];
    for (int c = 0; c < 3; ++c) {
      lo2[c] = lo[c] - rmax * grow;
      hi2[c] = hi[c] + rmax * grow;
    }
    const std::string name = prefix + std::to_string(j) + ".loadnodes";
    FILE* f = std::fopen(name.c_str(), "w");
    if (!f) return -2;
    for (const RegionPoint& p : P) {
      T v[3] = {(T)p.x[0], (T)p.x[1], (T)p.x[2]};
      bool in = true, core = true;
      for (int c = 0; c < 3; ++c) {
        in = in && v[c] > lo2[c] && v[c] < hi2[c];
        core = core && v[c] >= lo[c] && v[c] <= hi[c];
      }
      if (!in) continue;
      std::fprintf(f, " %.*g %.*g %.*g %.*g %lld %d\n", digits, (double)v[0], digits, (double)v[1],
                   digits, (double)v[2], digits, (double)(T)p.w, p.gal, core ? 0 : 1);
    }
    if (std::fclose(f) != 0) return -2;
  }
  *nregion = (int32_t)nreg;
  return 0;
}

}  // namespace

extern "C" {

int grh_decompose(const char* allpoints, const char* gal, const char* ran, double rmax,
                  int32_t nsplit, const char* prefix, int32_t* nregion) {
  std::vector<RegionPoint> P;
  const std::string pre = prefix ? prefix : "";
  *nregion = 0;
  if (allpoints && allpoints[0]) {
    // src/domain_decomposition.f90:14-33: count records, then READ
    // x y z w gal aux region per record; a READ error skips the record.
    Records R;
    if (!load_records(allpoints, R)) return -1;
    R.next = 0;
    for (;;) {
      if (R.next >= R.lines.size()) break;
      std::vector<std::string> tok;
      bool slash = false;
      // one list-directed READ of 7 items
      std::vector<std::string> items;
      while (items.size() < 7 && R.next < R.lines.size()) {
        split_tokens(R.lines[R.next++], tok, slash);
        for (const std::string& t : tok)
          if (items.size() < 7) items.push_back(t);
        if (slash) break;
      }
      if (items.size() < 7) break;  // end of file inside the READ
      float x[4], aux;
      long long g, r;
      bool ok = parse_real4(items[0], x[0]) && parse_real4(items[1], x[1]) &&
                parse_real4(items[2], x[2]) && parse_real4(items[3], x[3]) &&
                parse_int(items[4], g) && parse_real4(items[5], aux) && parse_int(items[6], r);
      if (!ok) continue;
      RegionPoint p;
      for (int c = 0; c < 3; ++c) p.x[c] = x[c];
      p.w = x[3];
      p.gal = g;
      p.region = r;
      P.push_back(p);
    }
    // `real rmax` read from the command line: one rounding to single precision
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", rmax);
    float rm;
    if (!parse_real4(buf, rm)) return -3;
    return write_regions<float>(P, rm, 1.0f, 9, pre, nregion);
  }
  if (!gal || !gal[0] || nsplit < 1 || !(rmax > 0.0)) return -3;
  double *xyz = nullptr, *w = nullptr;
  int64_t nd = 0, nr = 0;
  if (grh_read_catalogue(gal, ran, &xyz, &w, &nd, &nr) != 0) return -1;
  grh_normalise(w, nd, nr);
  const int64_t n = nd + nr;
  double lo[3], hi[3];
  for (int c = 0; c < 3; ++c) {
    lo[c] = std::numeric_limits<double>::infinity();
    hi[c] = -lo[c];
  }
  for (int64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::fmin(lo[c], xyz[3 * i + c]);
      hi[c] = std::fmax(hi[c], xyz[3 * i + c]);
    }
  P.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    long long cell[3];
    for (int c = 0; c < 3; ++c) {
      const double ext = hi[c] - lo[c];
      long long k = ext > 0.0 ? (long long)std::floor((xyz[3 * i + c] - lo[c]) / ext * nsplit) : 0;
      cell[c] = k < 0 ? 0 : (k >= nsplit ? nsplit - 1 : k);
    }
    RegionPoint& p = P[(size_t)i];
    for (int c = 0; c < 3; ++c) p.x[c] = xyz[3 * i + c];
    p.w = w[i];
    p.gal = i < nd ? 1 : 0;
    p.region = 1 + cell[0] + (long long)nsplit * (cell[1] + (long long)nsplit * cell[2]);
  }
  grh_free(xyz);
  grh_free(w);
  // subcubes are disjoint, so every point is a root in exactly one region;
  // the halo is grown by 1e-9 relative so that FP64 rounding of box - rmax
  // cannot drop a neighbour closer than rmax
  return write_regions<double>(P, rmax, 1.0 + 1e-9, 17, pre, nregion);
}

int grh_resum(int32_t query, int32_t n, const char* const* inputs, const char* out) {
  if (n < 1 || query < 2 || query > 6) return -3;
  // columns after the bin columns: N2, N3, N2/N3 [, disconnected terms]
  const int ndisc = query == 4 ? 3 : (query == 6 ? 1 : 0);
  std::vector<std::string> header;
  std::vector<std::vector<std::string>> bins;  // bin tokens per row
  std::vector<double> n2, n3;
  for (int f = 0; f < n; ++f) {
    Records R;
    if (!load_records(inputs[f], R)) return -1;
    size_t row = 0;
    for (const std::string& line : R.lines) {
      std::vector<std::string> tok;
      bool slash;
      split_tokens(line, tok, slash);
      double v0;
      if (tok.empty()) continue;
      if (!parse_real(tok[0], v0)) {  // header line
        if (f == 0) header.push_back(line);
        continue;
      }
      const int nt = (int)tok.size();
      const int nbin_col = nt - 3 - ndisc;
      if (nbin_col < 1) return -3;
      std::vector<std::string> b(tok.begin(), tok.begin() + nbin_col);
      double a, c;
      if (!parse_real(tok[nbin_col], a) || !parse_real(tok[nbin_col + 1], c)) return -3;
      if (f == 0) {
        bins.push_back(b);
        n2.push_back(a);
        n3.push_back(c);
      } else {
        if (row >= bins.size() || bins[row] != b) return -3;
        n2[row] += a;
        n3[row] += c;
      }
      row++;
    }
    if (row != bins.size()) return -3;
  }
  FILE* fo = std::fopen(out, "w");
  if (!fo) return -2;
  for (const std::string& h : header) std::fprintf(fo, "%s\n", h.c_str());
  for (size_t r = 0; r < bins.size(); ++r) {
    std::vector<double> v;
    for (const std::string& t : bins[r]) {
      double x;
      parse_real(t, x);
      v.push_back(x);
    }
    v.push_back(n2[r]);
    v.push_back(n3[r]);
    v.push_back(n2[r] / n3[r]);
    for (int k = 0; k < ndisc; ++k) v.push_back(std::numeric_limits<double>::quiet_NaN());
    write_record(fo, v.data(), (int)v.size());
  }
  return std::fclose(fo) == 0 ? 0 : -2;
}

}  // extern "C"
