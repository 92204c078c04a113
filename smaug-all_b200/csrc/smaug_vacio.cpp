// smaug_vacio.cpp -- VAC configuration files, the reference's on-disk format
// for initial conditions and snapshots (host only, no CUDA).
//
// ascii (.ini), as readasciivacconfig reads it (src/readwrite.c:982-1112):
//   line 1  a name
//   line 2  it  t  ndim  neqpar  nw
//   line 3  n_1 .. n_ndim
//   line 4  neqpar equation parameters (gamma, eta, g_1 .. g_ndim, ...)
//   line 5  variable names
//   then one line per cell, x fastest: ndim positions, nw values.
// binary (.out), as writevacconfig writes it (src/readwrite.c:160-368):
//   79-byte name | int32 it | float64 t | int32 ndim, neqpar, nw |
//   int32 n[ndim] | float64 eqpar[neqpar] | 79-byte names |
//   ndim position fields then nw state fields, each N float64 in x-fastest
//   order | one '\n' byte.
// In memory, positions are ndim arrays of N doubles and states nw arrays of N
// doubles (the wd[pos*] and wmod layouts), N = n_1 * .. * n_ndim.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smaug_b200.h"

namespace {

thread_local std::string g_vac_err;

int vfail(const std::string &m) {
  g_vac_err = m;
  return SMAUG_ERR_ARG;
}

struct File {
  FILE *f = nullptr;
  explicit File(FILE *p) : f(p) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

bool read_line(FILE *f, std::string &out) {
  out.clear();
  int ch;
  while ((ch = std::fgetc(f)) != EOF && ch != '\n') out.push_back((char)ch);
  if (ch == EOF && out.empty()) return false;
  while (!out.empty() && (out.back() == '\r' || out.back() == ' ')) out.pop_back();
  return true;
}

void copy_text(char *dst, const std::string &s) {
  std::memset(dst, 0, 80);
  std::strncpy(dst, s.c_str(), 79);
}

std::vector<double> numbers(const std::string &s) {
  std::vector<double> v;
  const char *p = s.c_str();
  char *end = nullptr;
  while (true) {
    errno = 0;
    const double x = std::strtod(p, &end);
    if (end == p) break;
    v.push_back(x);
    p = end;
  }
  return v;
}

long long cells(const smaug_vac_header *h) {
  long long N = 1;
  for (int d = 0; d < h->ndim; ++d) N *= h->n[d];
  return N;
}

const char *check_header(const smaug_vac_header *h) {
  if (h->ndim < 1 || h->ndim > 3) return "ndim must be 1..3";
  if (h->nw < 1 || h->nw > 64) return "nw must be 1..64";
  if (h->neqpar < 0 || h->neqpar > 16) return "neqpar must be 0..16";
  for (int d = 0; d < h->ndim; ++d)
    if (h->n[d] < 1 || h->n[d] > (1 << 24)) return "grid size out of range";
  return nullptr;
}

const char *check_buffers(const smaug_vac_header *h, const double *pos, size_t pos_count, const double *w,
                          size_t w_count) {
  const long long N = cells(h);
  if (pos && pos_count != (size_t)h->ndim * (size_t)N) return "positions must hold ndim * N doubles";
  if (w && w_count != (size_t)h->nw * (size_t)N) return "state must hold nw * N doubles";
  return nullptr;
}

}  // namespace

extern "C" {

const char *smaug_vac_last_error(void) { return g_vac_err.c_str(); }

int smaug_vac_read_ascii(const char *path, smaug_vac_header *hdr, double *pos, size_t pos_count, double *w,
                         size_t w_count) {
  if (!path || !hdr) return vfail("null argument");
  File f(std::fopen(path, "r"));
  if (!f.f) return vfail(std::string("cannot open ") + path);
  std::memset(hdr, 0, sizeof(*hdr));
  std::string line;
  if (!read_line(f.f, line)) return vfail("missing name line");
  copy_text(hdr->name, line);
  if (!read_line(f.f, line)) return vfail("missing line 2 (it t ndim neqpar nw)");
  std::vector<double> v = numbers(line);
  if (v.size() < 5) return vfail("line 2 needs it t ndim neqpar nw");
  hdr->it = (int)v[0];
  hdr->t = v[1];
  hdr->ndim = (int)v[2];
  hdr->neqpar = (int)v[3];
  hdr->nw = (int)v[4];
  if (!read_line(f.f, line)) return vfail("missing grid size line");
  v = numbers(line);
  if ((int)v.size() < hdr->ndim || hdr->ndim < 1 || hdr->ndim > 3) return vfail("grid size line does not match ndim");
  for (int d = 0; d < hdr->ndim; ++d) hdr->n[d] = (int)v[d];
  for (int d = hdr->ndim; d < 3; ++d) hdr->n[d] = 1;
  if (!read_line(f.f, line)) return vfail("missing equation parameter line");
  v = numbers(line);
  if ((int)v.size() < hdr->neqpar || hdr->neqpar > 16) return vfail("equation parameter line is short");
  for (int k = 0; k < hdr->neqpar; ++k) hdr->eqpar[k] = v[k];
  if (!read_line(f.f, line)) return vfail("missing variable names line");
  copy_text(hdr->names, line);
  if (const char *m = check_header(hdr)) return vfail(m);
  if (!pos && !w) return SMAUG_OK;  // header only
  if (const char *m = check_buffers(hdr, pos, pos_count, w, w_count)) return vfail(m);
  const long long N = cells(hdr);
  const int nc = hdr->ndim + hdr->nw;
  std::vector<double> row(nc);
  for (long long i = 0; i < N; ++i) {
    for (int k = 0; k < nc; ++k) {
      if (std::fscanf(f.f, "%lf", &row[k]) != 1)
        return vfail("cell " + std::to_string(i) + ": expected " + std::to_string(nc) + " numbers");
    }
    if (pos)
      for (int d = 0; d < hdr->ndim; ++d) pos[(size_t)d * N + i] = row[d];
    if (w)
      for (int k = 0; k < hdr->nw; ++k) w[(size_t)k * N + i] = row[hdr->ndim + k];
  }
  return SMAUG_OK;
}

int smaug_vac_write_ascii(const char *path, const smaug_vac_header *hdr, const double *pos, const double *w) {
  if (!path || !hdr || !pos || !w) return vfail("null argument");
  if (const char *m = check_header(hdr)) return vfail(m);
  File f(std::fopen(path, "w"));
  if (!f.f) return vfail(std::string("cannot create ") + path);
  std::fprintf(f.f, "%.79s\n", hdr->name);
  std::fprintf(f.f, "%7d %.17E %d %d %d\n", hdr->it, hdr->t, hdr->ndim, hdr->neqpar, hdr->nw);
  for (int d = 0; d < hdr->ndim; ++d) std::fprintf(f.f, " %d", hdr->n[d]);
  std::fprintf(f.f, "\n");
  for (int k = 0; k < hdr->neqpar; ++k) std::fprintf(f.f, " %.17E", hdr->eqpar[k]);
  std::fprintf(f.f, "\n%.79s\n", hdr->names);
  const long long N = cells(hdr);
  for (long long i = 0; i < N; ++i) {
    for (int d = 0; d < hdr->ndim; ++d) std::fprintf(f.f, " %.17E", pos[(size_t)d * N + i]);
    for (int k = 0; k < hdr->nw; ++k) std::fprintf(f.f, " %.17E", w[(size_t)k * N + i]);
    std::fprintf(f.f, "\n");
  }
  if (std::ferror(f.f)) return vfail("write error");
  return SMAUG_OK;
}

int smaug_vac_write_binary(const char *path, const smaug_vac_header *hdr, const double *pos, const double *w) {
  if (!path || !hdr || !pos || !w) return vfail("null argument");
  if (const char *m = check_header(hdr)) return vfail(m);
  File f(std::fopen(path, "wb"));
  if (!f.f) return vfail(std::string("cannot create ") + path);
  char text[80];
  std::memset(text, ' ', 79);
  std::memcpy(text, hdr->name, std::min<size_t>(std::strlen(hdr->name), 79));
  std::fwrite(text, 1, 79, f.f);
  const int it = hdr->it;
  const double t = hdr->t;
  const int dims[3] = {hdr->ndim, hdr->neqpar, hdr->nw};
  std::fwrite(&it, sizeof(int), 1, f.f);
  std::fwrite(&t, sizeof(double), 1, f.f);
  std::fwrite(dims, sizeof(int), 3, f.f);
  std::fwrite(hdr->n, sizeof(int), hdr->ndim, f.f);
  std::fwrite(hdr->eqpar, sizeof(double), hdr->neqpar, f.f);
  std::memset(text, ' ', 79);
  std::memcpy(text, hdr->names, std::min<size_t>(std::strlen(hdr->names), 79));
  std::fwrite(text, 1, 79, f.f);
  const long long N = cells(hdr);
  std::fwrite(pos, sizeof(double), (size_t)hdr->ndim * N, f.f);
  std::fwrite(w, sizeof(double), (size_t)hdr->nw * N, f.f);
  std::fputc('\n', f.f);
  if (std::ferror(f.f)) return vfail("write error");
  return SMAUG_OK;
}

int smaug_vac_read_binary(const char *path, smaug_vac_header *hdr, double *pos, size_t pos_count, double *w,
                          size_t w_count) {
  if (!path || !hdr) return vfail("null argument");
  File f(std::fopen(path, "rb"));
  if (!f.f) return vfail(std::string("cannot open ") + path);
  std::memset(hdr, 0, sizeof(*hdr));
  char text[80] = {0};
  int dims[3];
  if (std::fread(text, 1, 79, f.f) != 79) return vfail("short file: name");
  std::string s(text, 79);
  while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
  copy_text(hdr->name, s);
  if (std::fread(&hdr->it, sizeof(int), 1, f.f) != 1 || std::fread(&hdr->t, sizeof(double), 1, f.f) != 1 ||
      std::fread(dims, sizeof(int), 3, f.f) != 3)
    return vfail("short file: it, t, dimensions");
  hdr->ndim = dims[0];
  hdr->neqpar = dims[1];
  hdr->nw = dims[2];
  if (hdr->ndim < 1 || hdr->ndim > 3 || hdr->neqpar < 0 || hdr->neqpar > 16) return vfail("bad dimensions");
  if (std::fread(hdr->n, sizeof(int), hdr->ndim, f.f) != (size_t)hdr->ndim) return vfail("short file: grid size");
  for (int d = hdr->ndim; d < 3; ++d) hdr->n[d] = 1;
  if (std::fread(hdr->eqpar, sizeof(double), hdr->neqpar, f.f) != (size_t)hdr->neqpar)
    return vfail("short file: equation parameters");
  std::memset(text, 0, sizeof(text));
  if (std::fread(text, 1, 79, f.f) != 79) return vfail("short file: names");
  s.assign(text, 79);
  while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
  copy_text(hdr->names, s);
  if (const char *m = check_header(hdr)) return vfail(m);
  if (!pos && !w) return SMAUG_OK;
  if (const char *m = check_buffers(hdr, pos, pos_count, w, w_count)) return vfail(m);
  const long long N = cells(hdr);
  std::vector<double> tmp;
  double *pd = pos;
  if (!pd) {
    tmp.resize((size_t)hdr->ndim * N);
    pd = tmp.data();
  }
  if (std::fread(pd, sizeof(double), (size_t)hdr->ndim * N, f.f) != (size_t)hdr->ndim * N)
    return vfail("short file: positions");
  if (w && std::fread(w, sizeof(double), (size_t)hdr->nw * N, f.f) != (size_t)hdr->nw * N)
    return vfail("short file: state");
  return SMAUG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// smaug_initgrid: the metric from cell positions, as the reference's initgrid
// (init.cu:1118-1670) derives it from wd[pos1..] (the positions of every cell,
// ghosts included, as init_parallel sets them or a VAC file holds them):
//   * the positions go into a copy padded by one layer on each side of every
//     dimension (2-D: x and y only);
//   * dimension by dimension, every position component is extrapolated
//     linearly over the two outermost layers and the pad of each side,
//     q(ix) = (1 + |ixe - ix|) q(ixe) - |ixe - ix| q(ixf) with ixe, ixf the
//     first two inner cells of that side;
//   * delx_d = (x_d[c + 1] - x_d[c - 1]) / 2 along d, where 0 becomes dx[d].
// Built without FMA contraction (the build passes -ffp-contract=off), so the
// metric has the reference's bits.
// ---------------------------------------------------------------------------
extern "C" int smaug_initgrid(int ndim, const int *n, const double *pos, const double *dx, double *delx) {
  if (ndim != 2 && ndim != 3) return vfail("ndim must be 2 or 3");
  if (!n || !pos || !dx || !delx) return vfail("null argument");
  const int D = ndim;
  int nn[3] = {n[0], n[1], D == 3 ? n[2] : 1};
  for (int d = 0; d < D; ++d)
    if (nn[d] < 5 || nn[d] > (1 << 20)) return vfail("each dimension needs 5..2^20 cells including ghosts");
  const long long N = (long long)nn[0] * nn[1] * nn[2];
  const int pn[3] = {nn[0] + 2, nn[1] + 2, D == 3 ? nn[2] + 2 : 1};
  const size_t Np = (size_t)pn[0] * pn[1] * pn[2];
  const size_t ps[3] = {1, (size_t)pn[0], (size_t)pn[0] * pn[1]};
  const int off3 = D == 3 ? 1 : 0;
  std::vector<std::vector<double>> T(D, std::vector<double>(Np, 0.0));
  for (int d1 = 0; d1 < D; ++d1) {
    const double *src = pos + (size_t)d1 * N;
    for (int k = 0; k < nn[2]; ++k)
      for (int j = 0; j < nn[1]; ++j)
        for (int i = 0; i < nn[0]; ++i)
          T[d1][(size_t)(i + 1) + ps[1] * (j + 1) + ps[2] * (k + off3)] = src[i + (size_t)nn[0] * (j + (size_t)nn[1] * k)];
  }
  for (int d = 0; d < D; ++d) {
    const int m = nn[d];
    // the other two axes of the padded copy (full padded ranges)
    const int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2;
    const int sides[2][4] = {{m - 1, m + 1, m - 2, m - 3}, {0, 2, 3, 4}};
    for (const auto &sd : sides)
      for (int d1 = 0; d1 < D; ++d1)
        for (int ix = sd[0]; ix <= sd[1]; ++ix) {
          const double a = (double)std::abs(sd[2] - ix);
          for (int u = 0; u < pn[a2]; ++u)
            for (int v = 0; v < pn[a1]; ++v) {
              const size_t base = ps[a1] * v + ps[a2] * u;
              double *t = T[d1].data();
              t[base + ps[d] * ix] = (1.0 + a) * t[base + ps[d] * sd[2]] - a * t[base + ps[d] * sd[3]];
            }
        }
  }
  for (int d = 0; d < D; ++d) {
    const double *t = T[d].data();
    double *out = delx + (size_t)d * N;
    for (int k = 0; k < nn[2]; ++k)
      for (int j = 0; j < nn[1]; ++j)
        for (int i = 0; i < nn[0]; ++i) {
          const size_t c = (size_t)(i + 1) + ps[1] * (j + 1) + ps[2] * (k + off3);
          const double v = 0.5 * (t[c + ps[d]] - t[c - ps[d]]);
          out[i + (size_t)nn[0] * (j + (size_t)nn[1] * k)] = v == 0.0 ? dx[d] : v;
        }
  }
  return SMAUG_OK;
}
