// MatrixMarket reader/writer of libcgb200 (host code).
//
// The reader reproduces MatrixCOO::MatrixCOO (Matrix.cpp:13-111) entry for
// entry -- same banner checks and messages, same comment skipping, symmetric
// off-diagonal entries mirrored into the slot right after the entry, nz taken
// as 2*nz - N for symmetric files -- but parses the entry lines on several
// threads: the file is read whole, split at line boundaries, and each thread
// parses its lines with std::from_chars (correctly rounded, like the strtod
// behind the reference's stringstream). A prefix sum over per-chunk counts of
// off-diagonal lines gives each line its output slot.
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "cgx.h"

// Sets the message returned by cgx_last_error() (defined in api.cu).
void cgx_internal_set_error(const std::string &msg);

namespace {

cgx_status io_fail(const std::string &m) {
  cgx_internal_set_error(m);
  return CGX_ERROR_IO;
}

int worker_count(size_t work) {
  unsigned hc = std::thread::hardware_concurrency();
  int n = (int)std::max(1u, std::min(hc, 64u));
  size_t per = 1 << 20;  // at least ~1 MiB of text per thread
  n = (int)std::min<size_t>((size_t)n, std::max<size_t>(1, work / per));
  return n;
}

// Next line [b, e) starting at p; returns the start of the following line.
const char *line_end(const char *p, const char *end) {
  const char *q = (const char *)std::memchr(p, '\n', (size_t)(end - p));
  return q ? q : end;
}

const char *skip_ws(const char *p, const char *e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
  return p;
}

struct Entry {
  int r, c;
  double v;
};

// Parses "row col value" (1-based). Returns false on malformed input.
bool parse_entry(const char *p, const char *e, Entry &out) {
  p = skip_ws(p, e);
  auto r1 = std::from_chars(p, e, out.r);
  if (r1.ec != std::errc()) return false;
  p = skip_ws(r1.ptr, e);
  auto r2 = std::from_chars(p, e, out.c);
  if (r2.ec != std::errc()) return false;
  p = skip_ws(r2.ptr, e);
  if (p < e && *p == '+') p++;  // from_chars rejects a leading '+'
  auto r3 = std::from_chars(p, e, out.v);
  if (r3.ec != std::errc()) return false;
  return true;
}

}  // namespace

extern "C" void cgx_free(void *p) { std::free(p); }

extern "C" cgx_status cgx_mtx_read(const char *path, int *Nout, int *nzOut,
                                   int **Iout, int **Jout, double **Vout) {
  if (!path || !Nout || !nzOut || !Iout || !Jout || !Vout) {
    cgx_internal_set_error("NULL argument");
    return CGX_ERROR_INVALID_ARGUMENT;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) return io_fail("Can't open file with matrix!");
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<char> buf((size_t)std::max(sz, 0L) + 1);
  size_t got = sz > 0 ? std::fread(buf.data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  buf[got] = 0;
  const char *p = buf.data(), *end = buf.data() + got;

  // Banner (Matrix.cpp:25-57).
  const char *le = line_end(p, end);
  {
    std::string line(p, le);
    char w[5][64] = {{0}};
    std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2],
                w[3], w[4]);
    for (int k = 1; k < 5; k++)
      for (char *c = w[k]; *c; ++c) *c = (char)std::tolower((unsigned char)*c);
    if (std::strcmp(w[0], "%%MatrixMarket") || std::strcmp(w[1], "matrix") ||
        std::strcmp(w[2], "coordinate") || std::strcmp(w[3], "real"))
      return io_fail("Only supporting real matrices in coordinate format!");
    if (std::strcmp(w[4], "symmetric") && std::strcmp(w[4], "general"))
      return io_fail("Only supporting general or symmetric matrices!");
    *nzOut = 0;
    p = le < end ? le + 1 : end;
    bool symmetric = !std::strcmp(w[4], "symmetric");

    // Comments and empty lines (Matrix.cpp:50-53).
    for (;;) {
      if (p >= end)
        return io_fail("An exception occurred while reading the matrix!");
      le = line_end(p, end);
      if (le > p && *p != '%') break;
      p = le < end ? le + 1 : end;
    }
    int M = 0, N = 0, nzFile = 0;
    {
      std::string dims(p, le);
      if (std::sscanf(dims.c_str(), "%d %d %d", &M, &N, &nzFile) != 3)
        return io_fail("An exception occurred while reading the matrix!");
    }
    if (N != M) return io_fail("Need a square matrix!");
    if (N <= 0 || nzFile < 0)
      return io_fail("An exception occurred while reading the matrix!");
    p = le < end ? le + 1 : end;

    // Entry lines: the first nzFile lines after the size line. (The
    // reference reads exactly as many entries as it has slots; files that
    // follow the format have exactly nzFile entry lines.)
    std::vector<const char *> starts;
    starts.reserve((size_t)nzFile + 1);
    {
      const char *q = p;
      for (int i = 0; i < nzFile; i++) {
        if (q >= end)
          return io_fail("An exception occurred while reading the matrix!");
        starts.push_back(q);
        const char *e2 = line_end(q, end);
        q = e2 < end ? e2 + 1 : end;
      }
      starts.push_back(q);
    }

    const long long slots = symmetric ? 2LL * nzFile - N : (long long)nzFile;
    if (slots < 0 || slots > 0x7fffffffLL)
      return io_fail("An exception occurred while reading the matrix!");
    const int nz = (int)slots;
    int *I = (int *)std::malloc(sizeof(int) * (size_t)std::max(nz, 1));
    int *J = (int *)std::malloc(sizeof(int) * (size_t)std::max(nz, 1));
    double *V = (double *)std::malloc(sizeof(double) * (size_t)std::max(nz, 1));
    if (!I || !J || !V) {
      std::free(I);
      std::free(J);
      std::free(V);
      return io_fail("out of host memory reading the matrix");
    }

    const int T = worker_count((size_t)(end - p));
    std::vector<int> lo(T + 1);
    for (int t = 0; t <= T; t++) lo[t] = (int)((long long)nzFile * t / T);
    std::vector<long long> offdiag(T, 0);
    std::vector<int> bad(T, 0);
    std::vector<Entry> parsed((size_t)std::max(nzFile, 1));

    auto pass1 = [&](int t) {
      long long od = 0;
      for (int i = lo[t]; i < lo[t + 1]; i++) {
        const char *b = starts[i];
        const char *e2 = line_end(b, end);
        Entry en;
        if (!parse_entry(b, e2, en) || en.r < 1 || en.r > N || en.c < 1 ||
            en.c > N) {
          bad[t] = 1;
          return;
        }
        parsed[i] = en;
        if (symmetric && en.r != en.c) od++;
      }
      offdiag[t] = od;
    };
    {
      std::vector<std::thread> th;
      for (int t = 1; t < T; t++) th.emplace_back(pass1, t);
      pass1(0);
      for (auto &x : th) x.join();
    }
    bool anyBad = false;
    for (int t = 0; t < T; t++) anyBad |= bad[t] != 0;
    long long totalSlots = 0;
    std::vector<long long> base(T + 1, 0);
    for (int t = 0; t < T; t++) {
      base[t] = (long long)lo[t] + [&] {
        long long s = 0;
        for (int u = 0; u < t; u++) s += offdiag[u];
        return s;
      }();
    }
    for (int t = 0; t < T; t++) totalSlots += (lo[t + 1] - lo[t]) + offdiag[t];
    // The reference assumes every diagonal entry is present in a symmetric
    // file; otherwise its loop runs past the entries (undefined behaviour).
    if (anyBad || totalSlots != slots) {
      std::free(I);
      std::free(J);
      std::free(V);
      return io_fail(anyBad
                         ? "An exception occurred while reading the matrix!"
                         : "symmetric matrix without all diagonal entries");
    }
    auto pass2 = [&](int t) {
      long long s = base[t];
      for (int i = lo[t]; i < lo[t + 1]; i++) {
        const Entry &en = parsed[i];
        I[s] = en.r - 1;
        J[s] = en.c - 1;
        V[s] = en.v;
        s++;
        if (symmetric && en.r != en.c) {
          I[s] = en.c - 1;
          J[s] = en.r - 1;
          V[s] = en.v;
          s++;
        }
      }
    };
    {
      std::vector<std::thread> th;
      for (int t = 1; t < T; t++) th.emplace_back(pass2, t);
      pass2(0);
      for (auto &x : th) x.join();
    }
    *Nout = N;
    *nzOut = nz;
    *Iout = I;
    *Jout = J;
    *Vout = V;
  }
  return CGX_SUCCESS;
}

extern "C" cgx_status cgx_mtx_write_symmetric_crs(const char *path, int N,
                                                  const int *ptr,
                                                  const int *index,
                                                  const double *value) {
  if (!path || N <= 0 || !ptr || (ptr[N] > 0 && (!index || !value))) {
    cgx_internal_set_error("bad arguments");
    return CGX_ERROR_INVALID_ARGUMENT;
  }
  // Count the lower triangle.
  long long lower = 0;
  for (int i = 0; i < N; i++)
    for (int j = ptr[i]; j < ptr[i + 1]; j++)
      if (index[j] <= i) lower++;
  const int T = worker_count((size_t)ptr[N] * 24);
  std::vector<std::string> out(T);
  auto work = [&](int t) {
    const int r0 = (int)((long long)N * t / T), r1 = (int)((long long)N * (t + 1) / T);
    std::string &s = out[t];
    s.reserve((size_t)(ptr[r1] - ptr[r0]) * 20);
    char line[96];
    for (int i = r0; i < r1; i++)
      for (int j = ptr[i]; j < ptr[i + 1]; j++) {
        if (index[j] > i) continue;
        int n = std::snprintf(line, sizeof(line), "%d %d %.17g\n", i + 1,
                              index[j] + 1, value[j]);
        s.append(line, (size_t)n);
      }
  };
  {
    std::vector<std::thread> th;
    for (int t = 1; t < T; t++) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) return io_fail(std::string("cannot write ") + path);
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n");
  std::fprintf(f, "%d %d %lld\n", N, N, lower);
  for (auto &s : out) std::fwrite(s.data(), 1, s.size(), f);
  std::fclose(f);
  return CGX_SUCCESS;
}
