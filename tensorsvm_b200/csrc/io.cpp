// Host I/O of the training path: the LIBSVM text reader, the model-file writer and reader.
//
// The reference reads its training file with two single-threaded strtok/strtod passes
// (libsvmread, tensorsvm-train.cu:1162-1278) and writes the model with one fprintf per feature
// (writemodel, tensorsvm-train.cu:273-417); at a million rows both take seconds, longer than
// the GPU solve.  Here the file is mapped, split at line boundaries into one chunk per thread,
// and each thread parses its chunk in one pass over each token: plain decimal numbers by an
// exact fast path, anything else by std::from_chars (exact, no locale), so every value is the
// double strtod would give, then rounded to float as the reference does.  The dense matrix
// is then filled chunk by chunk.  The writer formats the support-vector
// lines in parallel chunks (6 fixed decimals, exactly the reference's "%7f", whose width never
// pads since every value prints at least 8 characters: std::to_chars for the coefficients, an
// exact integer rounding for the float features)
// and writes the chunks in order, so the file is byte-identical to a sequential writer's.
//
// Reader semantics kept from the reference: tokens separated by blanks, a label then
// index:value pairs with strictly increasing indices; indices are shifted by the smallest
// index seen (1 for 1-based files); -scale256 divides every value by 256.  Differences, each
// an error the reference ignores: a malformed or empty line is reported (its 1-based number)
// and nothing is returned, where the reference prints a message and trains on what it has
// read; a 0-based file gets max index + 1 columns (the reference allocates max index and
// writes one past the row).
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <charconv>
#include <string>
#include <thread>
#include <vector>

#include "tensorsvm.h"
#include "trace.h"

namespace {

int pick_threads(int requested) {
  int hw = (int)std::thread::hardware_concurrency();
  if (hw < 1) hw = 1;
  int t = requested > 0 ? requested : hw;
  return std::min(t, 256);
}

template <class F>
void parallel_for(int nt, F &&fn) {
  if (nt <= 1) {
    fn(0);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t) th.emplace_back(fn, t);
  for (auto &x : th) x.join();
}

inline bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// The training file, mapped read-only (the parsing threads fault its pages in, each in its own
// chunk); a file that cannot be mapped is read into memory instead.  As with any mapping, a
// file truncated by another process while it is being parsed raises SIGBUS.
class FileView {
 public:
  ~FileView() {
    if (map_) munmap(map_, size_);
  }
  bool open(const char *path) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) != 0) {
      close(fd);
      return false;
    }
    size_ = (size_t)st.st_size;
    if (size_ > 0) {
      void *m = mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m != MAP_FAILED) {
        map_ = m;
        data_ = static_cast<const char *>(m);
      } else {
        copy_.resize(size_);
        size_t got = 0;
        while (got < size_) {
          const ssize_t r = read(fd, &copy_[got], size_ - got);
          if (r <= 0) break;
          got += (size_t)r;
        }
        if (got != size_) {
          close(fd);
          return false;
        }
        data_ = copy_.data();
      }
    }
    close(fd);
    return true;
  }
  const char *data() const { return data_; }
  size_t size() const { return size_; }

 private:
  void *map_ = nullptr;
  const char *data_ = "";
  size_t size_ = 0;
  std::string copy_;
};

// strtod-like number: an optional '+' (from_chars takes only '-'), then from_chars.
template <class T>
bool parse_num(const char *b, const char *e, T &v) {
  if (b < e && *b == '+') ++b;
  if (b >= e) return false;
  auto r = std::from_chars(b, e, v);
  return r.ec == std::errc() && r.ptr == e;
}

// Exact decimal -> double for the common number form [+-]digits[.digits][(e|E)[+-]digits] with
// at most 19 digits, an integer part below 2^53 and a decimal exponent within +-22: the integer
// and the power of ten are exact doubles, so one IEEE multiplication or division rounds the
// value correctly, giving the double std::from_chars (and strtod) give (Clinger's fast path,
// PLDI 1990).  Scans from p and returns the end of the number, or nullptr when the text there
// is not of that form (the caller then applies the general token rules).
constexpr double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                               1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                               1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

inline bool is_digit(char c) { return (unsigned)(c - '0') < 10u; }

const char *scan_decimal(const char *p, const char *e, double &out) {
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) {
    neg = *p == '-';
    ++p;
  }
  uint64_t m = 0;
  int nd = 0, frac = 0;
  while (p < e && is_digit(*p)) {
    m = m * 10 + (uint64_t)(*p - '0');
    ++p;
    if (++nd > 19) return nullptr;
  }
  if (nd == 0) return nullptr;
  if (p < e && *p == '.') {
    ++p;
    if (p == e || !is_digit(*p)) return nullptr;
    while (p < e && is_digit(*p)) {
      m = m * 10 + (uint64_t)(*p - '0');
      ++p;
      ++frac;
      if (++nd > 19) return nullptr;
    }
  }
  int ex = 0;
  if (p < e && (*p == 'e' || *p == 'E')) {
    ++p;
    bool eneg = false;
    if (p < e && (*p == '+' || *p == '-')) {
      eneg = *p == '-';
      ++p;
    }
    int nde = 0;
    while (p < e && is_digit(*p)) {
      ex = ex * 10 + (*p - '0');
      ++p;
      if (++nde > 4) return nullptr;
    }
    if (nde == 0) return nullptr;
    if (eneg) ex = -ex;
  }
  if (m > (1ull << 53)) return nullptr;
  const int e10 = ex - frac;
  if (e10 > 22 || e10 < -22) return nullptr;
  double v = (double)m;
  v = e10 >= 0 ? v * kPow10[e10] : v / kPow10[-e10];
  out = neg ? -v : v;
  return p;
}

// A number token [b, first blank or eol): the fast scan when it covers the whole token, else
// parse_num on the token.  *end receives the token's end.
inline bool parse_token(const char *b, const char *eol, double &v, const char **end) {
  const char *r = scan_decimal(b, eol, v);
  if (r && (r == eol || is_blank(*r))) {
    *end = r;
    return true;
  }
  const char *t = b;
  while (t < eol && !is_blank(*t)) ++t;
  *end = t;
  return parse_num(b, t, v);
}

// A number occupying exactly [b, e), by the fast scan or parse_num.
inline bool parse_value(const char *b, const char *e, double &v) {
  const char *r = scan_decimal(b, e, v);
  return r == e || parse_num(b, e, v);
}

// index:value pair starting at q (not blank): the index as plain digits up to the colon, else
// the general rule (the token up to the first ':' or blank must parse as an integer).
inline bool parse_index(const char *q, const char *eol, int64_t &index, const char **colon) {
  const char *p = q;
  int64_t v = 0;
  int nd = 0;
  while (p < eol && is_digit(*p) && nd < 18) {
    v = v * 10 + (*p - '0');
    ++p;
    ++nd;
  }
  if (nd > 0 && p < eol && *p == ':') {
    index = v;
    *colon = p;
    return true;
  }
  p = q;
  while (p < eol && *p != ':' && !is_blank(*p)) ++p;
  *colon = p;
  if (p == eol || *p != ':') return false;
  return parse_num(q, p, index);
}

struct Chunk {
  const char *begin = nullptr, *end = nullptr;
  std::vector<float> labels;
  std::vector<int64_t> row_ptr{0};
  std::vector<int64_t> idx;
  std::vector<float> val;
  int64_t min_index = 1, max_index = 0;
  int64_t bad_local = -1;   // 0-based line within the chunk of the first malformed line
  int64_t lines = 0;
};

void parse_chunk(Chunk &c, bool scale256) {
  const char *p = c.begin;
  int64_t line = 0;
  while (p < c.end) {
    const char *eol = static_cast<const char *>(memchr(p, '\n', (size_t)(c.end - p)));
    if (!eol) eol = c.end;
    const char *q = p;
    while (q < eol && is_blank(*q)) ++q;
    if (q == eol) {   // empty line
      c.bad_local = line;
      return;
    }
    double lab;
    const char *t;
    if (!parse_token(q, eol, lab, &t)) {
      c.bad_local = line;
      return;
    }
    int64_t prev = -1;
    q = t;
    while (true) {
      while (q < eol && is_blank(*q)) ++q;
      if (q == eol) break;
      const char *colon;
      int64_t index;
      if (!parse_index(q, eol, index, &colon) || index <= prev || index < 0) {
        c.bad_local = line;
        return;
      }
      double v;
      const char *ve;
      if (!parse_token(colon + 1, eol, v, &ve)) {
        c.bad_local = line;
        return;
      }
      float fv = (float)v;
      if (scale256) fv /= 256;
      prev = index;
      c.idx.push_back(index);
      c.val.push_back(fv);
      c.min_index = std::min(c.min_index, index);
      c.max_index = std::max(c.max_index, index);
      q = ve;
    }
    c.labels.push_back((float)lab);
    c.row_ptr.push_back((int64_t)c.idx.size());
    ++line;
    p = eol < c.end ? eol + 1 : c.end;
  }
  c.lines = line;
}

// "%7f" digits of v (fixed, 6 decimals)
inline void put_fixed6(std::string &s, double v) {
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::fixed, 6);
  s.append(buf, r.ptr);
}

inline void put_int(std::string &s, int64_t v) {
  char buf[24];
  auto r = std::to_chars(buf, buf + sizeof buf, v);
  s.append(buf, r.ptr);
}

// "%7f" digits of a float, without the general conversion: x = m 2^e with |m| < 2^24, so
// x 10^6 = m 15625 2^(e+6) has at most 38 significant bits and is exact in double; rounding it
// to an integer to nearest, ties to even (as printf rounds the exact value) gives the six
// decimals.  The sign is x's, so a negative value that rounds to zero prints "-0.000000" as
// printf does.  Values of 9e9 and above, infinities and NaN take put_fixed6.
inline void put_fixed6_float(std::string &s, float x) {
  const double t = (double)x * 1e6;
  if (!(fabs(t) < 9.0e15)) {
    put_fixed6(s, (double)x);
    return;
  }
  const uint64_t q = (uint64_t)fabs(nearbyint(t));
  if (signbit(x)) s += '-';
  put_int(s, (int64_t)(q / 1000000));
  char frac[6];
  uint64_t f = q % 1000000;
  for (int i = 5; i >= 0; --i) {
    frac[i] = (char)('0' + f % 10);
    f /= 10;
  }
  s += '.';
  s.append(frac, 6);
}

// Support-vector lines of a model file ("coef idx:val ..."), parsed per chunk of lines as the
// training file is: a line is trimmed of trailing '\r' and ' ', empty lines are skipped, the
// coefficient is the first token, and each later token is "idx:val" with idx >= 1.
struct SvChunk {
  const char *begin = nullptr, *end = nullptr;
  std::vector<double> coef;
  std::vector<int64_t> row_ptr{0};
  std::vector<int> idx;
  std::vector<float> val;
  int maxi = 0;
  bool bad = false;
};

void parse_sv_chunk(SvChunk &c) {
  const char *p = c.begin;
  while (p < c.end) {
    const char *eol = static_cast<const char *>(memchr(p, '\n', (size_t)(c.end - p)));
    if (!eol) eol = c.end;
    const char *e = eol;
    while (e > p && (e[-1] == '\r' || e[-1] == ' ')) --e;
    const char *q = p;
    p = eol < c.end ? eol + 1 : c.end;
    if (q == e) continue;
    const char *t = q;
    while (t < e && !is_blank(*t)) ++t;
    double cv;
    if (!parse_value(q, t, cv)) {
      c.bad = true;
      return;
    }
    q = t;
    while (true) {
      while (q < e && is_blank(*q)) ++q;
      if (q >= e) break;
      const char *colon = q;
      while (colon < e && *colon != ':') ++colon;
      if (colon >= e) {
        c.bad = true;
        return;
      }
      const char *ve = colon + 1;
      while (ve < e && !is_blank(*ve)) ++ve;
      int index;
      double v;
      if (!parse_num(q, colon, index) || !parse_value(colon + 1, ve, v) || index < 1) {
        c.bad = true;
        return;
      }
      c.idx.push_back(index);
      c.val.push_back((float)v);
      c.maxi = std::max(c.maxi, index);
      q = ve;
    }
    c.coef.push_back(cv);
    c.row_ptr.push_back((int64_t)c.idx.size());
  }
}

}  // namespace

extern "C" {

void tsvm_free(void *p) { free(p); }

tsvm_status tsvm_read_libsvm(const char *path, int32_t scale256, int32_t threads, float **labels,
                             float **X, int64_t *n_out, int64_t *d_out, int64_t *nnz_out,
                             int64_t *bad_line) {
  if (!path || !labels || !X || !n_out || !d_out) return TSVM_ERR_INVALID_ARGUMENT;
  *labels = nullptr;
  *X = nullptr;
  if (bad_line) *bad_line = 0;
  tsvm::TraceRange trace_call("tsvm_read_libsvm");
  FileView text;
  if (!text.open(path)) return TSVM_ERR_IO;
  const int nt = pick_threads(threads);
  // chunk boundaries at line starts, about text.size() / nt bytes apart
  std::vector<Chunk> ch(nt);
  const char *base = text.data(), *end = base + text.size();
  const char *b = base;
  for (int t = 0; t < nt; ++t) {
    const char *e = t == nt - 1 ? end : base + (text.size() * (size_t)(t + 1)) / nt;
    if (e < b) e = b;
    if (t < nt - 1) {
      const char *nl = static_cast<const char *>(memchr(e, '\n', (size_t)(end - e)));
      e = nl ? nl + 1 : end;
    }
    ch[t].begin = b;
    ch[t].end = e;
    b = e;
  }
  parallel_for(nt, [&](int t) { parse_chunk(ch[t], scale256 != 0); });
  int64_t lines_before = 0, n = 0, nnz = 0, mn = 1, mx = 0;
  for (int t = 0; t < nt; ++t) {
    if (ch[t].bad_local >= 0) {
      if (bad_line) *bad_line = lines_before + ch[t].bad_local + 1;
      return TSVM_ERR_IO;
    }
    lines_before += ch[t].lines;
    n += (int64_t)ch[t].labels.size();
    nnz += (int64_t)ch[t].idx.size();
    mn = std::min(mn, ch[t].min_index);
    mx = std::max(mx, ch[t].max_index);
  }
  const int64_t d = mn == 0 ? mx + 1 : mx;
  float *L = static_cast<float *>(malloc(sizeof(float) * (size_t)std::max<int64_t>(n, 1)));
  float *M = static_cast<float *>(calloc((size_t)std::max<int64_t>(n * d, 1), sizeof(float)));
  if (!L || !M) {
    free(L);
    free(M);
    return TSVM_ERR_OUT_OF_MEMORY;
  }
  std::vector<int64_t> row0(nt + 1, 0);
  for (int t = 0; t < nt; ++t) row0[t + 1] = row0[t] + (int64_t)ch[t].labels.size();
  parallel_for(nt, [&](int t) {
    const Chunk &c = ch[t];
    for (size_t r = 0; r < c.labels.size(); ++r) {
      const int64_t i = row0[t] + (int64_t)r;
      L[i] = c.labels[r];
      for (int64_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; ++e)
        M[i * d + (c.idx[e] - mn)] = c.val[e];
    }
  });
  *labels = L;
  *X = M;
  *n_out = n;
  *d_out = d;
  if (nnz_out) *nnz_out = nnz;
  return TSVM_OK;
}

tsvm_status tsvm_write_model(const char *path, int32_t kernel, const float *X, const float *y,
                             const double *alpha, int64_t n, int32_t d, double C, double gamma,
                             double b, int32_t pos, int32_t neg, int32_t threads, int64_t *n_sv,
                             int64_t *n_free) {
  if (!path || !X || !y || !alpha || n < 0 || d < 1) return TSVM_ERR_INVALID_ARGUMENT;
  if (kernel != TSVM_KERNEL_RBF && kernel != TSVM_KERNEL_LINEAR) return TSVM_ERR_UNSUPPORTED;
  tsvm::TraceRange trace_call("tsvm_write_model");
  std::vector<int64_t> sv;
  int64_t nfree = 0;
  for (int64_t i = 0; i < n; ++i)
    if (alpha[i] > 1e-6) {
      sv.push_back(i);
      if (alpha[i] < C - 1e-6) ++nfree;
    }
  if (n_sv) *n_sv = (int64_t)sv.size();
  if (n_free) *n_free = nfree;
  FILE *f = fopen(path, "w");
  if (!f) return TSVM_ERR_IO;
  bool ok = true;
  if (kernel == TSVM_KERNEL_LINEAR) {
    // w = sum over SVs of alpha_j y_j x_j (writemodel, tensorsvm-train.cu:330-349)
    std::vector<double> w(d, 0.0);
    for (int64_t j : sv)
      for (int c = 0; c < d; ++c) w[c] += alpha[j] * y[j] * X[(size_t)j * d + c];
    ok &= fprintf(f, "solver_type L2R_L1LOSS_SVC_DUAL\n") > 0;
    ok &= fprintf(f, "nr_class 2\n") > 0;
    ok &= fprintf(f, "label %d %d\n", pos, neg) > 0;
    ok &= fprintf(f, "nr_feature %d\n", d) > 0;
    ok &= fprintf(f, "bias %d\n", 1) > 0;
    ok &= fprintf(f, "w\n") > 0;
    for (int c = 0; c < d; ++c) ok &= fprintf(f, "%.16f \n", w[c]) > 0;
    ok &= fprintf(f, "%.16f\n", b) > 0;
  } else {
    ok &= fprintf(f, "svm_type c_svc\n") > 0;
    ok &= fprintf(f, "kernel_type rbf\n") > 0;
    ok &= fprintf(f, "gamma %.7f\n", gamma) > 0;
    ok &= fprintf(f, "nr_class 2\n") > 0;
    ok &= fprintf(f, "total_sv %zu\n", sv.size()) > 0;
    ok &= fprintf(f, "rho %f\n", -b) > 0;
    ok &= fprintf(f, "label %d %d\n", pos, neg) > 0;
    ok &= fprintf(f, "nr_sv %lld %lld\n", (long long)nfree, (long long)(sv.size() - nfree)) > 0;
    ok &= fprintf(f, "SV\n") > 0;
    const int nt = pick_threads(threads);
    const size_t per = (sv.size() + nt - 1) / std::max(nt, 1);
    std::vector<std::string> out(nt);
    parallel_for(nt, [&](int t) {
      std::string &s = out[t];
      const size_t a = std::min(sv.size(), per * t), e = std::min(sv.size(), per * (t + 1));
      for (size_t q = a; q < e; ++q) {
        const int64_t j = sv[q];
        put_fixed6(s, (double)y[j] * alpha[j]);
        s += ' ';
        for (int c = 0; c < d; ++c) {
          const float v = X[(size_t)j * d + c];
          if (v > 0 || v < 0) {
            put_int(s, c + 1);
            s += ':';
            put_fixed6_float(s, v);
            s += ' ';
          }
        }
        s += '\n';
      }
    });
    for (auto &s : out) ok &= fwrite(s.data(), 1, s.size(), f) == s.size();
  }
  ok &= fclose(f) == 0;
  return ok ? TSVM_OK : TSVM_ERR_IO;
}

void tsvm_free_model(tsvm_model_view *m) {
  if (!m) return;
  free(const_cast<float *>(m->sv));
  free(const_cast<double *>(m->coef));
  m->sv = nullptr;
  m->coef = nullptr;
}

tsvm_status tsvm_read_model(const char *path, tsvm_model_view *m, int32_t *label_pos,
                            int32_t *label_neg) {
  if (!path || !m) return TSVM_ERR_INVALID_ARGUMENT;
  *m = tsvm_model_view{};
  FileView text;
  if (!text.open(path)) return TSVM_ERR_IO;
  const char *p = text.data(), *end = p + text.size();
  auto next_line = [&](std::string &line) -> bool {
    if (p >= end) return false;
    const char *eol = static_cast<const char *>(memchr(p, '\n', (size_t)(end - p)));
    if (!eol) eol = end;
    line.assign(p, eol);
    while (!line.empty() && (line.back() == '\r' || line.back() == ' ')) line.pop_back();
    p = eol < end ? eol + 1 : end;
    return true;
  };
  std::string line;
  int kernel = -1, pos = 0, neg = 0, nr_feature = 0;
  long long total_sv = -1;
  double gamma = 0.0, rho = 0.0;
  bool have_label = false;
  while (next_line(line)) {
    char key[64] = {0};
    if (sscanf(line.c_str(), "%63s", key) != 1) continue;
    const char *rest = line.c_str() + strlen(key);
    if (!strcmp(key, "solver_type")) kernel = TSVM_KERNEL_LINEAR;
    else if (!strcmp(key, "kernel_type")) {
      char kt[32] = {0};
      if (sscanf(rest, "%31s", kt) != 1 || strcmp(kt, "rbf") != 0) return TSVM_ERR_UNSUPPORTED;
      kernel = TSVM_KERNEL_RBF;
    } else if (!strcmp(key, "gamma")) gamma = strtod(rest, nullptr);
    else if (!strcmp(key, "rho")) rho = strtod(rest, nullptr);
    else if (!strcmp(key, "total_sv")) total_sv = strtoll(rest, nullptr, 10);
    else if (!strcmp(key, "nr_feature")) nr_feature = (int)strtol(rest, nullptr, 10);
    else if (!strcmp(key, "nr_class")) {
      if (strtol(rest, nullptr, 10) != 2) return TSVM_ERR_UNSUPPORTED;
    } else if (!strcmp(key, "label")) {
      have_label = sscanf(rest, "%d %d", &pos, &neg) == 2;
    } else if (!strcmp(key, "SV") || !strcmp(key, "w")) {
      break;
    }
  }
  if (!have_label || kernel < 0) return TSVM_ERR_IO;
  if (label_pos) *label_pos = pos;
  if (label_neg) *label_neg = neg;
  m->kernel = kernel;
  if (kernel == TSVM_KERNEL_LINEAR) {
    // nr_feature weights, then the bias value (the reference's bias line)
    if (nr_feature < 1) return TSVM_ERR_IO;
    float *w = static_cast<float *>(malloc(sizeof(float) * nr_feature));
    if (!w) return TSVM_ERR_OUT_OF_MEMORY;
    for (int c = 0; c < nr_feature; ++c) {
      if (!next_line(line)) {
        free(w);
        return TSVM_ERR_IO;
      }
      w[c] = (float)strtod(line.c_str(), nullptr);
    }
    double bias = 0.0;
    if (next_line(line)) bias = strtod(line.c_str(), nullptr);
    m->d = nr_feature;
    m->sv = w;
    m->rho = -bias;
    return TSVM_OK;
  }
  // RBF: one line per SV, "coef idx:val ..." with 1-based indices, parsed in parallel chunks
  const int nt = pick_threads(0);
  std::vector<SvChunk> ch(nt);
  const char *b = p;
  const size_t rest = (size_t)(end - p);
  for (int t = 0; t < nt; ++t) {
    const char *e = t == nt - 1 ? end : p + (rest * (size_t)(t + 1)) / nt;
    if (e < b) e = b;
    if (t < nt - 1) {
      const char *nl = static_cast<const char *>(memchr(e, '\n', (size_t)(end - e)));
      e = nl ? nl + 1 : end;
    }
    ch[t].begin = b;
    ch[t].end = e;
    b = e;
  }
  parallel_for(nt, [&](int t) { parse_sv_chunk(ch[t]); });
  size_t nsv = 0;
  int maxi = 0;
  std::vector<size_t> row0(nt + 1, 0);
  for (int t = 0; t < nt; ++t) {
    if (ch[t].bad) return TSVM_ERR_IO;
    nsv += ch[t].coef.size();
    row0[t + 1] = nsv;
    maxi = std::max(maxi, ch[t].maxi);
  }
  if (total_sv >= 0 && (long long)nsv != total_sv) return TSVM_ERR_IO;
  const int d = std::max(maxi, 1);
  float *S = static_cast<float *>(calloc(std::max<size_t>(nsv * d, 1), sizeof(float)));
  double *cf = static_cast<double *>(malloc(sizeof(double) * std::max<size_t>(nsv, 1)));
  if (!S || !cf) {
    free(S);
    free(cf);
    return TSVM_ERR_OUT_OF_MEMORY;
  }
  parallel_for(nt, [&](int t) {
    const SvChunk &c = ch[t];
    for (size_t r = 0; r < c.coef.size(); ++r) {
      const size_t i = row0[t] + r;
      cf[i] = c.coef[r];
      for (int64_t e = c.row_ptr[r]; e < c.row_ptr[r + 1]; ++e)
        S[i * d + (size_t)(c.idx[e] - 1)] = c.val[e];
    }
  });
  m->d = d;
  m->nsv = (int64_t)nsv;
  m->sv = S;
  m->coef = cf;
  m->rho = rho;
  m->gamma = gamma;
  return TSVM_OK;
}

}  // extern "C"
