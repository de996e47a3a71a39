// File -> CSR loaders with the interface and flag semantics of the
// reference's include/graph_io.h (read_graph :280-295, fill_data :21-130,
// mtx2csr :216-261, graph2csr :177-213, gr2csr :133-174).
//
// The steps a caller can observe are kept: the same per-format edge
// insertion order (including the reference's "symmetrize turns transposing
// off" behaviour), std::sort by column on the same Edge layout, order-
// preserving self-loop removal, adjacent-duplicate removal, and the same
// progress lines on stdout.  The parsing itself reads the whole file at once
// and scans it with a hand-written number parser instead of getline+sscanf,
// and the erase-in-a-loop passes are linear compactions with identical
// results.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <exception>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "gardenia_graph_io.h"
#include "gpr.h"

namespace gpr {
void set_error(const char *fmt, ...);
}

namespace {

struct Edge {
  int dst;
  WeightT wt;
};

bool by_column(const Edge &a, const Edge &b) { return a.dst < b.dst; }

struct Reader {
  std::string buf;
  size_t pos = 0;
  bool load(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n : 0);
    size_t got = n > 0 ? fread(&buf[0], 1, (size_t)n, f) : 0;
    fclose(f);
    buf.resize(got);
    return true;
  }
  bool eof() const { return pos >= buf.size(); }
  // Next line [b, e) without the newline.
  bool line(size_t *b, size_t *e) {
    if (pos >= buf.size()) return false;
    *b = pos;
    const char *nl = (const char *)memchr(buf.data() + pos, '\n', buf.size() - pos);
    *e = nl ? (size_t)(nl - buf.data()) : buf.size();
    pos = nl ? *e + 1 : buf.size();
    return true;
  }
};

// Integer starting at p (after blanks); returns false when there is none.
bool parse_int(const char *&p, const char *end, int *out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  if (p >= end) return false;
  bool neg = false;
  if (*p == '-' || *p == '+') {
    neg = *p == '-';
    ++p;
  }
  if (p >= end || *p < '0' || *p > '9') return false;
  long long v = 0;
  while (p < end && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
  *out = (int)(neg ? -v : v);
  return true;
}

bool parse_float(const char *&p, const char *end, float *out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  if (p >= end) return false;
  char tmp[64];
  size_t n = 0;
  while (p + n < end && n < sizeof(tmp) - 1 && p[n] != ' ' && p[n] != '\t' && p[n] != '\r' &&
         p[n] != '\n')
    ++n;
  memcpy(tmp, p, n);
  tmp[n] = 0;
  char *q = nullptr;
  float v = strtof(tmp, &q);
  if (q == tmp) return false;
  p += (q - tmp);
  *out = v;
  return true;
}

void fill_data(int m, int &nnz, int *&row_offsets, int *&column_indices, WeightT *&weight,
               std::vector<std::vector<Edge>> &vertices, bool symmetrize, bool sorted,
               bool remove_selfloops, bool remove_redundents) {
  if (sorted) {
    printf("Sorting the neighbor lists...");
    for (int i = 0; i < m; i++) std::sort(vertices[i].begin(), vertices[i].end(), by_column);
    printf(" Done\n");
  }
  int num_selfloops = 0;
  if (remove_selfloops) {
    printf("Removing self loops...");
    for (int i = 0; i < m; i++) {
      auto &v = vertices[i];
      auto it = std::remove_if(v.begin(), v.end(), [i](const Edge &e) { return e.dst == i; });
      num_selfloops += (int)(v.end() - it);
      v.erase(it, v.end());
    }
    printf(" %d selfloops are removed\n", num_selfloops);
  }
  int num_redundents = 0;
  if (remove_redundents) {
    printf("Removing redundent edges...");
    for (int i = 0; i < m; i++) {
      auto &v = vertices[i];
      auto it = std::unique(v.begin(), v.end(),
                            [](const Edge &a, const Edge &b) { return a.dst == b.dst; });
      num_redundents += (int)(v.end() - it);
      v.erase(it, v.end());
    }
    printf(" %d redundent edges are removed\n", num_redundents);
  }
  row_offsets = (int *)malloc((size_t)(m + 1) * sizeof(int));
  if (!row_offsets) throw std::bad_alloc();
  long long count = 0;
  for (int i = 0; i < m; i++) {
    row_offsets[i] = (int)count;
    count += (long long)vertices[i].size();
  }
  row_offsets[m] = (int)count;
  if (!symmetrize && count + num_selfloops + num_redundents != nnz)
    printf("Error reading graph, number of edges in edge list %d != %d\n", (int)count, nnz);
  nnz = (int)count;
  printf("num_vertices %d num_edges %d\n", m, nnz);
  column_indices = (int *)malloc((size_t)(count > 0 ? count : 1) * sizeof(int));
  weight = (WeightT *)malloc((size_t)(count > 0 ? count : 1) * sizeof(WeightT));
  if (!column_indices || !weight) throw std::bad_alloc();
  long long k = 0;
  for (int i = 0; i < m; i++)
    for (const Edge &e : vertices[i]) {
      column_indices[k] = e.dst;
      weight[k] = e.wt;
      ++k;
    }
}

// Adds edge src->dst with the reference's symmetrize / transpose rules.
inline void add_edge(std::vector<std::vector<Edge>> &v, int src, int dst, WeightT wt,
                     bool symmetrize, bool &transpose, bool sym_skips_selfloop) {
  if (symmetrize && (!sym_skips_selfloop || src != dst)) {
    v[dst].push_back(Edge{src, wt});
    transpose = false;
  }
  if (!transpose) v[src].push_back(Edge{dst, wt});
  else v[dst].push_back(Edge{src, wt});
}

bool in_range(int x, int m) { return x >= 0 && x < m; }

// An unreadable or malformed file.  read_graph turns it into the
// reference's message and exit; the C entry points into a status.
struct ReadError {
  const char *path;
  const char *why;
};

[[noreturn]] void bad(const char *path, const char *why) { throw ReadError{path, why}; }

void mtx2csr(const char *path, int &m, int &n, int &nnz, int *&rowptr, int *&col, WeightT *&w,
             bool symmetrize, bool transpose, bool sorted, bool rm_self, bool rm_dup) {
  printf("Reading (.mtx) input file %s\n", path);
  Reader R;
  if (!R.load(path)) bad(path, "cannot open");
  size_t b, e;
  if (!R.line(&b, &e)) bad(path, "empty file");
  while (b < e && R.buf[b] == '%')
    if (!R.line(&b, &e)) bad(path, "missing size line");
  const char *p = R.buf.data() + b, *pe = R.buf.data() + e;
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &n) || !parse_int(p, pe, &nnz) || m < 0)
    bad(path, "bad size line");
  if (m != n) printf("Warning, m(%d) != n(%d)\n", m, n);
  std::vector<std::vector<Edge>> v((size_t)m);
  int src = 0, dst = 0;
  WeightT wt = 1.0f;
  for (int i = 0; i < nnz; i++) {
    if (!R.line(&b, &e)) bad(path, "fewer entries than announced");
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    int num = 0;
    if (parse_int(p, pe, &src)) {
      ++num;
      if (parse_int(p, pe, &dst)) {
        ++num;
        if (parse_float(p, pe, &wt)) ++num;
      }
    }
    if (num == 2) wt = 1;
    if (wt < 0) wt = -wt;
    // decremented in place, as the reference does: a line that sets neither
    // number repeats the previous edge decremented once more
    --src;
    --dst;
    if (!in_range(src, m) || !in_range(dst, m)) bad(path, "index out of range");
    add_edge(v, src, dst, wt, symmetrize, transpose, true);
  }
  fill_data(m, nnz, rowptr, col, w, v, symmetrize, sorted, rm_self, rm_dup);
}

void graph2csr(const char *path, int &m, int &nnz, int *&rowptr, int *&col, WeightT *&w,
               bool symmetrize, bool transpose, bool sorted, bool rm_self, bool rm_dup) {
  printf("Reading .graph input file %s\n", path);
  Reader R;
  if (!R.load(path)) bad(path, "cannot open");
  size_t b, e;
  if (!R.line(&b, &e)) bad(path, "empty file");
  const char *p = R.buf.data() + b, *pe = R.buf.data() + e;
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz) || m < 0) bad(path, "bad size line");
  std::vector<std::vector<Edge>> v((size_t)m);
  for (int src = 0; src < m; src++) {
    if (!R.line(&b, &e)) break;
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    int dst;
    while (parse_int(p, pe, &dst)) {
      --dst;
      if (!in_range(dst, m)) bad(path, "index out of range");
      add_edge(v, src, dst, 1.0f, symmetrize, transpose, false);
    }
  }
  fill_data(m, nnz, rowptr, col, w, v, symmetrize, sorted, rm_self, rm_dup);
}

void gr2csr(const char *path, int &m, int &nnz, int *&rowptr, int *&col, WeightT *&w,
            bool symmetrize, bool transpose, bool sorted, bool rm_self, bool rm_dup) {
  printf("Reading RMAT (.gr) input file %s\n", path);
  Reader R;
  if (!R.load(path)) bad(path, "cannot open");
  size_t b, e;
  if (!R.line(&b, &e)) bad(path, "empty file");
  while (b < e && R.buf[b] == 'c')
    if (!R.line(&b, &e)) bad(path, "missing problem line");
  // "p sp <m> <nnz>"
  const char *p = R.buf.data() + b, *pe = R.buf.data() + e;
  if (p < pe) ++p;
  while (p < pe && (*p == ' ' || *p == '\t')) ++p;
  while (p < pe && *p != ' ' && *p != '\t') ++p;
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz) || m < 0) bad(path, "bad problem line");
  std::vector<std::vector<Edge>> v((size_t)m);
  int src = 0, dst = 0;  // kept across lines: a missing number keeps its last value
  for (int i = 0; i < nnz; i++) {
    if (!R.line(&b, &e)) bad(path, "fewer arcs than announced");
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (p < pe && *p != 'a') printf("line %d\n", __LINE__);
    if (p < pe) ++p;
    if (parse_int(p, pe, &src)) parse_int(p, pe, &dst);
    --src;
    --dst;
    if (!in_range(src, m) || !in_range(dst, m)) bad(path, "index out of range");
    add_edge(v, src, dst, 1.0f, symmetrize, transpose, false);
  }
  fill_data(m, nnz, rowptr, col, w, v, symmetrize, sorted, rm_self, rm_dup);
}

enum class Format { kMtx, kGraph, kGr, kUnknown };

// graph_io.h:281-291: the format is chosen by the first matching substring.
Format format_of(const char *path) {
  if (strstr(path, ".mtx")) return Format::kMtx;
  if (strstr(path, ".graph")) return Format::kGraph;
  if (strstr(path, ".gr")) return Format::kGr;
  return Format::kUnknown;
}

// read_graph for a file of a known format; throws ReadError or
// std::bad_alloc, after which the output pointers hold what was allocated.
void read_known(Format f, const char *path, int &m, int &n, int &nnz, int *&row_offsets,
                int *&column_indices, int *&degree, WeightT *&weight, bool is_symmetrize,
                bool is_transpose, bool sorted, bool remove_selfloops, bool remove_redundents) {
  if (f == Format::kMtx) {
    mtx2csr(path, m, n, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
            sorted, remove_selfloops, remove_redundents);
  } else if (f == Format::kGraph) {
    graph2csr(path, m, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
              sorted, remove_selfloops, remove_redundents);
    n = m;
  } else {
    gr2csr(path, m, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
           sorted, remove_selfloops, remove_redundents);
    n = m;
  }
  printf("Calculating degree...");
  degree = (int *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int));
  if (!degree) throw std::bad_alloc();
  for (int i = 0; i < m; i++) degree[i] = row_offsets[i + 1] - row_offsets[i];
  printf(" Done\n");
}

}  // namespace

// The reference's behaviour on a bad file is kept here: a message and exit.
void read_graph(int argc, char *argv[], int &m, int &n, int &nnz, int *&row_offsets,
                int *&column_indices, int *&degree, WeightT *&weight, bool is_symmetrize,
                bool is_transpose, bool sorted, bool remove_selfloops, bool remove_redundents) {
  if (argc < 2) {
    fprintf(stderr, "read_graph: no input file\n");
    exit(EXIT_FAILURE);
  }
  const char *path = argv[1];
  const Format f = format_of(path);
  if (f == Format::kUnknown) {
    printf("Unrecognizable input file format\n");
    exit(0);
  }
  try {
    read_known(f, path, m, n, nnz, row_offsets, column_indices, degree, weight, is_symmetrize,
               is_transpose, sorted, remove_selfloops, remove_redundents);
  } catch (const ReadError &e) {
    fprintf(stderr, "read_graph: %s: %s\n", e.path, e.why);
    exit(EXIT_FAILURE);
  } catch (const std::bad_alloc &) {
    fprintf(stderr, "read_graph: %s: out of host memory\n", path);
    exit(EXIT_FAILURE);
  }
}

namespace {

// ---------------------------------------------------------------------------
// Parallel parse into the reference's push order.
//
// The reference builds vector<vector<Edge>> by pushing, line by line, each
// edge into the list of one vertex (graph_io.h:133-261).  A push is a pure
// function of its line: the "symmetrize stops transposing" side effect never
// changes what is pushed (with symmetrize the reverse edge is pushed before
// the flag is read, and an .mtx self-loop lands in the same list either way).
// So the file can be parsed in parallel chunks of whole lines into an array
// of pushes (row, col, weight) in file order; a stable sort of the pushes by
// row then reproduces every per-vertex list exactly (gpr_csr_from_edges).
// Files with a line the reference would read with carried-over values (an
// .mtx entry line with fewer than two numbers) are parsed sequentially.
// ---------------------------------------------------------------------------
struct Pushes {
  std::vector<int> row, col;
  std::vector<float> wt;
  void add(int r, int c, float w) {
    row.push_back(r);
    col.push_back(c);
    wt.push_back(w);
  }
};

enum Fmt { kMtx, kGraph, kGr };

// Pushes of one edge src->dst (0-based) under the reference's rules.
inline void push_edge(Pushes &P, int src, int dst, float wt, bool symmetrize, bool transpose,
                      bool sym_skips_selfloop) {
  if (symmetrize) {
    if (!sym_skips_selfloop || src != dst) P.add(dst, src, wt);
    P.add(src, dst, wt);
  } else if (!transpose) {
    P.add(src, dst, wt);
  } else {
    P.add(dst, src, wt);
  }
}

struct ChunkResult {
  Pushes P;
  int err = 0;          // 1 index out of range, 3 a line the sequential reader must take
  long long lines = 0;  // lines parsed
};

// Parses lines [first_line, limit) of this chunk (global line numbers).
void parse_chunk(const std::string &buf, size_t cb, size_t ce, long long first_line,
                 long long limit, Fmt fmt, int m, bool symmetrize, bool transpose,
                 ChunkResult *out) {
  size_t pos = cb;
  long long ln = first_line;
  while (pos < ce && ln < limit) {
    const char *nl = (const char *)memchr(buf.data() + pos, '\n', ce - pos);
    const size_t e = nl ? (size_t)(nl - buf.data()) : ce;
    const char *p = buf.data() + pos, *pe = buf.data() + e;
    if (fmt == kMtx) {
      int src = 0, dst = 0;
      float wt = 1.0f;
      int num = 0;
      if (parse_int(p, pe, &src)) {
        ++num;
        if (parse_int(p, pe, &dst)) {
          ++num;
          if (parse_float(p, pe, &wt)) ++num;
        }
      }
      if (num < 2) {
        out->err = 3;
        return;
      }
      if (num == 2) wt = 1;
      if (wt < 0) wt = -wt;
      const int s = src - 1, d = dst - 1;
      if (!in_range(s, m) || !in_range(d, m)) {
        out->err = 1;
        return;
      }
      push_edge(out->P, s, d, wt, symmetrize, transpose, true);
    } else if (fmt == kGr) {
      if (p < pe) ++p;
      int src = 0, dst = 0;
      if (!parse_int(p, pe, &src) || !parse_int(p, pe, &dst)) {
        out->err = 3;  // carries values over from the previous line: sequential reader
        return;
      }
      --src;
      --dst;
      if (!in_range(src, m) || !in_range(dst, m)) {
        out->err = 1;
        return;
      }
      push_edge(out->P, src, dst, 1.0f, symmetrize, transpose, false);
    } else {
      const int src = (int)ln;
      int dst;
      while (parse_int(p, pe, &dst)) {
        --dst;
        if (!in_range(dst, m)) {
          out->err = 1;
          return;
        }
        push_edge(out->P, src, dst, 1.0f, symmetrize, transpose, false);
      }
    }
    ++ln;
    ++out->lines;
    pos = nl ? e + 1 : ce;
  }
}

int io_threads() {
  const char *env = getenv("GPR_IO_THREADS");
  int t = env ? atoi(env) : (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(t, 64));
}

// Parses `path` into pushes; returns 0, or -1 (cannot open / malformed:
// message in *why) or -2 (needs the sequential reader).
int parse_pushes(const char *path, bool symmetrize, bool transpose, int threads, int *m_out,
                 int *nnz_out, Pushes *out, const char **why) {
  Fmt fmt;
  if (strstr(path, ".mtx")) fmt = kMtx;
  else if (strstr(path, ".graph")) fmt = kGraph;
  else if (strstr(path, ".gr")) fmt = kGr;
  else {
    *why = "unrecognizable input file format";
    return -1;
  }
  Reader R;
  if (!R.load(path)) {
    *why = "cannot open";
    return -1;
  }
  size_t b, e;
  if (!R.line(&b, &e)) {
    *why = "empty file";
    return -1;
  }
  int m = 0, n = 0, nnz = 0;
  const char *p, *pe;
  if (fmt == kMtx) {
    while (b < e && R.buf[b] == '%')
      if (!R.line(&b, &e)) {
        *why = "missing size line";
        return -1;
      }
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (!parse_int(p, pe, &m) || !parse_int(p, pe, &n) || !parse_int(p, pe, &nnz)) {
      *why = "bad size line";
      return -1;
    }
  } else if (fmt == kGr) {
    while (b < e && R.buf[b] == 'c')
      if (!R.line(&b, &e)) {
        *why = "missing problem line";
        return -1;
      }
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (p < pe) ++p;
    while (p < pe && (*p == ' ' || *p == '\t')) ++p;
    while (p < pe && *p != ' ' && *p != '\t') ++p;
    if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz)) {
      *why = "bad problem line";
      return -1;
    }
  } else {
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz)) {
      *why = "bad size line";
      return -1;
    }
  }
  if (m < 0) {
    *why = "bad size line";
    return -1;
  }
  const long long limit = fmt == kGraph ? m : nnz;
  const size_t start = R.pos, size = R.buf.size();
  const int T = std::max(1, threads);
  std::vector<size_t> cut(T + 1, size);
  cut[0] = start;
  for (int k = 1; k < T; ++k) {
    size_t q = start + (size - start) / T * k;
    if (q < cut[k - 1]) q = cut[k - 1];
    const char *nl = q < size ? (const char *)memchr(R.buf.data() + q, '\n', size - q) : nullptr;
    cut[k] = nl ? (size_t)(nl - R.buf.data()) + 1 : size;
  }
  // Lines per chunk (a final line without a newline counts), then each
  // chunk's first global line number.
  std::vector<long long> nlines(T, 0), first(T + 1, 0);
  {
    std::vector<std::thread> th;
    for (int k = 0; k < T; ++k)
      th.emplace_back([&, k] {
        long long c = 0;
        for (size_t i = cut[k]; i < cut[k + 1]; ++i) c += R.buf[i] == '\n';
        if (cut[k + 1] == size && cut[k] < size && R.buf[size - 1] != '\n') ++c;
        nlines[k] = c;
      });
    for (auto &t : th) t.join();
  }
  for (int k = 0; k < T; ++k) first[k + 1] = first[k] + nlines[k];
  if (fmt != kGraph && first[T] < limit) {
    *why = fmt == kMtx ? "fewer entries than announced" : "fewer arcs than announced";
    return -1;
  }
  std::vector<ChunkResult> res(T);
  {
    std::vector<std::thread> th;
    for (int k = 0; k < T; ++k)
      th.emplace_back([&, k] {
        parse_chunk(R.buf, cut[k], cut[k + 1], first[k], limit, fmt, m, symmetrize, transpose,
                    &res[k]);
      });
    for (auto &t : th) t.join();
  }
  for (auto &r : res) {
    if (r.err == 3) return -2;
    if (r.err == 1) {
      *why = "index out of range";
      return -1;
    }
  }
  size_t total = 0;
  for (auto &r : res) total += r.P.row.size();
  out->row.resize(total);
  out->col.resize(total);
  out->wt.resize(total);
  size_t o = 0;
  for (auto &r : res) {
    std::copy(r.P.row.begin(), r.P.row.end(), out->row.begin() + o);
    std::copy(r.P.col.begin(), r.P.col.end(), out->col.begin() + o);
    std::copy(r.P.wt.begin(), r.P.wt.end(), out->wt.begin() + o);
    o += r.P.row.size();
  }
  *m_out = m;
  *nnz_out = nnz;
  return 0;
}

// Sequential fallback for files with lines the reference reads with values
// carried over from the previous line (.mtx and .gr): the numbers live across
// lines and are decremented in place, as in graph_io.h:155-158 and :238-245.
void parse_pushes_sequential(const char *path, bool symmetrize, bool transpose, int *m_out,
                             int *nnz_out, Pushes *out) {
  const bool gr = strstr(path, ".mtx") == nullptr;
  Reader R;
  if (!R.load(path)) bad(path, "cannot open");
  size_t b, e;
  if (!R.line(&b, &e)) bad(path, "empty file");
  while (b < e && R.buf[b] == (gr ? 'c' : '%'))
    if (!R.line(&b, &e)) bad(path, "missing size line");
  const char *p = R.buf.data() + b, *pe = R.buf.data() + e;
  int m = 0, n = 0, nnz = 0;
  if (gr) {
    if (p < pe) ++p;
    while (p < pe && (*p == ' ' || *p == '\t')) ++p;
    while (p < pe && *p != ' ' && *p != '\t') ++p;
    if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz) || m < 0) bad(path, "bad problem line");
  } else if (!parse_int(p, pe, &m) || !parse_int(p, pe, &n) || !parse_int(p, pe, &nnz) ||
             m < 0) {
    bad(path, "bad size line");
  }
  int src = 0, dst = 0;
  WeightT wt = 1.0f;
  for (int i = 0; i < nnz; i++) {
    if (!R.line(&b, &e)) bad(path, "fewer entries than announced");
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (gr) {
      if (p < pe) ++p;
      if (parse_int(p, pe, &src)) parse_int(p, pe, &dst);
      wt = 1.0f;
    } else {
      int num = 0;
      if (parse_int(p, pe, &src)) {
        ++num;
        if (parse_int(p, pe, &dst)) {
          ++num;
          if (parse_float(p, pe, &wt)) ++num;
        }
      }
      if (num == 2) wt = 1;
      if (wt < 0) wt = -wt;
    }
    --src;
    --dst;
    if (!in_range(src, m) || !in_range(dst, m)) bad(path, "index out of range");
    push_edge(*out, src, dst, wt, symmetrize, transpose, !gr);
  }
  *m_out = m;
  *nnz_out = nnz;
}

}  // namespace

// Pushes of `path` in the reference's order (row, col, weight), malloc'd
// here and released with gpr_read_graph_free.  threads <= 0: all cores
// (GPR_IO_THREADS overrides).
extern "C" int gpr_parse_edges(const char *path, int symmetrize, int transpose, int threads,
                               int *m_out, int *nnz_header, long long *n_push, int **row,
                               int **col, float **wt) {
  if (!path || !m_out || !nnz_header || !n_push || !row || !col || !wt) {
    gpr::set_error("gpr_parse_edges: NULL argument");
    return 1;
  }
  Pushes P;
  int m = 0, nnz = 0;
  try {
    const char *why = "";
    const int rc = parse_pushes(path, symmetrize != 0, transpose != 0,
                                threads > 0 ? threads : io_threads(), &m, &nnz, &P, &why);
    if (rc == -1) bad(path, why);
    if (rc == -2) {
      P = Pushes();
      parse_pushes_sequential(path, symmetrize != 0, transpose != 0, &m, &nnz, &P);
    }
  } catch (const ReadError &e) {
    fprintf(stderr, "gpr_parse_edges: %s: %s\n", e.path, e.why);
    gpr::set_error("gpr_parse_edges: %s: %s", e.path, e.why);
    return 1;
  } catch (const std::exception &e) {  // host memory or threads
    gpr::set_error("gpr_parse_edges: %s: %s", path, e.what());
    return 2;
  }
  const size_t k = P.row.size();
  *row = (int *)malloc(sizeof(int) * (k ? k : 1));
  *col = (int *)malloc(sizeof(int) * (k ? k : 1));
  *wt = (float *)malloc(sizeof(float) * (k ? k : 1));
  if (!*row || !*col || !*wt) {
    free(*row);
    free(*col);
    free(*wt);
    *row = *col = nullptr;
    *wt = nullptr;
    gpr::set_error("gpr_parse_edges: %s: out of host memory", path);
    return 2;
  }
  if (k) {
    memcpy(*row, P.row.data(), sizeof(int) * k);
    memcpy(*col, P.col.data(), sizeof(int) * k);
    memcpy(*wt, P.wt.data(), sizeof(float) * k);
  }
  *m_out = m;
  *nnz_header = nnz;
  *n_push = (long long)k;
  return 0;
}

// C entry point for foreign callers (ctypes / cgo): same flags, arrays
// malloc'd here and released with gpr_read_graph_free.
extern "C" int gpr_read_graph(const char *path, int symmetrize, int transpose, int sorted,
                              int remove_selfloops, int remove_redundents, int *m_out,
                              int *nnz_out, int **row_offsets, int **column_indices,
                              int **degree, float **weight) {
  if (!path || !m_out || !nnz_out || !row_offsets || !column_indices || !degree || !weight) {
    gpr::set_error("gpr_read_graph: NULL argument");
    return GPR_EINVAL;
  }
  const Format f = format_of(path);
  if (f == Format::kUnknown) {
    gpr::set_error("gpr_read_graph: %s: unrecognizable input file format", path);
    return GPR_EINVAL;
  }
  int m = 0, n = 0, nnz = 0;
  int *rp = nullptr, *ci = nullptr, *deg = nullptr;
  WeightT *w = nullptr;
  int rc = GPR_OK;
  try {
    read_known(f, path, m, n, nnz, rp, ci, deg, w, symmetrize != 0, transpose != 0, sorted != 0,
               remove_selfloops != 0, remove_redundents != 0);
  } catch (const ReadError &e) {
    gpr::set_error("gpr_read_graph: %s: %s", e.path, e.why);
    rc = GPR_EINVAL;
  } catch (const std::bad_alloc &) {
    gpr::set_error("gpr_read_graph: %s: out of host memory", path);
    rc = GPR_ENOMEM;
  }
  fflush(stdout);
  if (rc != GPR_OK) {
    free(rp);
    free(ci);
    free(deg);
    free(w);
    return rc;
  }
  *m_out = m;
  *nnz_out = nnz;
  *row_offsets = rp;
  *column_indices = ci;
  *degree = deg;
  *weight = w;
  return GPR_OK;
}

extern "C" void gpr_read_graph_free(void *p) { free(p); }
