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
#include <string>
#include <vector>

#include "gardenia_graph_io.h"

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

[[noreturn]] void bad(const char *path, const char *why) {
  fprintf(stderr, "read_graph: %s: %s\n", path, why);
  exit(EXIT_FAILURE);
}

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
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &n) || !parse_int(p, pe, &nnz))
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
    int s = src - 1, d = dst - 1;
    if (!in_range(s, m) || !in_range(d, m)) bad(path, "index out of range");
    add_edge(v, s, d, wt, symmetrize, transpose, true);
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
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz)) bad(path, "bad size line");
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
  if (!parse_int(p, pe, &m) || !parse_int(p, pe, &nnz)) bad(path, "bad problem line");
  std::vector<std::vector<Edge>> v((size_t)m);
  for (int i = 0; i < nnz; i++) {
    if (!R.line(&b, &e)) bad(path, "fewer arcs than announced");
    p = R.buf.data() + b;
    pe = R.buf.data() + e;
    if (p < pe && *p != 'a') printf("line %d\n", __LINE__);
    if (p < pe) ++p;
    int src = 0, dst = 0;
    if (!parse_int(p, pe, &src) || !parse_int(p, pe, &dst)) bad(path, "bad arc line");
    --src;
    --dst;
    if (!in_range(src, m) || !in_range(dst, m)) bad(path, "index out of range");
    add_edge(v, src, dst, 1.0f, symmetrize, transpose, false);
  }
  fill_data(m, nnz, rowptr, col, w, v, symmetrize, sorted, rm_self, rm_dup);
}

}  // namespace

void read_graph(int argc, char *argv[], int &m, int &n, int &nnz, int *&row_offsets,
                int *&column_indices, int *&degree, WeightT *&weight, bool is_symmetrize,
                bool is_transpose, bool sorted, bool remove_selfloops, bool remove_redundents) {
  if (argc < 2) {
    fprintf(stderr, "read_graph: no input file\n");
    exit(EXIT_FAILURE);
  }
  const char *path = argv[1];
  if (strstr(path, ".mtx")) {
    mtx2csr(path, m, n, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
            sorted, remove_selfloops, remove_redundents);
  } else if (strstr(path, ".graph")) {
    graph2csr(path, m, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
              sorted, remove_selfloops, remove_redundents);
    n = m;
  } else if (strstr(path, ".gr")) {
    gr2csr(path, m, nnz, row_offsets, column_indices, weight, is_symmetrize, is_transpose,
           sorted, remove_selfloops, remove_redundents);
    n = m;
  } else {
    printf("Unrecognizable input file format\n");
    exit(0);
  }
  printf("Calculating degree...");
  degree = (int *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int));
  for (int i = 0; i < m; i++) degree[i] = row_offsets[i + 1] - row_offsets[i];
  printf(" Done\n");
}

// C entry point for foreign callers (ctypes / cgo): same flags, arrays
// malloc'd here and released with gpr_read_graph_free.
extern "C" int gpr_read_graph(const char *path, int symmetrize, int transpose, int sorted,
                              int remove_selfloops, int remove_redundents, int *m_out,
                              int *nnz_out, int **row_offsets, int **column_indices,
                              int **degree, float **weight) {
  char *argv[2] = {(char *)"gpr", (char *)path};
  int m = 0, n = 0, nnz = 0;
  read_graph(2, argv, m, n, nnz, *row_offsets, *column_indices, *degree, *weight,
             symmetrize != 0, transpose != 0, sorted != 0, remove_selfloops != 0,
             remove_redundents != 0);
  *m_out = m;
  *nnz_out = nnz;
  fflush(stdout);
  return 0;
}

extern "C" void gpr_read_graph_free(void *p) { free(p); }
