// mmio.cpp -- MatrixMarket input and output for the seeded-problem type
// (host code in libab2), so that systems stored as files go through the
// same path as the generated ones.
//
// Reading follows Alien's MatrixMarket reader
// (src/movesemantic/alien/move/impl/MatrixMarketReader.cc):
//   * readBanner (:58-131): the first line starting with "%%MatrixMarket"
//     must say "coordinate" and "real" (case-insensitive), else the file is
//     rejected; symmetry "general" is taken as it is, any other value
//     ("symmetric", "skew-symmetric", "hermitian") as symmetric -- the reader
//     mirrors every off-diagonal entry with the same value (skew-symmetric
//     files therefore come out symmetric, as in the reference);
//   * '%' lines are comments; the first other line is "rows cols nnz";
//   * readValues (:133-157): each entry "row col value" (1-based) is added
//     into the matrix (DoK contribute = addNNZ: duplicates are summed in file
//     order), then its mirror when symmetric and row != col.
// The result is a CSR matrix with the columns of each row ascending, as
// Alien's profilers produce.  Right-hand side: an "array real" file with one
// value per line (readFromMatrixMarket for vectors, :189-273, which reads the
// first token of each line); without one, b = 1 everywhere as
// MatrixMarketProblem.cpp:33-43 does.  Only square matrices are accepted (the
// solvers need them).  Writing produces "coordinate real general" with 17
// significant digits (exact round trip) and the standard one-value-per-line
// array form for b (the reference's MatrixMarketSystemWriter writes
// "index value" pairs, which its own reader would take the index of).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ab2.h"
#include "ab2_problems.h"

namespace {

thread_local std::string g_mm_error;

int fail(const std::string& msg) {
  g_mm_error = msg;
  return AB2_ERR_BAD_ARG;
}

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return s;
}

bool skip_line(const std::string& line) {
  for (char c : line) {
    if (c == '%') return true;
    if (!std::isspace((unsigned char)c)) return false;
  }
  return true;  // blank
}

struct Entry {
  int r, c;
  double v;
};

}  // namespace

extern "C" {

const char* ab2_matrix_market_error(void) { return g_mm_error.c_str(); }

int ab2_problem_read_matrix_market(const char* matrix_path, const char* rhs_path, ab2_problem** out) {
  if (!matrix_path || !out) return fail("null argument");
  *out = nullptr;
  std::ifstream in(matrix_path);
  if (!in) return fail(std::string("cannot open ") + matrix_path);
  std::string line;
  bool header = false, symmetric = true;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string tag, object, format, scalar, symmetry;
    ss >> tag;
    if (tag != "%%MatrixMarket") continue;
    ss >> object >> format >> scalar >> symmetry;
    if (lower(format) != "coordinate" || lower(scalar) != "real")
      return fail("invalid header: only \"coordinate real\" matrices are read");
    symmetric = lower(symmetry) != "general";
    header = true;
    break;
  }
  if (!header) return fail("no %%MatrixMarket header");
  long long rows = -1, cols = -1, nnz = -1;
  while (std::getline(in, line)) {
    if (skip_line(line)) continue;
    std::istringstream ss(line);
    ss >> rows >> cols >> nnz;
    break;
  }
  if (rows < 0 || cols < 0 || nnz < 0) return fail("missing or bad size line");
  if (rows != cols) return fail("matrix is not square");
  if (rows > 0x7fffffffLL - 1) return fail("too many rows for 32-bit indices");
  const int n = (int)rows;
  std::vector<Entry> e;
  e.reserve((size_t)(symmetric ? 2 * nnz : nnz));
  long long seen = 0;
  while (seen < nnz && std::getline(in, line)) {
    if (skip_line(line)) continue;
    std::istringstream ss(line);
    long long r = 0, c = 0;
    double v = 0.0;
    if (!(ss >> r >> c >> v)) return fail("bad entry line: " + line);
    if (r < 1 || r > rows || c < 1 || c > cols) return fail("entry index out of range: " + line);
    ++seen;
    e.push_back(Entry{(int)r - 1, (int)c - 1, v});
    if (symmetric && r != c) e.push_back(Entry{(int)c - 1, (int)r - 1, v});
  }
  if (seen < nnz) return fail("file ends before its nnz entries");
  // contributions in file order per (row, col): a stable sort keeps it
  std::stable_sort(e.begin(), e.end(), [](const Entry& a, const Entry& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  std::vector<int> rp((size_t)n + 1, 0), ci;
  std::vector<double> vals;
  ci.reserve(e.size());
  vals.reserve(e.size());
  for (size_t k = 0; k < e.size();) {
    size_t m = k;
    double s = 0.0;
    for (; m < e.size() && e[m].r == e[k].r && e[m].c == e[k].c; ++m) s += e[m].v;
    ci.push_back(e[k].c);
    vals.push_back(s);
    rp[(size_t)e[k].r + 1] += 1;
    k = m;
  }
  for (int i = 0; i < n; ++i) rp[(size_t)i + 1] += rp[(size_t)i];
  std::vector<double> b((size_t)n, 1.0);
  if (rhs_path) {
    std::ifstream rin(rhs_path);
    if (!rin) return fail(std::string("cannot open ") + rhs_path);
    bool vheader = false;
    while (std::getline(rin, line)) {
      std::istringstream ss(line);
      std::string tag, object, format, scalar;
      ss >> tag;
      if (tag != "%%MatrixMarket") continue;
      ss >> object >> format >> scalar;
      if (lower(format) != "array" || lower(scalar) != "real")
        return fail("right-hand side must be an \"array real\" file");
      vheader = true;
      break;
    }
    if (!vheader) return fail("right-hand side has no %%MatrixMarket header");
    long long vrows = -1, vcols = -1;
    while (std::getline(rin, line)) {
      if (skip_line(line)) continue;
      std::istringstream ss(line);
      ss >> vrows >> vcols;
      break;
    }
    if (vcols != 1) return fail("right-hand side must hold exactly one vector");
    if (vrows != rows) return fail("right-hand side size does not match the matrix");
    long long got = 0;
    while (got < vrows && std::getline(rin, line)) {
      if (skip_line(line)) continue;
      std::istringstream ss(line);
      if (!(ss >> b[(size_t)got])) return fail("bad right-hand side line: " + line);
      ++got;
    }
    if (got < vrows) return fail("right-hand side ends early");
  }
  ab2_problem* p = new ab2_problem();
  p->n = n;
  p->nnz = (long long)ci.size();
  p->nx = n;
  p->ny = 1;
  p->nz = 1;
  p->row_ptr = new int[(size_t)n + 1];
  p->cols = new int[ci.size() + 1];
  p->vals = new double[vals.size() + 1];
  p->x_true = nullptr;
  p->b = new double[(size_t)n + 1];
  p->log10_k = nullptr;
  std::copy(rp.begin(), rp.end(), p->row_ptr);
  std::copy(ci.begin(), ci.end(), p->cols);
  std::copy(vals.begin(), vals.end(), p->vals);
  std::copy(b.begin(), b.end(), p->b);
  *out = p;
  return AB2_OK;
}

int ab2_problem_write_matrix_market(const ab2_problem* p, const char* matrix_path, const char* rhs_path) {
  if (!p || !matrix_path) return fail("null argument");
  {
    std::FILE* f = std::fopen(matrix_path, "w");
    if (!f) return fail(std::string("cannot write ") + matrix_path);
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%%\n%% #rows #cols #nonzeros\n");
    std::fprintf(f, "%d %d %lld\n", p->n, p->n, p->nnz);
    for (int i = 0; i < p->n; ++i)
      for (int k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k)
        std::fprintf(f, "%d %d %.17g\n", i + 1, p->cols[k] + 1, p->vals[k]);
    if (std::fclose(f) != 0) return fail(std::string("write failed: ") + matrix_path);
  }
  if (rhs_path && p->b) {
    std::FILE* f = std::fopen(rhs_path, "w");
    if (!f) return fail(std::string("cannot write ") + rhs_path);
    std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%%\n%d 1\n", p->n);
    for (int i = 0; i < p->n; ++i) std::fprintf(f, "%.17g\n", p->b[i]);
    if (std::fclose(f) != 0) return fail(std::string("write failed: ") + rhs_path);
  }
  return AB2_OK;
}

}  // extern "C"
