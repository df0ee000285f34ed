// formats.cpp -- host readers, converters and partitioners with the reference's
// semantics (SparseP support/matrix.h and support/partition.h), written as
// O(nnz) passes instead of the reference's nested loops.
//
// Every converter produces exactly the arrays the reference converter produces
// for sorted, duplicate-free input (and for duplicates: the reference's
// last-write-wins block fill, spmv/1D/BCSR-nnz/support/matrix.h:300-306).
// Allocation sizes follow the reference (e.g. values get nnz+8 entries,
// spmv/1D/CSR-row/support/matrix.h:121) so reference code that reads the
// padding keeps working on our structs.
#include <algorithm>
#include <type_traits>
#include <new>
#include <cmath>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "sparsep.h"
#include "internal.hpp"

namespace sparsep {

template <typename T>
static T *xcalloc(size_t n) {
  return static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
}

// ---------------------------------------------------------------------------
// .mtx readers
// ---------------------------------------------------------------------------
// readCOOMatrix, spmv/1D/CSR-row/support/matrix.h:44-96 (SoA, padded dims),
// spmv/1D/BCSR-nnz/support/matrix.h:63-110 (SoA, unpadded) and
// spmv/1D/COO-nnz/support/matrix.h:31-83 (AoS).  Tokens are separated by single
// spaces as strtok(line, " ") does; lines whose first token starts with '%' are
// comments; the first other line is "nrows ncols nnz"; values in the file are
// ignored and replaced with (T)(rand()%4+1), one rand() call per entry in file
// order.  Unlike the reference, a missing file, a short file, extra entries or
// 0 / out-of-range indices return SPARSEP_EBADF instead of crashing.
struct MtxEntries {
  uint32_t nrows = 0, ncols = 0, nnz = 0;
  std::vector<uint32_t> r, c;
  std::vector<int> v;  // rand()%4+1
};

static int read_mtx(const char *file, MtxEntries &m) {
  if (!file) return SPARSEP_EINVAL;
  FILE *fp = std::fopen(file, "r");
  if (!fp) return SPARSEP_EBADF;
  char line[1000];
  bool header = false;
  uint64_t i = 0;
  int st = SPARSEP_OK;
  while (std::fgets(line, sizeof line, fp) != nullptr) {
    char *save = nullptr;
    char *tok = strtok_r(line, " ", &save);
    if (!tok) continue;
    if (tok[0] == '%') continue;
    if (!header) {
      char *t2 = strtok_r(nullptr, " ", &save);
      char *t3 = t2 ? strtok_r(nullptr, " ", &save) : nullptr;
      if (!t2 || !t3) { st = SPARSEP_EBADF; break; }
      long a = std::atol(tok), b = std::atol(t2), c = std::atol(t3);
      if (a < 0 || b < 0 || c < 0 || a > 0xFFFFFFF0L || b > 0xFFFFFFF0L || c > 0xFFFFFFF0L) {
        st = SPARSEP_EBADF;
        break;
      }
      m.nrows = (uint32_t)a;
      m.ncols = (uint32_t)b;
      m.nnz = (uint32_t)c;
      m.r.resize(m.nnz);
      m.c.resize(m.nnz);
      m.v.resize(m.nnz);
      header = true;
      continue;
    }
    char *t2 = strtok_r(nullptr, " ", &save);
    if (!t2) { st = SPARSEP_EBADF; break; }
    if (i >= m.nnz) { st = SPARSEP_EBADF; break; }
    long rr = std::atol(tok), cc = std::atol(t2);
    if (rr < 1 || cc < 1 || (uint64_t)rr > m.nrows || (uint64_t)cc > m.ncols) {
      st = SPARSEP_EBADF;
      break;
    }
    m.r[i] = (uint32_t)(rr - 1);
    m.c[i] = (uint32_t)(cc - 1);
    m.v[i] = std::rand() % 4 + 1;
    ++i;
  }
  std::fclose(fp);
  if (st == SPARSEP_OK && (!header || i != m.nnz)) st = SPARSEP_EBADF;
  return st;
}

// ---------------------------------------------------------------------------
// Matrix Market with values (no reference counterpart: the reference reader
// above replaces every value by rand()%4+1).  Coordinate format; real /
// double / integer / pattern fields; general / symmetric / skew-symmetric
// (off-diagonal entries mirrored, negated for skew).  A file without a banner
// is read as real general.  Integer element types take the value rounded to
// the nearest integer, wrapped to the type's width.
// ---------------------------------------------------------------------------
struct MtxValues {
  uint32_t nrows = 0, ncols = 0;
  std::vector<uint32_t> r, c;
  std::vector<double> v;
};

static bool ieq(const char *a, const char *b) {
  for (; *a && *b; ++a, ++b)
    if (std::tolower((unsigned char)*a) != std::tolower((unsigned char)*b)) return false;
  return *a == *b;
}

static int read_mtx_values(const char *file, MtxValues &m) {
  if (!file) return SPARSEP_EINVAL;
  FILE *fp = std::fopen(file, "r");
  if (!fp) return SPARSEP_EBADF;
  char line[4096];
  bool header = false, first = true, pattern = false, sym = false, skew = false;
  uint64_t want = 0, got = 0;
  int st = SPARSEP_OK;
  while (st == SPARSEP_OK && std::fgets(line, sizeof line, fp) != nullptr) {
    if (first && std::strncmp(line, "%%MatrixMarket", 14) == 0) {
      char *save = nullptr, *t[5] = {};
      t[0] = strtok_r(line, " \t\r\n", &save);
      for (int i = 1; i < 5; ++i) t[i] = strtok_r(nullptr, " \t\r\n", &save);
      first = false;
      if (!t[1] || !t[2] || !t[3] || !t[4] || !ieq(t[1], "matrix")) {
        st = SPARSEP_EBADF;
        break;
      }
      if (!ieq(t[2], "coordinate")) { st = SPARSEP_ENOSYS; break; }  // dense array format
      if (ieq(t[3], "pattern")) pattern = true;
      else if (!ieq(t[3], "real") && !ieq(t[3], "double") && !ieq(t[3], "integer")) { st = SPARSEP_ENOSYS; break; }
      if (ieq(t[4], "symmetric")) sym = true;
      else if (ieq(t[4], "skew-symmetric")) sym = skew = true;
      else if (!ieq(t[4], "general")) { st = SPARSEP_ENOSYS; break; }  // hermitian
      continue;
    }
    first = false;
    char *p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (*p == '%' || *p == '\n' || *p == '\r' || *p == 0) continue;
    char *end = nullptr;
    if (!header) {
      const long long a = std::strtoll(p, &end, 10), b = std::strtoll(end, &end, 10), c = std::strtoll(end, &end, 10);
      if (a < 0 || b < 0 || c < 0 || a > 0xFFFFFFF0LL || b > 0xFFFFFFF0LL || c > 0xFFFFFFF0LL) {
        st = SPARSEP_EBADF;
        break;
      }
      m.nrows = (uint32_t)a;
      m.ncols = (uint32_t)b;
      want = (uint64_t)c;
      const uint64_t cap = sym ? 2 * want : want;
      if (cap > 0xFFFFFFF0ull) { st = SPARSEP_ERANGE; break; }
      m.r.reserve(cap);
      m.c.reserve(cap);
      m.v.reserve(cap);
      header = true;
      continue;
    }
    const long long rr = std::strtoll(p, &end, 10);
    char *e2 = nullptr;
    const long long cc = std::strtoll(end, &e2, 10);
    if (e2 == end || rr < 1 || cc < 1 || (uint64_t)rr > m.nrows || (uint64_t)cc > m.ncols || got >= want) {
      st = SPARSEP_EBADF;
      break;
    }
    double v = 1.0;
    if (!pattern) {
      char *e3 = nullptr;
      v = std::strtod(e2, &e3);
      if (e3 == e2) { st = SPARSEP_EBADF; break; }
    }
    m.r.push_back((uint32_t)(rr - 1));
    m.c.push_back((uint32_t)(cc - 1));
    m.v.push_back(v);
    if (sym && rr != cc) {
      if ((uint64_t)cc > m.nrows || (uint64_t)rr > m.ncols) { st = SPARSEP_EBADF; break; }
      m.r.push_back((uint32_t)(cc - 1));
      m.c.push_back((uint32_t)(rr - 1));
      m.v.push_back(skew ? -v : v);
    }
    ++got;
  }
  std::fclose(fp);
  if (st == SPARSEP_OK && (!header || got != want)) st = SPARSEP_EBADF;
  return st;
}

template <typename T> static T from_double(double v) {
  if constexpr (std::is_floating_point<T>::value) {
    return (T)v;
  } else {
    return (T)(typename std::make_unsigned<T>::type)(unsigned long long)std::llround(v);  // wraps
  }
}

template <typename T>
int read_coo_values(const char *file, typename Types<T>::coo **out) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  MtxValues m;
  int st;
  try {
    st = read_mtx_values(file, m);
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  if (st) return st;
  const uint32_t nnz = (uint32_t)m.r.size();
  auto *A = xcalloc<typename Types<T>::coo>(1);
  if (!A) return SPARSEP_ENOMEM;
  A->nrows = m.nrows;
  A->ncols = m.ncols;
  A->nnz = nnz;
  A->rowindx = xcalloc<uint32_t>(nnz ? nnz : 1);
  A->colind = xcalloc<uint32_t>(nnz ? nnz : 1);
  A->values = xcalloc<T>(nnz ? nnz : 1);
  if (!A->rowindx || !A->colind || !A->values) {
    free_coo<T>(A);
    return SPARSEP_ENOMEM;
  }
  for (uint32_t i = 0; i < nnz; ++i) {
    A->rowindx[i] = m.r[i];
    A->colind[i] = m.c[i];
    A->values[i] = from_double<T>(m.v[i]);
  }
  *out = A;
  return SPARSEP_OK;
}

static uint32_t pad_dim(uint32_t n, size_t s) {
  uint32_t g = (uint32_t)(8 / s);
  if (n % g) n += g - n % g;
  return n;
}

template <typename T>
int read_coo(const char *file, bool pad, typename Types<T>::coo **out) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  MtxEntries m;
  int st = read_mtx(file, m);
  if (st) return st;
  auto *A = xcalloc<typename Types<T>::coo>(1);
  if (!A) return SPARSEP_ENOMEM;
  A->nrows = pad ? pad_dim(m.nrows, sizeof(T)) : m.nrows;
  A->ncols = pad ? pad_dim(m.ncols, sizeof(T)) : m.ncols;
  A->nnz = m.nnz;
  A->rowindx = xcalloc<uint32_t>(m.nnz);
  A->colind = xcalloc<uint32_t>(m.nnz);
  A->values = xcalloc<T>(m.nnz);
  if (!A->rowindx || !A->colind || !A->values) {
    free_coo<T>(A);
    return SPARSEP_ENOMEM;
  }
  for (uint32_t i = 0; i < m.nnz; ++i) {
    A->rowindx[i] = m.r[i];
    A->colind[i] = m.c[i];
    A->values[i] = (T)m.v[i];
  }
  *out = A;
  return SPARSEP_OK;
}

template <typename T>
int read_cooe(const char *file, typename Types<T>::cooe **out) {
  if (!out) return SPARSEP_EINVAL;
  *out = nullptr;
  MtxEntries m;
  int st = read_mtx(file, m);
  if (st) return st;
  auto *A = xcalloc<typename Types<T>::cooe>(1);
  if (!A) return SPARSEP_ENOMEM;
  A->nrows = pad_dim(m.nrows, sizeof(T));
  A->ncols = pad_dim(m.ncols, sizeof(T));
  A->nnz = m.nnz;
  A->rows = xcalloc<uint32_t>(A->nrows);
  A->nnzs = xcalloc<typename Types<T>::elem>((size_t)m.nnz + 8);
  if (!A->rows || !A->nnzs) {
    free_cooe<T>(A);
    return SPARSEP_ENOMEM;
  }
  for (uint32_t i = 0; i < m.nnz; ++i) {
    A->nnzs[i].rowind = m.r[i];
    A->nnzs[i].colind = m.c[i];
    // the AoS reader stores rand()%4+1 through an int32_t (matrix.h:59,80)
    A->nnzs[i].val = (T)(int32_t)m.v[i];
  }
  *out = A;
  return SPARSEP_OK;
}

// sortCOOMatrix, spmv/1D/COO-nnz/support/matrix.h:88-125: order by (row, col)
// (glibc qsort is a merge sort here, so equal keys keep input order), then
// rows[r] = entries in row r.
template <typename T>
int sort_cooe(typename Types<T>::cooe *A) {
  if (!A || (A->nnz && !A->nnzs) || (A->nrows && !A->rows)) return SPARSEP_EINVAL;
  using E = typename Types<T>::elem;
  for (uint32_t n = 0; n < A->nnz; ++n)
    if (A->nnzs[n].rowind >= A->nrows || A->nnzs[n].colind >= A->ncols) return SPARSEP_EINVAL;
  std::stable_sort(A->nnzs, A->nnzs + A->nnz, [](const E &a, const E &b) {
    if (a.rowind != b.rowind) return a.rowind < b.rowind;
    return a.colind < b.colind;
  });
  std::memset(A->rows, 0, sizeof(uint32_t) * A->nrows);
  for (uint32_t n = 0; n < A->nnz; ++n) A->rows[A->nnzs[n].rowind]++;
  return SPARSEP_OK;
}

// coo2csr, spmv/1D/CSR-row/support/matrix.h:113-152: stable counting sort by
// row.  rowptr has nrows+2 entries (last one 0), colind nnz+1, values nnz+8.
template <typename T>
int coo2csr(const typename Types<T>::coo *B, typename Types<T>::csr **out) {
  if (!B || !out) return SPARSEP_EINVAL;
  *out = nullptr;
  for (uint32_t i = 0; i < B->nnz; ++i)
    if (B->rowindx[i] >= B->nrows || B->colind[i] >= B->ncols) return SPARSEP_EINVAL;
  auto *A = xcalloc<typename Types<T>::csr>(1);
  if (!A) return SPARSEP_ENOMEM;
  A->nrows = B->nrows;
  A->ncols = B->ncols;
  A->nnz = B->nnz;
  A->rowptr = xcalloc<uint32_t>((size_t)A->nrows + 2);
  A->colind = xcalloc<uint32_t>((size_t)A->nnz + 1);
  A->values = xcalloc<T>((size_t)A->nnz + 8);
  if (!A->rowptr || !A->colind || !A->values) {
    free_csr<T>(A);
    return SPARSEP_ENOMEM;
  }
  for (uint32_t i = 0; i < B->nnz; ++i) A->rowptr[B->rowindx[i] + 1]++;
  for (uint32_t r = 0; r < A->nrows; ++r) A->rowptr[r + 1] += A->rowptr[r];
  std::vector<uint32_t> next(A->rowptr, A->rowptr + A->nrows + (A->nrows ? 0 : 1));
  for (uint32_t i = 0; i < B->nnz; ++i) {
    uint32_t k = next[B->rowindx[i]]++;
    A->colind[k] = B->colind[i];
    A->values[k] = B->values[i];
  }
  *out = A;
  return SPARSEP_OK;
}

// Per-block-row block discovery shared by csr2bcsr and the 2D block converters:
// rows [row0, row0+nr) of a CSR whose entries k live at [ptr[i]+base, ptr[i+1]+base)
// are cut into rb x cb blocks; blocks of one block row come out sorted by block
// column (sortBCSRMatrix, spmv/1D/BCSR-nnz/support/matrix.h:460-469, leaves them so;
// the 2D converters keep discovery order, see sort flag), a later duplicate
// entry overwrites an earlier one as the reference's block fill does.
template <typename T>
struct BlockBuilder {
  uint32_t rb, cb, nbc;
  std::vector<uint32_t> slot;  // block col -> index into cur (or UINT32_MAX)
  std::vector<uint32_t> cur;   // block cols touched in this block row, discovery order
  std::vector<uint32_t> browptr, bcolind;
  std::vector<T> bval;
  BlockBuilder(uint32_t rb_, uint32_t cb_, uint32_t nbc_)
      : rb(rb_), cb(cb_), nbc(nbc_), slot(nbc_, UINT32_MAX) { browptr.push_back(0); }

  // rows: callback giving [begin, end) and column/value accessors
  template <typename RowFn>
  void block_row(uint32_t nrows_here, RowFn &&row, bool sort) {
    cur.clear();
    for (uint32_t di = 0; di < nrows_here; ++di) {
      row(di, [&](uint32_t j, T) {
        uint32_t J = j / cb;
        if (slot[J] == UINT32_MAX) {
          slot[J] = (uint32_t)cur.size();
          cur.push_back(J);
        }
      });
    }
    std::vector<uint32_t> order(cur.size());
    for (size_t i = 0; i < cur.size(); ++i) order[i] = (uint32_t)i;
    if (sort) std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cur[a] < cur[b]; });
    std::vector<uint32_t> pos(cur.size());
    size_t base = bcolind.size();
    for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = (uint32_t)(base + i);
    for (size_t i = 0; i < order.size(); ++i) bcolind.push_back(cur[order[i]]);
    bval.resize((bcolind.size()) * (size_t)rb * cb, T(0));
    for (uint32_t di = 0; di < nrows_here; ++di) {
      row(di, [&](uint32_t j, T v) {
        uint32_t J = j / cb;
        size_t b = pos[slot[J]];
        bval[b * rb * cb + (size_t)di * cb + (j - J * cb)] = v;
      });
    }
    for (uint32_t J : cur) slot[J] = UINT32_MAX;
    browptr.push_back((uint32_t)bcolind.size());
  }
};

template <typename T>
static uint32_t count_nonzero(const T *b, size_t n) {
  uint32_t c = 0;
  for (size_t i = 0; i < n; ++i) c += (b[i] != T(0));
  return c;
}

// csr2bcsr + sortBCSRMatrix + countNNZperBlockBCSRMatrix,
// spmv/1D/BCSR-nnz/support/matrix.h:202-485.  browptr has num_block_rows+2
// entries, bcolind num_blocks+1, bval (num_blocks+1)*rb*cb (calloc'd),
// nnz_per_block counts nonzero VALUES (matrix.h:474-485).
template <typename T>
int csr2bcsr(const typename Types<T>::csr *A, uint32_t rb, uint32_t cb,
             typename Types<T>::bcsr **out) {
  if (!A || !out || rb == 0 || cb == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  uint32_t nbr = (uint32_t)(((uint64_t)A->nrows + rb - 1) / rb);
  uint32_t nbc = (uint32_t)(((uint64_t)A->ncols + cb - 1) / cb);
  for (uint32_t k = 0; k < A->nnz; ++k)
    if (A->colind[k] >= A->ncols) return SPARSEP_EINVAL;
  BlockBuilder<T> bb(rb, cb, nbc);
  for (uint32_t I = 0; I < nbr; ++I) {
    uint32_t r0 = I * rb;
    uint32_t here = std::min<uint32_t>(rb, A->nrows - r0);
    bb.block_row(
        here,
        [&](uint32_t di, auto &&f) {
          for (uint32_t k = A->rowptr[r0 + di]; k < A->rowptr[r0 + di + 1]; ++k) f(A->colind[k], A->values[k]);
        },
        true);
  }
  auto *B = xcalloc<typename Types<T>::bcsr>(1);
  if (!B) return SPARSEP_ENOMEM;
  uint64_t nb = bb.bcolind.size();
  B->row_block_size = rb;
  B->col_block_size = cb;
  B->num_block_rows = nbr;
  B->num_block_cols = nbc;
  B->num_blocks = nb;
  B->num_rows_left = A->nrows % rb;
  B->nrows = A->nrows;
  B->ncols = A->ncols;
  B->nnz = A->nnz;
  B->browptr = xcalloc<uint32_t>((size_t)nbr + 2);
  B->bcolind = xcalloc<uint32_t>(nb + 1);
  B->bval = xcalloc<T>((nb + 1) * rb * cb);
  B->nnz_per_block = xcalloc<uint32_t>(nb);
  if (!B->browptr || !B->bcolind || !B->bval || !B->nnz_per_block) {
    free_bcsr<T>(B);
    return SPARSEP_ENOMEM;
  }
  std::memcpy(B->browptr, bb.browptr.data(), sizeof(uint32_t) * (nbr + 1));
  if (nb) std::memcpy(B->bcolind, bb.bcolind.data(), sizeof(uint32_t) * nb);
  if (nb) std::memcpy(B->bval, bb.bval.data(), sizeof(T) * nb * rb * cb);
  for (uint64_t b = 0; b < nb; ++b) B->nnz_per_block[b] = count_nonzero(B->bval + b * rb * cb, (size_t)rb * cb);
  *out = B;
  return SPARSEP_OK;
}

// bcsr2bcoo, spmv/1D/BCOO-nnz/support/matrix.h:549-578.
template <typename T>
int bcsr2bcoo(const typename Types<T>::bcsr *A, typename Types<T>::bcoo **out) {
  if (!A || !out) return SPARSEP_EINVAL;
  *out = nullptr;
  auto *B = xcalloc<typename Types<T>::bcoo>(1);
  if (!B) return SPARSEP_ENOMEM;
  B->row_block_size = A->row_block_size;
  B->col_block_size = A->col_block_size;
  B->num_block_rows = A->num_block_rows;
  B->num_block_cols = A->num_block_cols;
  B->num_blocks = A->num_blocks;
  B->num_rows_left = A->num_rows_left;
  B->nrows = A->nrows;
  B->ncols = A->ncols;
  B->nnz = A->nnz;
  size_t bs = (size_t)A->row_block_size * A->col_block_size;
  B->bind = xcalloc<sparsep_bind>(A->num_blocks);
  B->bval = xcalloc<T>((A->num_blocks + 1) * bs);
  B->nnz_per_block = xcalloc<uint32_t>(A->num_blocks);
  if (!B->bind || !B->bval || !B->nnz_per_block) {
    free_bcoo<T>(B);
    return SPARSEP_ENOMEM;
  }
  for (uint32_t n = 0; n < A->num_block_rows; ++n)
    for (uint32_t i = A->browptr[n]; i < A->browptr[n + 1]; ++i) {
      B->bind[i].rowind = n;
      B->bind[i].colind = A->bcolind[i];
    }
  std::memcpy(B->bval, A->bval, sizeof(T) * (A->num_blocks + 1) * bs);
  if (A->num_blocks) std::memcpy(B->nnz_per_block, A->nnz_per_block, sizeof(uint32_t) * A->num_blocks);
  *out = B;
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// 2D converters (input: sorted AoS COO)
// ---------------------------------------------------------------------------
template <typename T>
static int check_cooe(const typename Types<T>::cooe *C) {
  if (!C || (C->nnz && !C->nnzs)) return SPARSEP_EINVAL;
  for (uint32_t n = 0; n < C->nnz; ++n) {
    if (C->nnzs[n].rowind >= C->nrows || C->nnzs[n].colind >= C->ncols) return SPARSEP_EINVAL;
    if (n && (C->nnzs[n].rowind < C->nnzs[n - 1].rowind ||
              (C->nnzs[n].rowind == C->nnzs[n - 1].rowind && C->nnzs[n].colind < C->nnzs[n - 1].colind)))
      return SPARSEP_EINVAL;  // the reference converters assume sortCOOMatrix ran
  }
  return SPARSEP_OK;
}

static uint32_t ceil_div32(uint32_t a, uint32_t b) { return a / b + (a % b != 0); }

// Greedy nnz split of the columns into V stripes, coo2bdcsr
// spmv/2D/BDCSR/support/matrix.h:176-229: a stripe closes at the first column
// where its count reaches nnz/V; the last stripe takes every column left.
static void bd_stripes(const std::vector<uint32_t> &per_col, uint32_t ncols, uint64_t nnz, uint32_t V,
                       std::vector<uint32_t> &widths, std::vector<uint32_t> &per_part, uint32_t &maxw) {
  widths.assign(V + 1, 0);
  per_part.assign(V, 0);
  uint32_t nps = (uint32_t)(nnz / V);
  uint32_t cur = 0, cnt = 0;
  for (uint32_t t = 0; t < ncols; ++t) {
    cur += per_col[t];
    if (cur >= nps) {
      ++cnt;
      if (cnt <= V) {
        widths[cnt] = t + 1;
        per_part[cnt - 1] = cur;
      }
      cur = 0;
    }
  }
  // remaining columns (and everything past the V-th cut) go to the last stripe
  if (cnt < V) {
    widths[cnt + 1 <= V ? cnt + 1 : V] = ncols;
    if (cnt + 1 <= V) per_part[cnt] = cur;
    cnt = cnt + 1;
  }
  widths[V] = ncols;
  for (uint32_t t = cnt + 1; t <= V; ++t) {
    widths[t] = ncols;
    per_part[t - 1] = 0;
  }
  // recount exactly (the reference's totals assert, matrix.h:228)
  std::vector<uint32_t> exact(V, 0);
  uint32_t c = 0;
  for (uint32_t t = 0; t < ncols; ++t) {
    while (c + 1 < V && widths[c + 1] <= t) ++c;
    exact[c] += per_col[t];
  }
  per_part = exact;
  maxw = 0;
  for (uint32_t t = 0; t < V; ++t) maxw = std::max(maxw, widths[t + 1] - widths[t]);
}

static uint32_t stripe_of(const std::vector<uint32_t> &widths, uint32_t col) {
  // first p with widths[p+1] > col (the reference's linear scan, matrix.h:236-238)
  return (uint32_t)(std::upper_bound(widths.begin() + 1, widths.end(), col) - (widths.begin() + 1));
}

template <typename T>
int cooe2dcsr(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::dcsr **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::dcsr>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = H * V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  D->tile_height = ceil_div32(C->nrows, H);
  D->tile_width = ceil_div32(C->ncols, V);
  uint32_t th = D->tile_height, tw = D->tile_width;
  uint64_t P = (uint64_t)H * V;
  D->nnzs_per_partition = xcalloc<uint32_t>(P);
  D->drowptr = xcalloc<uint32_t>(((size_t)th + 2) * P);
  D->dcolind = xcalloc<uint32_t>((size_t)C->nnz + 2);
  D->dval = xcalloc<T>((size_t)C->nnz + 8);
  if (!D->nnzs_per_partition || !D->drowptr || !D->dcolind || !D->dval || th == 0 || tw == 0) {
    free_dcsr<T>(D);
    return th == 0 || tw == 0 ? SPARSEP_EINVAL : SPARSEP_ENOMEM;
  }
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pr = C->nnzs[n].rowind / th, pc = C->nnzs[n].colind / tw;
    uint64_t p = (uint64_t)pr * V + pc;
    D->nnzs_per_partition[p]++;
    D->drowptr[p * (th + 1) + (C->nnzs[n].rowind - pr * th)]++;
  }
  for (uint64_t p = 0; p < P; ++p) {
    uint32_t s = 0;
    for (uint32_t r = 0; r < th; ++r) {
      uint32_t c = D->drowptr[p * (th + 1) + r];
      D->drowptr[p * (th + 1) + r] = s;
      s += c;
    }
    D->drowptr[p * (th + 1) + th] = s;
  }
  std::vector<uint64_t> pos(P, 0);
  uint64_t tot = 0;
  for (uint64_t p = 0; p < P; ++p) { pos[p] = tot; tot += D->nnzs_per_partition[p]; }
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pr = C->nnzs[n].rowind / th, pc = C->nnzs[n].colind / tw;
    uint64_t k = pos[(uint64_t)pr * V + pc]++;
    D->dcolind[k] = C->nnzs[n].colind - pc * tw;
    D->dval[k] = C->nnzs[n].val;
  }
  *out = D;
  return SPARSEP_OK;
}

// Shared body of coo2rbdcsr (spmv/2D/RBDCSR/support/matrix.h:159-223) and
// coo2bdcsr (spmv/2D/BDCSR/support/matrix.h:161-282): per-stripe full-height CSR
// with stripe-local columns, stripes concatenated.
template <typename T>
static int stripe_csr(const typename Types<T>::cooe *C, uint32_t V, const std::vector<uint32_t> &widths,
                      uint32_t *&drowptr, uint32_t *&dcolind, T *&dval, std::vector<uint32_t> &per_part) {
  uint32_t nr = C->nrows;
  drowptr = xcalloc<uint32_t>(((size_t)nr + 2) * V);
  dcolind = xcalloc<uint32_t>((size_t)C->nnz + 2);
  dval = xcalloc<T>((size_t)C->nnz + 8);
  if (!drowptr || !dcolind || !dval) return SPARSEP_ENOMEM;
  per_part.assign(V, 0);
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pc = stripe_of(widths, C->nnzs[n].colind);
    per_part[pc]++;
    drowptr[(size_t)pc * (nr + 1) + C->nnzs[n].rowind]++;
  }
  for (uint32_t p = 0; p < V; ++p) {
    uint32_t s = 0;
    for (uint32_t r = 0; r < nr; ++r) {
      uint32_t c = drowptr[(size_t)p * (nr + 1) + r];
      drowptr[(size_t)p * (nr + 1) + r] = s;
      s += c;
    }
    drowptr[(size_t)p * (nr + 1) + nr] = s;
  }
  std::vector<uint64_t> pos(V, 0);
  uint64_t tot = 0;
  for (uint32_t p = 0; p < V; ++p) { pos[p] = tot; tot += per_part[p]; }
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pc = stripe_of(widths, C->nnzs[n].colind);
    uint64_t k = pos[pc]++;
    dcolind[k] = C->nnzs[n].colind - widths[pc];
    dval[k] = C->nnzs[n].val;
  }
  return SPARSEP_OK;
}

static std::vector<uint32_t> equal_widths(uint32_t ncols, uint32_t V, uint32_t tw) {
  std::vector<uint32_t> w(V + 1);
  for (uint32_t p = 0; p <= V; ++p) w[p] = (uint32_t)std::min<uint64_t>((uint64_t)p * tw, ncols);
  w[V] = std::max<uint32_t>(w[V], ncols);
  return w;
}

template <typename T>
int cooe2rbdcsr(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::rbdcsr **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::rbdcsr>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  D->tile_width = ceil_div32(C->ncols, V);
  if (D->tile_width == 0) { free_rbdcsr<T>(D); return SPARSEP_EINVAL; }
  std::vector<uint32_t> per;
  auto w = equal_widths(C->ncols, V, D->tile_width);
  int st = stripe_csr<T>(C, V, w, D->drowptr, D->dcolind, D->dval, per);
  D->nnzs_per_vert_partition = xcalloc<uint32_t>(V);
  if (st || !D->nnzs_per_vert_partition) { free_rbdcsr<T>(D); return SPARSEP_ENOMEM; }
  std::memcpy(D->nnzs_per_vert_partition, per.data(), sizeof(uint32_t) * V);
  *out = D;
  return SPARSEP_OK;
}

template <typename T>
int cooe2bdcsr(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::bdcsr **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::bdcsr>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  std::vector<uint32_t> per_col(C->ncols, 0), widths, per;
  for (uint32_t n = 0; n < C->nnz; ++n) per_col[C->nnzs[n].colind]++;
  bd_stripes(per_col, C->ncols, C->nnz, V, widths, per, D->max_tile_width);
  D->vert_tile_widths = xcalloc<uint32_t>((size_t)V + 1);
  D->nnzs_per_column = xcalloc<uint32_t>(C->ncols);
  D->nnzs_per_vert_partition = xcalloc<uint32_t>(V);
  std::vector<uint32_t> per2;
  int st = stripe_csr<T>(C, V, widths, D->drowptr, D->dcolind, D->dval, per2);
  if (st || !D->vert_tile_widths || !D->nnzs_per_column || !D->nnzs_per_vert_partition) {
    free_bdcsr<T>(D);
    return SPARSEP_ENOMEM;
  }
  std::memcpy(D->vert_tile_widths, widths.data(), sizeof(uint32_t) * (V + 1));
  if (C->ncols) std::memcpy(D->nnzs_per_column, per_col.data(), sizeof(uint32_t) * C->ncols);
  std::memcpy(D->nnzs_per_vert_partition, per2.data(), sizeof(uint32_t) * V);
  *out = D;
  return SPARSEP_OK;
}

// coo2dcoo, spmv/2D/DCOO/support/matrix.h:158-217: equal tiles, tile-local
// row and column, tiles concatenated in (row-tile, col-tile) order.
template <typename T>
int cooe2dcoo(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::dcoo **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::dcoo>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = H * V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  D->tile_height = ceil_div32(C->nrows, H);
  D->tile_width = ceil_div32(C->ncols, V);
  uint64_t P = (uint64_t)H * V;
  D->nnzs_per_partition = xcalloc<uint32_t>(P);
  D->nnzs = xcalloc<typename Types<T>::elem>((size_t)C->nnz + 2);
  if (!D->nnzs_per_partition || !D->nnzs || !D->tile_height || !D->tile_width) {
    free_dcoo<T>(D);
    return SPARSEP_ENOMEM;
  }
  uint32_t th = D->tile_height, tw = D->tile_width;
  for (uint32_t n = 0; n < C->nnz; ++n)
    D->nnzs_per_partition[(uint64_t)(C->nnzs[n].rowind / th) * V + C->nnzs[n].colind / tw]++;
  std::vector<uint64_t> pos(P);
  uint64_t tot = 0;
  for (uint64_t p = 0; p < P; ++p) { pos[p] = tot; tot += D->nnzs_per_partition[p]; }
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pr = C->nnzs[n].rowind / th, pc = C->nnzs[n].colind / tw;
    uint64_t k = pos[(uint64_t)pr * V + pc]++;
    D->nnzs[k].rowind = C->nnzs[n].rowind - pr * th;
    D->nnzs[k].colind = C->nnzs[n].colind - pc * tw;
    D->nnzs[k].val = C->nnzs[n].val;
  }
  *out = D;
  return SPARSEP_OK;
}

// Shared body of coo2rbdcoo (spmv/2D/RBDCOO/support/matrix.h:157) and coo2bdcoo
// (spmv/2D/BDCOO/support/matrix.h:158): stripes concatenated, GLOBAL row index,
// stripe-local column.
template <typename T>
static int stripe_coo(const typename Types<T>::cooe *C, uint32_t V, const std::vector<uint32_t> &widths,
                      typename Types<T>::elem *&nnzs, std::vector<uint32_t> &per_part) {
  nnzs = xcalloc<typename Types<T>::elem>((size_t)C->nnz + 2);
  if (!nnzs) return SPARSEP_ENOMEM;
  per_part.assign(V, 0);
  for (uint32_t n = 0; n < C->nnz; ++n) per_part[stripe_of(widths, C->nnzs[n].colind)]++;
  std::vector<uint64_t> pos(V);
  uint64_t tot = 0;
  for (uint32_t p = 0; p < V; ++p) { pos[p] = tot; tot += per_part[p]; }
  for (uint32_t n = 0; n < C->nnz; ++n) {
    uint32_t pc = stripe_of(widths, C->nnzs[n].colind);
    uint64_t k = pos[pc]++;
    nnzs[k].rowind = C->nnzs[n].rowind;
    nnzs[k].colind = C->nnzs[n].colind - widths[pc];
    nnzs[k].val = C->nnzs[n].val;
  }
  return SPARSEP_OK;
}

template <typename T>
int cooe2rbdcoo(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::rbdcoo **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::rbdcoo>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  D->tile_width = ceil_div32(C->ncols, V);
  if (!D->tile_width) { free_rbdcoo<T>(D); return SPARSEP_EINVAL; }
  std::vector<uint32_t> per;
  int st = stripe_coo<T>(C, V, equal_widths(C->ncols, V, D->tile_width), D->nnzs, per);
  D->nnzs_per_vert_partition = xcalloc<uint32_t>(V);
  if (st || !D->nnzs_per_vert_partition) { free_rbdcoo<T>(D); return SPARSEP_ENOMEM; }
  std::memcpy(D->nnzs_per_vert_partition, per.data(), sizeof(uint32_t) * V);
  *out = D;
  return SPARSEP_OK;
}

template <typename T>
int cooe2bdcoo(const typename Types<T>::cooe *C, uint32_t H, uint32_t V, typename Types<T>::bdcoo **out) {
  if (!out || H == 0 || V == 0) return SPARSEP_EINVAL;
  *out = nullptr;
  if (int st = check_cooe<T>(C)) return st;
  auto *D = xcalloc<typename Types<T>::bdcoo>(1);
  if (!D) return SPARSEP_ENOMEM;
  D->nrows = C->nrows;
  D->ncols = C->ncols;
  D->nnz = C->nnz;
  D->npartitions = V;
  D->horz_partitions = H;
  D->vert_partitions = V;
  std::vector<uint32_t> per_col(C->ncols, 0), widths, per, per2;
  for (uint32_t n = 0; n < C->nnz; ++n) per_col[C->nnzs[n].colind]++;
  bd_stripes(per_col, C->ncols, C->nnz, V, widths, per, D->max_tile_width);
  D->vert_tile_widths = xcalloc<uint32_t>((size_t)V + 1);
  D->nnzs_per_vert_partition = xcalloc<uint32_t>(V);
  D->nnzs_per_column = xcalloc<uint32_t>(C->ncols);
  int st = stripe_coo<T>(C, V, widths, D->nnzs, per2);
  if (st || !D->vert_tile_widths || !D->nnzs_per_vert_partition || !D->nnzs_per_column) {
    free_bdcoo<T>(D);
    return SPARSEP_ENOMEM;
  }
  std::memcpy(D->vert_tile_widths, widths.data(), sizeof(uint32_t) * (V + 1));
  std::memcpy(D->nnzs_per_vert_partition, per2.data(), sizeof(uint32_t) * V);
  if (C->ncols) std::memcpy(D->nnzs_per_column, per_col.data(), sizeof(uint32_t) * C->ncols);
  *out = D;
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// 2D block converters: each tile's CSR cut into blocks with tile-local block
// rows/cols.  D tiles: dcsr2dbcsr, spmv/2D/DBCSR/support/matrix.h:278-518 (blocks
// in discovery order, as the reference's DBCSR path does not sort them);
// DBCOO sorts them (sortDBCSRMatrix before dbcsr2dbcoo, spmv/2D/DBCOO/host/app.c:140).
// RBD/BD stripes: rbdcsr2rbdbcsr (spmv/2D/RBDBCSR-nnz/support/matrix.h:270),
// bdcsr2bdbcsr (spmv/2D/BDBCSR-nnz/support/matrix.h:334).
// ---------------------------------------------------------------------------
template <typename T>
struct TiledBlocks {
  std::vector<uint32_t> browptr, bcolind, blocks_per, nnz_per_block;
  std::vector<T> bval;
  uint32_t nbr = 0, nbc = 0, left = 0;
};

// tiles: P tiles, each with local rowptr at rowptr + t*stride (nrows_t rows),
// entries offset by nnz_base[t].
template <typename T>
static void build_tiled_blocks(uint32_t P, uint32_t nrows_t, uint32_t width_max, uint32_t stride,
                               const uint32_t *rowptr, const std::vector<uint64_t> &nnz_base,
                               const uint32_t *colind, const T *val, uint32_t rb, uint32_t cb, bool sort,
                               TiledBlocks<T> &tb) {
  tb.nbr = (uint32_t)(((uint64_t)nrows_t + rb - 1) / rb);
  tb.nbc = (uint32_t)(((uint64_t)width_max + cb - 1) / cb);
  tb.left = nrows_t % rb;
  tb.browptr.assign((size_t)P * (tb.nbr + 2), 0);
  tb.blocks_per.assign(P, 0);
  for (uint32_t p = 0; p < P; ++p) {
    BlockBuilder<T> bb(rb, cb, std::max<uint32_t>(tb.nbc, 1));
    const uint32_t *rp = rowptr + (size_t)p * stride;
    uint64_t base = nnz_base[p];
    for (uint32_t I = 0; I < tb.nbr; ++I) {
      uint32_t here = std::min<uint32_t>(rb, nrows_t - I * rb);
      bb.block_row(
          here,
          [&](uint32_t di, auto &&f) {
            uint32_t i = I * rb + di;
            for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) f(colind[base + k], val[base + k]);
          },
          sort);
    }
    std::memcpy(&tb.browptr[(size_t)p * (tb.nbr + 1)], bb.browptr.data(), sizeof(uint32_t) * (tb.nbr + 1));
    tb.blocks_per[p] = (uint32_t)bb.bcolind.size();
    tb.bcolind.insert(tb.bcolind.end(), bb.bcolind.begin(), bb.bcolind.end());
    tb.bval.insert(tb.bval.end(), bb.bval.begin(), bb.bval.end());
  }
  size_t bs = (size_t)rb * cb;
  tb.nnz_per_block.resize(tb.bcolind.size());
  for (size_t b = 0; b < tb.bcolind.size(); ++b) tb.nnz_per_block[b] = count_nonzero(&tb.bval[b * bs], bs);
}

template <typename B, typename T>
static int fill_block_arrays(B *X, const TiledBlocks<T> &tb, uint32_t P, uint32_t rb, uint32_t cb, bool coo) {
  size_t nb = tb.bcolind.size(), bs = (size_t)rb * cb;
  X->nblocks = (uint32_t)nb;
  X->row_block_size = rb;
  X->col_block_size = cb;
  X->num_block_rows = tb.nbr;
  X->num_block_cols = tb.nbc;
  X->num_rows_left = tb.left;
  X->bval = xcalloc<T>((nb + 1) * bs);
  X->nnz_per_block = xcalloc<uint32_t>(nb);
  if (!X->bval || !X->nnz_per_block) return SPARSEP_ENOMEM;
  if (nb) std::memcpy(X->bval, tb.bval.data(), sizeof(T) * nb * bs);
  if (nb) std::memcpy(X->nnz_per_block, tb.nnz_per_block.data(), sizeof(uint32_t) * nb);
  (void)P;
  (void)coo;
  return SPARSEP_OK;
}

template <typename X>
static void set_bcsr_index(X *D, const std::vector<uint32_t> &browptr, const std::vector<uint32_t> &bcolind,
                           uint32_t P, uint32_t nbr, int &st) {
  D->browptr = xcalloc<uint32_t>((size_t)P * (nbr + 2));
  D->bcolind = xcalloc<uint32_t>(bcolind.size() + 1);
  if (!D->browptr || !D->bcolind) { st = SPARSEP_ENOMEM; return; }
  std::memcpy(D->browptr, browptr.data(), sizeof(uint32_t) * browptr.size());
  if (!bcolind.empty()) std::memcpy(D->bcolind, bcolind.data(), sizeof(uint32_t) * bcolind.size());
}

template <typename X>
static void set_bcoo_index(X *D, const std::vector<uint32_t> &browptr, const std::vector<uint32_t> &bcolind,
                           const std::vector<uint32_t> &blocks_per, uint32_t P, uint32_t nbr, int &st) {
  D->bind = xcalloc<sparsep_bind>(bcolind.size() + 1);
  if (!D->bind) { st = SPARSEP_ENOMEM; return; }
  size_t off = 0;
  for (uint32_t p = 0; p < P; ++p) {
    const uint32_t *bp = &browptr[(size_t)p * (nbr + 1)];
    for (uint32_t n = 0; n < nbr; ++n)
      for (uint32_t i = bp[n]; i < bp[n + 1]; ++i) {
        D->bind[off + i].rowind = n;
        D->bind[off + i].colind = bcolind[off + i];
      }
    off += blocks_per[p];
  }
}

template <typename T, bool COO>
static int dcsr2dblock(const typename Types<T>::dcsr *A, uint32_t rb, uint32_t cb, void **out) {
  if (!A || !out || !rb || !cb) return SPARSEP_EINVAL;
  *out = nullptr;
  uint32_t P = A->npartitions;
  std::vector<uint64_t> base(P);
  uint64_t tot = 0;
  for (uint32_t p = 0; p < P; ++p) { base[p] = tot; tot += A->nnzs_per_partition[p]; }
  TiledBlocks<T> tb;
  build_tiled_blocks<T>(P, A->tile_height, A->tile_width, A->tile_height + 1, A->drowptr, base, A->dcolind,
                        A->dval, rb, cb, /*sort=*/COO, tb);
  int st = SPARSEP_OK;
  if (!COO) {
    auto *D = xcalloc<typename Types<T>::dbcsr>(1);
    if (!D) return SPARSEP_ENOMEM;
    D->nrows = A->nrows; D->ncols = A->ncols; D->nnz = A->nnz; D->npartitions = P;
    D->horz_partitions = A->horz_partitions; D->vert_partitions = A->vert_partitions;
    D->tile_height = A->tile_height; D->tile_width = A->tile_width;
    D->nnzs_per_partition = xcalloc<uint32_t>(P);
    D->blocks_per_partition = xcalloc<uint32_t>(P);
    if (!D->nnzs_per_partition || !D->blocks_per_partition) st = SPARSEP_ENOMEM;
    if (!st) {
      std::memcpy(D->nnzs_per_partition, A->nnzs_per_partition, sizeof(uint32_t) * P);
      std::memcpy(D->blocks_per_partition, tb.blocks_per.data(), sizeof(uint32_t) * P);
      st = fill_block_arrays(D, tb, P, rb, cb, false);
    }
    if (!st) set_bcsr_index(D, tb.browptr, tb.bcolind, P, tb.nbr, st);
    if (st) { free_dbcsr<T>(D); return st; }
    *out = D;
  } else {
    auto *D = xcalloc<typename Types<T>::dbcoo>(1);
    if (!D) return SPARSEP_ENOMEM;
    D->nrows = A->nrows; D->ncols = A->ncols; D->nnz = A->nnz; D->npartitions = P;
    D->horz_partitions = A->horz_partitions; D->vert_partitions = A->vert_partitions;
    D->tile_height = A->tile_height; D->tile_width = A->tile_width;
    D->nnzs_per_partition = xcalloc<uint32_t>(P);
    D->blocks_per_partition = xcalloc<uint32_t>(P);
    if (!D->nnzs_per_partition || !D->blocks_per_partition) st = SPARSEP_ENOMEM;
    if (!st) {
      std::memcpy(D->nnzs_per_partition, A->nnzs_per_partition, sizeof(uint32_t) * P);
      std::memcpy(D->blocks_per_partition, tb.blocks_per.data(), sizeof(uint32_t) * P);
      st = fill_block_arrays(D, tb, P, rb, cb, true);
    }
    if (!st) set_bcoo_index(D, tb.browptr, tb.bcolind, tb.blocks_per, P, tb.nbr, st);
    if (st) { free_dbcoo<T>(D); return st; }
    *out = D;
  }
  return SPARSEP_OK;
}

// Stripe (RBD/BD) block converters: each stripe is a full-height CSR.
template <typename T, typename SRC, typename DST, bool COO, bool BD>
static int stripe2block(const SRC *A, uint32_t rb, uint32_t cb, DST **out) {
  if (!A || !out || !rb || !cb) return SPARSEP_EINVAL;
  *out = nullptr;
  uint32_t V = A->vert_partitions;
  std::vector<uint64_t> base(V);
  uint64_t tot = 0;
  for (uint32_t p = 0; p < V; ++p) { base[p] = tot; tot += A->nnzs_per_vert_partition[p]; }
  uint32_t wmax;
  if constexpr (BD) wmax = A->max_tile_width; else wmax = A->tile_width;
  TiledBlocks<T> tb;
  // the BCSR stripe paths keep discovery order; the BCOO ones sort first
  // (sortRBDBCSRMatrix / sortBDBCSRMatrix, spmv/2D/RBDBCOO-nnz/host/app.c:149)
  build_tiled_blocks<T>(V, A->nrows, wmax, A->nrows + 1, A->drowptr, base, A->dcolind, A->dval, rb, cb, COO, tb);
  auto *D = xcalloc<DST>(1);
  if (!D) return SPARSEP_ENOMEM;
  int st = SPARSEP_OK;
  D->nrows = A->nrows; D->ncols = A->ncols; D->nnz = A->nnz; D->npartitions = V;
  D->horz_partitions = A->horz_partitions; D->vert_partitions = V;
  D->nnzs_per_vert_partition = xcalloc<uint32_t>(V);
  D->blocks_per_vert_partition = xcalloc<uint32_t>(V);
  if (!D->nnzs_per_vert_partition || !D->blocks_per_vert_partition) st = SPARSEP_ENOMEM;
  if (!st) {
    std::memcpy(D->nnzs_per_vert_partition, A->nnzs_per_vert_partition, sizeof(uint32_t) * V);
    std::memcpy(D->blocks_per_vert_partition, tb.blocks_per.data(), sizeof(uint32_t) * V);
  }
  if constexpr (BD) {
    D->max_tile_width = A->max_tile_width;
    D->vert_tile_widths = xcalloc<uint32_t>((size_t)V + 1);
    D->nnzs_per_column = xcalloc<uint32_t>(A->ncols);
    if (!D->vert_tile_widths || !D->nnzs_per_column) st = SPARSEP_ENOMEM;
    if (!st) {
      std::memcpy(D->vert_tile_widths, A->vert_tile_widths, sizeof(uint32_t) * (V + 1));
      if (A->ncols) std::memcpy(D->nnzs_per_column, A->nnzs_per_column, sizeof(uint32_t) * A->ncols);
    }
  } else {
    D->tile_width = A->tile_width;
  }
  if (!st) st = fill_block_arrays(D, tb, V, rb, cb, COO);
  if (!st) {
    if constexpr (COO) set_bcoo_index(D, tb.browptr, tb.bcolind, tb.blocks_per, V, tb.nbr, st);
    else set_bcsr_index(D, tb.browptr, tb.bcolind, V, tb.nbr, st);
  }
  if (st) { free_any(D); return st; }
  *out = D;
  return SPARSEP_OK;
}

// ---------------------------------------------------------------------------
// Partitioners
// ---------------------------------------------------------------------------
// Greedy prefix split shared by partition_by_nnz (spmv/1D/CSR-nnz/support/partition.h:35-77)
// and the per-stripe 2D splits (spmv/2D/BDCSR/support/partition.h:47-91): walk the
// units, close a part as soon as its weight reaches total/parts, merge what is
// left into the last part, pad with empty trailing parts.
void greedy_split(const uint64_t *prefix, uint32_t n, uint32_t parts, uint32_t *split) {
  split[0] = 0;
  if (parts == 1) { split[1] = n; return; }
  uint64_t total = prefix[n] - prefix[0];
  uint32_t nps = (uint32_t)(total / parts);
  uint64_t cur = 0;
  uint32_t cnt = 0;
  for (uint32_t i = 0; i < n; ++i) {
    cur += prefix[i + 1] - prefix[i];
    if (cur >= nps) {
      ++cnt;
      if (cnt <= parts) split[cnt] = i + 1;
      cur = 0;
    }
  }
  if (cur < nps && cnt <= parts) {
    ++cnt;
    if (cnt <= parts) split[cnt] = n;
  }
  if (cnt > parts) split[parts] = n;
  for (uint32_t i = cnt + 1; i <= parts; ++i) split[i] = n;
}

// BCSR/BCOO block-row variants (spmv/1D/BCSR-nnz/support/partition.h:39-112):
// the running counters reset only while fewer than `parts` cuts were made.
void greedy_split_bcsr(const uint64_t *prefix, uint32_t n, uint32_t parts, uint32_t *split) {
  split[0] = 0;
  if (parts == 1) { split[1] = n; return; }
  uint64_t total = prefix[n] - prefix[0];
  uint32_t nps = (uint32_t)(total / parts);
  uint64_t cur = 0;
  uint32_t cnt = 0;
  for (uint32_t i = 0; i < n; ++i) {
    cur += prefix[i + 1] - prefix[i];
    if (cur >= nps) {
      ++cnt;
      if (cnt <= parts) {
        split[cnt] = i + 1;
        cur = 0;
      }
    }
  }
  if (cur < nps && cnt <= parts) {
    ++cnt;
    if (cnt <= parts) split[cnt] = n;
  }
  if (cnt > parts) split[parts] = n;
  for (uint32_t i = cnt + 1; i <= parts; ++i) split[i] = n;
}

}  // namespace sparsep

using namespace sparsep;

extern "C" {

int sparsep_partition_by_row(uint32_t nrows, uint32_t parts, uint32_t *split) {
  // partition_by_row, spmv/1D/CSR-row/support/partition.h:35-60
  if (!split || parts == 0) return SPARSEP_EINVAL;
  uint32_t chunks = nrows / parts, rest = nrows % parts, cur = 0;
  split[0] = 0;
  for (uint32_t i = 0; i < parts; ++i) {
    cur += chunks + (i < rest ? 1 : 0);
    if (cur > nrows) cur = nrows;
    split[i + 1] = cur;
  }
  return SPARSEP_OK;
}

int sparsep_partition_by_nnz(const uint32_t *rowptr, uint32_t nrows, uint32_t parts, uint32_t *split) {
  if (!rowptr || !split || parts == 0) return SPARSEP_EINVAL;
  std::vector<uint64_t> pre(rowptr, rowptr + nrows + 1);
  greedy_split(pre.data(), nrows, parts, split);
  return SPARSEP_OK;
}

int sparsep_partition_by_elem(uint64_t nnz, uint32_t parts, uint64_t *split) {
  // equal nnz per part, the first nnz%parts parts one larger
  // (spmv/1D/COO-nnz/host/app.c:118-132)
  if (!split || parts == 0) return SPARSEP_EINVAL;
  uint64_t chunks = nnz / parts, rest = nnz % parts;
  for (uint32_t i = 0; i <= parts; ++i) split[i] = (uint64_t)i * chunks + std::min<uint64_t>(i, rest);
  return SPARSEP_OK;
}

int sparsep_partition_block_rows(const uint32_t *browptr, uint32_t nbr, const uint32_t *weights, uint32_t parts,
                                 uint32_t *split) {
  if (!browptr || !split || parts == 0) return SPARSEP_EINVAL;
  std::vector<uint64_t> pre(nbr + 1, 0);
  for (uint32_t i = 0; i < nbr; ++i) {
    uint64_t w = 0;
    if (weights)
      for (uint32_t b = browptr[i]; b < browptr[i + 1]; ++b) w += weights[b];
    else
      w = browptr[i + 1] - browptr[i];
    pre[i + 1] = pre[i] + w;
  }
  greedy_split_bcsr(pre.data(), nbr, parts, split);
  return SPARSEP_OK;
}

#define SPARSEP_FORMAT_ENTRIES(T, S)                                                                    \
  int sparsep_read_coo_##S(const char *f, sparsep_coo_##S **o) { return read_coo<T>(f, true, o); }      \
  int sparsep_read_coo_nopad_##S(const char *f, sparsep_coo_##S **o) { return read_coo<T>(f, false, o); } \
  int sparsep_read_cooe_##S(const char *f, sparsep_cooe_##S **o) { return read_cooe<T>(f, o); }         \
  int sparsep_read_mtx_values_##S(const char *f, sparsep_coo_##S **o) { return read_coo_values<T>(f, o); } \
  int sparsep_sort_cooe_##S(sparsep_cooe_##S *A) { return sort_cooe<T>(A); }                            \
  int sparsep_coo2csr_##S(const sparsep_coo_##S *A, sparsep_csr_##S **o) { return coo2csr<T>(A, o); }   \
  int sparsep_csr2bcsr_##S(const sparsep_csr_##S *A, uint32_t rb, uint32_t cb, sparsep_bcsr_##S **o) {  \
    return csr2bcsr<T>(A, rb, cb, o);                                                                   \
  }                                                                                                     \
  int sparsep_bcsr2bcoo_##S(const sparsep_bcsr_##S *A, sparsep_bcoo_##S **o) { return bcsr2bcoo<T>(A, o); } \
  int sparsep_cooe2dcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_dcsr_##S **o) {  \
    return cooe2dcsr<T>(A, h, v, o);                                                                    \
  }                                                                                                     \
  int sparsep_cooe2rbdcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_rbdcsr_##S **o) { \
    return cooe2rbdcsr<T>(A, h, v, o);                                                                  \
  }                                                                                                     \
  int sparsep_cooe2bdcsr_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_bdcsr_##S **o) { \
    return cooe2bdcsr<T>(A, h, v, o);                                                                   \
  }                                                                                                     \
  int sparsep_cooe2dcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_dcoo_##S **o) {  \
    return cooe2dcoo<T>(A, h, v, o);                                                                    \
  }                                                                                                     \
  int sparsep_cooe2rbdcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_rbdcoo_##S **o) { \
    return cooe2rbdcoo<T>(A, h, v, o);                                                                  \
  }                                                                                                     \
  int sparsep_cooe2bdcoo_##S(const sparsep_cooe_##S *A, uint32_t h, uint32_t v, sparsep_bdcoo_##S **o) { \
    return cooe2bdcoo<T>(A, h, v, o);                                                                   \
  }                                                                                                     \
  int sparsep_dcsr2dbcsr_##S(const sparsep_dcsr_##S *A, uint32_t rb, uint32_t cb, sparsep_dbcsr_##S **o) { \
    return dcsr2dblock<T, false>(A, rb, cb, (void **)o);                                                \
  }                                                                                                     \
  int sparsep_dcsr2dbcoo_##S(const sparsep_dcsr_##S *A, uint32_t rb, uint32_t cb, sparsep_dbcoo_##S **o) { \
    return dcsr2dblock<T, true>(A, rb, cb, (void **)o);                                                 \
  }                                                                                                     \
  int sparsep_rbdcsr2rbdbcsr_##S(const sparsep_rbdcsr_##S *A, uint32_t rb, uint32_t cb,                 \
                                 sparsep_rbdbcsr_##S **o) {                                             \
    return stripe2block<T, sparsep_rbdcsr_##S, sparsep_rbdbcsr_##S, false, false>(A, rb, cb, o);        \
  }                                                                                                     \
  int sparsep_rbdcsr2rbdbcoo_##S(const sparsep_rbdcsr_##S *A, uint32_t rb, uint32_t cb,                 \
                                 sparsep_rbdbcoo_##S **o) {                                             \
    return stripe2block<T, sparsep_rbdcsr_##S, sparsep_rbdbcoo_##S, true, false>(A, rb, cb, o);         \
  }                                                                                                     \
  int sparsep_bdcsr2bdbcsr_##S(const sparsep_bdcsr_##S *A, uint32_t rb, uint32_t cb, sparsep_bdbcsr_##S **o) { \
    return stripe2block<T, sparsep_bdcsr_##S, sparsep_bdbcsr_##S, false, true>(A, rb, cb, o);           \
  }                                                                                                     \
  int sparsep_bdcsr2bdbcoo_##S(const sparsep_bdcsr_##S *A, uint32_t rb, uint32_t cb, sparsep_bdbcoo_##S **o) { \
    return stripe2block<T, sparsep_bdcsr_##S, sparsep_bdbcoo_##S, true, true>(A, rb, cb, o);            \
  }

SPARSEP_FORMAT_ENTRIES(int8_t, i8)
SPARSEP_FORMAT_ENTRIES(int16_t, i16)
SPARSEP_FORMAT_ENTRIES(int32_t, i32)
SPARSEP_FORMAT_ENTRIES(int64_t, i64)
SPARSEP_FORMAT_ENTRIES(float, f32)
SPARSEP_FORMAT_ENTRIES(double, f64)

}  // extern "C"
