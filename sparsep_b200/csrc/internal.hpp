// internal.hpp -- type maps and helpers shared by the host sources of
// sparsep_b200 (not part of the C-ABI).
#pragma once
#include <cstdint>
#include <cstdlib>

#include "sparsep.h"

namespace sparsep {

template <typename T> struct Types;
#define SPARSEP_TYPES_SPEC(T, S, CODE)        \
  template <> struct Types<T> {               \
    using elem = sparsep_elem_##S;            \
    using coo = sparsep_coo_##S;              \
    using cooe = sparsep_cooe_##S;            \
    using csr = sparsep_csr_##S;              \
    using bcsr = sparsep_bcsr_##S;            \
    using bcoo = sparsep_bcoo_##S;            \
    using dcsr = sparsep_dcsr_##S;            \
    using rbdcsr = sparsep_rbdcsr_##S;        \
    using bdcsr = sparsep_bdcsr_##S;          \
    using dcoo = sparsep_dcoo_##S;            \
    using rbdcoo = sparsep_rbdcoo_##S;        \
    using bdcoo = sparsep_bdcoo_##S;          \
    using dbcsr = sparsep_dbcsr_##S;          \
    using dbcoo = sparsep_dbcoo_##S;          \
    using rbdbcsr = sparsep_rbdbcsr_##S;      \
    using rbdbcoo = sparsep_rbdbcoo_##S;      \
    using bdbcsr = sparsep_bdbcsr_##S;        \
    using bdbcoo = sparsep_bdbcoo_##S;        \
    static constexpr int dtype = CODE;        \
  };
SPARSEP_TYPES_SPEC(int8_t, i8, SPARSEP_INT8)
SPARSEP_TYPES_SPEC(int16_t, i16, SPARSEP_INT16)
SPARSEP_TYPES_SPEC(int32_t, i32, SPARSEP_INT32)
SPARSEP_TYPES_SPEC(int64_t, i64, SPARSEP_INT64)
SPARSEP_TYPES_SPEC(float, f32, SPARSEP_FP32)
SPARSEP_TYPES_SPEC(double, f64, SPARSEP_FP64)
#undef SPARSEP_TYPES_SPEC

// Frees of library-allocated structs (every pointer member, then the struct).
#define SPARSEP_F(m) std::free((void *)X->m)
#define SPARSEP_FREE_FN(KIND, ...)                        \
  template <typename S> inline void free_##KIND##_impl(S *X) { \
    if (!X) return;                                       \
    __VA_ARGS__;                                          \
    std::free(X);                                         \
  }
SPARSEP_FREE_FN(coo, SPARSEP_F(rowindx); SPARSEP_F(colind); SPARSEP_F(values))
SPARSEP_FREE_FN(cooe, SPARSEP_F(rows); SPARSEP_F(nnzs))
SPARSEP_FREE_FN(csr, SPARSEP_F(rowptr); SPARSEP_F(colind); SPARSEP_F(values))
SPARSEP_FREE_FN(bcsr, SPARSEP_F(browptr); SPARSEP_F(bcolind); SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(bcoo, SPARSEP_F(bind); SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(dcsr, SPARSEP_F(nnzs_per_partition); SPARSEP_F(drowptr); SPARSEP_F(dcolind); SPARSEP_F(dval))
SPARSEP_FREE_FN(rbdcsr, SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(drowptr); SPARSEP_F(dcolind); SPARSEP_F(dval))
SPARSEP_FREE_FN(bdcsr, SPARSEP_F(vert_tile_widths); SPARSEP_F(nnzs_per_column); SPARSEP_F(nnzs_per_vert_partition);
                SPARSEP_F(drowptr); SPARSEP_F(dcolind); SPARSEP_F(dval))
SPARSEP_FREE_FN(dcoo, SPARSEP_F(nnzs_per_partition); SPARSEP_F(nnzs))
SPARSEP_FREE_FN(rbdcoo, SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(nnzs))
SPARSEP_FREE_FN(bdcoo, SPARSEP_F(vert_tile_widths); SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(nnzs_per_column);
                SPARSEP_F(nnzs))
SPARSEP_FREE_FN(dbcsr, SPARSEP_F(nnzs_per_partition); SPARSEP_F(blocks_per_partition); SPARSEP_F(browptr);
                SPARSEP_F(bcolind); SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(dbcoo, SPARSEP_F(nnzs_per_partition); SPARSEP_F(blocks_per_partition); SPARSEP_F(bind);
                SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(rbdbcsr, SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(blocks_per_vert_partition); SPARSEP_F(browptr);
                SPARSEP_F(bcolind); SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(rbdbcoo, SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(blocks_per_vert_partition); SPARSEP_F(bind);
                SPARSEP_F(bval); SPARSEP_F(nnz_per_block))
SPARSEP_FREE_FN(bdbcsr, SPARSEP_F(nnzs_per_vert_partition); SPARSEP_F(nnzs_per_column);
                SPARSEP_F(blocks_per_vert_partition); SPARSEP_F(vert_tile_widths); SPARSEP_F(nnz_per_block);
                SPARSEP_F(browptr); SPARSEP_F(bcolind); SPARSEP_F(bval))
SPARSEP_FREE_FN(bdbcoo, SPARSEP_F(nnzs_per_column); SPARSEP_F(nnzs_per_vert_partition);
                SPARSEP_F(blocks_per_vert_partition); SPARSEP_F(vert_tile_widths); SPARSEP_F(nnz_per_block);
                SPARSEP_F(bind); SPARSEP_F(bval))
#undef SPARSEP_FREE_FN
#undef SPARSEP_F

template <typename T> inline void free_coo(typename Types<T>::coo *X) { free_coo_impl(X); }
template <typename T> inline void free_cooe(typename Types<T>::cooe *X) { free_cooe_impl(X); }
template <typename T> inline void free_csr(typename Types<T>::csr *X) { free_csr_impl(X); }
template <typename T> inline void free_bcsr(typename Types<T>::bcsr *X) { free_bcsr_impl(X); }
template <typename T> inline void free_bcoo(typename Types<T>::bcoo *X) { free_bcoo_impl(X); }
template <typename T> inline void free_dcsr(typename Types<T>::dcsr *X) { free_dcsr_impl(X); }
template <typename T> inline void free_rbdcsr(typename Types<T>::rbdcsr *X) { free_rbdcsr_impl(X); }
template <typename T> inline void free_bdcsr(typename Types<T>::bdcsr *X) { free_bdcsr_impl(X); }
template <typename T> inline void free_dcoo(typename Types<T>::dcoo *X) { free_dcoo_impl(X); }
template <typename T> inline void free_rbdcoo(typename Types<T>::rbdcoo *X) { free_rbdcoo_impl(X); }
template <typename T> inline void free_bdcoo(typename Types<T>::bdcoo *X) { free_bdcoo_impl(X); }
template <typename T> inline void free_dbcsr(typename Types<T>::dbcsr *X) { free_dbcsr_impl(X); }
template <typename T> inline void free_dbcoo(typename Types<T>::dbcoo *X) { free_dbcoo_impl(X); }

// Overloads picked by struct type (used by generic code).
#define SPARSEP_FREE_ANY(S)                                                   \
  inline void free_any(sparsep_coo_##S *X) { free_coo_impl(X); }             \
  inline void free_any(sparsep_cooe_##S *X) { free_cooe_impl(X); }           \
  inline void free_any(sparsep_csr_##S *X) { free_csr_impl(X); }             \
  inline void free_any(sparsep_bcsr_##S *X) { free_bcsr_impl(X); }           \
  inline void free_any(sparsep_bcoo_##S *X) { free_bcoo_impl(X); }           \
  inline void free_any(sparsep_dcsr_##S *X) { free_dcsr_impl(X); }           \
  inline void free_any(sparsep_rbdcsr_##S *X) { free_rbdcsr_impl(X); }       \
  inline void free_any(sparsep_bdcsr_##S *X) { free_bdcsr_impl(X); }         \
  inline void free_any(sparsep_dcoo_##S *X) { free_dcoo_impl(X); }           \
  inline void free_any(sparsep_rbdcoo_##S *X) { free_rbdcoo_impl(X); }       \
  inline void free_any(sparsep_bdcoo_##S *X) { free_bdcoo_impl(X); }         \
  inline void free_any(sparsep_dbcsr_##S *X) { free_dbcsr_impl(X); }         \
  inline void free_any(sparsep_dbcoo_##S *X) { free_dbcoo_impl(X); }         \
  inline void free_any(sparsep_rbdbcsr_##S *X) { free_rbdbcsr_impl(X); }     \
  inline void free_any(sparsep_rbdbcoo_##S *X) { free_rbdbcoo_impl(X); }     \
  inline void free_any(sparsep_bdbcsr_##S *X) { free_bdbcsr_impl(X); }       \
  inline void free_any(sparsep_bdbcoo_##S *X) { free_bdbcoo_impl(X); }
SPARSEP_FREE_ANY(i8)
SPARSEP_FREE_ANY(i16)
SPARSEP_FREE_ANY(i32)
SPARSEP_FREE_ANY(i64)
SPARSEP_FREE_ANY(f32)
SPARSEP_FREE_ANY(f64)
#undef SPARSEP_FREE_ANY

// Greedy prefix splits with the reference's semantics (formats.cpp).
void greedy_split(const uint64_t *prefix, uint32_t n, uint32_t parts, uint32_t *split);
void greedy_split_bcsr(const uint64_t *prefix, uint32_t n, uint32_t parts, uint32_t *split);

// Text of the last failure, returned by sparsep_last_error() on this thread.
void record_error(const char *msg);

// sparsep_opts.autotune on a CSR input (autotune.cu): the plan of the variant
// chosen by timing (2) or by the learned selector (1).
template <typename T>
int plan_autotuned(const typename Types<T>::csr *A, const sparsep_opts &o, sparsep_plan **out);
// Records in the plan's info.variant which variant autotuning chose and how.
void note_variant(sparsep_plan *p, const char *name, int mode);

}  // namespace sparsep
