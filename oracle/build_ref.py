"""Build the reference's own host-side code into oracle/_ref/ (TEST INFRASTRUCTURE).

For each SparseP kernel directory listed below and each element type, this
script writes a small C shim into oracle/_ref/src/ that #includes the
directory's support headers straight from the reference tree and the
`spmv_host` function cut out of its host/app.c (by pattern, at build time),
then compiles it with gcc into oracle/_ref/libref_<dir>_<dtype>.so.  Nothing
from the reference is copied into the repository: the shims and libraries are
build outputs (oracle/_ref/ is git-ignored) and exist only where the reference
tree does.  The UPMEM host runtime (dpu.h) is never included -- only
support/*.h and spmv_host, which are plain C.

Flags follow the reference build (-std=c11, spmv/1D/CSR-row/Makefile:29-42)
plus -fwrapv, which pins the signed wrap-around of `sum += x * val` for
int32/int64 that the reference relies on.

Usage: python oracle/build_ref.py [reference_root]

The reference root is the argument, else $SPARSEP_REFERENCE, else a
directory named `reference` beside the repository; without a reference tree
nothing is built.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
SRC = OUT / "src"
DTYPES = {"i8": "INT8", "i16": "INT16", "i32": "INT32", "i64": "INT64", "f32": "FP32", "f64": "FP64"}

# exported wrappers per reference directory: (return type, name, params, body)
COMMON = """
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <stdbool.h>
#include <string.h>
#include <assert.h>
#include <unistd.h>
#define NR_TASKLETS 16
"""

WRAPPERS = {
    "1D/CSR-row": ["partition.h:BLNC_TSKLT_ROW=1", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void *ref_coo2csr(void *B) { return coo2csr((struct COOMatrix *)B); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct CSRMatrix *)A, x); }
void ref_partition_by_row(void *A, int parts, uint32_t *split) {
  struct partition_info_t *p = partition_init(parts, NR_TASKLETS);
  partition_by_row((struct CSRMatrix *)A, p, parts);
  memcpy(split, p->row_split, sizeof(uint32_t) * (parts + 1));
  partition_free(p);
}
"""],
    "1D/CSR-nnz": ["partition.h:BLNC_TSKLT_NNZ=1", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void *ref_coo2csr(void *B) { return coo2csr((struct COOMatrix *)B); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct CSRMatrix *)A, x); }
void ref_partition_by_nnz(void *A, int parts, uint32_t *split) {
  /* partition_by_nnz may write split[parts+1] (one past its allocation) */
  struct partition_info_t *p = partition_init(parts + 1, NR_TASKLETS);
  partition_by_nnz((struct CSRMatrix *)A, p, parts);
  memcpy(split, p->row_split, sizeof(uint32_t) * (parts + 1));
  partition_free(p);
}
"""],
    "1D/COO-nnz": ["", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void ref_sort(void *A) { sortCOOMatrix((struct COOMatrix *)A); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct COOMatrix *)A, x); }
"""],
    "1D/BCSR-nnz": ["partition.h:BLNC_TSKLT_NNZ=1", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void *ref_coo2csr(void *B) { return coo2csr((struct COOMatrix *)B); }
void *ref_csr2bcsr(void *A, uint32_t rb, uint32_t cb) {
  struct BCSRMatrix *b = csr2bcsr((struct CSRMatrix *)A, rb, cb);
  sortBCSRMatrix(b);
  countNNZperBlockBCSRMatrix(b);
  return b;
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BCSRMatrix *)A, x); }
void ref_partition_by_nnz(void *A, int parts, uint32_t *split) {
  struct partition_info_t *p = partition_init(parts + 1, NR_TASKLETS);
  partition_by_nnz((struct BCSRMatrix *)A, p, parts);
  memcpy(split, p->brow_split, sizeof(uint32_t) * (parts + 1));
}
"""],
    "1D/BCSR-block": ["partition.h:BLNC_TSKLT_BLOCK=1", """
void ref_partition_by_blocks(void *A, int parts, uint32_t *split) {
  struct partition_info_t *p = partition_init(parts + 1, NR_TASKLETS);
  partition_by_blocks((struct BCSRMatrix *)A, p, parts);
  memcpy(split, p->brow_split, sizeof(uint32_t) * (parts + 1));
}
"""],
    "1D/BCOO-nnz": ["", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void *ref_coo2csr(void *B) { return coo2csr((struct COOMatrix *)B); }
void *ref_csr2bcoo(void *A, uint32_t rb, uint32_t cb) {
  struct BCSRMatrix *b = csr2bcsr((struct CSRMatrix *)A, rb, cb);
  sortBCSRMatrix(b);
  countNNZperBlockBCSRMatrix(b);
  return bcsr2bcoo(b);
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BCOOMatrix *)A, x); }
"""],
    "2D/DCSR": ["", """
void *ref_read(const char *f) { return readCOOMatrix(f); }
void ref_sort(void *A) { sortCOOMatrix((struct COOMatrix *)A); }
void *ref_convert(void *A, int h, int v) { return coo2dcsr((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct DCSRMatrix *)A, x); }
"""],
    "2D/RBDCSR": ["", """
void *ref_convert(void *A, int h, int v) { return coo2rbdcsr((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct RBDCSRMatrix *)A, x); }
"""],
    "2D/BDCSR": ["partition.h:BLNC_TSKLT_NNZ=1", """
void *ref_convert(void *A, int h, int v) { return coo2bdcsr((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BDCSRMatrix *)A, x); }
void ref_partition_by_nnz(void *A, uint32_t *split) {
  struct BDCSRMatrix *m = (struct BDCSRMatrix *)A;
  struct partition_info_t *p = partition_init(m, m->horz_partitions * m->vert_partitions, 1, NR_TASKLETS);
  partition_by_nnz(m, p);
  memcpy(split, p->row_split, sizeof(uint32_t) * m->vert_partitions * (m->horz_partitions + 1));
}
"""],
    "2D/DCOO": ["", """
void *ref_convert(void *A, int h, int v) { return coo2dcoo((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct DCOOMatrix *)A, x); }
"""],
    "2D/RBDCOO": ["", """
void *ref_convert(void *A, int h, int v) { return coo2rbdcoo((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct RBDCOOMatrix *)A, x); }
"""],
    "2D/BDCOO": ["", """
void *ref_convert(void *A, int h, int v) { return coo2bdcoo((struct COOMatrix *)A, h, v); }
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BDCOOMatrix *)A, x); }
"""],
    "2D/DBCSR": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct DBCSRMatrix *d = dcsr2dbcsr(coo2dcsr((struct COOMatrix *)A, h, v), rb, cb);
  countNNZperBlockDBCSRMatrix(d);
  return d;
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct DBCSRMatrix *)A, x); }
"""],
    "2D/DBCOO": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct DBCSRMatrix *d = dcsr2dbcsr(coo2dcsr((struct COOMatrix *)A, h, v), rb, cb);
  sortDBCSRMatrix(d);
  countNNZperBlockDBCSRMatrix(d);
  return dbcsr2dbcoo(d);
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct DBCOOMatrix *)A, x); }
"""],
    "2D/RBDBCSR-nnz": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct RBDBCSRMatrix *d = rbdcsr2rbdbcsr(coo2rbdcsr((struct COOMatrix *)A, h, v), rb, cb);
  countNNZperBlockRBDBCSRMatrix(d);
  return d;
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct RBDBCSRMatrix *)A, x); }
"""],
    "2D/RBDBCOO-nnz": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct RBDBCSRMatrix *d = rbdcsr2rbdbcsr(coo2rbdcsr((struct COOMatrix *)A, h, v), rb, cb);
  sortRBDBCSRMatrix(d);
  countNNZperBlockRBDBCSRMatrix(d);
  return rbdbcsr2rbdbcoo(d);
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct RBDBCOOMatrix *)A, x); }
"""],
    "2D/BDBCSR-nnz": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct BDBCSRMatrix *d = bdcsr2bdbcsr(coo2bdcsr((struct COOMatrix *)A, h, v), rb, cb);
  countNNZperBlockBDBCSRMatrix(d);
  return d;
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BDBCSRMatrix *)A, x); }
"""],
    "2D/BDBCOO-nnz": ["", """
void *ref_convert(void *A, int h, int v, uint32_t rb, uint32_t cb) {
  struct BDBCSRMatrix *d = bdcsr2bdbcsr(coo2bdcsr((struct COOMatrix *)A, h, v), rb, cb);
  sortBDBCSRMatrix(d);
  countNNZperBlockBDBCSRMatrix(d);
  return bdbcsr2bdbcoo(d);
}
void ref_spmv(val_dt *y, void *A, val_dt *x) { spmv_host(y, (struct BDBCOOMatrix *)A, x); }
"""],
}


def extract_spmv_host(app_c: Path) -> str:
    """Cut `spmv_host` out of a reference host/app.c (from its signature to the
    first line that is a lone closing brace)."""
    lines = app_c.read_text().splitlines()
    out, on = [], False
    for ln in lines:
        if not on and re.match(r"^(static )?void spmv_host\(", ln):
            on = True
        if on:
            out.append(ln)
            if ln.rstrip() == "}":
                break
    if not out:
        raise RuntimeError(f"spmv_host not found in {app_c}")
    return "\n".join(out) + "\n"


def shim_source(ref: Path, d: str, dtype_macro: str) -> tuple[str, list[str]]:
    part, body = WRAPPERS[d]
    sup = ref / "spmv" / d / "support"
    defs = [f"-D{dtype_macro}=1"]
    src = COMMON
    src += '#include "matrix.h"\n'
    if part:
        hdr, macro = part.split(":")
        defs.append(f"-D{macro}")
        src += f'#include "{hdr}"\n'
    src += extract_spmv_host(ref / "spmv" / d / "host" / "app.c")
    src += body
    return src, [f"-I{sup}", *defs]


def build_one(ref: Path, d: str, tag: str, macro: str) -> Path:
    SRC.mkdir(parents=True, exist_ok=True)
    name = d.replace("/", "_").replace("-", "_")
    c = SRC / f"{name}_{tag}.c"
    so = OUT / f"libref_{name}_{tag}.so"
    src, flags = shim_source(ref, d, macro)
    c.write_text(src)
    cmd = ["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-fwrapv", "-fPIC", "-shared", "-w", *flags, str(c),
           "-o", str(so)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)}\n{r.stderr}")
    return so


def reference_root(arg: str | os.PathLike | None = None) -> Path:
    """The reference tree: the argument, $SPARSEP_REFERENCE, or ../reference."""
    if arg:
        return Path(arg)
    env = os.environ.get("SPARSEP_REFERENCE")
    return Path(env) if env else HERE.parent.parent / "reference"


def build(ref_root: str | os.PathLike | None = None) -> list[Path]:
    ref = reference_root(ref_root)
    if not (ref / "spmv").is_dir():
        return []
    OUT.mkdir(parents=True, exist_ok=True)
    jobs = [(d, t, m) for d in WRAPPERS for t, m in DTYPES.items()]
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(lambda j: build_one(ref, *j), jobs))


if __name__ == "__main__":
    libs = build(sys.argv[1] if len(sys.argv) > 1 else None)
    print(f"built {len(libs)} reference libraries into {OUT}")
