"""ctypes binding of the sparsep_b200 C-ABI (include/sparsep.h).

This is the host-side mirror of the reference's interface for Python callers
(tests, bench, autotuner): the reference's matrix structs as ctypes structures
per element type, builders from numpy arrays, and a Plan object over
sparsep_plan.  The compute path is always libsparsep_b200.so; importing this
module raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np

PKG = Path(__file__).resolve().parent
# SPARSEP_CHECKED=1 selects the bounds-checked build (libsparsep_b200_check.so)
LIB_PATH = PKG / ("libsparsep_b200_check.so" if os.environ.get("SPARSEP_CHECKED") == "1" else "libsparsep_b200.so")

# status codes
OK, EIO, ENOMEM, ENODEV, EINVAL, ENOSYS, ERANGE, ETIMEDOUT, EBADF = 0, -5, -12, -19, -22, -38, -34, -110, -9
FMT_CSR, FMT_COO, FMT_BCSR, FMT_BCOO = range(4)
S1D, S2D_EQUAL, S2D_EQUAL_W, S2D_VAR = range(4)
BAL_ROW, BAL_NNZ, BAL_BLOCK, BAL_NNZ_ELEM, BAL_INTERLEAVE = range(5)
SYNC_LF, SYNC_ATOMIC, SYNC_CG = range(3)


@dataclass(frozen=True)
class DType:
    name: str       # suffix in the C-ABI (i8 ... f64)
    code: int       # sparsep_dtype
    np: Any         # numpy dtype
    ct: Any         # ctypes scalar
    macro: str      # reference -D macro


DTYPES = {
    "i8": DType("i8", 0, np.int8, C.c_int8, "INT8"),
    "i16": DType("i16", 1, np.int16, C.c_int16, "INT16"),
    "i32": DType("i32", 2, np.int32, C.c_int32, "INT32"),
    "i64": DType("i64", 3, np.int64, C.c_int64, "INT64"),
    "f32": DType("f32", 4, np.float32, C.c_float, "FP32"),
    "f64": DType("f64", 5, np.float64, C.c_double, "FP64"),
}

P32 = C.POINTER(C.c_uint32)


class Bind(C.Structure):
    _fields_ = [("rowind", C.c_uint32), ("colind", C.c_uint32)]


class Opts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "format", "scheme", "part_balance", "worker_balance", "sync", "nr_parts", "nr_workers",
        "vert_partitions", "row_block_size", "col_block_size", "lanes", "nrhs", "stage_x", "item_nnz", "pipeline",
        "autotune", "heavy_rows")] + [("reserved", C.c_int32 * 2)]


class PlanInfo(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("format", C.c_int32), ("scheme", C.c_int32), ("nrhs", C.c_int32),
                ("nrows", C.c_uint32), ("ncols", C.c_uint32), ("nnz", C.c_uint64), ("nblocks", C.c_uint64),
                ("items", C.c_uint64), ("tiles", C.c_uint64), ("compulsory_bytes", C.c_uint64),
                ("device_bytes", C.c_uint64), ("scratch_bytes", C.c_uint64), ("kernel_launches", C.c_int32),
                ("lanes", C.c_int32), ("workers", C.c_int32), ("stage_x", C.c_int32), ("variant", C.c_char * 96),
                ("y_bands", C.c_int32)]


def _struct_types(dt: DType) -> dict[str, type]:
    T = dt.ct
    PT = C.POINTER(T)

    class Elem(C.Structure):
        _fields_ = [("rowind", C.c_uint32), ("colind", C.c_uint32), ("val", T)]

    PE = C.POINTER(Elem)
    PB = C.POINTER(Bind)
    u32 = C.c_uint32
    u64 = C.c_uint64

    def mk(name, fields):
        return type(f"{name}_{dt.name}", (C.Structure,), {"_fields_": fields})

    d: dict[str, type] = {"elem": Elem}
    d["coo"] = mk("coo", [("nrows", u32), ("ncols", u32), ("nnz", u32), ("rowindx", P32), ("colind", P32),
                          ("values", PT)])
    d["cooe"] = mk("cooe", [("nrows", u32), ("ncols", u32), ("nnz", u32), ("rows", P32), ("nnzs", PE)])
    d["csr"] = mk("csr", [("nrows", u32), ("ncols", u32), ("nnz", u32), ("rowptr", P32), ("colind", P32),
                          ("values", PT)])
    blk = [("row_block_size", u64), ("col_block_size", u64), ("num_block_rows", u32), ("num_block_cols", u32),
           ("num_blocks", u64), ("num_rows_left", u32), ("nrows", u32), ("ncols", u32), ("nnz", u32)]
    d["bcsr"] = mk("bcsr", blk + [("browptr", P32), ("bcolind", P32), ("bval", PT), ("nnz_per_block", P32)])
    d["bcoo"] = mk("bcoo", blk + [("bind", PB), ("bval", PT), ("nnz_per_block", P32)])
    hd = [("nrows", u32), ("ncols", u32), ("nnz", u32), ("npartitions", u32), ("horz_partitions", u32),
          ("vert_partitions", u32)]
    d["dcsr"] = mk("dcsr", hd + [("tile_height", u32), ("tile_width", u32), ("nnzs_per_partition", P32),
                                 ("drowptr", P32), ("dcolind", P32), ("dval", PT)])
    d["rbdcsr"] = mk("rbdcsr", hd + [("tile_width", u32), ("nnzs_per_vert_partition", P32), ("drowptr", P32),
                                     ("dcolind", P32), ("dval", PT)])
    d["bdcsr"] = mk("bdcsr", hd + [("max_tile_width", u32), ("vert_tile_widths", P32), ("nnzs_per_column", P32),
                                   ("nnzs_per_vert_partition", P32), ("drowptr", P32), ("dcolind", P32),
                                   ("dval", PT)])
    d["dcoo"] = mk("dcoo", hd + [("tile_height", u32), ("tile_width", u32), ("nnzs_per_partition", P32),
                                 ("nnzs", PE)])
    d["rbdcoo"] = mk("rbdcoo", hd + [("tile_width", u32), ("nnzs_per_vert_partition", P32), ("nnzs", PE)])
    d["bdcoo"] = mk("bdcoo", hd + [("max_tile_width", u32), ("vert_tile_widths", P32),
                                   ("nnzs_per_vert_partition", P32), ("nnzs_per_column", P32), ("nnzs", PE)])
    geo = [("row_block_size", u64), ("col_block_size", u64), ("num_block_rows", u32), ("num_block_cols", u32),
           ("num_rows_left", u32)]
    d["dbcsr"] = mk("dbcsr", hd + [("nblocks", u32), ("tile_height", u64), ("tile_width", u64),
                                   ("nnzs_per_partition", P32), ("blocks_per_partition", P32)] + geo +
                    [("browptr", P32), ("bcolind", P32), ("bval", PT), ("nnz_per_block", P32)])
    d["dbcoo"] = mk("dbcoo", hd + [("nblocks", u32), ("tile_height", u64), ("tile_width", u64),
                                   ("nnzs_per_partition", P32), ("blocks_per_partition", P32)] + geo +
                    [("bind", PB), ("bval", PT), ("nnz_per_block", P32)])
    d["rbdbcsr"] = mk("rbdbcsr", hd + [("nblocks", u32), ("tile_width", u32), ("nnzs_per_vert_partition", P32),
                                       ("blocks_per_vert_partition", P32)] + geo +
                      [("browptr", P32), ("bcolind", P32), ("bval", PT), ("nnz_per_block", P32)])
    d["rbdbcoo"] = mk("rbdbcoo", hd + [("nblocks", u32), ("tile_width", u32), ("nnzs_per_vert_partition", P32),
                                       ("blocks_per_vert_partition", P32)] + geo +
                      [("bind", PB), ("bval", PT), ("nnz_per_block", P32)])
    d["bdbcsr"] = mk("bdbcsr", hd + [("nblocks", u32), ("max_tile_width", u32), ("nnzs_per_vert_partition", P32),
                                     ("nnzs_per_column", P32), ("blocks_per_vert_partition", P32),
                                     ("vert_tile_widths", P32), ("nnz_per_block", P32)] + geo +
                     [("browptr", P32), ("bcolind", P32), ("bval", PT)])
    d["bdbcoo"] = mk("bdbcoo", hd + [("nblocks", u32), ("max_tile_width", u32), ("nnzs_per_column", P32),
                                     ("nnzs_per_vert_partition", P32), ("blocks_per_vert_partition", P32),
                                     ("vert_tile_widths", P32), ("nnz_per_block", P32)] + geo +
                     [("bind", PB), ("bval", PT)])
    return d


STRUCTS = {k: _struct_types(v) for k, v in DTYPES.items()}
KINDS = ["csr", "coo", "cooe", "bcsr", "bcoo", "dcsr", "rbdcsr", "bdcsr", "dcoo", "rbdcoo", "bdcoo", "dbcsr",
         "dbcoo", "rbdbcsr", "rbdbcoo", "bdbcsr", "bdbcoo"]
CONVERTERS = {  # name: (input kind, output kind, extra uint32 args)
    "coo2csr": ("coo", "csr", 0), "csr2bcsr": ("csr", "bcsr", 2), "bcsr2bcoo": ("bcsr", "bcoo", 0),
    "cooe2dcsr": ("cooe", "dcsr", 2), "cooe2rbdcsr": ("cooe", "rbdcsr", 2), "cooe2bdcsr": ("cooe", "bdcsr", 2),
    "cooe2dcoo": ("cooe", "dcoo", 2), "cooe2rbdcoo": ("cooe", "rbdcoo", 2), "cooe2bdcoo": ("cooe", "bdcoo", 2),
    "dcsr2dbcsr": ("dcsr", "dbcsr", 2), "dcsr2dbcoo": ("dcsr", "dbcoo", 2),
    "rbdcsr2rbdbcsr": ("rbdcsr", "rbdbcsr", 2), "rbdcsr2rbdbcoo": ("rbdcsr", "rbdbcoo", 2),
    "bdcsr2bdbcsr": ("bdcsr", "bdbcsr", 2), "bdcsr2bdbcoo": ("bdcsr", "bdbcoo", 2),
}

_lib: C.CDLL | None = None


class SparsepError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().sparsep_strerror(status).decode() if _lib is not None else str(status)
        if status == EIO and _lib is not None:
            msg += ": " + _lib.sparsep_last_error().decode()
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


def check(st: int, what: str = "") -> None:
    if st != OK:
        raise SparsepError(st, what)


def lib() -> C.CDLL:
    """Load libsparsep_b200.so (in-tree).  No fallback: a missing library is an error."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m sparsep_b200.build` "
                          "(the CUDA path has no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    L.sparsep_strerror.restype = C.c_char_p
    L.sparsep_version.restype = C.c_char_p
    L.sparsep_last_error.restype = C.c_char_p
    L.sparsep_opts_default.argtypes = [C.POINTER(Opts)]
    L.sparsep_test_fail_alloc.argtypes = [C.c_int]
    L.sparsep_test_live_allocations.restype = C.c_longlong
    L.sparsep_test_wait_fault.argtypes = [C.c_int]
    L.sparsep_plan_free.argtypes = [C.c_void_p]
    L.sparsep_plan_get_info.argtypes = [C.c_void_p, C.POINTER(PlanInfo)]
    L.sparsep_timings.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.sparsep_execute_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sparsep_execute_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.sparsep_plan_x.argtypes = [C.c_void_p]
    L.sparsep_plan_x.restype = C.c_void_p
    L.sparsep_plan_y.argtypes = [C.c_void_p]
    L.sparsep_plan_y.restype = C.c_void_p
    L.sparsep_partition_by_row.argtypes = [C.c_uint32, C.c_uint32, P32]
    L.sparsep_partition_by_nnz.argtypes = [P32, C.c_uint32, C.c_uint32, P32]
    L.sparsep_partition_by_elem.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)]
    L.sparsep_partition_block_rows.argtypes = [P32, C.c_uint32, P32, C.c_uint32, P32]
    for s, dt in DTYPES.items():
        st = STRUCTS[s]
        PT = C.POINTER(dt.ct)
        for k in KINDS:
            f = getattr(L, f"sparsep_plan_{k}_{s}")
            f.argtypes = [C.POINTER(st[k]), C.POINTER(Opts), C.POINTER(C.c_void_p)]
            g = getattr(L, f"sparsep_spmv_{k}_{s}")
            g.argtypes = [C.POINTER(st[k]), PT, PT, C.POINTER(Opts)]
            h = getattr(L, f"sparsep_free_{k}_{s}")
            h.argtypes = [C.POINTER(st[k])]
            h.restype = None
        for rd in ("read_coo", "read_coo_nopad"):
            getattr(L, f"sparsep_{rd}_{s}").argtypes = [C.c_char_p, C.POINTER(C.POINTER(st["coo"]))]
        getattr(L, f"sparsep_read_cooe_{s}").argtypes = [C.c_char_p, C.POINTER(C.POINTER(st["cooe"]))]
        getattr(L, f"sparsep_sort_cooe_{s}").argtypes = [C.POINTER(st["cooe"])]
        for name, (a, b, nx) in CONVERTERS.items():
            f = getattr(L, f"sparsep_{name}_{s}")
            f.argtypes = [C.POINTER(st[a])] + [C.c_uint32] * nx + [C.POINTER(C.POINTER(st[b]))]
    _lib = L
    return L


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().sparsep_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, int(v))
    return o


def ptr(a: np.ndarray | None, ctype) -> Any:
    if a is None:
        return C.POINTER(ctype)()
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


class HostMatrix:
    """A reference struct over numpy arrays (the arrays are kept alive here)."""

    def __init__(self, kind: str, dtype: str, struct: C.Structure, arrays: dict[str, np.ndarray],
                 owned_by_lib: bool = False):
        self.kind, self.dtype, self.s, self.arrays = kind, dtype, struct, arrays
        self._owned = owned_by_lib

    @property
    def ref(self):
        return C.byref(self.s)

    def __del__(self):
        if getattr(self, "_owned", False) and _lib is not None:
            getattr(_lib, f"sparsep_free_{self.kind}_{self.dtype}")(C.pointer(self.s))
            self._owned = False


def _pad(a: np.ndarray, extra: int) -> np.ndarray:
    out = np.zeros(a.size + extra, dtype=a.dtype)
    out[: a.size] = a
    return out


def csr(dtype: str, nrows: int, ncols: int, rowptr, colind, values) -> HostMatrix:
    dt = DTYPES[dtype]
    rowptr = _pad(np.ascontiguousarray(rowptr, dtype=np.uint32), 1)
    colind = _pad(np.ascontiguousarray(colind, dtype=np.uint32), 1)
    values = _pad(np.ascontiguousarray(values, dtype=dt.np), 8)
    s = STRUCTS[dtype]["csr"](nrows, ncols, int(rowptr[nrows]), ptr(rowptr, C.c_uint32), ptr(colind, C.c_uint32),
                              ptr(values, dt.ct))
    return HostMatrix("csr", dtype, s, {"rowptr": rowptr, "colind": colind, "values": values})


def elems_array(dtype: str, rows, cols, vals) -> np.ndarray:
    """numpy structured array with the reference elem_t layout."""
    E = STRUCTS[dtype]["elem"]
    n = len(rows)
    buf = (E * (n + 8))()
    a = np.ctypeslib.as_array(buf)
    a["rowind"][:n] = rows
    a["colind"][:n] = cols
    a["val"][:n] = vals
    return a


def cooe(dtype: str, nrows: int, ncols: int, rows, cols, vals) -> HostMatrix:
    el = elems_array(dtype, rows, cols, vals)
    counts = np.bincount(np.asarray(rows, dtype=np.int64), minlength=nrows).astype(np.uint32)
    counts = _pad(counts, 1)
    E = STRUCTS[dtype]["elem"]
    s = STRUCTS[dtype]["cooe"](nrows, ncols, len(rows), ptr(counts, C.c_uint32), el.ctypes.data_as(C.POINTER(E)))
    return HostMatrix("cooe", dtype, s, {"rows": counts, "nnzs": el})


def coo(dtype: str, nrows: int, ncols: int, rows, cols, vals) -> HostMatrix:
    dt = DTYPES[dtype]
    r = _pad(np.ascontiguousarray(rows, dtype=np.uint32), 1)
    c = _pad(np.ascontiguousarray(cols, dtype=np.uint32), 1)
    v = _pad(np.ascontiguousarray(vals, dtype=dt.np), 1)
    s = STRUCTS[dtype]["coo"](nrows, ncols, len(rows), ptr(r, C.c_uint32), ptr(c, C.c_uint32), ptr(v, dt.ct))
    return HostMatrix("coo", dtype, s, {"rowindx": r, "colind": c, "values": v})


def bcsr(dtype: str, nrows: int, ncols: int, rb: int, cb: int, browptr, bcolind, bval, nnz: int,
         nnz_per_block=None) -> HostMatrix:
    """A BCSR struct over existing block arrays (block rows of rb x cb dense
    blocks sorted by block column, bval row-major per block), as the
    reference's csr2bcsr + sortBCSRMatrix + countNNZperBlockBCSRMatrix leave it."""
    dt = DTYPES[dtype]
    nbr = (nrows + rb - 1) // rb
    bp = _pad(np.ascontiguousarray(browptr, dtype=np.uint32), 1)
    bc = _pad(np.ascontiguousarray(bcolind, dtype=np.uint32), 1)
    bv = _pad(np.ascontiguousarray(np.asarray(bval).reshape(-1), dtype=dt.np), 1)
    nb = int(bp[nbr])
    if nnz_per_block is None:
        nnz_per_block = (np.asarray(bval).reshape(nb, -1) != 0).sum(axis=1) if nb else np.zeros(0)
    npb = _pad(np.ascontiguousarray(nnz_per_block, dtype=np.uint32), 1)
    s = STRUCTS[dtype]["bcsr"](rb, cb, nbr, (ncols + cb - 1) // cb, nb, nrows % rb, nrows, ncols, nnz,
                               ptr(bp, C.c_uint32), ptr(bc, C.c_uint32), ptr(bv, dt.ct), ptr(npb, C.c_uint32))
    return HostMatrix("bcsr", dtype, s, {"browptr": bp, "bcolind": bc, "bval": bv, "nnz_per_block": npb})


def convert(name: str, A: HostMatrix, *args: int) -> HostMatrix:
    a, b, nx = CONVERTERS[name]
    assert A.kind == a and len(args) == nx, (A.kind, name, args)
    out = C.POINTER(STRUCTS[A.dtype][b])()
    check(getattr(lib(), f"sparsep_{name}_{A.dtype}")(A.ref, *[C.c_uint32(v) for v in args], C.byref(out)), name)
    return HostMatrix(b, A.dtype, out.contents, {"_src": A}, owned_by_lib=True)


def read_mtx(path: str, dtype: str, flavour: str = "coo") -> HostMatrix:
    kind = "cooe" if flavour == "cooe" else "coo"
    fn = {"coo": "read_coo", "coo_nopad": "read_coo_nopad", "cooe": "read_cooe", "values": "read_mtx_values"}[flavour]
    out = C.POINTER(STRUCTS[dtype][kind])()
    check(getattr(lib(), f"sparsep_{fn}_{dtype}")(str(path).encode(), C.byref(out)), fn)
    return HostMatrix(kind, dtype, out.contents, {}, owned_by_lib=True)


def sort_cooe(A: HostMatrix) -> None:
    check(getattr(lib(), f"sparsep_sort_cooe_{A.dtype}")(A.ref), "sort_cooe")


class Plan:
    """A device-resident SpMV plan (sparsep_plan)."""

    def __init__(self, A: HostMatrix, opts: Opts | None = None):
        self.A = A
        self.dt = DTYPES[A.dtype]
        h = C.c_void_p()
        o = opts if opts is not None else default_opts()
        check(getattr(lib(), f"sparsep_plan_{A.kind}_{A.dtype}")(A.ref, C.byref(o), C.byref(h)),
              f"plan_{A.kind}_{A.dtype}")
        self.h = h
        self.info = PlanInfo()
        check(lib().sparsep_plan_get_info(self.h, C.byref(self.info)))

    @classmethod
    def from_device_csr(cls, dtype: str, nrows: int, ncols: int, nnz: int, d_rowptr: int, d_colind: int,
                        d_values: int, opts: Opts | None = None) -> "Plan":
        """A plan from CSR arrays already on the device (sparsep_plan_csr_device_*)."""
        p = cls.__new__(cls)
        p.A = None
        p.dt = DTYPES[dtype]
        h = C.c_void_p()
        o = opts if opts is not None else default_opts()
        f = getattr(lib(), f"sparsep_plan_csr_device_{dtype}")
        f.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p]
        check(f(nrows, ncols, nnz, d_rowptr, d_colind, d_values, C.byref(o), C.byref(h)), f"plan_csr_device_{dtype}")
        p.h = h
        p.info = PlanInfo()
        check(lib().sparsep_plan_get_info(p.h, C.byref(p.info)))
        return p

    @classmethod
    def from_device_bcsr(cls, dtype: str, nrows: int, ncols: int, rb: int, cb: int, nblocks: int, nnz: int,
                         d_browptr: int, d_bcolind: int, d_bval: int, d_nnz_per_block: int | None,
                         opts: Opts | None = None) -> "Plan":
        """A 1D BCSR plan from arrays already on the device (sparsep_plan_bcsr_device_*)."""
        p = cls.__new__(cls)
        p.A = None
        p.dt = DTYPES[dtype]
        h = C.c_void_p()
        o = opts if opts is not None else default_opts()
        f = getattr(lib(), f"sparsep_plan_bcsr_device_{dtype}")
        f.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        check(f(nrows, ncols, rb, cb, nblocks, nnz, d_browptr, d_bcolind, d_bval, d_nnz_per_block, C.byref(o),
                C.byref(h)), f"plan_bcsr_device_{dtype}")
        p.h = h
        p.info = PlanInfo()
        check(lib().sparsep_plan_get_info(p.h, C.byref(p.info)))
        return p

    @property
    def nrows(self) -> int:
        return int(self.info.nrows)

    @property
    def ncols(self) -> int:
        return int(self.info.ncols)

    def run_host(self, x: np.ndarray) -> np.ndarray:
        """y = A x on host buffers; with nrhs = k > 1, x is ncols x k and y
        nrows x k (row-major)."""
        k = max(1, int(self.info.nrhs))
        x = np.ascontiguousarray(x, dtype=self.dt.np)
        assert x.size >= self.ncols * k
        y = np.zeros((self.nrows, k) if k > 1 else self.nrows, dtype=self.dt.np)
        check(lib().sparsep_execute_host(self.h, x.ctypes.data, y.ctypes.data), "execute_host")
        return y

    def run_device(self, x_ptr: int, y_ptr: int, stream: int = 0) -> None:
        check(lib().sparsep_execute_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), C.c_void_p(stream)),
              "execute_device")

    def timings(self) -> list[float]:
        t = (C.c_double * 5)()
        check(lib().sparsep_timings(self.h, t))
        return list(t)

    @property
    def x_ptr(self) -> int:
        return lib().sparsep_plan_x(self.h)

    @property
    def y_ptr(self) -> int:
        return lib().sparsep_plan_y(self.h)

    def free(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            lib().sparsep_plan_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BcsrLayout:
    """The block structure of a device CSR (sparsep_bcsr_layout_device): sorts
    the nonzeros into rb x cb blocks once; fill() then writes the BCSR arrays
    of one value array into caller-allocated device buffers."""

    def __init__(self, d_rowptr: int, d_colind: int, nrows: int, ncols: int, nnz: int, rb: int, cb: int,
                 stream: int = 0):
        L = lib()
        L.sparsep_bcsr_layout_device.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                                 C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.sparsep_bcsr_layout_free.argtypes = [C.c_void_p]
        L.sparsep_bcsr_layout_free.restype = None
        self.h = C.c_void_p()
        nb = C.c_uint64()
        check(L.sparsep_bcsr_layout_device(d_rowptr, d_colind, nrows, ncols, nnz, rb, cb, C.byref(self.h),
                                           C.byref(nb), C.c_void_p(stream)), "bcsr_layout_device")
        self.nblocks = int(nb.value)
        self.nrows, self.ncols, self.nnz, self.rb, self.cb = nrows, ncols, nnz, rb, cb
        self.nbr = (nrows + rb - 1) // rb

    def fill(self, dtype: str, d_values: int, d_browptr: int, d_bcolind: int, d_bval: int, d_nnz_per_block: int,
             stream: int = 0) -> None:
        f = getattr(lib(), f"sparsep_csr2bcsr_device_{dtype}")
        f.argtypes = [C.c_void_p] * 7
        check(f(self.h, d_values, d_browptr, d_bcolind, d_bval, d_nnz_per_block, C.c_void_p(stream)),
              f"csr2bcsr_device_{dtype}")

    def free(self) -> None:
        if self.h:
            lib().sparsep_bcsr_layout_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def spmv(A: HostMatrix, x: np.ndarray, opts: Opts | None = None) -> np.ndarray:
    """One-shot SpMV through sparsep_spmv_<kind>_<dtype> (host buffers)."""
    dt = DTYPES[A.dtype]
    x = np.ascontiguousarray(x, dtype=dt.np)
    nrows = A.s.nrows
    y = np.zeros(nrows, dtype=dt.np)
    o = opts if opts is not None else default_opts()
    check(getattr(lib(), f"sparsep_spmv_{A.kind}_{A.dtype}")(A.ref, ptr(x, dt.ct), ptr(y, dt.ct), C.byref(o)),
          f"spmv_{A.kind}_{A.dtype}")
    return y


# ---------------------------------------------------------------------------
# batched multi-RHS SpMV
# ---------------------------------------------------------------------------
def row_pitch(k: int) -> int:
    """Elements between rows of a batch matrix's device x and y: k for
    k <= 2, else k rounded up to a multiple of 4."""
    return k if k <= 2 else (k + 3) // 4 * 4


class BatchVariant(C.Structure):
    _fields_ = [("mode", C.c_int32), ("lanes", C.c_int32), ("item_work", C.c_int32), ("vec", C.c_int32)]

    def as_tuple(self):
        return (int(self.mode), int(self.lanes), int(self.item_work), int(self.vec))

    def applies(self, k: int) -> bool:
        """Whether this variant can run a matrix with k right-hand sides
        (stored with rows of row_pitch(k) elements, all computed)."""
        v = max(1, int(self.vec))
        k = row_pitch(k)
        if k % v or (int(self.mode) & 2 and v != 4):  # window modes: 4-wide variants
            return False
        if int(self.mode) == 4:  # block items: 4-wide, one pass over the pitch (and a BCSR copy:
            return v == 4 and self.lanes * 4 >= k  # Batch.applies checks that per matrix)
        per = -(-k // (self.lanes * v))
        acc = 1
        while acc < per:
            acc *= 2
        return acc * v <= 8


def _batch_sigs(L):
    if getattr(L, "_batch_sigs", False):
        return
    PB = C.c_void_p
    for t in ("f32", "i32"):
        f = getattr(L, f"sparsep_batch_create_{t}")
        f.argtypes = [C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(BatchVariant), C.POINTER(C.c_void_p)]
    L.sparsep_batch_free.argtypes = [PB]
    L.sparsep_batch_free.restype = None
    L.sparsep_batch_x.argtypes = [PB, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    L.sparsep_batch_pitch.argtypes = [PB, C.c_uint32, C.POINTER(C.c_uint32)]
    L.sparsep_batch_item_kinds.argtypes = [PB, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.sparsep_batch_variant_applies.argtypes = [PB, C.c_uint32, C.POINTER(BatchVariant)]
    L.sparsep_batch_set_x.argtypes = [PB, C.c_uint32, C.c_void_p]
    L.sparsep_batch_get_y.argtypes = [PB, C.c_uint32, C.c_void_p]
    L.sparsep_batch_set_variant.argtypes = [PB, C.c_uint32, C.POINTER(BatchVariant)]
    L.sparsep_batch_get_variant.argtypes = [PB, C.c_uint32, C.POINTER(BatchVariant)]
    L.sparsep_batch_time_variant.argtypes = [PB, C.c_uint32, C.POINTER(BatchVariant), C.c_int,
                                             C.POINTER(C.c_double)]
    L.sparsep_batch_commit.argtypes = [PB]
    L.sparsep_batch_execute.argtypes = [PB, C.c_void_p]
    L.sparsep_batch_status.argtypes = [PB]
    L.sparsep_batch_set_ticket.argtypes = [PB, C.c_int]
    L.sparsep_batch_execute_per_matrix.argtypes = [PB, C.c_void_p]
    L.sparsep_batch_execute_one.argtypes = [PB, C.c_uint32, C.c_void_p]
    L.sparsep_batch_candidates.argtypes = [C.POINTER(BatchVariant), C.c_int]
    L.sparsep_batch_autotune.argtypes = [PB, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    L.sparsep_batch_get_info.argtypes = [PB, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.sparsep_batch_variant_default.argtypes = [C.c_uint32, C.POINTER(BatchVariant)]
    L.sparsep_batch_variant_default.restype = None
    L.sparsep_batch_features.argtypes = [PB, C.c_void_p]
    L.sparsep_batch_select.argtypes = [PB, C.c_void_p, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    L.sparsep_features.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    L.sparsep_mlp_nparams.restype = C.c_uint32
    L.sparsep_mlp_scratch_floats.argtypes = [C.c_uint32]
    L.sparsep_mlp_scratch_floats.restype = C.c_size_t
    L.sparsep_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    L.sparsep_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_float,
                                        C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sparsep_mlp_adam.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                   C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
    L.sparsep_mlp_to_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.sparsep_selector_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
    L.sparsep_selector_free.argtypes = [C.c_void_p]
    L.sparsep_selector_free.restype = None
    L.sparsep_selector_scores.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    L._batch_sigs = True


def batch_candidates() -> list[BatchVariant]:
    L = lib()
    _batch_sigs(L)
    n = L.sparsep_batch_candidates(None, 0)
    arr = (BatchVariant * n)()
    L.sparsep_batch_candidates(arr, n)
    return list(arr)


class Batch:
    """Many CSR matrices with their own right-hand-side counts, one persistent launch."""

    def __init__(self, dtype: str, mats: list[HostMatrix], nrhs: list[int], variants=None):
        assert dtype in ("f32", "i32")
        L = lib()
        _batch_sigs(L)
        self.dtype, self.mats, self.nrhs = dtype, mats, [int(k) for k in nrhs]
        ptrs = (C.c_void_p * len(mats))(*[C.addressof(m.s) for m in mats])
        ks = (C.c_uint32 * len(mats))(*self.nrhs)
        var = None
        if variants is not None:
            var = (BatchVariant * len(mats))(*variants)
        h = C.c_void_p()
        check(getattr(L, f"sparsep_batch_create_{dtype}")(len(mats), ptrs, ks, var, C.byref(h)), "batch_create")
        self.h = h
        self.np = DTYPES[dtype].np

    def set_x(self, m: int, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=self.np)
        assert x.size == self.mats[m].s.ncols * self.nrhs[m]
        check(lib().sparsep_batch_set_x(self.h, m, x.ctypes.data), "batch_set_x")

    def get_y(self, m: int) -> np.ndarray:
        y = np.empty((self.mats[m].s.nrows, self.nrhs[m]), dtype=self.np)
        check(lib().sparsep_batch_get_y(self.h, m, y.ctypes.data), "batch_get_y")
        return y

    def applies(self, m: int, v: BatchVariant) -> bool:
        """Whether variant v can run matrix m of this batch (block variants
        need the matrix's BCSR copy)."""
        return lib().sparsep_batch_variant_applies(self.h, m, C.byref(v)) == OK

    def item_kinds(self) -> tuple[int, int]:
        """Committed (window items, long-row chunk items)."""
        w, c = C.c_uint64(), C.c_uint64()
        check(lib().sparsep_batch_item_kinds(self.h, C.byref(w), C.byref(c)), "batch_item_kinds")
        return w.value, c.value

    def pitch(self, m: int) -> int:
        """Elements between consecutive rows of matrix m's device x and y."""
        p = C.c_uint32()
        check(lib().sparsep_batch_pitch(self.h, m, C.byref(p)), "batch_pitch")
        return p.value

    def device_xy(self, m: int):
        """Device x (ncols x pitch) and y (nrows x pitch) of matrix m."""
        dx, dy = C.c_void_p(), C.c_void_p()
        check(lib().sparsep_batch_x(self.h, m, C.byref(dx), C.byref(dy)))
        return dx.value, dy.value

    def execute(self, stream: int | None = None):
        check(lib().sparsep_batch_execute(self.h, C.c_void_p(stream) if stream else None), "batch_execute")

    def execute_per_matrix(self, stream: int | None = None):
        check(lib().sparsep_batch_execute_per_matrix(self.h, C.c_void_p(stream) if stream else None),
              "batch_execute_per_matrix")

    def status(self):
        """Raise if a work item's staging copy timed out since the last check."""
        check(lib().sparsep_batch_status(self.h), "batch_status")

    def set_ticket(self, on: bool):
        check(lib().sparsep_batch_set_ticket(self.h, int(bool(on))), "batch_set_ticket")

    def set_variant(self, m: int, v: BatchVariant):
        check(lib().sparsep_batch_set_variant(self.h, m, C.byref(v)), "batch_set_variant")

    def get_variant(self, m: int) -> BatchVariant:
        v = BatchVariant()
        check(lib().sparsep_batch_get_variant(self.h, m, C.byref(v)), "batch_get_variant")
        return v

    def time_variant(self, m: int, v: BatchVariant, reps: int = 3) -> float | None:
        """Median microseconds of matrix m alone under v; None if v does not apply."""
        us = C.c_double()
        st = lib().sparsep_batch_time_variant(self.h, m, C.byref(v), reps, C.byref(us))
        if st == ENOSYS:
            return None
        check(st, "batch_time_variant")
        return us.value

    def commit(self):
        check(lib().sparsep_batch_commit(self.h), "batch_commit")

    def features(self) -> np.ndarray:
        out = np.zeros((len(self.mats), NFEATURES), dtype=np.float32)
        check(lib().sparsep_batch_features(self.h, out.ctypes.data), "batch_features")
        return out

    def select(self, selector: "Selector", min_confidence: float = 0.0, reps: int = 3):
        """Learned variants (exhaustive autotuning where the network's
        confidence is below min_confidence); returns (chosen, fallback)."""
        ch = np.zeros(len(self.mats), dtype=np.int32)
        fb = np.zeros(len(self.mats), dtype=np.int32)
        check(lib().sparsep_batch_select(self.h, selector.h, float(min_confidence), int(reps), ch.ctypes.data,
                                         fb.ctypes.data), "batch_select")
        return ch, fb

    def autotune(self, reps: int = 3):
        nc = lib().sparsep_batch_candidates(None, 0)
        t = np.zeros((len(self.mats), nc), dtype=np.float64)
        ch = np.zeros(len(self.mats), dtype=np.int32)
        check(lib().sparsep_batch_autotune(self.h, reps, t.ctypes.data_as(C.POINTER(C.c_double)),
                                           ch.ctypes.data_as(C.POINTER(C.c_int32))), "batch_autotune")
        return t, ch

    def info(self):
        b, it, nz = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().sparsep_batch_get_info(self.h, C.byref(b), C.byref(it), C.byref(nz)))
        return dict(compulsory_bytes=b.value, items=it.value, nnz=nz.value)

    def free(self):
        if getattr(self, "h", None) and self.h.value:
            lib().sparsep_batch_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# learned variant selector
# ---------------------------------------------------------------------------
NFEATURES = 16
NVARIANTS = 36


def features(nrows: int, ncols: int, rowptr: np.ndarray, colind: np.ndarray, k: int) -> np.ndarray:
    """The selector's 16 features of a CSR structure with k right-hand sides."""
    L = lib()
    _batch_sigs(L)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    colind = np.ascontiguousarray(colind, dtype=np.uint32)
    out = np.zeros(NFEATURES, dtype=np.float32)
    check(L.sparsep_features(nrows, ncols, rowptr.ctypes.data, colind.ctypes.data, int(k), out.ctypes.data),
          "features")
    return out


class Selector:
    """A trained network (BF16 weight bits + feature standardisation) on the GPU."""

    def __init__(self, wb: np.ndarray, mean: np.ndarray, std: np.ndarray):
        L = lib()
        _batch_sigs(L)
        self.wb = np.ascontiguousarray(wb, dtype=np.uint16)
        self.mean = np.ascontiguousarray(mean, dtype=np.float32)
        self.std = np.ascontiguousarray(std, dtype=np.float32)
        assert self.wb.size == L.sparsep_mlp_nparams() and self.mean.size == NFEATURES == self.std.size
        h = C.c_void_p()
        check(L.sparsep_selector_create(self.wb.ctypes.data, self.mean.ctypes.data, self.std.ctypes.data,
                                        C.byref(h)), "selector_create")
        self.h = h

    def scores(self, feats: np.ndarray) -> np.ndarray:
        feats = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, NFEATURES)
        out = np.zeros((feats.shape[0], NVARIANTS), dtype=np.float32)
        check(lib().sparsep_selector_scores(self.h, feats.ctypes.data, feats.shape[0], out.ctypes.data),
              "selector_scores")
        return out

    def free(self):
        if getattr(self, "h", None) and self.h.value:
            lib().sparsep_selector_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# conjugate gradient on a plan
# ---------------------------------------------------------------------------
class CG:
    """Conjugate gradient (sparsep_cg_*) on an FP32 / FP64 plan of an SPD matrix."""

    def __init__(self, plan: "Plan"):
        L = lib()
        L.sparsep_cg_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.sparsep_cg_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_uint32,
                                       C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.c_void_p]
        L.sparsep_cg_free.argtypes = [C.c_void_p]
        L.sparsep_cg_free.restype = None
        self.plan = plan
        h = C.c_void_p()
        check(L.sparsep_cg_create(plan.h, C.byref(h)), "cg_create")
        self.h = h

    def solve(self, d_b: int, d_x: int, max_iters: int = 1000, rel_tol: float = 1e-8, check_every: int = 10,
              stream: int | None = None):
        """Solve in place on device vectors; returns (iterations, relative residual)."""
        it, r = C.c_uint32(), C.c_double()
        check(lib().sparsep_cg_solve(self.h, C.c_void_p(d_b), C.c_void_p(d_x), max_iters, rel_tol, check_every,
                                     C.byref(it), C.byref(r), C.c_void_p(stream) if stream else None), "cg_solve")
        return it.value, r.value

    def free(self):
        if getattr(self, "h", None) and self.h.value:
            lib().sparsep_cg_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PowerIteration:
    """Power iteration (sparsep_power_*) on a square FP32 / FP64 plan."""

    def __init__(self, plan: "Plan"):
        L = lib()
        L.sparsep_power_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.sparsep_power_run.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_uint32,
                                        C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.c_void_p]
        L.sparsep_power_free.argtypes = [C.c_void_p]
        L.sparsep_power_free.restype = None
        self.plan = plan
        h = C.c_void_p()
        check(L.sparsep_power_create(plan.h, C.byref(h)), "power_create")
        self.h = h

    def run(self, d_x: int, max_iters: int = 1000, rel_tol: float = 1e-10, check_every: int = 10,
            stream: int | None = None):
        """Iterate in place on the device vector d_x; returns (lambda, iterations)."""
        lam, it = C.c_double(), C.c_uint32()
        check(lib().sparsep_power_run(self.h, C.c_void_p(d_x), max_iters, rel_tol, check_every, C.byref(lam),
                                      C.byref(it), C.c_void_p(stream) if stream else None), "power_run")
        return lam.value, it.value

    def free(self):
        if getattr(self, "h", None) and self.h.value:
            lib().sparsep_power_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
