"""sparsep_b200: a B200 (sm_100a) SpMV library with SparseP's formats,
partitioning schemes, balance options and element types.

The compute path is the C-ABI library libsparsep_b200.so (include/sparsep.h);
this package is its Python binding (`capi`), the in-tree build (`build`) and
the seeded workload generators (`synth`).
"""
from . import capi, synth  # noqa: F401
from .capi import (DTYPES, HostMatrix, Opts, Plan, SparsepError, convert, coo, cooe, csr, default_opts, lib,  # noqa: F401
                   read_mtx, sort_cooe, spmv)

__all__ = ["capi", "synth", "DTYPES", "HostMatrix", "Opts", "Plan", "SparsepError", "convert", "coo", "cooe", "csr",
           "default_opts", "lib", "read_mtx", "sort_cooe", "spmv"]
