"""Exhaustive autotuner of single-matrix SpMV plans.

Given one CSR matrix, every plan the library offers for it is built and timed
on the GPU: format (CSR, COO, BCSR 4x4 / 8x8, BCOO 4x4) x scheme (1D, and the
reference's 2D tilings D / RBD / BD of CSR and COO at 16x16, 32x32 and 64x64
tiles = 256-4096 tiles) x balance (auto items, or 2048 parts split by rows,
nonzeros, blocks or elements) x sync (lock-free or red.global) x lanes per row
(1-32) and the TMA pipeline.  Each candidate is converted with the library's
converters, planned once, and timed with CUDA events on the launching stream
(median of `reps`, the L2 flushed by a 256 MB write before each run).  The
records form a timing database; the fastest is returned.  Integer results of
every candidate are compared with the first one (bit-exact); FP candidates'
largest relative difference is recorded.

    python -m sparsep_b200.tune --workload zipf --dtype f32 --out tune_zipf.json
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import capi, synth

PARTS = 2048
GRIDS = ((16, 16), (32, 32), (64, 64))
TWO_D = ("dcsr", "rbdcsr", "bdcsr", "dcoo", "rbdcoo", "bdcoo")


def _options(kind: str):
    """(label, opts dict) pairs for one struct kind."""
    if kind == "csr":
        out = [("auto", {}), ("pipeline", dict(pipeline=1))]
        out += [(f"lanes{L}", dict(lanes=L)) for L in (1, 2, 4, 8, 16, 32)]
        out += [("parts-row", dict(nr_parts=PARTS, part_balance=capi.BAL_ROW)),
                ("parts-nnz", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ, worker_balance=capi.BAL_NNZ))]
        return out
    if kind == "cooe":
        return [("auto-lf", {}), ("auto-atomic", dict(sync=capi.SYNC_ATOMIC)),
                ("parts-row", dict(nr_parts=PARTS, part_balance=capi.BAL_ROW)),
                ("parts-elem", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM))]
    if kind == "bcsr":
        return [("auto", {}), ("auto-atomic", dict(sync=capi.SYNC_ATOMIC)),
                ("parts-block", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
                ("parts-nnz", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ))]
    if kind == "bcoo":
        return [("auto", {}), ("auto-atomic", dict(sync=capi.SYNC_ATOMIC)),
                ("parts-block", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
                ("parts-elem", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM))]
    return [("merge", {}), ("atomic", dict(sync=capi.SYNC_ATOMIC)), ("no-smem-x", dict(stage_x=0))]


def _structs(A: capi.HostMatrix, grids=GRIDS, blocks=(4, 8)):
    """(label, kind, builder) for every struct the tuner tries; builders are
    called lazily so that only one converted copy lives at a time."""
    n, m = int(A.s.nrows), int(A.s.ncols)
    rp = A.arrays["rowptr"][: n + 1].astype(np.int64)
    nnz = int(rp[n])
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp))
    cols = A.arrays["colind"][:nnz]
    vals = A.arrays["values"][:nnz]

    def cooe():
        return capi.cooe(A.dtype, n, m, rows, cols, vals)

    out = [("csr", "csr", lambda: A), ("coo", "cooe", cooe)]
    for b in blocks:
        out.append((f"bcsr{b}x{b}", "bcsr", lambda b=b: capi.convert("csr2bcsr", A, b, b)))
    if blocks:
        b = blocks[0]
        out.append((f"bcoo{b}x{b}", "bcoo",
                    lambda b=b: capi.convert("bcsr2bcoo", capi.convert("csr2bcsr", A, b, b))))
    for kind in TWO_D:
        for h, v in grids:
            out.append((f"{kind}{h}x{v}", kind, lambda kind=kind, h=h, v=v: capi.convert(f"cooe2{kind}", cooe(), h, v)))
    return out


def autotune(A: capi.HostMatrix, x: np.ndarray, reps: int = 5, grids=GRIDS, blocks=(4, 8), log=print):
    """Time every candidate plan for CSR matrix A; returns (best, records)."""
    import torch

    assert A.kind == "csr"
    dt = capi.DTYPES[A.dtype]
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=dt.np)).cuda()
    yd = torch.zeros(int(A.s.nrows) + 64, dtype=xd.dtype, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()
    records, y0 = [], None
    for label, kind, build in _structs(A, grids, blocks):
        t0 = time.time()
        try:
            M = build()
        except capi.SparsepError as e:
            records.append(dict(struct=label, kind=kind, status=e.status, error=str(e)))
            continue
        conv_s = time.time() - t0
        for olabel, o in _options(kind):
            rec = dict(struct=label, kind=kind, option=olabel, opts=o, convert_s=round(conv_s, 3))
            try:
                p = capi.Plan(M, capi.default_opts(**o))
            except capi.SparsepError as e:
                rec.update(status=e.status, error=str(e))
                records.append(rec)
                continue
            for _ in range(2):
                p.run_device(xd.data_ptr(), yd.data_ptr(), st.cuda_stream)
            ts = []
            for _ in range(reps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                p.run_device(xd.data_ptr(), yd.data_ptr(), st.cuda_stream)
                e1.record(st)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1) * 1e3)
            y = yd[: int(A.s.nrows)].cpu().numpy()
            if y0 is None:
                y0 = y
            if np.dtype(dt.np).kind != "f":
                rec["matches_first"] = bool(np.array_equal(y, y0))
            else:
                rec["max_rel_diff_vs_first"] = float(np.abs(y.astype(np.float64) - y0).max()
                                                     / max(float(np.abs(y0).max()), 1e-300))
            us = float(np.median(ts))
            cb = int(p.info.compulsory_bytes)
            rec.update(status=0, us=round(us, 2), gbs=round(cb / (us * 1e-6) / 1e9, 1), compulsory_bytes=cb,
                       variant=p.info.variant.decode(), items=int(p.info.items))
            p.free()
            records.append(rec)
            if log:
                log(f"{label:>12} {olabel:>12} {us:9.1f} us {rec['gbs']:8.1f} GB/s")
        del M
    ok = [r for r in records if r.get("status") == 0]
    best = min(ok, key=lambda r: r["us"]) if ok else None
    return best, records


def workload(name: str, dtype: str):
    """CSR matrix and x of a benchmark configuration."""
    npdt = capi.DTYPES[dtype].np
    if name == "uniform8":
        n, m, r, c, v, x = synth.uniform_rows(4096, 4096, 8, 0, npdt)
    elif name == "zipf":
        n, m, r, c, v, x = synth.zipf_rows(seed=1, dtype=npdt)
    elif name in ("banded4", "banded8"):
        b = 4 if name == "banded4" else 8
        B = synth.block_banded(rb=b, cb=b, dtype=npdt)
        r, c, v = synth.bcsr_triplets(B)
        keep = v != 0
        r, c, v = r[keep], c[keep], v[keep]
        o = np.lexsort((c, r))
        r, c, v = r[o], c[o], v[o]
        n = m = B["nrows"]
        x = B["x"]
    else:
        raise ValueError(name)
    return capi.csr(dtype, n, m, *synth.to_csr(n, r, c, v)), x


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sparsep_b200.tune")
    ap.add_argument("--workload", default="zipf", choices=["uniform8", "zipf", "banded4", "banded8"])
    ap.add_argument("--dtype", default="f32", choices=list(capi.DTYPES))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", type=Path)
    a = ap.parse_args(argv)
    A, x = workload(a.workload, a.dtype)
    best, records = autotune(A, x, reps=a.reps)
    res = dict(workload=a.workload, dtype=a.dtype, nrows=int(A.s.nrows), nnz=int(A.s.nnz), best=best,
               records=records)
    if a.out:
        a.out.parent.mkdir(parents=True, exist_ok=True)
        a.out.write_text(json.dumps(res, indent=1))
    print(json.dumps(dict(workload=a.workload, dtype=a.dtype, best=best)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
