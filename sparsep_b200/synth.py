"""Seeded synthetic matrices with the shapes of the benchmark workloads.

The SuiteSparse inputs the reference scripts download are not available, so
every workload is generated here from a numpy PCG64 stream seeded as stated.
Matrices are returned as (nrows, ncols, rows, cols, vals) triplets sorted by
(row, col), plus CSR / BCSR builders.

Workloads (sizes as named):
  uniform8   4096 x 4096, 8 distinct uniform columns per row, integer values
             and x in [-8, 8], seed 0 (the plain CSR INT32 correctness case)
  zipf       1,048,576^2, row lengths Zipf(2.0) capped at 50,000 and rescaled
             to 16 * 2^20 nonzeros (mean 16), uniform distinct columns,
             values and x U[-1, 1], seed 1
  banded     2,097,152 rows, block-banded: block half-bandwidth 32 blocks, 30%
             of in-band blocks present, 60% fill inside present blocks,
             integer values U{-4..4} (FP: U[-1, 1]), seed 2
"""
from __future__ import annotations

import numpy as np


def _dedupe_cols(rng, row_of, ncols, cols):
    """Redraw duplicate (row, col) pairs until every row has distinct columns."""
    for _ in range(64):
        key = row_of.astype(np.int64) * ncols + cols
        order = np.argsort(key, kind="stable")
        k = key[order]
        dup = np.zeros(k.size, dtype=bool)
        dup[1:] = k[1:] == k[:-1]
        if not dup.any():
            return row_of[order], cols[order]
        bad = order[dup]
        cols[bad] = rng.integers(0, ncols, bad.size)
    raise RuntimeError("could not draw distinct columns")


def values(rng, n, dtype, lo_int=-8, hi_int=8):
    dt = np.dtype(dtype)
    if dt.kind == "f":
        return rng.uniform(-1.0, 1.0, n).astype(dt)
    return rng.integers(lo_int, hi_int + 1, n).astype(dt)


def uniform_rows(nrows, ncols, per_row, seed, dtype):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(nrows, dtype=np.uint32), per_row)
    cols = rng.integers(0, ncols, rows.size).astype(np.int64)
    rows, cols = _dedupe_cols(rng, rows, ncols, cols)
    vals = values(rng, rows.size, dtype)
    x = values(rng, ncols, dtype)
    return nrows, ncols, rows.astype(np.uint32), cols.astype(np.uint32), vals, x


def zipf_lengths(rng, nrows, nnz, a=2.0, cap=50_000):
    lens = np.minimum(rng.zipf(a, nrows), cap).astype(np.float64)
    lens = np.maximum(1, np.floor(lens * (nnz / lens.sum()))).astype(np.int64)
    lens = np.minimum(lens, cap)
    for _ in range(1000):
        diff = int(nnz - lens.sum())
        if diff == 0:
            break
        if diff > 0:
            room = np.nonzero(lens < cap)[0]
            idx = rng.choice(room, size=min(diff, room.size), replace=False)
            lens[idx] += 1
        else:
            room = np.nonzero(lens > 1)[0]
            idx = rng.choice(room, size=min(-diff, room.size), replace=False)
            lens[idx] -= 1
    assert lens.sum() == nnz
    return lens


def zipf_rows(nrows=1 << 20, ncols=1 << 20, nnz=16 << 20, seed=1, dtype=np.float32, a=2.0, cap=50_000):
    rng = np.random.default_rng(seed)
    lens = zipf_lengths(rng, nrows, nnz, a, cap)
    rows = np.repeat(np.arange(nrows, dtype=np.uint32), lens)
    cols = rng.integers(0, ncols, rows.size).astype(np.int64)
    rows, cols = _dedupe_cols(rng, rows, ncols, cols)
    vals = values(rng, rows.size, dtype)
    x = values(rng, ncols, dtype)
    return nrows, ncols, rows.astype(np.uint32), cols.astype(np.uint32), vals, x


def to_csr(nrows, rows, cols, vals):
    """Triplets sorted by (row, col) -> rowptr, colind, values."""
    rowptr = np.zeros(nrows + 1, dtype=np.uint32)
    np.cumsum(np.bincount(rows.astype(np.int64), minlength=nrows), out=rowptr[1:])
    return rowptr, cols.astype(np.uint32), vals


def block_banded(nrows=2_097_152, rb=4, cb=4, half_bw=32, p_block=0.3, p_fill=0.6, seed=2, dtype=np.int8,
                 chunk=16_384):
    """Block-banded matrix built directly as BCSR arrays.

    Generated in chunks of `chunk` block rows (one generator, drawn in chunk
    order), so the full 2M-row 8x8 case stays within a few GB.  Returns dict
    with nrows, ncols, browptr, bcolind, bval (nblocks x rb x cb, zeros at
    unfilled positions), nnz (filled positions), nnz_per_block (nonzero
    values, as the reference's countNNZperBlockBCSRMatrix) and x.
    """
    rng = np.random.default_rng(seed)
    ncols = nrows
    nbr = (nrows + rb - 1) // rb
    nbc = (ncols + cb - 1) // cb
    width = 2 * half_bw + 1
    dt = np.dtype(dtype)
    counts, bcols, bvals, npbs = [], [], [], []
    nnz = 0
    for b0 in range(0, nbr, chunk):
        b1 = min(nbr, b0 + chunk)
        present = rng.random((b1 - b0, width), dtype=np.float32) < p_block
        jj = np.arange(b0, b1)[:, None] - half_bw + np.arange(width)[None, :]
        present &= (jj >= 0) & (jj < nbc)
        counts.append(present.sum(axis=1))
        bc = jj[present].astype(np.uint32)  # row-major -> sorted by column within a block row
        nb = bc.size
        brow = np.repeat(np.arange(b0, b1), counts[-1])
        fill = rng.random((nb, rb, cb), dtype=np.float32) < p_fill
        # rows / cols past the matrix edge stay empty
        fill &= ((brow[:, None] * rb + np.arange(rb)[None, :]) < nrows)[:, :, None]
        fill &= ((bc[:, None].astype(np.int64) * cb + np.arange(cb)[None, :]) < ncols)[:, None, :]
        if dt.kind == "f":
            v = rng.uniform(-1.0, 1.0, (nb, rb, cb)).astype(dt)
        else:
            v = rng.integers(-4, 5, (nb, rb, cb), dtype=np.int8).astype(dt)
        v[~fill] = 0
        nnz += int(fill.sum())
        bcols.append(bc)
        bvals.append(v)
        npbs.append((v != 0).reshape(nb, -1).sum(axis=1).astype(np.uint32))
    browptr = np.zeros(nbr + 1, dtype=np.uint32)
    np.cumsum(np.concatenate(counts), out=browptr[1:])
    bval = np.concatenate(bvals) if bvals else np.zeros((0, rb, cb), dt)
    x = rng.uniform(-1.0, 1.0, ncols).astype(dt) if dt.kind == "f" else rng.integers(-4, 5, ncols).astype(dt)
    return dict(nrows=nrows, ncols=ncols, rb=rb, cb=cb, nbr=nbr, nbc=nbc, browptr=browptr,
                bcolind=np.concatenate(bcols), bval=bval, nnz=nnz, nnz_per_block=np.concatenate(npbs), x=x)


def bcsr_triplets(B):
    """(rows, cols, vals) of the stored block entries (explicit zeros included)."""
    rb, cb = B["rb"], B["cb"]
    nb = B["bcolind"].size
    counts = np.diff(B["browptr"].astype(np.int64))
    brow = np.repeat(np.arange(B["nbr"]), counts)
    r = (brow[:, None, None] * rb + np.arange(rb)[None, :, None]) + 0 * np.arange(cb)[None, None, :]
    c = (B["bcolind"][:, None, None].astype(np.int64) * cb + np.arange(cb)[None, None, :]) + 0 * np.arange(rb)[None, :, None]
    m = (r < B["nrows"]) & (c < B["ncols"])
    return r[m].astype(np.uint32), c[m].astype(np.uint32), B["bval"][m]


def stratified_cols(rng, lens, lo, hi):
    """Per row r, lens[r] <= hi[r] - lo[r] distinct sorted columns in
    [lo[r], hi[r]): one uniform draw inside each of the integer strata
    [floor(i w / len), floor((i + 1) w / len)), w = hi - lo, which are disjoint
    and non-empty (no sort, no redraw needed)."""
    lens = np.asarray(lens, dtype=np.int64)
    total = int(lens.sum())
    rowptr = np.zeros(lens.size + 1, dtype=np.int64)
    np.cumsum(lens, out=rowptr[1:])
    row_of = np.repeat(np.arange(lens.size), lens)
    i = np.arange(total, dtype=np.int64) - rowptr[:-1][row_of]
    w = (hi - lo).astype(np.int64)[row_of]
    ln = lens[row_of]
    a = i * w // ln
    span = (i + 1) * w // ln - a
    off = np.minimum(np.floor(rng.random(total) * span).astype(np.int64), span - 1)
    col = lo[row_of] + a + off
    return rowptr.astype(np.uint32), col.astype(np.uint32)


def batch_matrix(rng, n, kind, dtype):
    """One square matrix of the batch workload: 'uniform' (4-64 nnz/row),
    'zipf' (power-law row lengths, exponent 2, mean ~16) or 'banded'."""
    lo = np.zeros(n, dtype=np.int64)
    hi = np.full(n, n, dtype=np.int64)
    if kind == "uniform":
        lens = rng.integers(4, 65, n)
    elif kind == "zipf":
        lens = np.minimum(rng.zipf(2.0, n) * 4, min(n, 50_000))
    else:
        bw = int(rng.integers(8, 65))
        r = np.arange(n)
        lo = np.maximum(0, r - bw)
        hi = np.minimum(n, r + bw + 1)
        lens = np.minimum(hi - lo, rng.integers(4, 65, n))
    lens = np.minimum(lens, hi - lo)
    rowptr, cols = stratified_cols(rng, lens, lo, hi)
    dt = np.dtype(dtype)
    vals = rng.uniform(-1, 1, cols.size).astype(dt) if dt.kind == "f" else rng.integers(-8, 9, cols.size).astype(dt)
    return rowptr, cols, vals


def batch_workload(nmats=512, seed=3, dtype=np.float32, rows_lo=1_000, rows_hi=256_000, k_max=32):
    """The batched workload: nmats square matrices, rows log-uniform in
    [rows_lo, rows_hi], a mix of uniform / Zipf / banded structure, each with
    1..k_max right-hand sides (x uniform in [-1, 1], integers in [-8, 8])."""
    rng = np.random.default_rng(seed)
    out = []
    kinds = ("uniform", "zipf", "banded")
    for m in range(nmats):
        n = int(np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi))))
        kind = kinds[m % 3]
        k = int(rng.integers(1, k_max + 1))
        rowptr, cols, vals = batch_matrix(rng, n, kind, dtype)
        dt = np.dtype(dtype)
        x = rng.uniform(-1, 1, (n, k)).astype(dt) if dt.kind == "f" else rng.integers(-8, 9, (n, k)).astype(dt)
        out.append(dict(n=n, kind=kind, k=k, rowptr=rowptr, colind=cols, values=vals, x=x))
    return out


# ---------------------------------------------------------------------------
# Training and held-out matrices of the learned variant selector
# ---------------------------------------------------------------------------
SELECTOR_FAMILIES = ("uniform", "zipf", "banded", "blockdiag", "rmat")


def _rows_from_pairs(n, rows, cols):
    """Distinct (row, col) pairs sorted by row then column -> rowptr, colind."""
    key = np.unique(rows.astype(np.int64) * n + cols.astype(np.int64))
    r = (key // n).astype(np.int64)
    rowptr = np.zeros(n + 1, dtype=np.uint32)
    np.cumsum(np.bincount(r, minlength=n), out=rowptr[1:])
    return rowptr, (key % n).astype(np.uint32)


def selector_matrix(rng, family: str, n: int, mean_len: float):
    """One square training matrix (rowptr, colind) of a family:
    uniform   row lengths uniform in [1, 2 mean_len - 1], columns anywhere;
    zipf      power-law row lengths (exponent 2) scaled to mean_len;
    banded    columns within a band of half-width 2-64 x mean_len;
    blockdiag dense-ish diagonal blocks of 16-512 rows, columns inside the block;
    rmat      R-MAT graph, quadrant probabilities a/b/c/d = 0.57/0.19/0.19/0.05,
              n rounded to a power of two, about n * mean_len edges."""
    lo = np.zeros(n, dtype=np.int64)
    hi = np.full(n, n, dtype=np.int64)
    m = max(1, int(round(mean_len)))
    if family == "uniform":
        lens = rng.integers(1, 2 * m, n)
    elif family == "zipf":
        z = rng.zipf(2.0, n).astype(np.float64)
        lens = np.maximum(1, np.round(z * (m / z.mean()))).astype(np.int64)
    elif family == "banded":
        bw = int(m * rng.uniform(2, 64))
        r = np.arange(n)
        lo, hi = np.maximum(0, r - bw), np.minimum(n, r + bw + 1)
        lens = rng.integers(max(1, m // 2), 2 * m, n)
    elif family == "blockdiag":
        bs = int(rng.choice([16, 32, 64, 128, 256, 512]))
        r = np.arange(n)
        lo = (r // bs) * bs
        hi = np.minimum(n, lo + bs)
        lens = rng.integers(max(1, m // 2), 2 * m, n)
    elif family == "rmat":
        scale = max(4, int(round(np.log2(n))))
        n = 1 << scale
        ne = n * m
        rows = np.zeros(ne, dtype=np.int64)
        cols = np.zeros(ne, dtype=np.int64)
        a, b, c = 0.57, 0.19, 0.19
        for _ in range(scale):
            u = rng.random(ne)
            rows = rows * 2 + (u >= a + b)
            cols = cols * 2 + (((u >= a) & (u < a + b)) | (u >= a + b + c))
        rp, ci = _rows_from_pairs(n, rows, cols)
        return n, rp, ci
    else:
        raise ValueError(family)
    lens = np.minimum(np.minimum(lens, hi - lo), 50_000)
    rp, ci = stratified_cols(rng, lens, lo, hi)
    return n, rp, ci


def selector_one(seed: int, i: int, rows_lo=1_000, rows_hi=262_144, len_lo=2, len_hi=64, max_nnz=4_000_000,
                 k_max=32):
    """Training matrix i of the stream `seed` (its own generator, so any
    subset can be built in any process): family in turn, rows and mean row
    length log-uniform, k uniform in 1..k_max, nonzeros capped at max_nnz
    (the row count shrinks to fit).  -> dict(family, n, rowptr, colind, k)."""
    rng = np.random.default_rng([seed, i])
    fam = SELECTOR_FAMILIES[i % len(SELECTOR_FAMILIES)]
    n = int(np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi))))
    ml = float(np.exp(rng.uniform(np.log(len_lo), np.log(len_hi))))
    n = max(rows_lo // 2, min(n, int(max_nnz / ml)))
    k = int(rng.integers(1, k_max + 1))
    n, rp, ci = selector_matrix(rng, fam, n, ml)
    return dict(family=fam, n=n, rowptr=rp, colind=ci, k=k)


def selector_workload(count: int, seed: int, **kw):
    """Training matrices 0 .. count - 1 of the stream `seed`."""
    return [selector_one(seed, i, **kw) for i in range(count)]
