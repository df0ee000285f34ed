"""Learned choice of a CSR matrix's plan variant (sparsep_opts.autotune = 1).

A CSR input can run as any of SPARSEP_NPLANVARIANTS plans (CSR item sizes,
the TMA pipeline, the heavy-row stripes, COO lock-free / atomic, BCSR 4x4 /
8x8, BCOO 4x4, 2D equal-tile COO); sparsep_plan_autotune_csr_f32 times them
all.  This module builds a timing database of those times over seeded
synthetic matrices of the selector families (uniform, Zipf, banded,
block-diagonal, R-MAT a/b/c/d = 0.57/0.19/0.19/0.05; 10k-4M rows, 2-128
nonzeros per row, at most 8 M nonzeros per matrix so that a database is
timed in minutes), trains the selector network on it with the library's own
kernels (the MLP of the batch selector: its first SPARSEP_NPLANVARIANTS
outputs, the rest marked not applicable), evaluates its regret against the
exhaustive best and its speed-up over fixed CSR on held-out matrices, and
writes the weights into csrc/plan_model.cpp, which the library compiles in.

Command line (on a GPU box):
  python -m sparsep_b200.plan_selector gen --count N --seed S --out db.npz
  python -m sparsep_b200.plan_selector train --db db.npz --heldout h.npz --out model.npz
  python -m sparsep_b200.plan_selector export --model model.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import capi, selector, synth

NPLAN = 10
DATA = Path(__file__).resolve().parent / "selector_data"
MODEL = DATA / "plan_model.npz"
CPP = Path(__file__).resolve().parent / "csrc" / "plan_model.cpp"
FIXED_CSR = 0  # variant index of the default CSR plan


def variant_names() -> list[str]:
    L = capi.lib()
    L.sparsep_plan_variant_name.restype = C.c_char_p
    return [L.sparsep_plan_variant_name(v).decode() for v in range(NPLAN)]


def autotune_times(A: capi.HostMatrix, reps: int = 3) -> tuple[np.ndarray, int]:
    """Median time (us) of every plan variant of A (0: not applicable) and the best index."""
    L = capi.lib()
    f = getattr(L, f"sparsep_plan_autotune_csr_{A.dtype}")
    f.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    t = (C.c_double * NPLAN)()
    best = C.c_int32(-1)
    capi.check(f(A.ref, reps, t, C.byref(best)), "plan_autotune")
    return np.array(list(t), dtype=np.float64), int(best.value)


def _gen(args):
    seed, i = args
    d = synth.selector_one(seed, i, rows_lo=10_000, rows_hi=4_000_000, len_lo=2, len_hi=128, max_nnz=8_000_000,
                           k_max=1)
    d["feat"] = capi.features(d["n"], d["n"], d["rowptr"], d["colind"], 1)
    d["values"] = np.random.default_rng([seed, i, 7]).uniform(-1, 1, d["colind"].size).astype(np.float32)
    return i, d


def timing_db(count: int, seed: int, reps: int = 3, workers: int | None = None, log=print) -> dict:
    """Features and per-variant times (us; 0 = not applicable) of matrices
    0 .. count - 1 of stream `seed`, generated by spawned processes while the
    GPU times the previous ones."""
    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    feats = np.zeros((count, capi.NFEATURES), dtype=np.float32)
    times = np.zeros((count, NPLAN), dtype=np.float32)
    meta = np.zeros((count, 3), dtype=np.int64)  # family index, n, nnz
    t0 = time.time()
    with mp.get_context("spawn").Pool(workers) as pool:
        for i, d in pool.imap(_gen, [(seed, i) for i in range(count)], chunksize=2):
            A = capi.csr("f32", d["n"], d["n"], d["rowptr"], d["colind"], d["values"])
            times[i] = autotune_times(A, reps)[0]
            feats[i] = d["feat"]
            meta[i] = (synth.SELECTOR_FAMILIES.index(d["family"]), d["n"], int(d["rowptr"][-1]))
            if log and (i + 1) % 25 == 0:
                log(f"timed {i + 1}/{count} ({time.time() - t0:.0f}s)")
    return dict(feats=feats, times=times, meta=meta, seed=np.int64(seed), variants=np.array(variant_names()))


def padded(times: np.ndarray) -> np.ndarray:
    """Plan-variant times in the network's SPARSEP_NVARIANTS columns (the
    others 0: not applicable)."""
    out = np.zeros((times.shape[0], capi.NVARIANTS), dtype=np.float32)
    out[:, :NPLAN] = times
    return out


def evaluate(logits: np.ndarray, times: np.ndarray) -> dict:
    """Run time of the picks against the exhaustive best and fixed CSR,
    summed over the matrices (each timed alone)."""
    ok = (times > 0).any(axis=1) & (times[:, FIXED_CSR] > 0)
    t, lg = times[ok], logits[ok][:, :NPLAN]
    best = np.where(t > 0, t, np.inf).min(axis=1)
    pick = t[np.arange(len(t)), np.where(t > 0, lg, -np.inf).argmax(axis=1)]
    csr = t[:, FIXED_CSR]
    return dict(samples=int(len(t)), regret_total=float(pick.sum() / best.sum() - 1.0),
                regret_mean=float(np.mean(pick / best - 1.0)), regret_median=float(np.median(pick / best - 1.0)),
                fixed_csr_regret_total=float(csr.sum() / best.sum() - 1.0),
                speedup_vs_fixed_csr=float(csr.sum() / pick.sum()), exact_best=float(np.mean(pick == best)),
                best_counts=np.bincount(np.where(t > 0, t, np.inf).argmin(axis=1), minlength=NPLAN).tolist())


def export(model: dict, path: Path = CPP):
    """Write the trained weights as the library's compiled-in plan model."""
    wb = model["wb"].astype(np.uint16)
    lines = ["// plan_model.cpp -- weights of the plan-variant network used by",
             "// sparsep_opts.autotune = 1 (MLP 16-64-64-K, BF16 bits, then the feature",
             "// standardisation).  Written by `python -m sparsep_b200.plan_selector export`",
             f"// from the model trained on {model.get('note', 'the plan timing database')}.",
             "#include <cstdint>", "", "namespace sparsep {", "namespace {",
             f"const uint16_t kWb[{wb.size}] = {{"]
    for s in range(0, wb.size, 16):
        lines.append("    " + ", ".join(f"0x{v:04x}" for v in wb[s:s + 16]) + ",")
    lines.append("};")
    for name, arr in (("kMean", model["mean"]), ("kStd", model["std"])):
        lines.append(f"const float {name}[{arr.size}] = {{" + ", ".join(f"{float(v):.9e}f" for v in arr) + "};")
    lines += ["}  // namespace", "const uint16_t *plan_model_weights() { return kWb; }",
              "const float *plan_model_mean() { return kMean; }", "const float *plan_model_std() { return kStd; }",
              "}  // namespace sparsep", ""]
    path.write_text("\n".join(lines))


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sparsep_b200.plan_selector")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gen")
    g.add_argument("--count", type=int, required=True)
    g.add_argument("--seed", type=int, required=True)
    g.add_argument("--reps", type=int, default=3)
    g.add_argument("--out", type=Path, required=True)
    t = sub.add_parser("train")
    t.add_argument("--db", type=Path, nargs="+", required=True)
    t.add_argument("--heldout", type=Path, required=True)
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--out", type=Path, default=MODEL)
    x = sub.add_parser("export")
    x.add_argument("--model", type=Path, default=MODEL)
    x.add_argument("--cpp", type=Path, default=CPP)
    a = ap.parse_args(argv)
    if a.cmd == "gen":
        db = timing_db(a.count, a.seed, reps=a.reps)
        a.out.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(a.out, **db)
        return 0
    if a.cmd == "train":
        dbs = [np.load(p) for p in a.db]
        feats = np.concatenate([d["feats"] for d in dbs])
        times = np.concatenate([d["times"] for d in dbs])
        model = selector.train(feats, padded(times), steps=a.steps)
        sel = selector.selector(model)
        h = np.load(a.heldout)
        meta = dict(train_samples=int(len(feats)), heldout_samples=int(len(h["feats"])), steps=a.steps,
                    train_eval=evaluate(sel.scores(feats), times),
                    heldout_eval=evaluate(sel.scores(h["feats"]), h["times"]), variants=variant_names())
        a.out.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(a.out, wb=model["wb"], mean=model["mean"], std=model["std"], meta=json.dumps(meta))
        print(json.dumps(meta, indent=1))
        return 0
    if a.cmd == "export":
        z = np.load(a.model, allow_pickle=False)
        meta = json.loads(str(z["meta"]))
        export(dict(wb=z["wb"], mean=z["mean"], std=z["std"],
                    note=f"{meta['train_samples']} matrices (held-out regret "
                         f"{meta['heldout_eval']['regret_total']:.3f})"), a.cpp)
        return 0
    return 2


if __name__ == "__main__":
    sys.exit(main())
