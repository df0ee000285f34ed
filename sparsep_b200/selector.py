"""Learned variant selector for the batched multi-RHS SpMV.

The batch kernel runs every matrix with one of the SPARSEP_NVARIANTS row
routines (`capi.batch_candidates()`); the exhaustive autotuner times all of
them per matrix.  The selector replaces that search by a network: 16 cheap
sparsity features of the matrix and its right-hand-side count
(`capi.features`) go through an MLP 16-64-64-36 whose forward, loss/gradient
and Adam kernels are the library's own CUDA kernels (sparsep_mlp_*), BF16
weights with FP32 accumulation.  It is trained on the autotuner's timings of
seeded synthetic matrices; where its softmax confidence is low the batch
falls back to the exhaustive autotuner for that matrix
(`Batch.select(selector, min_confidence)`).  It only picks a schedule: every
variant computes the same result (integers bit-exact).

Command line (on a GPU box):
  python -m sparsep_b200.selector gen   --count N --seed S --out db.npz
  python -m sparsep_b200.selector train --db db.npz --out model.npz
  python -m sparsep_b200.selector eval  --model model.npz --db heldout.npz
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import capi, synth

DATA = Path(__file__).resolve().parent / "selector_data"
MODEL = DATA / "model.npz"


def candidates() -> np.ndarray:
    """(NVARIANTS, 4) int32: mode, lanes, item_work, vec of every candidate."""
    return np.array([v.as_tuple() for v in capi.batch_candidates()], dtype=np.int32)


def default_index(k: int) -> int:
    """Candidate index of the library's default (untuned) variant for k."""
    L = capi.lib()
    capi._batch_sigs(L)
    v = capi.BatchVariant()
    L.sparsep_batch_variant_default(int(k), v)
    cand = candidates()
    for i, c in enumerate(cand):
        if c[0] == v.mode and c[1] == v.lanes and c[3] == max(1, v.vec):
            return i
    raise RuntimeError("default variant is not a candidate")


# ---------------------------------------------------------------------------
# timing database
# ---------------------------------------------------------------------------
def _gen(args):
    seed, i, kw = args
    d = synth.selector_one(seed, i, **kw)
    d["feat"] = capi.features(d["n"], d["n"], d["rowptr"], d["colind"], d["k"])
    return i, d


def timing_db(count: int, seed: int, reps: int = 3, chunk: int = 48, workers: int | None = None,
              log=print, **ranges) -> dict:
    """Features and per-candidate median times (us; 0 = not applicable) of
    training matrices 0 .. count - 1 of stream `seed`, each timed alone on
    the current GPU.  Matrices are generated by a pool of spawned processes
    while the GPU times the previous chunk; `ranges` override the generator's
    row, row-length and size ranges (synth.selector_one)."""
    workers = workers or max(1, min(32, (os.cpu_count() or 2) - 1))
    ctx = mp.get_context("spawn")
    feats = np.zeros((count, capi.NFEATURES), dtype=np.float32)
    times = np.zeros((count, capi.NVARIANTS), dtype=np.float32)
    meta = np.zeros((count, 4), dtype=np.int64)  # family index, n, nnz, k
    cands = capi.batch_candidates()
    t0 = time.time()
    with ctx.Pool(workers) as pool:
        it = pool.imap(_gen, [(seed, i, ranges) for i in range(count)], chunksize=4)
        done = 0
        while done < count:
            ds = [next(it)[1] for _ in range(min(chunk, count - done))]
            mats = [capi.csr("f32", d["n"], d["n"], d["rowptr"], d["colind"],
                             np.ones(d["colind"].size, dtype=np.float32)) for d in ds]
            b = capi.Batch("f32", mats, [d["k"] for d in ds])
            for j, d in enumerate(ds):
                i = done + j
                feats[i] = d["feat"]
                meta[i] = (synth.SELECTOR_FAMILIES.index(d["family"]), d["n"], int(d["rowptr"][-1]), d["k"])
                for c, v in enumerate(cands):
                    us = b.time_variant(j, v, reps)
                    times[i, c] = 0.0 if us is None else us
            b.free()
            done += len(ds)
            if log:
                log(f"timed {done}/{count} ({time.time() - t0:.0f}s)")
    return dict(feats=feats, times=times, meta=meta, seed=np.int64(seed), candidates=candidates())


# ---------------------------------------------------------------------------
# training (the library's CUDA kernels; torch only holds device buffers)
# ---------------------------------------------------------------------------
def init_weights(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases, packed as the kernels expect."""
    rng = np.random.default_rng(seed)
    F, H, K = capi.NFEATURES, 64, capi.NVARIANTS
    parts = []
    for fan_in, fan_out in ((F, H), (H, H), (H, K)):
        lim = np.sqrt(6.0 / fan_in)
        parts += [rng.uniform(-lim, lim, fan_in * fan_out), np.zeros(fan_out)]
    return np.concatenate(parts).astype(np.float32)


def standardise(feats: np.ndarray):
    mean = feats.mean(axis=0).astype(np.float32)
    std = feats.std(axis=0).astype(np.float32)
    std[std <= 0] = 1.0
    return mean, std


def train(feats: np.ndarray, times: np.ndarray, steps: int = 3000, lr: float = 3e-3, seed: int = 0,
          weight_decay: float = 1e-4, alpha: float = 0.5, ce_weight: float = 0.02, tau: float = 0.05,
          log_every: int = 500, log=print) -> dict:
    """Full-batch Adam on the selector loss (expected regret of a softmax pick
    plus ce_weight x cross-entropy to softmax(-regret / tau), each matrix
    weighted by (its best time / the mean)^alpha); returns the model dict."""
    import torch

    L = capi.lib()
    capi._batch_sigs(L)
    dev = torch.device("cuda")
    n = feats.shape[0]
    mean, std = standardise(feats)
    X = torch.tensor((feats - mean) / std, dtype=torch.float32, device=dev).contiguous()
    T = torch.tensor(times, dtype=torch.float32, device=dev).contiguous()
    tb = np.where(times > 0, times, np.inf).min(axis=1)
    tb = tb[np.isfinite(tb)]
    wscale = float(1.0 / tb.mean())
    w = torch.tensor(init_weights(seed), device=dev)
    NP = w.numel()
    assert NP == L.sparsep_mlp_nparams()
    wb = torch.zeros(NP, dtype=torch.int16, device=dev)
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    g = torch.zeros_like(w)
    loss = torch.zeros(1, device=dev)
    scratch = torch.zeros(int(L.sparsep_mlp_scratch_floats(n)), device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    capi.check(L.sparsep_mlp_to_bf16(w.data_ptr(), wb.data_ptr(), stream), "mlp_to_bf16")
    history = []
    for step in range(1, steps + 1):
        capi.check(L.sparsep_mlp_loss_grad(wb.data_ptr(), X.data_ptr(), T.data_ptr(), n, wscale, alpha, ce_weight,
                                           tau, g.data_ptr(), loss.data_ptr(), scratch.data_ptr(), stream),
                   "mlp_loss_grad")
        if step == 1 or step % log_every == 0 or step == steps:
            history.append((step, float(loss.item())))
            if log:
                log(f"step {step} loss {history[-1][1]:.5f}")
        capi.check(L.sparsep_mlp_adam(w.data_ptr(), wb.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), step,
                                      lr, 0.9, 0.999, 1e-8, weight_decay, stream), "mlp_adam")
    torch.cuda.synchronize()
    return dict(w=w.cpu().numpy(), wb=wb.cpu().numpy().view(np.uint16), mean=mean, std=std,
                candidates=candidates(), history=np.array(history, dtype=np.float64))


def save(model: dict, path: Path, meta: dict | None = None):
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, wb=model["wb"], mean=model["mean"], std=model["std"], candidates=model["candidates"],
                        history=model.get("history", np.zeros((0, 2))), meta=json.dumps(meta or {}))


def load(path: Path = MODEL) -> dict:
    z = np.load(path, allow_pickle=False)
    model = {k: z[k] for k in z.files}
    model["meta"] = json.loads(str(model["meta"]))
    if not np.array_equal(model["candidates"], candidates()):
        raise ValueError("model was trained for another candidate list")
    return model


def selector(model: dict) -> capi.Selector:
    return capi.Selector(model["wb"], model["mean"], model["std"])


# ---------------------------------------------------------------------------
# evaluation against the exhaustive autotuner and the default variant
# ---------------------------------------------------------------------------
def applicable(times: np.ndarray) -> np.ndarray:
    return times > 0


def picks(logits: np.ndarray, times: np.ndarray) -> np.ndarray:
    return np.where(applicable(times), logits, -np.inf).argmax(axis=1)


def evaluate(logits: np.ndarray, times: np.ndarray, k: np.ndarray) -> dict:
    """Run time of the picks relative to the exhaustive best and to the
    default variant, summed over the matrices (each timed alone)."""
    ok = applicable(times).any(axis=1)
    t, lg, k = times[ok], logits[ok], k[ok]
    best = np.where(t > 0, t, np.inf).min(axis=1)
    pick = t[np.arange(len(t)), picks(lg, t)]
    dflt = t[np.arange(len(t)), [default_index(int(kk)) for kk in k]]
    return dict(samples=int(len(t)),
                regret_total=float(pick.sum() / best.sum() - 1.0),
                regret_mean=float(np.mean(pick / best - 1.0)),
                regret_median=float(np.median(pick / best - 1.0)),
                default_regret_total=float(dflt.sum() / best.sum() - 1.0),
                speedup_vs_default=float(dflt.sum() / pick.sum()),
                exact_best=float(np.mean(pick == best)))


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sparsep_b200.selector")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gen")
    g.add_argument("--count", type=int, required=True)
    g.add_argument("--seed", type=int, required=True)
    g.add_argument("--reps", type=int, default=3)
    g.add_argument("--out", type=Path, required=True)
    g.add_argument("--rows-lo", type=int, default=1_000)
    g.add_argument("--rows-hi", type=int, default=262_144)
    g.add_argument("--len-hi", type=int, default=64)
    g.add_argument("--max-nnz", type=int, default=4_000_000)
    t = sub.add_parser("train")
    t.add_argument("--db", type=Path, nargs="+", required=True)
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--heldout", type=Path)
    t.add_argument("--out", type=Path, default=MODEL)
    e = sub.add_parser("eval")
    e.add_argument("--model", type=Path, default=MODEL)
    e.add_argument("--db", type=Path, required=True)
    a = ap.parse_args(argv)
    if a.cmd == "gen":
        db = timing_db(a.count, a.seed, reps=a.reps, rows_lo=a.rows_lo, rows_hi=a.rows_hi, len_hi=a.len_hi,
                       max_nnz=a.max_nnz)
        a.out.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(a.out, **db)
        return 0
    if a.cmd == "train":
        dbs = [np.load(p) for p in a.db]
        feats = np.concatenate([d["feats"] for d in dbs])
        times = np.concatenate([d["times"] for d in dbs])
        model = train(feats, times, steps=a.steps, lr=a.lr, seed=a.seed)
        meta = dict(train_samples=int(len(feats)), steps=a.steps, lr=a.lr, seed=a.seed, alpha=0.5, ce_weight=0.02,
                    tau=0.05,
                    final_loss=float(model["history"][-1, 1]), db=[p.name for p in a.db])
        sel = selector(model)
        meta["train_eval"] = evaluate(sel.scores(feats), times, np.concatenate([d["meta"][:, 3] for d in dbs]))
        if a.heldout:
            h = np.load(a.heldout)
            meta["heldout_eval"] = evaluate(sel.scores(h["feats"]), h["times"], h["meta"][:, 3])
        save(model, a.out, meta)
        print(json.dumps(meta, indent=1))
        return 0
    if a.cmd == "eval":
        model = load(a.model)
        h = np.load(a.db)
        print(json.dumps(evaluate(selector(model).scores(h["feats"]), h["times"], h["meta"][:, 3]), indent=1))
        return 0
    return 2


if __name__ == "__main__":
    sys.exit(main())
