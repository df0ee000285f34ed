"""SpMV benchmark: GB/s and fraction of the HBM roofline on one B200.

Workload (default): FP32 CSR SpMV, 1D row partitions with nnz balance (the
GPU planner's auto items), on the 1,048,576 x 1,048,576 Zipf power-law matrix
(row lengths Zipf(2.0) capped at 50,000, mean 16, 16,777,216 nonzeros,
uniform distinct columns, values and x U[-1, 1], seed 1), synthetic.

One step = one SpMV over the whole matrix (inputs resident in HBM).  The L2
(126 MB) is flushed before every timed step by writing a 256 MB buffer; each
step is timed with CUDA events on the launching stream.  `value` is
compulsory bytes / device time summed over all ranks' steps (replicas, weak
scaling).  `e2e` is the same metric through sparsep_execute_host: pinned host
x in, pinned host y out, copies inside the timed region.  `clocks` is sampled
through NVML every millisecond during the timed region.

`batched` / `batched_i32` (one GPU): the batched multi-RHS path on 512
matrices, FP32 and INT32 -- plain per-matrix launches against the one-launch
work queue with the default, learned (sparsep_batch_select) and exhaustively
autotuned variants, a sample checked against the reference's host SpMV.

`configs` (one GPU): every other configuration of the workload list -- the
4096-row uniform INT32 CSR; the Zipf matrix in FP32 / FP64 as CSR and COO, 1D
with auto items, row / nnz balance over 2048 parts, lock-free and atomic, and
2D equal (D), equal-width (RBD) and variable (BD) tilings; the 2M-row
block-banded matrix as BCSR / BCOO 4x4 and 8x8 in INT8 / INT16 / INT64 /
FP32, block and nnz balance over 2048 parts.  Each entry: device time (L2
flushed), GB/s of compulsory bytes, fraction of the measured HBM copy
bandwidth, the reference's host SpMV for that kind on one core, and the check
against its result (integers bit-exact, FP within 2 gamma_n sum|a x|).

The headline run is gated: its y must match the reference's host SpMV within
that bound, or the run fails.

--impl reference times the reference's own host SpMV (spmv_host of
spmv/1D/CSR-row/host/app.c, compiled from the reference sources into
oracle/_ref) on the box's host cores: row slices of the matrix run the
unchanged reference loop on all threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "zipf-1M-csr-f32-1d"
METRIC = "SpMV GB/s (compulsory bytes / kernel time), FP32 CSR, 1M-row Zipf power-law matrix"
FALLBACK_HBM = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM)), "measured"
    return FALLBACK_HBM, "fallback"


def make_matrix():
    import sparsep_b200 as sp

    t0 = time.time()
    n, m, rows, cols, vals, x = sp.synth.zipf_rows(seed=1, dtype=np.float32)
    rowptr, colind, values = sp.synth.to_csr(n, rows, cols, vals)
    log(f"[bench] generated zipf matrix {n}x{m} nnz={rows.size} in {time.time() - t0:.1f}s "
        f"(max row {int(np.diff(rowptr.astype(np.int64)).max())})")
    return n, m, rowptr, colind, values, x


def compulsory_bytes(n, m, nnz, s=4):
    return nnz * (4 + s) + (n + 1) * 4 + m * s + n * s


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only
    queries) every millisecond by a thread during the timed region."""
    REASONS = (("nvmlClocksEventReasonHwSlowdown", "hw_slowdown"),
               ("nvmlClocksEventReasonHwThermalSlowdown", "hw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwThermalSlowdown", "sw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwPowerCap", "sw_power_cap"))

    def __init__(self, dev):
        self.dev = dev
        self.rows = []
        self.err = None

    def _handle(self):
        import pynvml as nv
        import torch

        nv.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.dev)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv, nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv, nv.nvmlDeviceGetHandleByIndex(self.dev)

    def _sample(self):
        sm = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
        r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        self.rows.append((sm, [name for bit, name in self.bits if r & bit]))

    def _run(self):
        try:
            while not self.stop.is_set():
                self._sample()
                self.stop.wait(0.001)
        except Exception as e:
            self.err = repr(e)

    def __enter__(self):
        import threading

        self.stop = threading.Event()
        self.t = None
        try:  # NVML set up (and one sample taken) before the timed region starts
            self.nv, self.h = self._handle()
            self.max_mhz = self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM)
            self.bits = [(getattr(self.nv, k), name) for k, name in self.REASONS]
            self._sample()
        except Exception as e:  # no NVML: reported, not fatal
            self.err = repr(e)
            return self
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.t:
            self.t.join(timeout=5)
        try:
            self._sample()  # one more after the last timed step
        except Exception:
            pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "error": self.err}
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": sorted({x for _, rs in self.rows for x in rs}), "samples": len(self.rows),
                "source": "nvml"}


def max_over_ranks(v: float, world: int, device: str) -> float:
    """The largest of every rank's v (the slowest rank times the job)."""
    if world <= 1:
        return float(v)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_step: int, steps: int, slowest_ms: float, world: int) -> float:
    """GB/s of the whole job: every rank (replica) moves bytes_per_step per
    step, and the job lasts as long as its slowest rank."""
    return world * bytes_per_step * steps / (slowest_ms * 1e-3) / 1e9


def run_ours(args, rank, world):
    import torch
    import torch.distributed as dist

    import sparsep_b200 as sp

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    n, m, rowptr, colind, values, x = make_matrix()
    nnz = int(rowptr[-1])
    A = sp.csr("f32", n, m, rowptr, colind, values)
    plan = sp.Plan(A, sp.default_opts(heavy_rows=args.heavy_rows))
    info = plan.info
    cb = int(info.compulsory_bytes)
    assert cb == compulsory_bytes(n, m, nnz)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty(n, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    launches_per_step = int(info.kernel_launches)

    # one untimed run; its y is checked in the CPU-baseline leg below
    plan.run_device(xd.data_ptr(), yd.data_ptr(), sh)
    torch.cuda.synchronize()
    y_first = yd.cpu().numpy()

    for _ in range(args.warmup):
        flush.zero_()
        plan.run_device(xd.data_ptr(), yd.data_ptr(), sh)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(dev) as clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(stream)
            plan.run_device(xd.data_ptr(), yd.data_ptr(), sh)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if world > 1:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in evs]
    tot_ms = max_over_ranks(sum(ms), world, "cuda")
    avg_ms = tot_ms / args.steps
    gbs_rank = cb / (avg_ms * 1e-3) / 1e9
    value = whole_job_gbs(cb, args.steps, tot_ms, world)

    # e2e through the C-ABI host path (pinned buffers, H2D x and D2H y per step)
    hx = torch.from_numpy(x).pin_memory()
    hy = torch.empty(n, dtype=torch.float32).pin_memory()
    lib = sp.lib()
    for _ in range(max(1, args.warmup)):
        sp.capi.check(lib.sparsep_execute_host(plan.h, C.c_void_p(hx.data_ptr()), C.c_void_p(hy.data_ptr())))
    e2e_ms, phase_steps = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sp.capi.check(lib.sparsep_execute_host(plan.h, C.c_void_p(hx.data_ptr()), C.c_void_p(hy.data_ptr())))
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
        phase_steps.append(plan.timings())  # device-timed phases of this call (outside the timed span)
    load_ms = plan.timings()[0]
    phases = np.mean(np.array(phase_steps), axis=0)  # slots 1..4 averaged over the timed calls
    e2e_avg = max_over_ranks(sum(e2e_ms) / len(e2e_ms), world, "cuda")
    y_dev = yd.cpu().numpy()
    assert np.array_equal(y_dev, hy.numpy()), "device and host paths disagree"
    # the same calls back to back, without the L2 flush and device
    # synchronisation in front of each (what those add to the spread)
    e2e_bb = []
    torch.cuda.synchronize()
    for _ in range(args.steps):
        t1 = time.perf_counter()
        sp.capi.check(lib.sparsep_execute_host(plan.h, C.c_void_p(hx.data_ptr()), C.c_void_p(hy.data_ptr())))
        e2e_bb.append((time.perf_counter() - t1) * 1e3)
    link = link_probe(hx, xd, hy, yd, reps=20)

    # the gather floor: x read at this matrix's column indices and nothing else
    ci_d = torch.from_numpy(colind[:nnz].view(np.int32)).cuda()
    probe_out = torch.empty(592 * 512, dtype=torch.float32, device="cuda")
    L = sp.lib()
    L.sparsep_probe_gather_f32.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    g_ms = []
    for i in range(args.warmup + 10):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sp.capi.check(L.sparsep_probe_gather_f32(ci_d.data_ptr(), nnz, xd.data_ptr(), probe_out.data_ptr(), 592,
                                                 C.c_void_p(sh)), "probe_gather")
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            g_ms.append(e0.elapsed_time(e1))
    gather_floor_ms = statistics.median(g_ms)
    del ci_d, probe_out

    peak, peak_kind = peaks()
    traffic = None
    tf = ROOT / "profiles" / "csr_f32_zipf1m_traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get("dram_bytes_per_launch")
    res = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(avg_ms, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Zipf power-law matrix, numpy PCG64 seed 1)",
        "config": {"workload": WORKLOAD, "nrows": n, "ncols": m, "nnz": nnz, "format": "csr",
                   "scheme": "1d", "balance": "nnz (auto items)", "variant": info.variant.decode(),
                   "items": int(info.items), "l2": "flushed (256 MB write) before every timed step",
                   "compulsory_bytes_per_step": cb, "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(gbs_rank, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(gbs_rank / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": cb, "avg_launch_ms": round(avg_ms, 5),
                     "gather_floor_ms": round(gather_floor_ms, 5),
                     "frac_of_gather_floor": round(gather_floor_ms / avg_ms, 4),
                     "gather_floor_note": "x read at this matrix's 16.7 M column indices and nothing else "
                                          "(sparsep_probe_gather_f32, 592 x 512 threads, L2 flushed): the "
                                          "random-gather bound of this SpMV"},
        "e2e": {"value": round(cb / (e2e_avg * 1e-3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": m * 4,
                "d2h_bytes_per_step": n * 4, "ms_per_step": round(e2e_avg, 4),
                "ms_quantiles": {q: round(float(np.quantile(e2e_ms, f)), 4)
                                 for q, f in (("min", 0.0), ("p50", 0.5), ("p90", 0.9), ("max", 1.0))},
                "y_bands": int(info.y_bands),
                "back_to_back_ms_quantiles": {q: round(float(np.quantile(e2e_bb, f)), 4)
                                              for q, f in (("min", 0.0), ("p50", 0.5), ("max", 1.0))},
                "link_probe": link,
                "phases_ms": {"load_input_vector": round(float(phases[1]), 4), "kernel": round(float(phases[2]), 4),
                              "retrieve_output_vector": round(float(phases[3]), 4),
                              "merge": round(float(phases[4]), 4), "load_matrix_once": round(load_ms, 3),
                              "note": "device events, mean over the timed calls; with y_bands > 0 the y copy "
                                      "overlaps the kernel and retrieve_output_vector is the part left after it"}},
        "gpu_launches": launches_per_step * args.steps,
        "gflops": round(2 * nnz / (avg_ms * 1e-3) / 1e9, 2),
        "wall_s_timed_region": round(wall, 4),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        res["cpu_baseline"], y_ref, y_abs = cpu_baseline(n, m, rowptr, colind, values, x,
                                                         budget_s=args.cpu_budget, threads=1)
        # the correctness gate: the benchmark's y (first run and last timed
        # run) against the reference's own host SpMV on the same matrix and x,
        # within 2 gamma_n sum|a x| per row; a failure ends the run
        counts = np.diff(rowptr.astype(np.int64))
        ok1, r1 = fp_check(y_first, y_ref, y_abs, counts, "f32")
        ok2, r2 = fp_check(y_dev, y_ref, y_abs, counts, "f32")
        res["check"] = {"ok": ok1 and ok2, "max_err_over_bound": round(max(r1, r2), 4),
                        "against": f"spmv_host of spmv/1D/CSR-row/host/app.c ({res['cpu_baseline']['kind']}), "
                                   "per row |y - y_ref| <= 2 gamma_n sum|a x|"}
        if not (ok1 and ok2):
            raise SystemExit(f"correctness gate failed: max err / bound = {max(r1, r2):.3g}")
    plan.free()
    return res


def link_probe(hx, xd, hy, yd, reps=20):
    """Host<->device copy rates of this box's link: the x and y sizes of the
    benchmark, pinned host memory, one copy per direction per rep on the
    current stream, device-timed; median GB/s of each direction."""
    import torch

    st = torch.cuda.current_stream()
    out = {}
    for name, dst, src in (("h2d", xd, hx), ("d2h", hy, yd)):
        ts = []
        for i in range(reps + 3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            dst.copy_(src, non_blocking=True)
            e1.record(st)
            torch.cuda.synchronize()
            if i >= 3:
                ts.append(e0.elapsed_time(e1))
        ms = statistics.median(ts)
        out[name] = {"bytes": int(src.numel() * src.element_size()), "ms": round(ms, 4),
                     "gbs": round(src.numel() * src.element_size() / (ms * 1e-3) / 1e9, 2)}
    return out


def run_batch(args, dt="f32"):
    """The batched multi-RHS path on the 512-matrix workload (FP32 or INT32):
    plain per-matrix launches (default variant per matrix) against the
    one-launch queue with the default, learned and exhaustively autotuned
    variants.  The batch's compulsory bytes (8.9 GB) exceed L2 many times over,
    so no flush is needed between timed runs.  A sample of matrices is checked
    column by column against the reference's CSR host SpMV (CPU-baseline leg:
    integers bit-exact, FP32 within 2 gamma_n sum|a x|), which is also timed."""
    import torch

    import sparsep_b200 as sp
    from sparsep_b200 import capi, selector

    t0 = time.time()
    npdt = capi.DTYPES[dt].np
    w = sp.synth.batch_workload(nmats=args.batch_mats, dtype=npdt)
    mats = [sp.csr(dt, d["n"], d["n"], d["rowptr"], d["colind"], d["values"]) for d in w]
    b = capi.Batch(dt, mats, [d["k"] for d in w])
    for m, d in enumerate(w):
        b.set_x(m, d["x"])
    setup_s = time.time() - t0
    info = b.info()
    cb = info["compulsory_bytes"]
    st = torch.cuda.Stream()

    def timeit(fn, reps=5):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    sample = list(range(0, len(w), max(1, len(w) // 24)))
    plain = timeit(lambda: b.execute_per_matrix(st.cuda_stream))
    y_plain = {m: b.get_y(m) for m in sample}
    default = timeit(lambda: b.execute(st.cuda_stream))
    sel = selector.selector(selector.load())
    t0 = time.time()
    ch_learned, _ = b.select(sel, min_confidence=0.0)
    select_s = time.time() - t0
    kinds_learned = b.item_kinds()
    learned = timeit(lambda: b.execute(st.cuda_stream))
    b.status()
    y_learned = {m: b.get_y(m) for m in sample}
    t0 = time.time()
    _, ch_tuned = b.autotune(reps=3)
    tune_s = time.time() - t0
    kinds_tuned = b.item_kinds()
    tuned = timeit(lambda: b.execute(st.cuda_stream))
    b.status()
    y_tuned = {m: b.get_y(m) for m in sample}
    b.free()

    check = {"matrices": len(sample), "columns": 0, "ok": True, "max_err_over_bound": 0.0}
    cpu_s, cpu_bytes = 0.0, 0
    if not args.no_cpu_baseline:
        ref = RefHost("csr", dt)
        for m in sample:
            d = w[m]
            A = mats[m]
            Aa = sp.csr(dt, d["n"], d["n"], d["rowptr"], d["colind"], np.abs(d["values"])) if dt == "f32" else None
            counts = np.diff(d["rowptr"].astype(np.int64))
            for j in sorted({0, d["k"] // 2, d["k"] - 1}):  # first, middle and last right-hand side
                xj = np.ascontiguousarray(d["x"][:, j])
                y_ref, sec = ref.run(A, xj)
                cpu_s += sec
                cpu_bytes += int(d["rowptr"][-1]) * 8 + (d["n"] + 1) * 4 + 2 * d["n"] * 4
                y_abs = ref.run(Aa, np.abs(xj))[0] if Aa is not None else None
                for y_all in (y_plain[m], y_learned[m], y_tuned[m]):
                    y = y_all.reshape(d["n"], d["k"])[:, j]
                    if y_abs is None:
                        ok, r = bool(np.array_equal(y, y_ref)), 0.0
                    else:
                        ok, r = fp_check(y, y_ref, y_abs, counts, dt)
                    check["ok"] &= ok
                    check["max_err_over_bound"] = max(check["max_err_over_bound"], round(r, 4))
                check["columns"] += 1
        check["against"] = ("spmv_host of spmv/1D/CSR-row/host/app.c per right-hand side, for the plain, learned "
                            "and autotuned runs: " + ("bit-exact" if dt != "f32" else "|y - y_ref| <= 2 gamma_n "
                                                      "sum|a x| per row"))

    def gbs(ms):
        return round(cb / (ms * 1e-3) / 1e9, 2)

    cands = capi.batch_candidates()

    def kinds(ch, items):
        modes = [int(cands[c].mode) for c in ch if c >= 0]
        return {"matrices_rows": modes.count(0), "matrices_merge": modes.count(1),
                "matrices_window_rows": modes.count(2), "matrices_window_merge": modes.count(3),
                "matrices_blocks": modes.count(4),
                "window_items": int(items[0]), "long_row_chunk_items": int(items[1])}

    out = {"workload": f"{len(w)} CSR matrices, rows log-uniform 1k-256k, uniform / Zipf / banded, 1-32 "
                       f"right-hand sides each, {dt.upper()} (seed 3)",
           "dtype": dt, "nnz": int(info["nnz"]), "compulsory_bytes": int(cb), "items": int(info["items"]),
           "plain_per_matrix_ms": round(plain, 3), "queue_default_ms": round(default, 3),
           "queue_learned_ms": round(learned, 3), "queue_autotuned_ms": round(tuned, 3),
           "learned_speedup_vs_plain": round(plain / learned, 3),
           "learned_over_autotuned": round(learned / tuned, 4),
           "gbs": {"plain": gbs(plain), "default": gbs(default), "learned": gbs(learned), "autotuned": gbs(tuned)},
           "select_s": round(select_s, 3), "autotune_s": round(tune_s, 2), "setup_s": round(setup_s, 1),
           "chosen": {"learned": kinds(ch_learned, kinds_learned), "autotuned": kinds(ch_tuned, kinds_tuned),
                      "note": "modes 2/3 are window items: a row range whose x tile is staged in shared "
                              "memory beside its nonzeros (a 2D tile); mode 4 block items on a 4x4 BCSR "
                              "copy (built for matrices with 4x4 block fill >= 0.25); rows "
                              "over 5120 nonzeros run as chunk items on many CTAs"},
           "check": check,
           "gpu_launches_per_step": {"plain": len(w), "queue": 1}}
    if cpu_s > 0:
        out["cpu_baseline"] = {"value": round(cpu_bytes / cpu_s / 1e9, 3), "unit": "GB/s", "cores": 1,
                               "kind": ref.kind, "sample": f"{check['columns']} single-vector passes of the "
                               f"reference's CSR spmv_host over {len(sample)} of the matrices"}
    log(f"[bench] batch {dt}: plain {plain:.2f} ms, learned {learned:.2f} ms, autotuned {tuned:.2f} ms, "
        f"check {check}")
    return out


# ---------------------------------------------------------------------------
# Every benchmark configuration: one device-timed number and one check each
# ---------------------------------------------------------------------------
# The reference directory whose spmv_host multiplies each struct kind
REF_DIR = {"csr": "1D_CSR_row", "cooe": "1D_COO_nnz", "bcsr": "1D_BCSR_nnz", "bcoo": "1D_BCOO_nnz",
           "dcsr": "2D_DCSR", "rbdcsr": "2D_RBDCSR", "bdcsr": "2D_BDCSR", "dcoo": "2D_DCOO", "rbdcoo": "2D_RBDCOO",
           "bdcoo": "2D_BDCOO"}


class RefHost:
    """The reference's own host SpMV for a struct kind and element type
    (spmv_host of that kind's host/app.c, built from the reference sources
    into oracle/_ref), else the oracle's restatement of it.  Used for the
    CPU baseline of each configuration and, with its result, as the check."""

    def __init__(self, kind, dtype):
        so = ROOT / "oracle" / "_ref" / f"libref_{REF_DIR[kind]}_{dtype}.so"
        if so.exists():
            self.fn, self.kind = C.CDLL(str(so)).ref_spmv, "reference"
        else:
            port = ROOT / "oracle" / "liboracle.so"
            if not port.exists():
                subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "liboracle.so"], check=True)
            self.fn, self.kind = getattr(C.CDLL(str(port)), f"oracle_spmv_{kind}_{dtype}"), "port"

    @staticmethod
    def lengths(A):
        """(x length, y length) the reference's host code reads and writes."""
        s = A.s
        if A.kind in ("bcsr", "bcoo"):
            return int(s.ncols) + 16, int(s.num_block_rows * s.row_block_size)
        if A.kind in ("dcsr", "dcoo"):
            return int(s.vert_partitions * s.tile_width) + 8, int(s.horz_partitions * s.tile_height)
        return int(s.ncols) + 16, int(s.nrows)

    def run(self, A, x, passes=1):
        """y and the seconds per pass of the reference's SpMV on A and x."""
        xl, yl = self.lengths(A)
        xp = np.zeros(max(xl, x.size), dtype=x.dtype)
        xp[: x.size] = x
        y = np.zeros(yl + 8, dtype=x.dtype)
        t0 = time.perf_counter()
        for _ in range(passes):
            self.fn(y.ctypes.data_as(C.c_void_p), A.ref, xp.ctypes.data_as(C.c_void_p))
        return y[: int(A.s.nrows)].copy(), (time.perf_counter() - t0) / passes


def fp_check(y, y_ref, y_abs, counts, dtype):
    """|y - y_ref| <= 2 gamma_n sum|a x| per row: both are sums of the same
    products, each within gamma_n sum|a x| of the exact value.  y_abs is the
    reference's own sum of |a||x| in the element type (within gamma_n of exact,
    covered by the 1.01 factor).  Returns (ok, max err / bound)."""
    u = 2.0 ** -24 if dtype == "f32" else 2.0 ** -53
    n = np.maximum(counts.astype(np.float64), 1.0)
    bound = 1.01 * 2 * (n * u / (1 - n * u)) * y_abs.astype(np.float64) + 1e-300
    err = np.abs(y.astype(np.float64) - y_ref.astype(np.float64))
    r = err / bound
    return bool((r <= 1.0).all()), float(r.max()) if r.size else 0.0


def time_device(plan, xd, yd, stream, flush, reps):
    """Median device time (ms) of plan on x/y with L2 flushed before each run."""
    import torch

    for _ in range(3):
        flush.zero_()
        plan.run_device(xd.data_ptr(), yd.data_ptr(), stream.cuda_stream)
    ts = []
    for _ in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.run_device(xd.data_ptr(), yd.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def measure_struct(cfg, workload, A, A_abs, x, counts, cases, peak, stream, flush, reps=10, ref_budget_s=2.0):
    """One struct: the reference's host SpMV once (CPU baseline, and its y as
    the check), then every option set in `cases` planned, device-timed and
    checked: integers bit for bit against the reference, FP within
    2 gamma_n sum|a x| of it.  A_abs: the same struct with |values| (FP)."""
    import torch

    import sparsep_b200 as sp

    dt = A.dtype
    ref = RefHost(A.kind, dt)
    y_ref, sec = ref.run(A, x)
    passes = max(1, min(10, int(ref_budget_s / max(sec, 1e-6))))
    if passes > 1:
        sec = ref.run(A, x, passes)[1]
    y_abs = ref.run(A_abs, np.abs(x))[0] if dt in ("f32", "f64") else None
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yd = torch.empty(int(A.s.nrows), dtype=xd.dtype, device="cuda")
    out = []
    for name, o in cases:
        plan = sp.Plan(A, sp.default_opts(**o))
        ms = time_device(plan, xd, yd, stream, flush, reps)
        y = yd.cpu().numpy()
        cb = int(plan.info.compulsory_bytes)
        if y_abs is None:
            ok, check = bool(np.array_equal(y, y_ref)), "bit-exact vs reference spmv_host"
        else:
            ok, r = fp_check(y, y_ref, y_abs, counts, dt)
            check = f"max |y - y_ref| / (2 gamma_n sum|ax|) = {r:.3g}"
        gbs = cb / (ms * 1e-3) / 1e9
        out.append({"config": cfg, "workload": workload, "dtype": dt, "kind": A.kind, "case": name,
                    "variant": plan.info.variant.decode(), "us": round(ms * 1e3, 2), "gbs": round(gbs, 1),
                    "frac": round(gbs / peak, 4), "compulsory_bytes": cb, "check_ok": ok, "check": check,
                    "cpu_baseline": {"value": round(cb / sec / 1e9, 3), "unit": "GB/s", "cores": 1,
                                     "kind": ref.kind, "ms_per_spmv": round(sec * 1e3, 2),
                                     "sample": f"{passes} full pass(es) of spmv_host ({REF_DIR[A.kind]})"}})
        log(f"[bench] C{cfg} {workload} {dt} {A.kind} {name}: {ms * 1e3:.1f} us, {gbs:.0f} GB/s, "
            f"ok={ok} ({check})")
        plan.free()
    del xd, yd
    return out


PARTS = 2048  # parts of the reference's 2048-DPU runs: one part = one CTA


def run_configs(args, peak):
    """Every single-matrix configuration of the workload list, one entry per
    format / scheme / balance / element type: device time, GB/s of compulsory
    bytes, fraction of the measured HBM copy bandwidth, the reference's own
    host SpMV for that kind on one core, and the check against it."""
    import torch

    import sparsep_b200 as sp
    from sparsep_b200 import capi

    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out = []
    t0 = time.time()

    # 1: uniform 4096 x 4096, 8 columns per row, INT32, CSR 1D nnz-balanced
    n, m, r, c, v, x = sp.synth.uniform_rows(4096, 4096, 8, 0, np.int32)
    A = sp.csr("i32", n, m, *sp.synth.to_csr(n, r, c, v))
    out += measure_struct(1, "uniform8-4096", A, None, x, None,
                          [("1d auto", {}), ("1d nnz-balanced 64 parts", dict(nr_parts=64, part_balance=capi.BAL_NNZ))],
                          peak, stream, flush)

    # 2: the 1M-row Zipf matrix, FP32 and FP64, CSR and COO, 1D and 2D
    for dt in ("f32", "f64"):
        n, m, r, c, v, x = sp.synth.zipf_rows(seed=1, dtype=capi.DTYPES[dt].np)
        counts = np.bincount(r.astype(np.int64), minlength=n)
        rp, ci, vals = sp.synth.to_csr(n, r, c, v)
        A, Aa = sp.csr(dt, n, m, rp, ci, vals), sp.csr(dt, n, m, rp, ci, np.abs(vals))
        out += measure_struct(2, "zipf-1M", A, Aa, x, counts,
                              [("1d auto", {}),
                               ("1d row-balanced 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_ROW)),
                               ("1d nnz-balanced 2048 parts",
                                dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ, worker_balance=capi.BAL_NNZ))],
                              peak, stream, flush)
        del A, Aa
        E, Ea = sp.cooe(dt, n, m, r, c, v), sp.cooe(dt, n, m, r, c, np.abs(v))
        out += measure_struct(2, "zipf-1M", E, Ea, x, counts,
                              [("1d lock-free auto", {}), ("1d atomic", dict(sync=capi.SYNC_ATOMIC)),
                               ("1d nnz-elem 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM))],
                              peak, stream, flush)
        for conv, hv, cases in (("cooe2dcsr", (16, 16), [("2d-D 16x16", {})]),
                                ("cooe2rbdcsr", (32, 32), [("2d-RBD 32x32", {})]),
                                ("cooe2bdcsr", (64, 64), [("2d-BD 64x64", {}),
                                                          ("2d-BD 64x64 atomic", dict(sync=capi.SYNC_ATOMIC))]),
                                ("cooe2dcoo", (16, 16), [("2d-D 16x16", {}),
                                                         ("2d-D 16x16 atomic", dict(sync=capi.SYNC_ATOMIC))]),
                                ("cooe2bdcoo", (64, 64), [("2d-BD 64x64", {})])):
            D, Da = sp.convert(conv, E, *hv), sp.convert(conv, Ea, *hv)
            out += measure_struct(2, "zipf-1M", D, Da, x, counts, cases, peak, stream, flush)
            del D, Da
        del E, Ea
    log(f"[bench] configs 1-2 in {time.time() - t0:.0f}s")

    # 3: the 2M-row block-banded matrix, BCSR and BCOO 4x4 / 8x8, block and nnz balance
    for rb in (4, 8):
        for dt in ("i8", "i16", "i64", "f32"):
            B = sp.synth.block_banded(rb=rb, cb=rb, dtype=capi.DTYPES[dt].np)
            A = capi.bcsr(dt, B["nrows"], B["ncols"], rb, rb, B["browptr"], B["bcolind"], B["bval"], B["nnz"],
                          B["nnz_per_block"])
            O = sp.convert("bcsr2bcoo", A)
            counts = Aa = Oa = None
            if dt == "f32":
                counts = np.repeat(np.diff(B["browptr"].astype(np.int64)) * rb, rb)[: B["nrows"]]
                Aa = capi.bcsr(dt, B["nrows"], B["ncols"], rb, rb, B["browptr"], B["bcolind"], np.abs(B["bval"]),
                               B["nnz"], B["nnz_per_block"])
                Oa = sp.convert("bcsr2bcoo", Aa)
            wl = f"banded-2M {rb}x{rb}"
            out += measure_struct(3, wl, A, Aa, B["x"], counts,
                                  [("1d block-balanced 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
                                   ("1d nnz-balanced 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ))],
                                  peak, stream, flush)
            out += measure_struct(3, wl, O, Oa, B["x"], counts,
                                  [("1d block-balanced 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_BLOCK)),
                                   ("1d nnz-elem 2048 parts", dict(nr_parts=PARTS, part_balance=capi.BAL_NNZ_ELEM))],
                                  peak, stream, flush)
            del A, O, Aa, Oa, B
    log(f"[bench] configs 1-3 in {time.time() - t0:.0f}s")
    del flush
    return out


def _ref_csr_lib():
    so = ROOT / "oracle" / "_ref" / "libref_1D_CSR_row_f32.so"
    if so.exists():
        return C.CDLL(str(so)), "reference"
    so = ROOT / "oracle" / "liboracle.so"
    if not so.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "liboracle.so"], check=True)
    return C.CDLL(str(so)), "port"


def cpu_baseline(n, m, rowptr, colind, values, x, budget_s=15.0, threads=1):
    """Time the reference's host CSR SpMV on a bounded number of full passes;
    also returns its y and its sum of |a||x| per row (the check's bound)."""
    import sparsep_b200 as sp

    L, kind = _ref_csr_lib()
    A = sp.csr("f32", n, m, rowptr, colind, values)
    ref = RefHost("csr", "f32")
    y_ref = ref.run(A, np.ascontiguousarray(x))[0]
    y_abs = ref.run(sp.csr("f32", n, m, rowptr, colind, np.abs(values)), np.abs(x))[0]
    y = np.zeros(n + 8, np.float32)
    xx = np.ascontiguousarray(x)
    nnz = int(rowptr[-1])
    cb = compulsory_bytes(n, m, nnz)

    def one():
        if threads == 1:
            if kind == "reference":
                L.ref_spmv(y.ctypes.data_as(C.c_void_p), A.ref, xx.ctypes.data_as(C.c_void_p))
            else:
                L.oracle_spmv_csr_f32(y.ctypes.data_as(C.c_void_p), A.ref, xx.ctypes.data_as(C.c_void_p))
        else:
            slices(L, kind, A, xx, y, threads)

    t0 = time.perf_counter()
    one()
    first = time.perf_counter() - t0
    reps = max(1, min(50, int(budget_s / max(first, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(reps):
        one()
    dt = (time.perf_counter() - t0) / reps
    return {"value": round(cb / dt / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": kind,
            "sample": f"{reps} full SpMV passes over the {n}-row matrix ({nnz} nnz), {dt * 1e3:.1f} ms each",
            "ms_per_spmv": round(dt * 1e3, 3), "cpu": _cpu_name()}, y_ref, y_abs


def slices(L, kind, A, x, y, threads):
    """Run the unchanged reference CSR loop on `threads` row slices in parallel."""
    import concurrent.futures as cf

    import sparsep_b200 as sp

    s = A.s
    n = int(s.nrows)
    rp = A.arrays["rowptr"]
    nnz = int(rp[n])
    bounds = [0]
    for t in range(1, threads):
        bounds.append(int(np.searchsorted(rp[: n + 1], nnz * t // threads)))
    bounds.append(n)
    views = []
    St = sp.capi.STRUCTS["f32"]["csr"]
    for t in range(threads):
        r0, r1 = bounds[t], bounds[t + 1]
        v = St(r1 - r0, s.ncols, s.nnz, C.cast(C.addressof(s.rowptr.contents) + 4 * r0, sp.capi.P32),
               s.colind, s.values)
        views.append((v, r0))
    fn = L.ref_spmv if kind == "reference" else L.oracle_spmv_csr_f32

    def work(vr):
        v, r0 = vr
        fn(C.c_void_p(y.ctypes.data + 4 * r0), C.byref(v), x.ctypes.data_as(C.c_void_p))

    with cf.ThreadPoolExecutor(threads) as ex:  # ctypes releases the GIL during the call
        list(ex.map(work, views))


def _cpu_name():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, rank, world):
    if rank != 0:
        return None
    n, m, rowptr, colind, values, x = make_matrix()
    threads = os.cpu_count() or 1
    L, kind = _ref_csr_lib()
    import sparsep_b200 as sp

    A = sp.csr("f32", n, m, rowptr, colind, values)
    y = np.zeros(n + 8, np.float32)
    nnz = int(rowptr[-1])
    cb = compulsory_bytes(n, m, nnz)
    for _ in range(args.warmup):
        slices(L, kind, A, x, y, threads)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        slices(L, kind, A, x, y, threads)
        ts.append(time.perf_counter() - t0)
    avg = sum(ts) / len(ts)
    v = round(cb / avg / 1e9, 3)
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(avg * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Zipf power-law matrix, numpy PCG64 seed 1)",
            "config": {"workload": WORKLOAD, "nrows": n, "ncols": m, "nnz": nnz, "format": "csr", "scheme": "1d"},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": f"{args.steps} full SpMV passes, rows split over {threads} threads, "
                                       "each slice running the reference's spmv_host loop",
                             "cpu": _cpu_name()},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default="all", choices=["all", "single", "batch", "configs"],
                    help="single: the FP32 CSR Zipf SpMV only; batch: the batched path only; configs: the "
                         "per-configuration entries only")
    ap.add_argument("--batch-mats", type=int, default=512)
    ap.add_argument("--heavy-rows", type=int, default=0,
                    help="headline plan: rows with at least this many nonzeros in shared-memory column stripes "
                         "(0: the planner's choice, -1: never)")
    ap.add_argument("--no-configs", action="store_true",
                    help="leave out the per-configuration entries (formats, schemes, element types)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.impl == "reference" and rank != 0:
            return
        if args.impl == "ours":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    elif args.only == "configs":
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        peak, _ = peaks()
        res = None
        if rank == 0:
            cfg = run_configs(args, peak)
            res = {"configs": cfg, "configs_checked": f"{sum(e['check_ok'] for e in cfg)}/{len(cfg)}"}
    elif args.only == "batch":
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        res = {"batched": run_batch(args, "f32"), "batched_i32": run_batch(args, "i32")} if rank == 0 else None
    else:
        res = run_ours(args, rank, world)
        if args.only == "all" and world == 1:
            res["batched"] = run_batch(args, "f32")
            res["batched_i32"] = run_batch(args, "i32")
            if not args.no_configs:
                peak, _ = peaks()
                res["configs"] = run_configs(args, peak)
                res["configs_checked"] = f"{sum(e['check_ok'] for e in res['configs'])}/{len(res['configs'])}"
    if world > 1 and args.impl == "ours":
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
