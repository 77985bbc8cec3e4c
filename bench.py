"""Benchmark: all-pairs trajectory similarity, 2000 x 2000 trajectories, all
six measures (DTW, EDR, LCSS, ERP, discrete Frechet, Hausdorff) per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the six all-pairs launches over one 2000 x 2000 block (random-walk
trajectories, lengths U{20..200}, float32; EDR/LCSS eps 3e-4 deg, ERP gap
point at the box centre).  Under torchrun the rows of that one block are
split across the ranks in contiguous blocks of near-equal work
(shard.row_shards); each rank computes its rows with no collective on the
data path, so the total work is fixed as N grows ("strong").

value    = DP cells/s of the whole block (Hausdorff: point-segment
           evaluations) over the slowest rank's device time from CUDA events
           around each step's six launches, inputs resident in HBM, L2 flushed
           (256 MB write) before every step.
e2e      = the same cells/s through the public API with host inputs (padded
           float64 arrays as the reference takes them): core.matrix_many on one
           GPU, core.matrix_sharded (row blocks + one all-gather per measure)
           on N; packing, H2D, the six launches, the results to the host as
           float64 arrays, wall clock per step (max over ranks).
cfg1     = the 1,000-pair paired call, core.<measure>(t1, len1, t2, len2), per
           measure: pairs/s through the call (host float64 in, float64 out)
           and on resident inputs, next to the CPU reference on the same pairs.
cfg3     = the 500k-pair uneven batch (lognormal lengths), DTW + Frechet + EDR
           in one autotuned persistent launch replayed as a CUDA graph, next to
           three plain tsm_pairs launches.
cfg5     = kNN, 1,000 queries x 1M trajectories, DTW top-10: exhaustive exact
           GPU DP against the learned filter (an encoder trained here on a
           reduced budget, stated in the line) + tensor-core candidate scan +
           exact rerank; queries/s and recall@10.
roofline = the dominant kernel's FP32-issue rate (algorithmic ops per unit x
           units / its event time) against SMs x 128 lanes x max SM clock.
cpu_baseline = the reference's C++ measures (oracle/_ref: DTW, ERP, Frechet,
           Hausdorff) and the FP64 port for EDR/LCSS, on rank 0 only, on a
           bounded row sample of the same workload, all host threads.
--impl reference: that CPU reference alone, as the reference arm.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURES = ["dtw", "edr", "lcss", "erp", "dfrechet", "hausdorff"]
MID = {"dtw": 0, "edr": 1, "lcss": 2, "erp": 3, "dfrechet": 4, "hausdorff": 5}
# Algorithmic FP32-pipe operations per unit (DP cell or point-segment
# evaluation): the ideal scalar recurrence, not the kernel's instruction count.
OPS_PER_UNIT = {"dtw": 7, "edr": 9, "lcss": 7, "erp": 9, "dfrechet": 7, "hausdorff": 12}
N_TRAJ = 2000
EPS = 3e-4
WORKLOAD = "allpairs_2000x2000_six_measures"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "numba"], default="ours",
                    help="reference: the reference's CPU measures (the reference arm); numba: the reference's "
                         "Numba-CUDA measures (baseline/_ref/core) on this GPU, 1,000 paired trajectories")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU work of the cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows", type=int, default=0, help="rows per thread (0 = library default)")
    ap.add_argument("--n-traj", type=int, default=N_TRAJ,
                    help="trajectories per set (smaller cases are for profiling, not bench lines)")
    ap.add_argument("--measures", default=",".join(MEASURES), help="comma-separated subset of the six measures")
    ap.add_argument("--flush-mb", type=int, default=256, help="L2 flush buffer written before each step (0: none)")
    ap.add_argument("--workload", choices=["allpairs", "uneven", "surrogate", "knn", "sym"], default="allpairs",
                    help="allpairs: the benchmark line; the others measure the uneven-batch, surrogate-training "
                         "and kNN configurations (one extra JSON line each)")
    ap.add_argument("--n-pairs", type=int, default=500_000, help="uneven: number of pairs")
    ap.add_argument("--pool", type=int, default=100_000, help="surrogate: trajectory pool")
    ap.add_argument("--train-pairs", type=int, default=200_000, help="surrogate: labelled pairs")
    ap.add_argument("--epochs", type=int, default=20, help="surrogate: training epochs")
    ap.add_argument("--n-db", type=int, default=1_000_000, help="knn: database size")
    ap.add_argument("--n-queries", type=int, default=1000, help="knn: queries")
    ap.add_argument("--checkpoint", default="", help="surrogate: save / knn: load the trained encoder here")
    ap.add_argument("--untrained-filter", action="store_true",
                    help="knn without a checkpoint: run the filter with an untrained encoder (profiling)")
    ap.add_argument("--no-extra", action="store_true", help="allpairs: skip the cfg1 / cfg3 keys")
    a = ap.parse_args()
    a.measures = [m for m in a.measures.split(",") if m]
    for m in a.measures:
        if m not in MID:
            ap.error(f"unknown measure {m}")
    return a


def _measured_peaks():
    """The driver-measured peaks of this pool's B200s (MEASURED_PEAKS.json at
    the repository root), {} when absent."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_sets(rank, n=N_TRAJ):
    from trajsimimeasures_b200 import datagen as D
    d = D.trajectory_set(n, seed=D.SEED_DB)
    q = d if rank == 0 else D.trajectory_set(n, seed=D.SEED_DB + rank)
    return q, d


def units(measure, lq, ld):
    lq = lq.astype(np.float64)
    ld = ld.astype(np.float64)
    if measure == "hausdorff":
        return float(lq.sum() * (ld - 1).sum() + ld.sum() * (lq - 1).sum())
    return float(lq.sum() * ld.sum())


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join("/tmp", f"tsm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None
            return
        t0 = time.time()  # nvidia-smi takes a moment to start: wait for its first sample
        while time.time() - t0 < 10 and self._lines() < 1 and self.p.poll() is None:
            time.sleep(0.05)
        self.skip = 0

    def _lines(self):
        self.f.flush()
        try:
            return sum(1 for ln in open(self.path) if ln.count(",") >= 8)
        except OSError:
            return 0

    def mark(self):
        """Samples before this call (the warm-up, idle) are not reported."""
        if self.p is not None:
            self.skip = self._lines()

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for ln in open(self.path) if ln.count(",") >= 8][getattr(self, "skip", 0):]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref + FP64 port), bounded sample
# ---------------------------------------------------------------------------

def cpu_reference_run(q, d, rows, threads):
    """Runs the CPU reference on rows `rows` of the Q x D block, all six
    measures.  Returns (units, seconds, per-measure dict, kind string)."""
    from oracle import oracle as O
    from trajsimimeasures_b200 import datagen as D
    qp, qo, ql = q
    dp, do, dl = d
    pts = np.concatenate([qp, dp])
    shift = qp.shape[0]
    nd = len(do)
    qi = np.repeat(rows, nd)
    di = np.tile(np.arange(nd), len(rows))
    have_ref = O.ref_available()
    rs = O.RefSet(pts, np.concatenate([qo, do + shift]), np.concatenate([ql, dl])) if have_ref else None
    O.set_threads(threads)
    tot_u, tot_t, per = 0.0, 0.0, {}
    for name in MEASURES:
        m = MID[name]
        u = units(name, ql[rows], dl)
        t0 = time.perf_counter()
        if rs is not None and m in (0, 3, 4, 5):
            rs.pairs(m, qi, di + len(qo), gpoint=D.BOX_CENTRE, threads=threads)
            kind = "reference"
        else:
            O.pairs_f64(m, pts, qo[qi], ql[qi], do[di] + shift, dl[di], eps=EPS, gpoint=D.BOX_CENTRE)
            kind = "port"
        dt = time.perf_counter() - t0
        per[name] = {"units_per_s": u / dt, "kind": kind}
        tot_u += u
        tot_t += dt
    if rs is not None:
        rs.close()
    kinds = sorted({v["kind"] for v in per.values()})
    return tot_u, tot_t, per, "+".join(kinds)


def parity_sample(q, d, outs, cnts, rows):
    """Checks rows `rows` of the GPU results of the timed step against the
    oracle: max/median relative error vs the FP64 restatement for the
    distance measures, count mismatches vs the FP32 same-arithmetic twin for
    EDR/LCSS (which must be 0)."""
    import torch
    from oracle import oracle as O
    from trajsimimeasures_b200 import datagen as D
    qp, qo, ql = q
    dp, do, dl = d
    res = {}
    for name in MEASURES:
        m = MID[name]
        if m in (1, 2):
            _, c32 = O.matrix_idx(O.pairs_f32, m, qp, qo[rows], ql[rows], dp, do, dl, eps=EPS, gpoint=D.BOX_CENTRE)
            got = cnts[name][torch.as_tensor(rows, device=cnts[name].device)].cpu().numpy()
            res[name] = {"count_mismatches": int((got != c32).sum()), "pairs": int(got.size)}
        else:
            d64, _ = O.matrix_idx(O.pairs_f64, m, qp, qo[rows], ql[rows], dp, do, dl, eps=EPS, gpoint=D.BOX_CENTRE)
            got = outs[name][torch.as_tensor(rows, device=outs[name].device)].cpu().numpy().astype(np.float64)
            with np.errstate(invalid="ignore", divide="ignore"):
                r = np.abs(got - d64) / np.maximum(np.abs(d64), 1e-30)
            res[name] = {"max_rel_err": float(r.max()), "median_rel_err": float(np.median(r)), "pairs": int(got.size)}
    return res


def cpu_sample_rows(q, d, target_s, threads):
    """Picks a row count whose six-measure CPU time is about target_s."""
    probe = np.arange(2)
    u, t, _, _ = cpu_reference_run(q, d, probe, threads)
    per_row = t / len(probe)
    nrows = int(max(1, min(N_TRAJ, target_s / max(per_row, 1e-6))))
    return np.arange(nrows)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    q, d = workload_sets(0)
    threads = host_threads()
    rows = cpu_sample_rows(q, d, 4.0, threads)
    vals = []
    for i in range(args.warmup + args.steps):
        u, t, per, kind = cpu_reference_run(q, d, rows, threads)
        if i >= args.warmup:
            vals.append((u, t))
    U = sum(v[0] for v in vals)
    T = sum(v[1] for v in vals)
    value = U / T
    line = {
        "metric": "DP cells/s (6 measures, all-pairs 2000x2000)", "value": value, "unit": "cells/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * T / len(vals), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_rows": int(len(rows)), "n_traj": N_TRAJ},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": threads, "kind": kind,
                         "sample": f"rows 0..{len(rows) - 1} of the 2000x2000 block x 6 measures per step "
                                   "(reference C++ Traj::DTW/ERP/Frechet/HausdorffDistance; FP64 port for EDR/LCSS)"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "per_measure": {k: v["units_per_s"] for k, v in per.items()},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def dram_traffic(measure):
    """DRAM bytes per launch (read + write) of the dominant kernel, from the
    committed ncu capture of the full-size launch; None if not captured."""
    path = os.path.join(ROOT, "profiles", "hausdorff_allpairs_2000x2000_dram.txt")
    if measure != "hausdorff" or not os.path.exists(path):
        return None
    vals = {}
    for line in open(path):
        if ":" in line and not line.startswith("#"):
            k, v = line.split(":", 1)
            vals[k.strip()] = v.strip()
    try:
        return int(vals["dram__bytes_read.sum"]) + int(vals["dram__bytes_write.sum"])
    except (KeyError, ValueError):
        return None


def run_ours(args, ws, rank, local):
    import torch
    import torch.distributed as dist
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet, matrix_raw
    from trajsimimeasures_b200.shard import row_shards

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    q, d = workload_sets(0, args.n_traj)  # one block, its rows split across the ranks
    r0, r1 = row_shards(q[2], ws)[rank]
    MEAS = args.measures
    qs = TrajSet.from_packed(q[0], q[1][r0:r1], q[2][r0:r1], device=dev)
    ds = TrajSet.from_packed(*d, device=dev)
    order = ds.order_by_length()
    nq, nd = qs.n, ds.n
    outs = {m: torch.empty((nq, nd), dtype=torch.float32, device=dev) for m in MEAS}
    cnts = {m: torch.empty((nq, nd), dtype=torch.int32, device=dev) for m in ("edr", "lcss") if m in MEAS}
    flush = torch.empty(max(args.flush_mb, 1) * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    U = {m: units(m, q[2][r0:r1], d[2]) for m in MEAS}  # this rank's block
    U_all = {m: units(m, q[2], d[2]) for m in MEAS}  # the whole block

    def step(evs=None):
        for i, m in enumerate(MEAS):
            if evs is not None:
                evs[i].record(stream)
            matrix_raw(MID[m], qs, ds, out=outs[m], counts=cnts.get(m), d_order=order, eps=EPS,
                       gpoint=D.BOX_CENTRE, rows=args.rows, stream=stream)
        if evs is not None:
            evs[len(MEAS)].record(stream)

    for _ in range(args.warmup):
        if args.flush_mb:
            flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if clk:
        clk.start()
        clk.mark()
    per_ms = {m: 0.0 for m in MEAS}
    step_ms = []
    launches = 0
    for _ in range(args.steps):
        if args.flush_mb:
            flush.fill_(1.0)
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(MEAS) + 1)]
        step(evs)
        launches += len(MEAS)
        torch.cuda.synchronize()
        for i, m in enumerate(MEAS):
            per_ms[m] += evs[i].elapsed_time(evs[i + 1])
        step_ms.append(evs[0].elapsed_time(evs[-1]))
    torch.cuda.synchronize()
    clocks = clk.stop() if clk else None
    if ws > 1:
        dist.barrier()
    tot_ms = float(sum(step_ms))
    t = torch.tensor([tot_ms], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    units_all = sum(U_all.values())
    value = units_all * args.steps / (max_ms / 1e3)

    # e2e through the public API, host inputs
    e2e = None
    if args.e2e_steps > 0:
        from trajsimimeasures_b200 import core
        Qpad = D.pad(D.unpack(*q))
        lq = q[2].copy()
        if ws == 1:
            call = lambda: core.matrix_many(MEAS, Qpad, lq, Qpad, lq, eps=EPS, gpoint=D.BOX_CENTRE)  # noqa: E731
            path = "core.matrix_many(padded float64 host arrays) -> float64 host arrays"
        else:
            call = lambda: core.matrix_sharded(MEAS, Qpad, lq, Qpad, lq, eps=EPS, gpoint=D.BOX_CENTRE)  # noqa: E731
            path = ("core.matrix_sharded(padded float64 host arrays): row blocks per rank, one NCCL all-gather per "
                    "measure -> float64 host arrays on every rank")
        call()  # warm
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.e2e_steps):
            if ws > 1:
                dist.barrier()
            t0 = time.perf_counter()
            call()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        tt = torch.tensor([sum(ts)], dtype=torch.float64, device=dev)
        if ws > 1:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        L = Qpad.shape[1]
        if ws == 1:  # one float32 upload of the set (Q is D), six float64 results back
            h2d = lq.shape[0] * (L * 8 + 12)
            d2h = nq * nd * 8 * len(MEAS)
        else:  # this rank's query rows and the whole database; every rank gets the gathered matrices
            h2d = (r1 - r0) * (L * 8 + 12) + lq.shape[0] * (L * 8 + 12)
            d2h = lq.shape[0] * nd * 4 * len(MEAS)
        e2e = {"value": units_all * args.e2e_steps / float(tt.item()), "unit": "cells/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": 1e3 * float(tt.item()) / args.e2e_steps, "path": path}

    if rank != 0:
        return
    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    max_mhz = (clocks or {}).get("sm_max_mhz") or 1965.0
    peak_ops = sms * 128 * max_mhz * 1e6
    per = {}
    for m in MEAS:
        sec = per_ms[m] / 1e3
        per[m] = {"units_per_s": U[m] * args.steps / sec, "pairs_per_s": nq * nd * args.steps / sec,
                  "ms": per_ms[m] / args.steps,
                  "fp32_issue_frac": U[m] * args.steps / sec * OPS_PER_UNIT[m] / peak_ops}
        if m in ("dtw", "erp"):  # one MUFU sqrt per cell; the SFU pipe runs 16 lanes per SM per clock
            per[m]["sfu_frac"] = U[m] * args.steps / sec / (sms * 16 * max_mhz * 1e6)
    dom = max(MEAS, key=lambda m: per_ms[m])
    traffic = dram_traffic(dom)
    ach = per[dom]["units_per_s"] * OPS_PER_UNIT[dom]
    roof = {"bound": "fp32-issue", "kernel": f"tsm::dp_matrix_kernel<{dom}>" if dom != "hausdorff"
            else "tsm::hausdorff_matrix_kernel", "achieved": ach / 1e9, "peak": peak_ops / 1e9, "unit": "Gop/s",
            "frac": ach / peak_ops, "traffic": traffic,
            "traffic_unit": "bytes per launch (ncu dram read + write of one full-size launch; the 16 MB result "
                            "is written back from L2 after the kernel)" if traffic is not None else None,
            "peak_source": f"{sms} SMs x 128 FP32 lanes x {max_mhz:.0f} MHz max SM clock (not in MEASURED_PEAKS, "
                           "which has HBM copy and bf16 GEMM only)",
            "ops_per_unit": OPS_PER_UNIT[dom], "units_per_launch": U[dom]}
    line = {
        "metric": "DP cells/s (6 measures, all-pairs 2000x2000)", "value": value, "unit": "cells/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random walks, Porto-like box)",
        "config": {"workload": WORKLOAD if (args.n_traj == N_TRAJ and MEAS == MEASURES)
                   else f"allpairs_{args.n_traj}x{args.n_traj}_{'+'.join(MEAS)} (profiling case)", "n_traj": args.n_traj, "lengths": "U{20..200}", "eps_deg": EPS,
                   "erp_gpoint": list(D.BOX_CENTRE), "l2": f"flushed before each step ({args.flush_mb} MB write)" if args.flush_mb else "not flushed",
                   "parallelism": f"strong: the rows of one 2000x2000 block split over {ws} rank(s) (rank 0: rows "
                                  f"{r0}..{r1 - 1})", "rows_per_thread": args.rows or "default (8; hausdorff 16)"},
        "e2e": e2e, "gpu_launches": launches, "roofline": roof, "clocks": clocks, "per_measure": per,
    }
    if not args.no_cpu_baseline:
        threads = host_threads()
        rows = cpu_sample_rows(q, d, args.cpu_seconds, threads)
        u, tcpu, cper, kind = cpu_reference_run(q, d, rows, threads)
        line["cpu_baseline"] = {"value": u / tcpu, "unit": "cells/s", "cores": threads, "kind": kind,
                                "seconds": tcpu,
                                "sample": f"rows 0..{len(rows) - 1} of the 2000x2000 block x 6 measures "
                                          "(reference C++ for DTW/ERP/Frechet/Hausdorff, FP64 port for EDR/LCSS)"}
        line["cpu_baseline"]["parity_rows_0_3"] = parity_sample(q, d, outs, cnts, np.arange(4))
    if ws == 1 and not args.no_extra:
        line["cfg1"] = cfg1_pairs(args)
        line["cfg3"] = uneven_result(args.n_pairs, 10, 3)
        cfg4, enc = surrogate_result(args)  # the surrogate training configuration (pool 100k, 200k pairs, 20 epochs)
        line["cfg4"] = cfg4
        k = run_knn(args, enc=enc, emit=False)
        k["encoder_training"] = "the cfg4 encoder"
        line["cfg5"] = k
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# other configurations (one JSON line each; not the benchmark line)
# ---------------------------------------------------------------------------

def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def cfg1_pairs(args, calls=20):
    """1,000 pairs (lengths U{20..200}, the box's random walks) through the
    reference-signature paired call core.<measure>(t1, len1, t2, len2), one
    call per measure on padded float64 host arrays: wall clock per call
    (staging, H2D, kernels, float64 result on the host), pairs/s; the same
    kernels on resident inputs (events); the CPU reference on the same pairs
    with all host threads (reference C++ for DTW/ERP/Frechet/Hausdorff, FP64
    port for EDR/LCSS).  The reference's paired driver:
    test_trajsimi_time.py:222-276."""
    import torch
    from oracle import oracle as O
    from trajsimimeasures_b200 import core, datagen as D
    from trajsimimeasures_b200.engine import pair_order, pairs_raw
    pts, off, lens, ia, ib = D.pairs_uniform(1000)
    la, lb = lens[ia], lens[ib]
    t1, t2 = D.pad(D.unpack(pts, off, lens, ia)), D.pad(D.unpack(pts, off, lens, ib))
    fns = {"dtw": lambda: core.dtw(t1, la, t2, lb), "edr": lambda: core.edr(t1, la, t2, lb, EPS),
           "lcss": lambda: core.lcss(t1, la, t2, lb, EPS), "erp": lambda: core.erp(t1, la, t2, lb, D.BOX_CENTRE),
           "dfrechet": lambda: core.dfrechet(t1, la, t2, lb), "hausdorff": lambda: core.hausdorff(t1, la, t2, lb)}
    dev = torch.device("cuda", torch.cuda.current_device())
    up = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)  # noqa: E731
    T = (up(pts, np.float32), up(off[ia], np.int64), up(la, np.int32), up(off[ib], np.int64), up(lb, np.int32))
    order = up(pair_order(la, lb), np.int32)
    out = torch.empty(1000, device=dev)
    cnt = torch.empty(1000, dtype=torch.int32, device=dev)
    mx = int(max(la.max(), lb.max()))
    threads = host_threads()
    O.set_threads(threads)
    have_ref = O.ref_available()
    rs = O.RefSet(pts, off, lens) if have_ref else None
    res = {}
    for name in MEASURES:
        m = MID[name]
        for _ in range(3):
            fns[name]()
        ts = []
        for _ in range(calls):
            t0 = time.perf_counter()
            fns[name]()
            ts.append(time.perf_counter() - t0)
        call_s = float(np.median(ts))
        kern = lambda: pairs_raw(m, *T, mx, out=out, counts=cnt if m in (1, 2) else None, order=order,  # noqa: E731
                                 eps=EPS, gpoint=D.BOX_CENTRE)
        for _ in range(3):
            kern()
        e0, e1 = _events()
        e0.record()
        for _ in range(calls):
            kern()
        e1.record()
        torch.cuda.synchronize()
        dev_s = e0.elapsed_time(e1) / 1e3 / calls
        t0 = time.perf_counter()
        if rs is not None and m in (0, 3, 4, 5):
            rs.pairs(m, ia, ib, gpoint=D.BOX_CENTRE, threads=threads)
            kind = "reference"
        else:
            O.pairs_f64(m, pts, off[ia], la, off[ib], lb, eps=EPS, gpoint=D.BOX_CENTRE)
            kind = "port"
        cpu_s = time.perf_counter() - t0
        res[name] = {"call_pairs_per_s": 1000 / call_s, "call_ms": 1e3 * call_s,
                     "device_pairs_per_s": 1000 / dev_s, "device_ms": 1e3 * dev_s,
                     "cpu_pairs_per_s": 1000 / cpu_s, "cpu_kind": kind, "call_vs_cpu": cpu_s / call_s}
    if rs is not None:
        rs.close()
    return {"workload": "pairs_1000_uniform_20_200_six_measures", "api": "core.<measure>(t1, len1, t2, len2), "
            "padded float64 host arrays in, float64 host array out, synchronous", "calls_per_measure": calls,
            "cpu_cores": threads, "per_measure": res,
            "h2d_bytes_per_call": int(t1.size * 4 + t2.size * 4 + 12 * 1000),
            "d2h_bytes_per_call": 1000 * 4}


def uneven_result(n_pairs, steps, warmup):
    """500k pairs, lognormal lengths (median 60, sigma 1, clipped 10..2000),
    DTW + Frechet + EDR in ONE persistent launch (autotuned tile/bucket shape,
    CUDA-graph replay), against three plain tsm_pairs launches."""
    import torch
    from trajsimimeasures_b200 import datagen as D, sched
    from trajsimimeasures_b200.engine import pairs_raw, pair_order
    t0 = time.perf_counter()
    pts, off, lens, ia, ib = D.pairs_lognormal(n_pairs, seed=D.SEED_DB)
    gen_s = time.perf_counter() - t0
    dev = torch.device("cuda", torch.cuda.current_device())
    up = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x, dtype=dt)).to(dev)  # noqa: E731
    la, lb = lens[ia], lens[ib]
    T = (up(pts, np.float32), up(off[ia], np.int64), up(la, np.int32), up(off[ib], np.int64), up(lb, np.int32))
    ms_ = ["dtw", "dfrechet", "edr"]
    cells = float((la.astype(np.float64) * lb).sum()) * len(ms_)
    t0 = time.perf_counter()
    best, tried = sched.autotune(*T, ms_, eps=EPS, len_a_host=la, len_b_host=lb)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    sc = sched.PairsScheduler(*T, ms_, eps=EPS, rows=best[0], warp_floats=best[1], max_steps=best[2], len_a_host=la,
                              len_b_host=lb)
    plan_s = time.perf_counter() - t0
    sc.capture()
    for _ in range(warmup):
        sc.replay()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        sc.replay()
    e1.record()
    torch.cuda.synchronize()
    ms_sched = e0.elapsed_time(e1) / steps
    # baseline: one tsm_pairs launch per measure (tile + wave kernels, shape-sorted order)
    order = up(pair_order(la, lb), np.int32)
    out = torch.empty(len(ia), device=dev)
    cnt = torch.empty(len(ia), dtype=torch.int32, device=dev)
    mx = int(max(la.max(), lb.max()))

    def plain():
        for m in ms_:
            pairs_raw(m, *T[:5], mx, out=out, counts=cnt if m == "edr" else None, order=order, eps=EPS)
    for _ in range(warmup):
        plain()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        plain()
    e1.record()
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1) / steps
    kinds = np.bincount(sc.plan.tasks[:, 0], minlength=7).tolist()
    return {
        "workload": f"uneven_{n_pairs}_pairs_lognormal_dtw+dfrechet+edr", "metric": "DP cells/s",
        "value": cells / (ms_sched / 1e3), "unit": "cells/s", "pairs_per_s": 3 * len(ia) / (ms_sched / 1e3),
        "ms_per_launch": ms_sched, "graph_replay": True,
        "autotuned": {"rows": best[0], "warp_floats": best[1], "max_steps": best[2], "candidates_ms": tried},
        "tasks_by_kind": {"tile": kinds[0], "group4": kinds[5], "group8": kinds[1], "group16": kinds[6],
                          "wave": kinds[2]},
        "plain_tsm_pairs_ms": ms_plain, "speedup_vs_plain": ms_plain / ms_sched,
        "host_s": {"generate": gen_s, "autotune": tune_s, "plan": plan_s}, "steps": steps,
        "cells_per_launch": cells}


def run_uneven(args):
    print(json.dumps(uneven_result(args.n_pairs, args.steps, args.warmup)), flush=True)


def _save_encoder(enc, path, extra):
    import torch
    torch.save({"params": enc.params.cpu(), "m": enc.m.cpu(), "v": enc.v.cpu(), "step": enc.step,
                "nrm": enc.nrm, **extra}, path)


def _load_encoder(path, dev):
    import torch
    from trajsimimeasures_b200.surrogate import Encoder
    ck = torch.load(path, weights_only=False)
    enc = Encoder(ck["params"].to(dev), np.asarray(ck["nrm"], np.float32), ck["m"].to(dev), ck["v"].to(dev),
                  int(ck["step"]))
    return enc, ck


def hit_ratios(Q, Dset, enc, exact_idx, ks=(10, 50), cands=(200, 500)):
    """HR@k of the embedding alone (the reference's learned-measure metric,
    utilities/tool_funcs.py:141-158): |top-k by embedding distance  intersect
    top-k by exact DTW| / k, averaged over the queries; and R10@c, the
    recall@10 of the top-c candidates, all with FP32 embedding distances."""
    import torch
    eq, ed = enc.embed(Q).double(), enc.embed(Dset).double()
    mu = ed.mean(0)
    eq, ed = (eq - mu).float(), (ed - mu).float()
    nd = (ed * ed).sum(1)
    kmax = max(max(ks), max(cands))
    tops = []
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for q0 in range(0, Q.n, 256):
            d = nd[None, :] - 2.0 * (eq[q0:q0 + 256] @ ed.T)
            tops.append(torch.topk(d, kmax, dim=1, largest=False).indices.cpu().numpy())
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    top = np.concatenate(tops)
    ex = np.asarray(exact_idx.cpu() if hasattr(exact_idx, "cpu") else exact_idx)
    out = {f"HR@{k}": float(np.mean([len(np.intersect1d(top[i, :k], ex[i, :k])) / k for i in range(len(top))]))
           for k in ks}
    out.update({f"R10@{c}": float(np.mean([len(np.intersect1d(top[i, :c], ex[i, :10])) / 10 for i in range(len(top))]))
                for c in cands})
    return out


def run_surrogate(args):
    print(json.dumps(surrogate_result(args)[0]), flush=True)


def surrogate_result(args):
    """Pool of random-walk trajectories; training pairs: random pairs (the
    reference protocol) plus each of 10k anchors with its 10 nearest pool
    trajectories by exact GPU DTW (neighbourhood pairs, as NEUTRAJ samples);
    labels from the GPU DTW kernel, normalised by the max label; the encoder
    trained with the relative squared error by the library's own kernels
    (MSE weighted by 1 / y^2, so that the near pairs count); held-out Spearman rho on
    random pairs; HR@10 / HR@50 of the embedding on 256 pool queries;
    FP64-oracle error of the labels.  -> (result dict, trained encoder)."""
    import torch
    from oracle import oracle as O
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.knn import _subset, knn_exhaustive
    from trajsimimeasures_b200.surrogate import Encoder, dtw_labels, neighbour_pairs, spearman
    dev = torch.device("cuda", 0)
    p, o, l = D.trajectory_set(args.pool, seed=D.SEED_DB)
    s = TrajSet.from_packed(p, o, l, device=dev)
    rng = np.random.Generator(np.random.PCG64(D.SEED_DB))
    n = args.train_pairs
    pa, pb = rng.integers(0, args.pool, n), rng.integers(0, args.pool, n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    na, nb = neighbour_pairs(s, args.pool // 10, k=10, seed=D.SEED_DB)
    torch.cuda.synchronize()
    nb_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    lab = dtw_labels(s, pa, pb)
    nlab = dtw_labels(s, na, nb)
    torch.cuda.synchronize()
    label_s = time.perf_counter() - t0
    sample = rng.choice(n, 2000, replace=False)
    d64, _ = O.pairs_idx(O.pairs_f64, 0, p, o, l, pa[sample], pb[sample])
    label_err = float(np.max(np.abs(lab[sample] - d64) / d64))
    mx = float(max(lab.max(), nlab.max()))
    y = lab / mx
    ntr = int(0.9 * n)
    tr_a, tr_b = np.concatenate([pa[:ntr], na]), np.concatenate([pb[:ntr], nb])
    tr_y = np.concatenate([y[:ntr], nlab / mx])
    hq = _subset(s, torch.as_tensor(np.sort(rng.choice(args.pool, 256, replace=False)), device=dev))
    _, hq_exact = knn_exhaustive(hq, s, 50)
    enc = Encoder.init(s, seed=0)
    rho0 = spearman(enc.predict_pairs(s, pa[ntr:], pb[ntr:]), y[ntr:])
    hr0 = hit_ratios(hq, s, enc, hq_exact)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = enc.fit(s, tr_a, tr_b, tr_y, epochs=args.epochs, batch_pairs=1024, lr=2e-3, relative=True)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    # one more step on a copy of the trained encoder, for launch lists (ncu --nvtx-include train_step/)
    cp = Encoder(enc.params.clone(), enc.nrm, enc.m.clone(), enc.v.clone())
    cp.step = enc.step
    sel = np.arange(min(1024, len(tr_a)))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("train_step")
    _, g, _ = cp.loss_grad(s, np.concatenate([tr_a[sel], tr_b[sel]]), sel, len(sel) + sel, tr_y[sel])
    cp.adam(g, lr=1e-3)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    del cp
    pred = enc.predict_pairs(s, pa[ntr:], pb[ntr:])
    rho = spearman(pred, y[ntr:])
    hr = hit_ratios(hq, s, enc, hq_exact)
    if args.checkpoint:
        _save_encoder(enc, args.checkpoint, {"max_label": mx, "rho": rho})
    return {
        "workload": f"surrogate_pool{args.pool}_pairs{n}+neighbours{len(na)}", "metric": "held-out Spearman rho",
        "value": rho, "rho_untrained": rho0, "hit_ratio": hr, "hit_ratio_untrained": hr0,
        "skip_weights": [round(float(x), 4) for x in torch.exp(enc.params[-16:]).tolist()],
        "mse_first_epoch": hist[0], "mse_last_epoch": hist[-1],
        "epochs": args.epochs, "train_pairs": int(len(tr_a)), "train_s": train_s,
        "train_pairs_per_s": args.epochs * len(tr_a) / train_s,
        "train_ms_per_step": 1e3 * train_s / (args.epochs * ((len(tr_a) + 1023) // 1024)), "label_s": label_s,
        "label_pairs_per_s": (n + len(na)) / label_s, "neighbour_pairs_s": nb_s,
        "label_max_rel_err_vs_fp64": label_err, "checkpoint": args.checkpoint or None}, enc


def run_knn(args, enc=None, emit=True):
    """1k queries against a 1M database (random walks, U{20..200}): exhaustive
    exact GPU DTW top-10 vs the calibrated learned filter + exact rerank."""
    import torch
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet
    from trajsimimeasures_b200.knn import SurrogateIndex, knn_exhaustive, recall_at_k
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    dp, do, dl = D.trajectory_set(args.n_db, seed=D.SEED_DB)
    qp, qo, ql = D.trajectory_set(args.n_queries, seed=D.SEED_QUERY)
    gen_s = time.perf_counter() - t0
    Dset = TrajSet.from_packed(dp, do, dl, device=dev)
    Q = TrajSet.from_packed(qp, qo, ql, device=dev)
    knn_exhaustive(TrajSet.from_packed(qp, qo[:4], ql[:4], device=dev), Dset, 10)  # warm
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    ex_d, ex_i = knn_exhaustive(Q, Dset, 10)
    e1.record()
    torch.cuda.synchronize()
    ex_s = e0.elapsed_time(e1) / 1e3
    out = {"workload": f"knn_{args.n_queries}q_x_{args.n_db}db_dtw_top10",
           "exhaustive_queries_per_s": args.n_queries / ex_s, "exhaustive_s": ex_s,
           "exhaustive_cells_per_s": float(ql.astype(np.float64).sum() * dl.astype(np.float64).sum()) / ex_s}
    if enc is None and getattr(args, "untrained_filter", False):
        from trajsimimeasures_b200.surrogate import Encoder
        enc = Encoder.init(Dset, seed=0)
    if enc is not None or (args.checkpoint and os.path.exists(args.checkpoint)):
        ck = {"rho": None}
        if enc is None:
            enc, ck = _load_encoder(args.checkpoint, dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        index = SurrogateIndex(enc, Dset)
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0
        cal = TrajSet.from_packed(*D.trajectory_set(256, seed=D.SEED_QUERY + 1), device=dev)
        t0 = time.perf_counter()
        c, rec = index.calibrate(cal, 10, target=0.99)
        torch.cuda.synchronize()
        cal_s = time.perf_counter() - t0
        # median of 5 timed queries (one query call is ~0.1 s: single shots are noisy)
        reps = []
        for _ in range(5):
            e0, e1 = _events()
            e0.record()
            f_d, f_i = index.query(Q, 10)
            e1.record()
            torch.cuda.synchronize()
            reps.append(e0.elapsed_time(e1) / 1e3)
        f_s = float(np.median(reps))
        # phase split of one query call: candidate selection (embedding + scan + select), exact rerank
        from trajsimimeasures_b200.knn import knn_rerank
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.nvtx.range_push("knn_query")  # the launches of one query call (ncu --nvtx-include knn_query/)
        scan_ev = []
        ev[0].record()
        cand = index.candidates(Q, min(c, Dset.n), scan_events=scan_ev) if c else None
        ev[1].record()
        if cand is not None:
            knn_rerank(Q, Dset, cand, 10)
        ev[2].record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        out["filtered_phase_s"] = {"candidates": ev[0].elapsed_time(ev[1]) / 1e3,
                                   "rerank": ev[1].elapsed_time(ev[2]) / 1e3}
        if scan_ev:  # the main candidate scan, timed with events on its stream
            ms = sum(a.elapsed_time(b) for a, b, _, _ in scan_ev)
            flop = sum(2.0 * q * r * 483 for _, _, q, r in scan_ev)  # K = 3 x 160 split products + 3 norm columns
            peak = _measured_peaks().get("bf16_tflops")
            out["scan_roofline"] = {
                "kernel": "scan::scan_kernel<false>", "bound": "tensor", "ms": ms, "unit": "TFLOP/s",
                "achieved": flop / ms / 1e9, "peak": peak, "frac": (flop / ms / 1e9 / peak) if peak else None,
                "flop_per_launch": flop, "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst), of measured",
                "note": "algorithmic FLOPs: 2 x queries x rows x 483 (FP16 split products, K padded to 512 "
                        "in the kernel)"}
        out["filtered_reps_s"] = reps
        out.update({"filtered_queries_per_s": args.n_queries / f_s, "filtered_s": f_s, "candidates": c,
                    "calibration_recall": {str(k): v for k, v in rec.items()},
                    "recall_at_10": recall_at_k(f_i, ex_i), "speedup_vs_exhaustive": ex_s / f_s,
                    "index_build_s": build_s, "calibration_s": cal_s, "encoder_rho": ck.get("rho")})
        out["branch_weight"] = index.beta
        out["calibration_by_weight"] = {str(b): {str(k): v for k, v in r.items()}
                                        for b, r in getattr(index, "calibration", {}).items()}
        # what training buys: the same filter with the untrained network (its
        # branch weight calibrated on the same sample), same budgets
        from trajsimimeasures_b200.surrogate import Encoder
        raw = SurrogateIndex(Encoder.init(Dset, seed=0), Dset)
        c_raw, _ = raw.calibrate(cal, 10, target=0.99)
        out["untrained_calibrated"] = {"candidates": c_raw, "branch_weight": raw.beta}
        counts = sorted(set(rec) | ({c} if c else set()) | {100, 200})
        out["recall_at_10_trained"] = {str(cc): recall_at_k(index.query(Q, 10, c=cc)[1], ex_i) for cc in counts}
        out["recall_at_10_untrained"] = {str(cc): recall_at_k(raw.query(Q, 10, c=cc)[1], ex_i) for cc in counts}
        _, ex50 = knn_exhaustive(Q, Dset, 50)
        out["skip_weights"] = {"trained": [round(float(x), 4) for x in enc.params[-16:].tolist()],
                               "untrained": [round(float(x), 4) for x in raw.enc.params[-16:].tolist()]}
        out["hit_ratio"] = hit_ratios(Q, Dset, enc, ex50)
        out["hit_ratio_untrained"] = hit_ratios(Q, Dset, raw.enc, ex50)
    out["host_generate_s"] = gen_s
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_sym(args):
    """Symmetric all-pairs of one 2000-trajectory set (the clustering shape):
    the upper-triangle driver (tsm_allpairs_sym, each unordered pair once,
    mirrored) against the full Q == D matrix, per measure, device time."""
    import torch
    from trajsimimeasures_b200 import datagen as D
    from trajsimimeasures_b200.engine import TrajSet, allpairs_sym_raw, matrix_raw
    dev = torch.device("cuda", 0)
    p, o, l = D.trajectory_set(args.n_traj, seed=D.SEED_DB)
    s = TrajSet.from_packed(p, o, l, device=dev)
    n = s.n
    order = s.order_by_length()
    out = torch.empty((n, n), dtype=torch.float32, device=dev)
    cnt = torch.empty((n, n), dtype=torch.int32, device=dev)
    res = {}
    for name in MEASURES:
        m = MID[name]
        c = cnt if m in (1, 2) else None
        full = lambda: matrix_raw(m, s, s, out=out, counts=c, d_order=order, eps=EPS, gpoint=D.BOX_CENTRE)
        sym = lambda: allpairs_sym_raw(m, s, out=out, counts=c, eps=EPS, gpoint=D.BOX_CENTRE)
        t = {}
        for key, fn in (("full_ms", full), ("sym_ms", sym)):
            for _ in range(args.warmup):
                fn()
            e0, e1 = _events()
            e0.record()
            for _ in range(args.steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            t[key] = e0.elapsed_time(e1) / args.steps
        t["unique_pairs_per_s_sym"] = n * (n + 1) / 2 / (t["sym_ms"] / 1e3)
        t["speedup"] = t["full_ms"] / t["sym_ms"]
        res[name] = t
    print(json.dumps({"workload": f"allpairs_symmetric_{n}_six_measures", "n_traj": n, "per_measure": res,
                      "total_full_ms": sum(v["full_ms"] for v in res.values()),
                      "total_sym_ms": sum(v["sym_ms"] for v in res.values())}), flush=True)


def run_numba_arm(args, ws, rank):
    """The reference's own GPU path on this GPU: core.dtw / erp / dfrechet /
    hausdorff / edr / lcss of the reference (Numba-CUDA, FP64, one 64-thread
    block per pair; core/dtw.py:56-77 etc.), installed unmodified in
    baseline/_ref by baseline/install_reference.py, called as the reference's
    paired driver calls them (test_trajsimi_time.py:222-276): 1,000 pairs,
    batches of 512 (config.py:45), padded float64 host arrays in, float64 out.
    ERP gets one trailing dummy pair whose second trajectory is as long as the
    padding, which keeps the reference kernel's gap-distance buffer (sized by
    the longest second trajectory, core/erp.py:106,112) in bounds.  Hausdorff
    is timed only: its host maximum reads uninitialised padded slots
    (core/hausdorff.py:114,121)."""
    if rank != 0:
        return
    ref = os.path.join(ROOT, "baseline", "_ref")
    line = {"impl": "numba", "metric": "pairs/s per measure (1,000 pairs, U{20..200}, reference Numba-CUDA)"}
    if not os.path.isdir(os.path.join(ref, "core")):
        line["unavailable"] = "baseline/_ref/core missing: run baseline/install_reference.py where the reference exists"
        print(json.dumps(line), flush=True)
        return
    try:
        sys.path.insert(0, ref)
        import core as rcore  # the reference's package
        from numba import cuda
        if not cuda.is_available():
            raise RuntimeError("numba.cuda reports no usable GPU")
        cc = cuda.get_current_device().compute_capability
    except Exception as e:  # noqa: BLE001 - reported, not hidden
        line["unavailable"] = f"{type(e).__name__}: {e}"[:300]
        print(json.dumps(line), flush=True)
        return
    from trajsimimeasures_b200 import datagen as D
    pts, off, lens, ia, ib = D.pairs_uniform(1000)
    la, lb = lens[ia].astype(np.int64), lens[ib].astype(np.int64)
    t1, t2 = D.pad(D.unpack(pts, off, lens, ia)), D.pad(D.unpack(pts, off, lens, ib))
    w = t1.shape[1]
    B = 512

    def batches(fn):
        for b0 in range(0, 1000, B):
            fn(slice(b0, min(b0 + B, 1000)))

    def erp_call(s):
        a = np.concatenate([t1[s], np.zeros((1, w, 2))])
        b = np.concatenate([t2[s], np.zeros((1, w, 2))])
        return rcore.erp(a, np.append(la[s], 1), b, np.append(lb[s], w), list(D.BOX_CENTRE), threads_per_traj=64)
    calls = {"dtw": lambda s: rcore.dtw(t1[s], la[s], t2[s], lb[s], threads_per_traj=64),
             "edr": lambda s: rcore.edr(t1[s], la[s], t2[s], lb[s], EPS, threads_per_traj=64),
             "lcss": lambda s: rcore.lcss(t1[s], la[s], t2[s], lb[s], EPS, threads_per_traj=64),
             "erp": erp_call,
             "dfrechet": lambda s: rcore.dfrechet(t1[s], la[s], t2[s], lb[s], threads_per_traj=64),
             "hausdorff": lambda s: rcore.hausdorff(t1[s], la[s], t2[s], lb[s], threads_per_traj=64)}
    per = {}
    try:
        for name, fn in calls.items():
            for _ in range(max(1, args.warmup)):
                batches(fn)  # the first call JIT-compiles the kernel
            cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                batches(fn)
            cuda.synchronize()
            dt = (time.perf_counter() - t0) / args.steps
            per[name] = {"pairs_per_s": 1000 / dt, "ms_per_1000_pairs": 1e3 * dt}
    except Exception as e:  # noqa: BLE001
        line["unavailable"] = f"{type(e).__name__}: {e}"[:300]
        line["per_measure"] = per
        print(json.dumps(line), flush=True)
        return
    line.update({"compute_capability": list(cc), "steps": args.steps, "warmup": args.warmup,
                 "batch": B, "threads_per_traj": 64, "per_measure": per,
                 "config": {"workload": "pairs_1000_uniform_20_200", "eps_deg": EPS, "erp_gpoint": list(D.BOX_CENTRE)}})
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "numba":
        run_numba_arm(args, ws, rank)
        return
    if args.workload != "allpairs":
        {"uneven": run_uneven, "surrogate": run_surrogate, "knn": run_knn, "sym": run_sym}[args.workload](args)
        return
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        return
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
