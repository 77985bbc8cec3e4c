"""Length-bucketed persistent scheduling of uneven paired batches, its
autotuner and CUDA-graph steady state.

The reference runs fixed batches of 512 pairs with 64 threads per pair
(config.py:43,45; test_trajsimi_time.py:222-276), whatever their lengths.
Here a batch of pairs (any lengths up to the per-warp capacity, any mix of
the six measures) is planned once on the host and executed by ONE persistent
launch (tsm_pairs_sched) whose warps pull tasks from a device queue:

* every (pair, measure) item goes to a bucket by the shape of its DP (rows =
  the longer trajectory, nr; columns = the shorter, nc):
    tile   (one pair per lane)        nc <= warp_floats/32 and a short loop
    groupG (one pair per G lanes)     G = 4, 8, 16 or 32 (wave), the smallest
                                      G whose super-strip loop takes at most
                                      max_steps steps, nc <= warp_floats*G/32
  Hausdorff items are one pair per lane, or one per warp when long.
* inside a bucket items are sorted by loop shape (row passes or super-strips,
  then columns) so a warp's lanes/groups get equal trip counts, then cut into
  warp tasks;
* the long tasks go first, largest first (longest-processing-time-first), so
  no long pair starts near the end; the rest follow one measure after the
  other, each largest first (task_order).

The autotuner picks (rows per strip, shared memory per warp, step budget) for a batch by
timing candidate plans on the device; choices are cached as JSON keyed by GPU
name, measures and a length-distribution signature.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .engine import _ptr, _stream_ptr, measure_id

KIND_TILE, KIND_GROUP8, KIND_WAVE, KIND_HAUSDORFF, KIND_HAUSDORFF_WARP, KIND_GROUP4, KIND_GROUP16 = 0, 1, 2, 3, 4, 5, 6
GROUP_KIND = {4: KIND_GROUP4, 8: KIND_GROUP8, 16: KIND_GROUP16, 32: KIND_WAVE}
# A pair may keep its lanes for at most this many loop steps (one step = R
# cells per lane) before the planner spreads it over more lanes.
MAX_STEPS = 4096
# Resident warps of a launch, for the task order when the caller gives none
# (B200: 148 SMs x 12 warps at 16 KB of shared memory per warp).
WARPS = 148 * 12
# Hausdorff pairs with more point-segment evaluations than this run one per
# warp (the lanes split the points) instead of one per lane.
HAUSDORFF_WARP_UNITS = 1 << 17
# (rows per strip, shared-memory floats per warp, step budget) tried by the autotuner
CANDIDATES = [(8, 3072, 4096), (8, 3072, 2048), (8, 4096, 4096), (8, 4096, 8192), (8, 2048, 4096),
              (8, 8192, 4096), (4, 4096, 4096)]


def group_steps(nr, nc, rows, G):
    """Loop steps of a pair on a G-lane group: super-strips of G*rows rows,
    nc + G - 1 steps each."""
    return ((nr + G * rows - 1) // (G * rows)) * (nc + G - 1)


def tile_steps(nr, nc, rows):
    """Loop steps of a pair on one lane of a tile task: passes of 2*rows rows,
    nc + 1 steps each (one step = 2*rows cells)."""
    return ((nr + 2 * rows - 1) // (2 * rows)) * (nc + 1)


@dataclass
class Plan:
    order: np.ndarray        # int32, pair indices; tasks index into it
    tasks: np.ndarray        # int32 [n_tasks, 4] = kind, measure, first, count
    rows: int
    warp_floats: int
    measures: list
    max_len: int
    cost: np.ndarray = field(repr=False, default=None)  # per task, lane-cell units

    @property
    def n_tasks(self):
        return int(self.tasks.shape[0])


def plan_pairs(len_a, len_b, measures, rows=8, warp_floats=4096, max_steps=MAX_STEPS, warps=None) -> Plan:
    """Buckets, orders and cuts the (pair, measure) items into warp tasks.
    warps: the number of warps the launch keeps resident (for task_order)."""
    warps = WARPS if warps is None else warps
    la = np.asarray(len_a, dtype=np.int64)
    lb = np.asarray(len_b, dtype=np.int64)
    n = la.shape[0]
    nr, nc = np.maximum(la, lb), np.minimum(la, lb)
    tile_cap, wave_cap = warp_floats // 32, warp_floats
    ms = [measure_id(m) for m in measures]
    dp_ms = [m for m in ms if m != _lib.HAUSDORFF]
    if dp_ms and n and nc.max() > wave_cap:
        raise ValueError(f"a pair's shorter side ({nc.max()}) exceeds the per-warp capacity {wave_cap}; "
                         "raise warp_floats")
    orders, tasks, costs = [], [], []
    pos = 0

    def emit(kind, m, idx, per_task, cost_of, shape_of=None):
        """Orders a bucket's items and cuts them into tasks of per_task items.
        shape_of (int64, larger = heavier), when given, is the sort key: lanes
        that run their own loops (one pair per lane) waste the steps by which
        their trip counts differ, so such tasks group items of equal loop
        shape, not merely of equal cost.  Otherwise the items go by cost."""
        nonlocal pos
        if idx.size == 0:
            return
        key = cost_of[idx] if shape_of is None else shape_of[idx]
        o = idx[np.argsort(-key, kind="stable")]
        starts = np.arange(0, o.size, per_task)
        cnt = np.minimum(per_task, o.size - starts)
        t = np.stack([np.full(starts.size, kind), np.full(starts.size, m), pos + starts, cnt], axis=1)
        orders.append(o.astype(np.int32))
        tasks.append(t.astype(np.int32))
        costs.append(np.maximum.reduceat(cost_of[o], starts).astype(np.float64))  # a task lasts as long as its largest item
        pos += o.size

    all_idx = np.arange(n, dtype=np.int64)
    for m in ms:
        if m == _lib.HAUSDORFF:
            units = (la * lb + lb * la).astype(np.float64)  # segments + the last vertex, both directions
            big = units > HAUSDORFF_WARP_UNITS
            hshape = ((nr + rows - 1) // rows) * 65536 + nc  # point blocks of the longer side, then the shorter side
            emit(KIND_HAUSDORFF, m, all_idx[~big], 32, units * 1.8, hshape)
            emit(KIND_HAUSDORFF_WARP, m, all_idx[big], 1, units * 1.8 / 32 + 64 * (la + lb))
            continue
        # a tile step does 2*rows cells per lane, about two group steps' work
        tile = (nc <= tile_cap) & (2 * tile_steps(nr, nc, rows) <= max_steps)
        passes = (nr + 2 * rows - 1) // (2 * rows)
        # a tile lane runs passes x (nc + 1) steps: group by passes, then by nc
        emit(KIND_TILE, m, all_idx[tile], 32, (passes * 2 * rows * (nc + 1)).astype(np.float64),
             passes * 65536 + nc)
        todo = ~tile
        gsize = np.zeros(n, np.int64)
        for G in (4, 8, 16, 32):  # the smallest group within the step budget
            fits = todo & (nc <= warp_floats * G // 32)
            pick = fits & (group_steps(nr, nc, rows, G) <= max_steps)
            if G == 32:
                pick = fits  # the widest group takes what is left
            gsize[pick] = G
            todo &= ~pick
        for G in (4, 8, 16, 32):
            sel = gsize == G
            strips = (nr + G * rows - 1) // (G * rows)
            emit(GROUP_KIND[G], m, all_idx[sel], 32 // G,
                 (group_steps(nr, nc, rows, G) * rows * 1.3).astype(np.float64), strips * 65536 + nc)
    if not tasks:
        return Plan(np.zeros(0, np.int32), np.zeros((0, 4), np.int32), rows, warp_floats, ms, 0, np.zeros(0))
    order = np.concatenate(orders)
    T = np.concatenate(tasks)
    C = np.concatenate(costs)
    s = task_order(T[:, 1], C, warps)
    return Plan(order, np.ascontiguousarray(T[s]), rows, warp_floats, ms,
                int(max(la.max(initial=0), lb.max(initial=0))), C[s])


def task_order(measure, cost, warps=WARPS):
    """Queue order of the tasks: the long ones first, largest first
    (longest-processing-time-first, so that no long task starts near the
    end), then the rest one measure after the other, each largest first.

    A task is long when it costs more than a quarter of the batch's cost per
    resident warp.  Grouping the rest by measure keeps the instructions that
    the SMs run at any one time to one measure's code: with the measures
    interleaved, the persistent kernel stalls on instruction fetch."""
    cost = np.asarray(cost, dtype=np.float64)
    if cost.size == 0:
        return np.zeros(0, np.int64)
    lpt = np.argsort(-cost, kind="stable")
    long = cost[lpt] > cost.sum() / max(int(warps), 1) / 4
    rest = lpt[~long]
    m = np.asarray(measure)[rest]
    by_total = sorted(set(m.tolist()), key=lambda x: -cost[rest][m == x].sum())
    return np.concatenate([lpt[long]] + [rest[m == x] for x in by_total])


class PairsScheduler:
    """A planned batch resident on the device: one persistent launch per run().

    pts/off/len tensors: the packed pairs (device); len_a/len_b host copies
    are used for planning.  Results: out[measure_id, pair] (float32) and
    counts[measure_id, pair] (int32, EDR/LCSS)."""

    def __init__(self, pts, off_a, len_a, off_b, len_b, measures, *, eps=0.0, gpoint=(0.0, 0.0), exact=False,
                 rows=8, warp_floats=4096, max_steps=MAX_STEPS, len_a_host=None, len_b_host=None, plan=None):
        self.dev = pts.device
        la = np.asarray(len_a_host if len_a_host is not None else len_a.cpu().numpy())
        lb = np.asarray(len_b_host if len_b_host is not None else len_b.cpu().numpy())
        self.plan = plan or plan_pairs(la, lb, measures, rows, warp_floats, max_steps)
        self.pts, self.off_a, self.len_a, self.off_b, self.len_b = pts, off_a, len_a, off_b, len_b
        self.n = int(off_a.shape[0])
        self.order = torch.from_numpy(self.plan.order).to(self.dev)
        self.tasks = torch.from_numpy(self.plan.tasks.reshape(-1)).to(self.dev)
        self.out = torch.full((6, self.n), float("nan"), dtype=torch.float32, device=self.dev)
        self.counts = torch.zeros((6, self.n), dtype=torch.int32, device=self.dev)
        nbytes = _lib.load().tsm_sched_workspace_bytes()
        self.workspace = torch.zeros(nbytes // 4, dtype=torch.int32, device=self.dev)
        self.params = _lib.params(eps, gpoint, exact, self.plan.rows)
        self.graph = None

    def run(self, stream=None):
        lib = _lib.load()
        rc = lib.tsm_pairs_sched(_ptr(self.pts), _ptr(self.off_a), _ptr(self.len_a), _ptr(self.off_b),
                                 _ptr(self.len_b), _ptr(self.order), _ptr(self.tasks), self.plan.n_tasks,
                                 self.plan.max_len, self.plan.warp_floats, ctypes.byref(self.params),
                                 _ptr(self.out), _ptr(self.counts), self.n, _ptr(self.workspace),
                                 _stream_ptr(stream))
        _lib.check(rc, "tsm_pairs_sched")

    def capture(self):
        """Records run() into a CUDA graph (steady-state replays via replay())."""
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.run(s)  # warm-up outside the graph (sets kernel attributes)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.run(s)
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()


# ---------------------------------------------------------------------------
# autotuner
# ---------------------------------------------------------------------------

def _cache_path():
    d = os.environ.get("TSM_CACHE_DIR", os.path.join(os.path.expanduser("~"), ".cache", "trajsimimeasures_b200"))
    return os.path.join(d, "autotune.json")


def signature(len_a, len_b, measures) -> str:
    """Length-distribution signature: deciles of the shorter and longer sides
    rounded to a power-of-two grid, plus the measure set."""
    la, lb = np.asarray(len_a), np.asarray(len_b)
    nr, nc = np.maximum(la, lb), np.minimum(la, lb)
    q = np.linspace(0.1, 0.9, 5)
    f = lambda x: [int(2 ** np.round(np.log2(max(v, 1)) * 2) / 2) for v in np.quantile(x, q)]  # noqa: E731
    ms = sorted(measure_id(m) for m in measures)
    return f"m{ms}_nc{f(nc)}_nr{f(nr)}_max{int(np.max(nc, initial=0))}"


def load_cache() -> dict:
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(c: dict):
    p = _cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(c, fh, indent=1, sort_keys=True)
    os.replace(tmp, p)


def autotune(pts, off_a, len_a, off_b, len_b, measures, *, eps=0.0, gpoint=(0.0, 0.0), exact=False,
             candidates=CANDIDATES, reps=3, use_cache=True, len_a_host=None, len_b_host=None):
    """Times each (rows, warp_floats, max_steps) candidate on this batch;
    returns (best (rows, warp_floats, max_steps), {candidate: ms}).  Cached
    per GPU/signature."""
    la = np.asarray(len_a_host if len_a_host is not None else len_a.cpu().numpy())
    lb = np.asarray(len_b_host if len_b_host is not None else len_b.cpu().numpy())
    gpu = torch.cuda.get_device_name(pts.device)
    key = f"{gpu}|{signature(la, lb, measures)}|{'exact' if exact else 'fast'}"
    cache = load_cache() if use_cache else {}
    if key in cache and len(cache[key].get("best", ())) == 3:
        return tuple(int(x) for x in cache[key]["best"]), cache[key].get("ms", {})
    times = {}
    nc_max = int(np.minimum(la, lb).max(initial=0))
    for rows, wf, mst in candidates:
        if any(measure_id(m) != _lib.HAUSDORFF for m in measures) and nc_max > wf:
            continue
        s = PairsScheduler(pts, off_a, len_a, off_b, len_b, measures, eps=eps, gpoint=gpoint, exact=exact,
                           rows=rows, warp_floats=wf, max_steps=mst, len_a_host=la, len_b_host=lb)
        s.run()
        torch.cuda.synchronize(pts.device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        for _ in range(reps):
            s.run()
        ev[1].record()
        torch.cuda.synchronize(pts.device)
        times[f"{rows},{wf},{mst}"] = ev[0].elapsed_time(ev[1]) / reps
    if not times:
        raise ValueError("no candidate can hold these pairs")
    best = min(times, key=times.get)
    choice = tuple(int(x) for x in best.split(","))
    if use_cache:
        cache[key] = {"best": list(choice), "ms": times}
        save_cache(cache)
    return choice, times
