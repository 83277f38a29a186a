"""Batched uneven workload: thousands of ciphertext operations of mixed ring
dimension (N = 2^12, 2^13), level (2..8 limbs) and kind (ct x ct + relin +
rescale, ct x pt + rescale) in one CUDA-graph replay per step.

Items are grouped into same-shape buckets (kind, log N, level).  Two
executions of the same buckets, bit-identical to each other:

* ``persistent`` (PersistentPlan, ckks_batch_plan_*): ONE launch of the
  persistent batch kernel drains a device work list of every bucket's work
  units (a ct x ct pair's tensor limbs, ModUp target primes and ModDown
  polynomials, a ct x pt item's two polynomials) with per-item dependency
  counters and bounded waits; a graph replay is one memset node and one
  kernel node.
* ``streams``: each bucket is one batched launch sequence of the library's
  kernels (one CTA per polynomial limb, so buckets of different shapes need
  no padding), spread over a pool of streams and captured into one graph.

The autotuner times every bucket alone under each launch shape (per-thread
radix 2^K, K = 2..5, balanced or tight register budget, limbs / work units
per CTA, the persistent TMA-fed tensor kernel, chunking of the bucket into
launches) and keeps the fastest, then times the persistent plan under each
lag (how far a dependent stage is listed after its producers); the choice
is baked into the graph at capture time.

The reference's batching is time multiplexing of four poly-mult instances on
one FPGA (rtl/m4/e2e_ckks_mult_ctrl_m4.sv:368-482, TIME_MULT = 4 in
scripts/exp_e17_energy_efficiency.py:32).
"""
from __future__ import annotations

import ctypes
import itertools
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, ops
from .evaluator import Evaluator
from .params import CkksParams

U64 = torch.uint64


@dataclass(frozen=True)
class Shape:
    op: str          # "ctct" or "ctpt"
    log_n: int
    level: int


def synthetic_workload(n_items: int = 4096, seed: int = 0, frac_ctct: float = 0.6,
                       log_ns=(12, 13), levels=tuple(range(2, 9))) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_items):
        op = "ctct" if rng.random() < frac_ctct else "ctpt"
        out.append(Shape(op, int(rng.choice(log_ns)), int(rng.choice(levels))))
    return out


@dataclass
class Bucket:
    shape: Shape
    count: int
    a: torch.Tensor = None
    b: torch.Tensor = None          # second ciphertext (ctct) or plaintext (ctpt)
    out: torch.Tensor = None
    scratch: torch.Tensor = None
    tune: dict = field(default_factory=lambda: {"k": 0, "minb": 0, "chunk": 0, "upc": 0})


# Per-thread radix 2^K the autotuner sweeps (K = log2 coefficients per thread).
RADIX_LOG2 = (2, 3, 4, 5)
# Work units (limbs, target primes, output polynomials) per CTA of the ct-mult kernels.
UNITS_PER_CTA = (1, 2, 4)


def cm_shape_built(log_n: int, k: int, minb: int) -> bool:
    """Whether the library builds the ct-mult kernels for (log N, K, budget):
    K = 3, 4 for log N in [6, 14] (at most 1024 threads), K = 2 for log N in
    [10, 12], K = 5 for log N in [10, 14] with the balanced budget only."""
    if not 6 <= log_n <= 14 or ((1 << log_n) >> k) > 1024:
        return False
    if k == 2:
        return 10 <= log_n <= 12
    if k == 5:
        return log_n >= 10 and minb == 1
    return k in (3, 4)


class PersistentPlan:
    """ckks_batch_plan over a list of Buckets: created once (validates, sizes
    and allocates its device memory, lists the work units), then run any
    number of times; ``run`` is capturable into a CUDA graph."""

    def __init__(self, evs: dict, buckets: list, lag_percent: int = 400):
        arr = (_lib.BatchBucket * max(1, len(buckets)))()
        for i, bk in enumerate(buckets):
            ev = evs[bk.shape.log_n]
            ctct = bk.shape.op == "ctct"
            arr[i] = _lib.BatchBucket(ev.ctx.handle, _lib.BATCH_CT_CT if ctct else _lib.BATCH_CT_PT, bk.count,
                                      bk.shape.level, 0 if ctct else 1, bk.a.data_ptr(), bk.b.data_ptr(),
                                      bk.out.data_ptr(), ev.rlk.data_ptr() if ctct else None)
        h = ctypes.c_void_p()
        _lib.call("ckks_batch_plan_create", arr, len(buckets), int(lag_percent), ctypes.byref(h))
        self.handle = h
        self.buckets = buckets
        self.lag_percent = lag_percent
        # True: the paired list (the default: N = 2^12 units two per slot);
        # False: the phased list (N = 2^13 whole-CTA slots, then N = 2^12 units
        # taken by each half on its own)
        self.paired = True

    def run(self, wait_cycles: int = 0, flags: int = 0, stream=None):
        st = (stream or torch.cuda.current_stream()).cuda_stream
        if not self.paired:
            flags |= _lib.BATCH_RUN_PHASED
        _lib.call("ckks_batch_plan_run", self.handle, int(wait_cycles), int(flags), st)

    def incomplete(self) -> tuple[int, list]:
        """(items of the last run whose output is incomplete, per-bucket complete flags)."""
        n = ctypes.c_int()
        flags = (ctypes.c_uint8 * max(1, len(self.buckets)))()
        _lib.call("ckks_batch_plan_incomplete", self.handle, ctypes.byref(n), flags)
        return n.value, [bool(flags[i]) for i in range(len(self.buckets))]

    def info(self) -> dict:
        nu, ns = ctypes.c_longlong(), ctypes.c_longlong()
        grid, smem, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        _lib.call("ckks_batch_plan_info", self.handle, ctypes.byref(nu), ctypes.byref(ns), ctypes.byref(grid),
                  ctypes.byref(smem), ctypes.byref(nb))
        return {"units": nu.value, "slots": ns.value, "grid": grid.value, "smem_bytes": smem.value,
                "device_bytes": nb.value, "lag_percent": self.lag_percent,
                "list": "paired" if self.paired else "phased"}

    def close(self):
        if self.handle:
            _lib.raw("ckks_batch_plan_destroy")(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchExecutor:
    def __init__(self, items: list, max_level: int = 8, seed: int = 0, n_streams: int = 4, device=None,
                 mode: str = "streams"):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        counts = {}
        for it in items:
            counts[it] = counts.get(it, 0) + 1
        self.n_items = len(items)
        self.evs = {}
        for log_n in sorted({s.log_n for s in counts}):
            ev = Evaluator(CkksParams.standard(log_n, max_level, seed=seed + log_n), device=self.device)
            ev.keygen()
            self.evs[log_n] = ev
        self.buckets = []
        for sh, cnt in sorted(counts.items(), key=lambda kv: (kv[0].op, kv[0].log_n, kv[0].level)):
            ev = self.evs[sh.log_n]
            bk = Bucket(sh, cnt)
            bk.a = ev.uniform(cnt * 2, sh.level).reshape(cnt, 2, sh.level, ev.n)
            if sh.op == "ctct":
                bk.b = ev.uniform(cnt * 2, sh.level).reshape(cnt, 2, sh.level, ev.n)
                need = ops.ct_mul_scratch_bytes(ev.ctx, cnt, sh.level)
                bk.scratch = torch.empty((need + 7) // 8, dtype=U64, device=self.device)
            else:
                bk.b = ev.uniform(cnt, sh.level)
            bk.out = torch.empty((cnt, 2, sh.level - 1, ev.n), dtype=U64, device=self.device)
            self.buckets.append(bk)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(n_streams)]
        self.graph = None
        self.plan = None
        self.mode = mode

    @property
    def mode(self) -> str:
        return self._mode

    @mode.setter
    def mode(self, m: str):
        if m not in ("streams", "persistent"):
            raise ValueError(f"mode={m!r}: 'streams' or 'persistent'")
        self._mode = m
        self.graph = None               # a captured step belongs to one mode

    def persistent_plan(self, lag_percent: int = 400) -> PersistentPlan:
        if self.plan is not None and self.plan.lag_percent == lag_percent:
            return self.plan
        if self.plan is not None:
            self.plan.close()
        self.plan = PersistentPlan(self.evs, self.buckets, lag_percent)
        self.graph = None
        return self.plan

    # ---------------------------------------------------------------- launches
    def launch(self, bk: Bucket):
        ev = self.evs[bk.shape.log_n]
        ctx = ev.ctx
        st = torch.cuda.current_stream().cuda_stream
        chunk = bk.tune["chunk"] or bk.count
        lvl = bk.shape.level
        if bk.shape.op == "ctct":
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 0, bk.tune["k"])
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 1, bk.tune["minb"])
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 4, bk.tune.get("upc", 0))
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 5, bk.tune.get("tma", 0))
            # buckets already overlap on the executor's streams: one sub-batch per call
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, 1)
            for s in range(0, bk.count, chunk):
                e = min(bk.count, s + chunk)
                n = e - s
                _lib.call("ckks_ct_mul_relin_rescale", ctx.handle, bk.out[s:e].data_ptr(), bk.a[s:e].data_ptr(),
                          bk.b[s:e].data_ptr(), ev.rlk.data_ptr(), n, lvl, bk.scratch.data_ptr(),
                          bk.scratch.numel() * 8, st)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 0, 0)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 1, 0)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 2, 0)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 4, 0)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 5, 0)
        else:
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 3, bk.tune["k"])
            for s in range(0, bk.count, chunk):
                e = min(bk.count, s + chunk)
                _lib.call("ckks_ct_mul_plain_rescale", ctx.handle, bk.out[s:e].data_ptr(), bk.a[s:e].data_ptr(),
                          bk.b[s:e].data_ptr(), 1, e - s, lvl, st)
            _lib.call("ckks_ctx_set_tuning", ctx.handle, 3, 0)

    def run(self):
        """One step in the selected mode, without a graph."""
        if self.mode == "persistent":
            (self.plan or self.persistent_plan()).run()
        else:
            self.run_eager()

    def run_eager(self):
        cur = torch.cuda.current_stream()
        fork = torch.cuda.Event()
        fork.record(cur)
        for s in self.streams:
            s.wait_event(fork)
        order = sorted(self.buckets, key=lambda b: -b.count * (1 << b.shape.log_n) * b.shape.level)
        for i, bk in enumerate(order):
            with torch.cuda.stream(self.streams[i % len(self.streams)]):
                self.launch(bk)
        for s in self.streams:
            j = torch.cuda.Event()
            j.record(s)
            cur.wait_event(j)

    def capture(self):
        self.run()                            # kernel attributes, lazy module loading
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def step(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def time_steps(self, steps: int = 10, warmup: int = 3, use_graph: bool = True) -> dict:
        fn = self.step if use_graph else self.run
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return {"ms_per_step": ms, "items_per_s": self.n_items / (ms / 1000.0), "graph": use_graph,
                "mode": self.mode}

    # ---------------------------------------------------------------- autotuner
    def autotune(self, reps: int = 3) -> dict:
        """Time each bucket alone under every launch shape; keep the fastest
        when it beats the default shape by more than 3 %."""
        choices = {}
        for bk in self.buckets:
            log_n = bk.shape.log_n
            cands = [{"k": 0, "minb": 0, "chunk": 0, "upc": 0}]  # the library's default shape first
            if bk.shape.op == "ctct":
                cands += [{"k": k, "minb": mb, "chunk": ch, "upc": u}
                          for k, mb, ch, u in itertools.product(RADIX_LOG2, (1, 2), (0, 128), UNITS_PER_CTA)
                          if cm_shape_built(log_n, k, mb) and not (ch and ch >= bk.count)]
                # the persistent TMA-fed tensor kernel at the default shape
                cands.append({"k": 0, "minb": 0, "chunk": 0, "upc": 0, "tma": 1})
            else:
                cands += [{"k": k, "minb": 0, "chunk": 0, "upc": 0} for k in RADIX_LOG2
                          if ((1 << log_n) >> k) <= 1024]
            best = None
            sweep = {}
            default_ms = None
            for c in cands:
                bk.tune = c
                self.launch(bk)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    self.launch(bk)
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / reps
                sweep[f"K{c['k']}/b{c['minb']}/c{c['chunk']}/u{c['upc']}/t{c.get('tma', 0)}"] = round(t, 4)
                if c is cands[0]:
                    default_ms = t
                if best is None or t < best[0]:
                    best = (t, c)
            # keep the default shape unless a candidate beats it clearly: the
            # buckets run concurrently in the graph, where a shape that wins
            # alone by a few per cent can lose
            if default_ms is not None and best[0] > 0.97 * default_ms:
                best = (default_ms, cands[0])
            bk.tune = best[1]
            choices[f"{bk.shape.op}/N=2^{bk.shape.log_n}/L={bk.shape.level}"] = {"ms": best[0], **best[1],
                                                                              "count": bk.count,
                                                                              "sweep": sweep}
        self.graph = None
        return choices

    def autotune_persistent(self, reps: int = 3, lags=(200, 400, 800)) -> dict:
        """Time the persistent plan under each lag (how far a dependent stage
        is listed after its producers, in % of a wave) and both of its unit
        lists (phased, paired); keep the fastest."""
        sweep = {}
        best = None
        for lag in lags:
            plan = PersistentPlan(self.evs, self.buckets, lag)
            keep = False
            for paired in (True, False):
                plan.paired = paired
                plan.run()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    plan.run()
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / reps
                sweep[f"{'paired' if paired else 'phased'}/lag{lag}"] = round(t, 4)
                if best is None or t < best[0]:
                    if best is not None and best[1] is not plan:
                        best[1].close()
                    best = (t, plan, paired)
                    keep = True
            if keep:
                plan.paired = best[2]
            else:
                plan.close()
        if self.plan is not None:
            self.plan.close()
        self.plan = best[1]
        self.graph = None
        return {"ms": best[0], **self.plan.info(), "sweep": sweep}


def main(argv=None) -> int:
    """Time the batched uneven workload: eager launches, one graph replay per
    step with the default launch shapes, then after autotuning."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--items", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--no-autotune", action="store_true")
    a = ap.parse_args(argv)
    items = synthetic_workload(a.items, seed=a.seed)
    ex = BatchExecutor(items)
    ex.mode = "persistent"
    ex.persistent_plan()
    persistent = ex.time_steps(a.steps, a.warmup, use_graph=True)
    ex.mode = "streams"
    res = {"workload": f"{a.items} items, 60% ct x ct + relin + rescale / 40% ct x pt + rescale, "
                       "N in {2^12, 2^13}, level uniform in 2..8",
           "buckets": len(ex.buckets),
           "ctct_items": sum(b.count for b in ex.buckets if b.shape.op == "ctct"),
           "eager": ex.time_steps(a.steps, a.warmup, use_graph=False),
           "graph_default": ex.time_steps(a.steps, a.warmup, use_graph=True),
           "persistent_default": {**persistent, **ex.plan.info()}}
    if not a.no_autotune:
        res["autotune"] = ex.autotune()
        res["graph_tuned"] = ex.time_steps(a.steps, a.warmup, use_graph=True)
        res["autotune_persistent"] = ex.autotune_persistent()
        ex.mode = "persistent"
        res["persistent_tuned"] = ex.time_steps(a.steps, a.warmup, use_graph=True)
    print(json.dumps(res, indent=1))
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
