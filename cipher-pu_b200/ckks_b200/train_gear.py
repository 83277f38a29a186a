"""Train the learned gear controller and compare it with the plain one.

    python -m ckks_b200.train_gear train   [--traces 200000] [--epochs 40] [--out PATH]
    torchrun --nproc-per-node G -m ckks_b200.train_gear train ...   (data-parallel)
    python -m ckks_b200.train_gear compare [--net PATH] [--model mlp|cnn|mlp_compressible] [--batches 8]

train: generates noise-monitor traces by running random encrypted layers of
the encrypted-MLP family (N = 2^13, L = 4) at every gear, trains the
16 -> 64 -> 64 -> 4 network on the GPU with the library's kernels and writes
the checkpoint (weights, feature normalisation, schema version).
compare: encrypted inference of a batch stream under the plain controller
(probe every layer) and the learned one (probe when uncertain), same model,
same inputs; prints samples/s, logit SNR vs FP64, top-1 agreement, probes.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

DEFAULT_NET = Path(__file__).resolve().parent / "data" / "gear_net.npz"


def train(n_traces: int = 200_000, epochs: int = 40, out: Path = DEFAULT_NET, seed: int = 0,
          log_n: int = 13, levels: int = 4) -> dict:
    from .dist import world
    from .evaluator import Evaluator
    from .gear_learn import GearNet, gen_traces
    from .params import CkksParams
    from .sharded import gen_traces as sharded_traces
    ev = Evaluator(CkksParams.standard(log_n, levels, seed=seed + 100))
    ev.keygen()
    t0 = time.perf_counter()
    # each rank generates its share (own seed), every rank gets all traces
    X, T = sharded_traces(n_traces, seed, lambda count, sd: gen_traces(ev, count, seed=sd))
    t_gen = time.perf_counter() - t0
    net = GearNet(seed=seed)
    t1 = time.perf_counter()
    hist = net.fit(X, T, epochs=epochs, seed=seed)   # data-parallel under torch.distributed
    t_fit = time.perf_counter() - t1
    out = Path(out)
    if world()[1] == 0:
        out.parent.mkdir(parents=True, exist_ok=True)
        net.save(out)
    return {"traces": len(X), "gen_s": t_gen, "fit_s": t_fit, "val_rmse_db": hist["val_rmse_db"][-1],
            "val_rmse_curve": hist["val_rmse_db"], "checkpoint": str(out)}


def compare(net_path: Path = DEFAULT_NET, model: str = "mlp", batches: int = 8, batch: int = 1024,
            target_db: float = 40.0, seed: int = 0) -> dict:
    from .evaluator import Evaluator
    from .gear_learn import GearNet, LearnedController, PlainController
    from .mlp import EncryptedMLP
    from .models import cnn_28x28, mlp_784_128_10, mlp_784_128_10_compressible, run_stream
    from .params import CkksParams
    if model not in ("mlp", "cnn", "mlp_compressible"):
        raise ValueError(f"model={model!r}")
    levels = 5 if model == "cnn" else 4
    ev = Evaluator(CkksParams.standard(13, levels, seed=seed + 7))
    ev.keygen()
    layers = {"mlp": mlp_784_128_10, "cnn": cnn_28x28, "mlp_compressible": mlp_784_128_10_compressible}[model](seed)
    # the compressible model runs on the integer pipe, whose layer time
    # shrinks with a gear's kept blocks (the tensor-core layer is dense)
    m = EncryptedMLP(ev, layers, tensor_cores=model != "mlp_compressible")
    rng = np.random.default_rng(seed + 1)
    data = [rng.uniform(0, 1, (batch, 784)) for _ in range(batches)]
    # warm-up: a full batch at every gear with every probe (kernels, weight
    # images, cached biases, allocator), so neither arm pays first-use costs
    for g in range(4):
        m.forward(data[0], lambda li, info, g=g: g)
    net = GearNet.load(net_path)
    # the arms alternate, twice each, with fresh controllers (so a warm or
    # cold GPU favours neither); the learned controller calibrates itself on
    # each stream's first batch (probes of every layer, timed, counted)
    runs = {"plain": [], "learned": []}
    for _ in range(2):
        runs["plain"].append(run_stream(m, PlainController(len(layers), target_db), data, fallback_db=target_db))
        runs["learned"].append(run_stream(m, LearnedController(m, net, target_db), data, fallback_db=target_db))

    def merged(rs):
        r = dict(rs[-1])
        r["seconds"] = sum(x["seconds"] for x in rs)
        r["samples"] = sum(x["samples"] for x in rs)
        r["samples_per_s"] = r["samples"] / r["seconds"]
        r["samples_per_s_runs"] = [x["samples_per_s"] for x in rs]
        return r
    rp, rl = merged(runs["plain"]), merged(runs["learned"])

    def hist(gears):
        h = np.zeros((len(layers), 4), dtype=int)
        for per_batch in gears:
            for li, g in enumerate(per_batch):
                h[li, g] += 1
        return h.tolist()
    drop = ("gears", "attempted_gears")
    return {"model": model, "target_db": target_db, "batch": batch, "batches": batches,
            "engine": "tensor cores" if m.tensor_cores else "integer pipe",
            "plain": {k: v for k, v in rp.items() if k not in drop}, "plain_gears": rp["gears"],
            "learned": {k: v for k, v in rl.items() if k not in drop}, "learned_gears": rl["gears"],
            "plain_gear_histogram": hist(rp["gears"]), "learned_gear_histogram": hist(rl["gears"]),
            "plain_attempted_histogram": hist(rp["attempted_gears"]),
            "learned_attempted_histogram": hist(rl["attempted_gears"]),
            "speedup": rl["samples_per_s"] / rp["samples_per_s"],
            "snr_gap_db": rl["snr_db"] - rp["snr_db"]}


def _init_distributed():
    """Under torchrun (WORLD_SIZE > 1): one process per GPU over NCCL."""
    import os
    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return False
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return True


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--traces", type=int, default=200_000)
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--out", default=str(DEFAULT_NET))
    c = sub.add_parser("compare")
    c.add_argument("--net", default=str(DEFAULT_NET))
    c.add_argument("--model", default="mlp", choices=["mlp", "cnn", "mlp_compressible"])
    c.add_argument("--batches", type=int, default=8)
    c.add_argument("--target-db", type=float, default=40.0)
    a = ap.parse_args(argv)
    distributed = _init_distributed() if a.cmd == "train" else False
    if a.cmd == "train":
        r = train(a.traces, a.epochs, Path(a.out))
    else:
        r = compare(Path(a.net), a.model, a.batches, target_db=a.target_db)
    from .dist import world
    if world()[1] == 0:
        print(json.dumps(r, default=float))
    if distributed:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
