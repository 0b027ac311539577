#!/usr/bin/env python
"""Throughput of the tsvdx4 timeSVD++ SGD epoch on B200.

One step = one training epoch (TxModel::fit_epoch, src/tx.rs:734-1115,
including the ycache rebuild) over the full synthetic Netflix-shaped
training set (480,189 users x 17,770 items, 100,480,507 ratings; seeded
stand-in for the real data, which is absent) at f=256 with the tsvdx4 `lm`
preset (src/bin/tsvdx4-new.rs:130-154) and 30 time bins.

  metric   SGD rating-updates/s (training ratings processed per second)
  value    device-timed (CUDA events on the launching stream) epochs with
           inputs resident in HBM; max over ranks
  e2e      the same metric through the C ABI from pinned host buffers:
           create() (H2D of both sets, setup, seeded init) plus per step
           fit_epoch + calc_rmse on the held-out set (H2D of the pr columns,
           D2H of the result)
  roofline the dominant kernel of the measured schedule (stratified: the item
           stratum, 8 f + 44 algorithmic bytes per rating; Hogwild: the user
           pass, 28 f + 64) over its CUDA-event duration, against the
           measured HBM copy peak

--impl reference runs the reference's CPU algorithm (the C++ restatement of
TxModel in oracle/, since the reference's Rust toolchain is absent) on a
bounded sample of the same workload and prints the same metric.
With --gpus N under torchrun the ranks train ONE model, sharded
(netflix_prize_b200/shard.py): user and item blocks per rank, the NSVD1
delta sums all-reduced and the blocks' rows all-gathered over NCCL; the job's
ratings per epoch stay fixed as N grows (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--f", type=int, default=256)
    ap.add_argument("--shape", choices=["c2", "c1", "c3"], default="c2")
    ap.add_argument("--schedule", choices=["hogwild", "stratified"], default="stratified")
    ap.add_argument("--precision", choices=["fp32", "bf16", "bf16all"], default="fp32",
                    help="BF16 read copies (stratified only): item and y tables, or also user rows")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ttr", action="store_true", help="skip the fold-in time-to-RMSE comparison")
    ap.add_argument("--sample-users", type=int, default=20000, help="users in the CPU sample")
    ap.add_argument("--no-train-ttr", action="store_true",
                    help="skip the training time to the reference's held-out RMSE")
    ap.add_argument("--batched", type=int, default=0, metavar="EPOCHS",
                    help="also time the 16 C3 variants trained together against one after another")
    return ap.parse_args()


def B_per_rating(f: int) -> int:
    """Algorithmic bytes per rating-update of the per-user pass, low_memory
    tx4 mode: q_i and q^f_i read+write (16 f), y_j gather (4 f) and
    read-modify-write (8 f), 64 bytes of stream and bias scalars."""
    return 28 * f + 64


def kernel_bytes_per_rating(kernel: str, f: int) -> int:
    """Algorithmic bytes per rating of the kernel the roofline is quoted on."""
    if kernel == "item_pass":
        # item stratum: the rating's two user rows, p_u + ycache_u (summed once
        # per user by the ycache rebuild) and p2_u (8 f), its 16-byte record and
        # 7 user-side bias scalars (28 B); item rows stay on chip per item
        return 8 * f + 44
    return B_per_rating(f)


def spec_for(shape: str):
    from netflix_prize_b200 import synth
    return {"c2": synth.spec_c2, "c1": synth.spec_c1, "c3": synth.spec_c3}[shape]()


def sample_spec(shape: str, users: int):
    from netflix_prize_b200 import synth
    s = spec_for(shape)
    n_train = int(round(s.n_train * users / s.n_users))
    out = synth.SynthSpec(users, s.n_items, n_train, s.zipf_s, s.median_cnt, s.max_cnt, None, s.max_heldout, None,
                          s.max_query, s.seed, s.rank, s.noise, f"{s.name}_sample")
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def traffic_record(kernel: str, workload: str):
    """DRAM bytes per launch from a committed ncu summary, when one exists."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    rec = d.get(f"{kernel}|{workload}")
    return None if rec is None else float(rec["dram_bytes_per_launch"])


class Clocks:
    """nvidia-smi sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm_sorted = sorted(sm)
        return {"sm_mhz": sm_sorted[len(sm_sorted) // 2], "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus:
        raise SystemExit(f"--gpus {n_gpus} but WORLD_SIZE={world}; launch with torchrun for N>1")
    return world, rank, local


def gpu_index_for(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def run_reference(args):
    """The reference's CPU algorithm (TxModel, sequential) on a bounded sample."""
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    from netflix_prize_b200 import synth
    from netflix_prize_b200.config import run_lm
    from netflix_prize_b200.data import MaskedDataset
    from oracle import pyoracle as po

    spec = sample_spec(args.shape, args.sample_users)
    tr, pr = synth.generate(spec)
    cfg = run_lm(args.f, args.warmup + args.steps, n_time_bins=30)
    m = po.OracleModel(tr, MaskedDataset(pr), cfg)
    for e in range(1, args.warmup + 1):
        m.fit_epoch(e)
    secs = m.time_epochs(args.warmup + 1, args.steps)
    value = tr.n_ratings * args.steps / secs
    sample = (f"{spec.n_users} users x {spec.n_items} items, {tr.n_ratings} ratings of the {args.shape} generator, "
              f"f={args.f}, one sequential TxModel epoch per step")
    line = {
        "impl": "reference", "metric": "SGD rating-updates/s", "value": value, "unit": "rating-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "rating-updates/s", "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "rating-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args, world: int = 1):
    spec = spec_for(args.shape)
    return {"workload": f"tsvdx4 lm preset, {args.shape} shape ({spec.n_users} users x {spec.n_items} items, "
                        f"{spec.n_train} ratings), f={args.f}, T=30, low_memory, schedule={args.schedule}, precision={args.precision}",
            "n_feat": args.f, "n_users": spec.n_users, "n_items": spec.n_items, "n_ratings": spec.n_train,
            "schedule": args.schedule, "precision": args.precision,
            "parallelism": "single GPU" if world == 1 else
            f"one model sharded over {world} GPUs (user and item blocks; NCCL all-reduce and all-gathers)",
            "l2": "inputs larger than L2 (16-byte rating records: 1.6 GB per epoch at the c2 shape)"}


def cpu_baseline(args):
    from netflix_prize_b200 import synth
    from netflix_prize_b200.config import run_lm
    from netflix_prize_b200.data import MaskedDataset
    from oracle import pyoracle as po

    spec = sample_spec(args.shape, args.sample_users)
    tr, pr = synth.generate(spec)
    cfg = run_lm(args.f, 2, n_time_bins=30)
    m = po.OracleModel(tr, MaskedDataset(pr), cfg)
    secs = m.time_epochs(1, 1)
    return {"value": tr.n_ratings / secs, "unit": "rating-updates/s", "cores": 1, "kind": "port",
            "sample": f"one sequential TxModel epoch (C++ restatement of src/tx.rs, -O2, 1 thread) over "
                      f"{spec.n_users} users x {spec.n_items} items, {tr.n_ratings} ratings of the "
                      f"{args.shape} generator, f={args.f}; host has {os.cpu_count()} cores"}


def time_to_rmse(model, tr, pr):
    """Time to a held-out RMSE target for new users (the C5 fold-in): the
    plain form (standard init + user-side SGD passes with item tables frozen)
    against the chosen form (encoder init + passes). The model's other
    480,189 - 80,189 users (same proportion at other shapes) train the
    encoder for 10 epochs; the 80,189 are reset and folded in. Target =
    plain RMSE after 8 passes + 0.001. Times are host wall clock around the
    synchronous C ABI calls."""
    import numpy as np
    from netflix_prize_b200.data import Dataset
    from netflix_prize_b200.encoder import UserEncoder, foldin, reset_users

    U = tr.n_users
    n_new = max(1, U - int(round(U * 400000 / 480189)))
    perm = np.random.default_rng(0).permutation(U).astype(np.uint32)
    new, old = np.sort(perm[:n_new]), perm[n_new:]
    keep = np.isin(pr.user_idxs, new) & (pr.is_test == 0)
    held = Dataset.from_ratings(pr.user_idxs[keep], pr.item_idxs[keep], pr.raw_ratings[keep], pr.dates[keep],
                                pr.n_users, pr.n_items, "held_new_users")
    model.synchronize()
    t0 = time.perf_counter()
    enc = UserEncoder(model, tr.raw_ratings, old, seed=5, lr=2e-3)
    losses = [enc.train_epoch(old, batch=1024) for _ in range(10)]
    model.synchronize()
    enc_s = time.perf_counter() - t0

    def run(k, warm):
        reset_users(model, new, 99)
        model.synchronize()
        t = time.perf_counter()
        if warm:
            enc.apply(model, new)
        if k:
            foldin(model, new, k)
        model.synchronize()
        return (time.perf_counter() - t) * 1000.0, model.calc_rmse(held)

    plain = [(k,) + run(k, False) for k in range(0, 9)]
    target = plain[-1][2] + 0.001
    warm = []
    for k in range(0, 5):
        warm.append((k,) + run(k, True))
        if warm[-1][2] <= target:
            break
    first = lambda rows: next((r for r in rows if r[2] <= target), None)
    p, w = first(plain), first(warm)
    enc.close()
    return {"scenario": f"fold-in of {n_new} held-out users of the trained model, item tables frozen",
            "target_rmse": target, "target_rule": "plain RMSE after 8 passes + 0.001",
            "plain": {"passes": p[0], "ms": p[1], "rmse": p[2]} if p else None,
            "chosen": {"form": "encoder init + fold-in passes", "passes": w[0], "ms": w[1], "rmse": w[2]}
            if w else None,
            "chosen_over_plain_time": (w[1] / p[1]) if (p and w and p[1] > 0) else None,
            "chosen_with_encoder_training_ms": (enc_s * 1000.0 + w[1]) if w else None,
            "chosen_with_encoder_training_over_plain_time": ((enc_s * 1000.0 + w[1]) / p[1])
            if (p and w and p[1] > 0) else None,
            "fold_in_batches_for_half_the_plain_time":
            (enc_s * 1000.0 / (0.5 * p[1] - w[1])) if (p and w and 0.5 * p[1] > w[1]) else None,
            "encoder_train_s": enc_s, "encoder_loss_first_last": [losses[0], losses[-1]],
            "plain_curve": [[k, round(ms, 3), r] for k, ms, r in plain],
            "chosen_curve": [[k, round(ms, 3), r] for k, ms, r in warm]}


def train_to_reference_rmse(tr, pr, cfg, device: int, shape: str):
    """Wall time of the plain GPU form to reach the reference's held-out RMSE
    (the best epoch of the oracle's sequential TxModel curve committed under
    tests/golden, + 0.001) from the standard init, epoch by epoch with the
    stratified schedule. Host wall clock around the synchronous calls; the
    per-epoch RMSE evaluations are timed apart."""
    path = os.path.join(ROOT, "tests", "golden", f"rmse_curve_{shape}_f{cfg.n_feat}.json")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        ref = json.load(fh)
    eps = ref["epochs"]
    best = min(eps, key=lambda r: r["heldout_rmse"])
    target = best["heldout_rmse"] + 0.001
    from netflix_prize_b200.data import MaskedDataset
    from netflix_prize_b200.model import TxModel
    m = TxModel(tr, MaskedDataset(pr), cfg.replace(n_epochs=len(eps)), device=device)
    train_ms = eval_ms = 0.0
    curve = []
    for e in range(1, len(eps) + 1):
        t = time.perf_counter()
        m.fit_epoch(tr, pr, e)
        m.synchronize()
        train_ms += (time.perf_counter() - t) * 1000.0
        t = time.perf_counter()
        r = m.calc_rmse(pr)
        eval_ms += (time.perf_counter() - t) * 1000.0
        curve.append([e, r, eps[e - 1]["heldout_rmse"]])
        if r <= target:
            break
    m.close()
    reached = curve[-1][1] <= target
    return {"target_rmse": target, "target_rule": "reference best held-out RMSE + 0.001",
            "reference": {"best_epoch": best["epoch"], "best_rmse": best["heldout_rmse"],
                          "epochs_in_curve": len(eps), "algorithm": ref["algorithm"]},
            "plain": {"reached": reached, "epochs": curve[-1][0], "train_ms": train_ms, "eval_ms": eval_ms},
            "curve_gpu_vs_reference": curve}


def c3_variants(base):
    """The batched configuration: f in {32, 64, 128, 256} x lr in {0.003,
    0.007} x reg in {0.005, 0.015}; lr sets lr_u and lr_i, reg sets reg_u and
    reg_i."""
    out = []
    for f in (32, 64, 128, 256):
        for lr in (0.003, 0.007):
            for reg in (0.005, 0.015):
                out.append(base.replace(n_feat=f, lr_u=lr, lr_i=lr, reg_u=reg, reg_i=reg))
    return out


def batched_leg(tr, pr, base_cfg, device: int, epochs: int):
    """The 16 C3 variants trained together (one graph per epoch, the
    autotuned whole-CTA thresholds) against the same variants trained one
    after another (CUDA events around each variant's epochs)."""
    import torch
    from netflix_prize_b200.data import MaskedDataset
    from netflix_prize_b200.model import TxGroup, TxModel
    cfgs = c3_variants(base_cfg.replace(n_epochs=epochs + 1))
    g = TxGroup(tr, MaskedDataset(pr), cfgs, device=device)
    thr = [int(x) for x in g.autotune()]
    g.fit_epoch(1)  # uncaptured first epoch
    group_ms = 0.0
    for e in range(2, epochs + 2):
        g.fit_epoch(e)
        group_ms += g.last_epoch_ms()
    rmse_group = [m.calc_rmse(pr) for m in g.models]
    g.close()
    sep_ms = 0.0
    for k, c in enumerate(cfgs):
        m = TxModel(tr, MaskedDataset(pr), c, device=device, heavy_item_ratings=min(thr[k], 2**31 - 1))
        m.fit_epoch(tr, pr, 1)
        m.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = torch.cuda.current_stream()
        m.set_stream(s.cuda_stream)
        e0.record(s)
        for e in range(2, epochs + 2):
            m.fit_epoch(tr, pr, e)
        e1.record(s)
        torch.cuda.synchronize()
        sep_ms += e0.elapsed_time(e1)
        m.close()
    R = tr.n_ratings
    return {"variants": len(cfgs), "epochs_timed": epochs, "group_ms_per_epoch": group_ms / epochs,
            "separate_ms_per_epoch": sep_ms / epochs, "speedup": sep_ms / group_ms,
            "group_rating_updates_per_s": R * len(cfgs) * epochs / (group_ms / 1000.0),
            "whole_cta_thresholds": thr, "heldout_rmse_group": rmse_group}


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from netflix_prize_b200 import synth
    from netflix_prize_b200.abi import SCHED_HOGWILD, SCHED_STRATIFIED
    from netflix_prize_b200.config import run_lm
    from netflix_prize_b200.data import MaskedDataset
    from netflix_prize_b200.model import TxModel

    sched = SCHED_HOGWILD if args.schedule == "hogwild" else SCHED_STRATIFIED
    prec = {"fp32": 0, "bf16": 1, "bf16all": 2}[args.precision]
    spec = spec_for(args.shape)
    tr, pr = synth.generate(spec)
    R = tr.n_ratings
    cfg = run_lm(args.f, args.warmup + args.steps, n_time_bins=30)

    from netflix_prize_b200 import dist

    def barrier():
        dist.barrier(world)

    def max_over_ranks(x: float) -> float:
        return dist.max_over_ranks(x, world)

    stream = torch.cuda.current_stream()

    def stepper(m):
        """One epoch of the job: the model's own epoch, or this rank's share
        of a sharded epoch."""
        if world == 1:
            return lambda e: m.fit_epoch(tr, pr, e)
        from netflix_prize_b200.shard import GpuEngine, Partition, ShardedEpochs, TorchComm
        sh = ShardedEpochs(GpuEngine(m), rank, Partition.for_data(tr, world), TorchComm(world, rank))
        return sh.fit_epoch

    # ---------------- value: device-resident epochs ----------------
    model = TxModel(tr, MaskedDataset(pr), cfg, schedule=sched, precision=prec, device=local)
    model.set_stream(stream.cuda_stream)
    step = stepper(model)
    for e in range(1, args.warmup + 1):
        step(e)
    barrier()
    model.reset_kernel_stats()
    model.set_profiling(True)
    clocks = Clocks(gpu_index_for(local))
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for k in range(args.steps):
        step(args.warmup + 1 + k)
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches = model.launch_count()
    kname = "user_pass_hogwild" if sched == SCHED_HOGWILD else "item_pass"
    kstats = {}
    for kn in ("user_pass_hogwild", "user_pass_stratified", "y_apply", "rebuild_ycache", "item_pass"):
        n, t = model.kernel_stats(kn)
        if n:
            kstats[kn] = {"launches": n, "avg_ms": t / n}
    model.set_profiling(False)
    rmse = model.calc_rmse(pr)
    value = R * args.steps / (ms / 1000.0)  # the job's ratings, whatever the number of ranks
    peak, peak_kind = measured_peaks()
    dom = kstats.get(kname, {"avg_ms": float("nan")})
    bpr = kernel_bytes_per_rating(kname, args.f)
    achieved = bpr * R / (dom["avg_ms"] / 1000.0) / 1e9
    workload = f"{args.shape}_f{args.f}_{args.schedule}"
    traffic = traffic_record(kname, workload)
    ttr = None
    if world == 1 and not args.no_ttr:
        ttr = time_to_rmse(model, tr, pr)
    del model
    train_ttr = None
    if world == 1 and not args.no_train_ttr:
        train_ttr = train_to_reference_rmse(tr, pr, cfg, local, args.shape)
    batched = None
    if world == 1 and args.batched > 0:
        batched = batched_leg(tr, pr, cfg, local, args.batched)

    # ---------------- e2e: through the C ABI from pinned host buffers ----------------
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.shape, dtype={np.int32: torch.int32, np.int16: torch.int16, np.int8: torch.int8,
                                            np.float32: torch.float32}[a.dtype.type], pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()

        import copy
        trp, prp = copy.copy(tr), copy.copy(pr)
        for d in (trp, prp):
            for f in ("user_idxs", "user_cnts", "item_idxs", "item_cnts", "raw_ratings", "residuals", "dates",
                      "is_test"):
                setattr(d, f, pinned(getattr(d, f)))
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m2 = TxModel(trp, MaskedDataset(prp), cfg, schedule=sched, precision=prec, device=local)
        m2.set_stream(stream.cuda_stream)
        step2 = stepper(m2)
        e2e_rmse = None
        for k in range(args.steps):
            step2(k + 1)
            e2e_rmse = m2.calc_rmse(prp)
        e1.record(stream)
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        tr_bytes = sum(getattr(trp, f).nbytes for f in ("user_idxs", "item_idxs", "residuals", "dates", "user_cnts"))
        pr_bytes = sum(getattr(prp, f).nbytes for f in ("user_idxs", "item_idxs", "dates", "user_cnts"))
        rmse_bytes = sum(getattr(prp, f).nbytes for f in ("user_idxs", "item_idxs", "dates", "residuals", "is_test"))
        del m2
        e2e = {"value": R * args.steps / (e2e_ms / 1000.0), "unit": "rating-updates/s",
               "h2d_bytes_per_step": int((tr_bytes + pr_bytes) / args.steps + rmse_bytes),
               "d2h_bytes_per_step": 16, "ms_total": e2e_ms,
               "includes": "create (H2D of train+pr, setup, seeded init) amortised over the steps; per step "
                           "fit_epoch + calc_rmse(held-out) with H2D of the pr columns and D2H of the SSE",
               "heldout_rmse": e2e_rmse}

    line = {
        "metric": "SGD rating-updates/s", "value": value, "unit": "rating-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                     "peak_source": f"{peak_kind} hbm_gbs", "bytes_per_rating": bpr},
        "kernels": kstats,
        "heldout_rmse_after_run": rmse,
        "clocks": clk,
        "gpu_launches": launches,
        "e2e": e2e,
        "time_to_rmse": ttr,
        "time_to_reference_rmse": train_ttr,
        "batched": batched,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
