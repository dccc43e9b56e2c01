"""Learned warm start end to end: solver-generated training data, surrogate training, and the cold vs warm
comparison on held-out designs.

    python -m xadvcool_b200.warmstart --train 2000 --heldout 256 --out warmstart.json

Designs are the seeded 148x128x32 gyroid cold plates (designs.gyroid_design); training seeds are 0..n_train-1,
held-out seeds start at HELDOUT_SEED0 so the two sets are disjoint. Training data are the fields of cold FP32
solves to the residual tolerance (batched persistent solver), kept resident on the GPU. The comparison times
each held-out design from mask upload to the scalars (delta_P, R_th), cold-started vs initialised from the
surrogate's prediction, and reports the relative error of the prediction against the converged fields.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import designs
from . import surrogate as S
from .batch import Batch
from .lattice import Lattice

TAU, POWER, T_IN = 0.55, 0.1, 25.0
HELDOUT_SEED0 = 1_000_000
SCALAR_KEYS = ("delta_P", "R_th")


def _sync():
    torch.cuda.synchronize()


def design(seed):
    return designs.gyroid_design(seed)


def _spec(mask, hs, u_in):
    return dict(mask=mask, heat_source=hs, tau_fluid=TAU, heat_power=POWER, t_inlet=T_IN, u_inlet_val=u_in)


# ------------------------------------------------------------------------------------------------ data
def generate(seeds, *, max_steps=30000, tol=1e-6, batch_size=64, log=print):
    """Cold batched solves of the given seeds -> (features [n,z,y,x,3] bf16, targets [n,z,y,x,5] fp32, info).

    Designs whose cold solve trips the divergence guard (max|u| > 0.17 or T > 1e4, src/simulation.py:146-153;
    at tau 0.55 most designs with u_in above about 0.045 do so in the impulsive start) give no target and are
    left out; ``info`` lists every seed with its outcome."""
    feats, tgts, info = [], [], []
    for b0 in range(0, len(seeds), batch_size):
        chunk = seeds[b0:b0 + batch_size]
        ds = [design(s) for s in chunk]
        b = Batch([_spec(m, h, u) for m, h, u, _ in ds])
        res = b.run(max_steps=max_steps, tol_ke=tol, tol_T=tol)
        for i, (m, h, u, _) in enumerate(ds):
            info.append({"seed": chunk[i], "u_in": u, "steps": res[i]["steps"], "converged": res[i]["converged"],
                         "diverged": res[i]["diverged"]})
            if res[i]["diverged"]:
                continue
            rho, uu, T = b.lattice(i).fields()
            feats.append(S.features(m, h, u)[..., :S.IN_FEATURES].clone())
            tgts.append(S.targets(rho, uu, T, u, POWER, T_IN))
        b.close()
        if log:
            nconv = sum(r["converged"] for r in res)
            log(f"generated {b0 + len(chunk)}/{len(seeds)} (batch converged {nconv}/{len(chunk)})")
    return torch.cat(feats, 0), torch.cat(tgts, 0), info


def _allreduce_(t):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return t


def _world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def gather_designs(feats, tgts):
    """Every rank's generated designs to every rank, in rank order (one all-gather of each tensor, padded to the
    largest shard; the counts are gathered first)."""
    import torch.distributed as dist
    rank, world = _world()
    if world == 1:
        return feats, tgts
    n = torch.tensor([feats.shape[0]], device=feats.device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c) for c in counts]
    m = max(counts)
    out = []
    for t in (feats, tgts):
        pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        pad[:t.shape[0]] = t
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad)
        out.append(torch.cat([p[:c] for p, c in zip(parts, counts)], 0))
    return out[0], out[1]


def train_surrogate(feats, tgts, *, epochs=30, batch=4, lr=5e-4, clip=1.0, val_frac=0.05, seed=0, log=print,
                    device="cuda", conv=None, micro=1):
    """Trains the surrogate on resident data (features expanded to 16 channels per mini-batch): AdamW, one-cycle
    schedule, MSE on per-channel normalised targets, gradient-norm clipping. The last ``val_frac`` of the designs
    are held back to report a validation loss per epoch.

    Data parallel when torch.distributed is initialised: every rank holds the same design list, takes the
    rank-th slice of each global mini-batch of ``batch`` designs (``batch`` divisible by the world size), and the
    gradients are averaged by ONE all-reduce per step over a flat buffer (NCCL on GPUs). Normalisation
    statistics and the shuffling are the same on every rank, so all ranks keep identical weights.

    ``micro`` > 1 splits each rank's share into that many micro-batches with gradient accumulation (less memory
    per step). The step's gradient is the sum over all world x micro slices divided by their count, so one process
    with micro = k reproduces k ranks with micro = 1 bit for bit."""
    rank, world = _world()
    if batch % (world * micro):
        raise ValueError(f"batch {batch} is not divisible by world size x micro-batches ({world} x {micro})")
    model = S.Surrogate(device, seed=seed)
    n_all = feats.shape[0]
    n_val = int(round(val_frac * n_all)) if n_all > 20 else 0
    n = n_all - n_val
    mean = tgts[:n].mean(dim=(0, 1, 2, 3))
    std = tgts[:n].std(dim=(0, 1, 2, 3)).clamp_min(1e-6)
    model.norm = (mean, std)
    params = model.parameters()
    opt = torch.optim.AdamW(params, lr=lr, weight_decay=1e-4)
    steps = epochs * math.ceil(n / batch)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=steps, pct_start=0.1)
    g = torch.Generator().manual_seed(seed)
    per = batch // world
    sl = batch // (world * micro)  # designs per slice
    flat = torch.zeros(sum(p.numel() for p in params), device=device)

    def inputs(idx):
        x = torch.zeros((len(idx),) + tuple(feats.shape[1:4]) + (16,), dtype=S.BF16, device=device)
        x[..., :S.IN_FEATURES] = feats[idx]
        return x

    hist = []
    for ep in range(epochs):
        order = torch.randperm(n, generator=g)
        tot = torch.zeros((), device=device)
        for i in range(0, n, batch):
            gidx = order[i:i + batch]
            opt.zero_grad(set_to_none=True)
            for m in range(micro):
                idx = gidx[(rank * micro + m) * sl:(rank * micro + m + 1) * sl].to(device)
                if not len(idx):
                    continue
                y = (tgts[idx] - mean) / std
                loss = torch.nn.functional.mse_loss(model.forward(inputs(idx), conv)[..., :S.OUT_FIELDS], y)
                # slice weight: the step's gradient is the mean over its designs (a short last batch included)
                k = len(idx) * world * micro / len(gidx)
                (loss * k if k != 1.0 else loss).backward()
                tot += loss.detach() * len(idx)
            if world > 1:
                # one all-reduce of every gradient per step
                off = 0
                for p in params:
                    k = p.numel()
                    flat[off:off + k] = p.grad.reshape(-1) if p.grad is not None else 0.0
                    off += k
                _allreduce_(flat)
                off = 0
                for p in params:
                    k = p.numel()
                    p.grad = flat[off:off + k].view_as(p).clone()
                    off += k
            if world * micro > 1:
                for p in params:
                    if p.grad is not None:
                        p.grad /= world * micro
            torch.nn.utils.clip_grad_norm_(params, clip)
            opt.step()
            sched.step()
        _allreduce_(tot)
        rec = {"epoch": ep, "mse": float(tot) / n}
        if n_val and rank == 0:
            with torch.no_grad():
                vt = torch.zeros((), device=device)
                for i in range(n, n_all, batch):
                    idx = torch.arange(i, min(i + batch, n_all), device=device)
                    y = (tgts[idx] - mean) / std
                    vt += torch.nn.functional.mse_loss(model.forward(inputs(idx), conv)[..., :S.OUT_FIELDS], y,
                                                       reduction="none").mean(dim=(1, 2, 3, 4)).sum()
                rec["val_mse"] = float(vt) / n_val
        hist.append(rec)
        if log and rank == 0:
            log(json.dumps(rec))
    return model, hist


# ------------------------------------------------------------------------------------------------ comparison
def _rel_err(a, b):
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def _rel(a, b):
    return abs(a - b) / abs(b)


def solve_solo(mask, hs, u_in, *, model=None, max_steps=150000, tol=1e-6, warm_min_steps=1000):
    """Mask upload -> (optional surrogate warm start) -> solve -> scalars, with the time of each phase; returns
    the record, the lattice and the prediction."""
    _sync()
    t0 = time.perf_counter()
    lat = Lattice(mask, tau_fluid=TAU, heat_power=POWER, t_inlet=T_IN, u_inlet_val=u_in, heat_source=hs)
    _sync()
    t1 = time.perf_counter()
    pred = None
    if model is not None:
        pred = S.predict(model, mask, hs, u_in, POWER)
        lat.init_fields(*pred)
    _sync()
    t2 = time.perf_counter()
    r = lat.run(max_steps=max_steps, tol_ke=tol, tol_T=tol, min_steps=warm_min_steps if model is not None else 0)
    t3 = time.perf_counter()
    sc = lat.scalars()
    _sync()
    t4 = time.perf_counter()
    rec = {"s": t4 - t0, "s_create": t1 - t0, "s_predict": t2 - t1, "s_run": t3 - t2, "s_scalars": t4 - t3,
           "steps": r["steps"], "converged": r["converged"], "diverged": r["diverged"],
           **{k: sc[k] for k in SCALAR_KEYS}}
    return rec, lat, pred


def compare(model, seeds, *, max_steps=150000, tol=1e-6, warm_min_steps=1000, tight_tol=1e-8, log=print):
    """Per held-out design: the cold and the warm solo solves (timed), then, untimed, the cold lattice continued
    to ``tight_tol`` as the steady-state reference; scalar agreement and the surrogate's field error against it."""
    rows = []
    for s in seeds:
        m, h, u, _ = design(s)
        cold, lat_c, _ = solve_solo(m, h, u, max_steps=max_steps, tol=tol)
        warm, lat_w, pred = solve_solo(m, h, u, model=model, max_steps=max_steps, tol=tol,
                                       warm_min_steps=warm_min_steps)
        lat_w.close()
        row = {"seed": s, "u_in": u, "cold": cold, "warm": warm}
        if not cold["diverged"]:
            rt = lat_c.run(max_steps=max_steps, tol_ke=tight_tol, tol_T=tight_tol, min_steps=200)
            sc = lat_c.scalars()
            tight = {"steps": cold["steps"] + rt["steps"], "converged": rt["converged"],
                     **{k: sc[k] for k in SCALAR_KEYS}}
            rho_c, u_c, T_c = lat_c.fields()
            fluid = torch.from_numpy(np.asarray(m) != 1).cuda()
            row.update(tight=tight, cold_vs_tight={k: _rel(cold[k], tight[k]) for k in SCALAR_KEYS},
                       warm_vs_cold={k: _rel(warm[k], cold[k]) for k in SCALAR_KEYS},
                       warm_vs_tight={k: _rel(warm[k], tight[k]) for k in SCALAR_KEYS},
                       pred_err={"u": _rel_err(pred[1][fluid], u_c[fluid]),
                                 "p": _rel_err(pred[0][fluid] - 1, rho_c[fluid] - 1),
                                 "T": _rel_err(pred[2] - T_IN, T_c - T_IN)},
                       speedup=cold["s"] / warm["s"])
        lat_c.close()
        rows.append(row)
        if log:
            log(json.dumps(row))
    return rows


def _batched(ds, model, *, max_steps, tol, warm_min_steps):
    """One batch of designs, cold (model None) or warm: wall seconds from mask upload to every design's scalars."""
    _sync()
    t0 = time.perf_counter()
    b = Batch([_spec(m, h, u) for m, h, u, _ in ds])
    if model is not None:
        for i, (m, h, u, _) in enumerate(ds):
            b.lattice(i).init_fields(*S.predict(model, m, h, u, POWER))
    res = b.run(max_steps=max_steps, tol_ke=tol, tol_T=tol, min_steps=warm_min_steps if model is not None else 0)
    sc = [b.lattice(i).scalars() for i in range(len(ds))]
    _sync()
    wall = time.perf_counter() - t0
    b.close()
    nconv = sum(r["converged"] for r in res)
    return {"wall_s": wall, "designs": len(ds), "converged": nconv, "s_per_converged_design": wall / max(nconv, 1),
            "diverged": sum(r["diverged"] for r in res), "steps": [r["steps"] for r in res],
            "ok": [bool(r["converged"]) for r in res], "scalars": [{k: s[k] for k in SCALAR_KEYS} for s in sc]}


def screen(seeds, steps=500):
    """Seeds whose cold start passes the divergence guard over its first ``steps`` steps (the impulsive start
    trips it at the first check, step 100, when it trips at all)."""
    ds = [design(s) for s in seeds]
    b = Batch([_spec(m, h, u) for m, h, u, _ in ds])
    res = b.run(max_steps=steps, tol_ke=0.0, tol_T=0.0)
    b.close()
    return [s for s, r in zip(seeds, res) if not r["diverged"]], [s for s, r in zip(seeds, res) if r["diverged"]]


def _vs(a, ref, ok_a, ok_ref):
    """Relative delta_P / R_th differences of batch ``a`` against batch ``ref`` over designs converged in both."""
    both = [j for j in range(len(ok_a)) if ok_a[j] and ok_ref[j]]
    dp = [_rel(a["scalars"][j]["delta_P"], ref["scalars"][j]["delta_P"]) for j in both]
    rt = [_rel(a["scalars"][j]["R_th"], ref["scalars"][j]["R_th"]) for j in both]
    return {"compared": len(both), "dP_rel_max": max(dp) if dp else None, "Rth_rel_max": max(rt) if rt else None,
            "Rth_rel_median": float(np.median(rt)) if rt else None,
            "within_half_percent": sum(1 for x, y in zip(dp, rt) if x <= 5e-3 and y <= 5e-3)}


def compare_batched(model, seeds, *, max_steps=150000, tol=1e-6, warm_min_steps=1000, tight_tol=None,
                    solve_cold_tripped=True):
    """Batched solves of the held-out designs whose cold start passes the divergence guard, cold and warm (same
    designs, same residual): wall seconds per converged design from mask upload to scalars, steps, and the
    scalar agreement per design. The designs whose cold start trips the guard are then solved warm, to count
    those the warm start solves. With ``tight_tol`` the same designs are also solved cold to that residual, and
    both the cold and the warm scalars are compared with those of the tight solve (``vs_tight``). ``per_design``
    lists, for every design that passes the guard, its seed, cold and warm steps, and the relative delta_P / R_th
    differences (warm vs cold; each vs the tight solve when there is one; None where a solve did not converge)."""
    good, bad = screen(seeds)
    out = {"screened_out": len(bad)}
    dg = [design(s) for s in good]
    out["cold"] = _batched(dg, None, max_steps=max_steps, tol=tol, warm_min_steps=warm_min_steps)
    out["warm"] = w = _batched(dg, model, max_steps=max_steps, tol=tol, warm_min_steps=warm_min_steps)
    c = out["cold"]
    both = [j for j in range(len(dg)) if w["ok"][j] and c["ok"][j]]
    dp = [_rel(w["scalars"][j]["delta_P"], c["scalars"][j]["delta_P"]) for j in both]
    rt = [_rel(w["scalars"][j]["R_th"], c["scalars"][j]["R_th"]) for j in both]
    out.update(compared=len(both), dP_rel_max=max(dp) if dp else None, Rth_rel_max=max(rt) if rt else None,
               dP_rel_median=float(np.median(dp)) if dp else None, Rth_rel_median=float(np.median(rt)) if rt else None,
               within_half_percent=sum(1 for a, b in zip(dp, rt) if a <= 5e-3 and b <= 5e-3),
               step_ratio=sum(c["steps"]) / max(sum(w["steps"]), 1),
               speedup=c["s_per_converged_design"] / w["s_per_converged_design"])
    t = None
    if tight_tol is not None:
        t = _batched(dg, None, max_steps=max_steps, tol=tight_tol, warm_min_steps=warm_min_steps)
        out["vs_tight"] = {"tol": tight_tol, "tight_converged": t["converged"],
                           "cold": _vs(c, t, c["ok"], t["ok"]), "warm": _vs(w, t, w["ok"], t["ok"])}

    def rel(a, b, j, key):
        return _rel(a["scalars"][j][key], b["scalars"][j][key]) if a["ok"][j] and b["ok"][j] else None

    rows = []
    for j, s in enumerate(good):
        r = {"seed": s, "cold_steps": c["steps"][j], "warm_steps": w["steps"][j],
             "dP_warm_vs_cold": rel(w, c, j, "delta_P"), "Rth_warm_vs_cold": rel(w, c, j, "R_th")}
        if t is not None:
            r.update(Rth_cold_vs_tight=rel(c, t, j, "R_th"), Rth_warm_vs_tight=rel(w, t, j, "R_th"))
        rows.append(r)
    out["per_design"] = rows
    if bad and solve_cold_tripped:
        r = _batched([design(s) for s in bad], model, max_steps=max_steps, tol=tol, warm_min_steps=warm_min_steps)
        out["warm_cold_tripped"] = {k: r[k] for k in ("designs", "converged", "diverged", "steps", "wall_s")}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=256)
    ap.add_argument("--solo", type=int, default=16, help="held-out designs also compared one at a time")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--gen-max-steps", type=int, default=30000)
    ap.add_argument("--max-steps", type=int, default=150000)
    ap.add_argument("--tol", type=float, default=1e-6, help="residual tolerance of the training solves")
    ap.add_argument("--eval-tols", default="1e-6,1e-7", help="residual tolerances of the cold vs warm comparison")
    ap.add_argument("--warm-min-steps", type=int, default=1000)
    ap.add_argument("--save", default=None, help="write the trained weights here (torch.save)")
    ap.add_argument("--load", default=None, help="skip data generation and training; load these weights")
    ap.add_argument("--out", default="warmstart.json")
    ap.add_argument("--ddp", action="store_true",
                    help="under torchrun: shard data generation over the ranks, gather it, train data-parallel (NCCL)")
    a = ap.parse_args(argv)
    report = {"args": vars(a)}
    rank, world = 0, 1
    if a.ddp:
        import datetime
        import os
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(minutes=30))
        rank, world = _world()
    if a.load:
        model = S.Surrogate("cuda")
        model.load_state_dict(torch.load(a.load))
    else:
        t = time.perf_counter()
        feats, tgts, info = generate(list(range(a.train))[rank::world], max_steps=a.gen_max_steps, tol=a.tol,
                                     log=print if rank == 0 else None)
        feats, tgts = gather_designs(feats, tgts)
        report["gen_s"] = time.perf_counter() - t
        report["gen"] = info
        report["gen_converged"] = sum(i["converged"] for i in info)  # this rank's shard
        report["gen_kept"] = int(feats.shape[0])
        print(json.dumps({k: report[k] for k in ("gen_s", "gen_converged", "gen_kept")}), flush=True)
        t = time.perf_counter()
        model, hist = train_surrogate(feats, tgts, epochs=a.epochs, batch=a.batch, lr=a.lr)
        _sync()
        report["train_s"] = time.perf_counter() - t
        report["train_mse"] = hist
        del feats, tgts
        if a.save and rank == 0:
            torch.save(model.state_dict(), a.save)
    if rank != 0:  # the comparison runs on rank 0
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
        return
    held = [HELDOUT_SEED0 + i for i in range(a.heldout)]
    report["eval"] = {}
    for tol in [float(t) for t in a.eval_tols.split(",")]:
        rows = compare(model, held[:a.solo], max_steps=a.max_steps, tol=tol, warm_min_steps=a.warm_min_steps)
        bat = compare_batched(model, held, max_steps=a.max_steps, tol=tol, warm_min_steps=a.warm_min_steps)
        report["eval"][f"{tol:g}"] = {"solo": rows, "batched": bat}
        json.dump(report, open(a.out, "w"), indent=1)
        sp = [r["speedup"] for r in rows if "speedup" in r]
        print(json.dumps({"tol": tol, "designs": len(held), "screened_out": bat["screened_out"],
                          "solo_speedup_median": float(np.median(sp)) if sp else None,
                          "batched_speedup": bat["speedup"], "step_ratio": bat["step_ratio"],
                          "cold_s_per_design": bat["cold"]["s_per_converged_design"],
                          "warm_s_per_design": bat["warm"]["s_per_converged_design"],
                          "compared": bat["compared"], "within_half_percent": bat["within_half_percent"],
                          "dP_rel_max": bat["dP_rel_max"], "Rth_rel_max": bat["Rth_rel_max"],
                          "Rth_rel_median": bat["Rth_rel_median"],
                          "rescued": bat.get("warm_cold_tripped", {}).get("converged")}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
