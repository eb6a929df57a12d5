"""Training and use of the learned surrogate on trajectories the solver generates.

Workloads:
  * training data: the plain-solver scenario generator (synth.scenario0: sloping terrain with
    Gaussian bumps and a channel, left z inflow, right open, top/bottom closed, fixed dt 0.1 s)
    with fresh seeds, kSt ~ U[20, 45] and the inflow level raised by U[1, 4] m; every member is
    run by the batched ensemble solver and snapshotted every 60 simulated seconds;
  * training: pairs (state at t, state at t + 60 s) of those trajectories, AdamW, MSE on the
    scaled change of depth and discharges;
  * evaluation: held-out trajectories; one-call (60 s) error against persistence (the method
    without the network: the state does not change) and closed-loop rollouts;
  * screening: an ensemble rolled out by the surrogate to max-depth maps; the most flooded
    fraction and every member whose mass-balance residual trips the fallback are re-run by the
    batched solver; the result is judged against the batched solver on every member (max-depth
    RMSE, flooded-extent IoU at 5 cm, wall time).

    python -m fip_b200.surrogate_run [--members 64 --size 512 --hours 1 --steps 2400 --unroll 3 ...]

prints one JSON object with the measurements.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import Ensemble, synth
from .surrogate import Surrogate

CALL_S = 60.0
LEVEL_MARGIN = 0.25  # m above the inflow level that a surrogate water surface may reach
UMAX = 10.0          # m/s: |q| <= UMAX * h after each surrogate call
DT = 0.1
STEPS_PER_CALL = int(round(CALL_S / DT))


def _torch():
    import torch

    return torch


def config3_members(outdir: str, n: int, size: int, seed: int, duration: float):
    """Scenario generator of the surrogate workloads (see module docstring)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kst = float(rng.uniform(20.0, 45.0))
        lvl = float(rng.uniform(1.0, 4.0))
        out.append(synth.scenario0(outdir, W=size, H=size, duration=duration, save_every=0, dt=DT,
                                   seed=seed * 100003 + i, name=f"s{seed}_{i}", kst=kst, level_add=lvl))
    return out


class Batch:
    """Static inputs of a set of equally sized scenarios on the GPU."""

    def __init__(self, scenarios, device=0):
        torch = _torch()
        self.n = len(scenarios)
        self.H, self.W = scenarios[0].H, scenarios[0].W
        dev = torch.device("cuda", device)
        terr = np.stack([s.terrain for s in scenarios]).astype(np.float32)
        self.terrain = torch.from_numpy(terr).to(dev)
        kst = np.stack([np.full((self.H, self.W), float(s.info.get("kst", 30.0)), np.float32) for s in scenarios])
        self.kst = torch.from_numpy(kst).to(dev)
        self.zref = torch.from_numpy(terr.reshape(self.n, -1).mean(1).astype(np.float32)).to(dev)
        # left z condition: h fixed at both boundary columns, qx = 0 on the boundary face
        mask = np.zeros((self.n, self.H, self.W), np.uint8)
        hv = np.zeros((self.n, self.H, self.W), np.float32)
        for k, s in enumerate(scenarios):
            lo, hi = s.info["bc_rows"]
            for c in (0, 1):
                hv[k, lo:hi + 1, c] = np.maximum(0.0, np.float32(s.info["zbc"]) - s.terrain[lo:hi + 1, c])
                mask[k, lo:hi + 1, c] |= 1
            mask[k, lo:hi + 1, 0] |= 2
        self.pins = {"mask": torch.from_numpy(mask).to(dev), "h": torch.from_numpy(hv).to(dev),
                     "qx": torch.zeros_like(self.terrain), "qy": torch.zeros_like(self.terrain)}
        self.no_value = -9999.0
        self.cells = self.n * self.H * self.W
        # level bound of the rollouts: the inflow level of each member plus LEVEL_MARGIN
        self.zcap = torch.tensor([float(s.info["zbc"]) + LEVEL_MARGIN for s in scenarios], dtype=torch.float32,
                                 device=dev)

    # edge types of the generator's scenarios (left z is pinned; right open; top and bottom close)
    SIDES = (0, 2, 1, 1)

    def state(self, h, qx, qy):
        return {"h": h, "qx": qx, "qy": qy, "terrain": self.terrain, "kst": self.kst, "zref": self.zref,
                "no_value": self.no_value, "sides": self.SIDES}


def solver_trajectories(scenarios, n_calls: int, device=0):
    """Snapshots [n_calls + 1][members][H][W] of h, qx, qy every 60 s (batched solver) and the
    solver's max-depth maps at the end."""
    torch = _torch()
    paths = [s.yaml_path for s in scenarios]
    B, H, W = len(scenarios), scenarios[0].H, scenarios[0].W
    snaps = {k: torch.empty((n_calls + 1, B, H, W), dtype=torch.float32, device=torch.device("cuda", device))
             for k in ("h", "qx", "qy")}
    t0 = time.perf_counter()
    with Ensemble(paths, device=device) as e:
        for k in ("h", "qx", "qy"):
            e.gather(k, snaps[k][0])
        for c in range(n_calls):
            e.step(STEPS_PER_CALL)
            for k in ("h", "qx", "qy"):
                e.gather(k, snaps[k][c + 1])
        hmax = torch.empty((B, H, W), dtype=torch.float32, device=snaps["h"].device)
        e.gather("hmax", hmax)
    torch.cuda.synchronize()
    return snaps, hmax, time.perf_counter() - t0


def train(net: Surrogate, batch: Batch, snaps, steps: int, bs: int = 32, lr: float = 1e-3, seed: int = 0,
          log_every: int = 50, pushforward: float = 0.0, unroll: int = 1):
    """AdamW on (state at t, state at t + 60 s) pairs with a cosine learning rate. With
    pushforward p > 0, after the first quarter of the steps a fraction p of the steps start from
    the network's own state after k calls (k drawn from 1..unroll, no gradient through them) out
    of the solver's state at t - 60 k s, and learn the change to the solver's state at t + 60 s,
    so that the network learns to correct the errors it makes itself in closed-loop use."""
    torch = _torch()
    T = snaps["h"].shape[0] - 1
    B, H, W = batch.n, batch.H, batch.W
    dev = snaps["h"].device
    rng = np.random.default_rng(seed)
    tgt = torch.empty((bs, H, W, 3), dtype=torch.float32, device=dev)
    cur = {k: torch.empty((bs, H, W), dtype=torch.float32, device=dev) for k in ("h", "qx", "qy")}
    nxt = {k: torch.empty((bs, H, W), dtype=torch.float32, device=dev) for k in ("h", "qx", "qy")}
    terr = torch.empty((bs, H, W), dtype=torch.float32, device=dev)
    kst = torch.empty_like(terr)
    zref = torch.empty(bs, dtype=torch.float32, device=dev)
    pins = {k: torch.empty((bs, H, W), dtype=v.dtype, device=dev) for k, v in batch.pins.items()}
    log = []
    t0 = time.perf_counter()
    for it in range(steps):
        push = pushforward > 0 and it >= steps // 4 and rng.random() < pushforward and T >= 2
        k_un = int(rng.integers(1, min(unroll, T - 1) + 1)) if push else 0
        ti_np = rng.integers(k_un, T, bs)
        ti = torch.from_numpy(ti_np).to(dev)
        mi = torch.from_numpy(rng.integers(0, B, bs)).to(dev)
        terr.copy_(batch.terrain[mi])
        kst.copy_(batch.kst[mi])
        zref.copy_(batch.zref[mi])
        for k in ("h", "qx", "qy"):
            cur[k].copy_(snaps[k][ti - k_un, mi])
            nxt[k].copy_(snaps[k][ti + 1, mi])
        for k, v in batch.pins.items():
            pins[k].copy_(v[mi])
        st = {"h": cur["h"], "qx": cur["qx"], "qy": cur["qy"], "terrain": terr, "kst": kst, "zref": zref,
              "no_value": batch.no_value, "sides": batch.SIDES}
        net.pin(st, pins)  # the first snapshot precedes the iteration-0 boundary conditions
        for _ in range(k_un):  # the network's own state at t
            net.advance(st, pins)
        net.target(cur, nxt, terr, batch.no_value, tgt)
        net.pack(cur["h"], cur["qx"], cur["qy"], terr, kst, zref, batch.no_value, bs, H, W, train=True)
        net.forward(bs, H, W, train=True)
        net.loss_acc.zero_()
        net.loss(tgt, bs, H, W)
        net.backward(bs, H, W)
        a = lr * 0.5 * (1 + np.cos(np.pi * it / max(steps, 1)))  # cosine schedule
        net.update(lr=float(a))
        if it % log_every == 0 or it == steps - 1:
            log.append((it, float(net.loss_acc.item()) / tgt.numel()))
    net.check_device()
    return log, time.perf_counter() - t0


def _rmse(a, b, mask=None):
    d = (a - b) if mask is None else (a - b)[mask]
    return float(np.sqrt(np.mean(d.astype(np.float64) ** 2))) if d.size else 0.0


def _iou(a, b, thr=0.05):
    wa, wb = a > thr, b > thr
    u = np.logical_or(wa, wb).sum()
    return float(np.logical_and(wa, wb).sum() / u) if u else 1.0


def rollout_trace(net: Surrogate, batch: Batch, snaps, calls=(1, 2, 5, 10, 20, 40, 60)):
    """Depth RMSE and water volume (surrogate / solver) of a closed-loop run at the given calls."""
    torch = _torch()
    T = snaps["h"].shape[0] - 1
    st = {k: snaps[k][0].clone() for k in ("h", "qx", "qy")}
    state = batch.state(st["h"], st["qx"], st["qy"])
    net.pin(state, batch.pins)
    out = []
    for c in range(1, T + 1):
        net.advance(state, batch.pins)
        if c in calls:
            ref = snaps["h"][c].cpu().numpy().astype(np.float64)
            got = st["h"].cpu().numpy().astype(np.float64)
            out.append({"call": c, "rmse_depth_m": float(np.sqrt(np.mean((got - ref) ** 2))),
                        "volume_ratio": float(got.sum() / max(ref.sum(), 1e-9))})
    torch.cuda.synchronize()
    return out


def evaluate_one_call(net: Surrogate, batch: Batch, snaps):
    """60-s prediction error of the depth over all held-out pairs: network vs persistence."""
    torch = _torch()
    T = snaps["h"].shape[0] - 1
    se_net = se_pers = 0.0
    n = 0
    for t in range(T):
        st = {k: snaps[k][t].clone() for k in ("h", "qx", "qy")}
        s0 = batch.state(st["h"], st["qx"], st["qy"])
        net.pin(s0, batch.pins)
        pers = st["h"].cpu().numpy()  # persistence = the untrained network: pinned input unchanged
        net.advance(s0, batch.pins)
        ref = snaps["h"][t + 1].cpu().numpy()
        got = st["h"].cpu().numpy()
        se_net += float(np.sum((got.astype(np.float64) - ref) ** 2))
        se_pers += float(np.sum((pers.astype(np.float64) - ref) ** 2))
        n += ref.size
    torch.cuda.synchronize()
    return {"rmse_depth_net_m": float(np.sqrt(se_net / n)), "rmse_depth_persistence_m": float(np.sqrt(se_pers / n))}


def rollout(net: Surrogate, batch: Batch, n_calls: int, h0, qx0, qy0, residual_threshold: float = 1e-3):
    """Closed-loop surrogate run from (h0, qx0, qy0) over n_calls calls: final state, max-depth
    maps (over the 60-s states) and, per member, whether the fallback indicator tripped and its
    worst value. The water of these scenarios comes from a level condition, so no surface may
    rise above that level: after every call the depth above the member's inflow level plus
    LEVEL_MARGIN is removed (and |q| <= UMAX h), and the removed volume -- water the network made
    up -- relative to the member's water volume (inner cells, floor 1 cm over 1 % of them) is the
    mass residual that trips the fallback above `residual_threshold` (1e-3 of the patch volume)
    at any call. The network's consistency residual (fip_sg_consistency) and the mass balance
    against the edge discharges are reported beside it."""
    torch = _torch()
    st = {"h": h0.clone(), "qx": qx0.clone(), "qy": qy0.clone()}
    state = batch.state(st["h"], st["qx"], st["qy"])
    net.pin(state, batch.pins)  # the iteration-0 boundary conditions
    hmax = st["h"].clone()
    worst = np.zeros(batch.n)
    worst_cons = np.zeros(batch.n)
    worst_mass = np.zeros(batch.n)
    dx = 3.0
    h_host = st["h"].cpu().numpy()
    vol = h_host[:, 1:-1, 2:-1].astype(np.float64).sum(axis=(1, 2))
    floor = 0.01 * 0.01 * (batch.H - 2) * (batch.W - 3)
    resid = torch.zeros(batch.n, dtype=torch.float64, device=net.dev)
    excess = torch.zeros(batch.n, dtype=torch.float64, device=net.dev)
    for c in range(n_calls):
        f0 = net.edge_flux(st["qx"], st["qy"])
        resid.zero_()
        excess.zero_()
        dvol = net.advance(state, batch.pins, hmax, resid=resid, bound=(batch.zcap, excess, UMAX))
        f1 = net.edge_flux(st["qx"], st["qy"])
        dv, a, b, r, ex = (t.cpu().numpy() for t in (dvol, f0, f1, resid, excess))
        denom = np.maximum(vol + dv, floor)
        worst = np.maximum(worst, ex / denom)
        worst_cons = np.maximum(worst_cons, r / denom)
        worst_mass = np.maximum(worst_mass, np.abs(dv - CALL_S / dx * 0.5 * (a + b)) / denom)
        vol = vol + dv - ex  # the limiter's removal (mostly inner cells) leaves the patch
    torch.cuda.synchronize()
    tripped = worst > residual_threshold
    return st, hmax, tripped, worst, worst_mass, worst_cons


def screen(net: Surrogate, sc, hours: float, chunk: int = 32, top_frac: float = 0.1, threshold: float = 1e-3):
    """Surrogate-screened ensemble: every member rolled out by the surrogate (chunks of `chunk`
    members) to max-depth maps; the most flooded `top_frac` and every member whose fallback
    indicator tripped are re-run by the batched solver. Judged against the batched solver on
    every member: max-depth RMSE, flooded-extent IoU at 5 cm, wall times."""
    torch = _torch()
    n_sc = int(round(hours * 3600 / CALL_S))
    n = len(sc)
    H, W = sc[0].H, sc[0].W
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ref_hmax = torch.empty((n, H, W), dtype=torch.float32, device="cuda")
    with Ensemble([s.yaml_path for s in sc]) as e:
        e.step(n_sc * STEPS_PER_CALL)
        e.gather("hmax", ref_hmax)
    torch.cuda.synchronize()
    t_solver_all = time.perf_counter() - t0
    t0 = time.perf_counter()
    s_hmax = torch.empty_like(ref_hmax)
    tripped = np.zeros(n, bool)
    worst = np.zeros(n)
    worst_mass = np.zeros(n)
    worst_cons = np.zeros(n)
    for c0 in range(0, n, chunk):
        part = sc[c0:c0 + chunk]
        bsc = Batch(part)
        h0 = torch.zeros((bsc.n, H, W), dtype=torch.float32, device="cuda")
        q0 = torch.zeros_like(h0)
        _, hm, tr, wo, wm, wc = rollout(net, bsc, n_sc, h0, q0, q0.clone(), residual_threshold=threshold)
        s_hmax[c0:c0 + bsc.n].copy_(hm)
        tripped[c0:c0 + bsc.n], worst[c0:c0 + bsc.n], worst_mass[c0:c0 + bsc.n] = tr, wo, wm
        worst_cons[c0:c0 + bsc.n] = wc
        del bsc, hm
    t_surrogate = time.perf_counter() - t0
    area = (s_hmax.cpu().numpy() > 0.05).sum(axis=(1, 2))
    k = max(1, int(round(top_frac * n)))
    rerun = sorted(set(np.argsort(-area)[:k].tolist()) | set(np.nonzero(tripped)[0].tolist()))
    final = s_hmax.clone()
    t0 = time.perf_counter()
    if rerun:
        with Ensemble([sc[i].yaml_path for i in rerun]) as e:
            e.step(n_sc * STEPS_PER_CALL)
            rh = torch.empty((len(rerun), H, W), dtype=torch.float32, device="cuda")
            e.gather("hmax", rh)
        for j, i in enumerate(rerun):
            final[i].copy_(rh[j])
    torch.cuda.synchronize()
    t_rerun = time.perf_counter() - t0
    fin, ref, sur = final.cpu().numpy(), ref_hmax.cpu().numpy(), s_hmax.cpu().numpy()
    t_screen = t_surrogate + t_rerun
    err = np.sqrt(((sur - ref) ** 2).mean(axis=(1, 2)))
    # the same screen at other thresholds: a re-run member gives exactly the solver's map (the
    # solver is deterministic and the members independent), its cost taken as its share of the
    # all-member solver time
    sweep = []
    for thr in (1e-4, 1e-3, 1e-2, 1e-1):
        rr = set(np.argsort(-area)[:k].tolist()) | set(np.nonzero(worst > thr)[0].tolist())
        f2 = sur.copy()
        for i in rr:
            f2[i] = ref[i]
        t2 = t_surrogate + t_solver_all * len(rr) / n
        sweep.append({"threshold": thr, "rerun": len(rr), "tripped": int((worst > thr).sum()),
                      "rmse_hmax_m": _rmse(f2, ref), "iou_5cm": float(np.mean([_iou(f2[i], ref[i]) for i in range(n)])),
                      "est_wall_s": round(t2, 2), "est_speedup": round(t_solver_all / t2, 3)})
    return {"members": n, "size": [H, W], "hours": hours, "rerun": len(rerun), "top_fraction": top_frac,
            "fallback_tripped": int(tripped.sum()), "fallback_threshold": threshold,
            "indicator_median": float(np.median(worst)), "indicator_max": float(np.max(worst)),
            "mass_balance_residual_median": float(np.median(worst_mass)),
            "wall_s_screened": round(t_screen, 2), "wall_s_surrogate": round(t_surrogate, 2),
            "wall_s_rerun": round(t_rerun, 2), "wall_s_batched_solver_all": round(t_solver_all, 2),
            "speedup": round(t_solver_all / max(t_screen, 1e-9), 3),
            "rmse_hmax_m": _rmse(fin, ref), "iou_5cm": float(np.mean([_iou(fin[i], ref[i]) for i in range(n)])),
            "rmse_hmax_surrogate_only_m": _rmse(sur, ref),
            "iou_5cm_surrogate_only": float(np.mean([_iou(sur[i], ref[i]) for i in range(n)])),
            "indicator_vs_error_spearman": _spearman(worst, err),
            "consistency_residual_median": float(np.median(worst_cons)),
            "consistency_vs_error_spearman": _spearman(worst_cons, err),
            "hmax_rmse_per_member_m_quantiles": [float(np.quantile(err, q)) for q in (0.1, 0.5, 0.9)],
            "threshold_sweep": sweep}


def _spearman(a, b):
    ra, rb = np.argsort(np.argsort(a)), np.argsort(np.argsort(b))
    if np.std(ra) == 0 or np.std(rb) == 0:
        return 0.0
    return float(np.corrcoef(ra, rb)[0, 1])


def main(argv=None, emit: bool = True):
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=64, help="training trajectories")
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--hours", type=float, default=1.0, help="simulated length of each training trajectory")
    ap.add_argument("--steps", type=int, default=2400, help="training steps")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--pushforward", type=float, default=0.5)
    ap.add_argument("--unroll", type=int, default=3, help="pushforward: up to this many own calls")
    ap.add_argument("--eval-members", type=int, default=8)
    ap.add_argument("--screen-members", type=int, default=32)
    ap.add_argument("--screen-size", type=int, default=512)
    ap.add_argument("--screen-hours", type=float, default=1.0)
    ap.add_argument("--screen-chunk", type=int, default=32, help="members per surrogate rollout batch")
    ap.add_argument("--threshold", type=float, default=1e-3, help="fallback: consistency residual / patch volume")
    ap.add_argument("--params", default="", help="trained parameters (.npy): skip data generation and training")
    ap.add_argument("--no-eval", action="store_true", help="skip the held-out evaluation")
    ap.add_argument("--out", default="", help="write the trained parameters (.npy) here")
    a = ap.parse_args(argv)
    torch = _torch()
    d = tempfile.mkdtemp(prefix="fip_sg_")
    n_calls = int(round(a.hours * 3600 / CALL_S))
    res = {"config": vars(a)}
    if a.params:
        net = Surrogate(params=np.load(a.params))
        res["train"] = {"params": a.params}
    else:
        # ---- training data from the solver
        tr = config3_members(d, a.members, a.size, seed=1, duration=a.hours * 3600 + 600)
        btr = Batch(tr)
        snaps, _, t_gen = solver_trajectories(tr, n_calls)
        res["train_data"] = {"pairs": a.members * n_calls, "solver_s": round(t_gen, 2)}
        # ---- training
        net = Surrogate(seed=0)
        log, t_train = train(net, btr, snaps, a.steps, bs=a.batch, lr=a.lr, pushforward=a.pushforward,
                             unroll=a.unroll)
        res["train"] = {"loss_log": log, "seconds": round(t_train, 2), "steps": a.steps,
                        "ms_per_step": round(1e3 * t_train / max(a.steps, 1), 2)}
        del snaps, btr
        torch.cuda.empty_cache()
        if a.out:
            np.save(a.out, net.params())
    if not a.no_eval:
        # ---- held-out evaluation
        ev = config3_members(d, a.eval_members, a.size, seed=2, duration=a.hours * 3600 + 600)
        bev = Batch(ev)
        esn, ehmax, _ = solver_trajectories(ev, n_calls)
        res["eval_one_call"] = evaluate_one_call(net, bev, esn)
        res["eval_trace"] = rollout_trace(net, bev, esn)
        st, hm, tripped, worst, worst_mass, worst_cons = rollout(net, bev, n_calls, esn["h"][0], esn["qx"][0],
                                                                 esn["qy"][0], residual_threshold=a.threshold)
        ref_h = esn["h"][n_calls].cpu().numpy()
        got_h = st["h"].cpu().numpy()
        pers = esn["h"][0].cpu().numpy()
        ehm = ehmax.cpu().numpy()
        hmn = hm.cpu().numpy()
        err = np.sqrt(((hmn - ehm) ** 2).mean(axis=(1, 2)))
        res["eval_rollout"] = {"calls": n_calls, "rmse_final_depth_m": _rmse(got_h, ref_h),
                               "rmse_final_depth_persistence_m": _rmse(pers, ref_h),
                               "rmse_hmax_m": _rmse(hmn, ehm),
                               "iou_hmax_5cm": float(np.mean([_iou(hmn[i], ehm[i]) for i in range(bev.n)])),
                               "fallback_tripped": int(tripped.sum()), "indicator": worst.tolist(),
                               "hmax_rmse_per_member_m": err.tolist(),
                               "indicator_vs_error_spearman": _spearman(worst, err),
                               "consistency_residual": worst_cons.tolist(),
                               "mass_balance_residual": worst_mass.tolist()}
        del esn
        torch.cuda.empty_cache()
    # ---- screening
    sc = config3_members(d, a.screen_members, a.screen_size, seed=3, duration=a.screen_hours * 3600)
    res["screening"] = screen(net, sc, a.screen_hours, chunk=a.screen_chunk, threshold=a.threshold)
    if emit:
        print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
