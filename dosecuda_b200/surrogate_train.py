"""Train and evaluate the photon-dose surrogate.

    python -m dosecuda_b200.surrogate_train --train 3000 --test 300 --epochs 50 \\
        --out surrogate_6mv.npz --report surrogate_report.json

Training data are phantoms of the surrogate workload (128^3 at 2.5 mm: a
water body ellipsoid with 1-5 random ellipsoids of HU uniform in [-900,
1500]; one 6 MV beam at a gantry angle in 5 degree steps; a square or
rectangular MLC field of 2-20 cm per side; 100 MU), whose TERMA, density and
CCCS dose this engine computes itself (``SampleMaker``).  Seeds 0..N-1 train,
seeds 1000000+i test.  Training uses the hand-written kernels (forward,
backward) with Adam on the fp32 master weights, one phantom per step.

The evaluation runs ``PhotonSurrogate`` on every test phantom (TERMA ->
network -> sparse CCCS probe -> probe gamma -> accept or full CCCS) and
checks every output against the full CCCS dose with gamma(2 %/2 mm, 10 %
cutoff, global max of the CCCS dose).  It reports the acceptance rate, the
gamma pass rates (vs CCCS) of accepted beams, the time per beam of the surrogate path
(fallbacks included) and of the CCCS path, and the same acceptance for the
untrained network (what training gains over the method without it).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np
import torch

from . import engine
from .surrogate import Dataset, PhotonSurrogate, SampleMaker, SurrogateNet, load_training_state, train

TEST_SEED0 = 1_000_000


def choose_scales(maker: SampleMaker, seeds):
    """terma_scale and dose_unit that bring the 99th percentile of the active
    voxels' TERMA and normalised dose to about 1."""
    ts, ds = [], []
    for s in seeds:
        density, terma, dose, cp = maker.make(s)
        act = terma > 0.01
        ts.append(float(torch.quantile(terma[act][::7].float(), 0.99)))
        ds.append(float(torch.quantile((dose[act] / maker.dose_scale(cp))[::7].float(), 0.99)))
    return 1.0 / float(np.median(ts)), float(np.median(ds))


def evaluate(net: SurrogateNet, maker: SampleMaker, seeds, accept_rate=0.99, log=None, time_it=True):
    """Accept/fallback results and timings on the given phantoms."""
    sur = PhotonSurrogate(net, maker.grid, maker.shape, maker.model, accept_rate=accept_rate)
    cccs_counts = torch.empty(4, dtype=torch.int32, device=net.device)
    rows = []
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if seeds:  # warm up (the network's CUDA graph is captured on the second call)
        from .surrogate import hu_to_density, random_field, random_phantom_hu
        rng = np.random.default_rng(seeds[0])
        density = hu_to_density(random_phantom_hu(rng, maker.shape, maker.spacing, maker.device), *maker.table)
        cp = maker.control_point(*random_field(rng))
        for _ in range(3):
            sur.dose(density.contiguous(), cp)
        torch.cuda.synchronize()
    for i, s in enumerate(seeds):
        rng = np.random.default_rng(s)
        from .surrogate import hu_to_density, random_field, random_phantom_hu
        hu = random_phantom_hu(rng, maker.shape, maker.spacing, maker.device)
        density = hu_to_density(hu, *maker.table).contiguous()
        cp = maker.control_point(*random_field(rng))
        # surrogate path (TERMA, network, probe, gamma, fallback when rejected)
        torch.cuda.synchronize()
        ev_a.record()
        dose, accepted, rate, n_probe = sur.dose(density, cp)
        ev_b.record()
        torch.cuda.synchronize()
        t_sur = ev_a.elapsed_time(ev_b)
        net_dose = sur.pred.clone()
        if not accepted:  # pred is in network units when rejected
            net_dose.mul_(maker.dose_scale(cp))
        # CCCS path (the method without the surrogate) and the reference dose
        ev_a.record()
        maker.beam.set_density(density)
        maker.beam.terma(maker.model, cp, views=maker.views(cp))
        cccs = maker.beam.dose()
        ev_b.record()
        torch.cuda.synchronize()
        t_cccs = ev_a.elapsed_time(ev_b)
        dmax = float(cccs.max())
        engine.gamma_counts(net_dose, maker.grid.spacing, cccs, dose_norm=dmax, counts=cccs_counts)
        e, p = (int(v) for v in cccs_counts[:2].cpu())
        vs_cccs = p / e if e else 1.0
        act = cccs > 0.1 * dmax
        mean_abs = float(((net_dose - cccs).abs()[act]).mean() / dmax) if bool(act.any()) else 0.0
        rows.append(dict(seed=int(s), gantry=float(cp.ga), accepted=bool(accepted), probe_pass=rate,
                         n_probe=int(n_probe), gamma_vs_cccs=vs_cccs, mean_abs_diff_frac=mean_abs, t_surrogate_ms=t_sur,
                         t_cccs_ms=t_cccs))
        if log and (i + 1) % 25 == 0:
            acc = np.mean([r["accepted"] for r in rows])
            log("eval %d/%d: accepted %.3f, gamma vs CCCS mean %.4f" % (i + 1, len(seeds), acc,
                                                               np.mean([r["gamma_vs_cccs"] for r in rows])))
    return rows


def summarize(rows, accept_rate):
    acc = [r for r in rows if r["accepted"]]
    t_sur = float(np.mean([r["t_surrogate_ms"] for r in rows]))
    t_cccs = float(np.mean([r["t_cccs_ms"] for r in rows]))
    return dict(
        n=len(rows),
        accepted_frac=len(acc) / max(len(rows), 1),
        gamma_vs_cccs_mean_all=float(np.mean([r["gamma_vs_cccs"] for r in rows])),
        gamma_vs_cccs_mean_accepted=float(np.mean([r["gamma_vs_cccs"] for r in acc])) if acc else None,
        gamma_vs_cccs_min_accepted=float(np.min([r["gamma_vs_cccs"] for r in acc])) if acc else None,
        false_accepts=int(sum(1 for r in acc if r["gamma_vs_cccs"] < accept_rate)),
        beams_gamma_vs_cccs_ge_99=float(np.mean([r["gamma_vs_cccs"] >= 0.99 for r in rows])),
        mean_abs_diff_frac=float(np.mean([r["mean_abs_diff_frac"] for r in rows])),
        ms_per_beam_surrogate_path=t_sur,
        ms_per_beam_cccs_path=t_cccs,
        speedup_vs_cccs_path=t_cccs / t_sur if t_sur > 0 else None,
        ms_per_beam_accepted=float(np.mean([r["t_surrogate_ms"] for r in acc])) if acc else None,
    )


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--train", type=int, default=3000)
    ap.add_argument("--test", type=int, default=300)
    ap.add_argument("--epochs", type=int, default=50)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--time-budget", type=float, default=None, help="stop training after this many seconds")
    ap.add_argument("--max-steps", type=int, default=None)
    ap.add_argument("--accept", type=float, default=0.99, help="probe gamma pass rate to accept")
    ap.add_argument("--out", default="surrogate_6mv.npz")
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--state", default=None, help="write a resumable training checkpoint here")
    ap.add_argument("--state-every", type=int, default=None, help="steps between training checkpoints")
    ap.add_argument("--resume", default=None, help="continue training from this training checkpoint")
    ap.add_argument("--report", default=None)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)

    def log(msg):
        print(msg, flush=True)

    torch.manual_seed(args.seed)
    maker = SampleMaker()
    t0 = time.time()
    if args.resume:  # scales (and weights, Adam state, schedule) come from the checkpoint
        meta = load_training_state(args.resume)["trainer"]["meta"]
        net = SurrogateNet(seed=args.seed, terma_scale=float(meta[2]), dose_unit=float(meta[3]))
    elif args.init:
        net = SurrogateNet.load(args.init)
    else:
        ts, du = choose_scales(maker, range(TEST_SEED0 * 2, TEST_SEED0 * 2 + 16))
        net = SurrogateNet(seed=args.seed, terma_scale=ts, dose_unit=du)
        log("terma_scale %.4g dose_unit %.4g" % (ts, du))
    untrained = SurrogateNet(seed=args.seed, terma_scale=net.terma_scale, dose_unit=net.dose_unit)
    hist, t_data, t_train = [], 0.0, 0.0
    if args.train > 0:  # --train 0 with --init: evaluate the given weights only
        data = Dataset(maker, range(args.train), dose_unit=net.dose_unit, log=log)
        t_data = time.time() - t0
        log("dataset: %d samples in %.1f s" % (len(data), t_data))
        t1 = time.time()
        hist = train(net, data, epochs=args.epochs, lr=args.lr, seed=args.seed, log=log, max_steps=args.max_steps,
                     time_budget_s=args.time_budget, checkpoint=args.out, state_path=args.state,
                     state_every=args.state_every, resume=args.resume)
        t_train = time.time() - t1
        net.save(args.out)
        del data
        torch.cuda.empty_cache()
    test_seeds = [TEST_SEED0 + i for i in range(args.test)]
    rows = evaluate(net, maker, test_seeds, accept_rate=args.accept, log=log)
    summ = summarize(rows, args.accept)
    rows_u = evaluate(untrained, maker, test_seeds[:min(20, len(test_seeds))], accept_rate=args.accept)
    summ_u = summarize(rows_u, args.accept)
    report = dict(train_samples=args.train, test_samples=args.test, epochs_requested=args.epochs, lr=args.lr,
                  steps=hist[-1][0] if hist else 0, train_seconds=t_train, data_seconds=t_data,
                  loss_history=hist, terma_scale=net.terma_scale, dose_unit=net.dose_unit,
                  flops_forward=SurrogateNet.flops(maker.shape), trained=summ, untrained=summ_u, rows=rows)
    log(json.dumps({"trained": summ, "untrained": summ_u}, indent=1))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
