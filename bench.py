"""Benchmark of the DoseCUDA B200 dose engines.

Headline: CCCS ms/beam on the small photon workload (128^3 voxels at 2.5 mm,
water with a lung block and a bone cube, one 10x10 cm 6 MV field, 100 MU,
72 cone directions).  One step = one control point: density -> ray trace ->
TERMA -> collapsed-cone dose.  Secondary (same JSON line): IMPT spots/s on the
small proton workload (96^3 at 2 mm, 6 energy layers x 100 spots); one step =
one beam: RLSP -> WET ray trace + smoothing -> pencil-beam dose.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

``value`` is measured with the inputs resident in HBM (CUDA events on the
launching stream, L2 flushed between steps with a 256 MiB write outside the
timed brackets); ``e2e`` goes through the drop-in ``dose_kernels`` API with
host buffers (pinned input, H2D + D2H inside the timed region).
``--impl reference`` times the reference DoseCUDA CUDA extension (built from
the reference sources into oracle/_ref/) through its own API on the same
inputs.  N > 1 (torchrun): N independent replicas, one per GPU, no
collective on the data path (weak scaling); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# DRAM bytes (read + write) per launch from one ncu --set full capture of each
# dominant kernel on these workloads, with the summary that records the
# capture (its command and figures).  A kernel change makes its entry stale
# until it is captured again.
NCU_TRAFFIC = {
    "cccs": (15107328, "profiles/cccs_photon_small.md"),
    "pencil_beam": (3622912, "profiles/pencil_beam_proton_small.md"),
    "conv_dec0": (67162880 + 26884352, "profiles/conv_gather_dec0_surrogate_128.md"),
}
SM_COUNT = 148
FP32_LANES_PER_SM = 128


# ----------------------------------------------------------------------------
# multi-process plumbing
# ----------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def aggregate_max(value: float, dist_mod) -> float:
    """Max of a per-rank scalar over all ranks (identity without a group)."""
    if dist_mod is None:
        return value
    import torch
    dev = "cuda" if dist_mod.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist_mod.all_reduce(t, op=dist_mod.ReduceOp.MAX)
    return float(t.item())


def barrier(dist_mod):
    if dist_mod is not None:
        dist_mod.barrier()


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
def photon_workload():
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.photon_small()
    model = plan.beam_models[0]
    cp = plan.beam_list[0].cp_list[0]
    density = grid.DensityFromHU(plan.machine_name)
    return grid, model, cp, density


def proton_workload():
    from dosecuda_b200 import phantoms
    grid, plan = phantoms.proton_small()
    model = plan.beam_models[0]
    beam = plan.beam_list[0]
    rlsp = grid.RLSPFromHU(plan.machine_name)
    return grid, model, beam, rlsp


def load_oracle():
    """The CPU oracle module (oracle/oracle.py), loaded by path: it is the
    checker and the CPU baseline, never part of the measured engine."""
    import importlib.util
    if "dc_oracle" in sys.modules:
        return sys.modules["dc_oracle"]
    spec = importlib.util.spec_from_file_location("dc_oracle", os.path.join(ROOT, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dc_oracle"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p, "measured"
    return PEAKS_FALLBACK, "fallback"


# ----------------------------------------------------------------------------
# algorithmic work (counted on the host from geometry, independent of the kernels)
# ----------------------------------------------------------------------------
def cccs_samples(dose_ref_mask_count: int, model, spacing_mm: float) -> int:
    """Cone samples per active voxel: 12 azimuths x sum over cones of the
    float sample count of the backward march (ray_length, -= spacing)."""
    per = 0
    sp = np.float32(spacing_mm) / np.float32(10.0)
    for rl in np.asarray(model.kernel, np.float32)[:, 5]:
        r = np.float32(rl)
        while r >= 0:
            per += 1
            r = np.float32(r - sp)
    return 12 * per * dose_ref_mask_count


# ----------------------------------------------------------------------------
def time_steps(step, k, flush):
    """Device time of k steps (CUDA events on the current stream around each
    step; the L2 flush between steps is outside the brackets)."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
    for i in range(k):
        flush()
        ev[i][0].record()
        step()
        ev[i][1].record()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def run_mine(args, ws, rank, local, dist_mod):
    import torch
    from dosecuda_b200 import _lib, dose_kernels, engine
    from dosecuda_b200.dose_kernels import ControlPointView, PhotonModelView
    from dosecuda_b200.plan import VolumeObject

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush():
        flush_buf.zero_()

    pk, pk_kind = peaks()
    out = {}

    # ---------------- photon (headline) ----------------
    grid, model, cp, density = photon_workload()
    dens_t = torch.from_numpy(density).to(dev)
    dose_t = torch.empty_like(dens_t)
    views = (PhotonModelView(model), ControlPointView(cp))

    def step_x():
        engine.photon_dose(dens_t, grid, model, cp, out=dose_t, views=views)

    for _ in range(args.warmup):
        flush()
        step_x()
    torch.cuda.synchronize()
    barrier(dist_mod)
    torch.cuda.synchronize()
    clk = ClockSampler(local).__enter__()  # sampled across all timed regions below
    t_ms = time_steps(step_x, args.steps, flush)
    torch.cuda.synchronize()
    barrier(dist_mod)
    t_ms = aggregate_max(t_ms, dist_mod)
    x_ms_per_beam = t_ms / (args.steps * ws)

    # kernel-level timing on the launching stream (profiled pass, separate from the timed one)
    _lib.raise_for(lib.dc_profile_enable(local, 1))
    _lib.raise_for(lib.dc_profile_reset(local))
    for _ in range(args.steps):
        flush()
        step_x()
    torch.cuda.synchronize()
    prof_x = _lib.profile_read(local)
    _lib.raise_for(lib.dc_profile_enable(local, 0))
    depth_mode = engine.photon_depth_mode(local)
    depth_marched = engine.photon_depth_marched(local)
    dose_np = dose_t.cpu().numpy()

    # the cone-direction sweep CCCS (an approximation, not the headline) beside
    # the per-voxel CCCS of the same TERMA: time and distance from it
    xbeam = engine.PhotonBeam(grid, dens_t.shape, device=dev)
    xbeam.set_density(dens_t)
    xbeam.terma(model, cp, views=views)
    exact, sweep = xbeam.dose(), xbeam.dose_sweep()
    torch.cuda.synchronize()
    sev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    sev[0].record()
    for _ in range(args.steps):
        xbeam.dose(out=exact)
    sev[1].record()
    sev[2].record()
    for _ in range(args.steps):
        xbeam.dose_sweep(out=sweep)
    sev[3].record()
    torch.cuda.synchronize()
    gc = engine.gamma_counts(sweep, grid.spacing, exact).cpu().numpy()
    e_np, s_np = exact.cpu().numpy().astype(np.float64), sweep.cpu().numpy().astype(np.float64)
    hi = e_np > 0.1 * e_np.max()
    sweep_rec = {"ms_sweep": round(sev[2].elapsed_time(sev[3]) / args.steps, 4),
                 "ms_per_voxel_cccs": round(sev[0].elapsed_time(sev[1]) / args.steps, 4),
                 "dD_frac_dmax": round(float(np.abs(s_np - e_np)[hi].max() / e_np.max()), 5),
                 "gamma_2_2": round(float(gc[1]) / max(int(gc[0]), 1), 5),
                 "what": "dc_photon_beam_dose_sweep against dc_photon_beam_dose on the same TERMA (CCCS only, "
                         "no ray trace or TERMA); an approximation outside the parity bar, not the headline"}
    xbeam.close()
    # active voxels = TERMA > 0.01 (the voxels the CCCS evaluates); from the
    # engine's TERMA mask we only need the count, taken as dose > 0 voxels.
    n_active = int((dose_np > 0).sum())
    samples = cccs_samples(n_active, model, float(grid.spacing[0]))
    c_launches, c_ms = prof_x.get("cccs", (1, float("nan")))
    cccs_avg_ms = c_ms / max(c_launches, 1)
    flops_per_sample = 18.0
    fp32_peak = SM_COUNT * FP32_LANES_PER_SM * 2 * pk.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved_tf = samples * flops_per_sample / (cccs_avg_ms * 1e-3) / 1e12
    nvox = density.size
    # algorithmic bytes: the (TERMA, density) float2 volume read once, the
    # electron term read once, the dose written once = 16 B per voxel
    cccs_bytes = nvox * 16

    # e2e through the drop-in API with host numpy in and out, H2D + D2H per
    # call: the headline passes the pageable array DensityFromHU returns, as
    # the reference's plan loop does (plan_imrt.py:126-158); the same call
    # with a page-locked input is reported beside it
    # calls per end-to-end leg: the K steps, and at least 30 so that the
    # wall-clock mean spans tens of milliseconds
    n_e2e = max(args.steps, 30)

    def e2e_photon(voxels):
        vol = VolumeObject()
        vol.voxel_data = voxels
        vol.origin = np.array(grid.origin, dtype=np.single)
        vol.spacing = np.array(grid.spacing, dtype=np.single)
        # warm-up as the timed loop runs: the previous result stays alive while
        # the next call allocates its page-locked output
        d = None
        for _ in range(max(2, args.warmup)):
            d = dose_kernels.photon_dose_cuda(model, vol, cp, local)
        torch.cuda.synchronize()
        barrier(dist_mod)
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            d = dose_kernels.photon_dose_cuda(model, vol, cp, local)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        barrier(dist_mod)
        return aggregate_max(ms, dist_mod), d


    # ---------------- proton (secondary) ----------------
    pgrid, pmodel, pbeam, rlsp = proton_workload()
    rl_t = torch.from_numpy(rlsp).to(dev)
    wet_t = torch.empty_like(rl_t)
    pdose_t = torch.empty_like(rl_t)
    dmodel = engine.ProtonModelDevice(pmodel, device=dev)
    n_spots = pbeam.spot_list.shape[0]

    def step_p():
        engine.proton_wet(rl_t, pgrid, pbeam, pmodel, out=wet_t)
        engine.proton_dose(wet_t, pgrid, pbeam, dmodel, out=pdose_t)

    for _ in range(args.warmup):
        flush()
        step_p()
    torch.cuda.synchronize()
    barrier(dist_mod)
    tp_ms = time_steps(step_p, args.steps, flush)
    clk.__exit__(None, None, None)  # the device-timed regions end here

    # end-to-end legs after the clock sampler has stopped: its polling takes
    # driver locks that stall host API calls, which a wall-clock figure over a
    # few milliseconds would pick up
    e2e_ms, d = e2e_photon(density)
    pinned = torch.from_numpy(density).pin_memory()
    e2e_pinned_ms, _ = e2e_photon(pinned.numpy())
    parity_e2e = float(np.abs(d - dose_np).max())
    barrier(dist_mod)
    tp_ms = aggregate_max(tp_ms, dist_mod)
    spots_per_s = n_spots * args.steps * ws / (tp_ms * 1e-3)
    _lib.raise_for(lib.dc_profile_enable(local, 1))
    _lib.raise_for(lib.dc_profile_reset(local))
    for _ in range(args.steps):
        flush()
        step_p()
    torch.cuda.synchronize()
    prof_p = _lib.profile_read(local)
    _lib.raise_for(lib.dc_profile_enable(local, 0))
    # (voxel, spot) pairs the pencil beam evaluates: voxels inside each layer's range
    wet_np = wet_t.cpu().numpy() * np.float32(10.0)
    pairs = 0
    for e in np.unique(pbeam.spot_list[:, 3].astype(int)):
        r80 = pmodel.divergence_params[e, 1]
        pairs += int((wet_np <= np.float32(1.1) * r80).sum()) * int((pbeam.spot_list[:, 3].astype(int) == e).sum())
    pb_launches, pb_ms = prof_p.get("pencil_beam", (1, float("nan")))
    pb_avg_ms = pb_ms / max(pb_launches, 1)
    def e2e_proton(voxels):
        pvol = VolumeObject()
        pvol.voxel_data = voxels
        pvol.origin = np.array(pgrid.origin, dtype=np.single)
        pvol.spacing = np.array(pgrid.spacing, dtype=np.single)

        def beam_call():
            # the reference's plan loop (plan_impt.py:124-160): WET, then the
            # dose from a fresh array copy of it
            w = dose_kernels.proton_raytrace_cuda(pmodel, pvol, pbeam, local)
            wv = VolumeObject()
            wv.voxel_data, wv.origin, wv.spacing = np.array(w, dtype=np.single), pvol.origin, pvol.spacing
            dose_kernels.proton_spot_cuda(pmodel, pvol, wv, pbeam, local)

        for _ in range(max(1, args.warmup)):
            beam_call()
        barrier(dist_mod)
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            beam_call()
        ms = (time.perf_counter() - t0) * 1e3
        barrier(dist_mod)
        return aggregate_max(ms, dist_mod)

    pe2e_ms = e2e_proton(rlsp)
    pe2e_pinned_ms = e2e_proton(torch.from_numpy(rlsp).pin_memory().numpy())

    out.update(dict(
        x_ms_per_beam=x_ms_per_beam, t_ms=t_ms, prof_x=prof_x, depth_mode=depth_mode, depth_marched=depth_marched, clocks=clk.summary(), samples=samples,
        n_active=n_active, cccs_avg_ms=cccs_avg_ms, achieved_tf=achieved_tf, fp32_peak=fp32_peak,
        cccs_bytes=cccs_bytes, e2e_ms=e2e_ms, e2e_pinned_ms=e2e_pinned_ms, parity_e2e=parity_e2e, nvox=nvox, pk=pk,
        pk_kind=pk_kind, spots_per_s=spots_per_s, tp_ms=tp_ms, prof_p=prof_p, pairs=pairs, pb_avg_ms=pb_avg_ms,
        pe2e_ms=pe2e_ms, pe2e_pinned_ms=pe2e_pinned_ms, n_spots=n_spots, pnvox=rlsp.size, n_e2e=n_e2e,
        sweep=sweep_rec,
    ))
    return out


def run_batched(args, local, dist_mod, ws):
    """Batched IMPT: 16 patient-like plans (256x256x160 at 1.5x1.5x2.0 mm,
    1-3 beams, 500-12,000 spots each) in one persistent launch, against the
    same beams evaluated by per-beam calls of the drop-in API."""
    import torch
    from dosecuda_b200 import dose_kernels, engine, phantoms
    from dosecuda_b200.plan import VolumeObject
    from dosecuda_b200.plan_impt import IMPTPlan
    dev = torch.device("cuda", local)
    model = IMPTPlan().beam_models[0]
    t0 = time.perf_counter()
    plans = [phantoms.batch_plan(seed + 1000 * local, model=model) for seed in range(args.batch_plans)]
    gen_s = time.perf_counter() - t0
    b = engine.ProtonBatch(model, device=dev)
    rls = []
    for grid, beams, _ in plans:
        rl = torch.from_numpy(grid.RLSPFromHU("HitachiProbeatJHU")).to(dev)
        rls.append(rl)
        pid = b.add_plan(grid, rl)
        for bm in beams:
            b.add_beam(pid, bm)
    b.commit()
    b.wet()
    torch.cuda.synchronize()
    variant = b.autotune(os.path.join(ROOT, "_build_autotune.json") if args.tune_cache else None)
    for _ in range(args.warmup):
        b.dose()
    torch.cuda.synchronize()
    barrier(dist_mod)
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        b.dose()
    e.record()
    torch.cuda.synchronize()
    t_batch = aggregate_max(a.elapsed_time(e) / args.steps, dist_mod)
    # the same launch replayed from a CUDA graph
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        b.dose()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        b.dose()
    g.replay()
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        g.replay()
    e.record()
    torch.cuda.synchronize()
    t_graph = aggregate_max(a.elapsed_time(e) / args.steps, dist_mod)
    del g
    # per-plan calls: every beam through dose_kernels.proton_spot_cuda (host buffers)
    wets = [w.cpu().numpy() for w in b.wets]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bi = 0
    for (grid, beams, _), rl in zip(plans, rls):
        vol = VolumeObject()
        vol.voxel_data = grid.HU  # the reference's call also reads the RLSP volume; its content is unused
        vol.origin = np.asarray(grid.origin, np.float32)
        vol.spacing = np.asarray(grid.spacing, np.float32)
        for bm in beams:
            wv = VolumeObject()
            wv.voxel_data, wv.origin, wv.spacing = wets[bi], vol.origin, vol.spacing
            # per-axis spacing is not expressible through the reference's call (it uses spacing[0]);
            # the timing of the call is what is compared here
            dose_kernels.proton_spot_cuda(model, vol, wv, bm, local)
            bi += 1
    t_calls = aggregate_max((time.perf_counter() - t0) * 1e3, dist_mod)
    # influence matrices (CSR, cutoff 1e-4 of each spot's maximum), beam by
    # beam, count then fill: one beam's matrix is alive at a time
    csr = None
    if args.batch_csr:
        b.influence_csr(0, cutoff=1e-4)  # warm-up (kernel attributes, allocator)
        torch.cuda.synchronize()
        nnz_tot, max_bytes, bytes_tot = 0, 0, 0
        t0 = time.perf_counter()
        for bid in range(b.n_beams):
            r, c, v = b.influence_csr(bid, cutoff=1e-4)
            nnz = c.numel()
            nnz_tot += nnz
            bytes_tot += r.numel() * 8 + nnz * 8
            max_bytes = max(max_bytes, r.numel() * 8 + nnz * 8)
            del r, c, v
        torch.cuda.synchronize()
        t_csr = aggregate_max((time.perf_counter() - t0) * 1e3, dist_mod)
        csr = {"ms_all_beams": round(t_csr, 2), "beams": b.n_beams, "nnz_total": int(nnz_tot),
               "entries_per_s": round(nnz_tot / (t_csr * 1e-3), 1),
               "gb_written": round(bytes_tot / 1e9, 3),
               "max_beam_gb": round(max_bytes / 1e9, 3),
               "what": "per beam: spot-max, count, scan, fill passes; float32 values, int32 spot columns, int64 "
                       "voxel row starts; entries >= 1e-4 x the spot's maximum; wall clock including the "
                       "count's host read and the arrays' allocation"}
    n_spots = b.n_spots
    out = {
        "metric": "batched IMPT dose: ms per optimisation iteration (all plans)",
        "value": round(t_batch, 3), "unit": "ms/iteration", "higher_is_better": False,
        "graph_replay_ms": round(t_graph, 3),
        "spots_per_s": round(n_spots * ws / (t_batch * 1e-3), 1),
        "per_plan_calls_ms": round(t_calls, 3),
        "speedup_vs_per_plan_calls": round(t_calls / t_batch, 2),
        "tile_variant": int(variant), "tile_ms": [round(x, 3) for x in getattr(b, "tune_ms", [])],
        "influence_csr": csr,
        "config": {"workload": "%d plans x 256x256x160 @ 1.5x1.5x2.0 mm, %d beams, %d spots; body ellipsoid "
                               "(20+-40 HU) with bone/lung/air ellipsoids, spherical target, layers at 3 mm R80 "
                               "spacing, 4-6 mm spot grid, lognormal(0, 0.5) weights" %
                               (args.batch_plans, b.n_beams, n_spots),
                   "iteration": "dose of every plan for new spot weights (WET resident)",
                   "per_plan_calls": "one dose_kernels.proton_spot_cuda call per beam, host buffers"},
        "generation_s": round(gen_s, 2),
    }
    b.close()
    return out


def run_optimisation(args, local, dist_mod):
    """Differentiable IMPT optimisation: 3 beams, ~7,500 spots; objective
    sum_target (D - 2 Gy)^2 + 10 sum_OAR max(D - 1 Gy, 0)^2 in FP64; gradient
    by the adjoint kernel through torch.autograd; 200 projected-Adam
    iterations (dosecuda_b200.optimize)."""
    import torch
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.optimize import DoseObjective, ImptOptimizer
    from dosecuda_b200.plan_impt import IMPTPlan
    dev = torch.device("cuda", local)
    model = IMPTPlan().beam_models[0]
    grid, beams, (c_t, r_t) = phantoms.batch_plan(102, model=model, n_beams=3)
    rl = torch.from_numpy(grid.RLSPFromHU("HitachiProbeatJHU")).to(dev)
    nz, ny, nx = rl.shape
    sp = np.asarray(grid.spacing, np.float64)
    zz = torch.arange(nz, device=dev, dtype=torch.float64) * sp[2] + grid.origin[2]
    yy = torch.arange(ny, device=dev, dtype=torch.float64) * sp[1] + grid.origin[1]
    xx = torch.arange(nx, device=dev, dtype=torch.float64) * sp[0] + grid.origin[0]
    Z, Y, X = torch.meshgrid(zz, yy, xx, indexing="ij")
    target = ((X - c_t[0]) ** 2 + (Y - c_t[1]) ** 2 + (Z - c_t[2]) ** 2) <= r_t ** 2
    # OAR: cylinder r = 10 mm along z, adjacent to the target
    oar = ((X - (c_t[0] + r_t + 10.0)) ** 2 + (Y - c_t[1]) ** 2) <= 10.0 ** 2
    oar &= (Z - c_t[2]).abs() <= r_t
    del X, Y, Z
    plans = [engine.ProtonBeamPlan(grid, bm, model, device=dev) for bm in beams]
    wets = [engine.proton_wet(rl, grid, bm, model) for bm in beams]
    objective = DoseObjective().uniform(target, 2.0).max_dose(oar, 1.0, weight=10.0)
    opt = ImptOptimizer(plans, wets, objective)
    opt.scale_to(target, 2.0)  # mean target dose 2 Gy; lr = 0.02 x the mean weight
    sizes = opt.sizes
    f0 = opt.evaluate()
    iters = args.opt_iters
    for _ in range(3):  # warm-up
        opt.step()
    torch.cuda.synchronize()
    barrier(dist_mod)
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    opt.run(iters)
    e.record()
    torch.cuda.synchronize()
    t = aggregate_max(a.elapsed_time(e) / iters, dist_mod)
    f1 = opt.evaluate()
    # the same optimisation with the dose and adjoint evaluated at the
    # objective's voxels only (voxel-list kernels); same start, same steps
    opt_v = ImptOptimizer(plans, wets, objective, voxels="objective")
    opt_v.scale_to(target, 2.0)
    for _ in range(3):  # warm-up
        opt_v.step()
    torch.cuda.synchronize()
    barrier(dist_mod)
    a.record()
    opt_v.run(iters)
    e.record()
    torch.cuda.synchronize()
    t_v = aggregate_max(a.elapsed_time(e) / iters, dist_mod)
    with torch.no_grad():
        f1_v = objective(opt_v.dose()).item()  # evaluated on the full-volume dose
    return {
        "metric": "IMPT plan optimisation: ms per iteration (dose + adjoint + Adam step)",
        "value": round(t, 3), "unit": "ms/iteration", "higher_is_better": False,
        "iterations": iters, "objective_start": round(f0, 3), "objective_end": round(f1, 3),
        "objective_voxels": {"ms_per_iteration": round(t_v, 4), "objective_end": round(f1_v, 3),
                             "voxels": int(objective.voxel_union().numel()),
                             "speedup_vs_volume": round(t / t_v, 2),
                             "what": "dose and adjoint at the objective's voxels only (target + OAR), "
                                     "voxel-list pencil-beam kernels; objective_end evaluated on the full volume"},
        "config": {"workload": "256x256x160 @ 1.5x1.5x2.0 mm, 3 beams, %d spots; target sphere r=%.1f mm, OAR "
                               "cylinder r=10 mm adjacent" % (sum(sizes), r_t),
                   "objective": "sum_target (D-2)^2 + 10 sum_OAR max(D-1,0)^2, FP64 reduction",
                   "gradient": "hand-written adjoint kernel (D^T g) behind torch.autograd"},
    }


def vmat_workload(n_cps=18):
    """The photon workload's phantom with one arc-like beam: n_cps control
    points of the 10x10 cm field at gantry 0, 20, ..., 100 MU in total."""
    from dosecuda_b200 import phantoms
    from dosecuda_b200.plan_imrt import IMRTControlPoint
    grid, plan = phantoms.photon_small(seed=1)
    beam = plan.beam_list[0]
    cp0 = beam.cp_list[0]
    beam.cp_list = [IMRTControlPoint(cp0.iso, 100.0 / n_cps, np.array(cp0.mlc, copy=True), 360.0 * i / n_cps, 0.0,
                                     0.0, None, None) for i in range(n_cps)]
    return grid, plan


def run_plan_loop(args, local, dist_mod, dose_kernels_module=None):
    """IMRT plan of one 18-control-point beam through the plan API: the
    reference's host loop (HU -> density on the host, one photon_dose_cuda
    call per control point with host buffers, numpy accumulation) and, for
    this engine, the device-resident loop (computeIMRTPlan(device=True):
    HU converted on the GPU, all control points in one call, one copy back).
    Both give the same dose bit for bit."""
    import torch
    from dosecuda_b200 import plan_imrt
    grid, plan = vmat_workload()
    saved = plan_imrt.dose_kernels
    if dose_kernels_module is not None:
        plan_imrt.dose_kernels = dose_kernels_module
    try:
        grid.computeIMRTPlan(plan, gpu_id=local)  # warm-up
        reps = max(2, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(reps):
            grid.computeIMRTPlan(plan, gpu_id=local)
        t_host = (time.perf_counter() - t0) * 1e3 / reps
        host_dose = grid.dose.copy()
    finally:
        plan_imrt.dose_kernels = saved
    out = {"metric": "IMRT plan, 1 beam x 18 control points (128^3): ms per plan",
           "host_loop_ms": round(t_host, 3), "unit": "ms/plan", "higher_is_better": False,
           "config": {"workload": "128^3 @ 2.5 mm photon phantom, 18 control points of a 10x10 cm 6 MV field at "
                                  "gantry 0..340 deg, 100 MU in total"}}
    if dose_kernels_module is not None:
        out["value"] = out["host_loop_ms"]
        return out
    grid.computeIMRTPlan(plan, gpu_id=local, device=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        grid.computeIMRTPlan(plan, gpu_id=local, device=True)
    t_dev = aggregate_max((time.perf_counter() - t0) * 1e3 / reps, dist_mod)
    out.update(value=round(t_dev, 3), device_loop_ms=round(t_dev, 3),
               speedup_vs_host_loop=round(t_host / t_dev, 2),
               bitwise_equal_to_host_loop=bool(np.array_equal(grid.dose, host_dose)))
    out["config"]["device_loop"] = "computeIMRTPlan(device=True): HU uploaded once and converted on the GPU, " \
                                   "the beam's control points in one call, one copy back"
    return out


SURROGATE_WEIGHTS = os.path.join(ROOT, "dosecuda_b200", "weights", "surrogate_6mv.npz")


def run_surrogate(args, local, dist_mod):
    """Learned photon surrogate with CCCS fallback on held-out phantoms of the
    surrogate workload (128^3 @ 2.5 mm, random ellipsoids, random gantry and
    MLC field): per beam the surrogate path (TERMA, network, sparse CCCS
    probe, probe gamma, full CCCS when rejected) against the CCCS path (TERMA
    + full CCCS), both timed with CUDA events; every network dose checked
    against the full CCCS with gamma(2%/2mm)."""
    import torch
    from dosecuda_b200 import engine
    from dosecuda_b200.surrogate import PhotonSurrogate, SampleMaker, SurrogateNet, hu_to_density, random_field, \
        random_phantom_hu
    if not os.path.exists(SURROGATE_WEIGHTS):
        return {"unavailable": "no trained weights at dosecuda_b200/weights/surrogate_6mv.npz"}
    dev = torch.device("cuda", local)
    net = SurrogateNet.load(SURROGATE_WEIGHTS, device=dev)
    maker = SampleMaker(device=dev)
    sur = PhotonSurrogate(net, maker.grid, maker.shape, maker.model, accept_rate=0.99)
    seeds = [1_000_000 + i for i in range(args.surrogate_beams)]
    cases = []
    for s in seeds:
        rng = np.random.default_rng(s)
        hu = random_phantom_hu(rng, maker.shape, maker.spacing, dev)
        cases.append((hu_to_density(hu, *maker.table).contiguous(), maker.control_point(*random_field(rng))))
    for _ in range(max(args.warmup, 3)):
        sur.dose(*cases[0])
        maker.beam.set_density(cases[0][0])
        maker.beam.terma(maker.model, cases[0][1], views=maker.views(cases[0][1]))
        maker.beam.dose()
    torch.cuda.synchronize()
    barrier(dist_mod)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    vs_cccs = torch.empty(4, dtype=torch.int32, device=dev)
    rows = []
    for density, cp in cases:
        ev[0].record()
        dose, accepted, rate, n_probe = sur.dose(density, cp)
        ev[1].record()
        torch.cuda.synchronize()
        net_dose = sur.pred.clone() if accepted else sur.pred * maker.dose_scale(cp)
        ev[2].record()
        maker.beam.set_density(density)
        maker.beam.terma(maker.model, cp, views=maker.views(cp))
        cccs = maker.beam.dose()
        ev[3].record()
        torch.cuda.synchronize()
        dmax = float(cccs.max())
        engine.gamma_counts(net_dose, maker.grid.spacing, cccs, dose_norm=dmax, counts=vs_cccs)
        e, p = (int(v) for v in vs_cccs[:2].cpu())
        rows.append((ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]), bool(accepted), rate, p / max(e, 1),
                     n_probe))
    t_sur = aggregate_max(float(np.mean([r[0] for r in rows])), dist_mod)
    t_cccs = aggregate_max(float(np.mean([r[1] for r in rows])), dist_mod)
    acc = [r for r in rows if r[2]]
    # network forward alone (one CUDA-graph replay), and the conv-stack roofline
    k = max(args.steps, 5)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(k):
        sur.run_network()
    b.record()
    torch.cuda.synchronize()
    t_net = a.elapsed_time(b) / k
    flops = SurrogateNet.flops(maker.shape)
    pk, pk_kind = peaks()
    bf16_peak = pk.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"])
    achieved = flops / (t_net * 1e-3) / 1e12
    # the dominant kernel alone: the last decoder convolution (16 -> 16, 3x3x3, full grid)
    from dosecuda_b200.surrogate import CONV3
    x16 = torch.randn((1,) + tuple(maker.shape) + (16,), device=dev).to(torch.bfloat16)
    y16 = torch.empty_like(x16)
    for _ in range(3):
        net.ops.conv(CONV3, x16, net._fw["dec0"], 16, out=y16)
    a.record()
    for _ in range(k):
        net.ops.conv(CONV3, x16, net._fw["dec0"], 16, out=y16)
    b.record()
    torch.cuda.synchronize()
    t_dec0 = a.elapsed_time(b) / k
    vox = int(np.prod(maker.shape))
    dec0_flops = 2 * vox * 27 * 16 * 16
    dec0_tf = dec0_flops / (t_dec0 * 1e-3) / 1e12
    del x16, y16
    return {
        "metric": "surrogate vs CCCS speed-up at gamma(2%/2mm) >= 99% (per beam, fallbacks included)",
        "value": round(t_cccs / t_sur, 3), "unit": "x", "higher_is_better": True,
        "ms_per_beam_surrogate_path": round(t_sur, 4), "ms_per_beam_cccs_path": round(t_cccs, 4),
        "ms_per_beam_accepted": round(float(np.mean([r[0] for r in acc])), 4) if acc else None,
        "beams": len(rows), "accepted_frac": round(len(acc) / len(rows), 4),
        "gamma_vs_cccs_mean_accepted": round(float(np.mean([r[4] for r in acc])), 5) if acc else None,
        "gamma_vs_cccs_min_accepted": round(float(np.min([r[4] for r in acc])), 5) if acc else None,
        "false_accepts": int(sum(1 for r in acc if r[4] < 0.99)),
        "gamma_vs_cccs_mean_all": round(float(np.mean([r[4] for r in rows])), 5),
        "probe_points_mean": round(float(np.mean([r[5] for r in rows])), 1),
        "network_forward_ms": round(t_net, 4),
        "roofline": {"bound": "tensor", "kernel": "conv_gather_kernel 16->16 3x3x3 @ 128^3 (bf16 mma.sync)",
                     "achieved": round(dec0_tf, 2), "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": round(dec0_tf / bf16_peak, 4), "peak_kind": pk_kind + " (cuBLAS bf16)",
                     "kernel_ms": round(t_dec0, 4),
                     "work": "%d FLOPs per launch (2 x voxels x 27 x 16 x 16)" % dec0_flops,
                     "traffic": NCU_TRAFFIC["conv_dec0"][0], "traffic_source": NCU_TRAFFIC["conv_dec0"][1],
                     "stack": {"achieved": round(achieved, 2), "frac": round(achieved / bf16_peak, 4),
                               "work": "%d FLOPs per forward (conv layers from their shapes + head)" % flops}},
        "config": {"workload": "photon surrogate: 128^3 @ 2.5 mm, water body + 1-5 random ellipsoids (HU -900..1500), "
                               "6 MV, gantry 0-355 in 5 deg steps, 2-20 cm MLC fields, 100 MU; held-out seeds "
                               "1000000+i",
                   "network": "4-level 3D encoder-decoder, 16-128 channels, bf16 activations, fp32 accumulation",
                   "acceptance": "probe gamma(2%%/2mm, 10%% cutoff) >= 99%% on CCCS at ~%d probe voxels"
                                 % int(np.mean([r[5] for r in rows])),
                   "l2": "per-beam working set (activations) above the 126 MB L2"},
    }


def texture_roof(gpu, achieved_per_s):
    """CCCS cone samples/s against the texture unit's measured rate of
    trilinear float2 3D fetches in the same access pattern."""
    import ctypes as C
    from dosecuda_b200 import _lib
    v = C.c_double()
    rc = _lib.load().dc_texture_fetch_rate(gpu, C.byref(v))
    if rc != 0:
        return None
    return {"achieved": round(achieved_per_s, 1), "peak": round(v.value, 1), "unit": "filtered float2 fetches/s",
            "frac": round(achieved_per_s / v.value, 4),
            "peak_kind": "measured (dc_texture_fetch_rate: all SMs, full occupancy, CCCS-like line marches)"}


def cpu_baseline_photon():
    """The FP64 C oracle on the host cores: one full control point of the
    photon workload (the whole 128^3 beam; about 10-30 s of CPU time).
    Also returns the oracle's CCCS sample count (voxels with TERMA > 0.01)."""
    oracle = load_oracle()
    grid, model, cp, density = photon_workload()
    t0 = time.perf_counter()
    _, _, _, samples = oracle.photon_dose(density, np.asarray(grid.spacing, np.float32)[[0, 0, 0]], grid.origin,
                                          model, cp.iso, cp.mu, cp.ga, cp.ca, cp.ta, np.ascontiguousarray(cp.mlc),
                                          intermediates=True)
    dt = time.perf_counter() - t0
    # samples of the radiological-depth march (geometry only: 1 mm steps from
    # every voxel to the volume's exit towards the source at SAD)
    _, march = oracle.proton_wet(density, np.asarray(grid.spacing, np.float32)[[0, 0, 0]], grid.origin, cp.iso,
                                 cp.ga, cp.ta, model.primary_source_distance, model.primary_source_distance)
    return {"value": round(dt * 1e3, 1), "unit": "ms/beam", "cores": oracle.num_threads(), "kind": "port",
            "sample": "one full control point of the 128^3 photon workload (FP64 C/OpenMP oracle)"}, samples, march


def cpu_baseline_proton():
    oracle = load_oracle()
    grid, model, beam, rlsp = proton_workload()
    sp = np.asarray(grid.spacing, np.float32)[[0, 0, 0]]
    t0 = time.perf_counter()
    wet, march = oracle.proton_wet(rlsp, sp, grid.origin, beam.iso, beam.gantry_angle, beam.couch_angle,
                                   model.VSADX, model.VSADY)
    _, dense, near = oracle.proton_dose(wet.astype(np.float32), sp, grid.origin, beam.iso, beam.gantry_angle,
                                        beam.couch_angle, model, beam.spot_list, near_pairs=True)
    dt = time.perf_counter() - t0
    return {"value": round(beam.spot_list.shape[0] / dt, 2), "unit": "spots/s", "cores": oracle.num_threads(),
            "kind": "port",
            "sample": "one full beam of the 96^3 proton workload (600 spots, FP64 C/OpenMP oracle)"}, march, near


def pencil_beam_roofline(r):
    """The pencil beam's roofline.  Work unit (the algorithmic count, from the
    oracle): a (voxel, spot) pair within the layer's range whose distance from
    the spot axis is inside 6 halo sigmas at that voxel, 20 FP32 flops and 2
    SFU ex2 each.  The kernel culls spots per CTA, so it evaluates somewhat
    more pairs than that; the dense count (every in-range voxel x every spot of
    the layer, the reference's work) is reported beside it."""
    sm_hz = r["pk"].get("sm_max_mhz", 1965.0) * 1e6
    sec = r["pb_avg_ms"] * 1e-3
    near = r.get("near_pairs")
    pairs = near if near else r["pairs"]
    out = {"bound": "sfu", "kernel": "pencil_beam",
           "achieved": round(2 * pairs / sec, 1), "peak": round(SM_COUNT * 16 * sm_hz, 1), "unit": "ex2/s",
           "frac": round(2 * pairs / sec / (SM_COUNT * 16 * sm_hz), 4),
           "peak_kind": "nominal (148 SMs x 16 SFU lanes x max SM clock); no measured SFU peak exists",
           "work": ("%d (voxel, spot) pairs inside the cut-off radius (oracle count) x 2 SFU ex2 + 20 FP32 flops"
                    % pairs) if near else ("%d dense in-range (voxel, spot) pairs (no oracle count: --no-cpu)"
                                            % pairs),
           "pairs_per_s": round(pairs / sec, 1), "kernel_ms": round(r["pb_avg_ms"], 4),
           "fp32": {"achieved_tflops": round(pairs * 20.0 / sec / 1e12, 3), "peak_tflops": round(r["fp32_peak"], 2),
                    "frac": round(pairs * 20.0 / sec / 1e12 / r["fp32_peak"], 4),
                    "peak_kind": "nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock)"},
           "dense": {"pairs": int(r["pairs"]), "pairs_per_s": round(r["pairs"] / sec, 1),
                     "what": "every in-range voxel x every spot of its layer (the reference's evaluated pairs)"},
           "traffic": NCU_TRAFFIC["pencil_beam"][0], "traffic_source": NCU_TRAFFIC["pencil_beam"][1]}
    return out


def stage_rates(prof, nvox, march_samples, fetch_rate):
    """Per-stage rates of one step from the kernel profile: the march's
    samples/s (samples counted by the oracle) against the measured texture
    fetch rate, voxels/s of the per-voxel stages, and the march + smoothing
    compulsory traffic (4 B read + 4 B write per voxel and pass)."""
    out = {}
    for name, (launches, total) in prof.items():
        ms = total / max(launches, 1)
        e = {"kernel_ms": round(ms, 4), "voxels_per_s": round(nvox / (ms * 1e-3), 1)}
        if name == "wet_march" and march_samples:
            rate = march_samples / (ms * 1e-3)
            e.update({"samples": int(march_samples), "samples_per_s": round(rate, 1)})
            if fetch_rate:
                e["texture_frac"] = round(rate / fetch_rate, 4)
                e["texture_peak_kind"] = "measured float2 fetch rate (dc_texture_fetch_rate); the march fetches float"
        if name in ("wet_march", "wet_smooth"):
            e["hbm_gbs_compulsory"] = round(8.0 * nvox / (ms * 1e-3) / 1e9, 2)
        out[name] = e
    return out


def depth_stage(r):
    """The photon radiological-depth pass of one step: its mode, its kernels'
    total time and, for the lattice, the voxels that fell back to the exact
    march."""
    names = [k for k in r["prof_x"] if k.startswith("xray_") or k == "wet_march"]
    ms = sum(r["prof_x"][k][1] / max(r["prof_x"][k][0], 1) for k in names)
    out = {"mode": r["depth_mode"], "kernels": names, "ms": round(ms, 4)}
    if r["depth_mode"] == "lattice" and r["depth_marched"] >= 0:
        out["voxels_marched_exactly"] = int(r["depth_marched"])
        out["marched_frac"] = round(r["depth_marched"] / r["nvox"], 5)
    return out


def main_mine(args):
    import torch
    ws, rank, local = dist_env()
    dist_mod = init_dist(ws, "nccl" if torch.cuda.is_available() else "gloo")
    r = run_mine(args, ws, rank, local, dist_mod)
    batched = run_batched(args, local, dist_mod, ws) if args.batch_plans > 0 else None
    optimisation = run_optimisation(args, local, dist_mod) if args.opt_iters > 0 else None
    surrogate = run_surrogate(args, local, dist_mod) if args.surrogate_beams > 0 else None
    plan_loop = run_plan_loop(args, local, dist_mod) if args.plan_loop else None
    if rank == 0:
        cpu_x = cpu_p = None
        march_x = march_p = None
        if ws == 1 and not args.no_cpu:
            cpu_x, oracle_samples, march_x = cpu_baseline_photon()
            cpu_p, march_p, r["near_pairs"] = cpu_baseline_proton()
            # algorithmic work counted by the oracle (TERMA > 0.01 voxels x cone samples)
            r["achieved_tf"] *= oracle_samples / max(r["samples"], 1)
            r["samples"] = oracle_samples
        pk = r["pk"]
        hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
        tex = texture_roof(local, r["samples"] / (r["cccs_avg_ms"] * 1e-3))
        fetch_rate = tex["peak"] if tex else None
        # this library's kernels per step: the profiled ones (depth pass, TERMA,
        # CCCS) plus the unprofiled one-block cone-direction kernel
        x_launch_per_step = sum(v[0] for v in r["prof_x"].values()) // max(args.steps, 1) + 1
        p_launch_per_step = sum(v[0] for v in r["prof_p"].values()) // max(args.steps, 1)
        line = {
            "metric": "CCCS ms/beam",
            "value": round(r["x_ms_per_beam"], 4),
            "unit": "ms/beam",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(r["t_ms"] / args.steps, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded phantoms; beam-model tables shipped with the reference)",
            "config": {"workload": "photon CCCS small: 128^3 @ 2.5 mm, water + lung block + bone cube, 6 MV "
                                   "10x10 cm MLC field, 100 MU, gantry 0, 72 cone directions",
                       "step": "one control point: ray trace + TERMA + CCCS, density resident in HBM",
                       "l2": "flushed between steps (256 MiB write, outside the timed brackets)",
                       "parallelism": "replicas" if ws > 1 else "single GPU"},
            "e2e": {"value": round(r["e2e_ms"] / (r["n_e2e"] * ws), 4), "unit": "ms/beam", "calls": r["n_e2e"],
                    "h2d_bytes_per_step": int(r["nvox"] * 4), "d2h_bytes_per_step": int(r["nvox"] * 4),
                    "api": "dosecuda_b200.dose_kernels.photon_dose_cuda (host numpy in/out: the pageable density "
                           "array DensityFromHU returns, as the reference's plan loop passes it; the returned "
                           "array page-locked by the call)",
                    "pinned_input": {"value": round(r["e2e_pinned_ms"] / (r["n_e2e"] * ws), 4), "unit": "ms/beam",
                                     "what": "the same call with a page-locked input array"}},
            # The CCCS's binding unit is the texture pipe (one filtered float2
            # fetch per cone sample; L1TEX ~95 % busy under ncu), so the
            # top-level roof is the fetch rate measured on this GPU by
            # dc_texture_fetch_rate; FP32 and HBM fractions are given beside it.
            "roofline": {
                "bound": "texture" if tex else "fp32",
                "kernel": "cccs",
                "achieved": (tex or {}).get("achieved", round(r["achieved_tf"], 3)),
                "peak": (tex or {}).get("peak", round(r["fp32_peak"], 2)),
                "unit": "filtered float2 fetches/s" if tex else "TFLOP/s",
                "frac": (tex or {}).get("frac", round(r["achieved_tf"] / r["fp32_peak"], 4)),
                "peak_kind": (tex or {}).get("peak_kind", "nominal FP32"),
                "work": f"{r['samples']} cone samples (oracle count), one filtered float2 fetch + 1 SFU exp + "
                        f"~18 FP32 flops each",
                "samples_per_s": round(r["samples"] / (r["cccs_avg_ms"] * 1e-3), 1),
                "kernel_ms": round(r["cccs_avg_ms"], 4),
                "fp32": {"achieved_tflops": round(r["achieved_tf"], 3), "peak_tflops": round(r["fp32_peak"], 2),
                         "frac": round(r["achieved_tf"] / r["fp32_peak"], 4),
                         "peak_kind": "nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock); "
                                      "no measured FP32 peak exists"},
                "hbm": {"achieved_gbs": round(r["cccs_bytes"] / (r["cccs_avg_ms"] * 1e-3) / 1e9, 2),
                        "peak_gbs": hbm, "frac": round(r["cccs_bytes"] / (r["cccs_avg_ms"] * 1e-3) / 1e9 / hbm, 5),
                        "peak_kind": r["pk_kind"]},
                # dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture
                # of this kernel on this workload (profiles/cccs_photon_small.md)
                "traffic": NCU_TRAFFIC["cccs"][0],
                "traffic_source": NCU_TRAFFIC["cccs"][1],
            },
            "kernels": {k: {"launches": v[0], "total_ms": round(v[1], 4)} for k, v in r["prof_x"].items()},
            "stages": stage_rates(r["prof_x"], r["nvox"], march_x, fetch_rate),
            "depth_pass": depth_stage(r),
            "cccs_sweep": r["sweep"],
            "gpu_launches": x_launch_per_step * args.steps,
            "clocks": r["clocks"],
            "cpu_baseline": cpu_x,
            "secondary": {
                "metric": "IMPT spots/s",
                "value": round(r["spots_per_s"], 1),
                "unit": "spots/s",
                "higher_is_better": True,
                "ms_per_step": round(r["tp_ms"] / args.steps, 4),
                "config": {"workload": "proton PB small: 96^3 @ 2 mm, water + bone cylinder + lung slab, gantry 0, "
                                       "6 layers (energy ids 34..59) x 100 spots",
                           "step": "one beam: WET ray trace + smoothing + pencil-beam dose, RLSP resident in HBM"},
                "e2e": {"value": round(r["n_spots"] * r["n_e2e"] * ws / (r["pe2e_ms"] * 1e-3), 1), "unit": "spots/s",
                        "calls": r["n_e2e"],
                        "h2d_bytes_per_step": int(r["pnvox"] * 4 * 2), "d2h_bytes_per_step": int(r["pnvox"] * 4 * 2),
                        "api": "dose_kernels.proton_raytrace_cuda + proton_spot_cuda (host numpy: the pageable "
                               "RLSP array RLSPFromHU returns, the WET passed back as a fresh array copy, as "
                               "the reference's plan loop does)",
                        "pinned_input": {"value": round(r["n_spots"] * r["n_e2e"] * ws / (r["pe2e_pinned_ms"] * 1e-3),
                                                        1), "unit": "spots/s",
                                         "what": "the same calls with a page-locked RLSP array"}},
                "roofline": pencil_beam_roofline(r),
                "kernels": {k: {"launches": v[0], "total_ms": round(v[1], 4)} for k, v in r["prof_p"].items()},
                "stages": stage_rates(r["prof_p"], r["pnvox"], march_p, fetch_rate),
                "gpu_launches": p_launch_per_step * args.steps,
                "cpu_baseline": cpu_p,
            },
            "batched": batched,
            "optimisation": optimisation,
            "surrogate": surrogate,
            "plan_loop": plan_loop,
        }
        print(json.dumps(line))
    if dist_mod is not None:
        dist_mod.destroy_process_group()


def load_reference_extension():
    """The reference's own compiled ``dose_kernels`` extension: the one the
    reference's package build installed into baseline/_ref (its CMake build,
    `pip install --target baseline/_ref`), else the same sources built by
    oracle/build_ref.sh into oracle/_ref.  Returns (module, where)."""
    import importlib.machinery
    import importlib.util
    for where in (os.path.join("baseline", "_ref", "DoseCUDA"), os.path.join("oracle", "_ref")):
        hits = sorted(glob.glob(os.path.join(ROOT, where, "dose_kernels*.so")))
        if hits:
            loader = importlib.machinery.ExtensionFileLoader("dose_kernels", hits[0])
            spec = importlib.util.spec_from_file_location("dose_kernels", hits[0], loader=loader)
            mod = importlib.util.module_from_spec(spec)
            loader.exec_module(mod)
            return mod, os.path.relpath(hits[0], ROOT)
    return None, None


# ----------------------------------------------------------------------------
def main_reference(args):
    """The reference DoseCUDA CUDA extension through its own API, same inputs."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    ref, ref_origin = load_reference_extension()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "no reference build: neither baseline/_ref (pip install "
                                                               "of the reference) nor oracle/_ref (oracle/build_ref.sh)"}))
        return
    from dosecuda_b200.plan import VolumeObject

    grid, model, cp, density = photon_workload()
    vol = VolumeObject()
    vol.voxel_data = np.ascontiguousarray(density)
    vol.origin = np.array(grid.origin, dtype=np.single)
    vol.spacing = np.array(grid.spacing, dtype=np.single)
    for _ in range(args.warmup):
        ref.photon_dose_cuda(model, vol, cp, local)
    n_calls = max(args.steps, 30)  # as the end-to-end legs of this engine's arm
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(n_calls):
            ref.photon_dose_cuda(model, vol, cp, local)
        x_ms = (time.perf_counter() - t0) * 1e3 / n_calls

    pgrid, pmodel, pbeam, rlsp = proton_workload()
    pvol = VolumeObject()
    pvol.voxel_data = np.ascontiguousarray(rlsp)
    pvol.origin = np.array(pgrid.origin, dtype=np.single)
    pvol.spacing = np.array(pgrid.spacing, dtype=np.single)

    def beam_step():
        # the reference's plan loop (plan_impt.py:124-160): WET, then the dose
        # from a fresh array copy of it, as this engine's end-to-end leg does
        w = ref.proton_raytrace_cuda(pmodel, pvol, pbeam, local)
        wv = VolumeObject()
        wv.voxel_data, wv.origin, wv.spacing = np.array(w, dtype=np.single), pvol.origin, pvol.spacing
        ref.proton_spot_cuda(pmodel, pvol, wv, pbeam, local)

    for _ in range(args.warmup):
        beam_step()
    t0 = time.perf_counter()
    for _ in range(n_calls):
        beam_step()
    p_s = (time.perf_counter() - t0) / n_calls
    n_spots = pbeam.spot_list.shape[0]

    batched = None
    if args.batch_plans > 0:
        # the batched workload as the reference computes it: one call per beam,
        # its WET kept between calls (computeIMPTPlanFromWET, plan_impt.py:192-211)
        from dosecuda_b200 import phantoms
        from dosecuda_b200.plan_impt import IMPTPlan
        bmodel = IMPTPlan().beam_models[0]
        calls = []
        for seed in range(args.batch_plans):
            grid, beams, _ = phantoms.batch_plan(seed, model=bmodel)
            rv = VolumeObject()
            rv.voxel_data = grid.RLSPFromHU("HitachiProbeatJHU")
            rv.origin = np.asarray(grid.origin, np.float32)
            rv.spacing = np.asarray(grid.spacing, np.float32)
            for bm in beams:
                wv = VolumeObject()
                wv.voxel_data = ref.proton_raytrace_cuda(bmodel, rv, bm, local)
                wv.origin, wv.spacing = rv.origin, rv.spacing
                calls.append((rv, wv, bm))
        ref.proton_spot_cuda(bmodel, *calls[0][:2], calls[0][2], local)  # warm-up
        t0 = time.perf_counter()
        for rv, wv, bm in calls:
            ref.proton_spot_cuda(bmodel, rv, wv, bm, local)
        t_calls = (time.perf_counter() - t0) * 1e3
        batched = {"metric": "batched IMPT dose: ms per optimisation iteration (all plans)",
                   "value": round(t_calls, 3), "unit": "ms/iteration", "higher_is_better": False,
                   "config": {"workload": "%d plans x 256x256x160 (same seeds as the engine's line), %d beams; "
                                          "the reference uses spacing[0] on all axes" % (args.batch_plans, len(calls)),
                              "iteration": "one proton_spot_cuda call per beam, WET reused"}}

    plan_loop = run_plan_loop(args, local, None, dose_kernels_module=ref) if args.plan_loop else None

    line = {
        "impl": "reference",
        "metric": "CCCS ms/beam",
        "value": round(x_ms, 4),
        "unit": "ms/beam",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(x_ms, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded phantoms; beam-model tables shipped with the reference)",
        "config": {"workload": "photon CCCS small: 128^3 @ 2.5 mm, water + lung block + bone cube, 6 MV "
                               "10x10 cm MLC field, 100 MU, gantry 0, 72 cone directions",
                   "step": "one control point through the reference's dose_kernels.photon_dose_cuda",
                   "parallelism": "single GPU"},
        "e2e": {"value": round(x_ms, 4), "unit": "ms/beam", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "calls": n_calls},
        "cpu_baseline": {"value": round(x_ms, 4), "unit": "ms/beam", "cores": 1, "kind": "reference",
                         "sample": "the reference's own implementation is CUDA-only: its extension (%s) built from "
                                   "the reference sources for sm_100a, run on the B200 through its Python API with "
                                   "host numpy buffers (its per-call allocation and copies included)" % ref_origin},
        "reference_build": ref_origin,
        "clocks": clk.summary(),
        "secondary": {"metric": "IMPT spots/s", "value": round(n_spots / p_s, 1), "unit": "spots/s",
                      "higher_is_better": True, "ms_per_step": round(p_s * 1e3, 4),
                      "e2e": {"value": round(n_spots / p_s, 1), "unit": "spots/s", "calls": n_calls}},
        "batched": batched,
        "plan_loop": plan_loop,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--batch-plans", type=int, default=16, help="plans in the batched workload (0: skip)")
    ap.add_argument("--no-batch-csr", dest="batch_csr", action="store_false",
                    help="skip the batched workload's influence matrices")
    ap.add_argument("--opt-iters", type=int, default=200, help="optimisation iterations (0: skip)")
    ap.add_argument("--tune-cache", action="store_true", help="keep the tile autotuner's JSON cache")
    ap.add_argument("--surrogate-beams", type=int, default=300, help="held-out beams for the surrogate (0: skip)")
    ap.add_argument("--no-plan-loop", dest="plan_loop", action="store_false",
                    help="skip the 18-control-point IMRT plan")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        main_reference(args)
    else:
        main_mine(args)


if __name__ == "__main__":
    main()
