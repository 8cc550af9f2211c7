"""Benchmark of the batched orientation search (CC evaluations per second).

Workload (one step): the 64^3 share of the batched uneven-alignment configuration --
1,200 synthetic 64^3 subtomograms, each searched over 256 local orientations within 8
degrees of its own seeded prior, peak radius 7, in one emc_search_run call (one CUDA graph).
307,200 CC evaluations per step per GPU.  The single-subtomogram plain search (one particle,
540 orientations on the 10 degree grid) is timed beside it and reported under "plain".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--particles P]

Under torchrun every rank runs its own full batch (weak scaling, no collective on the
data path); the step time is the max over ranks.  `--impl reference` times the
single-precision CPU port of the reference path (oracle/liboracle_f32.so) on all host
cores over a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BOX = 64
N_ORIENT = 256
PEAK_RADIUS = 7


def particle_bytes(n):
    """Per-particle input of the search: the particle spectrum (8 nh n^2) and its wedge.CTF weight
    wdgMask (4 nh n^2), read by every orientation of the particle (from L2 after the first)."""
    nh = n // 2 + 1
    return 12 * nh * n * n


def reference_bytes(n, store="f32"):
    """Per-reference input: the trilinear corner cells ((n+1)^3 x 32 B FP32 / 16 B BF16) and the
    real-space mask (4 n^3)."""
    return (n + 1) ** 3 * (32 if store == "f32" else 16) + 4 * n ** 3


def compulsory_bytes(n, evals, particles, references=1, store="f32"):
    """Compulsory HBM bytes of a launch that evaluates `evals` (particle, orientation) pairs of
    `particles` distinct particles: every input read once, 16 B written per evaluation."""
    return particles * particle_bytes(n) + references * reference_bytes(n, store) + 16 * evals


def bytes_per_eval(n):
    """Compulsory bytes per CC evaluation with N_ORIENT orientations per particle, the reference's share
    left out (it is read once per launch of hundreds of evaluations)."""
    return particle_bytes(n) / N_ORIENT + 16


def flops_per_eval(n):
    return 2 * 2.5 * n ** 3 * math.log2(n ** 3) + 30 * n ** 3 + 8 * (n // 2 + 1) * n * n


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
def build_batch(seed, n_particles):
    """Host (pinned) particle volumes and weights plus search descriptors for one rank."""
    import torch

    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(seed)
    ref = synthetic.blob_reference(rng, BOX)
    mask = synthetic.soft_sphere_mask(BOX, 28)
    grid = synthetic.local_grid(N_ORIENT, 8.0, 2.0)
    ref_g = torch.from_numpy(ref).cuda()
    parts = torch.empty((n_particles, BOX, BOX, BOX), dtype=torch.float32).pin_memory()
    weights = torch.empty((n_particles, BOX, BOX, BOX // 2 + 1), dtype=torch.float32).pin_memory()
    priors = []
    ft = api.FourierTransformer((BOX, BOX, BOX))
    for i in range(n_particles):
        prior = api.define_matrix(synthetic.random_euler(rng), "inv")
        jitter = api.define_matrix([rng.uniform(-6, 6), rng.uniform(0, 6), rng.uniform(-6, 6)], "inv")
        truth = prior @ jitter
        shift = rng.integers(-4, 5, 3)
        w = api.wedge_ctf_weight(BOX, -rng.uniform(50, 65), rng.uniform(50, 65),
                                 synthetic.ctf_dict(rng.uniform(15000, 40000)))
        p = synthetic.make_particle(ref_g, rng, truth, shift, w, 0.1, ft=ft)
        parts[i].copy_(p)
        weights[i].copy_(w)
        priors.append(prior)
    return dict(ref=ref_g, mask=torch.from_numpy(mask).cuda(), grid=grid, parts=parts, weights=weights,
                priors=priors, ref_np=ref, mask_np=mask)


def run_ours(args, world, rank, local):
    import torch

    from emclarity_b200 import api
    n = args.particles
    b = build_batch(1000 + rank, n)
    s = api.Search(peak_radius=PEAK_RADIUS, chunk_evals=args.chunk)
    if args.planes:
        s.set_planes(BOX, args.planes)
    if args.overlap:
        s.set_overlap(args.overlap)
    rid = s.add_reference(b["ref"], b["mask"])
    s.set_orientations(b["grid"])
    d_parts = b["parts"].cuda()
    d_w = b["weights"].cuda()
    d_w2 = torch.empty_like(d_w)
    spec = torch.empty((n, BOX, BOX, BOX // 2 + 1), dtype=torch.complex64, device="cuda")
    energy = torch.zeros(n, dtype=torch.float64, device="cuda")
    for i in range(n):
        L_call_spectrum(api, d_parts[i], None, spec[i], energy[i:i + 1])
    torch.cuda.synchronize()
    en = energy.cpu().numpy()
    # each particle's wedge.CTF weight is the CC's wdgMask, applied to the rotated reference
    # (BH_multi_xcf_Translational_2.m:35-38 with BH_multi_xcf_Rotational's binding)
    descs = [s.particle(spec[i], en[i], rid, prior=b["priors"][i], orient_count=N_ORIENT, wedge=d_w[i])
             for i in range(n)]
    descs_b = [s.particle(spec[i], en[i], rid, prior=b["priors"][i], orient_count=N_ORIENT, wedge=d_w2[i])
               for i in range(n)]
    evals = n * N_ORIENT
    cc = torch.empty(evals, device="cuda")
    best = torch.empty((n, 5), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        s.run(descs, cc=cc, best=best)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # ---------------- timed region: device-resident inputs, graph replay
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms_local = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms_local, world)
    device_best = best.cpu().clone()
    launches_per_step = s.timings()["launches_last_run"]

    # ---------------- per-pass device times (eager launches bracketed by CUDA events)
    s.set_profiling(True)
    s.timings(reset=True)
    torch.cuda.synchronize()
    for _ in range(max(1, min(args.steps, 3))):
        step()
    torch.cuda.synchronize()
    prof = s.timings(reset=True)
    s.set_profiling(False)

    # ---------------- end to end: pinned host volumes -> spectra -> search -> host results.
    # Every step copies its particles and weights from pinned host memory (on a copy stream, into
    # one of two device buffers), computes their spectra and energies, runs the search with the
    # energies read on the device (emc_search_run_energies: no host round trip between spectra and
    # search) and reads the best hits back.  Step k+1's copy overlaps step k's search.
    h_best = torch.empty((n, 5), dtype=torch.int32).pin_memory()
    h2d = b["parts"].numel() * 4 + b["weights"].numel() * 4
    d2h = h_best.numel() * 4
    in_bufs = [(d_parts, d_w), (torch.empty_like(d_parts), d_w2)]
    slot_descs = [descs, descs_b]  # the search reads the weights of the buffer its step copied into
    copy_stream = torch.cuda.Stream()
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]

    def issue_copy(k):
        slot = k % 2
        copy_stream.wait_event(consumed[slot])  # the spectra that last read this buffer are done
        with torch.cuda.stream(copy_stream):
            pa, wa = in_bufs[slot]
            pa.copy_(b["parts"], non_blocking=True)
            wa.copy_(b["weights"], non_blocking=True)
            copied[slot].record(copy_stream)

    def e2e_compute(k):
        slot = k % 2
        stream.wait_event(copied[slot])
        pa, wa = in_bufs[slot]
        api.particle_spectra(pa, out=spec, energies=energy)  # one batched call for the step
        s.run(slot_descs[slot], cc=cc, best=best, energies=energy)
        consumed[slot].record(stream)
        h_best.copy_(best, non_blocking=True)

    def e2e_steps(k_steps):
        copy_stream.wait_stream(stream)
        issue_copy(0)
        for k in range(k_steps):
            if k + 1 < k_steps:
                issue_copy(k + 1)
            e2e_compute(k)

    e2e_steps(2)  # warm-up: records the search graph of the device-energy variant
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    if not torch.equal(h_best, device_best):
        raise RuntimeError("end-to-end hits differ from the device-resident run")
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)

    # ---------------- plain single-subtomogram search (C0 shape), timed the same way
    plain = run_plain(args, api)

    value = world * evals / (ms / 1e3)
    res = {
        "metric": "CC evals/s at 64^3 (batched)",
        "value": value,
        "unit": "CC evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "batched alignment, 64^3 share: %d particles x %d local orientations (8 deg of a "
                               "seeded prior), peak radius %d, one emc_search_run (CUDA graph) per step" %
                               (n, N_ORIENT, PEAK_RADIUS),
                   "box": BOX, "particles_per_gpu": n, "orientations": N_ORIENT, "evals_per_step_per_gpu": evals,
                   "l2": "inputs larger than L2 (%.2f GB of particle spectra per GPU)" % (spec.numel() * 8 / 1e9),
                   "chunk_overlap_slots": args.overlap or 2, "chunk_evals": args.chunk or "library default",
                   "parallelism": "replicas%d" % world},
        "e2e": {"value": world * evals / (e2e_ms / 1e3), "unit": "CC evals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
                "path": "pinned host volumes + weights (copy stream, two device buffers) -> emc_particle_spectra "
                        "-> emc_search_run_energies (energies read on the device, the buffer's weights as "
                        "wdgMask) -> host hits; step k+1's copy overlaps step k's search; hits checked equal to "
                        "the device-resident run"},
        "gpu_launches": int(launches_per_step * args.steps),
        "plain": plain,
    }
    res["clocks"] = clk.summary()
    res["roofline"], res["passes"] = roofline(prof, res["clocks"])
    g, g_ms = s.planes(BOX)
    res["passes"]["fwd_xy"]["planes_per_cta"] = {"chosen": g, "tuning_ms_per_launch": g_ms}
    return res


def L_call_spectrum(api, part, w, q, e):
    """emc_particle_spectrum into preallocated buffers."""
    import ctypes as C

    from emclarity_b200 import _lib as L
    n = part.shape[-1]
    L.call("emc_particle_spectrum", n, C.c_void_p(part.data_ptr()), C.c_void_p(w.data_ptr()) if w is not None else None,
           None, C.c_void_p(q.data_ptr()), C.c_void_p(e.data_ptr()), api._stream())


def profiled_traffic():
    """DRAM bytes per CC evaluation from the committed ncu summary (None if absent)."""
    p = os.path.join(ROOT, "profiles", "search_batched64_passes.md")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_evaluation:"):
                    return float(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


def roofline(prof, clocks=None):
    """HBM roofline of the fused search on the compulsory-traffic model: per launch (one chunk of the
    three passes) the distinct particles' spectra and weights, the reference's cells and mask, and
    16 B per evaluation, over the measured per-launch device time.  The passes are bound on chip
    (shared memory, L1, issue), so the FP32 rate of the nominal FFT flop count is reported beside it
    against the nominal FP32 CUDA-core peak at the sampled SM clock."""
    peak, which = measured_peaks()
    nl = max(1, prof["launches"]["fwd_xy"])
    per_launch_ms = (prof["ms"]["fwd_xy"] + prof["ms"]["z_mul"] + prof["ms"]["inv_peak"]) / nl
    evals_per_launch = prof["evals"] / nl
    b = compulsory_bytes(BOX, evals_per_launch, evals_per_launch / N_ORIENT + 1)
    achieved = b / (per_launch_ms / 1e3) / 1e9
    passes = {k: {"ms_total": v, "launches": prof["launches"][k],
                  "us_per_launch": 1e3 * v / max(1, prof["launches"][k])} for k, v in prof["ms"].items()}
    total = sum(prof["ms"].values())
    for k in passes:
        passes[k]["share"] = prof["ms"][k] / total if total else None
    per_eval = profiled_traffic()
    traffic = per_eval * evals_per_launch if per_eval else None
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    fp32 = flops_per_eval(BOX) * evals_per_launch / (per_launch_ms / 1e3) / 1e12
    return ({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
             "peak_source": which + " (MEASURED_PEAKS.json hbm_gbs)" if which == "measured" else which,
             "traffic": traffic, "traffic_algorithmic": b,
             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per CC evaluation of a full "
                               "chunk (profiles/search_batched64_passes.md) x evaluations per launch"
                               if traffic else None,
             "model": "compulsory bytes per launch: distinct particles x (8 + 4) nh n^2 (spectrum + wdgMask) + "
                      "reference cells (n+1)^3 x 32 + mask 4 n^3 + 16 B per evaluation",
             "kernel": "fused search pipeline (fwd_xy + z_mul + inv_peak per chunk)",
             "compulsory_bytes_per_eval": b / evals_per_launch, "evals_per_launch": evals_per_launch,
             "us_per_launch": per_launch_ms * 1e3,
             "compute": {"unit": "TFLOP/s", "achieved": fp32, "peak": fp32_peak, "frac": fp32 / fp32_peak,
                         "flops_per_eval": flops_per_eval(BOX),
                         "peak_source": "nominal FP32 CUDA-core peak: 148 SMs x 128 lanes x 2 x %.0f MHz" % mhz}},
            passes)


def run_plain(args, api):
    """One particle, 540 orientations (10 degree grid), timed with CUDA events."""
    import torch

    from emclarity_b200 import synthetic
    case = synthetic.PlainCase(seed=11)
    g = case.to_gpu()
    q, e = api.particle_spectrum(g["particle"])
    s = api.Search(peak_radius=case.peak_radius)
    rid = s.add_reference(g["ref"], g["mask"])
    s.set_orientations(case.grid)
    d = [s.particle(q, e.item(), rid, orient_count=len(case.grid), wedge=g["weight"])]
    best = torch.empty((1, 5), dtype=torch.int32, device="cuda")
    for _ in range(max(3, args.warmup)):
        s.run(d, best=best)
    torch.cuda.synchronize()
    reps = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        s.run(d, best=best)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    s.close()
    return {"workload": "1 particle x %d orientations (C1 eulerSearch 40/10/40/10), 64^3" % len(case.grid),
            "ms_per_search": ms, "value": len(case.grid) / (ms / 1e3), "unit": "CC evals/s"}


# ---------------------------------------------------------------------------------------------
def _cpu_case():
    """One 64^3 particle of the default workload's shape (reference, mask, particle spectrum,
    wedge weight) and the local orientation grid, for the CPU arms."""
    from emclarity_b200 import synthetic
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    ref = synthetic.blob_reference(rng, BOX)
    mask = synthetic.soft_sphere_mask(BOX, 28)
    part = (np.roll(ref, 2, axis=0) + rng.standard_normal(ref.shape)).astype(np.float32)
    q, _ = O.particle_spectrum(part, precision="f32")
    wdg = O.even_weight_np(rng, BOX)[:, :, : BOX // 2 + 1].astype(np.float32)  # wdgMask operand
    grid = synthetic_local_grid_np()
    mats = [O.define_matrix([p, t, s - p], "inv") for p, t, s in grid]
    return ref, mask, q, wdg, mats


def cpu_rates(seconds=12.0):
    """The two CPU arms of the baseline on a bounded sample of the workload (one 64^3 particle over the
    local grid): the single-precision C port of the reference path (liboracle_f32.so, OpenMP over
    orientations on every host core) and the numpy / scipy.fft (pocketfft) restatement in one spawned
    process per host core.  Returns {arm: (evals/s, cores, sample description)} and the faster arm."""
    from oracle import oracle as O
    from oracle import pocketfft_arm as PF
    cores = os.cpu_count() or 1
    ref, mask, q, wdg, mats = _cpu_case()
    out = {}
    per = max(cores, 8)
    O.search(ref, q, mats[:per], mask=mask, wdg_mask=wdg, radius=PEAK_RADIUS, nthreads=cores, precision="f32")
    done, t0 = 0, time.time()
    while time.time() - t0 < seconds:
        sl = [mats[(done + k) % len(mats)] for k in range(per)]
        O.search(ref, q, sl, mask=mask, wdg_mask=wdg, radius=PEAK_RADIUS, nthreads=cores, precision="f32")
        done += per
    dt = time.time() - t0
    out["c_port"] = (done / dt, cores, "C port (FP32, OpenMP, %d threads): %d CC evaluations of one 64^3 particle "
                                       "over the local grid in %.1f s" % (cores, done, dt))
    with PF.Pool(ref, q, mask=mask, wdg_mask=wdg, radius=PEAK_RADIUS, processes=cores) as pool:
        pool.search(mats[:2 * cores])  # workers started and warm
        per = 4 * cores
        done, t0 = 0, time.time()
        while time.time() - t0 < seconds:
            pool.search([mats[(done + k) % len(mats)] for k in range(per)])
            done += per
        dt = time.time() - t0
    out["pocketfft"] = (done / dt, cores, "numpy + scipy.fft (pocketfft) in %d spawned processes: %d CC evaluations "
                                          "of one 64^3 particle over the local grid in %.1f s" % (cores, done, dt))
    best = max(out, key=lambda k: out[k][0])
    return out, best


def cpu_baseline_entry(seconds=12.0):
    rates, best = cpu_rates(seconds)
    r, cores, sample = rates[best]
    return {"value": r, "unit": "CC evals/s", "cores": cores, "kind": "port", "arm": best, "sample": sample,
            "cpu_model": _cpu_model(),
            "arms": {k: {"value": v[0], "cores": v[1], "sample": v[2]} for k, v in rates.items()}}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def synthetic_local_grid_np():
    from oracle import oracle as O
    g = O.euler_search_np("C1", 8.0, 2.0, 8.0, 2.0)
    mats = np.array([O.define_matrix([p, t, s - p], "inv") for p, t, s in g])
    ang = np.degrees(np.arccos(np.clip((np.trace(mats, axis1=1, axis2=2) - 1) / 2, -1, 1)))
    order = np.argsort(ang, kind="stable")[:N_ORIENT]
    return g[np.sort(order)]


def run_reference(args, world, rank):
    """The reference arm: the reference path's CPU implementation on the host cores.  The reference's
    own CPU path is MATLAB (absent here), so each step times both CPU restatements of it (the C port
    and the pocketfft arm) on a bounded sample of the workload and reports the faster."""
    if rank != 0:
        return None
    per_step = max(2.0, min(10.0, 60.0 / max(1, args.steps)))
    cpu_rates(seconds=1.0)  # warm-up
    steps = []
    for _ in range(args.steps):
        rates, best = cpu_rates(seconds=per_step)
        steps.append((rates, best))
    arms = {k: float(np.mean([r[k][0] for r, _ in steps])) for k in steps[0][0]}
    best = max(arms, key=arms.get)
    v = arms[best]
    cores = steps[-1][0][best][1]
    return {
        "metric": "CC evals/s at 64^3 (batched)", "value": v, "unit": "CC evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 2e3 * per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": "batched alignment, 64^3 share (bounded CPU sample: one particle over the local "
                               "grid per step, both CPU arms)", "box": BOX, "orientations": N_ORIENT,
                   "peak_radius": PEAK_RADIUS},
        "cpu_baseline": {"value": v, "unit": "CC evals/s", "cores": cores, "kind": "port", "arm": best,
                         "sample": steps[-1][0][best][2], "cpu_model": _cpu_model(), "arms": arms},
        "e2e": {"value": v, "unit": "CC evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# --------------------------------------------------------------------------------------------- other workloads
def _timed(fn, reps=1):
    import torch
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(reps):
        out = fn()
    torch.cuda.synchronize()
    return (time.time() - t0) / reps, out


def mixed_batch(n_part, seed=2024):
    """The batched uneven configuration: n_part particles split 60/30/10 over 64^3 / 96^3 / 128^3 in a
    seeded order, each made like the plain case with a seeded defocus in [1.5, 4] um, tilt range
    +/-U[50, 65] deg, SNR 0.1, and a truth within 8 degrees of a seeded prior.  Returns host-side
    records (box, prior, truth, shift) and device particles / wedges / references."""
    import torch

    from emclarity_b200 import api, synthetic
    sizes = synthetic.batched_sizes(n_part, seed=3)
    rng = np.random.default_rng(seed)
    refs, fts = {}, {}
    for n in (64, 96, 128):
        ref = synthetic.blob_reference(rng, n)
        mask = synthetic.soft_sphere_mask(n, 28 * n / 64)
        refs[n] = (ref, mask, torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda())
        fts[n] = api.FourierTransformer((n, n, n))
    parts = []
    for n in sizes:
        n = int(n)
        prior = api.define_matrix(synthetic.random_euler(rng), "inv")
        truth = prior @ api.define_matrix([rng.uniform(-6, 6), rng.uniform(0, 6), rng.uniform(-6, 6)], "inv")
        shift = rng.integers(-4, 5, 3)
        w = api.wedge_ctf_weight(n, -rng.uniform(50, 65), rng.uniform(50, 65),
                                 synthetic.ctf_dict(rng.uniform(15000, 40000)))
        p = synthetic.make_particle(refs[n][2], rng, truth, shift, w, 0.1, ft=fts[n])
        q, e = api.particle_spectrum(p)
        parts.append(dict(n=n, prior=prior, truth=truth, shift=shift, wedge=w, spec=q, energy=e.item(),
                          particle=p))
    return sizes, refs, parts


def time_mixed(parts, refs, store, steps, warmup, grid, overlap=0):
    """One emc_search_run over every particle of the batch with the reference stored as `store`."""
    import torch

    from emclarity_b200 import api
    s = api.Search(peak_radius=PEAK_RADIUS)
    if overlap:
        s.set_overlap(overlap)
    rids = {n: s.add_reference(refs[n][2], refs[n][3], store=store) for n in (64, 96, 128)}
    s.set_orientations(grid)
    descs = [s.particle(p["spec"], p["energy"], rids[p["n"]], prior=p["prior"], orient_count=len(grid),
                        wedge=p["wedge"]) for p in parts]
    best = torch.empty((len(descs), 5), dtype=torch.int32, device="cuda")
    for _ in range(warmup):
        s.run(descs, best=best)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        s.run(descs, best=best)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = s.timings()["launches_last_run"]
    s.close()
    return ms, launches, best.cpu().numpy()


def mixed_entry(sizes, parts, refs, store, steps, warmup, grid, overlap=0):
    ms, launches, _ = time_mixed(parts, refs, store, steps, warmup, grid, overlap)
    evals = len(parts) * len(grid)
    counts = {n: int(np.sum(sizes == n)) for n in (64, 96, 128)}
    byts = sum(compulsory_bytes(n, c * len(grid), c, 1, store) for n, c in counts.items())
    peak, which = measured_peaks()
    return {"metric": "CC evals/s, batched uneven boxes" + (" (BF16 reference storage)" if store == "bf16" else ""),
            "value": evals / (ms / 1e3), "unit": "CC evals/s", "steps": steps, "warmup": warmup, "ms_per_step": ms,
            "dtype": store, "gpu_launches_per_step": launches,
            "config": {"workload": "%d particles (%s) x %d local orientations (8 deg of a seeded prior), peak radius "
                                   "%d, one emc_search_run (CUDA graph) per step" % (len(parts), counts, len(grid),
                                                                                      PEAK_RADIUS), "store": store},
            "roofline": {"bound": "hbm", "achieved": byts / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": byts / (ms / 1e3) / 1e9 / peak, "peak_source": which,
                         "model": "compulsory bytes: particles x (8 + 4) nh n^2 + references' cells and masks + 16 B "
                                  "per evaluation"}}


def bf16_report(sizes, refs, parts, grid, n_sub=200, orient_stride=16):
    """Mixed precision against the FP64 oracle: over a seeded subset of n_sub particles (every box size
    in its share) and every orient_stride-th orientation of the local grid, the CCs and best
    orientations of the search with BF16 reference storage (and with FP32 storage, as the control)
    against the FP64 oracle on the unrounded reference."""
    import torch

    from emclarity_b200 import api
    from oracle import oracle as O
    rng = np.random.default_rng(200)
    sub = np.sort(rng.choice(len(parts), size=min(n_sub, len(parts)), replace=False))
    g = grid[::orient_stride]
    out = {}
    orc = []
    for i in sub:
        p = parts[i]
        ref, mask = refs[p["n"]][0], refs[p["n"]][1]
        P, _ = O.particle_spectrum(p["particle"].cpu().numpy())
        cc, pk = O.search(ref, P, api.search_matrices(g, p["prior"]), mask=mask, wdg_mask=p["wedge"].cpu().numpy(),
                          radius=PEAK_RADIUS)
        orc.append((cc, pk))
    for store in ("bf16", "f32"):
        s = api.Search(peak_radius=PEAK_RADIUS)
        rids = {n: s.add_reference(refs[n][2], refs[n][3], store=store) for n in (64, 96, 128)}
        s.set_orientations(g)
        descs = [s.particle(parts[i]["spec"], parts[i]["energy"], rids[parts[i]["n"]], prior=parts[i]["prior"],
                            orient_count=len(g), wedge=parts[i]["wedge"]) for i in sub]
        cc_g, pk_g, best = s.run_host(descs)
        s.close()
        cc_g = cc_g.reshape(len(sub), len(g))
        rel = np.concatenate([np.abs(cc_g[k] - orc[k][0]) / np.abs(orc[k][0]) for k in range(len(sub))])
        agree, near, ang = 0, 0, []
        for k in range(len(sub)):
            b_o = int(np.argmax(orc[k][0]))
            b_g = best[k][1]
            if b_g == b_o:
                agree += 1
            else:
                gap = abs(orc[k][0][b_g] - orc[k][0][b_o]) / abs(orc[k][0][b_o])
                near += gap <= 1e-3
                Ra = api.search_matrices([g[b_g]], parts[sub[k]]["prior"])[0]
                Rb = api.search_matrices([g[b_o]], parts[sub[k]]["prior"])[0]
                ang.append(float(np.degrees(np.arccos(np.clip((np.trace(Ra.T @ Rb) - 1) / 2, -1, 1)))))
        pk_agree = float(np.mean([np.array_equal(pk_g[k * len(g) + int(np.argmax(orc[k][0]))],
                                                 orc[k][1][int(np.argmax(orc[k][0]))]) for k in range(len(sub))]))
        out[store] = {"cc_rel_err_median": float(np.median(rel)), "cc_rel_err_p99": float(np.percentile(rel, 99)),
                      "cc_rel_err_max": float(rel.max()), "best_orientation_agreement": agree / len(sub),
                      "disagreements_within_1e-3_of_the_oracle_best": int(near),
                      "disagreement_angles_deg": ang, "peak_agreement_at_oracle_best": pk_agree}
    counts = {n: int(np.sum(np.array([parts[i]["n"] for i in sub]) == n)) for n in (64, 96, 128)}
    return {"particles": len(sub), "boxes": counts, "orientations_per_particle": len(g),
            "oracle": "FP64 CPU oracle on the unrounded (FP32) reference", **out}


def run_mixed(args, store="f32"):
    """Batched uneven alignment: 60% 64^3, 30% 96^3, 10% 128^3, 256 local orientations each, seeded
    defocus in [1.5, 4] um and tilt range in [+-50, +-65] deg, one emc_search_run per step.  With BF16
    storage, the report against the FP64 oracle on a 200-particle subset is added."""
    from emclarity_b200 import synthetic
    n_part = args.particles if args.particles != 1200 else 2000
    grid = synthetic.local_grid(N_ORIENT, 8.0, 2.0)
    sizes, refs, parts = mixed_batch(n_part)
    res = mixed_entry(sizes, parts, refs, store, args.steps, args.warmup, grid, args.overlap)
    res.update({"n_gpus": 1, "higher_is_better": True, "data": "synthetic"})
    if store == "bf16":
        res["vs_fp64_oracle"] = bf16_report(sizes, refs, parts, grid)
    return res


def run_tsearch(args):
    """Template search: 512x512x256 noise tomogram with 150 planted 48^3 copies, wedge + CTF (3 um),
    every orientation of eulerSearch(C1, 180, 12, 48, 12) (2,592) over the full volume."""
    import torch

    from emclarity_b200 import api, synthetic
    rng = np.random.default_rng(77)
    nz, ny, nx = 256, 512, 512
    t = 48
    tmpl = synthetic.blob_reference(rng, t)
    grid = api.euler_search("C1", 180, 12, 48, 12)
    if args.particles != 1200:
        grid = grid[:args.particles]
    tomo = torch.randn((nz, ny, nx), device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    tg = torch.from_numpy(tmpl).cuda()
    ip = api.Interpolator(tg)
    placed = []
    tries = 0
    while len(placed) < 150 and tries < 100000:
        tries += 1
        c = rng.integers([t, t, t], [nz - t, ny - t, nx - t])
        if all(np.sum((c - q) ** 2) >= t * t for q in placed):
            placed.append(c)
    for c in placed:
        o = grid[rng.integers(len(grid))]
        rot = ip.interp3d(api.define_matrix([o[0], o[1], o[2] - o[0]], "forward"), (0, 0, 0), "forward")
        z, y, x = (int(v) - t // 2 for v in c)
        tomo[z:z + t, y:y + t, x:x + t] -= 2.0 * rot
    ts = api.TemplateSearch(tomo.contiguous())
    peak = torch.empty_like(tomo)
    ang = torch.empty_like(tomo)
    ts.run(tg, grid[:4], peak, ang)
    dt, _ = _timed(lambda: ts.run(tg, grid, peak, ang))
    per_orient = dt / len(grid)
    byts = 8 * (nx // 2 + 1) * ny * nz + 16 * nx * ny * nz + 4 * t ** 3
    pk, which = measured_peaks()
    return {"metric": "template search orientations/s over 512x512x256", "value": len(grid) / dt,
            "unit": "orientations/s", "n_gpus": 1, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "512x512x256 tomogram, 150 planted 48^3 templates, %d orientations" % len(grid)},
            "roofline": {"bound": "hbm", "achieved": byts / per_orient / 1e9, "peak": pk, "unit": "GB/s",
                         "frac": byts / per_orient / 1e9 / pk, "peak_source": which}}


def run_average(args):
    """Subtomogram averaging (the accumulation loop of BH_average3d): P extracted 64^3 windows holding
    noisy rotated, shifted copies of a reference, seeded rotations / subvoxel shifts / peak weights,
    alternating half sets, 8 tilt-group wedge weights (64^3), C1.  One step = reset + add all P + read
    both half-set averages."""
    import torch

    from emclarity_b200 import api, synthetic
    from oracle import oracle as O
    n = nw = 64
    P = args.particles if args.particles != 1200 else 1024
    rng = np.random.default_rng(99)
    ref = synthetic.blob_reference(rng, n)
    ip = api.Interpolator(torch.from_numpy(ref).cuda(), interp="linear_border")
    d_parts = torch.empty((P, n, n, n), dtype=torch.float32, device="cuda")
    rots, shifts = [], []
    gen = torch.Generator(device="cuda").manual_seed(11)
    for i in range(P):
        R = api.define_matrix(synthetic.random_euler(rng), "inv")
        t = rng.uniform(-2, 2, 3)
        ip.interp3d(R.T, t, "forward", out=d_parts[i])
        rots.append(R)
        shifts.append(t)
    d_parts += 0.5 * torch.randn(d_parts.shape, device="cuda", generator=gen)
    rots = np.array(rots)
    shifts = np.array(shifts, np.float32)
    weights = rng.uniform(0.5, 1.0, P).astype(np.float32)
    halves = 1 + (np.arange(P) % 2)
    wedges = torch.rand((8, nw, nw, nw), device="cuda", generator=gen)
    widx = np.arange(P) % 8
    mask = torch.from_numpy(synthetic.soft_sphere_mask(n, 28)).cuda()
    avg = api.Average(mask, wedge_box=nw)
    h_parts = d_parts.cpu().pin_memory()
    h_avg = torch.empty((2, n, n, n), dtype=torch.float32).pin_memory()

    def step(src):
        avg.reset()
        avg.add(src, rots, halves, shifts=shifts, weights=weights, wedges=wedges, wedge_index=widx)
        return avg.result(1)[0], avg.result(2)[0]

    for _ in range(args.warmup):
        step(d_parts)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step(d_parts)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ref_avg = torch.stack(list(step(d_parts))).cpu()
    # end to end: pinned host windows -> device -> average -> both half averages back to the host.
    # The windows go over in batches of 128 on a copy stream into two device buffers; batch b+1's
    # copy is issued before emc_average_add(batch b) (which waits for its own work), so the copy
    # runs under the averaging.  The ordered accumulation makes the result independent of the
    # batch split (checked against the device-resident step).
    BT = 128
    bufs = [torch.empty((BT, n, n, n), dtype=torch.float32, device="cuda") for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]
    batches = [(b0, min(P, b0 + BT)) for b0 in range(0, P, BT)]

    def issue_copy(k):
        slot = k % 2
        b0, b1 = batches[k]
        copy_stream.wait_event(consumed[slot])
        with torch.cuda.stream(copy_stream):
            bufs[slot][:b1 - b0].copy_(h_parts[b0:b1], non_blocking=True)
            copied[slot].record(copy_stream)

    def e2e_step():
        avg.reset()
        copy_stream.wait_stream(stream)
        issue_copy(0)
        for k, (b0, b1) in enumerate(batches):
            if k + 1 < len(batches):
                issue_copy(k + 1)
            slot = k % 2
            stream.wait_event(copied[slot])
            avg.add(bufs[slot][:b1 - b0], rots[b0:b1], halves[b0:b1], shifts=shifts[b0:b1], weights=weights[b0:b1],
                    wedges=wedges, wedge_index=widx[b0:b1])
            consumed[slot].record(stream)
        h_avg[0].copy_(avg.result(1)[0], non_blocking=True)
        h_avg[1].copy_(avg.result(2)[0], non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    if not torch.equal(h_avg, ref_avg):
        raise RuntimeError("end-to-end averages differ from the device-resident step")
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    # CPU: the FP64 restatement on a bounded sample
    k = 8
    t0 = time.time()
    O.average_np(list(h_parts[:k].numpy()), mask.cpu().numpy(), list(rots[:k]), halves[:k], shifts=shifts[:k],
                 weights=weights[:k], wedges=list(wedges.cpu().numpy()), wedge_index=widx[:k])
    cpu_rate = k / (time.time() - t0)
    byts = 4 * n ** 3 + 4 * nw ** 3
    pk, which = measured_peaks()
    rate = P / (ms / 1e3)
    return {"metric": "particles/s averaged (64^3, with 64^3 wedge weights)", "value": rate,
            "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d extracted 64^3 windows, odd/even half sets, 8 wedge weights 64^3, C1, one "
                                   "emc_average_add per step" % P},
            "e2e": {"value": P / (e2e_ms / 1e3), "unit": "particles/s", "h2d_bytes_per_step": int(h_parts.numel() * 4),
                    "d2h_bytes_per_step": int(h_avg.numel() * 4)},
            "roofline": {"bound": "hbm", "achieved": byts * rate / 1e9, "peak": pk, "unit": "GB/s",
                         "frac": byts * rate / 1e9 / pk, "peak_source": which,
                         "algorithmic_bytes_per_particle": byts},
            "cpu_baseline": {"value": cpu_rate, "unit": "particles/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": "%d particles through the FP64 restatement (C rotation, numpy sums)" % k}}


def run_formats(args):
    """The data paths either side of the search: a 512x512x256 float32 tomogram (256 MiB) read from an
    MRC file into HBM, 2,000 64^3 windows extracted from it (BH_isWindowValid + zero padding), and
    per-particle SF3D weights (BH_weightMaskMex, 41 tilts, 64^3) for 64 positions."""
    import tempfile

    import torch

    from emclarity_b200 import api
    from oracle import oracle as O
    rng = np.random.default_rng(21)
    nz, ny, nx = 256, 512, 512
    tomo_h = rng.standard_normal((nz, ny, nx), dtype=np.float32)
    tmpdir = tempfile.mkdtemp(prefix="emc_bench_")
    path = os.path.join(tmpdir, "tomo.mrc")
    api.mrc_write(path, tomo_h, pixel_size=2.17)
    d_tomo = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    for _ in range(2):
        api.mrc_read_device(path, out=d_tomo)  # the file is in the page cache after the first read
    reps = max(3, args.steps)
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(reps):
        api.mrc_read_device(path, out=d_tomo)
    torch.cuda.synchronize()
    read_s = (time.time() - t0) / reps
    t0 = time.time()
    O.mrc_read_np(path)
    read_cpu_s = time.time() - t0
    # window extraction
    k, w = 2000, 64
    centers = np.stack([rng.uniform(1, nx, k), rng.uniform(1, ny, k), rng.uniform(1, nz, k)], axis=1)
    api.extract_windows(d_tomo, (w, w, w), centers[:8], 20.0)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        out, _, _ = api.extract_windows(d_tomo, (w, w, w), centers, 20.0)
    e1.record(stream)
    torch.cuda.synchronize()
    ext_ms = e0.elapsed_time(e1) / reps
    del out
    t0 = time.time()
    for c in centers[:20]:
        O.extract_window_np(tomo_h, (w, w, w), c, 20.0)
    ext_cpu = 20 / (time.time() - t0)
    # per-particle SF3D weights
    nt = 41
    t = np.zeros((nt, 22))
    t[:, 0] = np.arange(nt) + 1
    t[:, 3] = np.linspace(-60, 60, nt)
    t[:, 10] = np.linspace(0, 120, nt)
    t[:, 11], t[:, 12], t[:, 13] = 4.1e-8, -1.05, 1.0
    t[:, 14], t[:, 15], t[:, 16], t[:, 17], t[:, 18] = -3e-6, 2.17e-10, 2.7e-3, 1.968697e-12, 0.085
    n_sf = 2000
    xyz = np.stack([rng.uniform(1, 512, n_sf), rng.uniform(1, 512, n_sf), rng.uniform(1, 256, n_sf)], axis=1)
    rg = np.array([[512, 512, 256], [0.0, 0.0, 0.0]])
    api.sf3d_particles((64, 64, 64), 1.0, t, xyz[:2], rg)
    torch.cuda.synchronize()
    t0 = time.time()
    sf = api.sf3d_particles((64, 64, 64), 1.0, t, xyz, rg)
    torch.cuda.synchronize()
    sf_s = time.time() - t0
    del sf
    t0 = time.time()
    O.sf3d_particles_np((64, 64, 64), 1.0, t, xyz[:2], rg)
    sf_cpu = 2 / (time.time() - t0)
    os.remove(path)
    os.rmdir(tmpdir)
    pk, which = measured_peaks()
    ext_bytes = 2 * 4 * w ** 3 * k  # read + write of every window
    return {"metric": "windows/s extracted (64^3 from a 512x512x256 tomogram in HBM)", "value": k / (ext_ms / 1e3),
            "unit": "windows/s", "n_gpus": 1, "steps": reps, "ms_per_step": ext_ms, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "MRC read 512x512x256 float32 to HBM, 2,000 64^3 windows, 2,000 SF3D weights"},
            "roofline": {"bound": "hbm", "achieved": ext_bytes / (ext_ms / 1e3) / 1e9, "peak": pk, "unit": "GB/s",
                         "frac": ext_bytes / (ext_ms / 1e3) / 1e9 / pk, "peak_source": which},
            "mrc_read_device": {"gb_per_s": tomo_h.nbytes / read_s / 1e9, "ms": read_s * 1e3,
                                "cpu_numpy_gb_per_s": tomo_h.nbytes / read_cpu_s / 1e9,
                                "note": "file in the page cache; bound by the host read + PCIe"},
            "sf3d_particles": {"value": n_sf / sf_s, "unit": "particles/s", "particles": n_sf, "tilts": nt,
                               "cpu_restatement": sf_cpu},
            "cpu_baseline": {"value": ext_cpu, "unit": "windows/s", "cores": 1, "kind": "port",
                             "sample": "20 windows through the numpy restatement"}}


def run_tsearch_post(args):
    """Template-search pre / post-processing on a 512x512x256 map: local normalisation (feature size
    16) and greedy peak picking (300 peaks, spherical erase mask of radius 10, rmDim 17) on a map
    holding 400 planted peaks over noise."""
    import torch

    from emclarity_b200 import api
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    nz, ny, nx = 256, 512, 512
    gen = torch.Generator(device="cuda").manual_seed(3)
    vol = torch.randn((nz, ny, nx), device="cuda", generator=gen) + 2.0
    api.local_normalize(vol.clone(), 16)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(3, args.steps)
    work = [vol.clone() for _ in range(reps)]
    torch.cuda.synchronize()
    e0.record(stream)
    for w in work:
        api.local_normalize(w, 16)
    e1.record(stream)
    torch.cuda.synchronize()
    ln_ms = e0.elapsed_time(e1) / reps
    del work
    # peak map: noise + 400 Gaussian blobs, random angle indices, zero margin
    mag = 0.05 * torch.randn((nz, ny, nx), device="cuda", generator=gen)
    cz = rng.uniform(20, nz - 20, 400)
    cy = rng.uniform(20, ny - 20, 400)
    cx = rng.uniform(20, nx - 20, 400)
    hts = rng.uniform(0.5, 3.0, 400)
    r = 5
    g = torch.arange(-r, r + 1, device="cuda", dtype=torch.float32)
    blob = torch.exp(-(g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2) / (2 * 1.5 ** 2))
    for z, y, x, h in zip(cz.astype(int), cy.astype(int), cx.astype(int), hts):
        mag[z - r:z + r + 1, y - r:y + r + 1, x - r:x + r + 1] += float(h) * blob
    n_angles = 2592
    ang = torch.randint(1, n_angles + 1, (nz, ny, nx), device="cuda", generator=gen).float()
    angle_list = np.stack([rng.uniform(0, 360, n_angles), rng.uniform(0, 180, n_angles),
                           rng.uniform(-180, 180, n_angles)], axis=1)
    rm = 17
    gg = np.arange(2 * rm + 1) - rm
    zz, yy, xx = np.meshgrid(gg, gg, gg, indexing="ij")
    removal = ((xx ** 2 + yy ** 2 + zz ** 2) <= 100).astype(np.float32)
    m1 = mag.clone()
    api.tsearch_peaks(m1, ang, removal, rm, angle_list, max_peaks=10, high_thr=0.3)
    m2 = mag.clone()
    torch.cuda.synchronize()
    t0 = time.time()
    peaks = api.tsearch_peaks(m2, ang, removal, rm, angle_list, max_peaks=300, high_thr=0.3)
    torch.cuda.synchronize()
    pk_s = time.time() - t0
    # CPU restatements on bounded samples
    small = vol[:64, :128, :128].cpu().numpy()
    t0 = time.time()
    O.local_normalize_np(small, 16)
    ln_cpu_vox_s = small.size / (time.time() - t0)
    msm = m1[:96, :160, :160].cpu().numpy()
    t0 = time.time()
    ref = O.tsearch_peaks_np(msm, ang[:96, :160, :160].cpu().numpy(), removal, rm, angle_list, max_peaks=10,
                             high_thr=0.3)
    pk_cpu = max(1, len(ref)) / (time.time() - t0)
    pk, which = measured_peaks()
    nvox = nz * ny * nx
    byts = 2 * 4 * nvox  # read the volume once, write it once
    return {"metric": "peaks/s picked on a 512x512x256 template-search map", "value": len(peaks) / pk_s,
            "unit": "peaks/s", "n_gpus": 1, "steps": reps, "ms_per_step": pk_s * 1e3, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "512x512x256 map, 400 planted peaks, 300 picked, erase radius 10 (rmDim 17); "
                                   "local normalisation of a 512x512x256 tomogram, feature size 16"},
            "peaks_found": int(len(peaks)),
            "local_normalize": {"ms": ln_ms, "voxels_per_s": nvox / (ln_ms / 1e3),
                                "roofline": {"bound": "hbm", "achieved": byts / (ln_ms / 1e3) / 1e9, "peak": pk,
                                             "unit": "GB/s", "frac": byts / (ln_ms / 1e3) / 1e9 / pk,
                                             "peak_source": which},
                                "cpu_restatement_voxels_per_s": ln_cpu_vox_s},
            "cpu_baseline": {"value": pk_cpu, "unit": "peaks/s", "cores": 1, "kind": "port",
                             "sample": "10 peaks on a 96x160x160 crop through the numpy restatement"}}


def _rodrigues(axis, deg):
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    th = np.radians(deg)
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K


def run_refine(args, n_part=None):
    """Gradient pose refinement: 96^3 particles at SNR 0.05, coarse 15-degree local search (95
    orientations around a seeded prior within 12 degrees of the truth), then either 20 L-BFGS steps on
    the forward + adjoint CC or a dense 1-degree local grid (3,859 orientations) around the coarse best;
    wall-clock time and median pose error of both."""
    import torch

    from emclarity_b200 import api, refine, synthetic
    n = 96
    n_part = n_part or (args.particles if args.particles != 1200 else 1000)
    rng = np.random.default_rng(96)
    ref = synthetic.blob_reference(rng, n)
    mask = synthetic.soft_sphere_mask(n, 28 * n / 64)
    rg, mg = torch.from_numpy(ref).cuda(), torch.from_numpy(mask).cuda()
    ft = api.FourierTransformer((n, n, n))
    coarse = api.euler_search("C1", 30, 15, 30, 15)
    dense = api.euler_search("C1", 8, 1, 8, 1)
    s = api.Search(peak_radius=6)
    rid = s.add_reference(rg, mg)
    priors, truths, specs, hs, ens, wedges = [], [], [], [], [], []
    for _ in range(n_part):
        prior = api.define_matrix(synthetic.random_euler(rng), "inv")
        jitter = _rodrigues(rng.standard_normal(3), rng.uniform(0, 12))
        truth = prior @ jitter
        w = api.wedge_ctf_weight(n, -60, 60, synthetic.ctf_dict(rng.uniform(15000, 40000)))
        p = synthetic.make_particle(rg, rng, truth, rng.integers(-3, 4, 3), w, 0.05, ft=ft)
        q, e = api.particle_spectrum(p)
        priors.append(prior)
        truths.append(truth)
        specs.append(q)
        wedges.append(w)
        ens.append(e.item())
        # the adjoint's template h = F^-1(wdgMask .* P): its zero-lag numerator is the search's
        hs.append(api.particle_template(api.particle_spectrum(p, w)[0]))
    truths = np.array(truths)

    def coarse_search():
        s.set_orientations(coarse)
        d = [s.particle(specs[i], ens[i], rid, prior=priors[i], orient_count=len(coarse), wedge=wedges[i])
             for i in range(n_part)]
        _, _, best = s.run_host(d)
        return best

    t_coarse, best = _timed(coarse_search)
    Dc = [api.define_matrix([coarse[b[1]][0], coarse[b[1]][1], coarse[b[1]][2] - coarse[b[1]][0]], "inv")
          for b in best]
    R_coarse = np.array([priors[i] @ Dc[i] for i in range(n_part)])
    err_coarse = refine.geodesic_deg(R_coarse, truths)

    # (a) L-BFGS on the forward + adjoint, parameterised around the coarse best at theta = 90 deg
    rx90 = api.define_matrix([0.0, -90.0, 0.0], "inv")
    pri2 = [R_coarse[i] @ rx90 for i in range(n_part)]
    x0 = np.array([[0.0, 90.0, 0.0] + [float(v) for v in best[i][2]] for i in range(n_part)])

    def grad_refine(interp):
        obj = refine.BatchObjective(s, [rid] * n_part, hs, ens, pri2, interp=interp)
        x, f, hist = refine.lbfgs(obj, x0, n_iter=20)
        return x, obj.evals

    results = {}
    for interp in ("linear", "cubic"):
        t_ref, (x, nev) = _timed(lambda: grad_refine(interp))
        R = np.array([pri2[i] @ api.define_matrix([x[i, 0], x[i, 1], x[i, 2] - x[i, 0]], "inv")
                      for i in range(n_part)])
        err = refine.geodesic_deg(R, truths)
        results[interp] = {"seconds": t_ref, "median_err_deg": float(np.median(err)),
                           "p90_err_deg": float(np.percentile(err, 90)), "objective_evals": int(nev)}

    # (b) plain GPU grid search: dense 1-degree local grid around the coarse best
    def dense_search():
        s.set_orientations(dense)
        d = [s.particle(specs[i], ens[i], rid, prior=R_coarse[i], orient_count=len(dense), wedge=wedges[i])
             for i in range(n_part)]
        _, _, bd = s.run_host(d)
        return bd

    t_dense, bd = _timed(dense_search)
    R_dense = np.array([R_coarse[i] @ api.define_matrix(
        [dense[b[1]][0], dense[b[1]][1], dense[b[1]][2] - dense[b[1]][0]], "inv") for i, b in enumerate(bd)])
    err_dense = refine.geodesic_deg(R_dense, truths)
    lin = results["linear"]
    return {"metric": "pose-refine time at <= 0.5 deg median error", "value": lin["seconds"], "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d x 96^3 particles, SNR 0.05, coarse local 15-degree grid (%d orientations), "
                                   "20 L-BFGS steps vs dense 1-degree grid (%d orientations)" %
                                   (n_part, len(coarse), len(dense))},
            "coarse": {"seconds": t_coarse, "median_err_deg": float(np.median(err_coarse))},
            "lbfgs": results,
            "dense_grid": {"seconds": t_dense, "median_err_deg": float(np.median(err_dense)),
                           "p90_err_deg": float(np.percentile(err_dense, 90)), "evals": n_part * len(dense)},
            "speedup_refine_phase": t_dense / lin["seconds"],
            "speedup_total": (t_coarse + t_dense) / (t_coarse + lin["seconds"])}


def run_extras(args):
    """Keys of the default line beside the headline: the batched uneven configuration (2,000 particles,
    60/30/10 over 64^3 / 96^3 / 128^3, 256 local orientations each) with FP32 and with BF16 reference
    storage (three warm-up and two timed runs each), and a bounded pose refinement (200 x 96^3)."""
    import torch

    from emclarity_b200 import synthetic
    grid = synthetic.local_grid(N_ORIENT, 8.0, 2.0)
    sizes, refs, parts = mixed_batch(2000)
    out = {"mixed": mixed_entry(sizes, parts, refs, "f32", 2, 3, grid, args.overlap),
           "mixed_bf16": mixed_entry(sizes, parts, refs, "bf16", 2, 3, grid, args.overlap)}
    del parts, refs
    torch.cuda.empty_cache()
    out["refine"] = run_refine(args, n_part=200)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=1200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-uneven (FP32, BF16) and refinement keys of the default line")
    ap.add_argument("--planes", type=int, default=0, help="pass-A z-planes per CTA (0: timed choice)")
    ap.add_argument("--overlap", type=int, default=0, help="chunk scratch slots (0: the library default, 2)")
    ap.add_argument("--chunk", type=int, default=0, help="evaluations per chunk (0: the library default)")
    ap.add_argument("--workload", default="batched64", choices=["batched64", "mixed", "bf16", "tsearch", "refine", "average", "formats",
                                                                    "tsearch_post"])
    args = ap.parse_args()
    if args.impl == "ours" and args.workload != "batched64":
        import torch
        torch.cuda.set_device(0)
        fn = {"mixed": run_mixed, "bf16": lambda a: run_mixed(a, "bf16"), "tsearch": run_tsearch,
              "refine": run_refine, "average": run_average, "formats": run_formats,
              "tsearch_post": run_tsearch_post}[args.workload]
        print(json.dumps(fn(args)))
        return
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        res = run_reference(args, world, rank)
        if res is not None:
            print(json.dumps(res))
        return
    world, rank, local = dist_setup()
    res = run_ours(args, world, rank, local)
    if rank == 0:
        if not args.no_extras and world == 1:
            res.update(run_extras(args))
        if not args.no_cpu_baseline and world == 1:
            res["cpu_baseline"] = cpu_baseline_entry(seconds=10.0)
        print(json.dumps(res))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
