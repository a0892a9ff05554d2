"""Benchmark: raw echoes/s (facet x pulse x channel) of the B200 raw-data generator.

Workload (the two-channel along-track case): a 2048 x 2048 linear-wave surface at 1 m
(Elfouhaily spectrum, cos^2 spreading, U10 = 7 m/s at 45 deg, deep water), C band
5.405 GHz, 514 km altitude, 7600 m/s, 35 deg incidence, 2 along-track channels with a 10 m
baseline, 4096 pulses at 1500 Hz, 2048 range bins, Kodis specular + Romeiser Bragg NRCS,
vv.  Synthetic seeded input (no dataset exists for this path).  One step = one full scene:
the surface synthesis and the fused pulse kernel for all 4096 pulses, replayed from a CUDA
graph.  The working set (coefficients, scratch planes, fields, RCS, raw cube) is ~0.5 GB,
far above the 126 MB L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|f64] [--small]

``--impl reference`` times the CPU restatement of the reference's numba path (the oracle)
on the host cores, on a bounded window of pulses of the same workload, and prints the same
JSON line with "impl": "reference".  Multi-GPU runs (torchrun) are replicas: every rank
simulates its own scene (seed + rank); value = all ranks' echoes / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "raw echoes/s (facet*pulse*chan)"
UNIT = "echoes/s"

C2 = dict(name="C-band 2-channel ATI, 2048x2048 surface, 4096 pulses, 2048 bins",
          L=2048, d=1.0, wind_U=7.0, wind_dir=45.0, prf=1500.0, pulses=4096, bins=2048, num_ch=2,
          b_ati=10.0, b_xti=0.0, ant_l=2.742, pol="vv", inc=35.0)
C1 = dict(name="C-band 1-channel, 512x512 surface, 256 pulses, 512 bins",
          L=512, d=1.0, wind_U=10.0, wind_dir=0.0, prf=1000.0, pulses=256, bins=512, num_ch=1,
          b_ati=0.0, b_xti=0.0, ant_l=35.7, pol="vv", inc=35.0)

CFG = """[sar]
f0=5.405e9
inc_angle={inc}
pol={pol}
squint=0
prf={prf}
rg_bw=50e6
over_fs=1.1
alt=514e3
v_ground=7600.
heading=0.
ant_L_tx={ant_l}
ant_L_rx={ant_l}
num_ch={num_ch}
b_ati={b_ati}
b_xti={b_xti}
sigma_n_tx=0.
phase_n_tx=0.
sigma_beta_tx=0.
phase_beta_tx=0.
sigma_n_rx=0.
phase_n_rx=0.
sigma_beta_rx=0.
phase_beta_rx=0.

[ocean]
Lx={L}
Ly={L}
dx={d}
dy={d}
opt_res=True
fft_max_prime=2
dt=0.05
depth=1e5
wind_dir={wind_dir}
wind_U={wind_U}
wind_fetch=500e3
swell_dir_enable=False
sigf=0.007
freq_r=0.079
dir_swell_dir=120
sigs=8
Hs=0.8
swell_enable=False
swell_wl=60
swell_dir=20
swell_ampl=0.3
spec_model=elfouhaily
spread_model=cos2s
cutoff_wl=auto
current_mag=0
current_dir=0.
choppy_enable=False
frozen_ocean=False

[srg]
use_hmtf=False
nesz=-300.
wh_tol=2.73
scat_spec_enable=True
scat_spec_mode=kodis
scat_bragg_enable=True
scat_bragg_model=romeiser97
scat_bragg_spec=elfouhaily
scat_bragg_spread=cos2s
scat_bragg_d=0.125
use_lut=False
"""


def write_cfg(c, path):
    with open(path, "w") as f:
        f.write(CFG.format(**c))
    return path


def overrides(c):
    return dict(az_steps=c["pulses"], rg_samp=c["bins"], rg_samp_orig=c["bins"])


def echoes(c, pulses=None):
    return float(c["L"] / c["d"]) ** 2 * (c["pulses"] if pulses is None else pulses) * c["num_ch"]


# ----------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        out.update(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=reasons, samples=len(rows))
        return out


# ----------------------------------------------------------------------------------------
def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(c, cfg_path, pulses, seed=0):
    """Oracle (CPU restatement of the reference's numba path) over a bounded pulse window."""
    from oracle.sar_raw import SarRawSim
    sim = SarRawSim(cfg_path, overrides=overrides(c), seed=seed)
    sim.pulse(0)                               # JIT-free warm-up (FFT plans, first refresh)
    t0 = time.perf_counter()
    for a in range(1, 1 + pulses):
        sim.pulse(a)
    dt = time.perf_counter() - t0
    return echoes(c, pulses) / dt, dt


def run_reference(args, c, cfg_path):
    world, rank, _ = dist_info()
    if rank != 0:
        return
    from oracle.sar_raw import SarRawSim
    sim = SarRawSim(cfg_path, overrides=overrides(c), seed=0)
    steps = []
    pulses = 2 if args.small else 3
    a = 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for _ in range(pulses):
            sim.pulse(a % sim.az_steps)
            a += 1
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            steps.append((echoes(c, pulses) / dt, dt))
    value = float(np.mean([v for v, _ in steps]))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean([d for _, d in steps]) * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": c["name"], "sample": "%d pulses per step" % pulses},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": "%d pulses of the %dx%d scene per step, after one warm-up pulse; "
                                       "numpy FFT (single thread) + serial C accumulation" %
                                       (pulses, c["L"], c["L"])},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def accumulation_roofline(peak, peak_src, n=4096, nbins=2048, reps=10):
    """Standalone facet-to-bin accumulation (``ocs_chan_profile_2d_c64`` / ``_f64``) on a
    seeded n x n surface layout (slant range along the columns, azimuth curvature along the
    rows, 1 m jitter): algorithmic bytes = range (8 B) + scene (8 B c64 / 16 B c128) per
    facet; inputs (268 / 403 MB) exceed the L2."""
    import ctypes
    import torch
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim.range_profile import calc_sinc_vec
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.arange(n, device="cuda", dtype=torch.float64)
    y = x - n / 2
    sr0 = 627e3
    srg = (sr0 + x[None, :] * np.sin(np.radians(35.0)) + (y[:, None] + 3000.0) ** 2 / (2 * sr0) +
           torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)).contiguous()
    binsize = 2.99792458e8 / (2 * 50e6) / 1.1
    min_sr = float(srg.min()) - 10.0
    sinc = torch.tensor(calc_sinc_vec(8, 20, Fs=1.1), dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _capi.load()
    out = {}
    for name, fn, dt, bpf in (("c64", lib.ocs_chan_profile_2d_c64, torch.float32, 16),
                              ("f64", lib.ocs_chan_profile_2d_f64, torch.float64, 24)):
        sc = torch.randn(n, n, 2, generator=g, device="cuda", dtype=torch.float64).to(dt)
        o = torch.zeros(nbins, 2, device="cuda", dtype=dt)
        call = lambda: fn(srg.data_ptr(), sc.data_ptr(), n, n, binsize, min_sr, sinc.data_ptr(), 8, 20,  # noqa: E731
                          o.data_ptr(), nbins, st)
        for _ in range(3):
            assert call() == 0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            call()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = n * n * bpf / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 4), "facets_per_s": n * n / (ms * 1e-3), "GBps": round(gbs, 1),
                     "frac": round(gbs / peak, 4), "alg_bytes_per_facet": bpf}
        del sc, o
    try:
        traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))["accumulation"]["c64"]
    except (OSError, ValueError, KeyError):
        traffic = None
    out["c64"]["traffic"] = traffic
    out.update({"kernel": "chan_profile_2d_kernel", "grid": [n, n], "nbins": nbins, "peak": peak,
                "peak_source": peak_src, "bound": "hbm"})
    return out


# ----------------------------------------------------------------------------------------
# Batched and serving workloads (one GPU; replicas for N > 1 as for the default workload)
def _workload_reference(args, specs, what):
    """CPU oracle on a bounded sample of the workload's scenes (2 pulses of each of the
    first three), as echoes/s."""
    from oceansar_b200.serving import prepare_scene  # noqa: F401  (same cfg writer)
    from oracle.sar_raw import SarRawSim
    tot_e, tot_t = 0.0, 0.0
    tmpd = tempfile.mkdtemp(prefix="ocs_ref_")
    for k, sp in enumerate(specs[:3]):
        path = os.path.join(tmpd, "s%d.cfg" % k)
        with open(path, "w") as f:
            f.write(sp["cfg"])
        sim = SarRawSim(path, overrides=sp["overrides"], seed=sp["seed"])
        sim.pulse(0)
        t0 = time.perf_counter()
        for a in (1, 2):
            sim.pulse(a)
        tot_t += time.perf_counter() - t0
        tot_e += 2.0 * sim.surface.Nx * sim.surface.Ny * sim.num_ch
    v = tot_e / tot_t
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "2 pulses of each of the first 3 scenes of the %s workload (%.1f s)" % (what, tot_t)}


def run_workload(args):
    import torch
    from oceansar_b200 import replicas
    from oceansar_b200.serving import ScenePreparer, ServingLoop, batched_specs, run_batched, serving_requests
    from oceansar_b200.tune import Autotuner
    world, rank, local = dist_info()
    what = args.workload
    if what == "batched":
        specs = batched_specs(args.scenes, seed=1 + 1000 * rank)
    else:
        specs = serving_requests(rate=args.rate, duration=args.duration, seed=2 + 1000 * rank)
    if args.impl == "reference":
        if rank == 0:
            cpu = _workload_reference(args, specs, what)
            print(json.dumps({"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": args.gpus,
                              "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak",
                              "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                              "config": {"workload": what}, "cpu_baseline": cpu,
                              "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))
    prep = ScenePreparer(workers=args.workers)
    clocks = ClockSampler(local)
    tuner = Autotuner()
    try:
        if what == "batched":
            t0 = time.perf_counter()
            futs = [prep.submit(sp, args.precision) for sp in specs]
            gens = [f.result() for f in futs]
            host_prep = time.perf_counter() - t0
            clocks.start()
            rep = run_batched(gens, precision=args.precision, tuner=tuner)
            clk = clocks.stop()
            # end to end: spectra and scatterer indices from pinned host memory, the run,
            # every raw cube back to pinned host memory
            e2e = _batched_e2e(gens, args.precision, tuner, rep["pulse_block"])
            sec = replicas.max_over_ranks(rep["device_s"], device="cuda")
            ms = sec * 1e3
            value = replicas.sum_over_ranks(rep["echoes"], device="cuda") / sec
            line_extra = {"batched": {k: rep[k] for k in ("scenes", "echoes", "steps", "pulse_block", "tile_rows",
                                                          "tune_s", "launches_first_step")},
                          "host_prep_s": host_prep}
            launches = rep["kernel_launches"]
            e2e_d = e2e
        else:
            clocks.start()
            loop = ServingLoop(precision=args.precision, hbm_budget=150e9, max_slots=64, pulse_block=16,
                               preparer=prep, tuner=tuner)
            rep = loop.run(specs)
            clk = clocks.stop()
            sec = replicas.max_over_ranks(rep["span_s"], device="cuda")
            ms = sec * 1e3
            value = replicas.sum_over_ranks(rep["echoes"], device="cuda") / sec
            e2e_d = {"value": value, "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                     "note": "arrival to raw cube in host memory for every request (wall clock)"}
            line_extra = {"serving": {k: rep[k] for k in ("requests", "echoes", "span_s", "offered_echoes_per_s",
                                                          "latency_p50_s", "latency_p99_s", "latency_max_s",
                                                          "peak_reserved_bytes", "max_backlog",
                                                          "gpu_busy_frac", "capacity_echoes_per_s",
                                                          "queue_stable")},
                          "rate_per_s": args.rate, "arrival_window_s": args.duration}
            launches = None
    finally:
        prep.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = _workload_reference(args, specs, what)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 0,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": what, "precision": args.precision,
                           "parallelism": "replicas" if world > 1 else "single-gpu",
                           "l2": "working set of many scenes far above L2"},
                "clocks": clk, "e2e": e2e_d, "gpu_launches": launches, "roofline": None,
                "cpu_baseline": cpu}
        line.update(line_extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _batched_e2e(gens, precision, tuner, pulse_block):
    """Echoes/s of the whole batch with host inputs and outputs inside the timed region."""
    import torch
    from oceansar_b200.radarsim.batch import SceneBatch
    from oceansar_b200.serving import scene_echoes
    batch = SceneBatch(max_slots=len(gens), precision=precision)
    ins, outs = [], []
    for g in gens:
        cls = (g.surface.Nx, g.surface.Ny, g.npol * g.num_ch)
        batch.add(g, tile_rows=tuner.tile_rows_for(precision, cls))
        s = g.surface
        pairs = [(torch.from_numpy(s.wave_coefs).pin_memory(), s._coefs_d),
                 (torch.from_numpy(s.omega).pin_memory(), s._omega_d)]
        if g.scat_bragg_enable:
            pairs.append((torch.from_numpy(g.rndscat_m.ind0.astype(np.int32)).pin_memory(), g.rndscat_m.device()[1]))
            pairs.append((torch.from_numpy(g.rndscat_p.ind0.astype(np.int32)).pin_memory(), g.rndscat_p.device()[1]))
        ins.extend(pairs)
        outs.append((g.raw_d, torch.empty(g.raw_d.shape, dtype=g.raw_d.dtype).pin_memory()))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for h, d in ins:
        d.copy_(h, non_blocking=True)
    while True:
        for sl in batch.finished():
            batch.remove(sl)
        live = batch.live()
        if not live:
            break
        batch.graph_step(min(pulse_block, min(batch.remaining(sl) for sl in live)))
    for d, h in outs:
        h.copy_(d, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) * 1e-3
    batch.close()
    echoes = sum(scene_echoes(g) for g in gens)
    h2d = sum(h.numel() * h.element_size() for h, _ in ins)
    d2h = sum(h.numel() * h.element_size() for _, h in outs)
    return {"value": echoes / sec, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": sec * 1e3}


# ----------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--small", action="store_true", help="512^2 single-channel case (quick check)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--workload", default="c2", choices=["c2", "batched", "serving"],
                    help="c2: the two-channel 2048^2 scene (default); batched: many scenes in one "
                         "scene batch; serving: a Poisson request stream with continuous batching")
    ap.add_argument("--scenes", type=int, default=64, help="batched: number of scenes")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: requests per second")
    ap.add_argument("--duration", type=float, default=5.0, help="serving: seconds of arrivals")
    ap.add_argument("--workers", type=int, default=None, help="host set-up worker processes")
    ap.add_argument("--accumulation-only", action="store_true",
                    help="time only the standalone accumulation kernels and print their line")
    ap.add_argument("--profile-pulses", type=int, default=0,
                    help="run this many pulses with plain launches (for ncu) and exit")
    args = ap.parse_args()
    if args.workload != "c2":
        run_workload(args)
        return
    if args.accumulation_only:
        import torch
        torch.cuda.set_device(dist_info()[2])
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak, src = ((json.load(open(peaks_path))["hbm_gbs"], "measured") if os.path.exists(peaks_path)
                     else (6650.0, "fallback"))
        print(json.dumps({"accumulation": accumulation_roofline(peak, src)}), flush=True)
        return
    c = C1 if args.small else C2
    tmpd = tempfile.mkdtemp(prefix="ocs_bench_")
    cfg_path = write_cfg(c, os.path.join(tmpd, "scene.cfg"))
    if args.impl == "reference":
        run_reference(args, c, cfg_path)
        return

    import torch
    import torch.distributed as dist
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator

    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    from oceansar_b200 import replicas

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, device="cuda")

    def timed(gen, steps, warmup):
        for _ in range(warmup):
            gen.replay()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            gen.replay()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # ---- main arm ---------------------------------------------------------------------
    gen = RawGenerator(cfg_path, precision=args.precision, overrides=overrides(c),
                       seed=replicas.replica_seed(1000, rank))
    if args.profile_pulses:
        gen.run(range(args.profile_pulses))
        torch.cuda.synchronize()
        print("profiled %d pulses" % args.profile_pulses)
        return
    gen.capture()
    clocks = ClockSampler(local)
    clocks.start()
    ms = timed(gen, args.steps, args.warmup)
    clk = clocks.stop()
    value = echoes(c) * world / (ms * 1e-3)
    launches = gen.kernel_launches_per_scene() * args.steps

    # ---- per-kernel timing and roofline (dominant kernel) -----------------------------
    # Each kernel is bracketed alone by CUDA events on its launching stream, 64 pulses.
    npl = 64
    kt = gen.time_kernels(range(64, 64 + npl))
    nf = float(gen.surface.Nx * gen.surface.Ny)
    fields_pulse = 5 + (3 if gen.scat_spec_enable else 0)
    scat_b = ((8 if args.precision == "f64" else 4) * 2 * gen.npol) if gen.scat_bragg_enable else 0
    ind_b = 8 if gen.scat_bragg_enable else 0
    nfields = len(gen.surface._raw)
    npair = (nfields + 1) // 2
    # algorithmic bytes per launch: row pass reads c and omega and writes the packed row
    # transforms (one complex64 plane per field pair); column pass reads those planes and
    # writes the float32 fields; pulse kernel reads the fields it uses, sqrt(RCS) (m, p per
    # polarisation) and the two Bragg index maps.
    surf_rows_bytes = nf * (8 + 4 + 8 * npair)
    surf_cols_bytes = nf * (8 * npair + 4 * nfields)
    pulse_bytes = nf * (4 * fields_pulse + scat_b + ind_b)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    kern = {"surface_rows": {"ms": kt["surface_rows"], "bytes": surf_rows_bytes},
            "surface_cols": {"ms": kt["surface_cols"], "bytes": surf_cols_bytes},
            "pulse": {"ms": kt["pulse"], "bytes": pulse_bytes}}
    for k in kern.values():
        k["GBps"] = k["bytes"] / (k["ms"] * 1e-3) / 1e9
        k["frac"] = k["GBps"] / peak
    dom = max(kern, key=lambda k: kern[k]["ms"])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.precision, {}).get(dom)
        except (ValueError, OSError):
            traffic = None
    roofline = {"bound": "hbm", "achieved": kern[dom]["GBps"], "peak": peak, "unit": "GB/s",
                "frac": kern[dom]["frac"], "traffic": traffic, "kernel": dom, "peak_source": peak_src,
                "per_kernel": {k: {"ms": round(v["ms"], 5), "GBps": round(v["GBps"], 1),
                                   "frac": round(v["frac"], 4), "alg_bytes": v["bytes"]}
                               for k, v in kern.items()}}

    # ---- end to end through the public API with host buffers ---------------------------
    s = gen.surface
    host_in = {"coefs": torch.from_numpy(s.wave_coefs).pin_memory(),
               "omega": torch.from_numpy(s.omega).pin_memory()}
    if gen.scat_bragg_enable:
        host_in["ind0_m"] = torch.from_numpy(gen.rndscat_m.ind0.astype(np.int32)).pin_memory()
        host_in["ind0_p"] = torch.from_numpy(gen.rndscat_p.ind0.astype(np.int32)).pin_memory()
    dev_in = {"coefs": s._coefs_d, "omega": s._omega_d}
    if gen.scat_bragg_enable:
        dev_in["ind0_m"] = gen.rndscat_m.device()[1]
        dev_in["ind0_p"] = gen.rndscat_p.device()[1]
    host_out = torch.empty(gen.raw_d.shape, dtype=gen.raw_d.dtype).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in host_in.values())
    d2h = host_out.numel() * host_out.element_size()

    def e2e_step():
        for k, t in host_in.items():
            dev_in[k].copy_(t, non_blocking=True)
        gen.replay()
        host_out.copy_(gen.raw_d, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    e2e = {"value": echoes(c) * world / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms}

    # ---- FP64 drop-in form on the same workload (secondary figure) ---------------------
    fp64 = None
    if not args.no_fp64 and args.precision == "mixed":
        del gen
        torch.cuda.empty_cache()
        g64 = RawGenerator(cfg_path, precision="f64", overrides=overrides(c),
                           seed=replicas.replica_seed(1000, rank))
        g64.capture()
        ms64 = timed(g64, 1, 1)
        fp64 = {"value": echoes(c) * world / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64}
        del g64
        torch.cuda.empty_cache()

    # ---- standalone accumulation (chan_profile drop-in, [ny][nx] layout) -------------------
    accum = None
    if not args.small:
        accum = accumulation_roofline(peak, peak_src)

    # ---- CPU baseline (oracle port) -------------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        pulses = 2 if args.small else 3
        v, dt = cpu_baseline(c, cfg_path, pulses)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "%d pulses of the %dx%d scene (%.1f s), after one warm-up pulse; numpy FFT "
                         "(single thread) + serial C accumulation" % (pulses, c["L"], c["L"], dt)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
                "data": "synthetic",
                "config": {"workload": c["name"], "grid": [c["L"], c["L"]], "pulses": c["pulses"],
                           "channels": c["num_ch"], "range_bins": c["bins"], "precision": args.precision,
                           "parallelism": "replicas" if world > 1 else "single-gpu",
                           "l2": "inputs larger than L2 (~0.5 GB working set)",
                           "graph": "whole scene replayed from one CUDA graph"},
                "clocks": clk, "e2e": e2e, "gpu_launches": launches, "roofline": roofline,
                "cpu_baseline": cpu, "fp64": fp64, "accumulation": accum}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
