"""Batched and served raw-data generation on one GPU.

* ``batched_specs`` draws the batched workload: independent scenes of uneven grid size,
  wind, geometry, channel count and pulse count.
* ``serving_requests`` draws a Poisson stream of scene requests of the same kind.
* ``run_batched`` runs a set of scenes to completion in one ``SceneBatch`` (every step
  one launch per kernel class for all scenes, CUDA-graph replays, autotuned shapes).
* ``ServingLoop`` serves a request stream with continuous batching: a request is admitted
  when its device memory fits the budget, prepared on the host by a pool of worker
  processes (the spectrum, random phases and scatterer series are numpy work, as in the
  reference), placed in a slot of the running batch as soon as one frees up -- while the
  other scenes keep running -- and retired (raw cube copied to the host) when its last
  pulse has run.  It reports p50 / p99 end-to-end latency (arrival to raw cube on the
  host) and the sustained echoes/s.

The scene simulated for a request is the reference's ``sar_raw`` scene (the same ``.cfg``
parameters and seeded numpy draws), so a request's raw cube is the one that scene gives
when run alone, up to the order of floating-point atomics.
"""
import collections
import concurrent.futures as cf
import multiprocessing as mp
import os
import tempfile
import time

import numpy as np

C_LIGHT = 2.99792458e8

CFG_TEMPLATE = """[sar]
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
b_xti=0
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

GRIDS = (256, 512, 1024, 2048)


def _draw_scene(rng):
    """One scene of the batched workload.  Draw order: grid, U10, wind direction,
    incidence, channels, along-track span, pulses, surface seed."""
    L = int(rng.choice(GRIDS))
    wind_U = float(rng.uniform(3., 20.))
    wind_dir = float(rng.uniform(0., 360.))
    inc = float(rng.uniform(20., 45.))
    nch = int(rng.integers(1, 4))
    span = float(rng.uniform(0., 10.))
    pulses = int(rng.integers(512, 4097))
    seed = int(rng.integers(0, 2 ** 31 - 1))
    params = dict(L=L, d=1.0, wind_U=wind_U, wind_dir=wind_dir, inc=inc, pol='vv', prf=1000.0,
                  ant_l=2.742, num_ch=nch, b_ati=(span / (nch - 1)) if nch > 1 else 0.0)
    return dict(cfg=CFG_TEMPLATE.format(**params), seed=seed, overrides=dict(az_steps=pulses),
                params=params, pulses=pulses)


def batched_specs(n_scenes=64, seed=1):
    """The batched workload: ``n_scenes`` scenes drawn from ``numpy.random.default_rng(seed)``
    (grid uniform over 256^2..2048^2 at 1 m, U10 3-20 m/s, wind direction 0-360 deg,
    incidence 20-45 deg, 1-3 along-track channels spanning up to 10 m, 512-4096 pulses)."""
    rng = np.random.default_rng(seed)
    return [_draw_scene(rng) for _ in range(n_scenes)]


def serving_requests(rate=20.0, duration=600.0, seed=2):
    """Poisson request stream: exponential inter-arrival times at ``rate`` per second over
    ``duration`` seconds, each request's scene drawn as in ``batched_specs`` from the same
    ``numpy.random.default_rng(seed)`` stream (inter-arrival time first, then the scene)."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            return out
        spec = _draw_scene(rng)
        spec['arrival'] = t
        out.append(spec)


def prepare_scene(spec, precision):
    """Host set-up of a scene (no GPU): a RawGenerator to be uploaded with ``to_device``."""
    from .radarsim.sar_raw_nompi import RawGenerator
    fd, path = tempfile.mkstemp(suffix='.cfg')
    try:
        with os.fdopen(fd, 'w') as f:
            f.write(spec['cfg'])
        return RawGenerator(path, precision=precision, overrides=spec.get('overrides'), seed=spec['seed'],
                            device=False)
    finally:
        os.unlink(path)


def _warm(_):
    from .radarsim import sar_raw_nompi  # noqa: F401  (imports numpy / scipy / torch once)
    return os.getpid()


class ScenePreparer(object):
    """Host set-up of scenes in ``workers`` spawned processes (0: in this process)."""

    def __init__(self, workers=None):
        if workers is None:
            workers = max(1, min(8, (os.cpu_count() or 2) - 2))
        self.workers = int(workers)
        self._pool = None
        if self.workers > 0:
            self._pool = cf.ProcessPoolExecutor(max_workers=self.workers, mp_context=mp.get_context('spawn'))
            list(self._pool.map(_warm, range(self.workers)))

    def submit(self, spec, precision):
        if self._pool is None:
            f = cf.Future()
            f.set_result(prepare_scene(spec, precision))
            return f
        return self._pool.submit(prepare_scene, spec, precision)

    def close(self):
        if self._pool is not None:
            self._pool.shutdown(wait=True, cancel_futures=True)
            self._pool = None


def scene_echoes(gen):
    return float(gen.surface.Nx) * gen.surface.Ny * gen.az_steps * gen.num_ch


# ----------------------------------------------------------------------------------------
def run_batched(gens, precision='mixed', tuner=None, pulse_block=None, max_slots=None):
    """Run prepared scenes to completion in one SceneBatch; returns a report with the
    device time of the run (CUDA events, tuning excluded) and the tuned shapes."""
    import torch
    from .radarsim.batch import SceneBatch
    n = len(gens)
    batch = SceneBatch(max_slots=max_slots or max(1, n), precision=precision)
    for g in gens:
        batch.add(g)
    tuned_rows, t_tune = {}, 0.0
    if tuner is not None:
        t0 = time.perf_counter()
        tuned_rows, block = tuner.tune(batch)
        t_tune = time.perf_counter() - t0
        pulse_block = pulse_block or block
    pulse_block = pulse_block or 32
    launches = batch.launches_per_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps0 = batch.steps_run
    kernel_launches = [0]
    e0.record()
    t0 = time.perf_counter()
    while True:
        for s in batch.finished():
            batch.remove(s)
        live = batch.live()
        if not live:
            break
        k = min(pulse_block, min(batch.remaining(s) for s in live))
        kernel_launches[0] += k * batch.launches_per_step()
        batch.graph_step(k)
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) * 1e-3
    echoes = sum(scene_echoes(g) for g in gens)
    rep = dict(scenes=n, echoes=echoes, device_s=dev_s, wall_s=wall, echoes_per_s=echoes / dev_s,
               steps=batch.steps_run - steps0, pulse_block=pulse_block, tile_rows={
                   '%dx%d/%d%s' % (k[0], k[1], k[2], '/ka' if k[3] else ''): v for k, v in tuned_rows.items()}, tune_s=t_tune,
               launches_first_step=launches, kernel_launches=kernel_launches[0])
    batch.close()
    return rep


# ----------------------------------------------------------------------------------------
class _Req(object):
    __slots__ = ('i', 'spec', 'arrival', 'need', 'future', 'gen', 'slot', 't_admit', 't_start',
                 't_done', 'host_raw', 'event', 'echoes', 'nrcs')


class ServingLoop(object):
    """Continuous batching of scene requests on one GPU (see the module docstring).

    ``hbm_budget`` bounds the device memory of the scenes admitted at once (bytes, by
    ``RawGenerator.device_bytes``); ``max_slots`` the scenes running at once;
    ``pulse_block`` the steps enqueued between admission decisions.  ``keep_results``
    keeps every request's raw cube (host) and NRCS for inspection.
    """

    def __init__(self, precision='mixed', hbm_budget=150e9, max_slots=64, pulse_block=16, preparer=None,
                 tuner=None, keep_results=False, time_scale=1.0):
        self.precision = precision
        self.hbm_budget = float(hbm_budget)
        self.max_slots = int(max_slots)
        self.pulse_block = int(pulse_block)
        self.preparer = preparer if preparer is not None else ScenePreparer()
        self.tuner = tuner
        self.keep_results = keep_results
        self.time_scale = float(time_scale)

    def run(self, specs):
        import torch
        from .radarsim.batch import SceneBatch
        batch = SceneBatch(max_slots=self.max_slots, precision=self.precision)
        reqs = []
        for i, sp in enumerate(sorted(specs, key=lambda s: s['arrival'])):
            r = _Req()
            r.i, r.spec, r.arrival = i, sp, sp['arrival'] * self.time_scale
            r.future = r.gen = r.slot = r.host_raw = r.event = r.nrcs = r.need = None
            r.t_admit = r.t_start = r.t_done = None
            r.echoes = 0.0
            reqs.append(r)
        waiting = collections.deque(reqs)         # not yet admitted (arrival order)
        preparing = collections.deque()           # admitted, host set-up running
        ready = collections.deque()               # prepared, waiting for a slot
        running = {}                              # slot -> request
        retiring = []                             # raw cube copy to the host in flight
        inflight = collections.deque()            # events of enqueued blocks
        reserved = 0.0
        busy = 0.0                                # device time of the enqueued blocks
        peak_reserved = 0.0
        max_backlog = 0
        stream = torch.cuda.current_stream()
        t0 = time.perf_counter()
        first = None
        while waiting or preparing or ready or running or retiring:
            now = time.perf_counter() - t0
            # 1. admission: arrived requests in order, while their memory fits the budget
            while waiting and waiting[0].arrival <= now:
                r = waiting[0]
                if r.need is None:
                    r.need = self._need(r.spec)
                if reserved + r.need > self.hbm_budget and (running or preparing or ready or retiring):
                    break
                waiting.popleft()
                reserved += r.need
                peak_reserved = max(peak_reserved, reserved)
                r.t_admit = now
                r.future = self.preparer.submit(r.spec, self.precision)
                preparing.append(r)
            max_backlog = max(max_backlog, len(preparing) + len(ready) +
                              sum(1 for r in waiting if r.arrival <= now))
            # 2. prepared scenes, in admission order
            while preparing and preparing[0].future.done():
                r = preparing.popleft()
                r.gen = r.future.result()
                r.future = None
                ready.append(r)
            # 3. into free slots: the batch keeps running around them
            while ready and batch.free_slots():
                r = ready.popleft()
                rows = self.tuner.tile_rows_for(self.precision, (r.gen.surface.Nx, r.gen.surface.Ny,
                                                                 r.gen.npol * r.gen.num_ch)) if self.tuner else 0
                r.slot = batch.add(r.gen, tile_rows=rows)
                r.t_start = time.perf_counter() - t0
                r.echoes = scene_echoes(r.gen)
                running[r.slot] = r
                if first is None:
                    first = r.t_start
            # 4. finished scenes: raw cube to pinned host memory, slot freed
            for s in batch.finished():
                r = running.pop(s)
                batch.remove(s)
                r.host_raw = torch.empty(r.gen.raw_d.shape, dtype=r.gen.raw_d.dtype, pin_memory=True)
                r.host_raw.copy_(r.gen.raw_d, non_blocking=True)
                if self.keep_results:
                    r.nrcs = (r.gen.nrcs_spec_d.clone(), r.gen.nrcs_bragg_d.clone(), list(r.gen._refreshes))
                r.event = torch.cuda.Event()
                r.event.record(stream)
                retiring.append(r)
            # 5. one block of steps for the live scenes
            live = batch.live()
            if live:
                k = min(self.pulse_block, min(batch.remaining(s) for s in live))
                b0 = torch.cuda.Event(enable_timing=True)
                b0.record(stream)
                batch.graph_step(k)
                b1 = torch.cuda.Event(enable_timing=True)
                b1.record(stream)
                inflight.append((b0, b1))
                while len(inflight) > 2:            # keep the host at most two blocks ahead
                    e0, e1 = inflight.popleft()
                    e1.synchronize()
                    busy += e0.elapsed_time(e1) * 1e-3
            # 6. retired requests whose copy has landed
            still = []
            for r in retiring:
                if r.event.query():
                    r.t_done = time.perf_counter() - t0
                    if self.keep_results:
                        r.nrcs = self._nrcs(r.gen, r.nrcs)
                    else:
                        r.host_raw = None
                    r.gen = None                    # device buffers go back to the allocator
                    reserved -= r.need
                else:
                    still.append(r)
            retiring = still
            if not live and not retiring:
                if ready or preparing or (waiting and waiting[0].arrival > time.perf_counter() - t0):
                    time.sleep(0.0005)
        torch.cuda.synchronize()
        for e0, e1 in inflight:
            busy += e0.elapsed_time(e1) * 1e-3
        t_end = time.perf_counter() - t0
        batch.close()
        lat = np.array([r.t_done - r.arrival for r in reqs])
        echoes = sum(r.echoes for r in reqs)
        span = max(r.t_done for r in reqs) - (min(r.arrival for r in reqs) if reqs else 0.0)
        offered = echoes / max(1e-9, (max(r.arrival for r in reqs) if reqs else 1.0))
        rep = dict(requests=len(reqs), echoes=echoes, wall_s=t_end, span_s=span,
                   echoes_per_s=echoes / span if span > 0 else 0.0,
                   offered_echoes_per_s=offered,
                   latency_p50_s=float(np.percentile(lat, 50)), latency_p99_s=float(np.percentile(lat, 99)),
                   latency_max_s=float(lat.max()), peak_reserved_bytes=peak_reserved, max_backlog=max_backlog,
                   gpu_busy_s=busy, gpu_busy_frac=busy / span if span > 0 else 0.0,
                   capacity_echoes_per_s=echoes / busy if busy > 0 else 0.0,
                   # the queue is stable when the offered load is below what the GPU
                   # sustains while it has work (echoes per busy second)
                   queue_stable=bool(busy > 0 and offered < echoes / busy))
        self.requests = reqs
        return rep

    def _need(self, spec):
        """Device bytes of a request's scene, from its parameters (before any set-up)."""
        from .radarsim.sar_raw_nompi import scene_device_bytes
        p = spec['params']
        n = int(round(p['L'] / p['d']))
        # range bins are derived from the geometry; bound them by the ground-range span
        bins = int(np.ceil(n * p['d'] * 1.1 / (C_LIGHT / (2 * 50e6)))) + 2048
        return scene_device_bytes(n, n, 8, 1, p['num_ch'], spec['pulses'], bins, self.precision)

    @staticmethod
    def _nrcs(gen, saved):
        spec_d, bragg_d, refreshes = saved
        gen._refreshes = refreshes
        gen.nrcs_spec_d, gen.nrcs_bragg_d = spec_d, bragg_d
        return gen.nrcs_avg()
