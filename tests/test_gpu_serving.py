"""Serving loop and batched runner on the GPU.

The continuous-batching test sends a staggered stream of small requests through a
``ServingLoop`` with fewer slots than requests, so scenes are admitted while others run
and freed slots are reused, and checks that every request's raw cube and NRCS equal those
of the same scene run alone (``RawGenerator.run``) within the batch tolerance (relative
L2 1e-5 for the mixed form, whose float32 atomics may add in another order).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def spec(L, pulses, seed, nch, arrival, wind_dir=30.0):
    from oceansar_b200.serving import CFG_TEMPLATE
    params = dict(L=L, d=1.0, wind_U=9.0, wind_dir=wind_dir, inc=32.0, pol='vv', prf=1000.0, ant_l=2.742,
                  num_ch=nch, b_ati=4.0)
    return dict(cfg=CFG_TEMPLATE.format(**params), seed=seed, overrides=dict(az_steps=pulses),
                params=params, pulses=pulses, arrival=arrival)


def alone(s, precision):
    from oceansar_b200.serving import prepare_scene
    g = prepare_scene(s, precision).to_device()
    g.run()
    return g.raw(), g.nrcs_avg()


@pytest.mark.parametrize("workers", [0, 2])
def test_serving_results_equal_alone(workers):
    from oceansar_b200.serving import ScenePreparer, ServingLoop
    specs = [spec(128, 60, 11, 1, 0.00), spec(256, 40, 12, 2, 0.01, 100.0), spec(64, 90, 13, 3, 0.02),
             spec(128, 30, 14, 2, 0.05, 250.0), spec(256, 50, 15, 1, 0.06), spec(64, 20, 16, 1, 0.30)]
    prep = ScenePreparer(workers=workers)
    try:
        loop = ServingLoop(precision='mixed', hbm_budget=8e9, max_slots=3, pulse_block=8, preparer=prep,
                           keep_results=True)
        rep = loop.run(specs)
    finally:
        prep.close()
    assert rep['requests'] == len(specs)
    assert rep['latency_p50_s'] > 0 and rep['latency_p99_s'] >= rep['latency_p50_s']
    assert rep['echoes_per_s'] > 0
    by_i = {r.i: r for r in loop.requests}
    for i, s in enumerate(sorted(specs, key=lambda s: s['arrival'])):
        r = by_i[i]
        raw = r.host_raw.numpy().reshape(1, s['params']['num_ch'], s['pulses'], -1)
        raw0, nrcs0 = alone(s, 'mixed')
        assert raw.shape == raw0.shape
        assert rel_l2(raw, raw0) <= 1e-5, (i, rel_l2(raw, raw0))
        assert rel_l2(r.nrcs, nrcs0) <= 1e-6


def test_serving_budget_limits_admission():
    """A budget that fits one scene at a time serialises the requests but completes them."""
    from oceansar_b200.serving import ScenePreparer, ServingLoop
    specs = [spec(128, 20, 21, 1, 0.0), spec(128, 20, 22, 1, 0.0), spec(128, 20, 23, 1, 0.0)]
    prep = ScenePreparer(workers=0)
    loop = ServingLoop(precision='mixed', hbm_budget=1.0, max_slots=4, pulse_block=4, preparer=prep)
    rep = loop.run(specs)
    assert rep['requests'] == 3
    assert rep['peak_reserved_bytes'] <= max(r.need for r in loop.requests) * 1.0001
    starts = sorted(r.t_start for r in loop.requests)
    dones = sorted(r.t_done for r in loop.requests)
    assert starts[1] >= dones[0] - 1e-3 and starts[2] >= dones[1] - 1e-3


def test_run_batched_with_autotuner(tmp_path):
    from oceansar_b200.serving import prepare_scene, run_batched
    from oceansar_b200.tune import TILE_ROWS, Autotuner
    specs = [spec(128, 40, 31, 1, 0.0), spec(256, 24, 32, 2, 0.0), spec(128, 33, 33, 3, 0.0)]
    gens = [prepare_scene(s, 'mixed') for s in specs]
    tuner = Autotuner(path=str(tmp_path / 't.json'), steps=2, pulse_blocks=(2, 4))
    rep = run_batched(gens, precision='mixed', tuner=tuner)
    torch.cuda.synchronize()
    assert rep['scenes'] == 3 and rep['echoes_per_s'] > 0
    assert rep['pulse_block'] in (2, 4)
    assert set(rep['tile_rows'].values()) <= set(TILE_ROWS)
    for s, g in zip(specs, gens):
        raw0, _ = alone(s, 'mixed')
        assert rel_l2(g.raw(), raw0) <= 1e-5
