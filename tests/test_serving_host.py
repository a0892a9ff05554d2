"""Host side of the batched / served workloads (no GPU): workload draws, request stream,
scene preparation in spawned worker processes, memory estimates, autotuner cache."""
import pickle

import numpy as np


def test_batched_specs_are_seeded_and_in_range():
    from oceansar_b200.serving import batched_specs
    a = batched_specs(64, seed=1)
    b = batched_specs(64, seed=1)
    assert [s['cfg'] for s in a] == [s['cfg'] for s in b]
    assert [s['seed'] for s in a] == [s['seed'] for s in b]
    assert len(a) == 64
    for s in a:
        p = s['params']
        assert p['L'] in (256, 512, 1024, 2048)
        assert 3 <= p['wind_U'] <= 20 and 0 <= p['wind_dir'] <= 360 and 20 <= p['inc'] <= 45
        assert 1 <= p['num_ch'] <= 3 and (p['num_ch'] - 1) * p['b_ati'] <= 10 + 1e-9
        assert 512 <= s['pulses'] <= 4096
    assert len({s['params']['L'] for s in a}) == 4
    assert batched_specs(8, seed=2)[0]['cfg'] != a[0]['cfg']


def test_serving_requests_poisson():
    from oceansar_b200.serving import serving_requests
    r = serving_requests(rate=20.0, duration=60.0, seed=2)
    t = np.array([x['arrival'] for x in r])
    assert np.all(np.diff(t) > 0) and t[-1] < 60.0
    assert 1000 < len(r) < 1400                      # 20/s over 60 s
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 0.05) < 0.005
    assert serving_requests(rate=20.0, duration=60.0, seed=2)[5]['cfg'] == r[5]['cfg']


def small_spec(L=64, pulses=32, seed=0, nch=1):
    from oceansar_b200.serving import CFG_TEMPLATE
    params = dict(L=L, d=1.0, wind_U=8.0, wind_dir=30.0, inc=30.0, pol='vv', prf=1000.0, ant_l=2.742,
                  num_ch=nch, b_ati=5.0)
    return dict(cfg=CFG_TEMPLATE.format(**params), seed=seed, overrides=dict(az_steps=pulses),
                params=params, pulses=pulses, arrival=0.0)


def test_prepare_scene_host_only_and_pickles():
    from oceansar_b200.serving import prepare_scene
    g = prepare_scene(small_spec(), 'mixed')
    assert g.az_steps == 32 and g.surface.Nx == 64
    assert not g._on_device
    g2 = pickle.loads(pickle.dumps(g))
    np.testing.assert_array_equal(g2.surface.wave_coefs, g.surface.wave_coefs)
    assert g.device_bytes() > 64 * 64 * 40


def test_preparer_in_spawned_worker_matches_inline():
    from oceansar_b200.serving import ScenePreparer, prepare_scene
    p = ScenePreparer(workers=1)
    try:
        g = p.submit(small_spec(seed=5), 'f64').result(timeout=600)
    finally:
        p.close()
    h = prepare_scene(small_spec(seed=5), 'f64')
    np.testing.assert_array_equal(g.surface.wave_coefs, h.surface.wave_coefs)
    np.testing.assert_array_equal(g.rndscat_m.ind0, h.rndscat_m.ind0)


def test_scene_device_bytes_scales():
    from oceansar_b200.radarsim.sar_raw_nompi import scene_device_bytes
    a = scene_device_bytes(2048, 2048, 8, 1, 2, 4096, 2048, 'mixed')
    assert 480e6 < a < 560e6
    assert scene_device_bytes(2048, 2048, 8, 1, 2, 4096, 2048, 'f64') > a


def test_autotuner_cache_roundtrip(tmp_path):
    from oceansar_b200.tune import Autotuner
    t = Autotuner(path=str(tmp_path / 'tune.json'))
    t.cache[t._key('tile_rows', 'mixed', (256, 256, 2))] = 32
    t.save()
    u = Autotuner(path=str(tmp_path / 'tune.json'))
    assert u.tile_rows_for('mixed', (256, 256, 2)) == 32
    assert u.tile_rows_for('mixed', (512, 512, 2)) == 64
