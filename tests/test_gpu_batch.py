"""Scene batch (``ocs_batch_*``) against the same scenes run one at a time.

Every scene of a batch must produce the raw cube and NRCS that ``RawGenerator.run`` gives
for it alone: the batch runs the same per-pulse body with the same inputs, only the
order of the floating-point atomics of the accumulation differs.  Bars: relative L2 of the
raw cube 1e-5 (mixed: float32 accumulation) and 1e-12 (FP64), NRCS 1e-6 / 1e-12.

The mix covers four transform-length classes (64 x 64, 64 x 32, 256 x 256 and the generic
mixed-radix 48 x 54), one to four channels, dual polarisation, cross-track baselines,
directional swell, Kirchhoff specular scenes (facet approach and stationary phase, which
form pulse-kernel classes of their own), a choppy surface and pulse counts that differ, so
scenes finish at different steps.
"""
import os
import tempfile

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def scene_cfgs(tmp):
    """(cfg path, seed, overrides) of the mixed scene set."""
    import bench
    out = [(os.path.join(G, "cfg", "c1small.cfg"), 0, None),
           (os.path.join(G, "cfg", "c3small.cfg"), 1, None)]
    # the dual-polarisation two-channel case without choppy waves
    txt = open(os.path.join(G, "cfg", "c2small.cfg")).read().replace("choppy_enable=True", "choppy_enable=False")
    p = os.path.join(tmp, "c2nochop.cfg")
    open(p, "w").write(txt)
    out.append((p, 2, None))
    c = dict(bench.C1, L=256, pulses=48, bins=256, wind_U=12.0, wind_dir=30.0, num_ch=2, b_ati=5.0)
    out.append((bench.write_cfg(c, os.path.join(tmp, "s256.cfg")), 3, bench.overrides(c)))
    c = dict(bench.C1, L=256, pulses=80, bins=256, wind_U=6.0, wind_dir=200.0)
    out.append((bench.write_cfg(c, os.path.join(tmp, "s256b.cfg")), 4, bench.overrides(c)))
    # Kirchhoff specular scenes (their own pulse-kernel class): facet approach in dual
    # polarisation, stationary phase in vv
    out.append((os.path.join(G, "cfg", "c1fa.cfg"), 5, None))
    out.append((os.path.join(G, "cfg", "c1spa.cfg"), 6, None))
    # the choppy dual-polarisation case (slope / curvature step after the column pass)
    out.append((os.path.join(G, "cfg", "c2small.cfg"), 7, None))
    return out


def alone(cfgs, precision):
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator
    res = []
    for cfg, seed, ov in cfgs:
        g = RawGenerator(cfg, precision=precision, overrides=ov, seed=seed)
        g.run()
        res.append((g.raw(), g.nrcs_avg()))
        del g
    return res


def check(res, ref, precision):
    tol_raw = 1e-5 if precision == "mixed" else 1e-12
    tol_nrcs = 1e-6 if precision == "mixed" else 1e-12
    for (raw, nrcs), (raw0, nrcs0) in zip(res, ref):
        assert raw.shape == raw0.shape
        assert np.isfinite(raw).all()
        assert rel_l2(raw, raw0) <= tol_raw, rel_l2(raw, raw0)
        assert rel_l2(nrcs, nrcs0) <= tol_nrcs, rel_l2(nrcs, nrcs0)


@pytest.mark.parametrize("precision", ["mixed", "f64"])
@pytest.mark.parametrize("graphs", [False, True])
def test_batch_matches_scenes_alone(precision, graphs):
    from oceansar_b200 import build
    from oceansar_b200.radarsim.batch import SceneBatch
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator
    build.build()
    with tempfile.TemporaryDirectory() as tmp:
        cfgs = scene_cfgs(tmp)
        ref = alone(cfgs, precision)
        b = SceneBatch(max_slots=8, precision=precision)
        gens = [RawGenerator(cfg, precision=precision, overrides=ov, seed=seed) for cfg, seed, ov in cfgs]
        for g in gens:
            b.add(g)
        assert b.launches_per_step() >= 6
        finished = []
        b.run(pulse_block=16, use_graphs=graphs, on_finish=lambda s, g: finished.append(s))
        torch.cuda.synchronize()
        assert sorted(finished) == list(range(len(cfgs)))
        check([(g.raw(), g.nrcs_avg()) for g in gens], ref, precision)
        b.close()


def test_batch_admits_scenes_while_others_run():
    """Continuous batching: a scene put into a slot while others are mid-way gives the
    same result, and a freed slot is reused."""
    from oceansar_b200.radarsim.batch import SceneBatch
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator
    with tempfile.TemporaryDirectory() as tmp:
        cfgs = scene_cfgs(tmp)
        ref = alone(cfgs, "mixed")
        b = SceneBatch(max_slots=2, precision="mixed")
        gens = [RawGenerator(cfg, precision="mixed", overrides=ov, seed=seed) for cfg, seed, ov in cfgs]
        pending = list(range(len(gens)))
        placed = {}
        done = []
        while pending or b.slots():
            for s in b.finished():
                done.append(placed.pop(s))
                b.remove(s)
            while pending and b.free_slots():
                i = pending.pop(0)
                placed[b.add(gens[i])] = i
            live = b.live()
            if live:
                b.graph_step(min(7, min(b.remaining(s) for s in live)))
        torch.cuda.synchronize()
        assert sorted(done) == list(range(len(gens)))
        counters = b.counters()
        assert all(c == -1 for c in counters)
        check([(g.raw(), g.nrcs_avg()) for g in gens], ref, "mixed")
        b.close()


def test_batch_counters_and_errors():
    from oceansar_b200.radarsim.batch import SceneBatch
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator
    b = SceneBatch(max_slots=4, precision="mixed")
    g = RawGenerator(os.path.join(G, "cfg", "c1small.cfg"), precision="mixed", seed=0)
    s = b.add(g, slot=2)
    assert s == 2
    b.step(5)
    c = b.counters()
    assert c[2] == 5 and c[0] == -1 and c[1] == -1 and c[3] == -1
    with pytest.raises(ValueError):
        b.add(g, slot=2)                       # occupied
    with pytest.raises(ValueError):
        b.add(RawGenerator(os.path.join(G, "cfg", "c1small.cfg"), precision="f64", seed=0))
    b.step(1000)                               # runs to the end, then nothing more
    assert b.counters()[2] == g.az_steps
    b.close()
