"""Autotuner of the scene batch's launch shapes.

Two shapes are chosen by measurement on the GPU, for the scenes actually in the batch:

* ``tile_rows`` -- facet rows per pulse-kernel tile, per scene class (grid size and number
  of outputs).  Small scenes want short tiles (more CTAs for few facets), large ones long
  tiles (the register bin windows stay warm for longer).  Candidates are timed one class
  at a time on the whole batch (coordinate search), every other class at its current
  choice.
* ``pulse_block`` -- steps per CUDA-graph replay.  Longer blocks amortise the host's
  replay cost; shorter ones let a serving loop admit and retire scenes sooner.  Each
  candidate is timed by wall clock (host and device) over a replayed block.

Choices are cached in a JSON file (``$OCEANSAR_B200_TUNE_CACHE``, default
``~/.cache/oceansar_b200/tune.json``) keyed by device name, precision and class, so a
second run on the same machine skips the measurements.
"""
import json
import os
import time

import torch

TILE_ROWS = (16, 32, 64, 128)
PULSE_BLOCKS = (4, 16, 64)


def _default_path():
    return os.environ.get('OCEANSAR_B200_TUNE_CACHE') or os.path.join(
        os.path.expanduser('~'), '.cache', 'oceansar_b200', 'tune.json')


class Autotuner(object):
    def __init__(self, path=None, tile_rows=TILE_ROWS, pulse_blocks=PULSE_BLOCKS, steps=4, use_cache=True):
        self.path = path or _default_path()
        self.tile_rows_candidates = tuple(tile_rows)
        self.pulse_block_candidates = tuple(pulse_blocks)
        self.steps = int(steps)
        self.use_cache = use_cache
        self.cache = {}
        if use_cache and os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.cache = json.load(f)
            except (OSError, ValueError):
                self.cache = {}
        self.measurements = []           # (what, key, candidate, seconds per step)

    # ------------------------------------------------------------------------------------
    def _key(self, kind, precision, cls):
        name = torch.cuda.get_device_name() if torch.cuda.is_available() else 'cpu'
        return '|'.join([name, kind, precision, 'x'.join(str(v) for v in cls)])

    def save(self):
        if not self.use_cache:
            return
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            with open(self.path, 'w') as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
        except OSError:
            pass

    def tile_rows_for(self, precision, cls, default=64):
        """Cached tile height of a scene class (``default`` if never tuned)."""
        return int(self.cache.get(self._key('tile_rows', precision, cls), default))

    # ------------------------------------------------------------------------------------
    def _time_steps(self, batch, n):
        """Device seconds per step of the batch over n plain steps (after one warm-up)."""
        batch.step(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.step(n)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / n

    def tune_tile_rows(self, batch):
        """Choose the tile height of every scene class present; returns {class: rows}."""
        classes = {}
        for s in batch.slots():
            classes.setdefault(batch.scene_class(s), []).append(s)
        chosen = {}
        for cls, slots in sorted(classes.items()):
            key = self._key('tile_rows', batch.precision, cls)
            if key in self.cache:
                chosen[cls] = int(self.cache[key])
            else:
                best = None
                for cand in self.tile_rows_candidates:
                    for s in batch.slots():
                        batch.restart(s, cand if s in slots else None)
                    t = self._time_steps(batch, self.steps)
                    self.measurements.append(('tile_rows', cls, cand, t))
                    if best is None or t < best[0]:
                        best = (t, cand)
                chosen[cls] = best[1]
                self.cache[key] = best[1]
            for s in slots:
                batch.restart(s, chosen[cls])
        return chosen

    def tune_pulse_block(self, batch):
        """Choose the steps per graph replay for the batch's composition."""
        comp = sorted(batch.scene_class(s) for s in batch.slots())
        cls = (len(comp),) + tuple(v for c in comp for v in c)
        key = self._key('pulse_block', batch.precision, cls[:64])
        if key in self.cache:
            return int(self.cache[key])
        best = None
        for cand in self.pulse_block_candidates:
            for s in batch.slots():
                batch.restart(s)
            batch.graph_step(cand)                 # plain launches (first use)
            batch.graph_step(cand)                 # recorded and replayed
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            batch.graph_step(cand)
            torch.cuda.synchronize()
            t = (time.perf_counter() - t0) / cand
            self.measurements.append(('pulse_block', None, cand, t))
            if best is None or t < best[0] * 0.97:  # prefer shorter blocks unless clearly slower
                best = (t, cand)
        self.cache[key] = best[1]
        return best[1]

    def tune(self, batch):
        """Tile heights, then the pulse block; every scene restarts from pulse 0 after."""
        rows = self.tune_tile_rows(batch)
        block = self.tune_pulse_block(batch)
        for s in batch.slots():
            batch.restart(s)
        torch.cuda.synchronize()
        self.save()
        return rows, block
