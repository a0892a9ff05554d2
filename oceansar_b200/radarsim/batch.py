"""Scene batch: many independent ``sar_raw`` scenes on one GPU at once.

The reference simulates one scene per ``sar_raw`` call (``sar_raw_nompi.py:32-641``).  Here
every scene is a ``RawGenerator`` (the same host set-up, the same device buffers) placed in
a slot of the C-ABI scene batch (``ocs_batch_*``).  One step advances every live scene by
one pulse -- exactly the per-pulse body that ``RawGenerator.pulse`` runs -- with one launch
per transform-length class of the row and column passes, one row-table launch and one
pulse-kernel launch per output width, whatever the number of scenes.  The per-pulse
inputs (time, azimuth, refresh decisions, scatterer offsets) are uploaded once per scene
as device tables and a device-side pulse counter selects them, so a step needs no host
arguments and a run of steps can be recorded once into a CUDA graph and replayed.

Scenes of any grid size, geometry, channel count and pulse count mix freely.  A scene's
raw cube and NRCS are those of the same scene run alone (``RawGenerator.run``) up to the
order of the floating-point atomics of the accumulation.
"""
import ctypes

import numpy as np
import torch

from .. import _capi, _device
from .._structs import SceneDesc
from .sar_raw_nompi import PRECISIONS


class _Slot(object):
    __slots__ = ("gen", "tables", "desc", "sdesc", "cdesc", "done", "tile_rows", "key")


class SceneBatch(object):
    """Engine with ``max_slots`` scene slots for one precision ('mixed' or 'f64').

    ``add(gen)`` puts a ``RawGenerator`` in a free slot (its raw cube and NRCS restart from
    zero), ``step(n)`` enqueues n pulses of every live scene, ``finished()`` lists the
    slots whose scene has run all its pulses and ``remove(slot)`` frees a slot.
    ``run(pulse_block)`` drives everything present to completion with CUDA graphs of
    ``pulse_block`` steps.  All work is enqueued on ``stream`` (default: the current one).
    """

    def __init__(self, max_slots=64, precision='mixed', stream=None):
        if precision not in PRECISIONS:
            raise ValueError('precision must be f64 or mixed')
        self.precision = precision
        self.max_slots = int(max_slots)
        self.stream = stream
        h = ctypes.c_void_p()
        _capi.call("ocs_batch_create", self.max_slots, PRECISIONS[precision], ctypes.byref(h))
        self._h = h
        self._slots = [None] * self.max_slots
        self._upload = torch.cuda.Stream()
        self._graphs = {}
        self.max_graphs = 64
        self.steps_run = 0

    # ------------------------------------------------------------------------------------
    def close(self):
        if self._h is not None and self._h.value:
            self._graphs.clear()
            _capi.call("ocs_batch_destroy", self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sp(self):
        return _device.stream_ptr(self.stream)

    # ------------------------------------------------------------------------------------
    def free_slots(self):
        return [i for i, s in enumerate(self._slots) if s is None]

    def slots(self):
        """Occupied slot indices."""
        return [i for i, s in enumerate(self._slots) if s is not None]

    def generator(self, slot):
        return self._slots[slot].gen

    def add(self, gen, slot=None, tile_rows=0):
        """Place ``gen`` (a RawGenerator of this batch's precision) in a slot; returns it."""
        if gen.precision != self.precision:
            raise ValueError('scene precision %s differs from the batch (%s)' % (gen.precision, self.precision))
        if slot is None:
            free = self.free_slots()
            if not free:
                raise RuntimeError('no free slot')
            slot = free[0]
        if self._slots[slot] is not None:
            raise ValueError('slot %d is occupied' % slot)
        # uploads go on a stream of their own, so that placing a scene never waits for the
        # steps already enqueued; the batch's stream then waits for the uploads
        with torch.cuda.stream(self._upload):
            gen.to_device()
            sched = getattr(gen, '_batch_schedule', None)
            if sched is None:
                tables, refreshes, t_last = gen.pulse_schedule()
                dev = {k: (None if v is None else _device.to_device(v, v.dtype)) for k, v in tables.items()}
                sched = gen._batch_schedule = (dev, refreshes, t_last)
        dev, refreshes, t_last = sched
        compute = self.stream if self.stream is not None else torch.cuda.current_stream()
        compute.wait_stream(self._upload)
        with torch.cuda.stream(compute):
            gen.reset()
        gen._refreshes = list(refreshes)
        d = gen.desc
        d.az_step, d.az_now, d.refresh, d.tind = 0, 0.0, 0, 0
        sdesc = gen.surface.update_desc()
        p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        # choppy surfaces: the slope / curvature step after the column pass (its swell
        # rotation comes from the per-pulse table)
        cdesc = gen.surface.choppy_desc() if gen.surface._aux else None
        desc = SceneDesc(ctypes.addressof(sdesc), ctypes.addressof(d), int(tile_rows), p(dev['t']),
                         p(dev['add']), p(dev['swell_rot']), p(dev['az_now']), p(dev['flags']), p(dev['tmod']),
                         ctypes.addressof(cdesc) if cdesc is not None else None)
        _capi.call("ocs_batch_set", self._h, int(slot), ctypes.addressof(desc), self._sp())
        gen.t_last_rcs_bragg = t_last
        s = _Slot()
        s.gen, s.tables, s.desc, s.sdesc, s.done = gen, dev, desc, sdesc, 0
        s.cdesc = cdesc
        s.tile_rows = int(tile_rows) if tile_rows else 64
        s.key = (gen.surface.Nx, gen.surface.Ny, tuple(c for c, _, _, _ in gen.surface._raw),
                 gen.npol * gen.num_ch, s.tile_rows, self._kirchhoff(gen))
        self._slots[slot] = s
        return slot

    def restart(self, slot, tile_rows=None):
        """Put a slot's scene back to pulse 0 (raw cube and NRCS cleared), optionally with
        another pulse-kernel tile height (used by the autotuner)."""
        s = self._slots[slot]
        rows = s.tile_rows if tile_rows is None else int(tile_rows)
        self._slots[slot] = None
        _capi.call("ocs_batch_clear", self._h, int(slot), self._sp())
        self.add(s.gen, slot=slot, tile_rows=rows)

    def tile_rows(self, slot):
        return self._slots[slot].tile_rows

    @staticmethod
    def _kirchhoff(gen):
        """Whether the scene's specular term is a Kirchhoff model (its own pulse-kernel class)."""
        return bool(gen.scat_spec_enable and gen.scat_spec_mode != 'kodis')

    def scene_class(self, slot):
        """(Nx, Ny, outputs, Kirchhoff): scenes of one class share their launch shapes."""
        g = self._slots[slot].gen
        return (g.surface.Nx, g.surface.Ny, g.npol * g.num_ch, self._kirchhoff(g))

    def remove(self, slot):
        """Free a slot (the scene's buffers stay with its RawGenerator)."""
        if self._slots[slot] is None:
            return
        _capi.call("ocs_batch_clear", self._h, int(slot), self._sp())
        self._slots[slot] = None

    # ------------------------------------------------------------------------------------
    def step(self, pulses=1):
        """Enqueue ``pulses`` steps (no graph)."""
        _capi.call("ocs_batch_step", self._h, int(pulses), self._sp())
        self._advance(pulses)

    def _advance(self, pulses):
        self.steps_run += pulses
        for s in self._slots:
            if s is not None:
                s.done = min(s.gen.az_steps, s.done + pulses)

    def remaining(self, slot):
        s = self._slots[slot]
        return s.gen.az_steps - s.done

    def finished(self):
        return [i for i, s in enumerate(self._slots) if s is not None and s.done >= s.gen.az_steps]

    def live(self):
        return [i for i, s in enumerate(self._slots) if s is not None and s.done < s.gen.az_steps]

    def launches_per_step(self):
        return int(_capi.load().ocs_batch_launches_per_step(self._h))

    def counters(self):
        """Device pulse counters of all slots (-1: empty slot)."""
        out = (ctypes.c_int32 * self.max_slots)()
        _capi.call("ocs_batch_counters", self._h, ctypes.addressof(out), self._sp())
        return list(out)

    def composition(self):
        """Key of the launch sequence of a step: the occupied slots and their classes."""
        return tuple((i, s.key) for i, s in enumerate(self._slots) if s is not None)

    # ------------------------------------------------------------------------------------
    def graph_step(self, pulses):
        """Run ``pulses`` steps from a CUDA graph recorded for the current composition
        (recorded on first use; the first use of a composition runs plain launches)."""
        key = (self.composition(), int(pulses))
        g = self._graphs.get(key)
        if g is None:
            if not any(k[0] == key[0] for k in self._graphs):
                # first use of this composition: plain launches also set the kernels' shared-
                # memory limits before anything is recorded
                self.step(pulses)
                self._graphs[key] = None
                return
            cur = torch.cuda.current_stream() if self.stream is None else self.stream
            side = torch.cuda.Stream()
            side.wait_stream(cur)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                _capi.call("ocs_batch_step", self._h, int(pulses), ctypes.c_void_p(side.cuda_stream))
            cur.wait_stream(side)
            if len(self._graphs) >= self.max_graphs:
                for k in [k for k, v in self._graphs.items() if v is not None][:len(self._graphs) // 2]:
                    del self._graphs[k]
            self._graphs[key] = g
            # recording enqueued nothing: the steps still have to run
        with torch.cuda.stream(self.stream) if self.stream is not None else _nullctx():
            g.replay()
        self._advance(pulses)

    def run(self, pulse_block=32, on_finish=None, use_graphs=True):
        """Run every live scene to completion.  Steps go in blocks of at most
        ``pulse_block``, cut so that a block never runs past the end of a scene; finished
        scenes leave their slot (``on_finish(slot, gen)`` is called first) so that later
        blocks carry only live scenes."""
        while True:
            live = self.live()
            for i in self.finished():
                if on_finish is not None:
                    on_finish(i, self._slots[i].gen)
                self.remove(i)
            if not live:
                break
            n = min(int(pulse_block), min(self.remaining(i) for i in live))
            if use_graphs:
                self.graph_step(n)
            else:
                self.step(n)


class _nullctx(object):
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
