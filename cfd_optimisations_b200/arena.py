"""Many meshes in one device arena (include/hcfd_gpu.h, hcfd_arena_*): batched solves and the
building block of the serving loop (serve.py)."""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import native as _n
from . import FP32, GLOBAL_CFL, LIMITER_BJ, Mesh


class Arena:
    """An arena with an HBM budget; admit meshes, advance all of them together, retire."""

    def __init__(self, hbm_budget: int, precision: int = FP32, limiter: int = LIMITER_BJ, venkat_K: float = 5.0,
                 gma: float = 1.4, time_mode: int = GLOBAL_CFL, tile: int = 0, slots: int = 3,
                 max_instances: int = 1024, freeze_limiter_after: int = 0):
        p = _n.ArenaParams(int(hbm_budget), precision, limiter, venkat_K, gma, time_mode, tile, slots, max_instances,
                           freeze_limiter_after)
        h = ct.c_void_p()
        _n.check(_n.lib().hcfd_arena_create(ct.byref(p), ct.byref(h)))
        self._h = h
        self.gma = gma
        self.max_instances = max_instances
        self._mesh = {}
        self._nc = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _n.lib().hcfd_arena_destroy(h)
            self._h = None

    def admit(self, mesh: Mesh, bcmap, qbc, qic, dt_or_cfl: float):
        """Returns the instance slot, or None when the arena is full (HCFD_EAGAIN)."""
        v = mesh.view()
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
        qi = np.ascontiguousarray(qic, dtype=np.float64)
        slot = ct.c_int()
        rc = _n.lib().hcfd_arena_admit(self._h, ct.byref(v), bm.ctypes.data_as(_n._ip), len(bm),
                                       q.ctypes.data_as(_n._dp), qi.ctypes.data_as(_n._dp), dt_or_cfl, ct.byref(slot))
        if rc == _n.EAGAIN:
            return None
        _n.check(rc)
        self._mesh[slot.value] = mesh
        self._nc[slot.value] = v.Nc
        return slot.value

    def prepare(self, mesh: Mesh, bcmap, qbc, qic, dt_or_cfl: float) -> "Admission":
        """The host half of admit (tile plan, BC table); safe to call from worker threads
        while another thread steps the arena."""
        v = mesh.view()
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
        qi = np.ascontiguousarray(qic, dtype=np.float64)
        h = ct.c_void_p()
        _n.check(_n.lib().hcfd_arena_prepare(self._h, ct.byref(v), bm.ctypes.data_as(_n._ip), len(bm),
                                             q.ctypes.data_as(_n._dp), qi.ctypes.data_as(_n._dp), dt_or_cfl,
                                             ct.byref(h)))
        return Admission(h, mesh, v.Nc)

    def admit_prepared(self, adm: "Admission"):
        """The device half of admit; returns the slot, or None when the arena is full (the
        admission stays usable)."""
        slot = ct.c_int()
        rc = _n.lib().hcfd_arena_admit_prepared(self._h, adm._h, ct.byref(slot))
        if rc == _n.EAGAIN:
            return None
        _n.check(rc)
        self._mesh[slot.value] = adm.mesh
        self._nc[slot.value] = adm.Nc
        return slot.value

    def step(self, nsteps: int) -> None:
        _n.check(_n.lib().hcfd_arena_step(self._h, nsteps))

    def poll(self) -> dict:
        """{slot: stats dict} of the active instances (waits for the device)."""
        n = ct.c_int()
        slots = (ct.c_int * self.max_instances)()
        st = (_n.StepStats * self.max_instances)()
        _n.check(_n.lib().hcfd_arena_poll(self._h, self.max_instances, slots, st, ct.byref(n)))
        return {slots[i]: dict(dt=st[i].dt, res_l2=st[i].res_l2, res_first=st[i].res_first, steps=st[i].steps,
                               nonfinite=bool(st[i].nonfinite)) for i in range(n.value)}

    def fetch(self, slot: int, prims: bool = False) -> np.ndarray:
        out = np.empty((4, self._nc[slot]))
        ptrs = (ct.POINTER(ct.c_double) * 4)(*[out[v].ctypes.data_as(_n._dp) for v in range(4)])
        _n.check(_n.lib().hcfd_arena_fetch(self._h, slot, 1 if prims else 0, ptrs))
        return out

    def checkpoint(self, slot: int, path: str) -> None:
        """Exact snapshot of one instance (the format of Solver.checkpoint)."""
        _n.check(_n.lib().hcfd_arena_checkpoint(self._h, slot, os.fsencode(path)))

    def restore(self, slot: int, path: str) -> None:
        """Loads a checkpoint into an admitted instance of the same mesh."""
        _n.check(_n.lib().hcfd_arena_restore(self._h, slot, os.fsencode(path)))

    def release(self, slot: int) -> None:
        _n.check(_n.lib().hcfd_arena_release(self._h, slot))
        self._mesh.pop(slot, None)
        self._nc.pop(slot, None)

    def info(self) -> dict:
        i = _n.ArenaInfo()
        _n.check(_n.lib().hcfd_arena_info(self._h, ct.byref(i)))
        return {k: getattr(i, k) for k, _ in _n.ArenaInfo._fields_}


class Admission:
    """A prepared admission (hcfd_arena_prepare); holds the mesh it was built from."""

    def __init__(self, h, mesh: Mesh, Nc: int):
        self._h = h
        self.mesh = mesh
        self.Nc = Nc
        self.cells = int(_n.lib().hcfd_admission_cells(h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _n.lib().hcfd_admission_free(h)
            self._h = None
