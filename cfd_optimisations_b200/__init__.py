"""B200-native solver for the per-step residual-and-update loop of the 2-D unstructured
cell-centred finite-volume Euler solver of Hasti-Jalal-Aldeen/CFD_Optimisations.

The compute path is libhcfd_gpu.so (hand-written CUDA for sm_100a behind the C ABI of
include/hcfd_gpu.h).  This package is its Python binding:

* ``Mesh``    — .hmsh reader/writer, wedge generator, renumbering (the reference's Mesh,
                includes/Mesh.hpp).
* ``Solver``  — one mesh on one GPU: gather_bcs / initialise / step / download.
* ``GPU``     — classes with the names and signatures of the reference's Base layout
                (Domain, GaussGreen, Limiter, Flux, Euler, Writer), so a driver written
                against the reference swaps namespaces.
* ``arena``   — many meshes packed into one device arena (batched and served solves).

Nothing here computes on the CPU: without the native library or a CUDA device every
solver call raises.
"""
from __future__ import annotations

import ctypes as ct
import os
import struct

import numpy as np

from . import native as _n
from .native import (FIXED_DT, GLOBAL_CFL, LOCAL_CFL, FP32, FP64, KERNEL_CELL, KERNEL_TILED, LIMITER_BJ, LIMITER_VENKAT,
                     NUMBER_MORTON, NUMBER_NATURAL, NUMBER_RANDOM, NUMBER_RCM, SUBINLET, SUBOUTLET,
                     SUPINLET, SUPOUTLET, SYMMETRY, WALL, HcfdError)

__all__ = ["Mesh", "Solver", "HcfdError", "FIXED_DT", "GLOBAL_CFL", "LOCAL_CFL", "FP32", "FP64",
           "LIMITER_BJ", "LIMITER_VENKAT", "NUMBER_NATURAL", "NUMBER_RANDOM", "NUMBER_RCM",
           "NUMBER_MORTON", "SYMMETRY", "WALL", "SUPINLET", "SUBINLET", "SUPOUTLET", "SUBOUTLET",
           "write_hsln", "wedge_case", "checkpoint_info", "convert_checkpoint"]


def _dptr(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def _iptr(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_int))


class Mesh:
    """A host mesh owned by the native library (the reference's Mesh, src/Mesh.cpp)."""

    def __init__(self, path: str | None = None, _handle=None):
        L = _n.lib()
        if _handle is not None:
            self._h = _handle
        else:
            h = ct.c_void_p()
            _n.check(L.hcfd_mesh_load(path.encode(), ct.byref(h)))
            self._h = h

    @classmethod
    def wedge(cls, nx: int, ny: int, theta_deg: float = 15.0, jitter: float = 0.15, seed: int = 1234,
              numbering: int = NUMBER_RANDOM, length: float = 3.0, height: float = 1.5,
              x_ramp: float = 0.5) -> "Mesh":
        """Triangulated supersonic wedge (see hcfd_mesh_generate_wedge)."""
        spec = _n.WedgeSpec(nx, ny, length, height, x_ramp, theta_deg, jitter, seed, numbering)
        h = ct.c_void_p()
        _n.check(_n.lib().hcfd_mesh_generate_wedge(ct.byref(spec), ct.byref(h)))
        return cls(_handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _n.lib().hcfd_mesh_free(h)
            self._h = None

    def renumber(self, numbering: int, seed: int = 0) -> "Mesh":
        _n.check(_n.lib().hcfd_mesh_renumber(self._h, numbering, seed))
        return self

    def write(self, path: str) -> None:
        _n.check(_n.lib().hcfd_mesh_write(self._h, path.encode()))

    def view(self) -> _n.MeshView:
        v = _n.MeshView()
        _n.check(_n.lib().hcfd_mesh_view_of(self._h, ct.byref(v)))
        return v

    def arrays(self) -> dict:
        """Copies of the mesh arrays, keyed like the reference's Mesh members."""
        v = self.view()

        def take(ptr, n, dt):
            if not ptr or n == 0:
                return None
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)

        cn_off = take(v.cn_off, v.Nc + 1, np.int32)
        d = dict(dim=v.dim, Nn=v.Nn, Ncol=v.Ncol, NBCcol=v.NBCcol, Nc=v.Nc, Nf=v.Nf,
                 coltag=take(v.coltag, v.Ncol, np.int32), coloff=take(v.coloff, v.Ncol + 1, np.int32),
                 nodes=take(v.nodes, 2 * v.Nn, np.float64), fn_con=take(v.fn_con, 2 * v.Nf, np.int32),
                 fc_con=take(v.fc_con, 2 * v.Nf, np.int32), cn_off=cn_off,
                 cn_con=take(v.cn_con, int(cn_off[-1]), np.int32))
        if v.cc_off:
            cc_off = take(v.cc_off, v.Nc + 1, np.int32)
            d["cc_off"] = cc_off
            d["cc_con"] = take(v.cc_con, int(cc_off[-1]), np.int32)
        cfo, cfc = _n._ip(), _n._ip()
        _n.check(_n.lib().hcfd_mesh_cf(self._h, ct.byref(cfo), ct.byref(cfc)))
        d["cf_off"] = take(cfo, v.Nc + 1, np.int32)
        d["cf_con"] = take(cfc, int(d["cf_off"][-1]), np.int32)
        d["pnames"] = []
        for k in range(64):
            s = _n.lib().hcfd_mesh_pname(self._h, k)
            if s is None:
                break
            d["pnames"].append(s.decode())
        return d

    @property
    def Nc(self):
        return self.view().Nc

    @property
    def Nf(self):
        return self.view().Nf


class Solver:
    """One mesh on one GPU (include/hcfd_gpu.h, hcfd_gpu_*)."""

    def __init__(self, mesh: Mesh, gma: float = 1.4, limiter: int = LIMITER_BJ, venkat_K: float = 5.0,
                 precision: int = FP64, block: int = 0, kernel: int = 0, tile: int = 0,
                 keep_numbering: bool = False, freeze_limiter_after: int = 0, tile2: int = 0):
        self._mesh = mesh
        v = mesh.view()
        p = _n.Params(gma, limiter, venkat_K, precision, block, kernel, tile, 1 if keep_numbering else 0,
                      freeze_limiter_after, tile2)
        h = ct.c_void_p()
        _n.check(_n.lib().hcfd_gpu_create(ct.byref(v), ct.byref(p), ct.byref(h)))
        self._h = h
        self.gma = gma
        self.precision = precision
        Nc, Nf, Nr, W = ct.c_int(), ct.c_int(), ct.c_int(), ct.c_int()
        _n.check(_n.lib().hcfd_gpu_info(h, ct.byref(Nc), ct.byref(Nf), ct.byref(Nr), ct.byref(W)))
        self.Nc, self.Nf, self.Nreal, self.slots = Nc.value, Nf.value, Nr.value, W.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _n.lib().hcfd_gpu_destroy(h)
            self._h = None

    def gather_bcs(self, bcmap, qbc) -> None:
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64).reshape(-1)
        _n.check(_n.lib().hcfd_gpu_gather_bcs(self._h, _iptr(bm), len(bm), _dptr(q)))

    def initialise(self, qic) -> None:
        q = np.ascontiguousarray(qic, dtype=np.float64)
        _n.check(_n.lib().hcfd_gpu_initialise(self._h, _dptr(q)))

    def step(self, nsteps: int = 1, mode: int = FIXED_DT, dt_or_cfl: float = 1e-3, wait: bool = True):
        """Advances nsteps steps; returns the step statistics when wait is true."""
        st = _n.StepStats() if wait else None
        _n.check(_n.lib().hcfd_gpu_step(self._h, nsteps, mode, dt_or_cfl, ct.byref(st) if wait else None))
        return self._stats_dict(st) if wait else None

    @staticmethod
    def _stats_dict(st):
        return dict(dt=st.dt, res_l2=st.res_l2, res_first=st.res_first, steps=st.steps,
                    nonfinite=bool(st.nonfinite))

    def step_timed(self, nsteps: int, mode: int = FIXED_DT, dt_or_cfl: float = 1e-3) -> float:
        """Runs nsteps steps; returns their device time in ms (CUDA events on the handle's stream)."""
        ms = ct.c_double()
        _n.check(_n.lib().hcfd_gpu_step_timed(self._h, nsteps, mode, dt_or_cfl, ct.byref(ms)))
        return ms.value

    def launches_per_step(self) -> int:
        return _n.lib().hcfd_gpu_launches_per_step(self._h)

    def stats(self) -> dict:
        st = _n.StepStats()
        _n.check(_n.lib().hcfd_gpu_stats(self._h, ct.byref(st)))
        return self._stats_dict(st)

    def sync(self) -> None:
        _n.check(_n.lib().hcfd_gpu_sync(self._h))

    def download(self, prims: bool = False, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty((4, self.Nc)) if out is None else out
        ptrs = (ct.POINTER(ct.c_double) * 4)(*[_dptr(out[v]) for v in range(4)])
        _n.check(_n.lib().hcfd_gpu_download(self._h, 1 if prims else 0, ptrs))
        return out

    def U(self) -> np.ndarray:
        return self.download(False)

    def Q(self) -> np.ndarray:
        return self.download(True)

    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(4, self.Nc)
        ptrs = (ct.POINTER(ct.c_double) * 4)(*[_dptr(U[v]) for v in range(4)])
        _n.check(_n.lib().hcfd_gpu_upload(self._h, ptrs))

    def snapshot(self, out: np.ndarray, prims: bool = True) -> "Snapshot":
        """Starts copying the current state into `out` (4 x Nc float64, C order; pin it with
        `pin` for the copy to overlap later steps) and returns at once."""
        if out.shape != (4, self.Nc) or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("snapshot: out must be a C-contiguous float64 array of shape (4, Nc)")
        ptrs = (_n._dp * 4)(*[out[v].ctypes.data_as(_n._dp) for v in range(4)])
        t = ct.c_void_p()
        _n.check(_n.lib().hcfd_gpu_snapshot(self._h, 1 if prims else 0, ptrs, ct.byref(t)))
        return Snapshot(t, out)

    def checkpoint(self, path: str) -> None:
        """Exact snapshot (state, step statistics, recorded limiter values) for resuming."""
        _n.check(_n.lib().hcfd_gpu_checkpoint(self._h, os.fsencode(path)))

    def restore(self, path: str) -> None:
        """Continues a checkpointed solve: the next steps are bit-identical to the original's."""
        _n.check(_n.lib().hcfd_gpu_restore(self._h, os.fsencode(path)))

    def wall_cp(self, colour: int, rho_inf: float, p_inf: float, speed_inf: float) -> np.ndarray:
        out = np.empty(self.Nf)
        n = ct.c_int()
        _n.check(_n.lib().hcfd_gpu_wall_cp(self._h, colour, rho_inf, p_inf, speed_inf, _dptr(out), ct.byref(n)))
        return out[:n.value].copy()

    def profile(self, enable, every: int = 1) -> None:
        """Per-kernel CUDA-event timing of every `every`-th step while enabled."""
        _n.check(_n.lib().hcfd_gpu_profile(self._h, max(1, int(every)) if enable else 0))

    def profile_read(self) -> dict:
        m1, m2 = ct.c_double(), ct.c_double()
        n1, n2 = ct.c_longlong(), ct.c_longlong()
        _n.check(_n.lib().hcfd_gpu_profile_read(self._h, ct.byref(m1), ct.byref(n1), ct.byref(m2), ct.byref(n2)))
        return dict(ms_pass1=m1.value, n_pass1=n1.value, ms_pass2=m2.value, n_pass2=n2.value)


class Snapshot:
    """A snapshot in flight (Solver.snapshot): wait() returns the filled array."""

    def __init__(self, h, out: np.ndarray):
        self._h = h
        self.out = out

    def wait(self) -> np.ndarray:
        if self._h is not None:
            _n.check(_n.lib().hcfd_snapshot_wait(self._h))
        return self.out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _n.lib().hcfd_snapshot_free(h)
            self._h = None


def checkpoint_info(path: str) -> dict:
    """Header of a checkpoint file (no GPU needed)."""
    nc, prec, hl = ct.c_int(), ct.c_int(), ct.c_int()
    steps = ct.c_longlong()
    _n.check(_n.lib().hcfd_checkpoint_info(os.fsencode(path), ct.byref(nc), ct.byref(prec), ct.byref(steps),
                                           ct.byref(hl)))
    return dict(Nc=nc.value, precision=prec.value, steps=steps.value, has_limiter=bool(hl.value))


_CKPT_HEADER = struct.Struct("<8siiiiqdddii")   # magic, version, precision, Nc, has_limiter, steps, ...


def convert_checkpoint(src: str, dst: str, precision: int) -> dict:
    """Writes checkpoint `src` to `dst` as a checkpoint of `precision` (no GPU needed).
    To FP32, the state and the frozen limiter values are rounded to the nearest float, as an
    FP32 solver holds them, so the result is what that solver would have written; to FP64 the
    values are kept (FP32 values are exact in FP64).  Restoring the result into a solver of
    that precision, made for the same mesh with the same freezing step, hands the solve over:
    an FP64 solve frozen at step N continues in FP32 with the FP64 solve's limiter values.
    Returns the header of the written file (as checkpoint_info)."""
    if precision not in (FP64, FP32):
        raise ValueError("convert_checkpoint: precision must be FP64 or FP32")
    info = checkpoint_info(src)
    with open(src, "rb") as fh:
        raw = fh.read()
    n = 4 * info["Nc"] * (2 if info["has_limiter"] else 1)
    if len(raw) != _CKPT_HEADER.size + 8 * n:
        raise _n.HcfdError(_n.EIO, f"convert_checkpoint: {src} is not {n} values long")
    head = list(_CKPT_HEADER.unpack_from(raw, 0))
    head[2] = precision
    vals = np.frombuffer(raw, dtype="<f8", count=n, offset=_CKPT_HEADER.size)
    if precision == FP32:
        vals = vals.astype(np.float32).astype("<f8")
    tmp = dst + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(_CKPT_HEADER.pack(*head))
        fh.write(np.ascontiguousarray(vals, dtype="<f8").tobytes())
    os.replace(tmp, dst)
    return checkpoint_info(dst)


def plan_check(mesh: Mesh, tile: int = 0, keep_numbering: bool = False) -> dict:
    """Builds and checks the tiled kernels' plan on the host (see hcfd_plan_check)."""
    v = mesh.view()
    info = (ct.c_longlong * 8)()
    _n.check(_n.lib().hcfd_plan_check(ct.byref(v), tile, 1 if keep_numbering else 0, info))
    keys = ("tiles", "halo_max", "entries_max", "entries", "faces_once", "faces_cut", "slots", "halo_total")
    return dict(zip(keys, list(info)))


def set_device(device: int) -> int:
    """Selects the CUDA device for handles created afterwards; returns the device count."""
    n = ct.c_int()
    _n.check(_n.lib().hcfd_set_device(device, ct.byref(n)))
    return n.value


def device_mem_info() -> tuple[int, int]:
    """(free, total) bytes of device memory on the current device."""
    f, t = ct.c_size_t(), ct.c_size_t()
    _n.check(_n.lib().hcfd_device_mem_info(ct.byref(f), ct.byref(t)))
    return f.value, t.value


def device_sync() -> None:
    _n.check(_n.lib().hcfd_device_sync())


def pin(a: np.ndarray) -> None:
    """Page-locks a numpy array's memory for direct DMA (cudaHostRegister)."""
    _n.check(_n.lib().hcfd_host_pin(ct.c_void_p(a.ctypes.data), a.nbytes))


def unpin(a: np.ndarray) -> None:
    _n.check(_n.lib().hcfd_host_unpin(ct.c_void_p(a.ctypes.data)))


def write_hsln(path: str, arrs, varnames=("Density", "Velocity_X", "Velocity_Y", "Pressure")) -> None:
    """Writer::write_soln's file format (src/Writer.cpp:22-39)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
    nv, Nc = len(arrs), arrs[0].shape[0]
    names = (ct.c_char_p * nv)(*[s.encode() for s in varnames[:nv]])
    ptrs = (ct.POINTER(ct.c_double) * nv)(*[_dptr(a) for a in arrs])
    _n.check(_n.lib().hcfd_write_hsln(path.encode(), nv, names, Nc, ptrs))


def wedge_case(mach: float = 2.5, rho: float = 1.4, p: float = 1.0, gma: float = 1.4):
    """Boundary map and states of the supersonic-wedge family: colour tags 1 upper / 2 lower
    slip walls (SYMMETRY), 3 inlet SUPINLET, 4 outlet SUPOUTLET (src/Test.cpp:64); uniform
    freestream (rho, u = M a, 0, p) as the initial and boundary state."""
    a = (gma * p / rho) ** 0.5
    q = np.array([rho, mach * a, 0.0, p])
    bcmap = np.array([SYMMETRY, SYMMETRY, SYMMETRY, SUPINLET, SUPOUTLET], dtype=np.int32)
    qbc = np.tile(q, (4, 1))
    return bcmap, qbc, q
