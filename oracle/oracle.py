"""TEST INFRASTRUCTURE — Python access to the CPU oracle and to the reference build.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module, and
only as the checker or as the timed CPU baseline.  The product (cfd_optimisations_b200)
never imports it.

* ``Oracle``      — the C restatement in hcfd_oracle.c (built into _build/).
* ``Oracle32``    — the same source built with float step arithmetic (HCFD_ORACLE_FP32);
                    ``Oracle32NoComp`` without its compensated sums.
* ``RefSolver``   — the reference's own layouts, compiled unchanged into _ref/ by the
                    Makefile here (present only where the reference sources were
                    available at build time; the built library travels with the repo).
* ``wedge_hmsh``  — writes the triangulated wedge as a .hmsh file (hcfd_oracle_mesh.c), the
                    input of the timed reference arm, without the product library.
* ``read_hmsh`` / ``read_hsln`` — independent numpy readers of the two file formats,
  following src/Mesh.cpp:7-54 and src/Writer.cpp:22-39 of the reference.
"""
from __future__ import annotations

import ctypes as ct
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhcfd_oracle.so")
ORACLE32_SO = os.path.join(HERE, "_build", "libhcfd_oracle32.so")
ORACLE32NC_SO = os.path.join(HERE, "_build", "libhcfd_oracle32nc.so")
MESH_SO = os.path.join(HERE, "_build", "libhcfd_oracle_mesh.so")
REF_SO = os.path.join(HERE, "_ref", "libhcfd_ref.so")


def _reference_dir() -> str:
    """Where the reference sources lie: $HCFD_REFERENCE, else a checkout named `reference`
    beside this repository; "" when neither holds the reference's sources."""
    for d in (os.environ.get("HCFD_REFERENCE", ""),
              os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")):
        if d and os.path.exists(os.path.join(d, "src", "Mesh.cpp")):
            return d
    return ""


REF_DIR = _reference_dir()

# includes/Base/BoundaryConditions.hpp:6-13
SYMMETRY, WALL, SUPINLET, SUBINLET, SUPOUTLET, SUBOUTLET = range(6)
BJ, VENKAT = 0, 1
FIXED_DT, GLOBAL_CFL, LOCAL_CFL = 0, 1, 2
# fields of Oracle.get (hcfd_oracle.h)
F_U, F_Q, F_PHI, F_R, F_G, F_DTLOC, F_IV = range(7)

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def build(ref: bool = True) -> None:
    """Builds the oracle (and, when the reference sources are found, the reference library)."""
    targets = ["oracle"] + ([f"REF={REF_DIR}", "ref"] if ref and REF_DIR else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


NUMBER_NATURAL, NUMBER_RANDOM, NUMBER_RCM, NUMBER_MORTON = range(4)
_mesh_lib = None


def wedge_hmsh(path: str, nx: int, ny: int, theta_deg: float = 15.0, jitter: float = 0.15, seed: int = 1234,
               numbering: int = NUMBER_RANDOM, length: float = 3.0, height: float = 1.5, x_ramp: float = 0.5) -> None:
    """Writes the triangulated supersonic wedge to `path` (.hmsh), the same file the library's
    generator writes for the same arguments (hcfd_oracle_mesh.c)."""
    global _mesh_lib
    if _mesh_lib is None:
        if not os.path.exists(MESH_SO):
            raise RuntimeError(f"oracle mesh library missing: {MESH_SO} (run make -C oracle)")
        L = ct.CDLL(MESH_SO)
        L.hcfd_oracle_wedge_hmsh.argtypes = [ct.c_int, ct.c_int] + [ct.c_double] * 5 + [ct.c_ulonglong, ct.c_int,
                                                                                       ct.c_char_p]
        _mesh_lib = L
    rc = _mesh_lib.hcfd_oracle_wedge_hmsh(nx, ny, length, height, x_ramp, theta_deg, jitter, seed, numbering,
                                          os.fsencode(path))
    if rc != 0:
        raise ValueError(f"wedge_hmsh: {'bad arguments or an inverted triangle' if rc == -1 else 'I/O error'}")


def read_hmsh(path: str) -> dict:
    """Reads a .hmsh file (header of 8 int32, physical names, then the arrays in the order
    src/Mesh.cpp:31-44 reads them, then c_ctypes as interface/Mesh.py:463 writes it)."""
    with open(path, "rb") as fh:
        b = fh.read()
    dim, Nn, Ncol, NBCcol, Nc, Nf, Npn, Nch = struct.unpack_from("<8i", b, 0)
    off = 32
    names = b[off:off + Nch].split(b"\0")[:-1]
    off += Nch

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(b, dtype=dtype, count=n, offset=off).copy()
        off += a.nbytes
        return a

    m = dict(dim=dim, Nn=Nn, Ncol=Ncol, NBCcol=NBCcol, Nc=Nc, Nf=Nf,
             pnames=[s.decode() for s in names])
    m["coltag"] = take(np.int32, Ncol)
    m["coloff"] = take(np.int32, Ncol + 1)
    m["nodes"] = take(np.float64, Nn * dim)
    m["fn_con"] = take(np.int32, 2 * Nf)
    m["fc_con"] = take(np.int32, 2 * Nf)
    m["cn_off"] = take(np.int32, Nc + 1)
    m["cn_con"] = take(np.int32, int(m["cn_off"][-1]))
    m["cc_off"] = take(np.int32, Nc + 1)
    m["cc_con"] = take(np.int32, int(m["cc_off"][-1]))
    m["c_ctypes"] = take(np.int32, Nc) if off + 4 * Nc <= len(b) else None
    return m


def read_hsln(path: str):
    """Reads a .hsln file: int32 Nc, nvars, nchars, the names, then nvars x Nc float64."""
    with open(path, "rb") as fh:
        b = fh.read()
    Nc, nv, nch = struct.unpack_from("<3i", b, 0)
    names = [s.decode() for s in b[12:12 + nch].split(b"\0")[:-1]]
    data = np.frombuffer(b, dtype=np.float64, count=nv * Nc, offset=12 + nch).reshape(nv, Nc)
    return names, data.copy()


def prim_to_cons(q: np.ndarray, gma: float = 1.4) -> np.ndarray:
    """(rho, u, v, p) -> (rho, rho u, rho v, E), variable-major arrays."""
    r, u, v, p = q
    return np.stack([r, r * u, r * v, p / (gma - 1) + 0.5 * r * (u * u + v * v)])


def rel_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-variable relative L-infinity distance: max|a-b| / max|b| over cells."""
    a = np.asarray(a).reshape(4, -1)
    b = np.asarray(b).reshape(4, -1)
    den = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return np.abs(a - b).max(axis=1) / den


class Oracle:
    """The C restatement of the reference's Base solver (hcfd_oracle.c)."""

    _lib = None
    _so = "double"

    @classmethod
    def lib(cls):
        if cls._lib is None:
            so = {"double": ORACLE_SO, "float": ORACLE32_SO, "float-nocomp": ORACLE32NC_SO}[cls._so]
            if not os.path.exists(so):
                raise RuntimeError(f"oracle library missing: {so} (run make -C oracle)")
            L = ct.CDLL(so)
            L.hcfd_oracle_create.restype = ct.c_void_p
            L.hcfd_oracle_create.argtypes = [ct.c_int] * 5 + [_ip, _ip, _dp, _ip, _ip, _ip, _ip, ct.c_double]
            L.hcfd_oracle_free.argtypes = [ct.c_void_p]
            L.hcfd_oracle_gather_bcs.argtypes = [ct.c_void_p, _ip, ct.c_int, _dp]
            L.hcfd_oracle_initialise.argtypes = [ct.c_void_p, _dp]
            L.hcfd_oracle_set_limiter.argtypes = [ct.c_void_p, ct.c_int, ct.c_double]
            L.hcfd_oracle_set_freeze.argtypes = [ct.c_void_p, ct.c_longlong]
            L.hcfd_oracle_step.argtypes = [ct.c_void_p, ct.c_int, ct.c_double, _dp, _dp]
            L.hcfd_oracle_phase.argtypes = [ct.c_void_p, ct.c_int, ct.c_double]
            L.hcfd_oracle_get.argtypes = [ct.c_void_p, ct.c_int, _dp]
            L.hcfd_oracle_set_U.argtypes = [ct.c_void_p, _dp]
            L.hcfd_oracle_set_phi.argtypes = [ct.c_void_p, _dp]
            L.hcfd_oracle_wall_cp.argtypes = [ct.c_void_p, ct.c_int, ct.c_double, ct.c_double, ct.c_double, _dp]
            L.hcfd_oracle_domain.argtypes = [ct.c_void_p] + [_dp] * 6
            L.hcfd_oracle_nreal.argtypes = [ct.c_void_p]
            cls._lib = L
        return cls._lib

    def __init__(self, mesh: dict, gma: float = 1.4):
        L = self.lib()
        self.m = mesh
        self.Nc, self.Nf = int(mesh["Nc"]), int(mesh["Nf"])
        arrs = {k: np.ascontiguousarray(mesh[k], dtype=np.int32) for k in
                ("coltag", "coloff", "fn_con", "fc_con", "cn_off", "cn_con")}
        nodes = np.ascontiguousarray(mesh["nodes"], dtype=np.float64)
        self.h = L.hcfd_oracle_create(mesh["Nn"], self.Nc, self.Nf, mesh["Ncol"], mesh["NBCcol"],
                                      _i(arrs["coltag"]), _i(arrs["coloff"]), _d(nodes),
                                      _i(arrs["fn_con"]), _i(arrs["fc_con"]),
                                      _i(arrs["cn_off"]), _i(arrs["cn_con"]), gma)
        if not self.h:
            raise ValueError("oracle: invalid mesh")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().hcfd_oracle_free(self.h)
            self.h = None

    def gather_bcs(self, bcmap, qbc):
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64)
        if self.lib().hcfd_oracle_gather_bcs(self.h, _i(bm), len(bm), _d(q)) != 0:
            raise ValueError("oracle: bad BC map")

    def initialise(self, qic):
        q = np.ascontiguousarray(qic, dtype=np.float64)
        self.lib().hcfd_oracle_initialise(self.h, _d(q))

    def set_limiter(self, kind, K=0.0):
        if self.lib().hcfd_oracle_set_limiter(self.h, kind, K) != 0:
            raise ValueError("oracle: bad limiter")

    def set_freeze(self, after):
        if self.lib().hcfd_oracle_set_freeze(self.h, after) != 0:
            raise ValueError("oracle: bad freeze step")

    def step(self, mode=FIXED_DT, dt_or_cfl=1e-3):
        dt = np.zeros(1)
        res = np.zeros(1)
        self.lib().hcfd_oracle_step(self.h, mode, dt_or_cfl, _d(dt), _d(res))
        return float(dt[0]), float(res[0])

    def phase(self, which, dt=0.0):
        self.lib().hcfd_oracle_phase(self.h, which, dt)

    def get(self, which):
        n = 8 * self.Nc if which == 4 else (self.Nc if which in (5, 6) else 4 * self.Nc)
        out = np.zeros(n)
        self.lib().hcfd_oracle_get(self.h, which, _d(out))
        if which in (5, 6):
            return out
        return out.reshape(4, 2, self.Nc) if which == 4 else out.reshape(4, self.Nc)

    def U(self):
        return self.get(0)

    def Q(self):
        return self.get(1)

    def set_U(self, u):
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        self.lib().hcfd_oracle_set_U(self.h, _d(a))

    def set_phi(self, phi):
        a = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
        self.lib().hcfd_oracle_set_phi(self.h, _d(a))

    def wall_cp(self, colour, rho_inf, p_inf, speed_inf):
        out = np.zeros(self.Nf)
        n = self.lib().hcfd_oracle_wall_cp(self.h, colour, rho_inf, p_inf, speed_inf, _d(out))
        return out[:n]

    def nreal(self):
        return self.lib().hcfd_oracle_nreal(self.h)

    def domain(self):
        Nf, Nc = self.Nf, self.Nc
        rf, nf, Af, If = np.zeros(4 * Nf), np.zeros(2 * Nf), np.zeros(Nf), np.zeros(Nf)
        xc, iv = np.zeros(2 * Nc), np.zeros(Nc)
        self.lib().hcfd_oracle_domain(self.h, _d(rf), _d(nf), _d(Af), _d(If), _d(xc), _d(iv))
        return dict(rf=rf.reshape(Nf, 2, 2), nf=nf.reshape(Nf, 2), Af=Af, If=If,
                    xc=xc.reshape(Nc, 2), iv=iv)


class Oracle32(Oracle):
    """The same restatement built with float step arithmetic (HCFD_ORACLE_FP32): geometry in
    double rounded once, state, gradients, limiter and fluxes in IEEE float, each cell's
    residual summed with a compensated two-sum, dt minima and norms in double.  The CPU
    counterpart of the library's FP32 path, which differs from it by the hardware's approximate
    divisions and square roots (a few units in the last place per operation)."""

    _lib = None
    _so = "float"


class Oracle32NoComp(Oracle):
    """Oracle32 with plain float sums in place of the compensated ones (HCFD_ORACLE_NOCOMP)."""

    _lib = None
    _so = "float-nocomp"


class RefSolver:
    """One instance of the reference's own solver (compiled unchanged), driven phase by phase."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise RuntimeError(f"reference library missing: {REF_SO}")
            L = ct.CDLL(REF_SO)
            L.hcfd_ref_create.restype = ct.c_void_p
            L.hcfd_ref_create.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_double, _ip, ct.c_int, _dp, _dp]
            L.hcfd_ref_free.argtypes = [ct.c_void_p]
            L.hcfd_ref_nc.argtypes = [ct.c_void_p]
            L.hcfd_ref_steps.argtypes = [ct.c_void_p, ct.c_int, _dp, ct.c_int]
            L.hcfd_ref_phase.argtypes = [ct.c_void_p, ct.c_int, ct.c_double]
            L.hcfd_ref_get.argtypes = [ct.c_void_p, ct.c_int, _dp]
            L.hcfd_ref_get_G.argtypes = [ct.c_void_p, _dp]
            L.hcfd_ref_set_U.argtypes = [ct.c_void_p, _dp]
            L.hcfd_ref_mesh_info.argtypes = [ct.c_char_p, _ip]
            L.hcfd_ref_mesh_cf.argtypes = [ct.c_char_p, _ip, _ip]
            L.hcfd_ref_domain.argtypes = [ct.c_char_p] + [_dp] * 6
            L.hcfd_ref_bench.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_double, _ip, ct.c_int, _dp, _dp,
                                         ct.c_int, ct.c_int, ct.c_int, ct.c_double, _dp]
            cls._lib = L
        return cls._lib

    def __init__(self, mesh_path: str, bcmap, qbc, qic, layout: str = "Base", gma: float = 1.4):
        L = self.lib()
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64)
        qi = np.ascontiguousarray(qic, dtype=np.float64)
        self.h = L.hcfd_ref_create(layout.encode(), mesh_path.encode(), gma, _i(bm), len(bm), _d(q), _d(qi))
        if not self.h:
            raise ValueError(f"reference: cannot build {layout} on {mesh_path}")
        self.Nc = L.hcfd_ref_nc(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().hcfd_ref_free(self.h)
            self.h = None

    def steps(self, n, dt):
        dts = np.atleast_1d(np.asarray(dt, dtype=np.float64))
        self.lib().hcfd_ref_steps(self.h, n, _d(dts), len(dts))

    def phase(self, which, dt=0.0):
        self.lib().hcfd_ref_phase(self.h, which, dt)

    def get(self, which):
        out = np.zeros(4 * self.Nc)
        self.lib().hcfd_ref_get(self.h, which, _d(out))
        return out.reshape(4, self.Nc)

    def U(self):
        return self.get(0)

    def Q(self):
        return self.get(1)

    def G(self):
        out = np.zeros(8 * self.Nc)
        self.lib().hcfd_ref_get_G(self.h, _d(out))
        return out.reshape(4, 2, self.Nc)

    def set_U(self, u):
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        self.lib().hcfd_ref_set_U(self.h, _d(a))

    @classmethod
    def bench(cls, layout, mesh_path, bcmap, qbc, qic, nthreads, nwarm, nsteps, dt, gma=1.4):
        """Wall seconds of `nsteps` steps run by `nthreads` independent instances."""
        bm = np.ascontiguousarray(bcmap, dtype=np.int32)
        q = np.ascontiguousarray(qbc, dtype=np.float64)
        qi = np.ascontiguousarray(qic, dtype=np.float64)
        secs = np.zeros(1)
        rc = cls.lib().hcfd_ref_bench(layout.encode(), mesh_path.encode(), gma, _i(bm), len(bm), _d(q), _d(qi),
                                      nthreads, nwarm, nsteps, dt, _d(secs))
        if rc != 0:
            raise RuntimeError("reference bench failed")
        return float(secs[0])
