"""Host-side mirror of Hydra's QG caps module interface over the CUDA C-ABI.

``CaslGPU`` holds one simulation on one GPU and exposes the reference's
module procedures under their reference names (``con2grid``, ``velint``,
``main_invert``, ``gradient``, ``inversion``, ``advance``, ``surgery``,
``renode``, ``recontour``, ``ptospc``, ``spctop``) plus the driver loop of
caps.f90 (``initialise``, ``step``).  Every call goes through
``libhydra_casl.so`` (include/hydra_casl.h); there is no CPU fallback: if the
library or a GPU is missing, construction raises.

Array convention: a physical field q(ny,nx) is an (nx, ny) C-contiguous
float64 array indexed [ix-1, iy-1]; a spectral field s(nx,ny) is (ny, nx)
indexed [ky-1, kx-1]; contour index arrays are 1-based as in the reference.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhydra_casl.so")

CASL_OK, CASL_EINVAL, CASL_ECAPACITY, CASL_ECUDA, CASL_ENOMEM, CASL_EDOMAIN, CASL_ETIMEOUT, \
    CASL_EUNSUPPORTED = range(8)

FIELDS = {"qs": 0, "qd": 1, "qc": 2, "qq": 3, "pp": 4, "qspre": 5, "emq": 6, "epq": 7,
          "uu": 8, "vv": 9, "qr": 10}
SCALARS = {"t": 0, "dt": 1, "twist": 2, "ireg": 3, "zzrms": 4, "zzmax": 5, "uumax": 6, "qjump": 7,
           "node_steps": 8}


class CaslError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (code {code})")
        self.code = code


class CaslParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("ncontq", C.c_int),
        ("ellx", C.c_double), ("elly", C.c_double), ("kd", C.c_double), ("beta", C.c_double),
        ("rtherm", C.c_double), ("rekman", C.c_double), ("cdamp", C.c_double), ("nnu", C.c_double),
        ("npm", C.c_longlong), ("nm", C.c_longlong), ("nlevm", C.c_int),
        ("fixed_dt", C.c_double), ("dtmax", C.c_double), ("force_surgery", C.c_int),
        ("nregmax", C.c_int), ("twistmax", C.c_double),
    ]


_lib = None
_dp = C.POINTER(C.c_double)

# The network's output channels (CASL_NET_OUT): the velocity correction on a
# grid twice as fine as n, channel comp*4 + a*2 + b = component comp (u, v)
# at the fine point (2 ix + a, 2 iy + b).
NET_OUT = 8
# Its input channels (CASL_NET_IN): coarse contour PV, u, v, and the nine
# sub-cell deviations of the fine contour levels.
NET_IN = 12
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)

# name -> (restype, argtypes); the same list is checked against the header by tests
SIGNATURES = {
    "casl_create": (C.c_int, [C.POINTER(CaslParams), C.c_int, C.POINTER(C.c_void_p)]),
    "casl_destroy": (None, [C.c_void_p]),
    "casl_error_string": (C.c_char_p, [C.c_int]),
    "casl_last_cuda_error": (C.c_int, [C.c_void_p]),
    "casl_synchronize": (C.c_int, [C.c_void_p]),
    "casl_set_contours": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, _dp, _dp, _ip, _ip, _ip, _ip, _ip]),
    "casl_get_counts": (C.c_int, [C.c_void_p, _ip, _ip, _dp]),
    "casl_get_contours": (C.c_int, [C.c_void_p, _dp, _dp, _ip, _ip, _ip, _ip, _ip]),
    "casl_set_field": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "casl_get_field": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "casl_get_scalar": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "casl_set_scalar": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "casl_ptospc": (C.c_int, [C.c_void_p, _dp, _dp]),
    "casl_spctop": (C.c_int, [C.c_void_p, _dp, _dp]),
    "casl_con2grid": (C.c_int, [C.c_void_p, _dp, _ip]),
    "casl_velint": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "casl_main_invert": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "casl_gradient": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "casl_inversion": (C.c_int, [C.c_void_p]),
    "casl_advance": (C.c_int, [C.c_void_p]),
    "casl_surgery": (C.c_int, [C.c_void_p]),
    "casl_renode": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, C.c_int, _ip]),
    "casl_recontour": (C.c_int, [C.c_void_p, _dp]),
    "casl_initialise": (C.c_int, [C.c_void_p, _dp]),
    "casl_step": (C.c_int, [C.c_void_p, C.c_int]),
    "casl_diagnostics": (C.c_int, [C.c_void_p, _dp]),
    "casl_spec1d": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "casl_spec_tables": (C.c_int, [C.c_void_p, _ip, _ip, _dp, _dp]),
    "casl_con2grid_noalloc": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "casl_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "casl_launch_count": (C.c_int, [C.POINTER(C.c_longlong)]),
    "casl_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "casl_profile_read": (C.c_int, [C.c_void_p, _dp, C.POINTER(C.c_longlong), _dp]),
    "casl_kernel_times": (C.c_int, [C.c_int, C.c_char_p, C.c_longlong]),
    "casl_io_append_synopsis": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double]),
    "casl_io_append_ene": (C.c_int, [C.c_char_p, C.c_double, C.c_double, C.c_double]),
    "casl_io_append_norms": (C.c_int, [C.c_char_p, C.c_double, C.c_double]),
    "casl_io_append_spectrum": (C.c_int, [C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                          _dp, _dp]),
    "casl_io_append_monitor": (C.c_int, [C.c_char_p] + [C.c_double] * 6),
    "casl_io_append_complexity": (C.c_int, [C.c_char_p, C.c_double, C.c_int, C.c_int]),
    "casl_io_write_index": (C.c_int, [C.c_char_p, C.c_int, _ip, _ip, _ip]),
    "casl_io_read_index": (C.c_int, [C.c_char_p, C.c_int, _ip, _ip, _ip]),
    "casl_io_write_nodes": (C.c_int, [C.c_char_p, C.c_int, _dp, _dp]),
    "casl_io_read_nodes": (C.c_int, [C.c_char_p, C.c_int, _dp, _dp]),
    "casl_io_write_r4": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                   C.POINTER(C.c_float)]),
    "casl_io_read_r4": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float),
                                  C.POINTER(C.c_float)]),
    "casl_io_read_synopsis": (C.c_int, [C.c_char_p, C.c_int, _ip, _ip, _dp, _dp]),
    "casl_savecont": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "casl_savegrid": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "casl_set_saves": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double,
                                 C.c_int, C.c_int]),
    "casl_get_saves": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "casl_io_wait": (C.c_int, [C.c_void_p]),
    "casl_readcont": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "casl_genfg": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                             C.POINTER(C.c_float)]),
    "casl_net_param_count": (C.c_int, []),
    "casl_net_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "casl_net_destroy": (None, [C.c_void_p]),
    "casl_net_set_params": (C.c_int, [C.c_void_p, _fp, C.c_float, C.c_float]),
    "casl_net_get_params": (C.c_int, [C.c_void_p, _fp, _fp, _fp]),
    "casl_net_forward": (C.c_int, [C.c_void_p, _fp, _fp]),
    "casl_net_backward": (C.c_int, [C.c_void_p, _fp, _fp]),
    "casl_net_adam": (C.c_int, [C.c_void_p, C.c_float]),
    "casl_closure_judge": (C.c_int, [C.c_void_p, C.c_void_p, _dp, _dp, _dp, _dp]),
    "casl_closure_attach": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double]),
    "casl_closure_status": (C.c_int, [C.c_void_p, _ip, _dp, _dp, C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_longlong)]),
    "casl_closure_check": (C.c_int, [C.c_void_p, _dp, _dp]),
    "casl_closure_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, _dp]),
    "casl_closure_evaluate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _dp]),
    "casl_closure_features": (C.c_int, [C.c_void_p, C.c_void_p, _fp]),
    "casl_closure_correction": (C.c_int, [C.c_void_p, C.c_void_p, _dp, _dp]),
    "casl_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "casl_get_precision": (C.c_int, [C.c_void_p, _ip]),
    "casl_pvforce": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, _dp]),
    "casl_nb_forcing_init": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, _ip]),
    "casl_nb_forcing": (C.c_int, [C.c_void_p, C.c_double, _dp]),
    "casl_ensemble_create": (C.c_int, [C.POINTER(CaslParams), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "casl_ensemble_members": (C.c_int, [C.c_void_p, _ip]),
    "casl_ensemble_initialise": (C.c_int, [C.c_void_p, _dp, _ip]),
    "casl_ensemble_member_counts": (C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _dp]),
    "casl_ensemble_member_contours": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _ip, _ip, _ip, _ip, _ip]),
    "casl_ensemble_member_scalar": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
}


def load_library(path: str = LIB_PATH):
    """Load libhydra_casl.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"hydra_b200: CUDA library not built ({path}); run hydra_b200/build.py")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class CaslGPU:
    """One contour-advection simulation resident on one GPU."""

    def __init__(self, nx, ncontq=40, ellx=2 * np.pi, elly=None, kd=0.0, beta=0.0, rtherm=0.0,
                 rekman=0.0, cdamp=2.0, nnu=3.0, npm=None, nm=0, nlevm=2000, fixed_dt=0.0,
                 dtmax=0.05, force_surgery=0, nregmax=20, twistmax=2.5, device=0):
        self.lib = load_library()
        elly = ellx if elly is None else elly
        if npm is None:
            npm = 60 * nx * nx
        self.p = CaslParams(nx, nx, ncontq, ellx, elly, kd, beta, rtherm, rekman, cdamp, nnu,
                            int(npm), int(nm), nlevm, fixed_dt, dtmax, force_surgery, nregmax,
                            twistmax)
        h = C.c_void_p()
        self._check(self.lib.casl_create(C.byref(self.p), device, C.byref(h)), "casl_create")
        self.h = h
        self.nx = self.ny = nx

    def _check(self, rc, where):
        if rc != CASL_OK:
            msg = self.lib.casl_error_string(rc).decode()
            raise CaslError(rc, where, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.casl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- state ------------------------------------------------------------------
    def field(self, name):
        shape = (self.nx, self.ny)
        out = np.empty(shape)
        self._check(self.lib.casl_get_field(self.h, FIELDS[name], _d(out)), "casl_get_field")
        return out

    def set_field(self, name, arr):
        a = _f64(arr, (self.nx, self.ny))
        self._check(self.lib.casl_set_field(self.h, FIELDS[name], _d(a)), "casl_set_field")

    def scalar(self, name):
        v = C.c_double()
        self._check(self.lib.casl_get_scalar(self.h, SCALARS[name], C.byref(v)), "casl_get_scalar")
        return v.value

    def set_scalar(self, name, value):
        self._check(self.lib.casl_set_scalar(self.h, SCALARS[name], float(value)), "casl_set_scalar")

    def counts(self):
        nq, npt, qj = C.c_int(), C.c_int(), C.c_double()
        self._check(self.lib.casl_get_counts(self.h, C.byref(nq), C.byref(npt), C.byref(qj)),
                    "casl_get_counts")
        return nq.value, npt.value, qj.value

    def contours(self):
        nq, npt, qj = self.counts()
        xq = np.zeros(npt); yq = np.zeros(npt); nextq = np.zeros(npt, np.int32)
        indq = np.zeros(nq, np.int32); npq = np.zeros(nq, np.int32)
        i1q = np.zeros(nq, np.int32); i2q = np.zeros(nq, np.int32)
        self._check(self.lib.casl_get_contours(self.h, _d(xq), _d(yq), _i(nextq), _i(indq), _i(npq),
                                               _i(i1q), _i(i2q)), "casl_get_contours")
        return dict(nq=nq, nptq=npt, qjump=qj, xq=xq, yq=yq, nextq=nextq, indq=indq, npq=npq,
                    i1q=i1q, i2q=i2q)

    def set_contours(self, c):
        xq = _f64(c["xq"]); yq = _f64(c["yq"])
        nextq = np.ascontiguousarray(c["nextq"], np.int32)
        indq = np.ascontiguousarray(c["indq"], np.int32); npq = np.ascontiguousarray(c["npq"], np.int32)
        i1q = np.ascontiguousarray(c["i1q"], np.int32); i2q = np.ascontiguousarray(c["i2q"], np.int32)
        self._check(self.lib.casl_set_contours(self.h, len(indq), len(xq), float(c["qjump"]), _d(xq),
                                               _d(yq), _i(nextq), _i(indq), _i(npq), _i(i1q), _i(i2q)),
                    "casl_set_contours")

    # --- module procedures ------------------------------------------------------------
    def ptospc(self, q):
        a = _f64(q, (self.nx, self.ny)); out = np.empty((self.ny, self.nx))
        self._check(self.lib.casl_ptospc(self.h, _d(a), _d(out)), "casl_ptospc")
        return out

    def spctop(self, s):
        a = _f64(s, (self.ny, self.nx)); out = np.empty((self.nx, self.ny))
        self._check(self.lib.casl_spctop(self.h, _d(a), _d(out)), "casl_spctop")
        return out

    def con2grid(self, levels=False):
        qc = np.empty((self.nx, self.ny))
        lv = np.empty((4 * self.nx, 4 * self.ny), np.int32) if levels else None
        self._check(self.lib.casl_con2grid(self.h, _d(qc), _i(lv)), "casl_con2grid")
        return (qc, lv) if levels else qc

    def velint(self, uu, vv):
        _, npt, _ = self.counts()
        uu = _f64(uu, (self.nx, self.ny)); vv = _f64(vv, (self.nx, self.ny))
        uq = np.empty(npt); vq = np.empty(npt)
        self._check(self.lib.casl_velint(self.h, _d(uu), _d(vv), _d(uq), _d(vq)), "casl_velint")
        return uq, vq

    def main_invert(self, qq):
        qq = _f64(qq, (self.ny, self.nx))
        uu = np.empty((self.nx, self.ny)); vv = np.empty((self.nx, self.ny)); pp = np.empty((self.ny, self.nx))
        self._check(self.lib.casl_main_invert(self.h, _d(qq), _d(uu), _d(vv), _d(pp)), "casl_main_invert")
        return uu, vv, pp

    def gradient(self, ff):
        ff = _f64(ff, (self.ny, self.nx))
        fx = np.empty((self.nx, self.ny)); fy = np.empty((self.nx, self.ny))
        self._check(self.lib.casl_gradient(self.h, _d(ff), _d(fx), _d(fy)), "casl_gradient")
        return fx, fy

    def inversion(self):
        self._check(self.lib.casl_inversion(self.h), "casl_inversion")

    def advance(self):
        self._check(self.lib.casl_advance(self.h), "casl_advance")

    def surgery(self):
        self._check(self.lib.casl_surgery(self.h), "casl_surgery")

    def renode(self, xd, yd):
        xd = _f64(xd); yd = _f64(yd)
        cap = 8 * len(xd) + 64
        xr = np.empty(cap); yr = np.empty(cap); npr = C.c_int()
        self._check(self.lib.casl_renode(self.h, _d(xd), _d(yd), len(xd), _d(xr), _d(yr), cap,
                                         C.byref(npr)), "casl_renode")
        return xr[:npr.value], yr[:npr.value]

    def recontour(self, qq):
        qq = _f64(qq, (self.nx, self.ny))
        self._check(self.lib.casl_recontour(self.h, _d(qq)), "casl_recontour")

    def initialise(self, q0):
        q0 = _f64(q0, (self.nx, self.ny))
        self._check(self.lib.casl_initialise(self.h, _d(q0)), "casl_initialise")

    def step(self, nsteps=1):
        self._check(self.lib.casl_step(self.h, int(nsteps)), "casl_step")

    def synchronize(self):
        self._check(self.lib.casl_synchronize(self.h), "casl_synchronize")

    # --- benchmarking hooks --------------------------------------------------------
    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._check(self.lib.casl_get_stream(self.h, C.byref(p)), "casl_get_stream")
        return p.value or 0

    def launch_count(self) -> int:
        v = C.c_longlong()
        self._check(self.lib.casl_launch_count(C.byref(v)), "casl_launch_count")
        return v.value

    def profile(self, kernel_class: int):
        self._check(self.lib.casl_profile(self.h, kernel_class), "casl_profile")

    def profile_read(self):
        ms, n, b = C.c_double(), C.c_longlong(), C.c_double()
        self._check(self.lib.casl_profile_read(self.h, C.byref(ms), C.byref(n), C.byref(b)),
                    "casl_profile_read")
        return ms.value, n.value, b.value

    def kernel_times(self, mode: int) -> str:
        """Per-launch timing of every kernel (process-wide): 1 on, 0 off,
        2 returns the report (launches, total ms, mean us per kernel) and
        starts a new tally."""
        buf = C.create_string_buffer(1 << 16) if mode == 2 else None
        self._check(self.lib.casl_kernel_times(mode, buf, len(buf) if buf else 0),
                    "casl_kernel_times")
        return buf.value.decode() if buf else ""

    def diagnostics(self):
        out = np.zeros(4)
        self._check(self.lib.casl_diagnostics(self.h, _d(out)), "casl_diagnostics")
        return dict(ekin=out[0], epot=out[1], enstrophy=out[2], circulation=out[3])

    def savecont(self, rundir, icrec):
        """savecont (evolution.f90:731-774) into rundir/cont; the files are
        written by a background thread (see io_wait)."""
        self._check(self.lib.casl_savecont(self.h, os.fsencode(rundir), int(icrec)), "casl_savecont")

    def savegrid(self, rundir, irec):
        """savegrid (evolution.f90:648-727) at the current time."""
        self._check(self.lib.casl_savegrid(self.h, os.fsencode(rundir), int(irec)), "casl_savegrid")

    def set_saves(self, rundir, tgsave, tcsave, tinit=0.0, igrec=0, icrec=1):
        """The time loop's save schedule (evolution.f90:586-600): step() writes
        savegrid output (interpolated to each save time) every tgsave and
        savecont output every tcsave time units from tinit; rundir None
        turns it off."""
        d = None if rundir is None else os.fsencode(rundir)
        self._check(self.lib.casl_set_saves(self.h, d, float(tinit), float(tgsave), float(tcsave),
                                            int(igrec), int(icrec)), "casl_set_saves")

    def save_counters(self):
        g, c = C.c_int(), C.c_int()
        self._check(self.lib.casl_get_saves(self.h, C.byref(g), C.byref(c)), "casl_get_saves")
        return g.value, c.value

    def io_wait(self):
        self._check(self.lib.casl_io_wait(self.h), "casl_io_wait")

    def readcont(self, rundir, iind):
        """readcont (common.f90:30-100) + init: restart from save iind."""
        self._check(self.lib.casl_readcont(self.h, os.fsencode(rundir), int(iind)), "casl_readcont")

    def genfg(self, ix1v=1, nxv=None, iy1v=1, nyv=None, stride=1):
        """genfg (post/genfg.f90:79-194): ultra-fine PV of the contours plus the
        residual qr, float32 (nxv, nyv) array (iy fastest), 1-based starts."""
        nu = 16 * self.nx
        nxv = nxv or (nu - ix1v) // stride + 1
        nyv = nyv or (nu - iy1v) // stride + 1
        out = np.zeros((nxv, nyv), np.float32)
        self._check(self.lib.casl_genfg(self.h, ix1v, nxv, iy1v, nyv, stride,
                                        out.ctypes.data_as(C.POINTER(C.c_float))), "casl_genfg")
        return out

    def spec1d(self, ss, iopt=0):
        """spec1d (spectral.f90:370-424) of the spectral field ss(nx,ny), given
        as an (ny, nx) array; returns (spec[0..n], ss after the call)."""
        a = np.ascontiguousarray(ss, dtype=np.float64).copy()
        spec = np.zeros(self.nx + 1)
        self._check(self.lib.casl_spec1d(self.h, _d(a), _d(spec), int(iopt)), "casl_spec1d")
        return spec, a

    def pvforce(self, ivor, vorvor, rnd):
        """pvforce (evolution.f90:330-428) with the caller's uniforms in [0,1)
        (2 per vortex for ivor = 1, else 3)."""
        r = _f64(rnd).ravel()
        m = 2 if ivor == 1 else 3
        self._check(self.lib.casl_pvforce(self.h, int(ivor), float(vorvor), len(r) // m, _d(r)),
                    "casl_pvforce")

    def nb_forcing_init(self, kfmid, fwid, famp):
        k = C.c_int()
        self._check(self.lib.casl_nb_forcing_init(self.h, float(kfmid), float(fwid), float(famp),
                                                  C.byref(k)), "casl_nb_forcing_init")
        return k.value

    def nb_forcing(self, dt, rnd):
        r = _f64(rnd).ravel()
        self._check(self.lib.casl_nb_forcing(self.h, float(dt), _d(r)), "casl_nb_forcing")

    def set_precision(self, mode):
        """0 = FP64 (default); 1 = FP32 inversion (casl_set_precision)."""
        self._check(self.lib.casl_set_precision(self.h, int(mode)), "casl_set_precision")

    # --- learned velocity closure ---------------------------------------------------
    def judge(self, fine):
        """Node velocities of the fine-grid judge (handle `fine`, 2-8x the grid)
        and of the plain velint: (uJ, vJ, uP, vP)."""
        _, npt, _ = self.counts()
        out = [np.empty(npt) for _ in range(4)]
        self._check(self.lib.casl_closure_judge(self.h, fine.h, *[_d(a) for a in out]),
                    "casl_closure_judge")
        return tuple(out)

    def closure_attach(self, net, judge=None, check_every=0, budget=1e-3):
        self._check(self.lib.casl_closure_attach(self.h, net.h if net else None,
                                                 judge.h if judge else None, int(check_every),
                                                 float(budget)), "casl_closure_attach")

    def closure_status(self):
        a, ep, en = C.c_int(), C.c_double(), C.c_double()
        ch, fb = C.c_longlong(), C.c_longlong()
        self._check(self.lib.casl_closure_status(self.h, C.byref(a), C.byref(ep), C.byref(en),
                                                 C.byref(ch), C.byref(fb)), "casl_closure_status")
        return dict(active=a.value, err_plain=ep.value, err_net=en.value, checks=ch.value,
                    fallbacks=fb.value)

    def closure_check(self):
        ep, en = C.c_double(), C.c_double()
        self._check(self.lib.casl_closure_check(self.h, C.byref(ep), C.byref(en)), "casl_closure_check")
        return ep.value, en.value

    def closure_train(self, net, judge, lr):
        """One training sample; returns (plain error, corrected error, loss)."""
        out = np.zeros(3)
        self._check(self.lib.casl_closure_train(self.h, net.h, judge.h, float(lr), _d(out)),
                    "casl_closure_train")
        return tuple(out)

    def closure_evaluate(self, net, judge):
        out = np.zeros(3)
        self._check(self.lib.casl_closure_evaluate(self.h, net.h, judge.h, _d(out)),
                    "casl_closure_evaluate")
        return tuple(out)

    def closure_correction(self, net):
        """The network's correction at the nodes (du, dv) from the latest inversion."""
        _, npt, _ = self.counts()
        du, dv = np.empty(npt), np.empty(npt)
        self._check(self.lib.casl_closure_correction(self.h, net.h, _d(du), _d(dv)),
                    "casl_closure_correction")
        return du, dv

    def closure_features(self, net):
        x = np.empty((NET_IN, self.nx, self.ny), np.float32)
        self._check(self.lib.casl_closure_features(self.h, net.h, x.ctypes.data_as(_fp)),
                    "casl_closure_features")
        return x

    def spec_tables(self):
        """kmax, kmaxred, spmf, alk of init_spectral (spectral.f90:109-134)."""
        kmax, kred = C.c_int(), C.c_int()
        spmf, alk = np.zeros(self.nx + 1), np.zeros(self.nx + 1)
        self._check(self.lib.casl_spec_tables(self.h, C.byref(kmax), C.byref(kred), _d(spmf), _d(alk)),
                    "casl_spec_tables")
        return dict(kmax=kmax.value, kmaxred=kred.value, spmf=spmf, alk=alk)


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def _fptr(a):
    return a.ctypes.data_as(_fp) if a is not None else None


class CaslNet:
    """The learned velocity closure's network on one GPU (casl_net_*): four
    periodic 5x5 convolutions 3 -> 32 -> 32 -> 32 -> NET_OUT with GELU, BF16
    weights and activations, FP32 accumulation, on the tensor cores.  Arrays
    are channel-major (C, n, n) float32 with rows = ix, columns = iy."""

    def __init__(self, n, device=0):
        self.lib = load_library()
        h = C.c_void_p()
        self._check(self.lib.casl_net_create(int(n), int(device), C.byref(h)), "casl_net_create")
        self.h = h
        self.n = n
        self.count = self.lib.casl_net_param_count()

    _check = CaslGPU._check

    def close(self):
        if getattr(self, "h", None):
            self.lib.casl_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params, qscale=1.0, uscale=1.0):
        p = _f32(params, (self.count,))
        self._check(self.lib.casl_net_set_params(self.h, _fptr(p), float(qscale), float(uscale)),
                    "casl_net_set_params")

    def params(self):
        p = np.empty(self.count, np.float32)
        qs, us = C.c_float(), C.c_float()
        self._check(self.lib.casl_net_get_params(self.h, _fptr(p), C.byref(qs), C.byref(us)),
                    "casl_net_get_params")
        return p, qs.value, us.value

    def forward(self, x):
        x = _f32(x, (NET_IN, self.n, self.n))
        y = np.empty((NET_OUT, self.n, self.n), np.float32)
        self._check(self.lib.casl_net_forward(self.h, _fptr(x), _fptr(y)), "casl_net_forward")
        return y

    def backward(self, dy):
        """Gradient of sum(dy * y) for the last forward, flat in parameter order."""
        dy = _f32(dy, (NET_OUT, self.n, self.n))
        g = np.empty(self.count, np.float32)
        self._check(self.lib.casl_net_backward(self.h, _fptr(dy), _fptr(g)), "casl_net_backward")
        return g

    def adam(self, lr):
        self._check(self.lib.casl_net_adam(self.h, float(lr)), "casl_net_adam")


class CaslEnsemble(CaslGPU):
    """M independent simulations of one grid size in one handle
    (casl_ensemble_*): step() advances all members with single launches per
    stage; member_*() read one member back in its own numbering."""

    def __init__(self, nx, members, device=0, **kw):
        self.lib = load_library()
        kw = dict(kw)
        elly = kw.pop("elly", None)
        ellx = kw.pop("ellx", 2 * np.pi)
        elly = ellx if elly is None else elly
        npm = kw.pop("npm", None) or 60 * nx * nx * members
        d = dict(ncontq=40, kd=0.0, beta=0.0, rtherm=0.0, rekman=0.0, cdamp=2.0, nnu=3.0, nm=0,
                 nlevm=2000, fixed_dt=0.0, dtmax=0.05, force_surgery=1, nregmax=20, twistmax=2.5)
        d.update(kw)
        self.p = CaslParams(nx, nx, d["ncontq"], ellx, elly, d["kd"], d["beta"], d["rtherm"],
                            d["rekman"], d["cdamp"], d["nnu"], int(npm), int(d["nm"]), d["nlevm"],
                            d["fixed_dt"], d["dtmax"], d["force_surgery"], d["nregmax"],
                            d["twistmax"])
        h = C.c_void_p()
        self._check(self.lib.casl_ensemble_create(C.byref(self.p), int(members), int(device),
                                                  C.byref(h)), "casl_ensemble_create")
        self.h = h
        self.nx = self.ny = nx
        self.members = members

    def initialise_members(self, fields, ncontq=None):
        q = np.ascontiguousarray(np.stack([_f64(f, (self.nx, self.ny)) for f in fields]))
        if q.shape[0] != self.members:
            raise ValueError("one field per member")
        nc = None if ncontq is None else np.ascontiguousarray(ncontq, np.int32)
        self._check(self.lib.casl_ensemble_initialise(self.h, _d(q), _i(nc)), "casl_ensemble_initialise")

    def member_counts(self, m):
        nq, npt, qj = C.c_int(), C.c_int(), C.c_double()
        self._check(self.lib.casl_ensemble_member_counts(self.h, int(m), C.byref(nq), C.byref(npt),
                                                         C.byref(qj)), "casl_ensemble_member_counts")
        return nq.value, npt.value, qj.value

    def member_contours(self, m):
        nq, npt, qj = self.member_counts(m)
        xq = np.zeros(npt); yq = np.zeros(npt); nextq = np.zeros(npt, np.int32)
        indq = np.zeros(nq, np.int32); npq = np.zeros(nq, np.int32)
        i1q = np.zeros(nq, np.int32); i2q = np.zeros(nq, np.int32)
        self._check(self.lib.casl_ensemble_member_contours(self.h, int(m), _d(xq), _d(yq), _i(nextq),
                                                           _i(indq), _i(npq), _i(i1q), _i(i2q)),
                    "casl_ensemble_member_contours")
        return dict(nq=nq, nptq=npt, qjump=qj, xq=xq, yq=yq, nextq=nextq, indq=indq, npq=npq,
                    i1q=i1q, i2q=i2q)

    def member_scalar(self, m, name):
        v = C.c_double()
        self._check(self.lib.casl_ensemble_member_scalar(self.h, int(m), SCALARS[name], C.byref(v)),
                    "casl_ensemble_member_scalar")
        return v.value
