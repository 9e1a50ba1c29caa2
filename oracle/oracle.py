"""ctypes binding of the CPU oracle (``libcasl_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``, never by the product package.  The
oracle restates Hydra's ``ca/plane/qg/caps`` Fortran (contours.f90,
evolution.f90, spectral.f90, congen.f90, lib/stafft) in C; see
``casl_oracle.h`` for the file:line map and the "parity unpinned" note.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcasl_oracle.so")
_SRC = os.path.join(_HERE, "casl_oracle.c")


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (-O3, no FP contraction, as gfortran on x86-64)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC):
        cmd = ["gcc", "-O3", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-o", _LIB_PATH, _SRC, "-lm"]
        subprocess.check_call(cmd)
    return _LIB_PATH


class OParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("ncontq", C.c_int),
        ("ellx", C.c_double), ("elly", C.c_double), ("kd", C.c_double), ("beta", C.c_double),
        ("rtherm", C.c_double), ("rekman", C.c_double), ("cdamp", C.c_double), ("nnu", C.c_double),
        ("npm", C.c_long), ("nm", C.c_long), ("nlevm", C.c_int),
        ("fixed_dt", C.c_double), ("dtmax", C.c_double), ("force_surgery", C.c_int), ("nregmax", C.c_int),
        ("twistmax", C.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.o_create.restype = C.c_void_p
        L.o_create.argtypes = [C.POINTER(OParams)]
        L.o_destroy.argtypes = [C.c_void_p]
        L.o_forfft.argtypes = [C.c_int, C.c_int, dp]
        L.o_revfft.argtypes = [C.c_int, C.c_int, dp]
        L.o_ptospc.argtypes = [C.c_void_p, dp, dp]
        L.o_spctop.argtypes = [C.c_void_p, dp, dp]
        L.o_table.restype = dp
        L.o_table.argtypes = [C.c_void_p, C.c_int]
        L.o_set_contours.restype = C.c_int
        L.o_set_contours.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, dp, dp, ip, ip, ip, ip, ip]
        L.o_get_counts.argtypes = [C.c_void_p, ip, ip, dp]
        L.o_get_contours.argtypes = [C.c_void_p, dp, dp, ip, ip, ip, ip, ip]
        L.o_con2grid.argtypes = [C.c_void_p, dp, ip]
        L.o_velint.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.o_surgery.restype = C.c_int
        L.o_surgery.argtypes = [C.c_void_p]
        L.o_renode.restype = C.c_int
        L.o_renode.argtypes = [C.c_void_p, dp, dp, C.c_int, dp, dp]
        L.o_main_invert.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.o_gradient.argtypes = [C.c_void_p, dp, dp, dp]
        L.o_inversion.argtypes = [C.c_void_p]
        L.o_advance.argtypes = [C.c_void_p]
        L.o_recontour.restype = C.c_int
        L.o_recontour.argtypes = [C.c_void_p, dp]
        L.o_initialise.restype = C.c_int
        L.o_initialise.argtypes = [C.c_void_p, dp]
        L.o_step.restype = C.c_int
        L.o_step.argtypes = [C.c_void_p]
        L.o_field.restype = dp
        L.o_field.argtypes = [C.c_void_p, C.c_int]
        L.o_scalar.restype = C.c_double
        L.o_scalar.argtypes = [C.c_void_p, C.c_int]
        L.o_set_scalar.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.o_diagnostics.argtypes = [C.c_void_p, dp]
        L.o_spec1d.argtypes = [C.c_void_p, dp, dp, C.c_int]
        L.o_spec_tables.argtypes = [C.c_void_p, ip, ip, dp, dp]
        L.o_genfg.argtypes = [C.c_void_p, dp, C.POINTER(C.c_float)]
        L.o_pvforce.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, dp]
        L.o_nb_forcing_init.restype = C.c_int
        L.o_nb_forcing_init.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.o_nb_forcing.argtypes = [C.c_void_p, C.c_double, dp]
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def forfft(x: np.ndarray) -> np.ndarray:
    """stafft forfft on x(m,n) given as a C array of shape (n, m) (Fortran order of x(m,n))."""
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    n, m = a.shape
    lib().o_forfft(m, n, _dp(a))
    return a


def revfft(x: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float64).copy()
    n, m = a.shape
    lib().o_revfft(m, n, _dp(a))
    return a


FIELDS = {"qs": 0, "qd": 1, "qc": 2, "qq": 3, "pp": 4, "qspre": 5, "emq": 6, "epq": 7,
          "uu": 8, "vv": 9, "qr": 10}
TABLES = {"green": 0, "flo": 1, "fhi": 2, "qdiss": 3, "rksq": 4, "rk": 5,
          "rkx": 6, "hrkx": 7, "rky": 8, "hrky": 9, "bety": 10}
SCALARS = {"t": 0, "dt": 1, "twist": 2, "ireg": 3, "zzrms": 4, "zzmax": 5, "uumax": 6, "qjump": 7}


class Oracle:
    """One oracle simulation state (the module globals of the Fortran program).

    Arrays cross the boundary as numpy arrays whose C shape is the transpose
    of the Fortran shape: a physical field q(ny,nx) is a (nx, ny) C array
    (index [ix-1, iy-1]); a spectral field s(nx,ny) is a (ny, nx) C array.
    """

    def __init__(self, nx, ncontq=40, ellx=2 * np.pi, elly=None, kd=0.0, beta=0.0,
                 rtherm=0.0, rekman=0.0, cdamp=2.0, nnu=3.0, npm=None, nm=0, nlevm=2000,
                 fixed_dt=0.0, dtmax=0.05, force_surgery=0, nregmax=20, twistmax=2.5):
        elly = ellx if elly is None else elly
        if npm is None:
            npm = 60 * nx * nx
        self.p = OParams(nx, nx, ncontq, ellx, elly, kd, beta, rtherm, rekman, cdamp, nnu,
                         int(npm), int(nm), nlevm, fixed_dt, dtmax, force_surgery, nregmax, twistmax)
        self.h = lib().o_create(C.byref(self.p))
        if not self.h:
            raise ValueError("oracle: unsupported parameters (nx must equal ny and be a power of two)")
        self.nx = self.ny = nx

    def close(self):
        if self.h:
            lib().o_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- arrays -------------------------------------------------------------
    def field(self, name) -> np.ndarray:
        p = lib().o_field(self.h, FIELDS[name])
        return np.ctypeslib.as_array(p, shape=(self.nx, self.ny)).copy()

    def set_field(self, name, arr):
        p = lib().o_field(self.h, FIELDS[name])
        dst = np.ctypeslib.as_array(p, shape=(self.nx, self.ny))
        dst[...] = arr

    def table(self, name) -> np.ndarray:
        p = lib().o_table(self.h, TABLES[name])
        shape = (self.ny, self.nx) if TABLES[name] < 6 else (self.nx,)
        return np.ctypeslib.as_array(p, shape=shape).copy()

    def scalar(self, name) -> float:
        return lib().o_scalar(self.h, SCALARS[name])

    def set_scalar(self, name, v):
        lib().o_set_scalar(self.h, SCALARS[name], float(v))

    # --- contours -------------------------------------------------------------
    def counts(self):
        nq, npt, qj = C.c_int(), C.c_int(), C.c_double()
        lib().o_get_counts(self.h, C.byref(nq), C.byref(npt), C.byref(qj))
        return nq.value, npt.value, qj.value

    def contours(self) -> dict:
        nq, npt, qj = self.counts()
        xq = np.zeros(npt); yq = np.zeros(npt); nextq = np.zeros(npt, np.int32)
        indq = np.zeros(nq, np.int32); npq = np.zeros(nq, np.int32)
        i1q = np.zeros(nq, np.int32); i2q = np.zeros(nq, np.int32)
        lib().o_get_contours(self.h, _dp(xq), _dp(yq), _ip(nextq), _ip(indq), _ip(npq), _ip(i1q), _ip(i2q))
        return dict(nq=nq, nptq=npt, qjump=qj, xq=xq, yq=yq, nextq=nextq, indq=indq, npq=npq, i1q=i1q, i2q=i2q)

    def set_contours(self, c: dict):
        xq = np.ascontiguousarray(c["xq"], np.float64); yq = np.ascontiguousarray(c["yq"], np.float64)
        nextq = np.ascontiguousarray(c["nextq"], np.int32)
        indq = np.ascontiguousarray(c["indq"], np.int32); npq = np.ascontiguousarray(c["npq"], np.int32)
        i1q = np.ascontiguousarray(c["i1q"], np.int32); i2q = np.ascontiguousarray(c["i2q"], np.int32)
        rc = lib().o_set_contours(self.h, len(indq), len(xq), float(c["qjump"]), _dp(xq), _dp(yq),
                                  _ip(nextq), _ip(indq), _ip(npq), _ip(i1q), _ip(i2q))
        if rc:
            raise ValueError("oracle: contour capacity exceeded")

    # --- procedures -------------------------------------------------------------
    def ptospc(self, q):
        r = np.ascontiguousarray(q, np.float64).copy()
        out = np.zeros((self.ny, self.nx))
        lib().o_ptospc(self.h, _dp(r), _dp(out))
        return out

    def spctop(self, s):
        r = np.ascontiguousarray(s, np.float64).copy()
        out = np.zeros((self.nx, self.ny))
        lib().o_spctop(self.h, _dp(r), _dp(out))
        return out

    def con2grid(self, levels=False):
        qc = np.zeros((self.nx, self.ny))
        if levels:
            lv = np.zeros((4 * self.nx, 4 * self.ny), np.int32)
            lib().o_con2grid(self.h, _dp(qc), _ip(lv))
            return qc, lv
        lib().o_con2grid(self.h, _dp(qc), None)
        return qc

    def velint(self, uu, vv):
        _, npt, _ = self.counts()
        uu = np.ascontiguousarray(uu, np.float64); vv = np.ascontiguousarray(vv, np.float64)
        uq = np.zeros(npt); vq = np.zeros(npt)
        lib().o_velint(self.h, _dp(uu), _dp(vv), _dp(uq), _dp(vq))
        return uq, vq

    def main_invert(self, qq):
        qq = np.ascontiguousarray(qq, np.float64)
        uu = np.zeros((self.nx, self.ny)); vv = np.zeros((self.nx, self.ny)); pp = np.zeros((self.ny, self.nx))
        lib().o_main_invert(self.h, _dp(qq), _dp(uu), _dp(vv), _dp(pp))
        return uu, vv, pp

    def gradient(self, ff):
        ff = np.ascontiguousarray(ff, np.float64)
        fx = np.zeros((self.nx, self.ny)); fy = np.zeros((self.nx, self.ny))
        lib().o_gradient(self.h, _dp(ff), _dp(fx), _dp(fy))
        return fx, fy

    def renode(self, xd, yd):
        xd = np.ascontiguousarray(xd, np.float64); yd = np.ascontiguousarray(yd, np.float64)
        cap = 8 * len(xd) + 64
        xr = np.zeros(cap); yr = np.zeros(cap)
        n = lib().o_renode(self.h, _dp(xd), _dp(yd), len(xd), _dp(xr), _dp(yr))
        return xr[:max(n, 0)], yr[:max(n, 0)]

    def surgery(self):
        if lib().o_surgery(self.h):
            raise RuntimeError("oracle surgery: capacity exceeded")

    def inversion(self):
        lib().o_inversion(self.h)

    def advance(self):
        lib().o_advance(self.h)

    def recontour(self, qq):
        q = np.ascontiguousarray(qq, np.float64).copy()
        rc = lib().o_recontour(self.h, _dp(q))
        if rc:
            raise RuntimeError(f"oracle recontour failed ({rc})")

    def initialise(self, q0):
        q = np.ascontiguousarray(q0, np.float64)
        rc = lib().o_initialise(self.h, _dp(q))
        if rc:
            raise RuntimeError(f"oracle initialise failed ({rc})")

    def step(self):
        rc = lib().o_step(self.h)
        if rc:
            raise RuntimeError(f"oracle step failed ({rc}): "
                               + {1: "node capacity", 2: "contour capacity", 3: "surgery capacity",
                                  4: "node left the domain or became non-finite"}.get(rc, "?"))

    def diagnostics(self):
        out = np.zeros(4)
        lib().o_diagnostics(self.h, _dp(out))
        return dict(ekin=out[0], epot=out[1], enstrophy=out[2], circulation=out[3])

    def spec1d(self, ss, iopt=0):
        """spec1d (spectral.f90:370-424) of a spectral field ss(nx,ny) given as
        an (ny, nx) array; returns (spec[0..max(nx,ny)], ss after the call)."""
        a = np.ascontiguousarray(ss, dtype=np.float64).copy()
        spec = np.zeros(max(self.nx, self.nx) + 1)
        lib().o_spec1d(self.h, _dp(a), _dp(spec), int(iopt))
        return spec, a

    def genfg(self, qq):
        """genfg's ultra-fine PV (post/genfg.f90:79-113) of the current contours
        plus the residual qq (physical, (nx, ny) array), float32 (nxu, nyu)."""
        r = np.ascontiguousarray(qq, np.float64)
        out = np.zeros((16 * self.nx, 16 * self.nx), np.float32)
        lib().o_genfg(self.h, _dp(r), out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def pvforce(self, ivor, vorvor, rnd):
        """pvforce (evolution.f90:330-428) with the given uniforms."""
        r = np.ascontiguousarray(rnd, np.float64).ravel()
        m = 2 if ivor == 1 else 3
        lib().o_pvforce(self.h, int(ivor), float(vorvor), len(r) // m, _dp(r))

    def nb_forcing_init(self, kfmid, fwid, famp):
        return lib().o_nb_forcing_init(self.h, float(kfmid), float(fwid), float(famp))

    def nb_forcing(self, dt, rnd):
        r = np.ascontiguousarray(rnd, np.float64).ravel()
        lib().o_nb_forcing(self.h, float(dt), _dp(r))

    def spec_tables(self):
        """kmax, kmaxred, spmf, alk of init_spectral (spectral.f90:109-134)."""
        kmax = C.c_int(0)
        kred = C.c_int(0)
        spmf = np.zeros(self.nx + 1)
        alk = np.zeros(self.nx + 1)
        lib().o_spec_tables(self.h, C.byref(kmax), C.byref(kred), _dp(spmf), _dp(alk))
        return dict(kmax=kmax.value, kmaxred=kred.value, spmf=spmf, alk=alk)
