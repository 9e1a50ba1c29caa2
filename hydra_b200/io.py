"""Readers and writers of the caps output files (the reference's gfortran
I/O, evolution.f90:582-583, 648-774, common.f90:30-100), through the C ABI's
host-only entry points: no GPU is needed for these."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from hydra_b200.casl import CaslError, load_library


def _p(path):
    return os.fsencode(path)


def _chk(rc, where):
    if rc:
        lib = load_library()
        raise CaslError(rc, where, lib.casl_error_string(rc).decode())


def _ia(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


def _da(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def append_synopsis(path, nq, nptq, t, qjump):
    _chk(load_library().casl_io_append_synopsis(_p(path), nq, nptq, t, qjump), "append_synopsis")


def append_ene(path, tgrid, ekin, epot):
    _chk(load_library().casl_io_append_ene(_p(path), tgrid, ekin, epot), "append_ene")


def append_norms(path, tgrid, qql2):
    _chk(load_library().casl_io_append_norms(_p(path), tgrid, qql2), "append_norms")


def append_spectrum(path, tgrid, sumqspec, qql2, kmaxred, alk, qspec):
    a, pa = _da(alk)
    q, pq = _da(qspec)
    _chk(load_library().casl_io_append_spectrum(_p(path), tgrid, sumqspec, qql2, kmaxred, pa, pq),
         "append_spectrum")


def append_monitor(path, t, cfl, zzrms, zzmax, uumax, twist):
    _chk(load_library().casl_io_append_monitor(_p(path), t, cfl, zzrms, zzmax, uumax, twist),
         "append_monitor")


def append_complexity(path, t, nq, nptq):
    _chk(load_library().casl_io_append_complexity(_p(path), t, nq, nptq), "append_complexity")


def write_index(path, npq, i1q, indq):
    a, pa = _ia(npq)
    b, pb = _ia(i1q)
    c, pc = _ia(indq)
    _chk(load_library().casl_io_write_index(_p(path), len(a), pa, pb, pc), "write_index")


def read_index(path, nq):
    a, pa = _ia(np.zeros(nq))
    b, pb = _ia(np.zeros(nq))
    c, pc = _ia(np.zeros(nq))
    _chk(load_library().casl_io_read_index(_p(path), nq, pa, pb, pc), "read_index")
    return a, b, c


def write_nodes(path, xq, yq):
    x, px = _da(xq)
    y, py = _da(yq)
    _chk(load_library().casl_io_write_nodes(_p(path), len(x), px, py), "write_nodes")


def read_nodes(path, nptq):
    x, px = _da(np.zeros(nptq))
    y, py = _da(np.zeros(nptq))
    _chk(load_library().casl_io_read_nodes(_p(path), nptq, px, py), "read_nodes")
    return x, y


def write_r4(path, irec, t, a):
    """Record irec (1-based) of a direct-access r4 file: t, a(ny,nx) given
    as an (nx, ny) array (iy fastest)."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    nx, ny = f.shape
    _chk(load_library().casl_io_write_r4(_p(path), irec, nx, ny, float(t),
                                         f.ctypes.data_as(C.POINTER(C.c_float))), "write_r4")


def read_r4(path, irec, nx, ny):
    f = np.zeros((nx, ny), dtype=np.float32)
    t = C.c_float()
    _chk(load_library().casl_io_read_r4(_p(path), irec, nx, ny, C.byref(t),
                                        f.ctypes.data_as(C.POINTER(C.c_float))), "read_r4")
    return t.value, f


def read_synopsis(path, iind):
    nq, npt = C.c_int(), C.c_int()
    t, qj = C.c_double(), C.c_double()
    _chk(load_library().casl_io_read_synopsis(_p(path), iind, C.byref(nq), C.byref(npt),
                                              C.byref(t), C.byref(qj)), "read_synopsis")
    return nq.value, npt.value, t.value, qj.value
