"""casl_con2grid_noalloc: con2grid for callers that cannot allocate device memory.

Callers whose GPU memory is handed out by their own pool or by another
framework, callers that must not trigger cudaMalloc's device-wide
synchronisation inside a time-critical loop, and callers that hold no casl
handle, pass device arrays they already own; the entry point's scratch is a
fixed device array inside the library.  Checked against the handle-based
casl_con2grid on two calls in a row with different contour sets, so the
second call also shows that the first call's leftovers in the shared scratch
are cleared; at the largest grid it serves (n = 256) against the oracle, and
the device's free memory is the same before and after a call.  This file is
collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu

REL = 1e-12


def _call(gpu_lib, n, c, qc):
    import torch
    dev = qc.device
    xq = torch.tensor(c["xq"], dtype=torch.float64, device=dev)
    yq = torch.tensor(c["yq"], dtype=torch.float64, device=dev)
    nextq = torch.tensor(c["nextq"], dtype=torch.int32, device=dev)  # 1-based
    qc.fill_(float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    rc = gpu_lib.casl_con2grid_noalloc(n, 2 * np.pi, 2 * np.pi, int(c["nptq"]), float(c["qjump"]),
                                      ctypes.c_void_p(xq.data_ptr()), ctypes.c_void_p(yq.data_ptr()),
                                      ctypes.c_void_p(nextq.data_ptr()), ctypes.c_void_p(qc.data_ptr()),
                                      None)
    free1 = torch.cuda.mem_get_info(dev)[0]
    assert rc == 0, gpu_lib.casl_error_string(rc)
    return qc.cpu().numpy(), free0, free1


def test_noalloc_matches_con2grid(oracle_mod, gpu_lib):
    import torch

    from hydra_b200.casl import CaslGPU

    n = 128
    o = oracle_mod.Oracle(n, ncontq=20, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 8.0, 11))
    states = [o.contours()]
    o.step()
    o.step()
    states.append(o.contours())
    assert states[0]["nptq"] != states[1]["nptq"]

    g = CaslGPU(n, ncontq=20)
    qc = torch.empty((n, n), dtype=torch.float64, device="cuda:0")
    for c in states:  # two calls in a row
        g.set_contours(c)
        ref = g.con2grid()  # the existing entry point
        out, _, _ = _call(gpu_lib, n, c, qc)
        assert np.isfinite(out).all()
        assert np.abs(out - ref).max() <= REL * np.abs(ref).max()
    g.close()


def test_noalloc_largest_grid_matches_oracle_without_allocating(oracle_mod, gpu_lib):
    """n = 256 uses the whole scratch array; the first call is the warm-up
    that loads the array, the second must leave the free memory unchanged."""
    import torch

    n = 256
    o = oracle_mod.Oracle(n, ncontq=40, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 2))
    c = o.contours()
    ref = o.con2grid()
    qc = torch.empty((n, n), dtype=torch.float64, device="cuda:0")
    for call in range(2):
        out, free0, free1 = _call(gpu_lib, n, c, qc)
        assert np.abs(out - ref).max() <= REL * np.abs(ref).max()
        if call == 1:
            assert free1 == free0, (free0, free1)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_lib):
    # n = 512 would need a larger scratch array than the library holds
    rc = gpu_lib.casl_con2grid_noalloc(512, 2 * np.pi, 2 * np.pi, 0, 1.0, None, None, None,
                                      ctypes.c_void_p(1), None)
    assert rc == 1  # CASL_EINVAL
