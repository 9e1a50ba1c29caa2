"""Failure paths of the C ABI, made on the host (no GPU fault is caused).

The reference stops the program or overflows silently where these return a
status (common.f90:30-100 reads restart files without checks; the node and
contour capacities of constants.f90:35-41 are fixed arrays): a capacity that
the state or renode's growth exceeds gives CASL_ECAPACITY, a non-finite or
out-of-domain node CASL_EDOMAIN, broken links CASL_EINVAL, and a truncated
restart file CASL_EIO.  Every write past a capacity is skipped on the device
(renode placement and the write-back return when the output count is above
it), so these runs stay inside their buffers.
"""
import os

import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu

CASL_EINVAL, CASL_ECAPACITY, CASL_EDOMAIN, CASL_EUNSUPPORTED, CASL_EIO = 1, 2, 5, 7, 8


@pytest.fixture(scope="module")
def state(oracle_mod):
    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 4))
    c = o.contours()
    o.close()
    return n, c


def thin(c):
    """Every other node of each contour with at least 8 nodes: a valid state
    that renode grows back to about its former size."""
    xs, ys, nxt, npq, i1q = [], [], [], [], []
    start = 0
    for j in range(c["nq"]):
        a, m = c["i1q"][j] - 1, c["npq"][j]
        idx = np.arange(a, a + m)
        if m >= 8:
            idx = idx[::2]
        k = len(idx)
        xs.append(c["xq"][idx]); ys.append(c["yq"][idx])
        nxt.append(np.r_[np.arange(start + 2, start + k + 1), start + 1])
        npq.append(k); i1q.append(start + 1)
        start += k
    npq = np.array(npq, np.int32); i1q = np.array(i1q, np.int32)
    return dict(nq=c["nq"], nptq=start, qjump=c["qjump"], xq=np.concatenate(xs),
                yq=np.concatenate(ys), nextq=np.concatenate(nxt).astype(np.int32),
                indq=c["indq"].copy(), npq=npq, i1q=i1q, i2q=(i1q + npq - 1).astype(np.int32))


def test_capacity_on_upload(gpu_lib, state):
    from hydra_b200.casl import CaslError, CaslGPU
    n, c = state
    g = CaslGPU(n, ncontq=20, npm=c["nptq"] - 1, nm=10_000)
    with pytest.raises(CaslError) as e:
        g.set_contours(c)
    assert e.value.code == CASL_ECAPACITY
    g.close()


def test_capacity_on_renode_growth(gpu_lib, state):
    from hydra_b200.casl import CaslError, CaslGPU
    n, c = state
    t = thin(c)
    g = CaslGPU(n, ncontq=20, npm=t["nptq"] + 16, nm=10_000, force_surgery=1)
    g.set_contours(t)
    assert g.counts()[1] == t["nptq"]
    with pytest.raises(CaslError) as e:
        g.surgery()  # renode restores the node density: about twice the nodes
    assert e.value.code == CASL_ECAPACITY
    g.close()
    # the same state with room to grow renodes without error
    g = CaslGPU(n, ncontq=20, npm=4 * c["nptq"], nm=10_000, force_surgery=1)
    g.set_contours(t)
    g.surgery()
    assert g.counts()[1] > t["nptq"] + 16
    g.close()


@pytest.mark.parametrize("bad", ["nan", "outside", "link", "range"])
def test_bad_state_rejected(gpu_lib, state, bad):
    from hydra_b200.casl import CaslError, CaslGPU
    n, c = state
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in c.items()}
    if bad == "nan":
        d["xq"][17] = np.nan
    elif bad == "outside":
        d["yq"][5] = 4.0  # beyond elly/2 = pi
    elif bad == "link":
        d["nextq"][3] = d["nptq"] + 1
    else:
        d["npq"][0] += 1
    g = CaslGPU(n, ncontq=20)
    with pytest.raises(CaslError) as e:
        g.set_contours(d)
    assert e.value.code == (CASL_EDOMAIN if bad in ("nan", "outside") else CASL_EINVAL)
    assert g.counts()[:2] == (0, 0)  # nothing of the rejected state is kept
    g.set_contours(c)  # a good state is accepted afterwards
    assert g.counts()[:2] == (c["nq"], c["nptq"])
    g.step(1)
    g.close()


def test_truncated_restart_file(gpu_lib, tmp_path):
    from hydra_b200.casl import CaslError, CaslGPU
    n = 64
    g = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    g.initialise(random_pv(n, 6.0, 2))
    g.step(1)
    g.savecont(tmp_path, 1)
    g.io_wait()
    g.close()
    nodes = tmp_path / "cont" / "qqnodes001"
    size = os.path.getsize(nodes)
    with open(nodes, "r+b") as f:
        f.truncate(size // 2)
    g2 = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    with pytest.raises(CaslError) as e:
        g2.readcont(tmp_path, 1)
    assert e.value.code == CASL_EIO
    with pytest.raises(CaslError) as e:
        g2.readcont(tmp_path, 2)  # no such save
    assert e.value.code == CASL_EIO
    g2.close()


def test_save_schedule_arguments(gpu_lib, tmp_path):
    """casl_set_saves: both kinds off, a negative record counter or a
    contour counter below 1 is CASL_EINVAL; an ensemble handle has no save
    schedule (CASL_EUNSUPPORTED); a NULL directory turns the schedule off,
    after which steps write nothing."""
    from hydra_b200.casl import CaslEnsemble, CaslError, CaslGPU
    n = 32
    g = CaslGPU(n, ncontq=10, force_surgery=1, dtmax=0.05)
    g.initialise(random_pv(n, 4.0, 1))
    for args in [dict(tgsave=0.0, tcsave=0.0), dict(tgsave=0.1, tcsave=0.0, igrec=-1),
                 dict(tgsave=0.1, tcsave=0.2, icrec=0), dict(tgsave=float("nan"), tcsave=0.2)]:
        with pytest.raises(CaslError) as e:
            g.set_saves(tmp_path, **args)
        assert e.value.code == CASL_EINVAL, args
    g.set_saves(tmp_path / "on", tgsave=0.01, tcsave=0.0)
    g.set_saves(None, 0.0, 0.0)  # off again: nothing is written
    g.step(3)
    g.io_wait()
    assert not (tmp_path / "on").exists()
    assert g.save_counters() == (0, 1)
    g.close()
    e = CaslEnsemble(n, 2, dtmax=0.05)
    rc = e.lib.casl_set_saves(e.h, os.fsencode(str(tmp_path)), 0.0, 0.1, 0.1, 0, 1)
    assert rc == CASL_EUNSUPPORTED
    e.close()
