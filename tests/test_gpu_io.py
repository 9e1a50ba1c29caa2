"""savecont / savegrid / readcont through the C ABI (evolution.f90:648-774,
common.f90:30-100): the files hold the saved state in the reference's
layouts, a restart from them reproduces it, and savegrid's numbers match
the oracle's energy, l2 norm and spectrum at the same state."""
import numpy as np
import pytest

from hydra_b200.synthetic import random_pv

pytestmark = pytest.mark.gpu


def test_savecont_then_readcont(gpu_lib, tmp_path):
    from hydra_b200 import io
    from hydra_b200.casl import CaslGPU

    n = 64
    g = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    g.initialise(random_pv(n, 6.0, 2))
    g.step(3)
    g.savecont(tmp_path, 1)
    g.io_wait()
    c = g.contours()
    qq = g.field("qq")  # savecont inverts first (evolution.f90:87)
    t = g.scalar("t")
    cont = tmp_path / "cont"
    nq, npt, ts, qj = io.read_synopsis(cont / "qqsynopsis.asc", 1)
    assert (nq, npt) == (c["nq"], c["nptq"])
    assert abs(ts - t) <= 5e-6 and abs(qj - c["qjump"]) <= 5e-13
    npq, i1q, indq = io.read_index(cont / "qqindex001", nq)
    assert np.array_equal(npq, c["npq"]) and np.array_equal(i1q, c["i1q"])
    assert np.array_equal(indq, c["indq"])
    x, y = io.read_nodes(cont / "qqnodes001", npt)
    assert np.array_equal(x, c["xq"]) and np.array_equal(y, c["yq"])
    tr, qd = io.read_r4(cont / "qqresi.r4", 1, n, n)
    assert abs(tr - t) <= 1e-6 * max(1.0, t) and np.isfinite(qd).all()

    g2 = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    g2.readcont(tmp_path, 1)
    c2 = g2.contours()
    for k in ("nq", "nptq", "npq", "i1q", "i2q", "indq", "nextq", "xq", "yq"):
        assert np.array_equal(np.asarray(c2[k]), np.asarray(c[k])), k
    assert g2.scalar("t") == ts
    # qs = ptospc(con2grid + real(spctop(qq - qc))): the saved PV up to the
    # float32 rounding of the residual
    assert np.abs(g2.field("qs") - qq).max() <= 1e-6 * np.abs(qq).max()
    g2.step(2)  # the restarted run advances
    g.close()
    g2.close()


def test_savegrid_matches_oracle(oracle_mod, gpu_lib, tmp_path):
    from hydra_b200 import io
    from hydra_b200.casl import CaslGPU

    n = 64
    o = oracle_mod.Oracle(n, ncontq=20, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 6.0, 3))
    o.step()
    g = CaslGPU(n, ncontq=20, force_surgery=1, dtmax=0.05)
    g.set_contours(o.contours())
    for f in ("qs", "qd", "qr", "emq", "epq"):
        g.set_field(f, o.field(f))
    g.set_scalar("t", o.scalar("t"))
    g.savegrid(tmp_path, 1)
    g.io_wait()

    o.inversion()
    d = o.diagnostics()
    ene = (tmp_path / "ene.asc").read_text().split()
    assert abs(float(ene[0]) - o.scalar("t")) <= 5e-3
    assert abs(float(ene[1]) - d["ekin"]) <= 1e-10 * max(1.0, d["ekin"])
    norms = (tmp_path / "norms.asc").read_text().split()
    assert abs(float(norms[1]) - d["enstrophy"]) <= 1e-9 * d["enstrophy"]

    spec, _ = o.spec1d(o.field("qq"), 0)
    tb = o.spec_tables()
    lines = (tmp_path / "spectra.asc").read_text().splitlines()
    head = lines[0].split()
    kred = tb["kmaxred"]
    assert int(head[3]) == kred and len(lines) == 1 + kred
    sumq = 8.0 * spec[1:tb["kmax"] + 1].sum() / (n * n)
    assert abs(float(head[1]) - sumq) <= 1e-9 * sumq
    for k in range(1, kred + 1):
        a, lq = map(float, lines[k].split())
        assert abs(a - tb["alk"][k]) <= 5e-9
        assert abs(lq - np.log10(tb["spmf"][k] * spec[k])) <= 5e-8

    tq, q4 = io.read_r4(tmp_path / "qq.r4", 1, n, n)
    ref = o.spctop(o.field("qq"))
    assert np.abs(q4 - ref).max() <= 1e-6 * np.abs(ref).max()
    g.close()


def test_genfg_matches_oracle(oracle_mod, gpu_lib):
    """genfg's ultra-fine PV (post/genfg.f90:79-194): con2ugrid of the
    contours plus the bilinear residual, as float32; strided and wrapped
    window views are slices of the full image."""
    from hydra_b200.casl import CaslGPU

    n = 32
    o = oracle_mod.Oracle(n, ncontq=10, force_surgery=1, dtmax=0.05)
    o.initialise(random_pv(n, 4.0, 5))
    o.step()
    g = CaslGPU(n, ncontq=10, force_surgery=1, dtmax=0.05)
    g.set_contours(o.contours())
    rng = np.random.default_rng(6)
    qr = 0.3 * rng.standard_normal((n, n))
    g.set_field("qr", qr)
    ref = o.genfg(qr)
    full = g.genfg()
    assert full.shape == ref.shape == (16 * n, 16 * n)
    # integer-exact contour part; the residual terms agree to FP64 rounding
    assert np.abs(full - ref).max() <= 1e-6 * np.abs(ref).max()
    assert np.array_equal(g.genfg(stride=4), full[::4, ::4])
    nu = 16 * n
    win = g.genfg(ix1v=nu - 40 + 1, nxv=100, iy1v=7, nyv=nu)  # wraps in x and y
    cols = [(nu - 40 + i) % nu for i in range(100)]
    rows = [(6 + i) % nu for i in range(nu)]
    assert np.array_equal(win, full[np.ix_(cols, rows)])
    g.close()


def _ene_lines(path):
    return [list(map(float, ln.split())) for ln in path.read_text().splitlines() if ln.strip()]


def test_scheduled_saves_interpolate_to_the_save_times(oracle_mod, gpu_lib, tmp_path):
    """casl_set_saves: the time loop's own save schedule (evolution.f90:
    586-600, 200-204, 648-774).  The oracle steps beside the GPU run; the
    reference's flags (t + dt >= tgrid at adapt), the interpolation weights
    pt = (t - tgrid)/dt and the record counters are replayed here on its
    states, and every written value is compared: ene.asc, norms.asc, the
    spectra headers, qq.r4 records at the save times, and the contour saves'
    times."""
    from hydra_b200 import io
    from hydra_b200.casl import CaslGPU

    n, K = 64, 14
    q0 = random_pv(n, 6.0, 7)
    kw = dict(ncontq=20, force_surgery=1, dtmax=0.05)
    o = oracle_mod.Oracle(n, **kw)
    o.initialise(q0)
    ts, dts, qqs, ens = [], [], [], []
    # with force_surgery and no recontouring inside K < nregmax steps, a step
    # is surgery then advance; the saves read the state after the surgery
    for _ in range(K):
        o.surgery()
        o.inversion()
        d = o.diagnostics()
        ts.append(o.scalar("t"))
        qqs.append(o.field("qq").copy())
        ens.append((d["ekin"], d["epot"]))
        o.advance()
        dts.append(o.scalar("dt"))

    # save intervals from the run's own length: about 5 grid and 3 contour saves
    tg, tc = ts[-1] / 5.3, ts[-1] / 3.4
    g = CaslGPU(n, **kw)
    g.initialise(q0)
    g.set_saves(tmp_path, tg, tc)
    g.step(K)
    g.io_wait()

    # the reference's schedule on the oracle's states
    grid, cont = [], []
    igrec, icrec, gpend, cpend, tgrid = 0, 1, False, False, 0.0
    for k in range(K):
        if gpend:
            pt = (ts[k] - tgrid) / dts[k - 1]
            ptc = 1.0 - pt
            grid.append((tgrid, pt * qqs[k - 1] + ptc * qqs[k],
                         pt * ens[k - 1][0] + ptc * ens[k][0], pt * ens[k - 1][1] + ptc * ens[k][1],
                         pt))
            igrec += 1
            gpend = False
        if cpend:
            cont.append(ts[k])
            icrec += 1
            cpend = False
        tgrid, tcont = tg * igrec, tc * icrec
        gpend = ts[k] + dts[k] >= tgrid
        cpend = ts[k] + dts[k] >= tcont
    assert len(grid) >= 4 and len(cont) >= 3
    assert any(0.0 < gr[4] < 1.0 for gr in grid)  # saves between two steps
    assert g.save_counters() == (len(grid), 1 + len(cont))

    ene = _ene_lines(tmp_path / "ene.asc")
    norms = _ene_lines(tmp_path / "norms.asc")
    assert len(ene) == len(norms) == len(grid)
    tb = o.spec_tables()
    heads = [ln.split() for ln in (tmp_path / "spectra.asc").read_text().splitlines()
             if len(ln.split()) == 4]
    assert len(heads) == len(grid)
    for r, (tgr, qs_, ek, ep, _) in enumerate(grid):
        assert abs(ene[r][0] - tgr) <= 5e-3 and abs(norms[r][0] - tgr) <= 5e-3
        assert abs(ene[r][1] - ek) <= 1e-10 * max(1.0, ek)
        assert abs(ene[r][2] - ep) <= 1e-10 * max(1.0, ep)
        phys = o.spctop(qs_)
        l2 = (2 * np.pi / n) ** 2 * (phys ** 2).sum()
        assert abs(norms[r][1] - l2) <= 1e-9 * l2 + 1e-9
        spec, _ = o.spec1d(qs_, 0)
        sumq = 8.0 * spec[1:tb["kmax"] + 1].sum() / (n * n)
        assert abs(float(heads[r][1]) - sumq) <= 1e-9 * sumq + 1e-9
        tr, q4 = io.read_r4(tmp_path / "qq.r4", r + 1, n, n)
        assert abs(tr - tgr) <= 1e-6
        assert np.abs(q4 - phys).max() <= 1e-6 * np.abs(phys).max()
    syn = (tmp_path / "cont" / "qqsynopsis.asc").read_text().splitlines()
    assert len(syn) == len(cont)
    for line, t in zip(syn, cont):
        assert abs(float(line.split()[2]) - t) <= 5e-6
    g.close()
    o.close()
