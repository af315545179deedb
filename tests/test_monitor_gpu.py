"""GPU tests of the device statistics and monitors against numpy
restatements of the reference's formulas on the same fields:
calcStat (src/mod_statistics.f90:126-192), calcAndWriteSkf, calcAndWriteForcing,
extractAndWriteProbePoint and extractRegion (src/mod_monitor.f90:197-376)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _centred(u, v, w, u_crf=0.0):
    """cell-centred velocities from ghosted (nz+2, ny+2, nx+2) arrays"""
    uc = 0.5 * (u[1:-1, 1:-1, :-2] + u[1:-1, 1:-1, 1:-1]) + u_crf
    vc = 0.5 * (v[1:-1, :-2, 1:-1] + v[1:-1, 1:-1, 1:-1])
    wc = 0.5 * (w[:-2, 1:-1, 1:-1] + w[1:-1, 1:-1, 1:-1])
    return uc, vc, wc


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_statistics_match_numpy(gpu, prec):
    plb = gpu
    p = plb.PL_FP64 if prec == "fp64" else plb.PL_MIXED
    ch = plb.Channel(plb.ChannelConfig(nx=64, ny=48, nz=32, stretch_ratio=1.5, re_tau=180.0, precision=p))
    ch.init_flow(3, 0.1)
    ch.stat_enable(nt_init_stat=2, sample_interval=3)
    ref = {n: 0.0 for n in ch.STAT_NAMES}
    nspl = 0
    for nt in range(1, 12):
        ch.step(1)
        ch.stat_sample(nt)
        if (nt - 2) % 3 == 0:
            u, v, w, pp = ch.get_fields()
            uc, vc, wc = _centred(u, v, w)
            pi = pp[1:-1, 1:-1, 1:-1]
            for n, val in zip(ch.STAT_NAMES, (uc, vc, wc, uc * uc, vc * vc, wc * wc, uc * vc, uc * wc, vc * wc, pi,
                                                pi * pi)):
                ref[n] = ref[n] + val
            nspl += 1
    nts, nte, n = ch.stat_info()
    assert (nts, nte, n) == (3, 2 + 3 * nspl, nspl)
    for name in ch.STAT_NAMES:
        assert _rel(ch.stat_get(name), ref[name]) < TOL, name
    ch.stat_disable()
    ch.close()


def test_monitors_match_numpy(gpu):
    plb = gpu
    cfg = plb.ChannelConfig(nx=64, ny=48, nz=32, stretch_ratio=1.5, re_tau=180.0)
    ch = plb.Channel(cfg)
    ch.init_flow(5, 0.1)
    ch.step(3)
    u, v, w, pp = ch.get_fields()
    nz = cfg.nz
    zf = 0.5 * (1.0 + np.tanh((np.arange(nz + 1) / nz - 0.5) * 1.5) / np.tanh(0.75))
    dzf = cfg.lz * np.diff(zf)
    re_inv = 1.0 / plb.re_from_retau(cfg.re_tau)
    for wall, kw in ((0, 1), (1, nz)):
        tau = re_inv * u[kw, 1:-1, 1:-1].mean() / (0.5 * dzf[kw - 1])
        ut, cf = ch.skin_friction(wall)
        assert abs(ut - np.sqrt(tau)) <= TOL * np.sqrt(tau) and abs(cf - tau / 0.5) <= TOL * tau / 0.5
    means = ch.forcing_means()
    mref = (u[1:-1, 1:-1, 1:-1].mean(axis=(1, 2)) * dzf / cfg.lz).sum()
    assert abs(means[0] - mref) <= TOL and means[1] == 0.0 and means[2] == 0.0
    pr = ch.probe(7, 11, 13)
    assert np.array_equal(pr, [u[13, 11, 7], v[13, 11, 7], w[13, 11, 7], pp[13, 11, 7]])
    reg = ch.region((60, 70, 1, 5, 30, 40))  # clipped to i 60..64, k 30..32
    uc, vc, wc = _centred(u, v, w)
    sl = (slice(29, 32), slice(0, 5), slice(59, 64))
    for q, ref in enumerate((uc[sl], vc[sl], wc[sl], pp[1:-1, 1:-1, 1:-1][sl])):
        assert np.array_equal(reg[q], ref), q
    with pytest.raises(plb.PowerLLELError):
        ch.probe(0, 1, 1)
    ch.close()
