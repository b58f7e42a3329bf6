"""Grating-coupler flow (orf.gratingCouplerTE / orf.fiberCoupling) on the CPU:
the fiber overlap integral (tests/TestCPO.m:12-24), the TE0 source pick and
the monitor-box power balance of the short grating (tests/TestCPO.m:26-34),
the latter with the oracle standing in for the GPU run."""
import warnings

import numpy as np

import oracle
from opticrcwafdtd_b200 import coupler


def test_fiber_overlap_of_itself_is_one():
    x = np.arange(0, 20.0 + 1e-9, 0.02)
    th, w0, lam = np.deg2rad(8), 5.2, 1.55
    u = x - 10
    E = np.exp(-(u * np.cos(th) / w0) ** 2) * np.exp(1j * 2 * np.pi / lam * np.sin(th) * u)
    res = dict(xUp=x, EyUp=3 * E, lambdas=lam, nClad=1, Pup=0.6)
    eta, ov = coupler.fiberCoupling(res, th, 10, w0)
    assert abs(ov.item() - 1) < 1e-12
    assert abs(eta.item() - 0.6) < 1e-12
    # the wrong tilt sign must reduce the overlap
    assert coupler.fiberCoupling(res, -th, 10, w0)[0].item() / 0.6 < 0.5


def test_fiber_coupling_shapes():
    x = np.linspace(0, 20, 501)
    E = np.exp(-((x - 9) / 5) ** 2)[:, None] * np.ones((1, 3))
    res = dict(xUp=x, EyUp=E, lambdas=[1.5, 1.55, 1.6], nClad=1.0, Pup=np.array([0.5, 0.6, 0.7]))
    eta, ov = coupler.fiberCoupling(res, np.deg2rad([0, 5, 10, 15]), [8, 9, 10], 5.2)
    assert eta.shape == (4, 3, 3) and ov.shape == (4, 3, 3)
    assert np.all(ov <= 1 + 1e-12) and np.all(ov >= 0)
    np.testing.assert_allclose(eta, ov * np.array([0.5, 0.6, 0.7]), rtol=1e-14)


def test_short_grating_source_is_te0_not_a_substrate_mode():
    sim, bd = coupler.gratingCouplerTE_sim(dict(nPer=6, lambdas=[1.53, 1.55, 1.57]))
    assert abs(bd["neff"] - 2.835) < 0.01
    assert sim["pol"] == "TE" and len(sim["monitors"]) == 3 and len(sim["monitorsZ"]) == 2


def test_short_grating_power_balance_oracle():
    sim, bd = coupler.gratingCouplerTE_sim(dict(nPer=6, lambdas=[1.53, 1.55, 1.57]))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r = coupler.coupler_budget(oracle.fdtd2D(sim), bd)
    assert r["converged"]
    assert np.max(np.abs(r["balance"])) < 1e-3
    assert np.min(r["Pup"]) > 0 and np.min(r["Pdown"]) > 0 and np.min(r["R"]) > 0


def test_apodized_and_sidewall_geometry():
    per = np.linspace(0.6, 0.64, 5)
    ff = np.linspace(0.8, 0.5, 5)
    boxes, length = coupler._grating_boxes(coupler._params(dict(nPer=5, period=per, ff=ff)))
    assert abs(length - per.sum()) < 1e-12 and len(boxes) == 5
    # groove k starts at the end of tooth k (the unetched fraction comes first)
    assert abs(boxes[0][0] - (4.0 + ff[0] * per[0])) < 1e-12
    sw, _ = coupler._grating_boxes(coupler._params(dict(nPer=2, sidewall=80)))
    widths = [b[1] - b[0] for b in sw[: len(sw) // 2]]
    assert all(w2 < w1 for w1, w2 in zip(widths, widths[1:]))   # narrowing with depth


def test_best_fiber_coupling_finds_the_matching_fiber():
    """A field that is a tilted Gaussian at 9 deg centred at 10.3 um: the scan
    (bestFiberCoupling.m:1-8 interface) finds that fiber, eta = Pup there."""
    x = np.arange(0, 20.0 + 1e-9, 0.02)
    lam = np.array([1.53, 1.55, 1.57])
    th, w0, xc = np.deg2rad(9.0), 5.2, 10.3
    E = np.stack([np.exp(-((x - xc) * np.cos(th) / w0) ** 2) * np.exp(1j * 2 * np.pi / l * np.sin(th) * (x - xc))
                  for l in lam], axis=1)
    res = dict(xUp=x, EyUp=E, lambdas=lam, nClad=1.0, Pup=np.array([0.5, 0.6, 0.55]), grating=(4.0, 16.0),
               params=dict(lambda0=1.55))
    b = coupler.bestFiberCoupling(res, np.arange(5, 15.01, 0.5), w0)
    assert b["theta"] == 9.0 and abs(b["x0"] - 10.3) < 1e-9
    assert abs(b["eta"] - 0.6) < 1e-9 and abs(b["Pup"] - 0.6) < 1e-12
    assert b["spectrum"].shape == (3,) and b["band1dB"][0] <= 1.55 <= b["band1dB"][1]


def test_apodized_grating_meets_the_bragg_condition():
    per, ff = coupler.apodizedGrating(0.875, 0.435, 15, 25, 1.014)
    assert per.shape == (25,) and np.allclose(ff, np.linspace(0.875, 0.435, 25))
    q = coupler._params(None)
    nf = coupler._slab_te0(0.22, q)
    ne = coupler._slab_te0(0.22 - 0.07, q)
    assert 2.7 < nf < 2.95 and ne < nf                  # TE0 of 220 nm / 150 nm Si in air-clad SOI
    neff = ff * nf + (1 - ff) * ne
    np.testing.assert_allclose(per * (neff - np.sin(np.deg2rad(15))), 1.014 * 1.55, rtol=1e-12)
    assert np.all(np.diff(per) > 0)                     # weaker grating toward the end: longer periods
