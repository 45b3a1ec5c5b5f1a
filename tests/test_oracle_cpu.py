"""The C restatement of the oracle agrees with the numpy FP64 restatement
(CPU only), so either can serve as the checker."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def co():
    from coracle import COracle
    return COracle(64)


def test_c_channelise_matches_numpy(co, O):
    rng = np.random.default_rng(0)
    L = O.Layout(nave=2, muoslowfreq=384.0)
    p0 = rng.integers(0, 256, 12500 * 2 * 6, dtype=np.uint8)
    p1 = rng.integers(0, 256, 12500 * 2 * 6, dtype=np.uint8)
    a = co.channelise(p0, p1, L)
    b = O.channelise(p0, p1, L)
    assert np.max(np.abs(a - b) / np.abs(b)) < 1e-9


def test_c_chain_matches_numpy(co, O):
    rng = np.random.default_rng(1)
    rows, nch = 700, 64
    fb = rng.chisquare(20, (rows, nch)) * rng.uniform(1, 5, nch)
    bp_c = co.bandpass(fb)
    bp_n = O.subtract_bp_cal(fb)
    assert np.max(np.abs(bp_c - bp_n)) < 1e-9
    off, _ = O.delay_table(np.linspace(0, 40, 9).astype(np.float32), 384.0, 0.25, 0.001, nch)
    nt = rows - int(off.max())
    dd_c = co.dedisperse_cm(co.transpose(bp_c), off, nt)
    dd_n = O.dedisperse(bp_n, off, nt)
    assert np.max(np.abs(dd_c - dd_n)) < 1e-9
    s_c = co.calcstats_dm(dd_c)
    s_n = O.calcstats_dm(dd_n)
    for k in ("ave", "sigma", "peak", "frb", "argmax"):
        assert np.allclose(s_c[k], s_n[k], rtol=1e-6, atol=0), k
    a_c, g_c = co.dedisperse_sigma_cm(co.transpose(bp_c), off[:2], nt)
    a_n, g_n = O.dedisperse_sigma(bp_n, off[:2], nt)
    assert np.max(np.abs(a_c - a_n)) < 1e-9 and np.max(np.abs(g_c - g_n) / g_n) < 1e-9
    cs_c = co.chan_stats_cm(co.transpose(bp_c), 200, 3)
    cs_n = O.calcstats_chan(bp_n, 200, 3)
    for x, y in zip(cs_c, cs_n):
        assert np.allclose(x, y, rtol=1e-6, atol=1e-9)
