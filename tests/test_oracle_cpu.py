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


def _loop_subtract_bp_full(fb):
    """Statement-by-statement transcription of subtractbp (PIPE:1372-1424) in
    FP64 loops, checking the vectorised oracle on a small case."""
    x = np.array(fb, np.float64)
    nt, nch = x.shape
    for c in range(nch):
        ave = sum(x[j, c] for j in range(nt)) / nch  # PIPE:1380, divides by CNCHANOUT
        s = s2 = 0.0
        for j in range(nt):
            s2 += (x[j, c] - ave) ** 2
            s += x[j, c] - ave
        sig = (s2 - s * s / nt) / (nt - 1)
        hi, lo = ave + 3.0 * sig, ave - 3.0 * sig
        a, i = 0.0, 0
        for j in range(nt):
            if lo < x[j, c] < hi:
                a += x[j, c]
                i += 1
        m = a / i if i else float("nan")
        x[:, c] -= m
    return x


def _loop_subtract_zero(fb):
    """Transcription of subtractZERO (PIPE:1478-1515) in FP64 loops."""
    x = np.array(fb, np.float64)
    nt, nch = x.shape
    for t in range(nt):
        ave = sum(x[t]) / nch
        s = s2 = 0.0
        for j in range(nch):
            s2 += (x[t, j] - ave) ** 2
            s += x[t, j] - ave
        sig = (s2 - s * s / nch) / (nch - 1)
        hi, lo = ave + 3.0 * sig, ave - 3.0 * sig
        a, i = 0.0, 0
        for j in range(nch):
            if lo < x[t, j] < hi:
                a += x[t, j]
                i += 1
        x[t] -= a / max(i, 1)
    return x


def test_rfi_modes_oracle_matches_loops(O):
    rng = np.random.default_rng(5)
    nt, nch = 60, 9
    fb = rng.standard_normal((nt, nch)) * 0.2
    fb[:, 2] = fb[:, 2] * 50 + 40.0  # variance 100: the window about sum/nch = 267 keeps every row
    fb[:, 3] += 40.0        # variance 0.04 about 267: empty window, NaN (the sum/nch quirk)
    fb[7, 4] = 9.0          # clipped outlier
    fb[:, 6] = 3.0          # constant channel: empty clip, NaN (0/0) as the reference
    fb[11, :] = 1.5         # constant row: zero-DM count floor
    a = O.subtract_bp_full(fb)
    b = _loop_subtract_bp_full(fb)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    assert np.isnan(a[:, [3, 6]]).all() and not np.isnan(a[:, [0, 1, 2, 4, 5, 7, 8]]).any()
    assert np.allclose(a, b, rtol=0, atol=1e-12, equal_nan=True)
    assert abs(a[:, 2].mean()) < 1e-12  # all rows kept: the plain mean is subtracted
    z = O.subtract_zero(fb)
    assert np.allclose(z, _loop_subtract_zero(fb), rtol=0, atol=1e-12)
    assert np.array_equal(z[11], fb[11])  # sig 0: nothing inside the open interval, mean 0 subtracted
