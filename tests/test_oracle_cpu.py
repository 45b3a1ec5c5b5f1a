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


def _frames_np(duration, seed=0, rfi=None):
    from vlite_frb_b200 import synth
    spec = synth.StreamSpec(duration=duration, seed=seed, rfi=rfi)
    return synth.make_vdif(spec).numpy().reshape(-1, 2, 5032).copy()


def test_row_flags_known_answer(vf, O):
    """Pair flags from the reader restatement, pinned by hand: the invalid bit
    of either pol flags its pair (1); a missing pair becomes zero fill (2) and
    the frame that revealed the gap is used one pair later with its own bit."""
    fr = _frames_np(0.02)                      # 512 pairs, frames 0..511
    fr[7, 1, 3] |= 0x80                        # pol 1 of pair 7: invalid bit
    fr[30, 0, 3] |= 0x80                       # pol 0 of pair 30
    fr = np.delete(fr, 20, axis=0)             # pair 20 missing: frame 21 reveals the gap
    fr[20, 0, 3] |= 0x80                       # ... and frame 21 (now at index 20) is invalid on pol 0
    r = O.RefPairReader(fr.reshape(-1))
    assert r.initframe01() == 0
    while not r.readtwoframe():
        pass
    pf = np.array(r.pair_flags)
    want = np.zeros(512, np.uint8)
    want[7] = 1
    want[20] = 2          # the fill pair
    want[21] = 1          # frame 21, invalid, used after the fill
    want[30] = 1
    assert len(pf) == 512 and np.array_equal(pf, want)  # 511 pairs read + the fill pair
    L = O.Layout(nave=1, muoslowfreq=384.0)    # S = 12500 bytes = 2.5 pairs per row
    rf = O.row_flags(pf, L, 200)
    # pair 7 (bytes 35000-39999) straddles rows 2 and 3; pairs 20-21 lie in
    # row 8, pair 30 in row 12
    assert list(np.nonzero(rf)[0]) == [2, 3, 8, 12]
    assert rf[8] == 3 and rf[2] == rf[3] == rf[12] == 1


def test_block_rows_map(O):
    L = O.Layout(nave=2, muoslowfreq=384.0, maxtime=0.8)   # MAXNT 4096, NBUNDLE 32
    md = 100                                               # first = 96
    b1 = O.block_rows(L, md, 1)
    assert b1[0] == L.maxnt - md and b1[95] == L.maxnt - md + 95
    assert b1[96] == L.maxnt and b1[-1] == 2 * L.maxnt - 96 - 1
    b2 = O.block_rows(L, md, 2)
    assert b2[96] == b1[-1] + 1 and b2[0] == b1[-1] + 1 - md


def test_chan_sk_gaussian_expectation(O):
    """SK of Gamma(nsum) power (Gaussian-noise detection statistics) is 1 in
    expectation; a steady tone (constant power) drives it to 0, a burst far
    above 1."""
    rng = np.random.default_rng(3)
    nsum, m, nblk = 8, 1024, 6
    x = rng.gamma(nsum, 1.0 / nsum, (m * nblk, 64)) * 50.0
    x[:, 10] = 50.0                                   # constant: S2 = S1^2/M
    x[5:9, 20] *= 40.0                                # burst in block 0
    sk = O.chan_sk(x, m, nblk, nsum)
    ok = np.ones(64, bool)
    ok[[10, 20]] = False
    assert abs(sk[:, ok].mean() - 1.0) < 0.01
    assert np.allclose(sk[:, 10], 0.0, atol=1e-9)
    assert sk[0, 20] > 5 and abs(sk[1, 20] - 1) < 0.2
