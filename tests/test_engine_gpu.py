"""End-to-end parity of the plan/stream engine against the oracle chain.

Tolerances: dedispersed series max |gpu - oracle| <= 5e-5 * rms(oracle)
(FP32 channeliser + FP32 sums against FP64); per-DM ave/sigma relative
<= 1e-4, peak relative <= 1e-3, FRB flags identical; per-channel stats
relative <= 1e-4.  Streaming results are bit-identical however the input is
split and whether a stream runs alone or among others.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vdif(duration, seed=0, pulses=(), **kw):
    from vlite_frb_b200 import synth
    ps = [synth.Pulse(*p) for p in pulses]
    return synth.make_vdif(synth.StreamSpec(duration=duration, seed=seed, pulses=ps, **kw)).numpy()


@pytest.fixture(scope="module")
def co():
    from coracle import COracle
    return COracle(64)


def _oracle_rows(O, co, buf, L, mode="pipe"):
    """FB rows of every bundle the reference would process (raw, FP64)."""
    _, bundles, _ = O.read_bundles(buf, L, mode=mode)
    if not bundles:
        return np.zeros((0, L.nchanout))
    p0 = np.concatenate([b[0] for b in bundles])
    p1 = np.concatenate([b[1] for b in bundles])
    return co.channelise(p0, p1, L)


def _close(got, ref, tol, what):
    rms = np.sqrt(np.mean(ref ** 2))
    e = np.max(np.abs(got - ref)) / rms
    print(f"{what}: max err / rms = {e:.2e}")
    assert e <= tol, (what, e)


def test_block_mode_pipe_chain(vf, O, co):
    """PIPE semantics: MAXTIME blocks, leftover carry, block-relative BP,
    in-tree dedisperse + calcstats (PIPE:556-708)."""
    nave, maxtime = 2, 0.8
    dms = np.arange(0, 10.5, 0.5, dtype=np.float32)
    buf = _vdif(2.0, seed=11, pulses=[(0.7, 6.0, 2.0, 40.0)])
    plan = vf.Plan(dms, nave=nave, muoslowfreq=384.0, maxtime=maxtime, mode=vf.MODE_BLOCK,
                   outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_FB, fb_block=1)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, muoslowfreq=384.0, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    assert md == plan.max_delay
    rows = _oracle_rows(O, co, buf, L)
    blocks = list(O.run_blocks(rows, L, md))
    assert len(res) == len(blocks) == 2
    assert [r["row0"] for r in res] == [0, L.maxnt - md]  # absolute row of each block's row 0
    for r, (q, fb) in zip(res, blocks):
        bp = co.bandpass(fb)
        dd = co.dedisperse_cm(co.transpose(bp), off, L.maxnt - md)
        _close(r["dd"], dd, 5e-5, f"block {q} dedispersed")
        st = O.calcstats_dm(dd)
        assert np.array_equal(r["frb"], st["frb"])
        assert np.allclose(r["sigma"], st["sigma"], rtol=1e-4)
        assert np.allclose(r["peak"], st["peak"], rtol=1e-3)
        if q == 1:
            assert r["fb"] is not None
            _close(r["fb"], bp, 5e-5, "block 1 bandpassed FB")
        else:
            assert r["fb"] is None


def test_block_mode_rfi_modes(vf, O, co):
    """The reference's dead-code options as plan parameters: whole-block
    subtractbp (PIPE:1372) in place of subtractbpCAL, then subtractZERO
    (PIPE:1478), before dedispersion and calcstats."""
    nave, maxtime = 2, 0.8
    dms = np.arange(0, 10.5, 0.5, dtype=np.float32)
    buf = _vdif(1.2, seed=12, pulses=[(0.5, 6.0, 2.0, 40.0)])
    plan = vf.Plan(dms, nave=nave, muoslowfreq=384.0, maxtime=maxtime, mode=vf.MODE_BLOCK,
                   outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_FB, bp_mode=vf.BP_FULL, zero_dm=1)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, muoslowfreq=384.0, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    rows = _oracle_rows(O, co, buf, L)
    blocks = list(O.run_blocks(rows, L, md))
    assert len(res) == len(blocks) >= 1
    for r, (q, fb) in zip(res, blocks):
        x = O.subtract_zero(O.subtract_bp_full(fb))
        assert not np.isnan(x).any()
        _close(r["fb"], x, 5e-5, f"block {q} whole-block BP + zero-DM FB")
        dd = co.dedisperse_cm(co.transpose(x), off, L.maxnt - md)
        _close(r["dd"], dd, 5e-5, f"block {q} dedispersed")
        st = O.calcstats_dm(dd)
        # zero-DM removal leaves the DM-0 series at rounding level (its sigma
        # ~1e-14 in FP64, ~1e-6 in FP32): statistics of such trials are noise
        ok = st["sigma"] > 1e-6 * st["sigma"].max()
        assert not ok[0] and ok[1:].all()
        assert np.array_equal(r["frb"][ok], st["frb"][ok])
        assert np.allclose(r["sigma"][ok], st["sigma"][ok], rtol=1e-4)


def test_block_mode_ts_chain(vf, O, co):
    """TS semantics: 3840 channels, DM {0, 119.3}, dedisperseSTATS sigma."""
    dms = np.array([0.0, 119.3], np.float32)
    nave, maxtime = 4, 1.5  # MAXTIME must exceed the 1.0 s DM-119.3 sweep (TS:442)
    buf = _vdif(3.1, seed=5)
    plan = vf.Plan(dms, nave=nave, nchanout_fixed=3840, maxtime=maxtime, mode=vf.MODE_BLOCK,
                   reader=vf.READER_TS, outputs=vf.OUT_DEDISP | vf.OUT_SIGMA)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, nchanout_fixed=3840, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    rows = _oracle_rows(O, co, buf, L, mode="ts")
    blocks = list(O.run_blocks(rows, L, md))
    assert len(res) == len(blocks) >= 2
    for r, (q, fb) in zip(res, blocks):
        bp = co.bandpass(fb)
        a, s = co.dedisperse_sigma_cm(co.transpose(bp), off, L.maxnt - md)
        _close(r["dd"], a, 5e-5, f"TS block {q} mean")
        assert np.max(np.abs(r["dd_sigma"] - s) / s) <= 1e-4


def test_block_mode_stats_chain(vf, O, co):
    """STATS semantics: no overlap, per-channel stats per TIMESTATS block."""
    nave, maxtime, tstat = 4, 0.5, 0.1
    buf = _vdif(1.3, seed=9)
    plan = vf.Plan(None, nave=nave, maxtime=maxtime, timestats=tstat, mode=vf.MODE_BLOCK,
                   outputs=vf.OUT_CHANSTATS)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, maxtime=maxtime)
    rows = _oracle_rows(O, co, buf, L)
    ncol = int(tstat / L.tchan)
    nblk = int(np.float32(maxtime) / np.float32(tstat))
    blocks = list(O.run_stats_blocks(rows, L))
    assert len(res) == len(blocks) == 2
    assert [r["row0"] for r in res] == [0, L.maxnt]  # no overlap: blocks follow each other
    for r, (q, fb) in zip(res, blocks):
        bp = co.bandpass(fb)
        a, s, o = O.calcstats_chan(bp, ncol, nblk)
        assert np.max(np.abs(r["chan_ave"] - a)) <= 1e-4 * np.abs(bp).max()
        assert np.max(np.abs(r["chan_sig"] - s) / s) <= 1e-4
        assert np.array_equal(r["chan_outlier"], o)


def _stream_run(vf, dms, bufs, storage=0, chunk=0.25, splits=None, order=None, outputs=None, **kw):
    outputs = outputs if outputs is not None else vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_CANDS
    plan = vf.Plan(dms, nave=2, muoslowfreq=384.0, mode=vf.MODE_STREAM, storage=storage, chunk_seconds=chunk,
                   nstreams=len(bufs), outputs=outputs, **kw)
    rng = np.random.default_rng(0)
    pos = [0] * len(bufs)
    live = list(range(len(bufs)))
    while live:
        s = live[rng.integers(len(live))] if order is None else live[0]
        n = splits(rng) if splits else len(bufs[s])
        plan.push(s, bufs[s][pos[s]:pos[s] + n])
        pos[s] += n
        if pos[s] >= len(bufs[s]):
            plan.push(s, None)
            live.remove(s)
    res = plan.drain()
    per = {}
    for r in res:
        per.setdefault(r["stream"], []).append(r)
    return plan, per


def _rfi_vdif(duration, seed, drop=()):
    """RFI-heavy stream (tones, bursts, 10% invalid-flagged frames) with the
    listed frame pairs removed (gaps the reader zero-fills)."""
    from vlite_frb_b200 import synth
    fr = synth.make_vdif(synth.StreamSpec(duration=duration, seed=seed, rfi=synth.Rfi())).numpy()
    fr = fr.reshape(-1, 2, 5032)
    return np.ascontiguousarray(np.delete(fr, list(drop), axis=0)).reshape(-1)


def _pair_flags(O, buf, L, mode="pipe"):
    _, _, r = O.read_bundles(buf, L, mode=mode)
    return r.pair_flags


def test_stats_rfi_sk_and_row_flags(vf, O, co):
    """RFI-heavy STATS block mode: spectral kurtosis of the raw block per
    (channel, TIMESTATS block) within 1e-3 of the FP64 oracle; row flags
    (invalid bit, zero fill) identical to the oracle's."""
    nave, maxtime, tstat = 4, 0.5, 0.1
    buf = _rfi_vdif(1.3, seed=7, drop=(9000, 9001, 20000))
    plan = vf.Plan(None, nave=nave, maxtime=maxtime, timestats=tstat, mode=vf.MODE_BLOCK,
                   outputs=vf.OUT_CHANSTATS | vf.OUT_FLAGS)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, maxtime=maxtime)
    rows = _oracle_rows(O, co, buf, L)
    ncol = int(tstat / L.tchan)
    nblk = int(np.float32(maxtime) / np.float32(tstat))
    blocks = list(O.run_stats_blocks(rows, L))
    flags = O.row_flags(_pair_flags(O, buf, L), L, len(blocks) * L.maxnt)
    assert len(res) == len(blocks) == 2
    assert flags.any() and (flags & 2).any()
    for r, (q, fb) in zip(res, blocks):
        sk = O.chan_sk(fb, ncol, nblk, 2 * nave)
        e = np.max(np.abs(r["chan_sk"] - sk))
        print(f"block {q}: SK max abs err {e:.2e}, SK range {sk.min():.3f} .. {sk.max():.3f}")
        assert e <= 1e-3
        assert np.array_equal(r["row_flags"], flags[q * L.maxnt:(q + 1) * L.maxnt])


def test_pipe_block_and_stream_row_flags(vf, O, co):
    """Row flags in parity-block mode with the overlap carry (each block row
    maps to its absolute row) and in stream mode (rows [row0, row0 + nt) of
    each chunk), identical to the oracle's."""
    nave, maxtime = 2, 0.8
    dms = np.arange(0, 10.5, 0.5, dtype=np.float32)
    buf = _rfi_vdif(2.0, seed=8, drop=(15000, 30001))
    plan = vf.Plan(dms, nave=nave, muoslowfreq=384.0, maxtime=maxtime, mode=vf.MODE_BLOCK,
                   outputs=vf.OUT_DEDISP | vf.OUT_FLAGS)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    L = O.Layout(nave=nave, muoslowfreq=384.0, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    pf = _pair_flags(O, buf, L)
    flags = O.row_flags(pf, L, len(pf) * 5000 // (nave * 12500))
    assert len(res) == 2
    for q, r in enumerate(res):
        assert np.array_equal(r["row_flags"], flags[O.block_rows(L, md, q)])
    plan, per = _stream_run(vf, dms, [buf], outputs=vf.OUT_DEDISP | vf.OUT_FLAGS)
    got = np.concatenate([r["row_flags"] for r in per[0]])
    assert per[0][0]["row0"] == 0 and got.size > L.maxnt
    assert np.array_equal(got, flags[:got.size]) and (got & 2).any() and (got & 1).any()


def test_stream_mode_matches_oracle(vf, O, co):
    """Streaming: absolute 128-row BP windows, every sample dedispersed once."""
    dms = np.arange(0, 8.0, 0.5, dtype=np.float32)
    buf = _vdif(1.5, seed=21, pulses=[(0.6, 4.0, 2.0, 30.0)])
    plan, per = _stream_run(vf, dms, [buf])
    # stream mode uses every complete row (no bundle granularity): one-row bundles
    L = O.Layout(nave=2, muoslowfreq=384.0, nbundle=1)
    rows = _oracle_rows(O, co, buf, L)
    nbp = (rows.shape[0] // 128) * 128
    bp = co.bandpass(rows[:nbp])
    off, _ = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    md = int(off.max())
    dd = co.dedisperse_cm(co.transpose(bp), off, nbp - md)
    got = np.concatenate([r["dd"] for r in per[0]], axis=1)
    n = min(got.shape[1], dd.shape[1])
    assert n >= dd.shape[1] - 128
    _close(got[:, :n], dd[:, :n], 5e-5, "stream dedispersed")
    assert [r["row0"] for r in per[0]] == sorted(r["row0"] for r in per[0])


def test_stream_split_invariance_and_isolation(vf):
    """Results do not depend on how the input is cut, nor on other streams."""
    dms = np.arange(0, 6.0, 0.5, dtype=np.float32)
    bufs = [_vdif(0.9, seed=100 + i) for i in range(3)]
    _, alone = _stream_run(vf, dms, [bufs[1]])
    _, mixed = _stream_run(vf, dms, bufs, splits=lambda rng: int(rng.integers(1, 400000)))
    a = np.concatenate([r["dd"] for r in alone[0]], axis=1)
    m = np.concatenate([r["dd"] for r in mixed[1]], axis=1)
    assert a.shape == m.shape and np.array_equal(a, m)
    for s in range(3):
        assert all(r["device_errors"] == 0 for r in mixed[s])


def test_streams_open_close_and_admission(vf):
    """Serving: streams are opened while others run and closed when done;
    admission refuses a stream whose device memory does not fit the budget
    until another has closed and freed its memory; every stream's series
    equal its series run alone, bit for bit."""
    dms = np.arange(0, 6.0, 0.5, dtype=np.float32)
    bufs = [_vdif(0.9, seed=200 + i) for i in range(3)]
    alone = [np.concatenate([r["dd"] for r in _stream_run(vf, dms, [b])[1][0]], axis=1) for b in bufs]
    kw = dict(nave=2, muoslowfreq=384.0, mode=vf.MODE_STREAM, chunk_seconds=0.25, outputs=vf.OUT_DEDISP)
    probe = vf.Plan(dms, nstreams=1, **kw)
    one = probe.device_bytes
    probe.close()
    plan = vf.Plan(dms, nstreams=0, device_bytes=int(2.5 * one), **kw)
    assert plan.device_bytes == 0
    a, b = plan.open_stream(), plan.open_stream()
    assert (a, b) == (0, 1) and plan.device_bytes == 2 * one
    assert plan.open_stream() is None  # a third does not fit beside two
    got = {}

    def take(r):
        if r is not None:
            got.setdefault(r["stream"], []).append(r["dd"])

    half = len(bufs[0]) // 2 + 777  # cut inside a frame
    plan.push(a, bufs[0][:half])
    plan.push(b, bufs[1][:half])
    plan.push(a, bufs[0][half:])
    while not plan.close_stream(a):  # ends stream a; frees it once its results are polled
        take(plan.poll(wait=True))
    assert plan.device_bytes == one
    with pytest.raises(vf.VfrbError):
        plan.push(a, bufs[0][:10064])
    c = plan.open_stream()
    assert c == 2
    plan.push(c, bufs[2])
    plan.push(b, bufs[1][half:])
    plan.push(b, None)
    plan.push(c, None)
    for r in plan.drain():
        take(r)
    for i, sid in enumerate((a, b, c)):
        assert np.array_equal(np.concatenate(got[sid], axis=1), alone[i]), sid
    assert plan.close_stream(b) and plan.close_stream(c) and plan.device_bytes == 0
    plan.close()


def test_garbage_input_fails_cleanly(vf):
    """Bytes that are not VDIF end the stream at the reader (the reference's
    initframe01 failure, status 2) with no result and nothing launched on
    bad data; the plan stays usable for the next stream."""
    dms = np.arange(0, 6.0, 0.5, dtype=np.float32)
    plan = vf.Plan(dms, nave=2, muoslowfreq=384.0, mode=vf.MODE_STREAM, chunk_seconds=0.25, nstreams=1,
                   outputs=vf.OUT_DEDISP)
    garbage = np.random.default_rng(9).integers(0, 256, 3_000_000, dtype=np.uint8)
    for data in (garbage, None):
        try:
            plan.push(0, data)
        except vf.VfrbError as e:
            assert e.status == 2
            break
    assert plan.drain() == []
    sid = plan.open_stream()
    plan.push(sid, _vdif(0.9, seed=5))
    plan.push(sid, None)
    res = plan.drain()
    assert res and all(r["stream"] == sid and r["device_errors"] == 0 for r in res)
    plan.close()


def test_stream_fp16_form(vf):
    """FP16 storage: series within 3e-3 rms of FP32, identical candidates."""
    dms = np.arange(0, 12.0, 0.25, dtype=np.float32)
    buf = _vdif(1.5, seed=31, pulses=[(0.5, 5.0, 2.0, 40.0)])
    _, f32 = _stream_run(vf, dms, [buf], storage=0)
    _, f16 = _stream_run(vf, dms, [buf], storage=1)
    a = np.concatenate([r["dd"] for r in f32[0]], axis=1)
    b = np.concatenate([r["dd"] for r in f16[0]], axis=1)
    e = np.max(np.abs(a - b)) / np.sqrt(np.mean(a ** 2))
    print("fp16 vs fp32 err/rms", e)
    assert e <= 3e-3
    ca = [(c["dm_index"], c["t"]) for r in f32[0] for c in r["cands"]]
    cb = [(c["dm_index"], c["t"]) for r in f16[0] for c in r["cands"]]
    assert ca == cb and len(ca) >= 1
    sa = [c["snr"] for r in f32[0] for c in r["cands"]]
    sb = [c["snr"] for r in f16[0] for c in r["cands"]]
    assert np.max(np.abs(np.array(sa) - np.array(sb)) / np.array(sa)) <= 0.01


def test_stream_boxcar_candidates(vf, O, co):
    """Candidates with the boxcar width search (widths 1..32): per chunk they
    equal the oracle's rule applied to the same dedispersed series and
    statistics; the wide pulse is found at a width > 1 near its true DM, and
    against the FP64 oracle chain the candidate trials and SNRs agree."""
    dms = np.arange(0, 12.0, 0.25, dtype=np.float32)
    # chunks are 1280 rows (0.25 s): both pulses sit inside a chunk
    buf = _vdif(1.5, seed=41, pulses=[(0.62, 5.0, 8.0, 40.0), (1.05, 9.0, 1.0, 40.0)])
    plan, per = _stream_run(vf, dms, [buf], boxcar_max=32, cand_snr=8.0)
    found = []
    for r in per[0]:
        best, start, width = O.boxcar_best(r["dd"], r["ave"], r["sigma"], 32)
        assert np.array_equal(r["box_width"], width) and np.array_equal(r["box_start"], start)
        assert np.allclose(r["box_snr"], best, rtol=1e-5)
        want = O.candidates(best.astype(np.float32), start, width, dms, 8.0, r["row0"])
        got = [(c["dm_index"], c["t"], c["width"]) for c in r["cands"]]
        assert got == [(d, t, w) for d, t, w, _, _ in want]
        found += r["cands"]
    wide = [c for c in found if abs(c["dm"] - 5.0) <= 0.5]
    assert wide and max(c["width"] for c in wide) > 1
    assert any(abs(c["dm"] - 9.0) <= 0.5 for c in found)
    # the full FP64 oracle chain (stream semantics) gives the same candidate trials
    L = O.Layout(nave=2, muoslowfreq=384.0, nbundle=1)
    rows = _oracle_rows(O, co, buf, L)
    nbp = (rows.shape[0] // 128) * 128
    off, _ = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    ref = co.dedisperse_cm(co.transpose(co.bandpass(rows[:nbp])), off, nbp - int(off.max()))
    for r in per[0]:
        seg = ref[:, r["row0"]:r["row0"] + r["nt"]]
        if seg.shape[1] < r["nt"]:
            continue
        st = O.calcstats_dm(seg)
        best, start, width = O.boxcar_best(seg, st["ave"], st["sigma"], 32)
        want = O.candidates(best, start, width, dms, 8.0, r["row0"])
        # FP32 vs FP64 series: a near-tie between neighbouring trials may move a candidate by one trial
        assert len(r["cands"]) == len(want)
        for c, w in zip(r["cands"], want):
            assert abs(c["dm_index"] - w[0]) <= 1
            assert abs(c["snr"] - w[3]) <= 0.01 * w[3]


def test_stream_mode_chan_stats_sk_and_flags(vf, O, co):
    """Stream mode with VFRB_OUT_CHANSTATS: one result per absolute TIMESTATS
    block (rows [k*ncol, (k+1)*ncol)) holding calcstats per channel
    (STATS:910-946) of the bandpassed rows -- ave and variance within 1e-4 of
    the FP64 oracle (relative to the channel's level), outlier counts exact --
    the spectral kurtosis of the raw rows within 1e-3, and the block's row
    flags identical to the oracle's; RFI-heavy input with gaps.  The same
    stream among two others, pushed in random splits, gives identical
    results."""
    nave, tstat = 2, 0.25
    buf = _rfi_vdif(2.6, seed=9, drop=(7000, 7001, 40000))
    others = [_rfi_vdif(1.7, seed=10 + i) for i in range(2)]
    outputs = vf.OUT_CHANSTATS | vf.OUT_FLAGS
    _, alone = _stream_run(vf, None, [buf], outputs=outputs, timestats=tstat)
    _, mixed = _stream_run(vf, None, [others[0], buf, others[1]], outputs=outputs, timestats=tstat,
                           splits=lambda rng: int(rng.integers(1, 300000)))
    L = O.Layout(nave=nave, muoslowfreq=384.0, nbundle=1)
    ncol = int(tstat / L.tchan)
    rows = _oracle_rows(O, co, buf, L)
    nbp = rows.shape[0] // 128 * 128
    bp = co.bandpass(rows[:nbp])
    flags = O.row_flags(_pair_flags(O, buf, L), L, rows.shape[0])
    nblk = nbp // ncol
    res = [r for r in alone[0] if r["nstatblks"] == 1]
    assert len(res) == nblk >= 3 and [r["row0"] for r in res] == [k * ncol for k in range(nblk)]
    for k, r in enumerate(res):
        ave, sig, outl = O.calcstats_chan(bp[k * ncol:(k + 1) * ncol], ncol, 1)
        scale = np.abs(ave[0]) + np.sqrt(np.abs(sig[0])) + 1e-30
        assert np.max(np.abs(r["chan_ave"][0] - ave[0]) / scale) <= 1e-4
        assert np.max(np.abs(r["chan_sig"][0] - sig[0]) / (np.abs(sig[0]) + 1e-30)) <= 1e-4
        assert np.array_equal(r["chan_outlier"][0], outl[0])
        sk = O.chan_sk(rows[k * ncol:(k + 1) * ncol], ncol, 1, 2 * nave)
        e = np.max(np.abs(r["chan_sk"][0] - sk[0]))
        print(f"stream stats block {k}: SK max abs err {e:.2e}")
        assert e <= 1e-3
        assert np.array_equal(r["row_flags"], flags[k * ncol:(k + 1) * ncol])
    assert any((r["row_flags"] & 2).any() for r in res) and any((r["row_flags"] & 1).any() for r in res)
    mres = [r for r in mixed[1] if r["nstatblks"] == 1]
    assert len(mres) == len(res)
    for a, b in zip(res, mres):
        for key in ("chan_ave", "chan_sig", "chan_outlier", "chan_sk", "row_flags"):
            assert np.array_equal(a[key], b[key]), key


def test_stream_device_input_matches_host(vf):
    """Frames pushed from device memory (copied device to device, headers to
    the host for the reader) give results identical to the same bytes pushed
    from host memory, with splits that cut frames anywhere."""
    import torch
    dms = np.arange(0, 6.0, 0.5, dtype=np.float32)
    buf = _vdif(1.2, seed=31, pulses=[(0.5, 3.0, 2.0, 30.0)])
    dev = torch.from_numpy(buf).cuda()
    cuts = [0, 5031, 77777, 350001, 1000000, 2500003, len(buf)]
    out = []
    for src in (buf, dev):
        plan = vf.Plan(dms, nave=2, muoslowfreq=384.0, mode=vf.MODE_STREAM, chunk_seconds=0.25,
                       outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_FLAGS)
        for a, b in zip(cuts[:-1], cuts[1:]):
            plan.push(0, src[a:b])
        plan.push(0, None)
        out.append(plan.drain())
        plan.close()
    assert len(out[0]) == len(out[1]) > 2
    for x, y in zip(*out):
        assert x["row0"] == y["row0"] and np.array_equal(x["dd"], y["dd"])
        assert np.array_equal(x["row_flags"], y["row_flags"]) and x["device_errors"] == y["device_errors"] == 0


def test_stream_device_input_ordered_after_producer(vf):
    """Device chunks pushed the moment the kernels that write them are queued
    (on PyTorch's default stream, no synchronisation) are read only after
    those kernels: results equal the same chunks pushed from pinned host
    copies, bit for bit, with cuts anywhere.  12 s of one stream in chunks of
    0.5-4 s (device batches of a quarter of the 1-s frame ring), statistics
    blocks, the zero-DM series and its sigma, row flags."""
    import torch
    from vlite_frb_b200 import synth
    rng = np.random.default_rng(3)
    fps, total, sched, pos = 25600, 12 * 25600, [], 0
    while pos < total:
        n = min(total - pos, int(rng.uniform(0.5, 4.0) * fps) // 5 * 5)
        sched.append((pos, n))
        pos += n
    cuts = [sorted(set([0, n * 10064] + [int(x) for x in rng.integers(1, n * 10064, 2)])) for _, n in sched]

    def run(pinned):
        plan = vf.Plan(np.zeros(1, np.float32), nave=4, mode=vf.MODE_STREAM, chunk_seconds=1.0, ring_seconds=1.0,
                       timestats=1.0, outputs=vf.OUT_CHANSTATS | vf.OUT_DEDISP | vf.OUT_SIGMA | vf.OUT_FLAGS)
        res = []
        for k, (p0, n) in enumerate(sched):
            spec = synth.StreamSpec(duration=n / fps, seed=900 + k, frame0=p0, block0=p0 * 5000 // 12500,
                                    rfi=synth.Rfi(seed=9))
            fr = synth.make_vdif(spec, device="cuda")
            if pinned:
                h = torch.empty(fr.numel(), dtype=torch.uint8, pin_memory=True)
                h.copy_(fr)
                fr = h
            for a, b in zip(cuts[k][:-1], cuts[k][1:]):
                plan.push(0, fr[a:b])
            while (r := plan.poll(wait=False)) is not None:
                res.append(r)
        plan.push(0, None)
        res += plan.drain()
        plan.close()
        return res

    dev, host = run(False), run(True)
    assert len(dev) == len(host) > 10
    for x, y in zip(dev, host):
        assert (x["row0"], x["nt"], x["nstatblks"]) == (y["row0"], y["nt"], y["nstatblks"])
        for key in ("dd", "dd_sigma", "chan_ave", "chan_sig", "chan_outlier", "chan_sk", "row_flags"):
            assert (x[key] is None and y[key] is None) or np.array_equal(x[key], y[key]), key


def test_plans_on_host_threads_equal_sequential(vf):
    """Several single-stream plans, each pushed and polled by its own host
    thread at the same time (a plan is driven by one thread; plans are
    independent), give per stream exactly the results of the same plans run
    one after another: series, statistics and candidates bit-identical."""
    import threading
    dms = np.linspace(0.0, 40.0, 128).astype(np.float32)
    bufs = [_vdif(3.0, seed=70 + i, pulses=[(1.0 + 0.2 * i, 10.0 + 8 * i, 2.0, 30.0)]) for i in range(4)]

    def serve(i, out):
        plan = vf.Plan(dms, nave=2, muoslowfreq=384.0, mode=vf.MODE_STREAM, chunk_seconds=0.25,
                       outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=7.0)
        rng = np.random.default_rng(i)
        res, pos = [], 0
        while pos < len(bufs[i]):
            n = int(rng.integers(200000, 2000000))
            plan.push(0, bufs[i][pos:pos + n])
            pos += n
            while (r := plan.poll(wait=False)) is not None:
                res.append(r)
        plan.push(0, None)
        res += plan.drain()
        plan.close()
        out[i] = res

    seq, par = {}, {}
    for i in range(len(bufs)):
        serve(i, seq)
    threads = [threading.Thread(target=serve, args=(i, par)) for i in range(len(bufs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i in range(len(bufs)):
        a, b = seq[i], par[i]
        assert len(a) == len(b) >= 4, i
        for x, y in zip(a, b):
            assert (x["seq"], x["row0"], x["nt"]) == (y["seq"], y["row0"], y["nt"])
            for key in ("dd", "ave", "sigma", "peak", "frb", "argmax"):
                assert np.array_equal(x[key], y[key]), (i, key)
            assert x["cands"] == y["cands"] and y["device_errors"] == 0


@pytest.mark.parametrize("storage", [0, 1])
def test_stream_batched_dedispersion_equals_per_stream(vf, storage):
    """batch_streams = 1: the chunks that become ready in several streams are
    dedispersed by shared launches (one grid slice per stream); every
    series, statistic and candidate is bit-identical to per-stream launches,
    and each stream's results keep their order."""
    dms = np.linspace(0.0, 40.0, 128).astype(np.float32)
    bufs = [_vdif(3.0, seed=60 + i, pulses=[(1.0 + 0.2 * i, 10.0 + 8 * i, 2.0, 30.0)]) for i in range(3)]
    split = lambda rng: int(rng.integers(200000, 2000000))  # noqa: E731
    out = []
    for batch in (0, 1):
        _, per = _stream_run(vf, dms, bufs, storage=storage, splits=split, batch_streams=batch, cand_snr=7.0)
        out.append(per)
    for s in range(3):
        a, b = out[0][s], out[1][s]
        assert len(a) == len(b) >= 4
        for x, y in zip(a, b):
            assert (x["seq"], x["row0"], x["nt"]) == (y["seq"], y["row0"], y["nt"])
            for key in ("dd", "ave", "sigma", "peak", "frb", "argmax"):
                assert np.array_equal(x[key], y[key]), (s, key)
            assert x["cands"] == y["cands"] and y["device_errors"] == 0
        assert [r["seq"] for r in b] == sorted(r["seq"] for r in b)
