"""RFI-heavy statistics and zero-DM time series at their stated scale --
64 streams x 30 s -- served through the stream loop.

Workload: 64 independent streams (seeds 500..563) of 30 s of 2-pol 8-bit
VLITE VDIF each, with 40 narrowband sinusoids (5-50 counts), 1% of 1-ms
blocks carrying broadband bursts at 8x the noise rms, and the VDIF invalid
bit on 10% of frames; the reference's default layout (MUOSLOWFREQ 360 ->
3908 channels), NAVE 4.  One plan in stream mode computes, per stream:
  * VFRB_OUT_CHANSTATS: per 1-s TIMESTATS block (2560 rows) the STATS
    tool's per-channel mean, variance and outlier count (STATS:910-946) and
    the spectral kurtosis of the raw power;
  * VFRB_OUT_DEDISP | VFRB_OUT_SIGMA with the single trial DM 0: the TS
    tool's zero-DM time series and its per-sample channel sigma
    (dedisperseSTATS, TS:1450-1481);
  * VFRB_OUT_FLAGS: per-row data flags.
Streams are admitted one by one with vfrb_stream_open and fed chunks of
U(0.5, 8) s in random stream order, generated on the GPU and pushed from
device memory (split at arbitrary bytes).

Checks: the row flags of every stream bit-exact against the oracle's
(computed from the frames' invalid bits); streams 0 and 63 in full against
the FP64 oracle (channel mean within 1e-4 of the channel's level, variance
within 1e-4 relative, outlier counts exact, SK within 1e-3, zero-DM series
within 5e-5 of its rms, sigma within 1e-4 relative); stream 31 run alone
in a plan of its own gives results identical to those in the mix.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSTREAMS, DUR, NAVE, TSTAT = 64, 30.0, 4, 1.0
FPS, PAIR = 25600, 2 * 5032
CHECK, ISOLATE = (0, 63), 31


def _chunks(rng):
    """Chunk lengths of one stream in frame pairs (multiples of 5 pairs, so
    every chunk starts on a 12500-sample block), totalling DUR seconds."""
    total = int(DUR * FPS)
    out, done = [], 0
    while done < total:
        n = min(total - done, int(rng.uniform(0.5, 8.0) * FPS) // 5 * 5)
        out.append(n)
        done += n
    return out


def _gen(synth, stream, k, pair0, npairs):
    spec = synth.StreamSpec(duration=npairs / FPS, seed=(500 + stream) * 1000 + k, frame0=pair0,
                            block0=pair0 * 5000 // 12500, rfi=synth.Rfi(seed=500 + stream))
    return synth.make_vdif(spec, device="cuda")


def _plan(vf):
    return vf.Plan(np.zeros(1, np.float32), nave=NAVE, mode=vf.MODE_STREAM, chunk_seconds=1.0, ring_seconds=1.0,
                   timestats=TSTAT, nstreams=0,
                   outputs=vf.OUT_CHANSTATS | vf.OUT_DEDISP | vf.OUT_SIGMA | vf.OUT_FLAGS)


def _feed(plan, sched, keep, flags, drain):
    """Push the chunks in `sched` order ((stream, chunk k, pair0, npairs));
    bytes of streams in `keep` are also copied to the host."""
    import torch
    from vlite_frb_b200 import synth
    ids = {}
    rng = np.random.default_rng(7)
    for s, k, p0, n in sched:
        if s not in ids:
            ids[s] = plan.open_stream()
            assert ids[s] is not None, "stream not admitted"
        fr = _gen(synth, s, k, p0, n)
        if flags is not None:
            inv = ((fr.view(-1, 2, 5032)[:, :, 3] >> 7) & 1).to(torch.uint8)
            flags.setdefault(s, []).append((inv[:, 0] | inv[:, 1]).cpu().numpy())
        if s in keep:
            keep[s].append(fr.cpu().numpy())
        cuts = sorted(set([0, fr.numel()] + [int(x) for x in rng.integers(1, fr.numel(), int(rng.integers(0, 3)))]))
        for a, b in zip(cuts[:-1], cuts[1:]):
            plan.push(ids[s], fr[a:b])
        drain()
    return ids


@pytest.fixture(scope="module")
def served(vf):
    rng = np.random.default_rng(12345)
    per = {s: _chunks(rng) for s in range(NSTREAMS)}
    # random interleaving of the streams' chunks, each stream's in order
    queue = {s: list(enumerate(per[s])) for s in range(NSTREAMS)}
    pos = {s: 0 for s in range(NSTREAMS)}
    sched = []
    while queue:
        s = list(queue)[int(rng.integers(len(queue)))]
        k, n = queue[s].pop(0)
        sched.append((s, k, pos[s], n))
        pos[s] += n
        if not queue[s]:
            del queue[s]
    plan = _plan(vf)
    res = {}

    def drain(wait=False):
        while True:
            r = plan.poll(wait=wait)
            if r is None:
                return
            res.setdefault(r["stream"], []).append(r)

    keep = {s: [] for s in CHECK}
    flags = {}
    ids = _feed(plan, sched, keep, flags, drain)
    for s in range(NSTREAMS):
        plan.push(ids[s], None)
    drain(wait=True)
    plan.close()
    by_stream = {s: res.get(ids[s], []) for s in range(NSTREAMS)}
    # stream ISOLATE alone
    alone = _plan(vf)
    res1 = []

    def drain1(wait=False):
        while True:
            r = alone.poll(wait=wait)
            if r is None:
                return
            res1.append(r)

    ids1 = _feed(alone, [x for x in sched if x[0] == ISOLATE], {}, None, drain1)
    alone.push(ids1[ISOLATE], None)
    drain1(wait=True)
    alone.close()
    return dict(res=by_stream, keep={s: np.concatenate(v) for s, v in keep.items()},
                flags={s: np.concatenate(v) for s, v in flags.items()}, alone=res1)


def _split(res):
    stats = [r for r in res if r["nstatblks"] == 1]
    series = [r for r in res if r["nt"] > 0]
    return stats, series


def test_rfi_serving_flags_all_streams(O, served):
    L = O.Layout(nave=NAVE)
    S = L.nave * L.twonchan
    assert S % 5000 == 0
    ncol = int(TSTAT / L.tchan)
    nflagged = 0
    for s in range(NSTREAMS):
        stats, series = _split(served["res"][s])
        pf = served["flags"][s]
        nrows = len(pf) * 5000 // S
        rows_flags = np.bitwise_or.reduce(pf[:nrows * (S // 5000)].reshape(nrows, S // 5000), axis=1)
        assert len(stats) == int(DUR) and all(r["device_errors"] == 0 for r in stats + series)
        for r in stats:
            assert np.array_equal(r["row_flags"], rows_flags[r["row0"]:r["row0"] + ncol])
        got = np.concatenate([r["row_flags"] for r in series])
        assert np.array_equal(got, rows_flags[:got.size])
        nflagged += int((got & 1).astype(bool).sum())
    print(f"{NSTREAMS} streams x {DUR:g} s: row flags bit-exact; {nflagged} rows flagged invalid")


@pytest.mark.parametrize("stream", CHECK)
def test_rfi_serving_moments_vs_fp64(O, served, stream):
    from coracle import COracle
    co = COracle(64)
    L = O.Layout(nave=NAVE)
    ncol = int(TSTAT / L.tchan)
    fr = served["keep"][stream].reshape(-1, 2, 5032)
    p0 = np.ascontiguousarray(fr[:, 0, 32:]).reshape(-1)
    p1 = np.ascontiguousarray(fr[:, 1, 32:]).reshape(-1)
    rows = co.channelise(p0, p1, L)
    del p0, p1, fr
    nbp = rows.shape[0] // 128 * 128
    bp = co.bandpass(rows[:nbp])
    stats, series = _split(served["res"][stream])
    worst = dict(ave=0.0, var=0.0, sk=0.0)
    for r in stats:
        k = r["row0"] // ncol
        ave, sig, outl = O.calcstats_chan(bp[k * ncol:(k + 1) * ncol], ncol, 1)
        level = np.abs(ave[0]) + np.sqrt(np.abs(sig[0])) + 1e-30
        worst["ave"] = max(worst["ave"], float(np.max(np.abs(r["chan_ave"][0] - ave[0]) / level)))
        worst["var"] = max(worst["var"], float(np.max(np.abs(r["chan_sig"][0] - sig[0]) / (np.abs(sig[0]) + 1e-30))))
        assert np.array_equal(r["chan_outlier"][0], outl[0])
        sk = O.chan_sk(rows[k * ncol:(k + 1) * ncol], ncol, 1, 2 * NAVE)
        worst["sk"] = max(worst["sk"], float(np.max(np.abs(r["chan_sk"][0] - sk[0]))))
    a, sg = co.dedisperse_sigma_cm(co.transpose(bp), np.zeros((1, L.nchanout), np.int32), nbp)
    got = np.concatenate([r["dd"] for r in series], axis=1)
    gsg = np.concatenate([r["dd_sigma"] for r in series], axis=1)
    n = got.shape[1]
    assert n == nbp
    e_dd = float(np.max(np.abs(got - a[:, :n])) / np.sqrt(np.mean(a[:, :n] ** 2)))
    e_sg = float(np.max(np.abs(gsg - sg[:, :n]) / np.abs(sg[:, :n])))
    print(f"stream {stream}: {len(stats)} stats blocks; mean err/level {worst['ave']:.1e}, variance rel "
          f"{worst['var']:.1e}, SK abs {worst['sk']:.1e}; zero-DM series err/rms {e_dd:.1e}, sigma rel {e_sg:.1e}")
    assert worst["ave"] <= 1e-4 and worst["var"] <= 1e-4 and worst["sk"] <= 1e-3
    assert e_dd <= 5e-5 and e_sg <= 1e-4


def test_rfi_serving_alone_equals_mix(served):
    mix = served["res"][ISOLATE]
    alone = served["alone"]
    assert len(mix) == len(alone) > 0
    for a, b in zip(alone, mix):
        assert (a["row0"], a["nt"], a["nstatblks"]) == (b["row0"], b["nt"], b["nstatblks"])
        for key in ("dd", "dd_sigma", "chan_ave", "chan_sig", "chan_outlier", "chan_sk", "row_flags"):
            x, y = a[key], b[key]
            assert (x is None and y is None) or np.array_equal(x, y), key
