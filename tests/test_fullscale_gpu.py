"""The full-scale plain-FP32 configuration at its stated size, through the
plan API, against the FP64 C oracle on the same rows.

Workload: 60 s of 2-pol VLITE VDIF (seed 1) with the 20 dispersed pulses of
synth.injected_pulses (DM U(50, 1000), FWHM U(1, 10) ms, matched-filter SNR
U(8, 30)), full band (6250 channels), NAVE 10, 2048 DM trials on
linspace(0, 1000); stream mode with 1-s output chunks: every complete row is
channelised, bandpass windows are absolute 128-row windows, and each output
sample is dedispersed once, so 61,440 rows give 61,440 - 12,674 = 48,766
output samples per trial.

Checks, tolerances as written below:
  * the dedispersed series of all 2048 trials within 5e-5 of the oracle's rms;
  * per chunk, calcstats ave and sigma within 1e-4 (relative), peak within
    1e-3, FRB flags identical;
  * per chunk, the candidates (best boxcar over widths 1..16, threshold 7,
    DM-local maxima) identical to the oracle's rule applied to the oracle's
    series, near-ties excepted and printed (tests/candmatch.py);
  * injected-pulse recall: the clusters of candidates (within 16 trials and
    50 rows) are matched to the injected pulses and printed, with each
    pulse's state (found, missed, or outside the searched span); the CUDA
    path finds exactly the pulses the FP64 chain finds.
"""
import time

import numpy as np
import pytest

from candmatch import boxcar_snr_fn, check_candidates

pytestmark = pytest.mark.gpu

DURATION, NAVE, NDM, BOX, SNR_MIN = 60.0, 10, 2048, 16, 7.0
TCHAN = NAVE * 12500 / 128e6


@pytest.fixture(scope="module")
def full60(vf, O):
    import torch
    from coracle import COracle
    from vlite_frb_b200 import synth
    pulses = synth.injected_pulses(1, 20, DURATION, 50.0, 1000.0)
    spec = synth.StreamSpec(duration=DURATION, seed=1, pulses=pulses)
    dev = synth.make_vdif(spec, device="cuda")
    host = torch.empty(dev.numel(), dtype=torch.uint8, pin_memory=True)
    host.copy_(dev)
    del dev
    torch.cuda.empty_cache()
    dms = np.linspace(0.0, 1000.0, NDM).astype(np.float32)
    plan = vf.Plan(dms, nave=NAVE, muoslowfreq=384.0, mode=vf.MODE_STREAM, chunk_seconds=1.0, ring_seconds=2.0,
                   outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=SNR_MIN, boxcar_max=BOX)
    piece = 2 * 25600 * 5032
    res = []
    t0 = time.perf_counter()
    for off in range(0, host.numel(), piece):
        plan.push(0, host[off:off + piece])
        while True:
            r = plan.poll(wait=False)
            if r is None:
                break
            res.append(r)
    plan.push(0, None)
    res += plan.drain()
    t_gpu = time.perf_counter() - t0
    md = plan.max_delay
    plan.close()
    # The oracle on the same bytes: the stream has no gaps and starts on a
    # cal boundary, so its pol-pair sequence is the frame order itself.
    t0 = time.perf_counter()
    fr = host.numpy().reshape(-1, 2, 5032)
    p0 = np.ascontiguousarray(fr[:, 0, 32:]).reshape(-1)
    p1 = np.ascontiguousarray(fr[:, 1, 32:]).reshape(-1)
    del fr, host
    co = COracle(64)
    L = O.Layout(nave=NAVE, muoslowfreq=384.0, nbundle=1)
    rows = co.channelise(p0, p1, L)
    del p0, p1
    nbp = rows.shape[0] // 128 * 128
    bp = co.bandpass(rows[:nbp])
    del rows
    cm = co.transpose(bp)
    del bp
    off, _ = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    assert int(off.max()) == md  # stream mode carries the table's largest delay
    dd = co.dedisperse_cm(cm, off, nbp - md)
    del cm
    t_oracle = time.perf_counter() - t0
    print(f"60-s run: plan API {t_gpu:.1f} s wall (including result copies), FP64 oracle {t_oracle:.1f} s "
          f"on {co.threads()} threads")
    return dict(res=res, dd=dd, dms=dms, md=md, nbp=nbp, pulses=pulses, co=co)


def test_fullscale_series_and_stats(full60):
    res, dd = full60["res"], full60["dd"]
    assert sum(r["nt"] for r in res) == full60["nbp"] - full60["md"] == 48766
    assert all(r["device_errors"] == 0 for r in res)
    rms = float(np.sqrt(np.mean(dd ** 2)))
    worst = 0.0
    for r in res:
        seg = dd[:, r["row0"]:r["row0"] + r["nt"]]
        worst = max(worst, float(np.max(np.abs(r["dd"] - seg))) / rms)
        st = full60["co"].calcstats_dm(seg)
        assert np.allclose(r["ave"], st["ave"], rtol=1e-4, atol=1e-4 * rms)
        assert np.allclose(r["sigma"], st["sigma"], rtol=1e-4)
        assert np.allclose(r["peak"], st["peak"], rtol=1e-3, atol=1e-3)
        assert np.array_equal(r["frb"], st["frb"])
    print(f"60-s series: max |CUDA - FP64| / rms = {worst:.2e} over {len(res)} chunks x {NDM} trials")
    assert worst <= 5e-5


def _oracle_chunk_cands(O, co, dd, r, dms):
    seg = dd[:, r["row0"]:r["row0"] + r["nt"]]
    st = co.calcstats_dm(seg)
    best, start, width = O.boxcar_best(seg, st["ave"], st["sigma"], BOX)
    want = O.candidates(best, start, width, dms, SNR_MIN, r["row0"])
    return want, best, boxcar_snr_fn(seg, st["ave"], st["sigma"], r["row0"])


def test_fullscale_candidates_and_recall(vf, O, full60):
    res, dd, dms, co = full60["res"], full60["dd"], full60["dms"], full60["co"]
    got_all, want_all, ties = [], [], 0
    for r in res:
        want, best, snr_at = _oracle_chunk_cands(O, co, dd, r, dms)
        ties += check_candidates(r["cands"], want, best, snr_at, what=f"chunk {r['seq']}")
        got_all += r["cands"]
        want_all += [dict(dm_index=d, t=t, width=w, snr=s, dm=m) for d, t, w, s, m in want]
    print(f"candidates: {len(got_all)} (oracle {len(want_all)}), near-ties accepted: {ties}")
    got_cl = vf.cluster_cands(got_all, dm_tol=16, t_tol=50)[0]
    want_cl = vf.cluster_cands(want_all, dm_tol=16, t_tol=50)[0]
    assert len(got_cl) == len(want_cl)
    out_end = (full60["nbp"] - full60["md"]) * TCHAN  # last output sample (top-of-band arrival), s

    def near(c, p):
        return abs(c["t"] * TCHAN - p.t0) <= max(0.02, 3e-3 * p.fwhm_ms) and abs(c["dm"] - p.dm) <= 10.0

    matched = set()
    false_pos = []
    for c in got_cl:
        hit = [i for i, p in enumerate(full60["pulses"]) if near(c, p)]
        matched.update(hit)
        if not hit:
            false_pos.append(c)
        print(f"cluster t={c['t'] * TCHAN:.4f} s DM={c['dm']:.1f} SNR={c['snr']:.2f} width={c['width']}"
              f" -> {'pulse %d' % hit[0] if hit else 'no injected pulse'}")
    coverable = [i for i, p in enumerate(full60["pulses"]) if p.t0 + 0.05 < out_end]
    oracle_found = {i for i, p in enumerate(full60["pulses"]) for c in want_cl if near(c, p)}
    for i, p in enumerate(full60["pulses"]):
        state = "found" if i in matched else ("not in the searched span" if i not in coverable else "missed")
        print(f"pulse {i}: t0={p.t0:.3f} s DM={p.dm:.1f} FWHM={p.fwhm_ms:.1f} ms SNR={p.snr:.1f}: {state}")
    print(f"recall {len(matched & set(coverable))}/{len(coverable)} of the pulses in the searched span "
          f"(0-{out_end:.1f} s), {len(false_pos)} clusters with no injected pulse")
    # the CUDA path finds exactly the pulses the FP64 chain finds
    assert matched == oracle_found
