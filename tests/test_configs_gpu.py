"""The small plain-FP32 configuration and its reduced-precision forms at full
size, against the FP64 oracle chain.

Workload: 8.0 s of 2-pol VLITE VDIF (seed 0), one dispersed pulse at DM 150
(2 ms FWHM, matched-filter SNR 20, t = 3.0 s), 12500-point FFT -> 6250
channels (full band), NAVE 10, DM 0-200 in steps of 1 (201 trials), one
7.5-s block (7680 rows; the carry is the DM-200 delay at the band's lower
edge, TS:464, 2535 rows, leaving 5145 output samples).

Tolerances: FP32 dedispersed series <= 5e-5 rms of the oracle's; candidates
(DM-local maxima of the best boxcar SNR, widths 1..8) identical in trial
(+-1 for a near-tie between neighbouring trials), time and width, SNR within
1%.  FP16 storage: series <= 3e-3 rms, the same candidates as FP32 with
SNR within 1%.  int8 storage (q = 16): series <= 0.12 rms, the pulse found at
the same trial and time (errors printed).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DMS = np.arange(0, 201, dtype=np.float32)
NAVE, MAXTIME, BOX, SNR_MIN = 10, 7.5, 8, 8.0


@pytest.fixture(scope="module")
def cfg1():
    from vlite_frb_b200 import synth
    spec = synth.StreamSpec(duration=8.0, seed=0, pulses=[synth.Pulse(3.0, 150.0, 2.0, 20.0)])
    return synth.make_vdif(spec).numpy()


@pytest.fixture(scope="module")
def oracle1(O, cfg1):
    from coracle import COracle
    co = COracle(64)
    L = O.Layout(nave=NAVE, muoslowfreq=384.0, maxtime=MAXTIME)
    off, md = O.delay_table(DMS, L.fch1, L.chanbw, L.tchan, L.nchanout)
    _, bundles, _ = O.read_bundles(cfg1, L)
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    (q, fb), = list(O.run_blocks(rows, L, md))
    nt = L.maxnt - md
    dd = co.dedisperse_cm(co.transpose(co.bandpass(fb)), off, nt)
    st = O.calcstats_dm(dd)
    best, start, width = O.boxcar_best(dd, st["ave"], st["sigma"], BOX)
    cands = O.candidates(best, start, width, DMS, SNR_MIN, 0)
    return dict(L=L, md=md, nt=nt, dd=dd, cands=cands)


def _run(vf, buf, storage):
    plan = vf.Plan(DMS, nave=NAVE, muoslowfreq=384.0, maxtime=MAXTIME, mode=vf.MODE_BLOCK, storage=storage,
                   outputs=vf.OUT_DEDISP | vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=SNR_MIN, boxcar_max=BOX)
    plan.push(0, buf)
    plan.push(0, None)
    res = plan.drain()
    plan.close()
    assert len(res) == 1 and res[0]["device_errors"] == 0
    return res[0]


def _err(got, ref):
    return np.max(np.abs(got - ref)) / np.sqrt(np.mean(ref ** 2))


def _pulse(cands):
    return max(cands, key=lambda c: c["snr"] if isinstance(c, dict) else c[3])


def test_small_config_fp32(vf, cfg1, oracle1):
    r = _run(vf, cfg1, 0)
    assert r["nt"] == oracle1["nt"] == 7680 - oracle1["md"]
    e = _err(r["dd"], oracle1["dd"])
    print(f"FP32 series error / rms: {e:.2e}")
    assert e <= 5e-5
    want = oracle1["cands"]
    assert len(r["cands"]) == len(want) >= 1
    for c, w in zip(r["cands"], want):
        assert abs(c["dm_index"] - w[0]) <= 1 and c["t"] == w[1] and c["width"] == w[2]
        assert abs(c["snr"] - w[3]) <= 0.01 * w[3]
    p = _pulse(r["cands"])
    tchan = NAVE * 12500 / 128e6
    print("pulse candidate", p)
    assert abs(p["dm"] - 150.0) <= 2.0 and abs(p["t"] * tchan - 3.0) < 0.005


@pytest.mark.parametrize("storage,tol", [(1, 3e-3), (2, 0.12)])
def test_small_config_reduced_precision(vf, cfg1, oracle1, storage, tol):
    f32 = _run(vf, cfg1, 0)
    r = _run(vf, cfg1, storage)
    e = _err(r["dd"], oracle1["dd"])
    p32, p = _pulse(f32["cands"]), _pulse(r["cands"])
    dsnr = abs(p["snr"] - p32["snr"]) / p32["snr"]
    print(f"storage {storage}: series error / rms {e:.2e}, pulse dSNR vs FP32 {dsnr:.2e}")
    assert e <= tol
    assert (p["dm_index"], p["t"]) == (p32["dm_index"], p32["t"])
    if storage == 1:  # FP16: identical candidate list, SNR within 1%
        assert [(c["dm_index"], c["t"], c["width"]) for c in r["cands"]] == \
            [(c["dm_index"], c["t"], c["width"]) for c in f32["cands"]]
        assert max(abs(a["snr"] - b["snr"]) / b["snr"] for a, b in zip(r["cands"], f32["cands"])) <= 0.01
