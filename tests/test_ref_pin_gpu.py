"""Pins the oracle and the sm_100a kernels to the reference's own GPU code.

The harness libraries in oracle/_ref (built from the reference sources, see
oracle/build_ref.py) run the reference's convertarray + cuFFT R2C + sumpower
+ avepower + per-row copies, subtractbpCAL, the dead-code subtractbp and
subtractZERO, dedisperse + calcstats (PIPE),
dedisperseSTATS (TS) and the per-channel calcstats (STATS) with the
reference's launch shapes.  Three-way comparisons: reference vs FP64 oracle
(pins the oracle), product vs oracle (the parity bar).

Tolerances: the reference's FP32 cuFFT path keeps the 128 offset (its DC
term dominates the transform's rounding), so its filterbank agrees with FP64
to ~1e-4 of the row mean; the product's to 1e-5.  Stage outputs of the
reference kernels agree with the oracle to FP32 rounding (stated per test).
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib(tool):
    p = os.path.join(ROOT, "oracle", "_ref", f"libref_{tool}.so")
    if not os.path.exists(p):
        pytest.skip("reference build not present")
    lib = C.CDLL(p)
    vp, ci, cf = C.c_void_p, C.c_int, C.POINTER(C.c_float)
    lib.ref_gpu_channelise.argtypes = [vp, vp, ci, ci, ci, ci, ci, ci, vp, cf]
    lib.ref_gpu_bandpass.argtypes = [vp, ci, ci, cf]
    if tool in ("pipe", "ts"):
        lib.ref_gpu_subtract_mode.argtypes = [vp, ci, ci, ci, cf]
        lib.ref_gpu_dedisperse.argtypes = [vp, ci, ci, vp, ci, ci, vp, vp, vp, vp, vp, vp, cf]
    if tool == "stats":
        lib.ref_gpu_chanstats.argtypes = [vp, ci, ci, ci, ci, vp, vp, vp, cf]
    return lib


def _pols(seed=4, dur=0.2):
    from vlite_frb_b200 import synth
    fr = synth.make_vdif(synth.StreamSpec(duration=dur, seed=seed)).numpy().reshape(-1, 2, 5032)
    return np.ascontiguousarray(fr[:, 0, 32:].reshape(-1)), np.ascontiguousarray(fr[:, 1, 32:].reshape(-1))


@pytest.mark.parametrize("muos,nave", [(384.0, 10), (360.0, 4)])
def test_channeliser_reference_oracle_product(vf, O, muos, nave):
    import torch
    lib = _lib("pipe")
    nb = 8
    L = O.Layout(nave=nave, muoslowfreq=muos, nbundle=nb)
    p0, p1 = _pols()
    nbund = len(p0) // L.nloop
    n = nbund * L.nloop
    rows = nbund * nb
    ref = np.zeros((rows, L.nchanout), np.float32)
    ms = C.c_float(0)
    st = lib.ref_gpu_channelise(p0.ctypes.data, p1.ctypes.data, nbund, L.twonchan, nave, nb, L.nskip, L.nchanout,
                                ref.ctypes.data, C.byref(ms))
    assert st == 0
    orc = O.channelise(p0[:n], p1[:n], L)
    e_ref = np.max(np.abs(ref - orc) / orc.mean(axis=1, keepdims=True))
    print(f"reference cuFFT chain vs FP64: {e_ref:.2e} of row mean ({ms.value:.2f} ms)")
    assert e_ref <= 5e-4
    Lp = vf.layout(nave=nave, muoslowfreq=muos, nbundle=nb)
    dev = torch.device("cuda")
    d = torch.from_numpy(np.concatenate([p0, p1])).to(dev)
    nslot = len(p0) // 5000
    s0 = torch.arange(nslot, dtype=torch.int64, device=dev) * 5000
    got = vf.channelise(d, s0, s0 + len(p0), 0, rows, Lp)
    torch.cuda.synchronize()
    e_prod = np.max(np.abs(got.cpu().numpy() - orc) / orc.mean(axis=1, keepdims=True))
    print(f"product vs FP64: {e_prod:.2e} of row mean")
    assert e_prod <= 1e-5


@pytest.mark.parametrize("tool", ["pipe", "ts"])
def test_bandpass_reference_oracle_product(vf, O, tool):
    import torch
    lib = _lib(tool)
    rng = np.random.default_rng(3)
    maxnt, nch = 128 * 7 + 40, 300
    fb = (rng.chisquare(20, (maxnt, nch)) * rng.uniform(100, 900, nch) / 20).astype(np.float32)
    fb[10, 3] = 1e6
    ref = fb.copy()
    ms = C.c_float(0)
    assert lib.ref_gpu_bandpass(ref.ctypes.data, maxnt, nch, C.byref(ms)) == 0
    orc = O.subtract_bp_cal(fb.astype(np.float64))
    scale = np.abs(fb).max()
    # the reference sums 128 floats sequentially in FP32
    assert np.max(np.abs(ref - orc)) <= 2e-5 * scale
    got = vf.bandpass(torch.from_numpy(fb).cuda()).cpu().numpy().T
    assert np.max(np.abs(got - orc)) <= 1e-6 * scale


@pytest.mark.parametrize("tool", ["pipe", "ts"])
@pytest.mark.parametrize("kind", [0, 1])
def test_subtract_modes_reference_oracle_product(vf, O, tool, kind):
    """The dead-code modes subtractbp (kind 0) and subtractZERO (kind 1): the
    reference's kernels, the FP64 oracle and the product."""
    import torch
    lib = _lib(tool)
    rng = np.random.default_rng(30 + kind)
    maxnt, nch = 1500, 320
    fb = (rng.standard_normal((maxnt, nch)) * rng.uniform(1, 3, nch)).astype(np.float32)
    fb[rng.integers(0, maxnt, 50), rng.integers(0, nch, 50)] += 80.0
    if kind == 0:
        fb[:, 17] = fb[:, 17] * 30 + 200.0  # wide window about sum/NCHANOUT: every row kept
        fb[:, 40] = 4.0    # empty clip -> NaN in all three
    ref = fb.copy()
    ms = C.c_float(0)
    assert lib.ref_gpu_subtract_mode(ref.ctypes.data, maxnt, nch, kind, C.byref(ms)) == 0
    x64 = fb.astype(np.float64)
    orc = O.subtract_bp_full(x64) if kind == 0 else O.subtract_zero(x64)
    assert np.array_equal(np.isnan(ref), np.isnan(orc))
    ok = ~np.isnan(orc)
    scale = np.abs(fb).max()
    # the reference sums up to 1500 floats sequentially in FP32
    e_ref = np.max(np.abs(ref[ok] - orc[ok])) / scale
    print(f"reference kind {kind} vs FP64: {e_ref:.2e} of max|x| ({ms.value:.2f} ms)")
    assert e_ref <= 5e-5
    cm = torch.from_numpy(np.ascontiguousarray(fb.T)).cuda()
    (vf.subtract_bp_full if kind == 0 else vf.subtract_zero)(cm)
    got = cm.cpu().numpy().T
    assert np.array_equal(np.isnan(got), np.isnan(orc))
    assert np.max(np.abs(got[ok] - orc[ok])) <= 1e-6 * scale


def test_dedisperse_calcstats_reference_oracle_product(vf, O):
    import torch
    lib = _lib("pipe")
    rng = np.random.default_rng(8)
    L = O.Layout(nave=10, muoslowfreq=384.0)
    nch = 512
    dms = np.linspace(0, 60, 37).astype(np.float32)
    off, md = O.delay_table(dms, 384.0, 0.125, 0.001, nch)
    md = int(off.max())
    nt = 900
    maxnt = nt + md
    fb = (rng.standard_normal((maxnt, nch)) * 5).astype(np.float32)
    for c in range(nch):
        fb[300 + off[20, c], c] += 6.0
    out = np.zeros((len(dms), nt), np.float32)
    frb = np.zeros(len(dms), np.int32)
    ave, sig, peak = (np.zeros(len(dms), np.float32) for _ in range(3))
    ms = C.c_float(0)
    assert lib.ref_gpu_dedisperse(fb.ctypes.data, maxnt, nch, np.ascontiguousarray(off).ctypes.data, len(dms), nt,
                                  out.ctypes.data, None, frb.ctypes.data, ave.ctypes.data, sig.ctypes.data,
                                  peak.ctypes.data, C.byref(ms)) == 0
    orc = O.dedisperse(fb.astype(np.float64), off, nt)
    rms = np.sqrt(np.mean(orc ** 2))
    # the reference adds 512 channels one by one into FP32 global memory
    assert np.max(np.abs(out - orc)) <= 3e-5 * rms
    st = O.calcstats_dm(orc)
    assert np.array_equal(frb, st["frb"])
    assert np.allclose(ave, st["ave"], rtol=1e-4, atol=1e-6 * rms)
    assert np.allclose(sig, st["sigma"], rtol=1e-5)
    assert np.allclose(peak, st["peak"], rtol=1e-4)
    plan = vf.DedispPlan(off)
    got, gst = plan(torch.from_numpy(np.ascontiguousarray(fb.T)).cuda(), nt)
    torch.cuda.synchronize()
    # same summation order as the reference (channel by channel in FP32): same rounding
    assert np.max(np.abs(got.cpu().numpy() - orc)) <= 3e-5 * rms
    assert np.array_equal(gst["frb"].cpu().numpy(), frb)
    assert np.allclose(gst["peak"].cpu().numpy(), peak, rtol=1e-4)


def test_dedisperse_stats_ts_reference_oracle_product(vf, O):
    import torch
    lib = _lib("ts")
    rng = np.random.default_rng(12)
    L = O.Layout(nave=4, nchanout_fixed=3840)
    dms = np.array([0.0, 119.3], np.float32)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    nt = 600
    maxnt = nt + int(off.max())
    fb = (rng.standard_normal((maxnt, L.nchanout)) * 3).astype(np.float32)
    out = np.zeros((2, nt), np.float32)
    sg = np.zeros((2, nt), np.float32)
    ms = C.c_float(0)
    assert lib.ref_gpu_dedisperse(fb.ctypes.data, maxnt, L.nchanout, np.ascontiguousarray(off).ctypes.data, 2, nt,
                                  out.ctypes.data, sg.ctypes.data, None, None, None, None, C.byref(ms)) == 0
    a, s = O.dedisperse_sigma(fb.astype(np.float64), off, nt)
    assert np.max(np.abs(out - a)) <= 1e-5 * np.sqrt(np.mean(a ** 2))
    assert np.max(np.abs(sg - s) / s) <= 1e-4
    plan = vf.DedispPlan(off)
    gs = torch.empty((2, nt), device="cuda")
    got, _ = plan(torch.from_numpy(np.ascontiguousarray(fb.T)).cuda(), nt, sigma_out=gs, stats=False)
    torch.cuda.synchronize()
    assert np.max(np.abs(gs.cpu().numpy() - s) / s) <= 1e-5


def test_chanstats_reference_oracle_product(vf, O):
    import torch
    lib = _lib("stats")
    rng = np.random.default_rng(14)
    ncol, nblk, nch = 400, 5, 260
    maxnt = ncol * nblk
    fb = (rng.standard_normal((maxnt, nch)) * 4).astype(np.float32)
    fb[:, 7] = 2.0  # a constant channel: zero variance, no outliers
    ca, cs, co_ = (np.zeros((nblk, nch), np.float32) for _ in range(3))
    ms = C.c_float(0)
    assert lib.ref_gpu_chanstats(fb.ctypes.data, maxnt, nch, ncol, nblk, ca.ctypes.data, cs.ctypes.data,
                                 co_.ctypes.data, C.byref(ms)) == 0
    a, s, o = O.calcstats_chan(fb.astype(np.float64), ncol, nblk)
    assert np.max(np.abs(ca - a)) <= 1e-5 * 4
    assert np.max(np.abs(cs - s)[s > 0] / s[s > 0]) <= 1e-4
    assert np.array_equal(co_, o)
    ga, gs, go = vf.chan_stats(torch.from_numpy(np.ascontiguousarray(fb.T)).cuda(), maxnt, ncol, nblk)
    torch.cuda.synchronize()
    assert np.max(np.abs(ga.cpu().numpy() - a)) <= 1e-6 * 4
    assert np.array_equal(go.cpu().numpy(), o)
