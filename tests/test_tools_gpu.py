"""The drop-in command-line tools, run as processes on synthetic VDIF files,
against the oracle chain.

vdifFILE2dedisp_PIPELINE: NAME.head equals the SIGPROC header the reference
writes (bytes, tstart from the oracle reader); OUTDD.bin holds every DM
trial's value followed by the fifth block's dedispersed series and
NAME.nohead.fil the fifth block's bandpass-subtracted filterbank, both within
the engine tolerance (5e-5 of the rms) of the FP64 oracle.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "vlite-frb_b200", "bin")


def _tool(name):
    p = os.path.join(BIN, name)
    if not os.path.exists(p):
        pytest.fail(f"{p} not built (run vlite-frb_b200/build.py)")
    return p


@pytest.fixture(scope="module")
def co():
    from coracle import COracle
    return COracle(64)


def _close(got, ref, tol, what):
    rms = np.sqrt(np.mean(ref ** 2))
    e = np.max(np.abs(got - ref)) / rms
    print(f"{what}: max err / rms = {e:.2e}")
    assert e <= tol, (what, e)


def test_pipe_tool_outputs(vf, O, co, tmp_path):
    from vlite_frb_b200 import synth
    nave, maxtime = 2, 0.2
    dms = np.arange(0, 5.5, 0.5, dtype=np.float32)
    with open(tmp_path / "DM101.txt", "w") as f:
        for d in dms:
            f.write(f"{d:.1f}\n")
    spec = synth.StreamSpec(duration=1.0, seed=21, pulses=[synth.Pulse(0.62, 3.0, 2.0, 40.0)])
    buf = synth.make_vdif(spec).numpy()
    buf.tofile(tmp_path / "in.vdif")
    cmd = [_tool("vdifFILE2dedisp_PIPELINE"), "-nchan", "6250", "-nave", str(nave), "-nb", "32", "-i", "in.vdif",
           "-o", "out", "-fullband", "-maxtime", str(maxtime)]
    r = subprocess.run(cmd, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr, (tmp_path / "out.log").read_text())
    assert r.returncode == 0
    assert "TOTAL TIME" in r.stdout

    L = O.Layout(nave=nave, muoslowfreq=384.0, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    h0, bundles, _ = O.read_bundles(buf, L)
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    blocks = list(O.run_blocks(rows, L, md))
    assert len(blocks) >= 5
    tsamp = nave * 12500 / 128e6
    assert (tmp_path / "out.head").read_bytes() == O.sigproc_header(L.fch1, -L.chanbw, L.nchanout,
                                                                     O.vdif_dmjd(h0), tsamp)
    bp = co.bandpass(blocks[4][1])
    nt = L.maxnt - md
    dd = co.dedisperse_cm(co.transpose(bp), off, nt)
    raw = np.fromfile(tmp_path / "OUTDD.bin", np.float32).reshape(len(dms), 1 + nt)
    assert np.array_equal(raw[:, 0], dms)
    _close(raw[:, 1:], dd, 5e-5, "OUTDD.bin (block 4)")
    fil = np.fromfile(tmp_path / "out.nohead.fil", np.float32).reshape(L.maxnt, L.nchanout)
    _close(fil, bp, 5e-5, "nohead.fil (block 4)")


def test_pipe_tool_streaming_fil_cands_and_rfi_modes(vf, O, co, tmp_path):
    """Extensions: -filall streams every block's filterbank into NAME.fil (one
    continuous series after the header), -cands writes the clustered
    candidates, -bpfull/-zerodm switch on the reference's dead-code modes."""
    from vlite_frb_b200 import synth
    nave, maxtime = 2, 0.2
    dms = np.arange(0, 5.5, 0.5, dtype=np.float32)
    with open(tmp_path / "DM101.txt", "w") as f:
        for d in dms:
            f.write(f"{d:.1f}\n")
    spec = synth.StreamSpec(duration=0.9, seed=22, pulses=[synth.Pulse(0.55, 3.0, 2.0, 60.0)])
    buf = synth.make_vdif(spec).numpy()
    buf.tofile(tmp_path / "in.vdif")
    exe = _tool("vdifFILE2dedisp_PIPELINE")
    base = [exe, "-nchan", "6250", "-nave", str(nave), "-nb", "32", "-i", "in.vdif", "-fullband",
            "-maxtime", str(maxtime), "-filall"]
    r = subprocess.run(base + ["-o", "a", "-cands", "8", "-boxcar", "8"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.stderr, (tmp_path / "a.log").read_text())
    r = subprocess.run(base + ["-o", "b", "-bpfull", "-zerodm"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, (r.stderr, (tmp_path / "b.log").read_text())

    L = O.Layout(nave=nave, muoslowfreq=384.0, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    h0, bundles, _ = O.read_bundles(buf, L)
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    blocks = list(O.run_blocks(rows, L, md))
    assert len(blocks) >= 3
    hdr = O.sigproc_header(L.fch1, -L.chanbw, L.nchanout, O.vdif_dmjd(h0), nave * 12500 / 128e6)
    first = (md // L.nbundle) * L.nbundle
    for name, chain in (("a", co.bandpass), ("b", lambda fb: O.subtract_zero(O.subtract_bp_full(fb)))):
        raw = (tmp_path / f"{name}.fil").read_bytes()
        assert raw[:len(hdr)] == hdr
        got = np.frombuffer(raw[len(hdr):], np.float32).reshape(-1, L.nchanout)
        want = np.concatenate([chain(fb)[0 if q == 0 else first:] for q, fb in blocks])
        assert got.shape == want.shape
        _close(got, want, 5e-5, f"{name}.fil")
    lines = [ln.split() for ln in (tmp_path / "a.cands").read_text().splitlines() if not ln.startswith("#")]
    assert lines, "no candidate"
    best = max(lines, key=lambda v: float(v[3]))
    t_s, dm = float(best[1]), float(best[2])
    print("brightest cluster", best)
    assert abs(t_s - 0.55) < 0.003 and abs(dm - 3.0) <= 1.0


def test_pipe_tool_short_input_and_bad_args(vf, tmp_path):
    from vlite_frb_b200 import synth
    exe = _tool("vdifFILE2dedisp_PIPELINE")
    assert subprocess.run([exe], cwd=tmp_path, capture_output=True).returncode == 1
    assert subprocess.run([exe, "-bogus"], cwd=tmp_path, capture_output=True).returncode == 1
    # no DM101.txt: the reference logs the error and exits 2
    synth.make_vdif(synth.StreamSpec(duration=0.3, seed=2)).numpy().tofile(tmp_path / "in.vdif")
    r = subprocess.run([exe, "-d", "-i", "in.vdif", "-o", "o"], cwd=tmp_path, capture_output=True, timeout=120)
    assert r.returncode == 2
    # fewer than five blocks: outputs exist, the fifth block's buffers are zeros
    with open(tmp_path / "DM101.txt", "w") as f:
        f.write("0.0\n1.0\n")
    r = subprocess.run([exe, "-d", "-i", "in.vdif", "-o", "o", "-maxtime", "0.1"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    fil = np.fromfile(tmp_path / "o.nohead.fil", np.float32)
    assert fil.size > 0 and not fil.any()
    assert (tmp_path / "o.head").stat().st_size > 0


def test_stats_tool_file_and_ring(vf, O, co, tmp_path):
    """vdifDADA2stats: the .stats file holds, per block, CHANAVE, CHANSIGMA and
    CHANOUTLIER [NSTATBLKS][NCHANOUT]; reading the same bytes from the ring
    (fed by vfrb_dada_write) gives an identical file."""
    import random
    from vlite_frb_b200 import synth
    nave, maxtime, tstat = 4, 0.5, 0.1
    buf = synth.make_vdif(synth.StreamSpec(duration=1.3, seed=9)).numpy()
    buf.tofile(tmp_path / "in.vdif")
    args = ["-maxtime", str(maxtime), "-timestats", str(tstat)]
    r = subprocess.run([_tool("vdifDADA2stats"), "-i", "in.vdif", "-o", "f", *args], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stderr, (tmp_path / "f.log").read_text())
    L = O.Layout(nave=nave, maxtime=maxtime)
    _, bundles, _ = O.read_bundles(buf, L)
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    ncol = int(tstat / L.tchan)
    nblk = int(np.float32(maxtime) / np.float32(tstat))
    blocks = list(O.run_stats_blocks(rows, L))
    got = np.fromfile(tmp_path / "f.stats", np.float32).reshape(-1, 3, nblk, L.nchanout)
    assert got.shape[0] == len(blocks) == 2
    for g, (q, fb) in zip(got, blocks):
        bp = co.bandpass(fb)
        a, s, o = O.calcstats_chan(bp, ncol, nblk)
        assert np.max(np.abs(g[0] - a)) <= 1e-4 * np.abs(bp).max()
        assert np.max(np.abs(g[1] - s) / s) <= 1e-4
        assert np.array_equal(g[2], o)
    key = f"{random.randrange(0x10000000, 0x7fffffff):x}"
    w = subprocess.Popen([_tool("vfrb_dada_write"), "-k", key, "-i", "in.vdif", "-timeout", "120"], cwd=tmp_path)
    try:
        r = subprocess.run([_tool("vdifDADA2stats"), "-k", key, "-o", "k", *args], cwd=tmp_path,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (r.stderr, (tmp_path / "k.log").read_text())
        assert w.wait(timeout=120) == 0
    finally:
        if w.poll() is None:
            w.kill()
            w.wait()
    assert (tmp_path / "k.stats").read_bytes() == (tmp_path / "f.stats").read_bytes()


def test_timeseries_tool_outputs(vf, O, co, tmp_path):
    """vdifDADA2timeseries: DM 0 and DM 119.3 channel-mean and sigma series
    appended per block; the .inf headers (written at the end with -infatend)
    equal the reference's writeprestoheader text."""
    import glob
    from vlite_frb_b200 import synth
    nave, maxtime = 4, 1.5
    buf = synth.make_vdif(synth.StreamSpec(duration=3.1, seed=5)).numpy()
    buf.tofile(tmp_path / "in.vdif")
    r = subprocess.run([_tool("vdifDADA2timeseries"), "-d", "-i", "in.vdif", "-o", "ts", "-noskip", "-maxtime",
                        str(maxtime), "-infatend"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dms = np.array([0.0, 119.3], np.float32)
    L = O.Layout(nave=nave, nchanout_fixed=3840, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    h0, bundles, _ = O.read_bundles(buf, L, mode="ts")
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    blocks = list(O.run_blocks(rows, L, md))
    nt = L.maxnt - md
    ref_a, ref_s = [], []
    for q, fb in blocks:
        a, s = co.dedisperse_sigma_cm(co.transpose(co.bandpass(fb)), off, nt)
        ref_a.append(a)
        ref_s.append(s)
    ref_a = np.concatenate(ref_a, axis=1)
    ref_s = np.concatenate(ref_s, axis=1)
    tsamp = nave * 12500 / 128e6
    for d, name in enumerate(("DM0.0", "DM119.3")):
        # a run that crosses a UTC hour rotates the files: concatenate in time order
        dat = sorted(glob.glob(str(tmp_path / f"{name}_*[0-9].dat")))
        assert len(dat) >= 1
        base = dat[-1][:-4]
        a = np.concatenate([np.fromfile(f, np.float32) for f in dat])
        s = np.concatenate([np.fromfile(f[:-4] + "_SIGMA.dat", np.float32) for f in dat])
        assert a.size == s.size == ref_a.shape[1] == len(blocks) * nt
        _close(a, ref_a[d], 5e-5, f"{name} mean series")
        assert np.max(np.abs(s - ref_s[d]) / ref_s[d]) <= 1e-4
        if len(dat) == 1:
            inf = open(base + ".inf").read()
            assert inf == O.presto_inf(os.path.basename(base), O.vdif_dmjd(h0), a.size, tsamp, dms[d],
                                       320.0 + 0.5 * L.chanbw, L.nchanout * L.chanbw, L.nchanout, L.chanbw)
    assert glob.glob(str(tmp_path / "ts_*.log"))


def test_stats_and_timeseries_sk_and_flags(vf, O, co, tmp_path):
    """RFI-heavy input (tones, bursts, 10% invalid-flagged frames, two missing
    pairs): vdifDADA2stats -sk -flags writes per block the spectral kurtosis
    of the raw filterbank and the row flags; vdifDADA2timeseries -flags writes
    one flag byte per series sample.  SK within 1e-3 of the FP64 oracle,
    flags identical."""
    from vlite_frb_b200 import synth
    fr = synth.make_vdif(synth.StreamSpec(duration=3.2, seed=13, rfi=synth.Rfi())).numpy().reshape(-1, 2, 5032)
    buf = np.ascontiguousarray(np.delete(fr, [12345, 40000], axis=0)).reshape(-1)
    buf.tofile(tmp_path / "in.vdif")
    nave, maxtime, tstat = 4, 0.5, 0.1
    r = subprocess.run([_tool("vdifDADA2stats"), "-i", "in.vdif", "-o", "f", "-maxtime", str(maxtime), "-timestats",
                        str(tstat), "-sk", "-flags"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stderr, (tmp_path / "f.log").read_text())
    L = O.Layout(nave=nave, maxtime=maxtime)
    _, bundles, rd = O.read_bundles(buf, L)
    rows = co.channelise(np.concatenate([b[0] for b in bundles]), np.concatenate([b[1] for b in bundles]), L)
    ncol = int(tstat / L.tchan)
    nblk = int(np.float32(maxtime) / np.float32(tstat))
    blocks = list(O.run_stats_blocks(rows, L))
    sk = np.fromfile(tmp_path / "f.sk", np.float32).reshape(-1, nblk, L.nchanout)
    fl = np.fromfile(tmp_path / "f.flags", np.uint8).reshape(-1, L.maxnt)
    flags = O.row_flags(rd.pair_flags, L, len(blocks) * L.maxnt)
    assert sk.shape[0] == fl.shape[0] == len(blocks) >= 5
    for q, fb in blocks:
        assert np.max(np.abs(sk[q] - O.chan_sk(fb, ncol, nblk, 2 * nave))) <= 1e-3
        assert np.array_equal(fl[q], flags[q * L.maxnt:(q + 1) * L.maxnt])
    assert (flags & 1).any() and (flags & 2).any()
    # timeseries: 3840 channels, blocks with the max-delay carry
    maxtime = 1.5
    r = subprocess.run([_tool("vdifDADA2timeseries"), "-d", "-i", "in.vdif", "-o", "ts", "-noskip", "-maxtime",
                        str(maxtime), "-flags"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dms = np.array([0.0, 119.3], np.float32)
    L = O.Layout(nave=nave, nchanout_fixed=3840, maxtime=maxtime)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    _, bundles, rd = O.read_bundles(buf, L, mode="ts")
    nrows = len(bundles) * L.nbundle
    nblocks = len(list(O.run_blocks(np.zeros((nrows, 1)), L, md)))
    flags = O.row_flags(rd.pair_flags, L, nrows + L.maxnt)
    nt = L.maxnt - md
    want = np.concatenate([flags[O.block_rows(L, md, q)][:nt] for q in range(nblocks)])
    got = np.fromfile(tmp_path / "ts.flags", np.uint8)
    assert nblocks >= 1 and np.array_equal(got, want)
