"""Pins the oracle and the product's frame reader to the reference itself.

The reference ships no tests or golden data, so its own code is run here:
oracle/build_ref.py compiles vdifFILE2dedisp_PIPELINE.cu, vdifDADA2stats.cu
and vdifDADA2timeseries.cu (with stand-ins for psrdada/dedisp/vdifio) into
oracle/_ref/, and the harness calls the reference's initframe01 /
filltimebufferHOST on fixture files.  The bundles it produces must equal,
byte for byte, (a) the oracle's restatement and (b) the bundles implied by
the product reader's pair sequence (vfrb_read_pairs).
"""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def _reflib(tool):
    p = os.path.join(REF_DIR, f"libref_{tool}.so")
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (needs the reference checkout at build time)")
    lib = C.CDLL(p)
    lib.ref_read_bundles.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int]
    return lib


def ref_bundles(tool, path, twonchan, nave, nbundle, max_bundles=64, dada_skip=0):
    lib = _reflib(tool)
    nl = twonchan * nave * nbundle
    o0 = np.zeros(nl * max_bundles, np.uint8)
    o1 = np.zeros(nl * max_bundles, np.uint8)
    nb = C.c_int(0)
    ts = C.c_double(0)
    st = lib.ref_read_bundles(path.encode(), twonchan, nave, nbundle, max_bundles, o0.ctypes.data, o1.ctypes.data,
                              C.byref(nb), C.byref(ts), dada_skip)
    n = nb.value
    return st, [(o0[i * nl:(i + 1) * nl], o1[i * nl:(i + 1) * nl]) for i in range(n)], ts.value


def product_bundles(vf, data, mode, twonchan, nave, nbundle, split=0, max_bundles=64):
    lib = vf.lib()
    lib.vfrb_read_pairs.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_void_p,
                                    C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    cap = len(data) // 5032 + 8
    e0 = np.zeros(cap, np.int64)
    e1 = np.zeros(cap, np.int64)
    n = C.c_int64(0)
    ts = C.c_double(0)
    buf = np.ascontiguousarray(data)
    st = lib.vfrb_read_pairs(buf.ctypes.data, len(buf), mode, 0, split, e0.ctypes.data, e1.ctypes.data, cap,
                             C.byref(n), C.byref(ts))
    n = n.value
    fr = buf[:len(buf) // 5032 * 5032].reshape(-1, 5032)

    def stream(e):
        out = np.zeros(n * 5000, np.uint8)
        for k in range(n):
            if e[k] >= 0:
                out[k * 5000:(k + 1) * 5000] = fr[e[k], 32:]
        return out

    s0, s1 = stream(e0), stream(e1)
    nl = twonchan * nave * nbundle
    out = []
    b = 0
    while b < max_bundles and ((b + 1) * nl) // 5000 < n:  # the read-ahead pair must exist
        out.append((s0[b * nl:(b + 1) * nl], s1[b * nl:(b + 1) * nl]))
        b += 1
    return (0 if st == 0 else 2), out, ts.value


def _fixture(tmp_path, name, duration=0.25, frame0=0, seconds0=1000, drop=(), truncate=0, lead_pol1=False, seed=3):
    from vlite_frb_b200 import synth
    buf = synth.make_vdif(synth.StreamSpec(duration=duration, seed=seed, frame0=frame0, seconds0=seconds0)).numpy()
    buf = synth.edit_frames(buf, drop=drop, truncate=truncate, lead_pol1=lead_pol1)
    p = tmp_path / f"{name}.vdif"
    p.write_bytes(buf.tobytes())
    return str(p), buf


CASES = {
    "clean": dict(),
    "not_on_cal_boundary": dict(frame0=1234),
    "second_wrap": dict(frame0=25000),
    "lead_pol1": dict(lead_pol1=True),
    "gap_pol0": dict(drop=[2 * 700, 2 * 701, 2 * 702]),
    "gap_pol1": dict(drop=[2 * 900 + 1]),
    "gap_both": dict(drop=[2 * 1500, 2 * 1500 + 1, 2 * 1501, 2 * 1501 + 1]),
    "truncated_mid_frame": dict(truncate=1777),
    "truncated_header": dict(truncate=5010),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("geom", [(12500, 4, 32), (12500, 3, 7), (6250, 2, 5)])
def test_pipe_reader_matches_reference(tmp_path, vf, O, case, geom):
    twonchan, nave, nbundle = geom
    path, buf = _fixture(tmp_path, case, **CASES[case])
    st_r, ref, ts_r = ref_bundles("pipe", path, twonchan, nave, nbundle)
    L = O.Layout(twonchan=twonchan, nave=nave, nbundle=nbundle)
    h0, orc, _ = O.read_bundles(buf, L, mode="pipe", max_bundles=64)
    st_p, prod, ts_p = product_bundles(vf, buf, 0, twonchan, nave, nbundle)
    assert st_r == 0 and st_p == 0
    assert len(ref) > 0
    assert len(ref) == len(orc) == len(prod), (len(ref), len(orc), len(prod))
    for (a0, a1), (b0, b1), (c0, c1) in zip(ref, orc, prod):
        assert np.array_equal(a0, b0) and np.array_equal(a1, b1)
        assert np.array_equal(a0, c0) and np.array_equal(a1, c1)
    assert ts_r == ts_p == O.vdif_dmjd(h0)


@pytest.mark.parametrize("case", ["clean", "gap_pol0", "gap_both", "second_wrap", "truncated_mid_frame"])
def test_stats_reader_matches_reference(tmp_path, vf, O, case):
    path, buf = _fixture(tmp_path, case, **CASES[case])
    st_r, ref, _ = ref_bundles("stats", path, 12500, 4, 32)
    st_p, prod, _ = product_bundles(vf, buf, 0, 12500, 4, 32)
    assert st_r == 0 and len(ref) == len(prod) > 0
    for (a0, a1), (c0, c1) in zip(ref, prod):
        assert np.array_equal(a0, c0) and np.array_equal(a1, c1)


TS_CASES = dict(CASES)
TS_CASES["gap_across_second"] = dict(frame0=25000, drop=[2 * 650, 2 * 651, 2 * 652, 2 * 650 + 1])


@pytest.mark.parametrize("case", sorted(TS_CASES))
def test_ts_reader_matches_reference(tmp_path, vf, O, case):
    path, buf = _fixture(tmp_path, case, **TS_CASES[case])
    st_r, ref, ts_r = ref_bundles("ts", path, 12500, 4, 32)
    L = O.Layout(twonchan=12500, nave=4, nbundle=32)
    h0, orc, _ = O.read_bundles(buf, L, mode="ts", max_bundles=64)
    st_p, prod, ts_p = product_bundles(vf, buf, 1, 12500, 4, 32)
    assert st_r == 0 and st_p == 0
    assert len(ref) == len(orc) == len(prod) > 0
    for (a0, a1), (b0, b1), (c0, c1) in zip(ref, orc, prod):
        assert np.array_equal(a0, b0) and np.array_equal(a1, b1)
        assert np.array_equal(a0, c0) and np.array_equal(a1, c1)


@pytest.mark.parametrize("split", [5032 * 7 + 13, 100003, 5032])
def test_reader_independent_of_input_split(tmp_path, vf, split):
    """The resumable reader gives the same pairs however the input is cut."""
    case = "gap_both"
    path, buf = _fixture(tmp_path, case, **CASES[case])
    _, whole, _ = product_bundles(vf, buf, 0, 12500, 4, 32)
    _, parts, _ = product_bundles(vf, buf, 0, 12500, 4, 32, split=split)
    assert len(whole) == len(parts) > 0
    for (a0, a1), (b0, b1) in zip(whole, parts):
        assert np.array_equal(a0, b0) and np.array_equal(a1, b1)


def test_init_failure_matches_reference(tmp_path, vf, O):
    """Two stray pol-1 frames: the reference aborts initialisation (exit 2)."""
    from vlite_frb_b200 import synth
    buf = synth.make_vdif(synth.StreamSpec(duration=0.02, seed=1)).numpy()
    fr = buf.reshape(-1, 5032)
    bad = np.concatenate([fr[1], fr[1], buf])
    p = tmp_path / "bad.vdif"
    p.write_bytes(bad.tobytes())
    st_r, ref, _ = ref_bundles("pipe", str(p), 12500, 4, 32)
    st_p, prod, _ = product_bundles(vf, bad, 0, 12500, 4, 32)
    assert st_r == 2 and st_p == 2 and not ref and not prod


def _libc():
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    return libc


def test_sigproc_header_matches_reference_helpers(vf, O, tmp_path):
    """The reference's own send_string/send_int/send_double (PIPE:1177-1201)
    called in the order of PIPE:529-540 give the oracle's and the product's
    header bytes."""
    lib = _reflib("pipe")
    libc = _libc()
    ss = getattr(lib, "_Z11send_stringPKcP8_IO_FILE")
    si = getattr(lib, "_Z8send_intPKciP8_IO_FILE")
    sd = getattr(lib, "_Z11send_doublePKcdP8_IO_FILE")
    ss.argtypes = [C.c_char_p, C.c_void_p]
    si.argtypes = [C.c_char_p, C.c_int, C.c_void_p]
    sd.argtypes = [C.c_char_p, C.c_double, C.c_void_p]
    fch1, foff, nch, tstart, tsamp = 359.9949, -0.01024, 3908, 57083.6376284722, 0.000390625
    path = str(tmp_path / "x.head").encode()
    f = libc.fopen(path, b"wb")
    assert f
    ss(b"HEADER_START", f)
    si(b"barycentric", 1, f)
    si(b"telescope_id", 12, f)
    si(b"data_type", 1, f)
    sd(b"fch1", fch1, f)
    sd(b"foff", foff, f)
    si(b"nchans", nch, f)
    si(b"nbits", 32, f)
    sd(b"tstart", tstart, f)
    sd(b"tsamp", tsamp, f)
    si(b"nifs", 1, f)
    ss(b"HEADER_END", f)
    libc.fclose(f)
    ref = open(path, "rb").read()
    assert ref == O.sigproc_header(fch1, foff, nch, tstart, tsamp)
    plib = vf.lib()
    plib.vfrb_sigproc_header.restype = C.c_size_t
    plib.vfrb_sigproc_header.argtypes = [C.c_void_p, C.c_size_t, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                         C.c_double, C.c_double, C.c_int32]
    buf = (C.c_uint8 * len(ref))()
    assert plib.vfrb_sigproc_header(buf, len(ref), fch1, foff, nch, 32, tstart, tsamp, 1) == len(ref)
    assert bytes(buf) == ref


def test_presto_inf_matches_reference(vf, O, tmp_path):
    """writeprestoheader (TS:1483-1515) itself, against the oracle and the
    product."""
    lib = _reflib("ts")
    wp = getattr(lib, "_Z17writeprestoheaderPcdidfddid")
    wp.argtypes = [C.c_char_p, C.c_double, C.c_int, C.c_double, C.c_float, C.c_double, C.c_double, C.c_int,
                   C.c_double]
    wp.restype = C.c_int
    base = str(tmp_path / "DM119.3_2026-12-03_10:00:00")
    args = (60311.123456789012, 921600, 0.000390625, 119.3, 320.00512, 39.3216, 3840, 0.01024)
    assert wp(base.encode(), *args) == 0
    ref = open(base + ".inf").read()
    assert ref == O.presto_inf(base, *args)
    plib = vf.lib()
    plib.vfrb_presto_inf.restype = C.c_int
    plib.vfrb_presto_inf.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_double, C.c_int32, C.c_double,
                                     C.c_float, C.c_double, C.c_double, C.c_int32, C.c_double]
    buf = C.create_string_buffer(4096)
    assert plib.vfrb_presto_inf(buf, 4096, base.encode(), *args) == len(ref)
    assert buf.value.decode() == ref
