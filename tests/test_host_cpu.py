"""CPU-only checks: the C-ABI library loads and exports every declared symbol,
and its host-side arithmetic (header decode, MJD, layout, delay table)
matches the oracle exactly."""
import ctypes
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    txt = open(os.path.join(ROOT, "include", "vfrb.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vfrb_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(vf):
    names = _declared_functions()
    assert len(names) >= 14
    lib = ctypes.CDLL(vf.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_header_decode_matches_oracle(vf, O):
    rng = np.random.default_rng(0)
    for _ in range(200):
        b = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        a = vf.decode_header(b)
        o = O.decode_header(b)
        assert a["seconds"] == o["seconds"] and a["frame"] == o["frame"] and a["epoch"] == o["epoch"]
        assert a["threadid"] == o["threadid"] and a["invalid"] == o["invalid"] and a["legacymode"] == o["legacymode"]
        assert a["framelength8"] == o["framelength8"] and a["nbits_minus1"] == o["nbits"]
        assert a["stationid"] == o["stationid"] and a["iscomplex"] == o["iscomplex"]
        assert a["extended1"] == o["extended1"] and a["extended4"] == o["extended4"]
        assert vf.header_dmjd(b) == O.vdif_dmjd(o)


def test_header_roundtrip_known_values(vf, O):
    b = O.encode_header(seconds=12345678, frame=25599, epoch=33, framelength8=629, threadid=1, nbits=7,
                        stationid=0x5858, invalid=1)
    h = vf.decode_header(b)
    assert (h["seconds"], h["frame"], h["epoch"], h["threadid"], h["invalid"]) == (12345678, 25599, 33, 1, 1)
    # epoch 33 = 2016-07-01 (MJD 57570); 12345678 s = 142 d + 76878 s
    assert abs(vf.header_dmjd(b) - (57570 + 142 + 76878 / 86400 + 25599 / (25600 * 86400))) < 1e-9


@pytest.mark.parametrize("twonchan,nave,nb,muos,fixed,maxtime", [
    (12500, 4, 32, 360.0, 0, 70.0), (12500, 10, 32, 384.0, 0, 60.0), (12500, 4, 32, 360.0, 3840, 30.0),
    (12500, 4, 32, 360.0, 0, 60.0), (8000, 3, 16, 360.0, 0, 7.5), (12500, 10, 32, 384.0, 0, 7.5)])
def test_layout_matches_oracle(vf, O, twonchan, nave, nb, muos, fixed, maxtime):
    L = vf.layout(twonchan, nave, nb, muos, fixed, maxtime)
    o = O.Layout(twonchan=twonchan, nave=nave, nbundle=nb, muoslowfreq=muos, maxtime=maxtime,
                 nchanout_fixed=fixed or None)
    for k in ("nchan", "nfreq", "nchanout", "nskip", "nloop", "maxnt", "nhalfcyc"):
        assert getattr(L, k) == getattr(o, k), k
    for k in ("chanbw", "fch1", "foff", "tchan"):
        assert getattr(L, k) == getattr(o, k), k


def test_layout_reference_values(vf):
    L = vf.layout(12500, 10, 32, 384.0, 0, 60.0)
    assert (L.nchanout, L.nskip, L.maxnt) == (6250, 1, 61440)
    assert abs(L.fch1 - 383.99488) < 1e-9 and abs(L.tchan - 0.0009765625) < 1e-15
    L = vf.layout(12500, 4, 32, 360.0, 0, 70.0)
    assert (L.nchanout, L.nskip, L.maxnt, L.nhalfcyc) == (3908, 2343, 179200, 1400)


def test_delay_table_matches_oracle(vf, O):
    L = vf.layout(12500, 10, 32, 384.0, 0, 60.0)
    dms = np.linspace(0, 1000, 2048).astype(np.float32)[::97]
    off, md = vf.delay_table(L, dms)
    o_off, o_md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    assert np.array_equal(off, o_off) and md == o_md
    # TS: DM {0, 119.3}, 3840 channels (TS:441-464)
    L = vf.layout(12500, 4, 32, 360.0, 3840, 30.0)
    off, md = vf.delay_table(L, np.array([0.0, 119.3], np.float32))
    o_off, o_md = O.delay_table(np.array([0.0, 119.3], np.float32), L.fch1, L.chanbw, L.tchan, L.nchanout)
    assert np.array_equal(off, o_off) and md == o_md and off[0].max() == 0


def test_dm1000_sweep(vf):
    L = vf.layout(12500, 10, 32, 384.0, 0, 60.0)
    off, md = vf.delay_table(L, np.array([1000.0], np.float32))
    assert 12600 < md < 12700 and off.max() <= md


@pytest.mark.parametrize("fch1,foff,nch,tstart,tsamp", [(359.9949, -0.01024, 3908, 57083.6376284722, 0.000390625),
                                                        (383.99488, -0.01024, 6250, 60311.25, 0.0009765625)])
def test_sigproc_header_matches_oracle(vf, O, fch1, foff, nch, tstart, tsamp):
    lib = vf.lib()
    lib.vfrb_sigproc_header.restype = C.c_size_t
    lib.vfrb_sigproc_header.argtypes = [C.c_void_p, C.c_size_t, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                        C.c_double, C.c_double, C.c_int32]
    n = lib.vfrb_sigproc_header(None, 0, fch1, foff, nch, 32, tstart, tsamp, 1)
    buf = (C.c_uint8 * n)()
    assert lib.vfrb_sigproc_header(buf, n, fch1, foff, nch, 32, tstart, tsamp, 1) == n
    assert bytes(buf) == O.sigproc_header(fch1, foff, nch, tstart, tsamp)


def test_presto_inf_matches_oracle(vf, O):
    lib = vf.lib()
    lib.vfrb_presto_inf.restype = C.c_int
    lib.vfrb_presto_inf.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_double, C.c_int32, C.c_double,
                                    C.c_float, C.c_double, C.c_double, C.c_int32, C.c_double]
    args = (b"DM119.3_2026-12-03_10:00:00", 60311.123456789012, 921600, 0.000390625, 119.3, 320.00512, 39.3216,
            3840, 0.01024)
    n = lib.vfrb_presto_inf(None, 0, *args)
    buf = C.create_string_buffer(n + 1)
    assert lib.vfrb_presto_inf(buf, n + 1, *args) == n
    want = O.presto_inf(args[0].decode(), *args[1:])
    assert buf.value.decode() == want
    assert lib.vfrb_presto_inf(None, 0, None, *args[1:]) == -1


@pytest.mark.parametrize("kw,status", [
    (dict(bp_mode=2), 4),                                      # unknown bandpass mode: VFRB_ERR_ARG
    (dict(zero_dm=3), 4),
    (dict(bp_mode=1, mode=1), 5),                              # whole-block modes: block mode only
    (dict(zero_dm=1, mode=1), 5),
    (dict(bp_mode=1, storage=1), 5),                           # ... and FP32 storage only
    (dict(zero_dm=1, storage=2), 5),
])
def test_plan_rejects_unsupported_rfi_modes(vf, kw, status):
    """Parameter checks run before any CUDA call, so they need no GPU."""
    with pytest.raises(vf.VfrbError) as e:
        vf.Plan(np.array([0.0, 10.0], np.float32), **kw)
    assert e.value.status == status


def test_cluster_cands_known_answer(vf):
    c = [dict(dm_index=10, t=1000, width=4, snr=9.0), dict(dm_index=11, t=1002, width=1, snr=12.0),
         dict(dm_index=13, t=1001, width=2, snr=7.0),   # within 2 trials of 11: joins through it
         dict(dm_index=30, t=1000, width=1, snr=8.0),   # far in DM: its own cluster
         dict(dm_index=10, t=1010, width=1, snr=6.5),   # 6 samples after 1000+4: apart for t_tol 5
         dict(dm_index=12, t=900, width=1, snr=6.0)]
    cl, lab = vf.cluster_cands(c, dm_tol=2, t_tol=5)
    assert [(x["dm_index"], x["t"], x["snr"]) for x in cl] == [(12, 900, 6.0), (30, 1000, 8.0), (11, 1002, 12.0),
                                                             (10, 1010, 6.5)]
    assert list(lab) == [2, 2, 2, 1, 3, 0]
    cl, lab = vf.cluster_cands(c, dm_tol=2, t_tol=6)  # gap 1010 - 1004 = 6: now friends
    assert len(cl) == 3 and lab[4] == lab[0]
    cl, lab = vf.cluster_cands([], 2, 5)
    assert cl == [] and len(lab) == 0
    with pytest.raises(vf.VfrbError):
        vf.cluster_cands(c, dm_tol=-1)
    with pytest.raises(vf.VfrbError):
        vf.cluster_cands([dict(dm_index=0, t=0, width=0, snr=7.0)])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_cluster_cands_matches_oracle(vf, O, seed):
    rng = np.random.default_rng(seed)
    n = 300
    c = [dict(dm_index=int(rng.integers(0, 60)), t=int(rng.integers(0, 4000)), width=int(2 ** rng.integers(0, 5)),
              snr=float(np.float32(rng.integers(60, 90) / 8.0))) for _ in range(n)]  # repeated SNRs: tie rules
    for dm_tol, t_tol in ((0, 0), (2, 8), (5, 40)):
        cl, lab = vf.cluster_cands(c, dm_tol=dm_tol, t_tol=t_tol)
        tup = [(x["dm_index"], x["t"], x["width"], x["snr"]) for x in c]
        ocl, olab = O.cluster_cands(tup, dm_tol, t_tol)
        assert [(x["dm_index"], x["t"], x["width"], x["snr"]) for x in cl] == ocl
        assert list(lab) == olab


def test_cluster_cands_in_place(vf):
    """The output array may be the input array (clusters written in place)."""
    import ctypes as C
    rng = np.random.default_rng(11)
    n = 200
    arr = (vf.Cand * n)()
    for i in range(n):
        arr[i] = vf.Cand(dm_index=int(rng.integers(0, 40)), width=int(2 ** rng.integers(0, 4)),
                         t=int(rng.integers(0, 3000)), snr=float(rng.integers(60, 90) / 8.0), dm=0.0)
    cands = [dict(dm_index=a.dm_index, width=a.width, t=a.t, snr=a.snr) for a in arr]
    want, _ = vf.cluster_cands(cands, dm_tol=3, t_tol=20)
    nout = C.c_int32(0)
    lib = vf.lib()
    assert lib.vfrb_cluster_cands(arr, n, 3, 20, arr, C.byref(nout), None) == 0
    got = [dict(dm_index=a.dm_index, width=a.width, t=a.t, snr=a.snr, dm=a.dm) for a in arr[:nout.value]]
    assert got == want
