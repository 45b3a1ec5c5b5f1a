"""vlite-frb-b200: ctypes binding of libvfrb (the sm_100a FRB search chain).

The binding is thin: every call goes through the C ABI declared in
``include/vfrb.h``.  Device buffers are torch CUDA tensors (torch provides
device memory and streams only).  There is no CPU fallback: importing the
module on a machine without ``lib/libvfrb.so`` raises, and every stage call
raises ``VfrbError`` on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libvfrb.so")

VFRB_OK, VFRB_EOD, VFRB_ERR = 0, 1, 2
F32, F16, I8 = 0, 1, 2
DD_AUTO, DD_STAGED, DD_REG1, DD_REG2, DD_REG4, DD_DIRECT, DD_PAT4, DD_PAT2 = 0, 1, 2, 3, 4, 5, 6, 7
DD_NVARIANTS = 8


class VfrbError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib.vfrb_strerror(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({msg})")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libvfrb.so not built ({LIB_PATH}); run vlite-frb_b200/build.py")
    return C.CDLL(LIB_PATH)


_lib = None
_lib = _load()


def lib():
    return _lib


# ---- structures (mirror include/vfrb.h) --------------------------------------
class Hdr(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "seconds", "legacymode", "invalid", "frame", "epoch", "unassigned", "framelength8", "nchan_log2",
        "version", "stationid", "threadid", "nbits_minus1", "iscomplex", "eversion", "extended1",
        "extended2", "extended3", "extended4")]


class Layout(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "twonchan", "nchan", "nfreq", "nchanout", "nskip", "nave", "nbundle", "nloop", "maxnt", "nhalfcyc")] + [
        ("chanbw", C.c_double), ("fch1", C.c_double), ("foff", C.c_double), ("tchan", C.c_double),
        ("maxtime", C.c_float)]


class ChanArgs(C.Structure):
    _fields_ = [("frames", C.c_void_p), ("slots0", C.c_void_p), ("slots1", C.c_void_p), ("nslots", C.c_int64),
                ("sample0", C.c_int64), ("nrows", C.c_int32), ("twonchan", C.c_int32), ("nave", C.c_int32),
                ("nfreq", C.c_int32), ("nskip", C.c_int32), ("nchanout", C.c_int32), ("out", C.c_void_p),
                ("out_row_stride", C.c_int64), ("out_row0", C.c_int64), ("out_row_mask", C.c_uint32),
                ("d_err", C.c_void_p)]


class BpArgs(C.Structure):
    _fields_ = [("inp", C.c_void_p), ("in_row_stride", C.c_int64), ("in_row0", C.c_int64),
                ("in_row_mask", C.c_uint32), ("nchan", C.c_int32), ("nrows", C.c_int32), ("window", C.c_int32),
                ("storage", C.c_int32), ("out", C.c_void_p), ("out_chan_stride", C.c_int64),
                ("out_row0", C.c_int64), ("out_row_mask", C.c_uint32), ("inv_scale", C.c_void_p),
                ("q_scale", C.c_float), ("win_mean", C.c_void_p), ("win_var", C.c_void_p), ("tm_out", C.c_void_p),
                ("tm_row_stride", C.c_int64), ("d_err", C.c_void_p), ("subtract_mode", C.c_int32),
                ("out_shift1", C.c_void_p)]


class DdArgs(C.Structure):
    _fields_ = [("fb", C.c_void_p), ("storage", C.c_int32), ("chan_scale", C.c_void_p),
                ("uniform_scale", C.c_float), ("chan_stride", C.c_int64), ("row0", C.c_int64), ("row_mask", C.c_uint32),
                ("nrows_valid", C.c_int64), ("nt_out", C.c_int64), ("out", C.c_void_p), ("out_stride", C.c_int64),
                ("sigma_out", C.c_void_p), ("workspace", C.c_void_p), ("workspace_bytes", C.c_size_t),
                ("ave", C.c_void_p), ("sigma", C.c_void_p), ("peak", C.c_void_p), ("frb", C.c_void_p),
                ("argmax", C.c_void_p), ("d_err", C.c_void_p), ("fb_shift1", C.c_void_p)]


class CsArgs(C.Structure):
    _fields_ = [("fb", C.c_void_p), ("chan_stride", C.c_int64), ("row0", C.c_int64), ("row_mask", C.c_uint32),
                ("nchan", C.c_int32), ("nrows", C.c_int32), ("ncolstatblk", C.c_int32), ("nstatblks", C.c_int32),
                ("ave", C.c_void_p), ("sig", C.c_void_p), ("outlier", C.c_void_p)]


_lib.vfrb_strerror.restype = C.c_char_p
_lib.vfrb_strerror.argtypes = [C.c_int]
_lib.vfrb_decode_header.argtypes = [C.c_char_p, C.POINTER(Hdr)]
_lib.vfrb_header_dmjd.restype = C.c_double
_lib.vfrb_header_dmjd.argtypes = [C.POINTER(Hdr), C.c_int]
_lib.vfrb_layout_init.argtypes = [C.POINTER(Layout), C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_float]
_lib.vfrb_delay_table.argtypes = [C.POINTER(Layout), C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int32)]
for _n, _t in (("vfrb_channelise", ChanArgs), ("vfrb_bandpass", BpArgs), ("vfrb_chan_stats", CsArgs)):
    getattr(_lib, _n).argtypes = [C.POINTER(_t), C.c_void_p]
_lib.vfrb_ddplan_create.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_int]
_lib.vfrb_ddplan_destroy.argtypes = [C.c_void_p]
_lib.vfrb_ddplan_max_delay.argtypes = [C.c_void_p]
_lib.vfrb_ddplan_group_size.argtypes = [C.c_void_p]
_lib.vfrb_ddplan_set_variant.argtypes = [C.c_void_p, C.c_int, C.c_int]
_lib.vfrb_ddplan_variant.argtypes = [C.c_void_p, C.c_int]
_lib.vfrb_ddplan_autotune.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
_lib.vfrb_dedisperse_workspace_bytes.restype = C.c_size_t
_lib.vfrb_dedisperse_workspace_bytes.argtypes = [C.c_void_p, C.c_int64]
_lib.vfrb_dedisperse.argtypes = [C.c_void_p, C.POINTER(DdArgs), C.c_void_p]
_lib.vfrb_fb_to_time_major.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_uint32, C.c_int, C.c_int, C.c_void_p,
                                       C.c_int64, C.c_void_p]
_lib.vfrb_chan_sk.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                               C.c_void_p]
for _n in ("vfrb_subtract_bp_full", "vfrb_subtract_zero"):
    getattr(_lib, _n).argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_uint32, C.c_int, C.c_int64, C.c_void_p]


def _check(st: int, what: str):
    if st != 0:
        raise VfrbError(st, what)


# ---- host helpers -------------------------------------------------------------
def decode_header(b: bytes) -> dict:
    h = Hdr()
    _check(_lib.vfrb_decode_header(bytes(b[:32]), C.byref(h)), "vfrb_decode_header")
    return {n: getattr(h, n) for n, _ in Hdr._fields_}


def header_dmjd(b: bytes, fps: int = 25600) -> float:
    h = Hdr()
    _check(_lib.vfrb_decode_header(bytes(b[:32]), C.byref(h)), "vfrb_decode_header")
    return _lib.vfrb_header_dmjd(C.byref(h), fps)


def layout(twonchan=12500, nave=4, nbundle=32, muoslowfreq=360.0, nchanout_fixed=0, maxtime=70.0) -> Layout:
    L = Layout()
    _check(_lib.vfrb_layout_init(C.byref(L), twonchan, nave, nbundle, muoslowfreq, nchanout_fixed, maxtime),
           "vfrb_layout_init")
    return L


def delay_table(L: Layout, dms) -> tuple[np.ndarray, int]:
    d = np.ascontiguousarray(dms, dtype=np.float32)
    off = np.zeros((len(d), L.nchanout), np.int32)
    md = C.c_int32(0)
    _check(_lib.vfrb_delay_table(C.byref(L), d.ctypes.data, len(d), off.ctypes.data, C.byref(md)),
           "vfrb_delay_table")
    return off, int(md.value)


# ---- device stage wrappers (torch tensors) ---------------------------------------
def _torch():
    import torch  # noqa: WPS433  (torch only provides device memory and streams)
    return torch


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def contiguous_slots(nbytes_per_pol: int, device, base0: int = 0, base1: int | None = None):
    """Slot tables for two contiguous per-pol byte arrays (payloads back to back)."""
    torch = _torch()
    n = (nbytes_per_pol + 4999) // 5000
    s = torch.arange(n, dtype=torch.int64, device=device) * 5000
    return s + base0, s + (base1 if base1 is not None else base0)


def channelise(frames, slots0, slots1, sample0: int, nrows: int, L: Layout, out=None, out_row0=0,
               out_row_mask=0xFFFFFFFF, d_err=None, stream=None):
    torch = _torch()
    if out is None:
        out = torch.empty((nrows, L.nchanout), dtype=torch.float32, device=frames.device)
    a = ChanArgs(frames=frames.data_ptr(), slots0=slots0.data_ptr(), slots1=slots1.data_ptr(),
                 nslots=slots0.numel(), sample0=sample0, nrows=nrows, twonchan=L.twonchan, nave=L.nave,
                 nfreq=L.nfreq, nskip=L.nskip, nchanout=L.nchanout, out=out.data_ptr(),
                 out_row_stride=out.stride(0), out_row0=out_row0, out_row_mask=out_row_mask,
                 d_err=d_err.data_ptr() if d_err is not None else None)
    _check(_lib.vfrb_channelise(C.byref(a), _stream(stream)), "vfrb_channelise")
    return out


def bandpass(fb_tm, nrows=None, storage=F32, out=None, out_row0=0, out_row_mask=0xFFFFFFFF, inv_scale=None,
             q_scale=16.0, in_row0=0, in_row_mask=0xFFFFFFFF, window=128, win_mean=None, win_var=None,
             tm_out=None, d_err=None, subtract_mode=0, out_shift1=None, stream=None):
    torch = _torch()
    nrows = fb_tm.shape[0] if nrows is None else nrows
    nchan = fb_tm.shape[1]
    if out is None:
        dt = {F32: torch.float32, F16: torch.float16, I8: torch.int8}[storage]
        out = torch.empty((nchan, nrows), dtype=dt, device=fb_tm.device)
    a = BpArgs(inp=fb_tm.data_ptr(), in_row_stride=fb_tm.stride(0), in_row0=in_row0, in_row_mask=in_row_mask,
               nchan=nchan, nrows=nrows, window=window, storage=storage, out=out.data_ptr(),
               out_chan_stride=out.stride(0), out_row0=out_row0, out_row_mask=out_row_mask,
               inv_scale=_ptr(inv_scale), q_scale=q_scale, win_mean=_ptr(win_mean), win_var=_ptr(win_var),
               tm_out=_ptr(tm_out), tm_row_stride=tm_out.stride(0) if tm_out is not None else 0,
               d_err=_ptr(d_err), subtract_mode=subtract_mode, out_shift1=_ptr(out_shift1))
    _check(_lib.vfrb_bandpass(C.byref(a), _stream(stream)), "vfrb_bandpass")
    return out


def chan_sk(fb_tm, ncolstatblk, nstatblks, nsum, nrows=None, out=None, stream=None):
    """Spectral kurtosis per (channel, block of ncolstatblk rows) of a raw
    time-major FP32 FB (vfrb_chan_sk); returns [nstatblks][nchan] float32."""
    torch = _torch()
    nrows = fb_tm.shape[0] if nrows is None else nrows
    nchan = fb_tm.shape[1]
    if out is None:
        out = torch.empty((nstatblks, nchan), dtype=torch.float32, device=fb_tm.device)
    _check(_lib.vfrb_chan_sk(fb_tm.data_ptr(), fb_tm.stride(0), nchan, nrows, ncolstatblk, nstatblks, nsum,
                             out.data_ptr(), _stream(stream)), "vfrb_chan_sk")
    return out


def _rfi_call(fn, name, fb_cm, nrows, row0, row_mask, stream):
    if fb_cm.dtype != _torch().float32 or fb_cm.dim() != 2 or fb_cm.stride(1) != 1:
        raise ValueError(name + ": fb_cm must be a [nchan][rows] float32 tensor with unit row stride")
    nrows = fb_cm.shape[1] if nrows is None else nrows
    _check(fn(fb_cm.data_ptr(), fb_cm.stride(0), row0, row_mask, fb_cm.shape[0], nrows, _stream(stream)), name)
    return fb_cm


def subtract_bp_full(fb_cm, nrows=None, row0=0, row_mask=0xFFFFFFFF, stream=None):
    """In place: subtractbp (whole-block clipped channel mean, PIPE:1372-1424)."""
    return _rfi_call(_lib.vfrb_subtract_bp_full, "vfrb_subtract_bp_full", fb_cm, nrows, row0, row_mask, stream)


def subtract_zero(fb_cm, nrows=None, row0=0, row_mask=0xFFFFFFFF, stream=None):
    """In place: subtractZERO (per-row clipped mean across channels, PIPE:1478-1515)."""
    return _rfi_call(_lib.vfrb_subtract_zero, "vfrb_subtract_zero", fb_cm, nrows, row0, row_mask, stream)


class DedispPlan:
    """Device copy of a delay table [ndm][nchan] (vfrb_ddplan)."""

    def __init__(self, offsets: np.ndarray):
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        self.ndm, self.nchan = off.shape
        p = C.c_void_p()
        _check(_lib.vfrb_ddplan_create(C.byref(p), off.ctypes.data, self.ndm, self.nchan), "vfrb_ddplan_create")
        self._p = p
        self.max_delay = _lib.vfrb_ddplan_max_delay(p)
        self.group_size = _lib.vfrb_ddplan_group_size(p)

    def set_variant(self, storage: int, variant: int):
        _check(_lib.vfrb_ddplan_set_variant(self._p, storage, variant), "vfrb_ddplan_set_variant")

    def variant(self, storage: int = F32) -> int:
        return int(_lib.vfrb_ddplan_variant(self._p, storage))

    def autotune(self, storage: int, nt_out: int, stream=None):
        """Times each applicable kernel variant; returns {variant: ms} (n/a omitted)."""
        t = (C.c_float * DD_NVARIANTS)()
        _check(_lib.vfrb_ddplan_autotune(self._p, storage, nt_out, t, _stream(stream)), "vfrb_ddplan_autotune")
        return {i: t[i] for i in range(1, DD_NVARIANTS) if t[i] >= 0}

    def workspace_bytes(self, nt_out: int) -> int:
        return int(_lib.vfrb_dedisperse_workspace_bytes(self._p, nt_out))

    def __call__(self, fb_cm, nt_out: int, storage=F32, chan_scale=None, uniform_scale=0.0, row0=0, row_mask=0xFFFFFFFF,
                 nrows_valid=None, out=None, sigma_out=None, stats=True, workspace=None, d_err=None, fb_shift1=None,
                 stream=None):
        torch = _torch()
        dev = fb_cm.device
        if out is None:
            out = torch.empty((self.ndm, nt_out), dtype=torch.float32, device=dev)
        st = {}
        if stats:
            st = dict(ave=torch.empty(self.ndm, dtype=torch.float32, device=dev),
                      sigma=torch.empty(self.ndm, dtype=torch.float32, device=dev),
                      peak=torch.empty(self.ndm, dtype=torch.float32, device=dev),
                      frb=torch.empty(self.ndm, dtype=torch.int32, device=dev),
                      argmax=torch.empty(self.ndm, dtype=torch.int32, device=dev))
            if workspace is None:
                workspace = torch.empty(max(1, self.workspace_bytes(nt_out)), dtype=torch.uint8, device=dev)
        a = DdArgs(fb=fb_cm.data_ptr(), storage=storage, chan_scale=_ptr(chan_scale), uniform_scale=uniform_scale,
                   chan_stride=fb_cm.stride(0),
                   row0=row0, row_mask=row_mask,
                   nrows_valid=fb_cm.shape[1] if nrows_valid is None else nrows_valid, nt_out=nt_out,
                   out=out.data_ptr(), out_stride=out.stride(0), sigma_out=_ptr(sigma_out),
                   workspace=_ptr(workspace), workspace_bytes=workspace.numel() if workspace is not None else 0,
                   ave=_ptr(st.get("ave")), sigma=_ptr(st.get("sigma")), peak=_ptr(st.get("peak")),
                   frb=_ptr(st.get("frb")), argmax=_ptr(st.get("argmax")), d_err=_ptr(d_err),
                   fb_shift1=_ptr(fb_shift1))
        _check(_lib.vfrb_dedisperse(self._p, C.byref(a), _stream(stream)), "vfrb_dedisperse")
        return out, st

    def __del__(self):
        try:
            if getattr(self, "_p", None):
                _lib.vfrb_ddplan_destroy(self._p)
                self._p = None
        except Exception:
            pass


_lib.vfrb_boxcar.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.c_void_p]


def boxcar(dd, ave, sigma, max_width: int, nt=None, stream=None):
    """Best boxcar per trial over widths 1..max_width (vfrb_boxcar): (snr, start, width) device tensors."""
    torch = _torch()
    ndm = dd.shape[0]
    nt = dd.shape[1] if nt is None else nt
    snr = torch.empty(ndm, dtype=torch.float32, device=dd.device)
    start = torch.empty(ndm, dtype=torch.int32, device=dd.device)
    width = torch.empty(ndm, dtype=torch.int32, device=dd.device)
    _check(_lib.vfrb_boxcar(dd.data_ptr(), ndm, nt, dd.stride(0), ave.data_ptr(), sigma.data_ptr(), max_width,
                            snr.data_ptr(), start.data_ptr(), width.data_ptr(), _stream(stream)), "vfrb_boxcar")
    return snr, start, width


def chan_stats(fb_cm, nrows: int, ncolstatblk: int, nstatblks: int, row0=0, row_mask=0xFFFFFFFF, stream=None):
    torch = _torch()
    nchan = fb_cm.shape[0]
    dev = fb_cm.device
    ave = torch.empty((nstatblks, nchan), dtype=torch.float32, device=dev)
    sig = torch.empty_like(ave)
    outl = torch.empty_like(ave)
    a = CsArgs(fb=fb_cm.data_ptr(), chan_stride=fb_cm.stride(0), row0=row0, row_mask=row_mask, nchan=nchan,
               nrows=nrows, ncolstatblk=ncolstatblk, nstatblks=nstatblks, ave=ave.data_ptr(), sig=sig.data_ptr(),
               outlier=outl.data_ptr())
    _check(_lib.vfrb_chan_stats(C.byref(a), _stream(stream)), "vfrb_chan_stats")
    return ave, sig, outl


def fb_to_time_major(fb_cm, nrows=None, row0=0, row_mask=0xFFFFFFFF, out=None, stream=None):
    torch = _torch()
    nchan = fb_cm.shape[0]
    nrows = fb_cm.shape[1] if nrows is None else nrows
    if out is None:
        out = torch.empty((nrows, nchan), dtype=torch.float32, device=fb_cm.device)
    _check(_lib.vfrb_fb_to_time_major(fb_cm.data_ptr(), fb_cm.stride(0), row0, row_mask, nchan, nrows,
                                      out.data_ptr(), out.stride(0), _stream(stream)), "vfrb_fb_to_time_major")
    return out


# ---- plan / stream API -------------------------------------------------------------
MODE_BLOCK, MODE_STREAM = 0, 1
READER_PIPE, READER_TS = 0, 1
OUT_DEDISP, OUT_DMSTATS, OUT_SIGMA, OUT_CHANSTATS, OUT_FB, OUT_CANDS, OUT_FLAGS = 1, 2, 4, 8, 16, 32, 64
ROW_INVALID, ROW_FILL = 1, 2
BP_CAL, BP_FULL = 0, 1
VFRB_PENDING = 9
ERR_NOMEM = 6


class Params(C.Structure):
    _fields_ = [("twonchan", C.c_int32), ("nave", C.c_int32), ("nbundle", C.c_int32), ("muoslowfreq", C.c_double),
                ("nchanout_fixed", C.c_int32), ("maxtime", C.c_float), ("timestats", C.c_float),
                ("dms", C.c_void_p), ("ndm", C.c_int32), ("mode", C.c_int32), ("reader", C.c_int32),
                ("dada_skip", C.c_int32), ("storage", C.c_int32), ("q_scale", C.c_float), ("outputs", C.c_int32),
                ("fb_block", C.c_int32), ("nstreams", C.c_int32), ("chunk_seconds", C.c_float),
                ("ring_seconds", C.c_float), ("cand_snr", C.c_float), ("device", C.c_int32),
                ("device_bytes", C.c_int64), ("boxcar_max", C.c_int32), ("bp_mode", C.c_int32),
                ("zero_dm", C.c_int32), ("batch_streams", C.c_int32)]


class Cand(C.Structure):
    _fields_ = [("dm_index", C.c_int32), ("width", C.c_int32), ("t", C.c_int64), ("snr", C.c_float),
                ("dm", C.c_float)]


class Result(C.Structure):
    _fields_ = [("stream", C.c_int32), ("seq", C.c_int64), ("row0", C.c_int64), ("tstart_mjd", C.c_double),
                ("ndm", C.c_int32), ("nt", C.c_int64), ("dd", C.c_void_p), ("dd_sigma", C.c_void_p),
                ("ave", C.c_void_p), ("sigma", C.c_void_p), ("peak", C.c_void_p), ("frb", C.c_void_p),
                ("argmax", C.c_void_p), ("nchan", C.c_int32), ("fb_rows", C.c_int64), ("fb", C.c_void_p),
                ("nstatblks", C.c_int32), ("chan_ave", C.c_void_p), ("chan_sig", C.c_void_p),
                ("chan_outlier", C.c_void_p), ("ncand", C.c_int32), ("cands", C.c_void_p),
                ("latency_ms", C.c_double), ("device_errors", C.c_int32), ("box_snr", C.c_void_p),
                ("box_start", C.c_void_p), ("box_width", C.c_void_p), ("chan_sk", C.c_void_p),
                ("nflag_rows", C.c_int64), ("row_flags", C.c_void_p)]


_lib.vfrb_cluster_cands.argtypes = [C.POINTER(Cand), C.c_int32, C.c_int32, C.c_int64, C.POINTER(Cand),
                                    C.POINTER(C.c_int32), C.c_void_p]


def cluster_cands(cands, dm_tol=2, t_tol=0):
    """Friends-of-friends clustering of candidate dicts (dm_index, t, width,
    snr, dm) across trials and time (vfrb_cluster_cands).  Returns
    (clusters, labels): one dict per cluster -- its brightest member -- and
    the cluster index of each input."""
    n = len(cands)
    arr = (Cand * max(n, 1))()
    for i, c in enumerate(cands):
        arr[i] = Cand(dm_index=c["dm_index"], width=c["width"], t=c["t"], snr=c["snr"], dm=c.get("dm", 0.0))
    out = (Cand * max(n, 1))()
    nout = C.c_int32(0)
    lab = np.zeros(max(n, 1), np.int32)
    _check(_lib.vfrb_cluster_cands(arr, n, dm_tol, t_tol, out, C.byref(nout), lab.ctypes.data), "vfrb_cluster_cands")
    cl = [dict(dm_index=o.dm_index, width=o.width, t=o.t, snr=o.snr, dm=o.dm) for o in out[:nout.value]]
    return cl, lab[:n]


_lib.vfrb_params_default.argtypes = [C.POINTER(Params)]
_lib.vfrb_plan_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Params)]
_lib.vfrb_plan_destroy.argtypes = [C.c_void_p]
_lib.vfrb_plan_layout.argtypes = [C.c_void_p, C.POINTER(Layout), C.POINTER(C.c_int32)]
_lib.vfrb_plan_device_bytes.restype = C.c_int64
_lib.vfrb_plan_device_bytes.argtypes = [C.c_void_p]
_lib.vfrb_push_frames.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
_lib.vfrb_poll.argtypes = [C.c_void_p, C.POINTER(Result), C.c_int]
_lib.vfrb_stream_open.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
_lib.vfrb_stream_close.argtypes = [C.c_void_p, C.c_int]
_lib.vfrb_stream_log.restype = C.c_char_p
_lib.vfrb_stream_log.argtypes = [C.c_void_p, C.c_int]


def _arr(ptr, n, dt):
    if not ptr or n <= 0:
        return None
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(dt)), shape=(n,)).copy()


class Plan:
    """vfrb_plan: push raw VDIF bytes per stream, poll results (host copies)."""

    def __init__(self, dms=None, **kw):
        p = Params()
        _lib.vfrb_params_default(C.byref(p))
        self._dms = None
        if dms is not None:
            self._dms = np.ascontiguousarray(dms, dtype=np.float32)
            p.dms = self._dms.ctypes.data
            p.ndm = len(self._dms)
        for k, v in kw.items():
            if not hasattr(p, k):
                raise TypeError(f"unknown parameter {k}")
            setattr(p, k, v)
        self.params = p
        h = C.c_void_p()
        _check(_lib.vfrb_plan_create(C.byref(h), C.byref(p)), "vfrb_plan_create")
        self._h = h
        self.layout = Layout()
        md = C.c_int32(0)
        _check(_lib.vfrb_plan_layout(h, C.byref(self.layout), C.byref(md)), "vfrb_plan_layout")
        self.max_delay = md.value

    @property
    def device_bytes(self):
        return int(_lib.vfrb_plan_device_bytes(self._h))

    def open_stream(self):
        """Admit one more stream (vfrb_stream_open); returns its id, or None
        when its device memory does not fit the budget now."""
        i = C.c_int(-1)
        st = _lib.vfrb_stream_open(self._h, C.byref(i))
        if st == ERR_NOMEM:
            return None
        _check(st, "vfrb_stream_open")
        return i.value

    def close_stream(self, stream: int) -> bool:
        """End a stream and free it once its results are polled
        (vfrb_stream_close): True when freed, False while results remain."""
        st = _lib.vfrb_stream_close(self._h, stream)
        if st == VFRB_PENDING:
            return False
        _check(st, "vfrb_stream_close")
        return True

    def push(self, stream: int, data):
        """data: bytes / numpy uint8 / torch uint8 tensor -- CPU (pinned or not)
        or CUDA (device-resident frames are copied on the device, only their
        headers go to the host); None = end of data."""
        if data is None:
            _check(_lib.vfrb_push_frames(self._h, stream, None, 0), "vfrb_push_frames")
            return
        if hasattr(data, "data_ptr"):
            ptr, n = data.data_ptr(), data.numel()
        else:
            a = np.ascontiguousarray(np.frombuffer(data, np.uint8) if isinstance(data, (bytes, bytearray)) else data)
            ptr, n = a.ctypes.data, a.nbytes
            self._keep = a
        _check(_lib.vfrb_push_frames(self._h, stream, C.c_void_p(ptr), n), "vfrb_push_frames")

    def poll(self, wait=True, copy=True):
        r = Result()
        st = _lib.vfrb_poll(self._h, C.byref(r), 1 if wait else 0)
        if st in (VFRB_EOD, VFRB_PENDING):
            return None
        _check(st, "vfrb_poll")
        if not copy:
            return r
        ndm, nt, nch = r.ndm, r.nt, r.nchan
        out = dict(stream=r.stream, seq=r.seq, row0=r.row0, tstart_mjd=r.tstart_mjd, ndm=ndm, nt=nt,
                   latency_ms=r.latency_ms, device_errors=r.device_errors, nstatblks=r.nstatblks)
        dd = _arr(r.dd, ndm * nt, C.c_float)
        out["dd"] = dd.reshape(ndm, nt) if dd is not None else None
        ds = _arr(r.dd_sigma, ndm * nt, C.c_float)
        out["dd_sigma"] = ds.reshape(ndm, nt) if ds is not None else None
        for k, dt in (("ave", C.c_float), ("sigma", C.c_float), ("peak", C.c_float), ("frb", C.c_int32),
                      ("argmax", C.c_int32), ("box_snr", C.c_float), ("box_start", C.c_int32),
                      ("box_width", C.c_int32)):
            out[k] = _arr(getattr(r, k), ndm, dt)
        fb = _arr(r.fb, r.fb_rows * nch, C.c_float)
        out["fb"] = fb.reshape(r.fb_rows, nch) if fb is not None else None
        for k in ("chan_ave", "chan_sig", "chan_outlier", "chan_sk"):
            a = _arr(getattr(r, k), r.nstatblks * nch, C.c_float)
            out[k] = a.reshape(r.nstatblks, nch) if a is not None else None
        out["row_flags"] = _arr(r.row_flags, r.nflag_rows, C.c_uint8)
        cands = []
        if r.ncand and r.cands:
            ca = C.cast(r.cands, C.POINTER(Cand))
            for i in range(r.ncand):
                c = ca[i]
                cands.append(dict(dm_index=c.dm_index, width=c.width, t=c.t, snr=c.snr, dm=c.dm))
        out["cands"] = cands
        return out

    def drain(self):
        res = []
        while True:
            r = self.poll(wait=True)
            if r is None:
                return res
            res.append(r)

    def log(self, stream=0) -> str:
        return _lib.vfrb_stream_log(self._h, stream).decode()

    def close(self):
        if getattr(self, "_h", None):
            _lib.vfrb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
