"""FP64 CPU oracle for the vlite-frb FRB search chain.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may.
It restates, in numpy FP64, every stage of the reference's hot path, each
function citing the reference file:line it follows (paths are relative to the
paulray/vlite-frb checkout):

  PIPE  = vdifFILE2dedisp_PIPELINE.cu
  STATS = vdifDADA2stats.cu
  TS    = vdifDADA2timeseries.cu

Parity pinning.  The reference ships no tests, fixtures or golden vectors.  The
oracle is pinned against the reference itself: ``oracle/build_ref.py`` compiles
the reference's own .cu sources (in place, read-only) into ``oracle/_ref/``
together with project-written stand-ins for the absent psrdada/dedisp/vdifio
pieces, and ``tests/test_ref_pin.py`` runs the reference's host frame reader on
the CPU and the reference's kernels + cuFFT on the GPU against this module.
The dedisp library called at PIPE:671 is not vendored: its semantics are
unpinned, and the reference's own in-tree ``dedisperse`` kernel (PIPE:1517)
with the TS:454-464 delay table stands in for it.
"""
from __future__ import annotations

import datetime
import math
from dataclasses import dataclass, field

import numpy as np

# --- constants (PIPE:33-47, STATS:35-45, TS:34-48, TS:457) -----------------
FRAMELEN = 5032
HDRLEN = 32
DATALEN = 5000
FRAMESPERSEC = 25600
VLITERATE = 128e6
VLITEBW = 64.0
VLITELOWFREQ = 320.0
DELAY_CONST = 4.148808e3
NFRAMEDADAINIT = 256000  # TS:74


# --- a1: VDIF header decode (vdifio.h:53-72, gcc little-endian bitfields) ---
def decode_header(b) -> dict:
    w = [int(x) for x in np.frombuffer(bytes(b[:32]), dtype="<u4")]
    return dict(
        seconds=w[0] & 0x3FFFFFFF, legacymode=(w[0] >> 30) & 1, invalid=(w[0] >> 31) & 1,
        frame=w[1] & 0xFFFFFF, epoch=(w[1] >> 24) & 0x3F, unassigned=(w[1] >> 30) & 3,
        framelength8=w[2] & 0xFFFFFF, nchan=(w[2] >> 24) & 0x1F, version=(w[2] >> 29) & 7,
        stationid=w[3] & 0xFFFF, threadid=(w[3] >> 16) & 0x3FF, nbits=(w[3] >> 26) & 0x1F,
        iscomplex=(w[3] >> 31) & 1, eversion=w[4] & 0xFF, extended1=(w[4] >> 8) & 0xFFFFFF,
        extended2=w[5], extended3=w[6], extended4=w[7])


def encode_header(**f) -> bytes:
    """Inverse of decode_header (used to build fixtures)."""
    g = lambda k: int(f.get(k, 0))
    w0 = (g("seconds") & 0x3FFFFFFF) | (g("legacymode") & 1) << 30 | (g("invalid") & 1) << 31
    w1 = (g("frame") & 0xFFFFFF) | (g("epoch") & 0x3F) << 24 | (g("unassigned") & 3) << 30
    w2 = (g("framelength8") & 0xFFFFFF) | (g("nchan") & 0x1F) << 24 | (g("version") & 7) << 29
    w3 = (g("stationid") & 0xFFFF) | (g("threadid") & 0x3FF) << 16 | (g("nbits") & 0x1F) << 26 | (g("iscomplex") & 1) << 31
    w4 = (g("eversion") & 0xFF) | (g("extended1") & 0xFFFFFF) << 8
    return np.array([w0, w1, w2, w3, w4, g("extended2"), g("extended3"), g("extended4")], dtype="<u4").tobytes()


# --- a2: getVDIFDMJD (declared vdifio.h:87; body not vendored) --------------
def vdif_dmjd(h: dict, framepersec: int = FRAMESPERSEC) -> float:
    """Restated from the VDIF specification: ``epoch`` counts 6-month periods
    from 2000-01-01 00:00 UTC and ``seconds`` counts from the epoch start.
    MJD = MJD(epoch start) + seconds div 86400 + (seconds mod 86400)/86400
    + frame/(framepersec*86400), summed in that order in double."""
    year = 2000 + h["epoch"] // 2
    month = 1 + 6 * (h["epoch"] % 2)
    mjd_epoch = datetime.date(year, month, 1).toordinal() - datetime.date(1858, 11, 17).toordinal()
    imjd = mjd_epoch + h["seconds"] // 86400
    return float(imjd) + (h["seconds"] % 86400) / 86400.0 + h["frame"] / (framepersec * 86400.0)


# --- parameter derivation (PIPE:289-303; STATS:208-231; TS:277-298) ---------
@dataclass
class Layout:
    twonchan: int = 12500
    nave: int = 4
    nbundle: int = 32
    muoslowfreq: float = 360.0
    maxtime: float = 70.0
    nchanout_fixed: int | None = None  # TS hard-codes 3840 (TS:282)
    nchan: int = field(init=False)
    nfreq: int = field(init=False)
    chanbw: float = field(init=False)
    nchanout: int = field(init=False)
    nskip: int = field(init=False)
    nloop: int = field(init=False)
    fch1: float = field(init=False)
    foff: float = field(init=False)
    tchan: float = field(init=False)
    maxnt: int = field(init=False)
    nhalfcyc: int = field(init=False)

    def __post_init__(self):
        self.nchan = int(0.5 * self.twonchan)
        self.nfreq = self.nchan + 1
        self.chanbw = VLITEBW / self.nchan
        if self.nchanout_fixed is None:
            n = int((self.muoslowfreq - VLITELOWFREQ) / self.chanbw) + 1
            if n % 2 == 1:
                n += 1
        else:
            n = int(self.nchanout_fixed)
        self.nchanout = n
        self.nskip = (self.nchan - self.nchanout) + 1
        self.nloop = self.nbundle * self.nave * self.twonchan
        self.foff = -1.0 * self.chanbw
        self.fch1 = (VLITELOWFREQ + (self.nchanout * self.chanbw)) - (0.5 * self.chanbw)
        self.tchan = float(self.nave * self.twonchan) / VLITERATE
        # MAXTIME is a C float (PIPE:50); float/double is done in double.
        self.maxnt = int(float(np.float32(self.maxtime)) / self.tchan)
        self.nhalfcyc = self.maxnt // 128 + (1 if self.maxnt % 128 else 0)


# --- a3/a4: pol-pair frame reader (PIPE:829-1171; TS:829-1180) --------------
class RefPairReader:
    """Restates the reference's single-file pol-pair reader.

    mode 'pipe' (PIPE/STATS): a gap is (frame - expected) mod 25600
    (PIPE:888-930).  mode 'ts': the gap also counts seconds (TS:895-937).
    Fill frames hold byte 0 (PIPE:1044-1052).  The invalid bit is ignored.
    """

    def __init__(self, data, mode: str = "pipe"):
        self.buf = memoryview(bytes(data)) if not isinstance(data, memoryview) else data
        self.pos = 0
        self.mode = mode
        self.hdr = [None, None]
        self.data = [bytes(DATALEN), bytes(DATALEN)]
        self.tmp = [bytes(DATALEN), bytes(DATALEN)]
        self.nskip = [0, 0]
        self.expected = [0, 0]
        self.expsec = [0, 0]
        self.npartfill = 0
        self.npartleft = 0
        self.flag_eof = 1
        self.log: list[str] = []
        # row-flag bookkeeping (new-build extension; the reference ignores the
        # invalid bit): flag of the payload in data[p] / tmp[p] (1 = its
        # header had the invalid bit, 2 = zero fill), and per pair made
        # current (pair k = pol bytes [5000k, 5000(k+1))) the OR of both pols
        self.dflag = [0, 0]
        self.tflag = [0, 0]
        self.pair_flags: list[int] = []

    # fread of a header then a payload (PIPE:829-883)
    def _raw_read(self, p) -> int:
        if self.pos + HDRLEN > len(self.buf):
            self.pos = len(self.buf)
            self.flag_eof = 0
            return 1
        self.hdr[p] = decode_header(self.buf[self.pos:self.pos + HDRLEN])
        self.pos += HDRLEN
        if self.pos + DATALEN > len(self.buf):
            self.pos = len(self.buf)
            self.flag_eof = 0
            return 1
        self.data[p] = bytes(self.buf[self.pos:self.pos + DATALEN])
        self.pos += DATALEN
        self.dflag[p] = self.hdr[p]["invalid"]
        return 0

    def _checkframeskip(self, p):  # PIPE:888-930 / TS:895-937
        h = self.hdr[p]
        fnum = h["frame"]
        if self.mode == "ts":
            fsec = h["seconds"]
            if fnum != self.expected[p] or fsec != self.expsec[p]:
                self.nskip[p] = fnum - self.expected[p] + (fsec - self.expsec[p]) * FRAMESPERSEC
                self.tmp[p] = self.data[p]
                self.data[p] = bytes(DATALEN)
                self.tflag[p], self.dflag[p] = self.dflag[p], 2
                self.log.append(f"skip{p} {self.nskip[p]}")
            self.expected[p] = (fnum + 1) % FRAMESPERSEC
            self.expsec[p] = fsec + (1 if self.expected[p] == 0 else 0)
        else:
            if fnum != self.expected[p]:
                n = fnum - self.expected[p]
                if n < 0:
                    n += FRAMESPERSEC
                self.nskip[p] = n
                self.tmp[p] = self.data[p]
                self.data[p] = bytes(DATALEN)
                self.tflag[p], self.dflag[p] = self.dflag[p], 2
                self.log.append(f"skip{p} {n}")
            self.expected[p] = (fnum + 1) % FRAMESPERSEC

    def _readone(self, p) -> int:  # PIPE:934-1025
        if self.nskip[p]:
            self.nskip[p] -= 1
            if self.nskip[p] == 0:
                self.data[p] = self.tmp[p]
                self.dflag[p] = self.tflag[p]
            return 0
        if self._raw_read(p):
            return 1
        self._checkframeskip(p)
        return 0

    def readtwoframe(self) -> int:  # PIPE:1031-1040
        st = self._readone(0) or self._readone(1)
        if not st:
            self.pair_flags.append(self.dflag[0] | self.dflag[1])
        return st

    def init_dada(self) -> int:  # TS:767-826 (discard NFRAMEDADAINIT pairs)
        for _ in range(NFRAMEDADAINIT):
            if self._raw_read(0) or self._raw_read(1):
                return 1
        return 0

    def initframe01(self) -> int:  # PIPE:1058-1131, TS:1070-1145
        self.pair_flags = []
        if self._raw_read(0):
            return 1
        if self.hdr[0]["threadid"] != 0:
            if self._raw_read(0):
                return 1
        if self.hdr[0]["threadid"] != 0:
            return 1
        if self._raw_read(1):
            return 1
        if self.hdr[1]["threadid"] != 1:
            return 1
        ts = self.mode == "ts"
        fnum0, fnum1 = self.hdr[0]["frame"], self.hdr[1]["frame"]
        if fnum0 != fnum1 or (ts and self.hdr[0]["seconds"] != self.hdr[1]["seconds"]):
            return 2 if ts else 1
        while fnum0 % 2560 != 0:  # fmod((float)fnum0, 2560.f) < 1e-4 is exact below 2^24
            if self._raw_read(0) or self._raw_read(1):
                return 1
            fnum0 = self.hdr[0]["frame"]
        fnum1 = self.hdr[1]["frame"]
        if fnum0 != fnum1 or (ts and self.hdr[0]["seconds"] != self.hdr[1]["seconds"]):
            return 2 if ts else 1
        for p in (0, 1):
            self.expected[p] = (self.hdr[p]["frame"] + 1) % FRAMESPERSEC
            self.expsec[p] = self.hdr[p]["seconds"] + (1 if self.expected[p] == 0 else 0)
        self.pair_flags.append(self.dflag[0] | self.dflag[1])
        return 0

    def init_ts(self) -> int:
        """TS:516-523 retries initframe01 on status 1.  The reference loops for
        ever once the ring reports end of data; here the retry stops there."""
        while True:
            f = self.initframe01()
            if f == 0 or f == 2:
                return f
            if not self.flag_eof or self.pos >= len(self.buf):
                return 1

    def filltimebuffer(self, nloop: int):  # PIPE:1135-1171
        t0 = bytearray(nloop)
        t1 = bytearray(nloop)
        ifill = 0
        if self.npartleft:
            n = self.npartleft
            t0[0:n] = self.data[0][self.npartfill:self.npartfill + n]
            t1[0:n] = self.data[1][self.npartfill:self.npartfill + n]
            ifill += n
            if self.readtwoframe():
                return None
        ntot = nloop - self.npartleft
        nwhole = ntot // DATALEN
        self.npartfill = ntot % DATALEN
        self.npartleft = DATALEN - self.npartfill
        for _ in range(nwhole):
            t0[ifill:ifill + DATALEN] = self.data[0]
            t1[ifill:ifill + DATALEN] = self.data[1]
            ifill += DATALEN
            if self.readtwoframe():
                return None
        if self.npartfill:
            t0[ifill:ifill + self.npartfill] = self.data[0][:self.npartfill]
            t1[ifill:ifill + self.npartfill] = self.data[1][:self.npartfill]
        return np.frombuffer(bytes(t0), np.uint8), np.frombuffer(bytes(t1), np.uint8)


def read_bundles(data, L: Layout, mode="pipe", max_bundles=None, dada_skip=False):
    """All bundles the reference would process from one VDIF byte stream,
    as (tstart_header, [ (pol0 bytes, pol1 bytes), ... ])."""
    r = RefPairReader(data, mode)
    if dada_skip and r.init_dada():
        return None, [], r
    st = r.init_ts() if mode == "ts" else r.initframe01()
    if st != 0:
        return None, [], r
    h0 = dict(r.hdr[0])
    out = []
    while r.flag_eof:
        if max_bundles is not None and len(out) >= max_bundles:
            break
        b = r.filltimebuffer(L.nloop)
        if b is None:
            break
        out.append(b)
    return h0, out, r


def row_flags(pair_flags, L: Layout, nrows: int) -> np.ndarray:
    """Flags of FB rows 0 .. nrows-1 (new-build extension): row r holds pol
    bytes [r*S, (r+1)*S), S = NAVE*TWONCHAN, i.e. pairs r*S//5000 ..
    ((r+1)*S-1)//5000; its flag is the OR of theirs (1 = a frame with the
    VDIF invalid bit, 2 = a zero-filled missing frame)."""
    pf = np.asarray(pair_flags, np.uint8)
    S = L.nave * L.twonchan
    out = np.zeros(nrows, np.uint8)
    for r in range(nrows):
        out[r] = np.bitwise_or.reduce(pf[r * S // DATALEN:((r + 1) * S - 1) // DATALEN + 1])
    return out


def block_rows(L: Layout, max_delay: int, q: int) -> np.ndarray:
    """Absolute FB row of each row of block q (parity-block mode): block 0 is
    rows 0 .. MAXNT-1; a later block starts with the previous block's last
    max_delay rows, and its rows from first = (max_delay//NBUNDLE)*NBUNDLE
    on (where the refill starts, overwriting carried rows) follow the
    previous block's last row."""
    i = np.arange(L.maxnt, dtype=np.int64)
    if q == 0:
        return i
    first = (max_delay // L.nbundle) * L.nbundle
    end = L.maxnt + (q - 1) * (L.maxnt - first)  # absolute row after the previous block
    return np.where(i < first, end - max_delay + i, end - first + i)


# --- a5-a9: channeliser (PIPE:574-632, 1292-1322) ---------------------------
def channelise(pol0: np.ndarray, pol1: np.ndarray, L: Layout, batch_rows: int = 256) -> np.ndarray:
    """convertarray (no -128 offset, PIPE:1316) -> R2C FFT of TWONCHAN points
    (PIPE:589-596) -> sumpower /NFREQ (PIPE:1292) -> avepower over NAVE spectra
    (PIPE:1301) -> rows FB[row][c] = powAVE[NSKIP + c] (PIPE:627-632).
    Returns float64 [nrows][nchanout], time-major."""
    per_row = L.nave * L.twonchan
    nrows = len(pol0) // per_row
    out = np.empty((nrows, L.nchanout), np.float64)
    for r0 in range(0, nrows, batch_rows):
        r1 = min(nrows, r0 + batch_rows)
        x0 = pol0[r0 * per_row:r1 * per_row].astype(np.float64).reshape(-1, L.twonchan)
        x1 = pol1[r0 * per_row:r1 * per_row].astype(np.float64).reshape(-1, L.twonchan)
        X0 = np.fft.rfft(x0, axis=1)
        X1 = np.fft.rfft(x1, axis=1)
        p = (X0.real ** 2 + X0.imag ** 2 + X1.real ** 2 + X1.imag ** 2) / L.nfreq
        ave = p.reshape(r1 - r0, L.nave, L.nfreq).sum(axis=1) / L.nave
        out[r0:r1] = ave[:, L.nskip:L.nskip + L.nchanout]
    return out


# --- a11: subtractbpCAL (PIPE:1427-1474; STATS:869-908; TS:1365-1407) -------
def subtract_bp_cal(fb: np.ndarray, nrows: int | None = None, window: int = 128) -> np.ndarray:
    """Per (channel, 128-row window counted from row 0): mean; 'sig' is the
    variance (sum2 - sum^2/n)/(n-1); clip to the open interval ave +- 3*sig;
    clipped mean (count floored at 1); subtract it.  Returns a new array."""
    fb = np.array(fb, dtype=np.float64, copy=True)
    n_all = fb.shape[0] if nrows is None else nrows
    with np.errstate(invalid="ignore", divide="ignore"):
        for c0 in range(0, n_all, window):
            c1 = min(c0 + window, n_all)
            x = fb[c0:c1]
            npts = c1 - c0
            ave = x.sum(axis=0) / npts
            d = x - ave
            sig = ((d * d).sum(axis=0) - d.sum(axis=0) ** 2 / npts) / (npts - 1)
            hi = ave + 3.0 * sig
            lo = ave - 3.0 * sig
            m = (x < hi) & (x > lo)
            cnt = np.maximum(m.sum(axis=0), 1)
            cave = np.where(m, x, 0.0).sum(axis=0) / cnt
            fb[c0:c1] = x - cave
    return fb


# --- a12: DM delay table (TS:449-464; PIPE:449-461 commented) ---------------
def delay_table(dms, fch1: float, chanbw: float, tchan: float, nchanout: int):
    """OFF[i][j] = (int)(4.148808e3*DM_i*(pow(fch1-j*CHANBW,-2)-pow(fch1,-2))/tchan),
    OFF[i][0] = 0; DM values are C floats promoted to double.  max_delay uses
    the LAST list entry and one channel past the band (TS:464)."""
    dms32 = np.asarray(dms, dtype=np.float32)
    off = np.zeros((len(dms32), nchanout), np.int32)
    pf = math.pow(fch1, -2)
    for i, dm in enumerate(dms32):
        dmd = float(dm)
        for j in range(1, nchanout):
            dt = DELAY_CONST * dmd * (math.pow(fch1 - (j * chanbw), -2) - pf)
            off[i, j] = int(dt / tchan)
    dml = float(dms32[-1])
    max_delay = int((DELAY_CONST * dml * (math.pow(fch1 - (nchanout * chanbw), -2) - pf)) / tchan)
    return off, max_delay


# --- a13: dedisperse (PIPE:1517-1537; stands in for dedisp_execute PIPE:671) -
def dedisperse(fb_bp: np.ndarray, off: np.ndarray, ntime_out: int) -> np.ndarray:
    """out[d][t] = (1/NCHANOUT) * sum_c FB[t + OFF[d][c]][c]."""
    ndm, nch = off.shape
    out = np.zeros((ndm, ntime_out), np.float64)
    cols = np.arange(nch)
    for d in range(ndm):
        acc = np.zeros(ntime_out, np.float64)
        for c in range(nch):
            o = int(off[d, c])
            acc += fb_bp[o:o + ntime_out, cols[c]]
        out[d] = acc / nch
    return out


def dedisperse_sigma(fb_bp: np.ndarray, off: np.ndarray, ntime_out: int):
    """dedisperseSTATS (TS:1450-1481): channel mean, and
    sqrt((sum d^2 - (sum d)^2)/(N(N-1))) with d = x - mean."""
    ndm, nch = off.shape
    ave = np.zeros((ndm, ntime_out))
    sig = np.zeros((ndm, ntime_out))
    for d in range(ndm):
        g = np.empty((nch, ntime_out))
        for c in range(nch):
            o = int(off[d, c])
            g[c] = fb_bp[o:o + ntime_out, c]
        a = g.sum(axis=0) / nch
        dd = g - a
        ave[d] = a
        sig[d] = np.sqrt(((dd * dd).sum(axis=0) - dd.sum(axis=0) ** 2) / (nch * (nch - 1)))
    return ave, sig


# --- a14: calcstats per DM (PIPE:1337-1370) ---------------------------------
def calcstats_dm(outdd: np.ndarray):
    """FP64 mean; corrected two-pass variance; ave/sigma stored as float;
    peak = max(0, max_t (x - ave_f)/sigma_f) evaluated in float; FRB = any SNR > 3.
    Also returns the argmax time (a new-build extension)."""
    x = np.asarray(outdd, np.float64)
    n = x.shape[1]
    tave = x.sum(axis=1) / n
    d = x - tave[:, None]
    tsig = ((d * d).sum(axis=1) - d.sum(axis=1) ** 2 / n) / (n - 1)
    ave_f = tave.astype(np.float32)
    sig_f = np.sqrt(tsig).astype(np.float32)
    x32 = np.asarray(outdd, np.float32)
    snr = (x32 - ave_f[:, None]) / sig_f[:, None]
    peak = np.maximum(snr.max(axis=1), np.float32(0.0))
    arg = snr.argmax(axis=1)
    frb = (snr > 3.0).any(axis=1).astype(np.int32)
    return dict(ave=ave_f, sigma=sig_f, peak=peak.astype(np.float32), frb=frb, argmax=arg)


# --- dead-code bandpass modes (options; PIPE:1372-1424, 1478-1515) ----------
def subtract_bp_full(fb: np.ndarray) -> np.ndarray:
    """subtractbp (PIPE:1372-1424), one clipped mean per channel over the whole
    block, fb[MAXNT][NCHANOUT] time-major.  As in the reference, the first
    mean divides the sum by NCHANOUT (not by the number of rows), "sig" is the
    corrected two-pass variance about that value, the clip is the open
    interval ave +- 3 sig, and an empty clip window divides by zero (NaN)."""
    x = np.asarray(fb, np.float64)
    n, nch = x.shape
    ave = x.sum(axis=0) / nch
    d = x - ave
    sig = ((d * d).sum(axis=0) - d.sum(axis=0) ** 2 / n) / (n - 1)
    hi, lo = ave + 3.0 * sig, ave - 3.0 * sig
    keep = (x < hi) & (x > lo)
    with np.errstate(invalid="ignore", divide="ignore"):
        cm = (x * keep).sum(axis=0) / keep.sum(axis=0)
    return x - cm


def subtract_zero(fb: np.ndarray) -> np.ndarray:
    """subtractZERO (PIPE:1478-1515): per time row, the clipped mean over the
    channels (mean, corrected variance "sig", open interval ave +- 3 sig,
    count floored at 1) is subtracted from every channel (zero-DM removal)."""
    x = np.asarray(fb, np.float64)
    n, nch = x.shape
    ave = x.sum(axis=1) / nch
    d = x - ave[:, None]
    sig = ((d * d).sum(axis=1) - d.sum(axis=1) ** 2 / nch) / (nch - 1)
    hi, lo = ave + 3.0 * sig, ave - 3.0 * sig
    keep = (x < hi[:, None]) & (x > lo[:, None])
    cnt = np.maximum(keep.sum(axis=1), 1)
    cm = (x * keep).sum(axis=1) / cnt
    return x - cm[:, None]


# --- candidate search (new-build extension; no reference counterpart) -------
def boxcar_best(outdd: np.ndarray, ave_f, sig_f, max_width: int):
    """Per DM trial, the best boxcar over widths w = 1, 2, 4, ..., max_width:
    S_w(t) = sum_{i<w} x[t+i] (FP64, t = 0 .. nt-w) and
    snr_w(t) = (S_w(t) - w*ave) / (sigma*sqrt(w)) with the trial's calcstats
    ave and sigma (width 1 is calcstats' peak).  Ties: the smaller width, then
    the earlier start.  Returns (snr, start, width) arrays."""
    x = np.asarray(outdd, np.float64)
    ndm, nt = x.shape
    ave = np.asarray(ave_f, np.float32).astype(np.float64)
    sig = np.asarray(sig_f, np.float32).astype(np.float64)
    cs = np.concatenate([np.zeros((ndm, 1)), np.cumsum(x, axis=1)], axis=1)
    best = np.full(ndm, -np.inf)
    bt = np.zeros(ndm, np.int64)
    bw = np.ones(ndm, np.int64)
    w = 1
    while w <= max_width and w <= nt:
        s = cs[:, w:] - cs[:, :-w]
        snr = (s - w * ave[:, None]) / (sig[:, None] * np.sqrt(w))
        t = snr.argmax(axis=1)
        v = snr[np.arange(ndm), t]
        upd = v > best
        best[upd], bt[upd], bw[upd] = v[upd], t[upd], w
        w *= 2
    return best, bt, bw


def candidates(best, start, width, dms, threshold: float, row0: int = 0):
    """Candidates of one chunk: trials whose best boxcar SNR reaches the
    threshold and is a local maximum over neighbouring trials (ties go to the
    lower trial).  Returns a list of (dm_index, t, width, snr, dm)."""
    out = []
    n = len(best)
    for d in range(n):
        p = best[d]
        if not (p >= threshold):
            continue
        if d > 0 and best[d - 1] > p:
            continue
        if d + 1 < n and best[d + 1] >= p:
            continue
        out.append((d, row0 + int(start[d]), int(width[d]), float(p), float(dms[d])))
    return out


def cluster_cands(cands, dm_tol: int, t_tol: int):
    """Friends-of-friends clustering (new-build extension): candidates
    (dm_index, t, width, snr) are friends when |dm_a - dm_b| <= dm_tol and
    max(t_a, t_b) - min(t_a + w_a, t_b + w_b) <= t_tol; clusters are the
    connected components, each reported by its brightest member (ties: lower
    dm_index, then earlier t), ordered by (t, dm_index).  O(n^2) pairs, for
    small lists.  Returns (representatives, labels)."""
    n = len(cands)
    parent = list(range(n))

    def find(a):
        while parent[a] != a:
            a = parent[a]
        return a

    for i in range(n):
        for j in range(i + 1, n):
            a, b = cands[i], cands[j]
            gap = max(a[1], b[1]) - min(a[1] + a[2], b[1] + b[2])
            if abs(a[0] - b[0]) <= dm_tol and gap <= t_tol:
                ri, rj = find(i), find(j)
                if ri != rj:
                    parent[max(ri, rj)] = min(ri, rj)
    groups = {}
    for i in range(n):
        groups.setdefault(find(i), []).append(i)
    reps = []
    for root, mem in groups.items():
        best = min(mem, key=lambda k: (-cands[k][3], cands[k][0], cands[k][1]))
        reps.append((root, best))
    reps.sort(key=lambda rb: (cands[rb[1]][1], cands[rb[1]][0]))
    label_of_root = {root: k for k, (root, _) in enumerate(reps)}
    labels = [label_of_root[find(i)] for i in range(n)]
    return [cands[b] for _, b in reps], labels


def chan_sk(fb_raw: np.ndarray, ncolstatblk: int, nstatblks: int, nsum: int) -> np.ndarray:
    """Spectral kurtosis (new-build extension; the reference has none) per
    (stat block, channel) of the RAW FB (before bandpass subtraction): the
    generalised estimator of Nita & Gary (2010),
    SK = (M*nsum + 1)/(M - 1) * (M*S2/S1^2 - 1), M rows, S1 = sum x,
    S2 = sum x^2, nsum = raw power values per FB sample (2 pols x NAVE)."""
    x = np.asarray(fb_raw, np.float64)
    maxnt, nch = x.shape
    out = np.zeros((nstatblks, nch))
    for k in range(nstatblks):
        blk = x[ncolstatblk * k:min(ncolstatblk * (k + 1), maxnt)]
        m = blk.shape[0]
        s1 = blk.sum(axis=0)
        s2 = (blk * blk).sum(axis=0)
        out[k] = (m * nsum + 1.0) / (m - 1.0) * (m * s2 / (s1 * s1) - 1.0)
    return out


# --- a16: calcstats per channel (STATS:910-946) -----------------------------
def calcstats_chan(fb_bp: np.ndarray, ncolstatblk: int, nstatblks: int):
    """Per (channel, stat block of NCOLSTATBLK rows): mean, variance (named
    sig), outliers = count(x > ave + 5 sig) stored as integer i/npts."""
    maxnt, nch = fb_bp.shape
    ave = np.zeros((nstatblks, nch))
    sig = np.zeros((nstatblks, nch))
    outl = np.zeros((nstatblks, nch))
    for k in range(nstatblks):
        c0 = ncolstatblk * k
        c1 = min(c0 + ncolstatblk, maxnt)
        x = fb_bp[c0:c1]
        npts = c1 - c0
        a = x.sum(axis=0) / npts
        d = x - a
        s = ((d * d).sum(axis=0) - d.sum(axis=0) ** 2 / npts) / (npts - 1)
        i = (x > a + 5.0 * s).sum(axis=0)
        ave[k], sig[k], outl[k] = a, s, i // npts
    return ave, sig, outl


# --- a10: block manager for PIPE/TS (PIPE:649-704; TS:643-692) ---------------
def run_blocks(rows: np.ndarray, L: Layout, max_delay: int):
    """Yields (block_index, raw FB block) exactly as assembled by the
    reference: the first block is rows [0, MAXNT); each later block starts
    with the last max_delay raw rows of the previous block and new rows are
    written from row (max_delay/NBUNDLE)*NBUNDLE on."""
    nb = L.nbundle
    fb = np.zeros((L.maxnt, rows.shape[1]), np.float64)
    loopcnt = 0
    q = 0
    nbund = rows.shape[0] // nb
    for b in range(nbund):
        fb[loopcnt * nb:(loopcnt + 1) * nb] = rows[b * nb:(b + 1) * nb]
        loopcnt += 1
        if loopcnt == L.maxnt // nb:
            leftover = fb[L.maxnt - max_delay:L.maxnt].copy()
            yield q, fb.copy()
            fb[0:max_delay] = leftover
            loopcnt = max_delay // nb
            q += 1


def run_stats_blocks(rows: np.ndarray, L: Layout):
    """STATS:370-431: blocks of NLOOP=MAXNT/NBUNDLE bundles, no overlap."""
    nb = L.nbundle
    per = (L.maxnt // nb) * nb
    for q in range(rows.shape[0] // per):
        fb = np.zeros((L.maxnt, rows.shape[1]))
        fb[:per] = rows[q * per:(q + 1) * per]
        yield q, fb


# --- a17: writers -----------------------------------------------------------
def sigproc_header(fch1, foff, nchans, tstart, tsamp, nbits=32, nifs=1) -> bytes:
    """PIPE:529-540 via send_string/send_int/send_double (PIPE:1177-1201)."""
    import struct

    def s(x):
        return struct.pack("<i", len(x)) + x.encode()

    out = s("HEADER_START")
    out += s("barycentric") + struct.pack("<i", 1)
    out += s("telescope_id") + struct.pack("<i", 12)
    out += s("data_type") + struct.pack("<i", 1)
    out += s("fch1") + struct.pack("<d", fch1)
    out += s("foff") + struct.pack("<d", foff)
    out += s("nchans") + struct.pack("<i", nchans)
    out += s("nbits") + struct.pack("<i", nbits)
    out += s("tstart") + struct.pack("<d", tstart)
    out += s("tsamp") + struct.pack("<d", tsamp)
    out += s("nifs") + struct.pack("<i", nifs)
    out += s("HEADER_END")
    return out


def presto_inf(fbasename, mjdstart, ntimes, tsamp, dm, fchanlo, bw, nchan, chanbw) -> str:
    """TS:1483-1515 (dm is a C float printed with %f)."""
    dmf = float(np.float32(dm))
    return (
        f" Data file name without suffix          = {fbasename}\n"
        " Telescope used                         = VLA\n"
        " Instrument used                        = VLITE-FAST\n"
        " Object being observed                  = Unknown\n"
        " J2000 Right Ascension (hh:mm:ss.ssss)  = 00:00:00.0000\n"
        " J2000 Declination     (dd:mm:ss.ssss)  = 00:00:00.0000\n"
        " Data observed by                       = vdifDADA2timeseries\n"
        f" Epoch of observation (MJD)             = {mjdstart:.15f}\n"
        " Barycentered?                          = 1\n"
        f" Number of bins in the time series      = {ntimes:d}\n"
        f" Width of each time series bin (sec)    = {tsamp:.9f}\n"
        " Any breaks in the data? (1=yes, 0=no)  = 0\n"
        " Type of observation (EM band)          = Radio\n"
        " Beam diameter (arcsec)                 = 3600\n"
        f" Dispersion measure (cm-3 pc)           = {dmf:f}\n"
        f" Central freq of low channel (MHz)      = {fchanlo:f}\n"
        f" Total bandwidth (MHz)                  = {bw:f}\n"
        f" Number of channels                     = {nchan:d}\n"
        f" Channel bandwidth (MHz)                = {chanbw:f}\n"
        " Data analyzed by                       = vdifDADA2timeseries\n"
        " Any additional notes:\n    \n\n")


def outdd_bin(dms, outdd) -> bytes:
    """PIPE:734-739: per DM a float DM value then NTIME_OUTDD floats."""
    parts = []
    for dm, row in zip(np.asarray(dms, np.float32), np.asarray(outdd, np.float32)):
        parts.append(np.float32(dm).tobytes() + row.tobytes())
    return b"".join(parts)


# --- streaming semantics (new build; no reference counterpart) --------------
def stream_bandpass(fb: np.ndarray, window: int = 128):
    """Streaming form: absolute 128-row windows counted from the first row of
    the stream; same per-window estimator as subtractbpCAL.  Only complete
    windows are produced.  Returns (bp rows, per-window variance)."""
    n = (fb.shape[0] // window) * window
    out = subtract_bp_cal(fb[:n], window=window)
    return out
