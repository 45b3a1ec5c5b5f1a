"""ctypes wrapper of oracle.c (TEST INFRASTRUCTURE ONLY: tests and the CPU
baseline leg of bench.py).  `bits=64` is the FP64 checker, `bits=32` the
timed FP32 OpenMP host transcription."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class COracle:
    def __init__(self, bits=64):
        path = os.path.join(HERE, "_build", f"liboracle{bits}.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run oracle/build_oracle.py")
        self.lib = C.CDLL(path)
        self.dt = np.float64 if bits == 64 else np.float32
        L = self.lib
        p = C.c_void_p
        L.oc_channelise.argtypes = [p, p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, p]
        L.oc_bandpass.argtypes = [p, C.c_int64, C.c_int, C.c_int]
        L.oc_transpose.argtypes = [p, C.c_int64, C.c_int, p]
        L.oc_dedisperse.argtypes = [p, C.c_int64, C.c_int, p, C.c_int, C.c_int64, p]
        L.oc_calcstats_dm.argtypes = [p, C.c_int, C.c_int64, p, p, p, p, p]
        L.oc_dedisperse_sigma.argtypes = [p, C.c_int64, C.c_int, p, C.c_int, C.c_int64, p, p]
        L.oc_chan_stats.argtypes = [p, C.c_int64, C.c_int, C.c_int, C.c_int, p, p, p]

    def threads(self):
        return self.lib.oc_num_threads()

    def channelise(self, p0, p1, L):
        p0 = np.ascontiguousarray(p0, np.uint8)
        p1 = np.ascontiguousarray(p1, np.uint8)
        nrows = len(p0) // (L.nave * L.twonchan)
        out = np.empty((nrows, L.nchanout), self.dt)
        if self.lib.oc_channelise(p0.ctypes.data, p1.ctypes.data, nrows, L.twonchan, L.nave, L.nfreq, L.nskip,
                                  L.nchanout, out.ctypes.data):
            raise MemoryError("oc_channelise")
        return out

    def bandpass(self, fb, window=128):
        fb = np.array(fb, dtype=self.dt, copy=True, order="C")
        self.lib.oc_bandpass(fb.ctypes.data, fb.shape[0], fb.shape[1], window)
        return fb

    def transpose(self, fb):
        fb = np.ascontiguousarray(fb, self.dt)
        cm = np.empty((fb.shape[1], fb.shape[0]), self.dt)
        self.lib.oc_transpose(fb.ctypes.data, fb.shape[0], fb.shape[1], cm.ctypes.data)
        return cm

    def dedisperse_cm(self, cm, off, nt):
        cm = np.ascontiguousarray(cm, self.dt)
        off = np.ascontiguousarray(off, np.int32)
        out = np.empty((off.shape[0], nt), self.dt)
        self.lib.oc_dedisperse(cm.ctypes.data, cm.shape[1], cm.shape[0], off.ctypes.data, off.shape[0], nt,
                               out.ctypes.data)
        return out

    def calcstats_dm(self, out):
        out = np.ascontiguousarray(out, self.dt)
        n = out.shape[0]
        r = dict(ave=np.empty(n, np.float32), sigma=np.empty(n, np.float32), peak=np.empty(n, np.float32),
                 frb=np.empty(n, np.int32), argmax=np.empty(n, np.int32))
        self.lib.oc_calcstats_dm(out.ctypes.data, n, out.shape[1], r["ave"].ctypes.data, r["sigma"].ctypes.data,
                                 r["peak"].ctypes.data, r["frb"].ctypes.data, r["argmax"].ctypes.data)
        return r

    def dedisperse_sigma_cm(self, cm, off, nt):
        cm = np.ascontiguousarray(cm, self.dt)
        off = np.ascontiguousarray(off, np.int32)
        a = np.empty((off.shape[0], nt), self.dt)
        s = np.empty_like(a)
        self.lib.oc_dedisperse_sigma(cm.ctypes.data, cm.shape[1], cm.shape[0], off.ctypes.data, off.shape[0], nt,
                                     a.ctypes.data, s.ctypes.data)
        return a, s

    def chan_stats_cm(self, cm, ncol, nblk):
        cm = np.ascontiguousarray(cm, self.dt)
        nch = cm.shape[0]
        a = np.empty((nblk, nch), np.float32)
        s = np.empty_like(a)
        o = np.empty_like(a)
        self.lib.oc_chan_stats(cm.ctypes.data, cm.shape[1], nch, ncol, nblk, a.ctypes.data, s.ctypes.data,
                               o.ctypes.data)
        return a, s, o
