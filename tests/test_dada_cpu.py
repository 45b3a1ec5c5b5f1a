"""The DADA-style input ring (vfrb_dada_*) the STATS and TS tools read:
bytes arrive in order across wrap-around, a short read marks end of data
(ipcio_read / ipcbuf_eod semantics, STATS:444-462), waits are bounded, and
the writer tool feeds a reader in another process."""
import ctypes as C
import os
import random
import subprocess
import threading

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ERR_TIMEOUT = 7


def _lib(vf):
    lib = vf.lib()
    vp = C.c_void_p
    lib.vfrb_dada_create.argtypes = [C.c_uint32, C.c_uint64, C.POINTER(vp)]
    lib.vfrb_dada_connect.argtypes = [C.c_uint32, C.POINTER(vp)]
    lib.vfrb_dada_write.argtypes = [vp, vp, C.c_uint64, C.c_int]
    lib.vfrb_dada_write.restype = C.c_int64
    lib.vfrb_dada_read.argtypes = [vp, vp, C.c_uint64, C.c_int]
    lib.vfrb_dada_read.restype = C.c_int64
    lib.vfrb_dada_set_eod.argtypes = [vp]
    lib.vfrb_dada_eod.argtypes = [vp]
    lib.vfrb_dada_close.argtypes = [vp]
    lib.vfrb_dada_destroy.argtypes = [C.c_uint32]
    lib.vfrb_dada_acquire.argtypes = [vp, C.POINTER(C.c_void_p), C.c_uint64, C.c_int]
    lib.vfrb_dada_acquire.restype = C.c_int64
    lib.vfrb_dada_release.argtypes = [vp, C.c_uint64]
    lib.vfrb_dada_set_header.argtypes = [vp, C.c_char_p, C.c_uint64]
    lib.vfrb_dada_get_header.argtypes = [vp, C.c_char_p, C.c_uint64, C.c_int]
    lib.vfrb_dada_get_header.restype = C.c_int64
    lib.vfrb_dada_iread.argtypes = [vp]
    lib.vfrb_dada_force_iread.argtypes = [vp]
    lib.vfrb_dada_open_read.argtypes = [vp]
    return lib


def _key():
    return random.randrange(0x10000000, 0x7fffffff)


def test_ring_roundtrip_wrap_and_eod(vf):
    lib = _lib(vf)
    key = _key()
    w = C.c_void_p()
    assert lib.vfrb_dada_create(key, 1 << 16, C.byref(w)) == 0
    try:
        assert lib.vfrb_dada_create(key, 1 << 16, C.byref(C.c_void_p())) != 0  # key in use
        r = C.c_void_p()
        assert lib.vfrb_dada_connect(key, C.byref(r)) == 0
        data = np.random.default_rng(1).integers(0, 256, 1_000_003, dtype=np.uint8)

        def writer():
            pos = 0
            rng = np.random.default_rng(2)
            while pos < data.size:
                k = int(min(rng.integers(1, 40000), data.size - pos))
                assert lib.vfrb_dada_write(w, data[pos:].ctypes.data, k, 5000) == k
                pos += k
            lib.vfrb_dada_set_eod(w)

        t = threading.Thread(target=writer)
        t.start()
        got = np.zeros(data.size + 100, np.uint8)
        pos = 0
        while True:
            n = lib.vfrb_dada_read(r, got[pos:].ctypes.data, 5032, 5000)
            assert n >= 0
            pos += n
            if n < 5032:
                break
        t.join()
        assert pos == data.size and np.array_equal(got[:pos], data)
        assert lib.vfrb_dada_eod(r) == 1
        assert lib.vfrb_dada_read(r, got.ctypes.data, 10, 10) == 0
        lib.vfrb_dada_close(r)
        lib.vfrb_dada_close(w)
    finally:
        lib.vfrb_dada_destroy(key)


def test_ring_bounded_waits(vf):
    lib = _lib(vf)
    key = _key()
    w = C.c_void_p()
    assert lib.vfrb_dada_create(key, 4096, C.byref(w)) == 0
    try:
        buf = np.zeros(8192, np.uint8)
        assert lib.vfrb_dada_read(w, buf.ctypes.data, 16, 50) == -ERR_TIMEOUT  # nothing written, no EOD
        assert lib.vfrb_dada_write(w, buf.ctypes.data, 8192, 50) == 4096       # full after 4096 bytes
        assert lib.vfrb_dada_write(w, buf.ctypes.data, 1, 50) == -ERR_TIMEOUT
        assert lib.vfrb_dada_connect(key + 1, C.byref(C.c_void_p())) != 0       # no such ring
        assert lib.vfrb_dada_create(key + 2, 5000, C.byref(C.c_void_p())) == 4  # not a power of two
        lib.vfrb_dada_close(w)
    finally:
        lib.vfrb_dada_destroy(key)


def test_writer_tool_feeds_reader(vf, tmp_path):
    lib = _lib(vf)
    exe = os.path.join(ROOT, "vlite-frb_b200", "bin", "vfrb_dada_write")
    if not os.path.exists(exe):
        pytest.fail("vfrb_dada_write not built")
    key = _key()
    data = np.random.default_rng(3).integers(0, 256, 3_000_000, dtype=np.uint8)
    data.tofile(tmp_path / "x.bin")
    p = subprocess.Popen([exe, "-k", f"{key:x}", "-i", str(tmp_path / "x.bin"), "-cap", str(1 << 20),
                          "-chunk", "100000", "-timeout", "20"])
    try:
        r = C.c_void_p()
        for _ in range(500):
            if lib.vfrb_dada_connect(key, C.byref(r)) == 0:
                break
            threading.Event().wait(0.01)
        else:
            pytest.fail("ring never appeared")
        hdr = C.create_string_buffer(4096)
        n = lib.vfrb_dada_get_header(r, hdr, 4096, 20000)
        assert n > 0 and b"ENCODING VDIF" in hdr.raw[:n] and b"x.bin" in hdr.raw[:n]
        got = np.zeros(data.size, np.uint8)
        pos = 0
        while pos < data.size:
            n = lib.vfrb_dada_read(r, got[pos:].ctypes.data, min(65536, data.size - pos), 20000)
            assert n > 0
            pos += n
        assert lib.vfrb_dada_read(r, got.ctypes.data, 1, 20000) == 0  # end of data
        lib.vfrb_dada_close(r)
        assert p.wait(timeout=30) == 0
        assert np.array_equal(got, data)
    finally:
        if p.poll() is None:
            p.kill()
            p.wait()
        lib.vfrb_dada_destroy(key)


def test_ring_in_place_reading(vf):
    """acquire/release: the bytes are read in place in contiguous runs that
    stop at the ring's end, in order across wrap-around; releasing more than
    was written is refused; 0 bytes at end of data; a bounded wait."""
    lib = _lib(vf)
    key = _key()
    w = C.c_void_p()
    assert lib.vfrb_dada_create(key, 1 << 14, C.byref(w)) == 0
    try:
        r = C.c_void_p()
        assert lib.vfrb_dada_connect(key, C.byref(r)) == 0
        p = C.c_void_p()
        assert lib.vfrb_dada_acquire(r, C.byref(p), 1 << 20, 50) == -ERR_TIMEOUT  # nothing written yet
        data = np.random.default_rng(5).integers(0, 256, 300_001, dtype=np.uint8)

        def writer():
            pos = 0
            rng = np.random.default_rng(6)
            while pos < data.size:
                k = int(min(rng.integers(1, 9000), data.size - pos))
                assert lib.vfrb_dada_write(w, data[pos:].ctypes.data, k, 5000) == k
                pos += k
            lib.vfrb_dada_set_eod(w)

        t = threading.Thread(target=writer)
        t.start()
        got, runs = [], 0
        rng = np.random.default_rng(7)
        while True:
            n = lib.vfrb_dada_acquire(r, C.byref(p), int(rng.integers(1, 20000)), 5000)
            assert n >= 0
            if n == 0:
                break
            assert n <= (1 << 14)
            got.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(n,)).copy())
            take = int(rng.integers(1, n + 1))  # consume part of the run; the rest is acquired again
            got[-1] = got[-1][:take]
            assert lib.vfrb_dada_release(r, take) == 0
            runs += 1
        t.join()
        assert np.array_equal(np.concatenate(got), data) and runs > 20
        assert lib.vfrb_dada_release(r, 1) != 0  # nothing left to release
        lib.vfrb_dada_close(r)
    finally:
        lib.vfrb_dada_close(w)
        lib.vfrb_dada_destroy(key)


def test_header_block_and_eod_mid_frame(vf):
    """The header block: a reader's wait for it is bounded (timeout status)
    until the writer sets it, then the text comes back as written.  End of
    data in the middle of a frame: the reader gets the whole frames, then a
    short read with the partial frame, then 0 (ipcio_read at EOD)."""
    lib = _lib(vf)
    key = _key()
    w = C.c_void_p()
    assert lib.vfrb_dada_create(key, 1 << 16, C.byref(w)) == 0
    try:
        r = C.c_void_p()
        assert lib.vfrb_dada_connect(key, C.byref(r)) == 0
        buf = C.create_string_buffer(4096)
        assert lib.vfrb_dada_get_header(r, buf, 4096, 50) == -ERR_TIMEOUT
        text = b"HDR_VERSION 1.0\nHDR_SIZE 4096\nENCODING VDIF\n"
        assert lib.vfrb_dada_set_header(w, text, len(text)) == 0
        assert lib.vfrb_dada_set_header(w, text, 4097) == 4  # larger than the block: VFRB_ERR_ARG
        n = lib.vfrb_dada_get_header(r, buf, 4096, 50)
        assert n == len(text) and buf.raw[:n] == text
        frames = np.random.default_rng(4).integers(0, 256, 2 * 5032 + 2516, dtype=np.uint8)
        assert lib.vfrb_dada_write(w, frames.ctypes.data, frames.size, 1000) == frames.size
        assert lib.vfrb_dada_set_eod(w) == 0
        got = np.zeros(5032, np.uint8)
        sizes = [lib.vfrb_dada_read(r, got.ctypes.data, 5032, 1000) for _ in range(4)]
        assert sizes == [5032, 5032, 2516, 0]
        assert lib.vfrb_dada_eod(r) == 1
        lib.vfrb_dada_close(r)
    finally:
        lib.vfrb_dada_close(w)
        lib.vfrb_dada_destroy(key)


def test_primary_reader_lock_and_iread_force(vf):
    """One primary read client at a time (ipcio_open 'R'): a second reader's
    open fails while the first holds the role; forcing iread (the reference
    tools' ipcbuf_force_iread hack) clears it and returns the holder, after
    which the second reader opens; the first reader's close then leaves the
    second's role alone, and the second's close frees it."""
    lib = _lib(vf)
    key = _key()
    w = C.c_void_p()
    assert lib.vfrb_dada_create(key, 1 << 16, C.byref(w)) == 0
    try:
        r1, r2 = C.c_void_p(), C.c_void_p()
        assert lib.vfrb_dada_connect(key, C.byref(r1)) == 0
        assert lib.vfrb_dada_connect(key, C.byref(r2)) == 0
        assert lib.vfrb_dada_iread(r1) == -1
        assert lib.vfrb_dada_open_read(r1) == 0
        holder = lib.vfrb_dada_iread(r2)
        assert holder != -1
        assert lib.vfrb_dada_open_read(r2) == 2  # VFRB_ERR: another primary reader
        assert lib.vfrb_dada_force_iread(r2) == holder
        assert lib.vfrb_dada_iread(r2) == -1
        assert lib.vfrb_dada_open_read(r2) == 0
        mine = lib.vfrb_dada_iread(r1)
        assert mine not in (-1, holder)
        lib.vfrb_dada_close(r1)
        assert lib.vfrb_dada_iread(r2) == mine
        lib.vfrb_dada_close(r2)
        assert lib.vfrb_dada_iread(w) == -1
    finally:
        lib.vfrb_dada_close(w)
        lib.vfrb_dada_destroy(key)
