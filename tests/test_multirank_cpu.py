"""The N>1 path of bench.py on CPU: two ranks as separate processes over
gloo (world size 2, 127.0.0.1).  Each rank owns an independent stream (its
own seed, no data collective); the only collective is the max-over-ranks of
the step time.  A rank that leaves before the collective makes the other
rank's next collective end with an error within the short process-group
timeout instead of hanging (failure detected on the host)."""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("vfrb_bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, leave_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    b = _bench()
    dist = b.dist_init(world, backend="gloo", timeout_s=5)
    try:
        if rank == leave_rank:
            q.put((rank, "left", None, None))
            return  # leaves between steps, with nothing in flight
        b.dist_barrier(dist)
        v = b.dist_max(dist, 10.0 + rank)
        q.put((rank, "ok", v, b.stream_seed(rank)))
    except Exception as e:  # noqa: BLE001
        q.put((rank, "err", type(e).__name__, None))
    finally:
        try:
            import torch.distributed as d
            if leave_rank < 0:
                d.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _run(world, leave_rank, timeout=60):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q, leave_rank)) for r in range(world)]
    for p in ps:
        p.start()
    out = {}
    try:
        for _ in range(world):
            r = q.get(timeout=timeout)
            out[r[0]] = r[1:]
    finally:
        for p in ps:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
                p.join()
    return out


def test_two_ranks_max_time_and_independent_streams():
    out = _run(2, -1)
    assert out[0][0] == "ok" and out[1][0] == "ok", out
    assert out[0][1] == out[1][1] == 11.0  # max over ranks on every rank
    assert out[0][2] != out[1][2]  # each rank synthesises its own stream


def test_rank_leaving_is_detected_by_timeout():
    out = _run(2, 1)
    assert out[1][0] == "left"
    assert out[0][0] == "err", out  # the collective ends with an error, no hang


def test_reference_arm_line_contract():
    """`bench.py --impl reference` (the CPU port of the path, no GPU): one JSON
    line with the arm's keys; e2e repeats the value with no copies."""
    import json
    import subprocess
    import sys
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--cpu-sample", "0.05"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s data/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["warmup"] >= 3 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "s data/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the same workload object as the GPU arm; ms_per_step is the time of the
    # sample a step really ran (value = sample seconds / step seconds)
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.bench_config(bench.DURATION, 1)
    assert abs(d["ms_per_step"] / 1000.0 * d["value"] - 0.05) < 1e-6


def test_reference_arm_maps_no_product_library():
    """The reference arm's process loads the oracle's port and nothing of the
    product: libvfrb.so is never mapped."""
    import subprocess
    import sys
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', "
            "'--cpu-sample', '0.05']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); print('LIBVFRB' if 'libvfrb' in maps else 'CLEAN'); "
            "print('ORACLE' if 'liboracle32' in maps else 'NO-ORACLE')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "CLEAN" in r.stdout and "ORACLE" in r.stdout, r.stdout[-500:]


def _rank_pipeline(seed, drop_pair=None):
    """One rank's stream at toy size on the CPU: synthesise it (the rank's
    seed), pair its frames with the product's host reader (vfrb_read_pairs,
    C ABI), then channelise -> bandpass -> dedisperse -> calcstats with the
    FP64 C oracle.  Returns the per-trial statistics and the pair count."""
    import ctypes as C
    import sys

    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import vfrb_oracle as O
    from coracle import COracle
    b = _bench()
    synth = b.load_synth()
    buf = synth.make_vdif(synth.StreamSpec(duration=0.25, seed=seed, pulses=[synth.Pulse(0.08, 6.0, 2.0, 40.0)]))
    buf = buf.numpy()
    if drop_pair is not None:  # a gap the reader fills with zeros
        buf = np.ascontiguousarray(np.delete(buf.reshape(-1, 2, 5032), [drop_pair], axis=0)).reshape(-1)
    lib = C.CDLL(os.path.join(ROOT, "vlite-frb_b200", "lib", "libvfrb.so"))
    lib.vfrb_read_pairs.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_void_p,
                                    C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    cap = len(buf) // 5032 + 8
    e0, e1 = np.zeros(cap, np.int64), np.zeros(cap, np.int64)
    n, ts = C.c_int64(0), C.c_double(0)
    assert lib.vfrb_read_pairs(buf.ctypes.data, len(buf), 0, 0, 0, e0.ctypes.data, e1.ctypes.data, cap, C.byref(n),
                               C.byref(ts)) == 0
    fr = buf.reshape(-1, 5032)
    pay = [np.concatenate([fr[k, 32:] if k >= 0 else np.zeros(5000, np.uint8) for k in e[:n.value]])
           for e in (e0, e1)]
    L = O.Layout(nave=2, muoslowfreq=384.0, nbundle=1)
    co = COracle(64)
    rows = co.channelise(pay[0], pay[1], L)
    nbp = rows.shape[0] // 128 * 128
    dms = np.arange(0, 10.0, 0.5, dtype=np.float32)
    off, md = O.delay_table(dms, L.fch1, L.chanbw, L.tchan, L.nchanout)
    dd = co.dedisperse_cm(co.transpose(co.bandpass(rows[:nbp])), off, nbp - md)
    st = co.calcstats_dm(dd)
    return {k: v.tolist() for k, v in st.items()}, int(n.value), float(ts.value)


def _pipeline_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    b = _bench()
    dist = b.dist_init(world, backend="gloo", timeout_s=30)
    try:
        # each rank processes only its own stream: no collective on the data path
        stats, npairs, tstart = _rank_pipeline(b.stream_seed(rank), drop_pair=100 if rank == 1 else None)
        b.dist_barrier(dist)
        worst = b.dist_max(dist, float(npairs))
        q.put((rank, "ok", stats, npairs, tstart, worst))
    except Exception as e:  # noqa: BLE001
        q.put((rank, "err", repr(e), 0, 0.0, 0.0))
    finally:
        try:
            import torch.distributed as d
            d.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "vlite-frb_b200", "lib", "libvfrb.so")),
                    reason="libvfrb.so not built")
def test_two_rank_pipelines_equal_single_process():
    """Two gloo ranks, each driving its own stream (the rank's seed; rank 1's
    has a missing frame pair) through the product's host pair reader and the
    CPU chain, give per-rank results identical to one process running both
    streams; the only collective is the max over ranks."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_pipeline_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    try:
        for _ in range(2):
            r = q.get(timeout=300)
            out[r[0]] = r[1:]
    finally:
        for p in ps:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
                p.join()
    assert out[0][0] == "ok" and out[1][0] == "ok", out
    b = _bench()
    for rank in (0, 1):
        stats, npairs, tstart = _rank_pipeline(b.stream_seed(rank), drop_pair=100 if rank == 1 else None)
        assert out[rank][1] == stats and out[rank][2] == npairs and out[rank][3] == tstart
    assert out[0][1] != out[1][1]  # independent streams
    assert out[0][4] == out[1][4] == max(out[0][2], out[1][2])
