#!/usr/bin/env python3
"""Benchmark of the vlite-frb FRB search chain on B200.

Workload (the full-scale plain-FP32 configuration): 60 s of 2-pol 8-bit
VLITE VDIF (5032-byte frames, 25600 frames/s/pol, seed 1) with 20 injected
dispersed pulses (DM U(50,1000), FWHM U(1,10) ms, SNR U(8,30)), 12500-point
FFT -> 6250 channels (full band), NAVE = 10 (0.977 ms rows), bandpass
subtraction, 2048 DM trials on linspace(0, 1000), per-trial statistics.

A step is one pass of the chain over the 60 s batch.  `value` is the
real-time factor (seconds of data per second) with the raw VDIF resident in
HBM: channelise (K1) -> bandpass (K2) -> dedisperse + statistics (K3), with
the max-DM overlap carried in a device ring across steps, so every step
produces 61440 new output samples per trial.  `e2e` is the same metric
through the public plan API (vfrb_push_frames / vfrb_poll) from page-locked
host memory, host->device copies and result reads inside the timed region.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "vlite-frb_b200")
DURATION = 60.0
NAVE = 10
NDM = 2048
DM_MAX = 1000.0
SEED = 1
METRIC = "x-realtime (s data/s) + p99 chunk latency; FP16 vs FP32 form at ΔSNR≤1%"
WORKLOAD = "60 s 2-pol VLITE VDIF, 20 pulses DM 50-1000; 12500-pt FFT -> 6250 ch, NAVE 10; 2048 DMs 0-1000"


def load_pkg():
    if "vlite_frb_b200" in sys.modules:
        return sys.modules["vlite_frb_b200"]
    spec = importlib.util.spec_from_file_location("vlite_frb_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    m = importlib.util.module_from_spec(spec)
    sys.modules["vlite_frb_b200"] = m
    spec.loader.exec_module(m)
    return m


def load_synth():
    """The synthetic-input generator on its own, without the package (whose
    import maps libvfrb.so): the reference arm and the CPU baseline use it
    for their inputs and nothing else."""
    if "vfrb_synth_only" in sys.modules:
        return sys.modules["vfrb_synth_only"]
    spec = importlib.util.spec_from_file_location("vfrb_synth_only", os.path.join(PKG_DIR, "synth.py"))
    m = importlib.util.module_from_spec(spec)
    sys.modules["vfrb_synth_only"] = m
    spec.loader.exec_module(m)
    return m


def bench_config(duration, world):
    """The workload's `config` object, shared by both arms of the bench."""
    return {"workload": WORKLOAD, "seconds_per_step": duration, "nchan": 6250, "ndm": NDM, "nave": NAVE,
            "form": "plain FP32", "inputs_larger_than_l2": True,
            "l2_note": "inputs (15.5 GB of VDIF per step) exceed the 126 MB L2; no flush needed",
            "parallelism": f"streams x{world} (one independent stream per GPU)"}


def dm_grid():
    return np.linspace(0.0, DM_MAX, NDM).astype(np.float32)


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- device-resident chain
class DevicePipeline:
    """K1 -> K2 -> K3 over the resident 60 s batch through the stage C ABI,
    with the overlap ring persisting across steps."""

    def __init__(self, vf, frames, storage, variant=0):
        import torch
        self.vf, self.torch = vf, torch
        self.storage = storage
        dev = frames.device
        self.frames = frames
        self.L = vf.layout(nave=NAVE, muoslowfreq=384.0)
        npairs = frames.numel() // 10064
        idx = torch.arange(npairs, dtype=torch.int64, device=dev)
        self.s0 = idx * 10064 + 32
        self.s1 = self.s0 + 5032
        self.rows = (npairs * 5000) // (NAVE * 12500)
        self.rows = self.rows // 128 * 128
        nch = self.L.nchanout
        self.raw = torch.empty((self.rows, nch), dtype=torch.float32, device=dev)
        off, _ = vf.delay_table(self.L, dm_grid())
        self.plan = vf.DedispPlan(off)
        self.md = self.plan.max_delay
        R = 1 << math.ceil(math.log2(self.rows + self.md + 1024))
        self.R = R
        dt = {0: torch.float32, 1: torch.float16}[storage]
        self.ring = torch.zeros((nch, R), dtype=dt, device=dev)
        # FP16: the ring shifted by one row as well (written by the bandpass),
        # so the dedisperser reads windows of halves with 4-byte loads
        self.ring1 = torch.zeros_like(self.ring) if storage == 1 else None
        self.out = torch.empty((NDM, self.rows), dtype=torch.float32, device=dev)
        self.ws = torch.empty(self.plan.workspace_bytes(self.rows), dtype=torch.uint8, device=dev)
        self.scale = None
        self.k = 0
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        self.t_k = [0.0, 0.0, 0.0]
        self.n_timed = 0
        self.uscale = 0.0
        if storage != 0:
            # FP16 form: one scale per stream from the first window's variance
            vf.channelise(frames, self.s0, self.s1, 0, 128, self.L, out=self.raw)
            var = torch.empty((1, nch), device=dev)
            vf.bandpass(self.raw, nrows=128, win_var=var)
            S = float(torch.sqrt(torch.clamp(var[0], min=0).mean()).item())
            self.uscale = S
            self.inv = torch.full((nch,), 1.0 / S, device=dev)
        self.tune = self.plan.autotune(storage, self.rows)
        if variant:  # pinned kernel (profiling commands: the same kernel as the timed run)
            self.plan.set_variant(storage, variant)

    def step(self, timed=False):
        vf, torch = self.vf, self.torch
        k = self.k
        ev = self.ev
        if timed:
            ev[0].record()
        vf.channelise(self.frames, self.s0, self.s1, 0, self.rows, self.L, out=self.raw)
        if timed:
            ev[1].record()
        r0 = k * self.rows
        vf.bandpass(self.raw, storage=self.storage, out=self.ring, out_row0=r0, out_row_mask=self.R - 1,
                    inv_scale=self.inv if self.storage else None, out_shift1=self.ring1)
        if timed:
            ev[2].record()
        if k == 0:
            row0, nt = 0, self.rows - self.md
        else:
            row0, nt = r0 - self.md, self.rows
        out, st = self.plan(self.ring, nt, storage=self.storage, uniform_scale=self.uscale, row0=row0,
                            row_mask=self.R - 1, nrows_valid=nt + self.md, out=self.out, workspace=self.ws,
                            fb_shift1=self.ring1)
        self.stats = st
        if timed:
            ev[3].record()
        self.k += 1
        return nt

    def collect(self):
        e = self.ev
        return (e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), e[2].elapsed_time(e[3]))


def run_device(vf, frames, storage, steps, warmup, dist, variant=0):
    import torch
    pipe = DevicePipeline(vf, frames, storage, variant)
    for _ in range(max(warmup, 1)):
        pipe.step()
    torch.cuda.synchronize()
    stage = np.zeros(3)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(torch.cuda.current_device())
    dist_barrier(dist)
    torch.cuda.synchronize()
    with clk:
        start.record()
        for _ in range(steps):
            pipe.step(timed=True)
            torch.cuda.synchronize()  # so the per-step stage events can be read
            stage += np.array(pipe.collect())
        stop.record()
        torch.cuda.synchronize()
    dist_barrier(dist)
    ms = start.elapsed_time(stop) / steps
    ms = dist_max(dist, ms)
    stage /= steps
    return dict(ms=ms, stage_ms=stage.tolist(), rows=pipe.rows, md=pipe.md, clocks=clk.summary(),
                stats=pipe.stats, nchan=pipe.L.nchanout, launches=4, tune=pipe.tune,
                variant=pipe.plan.variant(storage))


# --------------------------------------------------------------------------- e2e through the plan API
def run_e2e(vf, host_frames, storage, steps, chunk_s=1.0, warmup=1):
    """Push the pinned 60 s buffer through vfrb_push_frames in 1-s pieces and
    poll every result; the stream continues across steps (frame numbers wrap
    consistently).  Returns seconds per step, bytes, latencies."""
    import torch
    plan = vf.Plan(dm_grid(), nave=NAVE, muoslowfreq=384.0, mode=vf.MODE_STREAM, storage=storage,
                   chunk_seconds=chunk_s, ring_seconds=2.0, outputs=vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=7.0)
    piece = 2 * 25600 * 5032  # one second of frames
    n = host_frames.numel()
    lat, cands, d2h = [], [], 0

    def one_step(record):
        nonlocal d2h
        for off in range(0, n, piece):
            plan.push(0, host_frames[off:off + piece])
            while True:
                r = plan.poll(wait=False)
                if r is None:
                    break
                if record:
                    lat.append(r["latency_ms"])
                    cands.extend(r["cands"])
                    d2h += NDM * 4 * 5
        torch.cuda.synchronize()

    for _ in range(warmup):
        one_step(False)
    t0 = time.perf_counter()
    for _ in range(steps):
        one_step(True)
    # drain what is in flight for this batch
    while True:
        r = plan.poll(wait=False)
        if r is None:
            break
        lat.append(r["latency_ms"])
        d2h += NDM * 4 * 5
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    plan.close()
    return dict(s_per_step=dt, h2d=n, d2h=d2h / steps, lat=lat, cands=cands, dev_bytes=None)


# --------------------------------------------------------------------------- baselines
_CPU_CACHE = {}


def run_serving(vf, storage, nstreams=16, paced_s=15.0, load=1.5, seed0=100):
    """The serving configuration: nstreams independent streams (seeds 100..,
    one dispersed pulse each) whose bytes arrive in chunks of U(0.5, 8.0) s
    (cut anywhere, not frame-aligned).  Each stream's frames are generated on
    the device as its chunks are needed (headers continue across chunks) and
    pushed from page-locked host memory.  First every stream is filled back
    to back past its pulse's output chunk plus the 12.4-s DM-1000 overlap,
    so every pulse is searched; then, for paced_s seconds, chunks arrive as
    one Poisson process with a mean gap of 1.25/load s (1.2 chunks/s at load
    1.5, i.e. 5.1 data-seconds per second on average for the mean 4.25-s
    chunk: more than the configuration's 1.5x real time; the rate realised,
    which the pushes' own time lowers, is returned as `offered`) and results
    are polled as they complete.  Returns the chunk latencies of that phase (data pushed
    -> result on the host) and every candidate."""
    import torch
    from vlite_frb_b200 import synth
    fps, pair = 25600, 2 * 5032
    # streams are admitted one by one as their data starts (vfrb_stream_open)
    plan = vf.Plan(dm_grid(), nave=NAVE, muoslowfreq=384.0, mode=vf.MODE_STREAM, storage=storage,
                   chunk_seconds=1.0, ring_seconds=2.0, nstreams=0,
                   outputs=vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=7.0)
    sid = []
    tchan = NAVE * 12500 / 128e6
    # the last pulse (t0 = 2.1 s) sits in output chunk 2 (rows 2048-3071)
    fill_s = (plan.max_delay + 3 * 1024) * tchan + 0.1
    buf = torch.empty(int(8.0 * fps + 2) * pair, dtype=torch.uint8, pin_memory=True)
    rng = np.random.default_rng(seed0)
    st = [{"pair": 0, "k": 0, "tail": torch.empty(0, dtype=torch.uint8), "sent": 0.0} for _ in range(nstreams)]
    # output sample t needs rows up to t + max_delay: pulses early in the
    # streams are searched once the paced data extend past their sweeps
    pulse = [(0.3 + 0.12 * i, 150.0 + 50.0 * i) for i in range(nstreams)]

    def push_chunk(i):
        s = st[i]
        nbytes = int(rng.uniform(0.5, 8.0) * fps * pair)
        nt = s["tail"].numel()
        buf[:nt] = s["tail"]
        npairs = max(0, -(-(nbytes - nt) // pair))
        total = nt
        if npairs:
            t0, dm = pulse[i]
            spec = synth.StreamSpec(duration=npairs / fps, seed=(seed0 + i) * 1000 + s["k"], frame0=s["pair"],
                                    pulses=[synth.Pulse(t0 - s["pair"] / fps, dm, 3.0, 25.0)])
            f = synth.make_vdif(spec, device="cuda")
            buf[nt:nt + f.numel()].copy_(f)
            total += f.numel()
            s["pair"] += npairs
            s["k"] += 1
        plan.push(sid[i], buf[:nbytes])
        s["tail"] = buf[nbytes:total].clone()
        s["sent"] += nbytes / (fps * pair)
        return nbytes / (fps * pair)

    lat, cands = [], []

    def drain(record, wait=False):
        while True:
            r = plan.poll(wait=wait)
            if r is None:
                return
            if record:
                lat.append(r["latency_ms"])
            cands.extend((r["stream"], c["dm_index"], c["t"], round(c["snr"], 4)) for c in r["cands"])

    for i in range(nstreams):  # admit each stream and fill it past the overlap, back to back
        k = plan.open_stream()
        if k is None:
            raise RuntimeError("stream %d not admitted" % i)
        sid.append(k)
        while st[i]["sent"] < fill_s:
            push_chunk(i)
            drain(False)
    drain(False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_next, data_s = t0, 0.0
    while time.perf_counter() - t0 < paced_s:
        t_next += rng.exponential(1.25 / load)
        while time.perf_counter() < t_next:
            drain(True)
        data_s += push_chunk(int(rng.integers(nstreams)))
        drain(True)
    wall = time.perf_counter() - t0
    for i in range(nstreams):
        plan.push(sid[i], None)
    drain(True, wait=True)
    for i in range(nstreams):
        plan.close_stream(sid[i])
    plan.close()
    return dict(lat=np.array(lat), cands=sorted(cands), offered=data_s / wall,
                data_s=sum(s["sent"] for s in st))


def run_capacity(vf, storage, nstreams=16, seconds_per_stream=24.0, seed0=100, buf_s=4.0, batch=1):
    """Serving capacity with the input already on the GPU: nstreams streams
    (seeds 100..), each a continuous stream built from a buf_s-second
    device-resident buffer repeated with its VDIF seconds advanced, arrive
    in chunks of U(0.5, 8) s of bytes (cut anywhere), as fast as the engine
    takes them (vfrb_push_frames with device memory: no PCIe).  The chunks
    come in rounds -- one for every live stream, in random order -- after
    which results are polled; with batch = 1 the dedispersion of the chunks
    a round completes runs as shared launches across the streams
    (batch_streams).  Returns the aggregate real-time factor (data seconds
    of all streams / wall seconds) and the chunk latencies."""
    import torch
    synth = load_synth()
    fps, pair = 25600, 2 * 5032
    plan = vf.Plan(dm_grid(), nave=NAVE, muoslowfreq=384.0, mode=vf.MODE_STREAM, storage=storage,
                   chunk_seconds=1.0, ring_seconds=2.0, nstreams=0, outputs=vf.OUT_DMSTATS | vf.OUT_CANDS,
                   cand_snr=7.0, batch_streams=batch)
    sid = [plan.open_stream() for _ in range(nstreams)]
    if any(k is None for k in sid):
        raise RuntimeError("capacity leg: streams not admitted")
    bufs = [synth.make_vdif(synth.StreamSpec(duration=buf_s, seed=seed0 + i), device="cuda") for i in range(nstreams)]
    nb = bufs[0].numel()
    words = [b.view(torch.int32).view(-1, 1258) for b in bufs]  # word 0 of each frame: seconds (30 bits)
    sec0 = [w[:, 0].clone() for w in words]
    rng = np.random.default_rng(seed0)
    total = int(seconds_per_stream * fps) * pair
    pos = [0] * nstreams
    lat = []

    def push_chunk(i, n):
        while n > 0:
            rep, off = divmod(pos[i], nb)
            if off == 0:  # a new repetition: advance the seconds of every frame
                words[i][:, 0] = sec0[i] + int(rep * buf_s)
            take = min(n, nb - off)
            plan.push(sid[i], bufs[i][off:off + take])
            pos[i] += take
            n -= take

    def drain(wait=False):
        while True:
            r = plan.poll(wait=wait)
            if r is None:
                return
            lat.append(r["latency_ms"])

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    live = list(range(nstreams))
    while live:
        for i in [live[k] for k in rng.permutation(len(live))]:
            n = min(int(rng.uniform(0.5, 8.0) * fps * pair), total - pos[i])
            push_chunk(i, n)
            if pos[i] >= total:
                plan.push(sid[i], None)
                live.remove(i)
        drain()
    drain(wait=True)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    for k in sid:
        plan.close_stream(k)
    plan.close()
    data_s = nstreams * total / (fps * pair)
    return dict(rtf=data_s / wall, lat=np.array(lat), data_s=data_s, wall=wall)


def run_capacity_threads(vf, storage, nstreams=16, seconds_per_stream=24.0, seed0=100, buf_s=4.0):
    """The capacity leg's streams served by one single-stream plan each, every
    plan pushed and polled by its own host thread (a plan is driven by one
    thread at a time; plans are independent, so their host work -- header
    reading, launches, copy waits -- runs in parallel).  Same data, chunking
    and measure as run_capacity."""
    import threading
    import torch
    synth = load_synth()
    fps, pair = 25600, 2 * 5032
    plans = [vf.Plan(dm_grid(), nave=NAVE, muoslowfreq=384.0, mode=vf.MODE_STREAM, storage=storage,
                     chunk_seconds=1.0, ring_seconds=2.0, outputs=vf.OUT_DMSTATS | vf.OUT_CANDS, cand_snr=7.0)
             for _ in range(nstreams)]
    bufs = [synth.make_vdif(synth.StreamSpec(duration=buf_s, seed=seed0 + i), device="cuda") for i in range(nstreams)]
    nb = bufs[0].numel()
    words = [b.view(torch.int32).view(-1, 1258) for b in bufs]  # word 0 of each frame: seconds (30 bits)
    sec0 = [w[:, 0].clone() for w in words]
    total = int(seconds_per_stream * fps) * pair
    lat = [[] for _ in range(nstreams)]
    errors = []

    def serve(i):
        try:
            rng = np.random.default_rng(seed0 + i)
            plan, pos = plans[i], 0
            while pos < total:
                n = min(int(rng.uniform(0.5, 8.0) * fps * pair), total - pos)
                while n > 0:
                    rep, off = divmod(pos, nb)
                    if off == 0:  # a new repetition: advance the seconds of every frame
                        words[i][:, 0] = sec0[i] + int(rep * buf_s)
                    take = min(n, nb - off)
                    plan.push(0, bufs[i][off:off + take])
                    pos += take
                    n -= take
                while True:
                    r = plan.poll(wait=False)
                    if r is None:
                        break
                    lat[i].append(r["latency_ms"])
            plan.push(0, None)
            lat[i].extend(r["latency_ms"] for r in plan.drain())
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    threads = [threading.Thread(target=serve, args=(i,)) for i in range(nstreams)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    for p in plans:
        p.close()
    if errors:
        raise errors[0]
    data_s = nstreams * total / (fps * pair)
    return dict(rtf=data_s / wall, lat=np.concatenate([np.array(x) for x in lat]), data_s=data_s, wall=wall)


def cpu_baseline(sample_s=1.0, min_cpu_s=0.0):
    """The oracle's FP32 C/OpenMP port on the host cores, on `sample_s` seconds
    of the workload (full 2048 trials, 6250 channels): channelise, bandpass,
    the transpose to the channel-major layout, dedisperse and per-trial
    statistics, all inside the timed region.  The pass repeats until at least
    `min_cpu_s` seconds of CPU time have been measured; the figures are per
    pass."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    if "co" not in _CPU_CACHE:
        subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "build_oracle.py")], check=False,
                       capture_output=True)
        from coracle import COracle  # the CPU port is the timed baseline only
        import vfrb_oracle as O
        synth = load_synth()
        co = COracle(32)
        L = O.Layout(nave=NAVE, muoslowfreq=384.0)
        off, md = O.delay_table(dm_grid(), L.fch1, L.chanbw, L.tchan, L.nchanout)
        nrow_s = int(round(sample_s / L.tchan))
        buf = synth.make_vdif(synth.StreamSpec(duration=sample_s + 0.02, seed=SEED)).numpy().reshape(-1, 2, 5032)
        p0 = np.ascontiguousarray(buf[:, 0, 32:].reshape(-1))
        p1 = np.ascontiguousarray(buf[:, 1, 32:].reshape(-1))
        cm_rows = nrow_s + int(off.max())
        cm = np.random.default_rng(0).standard_normal((L.nchanout, cm_rows)).astype(np.float32)
        _CPU_CACHE.update(co=co, L=L, off=off, nrow_s=nrow_s, p0=p0, p1=p1, cm=cm)
    c = _CPU_CACHE
    co, L, off, nrow_s, cm = c["co"], c["L"], c["off"], c["nrow_s"], c["cm"]
    tot = np.zeros(4)
    npass = 0
    while npass == 0 or tot.sum() < min_cpu_s:
        t0 = time.perf_counter()
        fb = co.channelise(c["p0"], c["p1"], L)[:nrow_s]
        t1 = time.perf_counter()
        bp = co.bandpass(fb)
        t2 = time.perf_counter()
        cm[:, :nrow_s] = co.transpose(bp)  # the rows past the sample stand in for the carried overlap
        t3 = time.perf_counter()
        dd = co.dedisperse_cm(cm, off, nrow_s)
        co.calcstats_dm(dd)
        t4 = time.perf_counter()
        tot += (t1 - t0, t2 - t1, t3 - t2, t4 - t3)
        npass += 1
    per = tot / npass
    secs = float(per.sum())
    rtf = sample_s / secs
    return dict(value=rtf, unit="s data/s", cores=co.threads(), kind="port",
                sample=f"{sample_s:g} s of the workload per pass ({npass} passes) through channelise + bandpass + "
                       f"transpose + dedisperse (2048 trials) + stats (FP32 C/OpenMP port of the oracle): per pass "
                       f"channelise {per[0]:.3f} s, bandpass {per[1]:.3f} s, transpose {per[2]:.3f} s, "
                       f"dedisperse {per[3]:.3f} s", seconds=secs)


def gpu_reference_baseline(vf, sample_bundles=32):
    """The reference's own CUDA chain (cuFFT + its kernels, built from its
    sources) on a sample: channeliser over `sample_bundles` bundles and the
    in-tree dedisperse + calcstats over 1 s of outputs, 2048 trials."""
    p = os.path.join(ROOT, "oracle", "_ref", "libref_pipe.so")
    if not os.path.exists(p):
        return None
    synth = load_synth()
    lib = C.CDLL(p)
    vp, ci, cf = C.c_void_p, C.c_int, C.POINTER(C.c_float)
    lib.ref_gpu_channelise.argtypes = [vp, vp, ci, ci, ci, ci, ci, ci, vp, cf]
    lib.ref_gpu_dedisperse.argtypes = [vp, ci, ci, vp, ci, ci, vp, vp, vp, vp, vp, vp, cf]
    L = vf.layout(nave=NAVE, muoslowfreq=384.0)
    dur = sample_bundles * L.nloop / 128e6 + 0.01
    buf = synth.make_vdif(synth.StreamSpec(duration=dur, seed=SEED)).numpy().reshape(-1, 2, 5032)
    p0 = np.ascontiguousarray(buf[:, 0, 32:].reshape(-1))
    p1 = np.ascontiguousarray(buf[:, 1, 32:].reshape(-1))
    rows = sample_bundles * L.nbundle
    fb = np.zeros((rows, L.nchanout), np.float32)
    ms_c = C.c_float(0)
    st = lib.ref_gpu_channelise(p0.ctypes.data, p1.ctypes.data, sample_bundles, L.twonchan, NAVE, L.nbundle, L.nskip,
                                L.nchanout, fb.ctypes.data, C.byref(ms_c))
    if st:
        return dict(error=f"ref_gpu_channelise status {st}")
    off, _ = vf.delay_table(L, dm_grid())
    nt = 1024
    md = int(off.max())
    rng = np.random.default_rng(1)
    big = rng.standard_normal((nt + md, L.nchanout)).astype(np.float32)
    out = np.zeros((NDM, nt), np.float32)
    z = [np.zeros(NDM, np.float32) for _ in range(3)]
    frb = np.zeros(NDM, np.int32)
    ms_d = C.c_float(0)
    st = lib.ref_gpu_dedisperse(big.ctypes.data, nt + md, L.nchanout, np.ascontiguousarray(off).ctypes.data, NDM, nt,
                                out.ctypes.data, None, frb.ctypes.data, z[0].ctypes.data, z[1].ctypes.data,
                                z[2].ctypes.data, C.byref(ms_d))
    if st:
        return dict(error=f"ref_gpu_dedisperse status {st}")
    data_s = rows * L.tchan
    ms_per_s = ms_c.value / data_s + ms_d.value / (nt * L.tchan)
    return dict(value=1000.0 / ms_per_s, unit="s data/s",
                channelise_ms_per_data_s=ms_c.value / data_s,
                dedisperse_calcstats_ms_per_data_s=ms_d.value / (nt * L.tchan),
                sample=f"reference cuFFT channeliser chain ({sample_bundles} bundles, synchronous per-bundle "
                       f"copies as PIPE:574-632) + in-tree dedisperse + calcstats (PIPE:1517, 1337) on {nt} "
                       f"samples x {NDM} trials; dedisp library unavailable")


# --------------------------------------------------------------------------- distributed helpers
def dist_init(n, backend="nccl", timeout_s=120):
    """One process per GPU (torchrun env).  The only collective on the path is
    the max-over-ranks of the step time; a short process-group timeout makes a
    rank that left end the others' next collective with an error."""
    if n <= 1 and "RANK" not in os.environ:
        return None
    import datetime
    import torch
    import torch.distributed as d
    rank = int(os.environ.get("RANK", 0))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if backend == "nccl":
        torch.cuda.set_device(local)
    d.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dict(rank=rank, world=d.get_world_size(), local=local, device="cuda" if backend == "nccl" else "cpu")


def stream_seed(rank):
    """Each rank synthesises and processes its own independent stream (antenna)."""
    return SEED + 1000 * rank


def dist_barrier(dist):
    if dist:
        import torch.distributed as d
        d.barrier()


def dist_max(dist, v):
    if not dist:
        return v
    import torch
    import torch.distributed as d
    t = torch.tensor([v], dtype=torch.float64, device=dist.get("device", "cuda"))
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------- arms
def reference_arm(args):
    """The reference arm: the reference has no CPU implementation of the path
    (its three tools are CUDA programs), so this times the oracle's FP32
    C/OpenMP port on the host cores with every host thread.  Each step is one
    pass over a bounded sample (`--cpu-sample` seconds of the workload, all
    2048 trials and 6250 channels), and ms_per_step is that pass's time.
    Under torchrun only rank 0 runs; the others exit at once."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    K, W = args.steps, args.warmup
    vals = []
    base = None
    for i in range(W + K):
        base = cpu_baseline(sample_s=args.cpu_sample)
        if i >= W:
            vals.append(base["seconds"])
    secs = float(np.mean(vals))
    value = args.cpu_sample / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s data/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": secs * 1000.0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded VLITE VDIF stand-in; no public dataset)",
            "config": bench_config(args.duration, args.gpus),
            "cpu_baseline": {"value": value, "unit": "s data/s", "cores": base["cores"], "kind": "port",
                             "sample": f"each step: {base['sample']}"},
            "e2e": {"value": value, "unit": "s data/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--duration", type=float, default=DURATION)
    ap.add_argument("--cpu-sample", type=float, default=1.0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--skip-extras", action="store_true",
                    help="only the primary line items and the FP16 device leg (no FP16 e2e, serving, capacity or "
                         "baselines)")
    ap.add_argument("--dd-variant", type=int, default=0,
                    help="dedispersion kernel variant for the device legs (0: the autotuner's choice)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)
    dist = dist_init(args.gpus)
    import torch
    vf = load_pkg()
    from vlite_frb_b200 import synth
    rank = dist["rank"] if dist else 0
    world = dist["world"] if dist else 1
    dev = torch.device("cuda")
    # each rank processes its own independent stream (antenna): weak scaling, no collective on the data path
    spec = synth.StreamSpec(duration=args.duration, seed=stream_seed(rank),
                            pulses=synth.injected_pulses(SEED, 20, args.duration, 50.0, DM_MAX))
    t_gen = time.perf_counter()
    frames = synth.make_vdif(spec, device=dev)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    data_s = args.duration

    f32 = run_device(vf, frames, 0, args.steps, args.warmup, dist, args.dd_variant)
    rtf = world * data_s / (f32["ms"] / 1000.0)
    # the FP16 form on the same resident data: the metric compares it with the FP32 form
    f16 = run_device(vf, frames, 1, args.steps, args.warmup, dist, args.dd_variant)
    # e2e through the public plan API from page-locked host memory
    host = torch.empty(frames.numel(), dtype=torch.uint8, pin_memory=True)
    host.copy_(frames)
    del frames
    torch.cuda.empty_cache()
    e2e = run_e2e(vf, host, 0, args.e2e_steps)
    e2e16 = run_e2e(vf, host, 1, args.e2e_steps) if not args.skip_extras else None
    del host
    e2e_s = dist_max(dist, e2e["s_per_step"])
    e2e_rtf = world * data_s / e2e_s
    # every rank takes the same collectives: the FP16 leg runs on all or none
    e2e16_s = dist_max(dist, e2e16["s_per_step"]) if e2e16 is not None else None
    lat = np.array(e2e["lat"]) if e2e["lat"] else np.array([float("nan")])
    if rank != 0:
        return 0
    # roofline of the dominant kernel (dedispersion, K3): it is bound by the
    # FP32 add rate (and the shared-memory reads that feed it), not by HBM
    from json import dumps
    nt, nch = f32["rows"], f32["nchan"]
    k3_ms = f32["stage_ms"][2]
    units = NDM * nt
    eff_bytes = units * nch * 4  # no-reuse convention: NCHANOUT * 4 B per DM-trial.sample
    comp_bytes = (nt + f32["md"]) * nch * 4 + units * 4
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    sm_mhz = float(peaks.get("sm_max_mhz") or f32["clocks"].get("sm_max_mhz") or 1965.0)
    fp32_peak_adds = nsm * 128 * sm_mhz * 1e6  # 128 FP32 lanes per SM
    adds_per_s = units * nch / (k3_ms / 1000.0)
    traffic, traffic_src = None, None
    try:  # DRAM bytes of a 16-s ncu capture of this kernel, scaled by output samples
        tr = json.load(open(os.path.join(ROOT, "profiles", "dedisperse_traffic.json")))
        traffic = tr["bytes_per_launch"] * (units / float(tr["units_per_launch"]))
        traffic_src = tr.get("source")
    except Exception:
        pass
    # K1: compulsory bytes = raw VDIF read + FP32 filterbank written
    k1_ms = f32["stage_ms"][0]
    k1_bytes = data_s * (2 * 25600 * 5032 + nch * (1.0 / (NAVE * 12500 / 128e6)) * 4)
    # K1 FFT work at the usual real-FFT count: 2.5 N log2 N per 12500-sample transform
    k1_flop = data_s * 2 * (128e6 / 12500) * 2.5 * 12500 * math.log2(12500)
    roofline = {"bound": "fp32_add", "achieved": adds_per_s / 1e12, "peak": fp32_peak_adds / 1e12,
                "unit": "Tadd/s", "frac": adds_per_s / fp32_peak_adds, "traffic": traffic,
                "kernel": "dedisperse (K3)",
                "peak_source": f"{nsm} SMs x 128 FP32 lanes x {sm_mhz:g} MHz (MEASURED_PEAKS.json has no FP32 "
                               f"figure)",
                "traffic_source": traffic_src,
                "hbm_no_reuse": {"achieved_gbs": eff_bytes / (k3_ms / 1000.0) / 1e9, "peak_gbs": hbm,
                                 "frac": eff_bytes / (k3_ms / 1000.0) / 1e9 / hbm,
                                 "convention": "NCHANOUT*4 B per DM-trial.sample, no reuse (values > 1 = on-chip "
                                               "reuse); peak " + peak_src},
                "compulsory_gbs": comp_bytes / (k3_ms / 1000.0) / 1e9,
                "k1_channelise": {"bound": "hbm", "achieved_gbs": k1_bytes / (k1_ms / 1000.0) / 1e9,
                                  "peak_gbs": hbm, "frac": k1_bytes / (k1_ms / 1000.0) / 1e9 / hbm,
                                  "bytes_per_step": k1_bytes,
                                  "note": "compulsory bytes (raw VDIF in + FP32 filterbank out); peak " + peak_src,
                                  "fp32": {"achieved_tflops": k1_flop / (k1_ms / 1000.0) / 1e12,
                                           "peak_tflops": 2 * fp32_peak_adds / 1e12,
                                           "frac": k1_flop / (k1_ms / 1000.0) / (2 * fp32_peak_adds),
                                           "flop_per_step": k1_flop,
                                           "convention": "2.5 N log2 N flop per real N = 12500 transform, two "
                                                         "per window (one per pol); peak = 2 flop x 128 FP32 "
                                                         "lanes per SM x SMs x clock"}}}
    line = {
        "metric": METRIC,
        "value": rtf,
        "unit": "s data/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": f32["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded VLITE VDIF stand-in generated on the device; no public dataset)",
        "config": bench_config(data_s, world),
        "roofline": roofline,
        "clocks": f32["clocks"],
        "stages_ms_per_step": {"channelise_K1": f32["stage_ms"][0], "bandpass_K2": f32["stage_ms"][1],
                               "dedisperse_stats_K3": f32["stage_ms"][2]},
        "dm_trial_samples_per_s": world * units / (f32["ms"] / 1000.0),
        "e2e": {"value": e2e_rtf, "unit": "s data/s", "h2d_bytes_per_step": int(e2e["h2d"]),
                "d2h_bytes_per_step": int(e2e["d2h"]), "steps": args.e2e_steps,
                "api": "vfrb_push_frames/vfrb_poll (stream mode, 1 s chunks), pinned host input"},
        "latency_ms": {"p50": float(np.nanpercentile(lat, 50)), "p99": float(np.nanpercentile(lat, 99)),
                       "chunk_ms": 1000.0, "n": int(len(lat))},
        "gpu_launches": f32["launches"] * args.steps,
        "dedisperse_autotune_ms": {"variant": f32["variant"], "times": {str(k): v for k, v in f32["tune"].items()}},
        "gen_seconds": t_gen,
    }
    if f16 is not None:
        k3_16 = units * nch / (f16["stage_ms"][2] / 1000.0)  # FP32 adds per second of the FP16 form's K3
        line["fp16"] = {"value": world * data_s / (f16["ms"] / 1000.0), "ms_per_step": f16["ms"],
                        "stages_ms_per_step": f16["stage_ms"], "speedup_vs_f32": f32["ms"] / f16["ms"],
                        "dedisperse_speedup_vs_f32": f32["stage_ms"][2] / f16["stage_ms"][2],
                        "dedisperse_add_rate_tadd_s": k3_16 / 1e12,
                        "dedisperse_fp32_add_peak_frac": k3_16 / fp32_peak_adds,
                        "autotune_ms": {"variant": f16["variant"], "times": {str(k): v for k, v in f16["tune"].items()}}}
        if e2e16_s is not None:  # through the plan API as well (PCIe-bound like the FP32 figure)
            line["fp16"]["e2e"] = {"value": world * data_s / e2e16_s, "unit": "s data/s",
                                   "h2d_bytes_per_step": int(e2e16["h2d"]), "d2h_bytes_per_step": int(e2e16["d2h"])}
    if not args.skip_extras:
        try:
            line["cpu_baseline"] = {k: v for k, v in cpu_baseline(args.cpu_sample, min_cpu_s=10.0).items() if k != "seconds"}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        try:
            line["gpu_reference"] = gpu_reference_baseline(vf)
        except Exception as e:  # noqa: BLE001
            line["gpu_reference"] = {"error": str(e)[:200]}
    if not args.skip_extras and world == 1:
        try:
            sv, cl = {}, {}
            for name, st in (("fp32", 0), ("fp16", 1)):
                r = run_serving(vf, st)
                lt = r["lat"]
                sv[name] = {"p50_ms": float(np.percentile(lt, 50)) if lt.size else None,
                            "p99_ms": float(np.percentile(lt, 99)) if lt.size else None,
                            "results": int(lt.size), "offered_rtf": r["offered"],
                            "data_seconds": r["data_s"], "candidates": len(r["cands"])}
                cl[name] = r["cands"]
            same = [x[:3] for x in cl["fp32"]] == [x[:3] for x in cl["fp16"]]
            dsnr = max((abs(x[3] - y[3]) / x[3] for x, y in zip(cl["fp32"], cl["fp16"])), default=0.0) if same \
                else None
            line["serving"] = {"streams": 16, "arrivals": "Poisson, 1.2 chunks/s (5.1x real time offered on average, "
                                                          "at least the configuration's 1.5x; offered_rtf = realised), "
                                                          "after a back-to-back fill past every pulse's chunk and the "
                                                          "12.4-s overlap",
                               "chunk_bytes": "U(0.5, 8.0) s, not frame-aligned", "output_chunk_ms": 1000.0,
                               "input": "page-locked host memory", **sv, "candidates_identical": same,
                               "max_dsnr": dsnr}
        except Exception as e:  # noqa: BLE001
            line["serving"] = {"error": str(e)[:200]}
        try:
            cap = {}
            for name, st, batch in (("fp32", 0, 1), ("fp16", 1, 1), ("fp32_per_stream_launches", 0, 0),
                                    ("fp32_plan_per_thread", 0, None), ("fp16_plan_per_thread", 1, None)):
                r = run_capacity(vf, st, batch=batch) if batch is not None else run_capacity_threads(vf, st)
                lt = r["lat"]
                cap[name] = {"rtf": r["rtf"], "p50_ms": float(np.percentile(lt, 50)),
                             "p99_ms": float(np.percentile(lt, 99)), "results": int(lt.size),
                             "data_seconds": r["data_s"], "wall_s": r["wall"]}
            line["capacity"] = {"streams": 16, "chunk_bytes": "U(0.5, 8.0) s, not frame-aligned, in rounds of one "
                                                              "chunk per stream (random order), as fast as accepted",
                                "dedispersion": "shared launches across the streams of a round (batch_streams), "
                                                "per-stream launches for comparison",
                                "plan_per_thread": "each stream in its own single-stream plan, pushed and polled "
                                                   "by its own host thread (chunks as they come, no rounds)",
                                "input": "device memory (vfrb_push_frames from the GPU: no PCIe)",
                                "output_chunk_ms": 1000.0, **cap,
                                "fp16_over_fp32": cap["fp16"]["rtf"] / cap["fp32"]["rtf"]}
        except Exception as e:  # noqa: BLE001
            line["capacity"] = {"error": str(e)[:200]}
    line["e2e_candidates"] = len(e2e["cands"])
    # the same candidates clustered across trials and chunks (vfrb_cluster_cands:
    # within 16 trials and 50 samples), i.e. one entry per detected pulse
    line["e2e_clusters"] = len(vf.cluster_cands(e2e["cands"], dm_tol=16, t_tol=50)[0])
    print(dumps(line))
    if dist:
        import torch.distributed as d
        d.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
