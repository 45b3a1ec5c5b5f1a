"""Seeded synthetic VLITE VDIF streams (stand-in for the absent VLITE recordings).

Frame format (VDIF v0): 32-byte header + 5000-byte payload, framelength8 =
629, 8-bit real offset-binary samples, log2nchan 0, threads 0/1 alternating
with equal frame numbers 0..25599 per second, seconds incrementing, fixed
epoch.  Samples are clip(round(128 + 12*N(0,1)), 0, 255).

Dispersed pulses are injected per 12500-sample block in the frequency
domain: the noise spectrum's bin k (sky frequency 384 - k*64/6250 MHz, the
band is spectrally inverted) is scaled by sqrt(1 + A*g(t_blk - t0 - delay_k))
with a Gaussian g of the given FWHM, then inverse-transformed.  A is set from
the target matched-filter SNR with the radiometer estimate
    SNR = A * sqrt(2 * NAVE * NCHAN * sum_t g(t)^2)
(2*NAVE exponential power samples per channel-row, NCHAN channels averaged).

RFI (optional): narrowband sinusoids, broadband bursts that multiply the
noise of 1-ms blocks by a factor, and the VDIF invalid bit on a fraction of
frames.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

FRAMELEN, HDRLEN, DATALEN, FPS = 5032, 32, 5000, 25600
RATE = 128e6
NBLK = 12500
DELAY_CONST = 4.148808e3


@dataclass
class Pulse:
    t0: float          # arrival time at the top of the band (384 MHz), s from stream start
    dm: float
    fwhm_ms: float = 2.0
    snr: float = 20.0


@dataclass
class Rfi:
    n_tones: int = 40
    tone_amp: tuple = (5.0, 50.0)
    burst_frac: float = 0.01
    burst_gain: float = 8.0
    invalid_frac: float = 0.10
    seed: int | None = None       # tones, bursts and flags (None: the stream's seed)


@dataclass
class StreamSpec:
    duration: float
    seed: int = 0
    pulses: list = field(default_factory=list)
    rfi: Rfi | None = None
    seconds0: int = 1000          # VDIF seconds of the first frame
    frame0: int = 0               # first frame number (0 = on a 10 Hz cal boundary)
    epoch: int = 30               # 2015-01-01
    nave_for_snr: int = 10
    nchan_for_snr: int = 6250
    block0: int = 0               # 12500-sample block of the stream where this piece starts (RFI time base)


def injected_pulses(seed: int = 1, n: int = 20, duration: float = 60.0, dm_lo: float = 50.0,
                    dm_hi: float = 1000.0) -> list:
    """The dispersed pulses of the full-scale workload: n pulses with arrival
    time U(0.2, duration - 0.5) s at the top of the band, DM U(dm_lo, dm_hi),
    FWHM U(1, 10) ms and matched-filter SNR U(8, 30), from
    default_rng(seed + 7).  Returns Pulse objects."""
    rng = np.random.default_rng(seed + 7)
    out = []
    for _ in range(n):
        dm = float(rng.uniform(dm_lo, dm_hi))
        out.append(Pulse(float(rng.uniform(0.2, duration - 0.5)), dm, float(rng.uniform(1, 10)),
                         float(rng.uniform(8, 30))))
    return out


def _headers(nframes_pairs: int, spec: StreamSpec, invalid: np.ndarray | None) -> np.ndarray:
    """uint8 [npairs, 2, 32] headers."""
    idx = np.arange(nframes_pairs, dtype=np.int64) + spec.frame0
    sec = spec.seconds0 + idx // FPS
    frm = idx % FPS
    h = np.zeros((nframes_pairs, 2, 8), dtype=np.uint32)
    for p in (0, 1):
        w0 = (sec & 0x3FFFFFFF).astype(np.uint32)
        if invalid is not None:
            w0 |= (invalid[:, p].astype(np.uint32) << 31)
        h[:, p, 0] = w0
        h[:, p, 1] = (frm.astype(np.uint32) & 0xFFFFFF) | np.uint32((spec.epoch & 0x3F) << 24)
        h[:, p, 2] = np.uint32(629)  # framelength8; log2nchan 0; version 0
        h[:, p, 3] = np.uint32(ord("X") | ord("X") << 8) | np.uint32(p << 16) | np.uint32(7 << 26)
    return h.view(np.uint8).reshape(nframes_pairs, 2, 32)


def pulse_amplitude(snr: float, fwhm_ms: float, tsamp: float, nave: int, nchan: int) -> float:
    sig = fwhm_ms * 1e-3 / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    t = np.arange(-50, 51) * tsamp
    g2 = float(np.sum(np.exp(-(t ** 2) / (sig ** 2))))
    return snr / math.sqrt(2.0 * nave * nchan * g2)


def _inject(x: torch.Tensor, spec: StreamSpec):
    """x: float32 [nblk, 12500] zero-mean noise for one pol, modified in place."""
    if not spec.pulses:
        return
    nblk = x.shape[0]
    dev = x.device
    k = torch.arange(NBLK // 2 + 1, device=dev, dtype=torch.float64)
    fk = 384.0 - k * (64.0 / (NBLK // 2))
    tblk = (torch.arange(nblk, device=dev, dtype=torch.float64) + 0.5) * (NBLK / RATE)
    tsamp = spec.nave_for_snr * NBLK / RATE
    for p in spec.pulses:
        sig = p.fwhm_ms * 1e-3 / (2.0 * math.sqrt(2.0 * math.log(2.0)))
        A = pulse_amplitude(p.snr, p.fwhm_ms, tsamp, spec.nave_for_snr, spec.nchan_for_snr)
        delay = DELAY_CONST * p.dm * (fk ** -2 - 384.0 ** -2)
        lo = p.t0 - 6 * sig
        hi = p.t0 + float(delay.max()) + 6 * sig
        b0 = max(0, int(lo / (NBLK / RATE)))
        b1 = min(nblk, int(hi / (NBLK / RATE)) + 2)
        for s0 in range(b0, b1, 4096):
            s1 = min(b1, s0 + 4096)
            X = torch.fft.rfft(x[s0:s1].to(torch.float64), dim=1)
            dt = tblk[s0:s1, None] - p.t0 - delay[None, :]
            gain = torch.sqrt(1.0 + A * torch.exp(-(dt ** 2) / (2 * sig ** 2)))
            x[s0:s1] = torch.fft.irfft(X * gain, n=NBLK, dim=1).to(torch.float32)


def _rfi(x: torch.Tensor, spec: StreamSpec, gen: torch.Generator, pol: int, blk0: int):
    """x: float32 [nblk, 12500] noise of one pol whose first block is block
    blk0 of the stream; adds the tones and scales the bursts in place.  The
    tones A sin(w n + phi) are built per block by angle addition,
    sin(w (n0 + m) + phi) = sin(w m) cos(w n0 + phi) + cos(w m) sin(w n0 + phi),
    with the block phases in float64: one float32 matrix product."""
    r = spec.rfi
    dev = x.device
    nblk = x.shape[0]
    rseed = spec.seed if r.seed is None else r.seed
    rng = np.random.default_rng(rseed * 7919 + 17)
    freqs = rng.uniform(0.0, 64e6, r.n_tones)
    amps = rng.uniform(r.tone_amp[0], r.tone_amp[1], r.n_tones)
    phs = rng.uniform(0, 2 * math.pi, (2, r.n_tones))
    flat = x.view(-1)
    # bursts: 1-ms blocks (128000 samples) with noise scaled by burst_gain
    bl = 128000
    first = blk0 * NBLK // bl
    nb = (blk0 * NBLK + flat.numel() + bl - 1) // bl - first
    brng = np.random.default_rng(rseed * 104729 + 3)
    hit = np.nonzero(brng.random(first + nb)[first:] < r.burst_frac)[0]
    for b in hit:
        a0 = max(0, (first + b) * bl - blk0 * NBLK)
        a1 = min(flat.numel(), (first + b + 1) * bl - blk0 * NBLK)
        if a1 > a0:
            flat[a0:a1] *= r.burst_gain
    w = 2 * math.pi * freqs / RATE                                      # rad per sample
    m = np.arange(NBLK, dtype=np.float64)
    wm = np.outer(w, m)
    sc = np.concatenate([amps[:, None] * np.sin(wm), amps[:, None] * np.cos(wm)]).astype(np.float32)
    th = np.outer((np.arange(nblk, dtype=np.float64) + blk0) * NBLK, w) + phs[pol][None, :]
    coef = np.concatenate([np.cos(th), np.sin(th)], axis=1).astype(np.float32)  # [nblk, 2*ntones]
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        x += torch.from_numpy(coef).to(dev) @ torch.from_numpy(sc).to(dev)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def make_vdif(spec: StreamSpec, device: str | torch.device = "cpu") -> torch.Tensor:
    """Interleaved pol0/pol1 frames as a uint8 tensor of npairs*2*5032 bytes."""
    npairs = int(round(spec.duration * FPS))
    nsamp = npairs * DATALEN
    nblk = (nsamp + NBLK - 1) // NBLK
    gen = torch.Generator(device=device)
    gen.manual_seed(spec.seed)
    pols = []
    for pol in (0, 1):
        samples = torch.empty(nblk * NBLK, dtype=torch.uint8, device=device)
        step = 10240  # 1 s of 12500-sample blocks per piece
        for b0 in range(0, nblk, step):
            b1 = min(nblk, b0 + step)
            x = torch.randn((b1 - b0, NBLK), generator=gen, device=device, dtype=torch.float32) * 12.0
            if spec.pulses:
                sub = StreamSpec(**{**spec.__dict__})
                sub.pulses = [Pulse(p.t0 - b0 * NBLK / RATE, p.dm, p.fwhm_ms, p.snr) for p in spec.pulses]
                _inject(x, sub)
            if spec.rfi is not None:
                _rfi(x, spec, gen, pol, spec.block0 + b0)
            samples[b0 * NBLK:b1 * NBLK] = torch.clamp(torch.round(x + 128.0), 0, 255).to(torch.uint8).view(-1)
        pols.append(samples[:nsamp].view(npairs, DATALEN))
    pay = torch.stack(pols, dim=1)  # [npairs, 2, 5000]
    del pols
    invalid = None
    if spec.rfi is not None and spec.rfi.invalid_frac > 0:
        irng = np.random.default_rng(spec.seed * 31 + 5 + spec.frame0)
        invalid = irng.random((npairs, 2)) < spec.rfi.invalid_frac
    hdr = torch.from_numpy(_headers(npairs, spec, invalid)).to(device)
    frames = torch.cat([hdr, pay], dim=2)  # [npairs, 2, 5032]
    return frames.reshape(-1)


def edit_frames(buf: np.ndarray, drop=(), truncate: int = 0, lead_pol1: bool = False) -> np.ndarray:
    """Fault fixtures on an interleaved frame buffer (numpy uint8): drop frames
    by global frame index (2*pair + pol), start with a stray pol-1 frame, or
    cut the last `truncate` bytes."""
    fr = buf.reshape(-1, FRAMELEN)
    keep = np.ones(fr.shape[0], bool)
    keep[list(drop)] = False
    fr = fr[keep]
    out = fr.reshape(-1)
    if lead_pol1:
        out = np.concatenate([fr[1], out])
    if truncate:
        out = out[:-truncate]
    return np.ascontiguousarray(out)
