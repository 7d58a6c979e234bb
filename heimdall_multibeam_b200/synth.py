"""Seeded synthetic filterbanks for the single-pulse search.

The reference ships no test data; its only generator (Formats/giant_maker.C:
183-445) is not built.  This module writes filterbanks to the workload
definitions used for parity tests and the benchmark:

* Gaussian noise of mean 128 and standard deviation 16, rounded and clipped
  to uint8 [0, 255];
* dispersed Gaussian pulses with arrival time t_c = t0 + 4148.808 * DM *
  (f_c^-2 - f_top^-2) s (f in MHz) in channel c = 0 (top of the band) ... C-1;
* optional RFI: persistent narrow-band channels and zero-DM broadband bursts.

Pulse amplitude follows the optimal matched-filter definition of integrated
S/N: S/N = sqrt(sum_c sum_t s_c(t)^2) / sigma over the pulse footprint, so a
pulse of S/N 20 carries amplitude 20 * sigma / sqrt(sum g^2) per sample.
(giant_maker.C:344-365 uses a width-adjusted convention instead.)

Random numbers come from numpy's Philox4x32-10 counter-based generator keyed by
(seed, beam), so every beam is reproducible on its own and on any machine.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Tuple, List, Optional, Sequence

import numpy as np

DISPERSION_K = 4148.808  # s MHz^2 pc^-1 cm^3


@dataclasses.dataclass
class Pulse:
    t0: float          # arrival sample at the top of the band (channel 0)
    dm: float
    fwhm_s: float      # full width at half maximum, seconds
    snr: float         # integrated S/N (optimal matched filter)


@dataclasses.dataclass
class Beam:
    data: np.ndarray   # (nsamps, nchans) uint8, time-major
    pulses: List[Pulse]
    nchans: int
    dt: float
    f0: float
    df: float
    seed: int
    beam: int


def _rng(seed: int, beam: int) -> np.random.Generator:
    key = (int(seed) & 0xFFFFFFFF) << 32 | (int(beam) & 0xFFFFFFFF)
    return np.random.Generator(np.random.Philox(key=key))


def dispersion_delay_s(dm: float, f_mhz: np.ndarray, f_top: float) -> np.ndarray:
    return DISPERSION_K * dm * (f_mhz ** -2.0 - f_top ** -2.0)


def inject_pulse(x: np.ndarray, p: Pulse, dt: float, f0: float, df: float,
                 sigma: float = 16.0) -> None:
    """Adds one dispersed Gaussian pulse to the float filterbank x (in place)."""
    nsamps, nchans = x.shape
    f = f0 + df * np.arange(nchans)
    centres = p.t0 + dispersion_delay_s(p.dm, f, f0) / dt
    s = max(p.fwhm_s / dt / (2.0 * math.sqrt(2.0 * math.log(2.0))), 0.3)
    half = int(math.ceil(6.0 * s)) + 1
    prof = []
    energy = 0.0
    for c in range(nchans):
        lo = int(math.floor(centres[c])) - half
        hi = int(math.floor(centres[c])) + half + 1
        t = np.arange(lo, hi)
        g = np.exp(-0.5 * ((t - centres[c]) / s) ** 2)
        keep = (t >= 0) & (t < nsamps)
        prof.append((c, t[keep], g[keep]))
        energy += float(np.sum(g * g))
    if energy <= 0.0:
        return
    amp = p.snr * sigma / math.sqrt(energy)
    for c, t, g in prof:
        x[t, c] += amp * g


def make_beam(nsamps: int, nchans: int, dt: float, f0: float, df: float,
              pulses: Sequence[Pulse] = (), seed: int = 1, beam: int = 0,
              rfi_chan_frac: float = 0.0, n_bursts: int = 0,
              rng: Optional[np.random.Generator] = None) -> Beam:
    """One beam of noise + pulses (+ RFI), rounded and clipped to uint8."""
    g = rng if rng is not None else _rng(seed, beam)
    x = g.standard_normal((nsamps, nchans), dtype=np.float32)
    x *= 16.0
    x += 128.0
    for p in pulses:
        inject_pulse(x, p, dt, f0, df)
    if rfi_chan_frac > 0.0:
        nbad = int(round(rfi_chan_frac * nchans))
        bad = g.choice(nchans, size=nbad, replace=False)
        x[:, bad] += 40.0 * 16.0
    for _ in range(n_bursts):
        width = int(g.integers(1, 51))
        start = int(g.integers(0, max(nsamps - width, 1)))
        x[start:start + width, :] += 8.0 * 16.0
    np.rint(x, out=x)
    np.clip(x, 0, 255, out=x)
    return Beam(x.astype(np.uint8), list(pulses), nchans, dt, f0, df, seed, beam)


def random_pulses(g: np.random.Generator, n: int, t_lo: float, t_hi: float,
                  dm_lo: float, dm_hi: float, fwhm_lo_s: float, fwhm_hi_s: float,
                  snr_lo: float, snr_hi: float) -> List[Pulse]:
    out = []
    for _ in range(n):
        dm = float(g.uniform(dm_lo, dm_hi))
        fwhm = float(math.exp(g.uniform(math.log(fwhm_lo_s), math.log(fwhm_hi_s))))
        snr = float(g.uniform(snr_lo, snr_hi))
        t0 = float(g.uniform(t_lo, t_hi))
        out.append(Pulse(t0, dm, fwhm, snr))
    return out


def max_delay_samples(dm: float, nchans: int, dt: float, f0: float, df: float) -> float:
    f_low = f0 + df * (nchans - 1)
    return float(dispersion_delay_s(dm, np.array([f_low]), f0)[0] / dt)


# --------------------------------------------------------------------------
# Workloads
# --------------------------------------------------------------------------

@dataclasses.dataclass
class Workload:
    name: str
    nchans: int
    dt: float
    f0: float
    df: float
    nsamps: int          # per beam
    nbeams: int
    dm_min: float
    dm_max: float
    boxcar_max: int
    clean: bool
    description: str


SEARCH_C0 = Workload("plain_c256_n65536", 256, 64e-6, 1500.0, -1.5625, 1 << 16, 1,
                     0.0, 1000.0, 1 << 10, False,
                     "plain single beam: 256 ch uint8, 1500 MHz top, -1.5625 MHz, 64 us, "
                     "2^16 samples, DM 0-1000, boxcars 2^0..2^10")
SEARCH_C1 = Workload("plain_c1024_n262144_rfi", 1024, 64e-6, 1520.0, -0.390625, 1 << 18, 1,
                     0.0, 2000.0, 1 << 12, True,
                     "plain single beam at survey size with RFI: 1024 ch uint8, 1520 MHz top, "
                     "-0.390625 MHz, 64 us, 2^18 samples, DM 0-2000, boxcars 2^0..2^12, "
                     "clean_filterbank_rfi on")
SEARCH_C2 = Workload("multibeam_36x_c320_n32768", 320, 655.36e-6, 851.0, -0.09765625, 1 << 15, 36,
                     0.0, 2000.0, 1 << 9, False,
                     "36 uniform beams x 320 ch uint8, 851 MHz top, -0.09765625 MHz, "
                     "655.36 us, 2^15 samples per beam, DM 0-2000, boxcars 2^0..2^9")


def make_c0(seed: int = 2024) -> Beam:
    w = SEARCH_C0
    md = max_delay_samples(w.dm_max, w.nchans, w.dt, w.f0, w.df)
    span = w.nsamps - md - w.boxcar_max
    pulses = [Pulse(w.boxcar_max + span * (k + 1) / 4.0, dm, fw, 20.0)
              for k, (dm, fw) in enumerate([(100.0, 0.5e-3), (500.0, 2e-3), (900.0, 8e-3)])]
    return make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df, pulses, seed=seed, beam=0)


def make_c1(seed: int = 2025, nsamps: Optional[int] = None, nchans: Optional[int] = None,
            npulses: int = 20, rfi: bool = True) -> Beam:
    w = SEARCH_C1
    ns = nsamps or w.nsamps
    nc = nchans or w.nchans
    df = w.df * (w.nchans / nc)
    g = _rng(seed, 0x5EED)
    md = max_delay_samples(w.dm_max, nc, w.dt, w.f0, df)
    hi = max(ns - md - 2 * w.boxcar_max, w.boxcar_max + 1)
    pulses = random_pulses(g, npulses, w.boxcar_max, hi, 50.0, 2000.0, 0.1e-3, 30e-3, 6.0, 50.0)
    return make_beam(ns, nc, w.dt, w.f0, df, pulses, seed=seed, beam=0,
                     rfi_chan_frac=0.05 if rfi else 0.0, n_bursts=10 if rfi else 0)


def make_multibeam(w: Workload, seed: int = 2026, pulses_per_beam: int = 2,
                   fwhm_lo_s: float = 1e-3, fwhm_hi_s: float = 50e-3,
                   snr_lo: float = 6.0, snr_hi: float = 30.0) -> List[Beam]:
    beams = []
    md = max_delay_samples(w.dm_max, w.nchans, w.dt, w.f0, w.df)
    hi = max(w.nsamps - md - 2 * w.boxcar_max, w.boxcar_max + 1)
    for b in range(w.nbeams):
        g = _rng(seed, b)
        pulses = random_pulses(g, pulses_per_beam, w.boxcar_max, hi, 50.0, w.dm_max,
                               fwhm_lo_s, fwhm_hi_s, snr_lo, snr_hi)
        beams.append(make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df, pulses, seed=seed,
                               beam=b, rng=g))
    return beams


def stf(beams: Sequence[Beam]) -> np.ndarray:
    """Concatenates beams in time (the reference's multibeam "STF" layout,
    Formats/PSRDadaRingBuffer.C:194-198)."""
    return np.ascontiguousarray(np.concatenate([b.data for b in beams], axis=0))


# ---------------------------------------------------------------------------
# Uneven beams: channel count, gulp length, sampling time and DM range differ
# from beam to beam (a 400 MHz band below 1520 MHz split into C channels)
# ---------------------------------------------------------------------------
UNEVEN_NCHANS = (128, 512, 2048, 4096)
UNEVEN_DT = (64e-6, 128e-6)
UNEVEN_DM_MAX = (500.0, 2000.0, 5000.0)
UNEVEN_F_TOP, UNEVEN_BW = 1520.0, 400.0
UNEVEN_BOXCAR_MAX = 1 << 12
UNEVEN_NSAMPS = (1 << 14, 1 << 17)


def uneven_shapes(nbeams: int, seed: int = 2027, nchans: Sequence[int] = UNEVEN_NCHANS,
                  nsamps_range: Tuple[int, int] = UNEVEN_NSAMPS,
                  dm_maxes: Sequence[float] = UNEVEN_DM_MAX,
                  boxcar_max: int = UNEVEN_BOXCAR_MAX) -> List[Workload]:
    """Per-beam shapes: channel counts in turn from `nchans`, sampling time
    alternating 64/128 us every len(nchans) beams, gulp length uniform in
    nsamps_range, and a DM range drawn among those of `dm_maxes` whose
    largest delay plus the widest boxcar (plus 5 % margin) fits the gulp
    (the smallest range otherwise; that beam then reports HD_TOO_FEW_NSAMPS
    or is not searched, as the reference would)."""
    g = _rng(seed, 0x0E7E)
    out = []
    for b in range(nbeams):
        c = int(nchans[b % len(nchans)])
        dt = UNEVEN_DT[(b // len(nchans)) % len(UNEVEN_DT)]
        n = int(g.integers(nsamps_range[0], nsamps_range[1] + 1))
        df = -UNEVEN_BW / c
        fits = [d for d in dm_maxes
                if 1.05 * max_delay_samples(d, c, dt, UNEVEN_F_TOP, df) + boxcar_max < n]
        dm_max = float(fits[int(g.integers(0, len(fits)))]) if fits else float(min(dm_maxes))
        out.append(Workload(f"uneven_b{b}_c{c}_n{n}", c, dt, UNEVEN_F_TOP, df, n, 1, 0.0, dm_max,
                            boxcar_max, True,
                            f"uneven beam {b}: {c} ch, {dt * 1e6:.0f} us, {n} samples, "
                            f"DM 0-{dm_max:.0f}"))
    return out


def make_uneven_beam(w: Workload, seed: int = 2027, beam: int = 0, rfi: bool = True) -> Beam:
    """Noise, injections and RFI as the survey-size beam, scaled to this
    beam's duration: 20 pulses and 10 zero-DM bursts per 2^18 x 64 us
    (at least one each; DM 50..dm_max, FWHM 0.1-30 ms, S/N 6-50) and 5 % of
    the channels persistently at +40 sd."""
    g = _rng(seed, 0x0E7E00 + beam)
    frac = w.nsamps * w.dt / ((1 << 18) * 64e-6)
    md = max_delay_samples(w.dm_max, w.nchans, w.dt, w.f0, w.df)
    hi = max(w.nsamps - md - 2 * w.boxcar_max, w.boxcar_max + 1)
    pulses = random_pulses(g, max(1, int(round(20 * frac))), w.boxcar_max, hi,
                           min(50.0, w.dm_max), w.dm_max, 0.1e-3, 30e-3, 6.0, 50.0)
    return make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df, pulses, seed=seed, beam=beam,
                     rfi_chan_frac=0.05 if rfi else 0.0,
                     n_bursts=max(1, int(round(10 * frac))) if rfi else 0, rng=g)


# ---------------------------------------------------------------------------
# Classifier training data: gulps with injected pulses and labelled RFI
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class RfiEvent:
    kind: str       # "burst" (zero-DM broadband), "narrow" (few channels), "drift"
    t0: float       # first sample
    length: float   # samples


TRAIN = Workload("train_c256_n32768", 256, 128e-6, 1500.0, -1.5625, 1 << 15, 1, 0.0, 500.0,
                 256, False, "classifier training gulps: 256 ch, 128 us, 2^15 samples, DM 0-500")


def make_training_beam(seed: int, w: Workload = TRAIN, n_pulses: int = 4, n_rfi: int = 2
                       ) -> Tuple[Beam, List[RfiEvent]]:
    """Noise + n_pulses dispersed pulses (DM 30..dm_max, FWHM 0.5-20 ms,
    S/N 8-40) + n_rfi RFI events, each event in its own slot of the gulp
    (separated by more than the clustering time window, so that an RFI
    cluster does not absorb a pulse).  RFI kinds: zero-DM broadband bursts
    (1-64 samples, +1..+3 sigma per channel), narrowband bursts (1-8 adjacent
    channels, 16-512 samples, +3..+8 sigma) and sinusoidal baseline drifts
    over all channels (period 5-50 ms, 1-3 periods, 0.3-1 sigma)."""
    g = _rng(seed, 0x7A11)
    md = max_delay_samples(w.dm_max, w.nchans, w.dt, w.f0, w.df)
    lo = 2 * w.boxcar_max
    hi = w.nsamps - md - 2 * w.boxcar_max
    nev = n_pulses + n_rfi
    slot = (hi - lo) / max(nev, 1)
    kinds = ["pulse"] * n_pulses + ["rfi"] * n_rfi
    g.shuffle(kinds)
    pulses: List[Pulse] = []
    events: List[RfiEvent] = []
    plan = []
    for k, kind in enumerate(kinds):
        t = lo + slot * (k + float(g.uniform(0.3, 0.7)))
        if kind == "pulse":
            dm = float(g.uniform(30.0, w.dm_max))
            fw = float(math.exp(g.uniform(math.log(0.5e-3), math.log(20e-3))))
            pulses.append(Pulse(t, dm, fw, float(g.uniform(8.0, 40.0))))
        else:
            plan.append((t, ("burst", "narrow", "drift")[int(g.integers(0, 3))]))
    b = make_beam(w.nsamps, w.nchans, w.dt, w.f0, w.df, pulses, seed=seed, beam=1, rng=g)
    x = b.data.astype(np.float32)
    for t, kind in plan:
        if kind == "burst":
            ln = int(g.integers(1, 65))
            t0 = int(t)
            x[t0:t0 + ln, :] += float(g.uniform(1.0, 3.0)) * 16.0
        elif kind == "narrow":
            ln = int(2 ** g.uniform(4, 9))
            t0 = int(t)
            nc = int(g.integers(1, 9))
            c0 = int(g.integers(0, w.nchans - nc))
            x[t0:t0 + ln, c0:c0 + nc] += float(g.uniform(3.0, 8.0)) * 16.0
        else:
            period = float(g.uniform(0.005, 0.05)) / w.dt
            ln = int(min(slot * 0.5, period * float(g.uniform(1.0, 3.0))))
            t0 = int(t)
            amp = float(g.uniform(0.3, 1.0)) * 16.0
            tt = np.arange(ln, dtype=np.float32)
            x[t0:t0 + ln, :] += (amp * np.sin(2.0 * np.pi * tt / period))[:, None]
        events.append(RfiEvent(kind, float(t0), float(ln)))
    np.rint(x, out=x)
    np.clip(x, 0, 255, out=x)
    b.data = x.astype(np.uint8)
    return b, events


def match_pulse(cand, pulses: Sequence[Pulse], dt: float) -> int:
    """Index of the injected pulse a candidate row recovers, or -1: |samp -
    t0| <= max(2^filter, FWHM/dt) + 2 and DM within max(5 %, 2 trial steps)
    (the recall rule of the benchmark)."""
    for k, p in enumerate(pulses):
        tol_t = max(2 ** int(cand["filter"]), p.fwhm_s / dt) + 2
        tol_dm = max(0.05 * p.dm, 2 * 1.25 * max(p.dm, 1.0) * 0.01)
        if abs(int(cand["samp_idx"]) - p.t0) <= tol_t and abs(float(cand["dm"]) - p.dm) <= tol_dm:
            return k
    return -1


# ---------------------------------------------------------------------------
# Classifier training gulps at survey size, generated on the GPU
# ---------------------------------------------------------------------------
def inject_pulse_device(torch, x, p: Pulse, dt: float, f0: float, df: float,
                        sigma: float = 16.0) -> None:
    """inject_pulse on a device tensor x (nsamps, nchans) float32: the same
    dispersed Gaussian (channel centre times, width, +-6 sigma window,
    amplitude for the integrated S/N over the whole window)."""
    nsamps, nchans = x.shape
    dev = x.device
    f = f0 + df * torch.arange(nchans, dtype=torch.float64, device=dev)
    centres = p.t0 + DISPERSION_K * p.dm * (f ** -2.0 - f0 ** -2.0) / dt
    s = max(p.fwhm_s / dt / (2.0 * math.sqrt(2.0 * math.log(2.0))), 0.3)
    half = int(math.ceil(6.0 * s)) + 1
    t = torch.floor(centres).long()[:, None] - half + torch.arange(2 * half + 1, device=dev)[None, :]
    g = torch.exp(-0.5 * ((t.double() - centres[:, None]) / s) ** 2)
    energy = float((g * g).sum())
    if energy <= 0.0:
        return
    amp = p.snr * sigma / math.sqrt(energy)
    keep = (t >= 0) & (t < nsamps)
    c = torch.arange(nchans, device=dev)[:, None].expand_as(t)
    x.index_put_((t[keep], c[keep]), (amp * g[keep]).float(), accumulate=True)


def make_training_gulps_device(torch, seeds: Sequence[int], w: Workload = None,
                               n_pulses: int = 40, n_rfi: int = 20, device: str = "cuda"):
    """Survey-shaped classifier training gulps (default: 1024 channels, 64 us,
    2^18 samples) generated on the GPU.  Each gulp: Gaussian noise (128, 16),
    n_pulses dispersed pulses (DM 50-dm_max, FWHM log-uniform 0.1-30 ms, S/N
    6-50) and n_rfi RFI events, each event in its own time slot: zero-DM
    broadband bursts (1-64 samples, +0.1..+0.5 sd per channel), narrowband
    bursts (1-32 adjacent channels, 16-512 samples, +1..+4 sd) and sinusoidal
    baseline drifts over all channels (period 5-50 ms, 1-3 periods,
    0.05-0.2 sd).  Over 1024 channels these integrate at DM 0 to S/N of a few
    to about a hundred (stronger events flood the list with candidates along
    the whole DM range and swallow neighbouring pulses).  Returns (uint8
    tensor [U, nsamps, nchans] on the device, pulses per gulp, RFI events per
    gulp)."""
    w = w or SEARCH_C1
    dev = torch.device(device)
    seeds = list(seeds)
    out = torch.empty((len(seeds), w.nsamps, w.nchans), dtype=torch.uint8, device=dev)
    md = max_delay_samples(w.dm_max, w.nchans, w.dt, w.f0, w.df)
    lo = 2 * w.boxcar_max
    hi = w.nsamps - md - 2 * w.boxcar_max
    nev = n_pulses + n_rfi
    slot = (hi - lo) / max(nev, 1)
    all_pulses, all_events = [], []
    for u, seed in enumerate(seeds):
        g = _rng(seed, 0xC1C1)
        tg = torch.Generator(device=dev).manual_seed(int(seed) * 7919 + 17)
        x = torch.randn((w.nsamps, w.nchans), generator=tg, device=dev)
        x.mul_(16.0).add_(128.0)
        kinds = ["pulse"] * n_pulses + ["rfi"] * n_rfi
        g.shuffle(kinds)
        pulses: List[Pulse] = []
        events: List[RfiEvent] = []
        for k, kind in enumerate(kinds):
            t = lo + slot * (k + float(g.uniform(0.3, 0.7)))
            if kind == "pulse":
                dm = float(g.uniform(50.0, w.dm_max))
                fw = float(math.exp(g.uniform(math.log(0.1e-3), math.log(30e-3))))
                pu = Pulse(t, dm, fw, float(g.uniform(6.0, 50.0)))
                inject_pulse_device(torch, x, pu, w.dt, w.f0, w.df)
                pulses.append(pu)
                continue
            kind = ("burst", "narrow", "drift")[int(g.integers(0, 3))]
            t0 = int(t)
            if kind == "burst":
                ln = int(g.integers(1, 65))
                x[t0:t0 + ln, :] += float(g.uniform(0.1, 0.5)) * 16.0
            elif kind == "narrow":
                ln = int(2 ** g.uniform(4, 9))
                nc = int(g.integers(1, 33))
                c0 = int(g.integers(0, w.nchans - nc))
                x[t0:t0 + ln, c0:c0 + nc] += float(g.uniform(1.0, 4.0)) * 16.0
            else:
                period = float(g.uniform(0.005, 0.05)) / w.dt
                ln = int(min(slot * 0.5, period * float(g.uniform(1.0, 3.0))))
                amp = float(g.uniform(0.05, 0.2)) * 16.0
                tt = torch.arange(ln, dtype=torch.float32, device=dev)
                x[t0:t0 + ln, :] += (amp * torch.sin(2.0 * math.pi * tt / period))[:, None]
            events.append(RfiEvent(kind, float(t0), float(ln)))
        out[u] = x.round_().clamp_(0, 255).to(torch.uint8)
        del x
        all_pulses.append(pulses)
        all_events.append(events)
    return out, all_pulses, all_events


# ---------------------------------------------------------------------------
# Sigproc filterbank files
# ---------------------------------------------------------------------------
SIGPROC_INT = ("nchans", "telescope_id", "machine_id", "data_type", "ibeam", "nbeams", "nbits",
               "barycentric", "pulsarcentric", "nbins", "nsamples", "nifs", "npuls")
SIGPROC_DOUBLE = ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "period",
                  "fch1", "foff", "refdm")
SIGPROC_STR = ("source_name", "rawdatafile")


def write_sigproc(path: str, data: Optional[np.ndarray] = None, order: Sequence[str] = (),
                  **fields) -> int:
    """Writes a sigproc file: HEADER_START, each field as its keyword string
    (4-byte length + characters) followed by its value (int32, float64, a
    string, or one byte for `signed`; an unknown keyword is written alone),
    HEADER_END, then data (time-major uint8 spectra).  `order` fixes the
    keyword order (the remaining fields follow).  Returns the header size."""
    import struct

    def w_str(f, t: str):
        b = t.encode()
        f.write(struct.pack("<i", len(b)))
        f.write(b)

    keys = list(order) + [k for k in fields if k not in order]
    with open(path, "wb") as f:
        w_str(f, "HEADER_START")
        for k in keys:
            v = fields[k]
            w_str(f, k)
            if k in SIGPROC_INT:
                f.write(struct.pack("<i", int(v)))
            elif k in SIGPROC_DOUBLE:
                f.write(struct.pack("<d", float(v)))
            elif k in SIGPROC_STR:
                w_str(f, str(v))
            elif k == "signed":
                f.write(struct.pack("<B", int(v)))
        w_str(f, "HEADER_END")
        size = f.tell()
        if data is not None:
            f.write(np.ascontiguousarray(data, dtype=np.uint8).tobytes())
    return size



def pack_filterbank(values: np.ndarray, nbits: int) -> np.ndarray:
    """Packs an (nsamps, nchans) array of sample values (each < 2^nbits) into
    one row of nbits-bit samples per spectrum, the layout hd_execute and
    dedisp_execute take for nbits = 1, 2, 4 and 16: channel c is the
    nbits-bit field at bit (c mod (32 / nbits)) * nbits of the little-endian
    32-bit word c / (32 / nbits) (the order of the reference's writer,
    Formats/giant_maker.C:385-392).  Returns uint8 rows of nchans * nbits / 8
    bytes (nchans * nbits a multiple of 32)."""
    v = np.asarray(values)
    nsamps, nchans = v.shape
    if nbits not in (1, 2, 4, 8, 16) or (nchans * nbits) % 32:
        raise ValueError("nbits in {1, 2, 4, 8, 16} and nchans * nbits a multiple of 32")
    if v.size and int(v.max()) >= (1 << nbits):
        raise ValueError("sample values must be below 2^nbits")
    cpw = 32 // nbits
    fields = v.astype(np.uint64).reshape(nsamps, nchans // cpw, cpw)
    shifts = (np.arange(cpw, dtype=np.uint64) * np.uint64(nbits))[None, None, :]
    words = (fields << shifts).sum(axis=2).astype(np.uint32)
    return np.ascontiguousarray(words.astype("<u4")).view(np.uint8).reshape(nsamps, -1)
