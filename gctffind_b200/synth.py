"""Seeded synthetic micrographs and tilt series with a known CTF.

The generator follows the image model used to benchmark the CTF path:

1. a white Gaussian object ``o ~ N(0, 1)`` drawn from the seed;
2. in Fourier space, multiplication by ``h = CTF * E`` with
   ``CTF = -sin(chi + phi_amp + phi_ext)``,
   ``chi = pi * lambda * s^2 * (df(theta) - 0.5 * lambda^2 * s^2 * Cs)``,
   ``df(theta) = mean + sigma * cos(2 * (theta - azimuth))`` and the
   B-factor envelope ``E = exp(-B * s^2 / 4)`` (s in 1/Angstrom), i.e. the
   same model and angle convention as GCalcCTF2D (FindCTF/GCalcCTF2D.cu:15-38):
   ``theta`` is measured from the +x frequency axis towards +y, where y is the
   row index of the image;
3. a smooth background field whose amplitude falls as ``1 / (f^2 + f0^2)``;
4. expected counts ``D * px^2 * (1 + c * (h * o) + b)`` clamped at zero,
   then a Poisson draw stored as float32.

A tilt series adds a defocus gradient along x: the defocus at column x is
``df0 + (x - W/2) * px * sin(tilt)``, realised by blending a small stack of
uniformly-filtered images column by column.

torch is used only as an array library here (CPU for the tests, CUDA for
large benchmark inputs); nothing in this module is on the estimation path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch


def wavelength_angstrom(kv: float) -> float:
    """Relativistic electron wavelength, CCTFTheory::mCalcWavelength
    (FindCTF/CCTFTheory.cpp:283-287)."""
    return 12.26 / math.sqrt(kv * 1000.0 + 0.9784 * kv * kv)


@dataclass
class MicrographSpec:
    width: int = 4096
    height: int = 4096
    pixel_size: float = 1.0          # Angstrom
    kv: float = 300.0
    cs_mm: float = 2.7
    amp_contrast: float = 0.07
    ext_phase_deg: float = 0.0
    df_min: float = 14850.0          # Angstrom
    df_max: float = 15150.0          # Angstrom
    azimuth_deg: float = 20.0
    bfactor: float = 100.0           # Angstrom^2, E = exp(-B s^2 / 4)
    dose: float = 1.0                # e / Angstrom^2
    contrast: float = 0.5            # c
    background: float = 0.3          # amplitude of b relative to 1
    bg_f0: float = 1.0 / 200.0       # 1/Angstrom
    tilt_deg: float = 0.0            # defocus gradient along x
    gradient_levels: int = 9
    seed: int = 0
    extra: dict = field(default_factory=dict)


def _freq_grid(h: int, w: int, px: float, device, dtype):
    ky = torch.fft.fftfreq(h, d=px, device=device, dtype=dtype)
    kx = torch.fft.rfftfreq(w, d=px, device=device, dtype=dtype)
    KY, KX = torch.meshgrid(ky, kx, indexing="ij")
    return KX, KY


def ctf_filter(spec: MicrographSpec, df_mean: float, h: int, w: int, device, dtype=torch.float64):
    """Half-plane transfer function CTF * E for a uniform defocus."""
    KX, KY = _freq_grid(h, w, spec.pixel_size, device, dtype)
    s2 = KX * KX + KY * KY
    theta = torch.atan2(KY, KX)
    sigma = 0.5 * (spec.df_max - spec.df_min)
    az = math.radians(spec.azimuth_deg)
    df = df_mean + sigma * torch.cos(2.0 * (theta - az))
    lam = wavelength_angstrom(spec.kv)
    cs = spec.cs_mm * 1e7
    ac = spec.amp_contrast
    phi = math.atan(ac / math.sqrt(1.0 - ac * ac)) + math.radians(spec.ext_phase_deg)
    chi = math.pi * lam * s2 * (df - 0.5 * lam * lam * s2 * cs) + phi
    env = torch.exp(-spec.bfactor * s2 / 4.0)
    return -torch.sin(chi) * env


def make_micrograph(spec: MicrographSpec, device="cpu") -> torch.Tensor:
    """Return one float32 micrograph (height x width) on `device`."""
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(spec.seed))
    h, w, px = spec.height, spec.width, spec.pixel_size
    dt = torch.float64 if dev.type == "cpu" else torch.float32
    obj = torch.randn((h, w), generator=gen, device=dev, dtype=dt)
    O = torch.fft.rfft2(obj)
    del obj
    df0 = 0.5 * (spec.df_min + spec.df_max)
    if abs(spec.tilt_deg) < 1e-6:
        img = torch.fft.irfft2(O * ctf_filter(spec, df0, h, w, dev, dt), s=(h, w))
    else:
        # defocus varies linearly with x; blend uniformly-filtered images
        span = 0.5 * w * px * math.sin(math.radians(spec.tilt_deg))
        nlev = max(2, int(spec.gradient_levels))
        levels = [df0 - span + 2.0 * span * i / (nlev - 1) for i in range(nlev)]
        xs = torch.arange(w, device=dev, dtype=dt)
        dfx = df0 + (xs - 0.5 * w) * px * math.sin(math.radians(spec.tilt_deg))
        pos = (dfx - levels[0]) / (levels[-1] - levels[0]) * (nlev - 1)
        pos = pos.clamp(0, nlev - 1)
        img = torch.zeros((h, w), device=dev, dtype=dt)
        for i, lv in enumerate(levels):
            wgt = (1.0 - (pos - i).abs()).clamp(min=0.0)
            if float(wgt.max()) <= 0:
                continue
            filt = torch.fft.irfft2(O * ctf_filter(spec, lv, h, w, dev, dt), s=(h, w))
            img += filt * wgt[None, :]
            del filt
    del O
    img = img / img.std().clamp(min=1e-12)
    # smooth background with amplitude ~ 1/(f^2 + f0^2)
    KX, KY = _freq_grid(h, w, px, dev, dt)
    f2 = KX * KX + KY * KY
    amp = 1.0 / (f2 + spec.bg_f0 ** 2)
    noise = torch.randn((h, w), generator=gen, device=dev, dtype=dt)
    bg = torch.fft.irfft2(torch.fft.rfft2(noise) * amp, s=(h, w))
    del noise, KX, KY, f2, amp
    bg = bg / bg.std().clamp(min=1e-12) * spec.background
    lam_e = spec.dose * px * px * (1.0 + spec.contrast * img + bg)
    lam_e = lam_e.clamp(min=0.0)
    del img, bg
    counts = torch.poisson(lam_e.to(torch.float32), generator=gen)
    return counts.to(torch.float32)


def tilt_series_specs(n_tilts: int = 41, step_deg: float = 3.0, size: int = 4096,
                      pixel_size: float = 1.35, dose: float = 3.0, df0: float = 30000.0,
                      seed: int = 1) -> list[MicrographSpec]:
    """Specs of a tilt series: tilts centred on 0 in `step_deg` steps, one
    astigmatism draw (uniform 0-800 Angstrom, random angle) for the series."""
    g = torch.Generator().manual_seed(seed)
    ast = float(torch.rand((), generator=g)) * 800.0
    ang = float(torch.rand((), generator=g)) * 180.0 - 90.0
    half = (n_tilts - 1) / 2.0
    specs = []
    for i in range(n_tilts):
        tilt = (i - half) * step_deg
        specs.append(MicrographSpec(width=size, height=size, pixel_size=pixel_size,
                                    df_min=df0 - 0.5 * ast, df_max=df0 + 0.5 * ast,
                                    azimuth_deg=ang, dose=dose, tilt_deg=tilt,
                                    seed=seed * 1000 + i))
    return specs


def tilt_angles(n_tilts: int = 41, step_deg: float = 3.0) -> list[float]:
    half = (n_tilts - 1) / 2.0
    return [(i - half) * step_deg for i in range(n_tilts)]


UNEVEN_SIZES = ((4096, 4096), (5760, 4092), (3838, 3710))


def uneven_batch_specs(n: int = 256, seed: int = 2, sizes=UNEVEN_SIZES) -> list[MicrographSpec]:
    """A seeded batch of independent micrographs of uneven size: each a
    uniform pick of `sizes`, pixel size U(0.8, 1.5) A, mean defocus
    U(5000, 40000) A, astigmatism (df_max - df_min) U(0, 1000) A at an angle
    U(0, 180) degrees (reported in (-90, 90]), dose U(0.5, 2) e/A^2."""
    g = torch.Generator().manual_seed(int(seed))

    def u(lo, hi):
        return lo + (hi - lo) * float(torch.rand((), generator=g, dtype=torch.float64))

    specs = []
    for k in range(n):
        w, h = sizes[int(torch.randint(0, len(sizes), (), generator=g))]
        px = u(0.8, 1.5)
        df = u(5000.0, 40000.0)
        ast = u(0.0, 1000.0)
        ang = u(0.0, 180.0)
        specs.append(MicrographSpec(width=w, height=h, pixel_size=px, df_min=df - 0.5 * ast,
                                    df_max=df + 0.5 * ast, azimuth_deg=ang if ang <= 90.0 else ang - 180.0,
                                    dose=u(0.5, 2.0), seed=int(seed) * 100003 + k))
    return specs


def inside_reference_envelope(spec: MicrographSpec) -> bool:
    """Whether the reference's full search can reach this micrograph's
    parameters: mean defocus inside CFindCtf1D's range [3000, 30000] px^2 A
    (FindCTF/CFindCtf1D.cpp:78-79; px after rescaling to >= 1.2 A) with 10 %
    to spare, and astigmatism ratio (df_max - df_min) / (df_max + df_min) at
    most the full search's 0.06 (FindCTF/CFindDefocus2D.cpp:117-118)."""
    px_n = max(spec.pixel_size, 1.2)
    mean = 0.5 * (spec.df_min + spec.df_max)
    ratio = (spec.df_max - spec.df_min) / (spec.df_max + spec.df_min)
    return 3300.0 * px_n * px_n <= mean <= 27000.0 * px_n * px_n and ratio <= 0.06
