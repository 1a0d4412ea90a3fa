"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset ships with the reference; every model here is generated from a fixed numpy seed.
Arrays follow the reference's in-memory layout: x-major, z fastest, float32
(forward/Acoustic_FD_by_ss/src/Acoustic_1order_FD.cpp:51-100, tools/get_vel_model.cpp:26-45).
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


def pad_edges(a: np.ndarray, pml_x: int, pml_z: int) -> np.ndarray:
    """Edge-replicated padding of an interior (nx, nz) model, the padding rule of
    forward/Q_forward/Q_multishot_fd_subroutine_fsbc_zy_rotated.f90:340-372."""
    return np.pad(a, ((pml_x, pml_x), (pml_z, pml_z)), mode="edge").astype(np.float32)


@dataclass
class AcousticCase:
    name: str
    NX: int            # interior cells along x
    NZ: int            # interior cells along z
    PML: int           # sponge width (cells)
    nt: int
    dx: float
    dz: float
    dt: float
    vp: np.ndarray     # padded (Nx, Nz) float32
    den: np.ndarray    # padded (Nx, Nz) float32
    src_x: List[int]   # padded source cells, one per shot
    src_z: List[int]
    rec_z: int         # padded depth of the horizontal receiver line (every interior x)
    f0: float
    radius: int = 8
    nt_per_shot: Optional[List[int]] = None
    extra: dict = field(default_factory=dict)

    @property
    def Nx(self) -> int:
        return self.NX + 2 * self.PML

    @property
    def Nz(self) -> int:
        return self.NZ + 2 * self.PML

    @property
    def nshot(self) -> int:
        return len(self.src_x)

    def receivers(self):
        rx = np.arange(self.PML, self.Nx - self.PML, dtype=np.int32)
        return rx, np.full_like(rx, self.rec_z)


def config1() -> AcousticCase:
    """Plain 2-D constant-density acoustic, single shot: 251 x 251, dx = dz = 10 m,
    dt = 1 ms, nt = 1000, two-layer vp (2000 m/s above interior z = 125, 3000 below),
    50-cell sponge, 25 Hz Ricker (tools/ricker.cpp:44 formula) at interior (z=2, x=125),
    receivers at every interior x on z = 2. 16th order (the reference's)."""
    NX = NZ = 251
    PML = 50
    z = np.arange(NZ)
    col = np.where(z < 125, 2000.0, 3000.0).astype(np.float32)
    vp = pad_edges(np.tile(col, (NX, 1)), PML, PML)
    den = np.full_like(vp, 2400.0)
    return AcousticCase("config1_plain_251x251", NX, NZ, PML, 1000, 10.0, 10.0, 1e-3, vp, den,
                        [PML + 125], [PML + 2], PML + 2, 25.0)


def layered_model(NX, NZ, nlayer, vmin, vmax, seed, lateral=0.05, anomalies=4, radius=40.0,
                  amp=400.0, dx=5.0):
    """Layered vp increasing with depth, a smooth +-`lateral` relative lateral field and
    Gaussian anomalies of +-`amp` m/s. Interior (NX, NZ) float32."""
    rng = np.random.default_rng(seed)
    bounds = np.sort(rng.uniform(0.05, 0.95, nlayer - 1)) * NZ
    vel = np.linspace(vmin, vmax, nlayer)
    z = np.arange(NZ)
    col = vel[np.searchsorted(bounds, z, side="right")]
    v = np.tile(col, (NX, 1)).astype(np.float64)
    x = np.arange(NX)
    # smooth lateral perturbation: a few low-wavenumber cosines in x and z
    lat = np.zeros((NX, NZ))
    for _ in range(4):
        kx, kz = rng.uniform(0.5, 3.0, 2) * 2 * np.pi
        px, pz = rng.uniform(0, 2 * np.pi, 2)
        lat += np.cos(kx * x[:, None] / NX + px) * np.cos(kz * z[None, :] / NZ + pz)
    lat /= np.abs(lat).max() + 1e-12
    v *= 1.0 + lateral * lat
    for _ in range(anomalies):
        cx, cz = rng.uniform(0.15, 0.85) * NX, rng.uniform(0.2, 0.85) * NZ
        sgn = rng.choice([-1.0, 1.0])
        v += sgn * amp * np.exp(-((x[:, None] - cx) ** 2 + (z[None, :] - cz) ** 2) / (2 * radius ** 2))
    return v.astype(np.float32)


def config2(nshot: int = 64, nt: int = 4000) -> AcousticCase:
    """Batched 2-D acoustic forward: 512 (z) x 2048 (x), dx = dz = 5 m, dt = 0.5 ms, nt = 4000,
    12 layers 1500-4500 m/s with +-5% lateral variation and 4 Gaussian anomalies (radius 40
    cells, +-400 m/s), 64 shots evenly spaced on interior z = 2, 30 Hz Ricker, 2048 receivers
    per shot (every interior x on z = 2), 50-cell sponge. Velocities are clipped at 4700 m/s
    so the 16th-order CFL number stays below 0.5 (limit 0.516)."""
    NX, NZ, PML = 2048, 512, 50
    v = np.clip(layered_model(NX, NZ, 12, 1500.0, 4500.0, seed=20261203), 1400.0, 4700.0)
    vp = pad_edges(v, PML, PML)
    den = np.full_like(vp, 2400.0)
    sx = [PML + int(round((i + 0.5) * NX / nshot)) for i in range(nshot)]
    return AcousticCase("config2_batched_512x2048", NX, NZ, PML, nt, 5.0, 5.0, 5e-4, vp, den,
                        sx, [PML + 2] * nshot, PML + 2, 30.0)


def config4(nshot: int = 32, nt: int = 3000):
    """2-D acoustic adjoint gradient: 384 (z) x 1536 (x), dx = dz = 10 m, dt = 1 ms, nt = 3000,
    32 shots on interior z = 2, receivers every x on z = 2, 25 Hz Ricker.  Returns
    (start case, true vp): the true model is layered plus 3 Gaussian anomalies, the starting
    model its Gaussian smoothing with sigma = 15 cells.  The checkpoint interval of the
    gradient is 55 steps."""
    from scipy.ndimage import gaussian_filter
    NX, NZ, PML = 1536, 384, 50
    true = np.clip(layered_model(NX, NZ, 10, 1500.0, 4000.0, seed=20261204, anomalies=3, radius=30.0, amp=350.0,
                                 dx=10.0), 1400.0, 4300.0)
    start = gaussian_filter(true.astype(np.float64), sigma=15.0, mode="nearest").astype(np.float32)
    vp_true = pad_edges(true, PML, PML)
    vp0 = pad_edges(start, PML, PML)
    den = np.full_like(vp0, 2200.0)
    sx = [PML + int(round((i + 0.5) * NX / nshot)) for i in range(nshot)]
    case = AcousticCase("config4_gradient_384x1536", NX, NZ, PML, nt, 10.0, 10.0, 1e-3, vp0, den, sx,
                        [PML + 2] * nshot, PML + 2, 25.0, extra={"checkpoint_interval": 55})
    return case, vp_true


def config3(nshot: int = 16):
    """2-D viscoacoustic (one SLS memory variable): 1024 x 1024 interior, dx = dz = 5 m,
    dt = 0.5 ms, the two-layer vp of config 1 rescaled to the grid (2000 m/s above interior
    z = 512, 3000 below), density 2000 kg/m^3, Q 20-200 as a seeded smooth random field with a
    low-Q lens (radius 60 cells, Q = 20), 20 Hz Ricker in the Q_forward convention, 16 shots on
    interior z = 2 with record lengths drawn uniformly from 2000-3000 steps, receivers at every
    interior x on z = 2, 50 pad cells (sponge) per side.  Returns a dict of padded arrays."""
    from scipy.ndimage import gaussian_filter
    NX = NZ = 1024
    PML = 50
    rng = np.random.default_rng(20261205)
    z = np.arange(NZ)
    x = np.arange(NX)
    vp = np.tile(np.where(z < NZ // 2, 2000.0, 3000.0), (NX, 1)).astype(np.float32)
    rho = np.full((NX, NZ), 2000.0, np.float32)
    f = gaussian_filter(rng.standard_normal((NX, NZ)), sigma=40.0, mode="wrap")
    f = (f - f.min()) / (f.max() - f.min())
    q = 20.0 + 180.0 * f
    lens = (x[:, None] - 0.6 * NX) ** 2 + (z[None, :] - 0.45 * NZ) ** 2 < 60.0 ** 2
    q = np.where(lens, 20.0, q).astype(np.float32)
    nts = [int(v) for v in rng.integers(2000, 3001, nshot)]
    sx = [PML + int(round((i + 0.5) * NX / nshot)) for i in range(nshot)]
    return {"name": "config3_viscoacoustic_1024x1024", "NX": NX, "NZ": NZ, "PML": PML, "dx": 5.0, "dz": 5.0,
            "dt": 5e-4, "f0": 20.0, "vp": pad_edges(vp, PML, PML), "rho": pad_edges(rho, PML, PML),
            "q": pad_edges(q, PML, PML), "src_x": sx, "src_z": [PML + 2] * nshot, "rec_z": PML + 2, "nt": nts,
            "interior": (vp, rho, q)}


def config5(nshot: int = 16, nt_scale: float = 1.0):
    """3-D acoustic, 8th order: 512^3 interior, dx = dy = dz = 10 m, dt = 1 ms, 50-cell sponge
    (612^3 padded), smooth layered vp 1500-4000 m/s (6 layers, Gaussian-smoothed with sigma = 6
    cells, +-3% smooth lateral variation), 16 shots on a 4 x 4 grid at interior depth 2, record
    lengths drawn uniformly from 1500-2500 steps (times nt_scale), a 256 x 256 receiver patch per
    shot at interior depth 2 with seeded offsets, 15 Hz Ricker (RIC formula).  Returns a dict; the
    velocity is built per x-slab (the grid holds 229M cells)."""
    from scipy.ndimage import gaussian_filter1d
    N, PML = 512, 50
    n = N + 2 * PML
    rng = np.random.default_rng(20261207)
    bounds = np.sort(rng.uniform(0.1, 0.9, 5)) * N
    z = np.arange(N)
    col = np.linspace(1500.0, 4000.0, 6)[np.searchsorted(bounds, z, side="right")]
    col = gaussian_filter1d(col, 6.0, mode="nearest")
    col = np.pad(col, (PML, PML), mode="edge").astype(np.float32)
    kx, ky = rng.uniform(1.0, 3.0, 2) * 2 * np.pi / n
    px, py = rng.uniform(0, 2 * np.pi, 2)
    yy = np.arange(n)

    def vp_slab(x0: int, x1: int) -> np.ndarray:
        xs = np.arange(x0, x1)
        lat = 1.0 + 0.03 * np.cos(kx * xs[:, None] + px) * np.cos(ky * yy[None, :] + py)
        return (lat[:, :, None] * col[None, None, :]).astype(np.float32)

    nts = [max(1, int(round(v * nt_scale))) for v in rng.integers(1500, 2501, nshot)]
    g = [PML + int(round((i + 0.5) * N / 4)) for i in range(4)]
    src = [(g[i % 4], g[i // 4], PML + 2) for i in range(nshot)]
    rec = []
    for s in src:
        ox, oy = rng.integers(-64, 65, 2)
        x0 = int(np.clip(s[0] - 128 + ox, PML, PML + N - 256))
        y0 = int(np.clip(s[1] - 128 + oy, PML, PML + N - 256))
        ry, rx = np.meshgrid(np.arange(y0, y0 + 256), np.arange(x0, x0 + 256), indexing="ij")
        rec.append((rx.ravel().astype(np.int32), ry.ravel().astype(np.int32),
                    np.full(256 * 256, PML + 2, np.int32)))
    return {"name": "config5_3d_512cube", "N": N, "PML": PML, "n": n, "d": 10.0, "dt": 1e-3, "f0": 15.0,
            "vp_slab": vp_slab, "src": src, "rec": rec, "nt": nts}


def vti_card(nshot: int = 64, nt: int = 2000, seed: int = 20261205):
    """The VTI modeller's shipped .par geometry (de-multiple/convolution_srm/vti_qa_2d_c3_demo1/
    vti_qa_2d_modelling_new.par): a 300 x 300 model at dx = dz = 5 m, dt = 0.5 ms, 30 Hz, PML 250 m
    on the left, right and bottom and none on top, offsets -1500 .. 1495 m (600 traces per shot),
    order 10 / 9 / 10; the card's shots step one cell from sx0 = 0.  The card's model files are
    not shipped: a seeded synthetic model stands in (8 layers, vz 1500-3500 m/s with a +-3% lateral
    field, epsilon 0.05-0.25 and delta 0.02-0.12 increasing with depth).  nshot shots spread over
    the 300 source positions; the card's nt is 10000."""
    rng = np.random.default_rng(seed)
    nxv = nzv = 300
    z = np.arange(nzv)
    layer = np.minimum((z * 8) // nzv, 7)
    vz1 = 1500.0 + 2000.0 * layer / 7.0
    lat = 1.0 + 0.03 * np.sin(2 * np.pi * np.arange(nxv) / nxv * rng.uniform(1.0, 3.0) + rng.uniform(0, 6.28))
    vz = (vz1[None, :] * lat[:, None]).astype(np.float32)
    eps = np.tile(0.05 + 0.20 * layer / 7.0, (nxv, 1)).astype(np.float32)
    de = np.tile(0.02 + 0.10 * layer / 7.0, (nxv, 1)).astype(np.float32)
    nsx = [1 + int(i * nxv / nshot) for i in range(nshot)]
    shots = [(s, 1, 1, s - 300, s + 299) for s in nsx]  # nint(offset / dx): -300 .. 299
    return {"name": "vti_card_300x300", "vz": vz, "eps": eps, "delta": de, "dx": 5.0, "dz": 5.0, "dt": 5e-4,
            "f0": 30.0, "nt": nt, "bounds": (50, 50, 0, 50), "shots": shots}


def small_varden(seed: int = 7) -> AcousticCase:
    """Non-square, variable-density case used to pin the restatement against the reference
    build: 80 (x) x 60 (z) interior, 15-cell sponge, 300 steps, off-centre source."""
    NX, NZ, PML = 80, 60, 15
    rng = np.random.default_rng(seed)
    v = layered_model(NX, NZ, 4, 1800.0, 3200.0, seed=seed, anomalies=2, radius=8.0, amp=200.0)
    d = (2000.0 + 400.0 * rng.random((NX, NZ))).astype(np.float32)
    return AcousticCase("small_varden_80x60", NX, NZ, PML, 300, 10.0, 10.0, 1e-3,
                        pad_edges(v, PML, PML), pad_edges(d, PML, PML), [PML + 30], [PML + 20],
                        PML + 3, 20.0)
