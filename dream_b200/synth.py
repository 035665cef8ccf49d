"""Seeded synthetic ultrasound scenes for the DAS beamformer.

No public dataset is involved: A-scans are synthesised from point scatterers
with a Gaussian-windowed sine pulse, plus Gaussian noise, all drawn from
``numpy.random.default_rng(seed)``. Geometry and units follow DREAM:
positions in mm, ``dt`` and delays in us, ``cp`` in m/s (so a path of
``r`` mm takes ``r / (cp / 1000)`` us). Arrays are Fortran ordered like the
reference bindings expect (``Ro`` is ``No x 3``, ``G`` is ``N x 3``,
``Y`` is ``K x (Nt*Nr)`` with A-scan column ``t*Nr + r``).

Full-size scenes (the sizes the benchmark and the large tests use):

* SAFT: 64 elements, pitch 0.5 mm, K=2048, dt=0.04, cp=1500, 256x256 grid.
* TFM: 64x64 full matrix capture, K=3000, dt=0.04, cp=1500, 512x512 grid.
* RCA: 128 columns x 128 rows, pitch 0.3 mm, row transmit, K=4096,
  dt=0.025, cp=1480, 128x128x256 grid (z in [5, 35] mm).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Scene",
    "linear_array",
    "rca_arrays",
    "grid_xz",
    "grid_xyz",
    "saft_scene",
    "tfm_scene",
    "rca_scene",
    "pulse",
]


@dataclass
class Scene:
    """Inputs of one ``das`` call, in the reference's argument order."""

    Y: np.ndarray
    Gt: np.ndarray
    Gr: np.ndarray
    Ro: np.ndarray
    dt: float
    delay: np.ndarray
    cp: float
    method: str
    grid_shape: tuple = ()
    extra: dict = field(default_factory=dict)

    @property
    def sums(self) -> int:
        """Number of (pixel, tx, rx) terms (SAFT: pixel, element)."""
        No = self.Ro.shape[0]
        if self.method == "saft":
            return No * self.Gt.shape[0]
        return No * self.Gt.shape[0] * self.Gr.shape[0]

    def astype(self, dtype) -> "Scene":
        f = lambda a: np.asfortranarray(np.asarray(a, dtype=dtype))
        return Scene(f(self.Y), f(self.Gt), f(self.Gr), f(self.Ro),
                     float(np.asarray(self.dt, dtype=dtype)), f(self.delay),
                     float(np.asarray(self.cp, dtype=dtype)), self.method,
                     self.grid_shape, dict(self.extra))


def linear_array(n: int, pitch: float) -> np.ndarray:
    """``n`` elements on the x axis, centred, ``y = z = 0`` (``n x 3``)."""
    x = (np.arange(n) - (n - 1) / 2.0) * pitch
    return np.asfortranarray(np.stack([x, np.zeros(n), np.zeros(n)], axis=1))


def rca_arrays(n_cols: int, n_rows: int, pitch: float):
    """Row-column array: columns spread along x, rows along y, z = 0.

    Returns ``(G_col, G_row)``; the reference requires ``Gt = G_col`` and
    ``Gr = G_row`` whichever direction transmits.
    """
    xc = (np.arange(n_cols) - (n_cols - 1) / 2.0) * pitch
    yr = (np.arange(n_rows) - (n_rows - 1) / 2.0) * pitch
    G_col = np.stack([xc, np.zeros(n_cols), np.zeros(n_cols)], axis=1)
    G_row = np.stack([np.zeros(n_rows), yr, np.zeros(n_rows)], axis=1)
    return np.asfortranarray(G_col), np.asfortranarray(G_row)


def grid_xz(nx: int, nz: int, x_rng, z_rng) -> np.ndarray:
    """``meshgrid(x, z)`` flattened column-major: z is the fastest index."""
    x = np.linspace(x_rng[0], x_rng[1], nx)
    z = np.linspace(z_rng[0], z_rng[1], nz)
    X, Z = np.meshgrid(x, z)
    return np.asfortranarray(
        np.stack([X.flatten("F"), np.zeros(X.size), Z.flatten("F")], axis=1))


def grid_xyz(nx: int, ny: int, nz: int, x_rng, y_rng, z_rng) -> np.ndarray:
    """3-D grid flattened with z fastest, then y, then x."""
    x = np.linspace(x_rng[0], x_rng[1], nx)
    y = np.linspace(y_rng[0], y_rng[1], ny)
    z = np.linspace(z_rng[0], z_rng[1], nz)
    Xg, Yg, Zg = np.meshgrid(x, y, z, indexing="ij")
    # index = iz + nz*(iy + ny*ix)
    return np.asfortranarray(np.stack(
        [Xg.reshape(-1), Yg.reshape(-1), Zg.reshape(-1)], axis=1))


def pulse(tau: np.ndarray, f0: float, sigma: float) -> np.ndarray:
    """Gaussian-windowed sine, ``exp(-tau^2 / (2 sigma^2)) * sin(2 pi f0 tau)``."""
    return np.exp(-tau * tau / (2.0 * sigma * sigma)) * np.sin(2.0 * np.pi * f0 * tau)


def _add_echoes(Y: np.ndarray, t_travel: np.ndarray, amp: np.ndarray, dt: float,
                f0: float, sigma: float) -> None:
    """Adds ``amp[s] * pulse(t_k - t_travel[col, s])`` to every column of Y.

    Only the +-5 sigma window around each arrival is evaluated.
    """
    K, C = Y.shape
    half = int(np.ceil(5.0 * sigma / dt)) + 1
    offs = np.arange(-half, half + 1)
    for s in range(t_travel.shape[1]):
        c0 = np.floor(t_travel[:, s] / dt).astype(np.int64)  # (C,)
        k = c0[:, None] + offs[None, :]                      # (C, W)
        ok = (k >= 0) & (k < K)
        tau = k * dt - t_travel[:, s][:, None]
        val = amp[s] * pulse(tau, f0, sigma)
        cols = np.broadcast_to(np.arange(C)[:, None], k.shape)
        np.add.at(Y, (k[ok], cols[ok]), val[ok])


def _dist(G: np.ndarray, P: np.ndarray) -> np.ndarray:
    """Euclidean distance between every element (rows of G) and point (rows of P)."""
    d = G[:, None, :] - P[None, :, :]
    return np.sqrt((d * d).sum(axis=2))


def saft_scene(seed: int = 0, n_el: int = 64, K: int = 2048, nx: int = 256, nz: int = 256,
               n_scat: int = 10, dt: float = 0.04, cp: float = 1500.0,
               pitch: float = 0.5) -> Scene:
    rng = np.random.default_rng(seed)
    G = linear_array(n_el, pitch)
    sx = rng.uniform(-12.0, 12.0, n_scat)
    sz = rng.uniform(10.0, 40.0, n_scat)
    amp = rng.uniform(0.5, 1.0, n_scat)
    S = np.stack([sx, np.zeros(n_scat), sz], axis=1)
    v = cp / 1000.0  # mm/us
    t = 2.0 * _dist(G, S) / v  # (n_el, n_scat)
    Y = np.zeros((K, n_el), order="F")
    _add_echoes(Y, t, amp, dt, 5.0, 0.1)
    Y += rng.normal(0.0, 0.01, Y.shape)
    Ro = grid_xz(nx, nz, (-16.0, 16.0), (5.0, 45.0))
    return Scene(np.asfortranarray(Y), G, np.zeros((0, 3), order="F"), Ro, dt,
                 np.zeros((1, 1), order="F"), cp, "saft", (nx, nz),
                 {"scatterers": S, "amp": amp})


def tfm_scene(seed: int = 1, n_el: int = 64, K: int = 3000, nx: int = 512, nz: int = 512,
              n_scat: int = 10, dt: float = 0.04, cp: float = 1500.0,
              pitch: float = 0.5) -> Scene:
    rng = np.random.default_rng(seed)
    G = linear_array(n_el, pitch)
    sx = rng.uniform(-12.0, 12.0, n_scat)
    sz = rng.uniform(10.0, 40.0, n_scat)
    amp = rng.uniform(0.5, 1.0, n_scat)
    S = np.stack([sx, np.zeros(n_scat), sz], axis=1)
    v = cp / 1000.0
    d = _dist(G, S)  # (n_el, n_scat)
    # column = tx * n_el + rx
    t = ((d[:, None, :] + d[None, :, :]) / v).reshape(n_el * n_el, n_scat)
    Y = np.zeros((K, n_el * n_el), order="F")
    _add_echoes(Y, t, amp, dt, 5.0, 0.1)
    Y += rng.normal(0.0, 0.01, Y.shape)
    Ro = grid_xz(nx, nz, (-20.0, 20.0), (2.0, 50.0))
    return Scene(np.asfortranarray(Y), G, G.copy(order="F"), Ro, dt,
                 np.zeros((1, 1), order="F"), cp, "tfm", (nx, nz),
                 {"scatterers": S, "amp": amp})


def _stripe_dist_cols(G_col, G_row, P):
    """Distance from each column stripe (along y, spanning the rows' extent) to P."""
    y_min, y_max = G_row[0, 1], G_row[-1, 1]
    dy = np.where(P[:, 1] < y_min, y_min - P[:, 1], np.where(P[:, 1] > y_max, y_max - P[:, 1], 0.0))
    dx = G_col[:, 0][:, None] - P[:, 0][None, :]
    dz = G_col[:, 2][:, None] - P[:, 2][None, :]
    return np.sqrt(dx * dx + dy[None, :] ** 2 + dz * dz)


def _stripe_dist_rows(G_col, G_row, P):
    """Distance from each row stripe (along x, spanning the columns' extent) to P."""
    x_min, x_max = G_col[0, 0], G_col[-1, 0]
    dx = np.where(P[:, 0] < x_min, x_min - P[:, 0], np.where(P[:, 0] > x_max, x_max - P[:, 0], 0.0))
    dy = G_row[:, 1][:, None] - P[:, 1][None, :]
    dz = G_row[:, 2][:, None] - P[:, 2][None, :]
    return np.sqrt(dx[None, :] ** 2 + dy * dy + dz * dz)


def rca_scene(seed: int = 2, n_cols: int = 128, n_rows: int = 128, K: int = 4096,
              nx: int = 128, ny: int = 128, nz: int = 256, n_scat: int = 20,
              dt: float = 0.025, cp: float = 1480.0, pitch: float = 0.3,
              method: str = "rca_rowtx", z_rng=(5.0, 35.0)) -> Scene:
    rng = np.random.default_rng(seed)
    G_col, G_row = rca_arrays(n_cols, n_rows, pitch)
    sx = rng.uniform(-19.0, 19.0, n_scat)
    sy = rng.uniform(-19.0, 19.0, n_scat)
    sz = rng.uniform(z_rng[0], z_rng[1], n_scat)
    amp = rng.uniform(0.5, 1.0, n_scat)
    S = np.stack([sx, sy, sz], axis=1)
    v = cp / 1000.0
    dc = _stripe_dist_cols(G_col, G_row, S)  # (n_cols, n_scat)
    dr = _stripe_dist_rows(G_col, G_row, S)  # (n_rows, n_scat)
    if method == "rca_rowtx":  # column = row * n_cols + col
        t = ((dr[:, None, :] + dc[None, :, :]) / v).reshape(n_rows * n_cols, n_scat)
    else:                      # column = col * n_rows + row
        t = ((dc[:, None, :] + dr[None, :, :]) / v).reshape(n_cols * n_rows, n_scat)
    Y = np.zeros((K, n_cols * n_rows), order="F", dtype=np.float64)
    _add_echoes(Y, t, amp, dt, 6.0, 0.1)
    Y += rng.normal(0.0, 0.005, Y.shape)
    Ro = grid_xyz(nx, ny, nz, (-19.0, 19.0), (-19.0, 19.0), z_rng)
    return Scene(np.asfortranarray(Y), G_col, G_row, Ro, dt, np.zeros((1, 1), order="F"),
                 cp, method, (nx, ny, nz), {"scatterers": S, "amp": amp})


def cg_scene(seed: int = 4, n_el: int = 32, K: int = 2048, nx: int = 256, nz: int = 256,
             density: float = 0.01, dt: float = 0.04, cp: float = 1500.0, pitch: float = 0.5,
             x_rng=(-8.0, 8.0), z_rng=(5.0, 37.0)):
    """Model-based reconstruction scene: a 32 x 32 TFM array, K = 2048, and a
    seeded sparse reflectivity image on a 256 x 256 grid (``density`` of the
    points nonzero, values N(0, 1)). The A-scans are synthesised by the
    adjoint (scatter) operator, so this returns the geometry and the image;
    ``Y`` is left empty (K x 0)."""
    rng = np.random.default_rng(seed)
    G = linear_array(n_el, pitch)
    Ro = grid_xz(nx, nz, x_rng, z_rng)
    x = np.zeros(Ro.shape[0])
    nnz = max(1, int(round(density * x.size)))
    idx = rng.choice(x.size, nnz, replace=False)
    x[idx] = rng.normal(0.0, 1.0, nnz)
    return Scene(np.zeros((K, 0), order="F"), G, G.copy(order="F"), Ro, dt, np.zeros((1, 1), order="F"),
                 cp, "tfm", (nx, nz), {"reflectivity": x})


def batch_specs(seed: int = 7, n_frames: int = 48):
    """Uneven frames for batched beamforming: elements per frame from
    {16, 32, 64, 128} (tx = rx), A-scan length K ~ U{1024..4096}, cp ~
    U[1450, 1550] m/s, square grids with a side ~ U{64..512}; dt = 0.04 us.
    The imaged depth follows K so most paths fit in the A-scan."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_frames):
        n_el = int(rng.choice([16, 32, 64, 128]))
        K = int(rng.integers(1024, 4097))
        cp = float(rng.uniform(1450.0, 1550.0))
        side = int(rng.integers(64, 513))
        out.append(dict(n_el=n_el, K=K, cp=cp, side=side, dt=0.04, seed=int(rng.integers(1 << 30))))
    return out


def tfm_frame_torch(spec: dict, device="cuda", n_scat: int = 10, noise: float = 0.01):
    """One batch frame with its A-scans synthesised on the GPU (torch): seeded
    point scatterers with the 5 MHz Gaussian-windowed sine plus N(0, noise).
    Returns (Y column-major FP32 (K, n_el^2) on the device, G, Ro, dt, cp)."""
    import torch
    rng = np.random.default_rng(spec["seed"])
    n_el, K, cp, side, dt = spec["n_el"], spec["K"], spec["cp"], spec["side"], spec["dt"]
    v = cp / 1000.0
    z_max = min(50.0, 0.35 * K * dt * v)
    x_half = min(20.0, 0.5 * z_max)
    G = linear_array(n_el, 0.5)
    Ro = grid_xz(side, side, (-x_half, x_half), (2.0, z_max))
    S = np.stack([rng.uniform(-0.6 * x_half, 0.6 * x_half, n_scat), np.zeros(n_scat),
                  rng.uniform(0.25 * z_max, 0.9 * z_max, n_scat)], axis=1)
    amp = rng.uniform(0.5, 1.0, n_scat)
    d = torch.from_numpy(_dist(G, S)).to(device)                       # (n_el, S)
    t = ((d[:, None, :] + d[None, :, :]) / v).reshape(n_el * n_el, n_scat)  # (C, S)
    C = n_el * n_el
    gen = torch.Generator(device=device).manual_seed(spec["seed"])
    Yc = torch.randn((C, K), generator=gen, device=device, dtype=torch.float32) * noise  # row c = column c
    half = int(np.ceil(0.5 / dt)) + 1
    offs = torch.arange(-half, half + 1, device=device, dtype=torch.float64)
    k = torch.floor(t / dt)[..., None] + offs                           # (C, S, W)
    tau = k * dt - t[..., None]
    val = torch.from_numpy(amp).to(device)[None, :, None] * torch.exp(-tau * tau / 0.02) * torch.sin(
        2.0 * np.pi * 5.0 * tau)
    ok = (k >= 0) & (k < K)
    cols = torch.arange(C, device=device, dtype=torch.float64)[:, None, None].expand_as(k)
    flat = (cols * K + k)[ok].long()
    Yc.view(-1).index_add_(0, flat, val[ok].float())
    return Yc.t(), G, Ro, dt, cp


def rca_frame_torch(seed: int = 2, n_cols: int = 128, n_rows: int = 128, K: int = 4096, nx: int = 128,
                    ny: int = 128, nz: int = 256, n_scat: int = 20, dt: float = 0.025, cp: float = 1480.0,
                    pitch: float = 0.3, method: str = "rca_rowtx", z_rng=(5.0, 35.0), noise: float = 0.005,
                    device="cuda"):
    """The RCA configuration with A-scans synthesised on the GPU (torch):
    seeded point scatterers in a 38 x 38 x 30 mm volume, 6 MHz Gaussian-windowed
    sine, N(0, noise). Returns (Y column-major FP32 (K, n_cols*n_rows) on the
    device, G_col, G_row, Ro). Row-tx columns are row*n_cols + col."""
    import torch
    rng = np.random.default_rng(seed)
    G_col, G_row = rca_arrays(n_cols, n_rows, pitch)
    S = np.stack([rng.uniform(-19.0, 19.0, n_scat), rng.uniform(-19.0, 19.0, n_scat),
                  rng.uniform(z_rng[0], z_rng[1], n_scat)], axis=1)
    amp = rng.uniform(0.5, 1.0, n_scat)
    v = cp / 1000.0
    dc = torch.from_numpy(_stripe_dist_cols(G_col, G_row, S)).to(device)
    dr = torch.from_numpy(_stripe_dist_rows(G_col, G_row, S)).to(device)
    if method == "rca_rowtx":
        t = ((dr[:, None, :] + dc[None, :, :]) / v).reshape(n_rows * n_cols, n_scat)
    else:
        t = ((dc[:, None, :] + dr[None, :, :]) / v).reshape(n_cols * n_rows, n_scat)
    C = n_cols * n_rows
    gen = torch.Generator(device=device).manual_seed(seed)
    Yc = torch.randn((C, K), generator=gen, device=device, dtype=torch.float32) * noise
    half = int(np.ceil(0.5 / dt)) + 1
    offs = torch.arange(-half, half + 1, device=device, dtype=torch.float64)
    k = torch.floor(t / dt)[..., None] + offs
    tau = k * dt - t[..., None]
    val = torch.from_numpy(amp).to(device)[None, :, None] * torch.exp(-tau * tau / 0.02) * torch.sin(
        2.0 * np.pi * 6.0 * tau)
    ok = (k >= 0) & (k < K)
    cols = torch.arange(C, device=device, dtype=torch.float64)[:, None, None].expand_as(k)
    Yc.view(-1).index_add_(0, (cols * K + k)[ok].long(), val[ok].float())
    Ro = grid_xyz(nx, ny, nz, (-19.0, 19.0), (-19.0, 19.0), z_rng)
    return Yc.t(), G_col, G_row, Ro
