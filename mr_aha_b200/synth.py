"""Seeded synthetic problems for the Toeplitz A^H A operator.

Every generator returns NumPy arrays in the row-major layout of the Python
binding (the column-major shapes of the C API reversed):

=============  ================================  ==============================
array          row-major shape                   column-major (C API)
=============  ================================  ==============================
``traj``       ``(ndim, Nkx, Ntrajs)`` float32   ``[Ntrajs, Nkx, ndim]``
``phi2``       ``(L, L, Ntrajs)`` / stack        ``[Ntrajs, L, L]`` /
               ``(L, L, Nkz, Ntrajs)``           ``[Ntrajs, Nkz, L, L]``
``x``          ``(L, [Nz,] Ny, Nx)``             ``[Nx, Ny, [Nz,] L]``
``SEs``        ``(C, [Nz,] Ny, Nx)``             ``[Nx, Ny, [Nz,] C]``
=============  ================================  ==============================

``phi2[j, i, ...]`` holds entry ``(i, j)`` of the Hermitian Gram block
``Phi Phi^H`` (rank x time ``Phi``), the convention of the reference's
``include/mr_aha/mr_aha.h:33-62``.

Two families of inputs are provided:

* the reference's own test recipe (``tests/make_reference.py:130-236`` of the
  reference): golden-angle radial / golden-means kooshball trajectories,
  random rank-2 Gram blocks per readout (and per kz), complex normal maps;
* the headline workloads: a stack-of-stars golden-angle trajectory, Gram blocks
  from a random orthonormal temporal basis with spokes assigned to frames,
  smoothed coil maps normalised to ``sum_c |S_c|^2 = 1``.
"""

from __future__ import annotations

import numpy as np

GOLDEN = (np.sqrt(5.0) - 1.0) / 2.0

#: The reference's synthetic test cases (``tests/make_reference.py:130-146``).
REFERENCE_CASES = [
    dict(name="2d_50x40_L3_c3", traj_type="2D", n_dim=(50, 40), L=3, n_coils=3,
         n_traj=61, n_kx=100, seed=1),
    dict(name="2d_33x27_L1_c2_odd", traj_type="2D", n_dim=(33, 27), L=1, n_coils=2,
         n_traj=45, n_kx=66, seed=2),
    dict(name="2d_50x40_L4_c2_M101x81", traj_type="2D", n_dim=(50, 40), L=4,
         n_coils=2, n_traj=61, n_kx=100, seed=3, phi2_dim=(101, 81)),
    dict(name="3d_24x20x16_L4_c2", traj_type="3D", n_dim=(24, 20, 16), L=4,
         n_coils=2, n_traj=400, n_kx=48, seed=4),
    dict(name="3d_25x21x15_L3_c2_odd", traj_type="3D", n_dim=(25, 21, 15), L=3,
         n_coils=2, n_traj=350, n_kx=50, seed=5),
    dict(name="stack_40x36x10_L3_c3", traj_type="stack", n_dim=(40, 36, 10), L=3,
         n_coils=3, n_traj=40, n_kx=80, seed=6),
    dict(name="stack_31x36x9_L4_c2_odd", traj_type="stack", n_dim=(31, 36, 9), L=4,
         n_coils=2, n_traj=35, n_kx=62, seed=7),
]

#: Headline workloads: a CPU-sized stack and the 320 x 320 x 56 stack.
WORKLOADS = {
    "stack64": dict(traj_type="stack", n_dim=(64, 64, 8), L=4, n_coils=4,
                    n_traj=64, n_kx=128, n_frames=32, frame_rule="mod", seed=0),
    "stack320": dict(traj_type="stack", n_dim=(320, 320, 56), L=16, n_coils=12,
                     n_traj=1000, n_kx=640, n_frames=200, frame_rule="div", seed=1),
    # small cases of the headline kernels for profiling (a few GB on the
    # device): the headline in-plane size, rank and coils on 4 kz planes; and
    # the headline 56-point z lines with rank 1 and 16 coils
    "slab320": dict(traj_type="stack", n_dim=(320, 320, 4), L=16, n_coils=12,
                    n_traj=1000, n_kx=640, n_frames=200, frame_rule="div", seed=2),
    "zlines320": dict(traj_type="stack", n_dim=(320, 320, 56), L=1, n_coils=16,
                      n_traj=1000, n_kx=640, n_frames=200, frame_rule="div", seed=3),
}


def default_phi2_dim(traj_type: str, n_dim) -> tuple:
    """``2 * n_dim``, except ``Mz = Nz`` for a stack (the reference's default)."""
    m = [2 * int(v) for v in n_dim]
    if traj_type == "stack":
        m[2] = int(n_dim[2])
    return tuple(m)


def radial_readout(n_kx: int) -> np.ndarray:
    """Readout positions ``pi * (2 s / n_kx - 1)`` in ``[-pi, pi)``."""
    return np.pi * (2.0 * np.arange(n_kx) / n_kx - 1.0)


def make_traj(traj_type: str, n_traj: int, n_kx: int) -> np.ndarray:
    """Golden-angle radial (2D, stack) or golden-means kooshball (3D) spokes.

    Follows ``tests/make_reference.py:172-201`` of the reference. Returns
    ``float32`` ``(ndim, Nkx, Ntrajs)`` in radians per image-grid unit.
    """
    r = radial_readout(n_kx)[:, None]
    t = np.arange(n_traj)[None, :]
    if traj_type in ("2D", "stack"):
        th = np.pi * GOLDEN * t
        traj = np.stack([r * np.cos(th), r * np.sin(th)])
    else:
        phi1, phi2 = 0.4656, 0.6823
        z = np.mod(t * phi1, 1.0)
        az = 2.0 * np.pi * np.mod(t * phi2, 1.0)
        s = np.sqrt(1.0 - z ** 2)
        traj = np.stack([r * s * np.cos(az), r * s * np.sin(az), r * z])
    return np.ascontiguousarray(traj, dtype=np.float32)


def crandn(rng, shape, dtype=np.complex64) -> np.ndarray:
    """Standard complex Gaussian array (real and imaginary parts N(0, 1))."""
    if np.dtype(dtype) == np.complex64:
        out = np.empty(shape, dtype=np.complex64)
        v = out.view(np.float32)
        v[...] = rng.standard_normal(v.shape, dtype=np.float32)
        return out
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def make_phi2_random(rng, L: int, n_traj: int, n_kz) -> np.ndarray:
    """Random rank-2 Hermitian PSD Gram blocks, as ``make_reference.py:204-231``.

    ``B = A^T conj(A) / 2`` with ``A`` complex normal ``(..., 2, L)``; stored
    ``phi2[j, i, (z,) t] = B[t, (z,) i, j]``.
    """
    lead = (n_traj,) if n_kz is None else (n_traj, n_kz)
    A = rng.standard_normal(lead + (2, L)) + 1j * rng.standard_normal(lead + (2, L))
    B = np.einsum("...ki,...kj->...ij", A, A.conj()) / 2.0
    phi2 = B.transpose(tuple(range(B.ndim))[::-1])
    return np.ascontiguousarray(phi2, dtype=np.complex64)


def make_basis(rng, L: int, n_frames: int) -> np.ndarray:
    """Random temporal basis ``Phi`` (L x T) with orthonormal rows (Q^H of a QR)."""
    G = rng.standard_normal((n_frames, L)) + 1j * rng.standard_normal((n_frames, L))
    Q, _ = np.linalg.qr(G)
    return np.ascontiguousarray(Q.conj().T)


def frames_of_spokes(n_traj: int, n_frames: int, rule: str) -> np.ndarray:
    """Frame index of every spoke: round robin (``mod``) or even split (``div``)."""
    t = np.arange(n_traj)
    if rule == "mod":
        return t % n_frames
    per = max(1, n_traj // n_frames)
    return np.minimum(t // per, n_frames - 1)


def make_phi2_basis(Phi: np.ndarray, frames: np.ndarray, n_kz) -> np.ndarray:
    """Per-spoke Gram blocks ``Phi[:, f] Phi[:, f]^H``, identical for every kz."""
    L = Phi.shape[0]
    cols = Phi[:, frames]                                 # (L, Ntrajs)
    B = np.einsum("it,jt->tij", cols, cols.conj())       # (Ntrajs, L, L)
    blk = B.transpose(2, 1, 0)                            # [j, i, t] = B[t, i, j]
    if n_kz is None:
        return np.ascontiguousarray(blk, dtype=np.complex64)
    out = np.empty((L, L, n_kz, B.shape[0]), dtype=np.complex64)
    out[...] = blk[:, :, None, :]
    return out


def make_smooth_maps(rng, n_coils: int, img_shape) -> np.ndarray:
    """Gaussian-smoothed complex normal maps with ``sum_c |S_c|^2 = 1`` per voxel.

    Smoothing is in-plane (the last two axes), periodic, with
    ``sigma = N / 8`` pixels per axis.
    """
    S = crandn(rng, (n_coils,) + tuple(img_shape), np.complex64)
    ny, nx = img_shape[-2], img_shape[-1]
    fy = np.fft.fftfreq(ny)[:, None]
    fx = np.fft.fftfreq(nx)[None, :]
    sy, sx = ny / 8.0, nx / 8.0
    H = np.exp(-2.0 * np.pi ** 2 * ((sy * fy) ** 2 + (sx * fx) ** 2)).astype(np.float32)
    for c in range(n_coils):
        F = np.fft.fft2(S[c], axes=(-2, -1))
        F *= H
        S[c] = np.fft.ifft2(F, axes=(-2, -1)).astype(np.complex64)
    norm = np.sqrt(np.sum(np.abs(S) ** 2, axis=0, dtype=np.float64)).astype(np.float32)
    norm[norm == 0] = 1.0
    S /= norm[None]
    return np.ascontiguousarray(S, dtype=np.complex64)


def reference_case(case: dict) -> dict:
    """Inputs of one reference test case (``make_reference.py:160-236``)."""
    rng = np.random.default_rng(case["seed"])
    tt, n_dim, L, nc = case["traj_type"], tuple(case["n_dim"]), case["L"], case["n_coils"]
    traj = make_traj(tt, case["n_traj"], case["n_kx"])
    n_kz = n_dim[2] if tt == "stack" else None
    phi2 = make_phi2_random(rng, L, case["n_traj"], n_kz)
    img = tuple(reversed(n_dim))
    x = crandn(rng, (L,) + img)
    SEs = crandn(rng, (nc,) + img)
    phi2_dim = case.get("phi2_dim") or default_phi2_dim(tt, n_dim)
    return dict(traj_type=tt, n_dim=n_dim, phi2_dim=tuple(phi2_dim), L=L,
                n_coils=nc, traj=traj, phi2=phi2, x=x, SEs=SEs)


def workload(name: str, with_x: bool = True) -> dict:
    """Inputs of a headline workload (``stack64`` or ``stack320``)."""
    w = WORKLOADS[name]
    rng = np.random.default_rng(w["seed"])
    tt, n_dim, L, nc = w["traj_type"], tuple(w["n_dim"]), w["L"], w["n_coils"]
    traj = make_traj(tt, w["n_traj"], w["n_kx"])
    Phi = make_basis(rng, L, w["n_frames"])
    frames = frames_of_spokes(w["n_traj"], w["n_frames"], w["frame_rule"])
    n_kz = n_dim[2] if tt == "stack" else None
    phi2 = make_phi2_basis(Phi, frames, n_kz)
    img = tuple(reversed(n_dim))
    SEs = make_smooth_maps(rng, nc, img)
    x = crandn(rng, (L,) + img) if with_x else None
    return dict(traj_type=tt, n_dim=n_dim, phi2_dim=default_phi2_dim(tt, n_dim),
                L=L, n_coils=nc, traj=traj, phi2=phi2, x=x, SEs=SEs, Phi=Phi,
                frames=frames)


# ---------------------------------------------------------------------------
# Uneven batches and served requests
# ---------------------------------------------------------------------------

BATCH_CHOICES = dict(n=(128, 192, 256, 320), nz=(8, 16, 32, 56), L=(4, 8, 16, 32),
                     coils=(8, 12, 16, 32))


def batch_specs(n_ops: int = 48, seed: int = 3, choices: dict = BATCH_CHOICES,
                spokes=(200, 1000)) -> list:
    """Seeded stack operators of uneven size: in-plane ``n``, ``Nz``, rank
    ``L`` and coil count drawn uniformly from ``choices``; spokes uniform in
    ``spokes``; ``Nkx = 2 n``; ``max(L, spokes // 5)`` frames split evenly."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_ops):
        n = int(rng.choice(choices["n"]))
        nz = int(rng.choice(choices["nz"]))
        L = int(rng.choice(choices["L"]))
        nc = int(rng.choice(choices["coils"]))
        n_traj = int(rng.integers(spokes[0], spokes[1] + 1))
        out.append(dict(traj_type="stack", n_dim=(n, n, nz), L=L, n_coils=nc, n_traj=n_traj,
                        n_kx=2 * n, n_frames=max(L, n_traj // 5), frame_rule="div",
                        seed=seed * 1000 + i))
    return out


def spec_inputs(spec: dict, with_x: bool = True) -> dict:
    """Inputs of one operator spec (same recipe as the headline workloads)."""
    rng = np.random.default_rng(spec["seed"])
    tt, n_dim, L, nc = spec["traj_type"], tuple(spec["n_dim"]), spec["L"], spec["n_coils"]
    traj = make_traj(tt, spec["n_traj"], spec["n_kx"])
    Phi = make_basis(rng, L, spec["n_frames"])
    frames = frames_of_spokes(spec["n_traj"], spec["n_frames"], spec["frame_rule"])
    n_kz = n_dim[2] if tt == "stack" else None
    phi2 = make_phi2_basis(Phi, frames, n_kz)
    img = tuple(reversed(n_dim))
    SEs = make_smooth_maps(rng, nc, img)
    x = crandn(rng, (L,) + img) if with_x else None
    return dict(traj_type=tt, n_dim=n_dim, phi2_dim=default_phi2_dim(tt, n_dim), L=L,
                n_coils=nc, traj=traj, phi2=phi2, x=x, SEs=SEs)


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of a Poisson process of ``rate`` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
