"""CPU oracle of the Toeplitz A^H A operator (FP64 NumPy restatement).

TEST INFRASTRUCTURE ONLY. Nothing in the shipped library imports, links or
calls this module. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline of ``bench.py`` use it, and only as the checker (or, in the CPU
baseline, as the timed CPU restatement).

It restates, in double precision, the reference's algorithm for the path:

* index conventions: ``mr_cent2nat`` / ``mr_nat2cent`` / ``mr_tri_offset``
  (``src/cuda/mr_internal.cuh:119-181``);
* Gram packing: ``mr_k_extract_tri`` (``src/cuda/mr_kernels.cu:307-333``);
* the Toeplitz kernel build ``mr_calc_toep`` (``src/cuda/mr_calc_toep.cu:
  498-643``): pack -> broadcast the packed element along each readout
  (``mr_k_fill_strengths``, ``mr_kernels.cu:335-362``) -> type-1 NUFFT with
  sign -1 and centered modes (``include/mr_aha/mr_aha.h:1169-1181``) ->
  centered inverse FFT scaled by ``1/prod(M)`` over the transformed axes
  (``mr_calc_toep.cu:171-200``; ``mr_kernels.cu:364-425``). The type-1 NUFFT
  is evaluated here as the EXACT non-uniform DFT (no spreading kernel), which
  is what cufinufft approximates to ``eps``;
* the apply ``mr_aha_plan_execute`` (``src/cuda/mr_aha.cu:694-790``): pad and
  multiply by the coil map (``mr_kernels.cu:98-142``), unnormalised forward
  DFT over the upsampled grid, packed Hermitian block multiply of the rank row
  vector from the right (``src/cuda/mr_kernels_bd.cu:56-139``), unnormalised
  inverse DFT, crop and conjugate-map coil sum (``mr_kernels.cu:144-176``);
  masked kernels through the grid-to-mask map (``mr_kernels.cu:221-301``);
* the independent NUFFT-route operator ``aha_nufft_plan.apply``
  (``python/mr_aha/nufft.py:473-552``), again with exact NUDFTs;
* the automatic mask ``mr_calc_mask`` (``src/cuda/mr_calc_mask.cu:63-404``),
  bit-exact (same float32 rounding of the grid-point search).

Because the 2x circulant embedding is exact, the Toeplitz apply with the exact
kernel equals the exact NUFFT route up to rounding: that identity is the
known-answer test that pins this restatement independently of any golden
file. Arrays use the row-major layout of the Python binding (column-major C
shapes reversed).
"""

from __future__ import annotations

import numpy as np

TWO_PI = 6.283185307179586


# --------------------------------------------------------------------------
# Index conventions (mr_internal.cuh:119-181)
# --------------------------------------------------------------------------

def cent2nat(k, M):
    """Centered index -> natural (FFT-order) index (``mr_internal.cuh:119-125``)."""
    j = np.asarray(k) - M // 2
    return np.where(j < 0, j + M, j)


def nat2cent(j, M):
    """Natural index -> centered index (``mr_internal.cuh:134-139``)."""
    k = np.asarray(j) + M // 2
    return np.where(k >= M, k - M, k)


def tri_offset(i: int, j: int, L: int, upper: bool):
    """Packed offset of element (i, j) and whether to conjugate (``:155-181``)."""
    r, c, cj = i, j, False
    if upper:
        if r > c:
            r, c, cj = c, r, True
        return c * (c + 1) // 2 + r, cj
    if r < c:
        r, c, cj = c, r, True
    return c * L - c * (c - 1) // 2 + (r - c), cj


def tri_pairs(L: int, upper: bool):
    """(row, col) of every packed component, in packed order."""
    rows, cols = [], []
    for c in range(L):
        rr = range(0, c + 1) if upper else range(c, L)
        for r in rr:
            rows.append(r)
            cols.append(c)
    return np.array(rows), np.array(cols)


def num_tri(L: int) -> int:
    return L * (L + 1) // 2 if L > 0 else 0


# --------------------------------------------------------------------------
# Gram packing and full blocks
# --------------------------------------------------------------------------

def pack_gram(phi2: np.ndarray, L: int, upper: bool) -> np.ndarray:
    """Packed Gram components ``[ntri, (Nkz,) Ntrajs]`` (``mr_kernels.cu:307-333``).

    ``phi2`` is row-major ``(L, L, [Nkz,] Ntrajs)`` with ``phi2[j, i] = B[i, j]``.
    Component ``t`` of ``(r, c)`` is ``B[r, c] = phi2[c, r]``.
    """
    rows, cols = tri_pairs(L, upper)
    return np.ascontiguousarray(phi2[cols, rows])


def unpack_blocks(packed: np.ndarray, L: int, upper: bool) -> np.ndarray:
    """Full Hermitian blocks ``A[..., r, c]`` from packed ``[ntri, ...]``."""
    rows, cols = tri_pairs(L, upper)
    shape = packed.shape[1:] + (L, L)
    A = np.zeros(shape, dtype=np.result_type(packed.dtype, np.complex128))
    moved = np.moveaxis(packed, 0, -1)
    for t, (r, c) in enumerate(zip(rows, cols)):
        A[..., r, c] = moved[..., t]
        if r != c:
            A[..., c, r] = np.conj(moved[..., t])
    return A


# --------------------------------------------------------------------------
# Geometry helpers
# --------------------------------------------------------------------------

def spatial_axes(traj_type: str, n_dim):
    """Row-major image shape (without rank/coil) for a configuration."""
    if traj_type == "2D":
        return (int(n_dim[1]), int(n_dim[0]))
    return (int(n_dim[2]), int(n_dim[1]), int(n_dim[0]))


def pad_index_maps(n_img, m_pad):
    """Per axis, the natural index ``(x - floor(N/2)) mod M`` of every image index."""
    return [((np.arange(n) - n // 2) % m) for n, m in zip(n_img, m_pad)]


# --------------------------------------------------------------------------
# Kernel build (mr_calc_toep), exact NUDFT
# --------------------------------------------------------------------------

def _centered_freqs(M: int) -> np.ndarray:
    """Centered mode frequencies ``[-floor(M/2), ceil(M/2))``."""
    return np.arange(M) - M // 2


def psf_exact(traj_type: str, phi2_dim, packed: np.ndarray, traj: np.ndarray,
              comps=None, kzs=None, spoke_chunk: int = 64) -> np.ndarray:
    """Exact type-1 NUDFT (sign -1, centered modes) of the broadcast strengths.

    ``psf[t, (z,) ky, kx] = sum_m c_{t,m} exp(-i (kx x_m + ky y_m [+ kz z_m]))``
    with ``c_{t,m}`` the packed Gram element ``t`` of sample ``m``'s readout
    (``mr_calc_toep.cu:537-567``). The strength is constant along a readout,
    so the sum is grouped per readout: ``psf = sum_s T[t, s] G_s`` with
    ``G_s`` the readout's own exact point-spread function.

    Args:
        packed: ``[ntri, (Nkz,) Ntrajs]`` from :func:`pack_gram`.
        traj: ``(ndim, Nkx, Ntrajs)``.
        comps / kzs: optional subsets of components / kz planes (stack).
    Returns:
        complex128 ``[ncomp, (nkz,) My, Mx]`` (stack/2D) or
        ``[ncomp, Mz, My, Mx]`` (3D).
    """
    tr = np.asarray(traj, dtype=np.float64)
    ntri = packed.shape[0]
    comps = np.arange(ntri) if comps is None else np.asarray(comps)
    Ntrajs = tr.shape[2]
    Mx, My = int(phi2_dim[0]), int(phi2_dim[1])
    fx, fy = _centered_freqs(Mx), _centered_freqs(My)
    if traj_type == "3D":
        Mz = int(phi2_dim[2])
        fz = _centered_freqs(Mz)
        out = np.zeros((len(comps), Mz, My, Mx), dtype=np.complex128)
        T = packed[comps]                                   # [nc, Ntrajs]
        for s0 in range(0, Ntrajs, spoke_chunk):
            s1 = min(Ntrajs, s0 + spoke_chunk)
            ex = np.exp(-1j * tr[0, :, s0:s1, None] * fx)   # [Nkx, ns, Mx]
            ey = np.exp(-1j * tr[1, :, s0:s1, None] * fy)
            ez = np.exp(-1j * tr[2, :, s0:s1, None] * fz)
            G = np.einsum("rsz,rsy,rsx->szyx", ez, ey, ex, optimize=True)
            out += np.einsum("cs,szyx->czyx", T[:, s0:s1], G, optimize=True)
        return out
    stack = traj_type == "stack"
    if stack:
        Nkz = packed.shape[1]
        kzs = np.arange(Nkz) if kzs is None else np.asarray(kzs)
        T = packed[comps][:, kzs, :]                        # [nc, nz, Ntrajs]
        out = np.zeros((len(comps), len(kzs), My, Mx), dtype=np.complex128)
    else:
        T = packed[comps]
        out = np.zeros((len(comps), My, Mx), dtype=np.complex128)
    for s0 in range(0, Ntrajs, spoke_chunk):
        s1 = min(Ntrajs, s0 + spoke_chunk)
        ex = np.exp(-1j * tr[0, :, s0:s1, None] * fx)       # [Nkx, ns, Mx]
        ey = np.exp(-1j * tr[1, :, s0:s1, None] * fy)       # [Nkx, ns, My]
        G = np.einsum("rsy,rsx->syx", ey, ex, optimize=True)  # [ns, My, Mx]
        if stack:
            out += np.einsum("czs,syx->czyx", T[:, :, s0:s1], G, optimize=True)
        else:
            out += np.einsum("cs,syx->cyx", T[:, s0:s1], G, optimize=True)
    return out


def psf_to_kernel(traj_type: str, psf: np.ndarray) -> np.ndarray:
    """Centered inverse FFT scaled by ``1/prod(M)`` (``mr_calc_toep.cu:171-200``).

    The unnormalised inverse DFT times ``1/prod(M)`` is NumPy's normalised
    ``ifftn``; the centering shifts are ``ifftshift`` before and ``fftshift``
    after (shift ``floor(M/2)``), over (y, x) for 2D / stack and (z, y, x)
    for 3D. The kz axis of a stack is neither shifted nor transformed.
    """
    axes = (-3, -2, -1) if traj_type == "3D" else (-2, -1)
    w = np.fft.ifftshift(psf, axes=axes)
    w = np.fft.ifftn(w, axes=axes)
    return np.fft.fftshift(w, axes=axes)


def calc_toep(traj_type: str, phi2_dim, L: int, phi2: np.ndarray,
              traj: np.ndarray, upper: bool = False, mask=None,
              comps=None, kzs=None) -> np.ndarray:
    """FP64 ``phi2_toep`` (``[ntri, (Mz,) My, Mx]``, or ``[ntri, num_masked]``).

    ``comps`` / ``kzs`` select a subset of components / kz planes (then the
    leading axes are those subsets and ``mask`` must be None).
    """
    packed = pack_gram(np.asarray(phi2), L, upper)
    psf = psf_exact(traj_type, phi2_dim, packed, traj, comps=comps, kzs=kzs)
    K = psf_to_kernel(traj_type, psf)
    if traj_type == "2D" and K.ndim == 3:
        pass
    if mask is not None:
        flat = K.reshape(K.shape[0], -1)
        return np.ascontiguousarray(flat[:, np.asarray(mask)])
    return K


# --------------------------------------------------------------------------
# Toeplitz apply (mr_aha_plan_execute)
# --------------------------------------------------------------------------

def kernel_natural_full(traj_type, phi2_dim, phi2_toep, L, upper, mask=None):
    """Full natural-order blocks ``A[q..., r, c]`` of a packed kernel.

    Unmasked: the kernel at natural index ``j`` is the centered entry
    ``nat2cent(j)`` (``mr_kernels.cu:178-219``), i.e. an ``ifftshift`` over
    every spatial axis (including kz of a stack, ``mr_aha.cu:639-691``).
    Masked: grid locations outside the mask have a zero block
    (``mr_kernels.cu:221-301``).
    """
    m_pad = spatial_axes(traj_type, phi2_dim)
    ntri = num_tri(L)
    if mask is not None:
        full = np.zeros((ntri, int(np.prod(m_pad))), dtype=np.complex128)
        full[:, np.asarray(mask)] = np.asarray(phi2_toep).reshape(ntri, -1)
        K = full.reshape((ntri,) + m_pad)
    else:
        K = np.asarray(phi2_toep, dtype=np.complex128).reshape((ntri,) + m_pad)
    Knat = np.fft.ifftshift(K, axes=tuple(range(1, K.ndim)))
    return unpack_blocks(Knat, L, upper)                 # [*m_pad, L, L]


def aha_toeplitz(traj_type: str, n_dim, phi2_dim, L: int, x: np.ndarray,
                 SEs: np.ndarray, phi2_toep: np.ndarray, upper: bool = False,
                 mask=None, blocks=None) -> np.ndarray:
    """FP64 Toeplitz ``A^H A x`` (``mr_aha.cu:694-790``).

    ``x``: ``(L, *img)``; ``SEs``: ``(C, *img)``; returns complex128 like ``x``.
    ``blocks`` may pass a precomputed :func:`kernel_natural_full`.
    """
    img = spatial_axes(traj_type, n_dim)
    m_pad = spatial_axes(traj_type, phi2_dim)
    x = np.asarray(x, dtype=np.complex128).reshape((L,) + img)
    S = np.asarray(SEs, dtype=np.complex128).reshape((-1,) + img)
    A = blocks if blocks is not None else kernel_natural_full(
        traj_type, phi2_dim, phi2_toep, L, upper, mask)
    maps = pad_index_maps(img, m_pad)
    ix = np.ix_(*maps)
    axes = tuple(range(1, 1 + len(img)))
    out = np.zeros((L,) + img, dtype=np.complex128)
    for c in range(S.shape[0]):
        pad = np.zeros((L,) + m_pad, dtype=np.complex128)
        pad[(slice(None),) + ix] = S[c][None] * x
        F = np.fft.fftn(pad, axes=axes)                      # unnormalised
        v = np.moveaxis(F, 0, -1)                            # [*m_pad, L]
        y = np.einsum("...r,...rc->...c", v, A)              # v <- v A
        F = np.moveaxis(y, -1, 0)
        back = np.fft.ifftn(F, axes=axes) * np.prod(m_pad)   # unnormalised
        out += np.conj(S[c])[None] * back[(slice(None),) + ix]
    return out


def aha_toeplitz_lean(traj_type: str, n_dim, phi2_dim, L: int, x: np.ndarray,
                      SEs: np.ndarray, phi2_toep: np.ndarray, upper: bool = False) -> np.ndarray:
    """FP64 Toeplitz ``A^H A x`` for grids too large for :func:`aha_toeplitz`'s
    full ``L x L`` blocks (unmasked kernels only).

    The same arithmetic as :func:`aha_toeplitz` (``mr_aha.cu:694-790``), one
    coil at a time: the spectrum is moved to centred order
    (``fftshift``, the inverse of the kernel's ``nat2cent`` read,
    ``mr_kernels.cu:178-219``) and multiplied by walking the packed triangle
    in place (``mr_kernels_bd.cu:56-139``: ``y_c += A_rc v_r`` and, off the
    diagonal, ``y_r += conj(A_rc) v_c``), so no expanded block array exists;
    the packed kernel is read as given (complex64 values are exact in
    complex128)."""
    img = spatial_axes(traj_type, n_dim)
    m_pad = spatial_axes(traj_type, phi2_dim)
    ntri = num_tri(L)
    x = np.asarray(x, dtype=np.complex128).reshape((L,) + img)
    S = np.asarray(SEs).reshape((-1,) + img)
    K = np.asarray(phi2_toep).reshape((ntri,) + m_pad)
    rows, cols = tri_pairs(L, upper)
    ix = np.ix_(*pad_index_maps(img, m_pad))
    axes = tuple(range(1, 1 + len(img)))
    out = np.zeros((L,) + img, dtype=np.complex128)
    for c in range(S.shape[0]):
        Sc = S[c].astype(np.complex128)
        pad = np.zeros((L,) + m_pad, dtype=np.complex128)
        pad[(slice(None),) + ix] = Sc[None] * x
        v = np.fft.fftshift(np.fft.fftn(pad, axes=axes), axes=axes)
        del pad
        y = np.zeros_like(v)
        for t in range(ntri):
            r, cc = int(rows[t]), int(cols[t])
            a = K[t]
            y[cc] += a * v[r]
            if r != cc:
                y[r] += np.conj(a) * v[cc]
        del v
        back = np.fft.ifftn(np.fft.ifftshift(y, axes=axes), axes=axes) * np.prod(m_pad)
        del y
        out += np.conj(Sc)[None] * back[(slice(None),) + ix]
    return out


# --------------------------------------------------------------------------
# NUFFT route (python/mr_aha/nufft.py:473-552), exact NUDFTs
# --------------------------------------------------------------------------

def aha_nufft(traj_type: str, n_dim, L: int, x: np.ndarray, SEs: np.ndarray,
              phi2: np.ndarray, traj: np.ndarray) -> np.ndarray:
    """Exact ``sum_c S_c^H F_+ B F_- S_c x`` (type-2 sign -1, type-1 sign +1).

    Centered modes; a stack first takes the centered, unnormalised DFT along
    z (``nufft.py:44-57, 397-404``) and applies the kz-dependent Gram block.
    """
    img = spatial_axes(traj_type, n_dim)
    tr = np.asarray(traj, dtype=np.float64)
    ndim_t, Nkx, Ntrajs = tr.shape
    Msmp = Nkx * Ntrajs
    pts = [tr[d].reshape(-1) for d in range(ndim_t)]      # m = t + Ntrajs * r
    spoke = np.tile(np.arange(Ntrajs), Nkx)
    x = np.asarray(x, dtype=np.complex128).reshape((L,) + img)
    S = np.asarray(SEs, dtype=np.complex128).reshape((-1,) + img)
    P = np.asarray(phi2, dtype=np.complex128)
    out = np.zeros((L,) + img, dtype=np.complex128)
    if traj_type == "3D":
        Nz, Ny, Nx = img
        ex = np.exp(-1j * np.outer(pts[0], _centered_freqs(Nx)))   # [M, Nx]
        ey = np.exp(-1j * np.outer(pts[1], _centered_freqs(Ny)))
        ez = np.exp(-1j * np.outer(pts[2], _centered_freqs(Nz)))
        Bm = P[:, :, spoke]                                        # [l, m', M]
        for c in range(S.shape[0]):
            u = S[c][None] * x                                     # [L, z, y, x]
            t1 = np.einsum("lzyx,mx->lzym", u, ex, optimize=True)
            t2 = np.einsum("lzym,my->lzm", t1, ey, optimize=True)
            k = np.einsum("lzm,mz->lm", t2, ez, optimize=True)     # [L, M]
            k = np.einsum("lpm,pm->lm", Bm, k)                     # v <- v B
            r1 = np.einsum("lm,mz->lzm", k, ez.conj(), optimize=True)
            r2 = np.einsum("lzm,my->lzym", r1, ey.conj(), optimize=True)
            im = np.einsum("lzym,mx->lzyx", r2, ex.conj(), optimize=True)
            out += np.conj(S[c])[None] * im
        return out
    if traj_type == "2D":
        Ny, Nx = img
        ex = np.exp(-1j * np.outer(pts[0], _centered_freqs(Nx)))
        ey = np.exp(-1j * np.outer(pts[1], _centered_freqs(Ny)))
        Bm = P[:, :, spoke]
        for c in range(S.shape[0]):
            u = S[c][None] * x
            t1 = np.einsum("lyx,mx->lym", u, ex, optimize=True)
            k = np.einsum("lym,my->lm", t1, ey, optimize=True)
            k = np.einsum("lpm,pm->lm", Bm, k)
            r1 = np.einsum("lm,my->lym", k, ey.conj(), optimize=True)
            im = np.einsum("lym,mx->lyx", r1, ex.conj(), optimize=True)
            out += np.conj(S[c])[None] * im
        return out
    # stack
    Nz, Ny, Nx = img
    ex = np.exp(-1j * np.outer(pts[0], _centered_freqs(Nx)))
    ey = np.exp(-1j * np.outer(pts[1], _centered_freqs(Ny)))
    zmod = np.exp(1j * TWO_PI * (Nz // 2) * np.arange(Nz) / Nz)[:, None, None]
    Bm = P[:, :, :, spoke]                                         # [l, p, z, M]
    for c in range(S.shape[0]):
        se = S[c] * zmod
        u = np.fft.fft(se[None] * x, axis=1)                       # [L, kz, y, x]
        t1 = np.einsum("lzyx,mx->lzym", u, ex, optimize=True)
        k = np.einsum("lzym,my->lzm", t1, ey, optimize=True)       # [L, kz, M]
        k = np.einsum("lpzm,pzm->lzm", Bm, k)
        r1 = np.einsum("lzm,my->lzym", k, ey.conj(), optimize=True)
        im = np.einsum("lzym,mx->lzyx", r1, ex.conj(), optimize=True)
        im = np.fft.ifft(im, axis=1, norm="forward")
        out += np.conj(se)[None] * im
    return out


# --------------------------------------------------------------------------
# Automatic mask (mr_calc_mask.cu), bit-exact
# --------------------------------------------------------------------------

def calc_mask(traj_type: str, phi2_dim, traj: np.ndarray, radius: int) -> np.ndarray:
    """Sorted centered linear indices kept by the neighborhood mask.

    Marks ``rint(k * float(M / 2pi)) + M/2 (mod M)`` per transformed axis in
    float32 (``mr_calc_mask.cu:63-90``), dilates by a ``(2r+1)^d`` periodic
    box (``:107-130``), compacts in ascending order, and for a stack repeats
    the in-plane set over every kz plane (``:144-152, 370-385``).
    """
    tr = np.asarray(traj, dtype=np.float32)
    three = traj_type == "3D"
    m = [int(phi2_dim[0]), int(phi2_dim[1]), int(phi2_dim[2]) if three else 1]
    nd = 3 if three else 2
    n_s = tr.shape[1] * tr.shape[2]
    grid = np.zeros((m[2], m[1], m[0]), dtype=bool)
    coords = []
    for a in range(nd):
        sc = np.float32(m[a] / TWO_PI)
        v = tr[a].reshape(-1).astype(np.float32) * sc          # float32 product
        i = np.rint(v).astype(np.int64) + m[a] // 2
        coords.append(np.mod(i, m[a]))
    if not three:
        coords.append(np.zeros(n_s, dtype=np.int64))
    grid[coords[2], coords[1], coords[0]] = True
    r = int(radius)
    if r > 0:
        for ax_c, ax in ((0, 2), (1, 1), (2, 0)):
            if m[ax_c] <= 1:
                continue
            acc = grid.copy()
            for d in range(-r, r + 1):
                acc |= np.roll(grid, d, axis=ax)
            grid = acc
    idx = np.flatnonzero(grid.reshape(-1))
    if traj_type == "stack":
        Mz = int(phi2_dim[2])
        plane = m[0] * m[1]
        idx = (idx[None, :] + plane * np.arange(Mz)[:, None]).reshape(-1)
    return idx.astype(np.int64)


# --------------------------------------------------------------------------
# Error metric
# --------------------------------------------------------------------------

def rel_l2(a, b) -> float:
    """``||a - b|| / ||b||`` in double precision (``tests/check_op.py:96-104``)."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb else 1.0)


# --------------------------------------------------------------------------
# Conjugate gradients (no reference counterpart: the reference stops at the
# operator; this is the FP64 oracle of the device solver)
# --------------------------------------------------------------------------

def cg(apply, b: np.ndarray, n_iter: int, lam: float = 0.0, x0=None):
    """FP64 conjugate gradients for ``(A^H A + lam I) x = b`` (Hestenes &
    Stiefel 1952), step for step what the device solver computes:
    ``q = apply(p) + lam p; alpha = |r|^2 / Re<p, q>`` (0 if not positive);
    ``x += alpha p; r -= alpha q; beta = |r_new|^2 / |r|^2; p = r + beta p``.
    ``apply`` maps a complex128 array to ``A^H A`` of it. Returns ``x`` and
    ``|r_k|^2`` for ``k = 0 .. n_iter``."""
    b = np.asarray(b, dtype=np.complex128)
    if x0 is None:
        x = np.zeros_like(b)
        r = b.copy()
    else:
        x = np.array(x0, dtype=np.complex128)
        r = b - apply(x) - lam * x
    p = r.copy()
    rr = float(np.vdot(r, r).real)
    hist = [rr]
    for _ in range(n_iter):
        q = apply(p) + lam * p
        pq = float(np.vdot(p, q).real)
        alpha = rr / pq if pq > 0 else 0.0
        x += alpha * p
        r -= alpha * q
        rr_new = float(np.vdot(r, r).real)
        beta = rr_new / rr if rr > 0 else 0.0
        rr = rr_new
        hist.append(rr)
        p = r + beta * p
    return x, np.array(hist)


def dequantized_kernel(K: np.ndarray, fmt: str) -> np.ndarray:
    """The complex64 values a 16-bit-stored kernel represents (no reference
    counterpart; the library's storage formats): per location q (last axes
    flattened; axis 0 is the packed component t), ``m = max |re|, |im|``;
    int16: ``scale = m / 32767``, ``code = rint(v / scale)`` (float32
    arithmetic, ties to even, clamped to +-32767), value ``code * scale``;
    bf16: ``scale = m``, value ``bf16(v / scale) * scale``. ``m = 0`` gives
    scale 1. Used as the kernel of the FP64 oracle of a 16-bit operator."""
    K = np.asarray(K, dtype=np.complex64)
    shape = K.shape
    K2 = K.reshape(shape[0], -1)
    re = K2.real.astype(np.float32)
    im = K2.imag.astype(np.float32)
    m = np.maximum(np.abs(re), np.abs(im)).max(axis=0).astype(np.float32)
    if fmt == "int16":
        sc = np.where(m > 0, m / np.float32(32767.0), np.float32(1.0)).astype(np.float32)
        inv = (np.float32(1.0) / sc).astype(np.float32)

        def q(v):
            c = np.clip((v * inv).astype(np.float32), -32767.0, 32767.0)
            return (np.rint(c).astype(np.int16).astype(np.float32) * sc).astype(np.float32)
    elif fmt == "bf16":
        sc = np.where(m > 0, m, np.float32(1.0)).astype(np.float32)
        inv = (np.float32(1.0) / sc).astype(np.float32)

        def q(v):
            u = (v * inv).astype(np.float32).view(np.uint32).astype(np.uint64)
            # round to nearest even on the upper 16 bits (finite inputs)
            u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
            return (u.astype(np.uint32).view(np.float32) * sc).astype(np.float32)
    else:
        raise ValueError(f"unknown 16-bit format {fmt!r}")
    out = (q(re) + 1j * q(im)).astype(np.complex64)
    return out.reshape(shape)
