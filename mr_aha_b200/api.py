"""Array-level interface of the library: the functions, argument meanings,
shapes and exceptions of the reference's Python binding
(``python/mr_aha/api.py``: ``make_config`` ``:211-324``, ``calc_mask``
``:393-447``, ``calc_toep`` ``:556-639``, ``aha_toeplitz`` ``:642-701``,
``AhAOp`` / ``create_op`` ``:745-1255``), implemented over this package's C
ABI.

Arrays live on the GPU: a CUDA ``torch.Tensor``, or any object exposing
``__cuda_array_interface__``. Every array is C-contiguous; data arrays are
``complex64``, ``traj`` is ``float32`` and ``mask`` ``int64``. Axis order is
row-major, so each shape reads right to left against the C header's
column-major one: an image ``x`` is ``(L, Nz, Ny, Nx)``, coil maps ``SEs``
``(C, Nz, Ny, Nx)``, the kernel ``phi2_toep`` ``(ntri, Mz, My, Mx)`` (or
``(ntri, num_masked)``), Gram blocks ``phi2`` ``(L, L, Nkz, Ntrajs)`` for a
stack (``(L, L, Ntrajs)`` otherwise) and the trajectory ``traj``
``(ndim, Nkx, Ntrajs)``; 2-D configurations drop the z axis.

Every size is checked against the C library's own size helpers
(``mr_x_size``, ``mr_se_size``, ``mr_phi2_toep_size``) by one routine,
:func:`_validate`, before any pointer crosses the ABI. Gram blocks act on the
rank row vector from the right (``v <- v B``), the reference's convention.
"""

from __future__ import annotations

import ctypes
import numbers
from typing import Optional, Sequence

from ._lib import (
    DEFAULT_MASK_RADIUS,
    KERNEL_FORMATS,
    OP_ALL_DEVICES,
    OP_SHARE_PRIMARY,
    OP_TOEP_SOURCES,
    MRConfig,
    MRError,
    MROpInfo,
    MROpInputs,
    MROpOptions,
    OpMethod,
    ToepDist,
    TrajType,
    Triangulation,
    backend,
    check,
    lib,
)

__all__ = [
    "DEFAULT_MASK_RADIUS", "MRConfig", "MRError", "TrajType", "Triangulation",
    "make_config", "num_tri", "phi2_toep_shape", "calc_mask", "calc_toep",
    "calc_toep_from_psf", "aha_toeplitz", "AhAPlan", "AhAOp", "create_op",
]

_DTYPES = {"complex64": 8, "float32": 4, "int64": 8}


def _torch():
    import torch  # noqa: PLC0415
    return torch


def _is_torch(a) -> bool:
    t = type(a)
    return t.__module__.startswith("torch") and hasattr(a, "data_ptr")


def _ptr(array, name: str, dtype: str, allow_none: bool = False):
    """Validate a device array and return its device pointer.

    Raises ``TypeError`` for host arrays or a wrong dtype and ``ValueError``
    for non-contiguous arrays, like the reference's ``_ptr`` (``api.py:155-209``).
    """
    if array is None:
        if allow_none:
            return None
        raise TypeError(f"{name} must not be None")
    if _is_torch(array):
        torch = _torch()
        want = {"complex64": torch.complex64, "float32": torch.float32,
                "int64": torch.int64}[dtype]
        if not array.is_cuda:
            raise TypeError(f"{name} must be a CUDA tensor for the {backend()} backend, "
                            f"got a tensor on {array.device}")
        if array.dtype != want:
            raise TypeError(f"{name} must have dtype {want}, got {array.dtype}")
        if not array.is_contiguous():
            raise ValueError(f"{name} must be C-contiguous; call .contiguous() first")
        return int(array.data_ptr()) or None
    cai = getattr(array, "__cuda_array_interface__", None)
    if cai is None:
        raise TypeError(f"{name} must be a CUDA device array (torch.Tensor on a CUDA device "
                        f"or __cuda_array_interface__), got {type(array).__name__}")
    import numpy as np  # noqa: PLC0415
    if np.dtype(cai["typestr"]) != np.dtype(dtype):
        raise TypeError(f"{name} must have dtype {dtype}, got {np.dtype(cai['typestr'])}")
    strides = cai.get("strides")
    if strides is not None:
        exp, acc = [], np.dtype(dtype).itemsize
        for n in reversed(cai["shape"]):
            exp.append(acc)
            acc *= n
        if tuple(reversed(exp)) != tuple(strides):
            raise ValueError(f"{name} must be C-contiguous")
    return int(cai["data"][0]) or None


def _size(array) -> int:
    if _is_torch(array):
        return int(array.numel())
    cai = getattr(array, "__cuda_array_interface__", None)
    if cai is None:
        return int(getattr(array, "size", 0))
    n = 1
    for s in cai["shape"]:
        n *= int(s)
    return n


def _shape(array) -> tuple:
    if _is_torch(array):
        return tuple(array.shape)
    return tuple(array.__cuda_array_interface__["shape"])


def _check_size(array, expected: int, name: str) -> None:
    if _size(array) != expected:
        raise ValueError(
            f"{name} has {_size(array)} elements but {expected} were expected "
            f"(remember that Python shapes are the reverse of the column-major shapes "
            f"in the documentation)")


def _device_of(*arrays):
    for a in arrays:
        if a is not None and _is_torch(a):
            return a.device
    torch = _torch()
    return torch.device("cuda", torch.cuda.current_device())


def _empty(shape, dtype: str, device):
    torch = _torch()
    td = {"complex64": torch.complex64, "int64": torch.int64, "float32": torch.float32}[dtype]
    return torch.empty(tuple(shape), dtype=td, device=device)


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream or None
    for attr in ("cuda_stream", "ptr"):
        v = getattr(stream, attr, None)
        if v is not None:
            return int(v) or None
    raise TypeError("stream must be None, an int handle, a torch.cuda.Stream or expose .ptr")


def _grid_dims(traj_type: int, n_dim, phi2_dim) -> tuple:
    """Column-major image and grid extents of a configuration. The grid
    defaults to twice the image along every transformed axis; a stack keeps
    its z extent (its kz axis is not oversampled)."""
    n_spatial = 2 if traj_type == TrajType.TWO_D else 3
    n = tuple(int(v) for v in n_dim)
    if len(n) != n_spatial:
        raise ValueError(f"n_dim must have {n_spatial} entries for this trajectory type, "
                         f"got {len(n)}")
    if phi2_dim is None:
        m = tuple(v if (traj_type == TrajType.STACK and ax == 2) else 2 * v
                  for ax, v in enumerate(n))
    else:
        m = tuple(int(v) for v in phi2_dim)
    if len(m) != n_spatial:
        raise ValueError(f"phi2_dim must have {n_spatial} entries, got {len(m)}")
    return n, m


def make_config(traj_type, n_dim: Sequence[int], L: int, *,
                phi2_dim: Optional[Sequence[int]] = None, triangulation="lower",
                is_masked: bool = False, num_masked: int = 0, n_coils: int = 1,
                eps: float = 1e-6, gpu_device_id: int = -1, stream=None,
                mem_fraction: float = 0.5, verbose: bool = False,
                mask_radius: int = DEFAULT_MASK_RADIUS) -> MRConfig:
    """A validated :class:`MRConfig` (the reference's ``make_config``).

    ``n_dim`` / ``phi2_dim`` are column-major ``(Nx, Ny[, Nz])``. A masked
    configuration may leave ``num_masked`` at 0: the count is taken from the
    mask when the configuration is first used with one.
    """
    tt = TrajType.parse(traj_type)
    n, m = _grid_dims(tt, n_dim, phi2_dim)
    cfg = MRConfig()
    check(lib.mr_config_defaults(ctypes.byref(cfg), tt), "mr_config_defaults")
    cfg.n_dim[:len(n)] = n
    cfg.phi2_dim[:len(m)] = m
    scalars = dict(L=int(L), triangulation=Triangulation.parse(triangulation),
                   is_masked=int(bool(is_masked)), num_masked=int(num_masked),
                   n_coils=int(n_coils), eps=float(eps), gpu_device_id=int(gpu_device_id),
                   mem_fraction=float(mem_fraction), verbose=int(bool(verbose)),
                   mask_radius=int(mask_radius), stream=_stream_ptr(stream))
    for field, value in scalars.items():
        setattr(cfg, field, value)
    # validate with a stand-in count of one masked location when the count
    # is still open; the real count is checked once a mask is supplied
    trial = MRConfig.from_buffer_copy(cfg)
    if trial.is_masked and trial.num_masked == 0:
        trial.num_masked = 1
    check(lib.mr_config_validate(ctypes.byref(trial)), "mr_config_validate")
    return cfg


def num_tri(L: int) -> int:
    return int(lib.mr_num_tri(int(L)))


def phi2_toep_shape(cfg: MRConfig) -> tuple:
    """Row-major shape of ``phi2_toep``: ``(ntri, num_masked)`` or ``(ntri, [Mz,] My, Mx)``."""
    ntri = num_tri(cfg.L)
    if cfg.is_masked:
        return (ntri, int(cfg.num_masked))
    dims = [cfg.phi2_dim[i] for i in range(cfg.n_spatial)]
    return tuple([ntri] + list(reversed(dims)))


def _image_shape(cfg: MRConfig) -> tuple:
    return tuple(reversed([cfg.n_dim[i] for i in range(cfg.n_spatial)]))


def _check_traj(cfg: MRConfig, traj):
    """``(Ntrajs, Nkx)`` of a trajectory shaped ``(ndim, Nkx, Ntrajs)``."""
    ndim_traj = 3 if cfg.traj_type == TrajType.THREE_D else 2
    shape = _shape(traj)
    if len(shape) != 3 or shape[0] != ndim_traj:
        raise ValueError(f"traj must be shaped (ndim, Nkx, Ntrajs) with ndim = {ndim_traj}, "
                         f"got {shape}")
    return int(shape[2]), int(shape[1])


def _gram_size(cfg: MRConfig, n_traj: int) -> int:
    """Elements of ``phi2``: one ``L x L`` block per readout (and per kz
    plane of a stack)."""
    n_kz = cfg.phi2_dim[2] if cfg.traj_type == TrajType.STACK else 1
    return cfg.L * cfg.L * n_kz * n_traj


_SIZE_OF = {"x": "mr_x_size", "out": "mr_x_size", "SEs": "mr_se_size",
            "phi2_toep": "mr_phi2_toep_size"}


def _validate(cfg: MRConfig, need_mask: bool = True, **arrays) -> tuple:
    """Check the arrays of one call against the configuration's contract.

    Image-, map- and kernel-sized arrays (``x``, ``out``, ``SEs``,
    ``phi2_toep``) must hold exactly the element count the C library's size
    helper gives for ``cfg``; ``phi2`` must match ``traj``'s readouts. A
    masked configuration needs a mask (when ``need_mask``) whose length is
    ``cfg.num_masked``, or sets that count when the configuration left it at
    0 (then ``cfg`` is validated again). Arrays passed as None are skipped.
    Returns ``(Ntrajs, Nkx)`` of ``traj`` (``(0, 0)`` without one). Raises
    ``ValueError`` for a size or mask mismatch."""
    traj = arrays.pop("traj", None)
    phi2 = arrays.pop("phi2", None)
    mask = arrays.pop("mask", None)
    n_traj, n_kx = _check_traj(cfg, traj) if traj is not None else (0, 0)
    if phi2 is not None:
        _check_size(phi2, _gram_size(cfg, n_traj), "phi2")
    if cfg.is_masked and (mask is not None or need_mask):
        if mask is None:
            raise ValueError("cfg.is_masked is set, so a mask is required")
        n_masked = _size(mask)
        if cfg.num_masked == 0:
            cfg.num_masked = n_masked
            check(lib.mr_config_validate(ctypes.byref(cfg)), "mr_config_validate")
        elif n_masked != int(cfg.num_masked):
            raise ValueError(f"mask has {n_masked} elements but cfg.num_masked is "
                             f"{cfg.num_masked}")
    for name, array in arrays.items():
        if array is not None:
            helper = getattr(lib, _SIZE_OF[name.lstrip("_")])
            _check_size(array, int(helper(ctypes.byref(cfg))), name)
    return n_traj, n_kx


def calc_mask(cfg: MRConfig, traj, *, radius: Optional[int] = None):
    """Neighbourhood mask from the trajectory (reference ``api.py:393-447``)."""
    Ntrajs, Nkx = _check_traj(cfg, traj)
    c = MRConfig.from_buffer_copy(cfg)
    if radius is not None:
        c.mask_radius = int(radius)
    dev = _device_of(traj)
    buf = _empty((int(lib.mr_pad_size(ctypes.byref(c))),), "int64", dev)
    n = ctypes.c_int64(0)
    check(lib.mr_calc_mask(ctypes.byref(c), _ptr(traj, "traj", "float32"), ctypes.c_int64(Ntrajs),
                           ctypes.c_int64(Nkx), _ptr(buf, "mask", "int64"), ctypes.byref(n)),
          "mr_calc_mask")
    mask = buf[: n.value].clone()
    del buf
    return mask


def calc_toep(cfg: MRConfig, phi2, traj, mask=None, out=None, nufft: Optional[str] = None):
    """The Toeplitz kernel ``phi2_toep`` of the Gram blocks ``phi2`` sampled
    at ``traj`` (the reference's ``calc_toep``), built on the GPU.

    ``nufft`` exists for signature compatibility: the library's own build is
    the only one (``None`` or ``'library'``).
    """
    if nufft not in (None, "library"):
        raise ValueError(f"nufft={nufft!r}: only the library build is available")
    n_traj, n_kx = _validate(cfg, traj=traj, phi2=phi2, mask=mask)
    if out is None:
        out = _empty(phi2_toep_shape(cfg), "complex64", _device_of(phi2, traj))
    _validate(cfg, need_mask=False, phi2_toep=out)
    check(lib.mr_calc_toep(ctypes.byref(cfg), _ptr(phi2, "phi2", "complex64"),
                           _ptr(traj, "traj", "float32"), ctypes.c_int64(n_traj),
                           ctypes.c_int64(n_kx), _ptr(mask, "mask", "int64", allow_none=True),
                           _ptr(out, "out", "complex64")), "mr_calc_toep")
    return out


def calc_toep_from_psf(cfg: MRConfig, psf, t0: int, out, mask=None):
    """Finish components ``[t0, t0 + n)`` of ``out`` from centred PSFs
    ``psf[n, Mz, My, Mx]`` (reference ``mr_calc_toep_from_psf``)."""
    vol = 1
    for i in range(3):
        vol *= cfg.phi2_dim[i]
    n = _size(psf) // vol
    check(lib.mr_calc_toep_from_psf(ctypes.byref(cfg), _ptr(psf, "psf", "complex64"),
                                    ctypes.c_int64(int(t0)), ctypes.c_int64(n),
                                    _ptr(mask, "mask", "int64", allow_none=True),
                                    _ptr(out, "out", "complex64")), "mr_calc_toep_from_psf")
    return out


def _host_ptr(array, name: str, expected: int) -> int:
    """Address of a complex64, C-contiguous host array (numpy, or a CPU torch
    tensor) of ``expected`` elements."""
    import numpy as np  # noqa: PLC0415

    if _is_torch(array):
        torch = _torch()
        if array.is_cuda:
            raise TypeError(f"{name} must be in host memory, got a tensor on {array.device}")
        if array.dtype != torch.complex64:
            raise TypeError(f"{name} must have dtype complex64, got {array.dtype}")
        if not array.is_contiguous():
            raise ValueError(f"{name} must be C-contiguous; call .contiguous() first")
        n, ptr = int(array.numel()), int(array.data_ptr())
    elif isinstance(array, np.ndarray):
        if array.dtype != np.complex64:
            raise TypeError(f"{name} must have dtype complex64, got {array.dtype}")
        if not array.flags["C_CONTIGUOUS"]:
            raise ValueError(f"{name} must be C-contiguous")
        if not array.flags["WRITEABLE"] and name == "out":
            raise ValueError("out must be writeable")
        n, ptr = int(array.size), int(array.ctypes.data)
    else:
        raise TypeError(f"{name} must be a numpy array or a CPU torch tensor, "
                        f"got {type(array).__name__}")
    if n != expected:
        raise ValueError(f"{name} has {n} elements but {expected} were expected")
    return ptr


def _host_empty_like(x):
    import numpy as np  # noqa: PLC0415

    if _is_torch(x):
        return _torch().empty(tuple(x.shape), dtype=x.dtype, pin_memory=x.is_pinned())
    return np.empty(x.shape, dtype=np.complex64)


def pinned_empty(shape):
    """A page-locked complex64 host array (a numpy view of a pinned CPU torch
    tensor; the array's base keeps the tensor alive): host buffers that let
    :meth:`AhAOp.apply_host` overlap its copies with applies."""
    return _torch().empty(tuple(shape), dtype=_torch().complex64, pin_memory=True).numpy()


def _out_like(x, out):
    """``out``, or a new complex64 array shaped like ``x`` on its device."""
    return _empty(_shape(x), "complex64", _device_of(x)) if out is None else out


def aha_toeplitz(cfg: MRConfig, x, SEs, phi2_toep, mask=None, out=None):
    """``A^H A x`` in one call from a ready kernel (the reference's
    ``aha_toeplitz``): a plan is made, applied once and released."""
    _validate(cfg, x=x, SEs=SEs, phi2_toep=phi2_toep, mask=mask, out=out)
    ptrs = (_ptr(x, "x", "complex64"), _ptr(SEs, "SEs", "complex64"),
            _ptr(phi2_toep, "phi2_toep", "complex64"),
            _ptr(mask, "mask", "int64", allow_none=True))
    out = _out_like(x, out)
    check(lib.mr_aha_toeplitz(ctypes.byref(cfg), *ptrs, _ptr(out, "out", "complex64")),
          "mr_aha_toeplitz")
    return out


class AhAPlan:
    """Reusable stateless plan (``mr_aha_plan_create/execute/destroy``)."""

    def __init__(self, cfg: MRConfig):
        self._cfg = MRConfig.from_buffer_copy(cfg)
        self._h = ctypes.c_void_p()
        check(lib.mr_aha_plan_create(ctypes.byref(self._cfg), ctypes.byref(self._h)),
              "mr_aha_plan_create")

    def execute(self, x, SEs, phi2_toep, mask=None, out=None):
        if not self._h:
            raise RuntimeError("this AhAPlan has already been closed")
        _validate(self._cfg, x=x, SEs=SEs, phi2_toep=phi2_toep, mask=mask, out=out)
        ptrs = (_ptr(x, "x", "complex64"), _ptr(SEs, "SEs", "complex64"),
                _ptr(phi2_toep, "phi2_toep", "complex64"),
                _ptr(mask, "mask", "int64", allow_none=True))
        out = _out_like(x, out)
        check(lib.mr_aha_plan_execute(self._h, *ptrs, _ptr(out, "out", "complex64")),
              "mr_aha_plan_execute")
        return out

    __call__ = execute

    def close(self):
        if self._h:
            lib.mr_aha_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass


def _devices_arg(devices):
    if devices is None:
        return None, 0
    if isinstance(devices, str):
        if devices.lower() != "all":
            raise ValueError(f"devices must be None, 'all', an int or a list; got {devices!r}")
        return None, OP_ALL_DEVICES
    if isinstance(devices, numbers.Integral):
        devices = [devices]
    devices = [int(d) for d in devices]
    if not devices:
        return None, 0
    return (ctypes.c_int * len(devices))(*devices), len(devices)


_NUFFT_OPTS = ("upsampfac", "gpu_method")


def _op_options(kind: int, cfg: MRConfig, devices, toep_dist, share_primary: bool,
                nufft_opts) -> tuple:
    """``mr_op_options`` of a create call, and the device list array it
    points to (kept alive by the caller until ``mr_op_create`` returns).
    NUFFT settings belong to ``method='nufft'`` only, which has no kernel and
    so no mask."""
    extra = dict(nufft_opts or {})
    if kind == OpMethod.NUFFT:
        if cfg.is_masked:
            raise ValueError("method='nufft' has no kernel to mask; build the configuration "
                             "with is_masked=False")
        unknown = sorted(set(extra) - set(_NUFFT_OPTS))
        if unknown:
            raise ValueError(f"unknown nufft_opts {unknown}; accepted: {list(_NUFFT_OPTS)}")
    elif extra:
        raise ValueError("nufft_opts is only used with method='nufft'")
    dev_array, n_dev = _devices_arg(devices)
    opt = MROpOptions()
    check(lib.mr_op_options_defaults(ctypes.byref(opt)), "mr_op_options_defaults")
    opt.method = kind
    opt.devices = ctypes.cast(dev_array, ctypes.POINTER(ctypes.c_int)) if dev_array else None
    opt.n_devices = n_dev
    opt.toep_dist = ToepDist.parse(toep_dist)
    opt.flags = OP_SHARE_PRIMARY if share_primary else 0
    opt.nufft_upsampfac = float(extra.get("upsampfac", 0.0))
    opt.nufft_gpu_method = int(extra.get("gpu_method", 0))
    return opt, dev_array


class AhAOp:
    """The ``A^H A`` operator (the reference's ``AhAOp``).

    ``op = create_op(cfg, SEs, phi2, traj)`` builds the Toeplitz kernel on the
    GPU and a plan; ``op(x)`` applies it on ``cfg.stream``. One GPU:
    ``devices`` other than the primary are accepted and served by the
    primary alone.
    """

    def __init__(self, *args, **kwargs):
        raise TypeError("AhAOp is created with mr_aha_b200.create_op(cfg, SEs, phi2, traj, ...) "
                        "(or AhAOp.create_op), not by calling the class")

    @classmethod
    def create_op(cls, cfg: MRConfig, SEs, phi2, traj, mask=None, *, method: str = "toeplitz",
                  devices=None, toep_dist: str = "auto", share_primary: bool = True,
                  nufft_opts: Optional[dict] = None, _phi2_toep=None,
                  kernel_format: str = "complex64", keep_complex64: bool = True) -> "AhAOp":
        """Create the operator (``mr_op_create``).

        The operator is built from the Gram blocks ``phi2`` at ``traj``, or,
        for ``method='toeplitz'`` with ``phi2`` and ``traj`` both None, from a
        ready kernel ``_phi2_toep``. ``kernel_format`` (``'complex64'``,
        ``'bf16'`` or ``'int16'``) selects the storage of the kernel read by
        every apply (no reference counterpart; ``mr_b200_op_set_kernel_format``).
        """
        kind = OpMethod.parse(method)
        opt, dev_array = _op_options(kind, cfg, devices, toep_dist, share_primary, nufft_opts)
        if _phi2_toep is not None and kind == OpMethod.NUFFT:
            raise ValueError("_phi2_toep is only used with method='toeplitz'")
        from_kernel = _phi2_toep is not None and phi2 is None and traj is None
        if not from_kernel and (phi2 is None or traj is None):
            raise ValueError("phi2 and traj are required (the operator is built from the "
                             "Gram blocks)")
        n_traj, n_kx = _validate(cfg, SEs=SEs, phi2=phi2, traj=traj, mask=mask,
                                 _phi2_toep=_phi2_toep)
        inputs = MROpInputs(
            d_SEs=_ptr(SEs, "SEs", "complex64"),
            d_phi2=_ptr(phi2, "phi2", "complex64", allow_none=from_kernel),
            d_traj=_ptr(traj, "traj", "float32", allow_none=from_kernel),
            Ntrajs=n_traj, Nkx=n_kx,
            d_mask=_ptr(mask, "mask", "int64", allow_none=True),
            d_phi2_toep=_ptr(_phi2_toep, "_phi2_toep", "complex64", allow_none=True))
        self = cls.__new__(cls)
        self._handle = ctypes.c_void_p()
        self._method = OpMethod._TO_STR[kind]
        self._cfg = MRConfig.from_buffer_copy(cfg)
        self._device = _device_of(SEs)
        # arrays the library may keep using in place (MR_OP_SHARE_PRIMARY)
        self._keep = (SEs, mask, _phi2_toep) if share_primary else ()
        self._host_pending = []
        check(lib.mr_op_create(ctypes.byref(cfg), ctypes.byref(inputs), ctypes.byref(opt),
                               ctypes.byref(self._handle)), "mr_op_create")
        del dev_array
        if kernel_format != "complex64":
            self.set_kernel_format(kernel_format, keep_complex64=keep_complex64)
        return self

    @property
    def config(self) -> MRConfig:
        return self._cfg

    @property
    def method(self) -> str:
        return self._method

    def _check_open(self):
        if not self._handle:
            raise RuntimeError("this AhAOp has already been closed")

    def apply(self, x, out=None):
        """``A^H A x`` (``mr_op_execute``), ordered on ``cfg.stream``."""
        self._check_open()
        _validate(self._cfg, need_mask=False, x=x, out=out)
        px = _ptr(x, "x", "complex64")
        out = _out_like(x, out)
        check(lib.mr_op_execute(self._handle, px, _ptr(out, "out", "complex64")),
              "mr_op_execute")
        return out

    __call__ = apply

    def set_kernel_format(self, fmt: str, keep_complex64: bool = True) -> None:
        """Store the kernel as ``'complex64'``, ``'bf16'`` or ``'int16'`` (+ scale)."""
        self._check_open()
        if fmt not in KERNEL_FORMATS:
            raise ValueError(f"kernel format must be one of {sorted(KERNEL_FORMATS)}")
        check(lib.mr_b200_op_set_kernel_format(self._handle, KERNEL_FORMATS[fmt],
                                               1 if keep_complex64 else 0),
              "mr_b200_op_set_kernel_format")
        if not keep_complex64 and fmt != "complex64" and len(self._keep) == 3:
            # a borrowed complex64 kernel is no longer referenced by the library
            self._keep = (self._keep[0], self._keep[1], None)

    @property
    def kernel_format(self) -> str:
        self._check_open()
        f = ctypes.c_int(0)
        check(lib.mr_b200_op_kernel_format(self._handle, ctypes.byref(f)),
              "mr_b200_op_kernel_format")
        return {v: k for k, v in KERNEL_FORMATS.items()}[f.value]

    def _kernel16_shapes(self):
        ntri = int(lib.mr_num_tri(int(self._cfg.L)))
        nloc = int(lib.mr_phi2_toep_size(ctypes.byref(self._cfg))) // ntri
        return (ntri, nloc, 2), (nloc,)

    def save_kernel16(self):
        """Checkpoint of the 16-bit kernel (``mr_b200_op_save_kernel16``):
        ``(fmt, codes, scale)`` with ``codes`` a new ``(ntri, nloc, 2)``
        tensor (int16, or bfloat16 for ``'bf16'``) of (re, im) codes and
        ``scale`` ``(nloc,)`` float32; value = scale * code per location."""
        self._check_open()
        torch = _torch()
        cshape, sshape = self._kernel16_shapes()
        fmt = self.kernel_format
        if fmt == "complex64":
            raise MRError(-1, "the operator's kernel is complex64; set a 16-bit format first")
        codes = torch.empty(cshape, dtype=torch.int16 if fmt == "int16" else torch.bfloat16,
                            device=self._device)
        scale = torch.empty(sshape, dtype=torch.float32, device=self._device)
        f = ctypes.c_int(0)
        check(lib.mr_b200_op_save_kernel16(self._handle, ctypes.byref(f), codes.data_ptr(),
                                           scale.data_ptr()), "mr_b200_op_save_kernel16")
        return fmt, codes, scale

    def load_kernel16(self, fmt: str, codes, scale) -> None:
        """Restore a 16-bit kernel saved by :meth:`save_kernel16`
        (``mr_b200_op_load_kernel16``); the operator then applies in ``fmt``
        only (its complex64 kernel is released)."""
        self._check_open()
        if fmt not in ("int16", "bf16"):
            raise ValueError("fmt must be 'int16' or 'bf16'")
        torch = _torch()
        cshape, sshape = self._kernel16_shapes()
        want = torch.int16 if fmt == "int16" else torch.bfloat16
        for name, t, shp, dt in (("codes", codes, cshape, want),
                                 ("scale", scale, sshape, torch.float32)):
            if not _is_torch(t) or not t.is_cuda or t.dtype != dt or not t.is_contiguous():
                raise TypeError(f"{name} must be a contiguous CUDA tensor of dtype {dt}")
            if tuple(t.shape) != shp:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {shp}")
        check(lib.mr_b200_op_load_kernel16(self._handle, KERNEL_FORMATS[fmt], codes.data_ptr(),
                                           scale.data_ptr()), "mr_b200_op_load_kernel16")
        if len(self._keep) == 3:
            self._keep = (self._keep[0], self._keep[1], None)

    def autotune(self, reps: int = 2) -> float:
        """Pick the fastest kernel of every pass by timing full applies
        (``mr_b200_op_autotune``); returns the tuned apply time in ms."""
        self._check_open()
        ms = ctypes.c_float(0.0)
        check(lib.mr_b200_op_autotune(self._handle, int(reps), ctypes.byref(ms)),
              "mr_b200_op_autotune")
        return float(ms.value)

    def blocked_copy(self, enable: bool) -> bool:
        """Free (False) or build (True, if it fits) the blocked copy of the
        operator's kernel in its current format (complex64, or the 16-bit
        codes for rank <= 16) read by pass 3 (``mr_b200_op_blocked_copy``);
        returns whether a copy exists."""
        self._check_open()
        built = ctypes.c_int(0)
        check(lib.mr_b200_op_blocked_copy(self._handle, 1 if enable else 0, ctypes.byref(built)),
              "mr_b200_op_blocked_copy")
        return bool(built.value)

    @property
    def device_bytes(self) -> int:
        """Device memory held by the operator (``mr_b200_op_device_bytes``)."""
        self._check_open()
        b = ctypes.c_uint64(0)
        check(lib.mr_b200_op_device_bytes(self._handle, ctypes.byref(b)),
              "mr_b200_op_device_bytes")
        return int(b.value)

    @property
    def device_status(self) -> int:
        """Status word of the operator's kernels since the last read (0 = no
        device-side error; ``mr_b200_op_device_status``). Synchronous."""
        self._check_open()
        st = ctypes.c_int(0)
        check(lib.mr_b200_op_device_status(self._handle, ctypes.byref(st)),
              "mr_b200_op_device_status")
        return int(st.value)

    def apply_host(self, x, out=None):
        """``A^H A x`` from and to HOST memory (``mr_b200_op_execute_host``):
        ``x`` and ``out`` are complex64, C-contiguous numpy arrays or CPU
        torch tensors of the image's size (``out`` is allocated like ``x``
        when None). Asynchronous and pipelined: the copies of consecutive
        calls overlap the applies around them when both buffers are
        page-locked (``pinned_empty``). The result is in ``out`` after
        :meth:`host_sync`; until then neither buffer may change."""
        self._check_open()
        m = int(lib.mr_x_size(ctypes.byref(self._cfg)))
        if out is None:
            out = _host_empty_like(x)
        px = _host_ptr(x, "x", m)
        po = _host_ptr(out, "out", m)
        check(lib.mr_b200_op_execute_host(self._handle, px, po), "mr_b200_op_execute_host")
        self._host_pending.append((x, out))
        return out

    def host_sync(self) -> None:
        """Wait for every queued :meth:`apply_host` (``mr_b200_op_host_sync``)."""
        self._check_open()
        check(lib.mr_b200_op_host_sync(self._handle), "mr_b200_op_host_sync")
        self._host_pending.clear()

    def host_release(self) -> None:
        """Wait, then free the device slots of :meth:`apply_host`."""
        self._check_open()
        check(lib.mr_b200_op_host_release(self._handle), "mr_b200_op_host_release")
        self._host_pending.clear()

    @property
    def launches_per_apply(self) -> int:
        self._check_open()
        n = ctypes.c_int(0)
        check(lib.mr_b200_op_launches(self._handle, ctypes.byref(n)), "mr_b200_op_launches")
        return int(n.value)

    def profile(self, x, out=None) -> list:
        """One apply with CUDA events around every kernel on the operator's
        stream: ``[(pass_name, ms), ...]`` in launch order (synchronous)."""
        self._check_open()
        if out is None:
            out = _empty(tuple(x.shape), "complex64", _device_of(x))
        nmax = 64
        ms = (ctypes.c_float * nmax)()
        names = ctypes.create_string_buffer(32 * nmax)
        n = ctypes.c_int(0)
        check(lib.mr_b200_op_profile(self._handle, _ptr(x, "x", "complex64"),
                                     _ptr(out, "out", "complex64"), ms, names, nmax,
                                     ctypes.byref(n)), "mr_b200_op_profile")
        raw = names.raw
        return [(raw[32 * k: 32 * k + 32].split(b"\0")[0].decode(), float(ms[k]))
                for k in range(n.value)]

    def cg(self, b, n_iter: int = 30, lam: float = 0.0, x0=None, out=None,
           graph: bool = True):
        """Solve ``(A^H A + lam I) x = b`` with ``n_iter`` conjugate-gradient
        iterations on the device (``mr_b200_cg_solve``; no reference
        counterpart). Starts from ``x0`` (copied into ``out``) or from zero.
        Returns ``(x, rr)`` with ``rr[k] = |r_k|^2`` (numpy float64,
        ``n_iter + 1`` values). Synchronous."""
        self._check_open()
        n = int(lib.mr_x_size(ctypes.byref(self._cfg)))
        _check_size(b, n, "b")
        pb = _ptr(b, "b", "complex64")
        if out is None:
            out = _empty(_shape(b), "complex64", _device_of(b))
        else:
            _check_size(out, n, "out")
        flags = CG_GRAPH if graph else 0
        if x0 is None:
            flags |= CG_ZERO_X
        else:
            _check_size(x0, n, "x0")
            out[...] = x0
        rr = (ctypes.c_double * (n_iter + 1))()
        check(lib.mr_b200_cg_solve(self._handle, pb, _ptr(out, "out", "complex64"), int(n_iter),
                                   float(lam), flags, rr), "mr_b200_cg_solve")
        import numpy as np

        return out, np.array(rr[:], dtype=np.float64)

    def cg_solver(self, b, x, lam: float = 0.0, max_iters: int = 1000, zero_x: bool = True,
                  graph: bool = True) -> "CGSolver":
        """A step-wise solver on this operator (``mr_b200_cg_create``): ``x``
        is updated in place by ``step(n)``; ``b`` and ``x`` must stay alive
        until ``close()``."""
        self._check_open()
        return CGSolver(self, b, x, lam, max_iters, zero_x, graph)

    @property
    def info(self) -> dict:
        self._check_open()
        inf = MROpInfo()
        check(lib.mr_op_info(self._handle, ctypes.byref(inf)), "mr_op_info")
        n = inf.n_devices
        return dict(
            method=OpMethod._TO_STR.get(int(inf.method), "unknown"),
            devices=list(inf.devices[:n]), coil_begin=list(inf.coil_begin[:n]),
            coil_count=list(inf.coil_count[:n]), group=list(inf.group[:n]),
            n_split_coils=int(inf.n_split_coils), peer_access=bool(inf.peer_access),
            peer_bandwidth_gbs=float(inf.peer_bandwidth_gbs),
            toep_source=OP_TOEP_SOURCES.get(int(inf.toep_source), "unknown"),
            toep_devices=int(inf.toep_devices), toep_ms=float(inf.toep_ms),
            toep_component_ms=float(inf.toep_component_ms),
            toep_gather_gbs=float(inf.toep_gather_gbs), create_ms=float(inf.create_ms),
        )

    def kernel(self, k: int = 0):
        """Read-only view of the operator's complex64 kernel (``mr_op_kernel``)."""
        self._check_open()
        ptr = ctypes.c_void_p()
        check(lib.mr_op_kernel(self._handle, int(k), ctypes.byref(ptr)), "mr_op_kernel")
        shape = phi2_toep_shape(self._cfg)
        size = int(lib.mr_phi2_toep_size(ctypes.byref(self._cfg)))
        torch = _torch()

        class _View:
            def __init__(self, p, n, owner):
                self.__cuda_array_interface__ = {
                    "shape": (n,), "typestr": "<c8", "data": (p, False), "version": 3,
                    "strides": None}
                self._owner = owner

        view = torch.as_tensor(_View(ptr.value, size, self), device=self._device)
        return view.view(shape)

    def close(self) -> None:
        if self._handle:
            lib.mr_op_destroy(self._handle)
            self._handle = ctypes.c_void_p()
        self._keep = ()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass


CG_ZERO_X = 1
CG_GRAPH = 2
BATCH_GRAPH = 1
BATCH_TUNE = 2


class Batch:
    """Apply many independent operators together (``mr_b200_batch_*``; no
    reference counterpart): ``batch(xs)`` returns ``[A_i^H A_i xs[i]]``.
    ``graph=True`` replays one captured CUDA graph per set of array
    pointers; ``tune=True`` autotunes each distinct geometry first."""

    def __init__(self, ops, n_streams: int = 4, graph: bool = True, tune: bool = False):
        self._ops = list(ops)
        if not self._ops:
            raise ValueError("a batch needs at least one operator")
        for o in self._ops:
            o._check_open()
        arr = (ctypes.c_void_p * len(self._ops))(*[o._handle.value for o in self._ops])
        self._handle = ctypes.c_void_p()
        flags = (BATCH_GRAPH if graph else 0) | (BATCH_TUNE if tune else 0)
        check(lib.mr_b200_batch_create(arr, len(self._ops), int(n_streams), flags,
                                       ctypes.byref(self._handle)), "mr_b200_batch_create")

    def __call__(self, xs, outs=None, stream=None):
        if not self._handle:
            raise RuntimeError("this Batch has already been closed")
        n = len(self._ops)
        if len(xs) != n:
            raise ValueError(f"expected {n} inputs, got {len(xs)}")
        if outs is None:
            outs = [_empty(_shape(x), "complex64", _device_of(x)) for x in xs]
        px = (ctypes.c_void_p * n)()
        po = (ctypes.c_void_p * n)()
        for i, (op, x, y) in enumerate(zip(self._ops, xs, outs)):
            m = int(lib.mr_x_size(ctypes.byref(op._cfg)))
            _check_size(x, m, f"xs[{i}]")
            _check_size(y, m, f"outs[{i}]")
            px[i] = _ptr(x, f"xs[{i}]", "complex64")
            po[i] = _ptr(y, f"outs[{i}]", "complex64")
        check(lib.mr_b200_batch_execute(self._handle, px, po, _stream_ptr(stream)),
              "mr_b200_batch_execute")
        return outs

    def close(self) -> None:
        if self._handle:
            lib.mr_b200_batch_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CGSolver:
    """Conjugate gradients kept resident on the device (``mr_b200_cg_*``):
    its vectors, step scalars and residual history stay in device memory
    between ``step`` calls, which return without waiting for the GPU."""

    def __init__(self, op: AhAOp, b, x, lam: float, max_iters: int, zero_x: bool, graph: bool):
        n = int(lib.mr_x_size(ctypes.byref(op._cfg)))
        _check_size(b, n, "b")
        _check_size(x, n, "x")
        self._op = op
        self._keep = (b, x)
        self.x = x
        self.max_iters = int(max_iters)
        self._handle = ctypes.c_void_p()
        flags = (CG_ZERO_X if zero_x else 0) | (CG_GRAPH if graph else 0)
        check(lib.mr_b200_cg_create(op._handle, _ptr(b, "b", "complex64"),
                                    _ptr(x, "x", "complex64"), float(lam), flags,
                                    self.max_iters, ctypes.byref(self._handle)),
              "mr_b200_cg_create")

    def step(self, n: int = 1) -> None:
        if not self._handle:
            raise RuntimeError("this CGSolver has already been closed")
        check(lib.mr_b200_cg_step(self._handle, int(n)), "mr_b200_cg_step")

    @property
    def busy(self) -> bool:
        """True while issued iterations are still running (does not wait)."""
        if not self._handle:
            return False
        v = ctypes.c_int(0)
        check(lib.mr_b200_cg_busy(self._handle, ctypes.byref(v)), "mr_b200_cg_busy")
        return bool(v.value)

    @property
    def iterations(self) -> int:
        """Iterations issued so far."""
        v = ctypes.c_int(0)
        check(lib.mr_b200_cg_iterations(self._handle, ctypes.byref(v)), "mr_b200_cg_iterations")
        return int(v.value)

    def residuals(self):
        """``|r_k|^2`` for the iterations done so far (waits for the GPU)."""
        import numpy as np

        if not self._handle:
            raise RuntimeError("this CGSolver has already been closed")
        buf = (ctypes.c_double * (self.max_iters + 1))()
        n = ctypes.c_int(0)
        check(lib.mr_b200_cg_residuals(self._handle, buf, self.max_iters + 1, ctypes.byref(n)),
              "mr_b200_cg_residuals")
        return np.array(buf[: min(n.value, self.max_iters + 1)], dtype=np.float64)

    def close(self) -> None:
        if self._handle:
            lib.mr_b200_cg_destroy(self._handle)
            self._handle = ctypes.c_void_p()
            self._keep = ()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_op(cfg: MRConfig, SEs, phi2, traj, mask=None, **kwargs) -> AhAOp:
    """Alias of :meth:`AhAOp.create_op` (reference ``api.py:1237-1255``)."""
    return AhAOp.create_op(cfg, SEs, phi2, traj, mask, **kwargs)
