"""ctypes binding of libtlbm.so (the C ABI declared in include/tlbm.h).

This is the only module that touches the shared library.  Everything above it
passes raw device pointers of the caller's torch tensors plus the current CUDA
stream.  There is no CPU or torch fallback: if the library is missing, or a
tensor is not on a CUDA device, the call raises.
"""

from __future__ import annotations

import ctypes
import os
import pathlib

import torch

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = pathlib.Path(os.environ.get("TLBM_LIB", _HERE / "libtlbm.so"))

# include/tlbm.h TLBM_ABI_VERSION this mirror (Desc, SIGNATURES) is written for
ABI_VERSION = 3
# tlbm_status
OK, ERR_SHAPE, ERR_DTYPE, ERR_ALIAS, ERR_LAUNCH, ERR_TIMEOUT, ERR_NONFINITE, ERR_ARG, ERR_UNSUPPORTED = range(9)
ERR_TOO_LARGE = 9
# tlbm_dtype
F32, F64, F16_SHIFTED, BF16_SHIFTED, F16, BF16 = 0, 1, 2, 3, 4, 5
# tlbm_collision
(COLL_NONE, COLL_BGK, COLL_MRT, COLL_CUMULANT, COLL_CUMULANT_GEIER, COLL_CUMULANT_D3Q19, COLL_SMAGORINSKY, COLL_TRT,
 COLL_CASCADED, COLL_RLBM) = range(10)
# tlbm_bc_bits / tlbm_flag_bits
BC_LID, BC_ZH_INLET, BC_ZH_OUTLET, BC_FAR_FIELD, BC_FAR_FIELD_Z = 1, 2, 4, 8, 16
FLAG_SOLID, FLAG_OBSTACLE, FLAG_HALFWAY, FLAG_MOVING, FLAG_CURVED = 1, 2, 4, 8, 16

TORCH_TO_DTYPE = {torch.float32: F32, torch.float64: F64}


class Desc(ctypes.Structure):
    """struct tlbm_desc"""

    _fields_ = [
        ("lattice", ctypes.c_int32),
        ("dtype", ctypes.c_int32),
        ("collision", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("bc", ctypes.c_uint32),
        ("tau", ctypes.c_double),
        ("s_e", ctypes.c_double),
        ("s_eps", ctypes.c_double),
        ("s_q", ctypes.c_double),
        ("s_pi", ctypes.c_double),
        ("omega_b", ctypes.c_double),
        ("omega_odd", ctypes.c_double),
        ("omega_even", ctypes.c_double),
        ("c_smag", ctypes.c_double),
        ("u_lid", ctypes.c_double),
        ("u_in", ctypes.c_double * 3),
        ("rho_out", ctypes.c_double),
        ("wall_velocity", ctypes.c_void_p),
        ("force_lin", ctypes.c_double),
        ("lambda_trt", ctypes.c_double),
        ("link_row", ctypes.c_void_p),
        ("link_q", ctypes.c_void_p),
        ("cm_s5", ctypes.c_double),
        ("cm_s6", ctypes.c_double),
        ("ff_inlet_du", ctypes.c_double * 3),
    ]


class BatchDomain(ctypes.Structure):
    """struct tlbm_batch_domain"""

    _fields_ = [("f_offset", ctypes.c_int64), ("cell_offset", ctypes.c_int64), ("nx", ctypes.c_int32),
                ("ny", ctypes.c_int32), ("tau", ctypes.c_double), ("u_in", ctypes.c_double),
                ("rho_out", ctypes.c_double), ("bc", ctypes.c_uint32), ("nz", ctypes.c_int32),
                ("u_lid", ctypes.c_double)]


class BatchDesc(ctypes.Structure):
    """struct tlbm_batch_desc"""

    _fields_ = [("lattice", ctypes.c_int32), ("dtype", ctypes.c_int32), ("collision", ctypes.c_int32),
                ("ndomains", ctypes.c_int32), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("cells_per_thread", ctypes.c_int32),
                ("domain_status", ctypes.c_void_p)]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES: dict[str, list] = {
    "tlbm_step": [ctypes.POINTER(Desc), _P, _P, _P, _P, _P, _P, _P],
    "tlbm_step_planes": [ctypes.POINTER(Desc), _P, _P, _P, _P, _P, _P, _I32, _I32, _P],
    "tlbm_collide": [ctypes.POINTER(Desc), _I32, _P, _P, _P, _P, _P],
    "tlbm_stream": [_I32, _I32, _I32, _I32, _I32, _P, _P, _P],
    "tlbm_equilibrium": [_I32, _I32, _I64, _P, _P, _P, _P, _P, _P],
    "tlbm_macroscopic": [_I32, _I32, _I64, _P, _P, _P, _P, _P, _P],
    "tlbm_bounce_back": [_I32, _I32, _I64, _P, _P, _P, _P],
    "tlbm_moving_wall_bounce_back": [_I32, _I32, _I64, _P, _P, _P, _P, _P],
    "tlbm_zou_he_inlet": [_I32, _I32, _I32, _I32, _I32, _P, _D, _D, _D, _P, _P, _P],
    "tlbm_zou_he_outlet": [_I32, _I32, _I32, _I32, _I32, _P, _D, _P],
    "tlbm_moving_lid": [_I32, _I32, _I32, _I32, _I32, _P, _D, _P],
    "tlbm_far_field": [_I32, _I32, _I32, _I32, _I32, _P, _D, _D, _D, _I32, _P],
    "tlbm_obstacle_force": [_I32, _I32, _I64, _P, _P, _P, _P],
    "tlbm_correct_mass": [_I32, _I64, _P, _P, _D, _P, _P],
    "tlbm_moment_sums": [_I32, _I32, _I64, _P, _P, _P],
    "tlbm_sphere_mask": [_I32, _I32, _I32, _D, _D, _D, _D, _P, _P],
    "tlbm_cylinder_mask": [_I32, _I32, _D, _D, _D, _P, _P],
    "tlbm_build_flags": [_I64, _P, _P, ctypes.c_uint32, _P, _P],
    "tlbm_missing_mask": [_I32, _I32, _I32, _I32, _P, _I32, _P, _P],
    "tlbm_link_blocks": [_I64],
    "tlbm_link_count": [_P, _I64, _P, _P, _P],
    "tlbm_link_list": [_P, _I64, _P, _P, _P],
    "tlbm_batch_step": [ctypes.POINTER(BatchDesc), _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P],
    "tlbm_batch_advance_slot": [_P, _P],
    "tlbm_batch_run": [ctypes.POINTER(BatchDesc), _P, _P, _I64, _P, _P, _P, _I32, _P, _I32, _P, _P, _I64, _P],
    "tlbm_link_list_noalloc": [_P, _I64, _P, _I64, _P, _P],
    "tlbm_sphere_links": [_I32, _I32, _I32, _I32, _D, _D, _D, _D, _P, _P, _P, _P],
    "tlbm_aa_load": [ctypes.POINTER(Desc), _P, _P, _P, _P, _P],
    "tlbm_step_aa": [ctypes.POINTER(Desc), _P, _I32, _P, _P, _P, _P, _P],
    "tlbm_aa_populations": [ctypes.POINTER(Desc), _P, _I32, _P, _P, _P, _P],
    "tlbm_bfl_bounce_back": [ctypes.POINTER(Desc), _P, _P, _P, _P, _P, _P, _P],
    "tlbm_link_momentum_sums": [ctypes.POINTER(Desc), _P, _P, _P, _P, _I32, _P, _P],
    "tlbm_link_list_static_capacity": [],
    "tlbm_les_filter_moments": [_P, _I32, _I32, _I32, _I32, _D, _P, _P],
    "tlbm_les_samples": [_P, _I32, _I32, _I32, _D, _D, _P, _P, _P, _P, _P],
    "tlbm_mlp_param_count": [],
    "tlbm_mlp_blob_bytes": [],
    "tlbm_mlp_grad_blocks": [_I64],
    "tlbm_mlp_grad": [_P, _P, _P, _P, _P, _P, _P, _I64, _P, _P],
    "tlbm_mlp_adam": [_P, _P, _P, _P, _I64, _D, _D, _D, _D, _I64, _P, _P, _P],
    "tlbm_mlp_eval": [_P, _P, _P, _P, _I64, _P, _P],
    "tlbm_mlp_pack": [_P, _P, _P, _P, _P, _D, _P, _P],
    "tlbm_mlp_infer": [_P, _P, _I64, _P, _P, _P],
    "tlbm_les_step": [_I32, _I32, _I32, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P],
    "tlbm_status_string": [ctypes.c_int],
    "tlbm_abi_version": [],
    "tlbm_struct_size": [_I32],
    "tlbm_set_row_staging": [_I32],
}
_RESTYPES = {"tlbm_link_blocks": _I64, "tlbm_link_list_static_capacity": _I64, "tlbm_status_string": ctypes.c_char_p,
             "tlbm_mlp_param_count": _I32, "tlbm_mlp_blob_bytes": _I32, "tlbm_mlp_grad_blocks": _I64,
             "tlbm_struct_size": _I64}

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Load (once) and type the shared library.  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"tensorlbm_b200: CUDA library {LIB_PATH} not found; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C tensorlbm_b200/csrc`"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.tlbm_abi_version.restype = ctypes.c_int
    if lib.tlbm_abi_version() != ABI_VERSION:
        raise RuntimeError(f"tensorlbm_b200: {LIB_PATH} has ABI version {lib.tlbm_abi_version()}, this package "
                           f"binds version {ABI_VERSION}; rebuild it")
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(status: int, what: str) -> None:
    """Map a tlbm_status to the exception type TensorLBM raises for that case."""
    if status == OK:
        return
    msg = f"{what}: {load().tlbm_status_string(status).decode()} (status {status})"
    if status in (ERR_SHAPE, ERR_DTYPE, ERR_ALIAS, ERR_ARG, ERR_TOO_LARGE):
        raise ValueError(msg)
    if status == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


def require_cuda(*tensors: torch.Tensor) -> torch.device:
    """All tensors on one CUDA device; returns it."""
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"expected a torch.Tensor, got {type(t).__name__}")
        if t.device.type != "cuda":
            raise RuntimeError(
                f"tensorlbm_b200 kernels run on CUDA devices only; got a tensor on {t.device}"
            )
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise RuntimeError(f"tensors on different devices: {dev} and {t.device}")
    if dev is None:
        raise RuntimeError("tensorlbm_b200 needs at least one CUDA tensor")
    return dev


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_of(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def real_dtype(t: torch.Tensor) -> int:
    try:
        return TORCH_TO_DTYPE[t.dtype]
    except KeyError:
        raise ValueError(f"unsupported dtype {t.dtype}; expected float32 or float64") from None


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def set_row_staging(enable: bool) -> bool:
    """Choose the kernel of the fused pull step: True runs the row-staged
    kernel where it is built and the layout allows it, False (the default)
    the two-cells-per-thread kernel (same results bit for bit).  Returns the
    previous setting."""
    return bool(load().tlbm_set_row_staging(1 if enable else 0))
