"""ctypes binding of libfeab200.so (declarations in include/feab200.h).

The library is the only compute path: importing this module raises ImportError when the
shared object is missing, and every call maps a non-zero status to the exception the
reference raises for the same condition.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfeab200.so")

FEAB_OK = 0
FEAB_BAD_ARG = 1
FEAB_DEGENERATE_ELEMENT = 2
FEAB_ZERO_DIAGONAL = 3
FEAB_NOT_SPD = 4
FEAB_NOT_CONVERGED = 5
FEAB_CUDA_ERROR = 6
FEAB_CAPACITY = 7
FEAB_SCRATCH_LIMIT = 8

KE_PACKED = 324
KE_FULL = 576
PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP32 = 2


class DeviceStatus(C.Structure):
    _fields_ = [("code", C.c_int32), ("reserved", C.c_int32), ("index", C.c_int64)]


class CSR(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_groups", C.c_int32), ("nnz", C.c_int64),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("vals64", C.c_void_p),
                ("vals32", C.c_void_p), ("group_ptr", C.c_void_p)]


class DiffOperator(C.Structure):
    _fields_ = [("tcol", C.c_void_p), ("vhi", C.c_void_p), ("vlo", C.c_void_p), ("gmask", C.c_void_p),
                ("S", C.c_void_p), ("goff", C.c_void_p), ("voff", C.c_void_p), ("vlo2", C.c_void_p)]


class SellOperator(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_slices", C.c_int32), ("soff", C.c_void_p), ("tcol", C.c_void_p),
                ("v64", C.c_void_p), ("vhi", C.c_void_p), ("vlo", C.c_void_p), ("gmask", C.c_void_p),
                ("S", C.c_void_p), ("tcol16", C.c_void_p)]


class TileOperator(C.Structure):
    _fields_ = [("n_tiles", C.c_int32), ("precision", C.c_int32), ("n_groups", C.c_int32), ("reserved", C.c_int32),
                ("tile_g0", C.c_void_p), ("group_tile", C.c_void_p), ("uoff", C.c_void_p), ("poff", C.c_void_p),
                ("ucol", C.c_void_p), ("upair", C.c_void_p), ("umask", C.c_void_p), ("v64", C.c_void_p),
                ("vhi", C.c_void_p), ("vlo", C.c_void_p), ("vlo2", C.c_void_p), ("cptr", C.c_void_p),
                ("chunk", C.c_void_p)]


TILE_GROUPS = 4   # FEAB_TILE_GROUPS: node row groups per tile of the block SpMM


class Batch(C.Structure):
    _fields_ = [("n_problems", C.c_int32), ("k", C.c_int32), ("n_items", C.c_int32), ("reserved", C.c_int32),
                ("item_problem", C.c_void_p), ("item_group0", C.c_void_p), ("item_group1", C.c_void_p),
                ("problem_items", C.c_void_p), ("problem_cols", C.c_void_p)]


class Band(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_tiles", C.c_int32), ("bands", C.c_int32), ("reserved", C.c_int32),
                ("storage", C.c_void_p)]


class PcgParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxiter", C.c_int32), ("precision", C.c_int32),
                ("reliable_delta", C.c_double), ("chunk", C.c_int32), ("use_dinv", C.c_int32),
                ("lanes_per_group", C.c_int32), ("reserved", C.c_int32)]


class PcgResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iters", C.c_int32), ("reliable_updates", C.c_int32),
                ("graph_launches", C.c_int32), ("relres", C.c_double), ("bnorm", C.c_double)]


_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_SZ = C.c_size_t
_D = C.c_double

# name -> (restype, argtypes); the exported set of include/feab200.h
SIGNATURES = {
    "feab_abi_version": (_I32, []),
    "feab_status_string": (C.c_char_p, [_I32]),
    "feab_set_device": (_I32, [_I32]),
    "feab_launch_count": (C.c_uint64, []),
    "feab_topology_scratch_bytes": (_SZ, [_I32, _I64]),
    "feab_node_incidence": (_I32, [_P, _I64, _I32, _P, _P, _P, _SZ, _P, C.POINTER(_I32), _P]),
    "feab_node_adjacency": (_I32, [_P, _P, _P, _I32, _P, _P, _P, _SZ, _P, C.POINTER(_I64), C.POINTER(_I32), _P]),
    "feab_csr_pattern": (_I32, [_P, _P, _I32, _P, _I32, _P, _P, _P, _P, _SZ, C.POINTER(_I64), C.POINTER(_I32), _P]),
    "feab_hex8_element_stiffness": (_I32, [_P, _P, _I64, C.POINTER(_D), _P, _D, _P, _I32, _P, _P]),
    "feab_hex8_bbar_element_stiffness": (_I32, [_P, _P, _I64, C.POINTER(_D), _P, _D, _P, _I32, _P, _P]),
    "feab_hex8_element_mass": (_I32, [_P, _P, _I64, C.POINTER(_D), _P, _D, _P, _I32, _P, _P]),
    "feab_assemble_csr": (_I32, [_P, _P, _P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "feab_hex8_apply": (_I32, [_P, _P, _P, _P, _I32, _P, _P, _P]),
    "feab_pcg_workspace_bytes": (_SZ, [_I32, _I32]),
    "feab_diff_operator_bytes": (_SZ, [_I32, _I64, _I32]),
    "feab_diff_operator_build": (_I32, [C.POINTER(CSR), _P, _P, _SZ, C.POINTER(DiffOperator), _P]),
    "feab_pcg_solve": (_I32, [C.POINTER(CSR), C.POINTER(SellOperator), _P, _P, _P, _P, _P, C.POINTER(PcgParams), _P,
                              _SZ, C.POINTER(PcgResult), _P]),
    "feab_pcg_noalloc_scratch_bytes": (_SZ, []),
    "feab_pcg_noalloc_max_n": (_I32, []),
    "feab_pcg_solve_noalloc": (_I32, [C.POINTER(CSR), _P, _P, _P, _P, C.POINTER(PcgParams), C.POINTER(PcgResult), _P]),
    "feab_sell_operator_bytes": (_SZ, [_I32, _I32, _I32, _I32]),
    "feab_sell_operator_build": (_I32, [C.POINTER(CSR), _P, _I32, _I32, _P, _SZ, C.POINTER(SellOperator), _P]),
    "feab_sell_spmv": (_I32, [C.POINTER(CSR), C.POINTER(SellOperator), _P, _P, _P]),
    "feab_csr_spmv": (_I32, [C.POINTER(CSR), C.POINTER(SellOperator), _I32, _I32, _P, _P, _P]),
    "feab_block_pcg_workspace_bytes": (_SZ, [_I32, _I32, _I32, _I32]),
    "feab_tile_scratch_bytes": (_SZ, [_I32, _I32]),
    "feab_tile_operator_build": (_I32, [C.POINTER(CSR), C.POINTER(DiffOperator), _P, _I32, _I32, _P, _SZ, _P, _SZ,
                                        C.POINTER(_SZ), C.POINTER(TileOperator), _P]),
    "feab_block_pcg_solve": (_I32, [C.POINTER(CSR), C.POINTER(DiffOperator), C.POINTER(TileOperator),
                                    C.POINTER(Batch), _P, _P, _P, C.POINTER(PcgParams), _P, _SZ, C.POINTER(_I32),
                                    C.POINTER(_D), C.POINTER(_I32), _P]),
    "feab_block_spmm": (_I32, [C.POINTER(CSR), C.POINTER(TileOperator), _P, _P, _I32, _P]),
    "feab_panel_gram_workspace_bytes": (_SZ, [_I64]),
    "feab_panel_gram": (_I32, [_P, _I32, _P, _I32, _I64, _I32, _P, _P, _SZ, _P]),
    "feab_panel_small": (_I32, [_P, _I32, _I64, _I32, _P, _I32, _P, _I32, _P]),
    "feab_gram_workspace_bytes": (_SZ, [_I64, _I32]),
    "feab_gram_bf16x3": (_I32, [_P, _I64, _I32, _P, _P, _SZ, _P, _P]),
    "feab_gram_fp64": (_I32, [_P, _I32, _I64, _I32, _P, _P, _SZ, _P]),
    "feab_gram_int8": (_I32, [_P, _I64, _I32, _P, _P, _SZ, _P, _P]),
    "feab_symeig_jacobi": (_I32, [_P, _I32, _P, _P, _I32, _P, _P]),
    "feab_hex8_simp_vjp": (_I32, [_P, _P, _I64, C.POINTER(_D), _P, _D, _D, _P, _P, _P, _P, _P]),
    "feab_element_centroids": (_I32, [_P, _P, _I64, _P, _P]),
    "feab_filter_scratch_bytes": (_SZ, [_I64]),
    "feab_filter_build": (_I32, [_P, _I64, _D, _P, _P, _P, _P, C.POINTER(_I64), _P, _SZ, _P]),
    "feab_filter_apply": (_I32, [_P, _P, _P, _P, _I64, _P, _P, _D, _P, _P]),
    "feab_oc_workspace_bytes": (_SZ, [_I64]),
    "feab_oc_update": (_I32, [_P, _P, _I64, _D, _D, _D, _D, _D, _I32, _P, _P, _P, _SZ, _P]),
    "feab_hex8_recover_scratch_bytes": (_SZ, [_I64]),
    "feab_hex8_recover": (_I32, [_P, _P, _I64, _I32, _P, _P, C.POINTER(_D), _P, _P, _P, _P, _P, _P, _SZ, _P, _P]),
    "feab_band_width": (_I32, [C.POINTER(CSR), _P, _P, C.POINTER(_I32), _P]),
    "feab_band_bytes": (_SZ, [_I32, _I32]),
    "feab_band_assemble": (_I32, [C.POINTER(CSR), _P, _I32, C.POINTER(Band), _P]),
    "feab_band_cholesky": (_I32, [C.POINTER(Band), C.POINTER(_D), _P]),
    "feab_band_solve": (_I32, [C.POINTER(Band), _P, _P, _P, _P]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"feab200: CUDA library {LIB_PATH} is missing -- build it with "
            f"`python computation-suite_b200/build.py` (nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def status_string(code):
    return lib.feab_status_string(int(code)).decode()


class FeabError(RuntimeError):
    """A CUDA-level failure inside libfeab200 (FEAB_CUDA_ERROR)."""


def raise_for(code, what, index=None):
    """Map a FEAB_* status to the reference's exception type."""
    code = int(code)
    if code == FEAB_OK:
        return
    where = "" if index is None else f" (index {int(index)})"
    msg = f"{what}: {status_string(code)}{where}"
    if code == FEAB_NOT_SPD:
        raise np.linalg.LinAlgError(msg + " -- A is not SPD.")
    if code == FEAB_NOT_CONVERGED:
        raise RuntimeError(msg)
    if code == FEAB_CUDA_ERROR:
        raise FeabError(msg)
    raise ValueError(msg)


def dptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else C.c_void_p(t.data_ptr())


_current = {}


def stream_ptr(device):
    """The torch stream of ``device`` as a cudaStream_t, after making ``device`` current in the
    library's runtime for this thread."""
    import threading
    import torch
    idx = torch.device(device).index
    idx = torch.cuda.current_device() if idx is None else idx
    tid = threading.get_ident()
    if _current.get(tid) != idx:
        raise_for(lib.feab_set_device(idx), "feab_set_device")
        _current[tid] = idx
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def dmat(D):
    """6x6 material matrix as a ctypes double[36] (host memory)."""
    a = np.ascontiguousarray(np.asarray(D, dtype=np.float64).reshape(36))
    return (C.c_double * 36)(*a.tolist())
