"""ctypes mirror of include/dgswem_cuda.h (the C-ABI of libdgswem_cuda.so).

Loading fails loudly when the built library is missing: there is no CPU or
Python fallback for the hydro step.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# DGSWEM_CUDA_LIB points at another build of the same library
LIB_PATH = Path(os.environ.get("DGSWEM_CUDA_LIB", Path(__file__).resolve().parent / "lib" / "libdgswem_cuda.so"))

# dgswem_cuda.h constants
MAX_SHAPES = 8        # DGSWEM_CUDA_MAX_SHAPES
TUNE_CACHED = 1       # DGSWEM_CUDA_TUNE_CACHED

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Setup(C.Structure):
    """struct dgswem_cuda_setup (field order matters)."""

    _fields_ = [
        ("ne", C.c_int), ("np", C.c_int), ("dofh", C.c_int), ("nrk", C.c_int), ("nedges", C.c_int),
        ("nieds", C.c_int), ("nleds", C.c_int), ("needs", C.c_int), ("nfeds", C.c_int), ("nreds", C.c_int),
        ("nebseg", C.c_int), ("nibseg", C.c_int),
        ("ics", C.c_int), ("nolifa", C.c_int), ("iflinbf", C.c_int), ("ifhybf", C.c_int), ("ifnlfa", C.c_int),
        ("nramp", C.c_int), ("nws", C.c_int), ("rainfall", C.c_int), ("slopeflag", C.c_int),
        ("load_manning", C.c_int),
        ("nleq", C.c_double), ("leq", C.c_double), ("g", C.c_double), ("h0", C.c_double),
        ("dtdp", C.c_double), ("statim", C.c_double), ("dramp", C.c_double),
        ("cf", C.c_double), ("hbreak", C.c_double), ("ftheta", C.c_double), ("fgamma", C.c_double),
        ("sfea0", C.c_double),
        ("atvd", _dp), ("btvd", _dp), ("dtvd", _dp),
        ("nm", _ip), ("x", _dp), ("y", _dp), ("dp", _dp),
        ("nedno", _ip), ("nedel", _ip), ("nedsd", _ip), ("neled", _ip),
        ("niedn", _ip), ("nledn", _ip), ("needn", _ip), ("nfedn", _ip), ("nredn", _ip), ("nebsegn", _ip),
        ("nibsegn", _ip),
        ("hb", _dp), ("cori_el", _dp), ("fric_el", _dp), ("manning", _dp),
        ("ze", _dp), ("qx", _dp), ("qy", _dp), ("wdflg", _ip),
        ("nbfr", C.c_int), ("amig", _dp), ("ff", _dp), ("face", _dp), ("per", _dp),
        ("emo_dg", _dp), ("efa_dg", _dp),
        ("nffr", C.c_int), ("famig", _dp), ("fff", _dp), ("fface", _dp), ("fper", _dp),
        ("qnam_dg", _dp), ("qnph_dg", _dp),
        ("ebht", _dp), ("ebcfsp", _dp), ("ibht", _dp), ("ibcfsb", _dp), ("ibcfsp", _dp),
    ]


# every entry point of the header: name -> (restype, argtypes)
SIGNATURES = {
    "dgswem_cuda_create": (C.c_int, [C.POINTER(Setup), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "dgswem_cuda_destroy": (None, [C.c_void_p]),
    "dgswem_cuda_hydro_timestep": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dgswem_cuda_synchronize": (C.c_int, [C.c_void_p]),
    "dgswem_cuda_upload_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip]),
    "dgswem_cuda_download_state": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip]),
    "dgswem_cuda_set_met": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "dgswem_cuda_met_file": (C.c_int, [C.c_void_p, C.c_char_p]),
    "dgswem_met_reader_open": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "dgswem_met_reader_next": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "dgswem_met_reader_calls": (C.c_long, [C.c_void_p]),
    "dgswem_met_reader_close": (None, [C.c_void_p]),
    "dgswem_cuda_modal2nodal": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip]),
    "dgswem_cuda_modal2nodal_noalloc": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _ip]),
    "dgswem_cuda_create_part": (C.c_int, [C.POINTER(Setup), C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.POINTER(C.c_void_p)]),
    "dgswem_cuda_part_info": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _ip]),
    "dgswem_cuda_stage_rhs": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dgswem_cuda_stage_rhs_tiles": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "dgswem_cuda_tile_split": (C.c_int, [C.c_void_p, _ip, _ip]),
    "dgswem_cuda_stage_limit": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_step_end": (C.c_int, [C.c_void_p]),
    "dgswem_cuda_halo_count": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _ip, _ip]),
    "dgswem_cuda_halo_pack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "dgswem_cuda_halo_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "dgswem_part_halo_ids": (C.c_int, [C.POINTER(Setup), C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip,
                                       _ip]),
    "dgswem_cuda_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "dgswem_cuda_last_error": (C.c_int, [C.c_char_p, C.c_int]),
    "dgswem_cuda_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dgswem_cuda_set_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_shapes": (C.c_int, [_ip, _ip, _ip, _ip, _ip, _ip]),
    "dgswem_cuda_set_shapes": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dgswem_cuda_get_shapes": (C.c_int, [C.c_void_p, _ip, _ip]),
    "dgswem_cuda_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "dgswem_cuda_stream": (C.c_void_p, [C.c_void_p]),
    "dgswem_cuda_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_profile_read": (C.c_int, [C.c_void_p, _dp, C.POINTER(C.c_longlong)]),
    "dgswem_deck_open": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "dgswem_deck_setup": (C.POINTER(Setup), [C.c_void_p]),
    "dgswem_deck_int": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int)]),
    "dgswem_deck_close": (None, [C.c_void_p]),
    "dgswem_deck_merge": (C.c_int, [C.POINTER(C.POINTER(Setup)), C.c_int, C.POINTER(C.c_void_p)]),
    "dgswem_cuda_set_params": (C.c_int, [C.c_void_p, _dp, _dp]),
    "dgswem_cuda_state_save": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_state_load": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_gauges": (C.c_int, [C.c_void_p, C.c_int, _ip, _dp]),
    "dgswem_cuda_gauge_eta": (C.c_int, [C.c_void_p, _dp]),
    "dgswem_cuda_adjoint_begin": (C.c_int, [C.c_void_p]),
    "dgswem_cuda_adjoint_seed": (C.c_int, [C.c_void_p, _dp]),
    "dgswem_cuda_adjoint_step": (C.c_int, [C.c_void_p, C.c_int]),
    "dgswem_cuda_adjoint_read": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "dgswem_cuda_misfit_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]),
    "dgswem_cuda_adjoint_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]),
    "dgswem_cuda_limit_state": (C.c_int, [C.c_void_p]),
    "dgswem_cuda_limiter_vjp": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]),
}

_lib = None


def load() -> C.CDLL:
    """Load libdgswem_cuda.so from the package (build it with dgswem_b200.build)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library with `python -m dgswem_b200.build`; "
                "the DG hydro step has no CPU fallback")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class DgswemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"libdgswem_cuda status {status}: {message}")
        self.status = status


def check(status: int) -> None:
    if status != 0:
        buf = C.create_string_buffer(1024)
        load().dgswem_cuda_last_error(buf, len(buf))
        raise DgswemError(status, buf.value.decode(errors="replace"))
