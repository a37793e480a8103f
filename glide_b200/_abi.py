"""ctypes binding of the C ABI in ``include/glide_b200.h``.

The library ``glide_b200/libglide_b200.so`` is loaded from the package
directory; importing this module never falls back to anything else: a missing
or stale library raises ``ImportError`` with the reason.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# GLIDE_B200_LIBRARY may name another build of the same library (e.g. a debug build)
LIB_PATH = Path(os.environ.get("GLIDE_B200_LIBRARY") or Path(__file__).resolve().parent / "libglide_b200.so")

GLIDE_OK = 0
GLIDE_MET_F32, GLIDE_MET_BF16, GLIDE_MET_F16 = 0, 1, 2
GLIDE_STATUS_NONFINITE_STATE, GLIDE_STATUS_BAD_ORDER = 1, 2
GLIDE_STATUS_BAD_ROW, GLIDE_STATUS_COMPACT_OVERFLOW = 4, 8
GLIDE_WORK_DONE, GLIDE_WORK_PENDING, GLIDE_WORK_CLASSES = 0, 63, 64
GLIDE_STEP_BATCH_MAX = 32
GLIDE_REGRID_MAX_LEVELS = 256
GLIDE_DIAG_DEG_SCALE, GLIDE_DIAG_M_SCALE = 1 << 20, 1 << 10

vp = C.c_void_p


class Grid(C.Structure):
    _fields_ = [("nz", C.c_int32), ("ny", C.c_int32), ("nx", C.c_int32), ("ascending", C.c_int32),
                ("lon_first", C.c_double), ("lon_last", C.c_double), ("lat_first", C.c_double),
                ("lat_last", C.c_double), ("level_sorted", vp), ("level_lut", vp), ("lut_n", C.c_int32),
                ("lut_inv_dz", C.c_float)]


class WindowDesc(C.Structure):
    _fields_ = [("grid", Grid), ("u", vp * 2), ("v", vp * 2), ("w", vp * 2), ("t", vp * 2), ("t_lowest", vp * 2),
                ("blh", vp * 2), ("sp", vp * 2), ("ustar", vp * 2), ("shf", vp * 2), ("height3d", vp),
                ("height_level", vp), ("pressure_hpa", vp), ("meander_coefficient", C.c_float),
                ("meander_radius", C.c_int32), ("build_meander", C.c_int32), ("met_dtype", C.c_int32),
                ("wind_packed", vp), ("surf_packed", vp), ("support_packed", vp), ("wind_sum", vp)]


class StepSched(C.Structure):
    _fields_ = [("cursor_off", C.c_float), ("delta", C.c_float), ("alpha", C.c_float), ("step_index", C.c_int32)]


class FootprintGrid(C.Structure):
    _fields_ = [("lon_min", C.c_double), ("lon_max", C.c_double), ("lat_min", C.c_double), ("lat_max", C.c_double),
                ("n_releases", C.c_int32), ("n_time_bins", C.c_int32), ("n_z", C.c_int32), ("n_y", C.c_int32),
                ("n_x", C.c_int32), ("z_edges", vp), ("ring", C.c_int32), ("value_f64", C.c_int32)]


class StepArgs(C.Structure):
    _fields_ = [("n", C.c_int64), ("lon", vp), ("lat", vp), ("z", vp), ("weight", vp), ("pos_stride", C.c_int64),
                ("u_prime", vp), ("v_prime", vp), ("w_prime", vp), ("u_meander", vp), ("v_meander", vp),
                ("rel_off", vp), ("win_end_off", vp), ("release_idx", vp), ("alive", vp), ("active_mask", vp),
                ("sim_length_s", C.c_float), ("wind_packed", vp), ("surf_packed", vp), ("support_packed", vp),
                ("met_dtype", C.c_int32), ("grid", Grid), ("substep_c", C.c_float), ("max_substeps", C.c_int32),
                ("z_ubl_m", C.c_float), ("flexpart_tl_floors", C.c_int32), ("surface_layer_override", C.c_int32),
                ("meander_enabled", C.c_int32), ("meander_timescale_s", C.c_float), ("sched", vp),
                ("sched0", StepSched), ("n_steps", C.c_int32), ("phys_begin", C.c_int32), ("post_begin", C.c_int32),
                ("noise_substep", vp), ("noise_meander", vp), ("seed", C.c_uint64), ("footprint", vp),
                ("fp", FootprintGrid), ("dom_lon_min", C.c_double), ("dom_lon_max", C.c_double),
                ("dom_lat_min", C.c_double), ("dom_lat_max", C.c_double), ("dom_alt_max", C.c_double),
                ("escaped_per_step", vp), ("active_per_step", vp), ("status", vp), ("launch_variant", C.c_int32),
                ("order", vp), ("work_key", vp), ("conv_column", vp), ("conv_step", C.c_int32),
                ("conv_nz", C.c_int32), ("conv_uniforms", vp), ("conv_moved", vp), ("diag_pos_fixed", vp)]


class ConvectArgs(C.Structure):
    _fields_ = [("n", C.c_int64), ("z", vp), ("z_stride", C.c_int64), ("rel_off", vp), ("alive", vp),
                ("active_mask", vp), ("sim_length_s", C.c_float), ("sched", StepSched), ("nz", C.c_int32),
                ("ny", C.c_int32), ("nx", C.c_int32), ("t", vp * 2), ("q", vp * 2), ("height3d", vp),
                ("height_level", vp), ("pressure_hpa", vp), ("alpha", C.c_float), ("closure_c", C.c_float),
                ("trigger_dtv_k", C.c_float), ("min_cape_j_kg", C.c_float), ("min_cloud_depth_m", C.c_float),
                ("uniforms", vp), ("seed", C.c_uint64), ("scratch", vp), ("n_moved", vp)]


class OuArgs(C.Structure):
    _fields_ = [("n", C.c_int64), ("w", vp), ("t_l", vp), ("t_l_scalar", C.c_float), ("sigma2", vp),
                ("sigma2_scalar", C.c_float), ("dt", vp), ("dt_scalar", C.c_float), ("drift", vp),
                ("drift_scalar", C.c_float), ("noise", vp), ("seed", C.c_uint64), ("counter", C.c_uint32)]


class RegridArgs(C.Structure):
    _fields_ = [("n_channels", C.c_int32), ("zp", C.c_int32), ("za", C.c_int32), ("ny", C.c_int32),
                ("nx", C.c_int32), ("height_agl_p", vp), ("agl_levels", vp), ("fields_p", vp), ("fields_agl", vp),
                ("pressure_p_hpa", vp), ("pressure_level_hpa", vp), ("u_channel", C.c_int32),
                ("v_channel", C.c_int32), ("w_channel", C.c_int32), ("dhdx", vp), ("dhdy", vp),
                ("slope_f32", C.c_int32), ("z_top_m", C.c_double), ("scratch", vp), ("scratch_bytes", C.c_size_t)]


class CompactArgs(C.Structure):
    _fields_ = [("rows", vp), ("n_rows", C.c_int64), ("cells", C.c_int64), ("row_index", vp), ("k", C.c_int32),
                ("clear", C.c_int32), ("slice_offset", vp), ("out_cell", vp), ("out_value", vp),
                ("capacity", C.c_int64), ("status", vp), ("scratch", vp), ("scratch_bytes", C.c_size_t),
                ("value_f64", C.c_int32)]


STRUCTS = (Grid, WindowDesc, StepSched, FootprintGrid, StepArgs, ConvectArgs, OuArgs, RegridArgs, CompactArgs)

# every exported symbol with (restype, argtypes)
SIGNATURES = {
    "glide_version": (C.c_int32, []),
    "glide_last_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "glide_abi_struct_sizes": (C.c_int32, [C.POINTER(C.c_size_t), C.c_int32]),
    "glide_window_packed_bytes": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_size_t),
                                              C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "glide_window_pack": (C.c_int32, [C.POINTER(WindowDesc), vp]),
    "glide_step": (C.c_int32, [C.POINTER(StepArgs), vp]),
    "glide_step_batched": (C.c_int32, [C.POINTER(StepArgs), C.c_int32, vp]),
    "glide_step_launch_variants": (C.c_int32, [C.POINTER(C.c_int32)]),
    "glide_step_launch_variant_info": (C.c_int32, [C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "glide_reorder_scratch_bytes": (C.c_int32, [C.c_int64, C.POINTER(C.c_size_t)]),
    "glide_reorder_by_key": (C.c_int32, [C.c_int64, vp, vp, vp, C.c_size_t, vp]),
    "glide_ou_update": (C.c_int32, [C.POINTER(OuArgs), vp]),
    "glide_displace_vertical": (C.c_int32, [C.c_int64, vp, C.c_int64, vp, vp, C.c_float, C.c_int32, vp]),
    "glide_displace_horizontal": (C.c_int32, [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_float, C.c_int32, vp]),
    "glide_reflect_surface": (C.c_int32, [C.c_int64, vp, C.c_int64, vp, C.c_float, vp]),
    "glide_rk2_stage": (C.c_int32, [C.c_int64, vp, C.c_int64, vp, C.c_int64, C.c_float, vp, C.c_int64, vp]),
    "glide_agl_regrid_scratch_bytes": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_size_t)]),
    "glide_agl_regrid": (C.c_int32, [C.POINTER(RegridArgs), vp]),
    "glide_footprint_compact_scratch_bytes": (C.c_int32, [C.c_int32, C.c_int64, C.POINTER(C.c_size_t)]),
    "glide_footprint_compact": (C.c_int32, [C.POINTER(CompactArgs), vp]),
    "glide_footprint_accumulate": (C.c_int32, [C.c_int64, vp, vp, vp, C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_float,
                                               C.POINTER(FootprintGrid), vp, vp]),
    "glide_convect_scratch_bytes": (C.c_int32, [C.c_int32, C.POINTER(C.c_size_t)]),
    "glide_convect": (C.c_int32, [C.POINTER(ConvectArgs), vp]),
    "glide_convect_noalloc": (C.c_int32, [C.POINTER(ConvectArgs), vp]),
    "glide_convect_redistribute": (C.c_int32, [C.POINTER(ConvectArgs), vp]),
    "glide_convect_column_info": (C.c_int32, [vp, C.c_int32, vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                              C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.POINTER(C.c_double)]),
}


class GlideError(RuntimeError):
    """A non-zero ``glide_status`` from the CUDA library, with its error text."""


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"glide_b200 CUDA library not built: {LIB_PATH} is missing "
                          "(run `python -m glide_b200.build`)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = (C.c_size_t * len(STRUCTS))()
    lib.glide_abi_struct_sizes(sizes, len(STRUCTS))
    for st, sz in zip(STRUCTS, sizes):
        if C.sizeof(st) != sz:
            raise ImportError(f"ABI mismatch: sizeof({st.__name__}) is {sz} in the library, "
                              f"{C.sizeof(st)} in the binding (rebuild the library)")
    return lib


lib = _load()


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib.glide_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str) -> None:
    if status != GLIDE_OK:
        raise GlideError(f"{what} failed (status {status}): {last_error()}")
