"""ctypes view of the B200 suites' C ABI (include/tealeaf_b200_{2d,3d}.h).

The structs restate the reference host layouts (2d/chunk.h:10-79,
2d/settings.h:69-150, 3d/chunk.h, 3d/settings.h); tests compare every offset
with the reference headers. The libraries are loaded from ``tealeaf_b200/lib``
only: there is no fallback, a missing library raises immediately.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"

_d, _i, _b, _p = C.c_double, C.c_int, C.c_bool, C.c_void_p
_dp = C.POINTER(C.c_double)


class ChunkExtension(C.Structure):
    _fields_ = [("suite", _p)]


class Settings2D(C.Structure):
    _fields_ = [
        ("kernel_profile", _p), ("application_profile", _p), ("wallclock_profile", _p),
        ("tea_out_fp", _p),
        ("rank", _i), ("end_step", _i), ("presteps", _i), ("max_iters", _i), ("coefficient", _i),
        ("ppcg_inner_steps", _i), ("summary_frequency", _i), ("halo_depth", _i), ("num_states", _i),
        ("num_chunks", _i), ("num_chunks_per_rank", _i), ("num_ranks", _i),
        ("fields_to_exchange", C.POINTER(C.c_bool)),
        ("is_offload", _b), ("error_switch", _b), ("check_result", _b), ("preconditioner", _b),
        ("eps", _d), ("dt_init", _d), ("end_time", _d), ("eps_lim", _d),
        ("tea_in_filename", C.c_char_p), ("tea_out_filename", C.c_char_p),
        ("test_problem_filename", C.c_char_p),
        ("solver", _i), ("solver_name", C.c_char_p), ("kernel_language", _i),
        ("grid_x_cells", _i), ("grid_y_cells", _i),
        ("grid_x_min", _d), ("grid_y_min", _d), ("grid_x_max", _d), ("grid_y_max", _d),
        ("dx", _d), ("dy", _d),
    ]


class Settings3D(C.Structure):
    _fields_ = [
        ("kernel_profile", _p), ("application_profile", _p), ("wallclock_profile", _p),
        ("tea_out_fp", _p),
        ("rank", _i), ("end_step", _i), ("presteps", _i), ("max_iters", _i), ("coefficient", _i),
        ("ppcg_inner_steps", _i), ("summary_frequency", _i), ("halo_depth", _i), ("num_states", _i),
        ("num_chunks", _i), ("num_chunks_per_rank", _i), ("num_ranks", _i),
        ("fields_to_exchange", C.POINTER(C.c_bool)),
        ("is_offload", _b), ("error_switch", _b), ("check_result", _b), ("preconditioner", _b),
        ("eps", _d), ("dt_init", _d), ("end_time", _d), ("eps_lim", _d),
        ("tea_in_filename", C.c_char_p), ("tea_out_filename", C.c_char_p),
        ("test_problem_filename", C.c_char_p),
        ("solver", _i), ("kernel_language", _i),
        ("grid_x_cells", _i), ("grid_y_cells", _i), ("grid_z_cells", _i),
        ("grid_x_min", _d), ("grid_y_min", _d), ("grid_z_min", _d),
        ("grid_x_max", _d), ("grid_y_max", _d), ("grid_z_max", _d),
        ("dx", _d), ("dy", _d), ("dz", _d),
    ]


class State2D(C.Structure):
    _fields_ = [("defined", _b), ("density", _d), ("energy", _d), ("x_min", _d), ("y_min", _d),
                ("x_max", _d), ("y_max", _d), ("radius", _d), ("geometry", _i)]


class State3D(C.Structure):
    _fields_ = [("defined", _b), ("density", _d), ("energy", _d), ("x_min", _d), ("y_min", _d),
                ("z_min", _d), ("x_max", _d), ("y_max", _d), ("z_max", _d), ("radius", _d),
                ("geometry", _i)]


_CHUNK_HEAD = [("dt_init", _d), ("neighbours", C.POINTER(C.c_int)),
               ("left_send", _dp), ("left_recv", _dp), ("right_send", _dp), ("right_recv", _dp),
               ("top_send", _dp), ("top_recv", _dp), ("bottom_send", _dp), ("bottom_recv", _dp)]
_CHUNK_TAIL = [("theta", _d), ("eigmin", _d), ("eigmax", _d),
               ("cg_alphas", _dp), ("cg_betas", _dp), ("cheby_alphas", _dp), ("cheby_betas", _dp),
               ("ext", C.POINTER(ChunkExtension))]


class Chunk2D(C.Structure):
    _fields_ = _CHUNK_HEAD + [
        ("left", _i), ("right", _i), ("bottom", _i), ("top", _i), ("x", _i), ("y", _i),
    ] + [(n, _p) for n in (
        "density0", "density", "energy0", "energy", "u", "u0", "p", "r", "mi", "w", "kx", "ky", "sd",
        "cell_x", "cell_y", "cell_dx", "cell_dy", "vertex_dx", "vertex_dy", "vertex_x", "vertex_y",
        "volume", "x_area", "y_area")] + _CHUNK_TAIL


class Chunk3D(C.Structure):
    _fields_ = _CHUNK_HEAD + [
        ("front_send", _dp), ("front_recv", _dp), ("back_send", _dp), ("back_recv", _dp),
        ("lr_page", _i), ("tb_page", _i), ("fb_page", _i),
        ("left", _i), ("right", _i), ("bottom", _i), ("top", _i), ("back", _i), ("front", _i),
        ("x", _i), ("y", _i), ("z", _i),
    ] + [(n, _p) for n in (
        "density0", "density", "energy0", "energy", "vec_u", "vec_u0", "vec_p", "vec_r", "vec_mi",
        "vec_w", "vec_kx", "vec_ky", "vec_kz", "vec_sd", "vec_z",
        "cell_x", "cell_y", "cell_z", "cell_dx", "cell_dy", "cell_dz",
        "vertex_dx", "vertex_dy", "vertex_dz", "vertex_x", "vertex_y", "vertex_z",
        "volume", "x_area", "y_area", "z_area")] + _CHUNK_TAIL


class StepStats(C.Structure):
    """TlStepStats of the device-resident driver."""
    _fields_ = [("cg_iters", _i), ("cheby_iters", _i), ("ppcg_iters", _i), ("jacobi_iters", _i),
                ("est_iters", _i), ("total_iters", _i), ("error", _d), ("eigmin", _d), ("eigmax", _d),
                ("exact_error", _d)]


class RefineStats(C.Structure):
    """TlRefineStats of the iterative-refinement timestep."""
    _fields_ = [("iterations", _i), ("residual_updates", _i), ("converged", _i), ("cg_trips", _i),
                ("rel_residual", _d), ("device_ms", _d)]


class AdjointStats(C.Structure):
    """TlAdjointStats of the 3D adjoint."""
    _fields_ = [("J", _d), ("device_ms", _d), ("forward_steps", _i), ("forward_iters", _i),
                ("adjoint_iters", _i), ("checkpoints", _i)]


class BatchStats(C.Structure):
    """TlBatchStats of the batched timestep."""
    _fields_ = [("problems", _i), ("converged", _i), ("max_iterations", _i), ("total_iterations", _i),
                ("kernel_iterations", _i), ("tile_rows", _i), ("grid_blocks", _i), ("graph", _i),
                ("device_ms", _d)]


# Entry points shared by both suites (name -> extra argtypes after Chunk*, Settings*).
_COMMON = {
    "run_set_chunk_data": [], "run_kernel_initialise": [],
    "run_local_halos": [_i], "run_pack_or_unpack": [_i, _i, _b, _p, _dp],
    "run_store_energy": [], "run_field_summary": [_dp, _dp, _dp, _dp],
    "run_ppcg_init": [], "run_ppcg_inner_iteration": [_d, _d],
    "run_calculate_residual": [], "run_calculate_2norm": [_p, _dp],
}
SIGS = {
    2: dict(_COMMON, **{
        "run_set_chunk_state": [C.POINTER(State2D)], "run_kernel_finalise": [],
        "run_cg_init": [_d, _d, _dp], "run_cg_calc_w": [_dp], "run_cg_calc_ur": [_d, _dp],
        "run_cg_calc_p": [_d], "run_cheby_init": [], "run_cheby_iterate": [_d, _d],
        "run_jacobi_init": [_d, _d], "run_jacobi_iterate": [_dp], "run_copy_u": [], "run_finalise": [],
    }),
    3: dict(_COMMON, **{
        "run_set_chunk_state": [C.POINTER(State3D)], "run_kernel_finalise": [],
        "run_cg_solver_init": [_d, _d, _d, _dp], "run_cg_solver_calc_w": [_dp],
        "run_cg_solver_calc_ur": [_d, _dp], "run_cg_solver_calc_p": [_d],
        "run_cheby_solver_init": [], "run_cheby_solver_iterate": [_d, _d],
        "run_jacobi_solver_init": [_d, _d, _d], "run_jacobi_solver_iterate": [_dp],
        "run_solver_copy_u": [], "run_solver_finalise": [],
    }),
}

LIB_NAMES = {2: "libtealeaf_b200_2d.so", 3: "libtealeaf_b200_3d.so"}
_loaded = {}


def lib_path(dims: int) -> Path:
    return LIB_DIR / LIB_NAMES[dims]


def load(dims: int) -> C.CDLL:
    """Load (once) the suite for 2 or 3 dimensions; raises if it was not built."""
    if dims in _loaded:
        return _loaded[dims]
    path = lib_path(dims)
    if not path.exists():
        raise FileNotFoundError(
            "B200 suite library %s not built (run `python -m tealeaf_b200.build`); "
            "there is no CPU fallback" % path)
    lib = C.CDLL(str(path))
    chunk_t = Chunk2D if dims == 2 else Chunk3D
    settings_t = Settings2D if dims == 2 else Settings3D
    head = [C.POINTER(chunk_t), C.POINTER(settings_t)]
    for name, extra in SIGS[dims].items():
        fn = getattr(lib, name)
        fn.argtypes = head + extra
        fn.restype = None
    pre = "tl%dd_" % dims
    getattr(lib, pre + "set_error_mode").argtypes = [_i]
    getattr(lib, pre + "set_device").argtypes = [_i]
    getattr(lib, pre + "get_error").argtypes = [C.c_char_p, _i]
    getattr(lib, pre + "get_error").restype = _i
    getattr(lib, pre + "stream").argtypes = [C.POINTER(chunk_t)]
    getattr(lib, pre + "stream").restype = _p
    for nm in ("upload_field", "download_field"):
        f = getattr(lib, pre + nm)
        f.argtypes = head + [_i, _p, C.c_longlong]
        f.restype = None
    getattr(lib, pre + "profile_enable").argtypes = [C.POINTER(chunk_t), _i]
    getattr(lib, pre + "profile_reset").argtypes = [C.POINTER(chunk_t)]
    f = getattr(lib, pre + "profile_read")
    f.argtypes = [C.POINTER(chunk_t), _i, C.c_char_p, _i, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
    f.restype = _i
    f = getattr(lib, pre + "launch_count")
    f.argtypes = [C.POINTER(chunk_t)]
    f.restype = C.c_longlong
    if hasattr(lib, pre + "calculate_2norm_noalloc"):
        f = getattr(lib, pre + "calculate_2norm_noalloc")
        f.argtypes = [_p, _i, _i, _i, _p, _p]
        f.restype = _i
    if hasattr(lib, pre + "solve_step"):
        f = getattr(lib, pre + "solve_step")
        f.argtypes = head + [_i, C.POINTER(StepStats)]
        f.restype = None
    if hasattr(lib, pre + "refine_solve_step"):
        f = getattr(lib, pre + "refine_solve_step")
        f.argtypes = head + [_i, _d, _i, C.POINTER(RefineStats)]
        f.restype = _i
    if hasattr(lib, pre + "flush"):
        f = getattr(lib, pre + "flush")
        f.argtypes = [C.POINTER(chunk_t)]
        f.restype = None
    if hasattr(lib, pre + "set_tma"):  # 2D and 3D
        f = getattr(lib, pre + "set_tma")
        f.argtypes = [C.POINTER(chunk_t), _i]
        f.restype = None
    if hasattr(lib, pre + "set_temporal_blocking"):
        f = getattr(lib, pre + "set_temporal_blocking")
        f.argtypes = [C.POINTER(chunk_t), _i]
        f.restype = None
    if hasattr(lib, pre + "batch_create"):
        lib.tl2d_batch_create.argtypes = [C.POINTER(C.POINTER(chunk_t)), C.POINTER(C.POINTER(settings_t)), _i, _i, _i]
        lib.tl2d_batch_create.restype = _p
        lib.tl2d_batch_destroy.argtypes = [_p]
        lib.tl2d_batch_destroy.restype = None
        lib.tl2d_batch_tune.argtypes = [_p, _i, C.POINTER(_d)]
        lib.tl2d_batch_tune.restype = _i
        lib.tl2d_batch_config.argtypes = [_p, C.POINTER(_i), C.POINTER(_i)]
        lib.tl2d_batch_config.restype = None
        lib.tl2d_batch_step.argtypes = [_p, C.POINTER(BatchStats)]
        lib.tl2d_batch_step.restype = _i
        lib.tl2d_batch_results.argtypes = [_p, _p, _p, _p]
        lib.tl2d_batch_results.restype = _i
        if hasattr(lib, "tl2d_batch_set_wait_limit"):
            lib.tl2d_batch_set_wait_limit.argtypes = [_p, C.c_longlong]
            lib.tl2d_batch_set_wait_limit.restype = _i
    if hasattr(lib, pre + "set_preconditioner"):
        f = getattr(lib, pre + "set_preconditioner")
        f.argtypes = [C.POINTER(chunk_t), _i]
        f.restype = _i
    if hasattr(lib, pre + "check_bounded_wait"):
        f = getattr(lib, pre + "check_bounded_wait")
        f.argtypes = [C.POINTER(chunk_t), C.c_longlong]
        f.restype = _i
    if hasattr(lib, pre + "adjoint_gradient"):
        f = getattr(lib, pre + "adjoint_gradient")
        f.argtypes = head + [_i, _i, C.POINTER(_d), _d, _p, C.POINTER(AdjointStats)]
        f.restype = _i
        f = getattr(lib, pre + "solve_step_backward")
        f.argtypes = head + [_p, _p, _p, _p, _d, C.POINTER(_i)]
        f.restype = _i
    if hasattr(lib, "diffuse_overload"):
        lib.diffuse_overload.argtypes = head
        lib.diffuse_overload.restype = None
    # Errors raise Python exceptions instead of exiting the interpreter.
    getattr(lib, pre + "set_error_mode")(1)
    _loaded[dims] = lib
    return lib


class SuiteError(RuntimeError):
    pass


def check(lib: C.CDLL, dims: int):
    """Raise SuiteError if the library recorded an error since the last check."""
    buf = C.create_string_buffer(512)
    code = getattr(lib, "tl%dd_get_error" % dims)(buf, 512)
    if code:
        raise SuiteError("B200 suite error %d: %s" % (code, buf.value.decode(errors="replace")))
