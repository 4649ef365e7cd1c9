"""ctypes binding of libvflip_gpu.so (the C ABI declared in include/vflip.h)."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "libvflip_gpu.so"

_P = C.c_void_p
_I = C.c_int
_U32 = C.c_uint32
_F = C.c_float
_D = C.c_double
_SZ = C.c_size_t


class VflipError(RuntimeError):
    """A negative status from the C ABI (argument or CUDA error)."""

    def __init__(self, code, msg):
        super().__init__(f"vflip error {code}: {msg}")
        self.code = code


class SolveStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int), ("vcycles", C.c_int), ("levels", C.c_int), ("converged", C.c_int),
                ("residual", C.c_double), ("rhs_norm", C.c_double), ("solve_ms", C.c_double)]


class ConfigC(C.Structure):
    _fields_ = [("precision", C.c_int), ("pre_sweeps", C.c_int), ("post_sweeps", C.c_int),
                ("coarse_sweeps", C.c_int), ("coarsest_max_unknowns", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p), ("sweep_kernel", C.c_int), ("smoother_depth", C.c_int),
                ("smoother_tile_rows", C.c_int), ("smoother_plane_ranges", C.c_int),
                ("smoother_ctas_per_sm", C.c_int), ("smoother_threads", C.c_int),
                ("smoother_prefetch", C.c_int), ("coarsest_solver", C.c_int), ("spmv_kernel", C.c_int),
                ("pcg_loop", C.c_int), ("pcg_vectors", C.c_int), ("batch_chunk", C.c_int),
                ("batch_ctas_per_sm", C.c_int), ("coarse_tail", C.c_int),
                ("tile_sweep_max_cells", C.c_int), ("p2g_kernel", C.c_int),
                ("advect_kernel", C.c_int)]


class SystemC(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("diag", C.c_void_p), ("xp", C.c_void_p),
                ("yp", C.c_void_p), ("zp", C.c_void_p), ("rhs", C.c_void_p), ("result", C.c_void_p)]


class SubdomainC(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("h", C.c_float), ("bmin", C.c_float * 3),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("nodal_phi", C.c_void_p)]


class LearnedStatsC(C.Structure):
    _fields_ = [("fallback", C.c_int), ("subspace", C.c_int), ("gamma", C.c_double * 4),
                ("init_residual", C.c_double), ("net_ms", C.c_double)]


# name -> (restype, argtypes); mirrors include/vflip.h one for one
SIGNATURES = {
    "vflip_config_default": (None, [C.POINTER(ConfigC)]),
    "vflip_config_size": (C.c_size_t, []),
    "vflip_create": (_I, [C.POINTER(_P), C.POINTER(ConfigC)]),
    "vflip_destroy": (_I, [_P]),
    "vflip_last_error": (C.c_char_p, [_P]),
    "vflip_synchronize": (_I, [_P]),
    "vflip_last_ms": (_D, [_P]),
    "vflip_amgpcg_solve_csr": (_I, [_P, _U32, _P, _P, _P, _P, _P, _D, _I, _P, _P, _I, _I, _I]),
    "vflip_amgpcg_solve": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _D, _I, C.POINTER(SolveStatsC)]),
    "vflip_build_levels": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _I, _P, _P]),
    "vflip_rbgs": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _I]),
    "vflip_vcycle": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "vflip_rbgs_noalloc": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _I]),
    "vflip_face_weights": (_I, [_P, _I, _I, _I, _P, _P, _P, _P]),
    "vflip_assemble": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "vflip_project": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _I,
                           C.POINTER(SolveStatsC)]),
    "vflip_project_subdomain": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _D, _I,
                                     C.POINTER(SolveStatsC)]),
    "vflip_advect_rk2_linear": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _P, _P]),
    "vflip_advect_rk2_linear2": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _P, _P, _P, _P]),
    "vflip_advect_cubic_clamp": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _P, _P]),
    "vflip_advect_velocity_cubic_clamp": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P]),
    "vflip_advect_velocity_rk2_linear": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P]),
    "vflip_advect_rk3_linear": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _P, _P]),
    "vflip_advect_rk3_linear2": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _P, _P, _P,
                                      _P]),
    "vflip_gen_heat": (_I, [_P, _I, _I, _I, _D, _F, _F, _F, _F, _F, _F, _F, _F, _F, _P, _P]),
    "vflip_add_smokeforce": (_I, [_P, _P, _I, _I, _I, _I, _D, _P, _P, _F, _F, _F]),
    "vflip_sub_particle_cells": (_I, [_P, _I, _I, _I, _F, _F, _F, _F, _P, _I, _P]),
    "vflip_sub_p2g": (_I, [_P, _I, _I, _I, _F, _F, _F, _F, _P, _I, _P, _P, _P, _P, _P, _P]),
    "vflip_sub_g2p": (_I, [_P, _I, _I, _I, _F, _F, _F, _F, _P, _I, _P, _P, _P]),
    "vflip_sub_reorder_flip": (_I, [_P, _I, _I, _I, _F, _F, _F, _F, _P, _I, _P, _P, _P, _P, C.c_uint, _P, _I,
                                    C.POINTER(_I)]),
    "vflip_advect_flip_nested": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, C.POINTER(SubdomainC)]),
    "vflip_reorder_flip_nested": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, C.c_uint, _P, _I, C.POINTER(_I),
                                       C.POINTER(SubdomainC)]),
    "vflip_halo_select": (_I, [_P, _P, _I, _F, C.POINTER(SubdomainC), _P, _I, C.POINTER(_I)]),
    "vflip_advect_tracers_nested": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, _F, C.POINTER(SubdomainC)]),
    "vflip_emit_tracers_nested": (_I, [_P, _P, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, C.c_uint, _I, _I, _I, _P,
                                       C.POINTER(SubdomainC), _P, _I, C.POINTER(_I)]),
    "vflip_emit_tracers": (_I, [_P, _P, _I, _F, _F, _F, _F, _F, _F, _F, _F, _I, C.c_uint, _P, _I, C.POINTER(_I)]),
    "vflip_advect_tracers": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F, _F]),
    "vflip_write_tracers": (_I, [_P, _P, _I, _F, C.c_char_p, _I]),
    "vflip_delta": (_I, [_P, _SZ, _P, _P, _P]),
    "vflip_particle_cells": (_I, [_P, _I, _I, _I, _F, _P, _I, _P]),
    "vflip_p2g": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _P, _P]),
    "vflip_advect_flip": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _F]),
    "vflip_reorder_flip": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, C.c_uint, _P, _I, C.POINTER(_I)]),
    "vflip_g2p": (_I, [_P, _I, _I, _I, _F, _P, _I, _P, _P, _P, _P, _P, _P, _D]),
    "vflip_set_profiling": (_I, [_P, _I]),
    "vflip_profile_sweeps": (_I, [_P, C.POINTER(_I), C.POINTER(_D), C.POINTER(_D)]),
    "vflip_profile_kernels": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_D)]),
    "vflip_launch_count": (C.c_ulonglong, [_P]),
    "vflip_plume_sources": (_I, [_P, _I, _I, _I, _F, _F, _P, _P, _P, _F, _F, _F, _F, _F, _F, _F, _F]),
    "vflip_bricks_to_linear": (_I, [_P, _I, _I, _I, _P, _P]),
    "vflip_linear_to_bricks": (_I, [_P, _I, _I, _I, _P, _P]),
    "vflip_unet_create": (_I, [C.POINTER(_P), _I, _P, C.c_ulonglong]),
    "vflip_unet_destroy": (_I, [_P]),
    "vflip_unet_last_error": (C.c_char_p, [_P]),
    "vflip_unet_num_params": (_I, []),
    "vflip_unet_get_params": (_I, [_P, _P]),
    "vflip_unet_set_params": (_I, [_P, _P]),
    "vflip_unet_forward": (_I, [_P, _I, _I, _I, _P, _P]),
    "vflip_unet_gradients": (_I, [_P, _I, _I, _I, _P, _P, _P, _F, _F, _P, C.POINTER(_D)]),
    "vflip_unet_train_step": (_I, [_P, _I, _I, _I, _P, _P, _P, _F, _F, _F, C.POINTER(_D)]),
    "vflip_unet_conv3": (_I, [_P, _I, _I, _I, _P, _I, _I, _P, _I, _I, _I, _P, _I, _P, _I, _I, _P, _I, _I, _P, _I,
                              _I]),
    "vflip_unet_conv3_wgrad": (_I, [_P, _I, _I, _I, _P, _I, _I, _I, _P, _I, _I, _I, _P]),
    "vflip_unet_launch_count": (C.c_longlong, [_P]),
    "vflip_unet_set_output_scale": (_I, [_P, _F, _F]),
    "vflip_batched_solve": (_I, [_P, _I, C.POINTER(SystemC), _D, _I, _I, C.POINTER(SolveStatsC)]),
    "vflip_learned_grid": (_I, [_I, _I, _I, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "vflip_project_learned": (_I, [_P, _P, _I, _I, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _I,
                                   _P, _P, _P, C.POINTER(SolveStatsC), C.POINTER(LearnedStatsC)]),
}

_lib = None


def lib_path():
    return os.path.join(HERE, _LIB_NAME)


def load():
    """Load libvflip_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m vflip_b200.build` "
                                "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.vflip_config_size() != C.sizeof(ConfigC):
        raise RuntimeError(f"{path} was built from another include/vflip.h: vflip_config is "
                           f"{lib.vflip_config_size()} bytes there, {C.sizeof(ConfigC)} here")
    _lib = lib
    return lib
