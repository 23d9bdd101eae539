"""Loader of the in-tree CUDA library libcss_b200.so (C ABI of
include/css_b200.h).  There is no CPU fallback: if the library is missing or
cannot be loaded, every entry point raises."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libcss_b200.so")
_LIB = None

dp = ctypes.POINTER(ctypes.c_double)


class CssError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("css error %d: %s" % (code, msg))
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBPATH):
            raise CssError(-1, "CUDA library %s not built (run __graft_entry__.build())" % LIBPATH)
        L = ctypes.CDLL(LIBPATH)
        L.css_last_error.restype = ctypes.c_char_p
        L.css_create.argtypes = [ctypes.c_void_p, dp, ctypes.POINTER(ctypes.c_void_p)]
        L.css_destroy.argtypes = [ctypes.c_void_p]
        L.css_destroy.restype = None
        L.css_upload_state.argtypes = [ctypes.c_void_p, dp]
        L.css_download_state.argtypes = [ctypes.c_void_p, dp]
        L.css_step_rk4.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.css_step_rk4_host.argtypes = [ctypes.c_void_p, dp, ctypes.c_double, ctypes.c_int]
        L.css_rhs.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_int]
        L.css_diffusion.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.css_deriv.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, ctypes.c_int]
        L.css_deriv_dev.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.css_dbyd1_dt0.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.css_compact_lines.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, dp, dp, dp, dp, ctypes.c_double, ctypes.c_double]
        L.css_sync.argtypes = [ctypes.c_void_p]
        L.css_state_device_ptr.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.css_kernel_launches.argtypes = [ctypes.c_void_p]
        L.css_kernel_launches.restype = ctypes.c_longlong
        L.css_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.css_compact_lines_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        L.css_profile.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.css_kernel_stats.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
        L.css_scalars.argtypes = [ctypes.c_void_p, dp]
        L.css_step_size.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.css_shell_averages.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, dp, dp]
        L.css_spectrum.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.css_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.css_checkpoint_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double]
        L.css_checkpoint_read.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.css_set_tiles.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.css_set_fused.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.css_dbydp_cyclic.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_int]
        L.css_deriv_adjoint_dev.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.css_dbydp_cyclic_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p]
        L.css_get_fused.argtypes = [ctypes.c_void_p]
        L.css_set_curl_pass.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.css_ensemble_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p)]
        L.css_ensemble_step.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        L.css_ensemble_launches.argtypes = [ctypes.c_void_p]
        L.css_ensemble_launches.restype = ctypes.c_longlong
        L.css_ensemble_last_ms.argtypes = [ctypes.c_void_p]
        L.css_ensemble_last_ms.restype = ctypes.c_double
        L.css_ensemble_destroy.argtypes = [ctypes.c_void_p]
        L.css_ensemble_destroy.restype = None
        vp, ll, fp = ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_float)
        L.css_set_sld_speed2.argtypes = [vp, vp]
        L.css_box_filter.argtypes = [vp, ctypes.c_int, vp, vp]
        L.css_closure_scales.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, fp]
        L.css_closure_features.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.css_closure_targets.argtypes = [ll, vp, vp, vp]
        L.css_closure_speed2.argtypes = [ll, vp, vp, vp]
        L.css_closure_speed2_shaped.argtypes = [vp, vp, vp, vp]
        L.css_restrict_state.argtypes = [vp, vp, ctypes.c_int, vp, vp]
        L.css_prolong_add.argtypes = [vp, vp, ctypes.c_int, vp]
        L.css_mlp_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                     ctypes.POINTER(vp)]
        L.css_mlp_destroy.argtypes = [vp]
        L.css_mlp_destroy.restype = None
        L.css_mlp_dims.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.css_mlp_forward.argtypes = [vp, vp, ll, vp]
        L.css_mlp_train_step.argtypes = [vp, vp, vp, ll, ctypes.c_float, fp]
        L.css_mlp_params.argtypes = [vp, ctypes.c_int, fp, fp, ctypes.c_int]
        L.css_mlp_grads.argtypes = [vp, ctypes.c_int, fp, fp]
        L.css_mlp_set_stream.argtypes = [vp, vp]
        L.css_mlp_set_fused.argtypes = [vp, ctypes.c_int]
        L.css_download_plane.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.css_bound.argtypes = [vp, dp]
        for nm in ("css_dbydr", "css_d2bydr2", "css_dbydt", "css_d2bydt2"):
            getattr(L, nm).argtypes = [vp, dp, dp, dp, dp, ctypes.c_int]
        for nm in ("css_dbydp", "css_d2bydp2"):
            getattr(L, nm).argtypes = [vp, dp, dp, ctypes.c_int]
        L.css_deriv_pencils.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        dp, dp, dp, dp, ctypes.c_int]
        L.css_set_clock.argtypes = [vp, ll, ctypes.c_double, ctypes.c_double]
        L.css_get_clock.argtypes = [vp, ctypes.POINTER(ll), dp]
        L.css_inout_init.argtypes = [vp]
        L.css_inout_state.argtypes = [vp, dp]
        L.css_set_rain_fields.argtypes = [vp, dp, dp]
        L.css_get_rain_fields.argtypes = [vp, dp, dp]
        L.css_build_squalls.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.css_add_squalls.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.css_build_lanes.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        ip = ctypes.POINTER(ctypes.c_int)
        L.css_voronoi.argtypes = [ctypes.c_int, dp, dp, ip, ip, ip, ip, dp]
        L.css_set_ash_slices.argtypes = [vp, dp, dp, ctypes.c_double]
        _LIB = L
    return _LIB


def check(rc):
    if rc != 0:
        raise CssError(rc, lib().css_last_error().decode())
    return rc


# exported symbols that include/css_b200.h declares
EXPORTS = [
    "css_last_error", "css_create", "css_destroy", "css_upload_state", "css_download_state", "css_step_rk4",
    "css_step_rk4_host", "css_rhs", "css_diffusion", "css_deriv", "css_deriv_dev", "css_dbyd1_dt0",
    "css_compact_lines", "css_checkpoint_write", "css_checkpoint_read", "css_sync", "css_state_device_ptr", "css_kernel_launches", "css_set_stream",
    "css_profile", "css_kernel_stats", "css_compact_lines_noalloc", "css_scalars", "css_step_size",
    "css_shell_averages", "css_spectrum", "css_autotune", "css_set_tiles", "css_set_fused", "css_get_fused", "css_set_curl_pass", "css_dbydp_cyclic", "css_dbydp_cyclic_dev", "css_deriv_adjoint_dev", "css_ensemble_create", "css_ensemble_step",
    "css_ensemble_launches", "css_ensemble_last_ms", "css_ensemble_destroy", "css_set_sld_speed2", "css_box_filter",
    "css_closure_scales", "css_closure_features", "css_closure_targets", "css_closure_speed2",
    "css_closure_speed2_shaped", "css_restrict_state", "css_prolong_add", "css_mlp_create",
    "css_mlp_destroy", "css_mlp_dims", "css_mlp_forward", "css_mlp_train_step", "css_mlp_params", "css_mlp_grads",
    "css_mlp_set_stream", "css_mlp_set_fused", "css_set_clock", "css_get_clock", "css_inout_init",
    "css_inout_state", "css_set_rain_fields", "css_get_rain_fields", "css_build_squalls", "css_add_squalls",
    "css_build_lanes", "css_voronoi",
    "css_set_ash_slices", "css_download_plane", "css_dbydr", "css_d2bydr2", "css_dbydt", "css_d2bydt2",
    "css_dbydp", "css_d2bydp2", "css_bound", "css_deriv_pencils",
]
