"""ctypes signatures of the C ABI (include/wavemoth.h, include/wavemoth_b200.h)."""
import ctypes

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
# pull_func_t of bfm_transpose_apply_d (src/butterfly.h.in:116-117)
PULL_FUNC = ctypes.CFUNCTYPE(None, _dp, _sz, _sz, _sz, _vp, _sz, _vp)

SIGNATURES = {
    "wavemoth_configure": (None, [ctypes.c_char_p]),
    "wavemoth_plan_to_healpix": (_vp, [ctypes.c_int] * 5 + [_vp, _vp, ctypes.c_int, ctypes.c_uint,
                                                           ctypes.c_char_p]),
    "wavemoth_plan_from_healpix": (_vp, [ctypes.c_int] * 5 + [_vp, _vp, ctypes.c_int, ctypes.c_uint,
                                                             ctypes.c_char_p]),
    "wavemoth_destroy_plan": (None, [_vp]),
    "wavemoth_execute": (None, [_vp]),
    "wavemoth_get_legendre_flops": (ctypes.c_int64, [_vp, ctypes.c_int, ctypes.c_int]),
    "wavemoth_query_resourcefile": (ctypes.c_int, [ctypes.c_char_p, _ip, _ip]),
    "wavemoth_create_healpix_grid_info": (_vp, [ctypes.c_int]),
    "wavemoth_free_grid_info": (None, [_vp]),
    "wavemoth_perform_legendre_transforms": (None, [_vp]),
    "wavemoth_perform_backward_ffts": (None, [_vp]),
    "wavemoth_disable_phase_shifting": (None, [_vp]),
    "wavemoth_last_error": (ctypes.c_char_p, []),
    "wavemoth_plan_status": (ctypes.c_int, [_vp]),
    "wavemoth_plan_device_status": (ctypes.c_int, [_vp, _vp]),
    "wavemoth_batch_create": (_vp, [ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "wavemoth_batch_execute": (ctypes.c_int, [_vp, _vp]),
    "wavemoth_batch_info": (ctypes.c_int, [_vp, _vp, _vp]),
    "wavemoth_batch_transforms": (ctypes.c_int, [_vp]),
    "wavemoth_batch_destroy": (None, [_vp]),
    "wavemoth_batch_create_scheduled": (_vp, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "wavemoth_batch_schedule": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_plan_set_grid_cap": (ctypes.c_int, [_vp, ctypes.c_int]),
    "wavemoth_execute_alm2map_device": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_execute_map2alm_device": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_get_work": (ctypes.c_int, [_vp, _dp]),
    "wavemoth_plan_nmaps": (ctypes.c_int, [_vp]),
    "wavemoth_plan_nside": (ctypes.c_int, [_vp]),
    "wavemoth_plan_lmax": (ctypes.c_int, [_vp]),
    "wavemoth_plan_device_bytes": (ctypes.c_int64, [_vp]),
    "wavemoth_plan_program_bytes": (ctypes.c_int64, [_vp]),
    "wavemoth_plan_image_bytes": (ctypes.c_int64, [_vp]),
    "wavemoth_set_device_memory_cap": (None, [ctypes.c_int64]),
    "wavemoth_plan_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "wavemoth_execute_adjoint": (None, [_vp]),
    "wavemoth_plan_set_ring_weights": (ctypes.c_int, [_vp, _dp]),
    "wavemoth_legendre_alm2map_device": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_legendre_map2alm_device": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_plan_shard": (_vp, [ctypes.c_int] * 4 + [ctypes.c_uint, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    "wavemoth_shard_layout": (ctypes.c_int, [_vp, _vp, _vp]),
    "wavemoth_shard_alm2map_legendre": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_shard_alm2map_rings": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "wavemoth_shard_map2alm_rings": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "wavemoth_shard_map2alm_legendre": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_map2alm_iterative_device": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    # kernel-level hooks (src/legendre_transform.h, src/butterfly.h.in)
    "wavemoth_legendre_transform_auxdata": (None, [_sz, _sz, _sz, _dp]),
    "wavemoth_legendre_transform": (None, [_sz, _sz, _sz, _dp, _dp, _dp, _dp, _dp, _dp]),
    "wavemoth_legendre_transform_sse": (None, [_sz, _sz, _sz, _dp, _dp, _dp, _dp, _dp, _dp, _vp]),
    "wavemoth_legendre_transform_sse_query_work": (_sz, [_sz]),
    "wavemoth_legendre_transform_pack": (None, [_sz, _sz, _dp, _dp]),
    "bfm_create_plan": (_vp, [_sz, _sz, _sz, _vp, _vp]),
    "bfm_destroy_plan": (None, [_vp]),
    "bfm_transpose_apply_d": (ctypes.c_int, [_vp, _vp, PULL_FUNC, _dp, _sz, _vp]),
    "bfm_query_matrix_data": (_vp, [_vp, _vp]),
    "bfm_scatter": (_vp, [_vp, _dp, _dp, _dp, _sz, _sz, _sz, ctypes.c_int, ctypes.c_int]),
    "wavemoth_legendre_alm2map_noalloc": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "wavemoth_plan_timing": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "wavemoth_plan_kernel_launches": (ctypes.c_int64, [_vp]),
    "wavemoth_plan_set_hemisphere_mode": (ctypes.c_int, [_vp, ctypes.c_int]),
    "wavemoth_plan_work": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "wavemoth_check_resourcefile": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.POINTER(ctypes.c_int64)]),
}


class GridInfo(ctypes.Structure):
    """wavemoth_grid_info (include/wavemoth.h; src/wavemoth_private.h:50-65)."""
    _fields_ = [("phi0s", _dp), ("ring_offsets", ctypes.POINTER(ctypes.c_int32)),
                ("nrings", ctypes.c_int32), ("mid_ring", ctypes.c_int32),
                ("npix", ctypes.c_int32), ("has_equator", ctypes.c_int)]


def declare(lib):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib.wavemoth_create_healpix_grid_info.restype = ctypes.POINTER(GridInfo)
    lib.wavemoth_free_grid_info.argtypes = [ctypes.POINTER(GridInfo)]
