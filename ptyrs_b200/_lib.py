"""ctypes binding of `libptyb200.so` (include/ptyb200.h). Loading fails loudly when the library
is not built: there is no fallback path."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libptyb200.so")

c_int32, c_int64, c_double, c_void_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
P = ctypes.POINTER


class Scan(ctypes.Structure):
    _fields_ = [("nframe", c_int32), ("ny", c_int32), ("nx", c_int32), ("counts_kind", c_int32),
                ("counts", c_void_p), ("pos_y", P(c_double)), ("pos_x", P(c_double)),
                ("wavelength", c_double), ("distance", c_double), ("detector_pixel", c_double)]


class Options(ctypes.Structure):
    _fields_ = [("device", c_int32), ("stack_size", c_int32), ("cluster", c_int32)]


class RpieParams(ctypes.Structure):
    _fields_ = [("update_object", c_int32), ("update_probe", c_int32), ("obj_step", c_double),
                ("probe_step", c_double), ("obj_alpha", c_double), ("probe_alpha", c_double),
                ("batch_size", c_int32), ("calc_llk", c_int32), ("seed", ctypes.c_uint64)]


class LsqmlParams(ctypes.Structure):
    _fields_ = [("batch_size", c_int32), ("cost", c_int32), ("seed", ctypes.c_uint64)]


class ApParams(ctypes.Structure):
    _fields_ = [("update_object", c_int32), ("update_probe", c_int32),
                ("obj_inertia", c_double), ("probe_inertia", c_double), ("calc_llk", c_int32),
                ("zero_phase_ramp", c_int32)]


class DmParams(ctypes.Structure):
    _fields_ = [("update_object", c_int32), ("update_probe", c_int32),
                ("obj_inertia", c_double), ("probe_inertia", c_double), ("alpha", c_double),
                ("loop_obj_probe", c_int32), ("calc_llk", c_int32), ("zero_phase_ramp", c_int32)]


class RaarParams(ctypes.Structure):
    _fields_ = [("update_object", c_int32), ("update_probe", c_int32),
                ("obj_inertia", c_double), ("probe_inertia", c_double), ("beta", c_double),
                ("loop_obj_probe", c_int32), ("calc_llk", c_int32), ("zero_phase_ramp", c_int32)]


class MlParams(ctypes.Structure):
    _fields_ = [("update_object", c_int32), ("update_probe", c_int32), ("calc_llk", c_int32),
                ("zero_phase_ramp", c_int32)]


class Llk(ctypes.Structure):
    _fields_ = [("poisson", c_double), ("gaussian", c_double), ("euclidian", c_double),
                ("nb_photons_calc", c_double)]


class LlkRecord(ctypes.Structure):
    _fields_ = [("cycle", c_int64), ("algorithm", c_int32), ("pad_", c_int32), ("llk", Llk)]


class LsqmlStep(ctypes.Structure):
    _fields_ = [("batch", c_int32), ("frame", c_int32), ("a_far", c_double), ("a_obj", c_double),
                ("a_probe", c_double)]


class BhParams(ctypes.Structure):
    _fields_ = [("batch_size", c_int32), ("pad_", c_int32), ("probe_rho", c_double),
                ("position_rho", c_double), ("seed", ctypes.c_uint64)]


class BhStep(ctypes.Structure):
    _fields_ = [("batch", c_int32), ("count", c_int32), ("beta", c_double), ("alpha", c_double),
                ("top", c_double), ("bottom", c_double)]


class LiveParams(ctypes.Structure):
    _fields_ = [("device", c_int32), ("n", c_int32), ("counts_kind", c_int32), ("slots", c_int32),
                ("capacity", c_int32), ("batch", c_int32), ("wavelength", c_double),
                ("distance", c_double), ("detector_pixel", c_double), ("pos_wait_ns", c_int64)]


class LiveStats(ctypes.Structure):
    _fields_ = [(k, c_int64) for k in ("committed", "landed", "ready", "dropped_no_position",
                                       "dropped_crowded", "dropped_invalid", "dropped_full",
                                       "stalls", "pos_waits", "batches")]


class CxiScan(ctypes.Structure):
    _fields_ = [("nframe", c_int32), ("ny", c_int32), ("nx", c_int32), ("pad_", c_int32),
                ("counts", P(ctypes.c_uint16)), ("y", P(c_double)), ("x", P(c_double)),
                ("wavelength", c_double), ("distance", c_double), ("detector_pixel", c_double)]


class Ptyr(ctypes.Structure):
    _fields_ = [("obj_shape", c_int32 * 3), ("probe_shape", c_int32 * 3),
                ("object", P(c_double)), ("probe", P(c_double)), ("psize", c_double * 2),
                ("origin", c_double * 2)]


# Every symbol include/ptyb200.h declares, with (restype, argtypes).
SIGNATURES = {
    "ptyb_create": (c_int32, [P(Scan), P(c_double), c_int32, c_int32, c_int32, P(c_double),
                              c_int32, P(Options), P(c_void_p)]),
    "ptyb_create_slices": (c_int32, [P(Scan), P(c_double), c_int32, P(c_double), c_int32,
                                     c_int32, P(c_double), c_int32, P(Options), P(c_void_p)]),
    "ptyb_nslice": (c_int32, [c_void_p]),
    "ptyb_get_objects": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_set_objects": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_rpie": (c_int32, [c_void_p, P(RpieParams), c_int32]),
    "ptyb_lsqml": (c_int32, [c_void_p, P(LsqmlParams), c_int32, c_int32]),
    "ptyb_ml": (c_int32, [c_void_p, P(MlParams), c_int32]),
    "ptyb_ap": (c_int32, [c_void_p, P(ApParams), c_int32]),
    "ptyb_bh": (c_int32, [c_void_p, P(BhParams), c_int32, c_int32]),
    "ptyb_bh_steps_len": (c_int32, [c_void_p]),
    "ptyb_bh_steps": (c_int32, [c_void_p, P(BhStep), c_int32]),
    "ptyb_dm": (c_int32, [c_void_p, P(DmParams), c_int32]),
    "ptyb_raar": (c_int32, [c_void_p, P(RaarParams), c_int32]),
    "ptyb_set_probe_variation": (c_int32, [c_void_p, P(c_double), c_int32, P(c_double), c_int32,
                                           P(c_double), c_int32]),
    "ptyb_get_probe_variation": (c_int32, [c_void_p, P(c_double), P(c_double), P(c_double)]),
    "ptyb_batch_run": (c_int32, [P(c_void_p), c_int32, P(RpieParams), c_int32, P(LsqmlParams),
                                 c_int32, c_int32, P(c_int32), P(ctypes.c_float)]),
    "ptyb_get_llk": (c_int32, [c_void_p, P(Llk)]),
    "ptyb_gradients": (c_int32, [c_void_p, P(c_double), P(c_double), P(c_double),
                                 P(c_double)]),
    "ptyb_forward_intensity": (c_int32, [c_void_p, P(c_int32), c_int32, P(ctypes.c_float)]),
    "ptyb_forward_intensity_noalloc": (c_int32, [c_void_p, P(c_int32), c_int32,
                                                 P(ctypes.c_float)]),
    "ptyb_set_positions": (c_int32, [c_void_p, P(c_double), c_int32]),
    "ptyb_get_positions": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_live_create": (c_int32, [P(LiveParams), P(c_void_p)]),
    "ptyb_live_reserve": (c_int32, [c_void_p, P(c_int64), P(c_void_p)]),
    "ptyb_live_commit": (c_int32, [c_void_p, c_int64, c_int64]),
    "ptyb_live_position": (c_int32, [c_void_p, c_int64, c_double, c_double]),
    "ptyb_live_flush": (c_int32, [c_void_p, c_int32]),
    "ptyb_live_get_stats": (c_int32, [c_void_p, P(LiveStats)]),
    "ptyb_live_landed": (c_int32, [c_void_p, P(c_int64), P(c_double), P(c_double), c_int32]),
    "ptyb_live_handle": (c_int32, [c_void_p, P(c_double), c_int32, c_int32, P(c_double),
                                   c_int32, P(Options), P(c_void_p), P(c_int32)]),
    "ptyb_live_last_error": (ctypes.c_char_p, [c_void_p]),
    "ptyb_live_destroy": (None, [c_void_p]),
    "ptyb_read_cxi": (c_int32, [ctypes.c_char_p, P(CxiScan)]),
    "ptyb_free_cxi": (None, [P(CxiScan)]),
    "ptyb_read_ptyr": (c_int32, [ctypes.c_char_p, P(Ptyr)]),
    "ptyb_free_ptyr": (None, [P(Ptyr)]),
    "ptyb_io_last_error": (ctypes.c_char_p, []),
    "ptyb_get_object": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_get_probe": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_set_object": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_set_probe": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_set_object_device": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p]),
    "ptyb_set_objects_device": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p]),
    "ptyb_set_probe_device": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_void_p]),
    "ptyb_gradients_device": (c_int32, [c_void_p, P(c_double), c_void_p, c_void_p,
                                        P(c_double)]),
    "ptyb_corners": (c_int32, [c_void_p, P(c_int32)]),
    "ptyb_history_len": (c_int32, [c_void_p]),
    "ptyb_history": (c_int32, [c_void_p, P(LlkRecord), c_int32]),
    "ptyb_cycle": (c_int64, [c_void_p]),
    "ptyb_lsqml_steps_len": (c_int32, [c_void_p]),
    "ptyb_lsqml_steps": (c_int32, [c_void_p, P(LsqmlStep), c_int32]),
    "ptyb_lsqml_slice_steps": (c_int32, [c_void_p, P(c_double)]),
    "ptyb_synchronize": (c_int32, [c_void_p]),
    "ptyb_launches": (c_int64, [c_void_p]),
    "ptyb_random_batches": (c_int32, [c_int32, c_int32, ctypes.c_uint64, ctypes.c_uint64,
                                      P(c_int32)]),
    "ptyb_view_corners": (c_int32, [P(c_double), P(c_double), c_int32, c_double, c_double,
                                    c_int32, c_int32, c_int32, c_int32, P(c_int32)]),
    "ptyb_set_timing": (c_int32, [c_void_p, c_int32]),
    "ptyb_kernel_kinds": (c_int32, []),
    "ptyb_kernel_name": (ctypes.c_char_p, [c_int32]),
    "ptyb_kernel_times": (c_int32, [c_void_p, P(c_double), P(c_int64), c_int32]),
    "ptyb_kernel_frames": (c_int32, [c_void_p, P(c_int64), c_int32]),
    "ptyb_last_call_ms": (c_double, [c_void_p]),
    "ptyb_last_error": (ctypes.c_char_p, [c_void_p]),
    "ptyb_destroy": (None, [c_void_p]),
}

_lib = None


def load():
    """The library with every signature set; raises when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: run `python -m ptyrs_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
