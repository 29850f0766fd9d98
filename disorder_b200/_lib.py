"""ctypes binding of libdisorder.so (the C ABI in include/disorder.h).

The library is built in-tree by ``python -m disorder_b200.build``. There is no
fallback: if the library or a CUDA device is missing, loading raises.
"""

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# DISORDER_LIB=checks loads the build with the device index checks
# (python -m disorder_b200.build --debug)
LIB_PATH = os.path.join(HERE, "libdisorder_checks.so" if os.environ.get("DISORDER_LIB") == "checks"
                        else "libdisorder.so")

STATUS = {0: "OK", 1: "BAD_ARG", 2: "UNSUPPORTED_FIELD", 3: "OOM", 4: "CUDA_ERR", 5: "TIMEOUT",
          6: "NONFINITE"}


class DisorderError(RuntimeError):
    """A libdisorder call returned a non-OK status (the MEX gateway maps the
    same statuses to MATLAB errors with identifier disorder:<status>)."""

    def __init__(self, status, msg):
        self.status = status
        super().__init__("disorder:%s %s" % (STATUS.get(status, status), msg))


class GridDesc(C.Structure):
    _fields_ = [("N", C.c_int32 * 3), ("rG", C.POINTER(C.c_float) * 3), ("kG", C.POINTER(C.c_float) * 3),
                ("cent", C.c_float * 3)]


class SamplingDesc(C.Structure):
    _fields_ = [("n_seg", C.c_int32), ("n_mot", C.c_int32), ("seg_offsets", C.POINTER(C.c_int64)),
                ("ky", C.POINTER(C.c_int32)), ("kz", C.POINTER(C.c_int32))]


VP = C.c_void_p
FP = C.POINTER(C.c_float)
DP = C.POINTER(C.c_double)
I32 = C.c_int32

# (name, restype, argtypes)
SIGNATURES = [
    ("disorder_ctx_create", C.c_int, [C.c_int, C.POINTER(VP)]),
    ("disorder_ctx_destroy", C.c_int, [VP]),
    ("disorder_last_error", C.c_char_p, [VP]),
    ("disorder_ctx_set_stream", C.c_int, [VP, VP]),
    ("disorder_ctx_get_stream", VP, [VP]),
    ("disorder_synchronize", C.c_int, [VP]),
    ("disorder_malloc", C.c_int, [VP, C.c_size_t, C.POINTER(VP)]),
    ("disorder_free", C.c_int, [VP, VP]),
    ("disorder_memcpy_h2d", C.c_int, [VP, VP, VP, C.c_size_t]),
    ("disorder_memcpy_d2h", C.c_int, [VP, VP, VP, C.c_size_t]),
    ("disorder_memcpy_d2d", C.c_int, [VP, VP, VP, C.c_size_t]),
    ("disorder_memset", C.c_int, [VP, VP, C.c_int, C.c_size_t]),
    ("disorder_upload", C.c_int, [VP, VP, C.c_size_t, C.POINTER(VP)]),
    ("disorder_download", C.c_int, [VP, VP, VP, C.c_size_t]),
    ("disorder_kernel_launches", C.c_int64, [VP]),
    ("disorder_workspace_bytes", C.c_int64, [VP]),
    ("disorder_ctx_inject_fault", C.c_int, [VP, I32]),
    ("disorder_ctx_set_precision", C.c_int, [VP, I32]),
    ("disorder_ctx_set_tuning", C.c_int, [VP, I32, I32]),
    ("disorder_event_record", C.c_int, [VP, I32]),
    ("disorder_event_elapsed", C.c_int, [VP, I32, I32, FP]),
    ("disorder_plan_create", C.c_int, [VP, C.POINTER(GridDesc), C.POINTER(SamplingDesc), C.POINTER(VP)]),
    ("disorder_plan_destroy", C.c_int, [VP]),
    ("disorder_sinc_rigid_transform", C.c_int, [VP, VP, VP, I32, FP, I32, I32, I32, I32, VP]),
    ("disorder_sinc_rigid_transform_static", C.c_int, [VP, VP, VP, I32, FP, I32, I32, I32, VP]),
    ("disorder_precompute_factors", C.c_int, [VP, VP, FP, I32, I32, VP, VP, VP, C.POINTER(C.c_uint8)]),
    ("disorder_sinc_rigid_transform_gradient", C.c_int, [VP, VP, VP, FP, I32, VP, VP]),
    ("disorder_encode", C.c_int, [VP, VP, VP, VP, I32, FP, VP]),
    ("disorder_decode", C.c_int, [VP, VP, VP, VP, I32, FP, VP, VP, VP]),
    ("disorder_encodedecode", C.c_int, [VP, VP, VP, VP, I32, FP, VP, VP]),
    ("disorder_compute_energy", C.c_int, [VP, VP, VP, VP, VP, I32, FP, VP, VP, VP, DP]),
    ("disorder_cg_solve", C.c_int, [VP, VP, VP, VP, I32, FP, VP, VP, VP, VP, VP, VP, VP, I32, I32, I32, C.c_double,
                                    DP, C.POINTER(I32), C.POINTER(I32)]),
    ("disorder_cg_solve_residual", C.c_int, [VP, VP, VP, VP, I32, FP, VP, VP, VP, VP, VP, VP, VP, I32, I32, I32,
                                             C.c_double, DP, C.POINTER(I32), C.POINTER(I32), VP]),
    ("disorder_lm_step", C.c_int, [VP, VP, VP, VP, I32, VP, FP, FP, C.POINTER(C.c_uint8), C.c_float, FP, I32, I32,
                                   DP, DP]),
    ("disorder_resample", C.c_int, [VP, VP, C.POINTER(I32), I32, C.POINTER(I32), VP]),
    ("disorder_gather_samples", C.c_int, [VP, VP, C.c_int64, C.c_int64, VP, C.c_int64, C.c_float, VP]),
    ("disorder_precondition_weights", C.c_int, [VP, VP, I32, C.c_int64, C.c_float, VP]),
    ("disorder_compress_coils", C.c_int, [VP, VP, I32, C.c_int64, VP, C.c_int64, C.c_double, I32, VP, VP,
                                          C.POINTER(I32), DP, DP]),
    ("disorder_state_energies", C.c_int, [VP, VP, VP, VP, I32, VP, FP, I32, I32, DP]),
    ("disorder_sample_energies", C.c_int, [VP, VP, VP, VP, I32, VP, FP, VP, DP]),
    ("disorder_residual_energies", C.c_int, [VP, VP, VP, I32, VP, DP]),
    ("disorder_backproject_states", C.c_int, [VP, VP, VP, VP, I32, VP, FP, I32, I32, VP]),
    ("disorder_synth_phantom", C.c_int, [VP, C.POINTER(I32), I32, FP, I32, FP, I32, VP]),
    ("disorder_synth_coils", C.c_int, [VP, C.POINTER(I32), I32, FP, C.c_float, VP]),
    ("disorder_add_noise", C.c_int, [VP, VP, C.c_int64, C.c_float, C.c_uint64]),
    ("disorder_electrostatic_order", C.c_int, [I32, I32, C.POINTER(C.c_int32)]),
    ("disorder_net_param_count", C.c_int64, []),
    ("disorder_net_create", C.c_int, [VP, C.POINTER(I32), I32, C.POINTER(VP)]),
    ("disorder_net_destroy", C.c_int, [VP]),
    ("disorder_net_set_params", C.c_int, [VP, VP, FP]),
    ("disorder_net_get_params", C.c_int, [VP, VP, FP]),
    ("disorder_net_forward", C.c_int, [VP, VP, VP, VP, I32, C.c_float, C.c_float, VP]),
    ("disorder_net_backward", C.c_int, [VP, VP, VP, I32, VP, DP]),
    ("disorder_net_adam", C.c_int, [VP, VP, VP, C.c_float, C.c_float, C.c_float, C.c_float, I32]),
    ("disorder_propose_motion", C.c_int, [VP, VP, VP, VP, VP, I32, VP, FP, I32, I32, C.c_float, FP]),
    ("disorder_shearlet_create", C.c_int, [VP, C.POINTER(I32), I32, VP, VP, VP, I32, C.POINTER(I32),
                                           C.POINTER(VP)]),
    ("disorder_shearlet_destroy", C.c_int, [VP]),
    ("disorder_shearlet_coefficients", C.c_int, [VP, VP, VP, C.c_float, C.c_float, VP]),
    ("disorder_shearlet_regularize", C.c_int, [VP, VP, VP, VP, C.c_float, C.c_float, VP]),
    ("disorder_shearlet_trace", C.c_int, [VP, VP, VP, VP, DP]),
    ("disorder_trace_probe", C.c_int, [VP, C.c_int64, C.c_uint64, VP, VP]),
    ("disorder_fidelity_trace", C.c_int, [VP, C.POINTER(I32), VP, VP, I32, VP, DP]),
    ("disorder_cg_solve_shearlet", C.c_int, [VP, VP, VP, VP, I32, FP, VP, VP, VP, VP, VP, VP, VP, VP, C.c_float,
                                             VP, I32, I32, I32, C.c_double, DP, C.POINTER(I32),
                                             C.POINTER(I32)]),
]

_lib = None


def load():
    """Load libdisorder.so once and declare the signatures. Raises OSError if
    the library was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("%s not built (run python -m disorder_b200.build%s)"
                          % (LIB_PATH, " --debug" if LIB_PATH.endswith("_checks.so") else ""))
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return [s[0] for s in SIGNATURES]
