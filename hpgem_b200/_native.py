"""ctypes binding of the C ABI in include/hpgem_b200.h.

The shared library is built in-tree by ``python -m hpgem_b200.build``.  There is
no fallback: if the library is missing or cannot be loaded, importing the
binding raises, and every solver entry point fails loudly.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libhpgem_b200.so")

# enum values of include/hpgem_b200.h
SHAPE_LINE, SHAPE_SQUARE, SHAPE_TRIANGLE, SHAPE_CUBE, SHAPE_TETRAHEDRON = 1, 2, 3, 4, 5
PHYSICS_ADVECTION, PHYSICS_WAVE, PHYSICS_WAVE_UPWIND = 0, 1, 2
PRECISION_FP64, PRECISION_FP32, PRECISION_BF16X3 = 0, 1, 2
ERRORS = {0: "HGG_OK", -1: "HGG_ERR_INVALID", -2: "HGG_ERR_UNSUPPORTED", -3: "HGG_ERR_CUDA",
          -4: "HGG_ERR_NOMEM", -5: "HGG_ERR_DEVICE", -6: "HGG_ERR_NOT_LOADED"}

# every symbol include/hpgem_b200.h declares (checked by the CPU tests)
EXPORTED = ["hgg_create", "hgg_destroy", "hgg_last_error", "hgg_set_state", "hgg_get_state",
            "hgg_step", "hgg_time_derivative", "hgg_synchronize", "hgg_vector_length",
            "hgg_kernel_kind", "hgg_set_store_last_stage", "hgg_set_stream", "hgg_set_kernel_variant", "hgg_launch_count",
            "hgg_test_arm_without_copy", "hgg_set_element_source", "hgg_set_boundary_source",
            "hgg_time_derivative_at",
            "hgg_create_structured", "hgg_structured_descriptor", "hgg_free_descriptor",
            "hgg_create_mesh_file", "hgg_mesh_file_descriptor",
            "hgg_create_linear", "hgg_linear_descriptor", "hgg_free_linear_descriptor",
            "hgg_create_linear_structured", "hgg_create_linear_mesh_file",
            "hgg_quadrature_points", "hgg_num_quadrature_points",
            "hgg_project", "hgg_num_error_points", "hgg_error_points", "hgg_l2_error", "hgg_max_error",
            "hgg_time_derivative_static", "hgg_step_adaptive", "hgg_set_error_estimate",
            "hgg_batch_create", "hgg_batch_destroy", "hgg_batch_last_error", "hgg_batch_add",
            "hgg_batch_remove", "hgg_batch_step", "hgg_batch_synchronize", "hgg_batch_remaining",
            "hgg_batch_set_autotune", "hgg_batch_launch_count", "hgg_batch_num_classes",
            "hgg_batch_class_info", "hgg_batch_profile_step", "hgg_batch_stream",
            "hgg_server_start", "hgg_server_submit", "hgg_server_poll", "hgg_server_result_length",
            "hgg_server_release", "hgg_server_times", "hgg_server_stats", "hgg_server_timing",
            "hgg_server_last_error",
            "hgg_server_stop"]

# void (*hgg_source_fn)(const double *xyz, const double *normals, int64_t n_points, int32_t dim,
#                       double time, double *values, void *user)
SOURCE_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int64,
                             ctypes.c_int32, ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)

# void (*hgg_initial_fn)(const double *xyz, int64_t n_points, int32_t dim, double *values, void *user)
INITIAL_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_int32,
                              ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


class ProblemDesc(ctypes.Structure):
    """Mirror of struct hgg_problem_desc."""
    _fields_ = [
        ("dim", ctypes.c_int32), ("shape", ctypes.c_int32), ("order", ctypes.c_int32),
        ("n_vars", ctypes.c_int32), ("physics", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("advection", ctypes.c_double * 3), ("c_inv", ctypes.c_double),
        ("n_elements", ctypes.c_int64), ("n_basis", ctypes.c_int32),
        ("n_quad", ctypes.c_int32), ("quad_weights", ctypes.c_void_p),
        ("basis_values", ctypes.c_void_p), ("basis_grads", ctypes.c_void_p),
        ("n_face_quad", ctypes.c_int32), ("face_weights", ctypes.c_void_p),
        ("n_face_tabs", ctypes.c_int32), ("face_tabs", ctypes.c_void_p),
        ("jacobians", ctypes.c_void_p),
        ("n_faces", ctypes.c_int64), ("face_elements", ctypes.c_void_p),
        ("face_local", ctypes.c_void_p), ("face_tab_index", ctypes.c_void_p),
        ("face_normals", ctypes.c_void_p),
        ("n_stages", ctypes.c_int32), ("rk_a", ctypes.c_void_p), ("rk_b", ctypes.c_void_p),
        ("rk_c", ctypes.c_void_p),
    ]


class LinearDesc(ctypes.Structure):
    """Mirror of struct hgg_linear_desc."""
    _fields_ = [
        ("n_rows", ctypes.c_int32), ("precision", ctypes.c_int32), ("n_elements", ctypes.c_int64),
        ("mass", ctypes.c_void_p), ("element_stiffness", ctypes.c_void_p),
        ("n_faces", ctypes.c_int64), ("face_elements", ctypes.c_void_p), ("face_stiffness", ctypes.c_void_p),
        ("n_stages", ctypes.c_int32), ("rk_a", ctypes.c_void_p), ("rk_b", ctypes.c_void_p),
        ("rk_c", ctypes.c_void_p),
    ]


class NativeError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, message))
        self.code = code


_lib = None


def load():
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("hpgem_b200 native library not built: %s is missing "
                          "(run python -m hpgem_b200.build)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    P = ctypes.c_void_p
    B = ctypes.c_void_p
    sig = {
        "hgg_create": (ctypes.c_int, [ctypes.POINTER(ProblemDesc), ctypes.POINTER(H)]),
        "hgg_destroy": (ctypes.c_int, [H]),
        "hgg_last_error": (ctypes.c_char_p, [H]),
        "hgg_set_state": (ctypes.c_int, [H, ctypes.c_int32, P]),
        "hgg_get_state": (ctypes.c_int, [H, ctypes.c_int32, P]),
        "hgg_step": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int32]),
        "hgg_time_derivative": (ctypes.c_int, [H, ctypes.c_int32, ctypes.c_int32]),
        "hgg_time_derivative_static": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p]),
        "hgg_test_arm_without_copy": (ctypes.c_int, [H, ctypes.c_int32]),
        "hgg_set_element_source": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p]),
        "hgg_set_boundary_source": (ctypes.c_int, [H, ctypes.c_void_p, ctypes.c_void_p]),
        "hgg_time_derivative_at": (ctypes.c_int, [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]),
        "hgg_step_adaptive": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_double,
                                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_int32)]),
        "hgg_set_error_estimate": (ctypes.c_int, [H, P, ctypes.c_int32]),
        "hgg_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
        "hgg_batch_destroy": (ctypes.c_int, [B]),
        "hgg_batch_last_error": (ctypes.c_char_p, [B]),
        "hgg_batch_add": (ctypes.c_int, [B, H, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
        "hgg_batch_remove": (ctypes.c_int, [B, ctypes.c_int32]),
        "hgg_batch_step": (ctypes.c_int, [B, ctypes.c_int32]),
        "hgg_batch_synchronize": (ctypes.c_int, [B]),
        "hgg_batch_remaining": (ctypes.c_int32, [B, ctypes.c_int32]),
        "hgg_batch_set_autotune": (ctypes.c_int, [B, ctypes.c_int32]),
        "hgg_batch_launch_count": (ctypes.c_int64, [B]),
        "hgg_batch_num_classes": (ctypes.c_int32, [B]),
        "hgg_batch_class_info": (ctypes.c_int, [B, ctypes.c_int32, P]),
        "hgg_batch_profile_step": (ctypes.c_int, [B, P, ctypes.c_int32]),
        "hgg_batch_stream": (ctypes.c_void_p, [B]),
        "hgg_server_start": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_void_p)]),
        "hgg_server_submit": (ctypes.c_int, [B, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P, ctypes.c_int32,
                                             ctypes.c_char_p, ctypes.c_int32, P, ctypes.c_int64, INITIAL_FN, P,
                                             ctypes.c_double, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
        "hgg_server_poll": (ctypes.c_int, [B, ctypes.c_int64, ctypes.c_int32, P, ctypes.c_int64,
                                           ctypes.POINTER(ctypes.c_double)]),
        "hgg_server_result_length": (ctypes.c_int64, [B, ctypes.c_int64]),
        "hgg_server_release": (ctypes.c_int, [B, ctypes.c_int64]),
        "hgg_server_times": (ctypes.c_int, [B, ctypes.c_int64, P]),
        "hgg_server_stats": (ctypes.c_int, [B, P]),
        "hgg_server_timing": (ctypes.c_int, [B, P]),
        "hgg_server_last_error": (ctypes.c_char_p, [B]),
        "hgg_server_stop": (ctypes.c_int, [B]),
        "hgg_synchronize": (ctypes.c_int, [H]),
        "hgg_vector_length": (ctypes.c_int64, [H]),
        "hgg_kernel_kind": (ctypes.c_int, [H]),
        "hgg_set_store_last_stage": (ctypes.c_int, [H, ctypes.c_int32]),
        "hgg_set_stream": (ctypes.c_int, [H, P]),
        "hgg_launch_count": (ctypes.c_int64, [H]),
        "hgg_set_kernel_variant": (ctypes.c_int, [H, ctypes.c_int32]),
        "hgg_create_structured": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                 ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(H)]),
        "hgg_structured_descriptor": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                     ctypes.c_char_p, ctypes.c_int32,
                                                     ctypes.POINTER(ProblemDesc), ctypes.POINTER(H)]),
        "hgg_free_descriptor": (None, [H]),
        "hgg_create_mesh_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(H)]),
        "hgg_mesh_file_descriptor": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                    ctypes.c_char_p, ctypes.c_int32,
                                                    ctypes.POINTER(ProblemDesc), ctypes.POINTER(H)]),
        "hgg_create_linear": (ctypes.c_int, [ctypes.POINTER(LinearDesc), ctypes.POINTER(H)]),
        "hgg_linear_descriptor": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                 ctypes.c_char_p, ctypes.c_int32,
                                                 ctypes.POINTER(LinearDesc), ctypes.POINTER(H)]),
        "hgg_free_linear_descriptor": (None, [H]),
        "hgg_create_linear_structured": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                        ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(H)]),
        "hgg_create_linear_mesh_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, P,
                                                       ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(H)]),
        "hgg_quadrature_points": (ctypes.c_int, [H, P]),
        "hgg_num_quadrature_points": (ctypes.c_int32, [H]),
        "hgg_project": (ctypes.c_int, [H, P, ctypes.c_int32]),
        "hgg_num_error_points": (ctypes.c_int32, [H]),
        "hgg_error_points": (ctypes.c_int, [H, P]),
        "hgg_l2_error": (ctypes.c_int, [H, ctypes.c_int32, P, ctypes.POINTER(ctypes.c_double)]),
        "hgg_max_error": (ctypes.c_int, [H, ctypes.c_int32, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code, handle=None):
    if code != 0:
        msg = load().hgg_last_error(handle)
        raise NativeError(code, msg.decode() if msg else "")
    return code


def check_server(code, server=None):
    if code < 0:
        msg = load().hgg_server_last_error(server)
        raise NativeError(code, msg.decode() if msg else "")
    return code


def check_batch(code, batch=None):
    if code != 0:
        msg = load().hgg_batch_last_error(batch)
        raise NativeError(code, msg.decode() if msg else "")
    return code
