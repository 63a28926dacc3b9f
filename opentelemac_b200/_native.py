"""ctypes binding of libbief_b200.so (the C ABI in include/bief_b200.h).

The library is required: importing a solver entry point without it raises
immediately.  There is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libbief_b200.so")

BIEF_OK = 0
BIEF_ERR_ARGS = -1
BIEF_ERR_BREAKDOWN = -2
BIEF_ERR_NAN = -3
BIEF_ERR_BAD_MESH = -4
BIEF_ERR_UNSUPPORTED = -5
BIEF_ERR_CUDA = -6
BIEF_ERR_DEVICE_TIMEOUT = -7
BIEF_ERR_NO_MATRIX = -8
BIEF_ERR_SIZE = -9

BIEF_SOLVE_MUTATE_INPUTS = 1
BIEF_SOLVE_INFOGR = 2
BIEF_SOLVE_MODASS3 = 4

# Every symbol include/bief_b200.h declares.
EXPORTS = [
    "bief_mesh_create", "bief_destroy", "bief_set_matrix", "bief_set_matrix_dev",
    "bief_get_matrix", "bief_get_matrix_dev", "bief_solve", "bief_solve_dev",
    "bief_solve_mixed", "bief_solve_mixed_dev", "bief_matvec", "bief_matvec_dev",
    "bief_matvec32_dev", "bief_assemble_wave_dev", "bief_assemble_mass_diff_dev",
    "bief_mass_diff_grad_dev", "bief_wave_coef_grad_dev", "bief_launch_info",
    "bief_matvec_format", "bief_set_blocks_per_sm", "bief_last_timing",
    "bief_kernel_launches", "bief_strerror", "bief_solve_noalloc",
    "bief_batch_solve_mixed_dev", "bief_set_segments", "bief_set_matrix_seg",
    "bief_set_matrix_seg_dev", "bief_ebe_to_seg", "bief_matrix_storage",
    "bief_selftest_timeout", "bief_diri01", "bief_diri01_dev",
]


class SlvCfg(ctypes.Structure):
    """Mirror of TYPE(SLVCFG) (bief_def.f:506-532)."""
    _fields_ = [("slv", ctypes.c_int), ("nitmax", ctypes.c_int), ("precon", ctypes.c_int),
                ("krylov", ctypes.c_int), ("eps", ctypes.c_double), ("zero", ctypes.c_double),
                ("ok", ctypes.c_int), ("nit", ctypes.c_int)]


class BiefError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib().bief_strerror(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({msg})" if what else f"status {status} ({msg})")


_lib = None


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(
                f"libbief_b200.so not found at {LIB}; build it with "
                "`python -m opentelemac_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB)
        vp, i, d, c = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char
        pi, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        pcfg = ctypes.POINTER(SlvCfg)
        sig = {
            "bief_mesh_create": ([i, i, i, vp, i, ctypes.POINTER(vp)], i),
            "bief_destroy": ([vp], i),
            "bief_set_matrix": ([vp, vp, vp, c, c], i),
            "bief_set_matrix_dev": ([vp, vp, vp, c, c], i),
            "bief_get_matrix": ([vp, vp, vp, ctypes.c_char_p], i),
            "bief_get_matrix_dev": ([vp, vp, vp, vp], i),
            "bief_solve": ([vp, vp, vp, pcfg, i, pd], i),
            "bief_solve_dev": ([vp, vp, vp, pcfg, i, pd, vp], i),
            "bief_solve_mixed": ([vp, vp, vp, i, d, d, i, i, pi, pi, pd], i),
            "bief_solve_mixed_dev": ([vp, vp, vp, i, d, d, i, i, pi, pi, pd, vp], i),
            "bief_matvec": ([vp, ctypes.c_char_p, vp, vp, d], i),
            "bief_matvec_dev": ([vp, ctypes.c_char_p, vp, vp, d, vp], i),
            "bief_matvec32_dev": ([vp, vp, vp, vp], i),
            "bief_assemble_mass_diff_dev": ([vp, vp, vp, d, d, i, vp, vp, vp], i),
            "bief_mass_diff_grad_dev": ([vp, vp, vp, d, i, vp, vp, vp, vp, vp, vp, vp], i),
            "bief_assemble_wave_dev": ([vp, vp, vp, vp, vp], i),
            "bief_wave_coef_grad_dev": ([vp, vp, vp, vp, vp, vp, vp], i),
            "bief_launch_info": ([vp, pi, pi], i),
            "bief_matvec_format": ([vp, pi], i),
            "bief_set_blocks_per_sm": ([vp, i], i),
            "bief_last_timing": ([vp, ctypes.POINTER(ctypes.c_float),
                                  ctypes.POINTER(ctypes.c_float)], i),
            "bief_kernel_launches": ([vp], ctypes.c_longlong),
            "bief_strerror": ([i], ctypes.c_char_p),
            "bief_solve_noalloc": ([i, i, i, vp, vp, vp, c, c, vp, vp, pcfg, pd, i, vp], i),
            "bief_batch_solve_mixed_dev": ([vp, i, vp, vp, vp, vp, i, d, d, i, i, i, i, vp, vp,
                                            vp, vp, vp], i),
            "bief_set_segments": ([vp, i, i, vp], i),
            "bief_set_matrix_seg": ([vp, vp, vp, c, c], i),
            "bief_set_matrix_seg_dev": ([vp, vp, vp, c, c], i),
            "bief_ebe_to_seg": ([vp, vp], i),
            "bief_matrix_storage": ([vp], i),
            "bief_selftest_timeout": ([i, ctypes.c_longlong], i),
            "bief_diri01": ([vp, i, vp, vp, i, vp, vp, vp, vp], i),
            "bief_diri01_dev": ([vp, i, vp, vp, i, vp, vp, vp, vp, vp], i),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib
