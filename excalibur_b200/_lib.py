"""ctypes binding of libexcalibur_b200.so (include/bbtsvd_b200.h).

The library is built in-tree by ``make -C excalibur_b200`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing, importing this module raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libexcalibur_b200.so")

BBT_OK = 0
STATUS = {0: "BBT_OK", 1: "BBT_ERR_ARG", 2: "BBT_ERR_CUDA", 3: "BBT_ERR_COUNT", 4: "BBT_ERR_NOMEM",
          5: "BBT_ERR_TIMEOUT", 6: "BBT_ERR_UNSUPPORTED", 7: "BBT_ERR_NUMERIC", 8: "BBT_ERR_IO"}

# Every extern "C" symbol declared in include/bbtsvd_b200.h.
EXPORTS = (
    "bbt_create", "bbt_destroy", "bbt_set_stream", "bbt_synchronize", "bbt_last_error",
    "bbt_status_string", "bbt_kernel_launches", "bbt_negative_count", "bbt_bisection",
    "bbt_twisted_vectors", "bbt_bidiagonal_svd", "bbt_givens_mask", "bbt_block_shift_mask",
    "bbt_local_qr", "bbt_fedsvd_run", "bbt_fedsvd_run_host", "bbt_fedsvd_run_files", "bbt_fedsvd_stage_ms",
    "bbt_dgemm", "bbt_profile", "bbt_profile_get", "bbt_twisted_vectors_noalloc",
    "bbt_svd_dense", "bbt_fedsvd_tune", "bbt_rademacher", "bbt_sketch_bf16x3", "bbt_mixed_local_qr",
    "bbt_mlp_param_count", "bbt_mlp_features", "bbt_mlp_forward", "bbt_mlp_grad", "bbt_mlp_adam",
    "bbt_mlp_brackets", "bbt_bisection_bracketed", "bbt_set_bracket_model", "bbt_bisection_stats", "bbt_gebrd",
    "bbt_dgemm_ozaki", "bbt_dgemm_crt", "bbt_gram_dd", "bbt_exact_local_qr", "bbt_exact_apply_q",
)
PROF_CLASSES = ("dgemm", "panel", "mask", "ralha", "bisect", "twisted", "sketch", "chol", "ozaki", "crt", "crt_prep",
                "crt_combine", "dd")


class FedSVDConfig(C.Structure):
    _fields_ = [
        ("participants", C.c_int),
        ("m", C.c_size_t),
        ("local_n", C.POINTER(C.c_size_t)),
        ("public_seed", C.c_uint),
        ("private_seeds", C.POINTER(C.c_uint)),
        ("top_k", C.c_int),
        ("svd_mode", C.c_int),
        ("precision", C.c_int),
        ("labels", C.c_void_p),
    ]


_lib = None


def load():
    """Load the library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise OSError(f"{LIBPATH} is missing: build it with `make -C excalibur_b200` "
                      "(there is no CPU fallback)")
    L = C.CDLL(LIBPATH)
    vp, i, st, d, u = C.c_void_p, C.c_int, C.c_size_t, C.c_double, C.c_uint
    sig = {
        "bbt_create": ([C.POINTER(vp), i], i),
        "bbt_destroy": ([vp], i),
        "bbt_set_stream": ([vp, vp], i),
        "bbt_synchronize": ([vp], i),
        "bbt_last_error": ([vp], C.c_char_p),
        "bbt_status_string": ([i], C.c_char_p),
        "bbt_kernel_launches": ([vp], C.c_uint64),
        "bbt_negative_count": ([vp, i, vp, vp, vp, i, vp], i),
        "bbt_bisection": ([vp, i, vp, vp, d, d, d, i, vp, C.POINTER(i)], i),
        "bbt_twisted_vectors": ([vp, i, i, vp, vp, vp, vp, vp], i),
        "bbt_bidiagonal_svd": ([vp, i, vp, vp, vp, vp, vp, i], i),
        "bbt_givens_mask": ([vp, st, st, st, vp, i, i, u], i),
        "bbt_block_shift_mask": ([vp, st, st, st, vp, i, i, u], i),
        "bbt_local_qr": ([vp, st, st, vp, vp, i], i),
        "bbt_fedsvd_run": ([vp, C.POINTER(FedSVDConfig), vp, vp, vp, vp, C.POINTER(i)], i),
        "bbt_fedsvd_run_host": ([vp, C.POINTER(FedSVDConfig), vp, vp, vp, vp, C.POINTER(i)], i),
        "bbt_fedsvd_run_files": ([vp, C.POINTER(FedSVDConfig), C.c_char_p, vp, vp, vp, C.POINTER(i)], i),
        "bbt_fedsvd_stage_ms": ([vp, vp, i], i),
        "bbt_dgemm": ([vp, i, i, i, i, C.c_long, d, vp, C.c_long, vp, C.c_long, d, vp, C.c_long], i),
        "bbt_profile": ([vp, i], i),
        "bbt_svd_dense": ([vp, i, vp, i, vp, vp, vp, C.POINTER(i)], i),
        "bbt_fedsvd_tune": ([vp, C.POINTER(FedSVDConfig), C.POINTER(i), C.POINTER(i), C.POINTER(d)], i),
        "bbt_twisted_vectors_noalloc": ([vp, i, i, vp, vp, vp, vp, vp], i),
        "bbt_profile_get": ([vp, i, C.POINTER(d), C.POINTER(C.c_uint64), C.POINTER(d)], i),
        "bbt_rademacher": ([vp, i, st, C.c_ulonglong, vp], i),
        "bbt_sketch_bf16x3": ([vp, i, st, vp, i, vp, vp], i),
        "bbt_mixed_local_qr": ([vp, st, st, vp, vp, vp], i),
        "bbt_mlp_param_count": ([], i),
        "bbt_mlp_features": ([vp, i, vp, vp, i, vp], i),
        "bbt_mlp_forward": ([vp, i, vp, vp, vp], i),
        "bbt_mlp_grad": ([vp, i, vp, vp, vp, vp, vp], i),
        "bbt_mlp_adam": ([vp, vp, vp, vp, vp, d, i], i),
        "bbt_mlp_brackets": ([vp, i, vp, vp, i, vp, d, vp], i),
        "bbt_bisection_bracketed": ([vp, i, vp, vp, d, d, d, i, vp, vp, C.POINTER(i), C.POINTER(C.c_longlong)], i),
        "bbt_set_bracket_model": ([vp, vp, d], i),
        "bbt_bisection_stats": ([vp, C.POINTER(C.c_longlong)], i),
        "bbt_gebrd": ([vp, i, vp, vp, vp], i),
        "bbt_dgemm_ozaki": ([vp, i, i, i, i, C.c_long, d, vp, C.c_long, vp, C.c_long, d, vp, C.c_long, i], i),
        "bbt_dgemm_crt": ([vp, i, i, C.c_long, d, vp, C.c_long, vp, C.c_long, d, vp, C.c_long, i], i),
        "bbt_gram_dd": ([vp, i, C.c_long, vp, C.c_long, vp, vp], i),
        "bbt_exact_local_qr": ([vp, i, st, vp, vp, vp, vp, vp], i),
        "bbt_exact_apply_q": ([vp, i, st, vp, C.c_long, vp, vp, vp, i, vp, C.c_long], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L
