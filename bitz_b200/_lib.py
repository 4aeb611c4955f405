"""ctypes binding of libbitz_b200.so (the C ABI declared in include/bitz_b200.h).

The library is built in-tree by ``make -C bitz_b200`` (or ``__graft_entry__.build()``).
Loading fails loudly when it is missing: there is no fallback implementation.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbitz_b200.so")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p

# (name, restype, argtypes) for every exported entry point.
SIGNATURES = [
    ("bitz_last_error", ctypes.c_char_p, []),
    ("bitz_device_count", ctypes.c_int, []),
    ("bitz_set_device", ctypes.c_int, [ctypes.c_int]),
    ("bitz_transcript_new", _vp, [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t]),
    ("bitz_transcript_free", None, [_vp]),
    ("bitz_transcript_public", ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    ("bitz_transcript_prover", ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    ("bitz_transcript_hint", ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    ("bitz_transcript_challenge_f128", ctypes.c_int, [_vp, _u64p]),
    ("bitz_transcript_grind", ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint32]),
    ("bitz_transcript_prime", ctypes.c_int, [_vp, ctypes.c_uint32, _u8p]),
    ("bitz_transcript_narg", ctypes.c_size_t, [_vp, _u8p, ctypes.c_size_t]),
    ("bitz_transcript_hints", ctypes.c_size_t, [_vp, _u8p, ctypes.c_size_t]),
    ("bitz_post_gkr_prove", ctypes.c_int,
     [_u64p, ctypes.c_int, _u64p, ctypes.c_int, _u64p, _u64p, ctypes.c_uint32, _vp, _u64p, _u64p]),
    ("bitz_post_gkr_prove_dev", ctypes.c_int,
     [_vp, ctypes.c_int, _vp, ctypes.c_int, _u64p, _vp, ctypes.c_uint32, _vp, _u64p, _u64p]),
    ("bitz_post_gkr_prove_noalloc", ctypes.c_int,
     [_vp, ctypes.c_int, _vp, ctypes.c_int, _u64p, _vp, ctypes.c_uint32, _vp, _vp, _u64p, _u64p]),
    ("bitz_gkr_prove", ctypes.c_int,
     [_u64p, _u64p, ctypes.c_int, _u64p, ctypes.c_uint32, _vp, _u64p, _u64p]),
    ("bitz_gkr_prove_dev", ctypes.c_int,
     [_vp, _vp, ctypes.c_int, _u64p, ctypes.c_uint32, _vp, _u64p, _u64p]),
    ("bitz_gkr_outputs", ctypes.c_int, [_u64p, _u64p, ctypes.c_int, _u64p]),
    ("bitz_system_new", ctypes.c_int,
     [ctypes.c_int, _vp, ctypes.c_size_t, _vp, ctypes.c_uint32, ctypes.POINTER(_vp)]),
    ("bitz_system_free", None, [_vp]),
    ("bitz_system_stats", ctypes.c_int, [_vp, _u64p]),
    ("bitz_system_prove", ctypes.c_int,
     [_vp, ctypes.POINTER(_u8p), ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_double)]),
    ("bitz_system_prove_ex", ctypes.c_int,
     [_vp, ctypes.c_int, ctypes.POINTER(_u8p), ctypes.POINTER(ctypes.c_size_t),
      ctypes.POINTER(ctypes.c_double)]),
    ("bitz_free", None, [_vp]),
    ("bitz_witness", ctypes.c_int, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    ("bitz_commit", ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    ("bitz_prove", ctypes.c_int,
     [_vp, _vp, _vp, ctypes.POINTER(_u8p), ctypes.POINTER(ctypes.c_size_t)]),
    ("bitz_witness_free", None, [_vp]),
    ("bitz_verify", ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    ("bitz_wire_decode", ctypes.c_int, [_vp, ctypes.c_size_t, _u64p]),
    ("bitz_blake3", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, _u8p]),
    ("bitz_committed_witness_free", None, [_vp]),
    ("bitz_launch_count", ctypes.c_ulonglong, []),
    ("bitz_resident_rounds", ctypes.c_int, []),
    ("bitz_round_wait_stats", ctypes.c_int, [ctypes.POINTER(ctypes.c_ulonglong)]),
    ("bitz_gate_stats", ctypes.c_int, [ctypes.POINTER(ctypes.c_ulonglong)]),
    ("bitz_system_witness", ctypes.c_int,
     [_vp, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t]),
    ("bitz_circuit_layout", ctypes.c_int,
     [ctypes.c_int, ctypes.c_size_t, _u64p, _u8p, _vp, _vp, _vp, _vp, _vp]),
    ("bitz_statement_digest", ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_size_t, _vp, _u8p]),
    ("bitz_batch_prove", ctypes.c_int,
     [_vp, ctypes.c_size_t, ctypes.c_int, _vp, _vp, _vp]),
    ("bitz_server_start", ctypes.c_int,
     [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_vp)]),
    ("bitz_server_submit", ctypes.c_int,
     [_vp, ctypes.c_int, _vp, ctypes.c_size_t, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("bitz_server_poll", ctypes.c_int,
     [_vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_u8p), ctypes.POINTER(ctypes.c_size_t),
      ctypes.POINTER(ctypes.c_double)]),
    ("bitz_server_stats", ctypes.c_int, [_vp, _u64p]),
    ("bitz_server_stop", ctypes.c_int, [_vp]),
    ("bitz_probe_kernel", ctypes.c_int, [ctypes.c_char_p]),
    ("bitz_probe_read", ctypes.c_int,
     [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_ulonglong)]),
    ("bitz_probe_kernels", ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
    ("bitz_l2_flush", ctypes.c_int, []),
    ("bitz_diag_fibers", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]),
    ("bitz_diag_gf_peak", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    ("bitz_diag_round_trip", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
]

_lib = None


def load():
    """Loads the library once and attaches the argument types."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `make -C bitz_b200` or __graft_entry__.build()")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
