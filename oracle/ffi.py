"""ctypes wrapper of the CPU oracle (oracle/liboracle.so). Test infrastructure only."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p


class F128(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64)]


_SIGS = [
    ("o_gf_mul", F128, [F128, F128]),
    ("o_gf_inv", F128, [F128]),
    ("o_ts_new", _vp, [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t]),
    ("o_ts_delete", None, [_vp]),
    ("o_ts_public", None, [_vp, _vp, ctypes.c_size_t]),
    ("o_ts_prover", None, [_vp, _vp, ctypes.c_size_t]),
    ("o_ts_hint", None, [_vp, _vp, ctypes.c_size_t]),
    ("o_ts_f128", F128, [_vp]),
    ("o_ts_grind", None, [_vp, ctypes.c_char_p, ctypes.c_uint32]),
    ("o_ts_narg", ctypes.c_size_t, [_vp, _vp, ctypes.c_size_t]),
    ("o_post_gkr_prove", ctypes.c_int,
     [_u64p, ctypes.c_int, _u64p, ctypes.c_int, F128, _u64p, ctypes.c_uint32, _vp, _u64p, _u64p]),
    ("o_gkr_prove", F128, [_u64p, _u64p, ctypes.c_int, _u64p, ctypes.c_uint32, _vp, _u64p]),
    ("o_gkr_outputs", None, [_u64p, _u64p, ctypes.c_int, _u64p]),
    ("o_fold_columns", None, [_u64p, ctypes.c_int, _u64p, _u64p]),
    ("o_mt_transpose", None,
     [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), ctypes.c_size_t, _u64p,
      ctypes.c_int, _u64p, _u64p]),
    ("o_set_clmul_mode", None, [ctypes.c_int]),
    ("o_blake3", None, [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]),
    ("o_blake3_derive_key", None,
     [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_char_p]),
]

_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def p64(a):
    return a.ctypes.data_as(_u64p)


def gf_mul(a, b):
    r = lib().o_gf_mul(F128(int(a[0]), int(a[1])), F128(int(b[0]), int(b[1])))
    return np.array([r.lo, r.hi], dtype=np.uint64)


class Transcript:
    def __init__(self, session: bytes, instance: bytes):
        self.h = lib().o_ts_new(session, len(session), instance, len(instance))

    def __del__(self):
        if getattr(self, "h", None):
            lib().o_ts_delete(self.h)
            self.h = None

    def public_message(self, b: bytes):
        lib().o_ts_public(self.h, b, len(b))

    def prover_message(self, b: bytes):
        lib().o_ts_prover(self.h, b, len(b))

    def verifier_message_f128(self):
        r = lib().o_ts_f128(self.h)
        return np.array([r.lo, r.hi], dtype=np.uint64)

    def grind(self, label: bytes, bits: int):
        lib().o_ts_grind(self.h, label, bits)

    def narg(self) -> bytes:
        n = lib().o_ts_narg(self.h, None, 0)
        buf = ctypes.create_string_buffer(max(n, 1))
        lib().o_ts_narg(self.h, buf, n)
        return buf.raw[:n]


def post_gkr_prove(rows, cols, target, packed, grind_bits, ts):
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    lr = rows.shape[0].bit_length() - 1
    lc = cols.shape[0].bit_length() - 1
    point = np.zeros((lr + lc, 2), dtype=np.uint64)
    value = np.zeros(2, dtype=np.uint64)
    rc = lib().o_post_gkr_prove(p64(rows), lr, p64(cols), lc, F128(int(target[0]), int(target[1])),
                                p64(packed), grind_bits, ts.h, p64(point), p64(value))
    return rc, point, value


def gkr_prove(images, cols, zeta, grind_bits, ts):
    images = np.ascontiguousarray(images, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    zeta = np.ascontiguousarray(zeta, dtype=np.uint64)
    s = cols.shape[0].bit_length() - 1
    point = np.zeros((s + 7, 2), dtype=np.uint64)
    claim = lib().o_gkr_prove(p64(images), p64(cols), s, p64(zeta), grind_bits, ts.h, p64(point))
    return point, np.array([claim.lo, claim.hi], dtype=np.uint64)


def gkr_outputs(images, cols):
    images = np.ascontiguousarray(images, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    s = cols.shape[0].bit_length() - 1
    out = np.zeros((1 << s, 2), dtype=np.uint64)
    lib().o_gkr_outputs(p64(images), p64(cols), s, p64(out))
    return out


def weighted_sum(rows, cols, packed):
    L = lib()
    L.o_weighted_sum.restype = F128
    L.o_weighted_sum.argtypes = [_u64p, ctypes.c_int, _u64p, ctypes.c_int, _u64p]
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    lr = rows.shape[0].bit_length() - 1
    lc = cols.shape[0].bit_length() - 1
    r = L.o_weighted_sum(p64(rows), lr, p64(cols), lc, p64(packed))
    return np.array([r.lo, r.hi], dtype=np.uint64)


class Circuit:
    """The oracle's replay of one SHA-256 circuit statement."""

    def __init__(self, kind: int, inputs, expected):
        L = lib()
        L.o_circuit_build.restype = _vp
        L.o_circuit_build.argtypes = [ctypes.c_int, _vp, ctypes.c_size_t, _vp]
        L.o_circuit_free.argtypes = [_vp]
        inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
        expected = np.ascontiguousarray(expected, dtype=np.uint8)
        self.h = L.o_circuit_build(kind, inputs.ctypes.data, inputs.size, expected.ctypes.data)
        sizes = np.zeros(7, dtype=np.uint64)
        L.o_circuit_sizes(ctypes.c_void_p(self.h), sizes.ctypes.data_as(_u64p))
        (self.f_len, self.h_len, self.rows, self.m_nnz, self.a_nnz, self.b_nnz,
         self.c_nnz) = [int(x) for x in sizes]

    def __del__(self):
        if getattr(self, "h", None):
            lib().o_circuit_free(self.h)
            self.h = None

    def _bytes(self, fn, n, dtype=np.uint8):
        out = np.zeros(n, dtype=dtype)
        getattr(lib(), fn)(ctypes.c_void_p(self.h), out.ctypes.data_as(ctypes.c_void_p))
        return out

    def outputs(self):
        return self._bytes("o_circuit_outputs", 256)

    def f(self):
        return self._bytes("o_circuit_f", self.f_len)

    def hbits(self):
        return self._bytes("o_circuit_h", self.h_len)

    def products(self):
        a = np.zeros(self.rows, dtype=np.int64)
        b = np.zeros(self.rows, dtype=np.int64)
        c = np.zeros(self.rows, dtype=np.int64)
        lib().o_circuit_products(ctypes.c_void_p(self.h), a.ctypes.data_as(_vp),
                                 b.ctypes.data_as(_vp), c.ctypes.data_as(_vp))
        return a, b, c

    def m_rows(self):
        off = np.zeros(self.h_len + 1, dtype=np.uint32)
        pos = np.zeros(max(self.m_nnz, 1), dtype=np.uint32)
        lib().o_circuit_m(ctypes.c_void_p(self.h), off.ctypes.data_as(_vp), pos.ctypes.data_as(_vp))
        return off, pos[: self.m_nnz]

    def matrix(self, which):
        nnz = [self.a_nnz, self.b_nnz, self.c_nnz][which]
        off = np.zeros(self.rows + 1, dtype=np.uint32)
        cols = np.zeros(max(nnz, 1), dtype=np.uint32)
        coef = np.zeros(max(nnz, 1), dtype=np.int64)
        lib().o_circuit_matrix(ctypes.c_void_p(self.h), which, off.ctypes.data_as(_vp),
                               cols.ctypes.data_as(_vp), coef.ctypes.data_as(_vp))
        return off, cols[:nnz], coef[:nnz]


def prove(kind: int, inputs, expected, security: int):
    """Runs the oracle's end-to-end prover; returns (status, proof bytes, times)."""
    L = lib()
    L.o_prover_run.restype = _vp
    L.o_prover_run.argtypes = [ctypes.c_int, _vp, ctypes.c_size_t, _vp, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int)]
    L.o_prover_proof.restype = ctypes.c_size_t
    L.o_prover_proof.argtypes = [_vp, _vp, ctypes.c_size_t]
    L.o_prover_times.argtypes = [_vp, _vp]
    L.o_prover_free.argtypes = [_vp]
    inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
    expected = np.ascontiguousarray(expected, dtype=np.uint8)
    st = ctypes.c_int(-1)
    h = L.o_prover_run(kind, inputs.ctypes.data, inputs.size, expected.ctypes.data, security,
                       ctypes.byref(st))
    n = L.o_prover_proof(h, None, 0)
    buf = ctypes.create_string_buffer(max(n, 1))
    L.o_prover_proof(h, buf, n)
    times = np.zeros(3, dtype=np.float64)
    L.o_prover_times(h, times.ctypes.data)
    L.o_prover_free(h)
    return st.value, buf.raw[:n], times


def verify(kind: int, inputs, expected, security: int, proof: bytes) -> int:
    """Runs the oracle's restated verifier; 0 when it accepts, else the code of
    the first failed check."""
    L = lib()
    L.o_verify.restype = ctypes.c_int
    L.o_verify.argtypes = [ctypes.c_int, _vp, ctypes.c_size_t, _vp, ctypes.c_int, ctypes.c_char_p,
                           ctypes.c_size_t]
    inputs = np.ascontiguousarray(inputs, dtype=np.uint8)
    expected = np.ascontiguousarray(expected, dtype=np.uint8)
    return L.o_verify(kind, inputs.ctypes.data, inputs.size, expected.ctypes.data, security,
                      proof, len(proof))
