"""The product's circuit setup against the oracle's replay (CPU only).

Both follow crates/circuit/src/sha256.rs and tooling/cli/src/circuits.rs; the
oracle also pins the layout counts to the reference's stats test
(crates/circuit/src/sha256.rs:792-813: 6,376 hint bits, 20,456 lifts and 184
rows per compression)."""
import ctypes

import numpy as np
import pytest

from bitz_b200 import _lib
from bitz_b200 import statements as ci
from oracle import ffi as of

CASES = [("sha256-compression", 1), ("sha256-chain", 1), ("sha256-chain", 3),
         ("sha256-block-aligned", 0), ("sha256-block-aligned", 2)]


def product_layout(kind, n_inputs):
    lib = _lib.load()
    sizes = np.zeros(8, dtype=np.uint64)
    dg = (ctypes.c_uint8 * 32)()
    rc = lib.bitz_circuit_layout(kind, n_inputs, sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 dg, None, None, None, None, None)
    assert rc == 0
    f_bits, h_len, rows, m_nnz, c_nnz = (int(x) for x in sizes[:5])
    m_off = np.zeros(h_len + 1, dtype=np.uint32)
    m_pos = np.zeros(m_nnz, dtype=np.uint32)
    c_off = np.zeros(rows + 1, dtype=np.uint32)
    c_col = np.zeros(max(c_nnz, 1), dtype=np.uint32)
    c_coef = np.zeros(max(c_nnz, 1), dtype=np.int64)
    rc = lib.bitz_circuit_layout(kind, n_inputs, sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 dg, m_off.ctypes.data, m_pos.ctypes.data, c_off.ctypes.data,
                                 c_col.ctypes.data, c_coef.ctypes.data)
    assert rc == 0
    return [int(x) for x in sizes], bytes(dg), m_off, m_pos, c_off, c_col[:c_nnz], c_coef[:c_nnz]


def csc_digest(h_len, f_cols, m_off, m_pos):
    """crates/circuit/src/matrix_transpose.rs:424-441 over the CSC of M."""
    counts = np.bincount(m_pos, minlength=f_cols).astype(np.uint32)
    col_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    rows = np.repeat(np.arange(h_len, dtype=np.uint32), np.diff(m_off))
    order = np.lexsort((rows, m_pos))
    row_idx = rows[order].astype(np.uint32)
    data = b"bitz/virtual-map/csc/v1" + np.array([h_len, f_cols, len(row_idx)], dtype="<u8").tobytes()
    data += col_off.astype("<u4").tobytes() + row_idx.astype("<u4").tobytes()
    out = ctypes.create_string_buffer(32)
    of.lib().o_blake3(data, len(data), out)
    return out.raw


@pytest.mark.parametrize("kind,blocks", CASES)
def test_layout_matches_oracle(kind, blocks):
    st = ci.random_state(1) if kind == "sha256-compression" else None
    inp, out, _ = ci.instance(kind, blocks, 5, st)
    oc = of.Circuit(ci.KINDS[kind], inp, out)
    sizes, digest, m_off, m_pos, c_off, c_col, c_coef = product_layout(ci.KINDS[kind], inp.size)
    assert sizes[0] == oc.f_len and sizes[1] == oc.h_len and sizes[2] == oc.rows
    o_off, o_pos = oc.m_rows()
    assert np.array_equal(m_off, o_off) and np.array_equal(m_pos, o_pos)
    oo, ocol, ocoef = oc.matrix(2)
    n_in = inp.size
    rows = oc.rows
    expected = np.concatenate([inp, out])
    for r in range(rows):
        o_entries = list(zip(ocol[oo[r]:oo[r + 1]], ocoef[oo[r]:oo[r + 1]]))
        p_entries = list(zip(c_col[c_off[r]:c_off[r + 1]], c_coef[c_off[r]:c_off[r + 1]]))
        if r < n_in or r >= rows - 256:
            bi = r if r < n_in else n_in + (r - (rows - 256))
            assert p_entries == []
            assert o_entries == ([(0, 1)] if expected[bi] else [])
        else:
            assert p_entries == o_entries, r
    assert digest == csc_digest(oc.h_len, oc.f_len + 1, o_off, o_pos)


def test_per_compression_counts():
    """sha256.rs:45 and 792-813: 6,376 hint bits, 20,456 lifts, 184 rows each."""
    a = product_layout(1, 512 * 2)[0]
    b = product_layout(1, 512 * 3)[0]
    assert b[0] - a[0] == 512 + 6376
    assert b[1] - a[1] == 512 + 20456
    assert b[2] - a[2] == 512 + 184
    # compression statement: 768 inputs + 6,376 hints; 1 + 768 + 20,456 + 256 lifts
    c = product_layout(0, 768)[0]
    assert c[0] == 7144 and c[1] == 21481 and c[2] == 1208


@pytest.mark.parametrize("kind,blocks,seed", [("sha256-compression", 1, 3), ("sha256-chain", 2, 4),
                                              ("sha256-block-aligned", 0, 5),
                                              ("sha256-block-aligned", 3, 6), ("sha256-2kb", 32, 7)])
def test_statement_digest_matches_oracle(kind, blocks, seed):
    """The integer-matrix digest with the statement's bit constants
    (crates/spartan/src/matrix.rs:562-661): the product hashes the
    statement-independent prefix once per shape and resumes from it."""
    st = ci.random_state(seed) if kind == "sha256-compression" else None
    inp, out, _ = ci.instance(kind, blocks, seed, st)
    L = _lib.load()
    got = (ctypes.c_uint8 * 32)()
    assert L.bitz_statement_digest(ci.KINDS[kind], inp.ctypes.data, inp.size, out.ctypes.data,
                                   got) == 0
    O = of.lib()
    O.o_matrix_digest.restype = None
    O.o_matrix_digest.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                  ctypes.c_void_p]
    want = (ctypes.c_uint8 * 32)()
    O.o_matrix_digest(ci.KINDS[kind], inp.ctypes.data, inp.size, out.ctypes.data, want)
    assert bytes(got) == bytes(want)
    # a different expected output changes the digest
    out2 = out.copy()
    out2[0] ^= 1
    got2 = (ctypes.c_uint8 * 32)()
    assert L.bitz_statement_digest(ci.KINDS[kind], inp.ctypes.data, inp.size, out2.ctypes.data,
                                   got2) == 0
    assert bytes(got2) != bytes(got)
