"""PCS parameter pins: the oracle's profile ladder and profile encoding against
the values the reference's own tests fix (crates/pcs/src/profiles.rs:170-260,
crates/pcs/src/commitment.rs:352-361), plus the closed-form bounds those
tests check for every supported size."""
import ctypes
import math

import pytest

from oracle import ffi


class Level(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("k", "log_inv_rate", "log_msg_cols", "queries", "fold_grinding", "grinding",
                 "ood_samples")]


class Config(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("log_n", ctypes.c_int), ("security_bits", ctypes.c_int),
                ("nlevels", ctypes.c_int), ("final_log_n", ctypes.c_int), ("levels", Level * 8)]


def config(m, security):
    L = ffi.lib()
    L.o_pcs_config.restype = ctypes.c_int
    L.o_pcs_config.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(Config)]
    c = Config()
    assert L.o_pcs_config(m, security, ctypes.byref(c)) == 0
    return c, [c.levels[i] for i in range(c.nlevels)]


def test_udr_m22_matches_audited_parameters():
    # profiles.rs:174-187
    c, levels = config(22, 128)
    assert levels[0].k == 4
    assert c.final_log_n == 5
    assert [l.queries for l in levels] == [311, 192, 161]
    assert [l.fold_grinding for l in levels] == [10, 9, 7]
    assert all(l.grinding == 4 for l in levels)
    assert all(l.ood_samples == 0 for l in levels)


@pytest.mark.parametrize("m,folds", [(20, [7, 4, 1]), (22, [9, 6, 3])])
def test_johnson_queries_replace_query_grinding(m, folds):
    # profiles.rs:234-245
    c, levels = config(m, 100)
    assert c.security_bits == 100
    assert [l.queries for l in levels] == [218, 106, 71]
    assert [l.fold_grinding for l in levels] == folds
    assert all(l.grinding == 0 for l in levels)
    assert [l.ood_samples for l in levels] == [int(i > 0) for i in range(len(levels))]


@pytest.mark.parametrize("m", range(20, 36))
def test_udr_all_supported_sizes_cover_combined_errors(m):
    # profiles.rs:190-231: the published bounds, rebuilt independently
    c, levels = config(m, 128)
    for index, lv in enumerate(levels):
        n = 2.0 ** (lv.log_msg_cols + lv.log_inv_rate)
        delta = 1.0 - 2.0 ** -lv.log_inv_rate
        gamma = delta / 2.0 - 3.0 / (delta * n)
        assert delta * delta * n >= 18.0
        assert delta / 3.0 <= gamma < delta / 2.0

        def fold_error(g):
            beta = float(index > 0 and g == 0)
            return (gamma * n + 3.0 + beta) * 2.0 ** (-128 - g)

        assert fold_error(lv.fold_grinding) <= 2.0 ** -128
        if lv.fold_grinding > 0:
            assert fold_error(lv.fold_grinding - 1) > 2.0 ** -128
        final_beta = int(index + 1 == len(levels))
        alpha = (1 << (lv.queries - 1).bit_length()).bit_length() - 1
        miss = (1.0 - gamma) ** lv.queries
        assert miss <= 2.0 ** -128
        assert (1.0 - gamma) ** (lv.queries - 1) > 2.0 ** -128
        query = (miss + (alpha + final_beta) * 2.0 ** -128) * 2.0 ** -lv.grinding
        assert query <= 2.0 ** -128
        if lv.grinding > 0:
            assert query * 2.0 > 2.0 ** -128
        assert lv.queries <= n
        assert lv.fold_grinding <= 32 and lv.grinding <= 32
        assert lv.fold_grinding >= lv.k


def test_profile_encoding_bytes():
    # commitment.rs:352-361: Shape::new(7, 13) is 2^20 committed bits
    L = ffi.lib()
    L.o_pcs_encoding.restype = ctypes.c_size_t
    L.o_pcs_encoding.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    buf = ctypes.create_string_buffer(64)
    n = L.o_pcs_encoding(20, 100, buf, 64)
    assert buf.raw[:n] == b"bitz/pcs/security/v1\x00\x00\x10\x00\x00\x00\x00\x00\x64\x00\x00\x00"
    n2 = L.o_pcs_encoding(20, 128, buf, 64)
    assert buf.raw[:n2] != b"bitz/pcs/security/v1\x00\x00\x10\x00\x00\x00\x00\x00\x64\x00\x00\x00"


def test_ladder_levels_shrink_to_the_final_block():
    # profiles.rs:66-126: each level folds k variables; the last leaves final_log_n
    for m in (20, 21, 22, 23, 25):
        for sec in (100, 128):
            c, levels = config(m, sec)
            assert sum(l.k for l in levels) + c.final_log_n == c.log_n
            assert math.isclose(levels[0].log_inv_rate, 1)
