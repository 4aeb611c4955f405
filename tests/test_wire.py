"""Strict decoding of the bitzPCS proof container (WireProof::from_bytes,
crates/host/src/wire_proof.rs:109-140) through the C ABI; needs no GPU.
Mirrors the reference's decoder tests: every header field checked, the
declared lengths exactly consumed, hostile lengths rejected without a crash."""
import struct

import pytest

import bitz_b200 as bz


def container(narg=b"\x01\x02\x03", hints=b"\xaa" * 5, magic=b"bitzPCS\x00", version=1,
              header_len=32, flags=0, narg_len=None, hint_len=None):
    return (magic + struct.pack("<HHI", version, header_len, flags)
            + struct.pack("<QQ", len(narg) if narg_len is None else narg_len,
                          len(hints) if hint_len is None else hint_len) + narg + hints)


def expect(data, variant):
    with pytest.raises(bz.BitzError) as e:
        bz.wire_decode(data)
    assert e.value.code == "MalformedProof"
    assert variant in str(e.value), str(e.value)


def test_round_trip():
    assert bz.wire_decode(container()) == (b"\x01\x02\x03", b"\xaa" * 5)
    assert bz.wire_decode(container(b"", b"")) == (b"", b"")


def test_header_fields_are_checked():
    expect(container(magic=b"bitzPCS\x01"), "BadMagic")
    expect(container(version=2), "UnsupportedVersion(2)")
    expect(container(header_len=31), "BadHeaderLen(31)")
    expect(container(flags=1), "ReservedFlagsSet(1)")


def test_lengths_must_match_exactly():
    good = container()
    expect(good[:31], "OutOfInput")
    expect(b"", "OutOfInput")
    expect(good[:-1], "LengthMismatch")
    expect(good + b"\x00", "LengthMismatch")
    expect(container(narg_len=4), "LengthMismatch")
    expect(container(hint_len=0), "LengthMismatch")


def test_hostile_lengths_do_not_overflow():
    expect(container(narg_len=2**64 - 1), "LengthOverflow")
    expect(container(narg_len=2**63, hint_len=2**63), "LengthOverflow")
    expect(container(narg_len=2**64 - 40, hint_len=8), "LengthOverflow")  # 32 + both = 2^64
    expect(container(narg_len=2**64 - 48, hint_len=8), "LengthMismatch")
