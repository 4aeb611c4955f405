"""The fibers that let one host thread drive several prover lanes
(bitz_b200/csrc/fiber.cpp): stack switches keep every fiber's registers,
control words, exceptions and device-gate counters its own. Needs no GPU."""
import ctypes

import pytest

from bitz_b200 import _lib


def run(threads, fibers, yields):
    out = ctypes.c_ulonglong(0)
    rc = _lib.load().bitz_diag_fibers(threads, fibers, yields, ctypes.byref(out))
    return rc, out.value


@pytest.mark.parametrize("threads,fibers,yields", [(1, 1, 4), (1, 7, 200), (4, 16, 100), (8, 3, 50)])
def test_fibers_interleave_and_keep_their_state(threads, fibers, yields):
    rc, h = run(threads, fibers, yields)
    assert rc == 0, _lib.load().bitz_last_error()
    assert run(threads, fibers, yields) == (0, h)  # round robin: the same order every time


def test_bad_arguments_are_rejected():
    assert run(0, 1, 4)[0] == 1
    assert run(1, 0, 4)[0] == 1
