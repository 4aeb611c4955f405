"""GPU parity of the GF(2^128) sumcheck stages against the CPU oracle.

Both provers drive the same transcript framing; equality of the narg strings
means every round message and every challenge matched bit for bit."""
import numpy as np
import pytest

import bitz_b200 as bz
from oracle import ffi as of

pytestmark = pytest.mark.gpu


def rand_f128(rng, n):
    return rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)


@pytest.fixture(autouse=True)
def fast_oracle():
    of.lib().o_set_clmul_mode(1)
    yield
    of.lib().o_set_clmul_mode(0)


@pytest.mark.parametrize("log_rows,log_cols,security", [
    (7, 1, 100), (8, 0, 100), (10, 3, 100), (12, 2, 128), (14, 0, 100), (16, 0, 128), (9, 6, 100),
])
def test_post_gkr_matches_oracle(log_rows, log_cols, security):
    rng = np.random.default_rng(log_rows * 100 + log_cols)
    rows = rand_f128(rng, 1 << log_rows)
    cols = rand_f128(rng, 1 << log_cols)
    packed = rand_f128(rng, (1 << (log_rows - 7)) << log_cols)
    target = of.weighted_sum(rows, cols, packed)
    grind = 1 if security == 128 else 0
    ot = of.Transcript(b"post_gkr-tests", b"reduce")
    rc, opoint, ovalue = of.post_gkr_prove(rows, cols, target, packed, grind, ot)
    assert rc == 0
    gt = bz.build_prover(b"post_gkr-tests", b"reduce")
    gpoint, gvalue = bz.post_gkr_prove(rows, cols, target, packed, security, gt)
    assert np.array_equal(gpoint, opoint)
    assert np.array_equal(gvalue, ovalue)
    assert gt.narg() == ot.narg()
    # the closing value is MLE[f](rho) over the bits: check the first coordinates'
    # expected narg length, 2 elements per round, the closing value, nonces
    rounds = log_rows + log_cols
    assert len(gt.narg()) == 32 * rounds + 16 + (8 * rounds if grind else 0)


def test_post_gkr_all_zero_and_all_one_bits():
    rng = np.random.default_rng(5)
    rows = rand_f128(rng, 1 << 10)
    cols = rand_f128(rng, 2)
    for fill in (0, 2**64 - 1):
        packed = np.full((16, 2), fill, dtype=np.uint64)
        target = of.weighted_sum(rows, cols, packed)
        ot = of.Transcript(b"s", b"i")
        rc, opoint, ovalue = of.post_gkr_prove(rows, cols, target, packed, 0, ot)
        gt = bz.build_prover(b"s", b"i")
        gpoint, gvalue = bz.post_gkr_prove(rows, cols, target, packed, 100, gt)
        assert np.array_equal(gvalue, ovalue) and gt.narg() == ot.narg()


def test_post_gkr_rejects_a_false_claim():
    rng = np.random.default_rng(3)
    rows = rand_f128(rng, 1 << 9)
    cols = rand_f128(rng, 1)
    packed = rand_f128(rng, 4)
    target = of.weighted_sum(rows, cols, packed)
    target[0] ^= np.uint64(1)
    with pytest.raises(bz.BitzError) as e:
        bz.post_gkr_prove(rows, cols, target, packed, 100, bz.build_prover(b"s", b"i"))
    assert e.value.code == "ClaimDoesNotHold"


@pytest.mark.parametrize("s", [4, 7, 10])
def test_gkr_outputs_match_oracle(s):
    rng = np.random.default_rng(s)
    images = rand_f128(rng, 128)
    cols = rand_f128(rng, 1 << s)
    assert np.array_equal(bz.gkr_outputs(images, cols), of.gkr_outputs(images, cols))


@pytest.mark.parametrize("s,security", [(4, 100), (6, 128), (9, 100), (11, 100)])
def test_gkr_prove_matches_oracle(s, security):
    rng = np.random.default_rng(1000 + s)
    images = rand_f128(rng, 128)
    cols = rand_f128(rng, 1 << s)
    zeta = rand_f128(rng, s)
    grind = 2 if security == 128 else 0
    ot = of.Transcript(b"gkr-tests", b"prove")
    opoint, oclaim = of.gkr_prove(images, cols, zeta, grind, ot)
    gt = bz.build_prover(b"gkr-tests", b"prove")
    gpoint, gclaim = bz.gkr_prove(images, cols, zeta, security, gt)
    assert gt.narg() == ot.narg()
    assert np.array_equal(gpoint, opoint)
    assert np.array_equal(gclaim, oclaim)


def test_gkr_zero_coordinate_sends_one():
    """A zero coordinate makes the round send sum(1) (crates/gkr/src/lib.rs:617)."""
    rng = np.random.default_rng(9)
    images = rand_f128(rng, 128)
    cols = rand_f128(rng, 1 << 5)
    zeta = rand_f128(rng, 5)
    zeta[2] = 0
    ot = of.Transcript(b"z", b"z")
    opoint, oclaim = of.gkr_prove(images, cols, zeta, 0, ot)
    gt = bz.build_prover(b"z", b"z")
    gpoint, gclaim = bz.gkr_prove(images, cols, zeta, 100, gt)
    assert gt.narg() == ot.narg() and np.array_equal(gclaim, oclaim)
