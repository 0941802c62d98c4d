"""The FP32 rounding identities the device kernels use for the reference's
round() (half away from zero), checked exhaustively over every float they are
applied to:

* round_half_away (dense C(q) kernels): trunc(fl(x + copysign(0.49999997, x)));
  the AC1D C(q) kernel's nearest bin floor(q + 1/2) is floor(fl(q + 0.49999997));
* round_away_rz_i / round_away_rz_f (photon-pair kernel): fl(|x| + 0.49999997)
  followed by a round-toward-zero add of 2^23, i.e. floor of that sum.

For every non-negative float a < 2^23, floor(fl(a + 0.49999997f)) must equal
floor(a + 1/2) computed exactly; negative x follow by symmetry (both kernels
round |x| and restore the sign)."""
import numpy as np

HALF_BELOW = np.float32(0.49999997)


def test_round_half_away_identity_exhaustive():
    top = int(np.float32(2.0 ** 23).view(np.uint32))  # bit patterns of [0, 2^23)
    step = 1 << 24
    for lo in range(0, top, step):
        bits = np.arange(lo, min(lo + step, top), dtype=np.uint32)
        a = bits.view(np.float32)
        got = np.floor(a + HALF_BELOW)                 # float32 add, round to nearest even
        want = np.floor(a.astype(np.float64) + 0.5)    # exact
        bad = np.nonzero(got.astype(np.float64) != want)[0]
        assert bad.size == 0, f"first mismatch at {a[bad[0]]!r}"


def test_round_toward_zero_add_is_floor():
    # __fadd_rz(y, 2^23) = 2^23 + floor(y) for 0 <= y < 2^23: the sum lies in
    # [2^23, 2^24), where floats are the integers, and rounding toward zero
    # drops the fraction.  Spot-check the float grid at every binade.
    for e in range(-30, 23):
        y = np.float32(2.0 ** e) * np.linspace(1, 2, 4097, dtype=np.float32)[:-1]
        s = y.astype(np.float64) + 2.0 ** 23
        assert np.all(np.floor(s) - 2.0 ** 23 == np.floor(y.astype(np.float64)))


def test_plain_half_add_misrounds_just_below_one_half():
    # why the kernels add 0.49999997f and not 0.5f before a floor: for the
    # largest float below 1/2 the float sum q + 0.5f is a tie between 1 - 2^-24
    # and 1, rounds to the even 1, and floor gives 1 where floor(q + 1/2) is 0
    q = np.float32(0.5) - np.float32(2.0 ** -25)
    assert q < np.float32(0.5)
    assert np.floor(q + np.float32(0.5)) == 1.0
    assert np.floor(np.float64(q) + 0.5) == 0.0
    assert np.floor(q + HALF_BELOW) == 0.0
