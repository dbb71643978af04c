"""The sweep sums of relax_brick.cuh, emulated lane by lane in IEEE double
arithmetic (numpy): the paired shuffle schedules give the same bits as the
plain xor butterflies they replace.

* Warp partials: a 32-cell group's squares are added along the xor
  butterfly (spans 16, 8, 4, 2, 1; lane l adds lane l ^ s).  Two groups of
  one thread's cells are taken together: at span 16 the lower lanes keep
  group r's pair sums and the upper lanes group r + 1's, then spans 8..1
  stay within a half.
* Level of a brick: its warp partials (up to 64) are added as two
  butterflies over 32 lanes (partials q and 32 + q, 0 where absent) and the
  halves' sums added; the paired form takes span 1 for both halves at once
  (even lanes the low half, odd lanes the high half), spans 2..16 within a
  parity, then one more span-1 shuffle adds the halves.

The device tests compare every block layout bit for bit; this pins the
arithmetic identity itself on adversarial values (mixed magnitudes, zeros,
subnormals)."""

import numpy as np

L = np.arange(32)


def butterfly(v, spans):
    v = v.copy()
    for s in spans:
        v = v + v[L ^ s]
    return v


def values(rng, n):
    mag = np.exp(rng.uniform(-60.0, 60.0, n))
    v = mag * rng.uniform(0.0, 1.0, n) ** 2
    v[rng.uniform(size=n) < 0.1] = 0.0
    v[rng.uniform(size=n) < 0.02] = 5e-324
    return v


def test_paired_group_butterflies_are_the_plain_ones():
    rng = np.random.default_rng(7)
    for _ in range(2000):
        a, b = values(rng, 32), values(rng, 32)
        ref_a = butterfly(a, (16, 8, 4, 2, 1))[0]
        ref_b = butterfly(b, (16, 8, 4, 2, 1))[0]
        up = L >= 16
        keep = np.where(up, b, a)
        give = np.where(up, a, b)
        v = keep + give[L ^ 16]
        v = butterfly(v, (8, 4, 2, 1))
        assert v[0] == ref_a and v[16] == ref_b
        # every lower lane holds group a's sum, every upper lane group b's
        assert np.all(v[:16] == ref_a) and np.all(v[16:] == ref_b)


def test_paired_level_sum_is_the_plain_tree():
    rng = np.random.default_rng(11)
    for nw in (16, 27, 54, 64):
        for _ in range(1000):
            p = values(rng, nw)
            lo = np.where(L < nw, np.concatenate([p, np.zeros(64)])[:32], 0.0)
            hi = np.where(32 + L < nw, np.concatenate([p, np.zeros(64)])[32:64], 0.0)
            ref = butterfly(lo, (1, 2, 4, 8, 16))[0]
            if nw > 32:
                ref = ref + butterfly(hi, (1, 2, 4, 8, 16))[0]
                odd = (L & 1) == 1
                v = np.where(odd, hi, lo) + np.where(odd, lo, hi)[L ^ 1]
                v = butterfly(v, (2, 4, 8, 16))
                v = v + v[L ^ 1]
            else:
                v = butterfly(lo, (1, 2, 4, 8, 16))
            assert np.all(v == ref), nw
