"""The surrogate's judge (ggems_b200/scatter.py: judge, judge_rescaled) and
its error measures, on synthetic projections.

A smooth "true" scatter image is sampled as Poisson counts (the low-count MC);
the network's output is the true image (kept), the true image off by 20 % in
magnitude (replaced by the MC; the rescaling variant rescales it to the MC's
integral), or an image of the wrong shape (the MC replaces it).  No GPU."""

import numpy as np

from ggems_b200 import scatter as S

SIDE, PRIMARIES = 64, 1_000_000


def _true_image():
    y, x = np.mgrid[0:SIDE, 0:SIDE] + 0.5
    return 1.0 + 0.8 * np.exp(-((x - 30.0) ** 2 + (y - 36.0) ** 2) / (2 * 14.0 ** 2))


def test_judge_keeps_rescales_and_replaces():
    rng = np.random.default_rng(5)
    true = _true_image()
    verdicts = {S.JUDGE_NETWORK: 0, S.JUDGE_RESCALED: 0, S.JUDGE_MC: 0}
    for trial in range(40):
        lam = true / true.sum() * 2000.0
        counts = rng.poisson(lam).astype(np.float64)
        mc = S.normalise(counts, PRIMARIES, SIDE)
        truth = lam * (SIDE * SIDE / PRIMARIES)  # the MC's expectation in the same units
        wrong_shape = np.roll(truth, SIDE // 2, axis=1) * np.linspace(0.2, 1.8, SIDE)[None, :]
        wrong_shape *= truth.sum() / wrong_shape.sum() * 1.3
        pred = np.stack([truth, 1.2 * truth, wrong_shape])
        plain, plain_used = S.judge(pred, np.stack([mc] * 3))
        # as specified: kept within 5 %, else the MC estimate
        assert plain_used[1] == S.JUDGE_MC and plain_used[2] == S.JUDGE_MC
        assert np.array_equal(plain[1], mc) and np.array_equal(plain[2], mc)
        if plain_used[0] == S.JUDGE_NETWORK:
            assert np.array_equal(plain[0], truth)
        final, used = S.judge_rescaled(pred, np.stack([mc] * 3), PRIMARIES, SIDE)
        for v in used:
            verdicts[int(v)] += 1
        # a kept network is returned unchanged; a rescaled one carries the MC's integral
        if used[0] == S.JUDGE_NETWORK:
            assert np.array_equal(final[0], truth)
        if used[1] == S.JUDGE_RESCALED:
            assert abs(final[1].sum() - mc.sum()) <= 1e-9 * mc.sum()
            assert np.allclose(final[1] / final[1].sum(), truth / truth.sum())
        assert used[2] == S.JUDGE_MC and np.array_equal(final[2], mc)
    # the MC integral's noise (~2.2 % at 2000 counts) rarely exceeds the 5 % tolerance
    assert verdicts[S.JUDGE_NETWORK] >= 35
    # the 20 %-off network is always rescaled: its shape is right (p >= 1e-3 fails rarely)
    assert verdicts[S.JUDGE_RESCALED] >= 38


def test_judge_without_counts_falls_back_to_mc():
    true = _true_image()
    mc = true.copy()
    final, used = S.judge(np.stack([1.2 * true]), np.stack([mc]))
    assert list(used) == [S.JUDGE_MC] and np.array_equal(final[0], mc)


def test_error_against_truth_removes_reference_noise():
    """error_vs_truth(relative_error(est, ref), reference_noise(ref)) recovers an
    estimate's error against the true image from a noisy reference, at full
    resolution and on the block grid."""
    rng = np.random.default_rng(9)
    true = _true_image()
    n_ref, n_est = 4_000_000, 250_000
    per_primary = true / true.sum() * 0.05  # counts per primary per element
    truth = per_primary * SIDE * SIDE       # normalise() units
    ref = S.normalise(rng.poisson(per_primary * n_ref).astype(np.float64), n_ref, SIDE)
    est = S.normalise(rng.poisson(per_primary * n_est).astype(np.float64), n_est, SIDE)
    for blocks in (None, 16):
        floor = S.reference_noise(ref, n_ref, blocks)
        expected_floor = S.relative_error(ref, truth, blocks)  # the reference's actual noise
        assert abs(floor - expected_floor) <= 0.1 * expected_floor
        err = S.error_vs_truth(S.relative_error(est, ref, blocks), floor)
        actual = S.relative_error(est, truth, blocks)
        assert abs(err - actual) <= 0.1 * actual, (blocks, err, actual)
        # the true image itself has (nearly) no error against the truth
        assert S.error_vs_truth(S.relative_error(truth, ref, blocks), floor) <= 0.3 * floor
