"""Batched runs on the GPU: several source runs (projection angles, phantoms)
in one persistent launch, its CUDA-graph replay and the launch autotuner.

A batched launch must give what running the jobs one after another gives:
the oracle runs each job in turn with the random states left by the previous
one, and every job's detector histogram and the final random streams are
compared (same tolerances as the single-run parity tests).
"""

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi

pytestmark = pytest.mark.gpu

DET = (64, 64, 1)


@pytest.fixture(scope="module")
def ctx():
    from ggems_b200 import _native
    c = _native.Context(0)
    yield c
    c.close()


def _job_scene(labels, voxel, angle_deg, k, n_jobs, tables):
    """Scene of job k: phantom + flat panel rotated by angle about z, histograms 2k / 2k+1."""
    sc = scenes.Scene()
    t = sc.add_tables(tables[0])
    sc.add_voxelized(labels, (voxel, voxel, voxel), t)
    td = sc.add_tables(tables[1])
    sc.add_flat_detector(td, DET, (6.4, 6.4, 10.0), sdd=1500.0, sid=1000.0, threshold=scenes.F(10.0) * scenes.KEV,
                         extra_rotation=(0.0, 0.0, float(angle_deg * scenes.DEG)))
    det = sc.solids[1]
    det.histogram, det.scatter_histogram = 2 * k, 2 * k + 1
    sc.histogram_sizes = [DET[0] * DET[1]] * (2 * n_jobs)
    src = scenes.XRaySource(rotation=(0.0, 0.0, float(angle_deg * scenes.DEG)), aperture_deg=11.0,
                            spectrum=scenes.synthetic_spectrum())
    return sc, src


def _jobs(phantoms, angles, n):
    tables = (scenes.Tables(["Air", "Water", "Bone185"]), scenes.Tables(["GOS"]))
    out = []
    k = 0
    total = len(phantoms) * len(angles)
    for labels, voxel in phantoms:
        for a in angles:
            out.append(_job_scene(labels, voxel, a, k, total, tables) + (n,))
            k += 1
    return out


def _sequential_oracle(jobs):
    states = scenes.seed_states(777)
    T_all = None
    for sc, src, n in jobs:
        P, T, states = parity.run_oracle(sc, src, n, states=states)
        if T_all is None:
            T_all = T
        else:
            for a, b in zip(T_all.histograms, T.histograms):
                a += b
    return P, T_all, states


def _spec(jobs):
    arrays = [(abi.gg_solid * len(sc.solids))(*sc.solids) for sc, _, _ in jobs]
    return [(src.struct, n, arr) for (sc, src, n), arr in zip(jobs, arrays)]


def _batched_gpu(ctx, jobs, graph_replays=0):
    first = jobs[0][0]
    ctx.upload_scene(first.struct())
    ctx.set_random_states(scenes.seed_states(777))
    spec = _spec(jobs)
    if graph_replays:
        g = ctx.capture_jobs(spec)
        for _ in range(graph_replays):
            g.launch()
        ctx.synchronize()
        g.close()
    else:
        ctx.run_jobs(spec)
    n0 = max(n for _, _, n in jobs)
    P = abi.Particles(min(n0, abi.GG_MAXIMUM_PARTICLES))
    ctx.read_particles(P)
    T = first.tallies()
    ctx.read_tallies(T)
    st = np.zeros((5, abi.GG_MAXIMUM_PARTICLES), np.uint32)
    ctx.get_random_states(st)
    return P, T, st


def _compare(Tg, To, sg, so, n):
    assert (sg[:, :n] == so[:, :n]).all(0).mean() > 0.999
    for hg, ho in zip(Tg.histograms, To.histograms):
        assert ho.sum() > 0
        assert abs(int(hg.sum()) - int(ho.sum())) <= 0.005 * ho.sum() + 3 * np.sqrt(ho.sum())
        z = parity.z_scores(hg.astype(float), ho.astype(float), hg.astype(float), ho.astype(float))
        assert (np.abs(z) < 3).mean() >= 0.997


def test_projection_angles_in_one_launch(ctx):
    """Four projection angles (source and panel rotated about z) of one phantom, one launch."""
    labels = scenes.ellipsoid_phantom(32, 8.0, seed=2, n_bones=4)
    jobs = _jobs([(labels, 8.0)], [0.0, 30.0, 90.0, 225.0], 150000)
    Pg, Tg, sg = _batched_gpu(ctx, jobs)
    Po, To, so = _sequential_oracle(jobs)
    _compare(Tg, To, sg, so, 150000)
    exact, close = parity.history_agreement(Pg, Po)
    print("batched angles: last job's histories bit-exact %.5f, within tolerance %.5f" % (exact, close))
    assert close > 0.995


def test_phantoms_of_uneven_size_in_one_launch(ctx):
    """Three phantoms of different sizes (and primaries) as jobs of one launch."""
    phantoms = [(scenes.ellipsoid_phantom(n, 256.0 / n, seed=s, n_bones=3), 256.0 / n)
                for n, s in ((16, 1), (32, 2), (24, 3))]
    jobs = _jobs(phantoms, [0.0], 0)
    jobs = [(sc, src, n) for (sc, src, _), n in zip(jobs, (120000, 60000, 90000))]
    Pg, Tg, sg = _batched_gpu(ctx, jobs)
    Po, To, so = _sequential_oracle(jobs)
    _compare(Tg, To, sg, so, 60000)


def test_graph_replay_equals_repeated_runs(ctx):
    """A captured batched launch replayed twice == the batched launch run twice."""
    labels = scenes.ellipsoid_phantom(32, 8.0, seed=2, n_bones=4)
    jobs = _jobs([(labels, 8.0)], [0.0, 90.0], 100000)
    _, Tg, sg = _batched_gpu(ctx, jobs, graph_replays=2)
    first = jobs[0][0]
    ctx.upload_scene(first.struct())
    ctx.set_random_states(scenes.seed_states(777))
    spec = _spec(jobs)
    ctx.run_jobs(spec)
    ctx.run_jobs(spec)
    T = first.tallies()
    ctx.read_tallies(T)
    st = np.zeros((5, abi.GG_MAXIMUM_PARTICLES), np.uint32)
    ctx.get_random_states(st)
    assert np.array_equal(st, sg)
    for a, b in zip(T.histograms, Tg.histograms):
        assert np.array_equal(a, b)


def test_autotune_restores_state(ctx):
    """gg_autotune searches the photon stash, resident blocks per SM, regroup
    ratio, block size and photons per thread (slots per work-queue claim),
    keeps the fastest, and leaves the random states and tallies as they were."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    ctx.upload_scene(sc.struct())
    st0 = scenes.seed_states(777)
    ctx.set_random_states(st0)
    ms = ctx.autotune(src.struct, 2 * abi.GG_MAXIMUM_PARTICLES)
    bps, lanes, ratio = ctx.tuning()
    threads, grain = ctx.launch()
    stash, swap, rnd = ctx.stash()
    print("autotune: %.2f ms for 2^21 primaries with %d blocks/SM of %d threads, regroup ratio %d/4, "
          "%d slot(s) per claim, stash %d registers" % (ms, bps, threads, ratio, grain, stash))
    assert ms > 0 and 1 <= bps <= 8 and 1 <= lanes <= 32
    assert threads in (128, 256, 512) and grain in (1, 2, 4, 8) and stash in (0, 64, 80)
    assert bps * threads <= 1024
    st = np.zeros_like(st0)
    ctx.get_random_states(st)
    assert np.array_equal(st, st0)
    T = sc.tallies()
    ctx.read_tallies(T)
    assert all(h.sum() == 0 for h in T.histograms)
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, 100000)
    Po, To, so = parity.run_oracle(sc, src, 100000)
    assert parity.history_agreement(Pg, Po)[1] > 0.995
    ctx.set_tuning()
    ctx.set_launch()
    ctx.set_stash()


def test_launch_shape_does_not_change_results(ctx):
    """Every slot's histories are the same whatever the launch shape: block
    size, blocks per SM, photons per thread and the photon stash (on, with
    either register budget, or off) change which lane runs a slot, not what
    the slot computes (final states, streams and integer tallies identical)."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 2_500_000
    try:
        ref = parity.run_gpu(ctx, sc, src, n)
        for threads, bps, grain, stash, rnd in ((128, 6, 1, 80, 40), (512, 1, 4, 80, 64), (256, 3, 8, 64, 24),
                                                (256, 0, 1, 0, 40), (128, 0, 2, 0, 40), (256, 0, 1, 64, 32)):
            ctx.set_launch(threads, grain)
            ctx.set_tuning(bps)
            ctx.set_stash(stash, 1 if stash == 64 else 4, rnd)
            shape = (threads, bps, grain, stash, rnd)
            P, T, st = parity.run_gpu(ctx, sc, src, n)
            assert np.array_equal(st, ref[2]), shape
            for f in ("E", "px", "py", "pz", "dx", "dy", "dz", "status", "scatter", "solid_id"):
                assert np.array_equal(getattr(P, f), getattr(ref[0], f)), shape + (f,)
            for a, b in zip(T.histograms, ref[1].histograms):
                assert np.array_equal(a, b), shape
    finally:
        ctx.set_tuning()
        ctx.set_launch()
        ctx.set_stash()
