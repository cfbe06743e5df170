"""Parity at each configuration's own size (GPU tests).

* C2 (256^3 phantom, 512^2 panel, 120 kVp): one full batch (1,041,667 slots)
  compared with the oracle history by history, and a 1e7-primary projection
  compared with an independent oracle projection of the same size (different
  seed) pixel by pixel.
* C1 (64^3 water, 60 keV): dose maps from independent random streams, dosel by
  dosel.
* C4 (the 245,760-triangle body of the meshed workload, BVH navigation on the
  GPU, GGEMS's octree scan in the oracle): history by history.
* C3 (360 angles of the 64^3 water phantom + 16 phantoms of 96-320 voxels, 376
  jobs in one launch): against the oracle running the jobs one after another.
* C5 (the U-Net at 256^2): forward and gradients against the numpy oracle.

Same-stream comparisons use the bars of tests/test_gpu_parity.py (>= 99.5 % of
histories within 1e-3 mm / 1e-5 relative energy, >= 99.9 % of random streams
identical).  Independent-stream comparisons apply the statistical criterion to
estimates that share no random numbers: per bin |z| < 3 in >= 99.7 % of bins,
integrated totals within 0.5 %.  Both sides have the same sample size (the
difference of two bins is then symmetric; with a 10:1 ratio the low-count
bins' Poisson skew alone puts ~0.7 % of pixels beyond 3 sigma), the 0.5 %
criterion is applied where the sample makes 0.5 % at least 4 standard
deviations of the difference of the totals (else the totals are held to 4
standard deviations), and the z of each bin uses the per-primary variance (E^2
tally for energy; pooled counts times the measured over-dispersion for
histograms).
"""

import ctypes as C
import os
import sys

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from ggems_b200 import _native
    c = _native.Context(0)
    yield c
    c.close()


def _cbct():
    sc, src = scenes.cbct_api_scene(256, 1.0, seed=1)
    return sc, src


def test_cbct_full_geometry_histories(ctx):
    """C2's own geometry, the projection's first batch: 1,041,667 histories."""
    sc, src = _cbct()
    n = 1_041_667
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    rng_exact = (sg[:, :n] == so[:, :n]).all(0).mean()
    print("C2 full geometry, one batch: bit-exact %.5f, within tolerance %.5f, streams identical %.5f"
          % (exact, close, rng_exact))
    assert exact > 0.8
    assert close > 0.995
    # A history whose path an ulp flips draws a different number of random
    # numbers; the 256 mm phantom's histories are long (~145 voxel steps), so
    # streams are held to the history bar.
    assert rng_exact > 0.995
    for hg, ho in zip(Tg.histograms, To.histograms):
        assert abs(int(hg.sum()) - int(ho.sum())) <= 0.005 * ho.sum()
        z = parity.count_z(hg, n, ho, n)
        assert (np.abs(z) < 3).mean() >= 0.997


def test_cbct_projection_independent_streams(ctx):
    """C2's geometry, 1e7 primaries on each side from independent random
    streams (GPU seed 777, oracle seed 778): per pixel |z| < 3 in >= 99.7 % of
    the 512^2 pixels for the total and the scatter histogram.

    The two samples have the same size, so the difference of two bins is
    symmetric; its variance is the pooled count times the histogram's
    over-dispersion E[k^2] / E[k] (a primary can count twice in one element:
    a Compton site then a photoelectric site), measured by the oracle's
    squared-count tally.  Detected counts per primary agree within 0.5 %
    (6.7 standard deviations at this size).  The scatter histogram holds about
    5e4 counts per 1e7 primaries (0.64 % relative standard deviation of the
    difference), so its total is held to 4 standard deviations here; the 0.5 %
    criterion would need about 4e8 primaries on each side."""
    sc, src = _cbct()
    n = 10_000_000
    _, Tg, _ = parity.run_gpu(ctx, sc, src, n, seed=777)
    To, sq = parity.run_oracle_squares(sc, src, n, seed=778)
    for k, name in ((0, "total"), (1, "scatter")):
        hg, ho = Tg.histograms[k].astype(np.int64), To.histograms[k].astype(np.int64)
        phi = sq[k].sum() / max(ho.sum(), 1)
        sd = np.sqrt(phi * (hg.sum() + ho.sum())) / ho.sum()  # relative sd of the difference of the totals
        rel = hg.sum() / ho.sum() - 1
        z = parity.z_scores(hg.astype(np.float64), ho.astype(np.float64), phi * hg, phi * ho)
        frac = (np.abs(z) < 3).mean()
        print("C2 %s: %d vs %d counts (rel %+.2e, sd %.2e, over-dispersion %.3f); |z|<3 in %.5f of pixels"
              % (name, hg.sum(), ho.sum(), rel, sd, phi, frac))
        assert frac >= 0.997
        assert abs(rel) <= 4 * sd
        if 0.005 >= 4 * sd:
            assert abs(rel) <= 0.005


def test_water_dose_independent_streams(ctx):
    """C1 dose (64^3 water, 60 keV cone) from independent random streams:
    GPU seed 777 against oracle seed 778, 2e7 primaries each."""
    sc = scenes.water_box_scene()
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 20_000_000
    _, Tg, _ = parity.run_gpu(ctx, sc, src, n, seed=777)
    _, To, _ = parity.run_oracle(sc, src, n, seed=778)
    eg, eo = Tg.edep[0], To.edep[0]
    qg, qo = Tg.edep_squared[0], To.edep_squared[0]
    # standard deviation of the difference of the totals, from the E^2 tallies
    sd = np.sqrt(max(qg.sum() - eg.sum() ** 2 / n, 0) + max(qo.sum() - eo.sum() ** 2 / n, 0))
    rel = eg.sum() / eo.sum() - 1
    z = parity.mean_z(eg, qg, n, eo, qo, n)
    busy = (Tg.hit[0] >= 25) & (To.hit[0] >= 25)
    print("C1 dose: total rel %.2e (0.5 %% = %.1f sd); |z|<3 in %.5f of dosels, %.5f of the %d dosels with "
          ">= 25 deposits on both sides" % (rel, 0.005 * eo.sum() / sd, (np.abs(z) < 3).mean(),
                                             (np.abs(z[busy]) < 3).mean(), busy.sum()))
    assert 0.005 * eo.sum() >= 4 * sd, "sample too small for the 0.5 % criterion"
    assert abs(rel) <= 0.005
    assert abs(int(Tg.hit[0].sum()) / int(To.hit[0].sum()) - 1) <= 0.005
    assert (np.abs(z) < 3).mean() >= 0.997
    assert busy.sum() > 10000 and (np.abs(z[busy]) < 3).mean() >= 0.997


def test_mesh_at_workload_size(ctx, tmp_path):
    """C4's mesh (body 120/100/150 mm + 8 inner ellipsoids, 245,760 triangles,
    the meshed workload's body): the GPU's BVH walk against the oracle's GGEMS
    octree scan (depth 4), 80 keV cone, 2 mm dose grid, 1e5 histories."""
    from ggems_b200 import workloads
    path = str(tmp_path / "body.stl")
    tris = workloads.body_mesh(6, 5, 8, seed=1)
    workloads.write_stl(path, tris)
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_meshed(path, t, depth=4, dose={"dosel_size": (2.0, 2.0, 2.0)})
    assert sc.solids[0].number_of_triangles == len(tris) >= 50000
    src = scenes.XRaySource(monoenergy=scenes.F(80.0) * scenes.KEV, aperture_deg=8.0)
    n = 100_000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po, pos_tol=1e-2)  # OBB push of the mesh exit
    rng_exact = (sg[:, :n] == so[:, :n]).all(0).mean()
    print("C4 mesh (%d triangles): bit-exact %.5f, within tolerance %.5f, streams identical %.5f"
          % (len(tris), exact, close, rng_exact))
    assert close > 0.995
    assert rng_exact > 0.999
    eg, eo = Tg.edep[0], To.edep[0]
    assert eo.sum() > 0 and abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()
    assert abs(int(Tg.hit[0].sum()) - int(To.hit[0].sum())) <= 0.005 * To.hit[0].sum()
    z = parity.mean_z(eg, Tg.edep_squared[0], n, eo, To.edep_squared[0], n)
    assert (np.abs(z) < 3).mean() >= 0.997


def _c3_jobs(primaries, angles=360, phantoms=16, seed=3, dosel=4.0):
    """The batched workload's job list in oracle form: the 64^3 water phantom
    (dose map 0) seen from `angles` source angles 1 degree apart, then
    `phantoms` ellipsoid phantoms of edge U{96..320} voxels of 1 mm, each with a
    dose map of `dosel` mm dosels.  Returns (master scene, jobs, edges)."""
    from ggems_b200 import workloads
    sc = scenes.water_box_scene()
    tp = sc.add_tables(scenes.Tables(["Air", "Water", "Bone185"]))
    edges = [int(x) for x in np.random.default_rng(seed).integers(96, 321, phantoms)]
    solids = []
    for p, e in enumerate(edges):
        sc.add_voxelized(workloads.cbct_labels(e, 1.0, seed + p), (1.0, 1.0, 1.0), tp,
                         dose={"dosel_size": (dosel, dosel, dosel)})
        solids.append((abi.gg_solid * 1)(sc.solids.pop()))
    jobs = []
    for k in range(angles):
        s = scenes.XRaySource(rotation=(0.0, 0.0, float(scenes.F(k) * scenes.DEG)),
                              monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
        jobs.append((s, primaries, None))
    base = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    for arr in solids:
        jobs.append((base, primaries, arr))
    return sc, jobs, edges


class _slots:
    """The final particle states of the slots selected by a boolean mask."""

    def __init__(self, P, mask):
        idx = np.nonzero(mask)[0]
        self.n = len(idx)
        for f in abi.Particles.FIELDS + ("status", "scatter", "solid_id"):
            setattr(self, f, getattr(P, f)[idx])


def test_batched_workload_at_size(ctx):
    """C3's 376 jobs (360 angles + 16 phantoms of 96-320 voxels) in one launch,
    2e4 primaries per job, against the oracle running the jobs one after another
    with the random streams carried from job to job: every dose map, the final
    streams and the last job's histories."""
    n = 20_000
    sc, jobs, edges = _c3_jobs(n)
    ss = sc.struct()
    ctx.upload_scene(ss)
    ctx.set_random_states(scenes.seed_states(777))
    ctx.run_jobs([(src.struct, m, arr) for src, m, arr in jobs])
    Pg = abi.Particles(n)
    ctx.read_particles(Pg)
    Tg = sc.tallies()
    ctx.read_tallies(Tg)
    sg = np.zeros((5, abi.GG_MAXIMUM_PARTICLES), np.uint32)
    ctx.get_random_states(sg)

    lib = scenes.oracle()
    states = scenes.seed_states(777)
    To = sc.tallies()
    Po = abi.Particles(n)
    for src, m, arr in jobs:
        job = abi.gg_scene()
        C.pointer(job)[0] = ss
        if arr is not None:
            job.solids = C.cast(arr, C.POINTER(abi.gg_solid))
        rc = lib.gg_oracle_run(C.byref(job), C.byref(src.struct), m, abi.ptr(states, C.c_uint32), C.byref(Po.struct),
                               C.byref(To.struct), os.cpu_count())
        assert rc == 0
    # Each slot runs 376 histories in a row: a slot whose stream left the
    # oracle's (an ulp flip in any of its histories) keeps a different stream
    # for the rest of the batch.  The bar is per history: the divergence rate
    # implied by the identical fraction, 1 - identical^(1/376), within the
    # single-run bar (streams identical in >= 99.9 % of single histories).
    same = (sg[:, :n] == states[:, :n]).all(0)
    rate = 1.0 - same.mean() ** (1.0 / len(jobs))
    Pg_s, Po_s = _slots(Pg, same), _slots(Po, same)
    exact, close = parity.history_agreement(Pg_s, Po_s)
    print("C3 376 jobs (phantom edges %s): streams identical %.5f (divergence %.2e per history); last job's "
          "histories of those slots bit-exact %.5f, within tolerance %.5f" % (edges, same.mean(), rate, exact, close))
    assert rate < 1e-3
    assert close > 0.995
    assert len(Tg.edep) == 17
    # The slots whose streams diverged (fraction f) contribute two independent
    # samples to the two runs' tallies: the totals may differ by that noise,
    # sqrt(2 f) x the standard deviation of a total (from the E^2 tally), on
    # top of the 0.5 % criterion.  It matters only for the phantom maps, which
    # hold a few hundred deposits at 2e4 primaries per job.
    f = 1.0 - same.mean()
    for d, (eg, eo) in enumerate(zip(Tg.edep, To.edep)):
        assert eo.sum() > 0, d
        sd = np.sqrt(2.0 * f * To.edep_squared[d].sum())
        assert abs(eg.sum() - eo.sum()) <= max(0.005 * eo.sum(), 4 * sd), d
        hits = int(To.hit[d].sum())
        assert abs(int(Tg.hit[d].sum()) - hits) <= max(0.005 * hits, 4 * np.sqrt(2.0 * f * hits)), d
        m = n * (360 if d == 0 else 1)
        z = parity.mean_z(eg, Tg.edep_squared[d], m, eo, To.edep_squared[d], m)
        assert (np.abs(z) < 3).mean() >= 0.997, d


def test_unet_at_256():
    """The surrogate's network at its own size (256^2, batch 2): the tile paths
    the scan runs (full-resolution levels with 4096-CTA grids, 64^2 / 32^2 levels
    with thinner channel tiles), forward and gradients against the numpy oracle
    with the tolerances of the 64^2 test."""
    import torch
    sys.path.insert(0, os.path.join(scenes.ROOT, "oracle"))
    import unet_oracle as uo
    from ggems_b200.scatter import UNet
    side, batch = 256, 2
    net = UNet(batch, side, seed=5)
    p = net.parameters()
    rng = np.random.default_rng(1)
    y, x = np.mgrid[0:side, 0:side] / side
    base = np.stack([np.exp(-2.0 * ((x - 0.5) ** 2 + (y - 0.5) ** 2)), 3.0 * x * y], -1)
    inp = np.stack([base + rng.uniform(0, 0.3, base.shape) for _ in range(batch)]).astype(np.float32)
    tgt = (0.5 * inp[..., 0] + 0.2 * inp[..., 1] ** 2 + rng.uniform(0, 0.05, inp.shape[:3])).astype(np.float32)
    xt, tt = torch.from_numpy(inp).cuda(), torch.from_numpy(tgt).cuda()
    out = net.forward(xt).cpu().numpy()
    loss, g = net.gradients(xt, tt)
    net.close()
    loss_ref, g_ref = uo.loss_and_gradients(p.astype(np.float64), inp.astype(np.float64), tgt.astype(np.float64))
    y_ref, _ = uo.forward(p.astype(np.float64), inp.astype(np.float64))
    fwd_err = np.linalg.norm(out - y_ref) / np.linalg.norm(y_ref)
    print("U-Net 256^2: forward relative error %.4f, loss %.6f vs %.6f" % (fwd_err, loss, loss_ref))
    assert fwd_err < 0.02
    assert abs(loss - loss_ref) <= 0.03 * loss_ref
    layers_g, wo_g, _, _ = uo.unpack(g.astype(np.float64))
    layers_r, wo_r, _, _ = uo.unpack(g_ref)
    for i, ((wg, bg), (wr, br)) in enumerate(zip(layers_g, layers_r)):
        if i == 0:
            wg, wr = wg[:, :, :uo.INPUT_CHANNELS], wr[:, :, :uo.INPUT_CHANNELS]
        for a, b in ((wg, wr), (bg, br)):
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            cos = float((a * b).sum() / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
            print("  layer %2d: rel %.4f cos %.5f" % (i, rel, cos))
            assert rel < 0.08 and cos > 0.995, (i, rel, cos)
    assert np.linalg.norm(wo_g - wo_r) / np.linalg.norm(wo_r) < 0.03
