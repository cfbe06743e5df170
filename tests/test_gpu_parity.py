"""Parity of the CUDA transport layer against the CPU oracle (GPU tests).

Both sides get the same scene, tables and JKISS states, so each random slot
follows the same history.  Float arithmetic is done in the same order on both
sides; only the math-library transcendentals (logf, expf, sinf, cosf, acos:
CUDA's versus the host libm's) may differ by an ulp, which perturbs the last
bits of a direction and can occasionally flip a later comparison.  The bar:
>= 99.5 % of histories within 1e-3 mm / 1e-5 relative energy of the oracle,
>= 99.9 % of random streams identical at the end (same number of draws), and
tallies statistically identical (|z| < 3 in >= 99.7 % of bins, totals within
0.5 %).  The bit-exact fraction is reported (about 0.9 for the water case).
Runs that share their random streams agree far more closely than independent
estimates would, so the tally z-tests here are consistency checks; the
statistical criterion proper, on independent streams, and the parity checks at
each configuration's full size are in tests/test_gpu_at_size.py.
"""

import numpy as np
import pytest

from ggems_b200 import abi

import parity
import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from ggems_b200 import _native
    c = _native.Context(0)
    yield c
    c.close()


def _report(name, exact, close):
    print("%s: bit-exact histories %.5f, within tolerance %.5f" % (name, exact, close))


def test_water_box_histories_and_dose(ctx):
    """C1 at its full size: 64^3 water at 2 mm, 60 keV cone from 1 m, dose map, 1e6 primaries."""
    sc = scenes.water_box_scene(photon_tracking=True)
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 1_000_000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("water", exact, close)
    rng_exact = (sg[:, :n] == so[:, :n]).all(0).mean()
    print("random states identical after the run: %.5f" % rng_exact)
    assert exact > 0.8
    assert close > 0.995
    assert rng_exact > 0.999
    # Tallies: totals and per-dosel agreement.
    eg, eo = Tg.edep[0], To.edep[0]
    assert abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()
    assert abs(int(Tg.hit[0].sum()) - int(To.hit[0].sum())) <= 0.005 * To.hit[0].sum()
    assert abs(int(Tg.photon_tracking[0].sum()) - int(To.photon_tracking[0].sum())) <= 0.005 * To.photon_tracking[0].sum()
    # per-dosel z-test using the E^2 tallies as variance estimates
    var_g = np.maximum(Tg.edep_squared[0] - eg ** 2 / np.maximum(Tg.hit[0], 1), 0)
    var_o = np.maximum(To.edep_squared[0] - eo ** 2 / np.maximum(To.hit[0], 1), 0)
    z = parity.z_scores(eg, eo, var_g, var_o)
    frac = (np.abs(z) < 3).mean()
    print("dosels with |z| < 3: %.5f" % frac)
    assert frac >= 0.997


def test_water_box_dose_finalisation(ctx):
    """compute_dose on the GPU vs the numpy restatement of the reference kernel."""
    sc = scenes.water_box_scene()
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 100000
    _, Tg, _ = parity.run_gpu(ctx, sc, src, n)
    nd = sc.dose_maps[0].total_number_of_dosels
    dose, unc = ctx.compute_dose(0, 0, nd, scale=1.0, water_reference=False, minimum_density=0.0)
    dref, uref = parity.oracle_dose(sc, Tg, 0, 0)
    np.testing.assert_allclose(dose, dref, rtol=1e-6, atol=0)
    np.testing.assert_allclose(unc, uref, rtol=1e-5, atol=1e-7)


def test_cbct_histories_and_projection(ctx):
    """C2 geometry at reduced size: ellipsoid phantom + flat GOS panel, 120 kVp."""
    sc = scenes.cbct_scene(n=64, voxel=4.0, elements=(128, 128, 1), element_size=(3.2, 3.2, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("cbct", exact, close)
    rng_exact = (sg[:, :n] == so[:, :n]).all(0).mean()
    print("random states identical after the run: %.5f" % rng_exact)
    assert exact > 0.8
    assert close > 0.995
    assert rng_exact > 0.999
    for hg, ho in zip(Tg.histograms, To.histograms):
        assert abs(int(hg.sum()) - int(ho.sum())) <= 0.005 * max(ho.sum(), 1)
        z = parity.z_scores(hg.astype(float), ho.astype(float), hg.astype(float), ho.astype(float))
        assert (np.abs(z) < 3).mean() >= 0.997


def test_cbct_full_size_properties(ctx):
    """C2 at its full size (256^3 phantom, 512^2 panel, 1e8 primaries in 96 batches),
    through properties that do not need the oracle to run 1e8 histories: two runs
    from the same random states give identical histograms and identical final
    streams (integer tallies are order-independent); every scatter count is also a
    total count; and the detected and scattered fractions per primary, and the
    projection's shape on a 16x16 grid of blocks, agree with the oracle's first batch
    (the same 1,041,667 slots from the same states) within binomial noise."""
    sc = scenes.cbct_scene()
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 100_000_000
    _, T1, s1 = parity.run_gpu(ctx, sc, src, n)
    _, T2, s2 = parity.run_gpu(ctx, sc, src, n)
    total, scat = T1.histograms[0].astype(np.int64), T1.histograms[1].astype(np.int64)
    assert np.array_equal(total, T2.histograms[0]) and np.array_equal(scat, T2.histograms[1])
    assert np.array_equal(s1, s2)
    assert (scat <= total).all() and total.sum() <= n
    n_ref = 1_041_667  # GGEMSSource::OrganizeParticlesInBatch: the first of 96 batches
    _, To, _ = parity.run_oracle(sc, src, n_ref)
    t_ref, s_ref = To.histograms[0].astype(np.int64), To.histograms[1].astype(np.int64)
    for g, r in ((total.sum(), t_ref.sum()), (scat.sum(), s_ref.sum())):
        p = r / n_ref
        sigma = np.sqrt(p * (1 - p) / n_ref + p * (1 - p) / n)
        print("fraction per primary: %.5f (GPU, 1e8) vs %.5f (oracle, 1 batch), z = %.2f" % (g / n, p, (g / n - p) / sigma))
        assert abs(g / n - p) < 4 * sigma
    side = total.reshape(512, 512)
    blocks_g = side.reshape(16, 32, 16, 32).sum((1, 3)).astype(float)
    blocks_r = t_ref.reshape(512, 512).reshape(16, 32, 16, 32).sum((1, 3)).astype(float)
    scale = n_ref / n
    z = (blocks_r - blocks_g * scale) / np.sqrt(np.maximum(blocks_r + blocks_g * scale * scale, 1.0))
    print("blocks with |z| < 4: %.4f, max |z| %.2f" % ((np.abs(z) < 4).mean(), np.abs(z).max()))
    assert (np.abs(z) < 4).mean() >= 0.99


def test_multi_batch_random_slot_reuse(ctx):
    """2.5 M primaries -> 3 batches; slot i draws batch after batch as in the reference."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 2500000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("multi-batch", exact, close)
    assert close > 0.99
    for hg, ho in zip(Tg.histograms, To.histograms):
        assert abs(int(hg.sum()) - int(ho.sum())) <= 0.005 * max(ho.sum(), 1)


def test_voxelized_source_with_dose(ctx):
    """GGEMSVoxelizedSource: activity-CDF voxel sampling + isotropic emission, dose in water."""
    sc = scenes.water_box_scene(n=32, voxel=4.0, photon_tracking=True)
    src = scenes.VoxelizedSource(scenes.hot_spot_activity(16), (4.0, 4.0, 4.0), position=(8.0, -4.0, 0.0),
                                 monoenergy=scenes.F(140.0) * scenes.KEV)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("voxelized source", exact, close)
    assert close > 0.995
    assert (sg[:, :n] == so[:, :n]).all(0).mean() > 0.999
    eg, eo = Tg.edep[0], To.edep[0]
    assert abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()


def test_curved_multi_module_detector(ctx):
    """46 detector modules on an arc (the ct_scanner layout): one box solid per module."""
    import numpy as np
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_voxelized(np.zeros((20, 20, 20), np.uint8), (5.0, 5.0, 5.0), t)
    td = sc.add_tables(scenes.Tables(["GOS"]))
    scenes.add_curved_detector(sc, td, (1, 46), (64, 16, 1), (0.6, 0.6, 0.6), 1085.6, 595.0,
                               scenes.F(10.0) * scenes.KEV)
    src = scenes.XRaySource(position=(-595.0, 0.0, 0.0), spectrum=scenes.synthetic_spectrum(), aperture_deg=12.5)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("curved CT", exact, close)
    assert close > 0.995
    tg = sum(int(h.sum()) for h in Tg.histograms[0::2])
    to = sum(int(h.sum()) for h in To.histograms[0::2])
    assert abs(tg - to) <= 0.005 * to


def test_tle_dose_water(ctx):
    """Track-length-estimator dose in water: same histories, same TLE tallies."""
    sc = scenes.water_box_scene(tle=True)
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("TLE water", exact, close)
    assert close > 0.995
    assert (sg[:, :n] == so[:, :n]).all(0).mean() > 0.999
    eg, eo = Tg.edep[0], To.edep[0]
    assert abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()
    assert abs(int(Tg.hit[0].sum()) - int(To.hit[0].sum())) <= 0.005 * To.hit[0].sum()
    var_g = np.maximum(Tg.edep_squared[0] - eg ** 2 / np.maximum(Tg.hit[0], 1), 0)
    var_o = np.maximum(To.edep_squared[0] - eo ** 2 / np.maximum(To.hit[0], 1), 0)
    z = parity.z_scores(eg, eo, var_g, var_o)
    assert (np.abs(z) < 3).mean() >= 0.997


def test_tle_dose_heterogeneous(ctx):
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Air", "Water", "Bone185"]))
    sc.add_voxelized(scenes.ellipsoid_phantom(32, 8.0, seed=5, n_bones=3), (8.0, 8.0, 8.0), t, dose={"tle": True})
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("TLE heterogeneous", exact, close)
    assert close > 0.995
    eg, eo = Tg.edep[0], To.edep[0]
    assert abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()


def test_meshed_phantom_histories_and_dose(ctx, tmp_path):
    """GGEMSMeshedPhantom (STL body with cavities, octree depth 4, rotated): histories,
    dose tallies and dose finalisation on the octree-box dose map."""
    deg = scenes.DEG
    sc = scenes.mesh_phantom_scene(str(tmp_path / "body.stl"), subdivisions=3, n_inner=4, depth=4, dose=True,
                                   ops=[("rotation", (float(90 * deg), float(30 * deg), 0.0)),
                                        ("translation", (10.0, -5.0, 0.0))])
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=8.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    # Leaving a meshed solid (dead or alive) carries the photon to the OBB
    # boundary, up to ~300 mm along its direction; an ulp-level direction
    # difference (CUDA vs host cosf/sinf after a few scatters) becomes a few
    # micrometres there, so positions are compared within 10 um here.
    exact, close = parity.history_agreement(Pg, Po, pos_tol=1e-2)
    _report("meshed phantom", exact, close)
    assert close > 0.995
    assert (sg[:, :n] == so[:, :n]).all(0).mean() > 0.999
    same = (Pg.status == Po.status) & (Pg.solid_id == Po.solid_id) & (Pg.scatter == Po.scatter)
    assert same.mean() > 0.999
    eg, eo = Tg.edep[0], To.edep[0]
    assert eo.sum() > 0
    assert abs(eg.sum() - eo.sum()) <= 0.005 * eo.sum()
    assert abs(int(Tg.hit[0].sum()) - int(To.hit[0].sum())) <= 0.005 * To.hit[0].sum()
    nd = sc.dose_maps[0].total_number_of_dosels
    dose, unc = ctx.compute_dose(0, 0, nd, scale=1.0, water_reference=False, minimum_density=0.0)
    dref, uref = parity.oracle_dose(sc, Tg, 0, 0)
    np.testing.assert_allclose(dose, dref, rtol=1e-6, atol=0)
    np.testing.assert_allclose(unc, uref, rtol=1e-5, atol=1e-7)


def test_meshed_phantom_with_detector(ctx, tmp_path):
    """Mesh phantom in front of a flat CT panel (the mesh example's layout)."""
    from ggems_b200 import workloads
    path = str(tmp_path / "body.stl")
    workloads.write_stl(path, workloads.body_mesh(3, 2, 6, seed=4))
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_meshed(path, t, depth=4)
    td = sc.add_tables(scenes.Tables(["GOS"]))
    sc.add_flat_detector(td, (128, 128, 1), (3.2, 3.2, 10.0), sdd=1500.0, sid=1000.0, threshold=scenes.F(10.0) * scenes.KEV)
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po, pos_tol=1e-2)  # OBB push of the mesh exit, as above
    _report("meshed phantom + detector", exact, close)
    assert close > 0.995
    for hg, ho in zip(Tg.histograms, To.histograms):
        assert abs(int(hg.sum()) - int(ho.sum())) <= 0.005 * max(ho.sum(), 1)


def test_meshed_phantom_bvh_matches_octree_scan(ctx, tmp_path, monkeypatch):
    """The BVH walk (used for large meshes) finds the same crossings as GGEMS's
    octree scan: same scene run both ways on the GPU, and against the oracle."""
    deg = scenes.DEG
    sc = scenes.mesh_phantom_scene(str(tmp_path / "body.stl"), subdivisions=3, n_inner=4, depth=4, dose=True,
                                   ops=[("rotation", (float(90 * deg), float(30 * deg), 0.0)),
                                        ("translation", (10.0, -5.0, 0.0))])
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=8.0)
    n = 200000
    monkeypatch.setenv("GGEMS_B200_MESH_BVH", "0")
    Ps, Ts, ss = parity.run_gpu(ctx, sc, src, n)
    monkeypatch.setenv("GGEMS_B200_MESH_BVH", "1")
    Pb, Tb, sb = parity.run_gpu(ctx, sc, src, n)
    exact, close = parity.history_agreement(Pb, Ps, pos_tol=1e-2)
    _report("mesh BVH vs octree scan (GPU)", exact, close)
    assert exact > 0.999
    assert (sb[:, :n] == ss[:, :n]).all(0).mean() > 0.9999
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pb, Po, pos_tol=1e-2)
    _report("mesh BVH vs oracle", exact, close)
    assert close > 0.995
    assert abs(Tb.edep[0].sum() - To.edep[0].sum()) <= 0.005 * To.edep[0].sum()


def test_large_mesh_bvh(ctx, tmp_path):
    """A 20k-triangle body (automatic BVH) against the oracle's octree scan."""
    from ggems_b200 import workloads
    path = str(tmp_path / "large.stl")
    workloads.write_stl(path, workloads.body_mesh(5, 3, 4, seed=9))
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_meshed(path, t, depth=4, dose={"dosel_size": (8.0, 8.0, 8.0)})
    assert sc.solids[0].number_of_triangles > 4096
    src = scenes.XRaySource(monoenergy=scenes.F(80.0) * scenes.KEV, aperture_deg=8.0)
    n = 100000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po, pos_tol=1e-2)
    _report("large mesh (BVH)", exact, close)
    assert close > 0.995
    assert (sg[:, :n] == so[:, :n]).all(0).mean() > 0.999
    assert abs(Tg.edep[0].sum() - To.edep[0].sum()) <= 0.005 * To.edep[0].sum()


def test_world_tracking(ctx):
    """GGEMSWorld on a CBCT scene: photon counts, energy, energy^2 and momentum
    on the world grid agree with the oracle (same histories; int64 fixed-point
    energy and momentum on the GPU against FP64 sums in the oracle)."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    sc.set_world((40, 30, 20), (60.0, 50.0, 40.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 200000
    Pg, Tg, sg = parity.run_gpu(ctx, sc, src, n)
    Po, To, so = parity.run_oracle(sc, src, n)
    exact, close = parity.history_agreement(Pg, Po)
    _report("world tracking", exact, close)
    assert close > 0.995
    wg, wo = Tg.world, To.world
    assert wo["photon_tracking"].sum() > 0
    cnt_g, cnt_o = wg["photon_tracking"].astype(np.int64), wo["photon_tracking"].astype(np.int64)
    assert abs(int(cnt_g.sum()) - int(cnt_o.sum())) <= 0.005 * cnt_o.sum()
    assert (cnt_g == cnt_o).mean() > 0.99
    for k in ("energy", "energy_squared", "momentum_x", "momentum_y", "momentum_z"):
        g, o = wg[k], wo[k]
        scale = np.abs(o).sum()
        assert scale > 0, k
        assert np.abs(g - o).sum() <= 0.005 * scale, k


def test_error_against_fp64_oracle(ctx):
    """The CUDA results' error against the oracle's FP64 build on the same
    random streams: water dose (C1 configuration) and the CBCT projection
    (total and scatter histograms)."""
    sc = scenes.water_box_scene()
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 1_000_000
    Pg, Tg, _ = parity.run_gpu(ctx, sc, src, n)
    P64, T64, _ = parity.run_oracle(sc, src, n, fp64=True)
    eg, e64 = Tg.edep[0], T64.edep[0]
    rel = abs(eg.sum() - e64.sum()) / e64.sum()
    var = np.maximum(T64.edep_squared[0] - e64 ** 2 / np.maximum(T64.hit[0], 1), 0)
    z = parity.z_scores(eg, e64, var, var)
    same = ((Pg.status == P64.status) & (Pg.solid_id == P64.solid_id) & (Pg.scatter == P64.scatter)).mean()
    print("water 1e6: edep GPU vs FP64 oracle rel %.2e, |z|<3 in %.5f of dosels, same outcome %.4f"
          % (rel, (np.abs(z) < 3).mean(), same))
    assert rel < 5e-3
    assert (np.abs(z) < 3).mean() >= 0.997
    sc = scenes.cbct_scene(n=64, voxel=4.0, elements=(128, 128, 1), element_size=(3.2, 3.2, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 1_000_000
    _, Tg, _ = parity.run_gpu(ctx, sc, src, n)
    _, T64, _ = parity.run_oracle(sc, src, n, fp64=True)
    for k, name in ((0, "total"), (1, "scatter")):
        hg, h64 = Tg.histograms[k].astype(np.float64), T64.histograms[k].astype(np.float64)
        rel = abs(hg.sum() - h64.sum()) / h64.sum()
        z = (hg - h64) / np.sqrt(np.maximum(hg + h64, 1.0))
        print("CBCT 1e6 %s histogram: GPU vs FP64 oracle rel %.2e, |z|<3 in %.5f of elements"
              % (name, rel, (np.abs(z) < 3).mean()))
        assert rel < 5e-3
        assert (np.abs(z) < 3).mean() >= 0.997


def test_particle_tracking(ctx):
    """GGEMS_TRACKING: the tracked slot's trajectory starts with its primary,
    enters solids before stepping in them, and ends dead at the slot's final
    state; the histories are the same with tracking on (it only records)."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 50000
    P0, T0, s0 = parity.run_gpu(ctx, sc, src, n)
    slot = int(np.nonzero(P0.scatter[:n] == 1)[0][0])  # a photon that scattered in the phantom
    ctx.set_tracking(slot)
    try:
        P1, T1, s1 = parity.run_gpu(ctx, sc, src, n)
        pts, count = ctx.read_tracking()
    finally:
        ctx.set_tracking(-1)
    assert np.array_equal(s0, s1)
    for f in ("E", "px", "py", "pz", "status"):
        assert np.array_equal(getattr(P0, f), getattr(P1, f)), f
    assert count == len(pts) and count >= 4
    assert pts[0].kind == abi.GG_TRACK_PRIMARY and pts[-1].kind == abi.GG_TRACK_DEAD
    kinds = [p.kind for p in pts]
    assert abi.GG_TRACK_ENTER in kinds and abi.GG_TRACK_SCATTER in kinds
    assert all(p.history == 0 for p in pts)  # one history per slot at n < 2^20
    inside = None
    for p in pts[1:]:
        if p.kind == abi.GG_TRACK_ENTER:
            inside = p.solid
        elif p.kind in (abi.GG_TRACK_STEP, abi.GG_TRACK_SCATTER):
            assert p.solid == inside
        elif p.kind == abi.GG_TRACK_LEAVE:
            inside = None
    last = pts[-1]
    assert last.E == P1.E[slot]
    assert [last.position[i] for i in range(3)] == [P1.px[slot], P1.py[slot], P1.pz[slot]]
    _, count_off = ctx.read_tracking()
    assert count_off == 0


def test_checkpoint_resume(ctx):
    """A run can stop and resume in another context (or process): the random
    streams and the tallies read back, a fresh context given them back, and
    the continuation equals the uninterrupted sequence of runs."""
    from ggems_b200 import _native
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 300000
    # uninterrupted: two runs in one context, tallies accumulating
    ss = sc.struct()
    ctx.upload_scene(ss)
    ctx.set_random_states(scenes.seed_states(777))
    ctx.run(src.struct, n)
    ctx.run(src.struct, n)
    T_ref = sc.tallies()
    ctx.read_tallies(T_ref)
    st_ref = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    ctx.get_random_states(st_ref)
    # checkpoint after the first run
    ctx.upload_scene(ss)
    ctx.set_random_states(scenes.seed_states(777))
    ctx.run(src.struct, n)
    T_ckpt = sc.tallies()
    ctx.read_tallies(T_ckpt)
    states = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    ctx.get_random_states(states)
    # resume in a new context
    other = _native.Context(0)
    try:
        other.upload_scene(sc.struct())
        other.set_random_states(states)
        other.run(src.struct, n)
        T_rest = sc.tallies()
        other.read_tallies(T_rest)
        st = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
        other.get_random_states(st)
    finally:
        other.close()
    assert np.array_equal(st, st_ref)
    for a, b, c in zip(T_ckpt.histograms, T_rest.histograms, T_ref.histograms):
        assert np.array_equal(a.astype(np.int64) + b, c)
    assert sum(int(h.sum()) for h in T_ref.histograms) > 0
