"""Helpers shared by the parity tests: run a scene through the CUDA layer and
through the CPU oracle with the same random states, and compare."""

import ctypes as C
import os

import numpy as np

import scenes
from ggems_b200 import abi


def reference_dir():
    """The GGEMS checkout the oracle pin is built from (oracle/build.py's
    choice: $GGEMS_REFERENCE_DIR or its default), or None when absent."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(scenes.ROOT, "oracle", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.reference_dir()


def slots_used(n):
    """Slots a run of n primaries fills (GGEMSSource::OrganizeParticlesInBatch:
    ceil(n / 2^20) batches, the first n mod batches of them one particle larger).
    Slots past these keep whatever an earlier run left there, on the device as in
    the reference, so only these are compared."""
    if n <= 0:
        return 0
    nb = -(-n // abi.GG_MAXIMUM_PARTICLES)
    q, r = divmod(n, nb)
    return q + (1 if r else 0)


def run_oracle(sc, src, n, seed=777, states=None, threads=None, fp64=False):
    st = scenes.seed_states(seed) if states is None else states.copy()
    ss = sc.struct()
    P = abi.Particles(min(n, abi.GG_MAXIMUM_PARTICLES))
    P.used = slots_used(n)
    T = sc.tallies()
    lib = scenes.oracle_fp64() if fp64 else scenes.oracle()
    rc = lib.gg_oracle_run(C.byref(ss), C.byref(src.struct), n, abi.ptr(st, C.c_uint32), C.byref(P.struct),
                           C.byref(T.struct), threads or os.cpu_count())
    assert rc == 0
    return P, T, st


def run_gpu(ctx, sc, src, n, seed=777, states=None):
    st = scenes.seed_states(seed) if states is None else states.copy()
    ss = sc.struct()
    ctx.upload_scene(ss)
    ctx.set_random_states(st)
    ctx.run(src.struct, n)
    P = abi.Particles(min(n, abi.GG_MAXIMUM_PARTICLES))
    P.used = slots_used(n)
    ctx.read_particles(P)
    T = sc.tallies()
    ctx.read_tallies(T)
    ctx.get_random_states(st)
    return P, T, st


def history_agreement(Pa, Pb, pos_tol=1e-3, e_rel=1e-5):
    """Fraction of slots whose final state agrees bit-exactly, and within tolerance
    (the slots both runs filled)."""
    k = min(getattr(Pa, "used", Pa.n), getattr(Pb, "used", Pb.n))
    Pa, Pb = _first(Pa, k), _first(Pb, k)
    ints = (Pa.status == Pb.status) & (Pa.solid_id == Pb.solid_id) & (Pa.scatter == Pb.scatter)
    exact = ints.copy()
    for f in ("E", "px", "py", "pz", "dx", "dy", "dz"):
        exact &= getattr(Pa, f).view(np.uint32) == getattr(Pb, f).view(np.uint32)
    pa = np.stack([Pa.px, Pa.py, Pa.pz], 1).astype(np.float64)
    pb = np.stack([Pb.px, Pb.py, Pb.pz], 1).astype(np.float64)
    close = ints & (np.abs(pa - pb).max(1) <= pos_tol) & \
        (np.abs(Pa.E.astype(np.float64) - Pb.E) <= e_rel * np.maximum(np.abs(Pb.E), 1e-6))
    return exact.mean(), close.mean()


class _Slice:
    def __init__(self, P, k):
        self.n = k
        for f in abi.Particles.FIELDS + ("status", "scatter", "solid_id"):
            setattr(self, f, getattr(P, f)[:k])


def _first(P, k):
    return P if P.n == k else _Slice(P, k)


def oracle_dose(sc, T, dose_map, solid, scale=1.0, water=False, min_density=0.0):
    """ComputeDoseGGEMSVoxelizedSolid.cl:53-121 (and the meshed variant,
    ComputeDoseGGEMSMeshSolid.cl:53-114: material 0, no labels) restated in
    numpy (double math, float stores)."""
    dm = sc.dose_maps[dose_map]
    s = sc.solids[solid]
    t = sc.tables[s.navigator]
    n = dm.total_number_of_dosels
    ids = np.arange(n)
    nx, ny = dm.number_of_dosels[0], dm.number_of_dosels[1]
    z = ids // dm.slice_number_of_dosels
    x = (ids - z * dm.slice_number_of_dosels) % nx
    y = (ids - z * dm.slice_number_of_dosels) // nx
    F = np.float32
    sz = [F(v) for v in dm.size_of_dosels]
    nd = list(dm.number_of_dosels)
    pos = [F(c.astype(np.float32) * sz[i]) + F(F(nd[i] - 1) * F(F(-0.5) * sz[i])) for i, c in enumerate((x, y, z))]
    pos = [(c.astype(np.float32) * sz[i]).astype(np.float32) + np.float32(F(nd[i] - 1) * F(F(-0.5) * sz[i]))
           for i, c in enumerate((x, y, z))]
    if s.type == abi.GG_SOLID_MESHED:
        mat = np.zeros(n, np.int64)
    else:
        vid = [np.trunc(((pos[i] - F(s.obb.border_min[i])).astype(np.float32) / F(s.voxel_sizes[i])).astype(np.float32))
               .astype(np.int64) for i in range(3)]
        lab = np.ctypeslib.as_array(s.labels, shape=(s.number_of_voxels[0] * s.number_of_voxels[1] * s.number_of_voxels[2],))
        mat = lab[vid[0] + vid[1] * s.number_of_voxels[0] + vid[2] * s.number_of_voxels[0] * s.number_of_voxels[1]]
    vol = F(F(sz[0] * sz[1]) * sz[2])
    g_cm3 = F(F(6.241509704e+21) / F(1.e3))
    density = np.full(n, F(F(1.0) * g_cm3), np.float32) if water else t.density[mat]
    edep = T.edep[dose_map]
    dose = np.where(density < F(min_density), F(0.0),
                    (((F(scale) * edep) / density.astype(np.float64)) / np.float64(vol) / np.float64(F(1.0e-12)))
                    .astype(np.float32))
    hit = T.hit[dose_map].astype(np.float64)
    e2 = T.edep_squared[dose_map]
    with np.errstate(divide="ignore", invalid="ignore"):
        unc = np.sqrt((hit * e2 - edep * edep) / ((hit - 1) * edep * edep)).astype(np.float32)
    unc = np.where((hit > 1) & (edep != 0.0), unc, F(1.0))
    return dose.astype(np.float32), unc.astype(np.float32)


def z_scores(a, b, var_a, var_b):
    """Per-bin z of a difference of two independent estimates."""
    v = var_a + var_b
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.where(v > 0, (a - b) / np.sqrt(v), 0.0)
    return z


def mean_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b):
    """Per-bin z of two independent tallies of a per-primary score, compared as
    means per primary: sum = sum of the scores in the bin, sq = sum of their
    squares (the E^2 tally), n = primaries.  Var(sum) is estimated as
    sq - sum^2 / n (the scores of one bin are taken as one score per primary)."""
    sum_a, sum_b = np.asarray(sum_a, np.float64), np.asarray(sum_b, np.float64)
    va = np.maximum(np.asarray(sq_a, np.float64) - sum_a ** 2 / n_a, 0.0) / float(n_a) ** 2
    vb = np.maximum(np.asarray(sq_b, np.float64) - sum_b ** 2 / n_b, 0.0) / float(n_b) ** 2
    return z_scores(sum_a / n_a, sum_b / n_b, va, vb)


def run_oracle_squares(sc, src, n, seed=777):
    """run_oracle plus the squared-count tally of every detector histogram:
    (tallies, [sum over primaries of k^2 per bin, one int64 array per histogram])."""
    sq = [np.zeros(h, np.int64) for h in sc.histogram_sizes]
    ptrs = (C.POINTER(C.c_int64) * max(len(sq), 1))(*[abi.ptr(a, C.c_int64) for a in sq])
    lib = scenes.oracle()
    lib.gg_oracle_set_histogram_squares.argtypes = [C.c_void_p]
    lib.gg_oracle_set_histogram_squares(C.cast(ptrs, C.c_void_p))
    try:
        _, T, _ = run_oracle(sc, src, n, seed=seed)
    finally:
        lib.gg_oracle_set_histogram_squares(None)
    return T, sq


def count_z_var(a, n_a, b, n_b, sq_b):
    """Per-bin z of two independent count histograms compared per primary, with
    each bin's variance per primary estimated from the second histogram's
    squared-count tally (sq_b = sum of k^2 over its primaries):
    s^2 = sq_b / n_b - (b / n_b)^2, bounded below by the pooled rate (a count
    made of whole counts per primary has variance >= mean)."""
    a, b, sq_b = np.asarray(a, np.float64), np.asarray(b, np.float64), np.asarray(sq_b, np.float64)
    s2 = sq_b / n_b - (b / n_b) ** 2
    p = (a + b) / (n_a + n_b)
    v = np.maximum(s2, p) * (1.0 / n_a + 1.0 / n_b)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(v > 0, (a / n_a - b / n_b) / np.sqrt(v), 0.0)


def count_z(a, n_a, b, n_b):
    """Per-bin z of two independent count histograms (Poisson), compared per
    primary with the pooled rate: p = (a + b) / (n_a + n_b), Var = p (1/n_a + 1/n_b)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    p = (a + b) / (n_a + n_b)
    v = p * (1.0 / n_a + 1.0 / n_b)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(v > 0, (a / n_a - b / n_b) / np.sqrt(v), 0.0)
