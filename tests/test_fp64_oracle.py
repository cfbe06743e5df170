"""The FP64 build of the oracle's transport restatement against its FP32 build
(the reference's precision), on the same random streams: what single precision
costs the tallies.  The GPU's own error against the FP64 oracle is measured
in tests/test_gpu_parity.py::test_error_against_fp64_oracle."""

import numpy as np

import parity
import scenes


def _totals(T):
    return float(T.edep[0].sum()), int(T.hit[0].sum())


def test_fp32_restatement_against_fp64():
    sc = scenes.water_box_scene()
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 100000
    P32, T32, s32 = parity.run_oracle(sc, src, n)
    P64, T64, s64 = parity.run_oracle(sc, src, n, fp64=True)
    e32, h32 = _totals(T32)
    e64, h64 = _totals(T64)
    same = (P32.status == P64.status) & (P32.solid_id == P64.solid_id) & (P32.scatter == P64.scatter)
    rel = abs(e32 - e64) / e64
    print("FP32 vs FP64 oracle: edep %.6f vs %.6f MeV (rel %.2e), hits %d vs %d, same outcome %.4f"
          % (e32, e64, rel, h32, h64, same.mean()))
    # same random streams: the two precisions follow the same histories but for
    # rare decisions that a last-bit difference flips
    assert same.mean() > 0.99
    assert rel < 2e-3
    assert abs(h32 - h64) <= 2e-3 * h64
    var = np.maximum(T64.edep_squared[0] - T64.edep[0] ** 2 / np.maximum(T64.hit[0], 1), 0)
    z = parity.z_scores(T32.edep[0], T64.edep[0], var, var)
    assert (np.abs(z) < 3).mean() >= 0.997
