"""Host-side statistics of the long-run precision comparison (longrun.py).

The window is cut into blocks; the batch-means standard error of each
quantity, the profiles folded about the channel centre, the comparison
against the FP64 run and the saved block averages (--save / --ref) are plain
numpy and run on the CPU.
"""
import math

import numpy as np

import longrun


def _blocks(seed, nb=8, nz=12, shift=0.0):
    rng = np.random.default_rng(seed)
    z = np.linspace(0.0, 1.0, nz)
    prof = 4.0 * z * (1.0 - z)  # symmetric about the centre
    bq = []
    for _ in range(nb):
        bq.append({"tau_w": 1e-5 * (1 + 0.01 * rng.standard_normal()), "u_tau": 3e-3, "re_tau": 180.0 + rng.standard_normal(),
                   "u_bulk": 0.08 * (1 + shift) + 1e-4 * rng.standard_normal(), "cf": 3e-3,
                   "mean_u": prof * (1 + shift) + 0.01 * rng.standard_normal(nz),
                   "u_rms": 0.1 * prof + 0.001 * rng.standard_normal(nz),
                   "v_rms": 0.05 * prof, "w_rms": 0.04 * prof + 0.001 * rng.standard_normal(nz)})
    return bq


def test_summary_standard_errors_and_fold():
    bq = _blocks(1)
    r = longrun.summarize(bq, 64, 1.0)
    vals = np.array([b["re_tau"] for b in bq])
    assert math.isclose(r["re_tau"], vals.mean())
    assert math.isclose(r["re_tau_se"], vals.std(ddof=1) / math.sqrt(len(bq)))
    mu = np.array([b["mean_u"] for b in bq])
    np.testing.assert_allclose(r["mean_u_fold"], 0.5 * (mu + mu[:, ::-1]).mean(axis=0))
    # folding two statistically equal halves lowers the standard error
    assert np.mean(r["mean_u_fold_se"]) < np.mean(r["mean_u_se"])


def test_compare_reports_difference_and_sigma():
    ref = longrun.summarize(_blocks(1), 64, 1.0)
    same = longrun.summarize(_blocks(2), 32, 1.0)
    off = longrun.summarize(_blocks(3, shift=0.05), 16, 1.0)
    e_same, e_off = longrun.compare(ref, same), longrun.compare(ref, off)
    # a 5 % shift of the profile stands out against the sampling error; a
    # second draw of the same statistics does not
    assert e_off["mean_u_fold_max_rel"] > 0.04
    assert e_off["mean_u_fold_max_z"] > 5 > e_same["mean_u_fold_max_z"]
    assert e_off["u_bulk_rel"] > 10 * e_off["u_bulk_sigma_rel"]


def test_saved_runs_round_trip(tmp_path):
    runs = []
    for label, seed in (("64", 1), ("64p", 2), ("16", 3)):
        r = longrun.summarize(_blocks(seed), int(label[:2]), 2.5)
        r["run"] = label
        runs.append(r)
    runs.append({"failed": "NaN", "run": "32"})
    path = tmp_path / "runs.npz"
    longrun.save_runs(str(path), runs)
    back = longrun.load_runs(str(path))
    assert sorted(back) == ["16", "64", "64p"]
    for r in runs[:3]:
        b = back[r["run"]]
        assert b["precision"] == r["precision"] and b["blocks"] == r["blocks"]
        for k in ("re_tau", "u_bulk", "re_tau_se"):
            assert math.isclose(b[k], r[k])
        for k in ("mean_u", "mean_u_fold_se", "u_rms"):
            np.testing.assert_array_equal(b[k], r[k])
