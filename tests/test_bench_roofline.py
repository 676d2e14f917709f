"""The bench's roofline arithmetic on CPU: the dominant kernel's bytes over
its stage time against the HBM peak, and the counted integer operations of
every stage (units x operations per unit) over the stage time against the
measured integer peak. Synthetic timings and counts; no GPU."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

TIMES = {"key": {"analyze": 2.0, "recon": 8.0, "filter": 0.2},
         "arf": {"motion_search": 0.4, "analyze": 0.3, "recon": 1.0, "filter": 0.2, "cdef_select": 0.03}}
COUNTS = {"key": {"analyze": {"ana_satd": 1000, "ana_intra_px": 4000}, "recon": {"fwd_mac": 10_000},
                  "filter": {"lf_taps": 100, "cdef_taps": 50}},
          "arf": {"motion_search": {"me_sad": 1_000_000, "me_satd": 10}, "analyze": {}, "recon": {"quant": 7},
                  "filter": {}, "cdef_select": {}},
          "int_peak_ops_s": 40e12}


def test_int_roofline_weighs_units_and_divides_by_stage_time_and_peak():
    r = bench.int_roofline(TIMES, COUNTS)
    assert r["peak_int_ops_per_s"] == 40.0
    by = {(s["frame"], s["stage"]): s for s in r["stages"]}
    me = by[("arf", "motion_search")]
    ops = 1_000_000 * bench.WORK_OPS["me_sad"] + 10 * bench.WORK_OPS["me_satd"]
    assert me["int_ops"] == ops
    assert abs(me["int_ops_per_s"] - ops / 0.4e-3 / 1e12) < 1e-4
    assert abs(me["frac_of_int_peak"] - ops / 0.4e-3 / 40e12) < 1e-5
    # stages without counted work report no rate
    assert by[("arf", "cdef_select")]["int_ops"] == 0 and "frac_of_int_peak" not in by[("arf", "cdef_select")]
    key_an = by[("key", "analyze")]
    assert key_an["int_ops"] == 1000 * bench.WORK_OPS["ana_satd"] + 4000 * bench.WORK_OPS["ana_intra_px"]


def test_every_counter_category_has_a_weight():
    import mav1cu
    assert set(bench.WORK_OPS) == set(mav1cu.WORK_NAMES)


def test_hbm_roofline_of_the_key_frame_recon():
    peaks = {"hbm_gbs": 6541.5}
    r = bench.roofline(TIMES, peaks, COUNTS)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak_source"] == "MEASURED_PEAKS.json"
    achieved = bench.KEY_RECON_BYTES / 8.0e-3 / 1e9
    assert abs(r["achieved"] - round(achieved, 2)) < 1e-9
    assert abs(r["frac"] - round(achieved / 6541.5, 6)) < 1e-9
    assert r["ms_per_launch"] == 8.0 and r["int_ops"]["stages"]
    assert bench.roofline(None, peaks) is None
    assert bench.roofline(TIMES, {}, None)["peak_source"] == "fallback"
