"""The bench's roofline arithmetic on CPU: the dominant kernel's bytes over
its stage time against the HBM peak, and the counted integer operations of
every stage (units x operations per unit) over the stage time against the
measured integer peak. Synthetic timings and counts; no GPU. Also the
bench's clock record (median and maximum SM clock, throttle reasons seen
active) from fake nvidia-smi samples, and the split of the benchmark clip's
coding plan into closed GOPs that the bench codes concurrently."""
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


def test_clock_summary_reads_median_max_and_active_reasons():
    c = bench.Clocks(0)
    c.samples = [["1965", "1965", "700.1", "Not Active", "Not Active", "Not Active", "Not Active"],
                 ["1900", "1965", "990.0", "Not Active", "Not Active", "Not Active", "Active"],
                 ["1950", "1965", "980.5", "Not Active", "Not Active", "Not Active", "Not Active"],
                 ["[N/A]", "1965", "1.0", "", "", "", ""]]
    s = c.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    c.samples = [["1965", "1965", "900", "Active", "Not Active", "Active", "Not Active"]]
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert bench.Clocks(0).summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_benchmark_clip_splits_into_two_closed_gops():
    import mav1cu
    cfg = mav1cu.cli_config(bench.SPEC.width, bench.SPEC.height, **bench.FLAGS)
    jobs = mav1cu.plan(cfg, bench.SPEC.frames)
    gops = bench.split_gops(jobs)
    assert len(gops) == 2
    for g in gops:
        assert g[0]["is_key"] and not any(j["is_key"] for j in g[1:])
    shown = sorted(int(j["disp"]) for g in gops for j in g)
    assert shown == sorted(set(shown)) and shown[0] == 0 and shown[-1] == bench.SPEC.frames - 1
    assert {int(j["disp"]) for j in gops[1]} == set(range(60, 120))
