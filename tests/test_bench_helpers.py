"""Host-side logic of bench.py that its reported claims rest on: the pick
comparison between correlation paths (equal picks, picks that differ only
at the threshold, moved peaks, score differences) and the per-unit FLOP
count of the roofline."""
import math
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _pick(angle, wx, wy, t, score, cx=10.0, cy=20.0):
    return {"angle_index": angle, "window_x": wx, "window_y": wy, "template_index": t,
            "score": score, "center_x": cx, "center_y": cy}


def test_identical_picks():
    a = [_pick(0, 1, 2, 3, 8.5), _pick(1, 0, 0, 4, 9.0)]
    r = bench.compare_picks(a, list(a), 7.0)
    assert r["equal_picks"] and r["picks"] == [2, 2] and r["picks_differing"] == 0
    assert r["max_rel_score_diff"] == 0.0 and r["peaks_moved"] == 0
    assert r["differing_picks_within_1e-3_of_threshold"]


def test_differing_pick_at_the_threshold_is_reported_as_such():
    base = [_pick(0, 1, 2, 3, 8.5), _pick(0, 1, 2, 4, 7.0005)]
    other = [_pick(0, 1, 2, 3, 8.5 * (1 + 2e-4))]
    r = bench.compare_picks(base, other, 7.0)
    assert not r["equal_picks"] and r["picks_differing"] == 1
    assert r["differing_picks_within_1e-3_of_threshold"]
    assert math.isclose(r["max_rel_score_diff"], 2e-4, rel_tol=1e-6)


def test_differing_pick_far_from_the_threshold_fails_the_check():
    base = [_pick(0, 1, 2, 3, 8.5)]
    other = [_pick(0, 1, 2, 3, 8.5), _pick(2, 0, 1, 5, 9.5)]
    r = bench.compare_picks(base, other, 7.0)
    assert r["picks_differing"] == 1 and not r["differing_picks_within_1e-3_of_threshold"]


def test_moved_peak_is_counted():
    base = [_pick(0, 1, 2, 3, 8.5, cx=10.0), _pick(0, 1, 2, 4, 8.0)]
    other = [_pick(0, 1, 2, 3, 8.5, cx=11.0), _pick(0, 1, 2, 4, 8.0)]
    r = bench.compare_picks(base, other, 7.0)
    assert r["equal_picks"] and r["peaks_moved"] == 1


def test_unit_flops():
    l = 720
    n = l * l
    assert math.isclose(bench.unit_flops(l), 2.5 * n * math.log2(n) + 6.0 * n)
