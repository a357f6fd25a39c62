"""CPU checks of bench.py's timed-window plan: the regroup cadence restarts
`pad` substeps before the window so that the window's regroupings fall at
cadence points around its middle, and the reported count is what a
substep-by-substep replay of the cadence gives."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def replay(steps, interval, pad):
    """Regroupings inside a window of `steps` substeps whose call follows a
    `pad`-substep call that a restarted cadence opened (no pad call when pad
    is 0: the window's own call opens with the regrouping)."""
    count = 0 if pad else 1
    since = pad
    for t in range(1, steps + 1):
        since += 1
        if since == interval:
            since = 0
            if t < steps:  # one due after the last substep opens the next call
                count += 1
    return count


@pytest.mark.parametrize("interval", [4, 8, 16, 32, 64, 128])
@pytest.mark.parametrize("steps", [1, 3, 20, 40, 64, 100, 128, 500])
def test_window_plan_matches_cadence_replay(steps, interval):
    pad, regroups = bench.window_plan(steps, interval)
    assert 0 <= pad < interval
    assert regroups == replay(steps, interval, pad)
    assert regroups >= 1
    # its share, rounded either way
    assert abs(regroups - steps / interval) < 1.0 + 1e-9 or regroups == 1


def test_window_plan_puts_a_short_windows_regrouping_mid_window():
    pad, regroups = bench.window_plan(20, 64)
    assert (pad, regroups) == (54, 1)  # after the window's 10th substep
