"""The M5 gate (scripts/engine_metrics.py:265-293) restated in metrics.py, on synthetic series."""
import numpy as np
import pytest


def test_m5_pass_fail_and_drift(me):
    from importlib import import_module
    m = import_module("motion_engine_b200.metrics")
    flat = np.full(600, 0.004)
    r = m.m5(flat)
    assert r["status"] == "PASS" and r["drift_class"] == "bounded" and abs(r["max_pen_over_R"] - 0.08) < 1e-12
    deep = np.full(600, 0.03)  # 0.6 R
    assert m.m5(deep)["status"] == "FAIL"
    # a slope whose extrapolation over the second half exceeds R / 10 is secular
    ramp = 0.001 + np.arange(600) * (0.1 * m.R / 300) * 1.5
    r = m.m5(ramp)
    assert r["drift_class"] == "secular" and r["status"] == "FAIL"
    with pytest.raises(ValueError):
        m.m5([0.0, 0.0])


def test_stack_penetration(me):
    from importlib import import_module
    m = import_module("motion_engine_b200.metrics")
    z = [2.998, 0.5, 1.4995]  # unsorted; spacings 0.9995 and 1.4985
    assert m.stack_penetration(z, 1.0) == pytest.approx(0.0005)
    assert m.stack_penetration(z, 1.0, ground=0.501) == pytest.approx(0.001)
