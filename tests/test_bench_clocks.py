"""Host-side helpers of bench.py's clock record (no GPU, no nvidia-smi):
which GPU the sampler asks nvidia-smi about, and how its samples become the
line's `clocks` object (median SM clock under load, max clock, throttle
reasons seen)."""
import os
import sys
import tempfile
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _fake_torch(uuid=None, fail=False):
    def props(dev):
        if fail:
            raise RuntimeError("no device")
        return types.SimpleNamespace(uuid=uuid)
    return types.SimpleNamespace(cuda=types.SimpleNamespace(get_device_properties=props))


def test_smi_id_prefers_the_device_uuid(monkeypatch):
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "4,5")
    assert bench._smi_id(_fake_torch("0a1b2c3d-0000-1111-2222-333344445555"), 1) == "GPU-0a1b2c3d-0000-1111-2222-333344445555"
    assert bench._smi_id(_fake_torch("GPU-0a1b"), 0) == "GPU-0a1b"


def test_smi_id_maps_through_the_visible_devices_without_a_uuid(monkeypatch):
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "4, 5")
    assert bench._smi_id(_fake_torch(fail=True), 1) == "5"
    assert bench._smi_id(_fake_torch(uuid=""), 0) == "4"
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES")
    assert bench._smi_id(_fake_torch(fail=True), 2) == "2"


def _summary(lines):
    fd, path = tempfile.mkstemp(suffix=".csv")
    with os.fdopen(fd, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    cs = bench.ClockSampler("0")
    cs.path = path
    out = cs.summary()
    assert not os.path.exists(path)          # the sample file is removed
    return out


def test_clock_summary_median_max_and_reasons():
    # index, clocks.sm, clocks.max.sm, power, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    rows = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 980.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 990.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage line",
        "0, [N/A], 1965, 0.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    out = _summary(rows)
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_summary_reports_slowdowns():
    rows = ["0, 1200, 1965, 500.0, 0x8, Active, Not Active, Active, Not Active"] * 3
    out = _summary(rows)
    assert out["sm_mhz"] == 1200.0 and out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_summary_without_samples():
    out = _summary([])
    assert out == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
