"""The bench's clock record (CPU): the summary of the timed region and the per-bin statistics
of the sustained workload, from fabricated NVML samples (no GPU, no NVML)."""
import types

import bench


def sampler(samples):
    c = bench.ClockSampler(0)
    c.ok = True
    c.max_mhz = 1965
    c.nv = types.SimpleNamespace(nvmlClocksEventReasonHwSlowdown=0x8,
                                 nvmlClocksEventReasonHwThermalSlowdown=0x40,
                                 nvmlClocksEventReasonSwThermalSlowdown=0x20,
                                 nvmlClocksEventReasonSwPowerCap=0x4)
    c.samples = samples
    return c


def test_summary_of_timed_region():
    # (t, sm_mhz, reasons bitmask, power_w)
    c = sampler([(0.00, 1965, 0x0, 250.0), (0.02, 1965, 0x0, 260.0), (0.04, 1830, 0x4, 400.0),
                 (0.50, 1500, 0x40, 900.0)])
    c.window = (0.0, 0.04)
    s = c.summary()
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]


def test_between_bins():
    c = sampler([(0.00, 1965, 0x0, 250.0), (0.01, 1965, 0x0, 270.0), (0.10, 1650, 0x4, 990.0),
                 (0.11, 1640, 0x4 | 0x8, 1000.0)])
    b0 = c.between(0.0, 0.05)
    assert b0 == {"sm_mhz": 1965.0, "power_w": 260.0, "reasons": [], "samples": 2}
    b1 = c.between(0.05, 0.2)
    assert b1["sm_mhz"] == 1645.0 and b1["power_w"] == 995.0
    assert b1["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert c.between(1.0, 2.0)["samples"] == 0


def test_unsampled():
    c = bench.ClockSampler(0)
    assert c.summary()["reasons"] == ["unsampled"]
    assert c.between(0.0, 1.0)["sm_mhz"] is None
