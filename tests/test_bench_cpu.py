"""CPU tests of bench.py's host helpers: the DRAM-traffic record is reported only for the kernel
sources it was captured on, and the clock record sampled during the timed region is summarised
(median SM clock under load, the throttle reasons seen)."""
import json

import bench


def test_recorded_traffic_follows_the_kernel_sources(tmp_path, monkeypatch):
    rec = {"ncc": {"kernel": "k", "dram_bytes": 1234, "command": "c", "sources_sha16": bench.kernel_sources_sha16()}}
    path = tmp_path / "traffic.json"
    path.write_text(json.dumps(rec))
    monkeypatch.setattr(bench, "TRAFFIC_FILE", str(path))
    value, why = bench.recorded_traffic("ncc")
    assert value == 1234 and "ncu capture of k" in why
    assert bench.recorded_traffic("mi") == (None, "no capture recorded for this workload")
    monkeypatch.setattr(bench, "kernel_sources_sha16", lambda: "0" * 16)
    value, why = bench.recorded_traffic("ncc")
    assert value is None and "other kernel sources" in why
    monkeypatch.setattr(bench, "TRAFFIC_FILE", str(tmp_path / "absent.json"))
    assert bench.recorded_traffic("ncc")[0] is None


def test_committed_traffic_record_matches_the_sources():
    """The committed captures were taken on the kernel sources as they are committed."""
    for workload in ("ncc", "mi"):
        value, why = bench.recorded_traffic(workload)
        assert value is not None and value > 0, (workload, why)


def test_kernel_sources_hash_covers_every_listed_file(tmp_path, monkeypatch):
    for f in bench.KERNEL_SOURCES:
        (tmp_path / f).parent.mkdir(parents=True, exist_ok=True)
        (tmp_path / f).write_text("a")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    base = bench.kernel_sources_sha16()
    for f in bench.KERNEL_SOURCES:
        (tmp_path / f).write_text("b")
        assert bench.kernel_sources_sha16() != base, f
        (tmp_path / f).write_text("a")
    assert bench.kernel_sources_sha16() == base


def test_clock_summary(tmp_path):
    rows = [
        "0, 1965 MHz, 1965 MHz, 700 W, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950 MHz, 1965 MHz, 900 W, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 345 MHz, 1965 MHz, 80 W, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1965 MHz, 1965 MHz, 800 W, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    path = tmp_path / "clocks.csv"
    # the sampler writes numbers without units (nounits); idle samples below half the peak are
    # not "under load"
    path.write_text("\n".join(r.replace(" MHz", "").replace(" W", "") for r in rows) + "\n")
    s = bench.ClockSampler.__new__(bench.ClockSampler)
    s.path = str(path)
    out = s.summary()
    assert out["samples"] == 4
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
