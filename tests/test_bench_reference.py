"""The reference arm of bench.py when one of its sample processes dies.

Each sample process builds the CPU oracle's operators, about 7 GB at its peak on the large
mesh, so on a host with too little memory the kernel's out-of-memory killer may end one.
The arm must then retry with half the processes, and once a single process dies too,
print its ``unavailable`` line and exit 0 rather than wait for a result that will never
come.  The
process death is made on the host: the sampling helper raises the executor's own error."""

import argparse
import json
import sys
from concurrent.futures.process import BrokenProcessPool

import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _args():
    return argparse.Namespace(steps=4, warmup=3, workload="single", ref_procs=4, gpus=1)


def _last_line(capsys):
    return json.loads(capsys.readouterr().out.strip().splitlines()[-1])


def test_reference_arm_retries_with_fewer_processes(monkeypatch, capsys):
    calls = []

    def samples(workload, procs, warm, steps):
        calls.append((procs, warm, steps))
        if len(calls) == 1:
            raise BrokenProcessPool("a sample process terminated abruptly")
        return [(2.0, 5, 100)] * steps, 4.0

    monkeypatch.setattr(bench, "_reference_samples", samples)
    monkeypatch.setattr(bench, "host_cores", lambda: 4)
    assert bench.run_reference(_args(), 1, 0) == 0
    line = _last_line(capsys)
    assert [c[0] for c in calls] == [4, 2]
    assert calls[-1][1:] == (3, 4)  # warm-up samples, then the timed steps
    assert line["impl"] == "reference" and line["value"] == pytest.approx(0.5)
    assert line["cpu_baseline"]["cores"] == 2 and line["steps"] == 4


def test_reference_arm_reports_unavailable_when_one_process_dies(monkeypatch, capsys):
    calls = []

    def samples(workload, procs, warm, steps):
        calls.append(procs)
        raise BrokenProcessPool("a sample process terminated abruptly")

    monkeypatch.setattr(bench, "_reference_samples", samples)
    monkeypatch.setattr(bench, "host_cores", lambda: 4)
    assert bench.run_reference(_args(), 1, 0) == 0
    line = _last_line(capsys)
    assert calls == [4, 2, 1]
    assert set(line) == {"impl", "unavailable"} and line["impl"] == "reference"
    assert "host memory" in line["unavailable"]


def test_host_memory_budget_is_within_the_host():
    import psutil

    avail = bench.host_memory_available()
    assert avail is not None and 0 <= avail <= psutil.virtual_memory().total
