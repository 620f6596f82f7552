"""bench.py's reading of the committed ncu summaries: every summary a bench
leg takes its DRAM traffic from is present under profiles/ and carries a
`dram_bytes_per_launch:` figure, and each names the command that made it."""
import os
import re

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _summaries_named_by_bench():
    text = open(os.path.join(ROOT, "bench.py")).read()
    return sorted(set(re.findall(r'ncu_traffic\("([^"]+\.md)"', text)) | {"project_kernel_4m_sh3.md"})


def test_every_traffic_summary_parses():
    names = _summaries_named_by_bench()
    assert len(names) >= 5, names
    for name in names:
        traffic = bench.ncu_traffic(name)
        assert traffic is not None and traffic > 0, name
        assert bench.ncu_traffic(name, 8) == 8 * traffic


def test_summaries_name_their_command():
    for name in os.listdir(os.path.join(ROOT, "profiles")):
        text = open(os.path.join(ROOT, "profiles", name)).read()
        assert "--clock-control none" in text, name
        assert "python bench.py" in text, name


def test_missing_summary_reads_as_none():
    assert bench.ncu_traffic("no_such_summary.md") is None
