"""Host-side pieces of bench.py that feed its JSON line: the DRAM traffic
of the dominant kernel read back from the committed ncu capture, and the
workload it applies to."""
import importlib.util
from pathlib import Path

from glasscamerapublic_b200 import scene

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_block_matching_traffic_comes_from_the_capture():
    b = _bench()
    t = b.bm_dram_traffic(scene.WORKLOADS["cfg2_4032x3024"])
    assert t is not None
    text = (ROOT / "profiles" / "block_match_pair_dram_4032x3024.txt").read_text()
    # the five launches' read + write bytes, summed as the capture lists them
    rows = [ln.split() for ln in text.splitlines() if ln[:1].isdigit() and len(ln.split()) >= 8]
    assert len(rows) == 5
    assert t["bytes"] == sum(int(r[-3]) + int(r[-2]) for r in rows)
    # no traffic figure for a workload the capture does not cover
    assert b.bm_dram_traffic(scene.WORKLOADS["cfg1_1024x768"]) is None
