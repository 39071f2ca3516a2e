"""Static checks of the CUDA sources for patterns that fault or hang a GPU.

A warp collective (__shfl*_sync, __ballot_sync, __any_sync, __all_sync) named
with the full mask must be executed by all 32 lanes.  Writing one as an
operand of a short-circuit (&&, ||) or conditional (?:) expression makes its
execution depend on the lane, which is undefined behaviour and can deadlock the
warp."""
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = glob.glob(os.path.join(ROOT, "coupled-bubble-control_b200", "csrc", "*.cu")) + \
    glob.glob(os.path.join(ROOT, "coupled-bubble-control_b200", "csrc", "*.cuh"))

COLLECTIVE = r"__(shfl|shfl_down|shfl_up|shfl_xor|ballot|any|all)_sync\s*\("


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def test_no_collective_in_short_circuit():
    bad = []
    for fn in SRC:
        for ln, line in enumerate(strip_comments(open(fn).read()).splitlines(), 1):
            if re.search(r"(&&|\|\||\?)\s*" + COLLECTIVE, line):
                bad.append(f"{os.path.basename(fn)}:{ln}: {line.strip()}")
    assert not bad, "warp collective inside a short-circuit/conditional:\n" + "\n".join(bad)

