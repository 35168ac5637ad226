"""Every reference citation in this repository must resolve.

Citations have the form `file.f90:a-b` (or `:a`, `:a-b, c, d-e`) and name a
file of the reference by its path within the project.  The table
tests/golden/reference_index.json (line counts and program-unit ranges of
every reference file, written by tests/golden/make_reference_index.py) lets
the check run without the reference mounted.  Checks:
  * the file exists in the reference and every cited line lies inside it;
  * a citation written as `routine (file:a-b)`, where routine is a program
    unit of that file, overlaps that unit's lines.
"""
import json
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INDEX = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_index.json")))
SCAN = ["oracle", "paes-channelflow_b200", "include", "tests", "bench.py", "__graft_entry__.py",
        "DESIGN.md", "INTEGRATION.md", "README.md"]
EXT = (".py", ".cpp", ".h", ".cu", ".cuh", ".f90", ".md", ".txt")
CITE = re.compile(r"(?:\b([A-Za-z_]\w*)\s*\(\s*)?\b([A-Za-z_][\w]*\.(?:f90|F90)):(\d+)(?:-(\d+))?"
                  r"((?:,\s*\d+(?:-\d+)?)*)")


def _files():
    for r in SCAN:
        p = os.path.join(ROOT, r)
        if os.path.isfile(p):
            yield p
            continue
        for dp, dn, fn in os.walk(p):
            if "_build" in dp or "__pycache__" in dp or "golden" in dp:
                continue
            for f in fn:
                if f.endswith(EXT):
                    yield os.path.join(dp, f)


def _citations():
    out = []
    for path in _files():
        for ln, line in enumerate(open(path, errors="replace"), 1):
            for m in CITE.finditer(line):
                routine, name = m.group(1), m.group(2)
                nums = [int(m.group(3))]
                if m.group(4):
                    nums.append(int(m.group(4)))
                extra = [int(x) for x in re.findall(r"\d+", m.group(5) or "")]
                out.append((os.path.relpath(path, ROOT), ln, routine, name, nums, extra))
    return out


CITATIONS = _citations()


def test_citations_found():
    assert len(CITATIONS) > 200


def test_every_citation_lies_inside_its_file():
    bad = []
    for path, ln, routine, name, nums, extra in CITATIONS:
        if name not in INDEX:
            bad.append("%s:%d %s (no such reference file)" % (path, ln, name))
            continue
        n = INDEX[name]["lines"]
        for v in nums + extra:
            if v < 1 or v > n:
                bad.append("%s:%d %s:%d (file has %d lines)" % (path, ln, name, v, n))
        if len(nums) == 2 and nums[1] < nums[0]:
            bad.append("%s:%d %s:%d-%d (empty range)" % (path, ln, name, nums[0], nums[1]))
    assert not bad, "\n".join(bad)


def test_named_routine_citations_overlap_the_routine():
    bad, checked = [], 0
    for path, ln, routine, name, nums, extra in CITATIONS:
        if not routine or name not in INDEX:
            continue
        units = {u[0]: (u[1], u[2]) for u in INDEX[name]["units"]}
        r = routine.lower()
        if r not in units:
            continue
        lo, hi = nums[0], nums[-1]
        a, b = units[r]
        checked += 1
        if hi < a or lo > b:
            bad.append("%s:%d %s (%s:%d-%d) outside %s at %d-%d" % (path, ln, routine, name, lo, hi, r, a, b))
    assert checked > 10
    assert not bad, "\n".join(bad)


@pytest.mark.skipif(not os.path.isdir("/root/reference"), reason="reference not mounted")
def test_index_matches_mounted_reference():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mkidx", os.path.join(ROOT, "tests", "golden", "make_reference_index.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for f, ent in INDEX.items():
        assert mod.index_file(os.path.join("/root/reference", f)) == ent, f
