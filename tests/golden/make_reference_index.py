"""Writes reference_index.json: for every source file of the reference
(fxie2/paes-channelflow, a flat directory of Fortran 90 files) its line count
and the line ranges of the program units it defines (program, module,
subroutine, function).  No source text is stored.  tests/test_citations.py
checks every file:line citation in this repository against the table, so
the citations stay checkable where the reference is not mounted.

    python tests/golden/make_reference_index.py [reference_dir]
"""
import json
import os
import re
import sys

UNIT = re.compile(r"^\s*(?:end\s+)?(program|module|subroutine|function)\s+([A-Za-z_]\w*)", re.I)
TYPED_FN = re.compile(r"^\s*(?:real|integer|logical)\s+function\s+([A-Za-z_]\w*)", re.I)


def index_file(path):
    lines = open(path, errors="replace").read().split("\n")
    if lines and lines[-1] == "":
        lines = lines[:-1]
    units, open_units = [], []
    for i, line in enumerate(lines, 1):
        code = line.split("!")[0]
        m = UNIT.match(code)
        if m is None:
            t = TYPED_FN.match(code)
            if t:
                open_units.append((t.group(1).lower(), i))
            continue
        kind, name = m.group(1).lower(), m.group(2).lower()
        if re.match(r"^\s*end\s", code, re.I):
            for k in range(len(open_units) - 1, -1, -1):
                if open_units[k][0] == name:
                    units.append([name, open_units[k][1], i])
                    del open_units[k]
                    break
        elif kind != "module" or not re.match(r"^\s*module\s+procedure", code, re.I):
            open_units.append((name, i))
    for name, start in open_units:  # a unit whose end statement is unnamed
        units.append([name, start, len(lines)])
    units.sort(key=lambda u: u[1])
    return {"lines": len(lines), "units": units}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = {}
    for f in sorted(os.listdir(ref)):
        p = os.path.join(ref, f)
        if os.path.isfile(p) and not f.endswith(".mod"):
            out[f] = index_file(p)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_index.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)
    print("wrote", dst, len(out), "files")


if __name__ == "__main__":
    main()
