"""Regenerate the golden fixtures of tests/golden from the reference tree.

Reads the reference's committed quadrature-point listing
(``_T/_200mesh/test_quadpoints.out``, written by
``_T/_200mesh/004test_quadpoints.f:42-246`` for sector 1 of a mesh of
ntp_global = 2 angular and nr_global = 2 radial zones, cut with iscale = 2
into one zone, logarithmic radial mesh between r = 10 and r = 11, no ghost
layers) and stores its numbers as JSON.  Needs the reference checkout; the
tests only read the JSON.

usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import re
import sys
from pathlib import Path


def parse(text: str) -> dict:
    out = {"vert": {}, "xb": {}, "yb": {}, "zb": {}}
    cur = None
    num = r"(-?\d+\.\d+)"
    for line in text.splitlines():
        m = re.match(r"\s*\((\d), (\d), (\d)\) =\s+" + num + r"\s+" + num + r"\s+" + num, line)
        if m:
            key = f"{m.group(1)}{m.group(2)}{m.group(3)}"
            out["vert"][key] = [float(m.group(4)), float(m.group(5)), float(m.group(6))]
            continue
        m = re.match(r"\s*([xyz]b)_quadpts_patch, face (\d)", line)
        if m:
            cur = (m.group(1), m.group(2))
            out[cur[0]][cur[1]] = []
            continue
        m = re.match(r"\s*Point :\s+" + num + r"\s+" + num + r"\s+" + num, line)
        if m and cur:
            out[cur[0]][cur[1]].append([float(m.group(1)), float(m.group(2)), float(m.group(3))])
    return out


def main() -> int:
    if len(sys.argv) != 2:
        print(__doc__.strip().splitlines()[-1], file=sys.stderr)
        return 2
    ref = Path(sys.argv[1])
    src = ref / "_T" / "_200mesh" / "test_quadpoints.out"
    data = parse(src.read_text())
    data["setting"] = {"isector": 1, "ntp_global": 2, "nr_global": 2, "iscale": 2, "rmin": 10.0, "rmax": 11.0,
                       "radial_mesh": "log", "decimals": 4,
                       "source": "_T/_200mesh/test_quadpoints.out (from _T/_200mesh/004test_quadpoints.f)"}
    dst = Path(__file__).resolve().parent / "quadpoints_sector1.json"
    dst.write_text(json.dumps(data, indent=1) + "\n")
    print(dst)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
