"""Check reference_known_answers.json against the reference's test sources it was transcribed
from: every number of an entry must appear among the numeric literals of the cited lines.

Usage: python tests/golden/check_transcription.py <reference checkout>
Exit status 0 when every entry checks out; the mismatches are printed otherwise.  The CPU test
suite runs it when a reference checkout is present on the machine (it is not needed to use
the fixtures)."""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = re.compile(r"(?<![\w.])-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?f?")
# entries whose numbers sit in a test fixture's set-up rather than in the cited test body
SETUP = {"intrinsics_rows": ("test/icp_tests.cpp", 1, 54), "rotation_90_rows": ("test/icp_tests.cpp", 1, 54)}


def literals(path, a, b):
    with open(path, encoding="utf-8", errors="replace") as f:
        lines = f.read().splitlines()[a - 1:b]
    out = set()
    for ln in lines:
        code = ln.split("//")[0]
        for m in NUM.findall(code):
            out.add(float(m.rstrip("fF")))
    return out


def flat(x):
    if isinstance(x, (list, tuple)):
        for y in x:
            yield from flat(y)
    elif isinstance(x, (int, float)) and not isinstance(x, bool):
        yield float(x)


def check(ref_root, fx=None):
    """[(entry, cited lines, numbers not found there)] for the fixture dict fx (default: the
    committed file)."""
    if fx is None:
        with open(os.path.join(HERE, "reference_known_answers.json")) as f:
            fx = json.load(f)
    bad = []
    for key, entry in fx.items():
        if key == "_source":
            continue
        if key in SETUP:
            rel, a, b = SETUP[key]
            values = set(flat(entry))
        else:
            m = re.match(r"(test/[\w.]+):(\d+)-(\d+)", entry["_source"])
            rel, a, b = m.group(1), int(m.group(2)), int(m.group(3))
            values = set(v for k, e in entry.items() if not k.startswith("_") for v in flat(e))
        lit = literals(os.path.join(ref_root, rel), a, b)
        # a literal x also stands for -x (negated vectors and matrix entries are written with
        # a separate minus sign, e.g. -glm::vec3(...))
        missing = sorted(v for v in values if v not in lit and -v not in lit)
        if missing:
            bad.append((key, "%s:%d-%d" % (rel, a, b), missing))
    return bad


if __name__ == "__main__":
    bad = check(sys.argv[1])
    for key, src, missing in bad:
        print("%s (%s): not in the source: %s" % (key, src, missing))
    sys.exit(1 if bad else 0)
