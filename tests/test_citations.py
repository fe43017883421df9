"""Reference citations stay checkable: every ``Name.F90:a-b`` (and ``.py``) citation in the
library, the oracle and the tests names a file of the reference checkout and a line range
inside it.  Runs only where the reference checkout is present (this is a source check, not a
numerical one); AFID_REFERENCE_ROOT overrides its location."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("AFID_REFERENCE_ROOT", "/root/reference")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")),
                                reason="reference checkout not present")

CITE = re.compile(r"([A-Za-z0-9_./-]+\.(?:F90|py))((?::\d+(?:-\d+)?)(?:,\s*\d+(?:-\d+)?)*)")


def _reference_lengths():
    lengths = {}
    for p in glob.glob(os.path.join(REF, "**", "*"), recursive=True):
        if os.path.isfile(p) and p.endswith((".F90", ".py")):
            with open(p, errors="replace") as f:
                n = sum(1 for _ in f)
            lengths.setdefault(os.path.basename(p), []).append((os.path.relpath(p, REF), n))
    return lengths


def _sources():
    pats = ["afid-murphfi_b200/*.py", "afid-murphfi_b200/csrc/*", "include/*.h", "oracle/*.py", "oracle/*.c",
            "tests/*.py", "tests/golden/*.py", "bench.py", "__graft_entry__.py"]
    for pat in pats:
        yield from sorted(glob.glob(os.path.join(ROOT, pat)))


def test_reference_citations_are_inside_their_files():
    lengths = _reference_lengths()
    checked, bad = 0, []
    for src in _sources():
        if src.endswith("test_citations.py"):
            continue
        with open(src, errors="replace") as f:
            lines = f.readlines()
        for ln, line in enumerate(lines, 1):
            for m in CITE.finditer(line):
                name, ranges = m.group(1), m.group(2)
                cands = lengths.get(os.path.basename(name))
                if not cands:
                    if name.endswith(".F90"):
                        bad.append(f"{os.path.relpath(src, ROOT)}:{ln}: {name} is not in the reference")
                    continue            # a .py citation of this repository's own files
                match = [n for rel, n in cands if rel.endswith(name)] or [n for _, n in cands]
                nlines = max(match)
                checked += 1
                for r in re.findall(r"\d+(?:-\d+)?", ranges):
                    lo, hi = (int(x) for x in (r.split("-") + r.split("-"))[:2]) if "-" in r else (int(r), int(r))
                    if not 1 <= lo <= hi <= nlines:
                        bad.append(f"{os.path.relpath(src, ROOT)}:{ln}: {name}{ranges} (file has {nlines} lines)")
                        break
    assert checked > 300
    assert not bad, "\n".join(bad)
