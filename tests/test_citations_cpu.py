"""Every ``code/<file>:<line>`` citation of the reference in this repository
points inside the cited file, and every cited line or range holds at least
one Fortran statement (not only blank or comment lines).

The line table (tests/golden/ref_lines.json) is written from the reference
sources by tests/golden/make_ref_lines.py, so this test runs without them."""
import json
import pathlib
import re

ROOT = pathlib.Path(__file__).resolve().parents[1]
TABLE = json.loads((ROOT / "tests" / "golden" / "ref_lines.json").read_text())
CITE = re.compile(r"code/([A-Za-z0-9_]+\.(?:f90|f))((?::\d+(?:-\d+)?(?:,\d+(?:-\d+)?)*))")
# written by the survey, the review and the round driver, not by this code
SKIP_FILES = {"SURVEY.md", "VERDICT.md", "ADVICE.md", "BASELINE.md"}
SKIP_DIRS = {".git", "_work", "gpurun_out", "data", "baseline", "__pycache__", "_build", ".pytest_cache"}
SUFFIXES = {".py", ".c", ".h", ".cpp", ".cu", ".cuh", ".md", ".txt", "Makefile"}


def _sources():
    for p in ROOT.rglob("*"):
        rel = p.relative_to(ROOT)
        if any(part in SKIP_DIRS for part in rel.parts) or not p.is_file():
            continue
        if rel.as_posix() in SKIP_FILES:
            continue
        if p.suffix in SUFFIXES or p.name in SUFFIXES:
            yield p


def _citations():
    for p in _sources():
        for ln, line in enumerate(p.read_text(errors="replace").splitlines(), 1):
            for m in CITE.finditer(line):
                for part in m.group(2)[1:].split(","):
                    a, _, b = part.partition("-")
                    yield p.relative_to(ROOT).as_posix(), ln, m.group(1), int(a), int(b or a)


def test_citations_exist_and_hold_statements():
    bad, n = [], 0
    for src, ln, ref, a, b in _citations():
        n += 1
        ent = TABLE.get(ref)
        if ent is None:
            bad.append(f"{src}:{ln} cites {ref}, which the reference does not have")
            continue
        if not (1 <= a <= b <= ent["lines"]):
            bad.append(f"{src}:{ln} cites {ref}:{a}-{b} (the file has {ent['lines']} lines)")
            continue
        if "1" not in ent["stmt"][a - 1:b]:
            bad.append(f"{src}:{ln} cites {ref}:{a}-{b}, which holds no statement")
    assert n > 100, f"only {n} citations found: the scan is broken"
    assert not bad, "\n".join(bad)
