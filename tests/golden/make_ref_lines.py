"""Write tests/golden/ref_lines.json: for each Fortran source of the reference
that this repository cites as ``code/<file>:<line>``, its line count and a
string with one character per line ('1' = a statement line, '0' = blank or a
comment), so tests/test_citations_cpu.py can check every citation without
the reference checkout.

    python tests/golden/make_ref_lines.py [REFERENCE_CODE_DIR]
"""
import json
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent
SRC = pathlib.Path(sys.argv[1]) if len(sys.argv) > 1 else pathlib.Path("/root/reference/code")


def is_statement(line: str) -> bool:
    s = line.rstrip("\n")
    if not s.strip():
        return False
    if s[:1] in ("c", "C", "*", "!"):          # fixed-form comment column 1
        return False
    return not s.strip().startswith("!")


def main() -> None:
    out = {}
    for p in sorted(SRC.iterdir()):
        if p.suffix not in (".f", ".f90"):
            continue
        lines = p.read_text(errors="replace").splitlines()
        out[p.name] = {"lines": len(lines), "stmt": "".join("1" if is_statement(x) else "0" for x in lines)}
    (HERE / "ref_lines.json").write_text(json.dumps(out, indent=0, sort_keys=True) + "\n")
    print(f"{len(out)} files")


if __name__ == "__main__":
    main()
