"""Regenerate ``seqtree_b200/_tables.py`` and ``seqtree_b200/csrc/builtin_tables.inc`` from the
reference's similarity grids.

The six built-in amino-acid similarity matrices must hold exactly the reference's numbers for
results to be bit-identical (seqtree 0.6.0 ``src/blosum62.inc``, ``blosum45.inc``,
``blosum80.inc``, ``pam250.inc``, ``pam100.inc``, ``structural.inc``; the first five are the
published NCBI/EMBOSS log-odds tables, the last one is generated by the reference's
``bench/gen_matrices.py``).  This script parses those files as text and writes the grids in
this package's own layout.  It needs the reference tree and is run by hand:

    python seqtree_b200/gen_tables.py <reference source tree>
"""
import re
import sys
from pathlib import Path

NAMES = ["blosum62", "blosum45", "blosum80", "pam250", "pam100", "structural"]


def parse(path: Path) -> list[list[int]]:
    text = path.read_text()
    body = text[text.index("{") + 1: text.rindex("}")]
    rows = []
    for line in body.splitlines():
        line = line.split("//")[0]
        nums = [int(x) for x in re.findall(r"-?\d+", line)]
        if nums:
            rows.append(nums)
    assert len(rows) == 24 and all(len(r) == 24 for r in rows), path
    return rows


def main(ref_root: str) -> None:
    out = ['"""Built-in similarity grids, row/column order ``ARNDCQEGHILKMFPSTWYVBZX*``.',
           "",
           "Generated by gen_tables.py from the reference's table files; do not edit by hand.",
           '"""', "", "SIMILARITY = {"]
    for name in NAMES:
        rows = parse(Path(ref_root) / "src" / f"{name}.inc")
        out.append(f'    "{name}": (')
        for r in rows:
            out.append("        (" + ", ".join(f"{v:3d}" for v in r) + "),")
        out.append("    ),")
    out.append("}")
    (Path(__file__).parent / "_tables.py").write_text("\n".join(out) + "\n")
    write_c_include(Path(__file__).parent / "csrc" / "builtin_tables.inc")


def write_c_include(path: Path) -> None:
    """The same grids as a C array for the library's ``st_builtin_similarity``."""
    from importlib import util
    spec = util.spec_from_file_location("_tables", Path(__file__).parent / "_tables.py")
    mod = util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = ["// Built-in similarity grids, row/column order ARNDCQEGHILKMFPSTWYVBZX*.",
           "// Generated by gen_tables.py; do not edit by hand.",
           "static const char* const kBuiltinNames[] = {" +
           ", ".join(f'"{n}"' for n in NAMES) + "};",
           f"static const int32_t kBuiltinSimilarity[{len(NAMES)}][24 * 24] = {{"]
    for name in NAMES:
        out.append(f"    {{  // {name}")
        for r in mod.SIMILARITY[name]:
            out.append("        " + ", ".join(f"{v:3d}" for v in r) + ",")
        out.append("    },")
    out.append("};")
    path.write_text("\n".join(out) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: gen_tables.py <reference source tree>")
    main(sys.argv[1])
