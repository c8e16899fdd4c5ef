"""Build step: generate the marching-cubes lookup tables header.

The case tables used by the reference (include/tables.h: edgeTable[256] at :22,
triTable[256][16] at :61 with X=255 as terminator, numVertsTable[256] at :323,
nrOfTriangles[256] at :584, offsets3[72] at :588) are the classic Lorensen/Bourke tables
in the reference's own edge numbering.  That file carries a third-party licence header,
so its text is not committed here: this script reads the numbers from the reference
checkout at build time and writes them, in this project's own format, to
csrc/generated/kf_mc_tables.inc (git-ignored; it ships beside the built libraries).

Usage: python gen_mc_tables.py [path/to/tables.h] [out.inc]

The reference's tables.h is looked for, in order, at: the first argument; $KF_MC_TABLES_H
(a path to tables.h); $KF_REFERENCE_DIR/include/tables.h (a checkout of the reference);
baseline/_ref/include/tables.h under the repository root; include/tables.h of a checkout
named `reference` beside the repository.  When none exists, a previously generated
header is kept; with neither, the script stops with an error naming these places.
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DEFAULT_OUT = os.path.join(HERE, "generated", "kf_mc_tables.inc")


def candidate_sources() -> list[str]:
    """Where the reference's tables.h may be, in the order they are tried."""
    c = []
    if os.environ.get("KF_MC_TABLES_H"):
        c.append(os.environ["KF_MC_TABLES_H"])
    if os.environ.get("KF_REFERENCE_DIR"):
        c.append(os.path.join(os.environ["KF_REFERENCE_DIR"], "include", "tables.h"))
    c.append(os.path.join(REPO, "baseline", "_ref", "include", "tables.h"))
    c.append(os.path.join(os.path.dirname(REPO), "reference", "include", "tables.h"))
    return c


def _array_body(text: str, name: str) -> str:
    m = re.search(r"\b" + re.escape(name) + r"\s*(\[[^\]]*\])+\s*=\s*\{", text)
    if not m:
        raise ValueError(f"table {name} not found")
    depth, i = 1, m.end()
    while depth:
        c = text[i]
        depth += c == "{"
        depth -= c == "}"
        i += 1
    return text[m.end():i - 1]


def _numbers(body: str) -> list[int]:
    body = re.sub(r"//[^\n]*", "", body)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for tok in re.findall(r"0x[0-9a-fA-F]+|\d+|\bX\b", body):
        out.append(255 if tok == "X" else int(tok, 0))
    return out


def parse(path: str) -> dict[str, list[int]]:
    with open(path, "r", encoding="latin-1") as f:
        text = f.read()
    tabs = {
        "edge": _numbers(_array_body(text, "edgeTable")),
        "tri": _numbers(_array_body(text, "triTable")),
        "nverts": _numbers(_array_body(text, "numVertsTable")),
        "ntri": _numbers(_array_body(text, "nrOfTriangles")),
        "offsets3": _numbers(_array_body(text, "offsets3")),
    }
    want = {"edge": 256, "tri": 4096, "nverts": 256, "ntri": 256, "offsets3": 72}
    for k, n in want.items():
        if len(tabs[k]) != n:
            raise ValueError(f"table {k}: {len(tabs[k])} entries, expected {n}")
    check(tabs)
    return tabs


def check(t: dict[str, list[int]]) -> None:
    """Self-consistency facts of the case tables."""
    for c in range(256):
        row = t["tri"][16 * c:16 * c + 16]
        n = next((i for i, e in enumerate(row) if e == 255), 16)
        assert all(e == 255 for e in row[n:]), c
        assert n == t["nverts"][c] == 3 * t["ntri"][c], c
        mask = 0
        for e in row[:n]:
            assert 0 <= e < 12
            mask |= 1 << e
        assert mask == t["edge"][c], c  # every cut edge is used, no other edge is
    assert sum(t["ntri"]) == 820


def emit(t: dict[str, list[int]], out: str) -> None:
    os.makedirs(os.path.dirname(out), exist_ok=True)

    def rows(vals, per):
        return ",\n".join("  " + ", ".join(str(v) for v in vals[i:i + per])
                          for i in range(0, len(vals), per))

    tri = [(-1 if v == 255 else v) for v in t["tri"]]
    src = [
        "/* generated by gen_mc_tables.py at build time; do not edit, do not commit */",
        "#define KF_MC_TABLES_GENERATED 1",
        f"KF_MC_TABLE_QUAL uint16_t kf_mc_edge_table[256] = {{\n{rows(t['edge'], 16)}\n}};",
        f"KF_MC_TABLE_QUAL int8_t kf_mc_tri_table[256 * 16] = {{\n{rows(tri, 16)}\n}};",
        f"KF_MC_TABLE_QUAL uint8_t kf_mc_num_verts[256] = {{\n{rows(t['nverts'], 16)}\n}};",
        f"KF_MC_TABLE_QUAL uint8_t kf_mc_nr_triangles[256] = {{\n{rows(t['ntri'], 16)}\n}};",
        f"KF_MC_TABLE_QUAL uint8_t kf_mc_offsets3[72] = {{\n{rows(t['offsets3'], 6)}\n}};",
        "",
    ]
    tmp = out + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(src))
    os.replace(tmp, out)


def main(argv: list[str]) -> int:
    tried = [argv[1]] if len(argv) > 1 else candidate_sources()
    out = argv[2] if len(argv) > 2 else DEFAULT_OUT
    src = next((p for p in tried if os.path.exists(p)), None)
    if src is None:
        if os.path.exists(out):
            print(f"gen_mc_tables: no tables.h found; keeping existing {out}")
            return 0
        print("gen_mc_tables: the reference's include/tables.h was not found (tried: "
              + ", ".join(tried) + ") and no previously generated " + out + " exists; "
              "pass its path as the first argument or set KF_MC_TABLES_H or KF_REFERENCE_DIR",
              file=sys.stderr)
        return 1
    emit(parse(src), out)
    print(f"gen_mc_tables: wrote {out}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
