"""Generate the golden marching-cubes triangle table from the Sharc.Volrus crate.

The crate's ``volume_to_mesh`` emits each cell's triangles from its constant
256 x 16 ``TRI_TABLE`` (src/tools/volume_to_mesh.rs:246-503, the classic
Lorensen & Cline / Bourke table that the crate's own doc comment names), so
triangle lists identical to the crate's need that exact table.  This script
reads the table out of the crate's source (the reference checkout must be
present, as it is where the fixtures are made; nothing at test time reads
it) and writes:

  * ``tests/golden/mc_tri_table.json``   the table, 256 rows of 16 entries
  * ``sharc/volrus_b200/csrc/mc_tri_table.inc``  the same rows as a C
    initialiser for the CUDA mesher (csrc/mesh.cu)

It also checks, before writing, that every row is a run of triangles
terminated by -1 (entry 15 always -1), that each row uses exactly the edges
the crate's EDGE_TABLE flags for its case (so no triangle reads an edge
without a vertex), and that EDGE_TABLE equals the classification rule (edge
e flagged iff its two corners classify differently).

Usage: python tests/golden/make_mc_tri_table.py [path/to/volume_to_mesh.rs]
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
DEFAULT_SRC = Path("/root/reference/src/tools/volume_to_mesh.rs")
EDGE_ENDPOINTS = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def _array_body(src: str, name: str) -> str:
    m = re.search(r"const\s+" + name + r"\s*:[^=]*=\s*\[", src)
    if not m:
        raise SystemExit(f"{name} not found")
    i, depth = m.end() - 1, 0
    for j in range(i, len(src)):
        if src[j] == "[":
            depth += 1
        elif src[j] == "]":
            depth -= 1
            if depth == 0:
                return src[i + 1:j]
    raise SystemExit(f"unterminated {name}")


def parse(src: str):
    tri_body = _array_body(src, "TRI_TABLE")
    rows = [[int(x) for x in r.split(",") if x.strip()] for r in re.findall(r"\[([^\[\]]*)\]", tri_body)]
    edge_body = _array_body(src, "EDGE_TABLE")
    edges = [int(x, 16) for x in re.findall(r"0x([0-9a-fA-F]+)", edge_body)]
    return rows, edges


def check(rows, edges):
    assert len(rows) == 256 and all(len(r) == 16 for r in rows), "256 rows of 16 entries"
    assert len(edges) == 256
    for case in range(256):
        rule = 0
        for e, (a, b) in enumerate(EDGE_ENDPOINTS):
            if ((case >> a) & 1) != ((case >> b) & 1):
                rule |= 1 << e
        assert edges[case] == rule, f"EDGE_TABLE[{case}] differs from the classification rule"
        r = rows[case]
        n = r.index(-1)
        assert n % 3 == 0 and n <= 15 and all(x == -1 for x in r[n:]), f"row {case} is not a -1 terminated run"
        used = 0
        for x in r[:n]:
            assert 0 <= x < 12
            used |= 1 << x
        assert used == rule, f"row {case} uses other edges than the case flags"


def write(rows):
    (HERE / "mc_tri_table.json").write_text(json.dumps(
        {"source": "Sharc.Volrus src/tools/volume_to_mesh.rs:246-503 (TRI_TABLE)", "rows": rows},
        separators=(",", ":")) + "\n")
    lines = [
        "// Marching-cubes triangle table of the Sharc.Volrus crate, 256 cases x 16",
        "// edge indices (-1 terminated), exactly as src/tools/volume_to_mesh.rs:246-503",
        "// holds it (the classic Lorensen & Cline / Bourke table).  Kept identical on",
        "// purpose: the crate's triangle lists are emitted from it, so an identical",
        "// mesh needs the identical table.  Written by tests/golden/make_mc_tri_table.py,",
        "// which also checks each row against the case's edge flags.",
    ]
    for r in rows:
        lines.append("{" + ", ".join(str(x) for x in r) + "},")
    (REPO / "sharc" / "volrus_b200" / "csrc" / "mc_tri_table.inc").write_text("\n".join(lines) + "\n")


def main():
    src = Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_SRC
    rows, edges = parse(src.read_text())
    check(rows, edges)
    write(rows)
    print(f"wrote {len(rows)} rows")


if __name__ == "__main__":
    main()
