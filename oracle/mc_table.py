"""ORACLE — test infrastructure only.

Marching-cubes tables for the oracle's restatement of ``volume_to_mesh``
(src/tools/volume_to_mesh.rs:46-201).

Corner and edge numbering follow the reference (src/tools/volume_to_mesh.rs:
110-122 and 203-217): corner i sits at the offsets below, edge e joins
EDGE_ENDPOINTS[e] and its vertex is interpolated from the first corner toward
the second.  The edge table is the rule itself (edge e carries a vertex iff
its two corners classify differently; the crate's EDGE_TABLE equals it, which
tests/golden/make_mc_tri_table.py checks when it reads the crate).  The
triangle table is the crate's own TRI_TABLE (src/tools/volume_to_mesh.rs:
246-503), read from the golden fixture tests/golden/mc_tri_table.json that
the same script writes from the crate's source.
"""
from __future__ import annotations

import json
from pathlib import Path

_GOLDEN = Path(__file__).resolve().parent.parent / "tests" / "golden" / "mc_tri_table.json"

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGE_ENDPOINTS = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
ROW = 16  # entries per case: up to 5 triangles, -1 padded (checked below)


def edge_table() -> list[int]:
    out = []
    for case in range(256):
        m = 0
        for e, (a, b) in enumerate(EDGE_ENDPOINTS):
            if ((case >> a) & 1) != ((case >> b) & 1):
                m |= 1 << e
        out.append(m)
    return out


def tri_table() -> list[list[int]]:
    """The crate's triangle table: 256 rows of 16 edge indices, -1 terminated."""
    rows = json.loads(_GOLDEN.read_text())["rows"]
    assert len(rows) == 256 and all(len(r) == ROW for r in rows)
    return [list(r) for r in rows]
