"""ORACLE — test infrastructure only.

Independent Python derivation of the marching-cubes tables that the CUDA
mesher (sharc/volrus_b200/csrc/mesh.cu) derives in C++; the tests compare the
two derivations entry for entry and then use this one to drive the oracle's
restatement of ``volume_to_mesh`` (src/tools/volume_to_mesh.rs:46-201).

Corner and edge numbering follow the reference (src/tools/volume_to_mesh.rs:
110-122 and 203-217): corner i sits at the offsets below, edge e joins
EDGE_ENDPOINTS[e] and its vertex is interpolated from the first corner toward
the second.  The edge table is the rule itself (edge e carries a vertex iff
its two corners classify differently).  The triangle table is derived here,
not copied: for each of the 256 corner classifications (bit i set: corner i
is below the isovalue, "inside")

  * on each cube face, walked counter-clockwise as seen from outside, a
    crossing where the walk leaves the inside is joined to the crossing where
    it last entered it (so an ambiguous face, with two diagonal inside
    corners, cuts each inside corner off on its own); the joins, run from the
    leaving crossing to the entering one, keep the inside on their left;
  * every crossing edge leaves on one of its two faces and enters on the
    other, so the joins chain into closed cycles; cycles are taken in order
    of their lowest edge index, each starting at that edge;
  * a cycle c0..c(k-1) becomes the fan (c0, c(i+1), c(i)), i = 1..k-2, wound
    so that the normals point toward increasing values (outward for a level
    set).

Neighbouring cells see a shared face with the same four corner classes and
join its crossings the same way, so the surface is closed across cells.
"""
from __future__ import annotations

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGE_ENDPOINTS = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]
# faces as corner cycles, counter-clockwise about the outward normal
FACES = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
ROW = 16  # entries per case: up to 5 triangles, -1 padded (checked below)


def _edge_of(a: int, b: int) -> int:
    for e, (p, q) in enumerate(EDGE_ENDPOINTS):
        if (p, q) == (a, b) or (p, q) == (b, a):
            return e
    raise ValueError((a, b))


def edge_table() -> list[int]:
    out = []
    for case in range(256):
        m = 0
        for e, (a, b) in enumerate(EDGE_ENDPOINTS):
            if ((case >> a) & 1) != ((case >> b) & 1):
                m |= 1 << e
        out.append(m)
    return out


def _cycles(case: int) -> list[list[int]]:
    inside = [(case >> i) & 1 for i in range(8)]
    succ: dict[int, int] = {}
    for face in FACES:
        leave, enter = [], []  # (walk position, edge)
        for k in range(4):
            a, b = face[k], face[(k + 1) % 4]
            if inside[a] and not inside[b]:
                leave.append((k, _edge_of(a, b)))
            elif inside[b] and not inside[a]:
                enter.append((k, _edge_of(a, b)))
        for k, e in leave:
            # the entering crossing that precedes this leaving one on the walk
            prev = max((p for p in enter if p[0] < k), default=None, key=lambda p: p[0])
            if prev is None:
                prev = max(enter, key=lambda p: p[0])
            assert e not in succ
            succ[e] = prev[1]
    cycles, seen = [], set()
    for e in sorted(succ):
        if e in seen:
            continue
        cyc, x = [], e
        while x not in seen:
            seen.add(x)
            cyc.append(x)
            x = succ[x]
        assert x == e, "joins chain into closed cycles"
        cycles.append(cyc)
    return cycles


def tri_table() -> list[list[int]]:
    out = []
    for case in range(256):
        row = []
        for cyc in _cycles(case):
            for i in range(1, len(cyc) - 1):
                row += [cyc[0], cyc[i + 1], cyc[i]]
        assert len(row) <= ROW - 1, (case, len(row))
        out.append(row + [-1] * (ROW - len(row)))
    return out


if __name__ == "__main__":
    t = tri_table()
    print("max triangles per case:", max(sum(1 for v in r if v >= 0) // 3 for r in t))
