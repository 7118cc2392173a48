"""Write tests/golden/trant3_kat.json: the table printed by the reference's TRANT3
known-answer program (tools/trant3/trant3.f:2-31) for nu=2.

The program fills a(1:8) = 1..8, applies TRANT3 id j (j=0 means none), then
prints each element of a beside b(:,id) = TRANT3(a, id) for id 1..5.  The
reference ships no expected output, so the table is computed here from the
documented action of each id (new(x,y,z) = old(...), tools/trant3/trant3.f:36-116)
using numpy axis permutations -- independent of the in-place swap loops that
oracle/triples_oracle.c restates.
"""
import json
import pathlib

import numpy as np

SPEC = {1: "acb", 2: "bac", 3: "cba", 4: "bca", 5: "cab"}   # new(a,b,c) = old(SPEC)


def apply(flat, tid, nu=2):
    v = flat.reshape((nu, nu, nu), order="F")
    return np.einsum(SPEC[tid] + "->abc", v).ravel(order="F")


def table():
    out = []
    for j in range(6):
        a = np.arange(1, 9, dtype=float)
        if j > 0:
            a = apply(a, j)
        cols = [apply(a, i) for i in range(1, 6)]
        rows = [[a[r]] + [c[r] for c in cols] for r in range(8)]
        out.append({"j": j, "rows": rows})
    return out


if __name__ == "__main__":
    path = pathlib.Path(__file__).with_name("trant3_kat.json")
    path.write_text(json.dumps({"nu": 2, "source": "tools/trant3/trant3.f:2-31", "blocks": table()}, indent=1))
    print("wrote", path)
