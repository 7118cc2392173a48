"""Write tests/golden/grad_no12-nu120.json: the hand-derived FP64 CPU gradient
(oracle.closed_grad) of E(T) for the seeded no=12/nu=120 system (seed 3,
normal distributions), sampled at 200 seeded random entries per input tensor,
with whole-tensor checksums.

Run from the repository root:  python tests/golden/make_grad_golden.py
(about 20 minutes on 8 cores).
"""
import json
import pathlib
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

from libcc_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = pathlib.Path(__file__).with_name("grad_no12-nu120.json")
NAMES = ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo")
SAMPLES = 200


def sample_indices(name: str, size: int):
    rng = np.random.default_rng(NAMES.index(name) + 7)
    return np.sort(rng.choice(size, size=min(SAMPLES, size), replace=False))


def main():
    cfg = S.WORKLOADS["no12-nu120"]
    inp = S.generate(cfg["no"], cfg["nu"], cfg["seed"], cfg["dist"], name="no12-nu120")
    t = time.time()
    g = O.closed_grad(inp)
    out = {"no": inp.no, "nu": inp.nu, "seed": inp.seed, "dist": cfg["dist"], "e_t": g["e_t"],
           "seconds": round(time.time() - t, 1), "tensors": {}}
    for name in NAMES:
        a = g[name]
        idx = sample_indices(name, a.size)
        out["tensors"][name] = {"size": int(a.size), "index": idx.tolist(), "value": a[idx].tolist(),
                                "sum": float(a.sum()), "sumsq": float(np.dot(a, a)),
                                "maxabs": float(np.abs(a).max())}
    OUT.write_text(json.dumps(out, indent=1))
    print("wrote", OUT, out["seconds"], "s")


if __name__ == "__main__":
    main()
