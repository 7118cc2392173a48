"""Write tests/golden/energies.json: oracle E(T) for the seeded synthetic workloads.

Run from the repository root:  python tests/golden/make_golden.py [names...]
Small systems use the literal C restatement (oracle/triples_oracle.c); larger
ones the literal numpy/OpenBLAS restatement (oracle/oracle.py), which
tests/test_oracle.py ties to the C one.  Values are merged into the JSON file.
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

OUT = pathlib.Path(__file__).with_name("energies.json")

CASES = {
    "water-avdz": ("c", S.WORKLOADS["water-avdz"]),
    "no12-nu120": ("np", S.WORKLOADS["no12-nu120"]),
    "no16-nu200": ("np", S.WORKLOADS["no16-nu200"]),
    "no24-nu320": ("np", S.WORKLOADS["no24-nu320"]),
}


def run(name):
    how, cfg = CASES[name]
    inp = S.generate(cfg["no"], cfg["nu"], cfg["seed"], cfg["dist"], name=name)
    t = time.time()
    if how == "c":
        ets, etd, v1 = O.c_cc_triples(inp)
    else:
        ets, etd, v1 = O.literal_cc_triples(inp)
        v1 = np.asarray(v1).ravel(order="F")
    return dict(no=inp.no, nu=inp.nu, seed=inp.seed, dist=cfg["dist"], restatement=how, ets=ets, etd=etd,
                e_t=ets + etd, v1_norm=float(np.linalg.norm(v1)), v1_sum=float(np.sum(v1)),
                seconds=round(time.time() - t, 1))


def main(names):
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    for n in names:
        data[n] = run(n)
        print(n, data[n], flush=True)
        OUT.write_text(json.dumps(data, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(sys.argv[1:] or ["water-avdz", "no12-nu120"])
