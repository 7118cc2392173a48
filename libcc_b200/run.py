"""Command-line (T) evaluation: ``python -m libcc_b200.run``.

Runs a named synthetic workload or a GAMESS ``triples.restart`` file through the
library and prints the reference's result line (``ets/etd/ets+etd=``,
triples.F90:316) with the device time.

    python -m libcc_b200.run --workload no16-nu200 --form fp64
    python -m libcc_b200.run --restart triples.restart --form int8:5
    python -m libcc_b200.run --workload no24-nu320 --tuples 4      # first 4 tuples only
    python -m libcc_b200.run --workload no12-nu120 --backward      # then the adjoint pass
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m libcc_b200.run", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--workload", help="named synthetic workload (libcc_b200.synthetic.WORKLOADS)")
    src.add_argument("--restart", help="path of a triples.restart file")
    ap.add_argument("--form", default="fp64",
                    help="fp64, int8 (automatic digits), int8:S (S digits) or int8@R (relative target R); "
                         "default fp64")
    ap.add_argument("--tuples", type=int, default=0, help="run only the first N tuples (default all)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--backward", action="store_true",
                    help="after the forward, run the adjoint (ccT_backward) over the same tuples")
    args = ap.parse_args(argv)

    from . import restart, synthetic
    from .api import TriplesPlan, format_energies
    inp = synthetic.workload(args.workload) if args.workload else restart.read(args.restart)
    with TriplesPlan.for_form(inp.no, inp.nu, args.form, args.device) as plan:
        t0 = time.perf_counter()
        plan.set_system(inp)
        t1 = time.perf_counter()
        end = args.tuples or plan.num_tuples
        ets, etd, _ = plan.forward(0, end)
        print(f" no={inp.no} nu={inp.nu} form={args.form} tuples={end}/{plan.num_tuples}")
        print(format_energies(ets, etd))
        print(f" device ms={plan.last_forward_ms:.3f} set_inputs s={t1 - t0:.3f} "
              f"launches={plan.last_forward_launches}")
        if plan.precision == "int8":
            print(" emulated digits: {digits} (calibrated |dE(T)| bound {est_err:.3g} Eh, target {target:.3g} Eh)"
                  .format(**plan.emu_digits()))
        if args.backward:
            plan.backward(0, end)
            print(f" backward device ms={plan.last_backward_ms:.3f} "
                  f"ratio={plan.last_backward_ms / plan.last_forward_ms:.2f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
