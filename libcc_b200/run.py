"""Command-line (T) evaluation: ``python -m libcc_b200.run``.

Runs a named synthetic workload or a GAMESS ``triples.restart`` file through the
library and prints the reference's result line (``ets/etd/ets+etd=``,
triples.F90:316) with the device time.

    python -m libcc_b200.run --workload no16-nu200 --form fp64
    python -m libcc_b200.run --restart triples.restart --form int8:5
    python -m libcc_b200.run --workload no24-nu320 --tuples 4      # first 4 tuples only
    python -m libcc_b200.run --workload no12-nu120 --backward      # then the adjoint pass
    python -m libcc_b200.run --workload no24-nu320 --ccsd-terms    # the CCSD T1-dressing terms
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
    ap.add_argument("--keep-w", action="store_true",
                    help="FP64 plans: the forward keeps every tuple's W-build output for the backward (keep_w)")
    ap.add_argument("--ccsd-terms", action="store_true",
                    help="instead of (T): one call of each CCSD T1-dressing entry point (ccT_ccsd_terms_29_31, "
                         "_32_35) on seeded device arrays of the workload's (no, nu); prints their device times")
    args = ap.parse_args(argv)
    if args.ccsd_terms:
        return ccsd_terms(args)

    from . import restart, synthetic
    from .api import TriplesPlan, format_energies
    inp = synthetic.workload(args.workload) if args.workload else restart.read(args.restart)
    with TriplesPlan.for_form(inp.no, inp.nu, args.form, args.device, keep_w=args.keep_w) as plan:
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
                  f"ratio={plan.last_backward_ms / plan.last_forward_ms:.2f} kept_tuples={plan.kept_tuples}")
    return 0


def ccsd_terms(args) -> int:
    import ctypes
    import torch
    from . import _native as N, synthetic
    if not args.workload:
        raise SystemExit("--ccsd-terms takes --workload (its no, nu)")
    no, nu = synthetic.WORKLOADS[args.workload]["no"], synthetic.WORKLOADS[args.workload]["nu"]
    dev = f"cuda:{args.device}"
    torch.cuda.set_device(args.device)
    nutr, n4 = nu * (nu + 1) // 2, no * nu * nu * no
    g = torch.Generator(device=dev).manual_seed(7)
    mk = lambda n: torch.randn(n, generator=g, device=dev, dtype=torch.float64) * 0.05
    o1, t2, vl, vr, vvvo = mk(no * nu), mk(n4), mk(n4), mk(n4), mk(nutr * nu * no)
    o2, vm, rl = mk(n4), mk(no ** 3 * nu), torch.zeros(n4, device=dev, dtype=torch.float64)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    lib = N.load()
    for name, call in (("29_31", lambda: lib.ccT_ccsd_terms_29_31(no, nu, vp(o1), vp(t2), vp(vl), vp(vr), vp(vvvo),
                                                                   N.CCT_MEM_DEVICE)),
                       ("32_35", lambda: lib.ccT_ccsd_terms_32_35(no, nu, vp(o1), vp(o2), vp(t2), vp(vm), vp(rl),
                                                                   vp(vvvo), N.CCT_MEM_DEVICE))):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = call()
        e1.record()
        torch.cuda.synchronize()
        N.check(st, "ccT_ccsd_terms_" + name)
        print(f" no={no} nu={nu} ccsd terms {name}: {e0.elapsed_time(e1):.3f} ms (first call: includes the workspace)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
