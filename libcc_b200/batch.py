"""Many independent (T) systems in one persistent kernel (``ccT_batch_*``).

    from libcc_b200 import batch, synthetic
    systems = synthetic.batch96()
    with batch.TriplesBatch([(s.no, s.nu) for s in systems]) as b:
        for k, s in enumerate(systems):
            b.set_system(k, s)
        b.tune()                      # optional: pick the N tile and tuple order
        ets, etd = b.forward()        # arrays, one entry per system

Every tuple of every system is a set of work items (W-build tiles, reduction
blocks) taken from one device-side queue by a persistent kernel, replayed
from a CUDA graph; per system the energies equal a single-system
``TriplesPlan`` bitwise.  ``TriplesBatch(shapes, form="int8")`` adds the
emulated executor (mode 2, its default): each system's digit count is
calibrated to the error target of the form ('int8': 1e-8 Eh, 'int8@R': R
|E(T)|, 'int8:S': S digits), and per system the energies equal
``TriplesPlan.for_form(no, nu, form)`` bitwise.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .api import _host, input_sizes


class TriplesBatch:
    def __init__(self, shapes, device: int = 0, form: str = "fp64"):
        from .api import parse_form
        lib = N.load()
        self.shapes = [(int(no), int(nu)) for no, nu in shapes]
        n = len(self.shapes)
        no = (ctypes.c_int64 * n)(*[s[0] for s in self.shapes])
        nu = (ctypes.c_int64 * n)(*[s[1] for s in self.shapes])
        opt = N.Options()
        lib.ccT_options_default(ctypes.byref(opt))
        opt.device = device
        kw = parse_form(form)
        self.emulated = kw["precision"] == "int8"
        opt.precision = N.CCT_PREC_INT8_EMU if self.emulated else N.CCT_PREC_FP64
        opt.emu_slices = kw.get("emu_slices", 0)
        if kw.get("emu_tol_rel"):
            opt.emu_tol_rel = kw["emu_tol_rel"]
        h = ctypes.c_void_p()
        N.check(lib.ccT_batch_create(ctypes.byref(h), n, no, nu, ctypes.byref(opt)), "ccT_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.load().ccT_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.shapes)

    def set_inputs(self, s: int, eh, ep, t1, t2, vm, voe, vvvo):
        no, nu = self.shapes[s]
        sizes = input_sizes(no, nu)
        arrs = dict(eh=eh, ep=ep, t1=t1, t2=t2, vm=vm, voe=voe, vvvo=vvvo)
        keep = [_host(a, sizes[k], k) for k, a in arrs.items()]
        ptrs = [ctypes.c_void_p(a.ctypes.data) for a in keep]
        N.check(N.load().ccT_batch_set_inputs(self._h, s, *ptrs, N.CCT_MEM_HOST), "ccT_batch_set_inputs")

    def set_system(self, s: int, inp):
        if (inp.no, inp.nu) != self.shapes[s]:
            raise ValueError(f"system {s}: shape {(inp.no, inp.nu)} != {self.shapes[s]}")
        self.set_inputs(s, *inp.arrays())

    def forward(self):
        """(ets, etd) arrays over the systems."""
        n = len(self.shapes)
        ets, etd = np.zeros(n), np.zeros(n)
        dp = ctypes.POINTER(ctypes.c_double)
        N.check(N.load().ccT_batch_forward(self._h, ets.ctypes.data_as(dp), etd.ctypes.data_as(dp)),
                "ccT_batch_forward")
        return ets, etd

    def v1(self, s: int) -> np.ndarray:
        no, nu = self.shapes[s]
        out = np.zeros(no * nu)
        N.check(N.load().ccT_batch_v1(self._h, s, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                "ccT_batch_v1")
        return out

    def configure(self, mode: int = 1, bn: int = 0, order: int = 0, group_bytes: int = 256 << 20):
        """mode 0: one persistent kernel over a device work queue; mode 1: grouped
        launches (W-build tiles / reduction blocks per tuple group, two streams);
        mode 2: grouped, with one emulated W-build launch per system and group
        (emulated batches).  bn: W-build N tile, 0 = per system (modes 1, 2)."""
        N.check(N.load().ccT_batch_configure(self._h, mode, bn, order, group_bytes), "ccT_batch_configure")

    def debug_stall(self, tuple_pos: int = 0, spin_limit: int = 0):
        """Testing hook (``ccT_batch_debug_stall``): make the persistent
        executor's counter wait of one tuple run out; ``tuple_pos`` < 0 clears it."""
        N.check(N.load().ccT_batch_debug_stall(self._h, tuple_pos, spin_limit), "ccT_batch_debug_stall")

    def tune(self):
        """Time every (mode, N tile, tuple order) candidate; keep the fastest.
        Returns (mode, bn, order, ms)."""
        mode, bn, order, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        N.check(N.load().ccT_batch_tune(self._h, ctypes.byref(mode), ctypes.byref(bn), ctypes.byref(order),
                                        ctypes.byref(ms)), "ccT_batch_tune")
        return mode.value, bn.value, order.value, ms.value

    @property
    def last_ms(self) -> float:
        return float(N.load().ccT_batch_last_ms(self._h))

    @property
    def work_items(self) -> int:
        return int(N.load().ccT_batch_work_items(self._h))

    def emu_digits(self, s: int) -> int:
        """Digit count of system s in the emulated executor (``ccT_batch_emu_digits``)."""
        d = ctypes.c_int32()
        N.check(N.load().ccT_batch_emu_digits(self._h, s, ctypes.byref(d)), "ccT_batch_emu_digits")
        return d.value


def main(argv=None) -> int:
    """``python -m libcc_b200.batch``: the first N systems of the 96-system
    batched workload through one executor configuration (or the tuner), one
    untimed and one timed forward; prints the device time and the energies."""
    import argparse
    from . import synthetic
    ap = argparse.ArgumentParser(prog="python -m libcc_b200.batch", description=main.__doc__)
    ap.add_argument("--systems", type=int, default=96, help="first N systems of the workload (default 96)")
    ap.add_argument("--form", default="fp64",
                    help="fp64, or int8 / int8@R / int8:S for the emulated W build (adds mode 2)")
    ap.add_argument("--mode", type=int, default=None,
                    help="0: one persistent kernel; 1: grouped launches; 2: grouped, emulated "
                         "(default: 1 for fp64, 2 for int8 forms)")
    ap.add_argument("--bn", type=int, default=0, help="W-build N tile, 0 = per system")
    ap.add_argument("--order", type=int, default=0, help="0: tuples by cost; 1: system by system")
    ap.add_argument("--group-mib", type=int, default=256, help="X scratch per tuple group, MiB")
    ap.add_argument("--tune", action="store_true", help="let the tuner pick mode, N tile and order")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    systems = synthetic.batch96(args.systems)
    with TriplesBatch([(s.no, s.nu) for s in systems], device=args.device, form=args.form) as b:
        for k, s in enumerate(systems):
            b.set_system(k, s)
        if args.tune:
            mode, bn, order, ms = b.tune()
            print(f"tuned: mode {mode} bn {bn} order {order} ({ms:.2f} ms)")
        else:
            mode = args.mode if args.mode is not None else (2 if b.emulated else 1)
            b.configure(mode, 0 if mode == 2 else args.bn, args.order, args.group_mib << 20)
        b.forward()
        ets, etd = b.forward()
        print(f"{len(systems)} systems, {b.work_items} work items, {b.last_ms:.2f} ms")
        for k, s in enumerate(systems):
            dg = ""
            try:
                dg = f" digits={b.emu_digits(k)}" if b.emulated else ""
            except N.CctError:  # the tuner chose an FP64 executor
                pass
            print(f"  {s.name} no={s.no} nu={s.nu} ets={ets[k]:.10f} etd={etd[k]:.10f}{dg}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
