"""Host-side mirror of the reference's (T) driver interface over the C ABI.

* ``cc_triples``     -- whole (T) evaluation, the single-GPU form of
                        ``cc_triples_acc`` (src/triples-ijk/triples.F90:1) with the
                        packed VVVO passed in place of the DDI handle.
* ``IjkGpuHooks``    -- ``ijk_gpu_init`` / ``ijk_gpu_driver`` / ``ijk_gpu_finalize``,
                        the per-tuple GPU hooks of the hybrid CUDA build
                        (triples_cpu.F90:363,465,497; ddcc_t_ijk_big_cuda.f:12).
* ``TriplesPlan``    -- the status-returning plan API (create, set inputs once,
                        forward over any tuple range).

Arrays are flat float64 in the reference's Fortran layouts (see
libcc_b200/synthetic.py).  Device arrays may be passed as CUDA tensors (any
object with ``data_ptr()`` and ``is_cuda``); they are read in place.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

_dp = ctypes.POINTER(ctypes.c_double)


def _host(a, n: int, name: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    if a.size != n:
        raise ValueError(f"{name}: expected {n} elements, got {a.size}")
    return a


def _is_device(a) -> bool:
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def format_energies(ets: float, etd: float) -> str:
    """The reference's result line (triples.F90:316,332: format '(1x,a,3F15.10)')."""
    return " ets/etd/ets+etd=" + "".join(f"{x:15.10f}" for x in (ets, etd, ets + etd))


def input_sizes(no: int, nu: int):
    nutr = nu * (nu + 1) // 2
    return dict(eh=no, ep=nu, t1=no * nu, t2=nu * nu * no * no, vm=no * nu * no * no,
                voe=nu * nu * no * no, vvvo=nutr * nu * no)


def parse_form(form: str) -> dict:
    """Plan keyword arguments of a form name: 'fp64' (native FP64), 'int8'
    (emulated, automatic digit count), 'int8:S' (emulated, S digits on every
    tile) or 'int8@R' (emulated, automatic digits with relative target R)."""
    if form == "fp64":
        return dict(precision="fp64")
    if form == "int8":
        return dict(precision="int8")
    if form.startswith("int8:"):
        return dict(precision="int8", emu_slices=int(form[5:]))
    if form.startswith("int8@"):
        return dict(precision="int8", emu_tol_rel=float(form[5:]))
    raise ValueError(f"unknown form {form!r}")


class TriplesPlan:
    """Device plan for one system: owns the HBM buffers that replace the DDI arrays.

    ``precision`` is "fp64" (native FP64 tensor-core W build) or "int8"
    (split-integer emulation).  Emulated plans take ``emu_slices`` (0: the
    digit count is calibrated in ``set_inputs`` against the target
    max(emu_tol, emu_tol_rel |E(T)|); 3..7: that many digits on every tile);
    ``emu_tol`` / ``emu_tol_rel`` of 0 keep the library defaults (1e-8 Eh,
    2e-14).  ``vvvo`` ("auto", "expanded", "packed") says whether an FP64 plan
    expands VVVO into the W build's operand or keeps the packed triangle
    resident and gathers rows from it (``CCT_VVVO_*``).  ``keep_w``: an FP64
    plan's forward keeps every tuple's W-build output on the device when it
    fits, and the backward reads it instead of rebuilding W
    (``ccT_options.keep_w``, ``kept_tuples``)."""

    def __init__(self, no: int, nu: int, precision: str = "fp64", device: int = 0, check_inputs: bool = True,
                 emu_slices: int = 0, emu_tol: float = 0.0, emu_tol_rel: float = 0.0, vvvo: str = "auto",
                 keep_w: bool = False):
        lib = N.load()
        opt = N.Options()
        lib.ccT_options_default(ctypes.byref(opt))
        opt.precision = {"fp64": N.CCT_PREC_FP64, "int8": N.CCT_PREC_INT8_EMU}[precision]
        opt.device = device
        opt.check_inputs = 1 if check_inputs else 0
        opt.emu_slices = emu_slices
        if emu_tol:
            opt.emu_tol = emu_tol
        if emu_tol_rel:
            opt.emu_tol_rel = emu_tol_rel
        opt.vvvo_mode = {"auto": N.CCT_VVVO_AUTO, "expanded": N.CCT_VVVO_EXPANDED, "packed": N.CCT_VVVO_PACKED}[vvvo]
        opt.keep_w = 1 if keep_w else 0
        h = ctypes.c_void_p()
        N.check(lib.ccT_plan_create(ctypes.byref(h), no, nu, ctypes.byref(opt)), "ccT_plan_create")
        self._h = h
        self.no, self.nu, self.precision, self.device = no, nu, precision, device
        self.num_tuples = int(lib.ccT_num_tuples(no))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.load().ccT_plan_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @classmethod
    def for_form(cls, no: int, nu: int, form: str, device: int = 0, **kw):
        """Plan for a form name (``parse_form``)."""
        return cls(no, nu, device=device, **parse_form(form), **kw)

    def set_inputs(self, eh, ep, t1, t2, vm, voe, vvvo):
        """Load the seven input arrays (all host numpy arrays, or all CUDA tensors).
        Device tensors are read after all work on the device has finished (the
        plan's own stream), or in order on the caller's stream after
        ``set_stream``."""
        arrs = dict(eh=eh, ep=ep, t1=t1, t2=t2, vm=vm, voe=voe, vvvo=vvvo)
        sizes = input_sizes(self.no, self.nu)
        dev = [_is_device(a) for a in arrs.values()]
        if any(dev) and not all(dev):
            raise ValueError("pass either all host arrays or all device tensors")
        if all(dev):
            ptrs = []
            for name, a in arrs.items():
                if a.numel() != sizes[name] or not a.is_contiguous() or str(a.dtype) != "torch.float64":
                    raise ValueError(f"{name}: need a contiguous float64 tensor of {sizes[name]} elements")
                ptrs.append(ctypes.c_void_p(a.data_ptr()))
            mem = N.CCT_MEM_DEVICE
            keep = None
        else:
            keep = [_host(a, sizes[name], name) for name, a in arrs.items()]
            ptrs = [ctypes.c_void_p(a.ctypes.data) for a in keep]
            mem = N.CCT_MEM_HOST
        N.check(N.load().ccT_set_inputs(self._h, *ptrs, mem), "ccT_set_inputs")
        del keep

    def set_system(self, inp):
        """Load a ``synthetic.TriplesInputs``."""
        self.set_inputs(*inp.arrays())

    def forward(self, begin: int = 0, end: int | None = None, want_v1: bool = True):
        """Run tuples [begin, end).  Returns (ets, etd, v1[nu*no] or None)."""
        end = self.num_tuples if end is None else end
        ets, etd = ctypes.c_double(), ctypes.c_double()
        v1 = np.zeros(self.nu * self.no) if want_v1 else None
        vptr = ctypes.c_void_p(v1.ctypes.data) if want_v1 else None
        N.check(N.load().ccT_forward(self._h, begin, end, ctypes.byref(ets), ctypes.byref(etd), vptr), "ccT_forward")
        return ets.value, etd.value, v1

    def backward(self, begin: int = 0, end: int | None = None) -> dict:
        """Gradient of E(T) = ets + etd of the last ``forward(begin, end)`` with
        respect to every input, as host arrays in the input layouts: keys eh,
        ep, t1, t2, vm, voe, vvvo (``ccT_backward``)."""
        end = self.num_tuples if end is None else end
        sizes = input_sizes(self.no, self.nu)
        out = {k: np.zeros(sizes[k]) for k in ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo")}
        ptrs = [ctypes.c_void_p(out[k].ctypes.data) for k in ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo")]
        N.check(N.load().ccT_backward(self._h, begin, end, *ptrs, N.CCT_MEM_HOST), "ccT_backward")
        return out

    def emu_digits(self) -> dict:
        """Emulated plans: the digit count the W build runs, the calibrated bound
        on |dE(T)| against the FP64 form and its target (``ccT_emu_digits``)."""
        dg, err, tgt = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        N.check(N.load().ccT_emu_digits(self._h, ctypes.byref(dg), ctypes.byref(err), ctypes.byref(tgt)),
                "ccT_emu_digits")
        return {"digits": dg.value, "est_err": err.value, "target": tgt.value}

    def tuple_w(self, tuple_index: int) -> np.ndarray:
        """W_abc of one tuple as this plan's W build forms it, flat in the
        reference's layout (a fastest), nu^3 doubles (``ccT_tuple_w``)."""
        w = np.empty(self.nu ** 3)
        N.check(N.load().ccT_tuple_w(self._h, tuple_index, ctypes.c_void_p(w.ctypes.data), N.CCT_MEM_HOST),
                "ccT_tuple_w")
        return w

    @property
    def last_backward_ms(self) -> float:
        return float(N.load().ccT_last_backward_ms(self._h))

    @property
    def kept_tuples(self) -> int:
        """Tuples whose W-build output the last forward kept for the backward
        (``keep_w``); 0 when it kept none."""
        return int(N.load().ccT_kept_tuples(self._h))

    def emu_slice_histogram(self) -> list:
        """Emulated plans: work items of the last forward per digit count
        (index s = digits per operand, 0..7); all zero for FP64 plans."""
        h = (ctypes.c_int64 * 8)()
        N.check(N.load().ccT_emu_slice_histogram(self._h, h, 8), "ccT_emu_slice_histogram")
        return [int(v) for v in h]

    def set_stream(self, stream_handle: int | None):
        """Run on a caller's CUDA stream (an integer cudaStream_t, e.g.
        ``torch.cuda.current_stream().cuda_stream``); None restores the plan's own."""
        N.check(N.load().ccT_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)), "ccT_set_stream")

    def time_wbuild(self, tuple_index: int = 0, reps: int = 3) -> float:
        """Mean milliseconds of one W-build launch of the given tuple (CUDA events)."""
        ms = ctypes.c_double()
        N.check(N.load().ccT_time_wbuild(self._h, tuple_index, reps, ctypes.byref(ms)), "ccT_time_wbuild")
        return ms.value

    @property
    def last_forward_ms(self) -> float:
        return float(N.load().ccT_last_forward_ms(self._h))

    @property
    def last_forward_launches(self) -> int:
        return int(N.load().ccT_last_forward_launches(self._h))


def cc_triples(no: int, nu: int, eh, ep, t1, t2, vm, voe, vvvo):
    """Whole (T) on one GPU through ``cc_triples_b200_``.  Returns (ets, etd, v1)."""
    sizes = input_sizes(no, nu)
    arrs = [_host(a, sizes[n], n) for n, a in zip(("eh", "ep", "t1", "t2", "vm", "voe", "vvvo"),
                                                    (eh, ep, t1, t2, vm, voe, vvvo))]
    v1 = np.zeros(no * nu)
    ets, etd = ctypes.c_double(), ctypes.c_double()
    n_o, n_u = ctypes.c_int64(no), ctypes.c_int64(nu)
    p = lambda a: a.ctypes.data_as(_dp)
    eh_, ep_, t1_, t2_, vm_, voe_, vvvo_ = arrs
    N.load().cc_triples_b200_(ctypes.byref(n_o), ctypes.byref(n_u), p(eh_), p(ep_), p(v1), p(t1_), p(t2_), p(vm_),
                              p(voe_), p(vvvo_), ctypes.byref(ets), ctypes.byref(etd))
    return ets.value, etd.value, v1


def ccsd_terms_29_31(no: int, nu: int, o1, t2, vl, vr, vvvo) -> np.ndarray:
    """The reference CCSD port's terms_29_30_31 (ccsd_acc.f:1-60) through
    ``ccT_ccsd_terms_29_31``; returns the updated t2 (host arrays in, host out)."""
    n4 = no * nu * nu * no
    nutr = nu * (nu + 1) // 2
    a = [_host(o1, no * nu, "o1"), _host(t2, n4, "t2").copy(), _host(vl, n4, "vl"), _host(vr, n4, "vr"),
         _host(vvvo, nutr * nu * no, "vvvo")]
    ptr = [ctypes.c_void_p(x.ctypes.data) for x in a]
    N.check(N.load().ccT_ccsd_terms_29_31(no, nu, *ptr, N.CCT_MEM_HOST), "ccT_ccsd_terms_29_31")
    return a[1]


def ccsd_terms_32_35(no: int, nu: int, o1, o2, t2, vm, vvvo):
    """The reference CCSD port's terms_32_33_34_35 (ccsd_acc.f:64-160) through
    ``ccT_ccsd_terms_32_35``; returns (t2, o2, vm, rl) as the routine leaves them."""
    n4 = no * nu * nu * no
    nutr = nu * (nu + 1) // 2
    o1h = _host(o1, no * nu, "o1")
    o2h, t2h, vmh = _host(o2, n4, "o2").copy(), _host(t2, n4, "t2").copy(), _host(vm, no ** 3 * nu, "vm").copy()
    rl = np.zeros(n4)
    vv = _host(vvvo, nutr * nu * no, "vvvo")
    ptr = [ctypes.c_void_p(x.ctypes.data) for x in (o1h, o2h, t2h, vmh, rl, vv)]
    N.check(N.load().ccT_ccsd_terms_32_35(no, nu, *ptr, N.CCT_MEM_HOST), "ccT_ccsd_terms_32_35")
    return t2h, o2h, vmh, rl


def ccsd_release_workspace() -> None:
    """Frees the device workspace the CCSD-term entry points keep between calls."""
    N.check(N.load().ccT_ccsd_release_workspace(), "ccT_ccsd_release_workspace")


def packed_columns(vvvo: np.ndarray, no: int, nu: int, x: int) -> np.ndarray:
    """The nu packed VVVO columns of occupied index x (0-based), as ddi_get fetches
    them for the GPU hook (triples_cpu.F90:428-450)."""
    nutr = nu * (nu + 1) // 2
    return np.ascontiguousarray(vvvo.reshape(nu * no, nutr)[x * nu:(x + 1) * nu]).ravel()


class IjkGpuHooks:
    """The hybrid build's GPU hooks.  Occupied indices are 1-based as in Fortran."""

    def __init__(self, no: int, nu: int, eh, ep, t2, vm, voe):
        self.no, self.nu = no, nu
        sizes = input_sizes(no, nu)
        self._keep = dict(eh=_host(eh, no, "eh"), ep=_host(ep, nu, "ep"), t2=_host(t2, sizes["t2"], "t2"),
                          vm=_host(vm, sizes["vm"], "vm"), voe=_host(voe, sizes["voe"], "voe"))
        self.v1 = np.zeros(no * nu)
        self.etd = ctypes.c_double(0.0)
        p = lambda a: a.ctypes.data_as(_dp)
        k = self._keep
        N.load().ijk_gpu_init_(ctypes.byref(ctypes.c_int64(no)), ctypes.byref(ctypes.c_int64(nu)), p(k["eh"]),
                               p(k["ep"]), p(self.v1), p(k["t2"]), p(k["vm"]), p(k["voe"]))

    def driver(self, i: int, j: int, k: int, ve_i, ve_j, ve_k):
        p = lambda a: a.ctypes.data_as(_dp)
        n = self.nu * (self.nu + 1) // 2 * self.nu
        vs = [_host(v, n, "ve") for v in (ve_i, ve_j, ve_k)]
        c = lambda v: ctypes.byref(ctypes.c_int64(v))
        N.load().ijk_gpu_driver_(c(self.nu), c(self.no), c(i), c(j), c(k), p(vs[0]), p(vs[1]), p(vs[2]),
                                 p(self.v1), p(self._keep["eh"]), p(self._keep["ep"]), ctypes.byref(self.etd))

    def finalize(self) -> float:
        c = lambda v: ctypes.byref(ctypes.c_int64(v))
        N.load().ijk_gpu_finalize_(c(self.no), c(self.nu), ctypes.byref(self.etd))
        return self.etd.value


def _kernel_profile(plan: TriplesPlan):
    """{class: (total_ms, launches)} of the last profiled forward."""
    out = {}
    for cls, name in ((0, "wbuild"), (1, "reduce")):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        N.check(N.load().ccT_last_kernel_ms(plan._h, cls, ctypes.byref(ms), ctypes.byref(n)), "ccT_last_kernel_ms")
        out[name] = (ms.value, n.value)
    return out


def _set_profiling(plan: TriplesPlan, on: bool):
    N.check(N.load().ccT_set_profiling(plan._h, 1 if on else 0), "ccT_set_profiling")


TriplesPlan.kernel_profile = _kernel_profile
TriplesPlan.set_profiling = _set_profiling
