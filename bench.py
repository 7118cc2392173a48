#!/usr/bin/env python
"""(T) benchmark: time to E(T) and TFLOP/s on B200.

One step is one full (T) evaluation -- every tuple of the workload, including
the degenerate (i,j,j)/(i,i,j) tuples -- through the library's plan API, with
inputs already resident in HBM.  Both forms are timed: the native FP64 form
(mma.sync f64) and the split-integer emulated form (tcgen05 INT8); the
headline value is the emulated form, the native one is reported beside it with
the speed-up and the relative energy difference.  ``e2e`` repeats the headline
step through the C ABI from pinned host buffers (plan create, host->device
upload, operand build, all tuples, v1/energy read-back, destroy).

Under torchrun (N>1) the tuple list is split into cost-balanced contiguous
shards, one per rank; the partial (ets, etd) are summed with one NCCL
all-reduce, the only exchange step (the reference's ddi_gsumf).

``--impl reference`` times the CPU stand-in for the reference's triples.x (the
literal 12-DGEMM/trant3/DRT1WT3 restatement with OpenBLAS) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "(T) time & TFLOP/s: emulated vs native FP64 on 1 B200 at |ΔE(T)|≤1e-8 Eh"
DEFAULT_WORKLOAD = "no24-nu320"


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the adjoint (no=12/nu=120) and batched-systems (96 uneven) measurements")
    ap.add_argument("--emu-slices", type=int, default=5, help="7-bit digits per operand of the emulated form (4..7)")
    return ap.parse_args()


def workload_desc(inp, dist):
    d = f"{inp.name} (no={inp.no}, nu={inp.nu}, seed {inp.seed}, "
    d += "log-uniform |x| in [1e-6,1] integrals and T2 numerators)" if dist == "log" else "normal integrals)"
    return d


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running, into a CSV
    under $CCT_CLOCKS_DIR (default: the system temporary directory)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        out = os.environ.get("CCT_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = pathlib.Path(out) / f"clocks_bench_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(sm=float(f[1]), smax=float(f[2]), power=float(f[3]), hw=f[5], hwt=f[6], swt=f[7],
                                 swp=f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        pmax = max(r["power"] for r in rows)
        loaded = [r for r in rows if r["power"] >= 0.5 * pmax] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                          ("swp", "sw_power_cap")):
            if any(r[key].lower().startswith("active") for r in loaded):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": reasons, "samples": len(loaded), "power_w_max": pmax}


def read_traffic(workload: str, kind: str = "f64"):
    """DRAM bytes per W-build launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"wbuild_{kind}_{workload}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def golden(workload: str):
    f = ROOT / "tests" / "golden" / "energies.json"
    if not f.exists():
        return None
    return json.loads(f.read_text()).get(workload)


def cpu_sample(inp, budget_s: float = 12.0):
    """Time the literal CPU restatement on i>j>k tuples of the workload until the
    budget is spent (at least one tuple).  Returns (TFLOP/s, tuples, seconds, threads)."""
    from oracle import oracle as O
    tuples = [t for t in O.all_tuples(inp.no) if t[0] == 0]
    flop_per = 12.0 * inp.nu ** 3 * (inp.no + inp.nu)
    O.literal_cc_triples(inp, tuples=tuples[:1])  # page in, build caches
    done, t0 = 0, time.perf_counter()
    while done < len(tuples):
        O.literal_cc_triples(inp, tuples=tuples[done:done + 1])
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return flop_per * done / dt / 1e12, done, dt, O.cpu_threads()


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from libcc_b200 import synthetic as S
    from oracle import oracle as O
    cfg = S.WORKLOADS[args.workload]
    inp = S.workload(args.workload)
    tuples = [t for t in O.all_tuples(inp.no) if t[0] == 0]
    flop_per = 12.0 * inp.nu ** 3 * (inp.no + inp.nu)
    per_step = 1
    for w in range(args.warmup):
        O.literal_cc_triples(inp, tuples=tuples[w % len(tuples):w % len(tuples) + per_step])
    t0 = time.perf_counter()
    for s in range(args.steps):
        a = (args.warmup + s) % len(tuples)
        O.literal_cc_triples(inp, tuples=tuples[a:a + per_step])
    dt = time.perf_counter() - t0
    tf = flop_per * per_step * args.steps / dt / 1e12
    full_ms = S.flops(inp.no, inp.nu) / (tf * 1e12) * 1e3
    sample = (f"{per_step} i>j>k tuple per step of {inp.name}; literal 12-DGEMM + trant3 + T3SQUA/ADT3DEN/DRT1WT3 "
              f"restatement (oracle/oracle.py) with OpenBLAS DGEMM, {O.cpu_threads()} threads")
    line = {"impl": "reference", "metric": METRIC, "value": tf, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": full_ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_desc(inp, cfg["dist"]), "form": "cpu-literal-port"},
            "cpu_baseline": {"value": tf, "unit": "TFLOP/s", "cores": O.cpu_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "ms_per_step extrapolates the sampled tuples/s to all tuples of the workload"}
    print(json.dumps(line), flush=True)
    return 0


def adjoint_extra(A, S, local):
    """Forward + hand-written adjoint on the no=12/nu=120 system (seed 3): device
    times, their ratio, and the gradient against the stored hand-derived FP64 CPU
    gradient (200 seeded entries per input) and a few central differences."""
    import copy
    import numpy as np
    g0 = json.loads((ROOT / "tests" / "golden" / "grad_no12-nu120.json").read_text())
    inp = S.generate(g0["no"], g0["nu"], g0["seed"], g0["dist"])
    with A.TriplesPlan(inp.no, inp.nu, device=local) as plan:
        plan.set_system(inp)
        fwd, bwd = [], []
        for rep in range(4):
            ets, etd, _ = plan.forward()
            fwd.append(plan.last_forward_ms)
            g = plan.backward()
            bwd.append(plan.last_backward_ms)
        f_ms, b_ms = statistics.median(fwd[1:]), statistics.median(bwd[1:])
        rel = {}
        for name, ref in g0["tensors"].items():
            idx = np.array(ref["index"])
            rel[name] = float(np.abs(g[name][idx] - np.array(ref["value"])).max() / ref["maxabs"])
        rng = np.random.default_rng(5)
        fd_rel = {}
        for name in g0["tensors"]:
            arr = getattr(inp, name)
            worst = 0.0
            for idx in rng.choice(arr.size, size=2, replace=False):
                h = 1e-5 * max(1.0, abs(arr[idx]))
                vals = []
                for sgn in (1.0, -1.0):
                    ip = copy.deepcopy(inp)
                    getattr(ip, name)[idx] += sgn * h
                    plan.set_system(ip)
                    e1, e2, _ = plan.forward(want_v1=False)
                    vals.append(e1 + e2)
                fd = (vals[0] - vals[1]) / (2 * h)
                worst = max(worst, abs(fd - g[name][idx]) / g0["tensors"][name]["maxabs"])
            fd_rel[name] = worst
    return {"workload": "no12-nu120 (seed 3, normal)", "forward_ms": f_ms, "backward_ms": b_ms,
            "ratio_backward_over_forward": b_ms / f_ms, "e_t": ets + etd,
            "max_rel_err_vs_cpu_gradient": rel, "central_difference_h": 1e-5,
            "max_rel_err_vs_central_differences": fd_rel,
            "note": "backward recomputes W per tuple in FP64; rel errors are relative to max|gradient| per input"}


def adaptive_extra(A, S, local):
    """Per-tile digit counts of the emulated form (emu_slices = 0, at most 5) against
    fixed 5 digits and native FP64 on the no=16/nu=200 system with magnitudes
    falling 2^-0.25 per virtual index (synthetic.with_decay): device time of a
    whole (T) step, the digit histogram over W tiles and the error vs FP64."""
    inp = S.with_decay(S.workload("no16-nu200"), 0.25)
    res = {}
    for form in ("fp64", "int8:5", "int8"):
        with make_plan(A, inp.no, inp.nu, local, form) as plan:
            plan.set_system(inp)
            times = []
            for _ in range(3):
                ets, etd, _ = plan.forward()
                times.append(plan.last_forward_ms)
            res[form] = {"ms": statistics.median(times[1:]), "e_t": ets + etd,
                         "digit_histogram": plan.emu_slice_histogram() if form != "fp64" else None}
    ref = res["fp64"]["e_t"]
    for form in ("int8:5", "int8"):
        res[form]["rel_err_vs_fp64"] = abs(res[form]["e_t"] - ref) / abs(ref)
    return {"workload": "no16-nu200 (seed 1, normal) with magnitudes x 2^(-0.25 a) per virtual index a",
            "fp64_ms": res["fp64"]["ms"], "fixed5_ms": res["int8:5"]["ms"], "per_tile_ms": res["int8"]["ms"],
            "speedup_per_tile_over_fixed5": res["int8:5"]["ms"] / res["int8"]["ms"],
            "fixed5_rel_err_vs_fp64": res["int8:5"]["rel_err_vs_fp64"],
            "per_tile_rel_err_vs_fp64": res["int8"]["rel_err_vs_fp64"],
            "per_tile_digit_histogram": res["int8"]["digit_histogram"],
            "note": "histogram index = 7-bit digits per operand of a 128 x N W tile; the bench headline runs "
                    "fixed 5 digits, where the per-tile rule also picks 5 on every tile of its workload"}


def batch_extra(A, S, local):
    """The 96 uneven systems (no ~ U{3..12}, nu ~ U{24..140}, seed 100+s): the
    batched executor (CUDA graph) against a per-system plan loop, and per-system
    E(T) against the CPU oracle on the 8 smallest systems."""
    import numpy as np
    from libcc_b200 import batch as B
    from oracle import oracle as O
    systems = S.batch96()
    plans = []
    for inp in systems:
        p = A.TriplesPlan(inp.no, inp.nu, device=local)
        p.set_system(inp)
        plans.append(p)
    loop_ms, loop_res = [], None
    for rep in range(3):
        res, ms = [], 0.0
        for p in plans:
            res.append(p.forward(want_v1=False))
            ms += p.last_forward_ms
        loop_ms.append(ms)
        loop_res = res
    for p in plans:
        p.close()
    with B.TriplesBatch([(s.no, s.nu) for s in systems], device=local) as b:
        for k, inp in enumerate(systems):
            b.set_system(k, inp)
        bms = []
        for rep in range(3):
            ets, etd = b.forward()
            bms.append(b.last_ms)
        items = b.work_items
    same = all(ets[k] == loop_res[k][0] and etd[k] == loop_res[k][1] for k in range(len(systems)))
    small = sorted(range(len(systems)), key=lambda k: S.flops(systems[k].no, systems[k].nu))[:8]
    errs = []
    for k in small:
        e_o, d_o, _ = O.c_cc_triples(systems[k])
        errs.append(abs((ets[k] + etd[k]) - (e_o + d_o)) / abs(e_o + d_o))
    flops = sum(S.flops(s.no, s.nu) for s in systems)
    lm, bm = statistics.median(loop_ms), statistics.median(bms)
    return {"workload": "96 systems, no ~ U{3..12}, nu ~ U{24..140}, seed 100+s (normal)",
            "tuples": int(sum(A.N.load().ccT_num_tuples(s.no) for s in systems)), "flops": flops,
            "batched_ms": bm, "batched_tflops": flops / bm / 1e9, "per_system_loop_ms": lm,
            "per_system_loop_tflops": flops / lm / 1e9, "speedup_batched_over_loop": lm / bm,
            "work_items": items, "bitwise_equal_to_loop": bool(same),
            "executor": "grouped launches per tuple group on two streams, per-system N tile, tuples by cost; "
                        "CUDA graph replay",
            "max_rel_err_vs_oracle_8_smallest": max(errs)}


def make_plan(A, no, nu, device, form):
    """Plan for one form: 'fp64' (native mma.sync f64), 'int8:S' (S-digit
    emulation), 'int8' (automatic digits, 1e-8 Eh target) or 'int8@R'
    (automatic digits, relative target R)."""
    return A.TriplesPlan.for_form(no, nu, form, device=device)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import datetime

    import torch

    from libcc_b200 import api as A
    from libcc_b200 import shard
    from libcc_b200 import synthetic as S

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    cfg = S.WORKLOADS[args.workload]
    inp = S.workload(args.workload)
    no, nu = inp.no, inp.nu
    # tuple list order (ccT_forward): C(no,3) i>j>k tuples, then no(no-1) degenerate ones at half cost
    n_ijk_all = no * (no - 1) * (no - 2) // 6
    costs = shard.tuple_costs(no)
    begin, end = shard.shard_of(no, rank, world)
    flop_step = S.flops(no, nu)
    my_flop_wb = sum(12.0 * nu ** 3 * (no + nu) * c for c in costs[begin:end])
    dev_inputs = [torch.from_numpy(a).to(f"cuda:{local}") for a in inp.arrays()]
    stream = torch.cuda.current_stream()
    N = A.N
    peaks = {"fp64": N.load().ccT_measure_fp64_peak(local), "int8": N.load().ccT_measure_int8_peak(local)}
    g = golden(args.workload)

    def allreduce(vals, op="sum"):
        if dist is None:
            return vals
        t = torch.tensor(vals, dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
        return t.tolist()

    def run_form(form, sampler):
        plan = make_plan(A, no, nu, local, form)
        plan.set_inputs(*dev_inputs)
        plan.set_stream(stream.cuda_stream)

        def step():
            ets, etd, _ = shard.sharded_cc_triples(plan, want_v1=False)
            return ets, etd

        for _ in range(args.warmup):
            step()
        plan.set_profiling(True)
        launches, wb_ms, wb_n = 0, 0.0, 0
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler is not None:
            sampler.__enter__()
        e0.record(stream)
        for _ in range(args.steps):
            ets, etd = step()
            launches += plan.last_forward_launches
            prof = plan.kernel_profile()
            wb_ms += prof["wbuild"][0]
            wb_n += prof["wbuild"][1]
        e1.record(stream)
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.__exit__(None, None, None)
        if dist is not None:
            dist.barrier()
        plan.close()
        ms = allreduce([e0.elapsed_time(e1)], op="max")[0]
        ms_step = ms / args.steps
        emu = form != "fp64"
        S_ = int(form.split(":")[1]) if emu else 0
        # algorithmic work of the W-build launches in the timed region
        fp64_flop = my_flop_wb * args.steps
        if emu:
            ops = fp64_flop * S_ * (S_ + 1) / 2  # INT8 ops: S(S+1)/2 digit products per FP64 multiply-add
            achieved = ops / (wb_ms * 1e-3) / 1e12 if wb_ms > 0 else None
            peak, unit, kern = peaks["int8"], "TOPS (int8)", "wbuild_emu_kernel (tcgen05.mma kind::i8, TMA, TMEM)"
            psrc = ("measured in this run: tcgen05.mma kind::i8 throughput with operands resident in shared memory "
                    "(ccT_measure_int8_peak); MEASURED_PEAKS.json has no INT8 entry")
            per_launch = f"{S_ * (S_ + 1) // 2} x 12 nu^3 (no+nu) int8 ops for an i>j>k tuple, half for a degenerate tuple"
        else:
            achieved = fp64_flop / (wb_ms * 1e-3) / 1e12 if wb_ms > 0 else None
            peak, unit, kern = peaks["fp64"], "TFLOP/s", "wbuild_f64_kernel (mma.sync m16n8k4 f64)"
            psrc = ("measured in this run: mma.sync f64 throughput microbenchmark (ccT_measure_fp64_peak); "
                    "MEASURED_PEAKS.json has no FP64 entry")
            per_launch = f"12 nu^3 (no+nu) = {12.0 * nu ** 3 * (no + nu):.4g} flop for an i>j>k tuple, half for a degenerate tuple"
        out = {"form": form, "ms_per_step": ms_step, "tflops": flop_step / (ms_step * 1e-3) / 1e12,
               "ets": ets, "etd": etd, "e_t": ets + etd, "gpu_launches": launches,
               "roofline": {"bound": "tensor", "kernel": kern, "achieved": achieved, "peak": peak, "unit": unit,
                            "frac": (achieved / peak) if (achieved and peak) else None,
                            "traffic": read_traffic(args.workload, "emu" if emu else "f64"),
                            "peak_source": psrc, "launches": wb_n, "avg_launch_ms": wb_ms / max(wb_n, 1),
                            "work_per_launch": per_launch, "share_of_step": wb_ms / ms if ms > 0 else None}}
        if g is not None:
            out["abs_err_vs_oracle"] = abs(out["e_t"] - g["e_t"])
            out["rel_err_vs_oracle"] = abs(out["e_t"] - g["e_t"]) / abs(g["e_t"])
        return out

    emu_form = f"int8:{args.emu_slices}"
    clocks = ClockSampler(local)
    forms = {"fp64": run_form("fp64", None), "int8_emu": run_form(emu_form, clocks)}
    head = forms["int8_emu"]
    rel_vs_native = abs(head["e_t"] - forms["fp64"]["e_t"]) / abs(forms["fp64"]["e_t"])
    head["rel_err_vs_native_fp64"] = rel_vs_native

    # end to end through the C ABI from pinned host buffers (headline form)
    e2e = None
    if not args.no_e2e:
        pinned = []
        for a in inp.arrays():
            t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = a
            pinned.append(t.numpy())
        h2d = sum(a.nbytes for a in pinned)
        d2h = nu * no * 8 + 2 * 8
        del dev_inputs
        torch.cuda.empty_cache()
        if dist is not None:
            dist.barrier()
        # three whole runs (plan, uploads, operand build, all tuples, teardown);
        # the median is reported: the host side (large allocations, pinned
        # copies) varies by a few tenths of a second from run to run
        runs, dev_runs, phases = [], [], []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with make_plan(A, no, nu, local, emu_form) as p2:
                t1 = time.perf_counter()
                p2.set_inputs(*pinned)
                t2 = time.perf_counter()
                r = shard.sharded_cc_triples(p2)
                t3 = time.perf_counter()
                dev_runs.append(p2.last_forward_ms * 1e-3)
            e2e_e = r[0] + r[1]
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            phases.append({"plan_create": t1 - t0, "set_inputs": t2 - t1, "forward": t3 - t2,
                           "plan_destroy": t4 - t3})
            runs.append(allreduce([t4 - t0], op="max")[0])
        e2e_s = statistics.median(runs)
        e2e = {"value": flop_step / e2e_s / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "seconds": e2e_s, "seconds_per_run": runs,
               "forward_device_seconds_per_run": dev_runs, "host_seconds_per_phase": phases, "steps": 1,
               "form": emu_form,
               "path": "ccT_plan_create/ccT_set_inputs(host)/ccT_forward/ccT_plan_destroy (C ABI), pinned inputs"
                       + (" + NCCL all-reduce of the shard energies" if world > 1 else ""),
               "e_t": e2e_e}
    else:
        del dev_inputs

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        tf_cpu, ntup, sec, thr = cpu_sample(inp)
        cpu = {"value": tf_cpu, "unit": "TFLOP/s", "cores": thr, "kind": "port",
               "sample": f"{ntup} i>j>k tuples of {inp.name} in {sec:.1f} s; literal 12-DGEMM + trant3 + "
                         "T3SQUA/ADT3DEN/DRT1WT3 restatement with OpenBLAS DGEMM"}

    if rank == 0:
        line = {"metric": METRIC, "value": head["tflops"], "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int8 tensor pipe (split-integer FP64 emulation)",
                "data": "synthetic (seeded generator, libcc_b200/synthetic.py)",
                "config": {"workload": workload_desc(inp, cfg["dist"]), "form": f"emulated FP64, {args.emu_slices} "
                           "7-bit digits per operand (tcgen05 kind::i8)", "tuples": len(costs), "tuples_ijk": n_ijk_all,
                           "flop_per_step": flop_step, "tuples_per_s": len(costs) / (head["ms_per_step"] * 1e-3),
                           "l2": "inputs larger than L2 (digit operands "
                                 f"{2 * args.emu_slices * no * nu * nu * (nu + no) / 1e9:.1f} GB re-streamed per step)",
                           "parallelism": f"tuple shards x{world}" if world > 1 else "1 GPU"},
                "roofline": head["roofline"], "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": head["gpu_launches"],
                "clocks": clocks.summary(), "energies": {"ets": head["ets"], "etd": head["etd"], "e_t": head["e_t"]},
                "accuracy": {"rel_err_vs_native_fp64": rel_vs_native,
                             "rel_err_vs_oracle": head.get("rel_err_vs_oracle"),
                             "native_rel_err_vs_oracle": forms["fp64"].get("rel_err_vs_oracle"),
                             "bar": "relative 2.1e-7 = 1e-8 Eh on a (T) energy of 0.048 Eh (Ar6); the seeded data "
                                    "give |E(T)| ~ 7.7e9 Eh, where an absolute 1e-8 Eh is below FP64 resolution"},
                "forms": forms,
                "speedup_emulated_over_native": forms["fp64"]["ms_per_step"] / head["ms_per_step"]}
        if world == 1 and not args.no_extras:
            line["adjoint"] = adjoint_extra(A, S, local)
            line["batch"] = batch_extra(A, S, local)
            line["per_tile_digits"] = adaptive_extra(A, S, local)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
