"""ccT_backward (hand-written adjoint kernels) against the hand-derived FP64 CPU
gradient and central finite differences of the GPU forward."""
import copy

import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu

NAMES = ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo")


@pytest.fixture(scope="module")
def api():
    from libcc_b200 import api as A
    return A


def _close(got, ref, rel=1e-10):
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(got - ref).max() <= rel * scale


@pytest.mark.parametrize("no,nu,seed", [(4, 7, 0), (5, 16, 1), (3, 9, 2), (2, 12, 3), (6, 40, 4), (5, 33, 6)])
def test_backward_matches_cpu_adjoint(api, no, nu, seed):
    from oracle import oracle as O
    inp = S.generate(no, nu, seed)
    ref = O.closed_grad(inp)
    with api.TriplesPlan(no, nu) as plan:
        plan.set_system(inp)
        plan.forward()
        g = plan.backward()
    for name in NAMES:
        assert _close(g[name], ref[name]), (name, np.abs(g[name] - ref[name]).max(), np.abs(ref[name]).max())


def test_backward_of_a_tuple_range(api):
    from oracle import oracle as O
    no, nu = 5, 20
    inp = S.generate(no, nu, 11)
    tuples = O.all_tuples(no)
    for begin, end in [(0, 4), (7, 10), (10, len(tuples))]:
        ref = O.closed_grad(inp, tuples[begin:end])
        with api.TriplesPlan(no, nu) as plan:
            plan.set_system(inp)
            plan.forward(begin, end)
            g = plan.backward(begin, end)
        for name in NAMES:
            assert _close(g[name], ref[name]), (begin, end, name)


def test_backward_needs_matching_forward(api):
    from libcc_b200 import _native as N
    inp = S.generate(4, 10, 3)
    with api.TriplesPlan(4, 10) as plan:
        plan.set_system(inp)
        with pytest.raises(N.CctError) as e:
            plan.backward()
        assert e.value.status == 6  # CCT_ERR_STATE
        plan.forward(0, 3)
        with pytest.raises(N.CctError):
            plan.backward(0, 4)
        plan.backward(0, 3)
        plan.set_system(inp)  # new inputs drop the saved context
        with pytest.raises(N.CctError):
            plan.backward(0, 3)


def test_backward_bitwise_reproducible(api):
    inp = S.generate(5, 24, 8)
    with api.TriplesPlan(5, 24) as plan:
        plan.set_system(inp)
        plan.forward()
        a = plan.backward()
        b = plan.backward()
    for name in NAMES:
        assert np.array_equal(a[name], b[name]), name


@pytest.mark.parametrize("no,nu,seed", [(5, 24, 8), (4, 17, 12)])
def test_backward_from_kept_w_equals_recompute(api, no, nu, seed):
    """keep_w: the forward keeps every tuple's W-build output and the backward
    reads it instead of rebuilding W; the FP64 W build is deterministic, so
    energies and every gradient are bitwise those of the recomputing
    backward, for the full range and for a tuple range."""
    inp = S.generate(no, nu, seed)
    for rng in [(), (2, 9)]:
        with api.TriplesPlan(no, nu) as plan:
            plan.set_system(inp)
            fa = plan.forward(*rng)
            ga = plan.backward(*rng)
            assert plan.kept_tuples == 0
        with api.TriplesPlan(no, nu, keep_w=True) as plan:
            plan.set_system(inp)
            fb = plan.forward(*rng)
            n = (rng[1] - rng[0]) if rng else plan.num_tuples
            assert plan.kept_tuples == n > 0
            gb = plan.backward(*rng)
            gc = plan.backward(*rng)  # the kept W is read, not consumed
        assert fa[0] == fb[0] and fa[1] == fb[1] and np.array_equal(fa[2], fb[2])
        for name in NAMES:
            assert np.array_equal(ga[name], gb[name]), (rng, name)
            assert np.array_equal(gb[name], gc[name]), (rng, name)


def test_keep_w_is_off_for_emulated_plans(api):
    inp = S.generate(4, 12, 5)
    with api.TriplesPlan(4, 12, precision="int8", emu_slices=4, keep_w=True) as plan:
        plan.set_system(inp)
        plan.forward()
        assert plan.kept_tuples == 0
        plan.backward()


def test_backward_after_emulated_forward(api):
    """An emulated plan's backward recomputes W in FP64: same gradient as FP64."""
    from oracle import oracle as O
    inp = S.generate(4, 18, 9)
    ref = O.closed_grad(inp)
    with api.TriplesPlan(4, 18, precision="int8") as plan:
        plan.set_system(inp)
        plan.forward()
        g = plan.backward()
    for name in NAMES:
        assert _close(g[name], ref[name]), name


def test_backward_central_differences_of_gpu_forward(api):
    """Central differences (h = 1e-5) of the GPU FP64 E(T) on random entries of
    every input.  E(T) is at most quadratic in each single T2/VM/VVVO entry and
    linear in T1/VOE, so the central difference is exact up to rounding there."""
    no, nu = 6, 30
    inp = S.generate(no, nu, 13)
    with api.TriplesPlan(no, nu) as plan:
        plan.set_system(inp)
        plan.forward()
        g = plan.backward()
        rng = np.random.default_rng(2)
        for name in NAMES:
            arr = getattr(inp, name)
            scale = np.abs(g[name]).max()
            for idx in rng.choice(arr.size, size=min(6, arr.size), replace=False):
                h = 1e-5 * max(1.0, abs(arr[idx]))
                vals = []
                for sgn in (1.0, -1.0):
                    ip = copy.deepcopy(inp)
                    getattr(ip, name)[idx] += sgn * h
                    plan.set_system(ip)
                    ets, etd, _ = plan.forward(want_v1=False)
                    vals.append(ets + etd)
                fd = (vals[0] - vals[1]) / (2 * h)
                assert abs(fd - g[name][idx]) <= 1e-6 * scale + 1e-8 * abs(fd), (name, idx, fd, g[name][idx])


def test_backward_matches_golden_gradient_no12_nu120(api):
    """The no=12/nu=120 system (seed 3): GPU gradient against the hand-derived FP64
    CPU gradient stored in tests/golden (200 seeded entries per input and
    whole-tensor checksums)."""
    import json
    import pathlib
    g0 = json.loads((pathlib.Path(__file__).parent / "golden" / "grad_no12-nu120.json").read_text())
    inp = S.generate(g0["no"], g0["nu"], g0["seed"], g0["dist"])
    with api.TriplesPlan(inp.no, inp.nu) as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
        g = plan.backward()
    assert abs((ets + etd) - g0["e_t"]) <= 1e-12 * abs(g0["e_t"])
    for name, ref in g0["tensors"].items():
        got = g[name]
        idx = np.array(ref["index"])
        assert np.abs(got[idx] - np.array(ref["value"])).max() <= 1e-10 * ref["maxabs"], name
        assert abs(got.sum() - ref["sum"]) <= 1e-10 * ref["maxabs"] * np.sqrt(got.size) + 1e-12 * abs(ref["sum"]), name
        assert abs(np.dot(got, got) - ref["sumsq"]) <= 1e-9 * ref["sumsq"], name
