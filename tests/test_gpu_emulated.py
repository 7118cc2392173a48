"""INT8 split-integer emulated FP64 W-build (tcgen05 kind::i8) against the oracle."""
import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _plan(api, inp, slices):
    from libcc_b200 import _native as N
    import ctypes
    lib = N.load()
    opt = N.Options()
    lib.ccT_options_default(ctypes.byref(opt))
    opt.precision = N.CCT_PREC_INT8_EMU
    opt.emu_slices = slices
    h = ctypes.c_void_p()
    N.check(lib.ccT_plan_create(ctypes.byref(h), inp.no, inp.nu, ctypes.byref(opt)), "ccT_plan_create")
    plan = api.TriplesPlan.__new__(api.TriplesPlan)
    plan._h, plan.no, plan.nu, plan.precision, plan.device = h, inp.no, inp.nu, "int8", 0
    plan.num_tuples = int(lib.ccT_num_tuples(inp.no))
    return plan


@pytest.fixture(scope="module")
def api():
    from libcc_b200 import api as A
    return A


@pytest.mark.parametrize("no,nu,seed", [(3, 7, 1), (4, 36, 0), (5, 64, 3), (6, 70, 5)])
def test_emulated_seven_slices_match_oracle(api, no, nu, seed):
    from oracle import oracle as O
    inp = S.generate(no, nu, seed)
    ets_o, etd_o, v1_o = O.c_cc_triples(inp)
    with _plan(api, inp, 7) as plan:
        plan.set_system(inp)
        ets, etd, v1 = plan.forward()
    assert abs(etd - etd_o) <= 1e-11 * abs(etd_o), (etd, etd_o)
    assert abs(ets - ets_o) <= 1e-9 * abs(ets_o) + 1e-12
    assert np.abs(v1 - v1_o).max() <= 1e-9 * np.abs(v1_o).max()


@pytest.mark.parametrize("dist", ["normal", "log"])
def test_default_emulation_meets_relative_bar(api, dist):
    """Default digit count against the oracle: relative 2.1e-7, i.e. 1e-8 Eh on a
    (T) energy of 0.048 Eh (the Ar6 magnitude)."""
    from oracle import oracle as O
    inp = S.generate(5, 40, 77, dist=dist)
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    with api.TriplesPlan(inp.no, inp.nu, precision="int8") as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
    assert abs((ets + etd) - (ets_o + etd_o)) <= 2.1e-7 * abs(ets_o + etd_o)


@pytest.mark.parametrize("slices,rel", [(4, 3e-6), (5, 3e-8), (6, 3e-10), (7, 1e-11)])
def test_error_falls_with_slice_count(api, slices, rel):
    inp = S.generate(5, 48, 9, dist="log")
    with api.TriplesPlan(inp.no, inp.nu) as ref:
        ref.set_system(inp)
        _, etd_ref, _ = ref.forward()
    with _plan(api, inp, slices) as plan:
        plan.set_system(inp)
        _, etd, _ = plan.forward()
    assert abs(etd - etd_ref) <= rel * abs(etd_ref), (slices, etd, etd_ref)


def test_emulated_tuple_kinds_and_shards(api):
    from oracle import oracle as O
    no, nu = 5, 17
    inp = S.generate(no, nu, 21)
    tuples = O.all_tuples(no)
    with _plan(api, inp, 7) as plan:
        plan.set_system(inp)
        for t in (0, 9, 10, 11, len(tuples) - 1):
            kind, i, j, k = tuples[t]
            e_ref, v1_ref = O.c_tuple(inp, kind, i, j, k)
            _, etd, v1 = plan.forward(t, t + 1)
            assert abs(etd - e_ref) <= 1e-11 * abs(e_ref), (kind, i, j, k)


@pytest.mark.parametrize("no,nu,slices", [(4, 70, 5), (3, 90, 5), (5, 150, 6), (4, 75, 4)])
def test_wide_n_tiles_meet_the_bar(api, no, nu, slices):
    """nu chosen so the plan picks the 80- and 96-column emulated N tiles."""
    from oracle import oracle as O
    inp = S.generate(no, nu, 31 + nu, dist="log")
    ets_o, etd_o, _ = O.literal_cc_triples(inp)
    with _plan(api, inp, slices) as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
    bar = {4: 3e-6, 5: 3e-8, 6: 3e-10}[slices]
    assert abs((ets + etd) - (ets_o + etd_o)) <= bar * abs(ets_o + etd_o), (ets + etd, ets_o + etd_o)


def test_emulated_deterministic(api):
    inp = S.generate(4, 40, 12)
    with api.TriplesPlan(inp.no, inp.nu, precision="int8") as plan:
        plan.set_system(inp)
        a = plan.forward()
        b = plan.forward()
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


def test_per_tile_digits_follow_exponent_spread(api):
    """emu_slices = 0: each 128 x N tile runs max(1, 5 - floor(gap/7)) digits, gap
    = bits its largest row scales sum below the system's top.  On a system whose
    magnitudes fall by half a bit per virtual index the tiles spread over 1..5
    digits; the energy keeps the 5-digit bar and stays close to fixed 5 digits."""
    from oracle import oracle as O
    inp = S.with_decay(S.generate(4, 64, 21, dist="normal"), 0.5)
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    e_ref = ets_o + etd_o
    with _plan(api, inp, 0) as plan:
        plan.set_system(inp)
        ets_a, etd_a, v1_a = plan.forward()
        hist = plan.emu_slice_histogram()
    with _plan(api, inp, 5) as plan:
        plan.set_system(inp)
        ets_f, etd_f, _ = plan.forward()
        hist_f = plan.emu_slice_histogram()
    assert sum(hist[1:5]) > 0 and hist[5] > 0 and sum(hist[6:]) == 0, hist
    assert hist_f[5] == sum(hist) and sum(hist_f) == hist_f[5], hist_f
    err_a, err_f = abs((ets_a + etd_a) - e_ref), abs((ets_f + etd_f) - e_ref)
    assert err_a <= 3e-8 * abs(e_ref), (err_a, e_ref)
    assert err_a <= 10.0 * err_f + 1e-14 * abs(e_ref), (err_a, err_f)


def test_per_tile_digits_uniform_system_equals_fixed(api):
    """Without an exponent spread every tile takes the maximum: bitwise the
    fixed 5-digit result."""
    inp = S.generate(4, 40, 12, dist="log")
    with _plan(api, inp, 0) as plan:
        plan.set_system(inp)
        a = plan.forward()
        hist = plan.emu_slice_histogram()
    with _plan(api, inp, 5) as plan:
        plan.set_system(inp)
        b = plan.forward()
    assert hist[5] == sum(hist) > 0, hist
    assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
