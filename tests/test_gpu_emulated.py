"""INT8 split-integer emulated FP64 W-build (tcgen05 kind::i8) against the oracle."""
import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _plan(api, inp, slices):
    return api.TriplesPlan(inp.no, inp.nu, precision="int8", emu_slices=slices)


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
def test_default_emulation_meets_its_target(api, dist):
    """Automatic digits against the oracle: |dE(T)| within the calibrated
    target max(1e-8 Eh, 2e-14 |E(T)|), and the calibrated bound itself below it."""
    from oracle import oracle as O
    inp = S.generate(5, 40, 77, dist=dist)
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    with api.TriplesPlan(inp.no, inp.nu, precision="int8") as plan:
        plan.set_system(inp)
        cal = plan.emu_digits()
        ets, etd, _ = plan.forward()
    e_o = ets_o + etd_o
    assert cal["target"] == pytest.approx(max(1e-8, 2e-14 * abs(e_o)), rel=0.5)
    assert 3 <= cal["digits"] <= 7 and cal["est_err"] <= cal["target"], cal
    assert abs((ets + etd) - e_o) <= cal["target"], (ets + etd, e_o, cal)


def test_water_avdz_default_meets_1e8_eh(api):
    """The water aug-cc-pVDZ shape (no=4, nu=36, seed 0; |E(T)| = 10.5 Eh, where
    1e-8 Eh is representable): the default emulated plan meets 1e-8 Eh
    absolute against the FP64 oracle."""
    import json
    import pathlib
    g = json.loads((pathlib.Path(__file__).parent / "golden" / "energies.json").read_text())["water-avdz"]
    inp = S.workload("water-avdz")
    with api.TriplesPlan(inp.no, inp.nu, precision="int8") as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
        cal = plan.emu_digits()
    assert cal["target"] == 1e-8, cal
    assert abs((ets + etd) - g["e_t"]) <= 1e-8, (ets + etd - g["e_t"], cal)


def test_relative_target_picks_fewer_digits(api):
    """A looser relative target (2.1e-7 |E|, the Ar6-scale reading of 1e-8 Eh)
    calibrates to fewer digits than the default and still meets its target."""
    from oracle import oracle as O
    inp = S.generate(5, 48, 9, dist="log")
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    e_o = ets_o + etd_o
    res = {}
    for rel in (0.0, 2.1e-7):
        with api.TriplesPlan(inp.no, inp.nu, precision="int8", emu_tol_rel=rel) as plan:
            plan.set_system(inp)
            ets, etd, _ = plan.forward()
            res[rel] = (plan.emu_digits(), ets + etd)
    assert res[2.1e-7][0]["digits"] < res[0.0][0]["digits"], res
    for rel, (cal, e) in res.items():
        assert abs(e - e_o) <= cal["target"], (rel, cal, e, e_o)


@pytest.mark.parametrize("slices,rel", [(3, 3e-7), (4, 3e-9), (5, 3e-11), (6, 3e-13), (7, 1e-14)])
def test_error_falls_with_slice_count(api, slices, rel):
    """Fixed digit counts with rounded digits: the energy error against the FP64
    form falls about 2^7 per digit."""
    inp = S.generate(5, 48, 9, dist="log")
    with api.TriplesPlan(inp.no, inp.nu) as ref:
        ref.set_system(inp)
        ets_r, etd_ref, _ = ref.forward()
    with _plan(api, inp, slices) as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
    assert abs(etd - etd_ref) <= rel * abs(etd_ref), (slices, etd, etd_ref)


@pytest.mark.parametrize("form,bar", [("fp64", 1e-13), ("int8:7", 1e-12), ("int8:5", 1e-8), ("int8:3", 1e-4)])
def test_tuple_w_matches_oracle(api, form, bar):
    """ccT_tuple_w against the oracle's literal formv3/SYMT311/ZEROT3 W for every
    tuple kind: max |dW| / max |W|."""
    from oracle import oracle as O
    no, nu = 5, 29
    inp = S.generate(no, nu, 61, dist="log")
    tuples = O.all_tuples(no)
    pick = [next(t for t, tup in enumerate(tuples) if tup[0] == kd) for kd in (0, 1, 2)] + [len(tuples) - 1]
    with api.TriplesPlan.for_form(no, nu, form) as plan:
        plan.set_system(inp)
        for t in pick:
            w = plan.tuple_w(t)
            w_ref = O.c_tuple_w(inp, *tuples[t])
            err = np.abs(w - w_ref).max() / np.abs(w_ref).max()
            assert err <= bar, (form, tuples[t], err)


def test_emu_digits_on_fp64_plan_is_state_error(api):
    from libcc_b200._native import CctError
    with api.TriplesPlan(3, 5) as plan:
        with pytest.raises(CctError) as e:
            plan.emu_digits()
        assert e.value.status == 6


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


@pytest.mark.parametrize("no,nu,slices", [(4, 70, 5), (3, 90, 5), (5, 150, 6), (4, 75, 4), (3, 96, 3)])
def test_wide_n_tiles_meet_the_bar(api, no, nu, slices):
    """nu chosen so the plan picks the 80- and 96-column emulated N tiles."""
    from oracle import oracle as O
    inp = S.generate(no, nu, 31 + nu, dist="log")
    ets_o, etd_o, _ = O.literal_cc_triples(inp)
    with _plan(api, inp, slices) as plan:
        plan.set_system(inp)
        ets, etd, _ = plan.forward()
    bar = {3: 3e-7, 4: 3e-9, 5: 3e-11, 6: 3e-13}[slices]
    assert abs((ets + etd) - (ets_o + etd_o)) <= bar * abs(ets_o + etd_o), (ets + etd, ets_o + etd_o)


def test_emulated_deterministic(api):
    inp = S.generate(4, 40, 12)
    with api.TriplesPlan(inp.no, inp.nu, precision="int8") as plan:
        plan.set_system(inp)
        a = plan.forward()
        b = plan.forward()
    assert a[1] == b[1] and np.array_equal(a[2], b[2])


def test_per_tile_digits_follow_exponent_spread(api):
    """Automatic plans: each 128 x N tile runs max(1, S - floor(gap/7)) digits, S
    the calibrated count, gap = bits its largest row scales sum below the
    system's top.  On a system whose magnitudes fall by half a bit per virtual
    index the tiles spread over several counts; the energy meets the target."""
    from oracle import oracle as O
    inp = S.with_decay(S.generate(4, 64, 21, dist="normal"), 0.5)
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    e_ref = ets_o + etd_o
    with _plan(api, inp, 0) as plan:
        plan.set_system(inp)
        ets_a, etd_a, v1_a = plan.forward()
        hist = plan.emu_slice_histogram()
        cal = plan.emu_digits()
    top = cal["digits"]
    assert hist[top] > 0 and sum(hist[1:top]) > 0 and sum(hist[top + 1:]) == 0, (hist, cal)
    assert abs((ets_a + etd_a) - e_ref) <= cal["target"], (ets_a + etd_a, e_ref, cal)


def test_per_tile_digits_uniform_system_equals_fixed(api):
    """Without an exponent spread every tile takes the calibrated count: bitwise
    the fixed-count result (the same leading digits, the same N tile)."""
    inp = S.generate(4, 40, 12, dist="log")
    with _plan(api, inp, 0) as plan:
        plan.set_system(inp)
        a = plan.forward()
        hist = plan.emu_slice_histogram()
        top = plan.emu_digits()["digits"]
    with _plan(api, inp, top) as plan:
        plan.set_system(inp)
        b = plan.forward()
    assert hist[top] == sum(hist) > 0, hist
    assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("no,nu,seed,rel", [(4, 40, 12, 1e-4), (5, 48, 9, 2.1e-7), (4, 64, 21, 1e-6)])
def test_loose_target_calibration_is_the_first_passing_count(api, no, nu, seed, rel):
    """A target looser than 3.5 digits' worth of bits is tried at 3 digits
    first, on 3-digit operands: the count it keeps has its bound within the
    target, the energy meets the target against the oracle, and with every
    tile at the calibrated count the energies are bitwise those of the
    fixed-count plan."""
    from oracle import oracle as O
    inp = S.generate(no, nu, seed, dist="log")
    e_o = sum(O.c_cc_triples(inp)[:2])
    with api.TriplesPlan(no, nu, precision="int8", emu_tol_rel=rel) as plan:
        plan.set_system(inp)
        a = plan.forward()
        cal = plan.emu_digits()
        hist = plan.emu_slice_histogram()
    assert cal["est_err"] <= cal["target"], cal
    assert abs(a[0] + a[1] - e_o) <= cal["target"], (cal, a[0] + a[1], e_o)
    top = cal["digits"]
    with _plan(api, inp, top) as plan:
        plan.set_system(inp)
        b = plan.forward()
    if hist[top] == sum(hist):
        assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])

