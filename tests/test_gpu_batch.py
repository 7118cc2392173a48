"""Batched systems in one persistent kernel (ccT_batch_*) against single-system
plans (bitwise) and the oracle."""
import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu

SHAPES = [(3, 24), (5, 17), (4, 40), (2, 9), (6, 33), (3, 61), (7, 20)]


@pytest.fixture(scope="module")
def systems():
    return [S.generate(no, nu, 100 + k) for k, (no, nu) in enumerate(SHAPES)]


@pytest.fixture(scope="module")
def single(systems):
    from libcc_b200 import api as A
    out = []
    for inp in systems:
        with A.TriplesPlan(inp.no, inp.nu) as p:
            p.set_system(inp)
            out.append(p.forward())
    return out


def _batch(systems):
    from libcc_b200 import batch as B
    b = B.TriplesBatch([(s.no, s.nu) for s in systems])
    for k, s in enumerate(systems):
        b.set_system(k, s)
    return b


def test_batch_equals_single_plans_bitwise(systems, single):
    with _batch(systems) as b:
        ets, etd = b.forward()
        for k in range(len(systems)):
            assert ets[k] == single[k][0] and etd[k] == single[k][1], k
            assert np.array_equal(b.v1(k), single[k][2]), k


def test_batch_matches_oracle(systems):
    from oracle import oracle as O
    with _batch(systems) as b:
        ets, etd = b.forward()
    for k, inp in enumerate(systems):
        ets_o, etd_o, _ = O.c_cc_triples(inp)
        assert abs(etd[k] - etd_o) <= 1e-12 * abs(etd_o), k
        assert abs(ets[k] - ets_o) <= 1e-11 * abs(ets_o) + 1e-15, k


@pytest.mark.parametrize("mode,bn,order,group_mib", [
    (0, 32, 0, 512), (0, 64, 1, 512), (0, 48, 0, 1), (0, 32, 1, 1),
    (1, 0, 0, 512), (1, 0, 1, 1), (1, 64, 1, 512), (1, 48, 0, 1), (1, 32, 1, 1)])
def test_schedules_agree(systems, single, mode, bn, order, group_mib):
    """Both executors, every N tile, tuple order and group size (1 MiB forces many
    groups, so the X scratch ring is reused and the group waits / stream events
    are exercised) give the same bits."""
    with _batch(systems) as b:
        b.configure(mode, bn, order, group_mib << 20)
        for _ in range(2):  # second call replays the CUDA graph
            ets, etd = b.forward()
            for k in range(len(systems)):
                assert ets[k] == single[k][0] and etd[k] == single[k][1], (mode, bn, order, group_mib, k)


def test_tune_picks_a_candidate(systems, single):
    with _batch(systems) as b:
        mode, bn, order, ms = b.tune()
        assert mode in (0, 1) and bn in (0, 32, 48, 64) and order in (0, 1) and ms > 0
        ets, etd = b.forward()
        assert b.last_ms > 0 and b.work_items > 0
        for k in range(len(systems)):
            assert etd[k] == single[k][1]


def test_forward_needs_inputs():
    from libcc_b200 import _native as N
    from libcc_b200 import batch as B
    with B.TriplesBatch([(3, 8), (4, 9)]) as b:
        b.set_system(0, S.generate(3, 8, 1))
        with pytest.raises(N.CctError) as e:
            b.forward()
        assert e.value.status == 6


def test_bounded_wait_runs_out_and_context_survives(systems, single):
    """The persistent executor's counter wait, made unmeetable on the host
    (one tuple's reduction blocks wait for a W-build tile more than it has)
    with a short spin limit: the forward returns CCT_ERR_TIMEOUT, and with the
    stall cleared the same batch gives the single-plan bits again."""
    from libcc_b200 import _native as N
    with _batch(systems) as b:
        b.configure(0, 32, 0, 1 << 20)
        b.debug_stall(0, 20000)
        with pytest.raises(N.CctError) as e:
            b.forward()
        assert e.value.status == 7  # CCT_ERR_TIMEOUT
        b.debug_stall(-1, 0)
        ets, etd = b.forward()
        for k in range(len(systems)):
            assert ets[k] == single[k][0] and etd[k] == single[k][1]


@pytest.fixture(scope="module")
def single_emulated(systems):
    from libcc_b200 import api as A
    out = []
    for inp in systems:
        with A.TriplesPlan.for_form(inp.no, inp.nu, "int8") as p:
            p.set_system(inp)
            ets, etd, _ = p.forward()
            out.append((ets, etd, p.emu_digits()["digits"]))
    return out


@pytest.mark.parametrize("order", [0, 1])
def test_emulated_batch_equals_emulated_plans_bitwise(systems, single_emulated, order):
    """Mode 2 (one emulated W-build launch per system and tuple group; 1 MiB
    groups, so the X ring is reused): per system the calibrated digit count and
    the energies of a single emulated plan with the same options, bitwise."""
    from libcc_b200 import batch as B
    with B.TriplesBatch([(s.no, s.nu) for s in systems], form="int8") as b:
        for k, s in enumerate(systems):
            b.set_system(k, s)
        b.configure(2, 0, order, 1 << 20)
        for _ in range(2):  # the second call replays the CUDA graph
            ets, etd = b.forward()
            for k in range(len(systems)):
                assert b.emu_digits(k) == single_emulated[k][2]
                assert ets[k] == single_emulated[k][0] and etd[k] == single_emulated[k][1], (order, k)


def test_emulated_batch_meets_target_and_tunes(systems):
    """The emulated batch's energies are within the 1e-8 Eh target of the FP64
    oracle for every system, and its tuner chooses among all three executors."""
    from libcc_b200 import batch as B
    from oracle import oracle as O
    with B.TriplesBatch([(s.no, s.nu) for s in systems], form="int8") as b:
        for k, s in enumerate(systems):
            b.set_system(k, s)
        ets, etd = b.forward()
        for k, inp in enumerate(systems):
            ets_o, etd_o, _ = O.c_cc_triples(inp)
            assert abs((ets[k] + etd[k]) - (ets_o + etd_o)) <= 1e-8, k
        mode, bn, order, ms = b.tune()
        assert mode in (0, 1, 2) and ms > 0
        ets2, etd2 = b.forward()
        for k in range(len(systems)):
            assert abs((ets2[k] + etd2[k]) - (ets[k] + etd[k])) <= 2e-8


def test_emulated_mode_needs_an_emulated_batch(systems):
    from libcc_b200 import _native as N
    with _batch(systems) as b:
        with pytest.raises(N.CctError):
            b.configure(2, 0, 0, 1 << 20)
