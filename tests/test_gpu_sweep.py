"""Seeded sweep over small and edge-sized systems (nu from 1 to 129, no from 2
to 8, normal and log-uniform magnitudes): the FP64 forward against the C
oracle, both emulated forms (7 fixed digits; automatic digits against the
default 1e-8 Eh target) against the oracle, the gradient against the hand-derived CPU adjoint where
nu <= 24, and the batch against single-system plans bitwise."""
import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(12345)
    out = []
    for c in range(36):
        no, nu = int(rng.integers(2, 8)), int(rng.integers(1, 72))
        out.append((no, nu, 1000 + c, "log" if c % 3 == 0 else "normal"))
    out += [(2, 1, 7, "normal"), (3, 2, 8, "normal"), (8, 3, 9, "normal"), (2, 129, 10, "normal"),
            (3, 97, 11, "log")]
    return out


CASES = _cases()


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("no,nu,seed,dist", CASES)
def test_sweep_forward_gradient_and_emulation(no, nu, seed, dist):
    from libcc_b200 import api as A
    from oracle import oracle as O
    inp = S.generate(no, nu, seed, dist)
    ets_o, etd_o, v1_o = O.c_cc_triples(inp)
    e_o = ets_o + etd_o
    with A.TriplesPlan(no, nu) as p:
        p.set_system(inp)
        ets, etd, v1 = p.forward()
        assert abs(ets + etd - e_o) <= 1e-12 * abs(e_o)
        assert _rel(v1, v1_o) <= 1e-12
        if nu <= 24:
            g = p.backward()
            ref = O.closed_grad(inp)
            for k in g:
                assert _rel(g[k], ref[k]) <= 1e-12, k
    with A.TriplesPlan.for_form(no, nu, "int8:7") as p:
        p.set_system(inp)
        ets, etd, _ = p.forward()
    assert abs(ets + etd - e_o) <= 1e-11 * abs(e_o) + 1e-14
    with A.TriplesPlan.for_form(no, nu, "int8") as p:  # automatic digits, 1e-8 Eh target
        p.set_system(inp)
        ets, etd, _ = p.forward()
        cal = p.emu_digits()
    assert abs(ets + etd - e_o) <= cal["target"] + 2e-14 * abs(e_o), (cal, ets + etd, e_o)


def test_sweep_batch_equals_plans_bitwise():
    from libcc_b200 import api as A
    from libcc_b200 import batch as B
    systems = [S.generate(no, nu, seed, dist) for (no, nu, seed, dist) in CASES]
    with B.TriplesBatch([(s.no, s.nu) for s in systems]) as b:
        for k, inp in enumerate(systems):
            b.set_system(k, inp)
        ets, etd = b.forward()
    for k, inp in enumerate(systems):
        with A.TriplesPlan(inp.no, inp.nu) as p:
            p.set_system(inp)
            e1, e2, _ = p.forward()
        assert ets[k] == e1 and etd[k] == e2, (inp.no, inp.nu)
