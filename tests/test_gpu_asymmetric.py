"""Inputs without the integral/amplitude permutation symmetries: the kernels read
exactly the entries the reference's formulas name, so E(T) and the gradient
match the oracle for arbitrary arrays, not only for symmetric ones."""
import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _asymmetric(no, nu, seed):
    inp = S.generate(no, nu, seed)
    rng = np.random.default_rng(seed + 1000)
    for name in ("t1", "t2", "vm", "voe", "vvvo"):
        a = getattr(inp, name)
        a += 0.05 * np.abs(a).max() * rng.standard_normal(a.size)
    return inp


@pytest.mark.parametrize("no,nu,seed", [(4, 9, 0), (5, 21, 1), (3, 16, 2)])
def test_forward_matches_oracle_without_symmetry(no, nu, seed):
    from libcc_b200 import api as A
    from oracle import oracle as O
    inp = _asymmetric(no, nu, seed)
    ets_o, etd_o, v1_o = O.c_cc_triples(inp)
    with A.TriplesPlan(no, nu) as plan:
        plan.set_system(inp)
        ets, etd, v1 = plan.forward()
    assert abs(etd - etd_o) <= 1e-12 * abs(etd_o)
    assert abs(ets - ets_o) <= 1e-11 * abs(ets_o) + 1e-15
    assert np.abs(v1 - v1_o).max() <= 1e-11 * np.abs(v1_o).max()


def test_backward_matches_oracle_without_symmetry():
    from libcc_b200 import api as A
    from oracle import oracle as O
    inp = _asymmetric(4, 11, 5)
    ref = O.closed_grad(inp)
    with A.TriplesPlan(4, 11) as plan:
        plan.set_system(inp)
        plan.forward()
        g = plan.backward()
    for name in ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo"):
        assert np.abs(g[name] - ref[name]).max() <= 1e-10 * np.abs(ref[name]).max(), name
