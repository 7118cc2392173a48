"""The hand-derived FP64 CPU gradient (oracle.closed_grad) against central finite
differences of the oracle's E(T), for every input and every tuple kind."""
import copy

import numpy as np
import pytest

from libcc_b200 import synthetic as S

NAMES = ("eh", "ep", "t1", "t2", "vm", "voe", "vvvo")


def _energy(O, inp):
    ets, etd, _ = O.c_cc_triples(inp)
    return ets + etd


@pytest.mark.parametrize("no,nu,seed", [(4, 5, 5), (3, 4, 1), (2, 6, 7)])
def test_closed_grad_matches_central_differences(no, nu, seed):
    from oracle import oracle as O
    inp = S.generate(no, nu, seed)
    g = O.closed_grad(inp)
    assert abs(g["e_t"] - _energy(O, inp)) <= 1e-12 * abs(g["e_t"])
    rng = np.random.default_rng(seed)
    for name in NAMES:
        arr = getattr(inp, name)
        scale = np.abs(g[name]).max()
        for idx in rng.choice(arr.size, size=min(5, arr.size), replace=False):
            h = 1e-5 * max(1.0, abs(arr[idx]))
            ip, im = copy.deepcopy(inp), copy.deepcopy(inp)
            getattr(ip, name)[idx] += h
            getattr(im, name)[idx] -= h
            fd = (_energy(O, ip) - _energy(O, im)) / (2 * h)
            assert abs(fd - g[name][idx]) <= 1e-7 * scale + 1e-9 * abs(fd), (name, idx, fd, g[name][idx])


def test_closed_grad_is_additive_over_tuple_ranges():
    """The gradient of a tuple range plus that of its complement is the whole
    gradient (the backward of a shard composes like the forward)."""
    from oracle import oracle as O
    inp = S.generate(4, 6, 2)
    tuples = O.all_tuples(4)
    whole = O.closed_grad(inp)
    a = O.closed_grad(inp, tuples[:5])
    b = O.closed_grad(inp, tuples[5:])
    for name in NAMES:
        assert np.allclose(a[name] + b[name], whole[name], rtol=1e-12, atol=1e-15 * np.abs(whole[name]).max())
