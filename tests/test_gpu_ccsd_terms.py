"""The CCSD T1-dressing terms on the GPU (ccT_ccsd_terms_29_31 / _32_35)
against the oracle's literal restatement of ccsd_acc.f."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(no, nu, seed):
    rng = np.random.default_rng(seed)
    nutr = nu * (nu + 1) // 2
    n4 = no * nu * nu * no
    return dict(o1=rng.normal(0, 0.1, no * nu), t2=rng.normal(size=n4), vl=rng.normal(size=n4),
                vr=rng.normal(size=n4), vvvo=rng.normal(size=nutr * nu * no), o2=rng.normal(size=n4),
                vm=rng.normal(size=no ** 3 * nu))


@pytest.mark.parametrize("no,nu,seed", [(3, 5, 1), (4, 17, 2), (6, 40, 3), (8, 64, 4), (20, 24, 5), (24, 33, 6)])
def test_terms_29_31_match_oracle(no, nu, seed):
    from libcc_b200 import api as A
    from oracle import oracle as O
    a = _inputs(no, nu, seed)
    got = A.ccsd_terms_29_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
    ref = O.literal_terms_29_30_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("no,nu,seed", [(3, 5, 1), (4, 17, 2), (6, 40, 3), (8, 64, 4), (20, 24, 5), (24, 33, 6)])
def test_terms_32_35_match_oracle(no, nu, seed):
    from libcc_b200 import api as A
    from oracle import oracle as O
    a = _inputs(no, nu, seed)
    got = A.ccsd_terms_32_35(no, nu, a["o1"], a["o2"], a["t2"], a["vm"], a["vvvo"])
    ref = O.literal_terms_32_35(no, nu, a["o1"], a["o2"], a["t2"], a["vm"], a["vvvo"])
    for name, g, r in zip(("t2", "o2", "vm", "rl"), got, ref):
        assert np.abs(g - r).max() <= 1e-12 * max(np.abs(r).max(), 1e-300), name


def test_workspace_reuse_across_shapes_and_release():
    """The entry points keep their device workspace between calls: a large
    shape, then a smaller one in the grown slots, then the large one again
    after ccT_ccsd_release_workspace, each bitwise equal to its first call and
    within the oracle tolerance."""
    from libcc_b200 import api as A
    from oracle import oracle as O
    shapes = [(6, 40, 7), (3, 9, 8)]
    first = {}
    for rep in range(2):
        for no, nu, seed in shapes:
            a = _inputs(no, nu, seed)
            g1 = A.ccsd_terms_29_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
            g2 = A.ccsd_terms_32_35(no, nu, a["o1"], a["o2"], a["t2"], a["vm"], a["vvvo"])
            if rep == 0:
                first[no] = (g1, g2)
                ref = O.literal_terms_29_30_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
                assert np.abs(g1 - ref).max() <= 1e-12 * np.abs(ref).max()
            else:
                assert np.array_equal(g1, first[no][0])
                assert all(np.array_equal(x, y) for x, y in zip(g2, first[no][1]))
        A.ccsd_release_workspace()
