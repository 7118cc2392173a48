"""The CCSD T1-dressing terms of the reference's CCSD port (ccsd_acc.f): the
oracle's literal DGEMM / permutation restatement against its closed form."""
import numpy as np

from oracle import oracle as O


def _inputs(no, nu, seed):
    rng = np.random.default_rng(seed)
    nutr = nu * (nu + 1) // 2
    return dict(o1=rng.normal(size=no * nu), t2=rng.normal(size=no * nu * nu * no),
                vl=rng.normal(size=no * nu * nu * no), vr=rng.normal(size=nu * no * nu * no),
                vvvo=rng.normal(size=nutr * nu * no), o2=rng.normal(size=no * nu * nu * no),
                vm=rng.normal(size=no ** 3 * nu))


def test_terms_29_30_31_literal_equals_closed_form():
    for no, nu, seed in ((3, 5, 1), (4, 7, 2), (2, 9, 3)):
        a = _inputs(no, nu, seed)
        lit = O.literal_terms_29_30_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
        clo = O.closed_terms_29_30_31(no, nu, a["o1"], a["t2"], a["vl"], a["vr"], a["vvvo"])
        assert np.abs(lit - clo).max() <= 1e-12 * np.abs(lit).max()


def test_terms_32_35_shapes_and_transposes():
    """t2 and rl come back transposed as (nou x nou) matrices, o2 permuted to
    (nu,nu,no,no); a zero O1 and O2 leave vm only permuted (312 then 23)."""
    no, nu = 3, 4
    a = _inputs(no, nu, 5)
    t2, o2, vm, rl = O.literal_terms_32_35(no, nu, np.zeros(no * nu), np.zeros_like(a["o2"]), a["t2"], a["vm"],
                                           a["vvvo"])
    nou = no * nu
    assert np.array_equal(t2.reshape((nou, nou), order="F"), a["t2"].reshape((nou, nou), order="F").T)
    assert not rl.any()
    V = a["vm"].reshape((no, no, no, nu), order="F")
    want = np.einsum("yxza->xyza", V)  # VM_out(x,y,z,a) = VM_in(y,x,z,a)
    assert np.array_equal(vm.reshape((no, no, no, nu), order="F"), want)
