"""The oracle against the reference's known answers, and its restatements against each other."""
import json
import pathlib

import numpy as np
import pytest

from libcc_b200 import synthetic as S
from oracle import oracle as O

GOLD = pathlib.Path(__file__).parent / "golden"


def test_trant3_known_answer_table():
    """tools/trant3/trant3.f:2-31 on nu=2: the oracle's in-place TRANT3 loops
    reproduce the table derived independently in tests/golden/make_trant3_kat.py."""
    kat = json.loads((GOLD / "trant3_kat.json").read_text())
    for block in kat["blocks"]:
        j = block["j"]
        a = np.arange(1, 9, dtype=float)
        if j > 0:
            a = O.c_trant3(a, 2, j)
        cols = [O.c_trant3(a, 2, tid) for tid in range(1, 6)]
        got = [[a[r]] + [c[r] for c in cols] for r in range(8)]
        assert got == block["rows"], j


@pytest.mark.parametrize("nu", [3, 5, 8])
@pytest.mark.parametrize("tid", [1, 2, 3, 4, 5])
def test_trant3_in_place_loops_are_the_documented_permutations(nu, tid):
    v = np.random.default_rng(nu * 10 + tid).standard_normal(nu ** 3)
    spec = {1: "acb", 2: "bac", 3: "cba", 4: "bca", 5: "cab"}[tid]
    want = np.einsum(spec + "->abc", v.reshape((nu, nu, nu), order="F")).ravel(order="F")
    assert np.array_equal(O.c_trant3(v, nu, tid), want)


def test_trant3_4_and_5_are_inverse():
    v = np.random.default_rng(3).standard_normal(7 ** 3)
    assert np.array_equal(O.c_trant3(O.c_trant3(v, 7, 4), 7, 5), v)


def test_task_enumeration_and_div_even():
    """DDCC_T_TASK (common_functions.f:62-86) and DIV_EVEN (:88-104)."""
    no = 6
    tasks = [O.c_task(t, no) for t in range(no * (no - 1) * (no - 2) // 6)]
    assert tasks == [(i, j, k) for i in range(no) for j in range(i) for k in range(j)]
    for n, np_ in [(20, 3), (2024, 7), (5, 8)]:
        parts = [O.c_div_even(n, np_, me) for me in range(np_)]
        starts = [sr - 1 for _, sr in parts]
        assert sum(nr for nr, _ in parts) == n
        assert starts == sorted(starts) and starts[0] == 0
        assert max(nr for nr, _ in parts) - min(nr for nr, _ in parts) <= 1


def test_getve_expands_packed_columns():
    inp = S.generate(3, 6, 1)
    for x in range(inp.no):
        assert np.array_equal(O.c_getve(inp, x), O.expand_vvvo(inp, x).ravel(order="F"))


@pytest.mark.parametrize("no,nu,seed", [(3, 5, 0), (4, 9, 1), (5, 7, 2), (6, 6, 3)])
def test_three_restatements_agree(no, nu, seed):
    inp = S.generate(no, nu, seed)
    c = O.c_cc_triples(inp)
    lit = O.literal_cc_triples(inp)
    cl = O.closed_cc_triples(inp)
    for other in (lit, cl):
        assert abs(other[1] - c[1]) <= 1e-13 * max(1.0, abs(c[1]))
        assert abs(other[0] - c[0]) <= 1e-13 * max(1.0, abs(c[0]))
        assert np.abs(np.asarray(other[2]).ravel(order="F") - c[2]).max() <= 1e-13


def test_fused_t1wt3_equals_t3squa_plus_drt1wt3():
    """t1wt3.f90 (triples-ijk fused form) and T3SQUA+ADT3DEN+DRT1WT3IJK (triples-abc)
    give the same tuple contributions."""
    import ctypes
    inp = S.generate(5, 8, 4)
    no, nu = inp.no, inp.nu
    lib = O.lib()
    for (i, j, k) in [(3, 1, 0), (4, 2, 1)]:
        w = O.c_tuple_w(inp, 0, i, j, k)
        v1 = np.zeros(nu * no)
        x3 = lib.orc_t1wt3_fused(i, j, k, no, nu, O._p(w), O._p(inp.voe), O._p(v1), O._p(inp.eh), O._p(inp.ep))
        e_ref, v1_ref = O.c_tuple(inp, 0, i, j, k)
        assert abs(x3 - e_ref) <= 1e-14 * max(1.0, abs(e_ref))
        assert np.abs(v1 - v1_ref).max() <= 1e-15
    del ctypes


def test_degenerate_tuples_are_half_weighted_closed_form():
    """ijj/iij pipelines (SYMT311 + T3SQUA CF=1/2 + DRT1WT3IJ/JK) equal the
    closed-form W with a repeated index and weight 1/2."""
    inp = S.generate(5, 7, 9)
    V = O._Views(inp)
    veo = {x: O.expand_vvvo(inp, x) for x in range(inp.no)}
    for kind, i, j, k in [(1, 3, 1, 1), (2, 3, 3, 1), (1, 4, 0, 0), (2, 2, 2, 0)]:
        e_ref, v1_ref = O.c_tuple(inp, kind, i, j, k)
        v1 = np.zeros((inp.nu, inp.no), order="F")
        e = O.closed_reduce(V, i, j, k, O.closed_w(V, i, j, k, veo), 0.5, v1)
        assert abs(e - e_ref) <= 1e-14 * max(1.0, abs(e_ref))
        assert np.abs(v1.ravel(order="F") - v1_ref).max() <= 1e-15


def test_long_double_spot_check():
    """One tuple's E[4] in extended precision agrees with the FP64 oracle."""
    inp = S.generate(4, 6, 5)
    V = O._Views(inp)
    veo = {x: O.expand_vvvo(inp, x).astype(np.longdouble) for x in range(inp.no)}

    class LD:
        T2f = V.T2f.astype(np.longdouble)
        VM = V.VM.astype(np.longdouble)
        nu = V.nu
    w = O.closed_w(LD, 3, 2, 0, veo)
    d = 1.0 / ((np.longdouble(inp.eh[3]) + inp.eh[2] + inp.eh[0]) -
               (inp.ep[:, None, None] + inp.ep[None, :, None] + inp.ep[None, None, :]).astype(np.longdouble))
    P = lambda s: np.einsum(s + "->abc", w)
    x3 = np.sum((8 * w - 4 * (P("acb") + P("cba") + P("bac")) + 2 * (P("bca") + P("cab"))) * w * d)
    e_ref, _ = O.c_tuple(inp, 0, 3, 2, 0)
    assert abs(float(x3) - e_ref) <= 1e-14 * abs(e_ref)


def test_golden_fixture_reproduced_by_oracle():
    g = json.loads((GOLD / "energies.json").read_text())["water-avdz"]
    inp = S.workload("water-avdz")
    ets, etd, v1 = O.c_cc_triples(inp)
    assert ets == pytest.approx(g["ets"], abs=1e-14) and etd == pytest.approx(g["etd"], rel=1e-14)


def test_blas_pipeline_matches_plain_oracle():
    """The timed CPU baseline (the literal pipeline with OpenBLAS DGEMMs) gives
    the plain-loop oracle's energies and v1 on every tuple kind."""
    from oracle import oracle as O
    inp = S.generate(5, 23, 4)
    ets_o, etd_o, v1_o = O.c_cc_triples(inp)
    ets, etd, v1, secs, dg = O.blas_cc_triples(inp)
    assert abs(etd - etd_o) <= 1e-13 * abs(etd_o)
    assert abs(ets - ets_o) <= 1e-13 * abs(ets_o) + 1e-16
    assert np.abs(v1 - v1_o).max() <= 1e-13 * np.abs(v1_o).max()
    assert 0.0 < dg <= secs


def test_blas_tuple_w_matches_plain_oracle():
    from oracle import oracle as O
    inp = S.generate(4, 13, 6)
    for t in (O.all_tuples(4)[0], O.all_tuples(4)[-1], O.all_tuples(4)[-2]):
        assert np.abs(O.blas_tuple_w(inp, *t) - O.c_tuple_w(inp, *t)).max() <= 1e-14
