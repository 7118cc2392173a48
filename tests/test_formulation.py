"""CPU model of the device formulation, checked against the oracle.

The CUDA path never forms the reference's twelve GEMMs: it builds E and F
(libcc_b200/csrc/cct_layout.cu), runs three grouped GEMMs per tuple
(cct_wbuild_f64.cu) and assembles W with per-kind index permutations
(cct_reduce.cu).  This file restates those three steps with numpy and checks
the assembled W against the literal reference pipeline of the oracle for every
tuple kind, so a formulation error shows up here without a GPU.
"""
import numpy as np
import pytest

from libcc_b200 import synthetic as S
from oracle import oracle as O


def model_E_F(inp):
    no, nu = inp.no, inp.nu
    KP = nu + no
    T2 = inp.t2.reshape((nu, nu, no, no), order="F")
    VM = inp.vm.reshape((no, nu, no, no), order="F")
    E = np.zeros((no, nu, nu, KP))
    for x in range(no):
        veo = O.expand_vvvo(inp, x)               # veo[a,b,c] = (ab|c x)
        # E[x][r1][r2][d] = (d r2 | r1 x) = veo[d, r2, r1]
        E[x, :, :, :nu] = np.transpose(veo, (2, 1, 0))
        # E[x][r1][r2][nu+l] = -T2(r1, r2, l, x)
        E[x, :, :, nu:] = -T2[:, :, :, x]
    F = np.zeros((no, no, nu, KP))
    for y in range(no):
        for z in range(no):
            F[y, z, :, :nu] = T2[:, :, y, z]                 # F[y][z][s][d] = T2(s,d,y,z)
            F[y, z, :, nu:] = VM[:, :, z, y].T               # F[y][z][s][nu+l] = VM(l,s,z,y)
    return E, F


def model_G(E, F, x1, x2, x3, halves=2):
    """X(p,q,s) = sum_k E[x1][p][q][k] F[x2][x3][s][k] (+ E[x2][q][p][k] F[x1][x3][s][k])."""
    X = np.einsum("pqk,sk->pqs", E[x1], F[x2, x3])
    if halves == 2:
        X = X + np.einsum("qpk,sk->pqs", E[x2], F[x1, x3])
    return X


def model_W(E, F, kind, i, j, k):
    P = lambda X, spec: np.einsum(spec + "->abc", X)
    if kind == 0:
        X0, X1, X2 = model_G(E, F, i, j, k), model_G(E, F, i, k, j), model_G(E, F, j, k, i)
        W = X0 + P(X1, "acb") + P(X2, "bca")
    elif kind == 1:   # (i, j, j)
        X0, X1 = model_G(E, F, i, j, j), model_G(E, F, j, j, i, halves=1)
        W = X0 + P(X0, "acb") + P(X1, "bca") + P(X1, "cba")
    else:             # (i, i, k)
        X0, X1 = model_G(E, F, i, i, k, halves=1), model_G(E, F, i, k, i)
        W = X0 + P(X0, "bac") + P(X1, "acb") + P(X1, "bca")
    nu = W.shape[0]
    r = np.arange(nu)
    W[r, r, r] = 0.0
    return W


@pytest.mark.parametrize("no,nu,seed", [(4, 7, 0), (5, 9, 3), (6, 5, 11)])
def test_grouped_gemms_reproduce_reference_w(no, nu, seed):
    inp = S.generate(no, nu, seed)
    E, F = model_E_F(inp)
    for kind, i, j, k in O.all_tuples(no):
        ref = O.c_tuple_w(inp, kind, i, j, k).reshape((nu, nu, nu), order="F")
        got = model_W(E, F, kind, i, j, k)
        assert np.abs(got - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max()), (kind, i, j, k)
