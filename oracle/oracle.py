"""ORACLE: CPU restatements of libcc's (T) triples correction.

TEST INFRASTRUCTURE ONLY.  Imported solely by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / ``--impl reference`` legs, as the checker or as
the timed stand-in for the reference's CPU ``triples.x``.  The product package
``libcc_b200`` never imports it.

Parity status: PARTIALLY PINNED (see the header of triples_oracle.c): the TRANT3
known-answer table and the restart-file sizes are pinned against the reference;
the energies are not, because the reference's ``triples.restart`` inputs are
missing from its tree.

Three restatements live here:

* ``c_*``       ctypes front-end of ``triples_oracle.c`` -- the literal
                triples-abc pipeline with plain-loop DGEMMs (small sizes).
* ``literal_*`` the same literal sequence with numpy/OpenBLAS DGEMMs (the
                reference also calls a vendor DGEMM); fast enough for the full
                workloads, so it is the timed CPU baseline.
* ``closed_*``  the closed form of W_abc (one expression per reference term
                label #0..#11, ``ijk_tuple.f90:56-80``) with the unified
                degenerate-tuple handling; an independent cross-check.
"""
from __future__ import annotations

import ctypes
import math
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
_lib = None


# --------------------------------------------------------------------------- build / load

def build(force: bool = False) -> pathlib.Path:
    """Compile triples_oracle.c into oracle/_build/liboracle.so with gcc."""
    src = HERE / "triples_oracle.c"
    LIB_PATH.parent.mkdir(exist_ok=True)
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-o", str(LIB_PATH), str(src), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        i64 = ctypes.c_int64
        _lib.orc_trant3.argtypes = [dp, i64, ctypes.c_int]
        _lib.orc_cc_triples.argtypes = [i64, i64] + [dp] * 7 + [dp, dp, dp]
        _lib.orc_cc_triples.restype = ctypes.c_int
        _lib.orc_getve.argtypes = [dp, i64, i64, dp]
        _lib.orc_ijk_formv3.argtypes = [i64] * 5 + [dp] * 6
        _lib.orc_ijj_formv3.argtypes = [i64] * 4 + [dp] * 5
        _lib.orc_iij_formv3.argtypes = [i64] * 4 + [dp] * 5
        _lib.orc_symt311.argtypes = [dp, i64, ctypes.c_int]
        _lib.orc_t1wt3_fused.argtypes = [i64] * 5 + [dp, dp, dp, dp, dp]
        _lib.orc_t1wt3_fused.restype = ctypes.c_double
        _lib.orc_task.argtypes = [i64, i64, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)]
        _lib.orc_div_even.argtypes = [i64, i64, i64, ctypes.POINTER(i64), ctypes.POINTER(i64)]
        _lib.orc_tuple.argtypes = [ctypes.c_int] + [i64] * 5 + [dp] * 11 + [dp]
        _lib.orc_reduce_tuple.argtypes = [ctypes.c_int] + [i64] * 5 + [dp] * 7
        _lib.orc_set_blas.argtypes = [ctypes.c_void_p]
        _lib.orc_dgemm_seconds.argtypes = [ctypes.c_int]
        _lib.orc_dgemm_seconds.restype = ctypes.c_double
        _lib.orc_cc_triples_list.argtypes = [i64, i64] + [dp] * 6 + [ctypes.POINTER(i64), i64, dp, dp]
        _lib.orc_cc_triples_list.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# --------------------------------------------------------------------------- C oracle front-end

def c_trant3(v: np.ndarray, nu: int, tid: int) -> np.ndarray:
    """TRANT3_SMP(v, nu, id) in place on a copy of the flat Fortran array."""
    out = np.ascontiguousarray(v, dtype=np.float64).copy()
    lib().orc_trant3(_p(out), nu, tid)
    return out


def c_cc_triples(inp):
    """Whole (T) driver (triples-abc semantics).  Returns (ets, etd, v1[nu*no])."""
    v1 = np.zeros(inp.nu * inp.no)
    ets = ctypes.c_double()
    etd = ctypes.c_double()
    rc = lib().orc_cc_triples(inp.no, inp.nu, _p(inp.eh), _p(inp.ep), _p(inp.t1), _p(inp.t2),
                              _p(inp.vm), _p(inp.voe), _p(inp.vvvo), _p(v1),
                              ctypes.byref(ets), ctypes.byref(etd))
    if rc != 0:
        raise MemoryError("oracle out of memory")
    return ets.value, etd.value, v1


def c_task(task: int, no: int):
    i, j, k = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    lib().orc_task(task, no, ctypes.byref(i), ctypes.byref(j), ctypes.byref(k))
    return i.value, j.value, k.value


def c_div_even(n: int, np_: int, me: int):
    nr, sr = ctypes.c_int64(), ctypes.c_int64()
    lib().orc_div_even(n, np_, me, ctypes.byref(nr), ctypes.byref(sr))
    return nr.value, sr.value


def c_getve(inp, x: int) -> np.ndarray:
    ve = np.zeros(inp.nu ** 3)
    lib().orc_getve(_p(inp.vvvo), inp.nu, x, _p(ve))
    return ve


def c_tuple_w(inp, kind: int, i: int, j: int, k: int) -> np.ndarray:
    """W (flat Fortran nu^3) of one tuple from the literal formv3 sequence, after
    SYMT311/ZEROT3 as the reference's pipeline applies them.  0-based i,j,k."""
    nu = inp.nu
    ve = {}
    for x in {i, j, k}:
        v = c_getve(inp, x)
        lib().orc_trant3(_p(v), nu, 1)
        ve[x] = v
    v3 = np.zeros(nu ** 3)
    if kind == 0:
        lib().orc_ijk_formv3(inp.no, nu, i, j, k, _p(inp.t2), _p(inp.vm), _p(ve[i]), _p(ve[j]), _p(ve[k]), _p(v3))
    elif kind == 1:  # (i, j, j)
        lib().orc_ijj_formv3(inp.no, nu, i, j, _p(inp.t2), _p(inp.vm), _p(ve[i]), _p(ve[j]), _p(v3))
        lib().orc_symt311(_p(v3), nu, 23)
        v3.reshape(nu, nu, nu)[np.arange(nu), np.arange(nu), np.arange(nu)] = 0.0
    else:  # (i, i, j)
        lib().orc_iij_formv3(inp.no, nu, i, k, _p(inp.t2), _p(inp.vm), _p(ve[i]), _p(ve[k]), _p(v3))
        lib().orc_symt311(_p(v3), nu, 12)
        v3.reshape(nu, nu, nu)[np.arange(nu), np.arange(nu), np.arange(nu)] = 0.0
    return v3


def c_tuple(inp, kind: int, i: int, j: int, k: int):
    """One tuple through the reference pipeline: returns (etd contribution, v1 contribution)."""
    nu, no = inp.nu, inp.no
    ve = {}
    for x in {i, j, k}:
        v = c_getve(inp, x)
        lib().orc_trant3(_p(v), nu, 1)
        ve[x] = v
    v3 = np.zeros(nu ** 3)
    t3 = np.zeros(nu ** 3)
    v1 = np.zeros(nu * no)
    e = ctypes.c_double(0.0)
    a, b, c = ve[i], ve[j], ve[k]
    lib().orc_tuple(kind, no, nu, i, j, k, _p(inp.t2), _p(inp.vm), _p(inp.voe), _p(inp.eh), _p(inp.ep),
                    _p(a), _p(b), _p(c), _p(v3), _p(t3), _p(v1), ctypes.byref(e))
    return e.value, v1


# --------------------------------------------------------------------------- numpy helpers

def _fv(flat: np.ndarray, shape):
    """Fortran-order view of a flat array."""
    return flat.reshape(shape, order="F")


def _perm(w: np.ndarray, spec: str) -> np.ndarray:
    """X[a,b,c] = w[spec] e.g. spec='bca' -> X[a,b,c] = w[b,c,a]."""
    return np.einsum(spec + "->abc", w)


def _trant3_np(v: np.ndarray, tid: int) -> np.ndarray:
    spec = {1: "acb", 2: "bac", 3: "cba", 4: "bca", 5: "cab"}[tid]
    return np.asfortranarray(_perm(v, spec))


def expand_vvvo(inp, x: int) -> np.ndarray:
    """VEo_x(a,b,c) = (ab|c x) as an (nu,nu,nu) Fortran array (DDCC_T_GETVE)."""
    nu = inp.nu
    nutr = nu * (nu + 1) // 2
    cols = inp.vvvo.reshape(nu * inp.no, nutr)[x * nu:(x + 1) * nu]  # [c][packed]
    rows, colsidx = np.tril_indices(nu)  # packed order: (I >= J), I outer, J inner
    ve = np.zeros((nu, nu, nu), order="F")
    for c in range(nu):
        sq = np.zeros((nu, nu))
        sq[rows, colsidx] = cols[c]
        sq[colsidx, rows] = cols[c]
        ve[:, :, c] = sq
    return ve


class _Views:
    def __init__(self, inp):
        no, nu = inp.no, inp.nu
        self.no, self.nu = no, nu
        self.T2 = _fv(inp.t2, (nu * nu, no, no))        # T2(ab, l, x)
        self.T2f = _fv(inp.t2, (nu, nu, no, no))
        self.VM = _fv(inp.vm, (no, nu, no, no))
        self.VOE = _fv(inp.voe, (nu * nu, no, no))
        self.eh, self.ep = inp.eh, inp.ep
        self.t1 = _fv(inp.t1, (no, nu))

    def t2x(self, x):            # (nu2, no)
        return self.T2[:, :, x]

    def t2xy(self, x, y):        # T2(:,:,y,x) as (nu, nu)
        return self.T2f[:, :, y, x]

    def vmxy(self, x, y):        # (no, nu)
        return self.VM[:, :, x, y]


# --------------------------------------------------------------------------- literal numpy pipeline

def _dgemm(ta: str, tb: str, alpha: float, a: np.ndarray, b: np.ndarray, beta: float, c: np.ndarray):
    """C := alpha op(A) op(B) + beta C in place, through the BLAS DGEMM the
    reference calls (scipy's handle on the image's OpenBLAS)."""
    from scipy.linalg.blas import dgemm
    out = dgemm(alpha, a, b, beta=beta, c=c, trans_a=int(ta == "t"), trans_b=int(tb == "t"), overwrite_c=1)
    if out is not c and not np.shares_memory(out, c):
        c[...] = out


def literal_ijk_w(V: _Views, i, j, k, ve_i, ve_j, ve_k) -> np.ndarray:
    """ijk_tuple_formv3 (triples-abc/ijk_tuple.f90:1-53) with BLAS DGEMMs; ve_x are the
    swapped slices ve_x(a,b,c) = (ac|b x).  Returns W (nu,nu,nu) Fortran order."""
    nu = V.nu
    nu2 = nu * nu
    v3 = np.zeros((nu, nu, nu), order="F")
    m2 = lambda v: v.reshape((nu2, nu), order="F")
    m1 = lambda v: v.reshape((nu, nu2), order="F")
    vi, vj, vk = m1(ve_i), m1(ve_j), m1(ve_k)
    _dgemm("n", "n", -1.0, V.t2x(i), V.vmxy(k, j), 0.0, m2(v3))      # #0
    _dgemm("t", "t", 1.0, vi, V.t2xy(k, j), 1.0, m2(v3))            # #11
    _dgemm("n", "n", 1.0, V.t2xy(i, k), vj, 1.0, m1(v3))            # #8
    _dgemm("t", "t", -1.0, V.vmxy(i, k), V.t2x(j), 1.0, m1(v3))     # #3
    v3 = _trant3_np(v3, 1)
    _dgemm("n", "n", -1.0, V.t2x(i), V.vmxy(j, k), 1.0, m2(v3))     # #1
    _dgemm("t", "t", 1.0, vi, V.t2xy(j, k), 1.0, m2(v3))            # #10
    _dgemm("n", "n", 1.0, V.t2xy(i, j), vk, 1.0, m1(v3))            # #6
    _dgemm("t", "t", -1.0, V.vmxy(i, j), V.t2x(k), 1.0, m1(v3))     # #5
    v3 = _trant3_np(v3, 4)
    _dgemm("n", "n", -1.0, V.t2x(j), V.vmxy(k, i), 1.0, m2(v3))     # #2
    _dgemm("t", "t", 1.0, vj, V.t2xy(k, i), 1.0, m2(v3))            # #9
    v3 = _trant3_np(v3, 1)
    _dgemm("t", "t", -1.0, V.vmxy(j, i), V.t2x(k), 1.0, m1(v3))     # #4
    _dgemm("n", "n", 1.0, V.t2xy(j, i), vk, 1.0, m1(v3))            # #7
    v3 = _trant3_np(v3, 4)
    r = np.arange(nu)
    v3[r, r, r] = 0.0                                                  # ZEROT3
    return v3


def literal_ijj_w(V: _Views, i, j, ve_i, ve_j) -> np.ndarray:
    """ijj_tuple_formv3 (triples-abc/ijj_tuple.f90) + SYMT311(23) + ZEROT3 for (i,j,j)."""
    nu = V.nu
    nu2 = nu * nu
    m2 = lambda v: v.reshape((nu2, nu), order="F")
    m1 = lambda v: v.reshape((nu, nu2), order="F")
    v3 = np.zeros((nu, nu, nu), order="F")
    _dgemm("n", "n", -1.0, V.t2x(i), V.vmxy(j, j), 0.0, m2(v3))
    v3 = _trant3_np(v3, 2)
    _dgemm("n", "n", -1.0, V.t2x(j), V.vmxy(j, i), 1.0, m2(v3))
    v3 = _trant3_np(v3, 1)
    _dgemm("n", "n", -1.0, V.t2x(j), V.vmxy(i, j), 1.0, m2(v3))
    v3 = _trant3_np(v3, 4)
    _dgemm("n", "n", 1.0, V.t2xy(i, j), m1(ve_j), 1.0, m1(v3))
    v3 = _trant3_np(v3, 3)
    _dgemm("n", "n", 1.0, V.t2xy(j, i), m1(ve_j), 1.0, m1(v3))
    v3 = _trant3_np(v3, 1)
    _dgemm("n", "n", 1.0, V.t2xy(j, j), m1(ve_i), 1.0, m1(v3))
    v3 = _trant3_np(v3, 2)
    v3 = np.asfortranarray(v3 + _perm(v3, "acb"))
    r = np.arange(nu)
    v3[r, r, r] = 0.0
    return v3


def literal_iij_w(V: _Views, i, k, ve_i, ve_k) -> np.ndarray:
    """iij_tuple_formv3 (triples-abc/iij_tuple.f90) + SYMT311(12) + ZEROT3 for (i,i,k)."""
    nu = V.nu
    nu2 = nu * nu
    m2 = lambda v: v.reshape((nu2, nu), order="F")
    m1 = lambda v: v.reshape((nu, nu2), order="F")
    v3 = np.zeros((nu, nu, nu), order="F")
    _dgemm("n", "n", -1.0, V.t2x(i), V.vmxy(k, i), 0.0, m2(v3))
    v3 = _trant3_np(v3, 1)
    _dgemm("n", "n", -1.0, V.t2x(i), V.vmxy(i, k), 1.0, m2(v3))
    v3 = _trant3_np(v3, 2)
    _dgemm("n", "n", -1.0, V.t2x(k), V.vmxy(i, i), 1.0, m2(v3))
    v3 = _trant3_np(v3, 2)
    _dgemm("n", "n", 1.0, V.t2xy(i, i), m1(ve_k), 1.0, m1(v3))
    v3 = _trant3_np(v3, 1)
    _dgemm("n", "n", 1.0, V.t2xy(i, k), m1(ve_i), 1.0, m1(v3))
    v3 = _trant3_np(v3, 3)
    _dgemm("n", "n", 1.0, V.t2xy(k, i), m1(ve_i), 1.0, m1(v3))
    v3 = _trant3_np(v3, 3)
    v3 = np.asfortranarray(v3 + _perm(v3, "bac"))
    r = np.arange(nu)
    v3[r, r, r] = 0.0
    return v3


def _smt3four(v):
    return 2.0 * (v - _perm(v, "bac")) - _perm(v, "acb") + _perm(v, "bca")


def _dinv(V: _Views, i, j, k):
    ep = V.ep
    dabc = ep[:, None, None] + ep[None, :, None] + ep[None, None, :]
    return 1.0 / ((V.eh[i] + V.eh[j] + V.eh[k]) - dabc)


def literal_reduce(V: _Views, i, j, k, w: np.ndarray, weight: float, v1: np.ndarray) -> float:
    """T3SQUA + ADT3DEN + DRT1WT3IJK for a W with W_aaa = 0.  The six T1WT3IJK calls
    of DRT1WT3IJK (triples-abc/ddcc_aux.f:146-169) are written with the permutation
    each trant3 step leaves in TI.  ``weight`` is CF (1 or 1/2).  v1 is (nu,no)."""
    nu = V.nu
    d = _dinv(V, i, j, k)
    f = 8.0 * w - 4.0 * (_perm(w, "acb") + _perm(w, "cba") + _perm(w, "bac")) + 2.0 * (_perm(w, "bca") + _perm(w, "cab"))
    x3 = float(np.sum(f * w * d))
    ti = np.asfortranarray(w * d)
    seq = [((i, j, k), None), ((i, k, j), 1), ((j, i, k), 4), ((j, k, i), 1), ((k, i, j), 5), ((k, j, i), 1)]
    for (I, J, K), t in seq:
        if t is not None:
            ti = _trant3_np(ti, t)
        z = _smt3four(ti)
        v1[:, I] += weight * (z.reshape((nu, nu * nu), order="F") @ V.VOE[:, J, K])
    return weight * x3


def literal_cc_triples(inp, tuples=None, threads=None):
    """(T) through the literal numpy pipeline.  ``tuples`` optionally restricts the
    work to a list of (kind, i, j, k) (kind 0: i>j>k, 1: (i,j,j), 2: (i,i,k));
    degenerate tuples go through the literal ijj/iij_tuple_formv3 sequences with
    SYMT311; every tuple then goes through the C restatement of T3SQUA, ADT3DEN
    and DRT1WT3IJK/IJ/JK.  Tuple energies are summed with math.fsum.  Returns (ets, etd, v1[nu,no])."""
    V = _Views(inp)
    no, nu = inp.no, inp.nu
    v1 = np.zeros((nu, no), order="F")
    etd_parts = []
    if tuples is None:
        tuples = all_tuples(no)
    cache = {}

    def ve(x):
        if x not in cache:
            if len(cache) > 3:
                cache.pop(next(iter(cache)))
            cache[x] = _trant3_np(expand_vvvo(inp, x), 1)
        return cache[x]

    v1c = np.zeros(nu * no)
    t3 = np.zeros(nu ** 3)
    for kind, i, j, k in tuples:
        if kind == 0:
            w = literal_ijk_w(V, i, j, k, ve(i), ve(j), ve(k))
        elif kind == 1:
            w = literal_ijj_w(V, i, j, ve(i), ve(j))
        else:
            w = literal_iij_w(V, i, k, ve(i), ve(k))
        wf = np.ascontiguousarray(w.ravel(order="F"))
        e = ctypes.c_double(0.0)
        lib().orc_reduce_tuple(kind, no, nu, i, j, k, _p(wf), _p(t3), _p(inp.voe), _p(inp.eh), _p(inp.ep),
                               _p(v1c), ctypes.byref(e))
        etd_parts.append(e.value)
    etd = math.fsum(etd_parts)
    v1[...] = v1c.reshape((nu, no), order="F")
    ets = 2.0 * float(np.sum(V.t1.T * v1))
    return ets, etd, v1


def all_tuples(no: int):
    """Every tuple with work: i>j>k in DDCC_T_TASK order, then for i, j<i the
    (i,j,j) and (i,i,j) tuples (triples-abc/triples.f90:232-313).  0-based."""
    out = []
    for i in range(no):
        for j in range(i):
            for k in range(j):
                out.append((0, i, j, k))
    for i in range(no):
        for j in range(i):
            out.append((1, i, j, j))
            out.append((2, i, i, j))
    return out


# --------------------------------------------------------------------------- closed form

def closed_w(V: _Views, i, j, k, veo) -> np.ndarray:
    """W_abc of tuple (i,j,k) from the twelve reference terms in closed form.
    ``veo[x]`` is VEo_x(a,b,c) = (ab|c x).  Term labels follow ijk_tuple.f90:56-80.
    With a repeated occupied index the same expression gives the symmetrised W of
    the degenerate pipelines (SYMT311 after ijj/iij_tuple_formv3), W_aaa = 0."""
    E = np.einsum
    T2 = V.T2f
    VM = V.VM
    w = -E("abl,lc->abc", T2[:, :, :, i], VM[:, :, k, j])      # 0
    w += E("dba,cd->abc", veo[i], T2[:, :, j, k])             # 11
    w += E("ad,dcb->abc", T2[:, :, k, i], veo[j])             # 8
    w -= E("la,bcl->abc", VM[:, :, i, k], T2[:, :, :, j])      # 3
    w -= E("acl,lb->abc", T2[:, :, :, i], VM[:, :, j, k])      # 1
    w += E("dca,bd->abc", veo[i], T2[:, :, k, j])             # 10
    w += E("ad,dbc->abc", T2[:, :, j, i], veo[k])             # 6
    w -= E("la,cbl->abc", VM[:, :, i, j], T2[:, :, :, k])      # 5
    w -= E("bal,lc->abc", T2[:, :, :, j], VM[:, :, k, i])      # 2
    w += E("dab,cd->abc", veo[j], T2[:, :, i, k])             # 9
    w -= E("lb,cal->abc", VM[:, :, j, i], T2[:, :, :, k])      # 4
    w += E("bd,dac->abc", T2[:, :, i, j], veo[k])             # 7
    w = np.asfortranarray(w)
    r = np.arange(V.nu)
    w[r, r, r] = 0.0
    return w


def closed_reduce(V: _Views, i, j, k, w: np.ndarray, weight: float, v1: np.ndarray) -> float:
    """E[4] and the v1 update in the fused full-sum form of t1wt3.f90:46-95:
    v1(a,i) += sum_bc [Z1 VOE(b,c,j,k) + Z2 VOE(b,c,k,j)] / D, etc."""
    nu = V.nu
    d = _dinv(V, i, j, k)
    P = lambda s: _perm(w, s)
    wabc, wacb, wbac, wbca, wcab, wcba = w, P("acb"), P("bac"), P("bca"), P("cab"), P("cba")
    x3 = float(np.sum((8 * wabc - 4 * (wacb + wcba + wbac) + 2 * (wbca + wcab)) * wabc * d))
    z1 = (wabc - wbac) * 2 - wacb + wbca
    z2 = (wacb - wbca) * 2 - wabc + wbac
    z3 = (wbac - wabc) * 2 - wcab + wcba
    z4 = (wbca - wacb) * 2 - wcba + wcab
    z5 = (wcab - wcba) * 2 - wbac + wabc
    z6 = (wcba - wcab) * 2 - wbca + wacb
    VOE = V.VOE.reshape((nu, nu, V.no, V.no), order="F")
    red = lambda z, x, y: np.einsum("abc,bc->a", z * d, VOE[:, :, x, y])
    v1[:, i] += weight * (red(z1, j, k) + red(z2, k, j))
    v1[:, j] += weight * (red(z3, i, k) + red(z5, k, i))
    v1[:, k] += weight * (red(z4, i, j) + red(z6, j, i))
    return weight * x3


def closed_cc_triples(inp, tuples=None):
    """(T) with closed-form W and the fused reduction for every tuple kind
    (weight 1/2 for degenerate tuples).  Returns (ets, etd, v1[nu,no])."""
    V = _Views(inp)
    no, nu = inp.no, inp.nu
    v1 = np.zeros((nu, no), order="F")
    etd = 0.0
    veo = {x: expand_vvvo(inp, x) for x in range(no)}
    for kind, i, j, k in (tuples or all_tuples(no)):
        w = closed_w(V, i, j, k, veo)
        etd += closed_reduce(V, i, j, k, w, 1.0 if kind == 0 else 0.5, v1)
    ets = 2.0 * float(np.sum(V.t1.T * v1))
    return ets, etd, v1


# --------------------------------------------------------------------------- adjoint (hand-derived)
#
# E(T) = sum_t w_t sum_abc [ W (P W) + sum_m z_m S_m ] / D           (closed_reduce, with
#   P W = 8W_abc - 4(W_acb + W_cba + W_bac) + 2(W_bca + W_cab),      ets = 2 sum T1 v1
#   S_m(a,b,c) = u_x(a) VOE(b,c,y,z),  u_x(a) = 2 T1(x,a)             written per tuple)
# D is symmetric in (a,b,c), so  dE/dW = w (2 P W + H) / D  with H the adjoint of the
# z_m combinations applied to S_m (each W at a permuted index moves to S at the
# inverse permutation).  The W-build is bilinear: every closed-form term
# W ±= A (x) B gives dA ±= dW (x) B and dB ±= A (x) dW.

# (sign, einsum spec, operand A, operand B) of the twelve closed_w terms; operands
# are ('T2', l-or-':' slice) etc. resolved per tuple.
_W_TERMS = (
    (-1, "abl,lc->abc", ("T2x", "i"), ("VM", "k", "j")),     # 0
    (+1, "dba,cd->abc", ("veo", "i"), ("T2", "j", "k")),     # 11
    (+1, "ad,dcb->abc", ("T2", "k", "i"), ("veo", "j")),     # 8
    (-1, "la,bcl->abc", ("VM", "i", "k"), ("T2x", "j")),     # 3
    (-1, "acl,lb->abc", ("T2x", "i"), ("VM", "j", "k")),     # 1
    (+1, "dca,bd->abc", ("veo", "i"), ("T2", "k", "j")),     # 10
    (+1, "ad,dbc->abc", ("T2", "j", "i"), ("veo", "k")),     # 6
    (-1, "la,cbl->abc", ("VM", "i", "j"), ("T2x", "k")),     # 5
    (-1, "bal,lc->abc", ("T2x", "j"), ("VM", "k", "i")),     # 2
    (+1, "dab,cd->abc", ("veo", "j"), ("T2", "i", "k")),     # 9
    (-1, "lb,cal->abc", ("VM", "j", "i"), ("T2x", "k")),     # 4
    (+1, "bd,dac->abc", ("T2", "i", "j"), ("veo", "k")),     # 7
)


def _z_adjoint(s):
    """H contributions of the six z_m: for z_m = sum_pi c_pi W(pi), sum_abc z_m S d =
    sum_abc W (sum_pi c_pi S(pi^-1)) d.  Returns the six adjoint combinations in the
    order z1..z6, each a list of (coefficient, spec) applied to that z's S."""
    return {
        1: ((2, "abc"), (-2, "bac"), (-1, "acb"), (1, "cab")),
        2: ((2, "acb"), (-2, "cab"), (-1, "abc"), (1, "bac")),
        3: ((2, "bac"), (-2, "abc"), (-1, "bca"), (1, "cba")),
        4: ((2, "cab"), (-2, "acb"), (-1, "cba"), (1, "bca")),
        5: ((2, "bca"), (-2, "cba"), (-1, "bac"), (1, "abc")),
        6: ((2, "cba"), (-2, "bca"), (-1, "cab"), (1, "acb")),
    }[s]


def closed_grad(inp, tuples=None):
    """Hand-derived FP64 gradient of E(T) = ets + etd with respect to every input,
    in the input layouts: dict with eh (no), ep (nu), t1 (no*nu, file layout),
    t2 (nu*nu*no*no), vm (no*nu*no*no), voe (nu*nu*no*no), vvvo (packed, like
    the input), and e_t.  W is recomputed per tuple (nothing of size nu^3 is kept
    across tuples)."""
    V = _Views(inp)
    no, nu = inp.no, inp.nu
    tuples = tuples or all_tuples(no)
    veo = {x: expand_vvvo(inp, x) for x in range(no)}
    ets, etd, v1 = closed_cc_triples(inp, tuples)
    gT2 = np.zeros((nu, nu, no, no), order="F")
    gVM = np.zeros((no, nu, no, no), order="F")
    gVOE = np.zeros((nu, nu, no, no), order="F")
    gveo = {x: np.zeros((nu, nu, nu), order="F") for x in range(no)}
    geh, gep = np.zeros(no), np.zeros(nu)
    VOE4 = V.VOE.reshape((nu, nu, no, no), order="F")
    u = 2.0 * V.t1  # u[x, a] = 2 T1(x, a)
    r = np.arange(nu)
    for kind, i, j, k in tuples:
        weight = 1.0 if kind == 0 else 0.5
        w = closed_w(V, i, j, k, veo)
        d = _dinv(V, i, j, k)
        P = lambda s, a=w: _perm(a, s)
        pw = 8 * w - 4 * (P("acb") + P("cba") + P("bac")) + 2 * (P("bca") + P("cab"))
        smap = {1: (i, j, k), 2: (i, k, j), 3: (j, i, k), 4: (k, i, j), 5: (j, k, i), 6: (k, j, i)}
        H = np.zeros((nu, nu, nu))
        for m, (x, y, z) in smap.items():
            S = u[x][:, None, None] * VOE4[None, :, :, y, z]
            for c, spec in _z_adjoint(m):
                H += c * _perm(S, spec)
        gw = weight * d * (2.0 * pw + H)
        gw[r, r, r] = 0.0
        # denominators: E_t = w sum N d with N ~ W (P W + H) on each permutation orbit
        Mw = weight * w * (pw + H) * d * d
        tot = float(Mw.sum())
        for x in (i, j, k):
            geh[x] -= tot
        gep += Mw.sum(axis=(1, 2)) + Mw.sum(axis=(0, 2)) + Mw.sum(axis=(0, 1))
        # VOE: dVOE(b,c,y,z) += w sum_a z_m(a,b,c) u_x(a) d(a,b,c)
        zs = {1: (w - P("bac")) * 2 - P("acb") + P("bca"), 2: (P("acb") - P("bca")) * 2 - w + P("bac"),
              3: (P("bac") - w) * 2 - P("cab") + P("cba"), 4: (P("bca") - P("acb")) * 2 - P("cba") + P("cab"),
              5: (P("cab") - P("cba")) * 2 - P("bac") + w, 6: (P("cba") - P("cab")) * 2 - P("bca") + P("acb")}
        for m, (x, y, z) in smap.items():
            gVOE[:, :, y, z] += weight * np.einsum("abc,a->bc", zs[m] * d, u[x])
        # the twelve W-build terms
        idx = {"i": i, "j": j, "k": k}

        def operand(spec):
            kind_, *ix = spec
            if kind_ == "T2x":
                x = idx[ix[0]]
                return V.T2f[:, :, :, x], gT2[:, :, :, x]
            if kind_ == "T2":
                return V.T2f[:, :, idx[ix[0]], idx[ix[1]]], gT2[:, :, idx[ix[0]], idx[ix[1]]]
            if kind_ == "VM":
                return V.VM[:, :, idx[ix[0]], idx[ix[1]]], gVM[:, :, idx[ix[0]], idx[ix[1]]]
            x = idx[ix[0]]
            return veo[x], gveo[x]

        for sign, spec, sa, sb in _W_TERMS:
            ins, out = spec.split("->")
            sA, sB = ins.split(",")
            A, gA = operand(sa)
            B, gB = operand(sb)
            gA += sign * np.einsum(f"{out},{sB}->{sA}", gw, B, optimize=True)
            gB += sign * np.einsum(f"{sA},{out}->{sB}", A, gw, optimize=True)
    # packed VVVO: column x*nu + c holds (I >= J) of (I J | c x), tril order
    nutr = nu * (nu + 1) // 2
    gvvvo = np.zeros((nu * no, nutr))
    I, J = np.tril_indices(nu)
    for x in range(no):
        g = gveo[x]
        for c in range(nu):
            sq = g[:, :, c]
            gvvvo[x * nu + c] = np.where(I == J, sq[I, J], sq[I, J] + sq[J, I])
    gt1 = 2.0 * v1.T  # dE/dT1(x,a) = 2 v1(a,x)
    return {"eh": geh, "ep": gep, "t1": np.asfortranarray(gt1).ravel(order="F"),
            "t2": gT2.ravel(order="F"), "vm": gVM.ravel(order="F"), "voe": gVOE.ravel(order="F"),
            "vvvo": gvvvo.ravel(), "e_t": ets + etd}


# --------------------------------------------------------------------------- BLAS-backed C pipeline

def _blas_dgemm_pointer() -> int:
    """Address of the BLAS DGEMM behind scipy.linalg (the image's OpenBLAS),
    Fortran calling convention with 32-bit integers."""
    import scipy.linalg.cython_blas as cb
    cap = cb.__pyx_capi__["dgemm"]
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype, get_name.argtypes = ctypes.c_char_p, [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype, get_ptr.argtypes = ctypes.c_void_p, [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(cap, get_name(cap))


def blas_cc_triples(inp, tuples=None):
    """The literal triples-abc pipeline of triples_oracle.c (OpenMP TRANT3,
    T3SQUA, ADT3DEN, SMT3FOUR/T1WT3IJK loops) with every DGEMM sent to the
    image's OpenBLAS: the reference CPU algorithm, the timed CPU baseline.
    Returns (ets, etd, v1[nu*no], seconds, dgemm_seconds)."""
    import time
    L = lib()
    L.orc_set_blas(_blas_dgemm_pointer())
    tuples = all_tuples(inp.no) if tuples is None else tuples
    arr = np.ascontiguousarray(np.array(tuples, dtype=np.int64).reshape(-1, 4))
    v1 = np.zeros(inp.nu * inp.no)
    etd = ctypes.c_double(0.0)
    L.orc_dgemm_seconds(1)
    t0 = time.perf_counter()
    rc = L.orc_cc_triples_list(inp.no, inp.nu, _p(inp.eh), _p(inp.ep), _p(inp.t2), _p(inp.vm), _p(inp.voe),
                               _p(inp.vvvo), arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(arr),
                               _p(v1), ctypes.byref(etd))
    secs = time.perf_counter() - t0
    dg = L.orc_dgemm_seconds(1)
    L.orc_set_blas(None)
    if rc != 0:
        raise MemoryError("oracle out of memory")
    t1 = _fv(inp.t1, (inp.no, inp.nu))
    ets = 2.0 * float(np.sum(t1.T * v1.reshape((inp.nu, inp.no), order="F")))
    return ets, etd.value, v1, secs, dg


def blas_tuple_w(inp, kind: int, i: int, j: int, k: int) -> np.ndarray:
    """``c_tuple_w`` (the literal formv3 / SYMT311 / ZEROT3 W of one tuple) with
    its DGEMMs sent to the image's OpenBLAS: fast enough at nu = 320."""
    L = lib()
    L.orc_set_blas(_blas_dgemm_pointer())
    try:
        return c_tuple_w(inp, kind, i, j, k)
    finally:
        L.orc_set_blas(None)


def openblas_dgemm_tflops(n: int = 4096, reps: int = 3) -> float:
    """Best-of-reps TFLOP/s of an n^3 DGEMM through the same OpenBLAS."""
    import time
    from scipy.linalg.blas import dgemm
    a = np.asfortranarray(np.random.default_rng(0).standard_normal((n, n)))
    b = np.asfortranarray(np.random.default_rng(1).standard_normal((n, n)))
    dgemm(1.0, a[:256, :256], b[:256, :256])
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        dgemm(1.0, a, b)
        best = min(best, time.perf_counter() - t0)
    return 2.0 * n ** 3 / best / 1e12


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


# --------------------------------------------------------------------------- CCSD T1-dressing terms
#
# The two routines of the reference's OpenACC CCSD port, src/triples-ijk/ccsd_acc.f
# (terms_29_30_31, lines 1-60; terms_32_33_34_35, lines 64-160), restated as
# their literal DGEMM / permutation sequence for one process that holds every
# occupied index (DIV_EVEN over one rank).  Nothing in the reference tree calls
# them.  Permutation helpers, from the reference's TRANMD_SMP
# (common_functions.f:141-421) and GAMESS conventions for the two the tree
# does not define:
#   TRANMD(A,n1,n2,n3,n4,13): new(a,b,c,l) = old(c,b,a,l);   12: old(b,a,c,l);
#                            23: old(a,c,b,l);  312: new(x,y,z,l) = old(z,x,y,l)
#   INSITU(n1,n2,n3,n4,tmp,V,12): V(n1,n2,n3,n4) becomes V'(n2,n1,n3,n4),
#                            V'(x,y,z,w) = V(y,x,z,w); 13 and 23 likewise
#   TRANSQ(A,n): the n x n matrix A transposed in place.
# Two places of the literal code are not followed: the TRANMD of the scratch
# buffer tmp at ccsd_acc.f:33 (it transposes a buffer of nutr*nu doubles as if
# it held nu^3, and nothing reads it afterwards except as scratch), and the VM
# update loop at ccsd_acc.f:136-144, whose vm(iof1+i) / tmp(iof2+i) with iof1
# and i both starting at 1 skip the first element of every (j, a) block and add
# into the next one; the restatement adds tmp((k,l),a) to VM(k,l,j,a).

def _tranmd(a: np.ndarray, code: int) -> np.ndarray:
    """TRANMD on a 4-index Fortran array (returns a new array)."""
    spec = {12: "bacd", 13: "cbad", 23: "acbd", 312: "cabd"}[code]
    return np.asfortranarray(np.einsum(spec + "->abcd", a))


def _insitu(a: np.ndarray, code: int) -> np.ndarray:
    """INSITU: the two named indices of a 4-index array exchanged (new shape)."""
    axes = {12: (1, 0, 2, 3), 13: (2, 1, 0, 3), 23: (0, 2, 1, 3)}[code]
    return np.asfortranarray(np.transpose(a, axes))


def _transq(flat: np.ndarray, n: int) -> np.ndarray:
    return np.ascontiguousarray(flat.reshape((n, n), order="F").T.ravel(order="F"))


def _vvvo_slice(vvvo: np.ndarray, no: int, nu: int, j: int) -> np.ndarray:
    """DDCC_T_GETVE_acc (ddcc_aux.f:18-45): VE(x,y,z) = (xy|z j), Fortran (nu,nu,nu)."""
    nutr = nu * (nu + 1) // 2
    cols = vvvo.reshape(nu * no, nutr)[j * nu:(j + 1) * nu]
    r, c = np.tril_indices(nu)
    ve = np.zeros((nu, nu, nu), order="F")
    for z in range(nu):
        ve[r, c, z] = cols[z]
        ve[c, r, z] = cols[z]
    return ve


def literal_terms_29_30_31(no, nu, o1, t2, vl, vr, vvvo):
    """terms_29_30_31: returns the new t2 (no,nu,nu,no).  o1 (no,nu); vl the DDI
    array D_VL as (no,nu,nu,no); vr D_VR_IBT as (nu,no,nu,no); vvvo packed."""
    O1 = o1.reshape((no, nu), order="F")
    T2 = np.array(t2, dtype=np.float64).reshape((no, nu * nu, no), order="F").copy(order="F")
    VL = vl.reshape((no, nu * nu, no), order="F")
    VR = vr.reshape((nu, no, nu, no), order="F")
    for j in range(no):
        ve = _vvvo_slice(vvvo, no, nu, j)
        ve2 = ve.reshape((nu, nu * nu), order="F") - O1.T @ VL[:, :, j]               # DGEMM('T','N') line 37
        ve = _tranmd(ve2.reshape((nu, nu, nu, 1), order="F"), 13)                      # line 44
        rl = _insitu(_insitu(VR[:, :, :, j].reshape((nu, no, nu, 1), order="F"), 13), 12)  # lines 46-47
        ve2 = ve.reshape((nu, nu * nu), order="F") - O1.T @ rl.reshape((no, nu * nu), order="F")  # line 49
        ve = _tranmd(ve2.reshape((nu, nu, nu, 1), order="F"), 12)                      # line 52
        T2[:, :, j] += O1 @ ve.reshape((nu, nu * nu), order="F")                       # line 54
    return T2.ravel(order="F")


def literal_terms_32_35(no, nu, o1, o2, t2, vm, vvvo):
    """terms_32_33_34_35: returns (t2, o2, vm, rl) as the routine leaves them:
    t2 transposed as an (nou x nou) matrix, o2 permuted to (nu,nu,no,no), vm
    updated, rl the new (nou x nou) array.  o1 (no,nu); o2 (no,nu,nu,no);
    t2 (no,nu,nu,no); vm (no,no,no,nu); vvvo packed."""
    nou = no * nu
    O1 = o1.reshape((no, nu), order="F")
    t2n = _transq(np.asarray(t2, dtype=np.float64), nou)                               # line 83
    O2 = _insitu(_insitu(np.asarray(o2).reshape((no, nu, nu, no), order="F"), 12), 23)  # lines 84-85
    VM = _tranmd(np.asarray(vm).reshape((no, no, no, nu), order="F"), 312)             # line 86
    RL = np.zeros((no, nu * nu, no), order="F")
    for j in range(no):
        ve = _vvvo_slice(vvvo, no, nu, j)
        RL[:, :, j] = O1 @ ve.reshape((nu, nu * nu), order="F")                        # line 109
        ve13 = _tranmd(ve.reshape((nu, nu, nu, 1), order="F"), 13)                     # line 114
        tmp = O2.reshape((nu * nu, no * no), order="F").T @ ve13.reshape((nu * nu, nu), order="F")  # line 119
        VM[:, :, j, :] += tmp.reshape((no, no, nu), order="F")                          # lines 125-131 (intended)
    rl = _transq(RL.ravel(order="F"), nou)                                             # line 151
    VM = _tranmd(VM, 23)                                                               # line 154
    return t2n, O2.ravel(order="F"), VM.ravel(order="F"), rl


def closed_terms_29_30_31(no, nu, o1, t2, vl, vr, vvvo, only_j=None):
    """The same update in closed form (derived from the sequence above):
    T2(i,y,z,j) += sum_x O1(i,x) [ (z x|y j) - sum_k O1(k,z) VL(k,x,y,j)
                                   - sum_k O1(k,y) VR(z,k,x,j) ].
    With only_j set, returns just the updated slab T2(:,:,:,only_j)."""
    O1 = o1.reshape((no, nu), order="F")
    VL = vl.reshape((no, nu, nu, no), order="F")
    VR = vr.reshape((nu, no, nu, no), order="F")
    T2 = np.array(t2, dtype=np.float64).reshape((no, nu, nu, no), order="F").copy(order="F")
    for j in (range(no) if only_j is None else [only_j]):
        V = _vvvo_slice(vvvo, no, nu, j)                  # V[x,y,z] = (xy|z j)
        G = np.einsum("zxy->xyz", V) - np.einsum("kz,kxy->xyz", O1, VL[:, :, :, j], optimize=True) \
            - np.einsum("ky,zkx->xyz", O1, VR[:, :, :, j], optimize=True)
        T2[:, :, :, j] += np.einsum("ix,xyz->iyz", O1, G, optimize=True)
    return T2.ravel(order="F") if only_j is None else T2[:, :, :, only_j]
