"""The allocation-free reduction entry point, ccT_reduce_w_noalloc.

Some callers cannot let a library allocate device memory: codes that reserve
all of their GPU buffers in one arena when they start, and drivers that must
not risk the device synchronisation a cudaMalloc/cudaFree can bring in the
middle of their own asynchronous work.  For them the library offers this one
entry point, which keeps its scratch in a fixed device array (sized for
nu <= CCT_NOALLOC_MAX_NU) instead of allocating.

Here it is called through the C ABI, twice in a row on different tuples (so
the second call starts from the first call's leftovers in the shared scratch
array), then once more on the first tuple, and each result is checked against
the plan path (ccT_forward over that single tuple) with the tolerance of the
other parity tests.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from libcc_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def tol(e_ref: float) -> float:
    return max(1e-10, 2e-14 * abs(e_ref))


def test_noalloc_reduction_matches_plan_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    from libcc_b200 import _native as N
    from libcc_b200 import api as A
    from oracle import oracle as O

    lib = N.load()
    no, nu = 5, 23
    inp = S.generate(no, nu, 41)
    tuples = O.all_tuples(no)
    first_ijk = next(t for t, tup in enumerate(tuples) if tup[0] == 0)
    first_ijj = next(t for t, tup in enumerate(tuples) if tup[0] == 1)
    first_iij = next(t for t, tup in enumerate(tuples) if tup[0] == 2)
    order = [first_ijk, first_ijj, first_iij, first_ijk]

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()

    eh, ep, voe = dev(inp.eh), dev(inp.ep), dev(inp.voe)
    with A.TriplesPlan(no, nu) as plan:
        plan.set_system(inp)
        for tix in order:
            kind, i, j, k = tuples[tix]
            _, etd_ref, v1_ref = plan.forward(tix, tix + 1)
            w = dev(O.c_tuple_w(inp, kind, i, j, k))
            etd_acc = torch.zeros(2, dtype=torch.float64, device="cuda")
            v1_acc = torch.zeros(nu * no, dtype=torch.float64, device="cuda")
            p = lambda t: ctypes.c_void_p(t.data_ptr())
            rc = lib.ccT_reduce_w_noalloc(no, nu, i, j, k, p(w), p(eh), p(ep), p(voe), p(etd_acc), p(v1_acc), None)
            assert rc == 0, lib.ccT_last_error()
            torch.cuda.synchronize()
            etd = float(etd_acc[0] + etd_acc[1])
            v1 = v1_acc.cpu().numpy()
            assert abs(etd - etd_ref) <= tol(etd_ref), (tuples[tix], etd, etd_ref)
            assert np.abs(v1 - v1_ref).max() <= 1e-13 * max(1.0, np.abs(v1_ref).max()), tuples[tix]


@pytest.mark.parametrize("no,nu", [(3, 64), (4, 320)])
def test_noalloc_reduction_at_block_multiple_and_limit(no, nu):
    """nu a multiple of the 8-wide reduction block (64), and nu at the limit
    (320: 40 blocks, 11480 block triples, the whole scratch array): a W from
    the FP64 plan (ccT_tuple_w) through the allocation-free reduction, twice in
    a row, against the plan's own forward over that one tuple."""
    torch = pytest.importorskip("torch")
    from libcc_b200 import _native as N
    from libcc_b200 import api as A
    from oracle import oracle as O

    lib = N.load()
    inp = S.generate(no, nu, 43 + nu)
    tuples = O.all_tuples(no)
    pick = [next(t for t, tup in enumerate(tuples) if tup[0] == kd) for kd in (0, 2)]

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()

    eh, ep, voe = dev(inp.eh), dev(inp.ep), dev(inp.voe)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    with A.TriplesPlan(no, nu) as plan:
        plan.set_system(inp)
        for tix in pick:
            kind, i, j, k = tuples[tix]
            _, etd_ref, v1_ref = plan.forward(tix, tix + 1)
            w = dev(plan.tuple_w(tix))
            for _ in range(2):
                etd_acc = torch.zeros(2, dtype=torch.float64, device="cuda")
                v1_acc = torch.zeros(nu * no, dtype=torch.float64, device="cuda")
                rc = lib.ccT_reduce_w_noalloc(no, nu, i, j, k, p(w), p(eh), p(ep), p(voe), p(etd_acc), p(v1_acc),
                                              None)
                assert rc == 0, lib.ccT_last_error()
                torch.cuda.synchronize()
                etd = float(etd_acc[0] + etd_acc[1])
                assert abs(etd - etd_ref) <= tol(etd_ref), (tuples[tix], etd, etd_ref)
                v1 = v1_acc.cpu().numpy()
                assert np.abs(v1 - v1_ref).max() <= 1e-13 * max(1.0, np.abs(v1_ref).max()), tuples[tix]


def test_noalloc_rejects_nu_beyond_its_scratch():
    from libcc_b200 import _native as N
    lib = N.load()
    cap = 320
    dummy = ctypes.c_void_p(16)
    rc = lib.ccT_reduce_w_noalloc(4, cap + 1, 2, 1, 0, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == 1
    assert b"320" in lib.ccT_last_error()
