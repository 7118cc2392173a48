"""Rank body for the multi-process shard tests (spawned; gloo on CPU).

Each rank computes its tuple shard with the oracle's per-tuple pipeline and the
ranks' partial sums are combined by ``libcc_b200.shard.sharded_forward``."""
import datetime
import os
import sys


def oracle_forward(inp):
    """forward(begin, end) over the oracle's tuple list (plan order)."""
    import numpy as np
    from oracle import oracle as O
    tuples = O.all_tuples(inp.no)

    def fwd(b, e):
        etd, v1 = 0.0, np.zeros(inp.nu * inp.no)
        for kind, i, j, k in tuples[b:e]:
            de, dv = O.c_tuple(inp, kind, i, j, k)
            etd += de
            v1 += dv
        # ets = 2 ddot(trpose(t1), v1): t1 is (no,nu), v1 is (nu,no), both column-major
        t1 = inp.t1.reshape(inp.nu, inp.no)
        ets = 2.0 * float(np.sum(t1 * v1.reshape(inp.no, inp.nu).T))
        return ets, etd, v1
    return fwd


def run(rank, world, port, no, nu, seed, want_v1, out_dir):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import numpy as np
    import torch.distributed as dist
    from libcc_b200 import shard, synthetic
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        inp = synthetic.generate(no, nu, seed)
        calls = []
        base = oracle_forward(inp)

        def fwd(b, e):
            calls.append((b, e))
            return base(b, e)
        ets, etd, v1 = shard.sharded_forward(fwd, no, nu, want_v1=want_v1)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), ets=ets, etd=etd,
                 v1=v1 if v1 is not None else np.zeros(0), calls=np.array(calls, dtype=np.int64).reshape(-1, 2))
    finally:
        dist.destroy_process_group()
