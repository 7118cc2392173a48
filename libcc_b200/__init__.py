"""libcc_b200: B200-native (sm_100a) CCSD(T) triples correction E(T).

A from-scratch CUDA implementation of the (T) path of libcc's ``triples.x``
(src/triples-ijk, src/triples-abc, tools/trant3) behind the C ABI declared in
``include/libcc_b200.h``.  Python here is host glue only; every number comes
from the CUDA kernels in ``libcc_b200/csrc``.
"""
from . import synthetic  # noqa: F401
from . import api  # noqa: F401
