"""CPU oracle for the block-sparse symmetric contraction hot path.

TEST INFRASTRUCTURE ONLY.  This package is a float64 NumPy restatement of the
reference algorithms (tenax ``core/tensor.py``, ``contraction/contractor.py``,
``algorithms/dmrg.py``, ``linalg.py``, ``algorithms/ipeps.py``); every
function cites the reference file:line it follows.  It is imported only by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` -- as the checker and as the timed
CPU baseline, never as a product code path.  The product package
(``tenax_b200``) never imports it and fails loudly when its CUDA library is
missing.

Parity pin: the restatement is checked against golden fixtures in
``tests/golden/`` that were produced by executing the reference's own source
(with a NumPy stand-in for jax) -- see ``tests/golden/make_golden.py``.
"""

from oracle.blocksparse import (  # noqa: F401
    OTensor,
    Leg,
    block_shape,
    blockwise_contract,
    contract_symmetric,
    inner,
    norm,
    t_add,
    t_scale,
    valid_blocks,
)
