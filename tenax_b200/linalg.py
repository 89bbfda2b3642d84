"""FP64 decompositions on the library's own cuSOLVER workers.

The reference computes one ``jnp.linalg.svd(matrix, full_matrices=False)``
per charge sector of a block SVD (linalg.py:186-192) and one per split-CTM
edge (algorithms/_split_ctm_tensor.py:1058-1074).  Here every such SVD goes
through ``tnx_svd_batch``: cuSOLVER's polar-decomposition SVD for matrices
with min(m, k) >= ``POLAR_MIN`` and its Jacobi SVD for smaller ones, on up to
``n_workers`` library-owned streams with one host thread each.
"""

from __future__ import annotations

import ctypes as C

import torch

from tenax_b200 import _capi

# below this min(m, k) the Jacobi driver is faster than the polar one
# (chi = 2048 DMRG sectors: 66 -> 2.8 vs 4.0 ms, 220 -> 14 vs 7.9 ms)
POLAR_MIN = 128


def svd_batch(mats, n_workers: int = 8, polar_min: int = POLAR_MIN):
    """Thin SVD of every matrix in ``mats`` (device tensors, any float type,
    decomposed in FP64).  Returns ``[(U, S, Vh), ...]`` like
    ``torch.linalg.svd(M, full_matrices=False)``; singular values descend.
    Blocks the calling thread until all decompositions are done; the current
    stream is ordered after them."""
    if not mats:
        return []
    dev = mats[0].device
    A = [M.to(torch.float64).contiguous() for M in mats]
    n = len(A)
    r = [min(M.shape) for M in A]
    U = [torch.empty((M.shape[0], k), dtype=torch.float64, device=dev) for M, k in zip(A, r)]
    S = [torch.empty((k,), dtype=torch.float64, device=dev) for k in r]
    Vh = [torch.empty((k, M.shape[1]), dtype=torch.float64, device=dev) for M, k in zip(A, r)]
    i64 = C.c_int64 * n
    ptrs = C.c_void_p * n
    _capi.check(_capi.LIB.tnx_svd_batch(
        n, i64(*[M.shape[0] for M in A]), i64(*[M.shape[1] for M in A]), ptrs(*[M.data_ptr() for M in A]),
        ptrs(*[x.data_ptr() for x in U]), ptrs(*[x.data_ptr() for x in S]), ptrs(*[x.data_ptr() for x in Vh]),
        int(polar_min), int(n_workers), None, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    return list(zip(U, S, Vh))


def svd(M: torch.Tensor, polar_min: int = POLAR_MIN):
    """(U, S, Vh) of one matrix through ``svd_batch``."""
    return svd_batch([M], 1, polar_min)[0]
