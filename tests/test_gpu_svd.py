"""GPU sector SVDs (tnx_svd_batch: cuSOLVER's polar-decomposition SVD for
large sectors, its Jacobi SVD for small ones) against
LAPACK's SVD (numpy.linalg.svd, what jnp.linalg.svd runs on the reference's
CPU backend, linalg.py:190), and the block-diagonal truncated SVD built on
them against the Jacobi driver.

Bars: singular values within 1e-12 * sigma_max of LAPACK's; U diag(s) Vh
reproduces the input to 1e-12 relative (Frobenius); U's columns and Vh's
rows orthonormal to 1e-12; the input is left unchanged."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tenax_b200 import dmrg as D  # noqa: E402


def _graded(m, k, decades, rng):
    """m x k with singular values spread log-uniformly over `decades` decades."""
    r = min(m, k)
    qu, _ = np.linalg.qr(rng.standard_normal((m, r)))
    qv, _ = np.linalg.qr(rng.standard_normal((k, r)))
    s = 10.0 ** (-decades * np.arange(r) / max(r - 1, 1))
    return (qu * s) @ qv.T


def _check(M, usv):
    U, S, Vh = (x.cpu().numpy() for x in usv)
    r = min(M.shape)
    assert U.shape == (M.shape[0], r) and S.shape == (r,) and Vh.shape == (r, M.shape[1])
    if r == 0:
        return
    s_ref = np.linalg.svd(M, compute_uv=False)
    assert np.all(np.diff(S) <= 0.0)
    np.testing.assert_allclose(S, s_ref, rtol=0, atol=1e-12 * s_ref[0])
    assert np.linalg.norm((U * S) @ Vh - M) <= 1e-12 * np.linalg.norm(M)
    np.testing.assert_allclose(U.T @ U, np.eye(r), atol=1e-12)
    np.testing.assert_allclose(Vh @ Vh.T, np.eye(r), atol=1e-12)


SHAPES = [(512, 512), (300, 120), (120, 300), (1, 1), (1, 7), (7, 1), (64, 63), (63, 64), (257, 33), (0, 5)]


@pytest.mark.parametrize("polar_min", [0, 128, 1 << 40], ids=["polar", "split", "jacobi"])
def test_sector_svds_match_lapack(polar_min):
    rng = np.random.default_rng(11)
    mats = [_graded(m, k, 10, rng) if min(m, k) > 0 else np.zeros((m, k)) for m, k in SHAPES]
    dev = [torch.as_tensor(M, device="cuda") for M in mats]
    before = [d.clone() for d in dev]
    out = D.native_sector_svds(dev, 8, polar_min)
    torch.cuda.synchronize()
    for M, usv in zip(mats, out):
        _check(M, usv)
    for a, b in zip(dev, before):
        assert torch.equal(a, b)


@pytest.mark.parametrize("workers", [1, 3, 32])
def test_worker_counts_give_identical_results(workers):
    rng = np.random.default_rng(5)
    mats = [torch.as_tensor(rng.standard_normal((m, k)), device="cuda") for m, k in SHAPES[:7]]
    ref = D.native_sector_svds(mats, 8)
    got = D.native_sector_svds(mats, workers)
    for a, b in zip(ref, got):
        for x, y in zip(a, b):
            assert torch.equal(x, y)


def test_degenerate_spectrum_reconstructs():
    """Repeated singular values: the vectors inside a degenerate cluster are
    the solver's own choice, so only the factorisation is compared."""
    rng = np.random.default_rng(3)
    qu, _ = np.linalg.qr(rng.standard_normal((200, 200)))
    qv, _ = np.linalg.qr(rng.standard_normal((150, 150)))
    s = np.repeat([1.0, 0.5, 0.25, 1e-3, 1e-6], 30)
    M = (qu[:, :150] * s) @ qv.T
    for polar_min in (0, 1 << 40):
        _check(M, D.native_sector_svds([torch.as_tensor(M, device="cuda")], 2, polar_min)[0])


def test_bad_extent_raises():
    import ctypes as C

    from tenax_b200 import _capi

    i64 = C.c_int64 * 1
    p = C.c_void_p * 1
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    with pytest.raises(ValueError):
        _capi.check(_capi.LIB.tnx_svd_batch(1, i64(-1), i64(4), p(None), p(None), p(None), p(None), 0, 1, None, st))
    with pytest.raises(ValueError):
        _capi.check(_capi.LIB.tnx_svd_batch(1, i64(3), i64(4), p(None), p(None), p(None), p(None), 0, 1, None, st))
    _capi.check(_capi.LIB.tnx_svd_batch(0, None, None, None, None, None, None, 0, 1, None, st))


def test_truncated_svd_drivers_agree():
    """The block-diagonal truncated SVD (linalg.py:75-333) of a two-site
    tensor with the library's batch and with torch's Jacobi driver:
    the same kept singular values (1e-12 relative to the largest), the same
    bond charges, and the same truncated tensor U s Vh."""
    from tenax_b200 import workloads as W
    from tenax_b200.contraction import contract

    Wl, Wr = W.chain_bulk_w()
    p = W.make_heff_problem(96, 96, Wl, Wr, np.random.default_rng(2), n_sectors=9, hi=24)
    th = p.theta
    labels = th.labels()
    left, right = list(labels[:2]), list(labels[2:])
    res = {}
    for drv in ("native", "gesvdj"):
        A, s, B, s_full = D.truncated_svd(th, left, right, "bond", 60, None, driver=drv, n_streams=4)
        res[drv] = (A, s, B, s_full)
    (A1, s1, B1, f1), (A2, s2, B2, f2) = res["native"], res["gesvdj"]
    np.testing.assert_allclose(s1, s2, rtol=0, atol=1e-12 * s2[0])
    np.testing.assert_allclose(f1, f2, rtol=0, atol=1e-12 * f2[0])
    np.testing.assert_array_equal(A1.indices[-1].charges, A2.indices[-1].charges)
    t1 = contract(D.scale_bond_axis(A1, "bond", s1), B1).todense().cpu().numpy()
    t2 = contract(D.scale_bond_axis(A2, "bond", s2), B2).todense().cpu().numpy()
    assert np.linalg.norm(t1 - t2) <= 1e-11 * np.linalg.norm(t2)
