"""Failure detection without a GPU fault: a device wait that nobody
satisfies gives up at its deadline and reports TNX_ERR_TIMEOUT through a
status word, and the context stays usable afterwards (the same deadline
discipline as the mbarrier waits inside the GEMM kernels)."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tenax_b200 import dense  # noqa: E402
from tenax_b200 import _capi  # noqa: E402

TNX_ERR_TIMEOUT = 5


def _wait(flag, expected, timeout_ns, status):
    st = torch.cuda.current_stream().cuda_stream
    _capi.check(_capi.LIB.tnx_wait_flag(flag.data_ptr(), expected, timeout_ns, status.data_ptr(), st))


def test_unsatisfied_wait_times_out_and_context_survives():
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _wait(flag, 1, 50_000_000, status)  # 50 ms; nothing ever sets the flag
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert int(status.item()) == TNX_ERR_TIMEOUT
    assert 0.04 <= dt < 5.0
    # a satisfied wait reports success at once
    flag.fill_(1)
    status.fill_(-1)
    _wait(flag, 1, 50_000_000, status)
    assert int(status.item()) == 0
    # the context is still usable: a contraction runs and is right
    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.standard_normal((64, 48))).cuda()
    b = torch.from_numpy(rng.standard_normal((48, 32))).cuda()
    got = dense.einsum("ik,kj->ij", a, b)
    torch.testing.assert_close(got, a @ b, rtol=1e-12, atol=1e-12)


def test_wait_rejects_bad_arguments():
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for bad in (0, -1, 20_000_000_000):
        with pytest.raises(ValueError, match="timeout"):
            _wait(flag, 1, bad, status)
