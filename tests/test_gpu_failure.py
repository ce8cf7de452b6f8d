"""Failure detection without a GPU fault: every device-side wait of the library is bounded. A
wavefront triangular solve whose block never publishes its result makes the blocks after it run
into a short wait limit: they give up, publish NaN and record the timeout, which the host reads;
the context stays usable and the next solve is exact."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _solve(L, v, dead_block, limit):
    from nqs import _lib
    n = L.shape[0]
    ws = torch.empty((2 * 64 + 64 * 64 * ((n + 63) // 64)) * 8, dtype=torch.uint8, device="cuda")
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    x = v.clone()
    _lib.check(_lib.lib().nqs_selftest_bounded_wait(_lib.ptr(L), n, dead_block, limit,
                                                    _lib.ptr(x), _lib.ptr(ws), ws.numel(),
                                                    _lib.ptr(st), _lib.stream_ptr()),
               "nqs_selftest_bounded_wait")
    torch.cuda.synchronize()
    return x, int(st.item())


def test_flag_wait_runs_out_and_reports():
    rng = np.random.default_rng(1)
    n = 640  # ten 64-row blocks
    A = np.tril(rng.uniform(-0.1, 0.1, (n, n))) + np.eye(n) * 2.0
    L = torch.as_tensor(A).cuda().contiguous()
    v = torch.as_tensor(rng.standard_normal(n)).cuda()
    ref = torch.linalg.solve_triangular(L, v[:, None], upper=False)[:, 0]
    x, st = _solve(L, v, -1, 1 << 20)
    assert st == 0 and float((x - ref).abs().max()) < 1e-12
    # block 3 never publishes: blocks 0..3 are solved, 4..9 give up after the short limit
    x, st = _solve(L, v, 3, 4096)
    assert st == 1
    assert float((x[:256] - ref[:256]).abs().max()) < 1e-12
    assert torch.isnan(x[256:]).all()
    # the context is still usable and the next solve exact
    x, st = _solve(L, v, -1, 1 << 20)
    assert st == 0 and float((x - ref).abs().max()) < 1e-12


def test_wait_limit_setting_keeps_results():
    """A process-wide limit set and restored (0 = defaults) leaves a normal pass unchanged."""
    from nqs import _lib
    from nqs.minsr import gram_lower
    A = torch.randn(300, 1000, dtype=torch.float32, device="cuda")
    T0 = gram_lower(A, "bf16")
    _lib.check(_lib.lib().nqs_set_wait_limit(1 << 23), "nqs_set_wait_limit")
    try:
        T1 = gram_lower(A, "bf16")
    finally:
        _lib.lib().nqs_set_wait_limit(0)
    assert torch.equal(T0, T1)
