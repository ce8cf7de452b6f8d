"""nqs_energy_gradient_noalloc (static device scratch, no workspace) against nqs_energy_gradient
(caller workspace) through the C ABI: same O, same energies, two calls in a row each."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grad_ws(lib, _lib, O, o_dtype, e, W, P, out):
    ws = _lib.workspace.get(16 * W + 4096)
    _lib.check(lib.nqs_energy_gradient(_lib.ptr(O), o_dtype, _lib.ptr(e), W, P, _lib.ptr(out),
                                       _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
               "nqs_energy_gradient")


def _grad_noalloc(lib, _lib, O, o_dtype, e, W, P, out):
    _lib.check(lib.nqs_energy_gradient_noalloc(_lib.ptr(O), o_dtype, _lib.ptr(e), W, P,
                                               _lib.ptr(out), _lib.stream_ptr()),
               "nqs_energy_gradient_noalloc")


@pytest.mark.parametrize("o_dtype", [0, 1])
def test_noalloc_matches_workspace_entry_twice(o_dtype):
    import torch
    from nqs import _lib
    lib = _lib.lib()
    dev = _lib.device()
    rng = np.random.default_rng(11 + o_dtype)
    tdt = torch.float64 if o_dtype == 0 else torch.float32
    # a large call, then a smaller one that reuses the shared scratch, then the large one again
    for W, P in [(4096, 3001), (1000, 517), (4096, 3001)]:
        O = torch.as_tensor(rng.standard_normal((2 * W, P)), dtype=tdt, device=dev)
        e = torch.as_tensor(rng.standard_normal(W) * 0.3 - 2.0 + 1j * rng.standard_normal(W) * 0.01,
                            dtype=torch.complex128, device=dev)
        ref = torch.full((P,), float("nan"), dtype=torch.float64, device=dev)
        _grad_ws(lib, _lib, O, o_dtype, e, W, P, ref)
        for _ in range(2):
            got = torch.full((P,), float("nan"), dtype=torch.float64, device=dev)
            _grad_noalloc(lib, _lib, O, o_dtype, e, W, P, got)
            torch.cuda.synchronize()
            scale = float(ref.abs().max())
            assert torch.isfinite(got).all()
            assert float((got - ref).abs().max()) <= 1e-12 * scale, (W, P)


def test_noalloc_rejects_more_walkers_than_its_scratch():
    import torch
    from nqs import _lib
    lib = _lib.lib()
    dev = _lib.device()
    W = 32769  # one more than NQS_NOALLOC_MAX_WALKERS; buffers sized for it, P = 1
    O = torch.zeros((2 * W, 1), dtype=torch.float64, device=dev)
    e = torch.zeros(W, dtype=torch.complex128, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    s = lib.nqs_energy_gradient_noalloc(_lib.ptr(O), 0, _lib.ptr(e), W, 1, _lib.ptr(out),
                                        _lib.stream_ptr())
    assert s == 2  # NQS_ERR_UNSUPPORTED
    assert b"static scratch limit" in lib.nqs_last_error()
