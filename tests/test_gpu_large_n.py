"""Shapes past 16 electrons (the sizes of the reference's configurations 4 and 5): the head and
attention kernels take their general paths there. log psi, the local energy (forward Laplacian and
spin-orbit flips) and the per-sample Jacobian against the FP64 oracle (reference
src/nqs/psiformer.py:118-189, src/nqs/local_energy.py:40-117, src/nqs/minsr.py:56-65)."""
import numpy as np
import pytest

from helpers import build, configs, perturb
from oracle import nqs_oracle as O

pytestmark = pytest.mark.gpu


def _close_mod_2pi(a, b, tol):
    d = complex(a) - complex(b)
    return abs(d.real) < tol and abs((d.imag + np.pi) % (2 * np.pi) - np.pi) < tol


@pytest.mark.parametrize("kw", [
    # configuration-4-like: width 64, 3 blocks, 2 determinants, N between 16 and 26
    dict(N=20, L=9.0, embed=64, depth=3, heads=4, n_freq=8, n_dets=2),
    # configuration-5 shape: N = 48, width 128, 8 heads, 8 determinants, RBF Jastrow
    dict(N=48, L=14.0, embed=128, depth=2, heads=8, n_freq=8, n_dets=8, use_jastrow=True,
         n_knots=16),
])
def test_logpsi_large_n_matches_oracle(kw):
    from nqs.psiformer import make_logpsi
    g, model = build(**kw)
    p = perturb(model.init(0), 0.02, 41)
    R, S = configs(model.n_elec, model.L, 3, 42)
    lp = make_logpsi(model, p)(R, S).cpu()
    for w in range(R.shape[0]):
        ref = O.logpsi(model, p, R[w], S[w])
        assert _close_mod_2pi(lp[w], ref, 1e-10), (w, complex(lp[w]), complex(ref))
    # antisymmetry: swapping electrons 0 and 1 (positions and spins) flips the sign
    perm = list(range(model.n_elec))
    perm[0], perm[1] = 1, 0
    l1 = make_logpsi(model, p)(R[:, perm], S[:, perm]).cpu()
    ratio = np.exp(complex(l1[0] - lp[0]))
    assert abs(ratio + 1) < 1e-9


def test_local_energy_n18_matches_oracle():
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(N=18, L=8.5, n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 43)
    R, S = configs(model.n_elec, model.L, 2, 44)
    e = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.5)(R, S).cpu()
    for w in range(2):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.5)
        assert abs(complex(e[w]) - complex(ref)) < 1e-9 * max(1.0, abs(complex(ref)))


def test_per_sample_O_n18_matches_oracle():
    from nqs.minsr import per_sample_O, real_ravel
    g, model = build(N=18, L=8.5, n_dets=2, use_jastrow=True, n_knots=4)
    p = perturb(model.init(0), 0.05, 45)
    theta, unravel = real_ravel(p)
    R, S = configs(model.n_elec, model.L, 2, 46)
    Og = per_sample_O(model, theta.cuda(), unravel, R, S).cpu()
    ot, ou = O.real_ravel(p["params"])
    Oo = O.per_sample_O(model, ot, ou, R, S)
    assert (Og - Oo).abs().max() < 1e-10 * max(1.0, float(Oo.abs().max()))


def test_local_energy_n40_matches_oracle():
    """N = 40 (the CTA-per-job head with 3 x 3 tiles of the tangent products per thread): the
    local energy, forward Laplacian and spin-orbit flips included, against the dense-Hessian
    oracle."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(N=40, L=12.0, embed=16, depth=1, heads=4, n_dets=2, use_jastrow=True,
                     n_knots=4)
    p = perturb(model.init(0), 0.05, 47)
    R, S = configs(model.n_elec, model.L, 2, 48)
    e = make_local_energy(make_logpsi(model, p), 1.0, 1.0, 0.5)(R, S).cpu()
    for w in range(2):
        ref = O.local_energy(lambda r, s: O.logpsi(model, p, r, s), R[w], S[w], 1.0, 1.0, 0.5)
        assert abs(complex(e[w]) - complex(ref)) < 1e-9 * max(1.0, abs(complex(ref)))


@pytest.mark.parametrize("N,K,prec", [(24, 3, "fp64"), (40, 2, "fp64"), (24, 3, "mixed"),
                                      (33, 2, "mixed")])
def test_cta_kernels_equal_warp_kernels(N, K, prec):
    """The CTA-per-job determinant head and CTA-per-(job, head) attention (default past 16
    electrons) against the warp-per-task kernels they replace (nqs_set_large_n_kernels(0)).
    Float64: log psi and local energies (forward-Laplacian batch and spin-orbit flips) agree to
    1e-10 relative (the two sum in different orders). Mixed: the float32 attention's summation
    order changes the float32 rounding, so each is compared with the float64 path: log psi to
    1e-5 of each other, and the new kernels' median local-energy error no larger than 2 x the
    old kernels'."""
    from nqs import _lib
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(N=N, L=1.9 * np.sqrt(N), embed=32, depth=2, heads=4, n_dets=K,
                     use_jastrow=True, n_knots=6)
    p = perturb(model.init(0), 0.05, 50 + N)
    R, S = configs(model.n_elec, model.L, 37, 51 + N)

    def run(prec_):
        lp = make_logpsi(model, p, precision=prec_)
        return lp(R, S).cpu(), make_local_energy(lp, 1.0, 0.7, 0.3)(R, S).cpu()

    out = {}
    for on in (1, 0):
        _lib.lib().nqs_set_large_n_kernels(on)
        try:
            out[on] = run(prec)
        finally:
            _lib.lib().nqs_set_large_n_kernels(1)

    def rel(a, b):
        d = a - b
        d = d.real.abs() + ((d.imag + np.pi) % (2 * np.pi) - np.pi).abs()
        return d / b.abs().clamp(min=1.0)

    if prec == "fp64":
        for a, b in zip(out[1], out[0]):
            assert float(rel(a, b).max()) < 1e-10
        return
    l64, e64 = run("fp64")
    for q, stat in ((0, "max"), (1, "median")):  # log psi: worst walker; E_loc: median walker
        err_new = float(getattr(rel(out[1][q], l64 if q == 0 else e64), stat)())
        err_old = float(getattr(rel(out[0][q], l64 if q == 0 else e64), stat)())
        assert err_new <= 2.0 * err_old + 1e-12, (q, err_new, err_old)


def test_width128_network_runs_on_tensor_cores():
    """Width 128 with 8 determinants (the configuration-5 layer widths: QKV 384, feed-forward
    256 -> 128, backflow 2 K N = 640 outputs): the mixed path's Dense layers run as tcgen05 row-
    GEMM pieces (K <= 128, N <= 256 per launch) and its log psi and local energies follow the
    float64 path to TF32 accuracy."""
    import ctypes

    import torch
    from nqs import _lib
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    g, model = build(N=40, L=12.0, embed=128, depth=2, heads=8, n_freq=8, n_dets=8)
    p = perturb(model.init(0), 0.02, 52)
    R, S = configs(model.n_elec, model.L, 16, 53)
    L = _lib.lib()
    L.nqs_profile_gemm_read(None, None, None)
    L.nqs_profile_gemm(1)
    try:
        lm = make_logpsi(model, p, precision="mixed")
        lp32 = lm(R, S).cpu()
        em = make_local_energy(lm, 1.0, 0.7, 0.3)(R, S).cpu()
        torch.cuda.synchronize()
    finally:
        L.nqs_profile_gemm(0)
    n = ctypes.c_longlong(0)
    L.nqs_profile_gemm_read(None, None, ctypes.byref(n))
    assert n.value > 0
    l64 = make_logpsi(model, p)
    lp64 = l64(R, S).cpu()
    e64 = make_local_energy(l64, 1.0, 0.7, 0.3)(R, S).cpu()
    d = lp32 - lp64
    assert float(d.real.abs().max()) < 5e-3 * max(1.0, float(lp64.real.abs().max()))
    assert float((em - e64).abs().median()) < 1e-2 * max(1.0, float(e64.abs().median()))
