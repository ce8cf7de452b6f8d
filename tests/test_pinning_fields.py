"""Pinning fields (reference src/nqs/pinning.py:20-119) on the CPU: the vectorised ext_field
callables against the per-point oracle, the competitor dispatch of make_pin, and the field
magnitude h_pin the reference's own production test checks (tests/test_nqs_production.py:47-60)."""
import numpy as np
import pytest
import torch

from oracle import pinning_oracle as OO

QSTAR = 0.9548
Q1 = QSTAR * np.array([1.0, 0.0])
Q2 = QSTAR * np.array([-0.5, np.sqrt(3) / 2])


def _points(n, seed):
    return np.random.default_rng(seed).uniform(-9.0, 9.0, (n, 2))


def _check(field, ref, pts, tol=1e-13):
    got = field(torch.as_tensor(pts)).numpy()
    assert got.shape == (len(pts), 3)
    for r, g in zip(pts, got):
        assert np.abs(g - np.asarray(ref(r))).max() < tol
    # a single position (the local energy's per-electron call) gives one 3-vector
    one = field(torch.as_tensor(pts[0])).numpy()
    assert one.shape == (3,) and np.abs(one - got[0]).max() < 1e-15


@pytest.mark.parametrize("neel", [True, False])
def test_skx_field_matches_oracle(neel):
    from nqs.pinning import make_skx_pin
    f = make_skx_pin(Q1, Q2, 0.7, m0=0.4, chirality=-1.0, neel=neel)
    _check(f, lambda r: OO.skx_field(r, Q1, Q2, 0.7, 0.4, -1.0, neel), _points(50, 1))
    n = np.linalg.norm(f(torch.as_tensor(_points(50, 2))).numpy(), axis=-1)
    assert np.abs(n - 0.7).max() < 1e-9  # a unit texture times h_pin


def test_spiral_fm_overhauser_fields_match_oracle():
    from nqs.pinning import make_fm_pin, make_overhauser_pin, make_spiral_pin
    Q = np.array([0.8, -0.3])
    pts = _points(40, 3)
    _check(make_spiral_pin(Q, 0.5), lambda r: OO.spiral_field(r, Q, 0.5, True), pts)
    _check(make_spiral_pin(Q, 0.5, cycloidal=False), lambda r: OO.spiral_field(r, Q, 0.5, False),
           pts)
    _check(make_overhauser_pin(Q, 0.25), lambda r: OO.overhauser_field(r, Q, 0.25), pts)
    _check(make_fm_pin(0.3, axis=(1.0, 2.0, -2.0)),
           lambda r: OO.fm_field(r, 0.3, (1.0, 2.0, -2.0)), pts)


def test_make_pin_dispatch():
    from nqs.pinning import make_pin
    assert make_pin("fluid", Q1, Q2, 1.0) is None
    r = torch.as_tensor(_points(5, 6))
    assert torch.allclose(make_pin("skx_bloch", Q1, Q2, 1.0, m0=0.2)(r),
                          torch.as_tensor([OO.skx_field(p, Q1, Q2, 1.0, 0.2, 1.0, False)
                                           for p in r.numpy()]), atol=1e-13)
    for kind in ("fm", "spiral", "spiral_xy", "overhauser", "skx"):
        assert make_pin(kind, Q1, Q2, 1.0)(r).shape == (5, 3)
    with pytest.raises(ValueError):
        make_pin("stripes", Q1, Q2, 1.0)


def test_pins_have_magnitude_h_pin():
    """Skyrmion (m0 = 0.3, the default), FM and cycloidal-spiral fields are h_pin times a unit
    vector at any position (reference tests/test_nqs_production.py:47-60)."""
    from nqs.pinning import make_fm_pin, make_skx_pin, make_spiral_pin
    pts = torch.as_tensor(np.vstack([[1.3, -0.7], _points(20, 9)]))
    for pin in (make_skx_pin(Q1, Q2, 0.7), make_fm_pin(0.7), make_spiral_pin(Q1, 0.7)):
        n = np.linalg.norm(pin(pts).numpy(), axis=-1)
        assert np.abs(n - 0.7).max() < 1e-9
