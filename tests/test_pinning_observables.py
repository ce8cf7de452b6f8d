"""Pinning fields (reference src/nqs/pinning.py) and the texture diagnostics of the observables
module (src/nqs/observables.py:77-90, 123-130, 150-165) on the CPU: the vectorised package
versions against the per-point oracle, and the known answers of the reference's own test
(tests/test_nqs_observables.py:42-66: zero skyrmion number for a uniform texture, a nonzero
integer for the triple-Q field over one magnetic cell)."""
import numpy as np
import pytest
import torch

from oracle import observables_oracle as OO

QSTAR = 0.9548
Q1 = QSTAR * np.array([1.0, 0.0])
Q2 = QSTAR * np.array([-0.5, np.sqrt(3) / 2])
CELL = 2.0 * np.pi * np.linalg.inv(np.array([Q1, Q2]))  # one magnetic cell


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


def test_hf_texture_field_and_file(tmp_path):
    from nqs.pinning import load_hf_texture, make_hf_skx_pin
    rng = np.random.default_rng(4)
    keys = np.array([[0, 0], [1, 0], [0, 1], [-1, -1], [2, -1]])
    vals = rng.normal(size=(5, 3)) + 1j * rng.normal(size=(5, 3))
    path = tmp_path / "tex.npz"
    np.savez(path, q1=Q1, q2=Q2, s_keys=keys, s_vals=vals, BL=1.0, E_var=-0.5, q_star=QSTAR,
             e_per_cell=3.0)
    d = load_hf_texture(str(path))
    assert d["BL"] == 1.0 and d["e_per_cell"] == 3.0 and "n_keys" not in d
    f = make_hf_skx_pin(d["s_keys"], d["s_vals"], d["q1"], d["q2"], 0.9)
    _check(f, lambda r: OO.hf_field(r, keys, vals, Q1, Q2, 0.9), _points(30, 5))


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


def test_berg_luscher_matches_oracle():
    from nqs.observables import berg_luscher
    rng = np.random.default_rng(7)
    for shape in ((6, 6), (5, 7)):
        m = rng.normal(size=shape + (3,))
        assert abs(berg_luscher(m) - OO.berg_luscher(m)) < 1e-12
    up = np.zeros((16, 16, 3))
    up[..., 2] = 1.0
    assert abs(berg_luscher(up)) < 1e-12


def test_skyrmion_number_of_pinning_textures():
    """The triple-Q field over one magnetic cell has skyrmion number 1 (both chiralities of the
    in-plane part); single-Q, collinear and uniform textures have none."""
    from nqs.pinning import berg_luscher_realspace, make_pin
    for kind in ("skx", "skx_bloch"):
        Qn = berg_luscher_realspace(make_pin(kind, Q1, Q2, 1.0, m0=0.5), CELL, ngrid=30)
        assert abs(Qn - round(Qn)) < 0.05 and abs(Qn) > 0.5, (kind, Qn)
        m = make_pin(kind, Q1, Q2, 1.0, m0=0.5)
        f = (np.arange(30) + 0.5) / 30
        grid = np.stack(np.meshgrid(f, f, indexing="ij"), -1) @ CELL.T
        assert abs(OO.berg_luscher(m(torch.as_tensor(grid)).numpy()) - Qn) < 1e-9
    for kind in ("fm", "spiral", "spiral_xy", "overhauser"):
        assert abs(berg_luscher_realspace(make_pin(kind, Q1, Q2, 1.0), CELL, ngrid=30)) < 1e-9


def test_skx_arms():
    from nqs.observables import skx_arms
    G = skx_arms(Q1, Q2, nharm=2)
    assert G.shape == (13, 2) and np.all(G[0] == 0)
    q3 = -(Q1 + Q2)
    assert np.allclose(G[1:7], [Q1, -Q1, Q2, -Q2, q3, -q3])
    assert np.allclose(G[7:], 2 * np.array([Q1, -Q1, Q2, -Q2, q3, -q3]))


def test_slater_spin_density_matches_oracle():
    from nqs.observables import slater_spin_density
    rng = np.random.default_rng(8)
    A = np.array([[6.0, 1.0], [0.0, 5.0]])
    Gs = rng.normal(size=(7, 2))
    W = rng.normal(size=(3, 7, 2)) + 1j * rng.normal(size=(3, 7, 2))
    m = slater_spin_density(Gs, W, A, ngrid=5)
    f = (np.arange(5) + 0.5) / 5
    for i in range(5):
        for j in range(5):
            r = A @ np.array([f[i], f[j]])
            assert np.abs(m[i, j] - OO.slater_spin_density_at(r, Gs, W)).max() < 1e-11
    # spin-up orbitals only: m = (0, 0, density)
    Wu = W.copy()
    Wu[..., 1] = 0
    mu = slater_spin_density(Gs, Wu, A, ngrid=4)
    assert np.abs(mu[..., :2]).max() < 1e-12 and (mu[..., 2] > 0).all()


def test_pins_have_magnitude_h_pin():
    """Skyrmion (m0 = 0.3, the default), FM and cycloidal-spiral fields are h_pin times a unit
    vector at any position (reference tests/test_nqs_production.py:47-60)."""
    from nqs.pinning import berg_luscher_realspace, make_fm_pin, make_skx_pin, make_spiral_pin
    pts = torch.as_tensor(np.vstack([[1.3, -0.7], _points(20, 9)]))
    for pin in (make_skx_pin(Q1, Q2, 0.7), make_fm_pin(0.7), make_spiral_pin(Q1, 0.7)):
        n = np.linalg.norm(pin(pts).numpy(), axis=-1)
        assert np.abs(n - 0.7).max() < 1e-9
    assert abs(berg_luscher_realspace(make_skx_pin(Q1, Q2, 1.0, m0=0.3), CELL, ngrid=36)) > 0.5
