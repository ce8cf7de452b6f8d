"""The host-side Rashba setup (nqs.rashba) on the analytic checks the reference applies to its own
module (tests/test_nqs_rashba_reference.py:14-76): eigensolver bands against the closed form,
the Hamiltonian's SOC convention, the h_z = 0 ring minimum, the ground state as the sum of the
lowest levels with a closed shell, occupied spinors as normalised eigenstates, and cutoff
convergence. CPU only."""
import numpy as np

from nqs import rashba

SX = np.array([[0, 1], [1, 0]], dtype=complex)
SY = np.array([[0, -1j], [1j, 0]], dtype=complex)
SZ = np.array([[1, 0], [0, -1]], dtype=complex)


def test_eigensolver_bands_equal_closed_form():
    rng = np.random.default_rng(21)
    for _ in range(60):
        kx, ky = 2.0 * rng.normal(size=2)
        ms, lr, hz = rng.uniform(0.3, 2.0), rng.uniform(0.0, 3.0), rng.uniform(0.0, 1.0)
        lo, up, _, _ = rashba.bands_k(kx, ky, ms, lr, hz)
        alo, aup = rashba.bands_analytic(kx, ky, ms, lr, hz)
        assert abs(lo - alo) < 1e-10 and abs(up - aup) < 1e-10


def test_h0_hermitian_with_the_reference_soc_convention():
    kx, ky, lr, hz = 0.7, -1.3, 1.1, 0.4
    H = rashba.h0_k(kx, ky, 1.0, lr, hz)
    assert np.allclose(H, H.conj().T)
    soc = H - 0.5 * (kx * kx + ky * ky) * np.eye(2) + 0.5 * hz * SZ
    assert np.allclose(soc, lr * (SX * ky + SY * kx))  # lambda_R (sigma_x k_y + sigma_y k_x)


def test_ground_state_is_the_lowest_levels_and_closed():
    g = rashba.noninteracting_gs(N=7, L=8.0, m_star=1.0, lambda_r=1.0, h_z=0.5, n_cut=10,
                                 twist=(0.1, 0.17))
    assert g["gap"] > 1e-6 and g["cutoff_ok"]
    E = sorted(d["E"] for d in rashba.single_particle_levels(8.0, 1.0, 1.0, 0.5, 10, (0.1, 0.17)))
    assert abs(g["E_gs"] - sum(E[:7])) < 1e-12


def test_occupied_spinors_are_normalised_eigenstates():
    g = rashba.noninteracting_gs(N=9, L=9.0, m_star=1.0, lambda_r=1.0, h_z=0.5, n_cut=10,
                                 twist=(0.07, 0.13))
    K, Chi = rashba.occupied_orbital_matrix(g)
    assert K.shape == (9, 2) and Chi.shape == (9, 2)
    for k, chi in zip(K, Chi):
        assert abs(np.vdot(chi, chi) - 1.0) < 1e-10
        Hc = rashba.h0_k(k[0], k[1], 1.0, 1.0, 0.5) @ chi
        assert np.allclose(Hc, np.vdot(chi, Hc) * chi, atol=1e-9)


def test_ground_state_converged_in_the_cutoff():
    kw = dict(N=11, L=10.0, m_star=1.0, lambda_r=1.0, h_z=0.5, twist=(0.1, 0.2))
    assert abs(rashba.noninteracting_gs(n_cut=8, **kw)["E_gs"]
               - rashba.noninteracting_gs(n_cut=12, **kw)["E_gs"]) < 1e-12
