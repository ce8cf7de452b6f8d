"""train_minsr on the device (reference tests/test_nqs_minsr.py:64-76): perturbed backflow,
MinSR brings the energy back to E_gs."""
import numpy as np
import pytest

from helpers import build, perturb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_minsr_descends_to_Egs(precision):
    from nqs.minsr import train_minsr
    g, model = build(N=5, L=7.0, hz=0.5, embed=16, heads=4)
    params = perturb(model.init(0), 0.1, 7, only="backflow")
    params, hist = train_minsr(model, params, 7.0, 5, 3, m_star=1.0, lambda_r=1.0, h_z=0.5,
                               n_walkers=256, n_steps=80, lr=0.1, lam=1e-3, n_sweeps=8,
                               step_size=0.5, burn=40, log_every=0, precision=precision)
    E_final = float(np.mean(hist["E"][-5:]))
    assert E_final < g["E_gs"] + 1e-2, (E_final, g["E_gs"])
    assert E_final > g["E_gs"] - 2e-2
    assert hist["E"][0] > E_final


def test_adam_training_descends_to_Egs():
    """tests/test_nqs_train.py:36-72: Adam removes >= 95% of the perturbation's energy excess."""
    from nqs.local_energy import make_local_energy
    from nqs.psiformer import make_logpsi
    from nqs.sampler import run_chain, vmc_energy
    from nqs.train import train
    g, model = build(N=5, L=7.0, hz=0.5, embed=16, heads=4)
    params = perturb(model.init(0), 0.15, 2, only="backflow")

    def energy_now(p):
        lp = make_logpsi(model, p)
        R, S, _, _ = run_chain(lp, 7.0, 5, 7, n_walkers=256, n_sweeps=80, burn=80, step=0.5)
        return vmc_energy(make_local_energy(lp, 1.0, 1.0, 0.5), R, S)[0]

    E_init = energy_now(params)
    params, hist = train(model, params, 7.0, 5, 3, m_star=1.0, lambda_r=1.0, h_z=0.5,
                         n_walkers=256, n_steps=120, lr=3e-3, n_sweeps=8, step_size=0.5, burn=40,
                         log_every=0)
    E_final = energy_now(params)
    excess = E_init - g["E_gs"]
    assert excess > 1e-2
    assert E_final < E_init - 1e-3
    assert (E_final - g["E_gs"]) / excess < 0.05, (E_init, E_final, g["E_gs"])
    assert E_final > g["E_gs"] - 0.02


def test_checkpoint_resume_is_bit_identical(tmp_path):
    """Two VMC steps straight through equal one step, a checkpoint written to disk, a fresh
    iteration restored from it, and one more step (same theta, walkers and random stream)."""
    import torch
    from nqs.minsr import VMCIteration, load_checkpoint, save_checkpoint, real_ravel
    from nqs.sampler import init_walkers_uniform
    g, model = build(N=5, L=7.0, hz=0.5, embed=16, heads=4)
    theta, _ = real_ravel(perturb(model.init(0), 0.05, 8, only="backflow"))
    R0, S0 = init_walkers_uniform(5, 64, 5, 7.0)
    kw = dict(m_star=1.0, lambda_r=1.0, h_z=0.5, lr=0.05, lam=1e-3, n_sweeps=4, step_size=0.5,
              seed=11)
    a = VMCIteration(model, theta, R0, S0, **kw)
    a.step()
    save_checkpoint(tmp_path / "ck.npz", a)
    a.step()
    b = VMCIteration(model, theta, R0, S0, **kw)  # different state until restored
    b.load_state_dict(load_checkpoint(tmp_path / "ck.npz"))
    b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.theta, b.theta)
    assert torch.equal(a.R, b.R) and torch.equal(a.S, b.S)
    assert a.counter == b.counter
