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
