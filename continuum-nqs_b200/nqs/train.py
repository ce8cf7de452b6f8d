"""VMC training with Adam (drop-in for src/nqs/train.py:28-96).

One step: n_sweeps Metropolis sweeps -> local energies -> the surrogate-loss gradient
g = 2 mean_w Re[conj(e_w - mean e) d log psi_w / d theta] -> an Adam update, all on the device.
The gradient is the per-sample Jacobian contracted with the centred energies (nqs_energy_gradient),
so it is exactly the derivative of the reference's surrogate with respect to the REAL ravel theta.
(For complex leaves JAX's grad returns d/dRe - i d/dIm and optax's Adam then keeps one second
moment per complex element; here every real component has its own moment — stated difference.)
"""
from __future__ import annotations

import torch

from . import _lib
from .minsr import real_ravel


class Adam:
    """optax.adam-like: init(theta) -> state; update(grad, state, theta) applies the step."""

    def __init__(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = float(lr), float(b1), float(b2), float(eps)

    def init(self, theta):
        return {"m": torch.zeros_like(theta), "v": torch.zeros_like(theta), "t": 0}

    def update(self, grad, state, theta):
        state["t"] += 1
        _lib.check(_lib.lib().nqs_adam_update(
            _lib.ptr(theta), _lib.ptr(grad), _lib.ptr(state["m"]), _lib.ptr(state["v"]),
            theta.numel(), self.lr, self.b1, self.b2, self.eps, state["t"], _lib.stream_ptr()),
            "nqs_adam_update")
        return state


def adam(lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    return Adam(lr, b1, b2, eps)


def make_train_step(model, L, n_elec, m_star=1.0, lambda_r=1.0, h_z=0.0, coulomb=None,
                    optimizer=None, n_sweeps=10, step_size=0.4, n_spin_flips=2):
    """Return (optimizer, step(theta, opt_state, R, S, key)) (train.py:28-65). theta is the real
    ravel on the device and is updated in place; returns
    (theta, opt_state, R, S, E, Eerr, acc_pos, acc_spin)."""
    from .minsr import VMCIteration
    from .random import as_key, key_to_seed
    optimizer = optimizer or adam(1e-3)
    cache = {}

    def step(theta, opt_state, R, S, key):
        s, c = as_key(key)
        it = cache.get("it")
        if it is None or it.W != torch.as_tensor(S).shape[0]:
            it = VMCIteration(model, theta, R, S, m_star=m_star, lambda_r=lambda_r, h_z=h_z,
                              coulomb=coulomb, n_sweeps=n_sweeps, step_size=step_size,
                              n_spin_flips=n_spin_flips, precision="fp64")
            cache["it"] = it
            cache["g"] = torch.empty_like(it.theta)
        it.theta = theta
        it.R.copy_(torch.as_tensor(R))
        it.S.copy_(torch.as_tensor(S))
        it.seed, it.counter = key_to_seed((s, 0)), c
        it.sample()
        it.energies()
        it.jacobian()
        g = cache["g"]
        ws = _lib.workspace.get(16 * it.W + 4096)
        _lib.check(_lib.lib().nqs_energy_gradient(
            _lib.ptr(it.O), 0, _lib.ptr(it.e), it.W, it.P, _lib.ptr(g), _lib.ptr(ws), ws.numel(),
            _lib.stream_ptr()), "nqs_energy_gradient")
        opt_state = optimizer.update(g, opt_state, theta)
        er = it.e.real
        return (theta, opt_state, it.R, it.S, er.mean(), er.std(unbiased=False) / it.W ** 0.5,
                it.acc_pos.mean(), it.acc_spin.mean())

    return optimizer, step


def init_walkers(key, n_walkers, n_elec, L):
    from .sampler import init_walkers_uniform
    return init_walkers_uniform(key, n_walkers, n_elec, L)


def train(model, params, L, n_elec, key, *, m_star=1.0, lambda_r=1.0, h_z=0.0, coulomb=None,
          n_walkers=256, n_steps=200, lr=1e-3, n_sweeps=10, step_size=0.4, burn=50,
          optimizer=None, log_every=20, history=None):
    """Run VMC training with Adam; return (params, history) (train.py:75-96)."""
    from .random import as_key, fold_in, split
    optimizer, step = make_train_step(model, L, n_elec, m_star, lambda_r, h_z, coulomb,
                                      optimizer or adam(lr), n_sweeps, step_size)
    theta, unravel = real_ravel(params)
    theta = theta.to(_lib.device()).contiguous()
    opt_state = optimizer.init(theta)
    kw, ks = split(as_key(key), 2)
    R, S = init_walkers(kw, n_walkers, n_elec, L)
    # burn-in at the initial parameters: sweeps only (the reference discards these updates)
    from .minsr import VMCIteration
    it = VMCIteration(model, theta, R, S, m_star=m_star, lambda_r=lambda_r, h_z=h_z,
                      n_sweeps=n_sweeps, step_size=step_size)
    it.sample((burn // n_sweeps + 1) * n_sweeps)
    R, S = it.R, it.S
    hist = history if history is not None else {"E": [], "Eerr": [], "acc_pos": []}
    for i in range(n_steps):
        theta, opt_state, R, S, E, Eerr, ap, asp = step(theta, opt_state, R, S,
                                                        fold_in(ks, 1000 + i))
        hist["E"].append(float(E))
        hist["Eerr"].append(float(Eerr))
        hist["acc_pos"].append(float(ap))
        if log_every and (i % log_every == 0 or i == n_steps - 1):
            print(f"    step {i:4d}: E={float(E):+.6f} +/- {float(Eerr):.1e}  "
                  f"acc_pos={float(ap):.2f} acc_spin={float(asp):.2f}", flush=True)
    return unravel(theta.cpu()), hist
