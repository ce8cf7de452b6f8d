"""VMC training with Adam (drop-in for src/nqs/train.py:28-96).

One step: n_sweeps Metropolis sweeps -> local energies -> the gradient of the reference's
surrogate loss 2 mean_w Re[conj(e_w - mean e) log psi_w] (train.py:53-59), taken by torch autograd
through the differentiable log psi of nqs.psiformer (forward nqs_logpsi, backward the hand-written
vector-Jacobian product nqs_logpsi_vjp, which never forms the per-sample Jacobian) -> the Adam
step of optax.adam as train.py applies it to jax.grad's tree: a complex leaf element moves as one
complex number with JAX's gradient dL/dRe - i dL/dIm, one complex first moment and one shared
second moment |G|^2 (nqs_adam_update_complex). Everything runs on the device.
"""
from __future__ import annotations

import torch

from . import _lib
from .minsr import real_ravel


def complex_partners(model):
    """int64[P]: for each component of a complex leaf element the theta index of the other
    component (re block k <-> im block k + n), -1 for a real parameter."""
    P = model.n_params()
    partner = torch.full((P,), -1, dtype=torch.int64)
    for _, shape, is_c, off in model.leaves():
        if is_c:
            n = 1
            for x in shape:
                n *= int(x)
            k = torch.arange(off, off + n, dtype=torch.int64)
            partner[k] = k + n
            partner[k + n] = k
    return partner


class Adam:
    """optax.adam on the real ravel: init(theta) -> state; update(grad, state, theta) applies the
    step in place. grad is the real-ravel gradient (dL/dRe, dL/dIm for complex leaves). With a
    model (partner table from complex_partners) complex leaf elements take optax's complex step;
    without one every component is a real parameter."""

    def __init__(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, model=None):
        self.lr, self.b1, self.b2, self.eps = float(lr), float(b1), float(b2), float(eps)
        self.model = model

    def init(self, theta):
        st = {"m": torch.zeros_like(theta), "v": torch.zeros_like(theta), "t": 0}
        if self.model is not None:
            st["partner"] = complex_partners(self.model).to(theta.device)
        return st

    def update(self, grad, state, theta):
        state["t"] += 1
        if "partner" in state:
            _lib.check(_lib.lib().nqs_adam_update_complex(
                _lib.ptr(theta), _lib.ptr(grad), _lib.ptr(state["m"]), _lib.ptr(state["v"]),
                _lib.ptr(state["partner"]), theta.numel(), self.lr, self.b1, self.b2, self.eps,
                state["t"], _lib.stream_ptr()), "nqs_adam_update_complex")
        else:
            _lib.check(_lib.lib().nqs_adam_update(
                _lib.ptr(theta), _lib.ptr(grad), _lib.ptr(state["m"]), _lib.ptr(state["v"]),
                theta.numel(), self.lr, self.b1, self.b2, self.eps, state["t"],
                _lib.stream_ptr()), "nqs_adam_update")
        return state


def adam(lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, model=None):
    return Adam(lr, b1, b2, eps, model)


def surrogate_gradient(model, theta, R, S, e, precision="fp64"):
    """d/dtheta of the reference's surrogate 2 mean_w Re[conj(e_w - mean e) log psi_theta(R_w,
    S_w)] (train.py:53-59) by torch autograd through the differentiable log psi (backward =
    nqs_logpsi_vjp). Returns the real-ravel gradient float64[P]."""
    from .psiformer import LogPsi
    th = theta.detach().requires_grad_(True)
    with torch.enable_grad():
        lp = LogPsi(model, th, precision)(R, S)
        ec = torch.conj(e - e.mean()).detach()
        loss = 2.0 * torch.real(ec * lp).mean()
        (g,) = torch.autograd.grad(loss, th)
    return g


def make_train_step(model, L, n_elec, m_star=1.0, lambda_r=1.0, h_z=0.0, coulomb=None,
                    optimizer=None, n_sweeps=10, step_size=0.4, n_spin_flips=2):
    """Return (optimizer, step(theta, opt_state, R, S, key)) (train.py:28-65). theta is the real
    ravel on the device and is updated in place; returns
    (theta, opt_state, R, S, E, Eerr, acc_pos, acc_spin). The default optimizer is optax.adam(1e-3)
    with the complex-leaf treatment of the reference."""
    from .minsr import VMCIteration
    from .random import as_key, key_to_seed
    optimizer = optimizer or adam(1e-3, model=model)
    cache = {}

    def step(theta, opt_state, R, S, key):
        s, c = as_key(key)
        it = cache.get("it")
        if it is None or it.W != torch.as_tensor(S).shape[0]:
            it = VMCIteration(model, theta, R, S, m_star=m_star, lambda_r=lambda_r, h_z=h_z,
                              coulomb=coulomb, n_sweeps=n_sweeps, step_size=step_size,
                              n_spin_flips=n_spin_flips, precision="fp64")
            cache["it"] = it
        it.theta = theta
        it.R.copy_(torch.as_tensor(R))
        it.S.copy_(torch.as_tensor(S))
        it.seed, it.counter = key_to_seed((s, 0)), c
        it.sample()
        it.energies()
        g = surrogate_gradient(model, theta, it.R, it.S, it.e)
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
                                      optimizer or adam(lr, model=model), n_sweeps, step_size)
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
