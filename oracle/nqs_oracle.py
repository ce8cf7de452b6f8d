"""FP64 CPU oracle for the VMC iteration — TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it. The CUDA product
path never calls into it and fails loudly when its extension is missing.

It restates, in plain torch float64/complex128 on the CPU, the reference algorithm of
wenqin-chen/continuum-nqs (a JAX/Flax package that cannot be imported here: jax, flax, optax and
folx are absent). Each function cites the reference file:line it follows. Derivatives use
``torch.func`` (reverse mode for gradients and per-sample Jacobians, forward-over-reverse for the
dense Hessian) exactly where the reference uses ``jax.grad`` / ``jax.hessian``.

Parity pinning: the reference ships no stored golden vectors for this path. The oracle is pinned
by (i) the reference's own pure-numpy module ``rashba_reference.py`` (imported in the build
container; its outputs are committed as ``tests/golden/rashba_gs.npz``), and (ii) the reference's
analytic known-answer tests re-expressed against this oracle: zero-variance E_loc = E_gs,
the Zeeman-polarised limit, antisymmetry, Ewald eta-independence / periodicity / alpha scaling /
1/r limit, and MinSR == parameter-space SR. Quantities that only an actual JAX run would fix
(threefry random streams, flax's LayerNorm variance formula, JAX's erfc rounding) are
"parity unpinned" and are stated as such in the tests that touch them.
"""
from __future__ import annotations

import math
from typing import Any, Callable

import numpy as np
import torch
from scipy.special import erfc as _erfc_np
from torch.func import grad, hessian, jacrev, vmap

F64 = torch.float64
C128 = torch.complex128


# ----------------------------------------------------------------------------------------------
# cell helpers  (reference: src/nqs/cell.py:21-53, src/nqs/sampler.py:19-22)
# ----------------------------------------------------------------------------------------------
def cell_matrix(cell) -> np.ndarray:
    """Scalar L -> L*I; 2x2 A (columns = lattice vectors) passes through (cell.py:21-32)."""
    if np.ndim(cell) == 0:
        return np.array([[float(cell), 0.0], [0.0, float(cell)]])
    return np.asarray(cell, dtype=float)


def _t(x, dtype=F64):
    if isinstance(x, torch.Tensor):
        return x.detach().to("cpu", dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype)


# ----------------------------------------------------------------------------------------------
# wavefunction  (reference: src/nqs/psiformer.py:38-196)
# ----------------------------------------------------------------------------------------------
def periodic_features(R, A, n_freq):
    """psiformer.py:84-97 — s = R A^-T (no mod); per electron [x: sin m=1..nf, cos m=1..nf,
    y: sin m=1..nf, cos m=1..nf]."""
    Ainv = torch.linalg.inv(_t(A))
    s = R @ Ainv.T
    ph = 2.0 * math.pi * s
    m = torch.arange(1, n_freq + 1, dtype=F64)
    ang = ph[:, :, None] * m[None, None, :]
    feats = torch.cat([torch.sin(ang), torch.cos(ang)], dim=-1)
    return feats.reshape(R.shape[0], -1)


def layer_norm(x, p, eps=1e-6):
    """flax.linen.LayerNorm defaults (epsilon 1e-6, scale and bias). Two-pass variance; flax's
    fast-variance form E[x^2]-E[x]^2 agrees to rounding (parity unpinned at the ulp level)."""
    mu = x.mean(-1, keepdim=True)
    u = x - mu
    var = (u * u).mean(-1, keepdim=True)
    return u / torch.sqrt(var + eps) * p["scale"] + p["bias"]


def gelu_tanh(x):
    """jax.nn.gelu default (approximate=True): 0.5 x (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))."""
    return 0.5 * x * (1.0 + torch.tanh(math.sqrt(2.0 / math.pi) * (x + 0.044715 * x ** 3)))


# Emulation hook for tests of the tensor-core precisions: when set to a function f, the operands
# of every Dense product whose K (input width) is a multiple of 64, and of the backflow product,
# become f(x) and f(kernel) (e.g. rounding to BF16); the products themselves stay float64.
OPERAND_ROUND: Callable | None = None


def dense(x, p):
    if OPERAND_ROUND is not None and x.shape[-1] % 64 == 0:
        return OPERAND_ROUND(x) @ OPERAND_ROUND(p["kernel"]) + p["bias"]
    return x @ p["kernel"] + p["bias"]


def mha(x, p, n_heads):
    """psiformer.py:50-64 — q,k,v Dense(d); softmax(QK^T/sqrt(hd)) over keys; merge; Dense o."""
    N, d = x.shape
    hd = d // n_heads

    def split(t):
        return t.reshape(N, n_heads, hd).permute(1, 0, 2)

    Q, K, V = split(dense(x, p["q"])), split(dense(x, p["k"])), split(dense(x, p["v"]))
    att = torch.softmax(torch.einsum("hid,hjd->hij", Q, K) / math.sqrt(hd), dim=-1)
    out = torch.einsum("hij,hjd->hid", att, V).permute(1, 0, 2).reshape(N, d)
    return dense(out, p["o"])


def transformer_block(x, p, n_heads):
    """psiformer.py:67-81 — pre-norm MHA and GELU MLP, both residual."""
    x = x + mha(layer_norm(x, p["LayerNorm_0"]), p["attn"], n_heads)
    h = layer_norm(x, p["LayerNorm_1"])
    h = gelu_tanh(dense(h, p["Dense_0"]))
    return x + dense(h, p["Dense_1"])


def complex_logsumexp(z):
    """jax.scipy.special.logsumexp on a complex vector: shift by max Re, principal log."""
    amax = torch.max(z.real).detach()
    return torch.log(torch.sum(torch.exp(z - amax))) + amax


def logpsi(spec, params, R, S):
    """ContinuumSpinorPsiformer.__call__ (psiformer.py:118-189) for ONE configuration.

    R (N,2) float64, S (N,) int -> complex128 scalar log psi."""
    p = params["params"] if "params" in params else params
    N = spec.n_elec
    A = cell_matrix(spec.L)
    Gs = _t(spec.Gs)
    W = _t(spec.W, C128)
    if spec.learnable_env:
        W = W + p["dW"]
    pos = periodic_features(R, A, spec.n_freq)
    spin = torch.nn.functional.one_hot(S.long(), 2).to(F64)
    x = dense(torch.cat([pos, spin], dim=-1), p["embed"])
    for b in range(spec.depth):
        x = transformer_block(x, p[f"TransformerBlock_{b}"], spec.n_heads)
    x = layer_norm(x, p["LayerNorm_0"])
    if OPERAND_ROUND is not None and x.shape[-1] % 64 == 0:
        kb = p["backflow"]["kernel"]
        kr = torch.complex(OPERAND_ROUND(kb.real), OPERAND_ROUND(kb.imag))
        bf = OPERAND_ROUND(x).to(C128) @ kr + p["backflow"]["bias"]
    else:
        bf = x.to(C128) @ p["backflow"]["kernel"] + p["backflow"]["bias"]  # (N, K*N)
    bf = bf.reshape(N, spec.n_dets, N).permute(1, 2, 0)                  # (K, n_orb, N)
    phase = torch.exp(1j * (Gs @ R.T))                                    # (n_G, N)
    Ws = W[:, :, S.long()]                                                # (n_orb, n_G, N)
    env = torch.einsum("gi,agi->ai", phase, Ws)
    M = env[None] * (1.0 + bf)
    sign, logabs = torch.linalg.slogdet(M)
    logdets = logabs + torch.log(sign)
    if spec.n_dets == 1:
        lp = logdets[0]
    else:
        lp = complex_logsumexp(logdets + p["det_logw"])
    if spec.use_jastrow:
        lp = lp + jastrow(spec, p, R, S).to(C128)
    return lp


def jastrow(spec, p, R, S):
    """psiformer.py:162-188 — minimum-image pair Jastrow, rbf or cusp form, summed over i<j."""
    A = _t(cell_matrix(spec.L))
    Ainv = torch.linalg.inv(A)
    N = spec.n_elec
    d = R[:, None, :] - R[None, :, :]
    dfrac = d @ Ainv.T
    dmin = (dfrac - torch.round(dfrac)) @ A.T
    r = torch.sqrt(torch.sum(dmin * dmin, -1) + 1e-12)
    same = S[:, None] == S[None, :]
    if spec.jastrow_kind == "rbf":
        area = float(abs(np.linalg.det(cell_matrix(spec.L))))
        rcut = 0.5 * math.sqrt(area)
        mu = torch.as_tensor(np.linspace(0.0, rcut, spec.n_knots), dtype=F64)
        wdt = rcut / max(spec.n_knots - 1, 1)
        rbf = torch.exp(-(((r[..., None] - mu) / wdt) ** 2))
        uij = torch.where(same, (rbf * p["jas_c_same"]).sum(-1), (rbf * p["jas_c_opp"]).sum(-1))
    else:
        a = torch.nn.functional.softplus(p["jastrow_loga"]) + 0.05
        alpha = torch.where(same, torch.full_like(r, spec.cusp / 3.0), torch.full_like(r, spec.cusp))
        uij = alpha * a * (1.0 - torch.exp(-r / a))
    iu = torch.triu_indices(N, N, 1)
    return torch.sum(uij[iu[0], iu[1]])


def slater_logpsi(Gs, W, R, S):
    """slater_reference.py:21-35 — general multi-G spinor determinant."""
    Gs = _t(Gs)
    W = _t(W, C128)
    phase = torch.exp(1j * (Gs @ R.T))
    M = torch.einsum("gi,agi->ai", phase, W[:, :, S.long()])
    sign, logabs = torch.linalg.slogdet(M)
    return logabs + torch.log(sign)


# ----------------------------------------------------------------------------------------------
# local energy  (reference: src/nqs/local_energy.py:40-117, dense-Hessian default path)
# ----------------------------------------------------------------------------------------------
def local_energy(lp: Callable, R, S, m_star=1.0, lambda_r=1.0, h_z=0.0, ext_field=None):
    """E_loc(R,S) for a single configuration with a dense Hessian kinetic term
    (local_energy.py:63-115). lp(R,S) -> complex. ext_field(r) -> (3,) real (one position) adds
    -sum_i f_z (sigma_z)_{s_i s_i} - sum_i [f_x sigma_x + f_y sigma_y]_{s_i s'} ratio_i
    (local_energy.py:86-88,109-111)."""
    N = R.shape[0]
    rf = R.reshape(-1)

    def Lr(rf_, S_):
        return lp(rf_.reshape(N, 2), S_).real

    def Li(rf_, S_):
        return lp(rf_.reshape(N, 2), S_).imag

    L0 = lp(R, S)
    g = grad(Lr)(rf, S) + 1j * grad(Li)(rf, S)
    lap = torch.trace(hessian(Lr)(rf, S)) + 1j * torch.trace(hessian(Li)(rf, S))
    E_kin = -1.0 / (2.0 * m_star) * (lap + torch.sum(g * g))
    sgn = 1.0 - 2.0 * S.to(F64)
    E_Z = -0.5 * h_z * torch.sum(sgn)
    fields = None
    if ext_field is not None:
        fields = [torch.as_tensor(ext_field(R[i]), dtype=F64) for i in range(N)]
        E_Z = E_Z - sum(float(fields[i][2]) * float(sgn[i]) for i in range(N))
    E_soc = torch.zeros((), dtype=C128)
    for i in range(N):
        s_i = int(S[i])
        s_p = 1 - s_i
        Sf = S.clone()
        Sf[i] = s_p
        Lf = lp(R, Sf)
        if not torch.isfinite(Lf.real):
            # exactly singular flipped determinant: Psi(s') = 0, the reference's guarded
            # ratio * gradient is 0 (local_energy.py:99-105); so is the field term
            continue
        ratio = torch.exp(Lf - L0)
        if fields is not None:
            sy_f = -1j if s_i == 0 else 1j
            E_soc = E_soc - (float(fields[i][0]) + float(fields[i][1]) * sy_f) * ratio
        gf = grad(Lr)(rf, Sf) + 1j * grad(Li)(rf, Sf)
        ampgx = ratio * gf[2 * i]
        ampgy = ratio * gf[2 * i + 1]
        if not torch.isfinite(ampgx.real) or not torch.isfinite(ampgx.imag):
            ampgx = torch.zeros((), dtype=C128)
        if not torch.isfinite(ampgy.real) or not torch.isfinite(ampgy.imag):
            ampgy = torch.zeros((), dtype=C128)
        sx = 1.0 + 0j                                   # (sigma_x)_{s,1-s} = 1
        sy = -1j if s_i == 0 else 1j                    # (sigma_y)_{0,1} = -i, _{1,0} = +i
        E_soc = E_soc + lambda_r * (sx * (-1j) * ampgy + sy * (-1j) * ampgx)
    return E_kin + E_Z + E_soc


def grad_and_lap(lp: Callable, R, S):
    """(log psi, complex gradient (2N,), complex Laplacian) via the dense Hessian."""
    N = R.shape[0]
    rf = R.reshape(-1)

    def Lr(rf_):
        return lp(rf_.reshape(N, 2), S).real

    def Li(rf_):
        return lp(rf_.reshape(N, 2), S).imag

    g = grad(Lr)(rf) + 1j * grad(Li)(rf)
    lap = torch.trace(hessian(Lr)(rf)) + 1j * torch.trace(hessian(Li)(rf))
    return lp(R, S), g, lap


# ----------------------------------------------------------------------------------------------
# Ewald  (reference: src/nqs/ewald.py:26-73)
# ----------------------------------------------------------------------------------------------
class Ewald:
    """make_ewald_lattice (ewald.py:26-67): images A n, |n_x|,|n_y| <= n_real; G = B m over the
    square index box |m_x|,|m_y| <= n_recip, m != 0; RECIP = (2 pi/area) erfc(|G|/2eta)/|G|."""

    def __init__(self, A, alpha=1.0, ewald_alpha=None, n_real=5, n_recip=10):
        A = cell_matrix(A)
        self.A = A
        self.area = float(abs(np.linalg.det(A)))
        B = 2.0 * np.pi * np.linalg.inv(A).T
        self.eta = (float(np.sqrt(np.pi) / np.sqrt(self.area)) if ewald_alpha is None
                    else float(ewald_alpha))
        self.alpha = float(alpha)
        nx, ny = np.meshgrid(np.arange(-n_real, n_real + 1), np.arange(-n_real, n_real + 1),
                             indexing="ij")
        cells = np.stack([nx.ravel(), ny.ravel()], -1).astype(float)
        self.R_lat = cells @ A.T
        mx, my = np.meshgrid(np.arange(-n_recip, n_recip + 1), np.arange(-n_recip, n_recip + 1),
                             indexing="ij")
        mc = np.stack([mx.ravel(), my.ravel()], -1).astype(float)
        keep = (mc[:, 0] ** 2 + mc[:, 1] ** 2) > 0
        self.G = mc[keep] @ B.T
        Gm = np.linalg.norm(self.G, axis=-1)
        self.RECIP = (2.0 * np.pi / self.area) * _erfc_np(Gm / (2.0 * self.eta)) / Gm
        self.V_G0 = -2.0 * np.sqrt(np.pi) / (self.area * self.eta)
        Rs = np.linalg.norm(self.R_lat, axis=-1)
        real_nz = float(sum(_erfc_np(self.eta * d) / d for d in Rs if d > 1e-10))
        V_self = -2.0 * self.eta / np.sqrt(np.pi)
        self.zeta_M = float(self.alpha * (real_nz + V_self + float(np.sum(self.RECIP)) + self.V_G0))

    def pair(self, r):
        """ewald_pair (ewald.py:47-51) for r (2,) or (M,2) -> float64."""
        r = np.asarray(r, dtype=float)
        single = r.ndim == 1
        r = np.atleast_2d(r)
        d = np.linalg.norm(r[:, None, :] + self.R_lat[None], axis=-1)
        V_real = np.sum(_erfc_np(self.eta * d) / d, axis=-1)
        V_rec = np.sum(self.RECIP[None] * np.cos(r @ self.G.T), axis=-1)
        out = self.alpha * (V_real + V_rec + self.V_G0)
        return out[0] if single else out

    def energy(self, R):
        """coulomb_energy (ewald.py:60-65): sum_{i<j} ewald_pair(r_i - r_j) + N zeta_M / 2."""
        R = np.asarray(R, dtype=float)
        if R.ndim == 3:
            return np.array([self.energy(x) for x in R])
        N = R.shape[0]
        iu = np.triu_indices(N, 1)
        dr = (R[:, None, :] - R[None, :, :])[iu]
        return float(np.sum(self.pair(dr)) + N * self.zeta_M / 2.0)


# ----------------------------------------------------------------------------------------------
# Metropolis sweep with injected randomness  (reference: src/nqs/sampler.py:25-59)
# ----------------------------------------------------------------------------------------------
def wrap(R, A):
    """sampler.py:30-31 — mod(r A^-T, 1) A^T."""
    At = _t(cell_matrix(A))
    Ainv = torch.linalg.inv(At)
    return torch.remainder(R @ Ainv.T, 1.0) @ At.T


def mcmc_sweep(lp: Callable, A, R, S, step, normals, u_pos, flip_idx, u_flip, L_cur=None):
    """One sweep for ONE walker with the proposal normals / uniforms / flip indices given.

    Accept rule (sampler.py:39-53): d = 2 Re L' - 2 Re L; accept iff u < exp(min(0, d)).
    Returns (R, S, acc_pos, n_acc_spin, L_cur, d_values) where d_values lists every d."""
    if L_cur is None:
        L_cur = lp(R, S)
    ds = []
    Rp = wrap(R + step * normals, A)
    Lp = lp(Rp, S)
    d = 2.0 * Lp.real - 2.0 * L_cur.real
    ds.append(float(d))
    acc = bool(u_pos < math.exp(min(0.0, float(d))))
    if acc:
        R, L_cur = Rp, Lp
    nacc = 0
    for j in range(len(flip_idx)):
        i = int(flip_idx[j])
        Sp = S.clone()
        Sp[i] = 1 - Sp[i]
        Lp = lp(R, Sp)
        d = 2.0 * Lp.real - 2.0 * L_cur.real
        ds.append(float(d))
        a = bool(u_flip[j] < math.exp(min(0.0, float(d))))
        if a:
            S, L_cur = Sp, Lp
            nacc += 1
    return R, S, acc, nacc, L_cur, ds


# ----------------------------------------------------------------------------------------------
# parameter layout, per-sample Jacobian and MinSR  (reference: src/nqs/minsr.py:30-88)
# ----------------------------------------------------------------------------------------------
def flatten_sorted(tree, prefix=()):
    """JAX pytree flatten order for nested dicts: keys sorted; returns [(path, leaf)]."""
    out = []
    for k in sorted(tree.keys()):
        v = tree[k]
        if isinstance(v, dict):
            out.extend(flatten_sorted(v, prefix + (k,)))
        else:
            out.append((prefix + (k,), v))
    return out


def real_ravel(params):
    """minsr.py:30-53 — complex leaf -> [re.ravel(), im.ravel()]; returns (theta, unravel)."""
    leaves = flatten_sorted(params)
    specs, flats = [], []
    for path, l in leaves:
        l = torch.as_tensor(l)
        if l.is_complex():
            specs.append((path, True, tuple(l.shape), l.numel()))
            flats += [l.real.reshape(-1).to(F64), l.imag.reshape(-1).to(F64)]
        else:
            specs.append((path, False, tuple(l.shape), l.numel()))
            flats.append(l.reshape(-1).to(F64))
    theta = torch.cat(flats)

    def unravel(v):
        out: dict = {}
        i = 0
        for path, is_c, shape, size in specs:
            if is_c:
                leaf = torch.complex(v[i:i + size], v[i + size:i + 2 * size]).reshape(shape)
                i += 2 * size
            else:
                leaf = v[i:i + size].reshape(shape)
                i += size
            node = out
            for k in path[:-1]:
                node = node.setdefault(k, {})
            node[path[-1]] = leaf
        return out

    return theta, unravel


def per_sample_O(spec, theta, unravel, R, S):
    """minsr.py:56-65 — O[s,k] = d Re L/d theta_k + i d Im L/d theta_k, (W, P) complex."""
    def lr(t, r, s):
        return logpsi(spec, unravel(t), r, s).real

    def li(t, r, s):
        return logpsi(spec, unravel(t), r, s).imag

    rows = []
    for w in range(R.shape[0]):
        rows.append(grad(lr)(theta, R[w], S[w]) + 1j * grad(li)(theta, R[w], S[w]))
    return torch.stack(rows)


def otil_etil(O, eps):
    """minsr.py:68-73 — centre, stack [Re; Im] (no 1/sqrt(W) scaling)."""
    dO = O - O.mean(0, keepdim=True)
    Otil = torch.cat([dO.real, dO.imag], 0)
    ec = eps - eps.mean()
    etil = torch.cat([ec.real, ec.imag])
    return Otil, etil


def minsr_direction(O, eps, lam):
    """minsr.py:76-81 — dtheta = Otil^T (Otil Otil^T + lam I)^-1 etil (LU solve)."""
    Otil, etil = otil_etil(O, eps)
    T = Otil @ Otil.T
    y = torch.linalg.solve(T + lam * torch.eye(T.shape[0], dtype=F64), etil)
    return Otil.T @ y


def paramsr_direction(O, eps, lam):
    """minsr.py:84-88 — the explicit P x P solve."""
    Otil, etil = otil_etil(O, eps)
    P = Otil.shape[1]
    return torch.linalg.solve(Otil.T @ Otil + lam * torch.eye(P, dtype=F64), Otil.T @ etil)


def _median(x):
    """jnp.median: midpoint of the two middle order statistics for an even count."""
    v, _ = torch.sort(x)
    n = v.numel()
    return v[n // 2] if n % 2 == 1 else 0.5 * (v[n // 2 - 1] + v[n // 2])


def clip_energies(e, clip_k):
    """minsr.py:145-148 — median-MAD clip of Re e (gradient only); Im kept."""
    e_re = e.real
    med = _median(e_re)
    mad = _median(torch.abs(e_re - med)) + 1e-12
    return torch.clamp(e_re, med - clip_k * mad, med + clip_k * mad) + 1j * e.imag


# ----------------------------------------------------------------------------------------------
# one VMC iteration on CPU (the timed CPU baseline): minsr.py:139-156 with injected randomness
# ----------------------------------------------------------------------------------------------
def vmc_iteration(spec, theta, unravel, R, S, *, A, step, n_sweeps, n_spin_flips, rng,
                  m_star, lambda_r, h_z, ewald: Ewald | None, lam, lr, clip_k,
                  n_walkers_elocal=None, draws=None):
    """Sample (n_sweeps Metropolis sweeps), E_loc (dense Hessian), O (reverse mode), clip,
    MinSR direction, update. `rng` is a numpy Generator supplying the proposals, or `draws` the
    pre-drawn randomness in the device's injected layout (normals [n_sweeps][W][N][2], position
    uniforms [n_sweeps][W], flip indices and flip uniforms [n_sweeps][n_spin_flips][W]). When
    `n_walkers_elocal` is given only that many walkers enter E_loc / O / MinSR (a bounded
    sample for timing)."""
    params = unravel(theta)
    lp = lambda r, s: logpsi(spec, params, r, s)  # noqa: E731
    Wn, N = S.shape
    for sw in range(n_sweeps):
        for w in range(Wn):
            if draws is None:
                nrm, up = torch.as_tensor(rng.standard_normal((N, 2))), rng.uniform()
                fi, uf = rng.integers(0, N, n_spin_flips), rng.uniform(size=n_spin_flips)
            else:
                nrm, up = torch.as_tensor(draws[0][sw, w]), float(draws[1][sw, w])
                fi, uf = draws[2][sw, :, w], draws[3][sw, :, w]
            R[w], S[w], *_ = mcmc_sweep(lp, A, R[w], S[w], step, nrm, up, fi, uf)
    Wm = Wn if n_walkers_elocal is None else n_walkers_elocal
    e = torch.stack([local_energy(lp, R[w], S[w], m_star, lambda_r, h_z) for w in range(Wm)])
    if ewald is not None:
        e = e + torch.as_tensor(ewald.energy(R[:Wm].numpy()))
    O = per_sample_O(spec, theta, unravel, R[:Wm], S[:Wm])
    d = minsr_direction(O, clip_energies(e, clip_k), lam)
    return theta - lr * d, R, S, e


# ----------------------------------------------------------------------------------------------
# the Adam driver's gradient and step  (reference: src/nqs/train.py:53-61 with optax.adam)
# ----------------------------------------------------------------------------------------------
def surrogate_grad(spec, theta, unravel, R, S, e):
    """train.py:53-59 — the real-ravel gradient of 2 mean_w Re[conj(e_w - mean e) log psi(R_w,
    S_w)] (reverse mode through the oracle log psi), (dL/dRe, dL/dIm) for complex leaves."""
    ec = torch.conj(e - e.mean())

    def loss(t):
        p = unravel(t)
        lp = torch.stack([logpsi(spec, p, R[w], S[w]) for w in range(R.shape[0])])
        return 2.0 * torch.real(ec * lp).mean()

    return grad(loss)(theta)


def jax_grad_tree(unravel, g):
    """The tree jax.grad returns for a real loss, from the real-ravel gradient g: a real leaf
    takes its components, a complex leaf c = a + i b the complex number dL/da - i dL/db (JAX's
    transpose convention for complex inputs)."""
    tree = unravel(g)

    def conj_tree(node):
        return {k: conj_tree(v) if isinstance(v, dict) else (torch.conj(v) if v.is_complex() else v)
                for k, v in node.items()}

    return conj_tree(tree)


def optax_adam(params, grads, state, lr, b1=0.9, b2=0.999, eps=1e-8):
    """optax.adam(lr) = scale_by_adam(b1, b2, eps) then scale_by_learning_rate, applied with
    optax.apply_updates, on trees of torch tensors (complex leaves included):
    mu <- b1 mu + (1 - b1) g;  nu <- b2 nu + (1 - b2) |g|^2;  t <- t + 1;
    p <- p - lr (mu / (1 - b1^t)) / (sqrt(nu / (1 - b2^t)) + eps).
    state: None (zeros) or the (t, mu, nu) this function returned. Returns (params, state)."""
    flat_p = flatten_sorted(params)
    flat_g = dict(flatten_sorted(grads))
    if state is None:
        state = (0, {k: torch.zeros_like(v) for k, v in flat_p},
                 {k: torch.zeros(v.shape, dtype=F64) for k, v in flat_p})
    t, mu, nu = state
    t += 1
    out, mu2, nu2 = {}, {}, {}
    for k, p in flat_p:
        gk = flat_g[k]
        mu2[k] = b1 * mu[k] + (1.0 - b1) * gk
        sq = (gk.real ** 2 + gk.imag ** 2) if gk.is_complex() else gk ** 2
        nu2[k] = b2 * nu[k] + (1.0 - b2) * sq
        upd = (mu2[k] / (1.0 - b1 ** t)) / (torch.sqrt(nu2[k] / (1.0 - b2 ** t)) + eps)
        node = out
        for q in k[:-1]:
            node = node.setdefault(q, {})
        node[k[-1]] = p - lr * upd
    return out, (t, mu2, nu2)
