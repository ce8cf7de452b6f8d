"""MinSR natural-gradient optimizer and driver (drop-in for src/nqs/minsr.py:30-159).

real_ravel flattens the parameter tree exactly as the reference (sorted keys; complex leaf ->
[re, im]), so theta / O columns line up with the reference's. per_sample_O, minsr_direction and
paramsr_direction run in libnqs kernels.
"""
from __future__ import annotations

import numpy as np
import torch

F64 = torch.float64


def _flatten_sorted(tree, prefix=()):
    out = []
    for k in sorted(tree.keys()):
        v = tree[k]
        if isinstance(v, dict):
            out.extend(_flatten_sorted(v, prefix + (k,)))
        else:
            out.append((prefix + (k,), v))
    return out


def real_ravel(pytree):
    """Flatten a param tree to a REAL float64 vector (complex leaves -> [re, im]); returns
    (vec, unravel) (minsr.py:30-53). The vector lives on the leaves' device."""
    if "params" in pytree and isinstance(pytree["params"], dict) and len(pytree) == 1:
        wrapped = True
        tree = pytree["params"]
    else:
        wrapped = False
        tree = pytree
    leaves = _flatten_sorted(tree)
    specs, flats = [], []
    for path, leaf in leaves:
        leaf = torch.as_tensor(leaf)
        if leaf.is_complex():
            specs.append((path, True, tuple(leaf.shape), leaf.numel()))
            flats += [leaf.real.reshape(-1).to(F64), leaf.imag.reshape(-1).to(F64)]
        else:
            specs.append((path, False, tuple(leaf.shape), leaf.numel()))
            flats.append(leaf.reshape(-1).to(F64))
    dev = flats[0].device
    vec = torch.cat([f.to(dev) for f in flats])

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
        return {"params": out} if wrapped else out

    return vec, unravel


# ---------------------------------------------------------------------------------------------
# per-sample Jacobian and the sample-space solve (libnqs)
# ---------------------------------------------------------------------------------------------
def per_sample_O_rows(model, theta, R, S, dtype=torch.float64, precision="fp64"):
    """O as the [2W][P] real matrix (rows 0..W-1 = Re O, W..2W-1 = Im O) on the device."""
    from . import _lib
    from .psiformer import _prec, as_batch
    R, S, _ = as_batch(R, S)
    W = R.shape[0]
    P = model.n_params()
    theta = theta.to(R.device, F64).contiguous()
    out = torch.empty(2 * W, P, dtype=dtype, device=R.device)
    prec = _prec(precision)
    h = model.native().handle
    ws, _ = _lib.workspace_for(h, _lib.OP_PER_SAMPLE_O, W, prec)
    _lib.check(_lib.lib().nqs_per_sample_O(
        h, _lib.ptr(theta), _lib.ptr(R), _lib.ptr(S), W, _lib.ptr(out),
        0 if dtype == torch.float64 else 1, prec, _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
        "nqs_per_sample_O")
    return out


def per_sample_O(model, theta, unravel, R, S):
    """O[s,k] = d log Psi(x_s) / d theta_k, complex (W, P) (minsr.py:56-65)."""
    rows = per_sample_O_rows(model, theta, R, S)
    W = rows.shape[0] // 2
    return torch.complex(rows[:W], rows[W:])


def _as_rows(O):
    """Complex (W, P) -> real [2W][P] (copy); real [2W][P] passes through."""
    if O.is_complex():
        return torch.cat([O.real, O.imag], 0).contiguous()
    return O


_GRAM = {"fp64": 0, "bf16": 1, "tf32": 2}


PCG_MAX_ITERS = 24  # conjugate-gradient iterations allowed to a tensor-core Gram's solve
PCG_TOL = 1e-2      # ... and the preconditioned-residual reduction at which it stops


def minsr_step(O_rows, eps, lam, gram="fp64", theta=None, lr=0.0, want_direction=True,
               n_refine=None, damping_out=None, info=None, tol=PCG_TOL):
    """Sample-space natural gradient on the device, at damping lam. O_rows is [2W][P] (f64 or
    f32; a float64 O_rows is centred in place by the float64 Gram). gram "fp64": float64 Gram,
    Cholesky and n_refine (default 1) refinement steps; "bf16" / "tf32": tensor-core Gram whose
    factor preconditions conjugate gradients on the exact system (n_refine = iteration limit,
    default PCG_MAX_ITERS, stopping at tol). info (optional int32[5] on the device) receives
    the status and the CG iteration count (nqs_minsr_direction_ex). Returns dtheta (P,) and
    updates theta in place by -lr dtheta when given."""
    from . import _lib
    _lib.require_cuda()
    dev = O_rows.device
    n, P = O_rows.shape
    W = n // 2
    eps = torch.as_tensor(eps).to(dev, torch.complex128).resolve_conj().contiguous()
    od = 0 if O_rows.dtype == torch.float64 else 1
    g = _GRAM[gram]
    if n_refine is None:
        n_refine = 1 if g == 0 else PCG_MAX_ITERS
    nb = ctypes_size(W, P, od, g)
    ws = _lib.workspace.get(nb)
    d = torch.empty(P, dtype=F64, device=dev) if want_direction else None
    _lib.check(_lib.lib().nqs_minsr_direction_ex(
        _lib.ptr(O_rows), od, _lib.ptr(eps), W, P, float(lam), g, int(n_refine), float(tol),
        _lib.ptr(d), _lib.ptr(theta), float(lr), _lib.ptr(info), _lib.ptr(damping_out),
        _lib.ptr(ws), ws.numel(), _lib.stream_ptr()), "nqs_minsr_direction_ex")
    return d


def ctypes_size(W, P, od, g):
    import ctypes
    from . import _lib
    n = ctypes.c_size_t(0)
    _lib.check(_lib.lib().nqs_minsr_workspace_size(W, P, od, g, ctypes.byref(n)),
               "nqs_minsr_workspace_size")
    return n.value


def minsr_direction(O, eps, lam, gram="fp64", n_refine=None):
    """Natural-gradient direction via the SAMPLE-space (2W x 2W) solve (minsr.py:76-81).
    O: complex (W, P) or real [2W][P]; the input is not modified."""
    rows = _as_rows(O)
    if rows is O:
        rows = rows.clone()
    return minsr_step(rows, eps, lam, gram, n_refine=n_refine)


def gram_solve(A, rhs, lam):
    """x = (A A^T + lam I)^-1 rhs for a float64 row-major A (M x K) on the device, with the
    library's float64 Gram and Cholesky (nqs_gram_solve)."""
    from . import _lib
    A = A.to(F64).contiguous()
    M, K = A.shape
    rhs = rhs.to(A.device, F64).contiguous()
    x = torch.empty(M, dtype=F64, device=A.device)
    import ctypes
    n = ctypes.c_size_t(0)
    _lib.check(_lib.lib().nqs_gram_solve_workspace_size(M, K, ctypes.byref(n)),
               "nqs_gram_solve_workspace_size")
    ws = _lib.workspace.get(n.value)
    _lib.check(_lib.lib().nqs_gram_solve(_lib.ptr(A), M, K, float(lam), _lib.ptr(rhs), _lib.ptr(x),
                                         _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
               "nqs_gram_solve")
    return x


def paramsr_direction(O, eps, lam):
    """The same direction via the explicit PARAMETER-space (P x P) solve (minsr.py:84-88):
    (Otil^T Otil + lam I)^-1 Otil^T etil, with Otil^T as the Gram operand (test-sized P)."""
    rows = _as_rows(O).to(F64)
    W = rows.shape[0] // 2
    Ot = torch.cat([rows[:W] - rows[:W].mean(0, keepdim=True),
                    rows[W:] - rows[W:].mean(0, keepdim=True)], 0)
    eps = torch.as_tensor(eps).to(rows.device, torch.complex128)
    ec = eps - eps.mean()
    et = torch.cat([ec.real, ec.imag])
    At = Ot.T.contiguous()
    return gram_solve(At, At @ et, lam)


def clip_energies(e, clip_k):
    """median-MAD clip of Re e (minsr.py:145-148) and the energy statistics, on the device.
    Returns (e_clip complex (W,), stats f64[5] = mean, err, var, median, mad)."""
    from . import _lib
    e = torch.as_tensor(e).to(torch.complex128).resolve_conj().contiguous()
    out = torch.empty_like(e)
    stats = torch.empty(5, dtype=F64, device=e.device)
    _lib.check(_lib.lib().nqs_clip_energies(_lib.ptr(e), e.shape[0], float(clip_k), _lib.ptr(out),
                                            _lib.ptr(stats), _lib.stream_ptr()),
               "nqs_clip_energies")
    return out, stats


def gram_lower(A, kind="bf16"):
    """Lower triangle of A A^T (float64 out) on the tcgen05 tensor cores; A (M, K) float32 on
    the device is rounded to BF16 (kind 'bf16') or read as TF32 (kind 'tf32')."""
    from . import _lib
    _lib.require_cuda()
    M, K = A.shape
    if kind == "bf16":
        lda = (K + 7) // 8 * 8
        Ad = torch.zeros(M, lda, dtype=torch.bfloat16, device=A.device)
        Ad[:, :K] = A.to(torch.bfloat16)
        code = 1
    else:
        lda = (K + 3) // 4 * 4
        Ad = torch.zeros(M, lda, dtype=torch.float32, device=A.device)
        Ad[:, :K] = A.to(torch.float32)
        code = 2
    T = torch.zeros(M, M, dtype=F64, device=A.device)
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    _lib.check(_lib.lib().nqs_gram(_lib.ptr(Ad), code, M, K, lda, _lib.ptr(T), M, _lib.ptr(err),
                                   _lib.stream_ptr()), "nqs_gram")
    if int(err.item()) != 0:
        raise RuntimeError("nqs_gram: a tensor-core CTA hit its bounded-wait limit")
    return T


# ---------------------------------------------------------------------------------------------
# the VMC iteration and the MinSR training loop (minsr.py:92-159)
# ---------------------------------------------------------------------------------------------
class VMCIteration:
    """Device-resident state of one VMC run: theta, walkers, and the buffers of one iteration.

    step() = n_sweeps Metropolis sweeps (nqs_mcmc_sweeps) -> local energies with the Ewald term
    fused (nqs_local_energy) -> per-sample Jacobian (nqs_per_sample_O) -> median-MAD clip
    (nqs_clip_energies) -> MinSR direction with the update theta -= lr dtheta fused
    (nqs_minsr_direction). No host synchronisation happens inside step().

    precision "fp64": every stage float64 (float64 O, float64 Gram).
    precision "mixed": float32 network, float32 O, BF16 tcgen05 Gram ("gram" may override:
    "bf16" or "tf32"); determinants, energies, Cholesky and solves stay float64."""

    def __init__(self, model, theta, R, S, *, m_star=1.0, lambda_r=1.0, h_z=0.0, coulomb=None,
                 lr=0.05, lam=1e-3, n_sweeps=10, step_size=0.4, clip_k=5.0, n_spin_flips=2,
                 seed=0, counter=0, precision="fp64", gram=None, n_refine=None, ext_field=None,
                 checkpoint_blocks=False, device_counter=False, O_buffer=None):
        from . import _lib
        from .psiformer import _prec, as_batch
        _lib.require_cuda()
        self.model = model
        self.theta = theta.to(_lib.device(), F64).contiguous().clone()
        self.R, self.S, _ = as_batch(R, S)
        self.R, self.S = self.R.clone(), self.S.clone()
        self.W, self.N = self.S.shape
        self.P = model.n_params()
        self.m_star, self.lambda_r, self.h_z = float(m_star), float(lambda_r), float(h_z)
        self.ewald = None
        if coulomb is not None:
            if not hasattr(coulomb, "ewald"):
                raise NotImplementedError("coulomb must come from nqs.ewald.make_ewald")
            self.ewald = coulomb.ewald
        self.lr, self.lam, self.clip_k = float(lr), float(lam), float(clip_k)
        self.n_sweeps, self.step_size, self.n_flips = int(n_sweeps), float(step_size), n_spin_flips
        self.seed, self.counter = int(seed), int(counter)
        self.prec_name = precision
        self.prec = _prec(precision)
        self.checkpoint_blocks = bool(checkpoint_blocks)
        self.gram = gram or ("fp64" if self.prec == _lib.PREC_FP64 else "bf16")
        self.n_refine = int(n_refine if n_refine is not None
                            else (1 if self.gram == "fp64" else PCG_MAX_ITERS))
        dev = self.R.device
        self.o_dtype = torch.float64 if self.prec == _lib.PREC_FP64 else torch.float32
        self._O = None  # the [2W][P] Jacobian, allocated on first use
        if O_buffer is not None:  # a caller-owned buffer (several iterations may share one)
            if O_buffer.dtype != self.o_dtype or O_buffer.numel() < 2 * self.W * self.P:
                raise ValueError("O_buffer: wrong dtype or too small")
            self._O = O_buffer.view(-1)[:2 * self.W * self.P].view(2 * self.W, self.P)
        # the random stream's sweep counter in device memory (CUDA-graph replay draws fresh
        # proposals each time); the host counter is then not advanced
        self.counter_dev = (torch.tensor([self.counter], dtype=torch.int64, device=dev)
                            if device_counter else None)
        self.e = torch.empty(self.W, dtype=torch.complex128, device=dev)
        self.e_clip = torch.empty_like(self.e)
        self.stats = torch.zeros(5, dtype=F64, device=dev)
        self.acc_pos = torch.zeros(self.W, dtype=F64, device=dev)
        self.acc_spin = torch.zeros(self.W, dtype=F64, device=dev)
        # [0] non-positive pivot, [1] Gram timeout, [2] floored pivots, [3] CG iterations,
        # [4] CG stop reason (nqs_minsr_direction_ex)
        self.status = torch.zeros(5, dtype=torch.int32, device=dev)
        self.damping = torch.zeros(1, dtype=F64, device=dev)  # preconditioner shift of a TC Gram
        # external spin field (vectorised ext_field: positions (..., 2) -> (..., 3))
        self.ext_field = ext_field
        self.field = (torch.empty(self.W, self.N, 3, dtype=F64, device=dev)
                      if ext_field is not None else None)
        h = model.native().handle
        self.h = h
        op_o = _lib.OP_PER_SAMPLE_O_CKPT if self.checkpoint_blocks else _lib.OP_PER_SAMPLE_O
        sizes = [_lib.workspace_for(h, op, self.W, self.prec)[1]
                 for op in (_lib.OP_MCMC, _lib.OP_LOCAL_E, op_o)]
        sizes.append(ctypes_size(self.W, self.P, 0 if self.o_dtype == torch.float64 else 1,
                                 _GRAM[self.gram]))
        self.ws = _lib.workspace.get(max(sizes))

    @property
    def O(self):
        if self._O is None:
            self._O = torch.empty(2 * self.W, self.P, dtype=self.o_dtype, device=self.R.device)
        return self._O

    def sample(self, n_sweeps=None, inject=None):
        """n_sweeps Metropolis sweeps (default: the iteration's). inject: optional pre-drawn
        randomness (normals [n][W][N][2], position uniforms [n][W], flip indices and flip
        uniforms [n][n_spin_flips][W]) used verbatim instead of the counter-based stream (the
        counter still advances)."""
        from . import _lib
        L = _lib.lib()
        n = self.n_sweeps if n_sweeps is None else n_sweeps
        if self.counter_dev is not None:
            if inject is not None:
                raise ValueError("injected randomness needs the host counter")
            _lib.check(L.nqs_mcmc_sweeps_devctr(
                self.h, _lib.ptr(self.theta), _lib.ptr(self.R), _lib.ptr(self.S), None, self.W,
                n, self.n_flips, self.step_size, self.seed, _lib.ptr(self.counter_dev),
                _lib.ptr(self.acc_pos), _lib.ptr(self.acc_spin), self.prec, _lib.ptr(self.ws),
                self.ws.numel(), _lib.stream_ptr()), "nqs_mcmc_sweeps_devctr")
            return
        inj = [None] * 4
        if inject is not None:
            dev = self.R.device
            inj = [torch.as_tensor(inject[0], dtype=F64).to(dev).contiguous(),
                   torch.as_tensor(inject[1], dtype=F64).to(dev).contiguous(),
                   torch.as_tensor(inject[2]).to(dev, torch.int32).contiguous(),
                   torch.as_tensor(inject[3], dtype=F64).to(dev).contiguous()]
            if (tuple(inj[0].shape) != (n, self.W, self.N, 2) or tuple(inj[1].shape) != (n, self.W)
                    or tuple(inj[2].shape) != (n, self.n_flips, self.W)
                    or tuple(inj[3].shape) != (n, self.n_flips, self.W)):
                raise ValueError("injected randomness has the wrong shape")
        _lib.check(L.nqs_mcmc_sweeps(
            self.h, _lib.ptr(self.theta), _lib.ptr(self.R), _lib.ptr(self.S), None, self.W, n,
            self.n_flips, self.step_size, self.seed, self.counter, *[_lib.ptr(x) for x in inj],
            _lib.ptr(self.acc_pos), _lib.ptr(self.acc_spin), None, self.prec, _lib.ptr(self.ws),
            self.ws.numel(), _lib.stream_ptr()), "nqs_mcmc_sweeps")
        self.counter += n

    def energies(self):
        from . import _lib
        ew = self.ewald.handle if self.ewald else None
        if self.ext_field is None:
            _lib.check(_lib.lib().nqs_local_energy(
                self.h, _lib.ptr(self.theta), _lib.ptr(self.R), _lib.ptr(self.S), self.W,
                self.m_star, self.lambda_r, self.h_z, ew, _lib.ptr(self.e), None, self.prec,
                _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr()), "nqs_local_energy")
        else:
            self.field.copy_(torch.as_tensor(self.ext_field(self.R), dtype=F64))
            _lib.check(_lib.lib().nqs_local_energy_field(
                self.h, _lib.ptr(self.theta), _lib.ptr(self.R), _lib.ptr(self.S), self.W,
                self.m_star, self.lambda_r, self.h_z, ew, _lib.ptr(self.field), _lib.ptr(self.e),
                None, self.prec, _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr()),
                "nqs_local_energy_field")

    def jacobian(self):
        """The per-sample Jacobian O (nqs_per_sample_O_ex; with checkpoint_blocks the reverse
        pass recomputes each block's activations instead of storing them)."""
        from . import _lib
        _lib.check(_lib.lib().nqs_per_sample_O_ex(
            self.h, _lib.ptr(self.theta), _lib.ptr(self.R), _lib.ptr(self.S), self.W,
            _lib.ptr(self.O), 0 if self.o_dtype == torch.float64 else 1, self.prec,
            int(self.checkpoint_blocks), _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr()),
            "nqs_per_sample_O_ex")

    def release_jacobian(self):
        """Free the [2W][P] Jacobian buffer (it is reallocated by the next jacobian())."""
        self._O = None

    def update(self):
        from . import _lib
        L = _lib.lib()
        _lib.check(L.nqs_clip_energies(_lib.ptr(self.e), self.W, self.clip_k,
                                       _lib.ptr(self.e_clip), _lib.ptr(self.stats),
                                       _lib.stream_ptr()), "nqs_clip_energies")
        _lib.check(L.nqs_minsr_direction_ex(
            _lib.ptr(self.O), 0 if self.o_dtype == torch.float64 else 1, _lib.ptr(self.e_clip),
            self.W, self.P, self.lam, _GRAM[self.gram], self.n_refine, PCG_TOL, None,
            _lib.ptr(self.theta), self.lr, _lib.ptr(self.status), _lib.ptr(self.damping),
            _lib.ptr(self.ws), self.ws.numel(), _lib.stream_ptr()), "nqs_minsr_direction_ex")

    def step(self, inject=None):
        """One iteration; inject as in sample() replaces the sweeps' random draws."""
        self.sample(inject=inject)
        self.energies()
        self.jacobian()
        self.update()

    def state_dict(self):
        """What a resume needs beyond the constructor arguments: theta, the walkers and the
        position of the Metropolis random stream (seed, sweep counter), as host copies."""
        counter = int(self.counter_dev.item()) if self.counter_dev is not None else self.counter
        return {"theta": self.theta.cpu(), "R": self.R.cpu(), "S": self.S.cpu(),
                "seed": self.seed, "counter": counter}

    def load_state_dict(self, st):
        """Restore a state_dict (shapes must match this iteration's model and walker count); the
        next sweeps continue the same random stream."""
        theta = torch.as_tensor(st["theta"], dtype=F64)
        R = torch.as_tensor(st["R"], dtype=F64)
        S = torch.as_tensor(st["S"])
        if theta.shape != self.theta.shape or R.shape != self.R.shape or S.shape != self.S.shape:
            raise ValueError("checkpoint shapes do not match this VMC iteration")
        self.theta.copy_(theta)
        self.R.copy_(R)
        self.S.copy_(S.to(self.S.dtype))
        self.seed, self.counter = int(st["seed"]), int(st["counter"])
        if self.counter_dev is not None:
            self.counter_dev.fill_(self.counter)


def save_checkpoint(path, it):
    """Write a VMC iteration's state_dict (theta, walkers, random-stream position) to an .npz."""
    st = it.state_dict()
    np.savez(path, theta=st["theta"].numpy(), R=st["R"].numpy(), S=st["S"].numpy(),
             seed=np.int64(st["seed"]), counter=np.int64(st["counter"]))


def load_checkpoint(path):
    """The state_dict saved by save_checkpoint (torch tensors on the host, ints)."""
    z = np.load(path)
    return {"theta": torch.as_tensor(z["theta"]), "R": torch.as_tensor(z["R"]),
            "S": torch.as_tensor(z["S"]), "seed": int(z["seed"]), "counter": int(z["counter"])}


def train_minsr(model, params, L, n_elec, key, *, m_star=1.0, lambda_r=1.0, h_z=0.0,
                ext_field=None, coulomb=None, use_folx=False, n_walkers=256, n_steps=100,
                lr=0.05, lam=1e-3, n_sweeps=10, step_size=0.4, burn=80, clip_k=5.0,
                log_every=20, history=None, R0=None, S0=None, return_walkers=False,
                precision="fp64", gram=None):
    """Optimise the Psiformer with MinSR on the device (minsr.py:92-159). Returns
    (params, history) or (params, history, R, S) when return_walkers=True. Cold start draws
    uniform walkers and `burn` sweeps; a warm ensemble (R0, S0) skips the burn stage."""
    from .random import as_key, key_to_seed, split
    from .sampler import init_walkers_uniform
    theta, unravel = real_ravel(params)
    kk, ks = split(as_key(key), 2)
    if R0 is None:
        R, S = init_walkers_uniform(kk, n_walkers, n_elec, L)
    else:
        R, S = torch.as_tensor(R0), torch.as_tensor(S0)
    it = VMCIteration(model, theta, R, S, m_star=m_star, lambda_r=lambda_r, h_z=h_z,
                      coulomb=coulomb, lr=lr, lam=lam, n_sweeps=n_sweeps, step_size=step_size,
                      clip_k=clip_k, seed=key_to_seed(ks), precision=precision, gram=gram,
                      ext_field=ext_field)
    if R0 is None and burn > 0:
        it.sample(burn)
    hist = history if history is not None else {"E": [], "Eerr": []}
    for i in range(n_steps):
        it.step()
        st = it.stats.cpu()
        hist["E"].append(float(st[0]))
        hist["Eerr"].append(float(st[1]))
        if log_every and (i % log_every == 0 or i == n_steps - 1):
            print(f"    minsr {i:4d}: E={float(st[0]):+.6f} +/- {float(st[1]):.1e} "
                  f"acc={float(it.acc_pos.mean()):.2f}", flush=True)
    out = unravel(it.theta.to(theta.device))
    if return_walkers:
        return out, hist, it.R, it.S
    return out, hist
