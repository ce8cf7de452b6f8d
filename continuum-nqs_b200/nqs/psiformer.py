"""Continuum spinful Psiformer — the wavefunction module (drop-in for src/nqs/psiformer.py).

Same constructor fields, parameter tree (flax names and shapes) and ``init`` / ``apply`` /
``make_logpsi`` entry points as the reference (psiformer.py:100-196). The forward pass runs in the
CUDA kernels of libnqs (``nqs_logpsi``); parameters live on the device as the real ravel ``theta``
(float64) whose layout is the JAX flatten order of the flax tree (minsr.py:30-53).

Adaptations forced by the absence of JAX: ``key`` is an integer seed (or a ``nqs.random`` key),
``apply`` accepts one configuration ``R (N,2), S (N,)`` or a batch ``R (W,N,2), S (W,N)``, and the
parameter leaves are torch tensors.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from . import _lib
from .cell import cell_matrix

F64 = torch.float64
C128 = torch.complex128


def _key_seed(key) -> int:
    from .random import key_to_seed
    return key_to_seed(key)


@dataclass(eq=False)
class ContinuumSpinorPsiformer:
    """Single generalized-spinor-determinant Psiformer (psiformer.py:100-116)."""
    n_elec: int
    Gs: Any
    W: Any
    L: Any
    embed_dim: int = 32
    depth: int = 3
    n_heads: int = 4
    ff_mult: int = 2
    n_freq: int = 4
    n_dets: int = 1
    learnable_env: bool = False
    use_jastrow: bool = False
    jastrow_kind: str = "rbf"
    n_knots: int = 10
    cusp: float = 1.0
    _native: dict = field(default_factory=dict, repr=False)

    # ---------------------------------------------------------------- parameter tree layout
    def param_shapes(self) -> dict:
        """Nested dict path -> (shape, is_complex), flax module names (psiformer.py:50-188)."""
        d, N, K = self.embed_dim, self.n_elec, self.n_dets
        D = self.ff_mult * d
        dense = lambda i, o: {"bias": ((o,), False), "kernel": ((i, o), False)}  # noqa: E731
        ln = lambda n: {"bias": ((n,), False), "scale": ((n,), False)}  # noqa: E731
        tree: dict = {"LayerNorm_0": ln(d)}
        for b in range(self.depth):
            tree[f"TransformerBlock_{b}"] = {
                "Dense_0": dense(d, D), "Dense_1": dense(D, d),
                "LayerNorm_0": ln(d), "LayerNorm_1": ln(d),
                "attn": {"k": dense(d, d), "o": dense(d, d), "q": dense(d, d), "v": dense(d, d)},
            }
        tree["backflow"] = {"bias": ((K * N,), True), "kernel": ((d, K * N), True)}
        if self.learnable_env:
            tree["dW"] = ((N, int(np.asarray(self.Gs).shape[0]), 2), True)
        if K > 1:
            tree["det_logw"] = ((K,), True)
        tree["embed"] = dense(4 * self.n_freq + 2, d)
        if self.use_jastrow:
            if self.jastrow_kind == "rbf":
                tree["jas_c_opp"] = ((self.n_knots,), False)
                tree["jas_c_same"] = ((self.n_knots,), False)
            else:
                tree["jastrow_loga"] = ((), False)
        return tree

    def leaves(self):
        """[(path, shape, is_complex, offset)] in theta order (sorted keys, complex -> re, im)."""
        out, off = [], 0

        def walk(node, prefix):
            nonlocal off
            for k in sorted(node.keys()):
                v = node[k]
                if isinstance(v, dict):
                    walk(v, prefix + (k,))
                else:
                    shape, is_c = v
                    n = int(np.prod(shape)) if len(shape) else 1
                    out.append((prefix + (k,), shape, is_c, off))
                    off += 2 * n if is_c else n

        walk(self.param_shapes(), ())
        return out

    def n_params(self) -> int:
        last = self.leaves()[-1]
        n = int(np.prod(last[1])) if len(last[1]) else 1
        return last[3] + (2 * n if last[2] else n)

    # ---------------------------------------------------------------- init
    def init(self, key, R0=None, S0=None):
        """flax default initialisation (psiformer.py:100-188): Dense kernels lecun_normal
        (truncated normal, std sqrt(1/fan_in)/0.8796), biases 0, LayerNorm scale 1 / bias 0,
        backflow / det_logw / Jastrow / dW zero. Returns {'params': tree} of CPU tensors.
        The random stream is numpy's (keyed by `key`), not JAX's threefry."""
        rng = np.random.default_rng(_key_seed(key))
        tree: dict = {}
        for path, shape, is_c, _ in self.leaves():
            name = path[-1]
            zero_init = path[0] in ("backflow", "dW", "det_logw", "jas_c_opp", "jas_c_same",
                                    "jastrow_loga")
            if name == "kernel" and not zero_init:
                std = math.sqrt(1.0 / shape[0]) / 0.87962566103423978
                v = rng.standard_normal(size=shape)
                bad = np.abs(v) > 2.0
                while bad.any():
                    v[bad] = rng.standard_normal(size=int(bad.sum()))
                    bad = np.abs(v) > 2.0
                leaf = torch.as_tensor(v * std, dtype=F64)
            elif name == "scale":
                leaf = torch.ones(shape, dtype=F64)
            else:
                leaf = torch.zeros(shape, dtype=C128 if is_c else F64)
            node = tree
            for k in path[:-1]:
                node = node.setdefault(k, {})
            node[path[-1]] = leaf
        return {"params": tree}

    def init_normal(self, key, std=0.02, backflow_std=1e-3, jastrow_std=0.02, logw_std=0.0):
        """The synthetic initialisation of the benchmark configurations: every Dense kernel
        ~N(0, std^2), biases 0, LayerNorm 1/0, backflow kernel re/im ~N(0, backflow_std^2),
        Jastrow coefficients ~N(0, jastrow_std^2), det_logw ~N(0, logw_std^2)."""
        rng = np.random.default_rng(_key_seed(key))
        p = self.init(key)
        for path, shape, is_c, _ in self.leaves():
            node = p["params"]
            for k in path[:-1]:
                node = node[k]
            name = path[-1]
            if path[0] == "backflow" and name == "kernel":
                node[name] = torch.complex(
                    torch.as_tensor(rng.normal(0, backflow_std, shape), dtype=F64),
                    torch.as_tensor(rng.normal(0, backflow_std, shape), dtype=F64))
            elif path[0] in ("jas_c_opp", "jas_c_same"):
                node[name] = torch.as_tensor(rng.normal(0, jastrow_std, shape), dtype=F64)
            elif path[0] == "det_logw" and logw_std > 0:
                node[name] = torch.complex(torch.as_tensor(rng.normal(0, logw_std, shape)),
                                           torch.as_tensor(rng.normal(0, logw_std, shape)))
            elif name == "kernel" and path[0] not in ("backflow",):
                node[name] = torch.as_tensor(rng.normal(0, std, shape), dtype=F64)
        return p

    # ---------------------------------------------------------------- native handle
    def native(self):
        """The libnqs model handle for the current device (created once per device)."""
        dev = _lib.device()
        h = self._native.get(dev.index)
        if h is not None:
            return h
        torch.cuda.init()
        L = _lib.lib()
        desc, keep = self.descriptor()
        handle = ctypes.c_void_p()
        _lib.check(L.nqs_model_create(ctypes.byref(desc), ctypes.byref(handle)),
                   "nqs_model_create")
        del keep  # the constants were copied to the device by nqs_model_create
        h = _NativeModel(handle)
        self._native[dev.index] = h
        return h

    def descriptor(self):
        """(NqsModelDesc, host arrays it points to) for nqs_model_create; keep the arrays alive
        until the call returns."""
        desc = _lib.NqsModelDesc()
        desc.n_elec, desc.embed_dim, desc.depth = self.n_elec, self.embed_dim, self.depth
        desc.n_heads, desc.ff_mult, desc.n_freq = self.n_heads, self.ff_mult, self.n_freq
        desc.n_dets = self.n_dets
        Gs = np.ascontiguousarray(np.asarray(self.Gs, dtype=np.float64))
        W = np.ascontiguousarray(np.asarray(self.W, dtype=np.complex128))
        desc.n_g = Gs.shape[0]
        desc.learnable_env = int(self.learnable_env)
        desc.use_jastrow = int(self.use_jastrow)
        desc.jastrow_kind = 0 if self.jastrow_kind == "rbf" else 1
        desc.n_knots = self.n_knots
        desc.cusp = float(self.cusp)
        A = cell_matrix(self.L)
        for i in range(4):
            desc.A[i] = float(A.reshape(-1)[i])
        area = float(abs(np.linalg.det(A)))
        knots = np.ascontiguousarray(np.linspace(0.0, 0.5 * math.sqrt(area), self.n_knots))
        Wri = np.ascontiguousarray(W.view(np.float64))
        desc.Gs_host = Gs.ctypes.data
        desc.W_host = Wri.ctypes.data
        desc.knots_host = knots.ctypes.data
        offs = {path: off for path, _, _, off in self.leaves()}
        desc.n_params = self.n_params()
        g = lambda *p: offs.get(tuple(p), -1)  # noqa: E731
        desc.off_final_ln_bias = g("LayerNorm_0", "bias")
        desc.off_final_ln_scale = g("LayerNorm_0", "scale")
        desc.off_embed_bias = g("embed", "bias")
        desc.off_embed_kernel = g("embed", "kernel")
        desc.off_backflow_bias = g("backflow", "bias")
        desc.off_backflow_kernel = g("backflow", "kernel")
        desc.off_dW = g("dW")
        desc.off_det_logw = g("det_logw")
        desc.off_jas_c_opp = g("jas_c_opp")
        desc.off_jas_c_same = g("jas_c_same")
        desc.off_jastrow_loga = g("jastrow_loga")
        for b in range(self.depth):
            for q, sub in enumerate(_lib.BLOCK_PARAMS):
                desc.off_block[b][q] = g(f"TransformerBlock_{b}", *sub)
        return desc, (Gs, Wri, knots)

    # ---------------------------------------------------------------- forward
    def apply(self, params, R, S, precision: str = "fp64"):
        """log psi(R, S) (complex) for one configuration or a batch (psiformer.py:118-189)."""
        return make_logpsi(self, params, precision=precision)(R, S)

    def theta(self, params) -> torch.Tensor:
        """Real ravel of the parameter tree on the current CUDA device."""
        from .minsr import real_ravel
        t, _ = real_ravel(params["params"] if "params" in params else params)
        return t.to(_lib.device(), F64).contiguous()


class _NativeModel:
    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        try:
            if self.handle:
                _lib.lib().nqs_model_destroy(self.handle)
        except Exception:
            pass


def _prec(precision) -> int:
    if precision in (0, "fp64", "float64"):
        return _lib.PREC_FP64
    if precision in (1, "mixed", "tf32"):
        return _lib.PREC_MIXED
    if precision in (2, "mixed_simt", "fp32"):
        return _lib.PREC_MIXED_SIMT
    if precision in (3, "mixed_bf16", "bf16"):
        return _lib.PREC_MIXED_BF16
    raise ValueError(f"unknown precision {precision!r}")


def as_batch(R, S):
    """Move (R, S) to the device as float64 (W,N,2) / int32 (W,N); report whether single."""
    dev = _lib.device()
    R = torch.as_tensor(R)
    S = torch.as_tensor(S)
    single = R.dim() == 2
    if single:
        R, S = R[None], S[None]
    R = R.to(dev, F64).contiguous()
    S = S.to(dev, torch.int32).contiguous()
    return R, S, single


def split_heads(x, n_heads):
    """(..., N, d) -> (..., n_heads, N, d / n_heads): head h holds features [h hd, (h + 1) hd)
    (reference psiformer.py:38-41; the attention kernels use this feature-to-head map)."""
    x = torch.as_tensor(x)
    *lead, N, d = x.shape
    return x.reshape(*lead, N, n_heads, d // n_heads).movedim(-2, -3)


def merge_heads(x):
    """Inverse of split_heads: (..., n_heads, N, hd) -> (..., N, n_heads hd)."""
    x = torch.as_tensor(x).movedim(-3, -2)
    *lead, N, nh, hd = x.shape
    return x.reshape(*lead, N, nh * hd)


def periodic_features(R, cell, n_freq):
    """The network's input features (reference psiformer.py:84-97), as a host / device torch
    function: fractional coordinates s = R A^-T (no wrap: the features are lattice-periodic) and,
    per electron, [sin(2 pi m s_x), cos(2 pi m s_x), sin(2 pi m s_y), cos(2 pi m s_y)] blocks for
    m = 1..n_freq, i.e. (..., N, 2) -> (..., N, 4 n_freq) in the order [x: sin, cos; y: sin, cos].
    The kernels compute the same features in-kernel; this is for inspection and tests."""
    from .cell import cell_matrix
    R = torch.as_tensor(R)
    A = torch.as_tensor(cell_matrix(cell), dtype=R.dtype, device=R.device)
    s = R @ torch.linalg.inv(A).T
    m = torch.arange(1, n_freq + 1, dtype=R.dtype, device=R.device)
    ang = (2.0 * np.pi) * s[..., :, None] * m
    return torch.cat([torch.sin(ang), torch.cos(ang)], dim=-1).reshape(*R.shape[:-1], 4 * n_freq)


def _logpsi_values(model, theta, R, S, prec):
    W = R.shape[0]
    out = torch.empty(W, dtype=C128, device=R.device)
    h = model.native().handle
    ws, _ = _lib.workspace_for(h, _lib.OP_LOGPSI, W, prec)
    _lib.check(_lib.lib().nqs_logpsi(h, _lib.ptr(theta), _lib.ptr(R), _lib.ptr(S), W,
                                     _lib.ptr(out), prec, _lib.ptr(ws), ws.numel(),
                                     _lib.stream_ptr()), "nqs_logpsi")
    return out


def logpsi_vjp(model, theta, R, S, cotangent, precision="fp64", checkpoint_blocks=False):
    """sum_w Re(cotangent_w d log psi(R_w, S_w) / d theta) as float64[P] (nqs_logpsi_vjp): the
    derivative the Adam driver takes of its surrogate loss (train.py:53-59) without forming the
    per-sample Jacobian."""
    prec = _prec(precision)
    R, S, _ = as_batch(R, S)
    W = R.shape[0]
    theta = theta.detach().to(R.device, F64).contiguous()
    # resolve_conj: a lazily conjugated view (torch.conj) keeps the unconjugated numbers in memory
    ct = torch.as_tensor(cotangent).to(R.device, C128).reshape(W).resolve_conj().contiguous()
    out = torch.empty(model.n_params(), dtype=F64, device=R.device)
    h = model.native().handle
    op = _lib.OP_LOGPSI_VJP_CKPT if checkpoint_blocks else _lib.OP_LOGPSI_VJP
    ws, _ = _lib.workspace_for(h, op, W, prec)
    _lib.check(_lib.lib().nqs_logpsi_vjp(h, _lib.ptr(theta), _lib.ptr(R), _lib.ptr(S), W,
                                         _lib.ptr(ct), _lib.ptr(out), prec,
                                         int(bool(checkpoint_blocks)), _lib.ptr(ws), ws.numel(),
                                         _lib.stream_ptr()), "nqs_logpsi_vjp")
    return out


class _LogPsiFn(torch.autograd.Function):
    """log psi as a differentiable function of theta: forward nqs_logpsi, backward nqs_logpsi_vjp.
    PyTorch hands a complex output the gradient g = dL/dRe + i dL/dIm, so dL/dtheta =
    sum_w Re(conj(g_w) d log psi_w / d theta): the VJP with cotangent conj(g)."""

    @staticmethod
    def forward(ctx, theta, R, S, model, prec, checkpoint_blocks):
        ctx.model, ctx.prec, ctx.ckpt = model, prec, checkpoint_blocks
        ctx.save_for_backward(theta, R, S)
        return _logpsi_values(model, theta.detach().contiguous(), R, S, prec)

    @staticmethod
    def backward(ctx, g):
        theta, R, S = ctx.saved_tensors
        gt = None
        if ctx.needs_input_grad[0]:
            gt = logpsi_vjp(ctx.model, theta, R, S, torch.conj(g), ctx.prec, ctx.ckpt)
        return gt, None, None, None, None, None


class LogPsi:
    """logpsi(R, S) bound to a model and parameters (make_logpsi, psiformer.py:192-196). When
    theta requires grad (and grad mode is on) the output is differentiable with respect to theta
    through the hand-written reverse mode (nqs_logpsi_vjp)."""

    def __init__(self, model: ContinuumSpinorPsiformer, theta: torch.Tensor, precision="fp64",
                 checkpoint_blocks=False):
        self.model = model
        self.theta = theta
        self.precision = _prec(precision)
        self.checkpoint_blocks = bool(checkpoint_blocks)

    def __call__(self, R, S):
        R, S, single = as_batch(R, S)
        if torch.is_grad_enabled() and self.theta.requires_grad:
            out = _LogPsiFn.apply(self.theta, R, S, self.model, self.precision,
                                  self.checkpoint_blocks)
        else:
            out = _logpsi_values(self.model, self.theta.detach(), R, S, self.precision)
        return out[0] if single else out


def make_logpsi(model, params, precision="fp64"):
    """Bind params -> logpsi(R, S) -> complex (psiformer.py:192-196). params is the flax-style
    tree or the real ravel theta; a float64 CUDA theta that requires grad is kept as is, so the
    log psi values are differentiable with respect to it."""
    if isinstance(params, torch.Tensor):
        theta = params if (params.is_cuda and params.dtype == F64 and params.is_contiguous()) \
            else params.to(_lib.device(), F64).contiguous()
    else:
        theta = model.theta(params)
    return LogPsi(model, theta, precision)
