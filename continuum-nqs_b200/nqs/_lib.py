"""ctypes binding of libnqs.so (the C ABI declared in include/nqs.h).

The library is the only compute path: there is no CPU fallback. Loading it needs no GPU, but every
compute call requires CUDA tensors and raises RuntimeError on a machine without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os
import threading
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, \
    c_uint64, c_void_p

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnqs.so")

NQS_OK = 0
NQS_ERR_INVALID_ARG = 1
NQS_ERR_UNSUPPORTED = 2
NQS_ERR_WORKSPACE = 3
NQS_ERR_CUDA = 4
NQS_ERR_NONFINITE = 5
NQS_ERR_TIMEOUT = 6
NQS_ERR_NOT_SPD = 7

PREC_FP64 = 0
PREC_MIXED = 1
PREC_MIXED_SIMT = 2
PREC_MIXED_BF16 = 3

OP_LOGPSI, OP_LOCAL_E, OP_MCMC, OP_PER_SAMPLE_O = 0, 1, 2, 3
OP_PER_SAMPLE_O_CKPT, OP_LOGPSI_VJP, OP_LOGPSI_VJP_CKPT = 4, 5, 6

MAX_DEPTH = 16
B_NPARAM = 16
# order of NqsBlockParam
BLOCK_PARAMS = [("Dense_0", "bias"), ("Dense_0", "kernel"), ("Dense_1", "bias"),
                ("Dense_1", "kernel"), ("LayerNorm_0", "bias"), ("LayerNorm_0", "scale"),
                ("LayerNorm_1", "bias"), ("LayerNorm_1", "scale"), ("attn", "k", "bias"),
                ("attn", "k", "kernel"), ("attn", "o", "bias"), ("attn", "o", "kernel"),
                ("attn", "q", "bias"), ("attn", "q", "kernel"), ("attn", "v", "bias"),
                ("attn", "v", "kernel")]


class NqsModelDesc(Structure):
    _fields_ = [
        ("n_elec", c_int32), ("embed_dim", c_int32), ("depth", c_int32), ("n_heads", c_int32),
        ("ff_mult", c_int32), ("n_freq", c_int32), ("n_dets", c_int32), ("n_g", c_int32),
        ("learnable_env", c_int32), ("use_jastrow", c_int32), ("jastrow_kind", c_int32),
        ("n_knots", c_int32), ("cusp", c_double), ("A", c_double * 4),
        ("Gs_host", c_void_p), ("W_host", c_void_p), ("knots_host", c_void_p),
        ("n_params", c_int64),
        ("off_final_ln_bias", c_int64), ("off_final_ln_scale", c_int64),
        ("off_embed_bias", c_int64), ("off_embed_kernel", c_int64),
        ("off_backflow_bias", c_int64), ("off_backflow_kernel", c_int64),
        ("off_dW", c_int64), ("off_det_logw", c_int64), ("off_jas_c_opp", c_int64),
        ("off_jas_c_same", c_int64), ("off_jastrow_loga", c_int64),
        ("off_block", (c_int64 * B_NPARAM) * MAX_DEPTH),
    ]


_lib = None
_lock = threading.Lock()

_SIGS = {
    "nqs_version": ([], c_int),
    "nqs_status_string": ([c_int], c_char_p),
    "nqs_last_error": ([], c_char_p),
    "nqs_model_create": ([POINTER(NqsModelDesc), POINTER(c_void_p)], c_int),
    "nqs_model_destroy": ([c_void_p], c_int),
    "nqs_model_n_params": ([c_void_p], c_int64),
    "nqs_workspace_size": ([c_void_p, c_int, c_int, c_int, POINTER(c_size_t)], c_int),
    "nqs_logpsi": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p,
                    c_size_t, c_void_p], c_int),
    "nqs_local_energy": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double, c_double,
                          c_double, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_size_t,
                          c_void_p], c_int),
    "nqs_spin_estimators": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                             c_void_p, c_int, c_void_p, c_size_t, c_void_p], c_int),
    "nqs_local_energy_field": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double,
                                c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                c_void_p, c_size_t, c_void_p], c_int),
    "nqs_grad_laplacian": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                            c_void_p, c_int, c_void_p, c_size_t, c_void_p], c_int),
    "nqs_mcmc_sweeps": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                         c_double, c_uint64, c_uint64, c_void_p, c_void_p, c_void_p, c_void_p,
                         c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_size_t, c_void_p], c_int),
    "nqs_per_sample_O": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int,
                          c_void_p, c_size_t, c_void_p], c_int),
    "nqs_per_sample_O_ex": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                             c_int, c_int, c_void_p, c_size_t, c_void_p], c_int),
    "nqs_logpsi_vjp": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                        c_int, c_void_p, c_size_t, c_void_p], c_int),
    "nqs_ewald_create": ([POINTER(c_double), c_double, c_double, c_int, c_int, POINTER(c_void_p)],
                         c_int),
    "nqs_ewald_destroy": ([c_void_p], c_int),
    "nqs_ewald_zeta": ([c_void_p, POINTER(c_double)], c_int),
    "nqs_ewald_pair": ([c_void_p, c_void_p, c_int, c_void_p, c_void_p], c_int),
    "nqs_ewald_energy": ([c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p], c_int),
}


def lib():
    """Load libnqs.so once; bind every entry point with its C signature."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libnqs.so not built at {LIB_PATH}: run "
                                   "`python continuum-nqs_b200/build.py`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                f = getattr(L, name, None)
                if f is None:
                    continue
                f.argtypes = args
                f.restype = res
            _lib = L
        return _lib


def exported_symbols():
    """Names of _SIGS entry points the loaded library exports."""
    L = lib()
    return [n for n in _SIGS if getattr(L, n, None) is not None]


def check(status: int, what: str):
    if status == NQS_OK:
        return
    msg = lib().nqs_last_error().decode(errors="replace")
    text = f"{what} failed: {lib().nqs_status_string(status).decode()} ({msg})"
    if status in (NQS_ERR_INVALID_ARG, NQS_ERR_UNSUPPORTED):
        raise ValueError(text)
    raise RuntimeError(text)


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("nqs: the CUDA kernels need a CUDA device (there is no CPU fallback)")


def device() -> torch.device:
    require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def ptr(t):
    return None if t is None else c_void_p(t.data_ptr())


def stream_ptr():
    return c_void_p(torch.cuda.current_stream().cuda_stream)


class _Workspace:
    """Caller-side scratch buffers (one per device) grown on demand; the library allocates nothing."""

    def __init__(self):
        self.buf = {}

    def get(self, nbytes: int) -> torch.Tensor:
        dev = torch.cuda.current_device()
        b = self.buf.get(dev)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes * 1.25), 1 << 20), dtype=torch.uint8,
                            device=f"cuda:{dev}")
            self.buf[dev] = b
        return b


workspace = _Workspace()


def workspace_for(model_handle, op: int, n_walkers: int, prec: int) -> tuple[torch.Tensor, int]:
    n = c_size_t(0)
    check(lib().nqs_workspace_size(model_handle, op, n_walkers, prec, ctypes.byref(n)),
          "nqs_workspace_size")
    return workspace.get(n.value), n.value

_SIGS.update({
    "nqs_minsr_workspace_size": ([c_int, c_int64, c_int, c_int, POINTER(c_size_t)], c_int),
    "nqs_minsr_direction": ([c_void_p, c_int, c_void_p, c_int, c_int64, c_double, c_int, c_int,
                             c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_size_t,
                             c_void_p], c_int),
    "nqs_minsr_direction_ex": ([c_void_p, c_int, c_void_p, c_int, c_int64, c_double, c_int, c_int,
                                c_double, c_void_p, c_void_p, c_double, c_void_p, c_void_p,
                                c_void_p, c_size_t, c_void_p], c_int),
    "nqs_clip_energies": ([c_void_p, c_int, c_double, c_void_p, c_void_p, c_void_p], c_int),
    "nqs_energy_gradient": ([c_void_p, c_int, c_void_p, c_int, c_int64, c_void_p, c_void_p, c_size_t,
                             c_void_p], c_int),
    "nqs_energy_gradient_noalloc": ([c_void_p, c_int, c_void_p, c_int, c_int64, c_void_p,
                                     c_void_p], c_int),
    "nqs_adam_update": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_double, c_double,
                         c_double, c_double, c_int, c_void_p], c_int),
    "nqs_adam_update_complex": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                 c_double, c_double, c_double, c_double, c_int, c_void_p], c_int),
    "nqs_kernel_launches": ([], ctypes.c_ulonglong),
    "nqs_set_wait_limit": ([ctypes.c_uint], c_int),
    "nqs_selftest_bounded_wait": ([c_void_p, c_int, c_int, ctypes.c_uint, c_void_p, c_void_p,
                                   c_size_t, c_void_p, c_void_p], c_int),
    "nqs_profile_gemm": ([c_int], c_int),
    "nqs_set_block_fusion": ([c_int], c_int),
    "nqs_set_large_n_kernels": ([c_int], c_int),
    "nqs_set_attention_cta_small": ([c_int], c_int),
    "nqs_set_jacobian_tc": ([c_int], c_int),
    "nqs_set_attention_mma": ([c_int], c_int),
    "nqs_set_cholesky_dag": ([c_int], c_int),
    "nqs_set_cholesky_tc": ([c_int], c_int),
    "nqs_set_gram_wide": ([c_int], c_int),
    "nqs_set_preconditioner_shift": ([c_double], c_int),
    "nqs_set_rowgemm_stages": ([c_int], c_int),
    "nqs_mcmc_sweeps_devctr": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                c_int, c_double, c_uint64, c_void_p, c_void_p, c_void_p, c_int,
                                c_void_p, c_size_t, c_void_p], c_int),
    "nqs_profile_block_read": ([c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "nqs_profile_gemm_read": ([c_void_p, c_void_p, c_void_p], c_int),
    "nqs_profile_events": ([c_void_p, c_void_p], c_int),
    "nqs_gram": ([c_void_p, c_int, c_int, c_int64, c_int64, c_void_p, c_int64, c_void_p, c_void_p],
                 c_int),
    "nqs_gram_solve_workspace_size": ([c_int, c_int64, POINTER(c_size_t)], c_int),
    "nqs_gram_solve": ([c_void_p, c_int, c_int64, c_double, c_void_p, c_void_p, c_void_p, c_size_t,
                        c_void_p], c_int),
})
