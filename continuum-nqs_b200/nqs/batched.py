"""Many independent VMC instances advanced together (the reference runs one train_minsr per
instance, src/nqs/minsr.py:92-159; here a whole batch of them is one unit of work).

Each instance has its own model (electron count, cell, envelope), walker count, Hamiltonian
(Rashba, Zeeman), damping and random stream. One MultiVMC.step() runs one VMC iteration of every
instance (Metropolis sweeps, local energies with Ewald, per-sample Jacobian, clip, MinSR update).
The instances share one Jacobian buffer and one workspace (they run one after the other on the
stream), and their random-stream counters live in device memory, so the whole step is captured
ONCE as a CUDA graph and each later step is a single graph launch.

Per (electron-count, walker-count) bucket an autotuner picks the implementation knobs of that
bucket's launches by timing them on a representative instance: the fused value-pass block on or
off, the row GEMMs' pipeline depth (2-4 operand tiles in flight) and the checkpointed reverse pass
on or off. The choices are applied while the graph is captured (each instance's launches are
recorded with its bucket's knobs) and are returned as a table.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import torch

from . import _lib
from .minsr import VMCIteration

F64 = torch.float64

N_EDGES = (10, 16, 22)        # electron-count buckets: <= 10, <= 16, <= 22, larger
W_EDGES = (1536, 2816)        # walker-count buckets: <= 1536, <= 2816, larger


def bucket_of(N: int, W: int) -> tuple[int, int]:
    """(electron bucket, walker bucket) indices."""
    return (sum(N > e for e in N_EDGES), sum(W > e for e in W_EDGES))


@dataclass
class Knobs:
    fusion: int = 1            # fused value-pass block (nqs_set_block_fusion)
    stages: int = 4            # row-GEMM pipeline depth (nqs_set_rowgemm_stages)
    checkpoint: bool = False   # checkpointed reverse pass for the Jacobian

    def apply(self):
        L = _lib.lib()
        _lib.check(L.nqs_set_block_fusion(int(self.fusion)), "nqs_set_block_fusion")
        _lib.check(L.nqs_set_rowgemm_stages(int(self.stages)), "nqs_set_rowgemm_stages")

    @staticmethod
    def restore():
        L = _lib.lib()
        L.nqs_set_block_fusion(1)
        L.nqs_set_rowgemm_stages(0)


CANDIDATES = [Knobs(f, s, c) for f, s, c in itertools.product((1, 0), (4, 3, 2), (False, True))]


@dataclass
class Instance:
    """One VMC problem: model + walkers + the VMCIteration keyword arguments (m_star,
    lambda_r, h_z, coulomb, lr, lam, n_sweeps, step_size, clip_k, seed, ...)."""
    model: object
    theta: torch.Tensor
    R: torch.Tensor
    S: torch.Tensor
    kwargs: dict = field(default_factory=dict)


class MultiVMC:
    def __init__(self, instances, precision="mixed", tuning=None, use_graph=True):
        _lib.require_cuda()
        self.precision = precision
        self.use_graph = use_graph
        o_dtype = torch.float64 if precision == "fp64" else torch.float32
        dev = _lib.device()
        need = max(2 * int(torch.as_tensor(x.S).shape[0]) * x.model.n_params() for x in instances)
        self.O_shared = torch.empty(need, dtype=o_dtype, device=dev)
        # workspaces are sized with every block's activations kept, which also covers the
        # checkpointed reverse pass the autotuner may pick
        # (created largest first, so that the shared workspace is sized once)
        order = sorted(range(len(instances)),
                       key=lambda i: -int(torch.as_tensor(instances[i].S).shape[0])
                       * instances[i].model.n_params())
        its = {}
        for i in order:
            x = instances[i]
            its[i] = VMCIteration(x.model, x.theta, x.R, x.S, precision=precision,
                                  device_counter=True, O_buffer=self.O_shared,
                                  **{k: v for k, v in x.kwargs.items() if k != "checkpoint_blocks"})
        self.its = [its[i] for i in range(len(instances))]
        self.tuning = dict(tuning or {})
        self.graph = None

    def knobs(self, it) -> Knobs:
        return self.tuning.get(bucket_of(it.N, it.W), Knobs())

    def _enqueue(self):
        try:
            for it in self.its:
                k = self.knobs(it)
                k.apply()
                it.checkpoint_blocks = k.checkpoint
                it.step()
        finally:
            Knobs.restore()

    def autotune(self, reps=1):
        """Time every candidate knob set on the largest-W instance of each bucket (eager, one
        warm step first) and keep the fastest; returns {bucket: (Knobs, ms)}."""
        reps = max(1, int(reps))
        report = {}
        buckets = {}
        for it in self.its:
            b = bucket_of(it.N, it.W)
            if b not in buckets or it.W > buckets[b].W:
                buckets[b] = it
        for b, it in sorted(buckets.items()):
            st = it.state_dict()
            best = None
            for k in CANDIDATES:
                try:
                    k.apply()
                    it.checkpoint_blocks = k.checkpoint
                    it.step()  # warm (first-launch set-up outside the timing)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(reps):
                        it.step()
                    e1.record()
                    torch.cuda.synchronize()
                    ms = e0.elapsed_time(e1) / reps
                finally:
                    Knobs.restore()
                if best is None or ms < best[1]:
                    best = (k, ms)
            it.load_state_dict(st)  # the tuning steps do not count
            self.tuning[b] = best[0]
            report[b] = best
        return report

    def capture(self, warmup=1):
        """Eager warm-up steps (first-launch set-up, workspace sizes), then the whole step is
        captured once as a CUDA graph."""
        for _ in range(warmup):
            self._enqueue()
        torch.cuda.synchronize()
        if not self.use_graph:
            return
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._enqueue()
        torch.cuda.synchronize()
        self.graph = g

    def step(self):
        """One VMC iteration of every instance (a single graph launch once captured)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._enqueue()

    def energies(self):
        """(W, N, mean E, error) per instance from the last step's statistics."""
        return [(it.W, it.N, float(it.stats[0]), float(it.stats[1])) for it in self.its]


def tuning_table(report):
    """JSON-friendly form of an autotune() report."""
    return [{"electron_bucket": b[0], "walker_bucket": b[1], "fusion": k.fusion,
             "rowgemm_stages": k.stages, "checkpoint": k.checkpoint, "ms_per_step": ms}
            for b, (k, ms) in sorted(report.items())]


def walker_steps(its):
    return sum(it.W * it.n_sweeps for it in its)

