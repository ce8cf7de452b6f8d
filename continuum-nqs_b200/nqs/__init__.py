"""nqs — B200-native (sm_100a) VMC iteration for the continuum spinor Psiformer.

Modules mirror the reference package src/nqs of wenqin-chen/continuum-nqs: psiformer, local_energy,
ewald, sampler, minsr, train, plus the host-side setup helpers cell and rashba. Every compute call
goes through libnqs.so (C ABI, include/nqs.h); there is no CPU fallback.
"""
__all__ = ["psiformer", "local_energy", "ewald", "sampler", "minsr", "train", "cell", "rashba",
           "random"]
