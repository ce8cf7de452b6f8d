"""Many independent VMC instances in one unit of work (nqs.batched.MultiVMC, configuration 4's
shape at reduced walker counts): the whole step captured once as a CUDA graph and replayed equals
the same instances stepped one by one as separate VMCIterations (bit for bit: same kernels, same
inputs, random streams in device memory), and the autotuner returns one choice per bucket."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _instances(n=3):
    from nqs.configs import config4_instances
    return config4_instances(n_instances=n, seed=5, scale_walkers=0.08)


def test_graph_step_equals_separate_iterations():
    from nqs.batched import MultiVMC
    from nqs.minsr import VMCIteration
    inst = _instances()
    mv = MultiVMC(inst, precision="mixed", use_graph=True)
    mv.capture(warmup=1)
    assert mv.graph is not None
    mv.step()
    mv.step()
    torch.cuda.synchronize()
    for x, got in zip(inst, mv.its):
        ref = VMCIteration(x.model, x.theta, x.R, x.S, precision="mixed", device_counter=True,
                           **x.kwargs)
        for _ in range(3):
            ref.step()
        torch.cuda.synchronize()
        assert torch.equal(ref.theta, got.theta)
        assert torch.equal(ref.R, got.R) and torch.equal(ref.S, got.S)
        assert int(ref.counter_dev.item()) == int(got.counter_dev.item()) == 3 * x.kwargs["n_sweeps"]


def test_autotune_picks_one_choice_per_bucket():
    from nqs.batched import MultiVMC, bucket_of, tuning_table
    inst = _instances(4)
    mv = MultiVMC(inst, precision="mixed", use_graph=False)
    st0 = [it.state_dict() for it in mv.its]
    rep = mv.autotune()
    buckets = {bucket_of(it.N, it.W) for it in mv.its}
    assert set(rep) == buckets
    tab = tuning_table(rep)
    assert len(tab) == len(buckets) and all(r["ms_per_step"] > 0 for r in tab)
    # tuning leaves the instances' state as it found it
    for st, it in zip(st0, mv.its):
        s1 = it.state_dict()
        assert torch.equal(st["theta"], s1["theta"]) and torch.equal(st["R"], s1["R"])
        assert st["counter"] == s1["counter"]
    mv.capture(warmup=1)
    mv.step()
    assert all(torch.isfinite(it.stats[:3]).all() for it in mv.its)
