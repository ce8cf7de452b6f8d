"""On-disk checkpoint of a VMC iteration (theta, walkers, random-stream position; the reference
resumes in memory only, src/nqs/minsr.py:95-103,136-138,157-158): the file format round trip on
the CPU. The bit-identical device resume is in tests/test_gpu_train.py."""
import torch


def test_checkpoint_file_roundtrip(tmp_path):
    """save_checkpoint / load_checkpoint keep theta, walkers and the random-stream position
    (a stand-in object with the iteration's state_dict)."""
    from nqs.minsr import load_checkpoint, save_checkpoint

    class It:
        def state_dict(self):
            return {"theta": torch.arange(5, dtype=torch.float64),
                    "R": torch.ones(2, 3, 2, dtype=torch.float64),
                    "S": torch.tensor([[0, 1, 1], [1, 0, 0]], dtype=torch.int32),
                    "seed": 7, "counter": 123456789012}

    p = tmp_path / "ck.npz"
    save_checkpoint(p, It())
    st = load_checkpoint(p)
    ref = It().state_dict()
    for k in ("theta", "R", "S"):
        assert torch.equal(st[k], ref[k])
    assert st["seed"] == 7 and st["counter"] == 123456789012
