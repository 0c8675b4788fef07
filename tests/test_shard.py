"""Multi-rank path on CPU: two gloo ranks split the samples of a frame and one
all-reduce reproduces the single-process film. The per-pixel sample values
come from the restated Luz sampler, so the test exercises the same keying
(seed, x, y, sample) the GPU kernels use."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from luz_b200.shard import render_sharded, sample_range

W, H, SPP, SEED = 6, 5, 7, 99


def fake_render_mean(offset, count):
    import oracle as O
    R = O.Restate()
    img = np.zeros((H, W, 3))
    for y in range(H):
        for x in range(W):
            for s in range(offset, offset + count):
                img[y, x] += [R.sample1d(SEED, x, y, s, 0, 0, 9), R.sample1d(SEED, x, y, s, 0, 1, 9),
                              R.sample1d(SEED, x, y, s, 0, 2, 9)]
    return torch.from_numpy(img / max(count, 1))


def worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    dist.init_process_group("gloo", rank=rank, world_size=world)
    film = render_sharded(fake_render_mean, SPP, rank, world, lambda t: dist.all_reduce(t))
    torch.save(film, os.path.join(out, f"film{rank}.pt"))
    dist.barrier()
    dist.destroy_process_group()


def test_sample_range_partition():
    for spp in (1, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [sample_range(spp, r, world) for r in range(world)]
            assert sum(c for _, c in parts) == spp
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))
    with pytest.raises(ValueError):
        sample_range(4, 2, 2)


def test_two_rank_gloo_matches_single_process(tmp_path):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    f0 = torch.load(tmp_path / "film0.pt")
    f1 = torch.load(tmp_path / "film1.pt")
    ref = fake_render_mean(0, SPP)
    assert torch.equal(f0, f1)
    assert torch.allclose(f0, ref, rtol=1e-12, atol=1e-12)
