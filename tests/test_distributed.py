"""Multi-rank sample sharding on CPU (gloo, world size 2): disjoint seeds per rank, one all-reduce,
and the combined image equals the mean of every rank's frames rendered by the oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from lambent_b200 import distributed as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from lambent_b200 import scenes
    from oracle import oracle_py as O
    s = scenes.cornell_box(32, 32)
    osc = O.OracleScene(s)
    seeds = []

    def frame(seed):
        seeds.append(seed)
        return torch.from_numpy(osc.render(s.camera, 32, 32, samples=2, threads=1, seed_offset=seed)["color"])

    img = D.render_sharded(frame, 3, base_seed=11)
    np.save(os.path.join(out_dir, f"img{rank}.npy"), img.numpy())
    np.save(os.path.join(out_dir, f"seeds{rank}.npy"), np.array(seeds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sample_sharding(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    imgs = [np.load(tmp_path / f"img{r}.npy") for r in range(world)]
    seeds = [np.load(tmp_path / f"seeds{r}.npy") for r in range(world)]
    np.testing.assert_array_equal(imgs[0], imgs[1])
    assert not set(seeds[0]) & set(seeds[1])
    from lambent_b200 import scenes
    from oracle import oracle_py as O
    s = scenes.cornell_box(32, 32)
    osc = O.OracleScene(s)
    ref = np.mean([osc.render(s.camera, 32, 32, samples=2, threads=1, seed_offset=int(sd))["color"]
                   for r in range(world) for sd in seeds[r]], axis=0)
    np.testing.assert_allclose(imgs[0], ref, rtol=1e-5, atol=1e-6)


def test_rank_seed_range():
    assert D.rank_seed(0, 1, 0) == D.SEED_STRIDE
    with pytest.raises(ValueError):
        D.rank_seed(0, 0, D.SEED_STRIDE)


def _worker_offset(rank, world, port, out_dir):
    """render_sharded with first_step: the seeds continue the rank's range after the warm-up steps,
    as bench.py's timed loop uses them."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seeds = []

    def frame(seed):
        seeds.append(seed)
        return torch.full((4, 4), float(seed % 97), dtype=torch.float64)

    img = D.render_sharded(frame, 3, first_step=2)
    np.save(os.path.join(out_dir, f"img{rank}.npy"), img.numpy())
    np.save(os.path.join(out_dir, f"seeds{rank}.npy"), np.array(seeds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_after_warmup(tmp_path):
    world = 2
    mp.start_processes(_worker_offset, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    seeds = [np.load(tmp_path / f"seeds{r}.npy").tolist() for r in range(world)]
    assert seeds == [[D.rank_seed(0, r, k) for k in (2, 3, 4)] for r in range(world)]
    want = np.mean([s % 97 for r in range(world) for s in seeds[r]])
    for r in range(world):
        np.testing.assert_allclose(np.load(tmp_path / f"img{r}.npy"), np.full((4, 4), want))
