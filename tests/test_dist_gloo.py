"""Multi-process host logic of the multi-GPU path on CPU: world size 2 over gloo.

Each rank renders the Cornell box with its own seed family (here with the CPU oracle
standing in for a GPU), the accumulators are summed with an all-reduce, and the step time
is the maximum over ranks.  The reduced accumulators must equal the two renders summed
serially, and the whole-job value must count both ranks' paths.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from naivetrace_b200 import dist as nd
    from naivetrace_b200 import scenes
    from naivetrace_b200.scene import make_params
    from oracle.oracle import OracleScene

    r = nd.init_from_env(prefer="gloo", timeout_s=60)
    assert r.world == world and r.rank == rank and r.backend == "gloo"
    scene = scenes.cornell_box(16, 16)
    o = OracleScene(scene, make_params(max_ray_depth=5))
    acc, light, _ = o.render(2, seed=nd.rank_seed(1, rank), nthreads=1)
    t_acc, t_light = torch.from_numpy(acc.copy()), torch.from_numpy(light.copy())
    nd.allreduce_sum_([t_acc, t_light], r)
    worst = nd.max_over_ranks(10.0 + rank, r)
    nd.barrier(r)
    np.save(os.path.join(out_dir, f"acc{rank}.npy"), t_acc.numpy())
    np.save(os.path.join(out_dir, f"worst{rank}.npy"), np.array([worst]))
    nd.shutdown(r)


def test_two_rank_allreduce_and_max(tmp_path, oracle_lib):
    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    from naivetrace_b200 import dist as nd
    from naivetrace_b200 import scenes
    from naivetrace_b200.scene import make_params
    from oracle.oracle import OracleScene

    scene = scenes.cornell_box(16, 16)
    o = OracleScene(scene, make_params(max_ray_depth=5))
    expect = o.render(2, seed=nd.rank_seed(1, 0), nthreads=1)[0] + o.render(2, seed=nd.rank_seed(1, 1), nthreads=1)[0]
    for rank in range(world):
        np.testing.assert_allclose(np.load(tmp_path / f"acc{rank}.npy"), expect, rtol=1e-12, atol=1e-15)
        assert np.load(tmp_path / f"worst{rank}.npy")[0] == 11.0
    assert nd.weak_scaling_value(1000, 2, 2.0) == pytest.approx(1.0)
