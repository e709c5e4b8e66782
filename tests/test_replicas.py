"""The N-GPU bench runs independent replicas (the solve does not shard): the
whole-job figure is the iterations of all ranks over the slowest rank's time.
Checked here with two gloo ranks on the CPU."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ms, units = [40.0, 55.0][rank], [180, 175][rank]
    res = bench.combine_ranks(ms, units, world)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out, f"r{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_replicas_combine(tmp_path):
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        ms, units = json.load(open(tmp_path / f"r{r}.json"))
        assert ms == 55.0 and units == 355.0  # slowest rank's time, all ranks' iterations


def test_single_rank_is_identity():
    assert bench.combine_ranks(12.5, 7, 1) == (12.5, 7.0)


def test_reference_batch_sample_runs_one_process_per_model():
    """The batch bench's CPU baseline: the reference binary on two small batch
    models at once gives a positive aggregate rate over both."""
    import os
    import bench
    from efem_b200 import meshgen as mg

    if not os.path.exists(os.path.join(bench.ROOT, "oracle", "_ref", "efem_ref")):
        pytest.skip("oracle/_ref is not built")
    cases = mg.batch_beams(n=2, el_max=2000)
    rate, used, meta = bench.reference_batch_sample(cases, 2, ipstep=2, warmup=1, steps=1)
    assert rate is not None, meta
    assert used == 2 and rate > 0.0
