"""The multi-rank logic of bench.py on CPU: two gloo ranks agree on the
slowest rank's time and on the whole-job throughput, and the reference arm
does its work on rank 0 only."""
import os
import socket
from datetime import timedelta

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench.barrier(world)
        dev_ms = [10.0, 12.5][rank]
        q.put((rank,) + bench.aggregate(world, 1000, 4, dev_ms, torch.device("cpu")))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    want = 2 * 1000 * 4 / (12.5 / 1e3) / 1e6
    for rank, ms_max, value in got:
        assert ms_max == 12.5
        assert value == pytest.approx(want)


def test_single_rank_aggregate():
    import bench
    ms, v = bench.aggregate(1, 500, 10, 5.0, None)
    assert ms == 5.0 and v == pytest.approx(500 * 10 / 5e-3 / 1e6)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import bench
    import voxelg_b200.configs as configs
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(None, configs.CONFIGS[bench.CONFIG_NAME]) is None
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("content,want", [('{"hbm_gbs": 7100.5}', (7100.5, "measured")),
                                          ('{"hbm_gbs": {"burst": 7000}}', (7000.0, "measured")),
                                          ("not json", (6650.0, "fallback")),
                                          ('{"bf16_tflops": 1590}', (6650.0, "fallback")),
                                          (None, (6650.0, "fallback"))])
def test_measured_peaks_file_shapes(monkeypatch, tmp_path, content, want):
    """The roofline denominator: the driver-written HBM figure when readable,
    else the fallback, never an exception."""
    import bench
    if content is not None:
        (tmp_path / "MEASURED_PEAKS.json").write_text(content)
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    got = bench.measured_peaks()
    assert (got["hbm_gbs"], got["source"]) == want
