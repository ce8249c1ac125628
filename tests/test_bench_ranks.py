"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (127.0.0.1).

bench.py --gpus N runs N independent replicas (one mesh per GPU, no
collective on the data path). What crosses ranks is timing: every rank's
time is reduced with a MAX, the job's throughput is N meshes over the
slowest rank's time, and the reference arm runs on rank 0 only while the
other ranks exit 0 without work. The same helpers run here over gloo.
"""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.0 + rank, dist, "cpu")      # rank r took 1 + r seconds
        v = bench.job_gfaces(world, 2_000_000_000, t)
        args = bench.argparse.Namespace(gpus=world, steps=3, warmup=3, n=6, cpu_n=6, cpu_reps=3, order=2)
        out = io.StringIO()
        with redirect_stdout(out):
            rc = bench.run_reference(args)
        dist.barrier()
        q.put((rank, t, v, rc, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_max_and_reference_arm_on_rank0():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v, rc, out in res:
        assert t == 2.0                                  # the slowest rank's time on every rank
        assert v == pytest.approx(2 * 2.0 / 2.0)         # 2 meshes x 2e9 faces / 2 s = 2 Gfaces/s
        assert rc == 0
    assert res[1][4] == ""                               # rank 1: no work, no line
    line = json.loads(res[0][4])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["value"] == line["value"] > 0
    # the reference arm runs the GPU arm's workload, with its steps and warm-up
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.workload_config(6, 2, 2)
    assert line["steps"] == 3 and line["warmup"] == 3


class _DoneProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_sampler_reads_power_cap_and_memory_clock(tmp_path):
    """bench.Clocks parses nvidia-smi rows in the order it asks for them
    (index, SM clock, SM max, power, active mask, hw_slowdown,
    hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap, memory clock):
    the SM clock's median and minimum, the memory clock, the highest power
    and every throttle reason seen, with the samples that had the power cap;
    unreadable rows are skipped."""
    sys.path.insert(0, ROOT)
    import bench
    rows = ["0, 1965, 1965, 268.4, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active, 3996",
            "0, 1965, 1965, 730.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active, 3996",
            "0, 1612, 1965, 995.8, 0x0000000000000004, Not Active, Not Active, Not Active, Active, 3996",
            "0, 1567, 1965, 1014.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active, 3996",
            "0, 1560, 1965, 997.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active, 3996",
            "0, [N/A], 1965, 990.0, 0x0, Not Active, Not Active, Not Active, Not Active, 3996",
            "garbage"]
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    with open(c.path, "w") as fh:
        fh.write("\n".join(rows) + "\n")
    c.proc = _DoneProc()
    out = c.stop()
    assert out["samples"] == 5
    assert out["sm_mhz"] == 1612.0 and out["sm_mhz_min"] == 1560.0 and out["sm_max_mhz"] == 1965.0
    assert out["mem_mhz"] == 3996.0 and out["power_w_max"] == 1014.0
    assert out["reasons"] == ["sw_power_cap"] and out["sw_power_cap_samples"] == 3
    assert not os.path.exists(c.path)


def test_clock_sampler_without_nvidia_smi():
    """No sampler process: the line says so instead of inventing clocks."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.Clocks(0)
    assert c.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
