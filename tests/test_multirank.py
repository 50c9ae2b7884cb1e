"""Multi-rank logic of bench.py on the CPU: the cross-rank reductions over a
world-size-2 gloo group, the per-rank slices, and the reference arm under
torchrun (rank 0 alone prints one line)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _reduce_worker(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev = torch.device("cpu")
        mx = bench.reduce_over_ranks([rank, -rank, 10.0 * rank + 1], "max", dev, world)
        mn = bench.reduce_over_ranks([rank, -rank, 10.0 * rank + 1], "min", dev, world)
        (Path(out_dir) / f"r{rank}.json").write_text(json.dumps({"max": mx, "min": mn}))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_reduce_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        d = json.loads((tmp_path / f"r{r}.json").read_text())
        assert d["max"] == [1.0, 0.0, 11.0]
        assert d["min"] == [0.0, -1.0, 1.0]


def test_reduce_over_ranks_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_over_ranks([3, 1.5], "max", None, 1) == [3.0, 1.5]


def test_each_rank_gets_its_own_slice():
    """Weak scaling: rank r simulates the slice seeded by r; the same rank
    always gets the same slice, and the B1 field is the same on every rank."""
    sys.path.insert(0, str(ROOT))
    import bench
    a0 = bench.phantom(0, nx=32)
    a0b = bench.phantom(0, nx=32)
    a1 = bench.phantom(1, nx=32)
    for x, y in zip(a0, a0b):
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(a0[1], a1[1])
    np.testing.assert_array_equal(a0[0], a1[0])


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=540, env=env,
                       stdin=subprocess.DEVNULL)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["extrapolated"] is False
    assert d["config"]["atoms"] == 284458 and d["config"]["voxels"] == 57600


def test_reference_arm_loads_no_product_code():
    """The CPU arm runs the oracle alone: after one of its steps neither the
    product package nor its library is loaded in the process."""
    code = ("import sys; sys.path.insert(0, '.'); import bench; r = bench.cpu_step(3); "
            "assert r['atoms'] == 6938 and r['voxels'] == 1405, r; "
            "assert not any(m.startswith('snapmrf_b200') for m in sys.modules), sorted(sys.modules); "
            "maps = open('/proc/self/maps').read(); assert 'libsnapmrf' not in maps; print('ok')")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300,
                       env=env, stdin=subprocess.DEVNULL)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-3000:]


def _shard_maps(r, nvox=64):
    """Synthetic per-shard matching results (shard r of 2) with ties built in:
    the B1 values of the shard's blocks, PDs that repeat across shards."""
    rng = np.random.default_rng(100 + r)
    maps = np.zeros((nvox, 5), np.float32)
    maps[:, 0] = rng.uniform(100, 3000, nvox)
    maps[:, 1] = rng.uniform(10, 90, nvox)
    maps[:, 3] = np.float32([0.8, 0.9][r]) + np.float32(0.1) * (np.arange(nvox) % 2)
    maps[:, 4] = np.round(rng.uniform(0, 4, nvox)).astype(np.float32)   # few distinct values: ties
    index = (r * 1000 + np.arange(nvox)).astype(np.int64)
    return maps, index


def _reference_merge(maps_list, index_list, b1):
    """merge_maps restated (src/functions.cu:1351-1384): nearest B1 from an
    initial 10 with strict '<', else the largest PD with strict '>'."""
    nvox = maps_list[0].shape[0]
    out = np.zeros_like(maps_list[0])
    idx = np.zeros(nvox, np.int64)
    for v in range(nvox):
        k = 0
        if b1 is not None:
            best = np.float32(10.0)
            for r, m in enumerate(maps_list):
                d = np.float32(abs(np.float32(b1[v]) - m[v, 3]))
                if d < best:
                    best, k = d, r
        else:
            best = maps_list[0][v, 4]
            for r, m in enumerate(maps_list[1:], start=1):
                if m[v, 4] > best:
                    best, k = m[v, 4], r
        out[v] = maps_list[k][v]
        idx[v] = index_list[k][v]
    return out, idx


def _b1_for(nvox=64):
    b1 = np.linspace(0.7, 1.2, nvox).astype(np.float32)
    b1[5] = np.nan
    b1[6] = 50.0
    b1[7] = np.float32(0.85)  # equidistant from 0.8 and 0.9 within rounding
    return b1


def _sharded_worker(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from snapmrf_b200 import sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m, i = _shard_maps(rank)
        res = {}
        for name, b1 in (("pd", None), ("b1", _b1_for())):
            maps, index = sharded.exchange_and_merge(torch.from_numpy(m), torch.from_numpy(i),
                                                     None if b1 is None else torch.from_numpy(b1))
            res[name] = (maps.numpy().tolist(), index.numpy().tolist())
        (Path(out_dir) / f"s{rank}.json").write_text(json.dumps(res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_merge_gloo(tmp_path):
    """Two ranks, each with the matching results of its half of the B1
    blocks: one all_gather and the reference's merge rule give every rank the
    same maps, equal to merge_maps restated over both shards."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_sharded_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    shards = [_shard_maps(r) for r in range(2)]
    for name, b1 in (("pd", None), ("b1", _b1_for())):
        want_maps, want_idx = _reference_merge([s[0] for s in shards], [s[1] for s in shards], b1)
        for r in range(2):
            got_maps, got_idx = json.loads((tmp_path / f"s{r}.json").read_text())[name]
            np.testing.assert_array_equal(np.array(got_maps, np.float32), want_maps)
            np.testing.assert_array_equal(np.array(got_idx, np.int64), want_idx)
