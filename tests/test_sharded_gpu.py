"""Matching against a dictionary sharded by B1 blocks (snapmrf_b200.sharded):
each shard matched on its own, the results merged with the reference's
merge_maps rule, equals one MRF_match over the whole dictionary.  The shards
run one after another on one GPU (no rank waits on another); the exchange
itself is covered on the CPU (tests/test_multirank.py) and here through a
one-rank NCCL group.  Criteria:
  - with a B1 map (FP32 and FP16 tensor-core forms): maps and indices equal;
  - without one (FP32): every merged pick has the unsharded pick's PD to
    1e-6 (relative), and >= 99 % of the picks are the same atom.
"""
import numpy as np
import pytest

from cases import mrf_schedule
from gpu_util import run_dict, torch_cuda

pytestmark = pytest.mark.gpu


def _setup(snap, T=300, b1s=(0.8, 0.9, 1.0, 1.1), nvox=2000, seed=31):
    torch = torch_cuda()
    h = mrf_schedule(T, seed=seed)
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 800, 12)
            for a in np.geomspace(100, 3000, 14) if a > b]
    params = np.array(rows, np.float32)
    natoms = params.shape[0] // len(b1s)
    atoms = run_dict(snap, "epg_fisp", params, h, T, natoms=natoms, nstates=20,
                     flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    rng = np.random.default_rng(seed)
    j = rng.integers(0, atoms.shape[0], nvox)
    img = atoms[j] * (rng.uniform(0.5, 1, nvox) * np.exp(1j * rng.uniform(0, 6.28, nvox)))[:, None]
    img = img + 0.01 * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape))
    b1 = (params[j, 3] + rng.uniform(-0.04, 0.04, nvox)).astype(np.float32)
    dev = torch.device("cuda")
    d_atoms = torch.from_numpy(atoms.view(np.float32)).to(dev).reshape(atoms.shape[0], T, 2)
    d_params = torch.from_numpy(params).to(dev)
    d_img = torch.from_numpy(img.astype(np.complex64).view(np.float32)).to(dev).reshape(nvox, T, 2)
    return torch, d_atoms, d_params, d_img, torch.from_numpy(b1).to(dev), T, natoms, nvox


def _match(snap, torch, d_atoms, d_params, d_img, T, NATOMS, natoms, nvox, b1, **kw):
    d_maps = torch.empty((nvox, 5), dtype=torch.float32, device="cuda")
    d_index = torch.empty(nvox, dtype=torch.int64, device="cuda")
    snap.MRF_match(d_maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, nvox, in_b1map=b1,
                   d_index=d_index, **kw)
    return d_maps, d_index


def _sharded(snap, torch, d_atoms, d_params, d_img, T, natoms, nvox, b1, nshards, **kw):
    from snapmrf_b200 import sharded
    NATOMS = d_atoms.shape[0]
    nb = NATOMS // natoms
    per = nb // nshards
    maps_l, idx_l = [], []
    for s in range(nshards):
        a0, a1 = s * per * natoms, (s + 1) * per * natoms
        m, i = _match(snap, torch, d_atoms[a0:a1], d_params[a0:a1], d_img, T, a1 - a0, natoms, nvox, b1, **kw)
        maps_l.append(m)
        idx_l.append(i + a0)
    return sharded.merge_maps(maps_l, idx_l, b1)


@pytest.mark.parametrize("prec", [0, 2], ids=["fp32", "fp16"])
def test_sharded_with_b1_map_equals_whole(snap, prec):
    torch, d_atoms, d_params, d_img, b1, T, natoms, nvox = _setup(snap)
    kw = dict(precision=prec, flags=snap.MATCH_IMAG_ATOMS if prec else 0)
    m0, i0 = _match(snap, torch, d_atoms, d_params, d_img, T, d_atoms.shape[0], natoms, nvox, b1, **kw)
    m2, i2 = _sharded(snap, torch, d_atoms, d_params, d_img, T, natoms, nvox, b1, 2, **kw)
    torch.cuda.synchronize()
    assert snap.device_error(reset=True) == 0
    assert torch.equal(i0, i2)
    assert torch.equal(m0, m2)


def test_sharded_without_b1_map_keeps_the_best_pd(snap):
    torch, d_atoms, d_params, d_img, _, T, natoms, nvox = _setup(snap)
    m0, i0 = _match(snap, torch, d_atoms, d_params, d_img, T, d_atoms.shape[0], natoms, nvox, None)
    m2, i2 = _sharded(snap, torch, d_atoms, d_params, d_img, T, natoms, nvox, None, 2)
    pd0, pd2 = m0[:, 4].cpu().numpy(), m2[:, 4].cpu().numpy()
    assert np.all(pd2 >= pd0 * (1 - 1e-6))
    same = (i0 == i2).float().mean().item()
    print(f"same atom for {same:.4f} of the voxels")
    assert same >= 0.99


def test_match_sharded_one_rank_group(snap):
    """MRF_match_sharded through a one-rank NCCL group: the exchange path."""
    import datetime
    import socket

    import torch.distributed as dist
    from snapmrf_b200 import sharded
    torch, d_atoms, d_params, d_img, b1, T, natoms, nvox = _setup(snap, nvox=500)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        d_maps = torch.empty((nvox, 5), dtype=torch.float32, device="cuda")
        idx = sharded.MRF_match_sharded(d_maps, d_img, d_atoms, d_params, T, T, d_atoms.shape[0], natoms, nvox,
                                        0, in_b1map=b1)
        m0, i0 = _match(snap, torch, d_atoms, d_params, d_img, T, d_atoms.shape[0], natoms, nvox, b1)
        torch.cuda.synchronize()
        assert torch.equal(idx, i0) and torch.equal(d_maps, m0)
    finally:
        dist.destroy_process_group()
