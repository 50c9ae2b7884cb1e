"""Matching against a dictionary sharded across processes (one per GPU).

Each rank holds a contiguous range of whole B1 blocks of the dictionary (its
atoms and their parameter rows), matches every voxel against them with
MRF_match, and the ranks exchange their per-voxel results once: an
all_gather of the maps (T1, T2, B0, B1, PD) and the chosen global atom index,
28 bytes per voxel.  The merge is the reference's own rule for combining the
per-block results (merge_maps, src/functions.cu:1351-1384):

  * with a B1 map: the result whose B1 is nearest the voxel's map value
    (strict '<' from an initial 10, so ties go to the lower block and a voxel
    10 or more away from every result takes block 0's);
  * without one: the largest PD (strict '>', ties to the lower block).

Each rank's local match already applies that rule within its blocks, and the
ranks hold the blocks in order, so the merged maps are those of one
MRF_match over the whole dictionary whose blocks were matched one by one.
The exchange goes through torch.distributed (NCCL between GPUs, gloo on the
CPU); no kernel waits on another rank.
"""
from __future__ import annotations

from . import api


def merge_maps(maps_list, index_list, b1map=None):
    """Merges per-shard results, shards in block order.

    maps_list: sequence of [nvox][5] float tensors (T1, T2, B0, B1, PD);
    index_list: sequence of [nvox] int64 tensors (global atom index);
    b1map: optional [nvox] float tensor.  Returns (maps, index)."""
    import torch
    maps = maps_list[0].clone()
    index = index_list[0].clone()
    if b1map is not None:
        b1 = b1map.reshape(-1).to(maps.dtype)
        best = torch.full_like(b1, 10.0)
        chosen = torch.zeros(b1.shape, dtype=torch.int64, device=maps.device)
        for r, m in enumerate(maps_list):
            d = (b1 - m[:, 3]).abs()
            take = d < best
            best = torch.where(take, d, best)
            chosen = torch.where(take, torch.full_like(chosen, r), chosen)
    else:
        best = maps_list[0][:, 4].clone()
        chosen = torch.zeros(best.shape, dtype=torch.int64, device=maps.device)
        for r, m in enumerate(maps_list[1:], start=1):
            take = m[:, 4] > best
            best = torch.where(take, m[:, 4], best)
            chosen = torch.where(take, torch.full_like(chosen, r), chosen)
    stacked_maps = torch.stack(list(maps_list))             # [R][nvox][5]
    stacked_index = torch.stack(list(index_list))           # [R][nvox]
    ar = torch.arange(maps.shape[0], device=maps.device)
    maps = stacked_maps[chosen, ar]
    index = stacked_index[chosen, ar]
    return maps, index


def exchange_and_merge(d_maps, d_index, b1map=None, group=None):
    """All-gathers this rank's (maps, index) and merges them in rank order
    (ranks must hold the dictionary's B1 blocks in rank order).  Returns the
    merged (maps, index), identical on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    maps_all = [torch.empty_like(d_maps) for _ in range(world)]
    index_all = [torch.empty_like(d_index) for _ in range(world)]
    dist.all_gather(maps_all, d_maps.contiguous(), group=group)
    dist.all_gather(index_all, d_index.contiguous(), group=group)
    return merge_maps(maps_all, index_all, b1map)


def MRF_match_sharded(d_maps, img, d_atoms, d_params, NREPS: int, nreps: int, natoms_shard: int, natoms: int,
                      nvoxels: int, atom_offset: int, in_b1map=None, *, group=None, **match_kw):
    """MRF_match of this rank's shard (natoms_shard atoms, whole B1 blocks of
    natoms each, starting at global atom atom_offset), then the exchange and
    merge.  d_maps receives the merged maps; returns the merged global atom
    index per voxel.  Extra keywords go to MRF_match (precision, flags, ...).

    in_b1map must be a device tensor here (the merge reads it)."""
    import torch
    if natoms_shard % natoms:
        raise api.SnapMRFError(1, "a shard must hold whole B1 blocks")
    d_index = torch.empty(nvoxels, dtype=torch.int64, device=d_maps.device)
    local = torch.empty_like(d_maps)
    api.MRF_match(local, img, d_atoms, d_params, NREPS, nreps, natoms_shard, natoms, nvoxels,
                  in_b1map=in_b1map, d_index=d_index, **match_kw)
    d_index += atom_offset
    maps, index = exchange_and_merge(local, d_index, in_b1map, group)
    d_maps.copy_(maps)
    return index
