"""Helpers for the GPU tests: run the product's entry points on torch CUDA
buffers and bring results back as numpy."""
from __future__ import annotations

import numpy as np


def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def run_dict(snap, echo, params, h_mrf, nreps, natoms=None, nstates=101, flags=0, n_iso=1,
             fill=None, want_norms=False):
    """MRF_dict on the GPU; returns complex64 [NATOMS][nreps] (and norms)."""
    torch = torch_cuda()
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 4)
    NATOMS = params.shape[0]
    natoms = natoms or NATOMS
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.zeros((NATOMS, nreps, 2), dtype=torch.float32, device="cuda")
    if fill is not None:
        d_atoms.fill_(fill)
    d_norms = torch.full((NATOMS,), -1.0, dtype=torch.float32, device="cuda") if want_norms else None
    h_mrf = np.ascontiguousarray(h_mrf, np.float32)
    snap.MRF_dict(d_atoms, d_params, h_mrf, nreps, h_mrf.shape[1], NATOMS, natoms, 4, nstates, echo,
                  flags=flags, n_iso=n_iso, d_norms=d_norms)
    torch.cuda.synchronize()
    a = d_atoms.cpu().numpy()
    atoms = a[..., 0] + 1j * a[..., 1]
    if want_norms:
        return atoms.astype(np.complex64), d_norms.cpu().numpy()
    return atoms.astype(np.complex64)


def run_match(snap, img, atoms, params, nreps=None, natoms=None, b1map=None, device_img=False,
              flags=0, b1_device=False, precision=0):
    """MRF_match on the GPU; returns (maps [nvox][5], index [nvox])."""
    torch = torch_cuda()
    atoms = np.ascontiguousarray(atoms, np.complex64)
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 4)
    img = np.ascontiguousarray(img, np.complex64)
    NATOMS, T = atoms.shape
    nreps = nreps or T
    natoms = natoms or NATOMS
    nvox = img.shape[0]
    d_atoms = torch.from_numpy(atoms.view(np.float32)).cuda()
    d_params = torch.from_numpy(params).cuda()
    d_maps = torch.full((nvox, 5), -7.0, dtype=torch.float32, device="cuda")
    d_index = torch.full((nvox,), -1, dtype=torch.int64, device="cuda")
    src = img
    if device_img:
        src = torch.from_numpy(img.view(np.float32)).cuda()
    b1 = b1map
    if b1map is not None and b1_device:
        b1 = torch.from_numpy(np.ascontiguousarray(b1map, np.float32)).cuda()
    snap.MRF_match(d_maps, src, d_atoms, d_params, T, nreps, NATOMS, natoms, nvox, in_b1map=b1,
                   flags=flags, d_index=d_index, img_stride=img.shape[1], precision=precision)
    torch.cuda.synchronize()
    return d_maps.cpu().numpy(), d_index.cpu().numpy()
