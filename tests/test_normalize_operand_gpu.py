"""A dictionary whose 16-bit matching operand is normalised while the FP32
atoms stay as generated (DICT_NORMALIZE_OPERAND), matched with atom_norms,
against the normalised dictionary matched as usual.  Criteria:
  - the FP32 atoms equal those generated without normalisation, and the
    norms and the packed operand equal those of the normalised run (bitwise);
  - the matched atom equal on every voxel, (T1, T2, B0, B1) equal, and PD
    within 1e-6 relative (the rescoring divides the inner product by the norm
    instead of using atoms scaled beforehand: rounding only).
"""
import numpy as np
import pytest

from cases import mrf_schedule
from gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def _inputs(T=300, b1s=(0.8, 0.9, 1.0, 1.1), nvox=3000, seed=41):
    h = mrf_schedule(T, seed=seed)
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 800, 14)
            for a in np.geomspace(100, 3000, 16) if a > b]
    params = np.array(rows, np.float32)
    return h, params, params.shape[0] // len(b1s), nvox, seed


def _dict(snap, torch, h, params, T, natoms, flags, prec):
    NATOMS = params.shape[0]
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.full((NATOMS, T, 2), 5.0, dtype=torch.float32, device="cuda")
    d_norms = torch.full((NATOMS,), -1.0, dtype=torch.float32, device="cuda")
    d_packed = torch.full((NATOMS, snap.packed_pitch(T)), 3, dtype=torch.int16, device="cuda")
    snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, 20, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS | flags, d_norms=d_norms, d_packed=d_packed, packed_precision=prec)
    return d_params, d_atoms, d_norms, d_packed


@pytest.mark.parametrize("prec_name", ["fp16", "bf16"])
def test_normalized_operand_matches_like_normalized_atoms(snap, prec_name):
    torch = torch_cuda()
    prec = snap.PREC_FP16 if prec_name == "fp16" else snap.PREC_BF16
    h, params, natoms, nvox, seed = _inputs()
    T = h.shape[1]
    NATOMS = params.shape[0]
    _, a_norm, n_norm, p_norm = _dict(snap, torch, h, params, T, natoms, snap.DICT_NORMALIZE, prec)
    d_params, a_op, n_op, p_op = _dict(snap, torch, h, params, T, natoms, snap.DICT_NORMALIZE_OPERAND, prec)
    _, a_raw, n_raw, _ = _dict(snap, torch, h, params, T, natoms, 0, prec)
    torch.cuda.synchronize()
    assert torch.equal(a_op, a_raw)
    assert torch.equal(n_op, n_norm) and torch.equal(n_op, n_raw)
    assert torch.equal(p_op, p_norm)

    rng = np.random.default_rng(seed)
    atoms = a_norm.cpu().numpy()
    atoms = atoms[..., 0] + 1j * atoms[..., 1]
    j = rng.integers(0, NATOMS, nvox)
    img = atoms[j] * (rng.uniform(0.5, 1, nvox) * np.exp(1j * rng.uniform(0, 6.28, nvox)))[:, None]
    img = img + 0.005 * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape))
    b1 = (params[j, 3] + rng.uniform(-0.04, 0.04, nvox)).astype(np.float32)
    d_img = torch.from_numpy(img.astype(np.complex64).view(np.float32)).cuda().reshape(nvox, T, 2)
    d_b1 = torch.from_numpy(b1).cuda()
    flags = snap.MATCH_IMAG_ATOMS | snap.MATCH_ASSUME_UNIFORM_B1
    out = []
    for atoms_d, packed, norms in ((a_norm, p_norm, None), (a_op, p_op, n_op)):
        d_maps = torch.empty((nvox, 5), dtype=torch.float32, device="cuda")
        d_index = torch.empty(nvox, dtype=torch.int64, device="cuda")
        snap.MRF_match(d_maps, d_img, atoms_d, d_params, T, T, NATOMS, natoms, nvox, in_b1map=d_b1,
                       flags=flags, precision=prec, d_index=d_index, packed_atoms=packed, atom_norms=norms)
        out.append((d_maps.cpu().numpy(), d_index.cpu().numpy()))
    torch.cuda.synchronize()
    assert snap.device_error(reset=True) == 0
    (m0, i0), (m1, i1) = out
    assert np.array_equal(i0, i1)
    assert np.array_equal(m0[:, :4], m1[:, :4])
    rel = np.abs(m1[:, 4] - m0[:, 4]) / np.maximum(m0[:, 4], 1e-30)
    print(f"{prec_name}: PD max rel diff {rel.max():.2e}")
    assert rel.max() <= 1e-6
