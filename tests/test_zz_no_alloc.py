"""snapmrf_mrf_match_noalloc: matching for callers that cannot allocate
device memory while they run (a framework whose caching allocator already
holds the GPU's free memory, or a reconstruction pipeline that must not
allocate after start-up).  Its working arrays live in one fixed array per
GPU that every call shares, so this test calls it several times in a row,
with different inputs, and checks each result against the ordinary
snapmrf_mrf_match (same tolerance as the other matching tests: identical
indices and parameters, PD within 1e-5 relative).

The file is named to be collected last, and passes both alone in a fresh
process and after the rest of the suite.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(snap, torch):
    from cases import mrf_schedule
    T = 120
    h = mrf_schedule(T, seed=21)
    b1s = np.float32([0.8, 0.95, 1.1, 1.25])
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 600, 9)
            for a in np.geomspace(100, 3000, 11) if a > b]
    params = np.array(rows, np.float32)
    NATOMS = params.shape[0]
    natoms = NATOMS // len(b1s)
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.empty((NATOMS, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, 20, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    torch.cuda.synchronize()
    a = d_atoms.cpu().numpy()
    atoms = (a[..., 0] + 1j * a[..., 1]).astype(np.complex64)
    return T, params, NATOMS, natoms, d_params, d_atoms, atoms


def _voxels(atoms, n, seed):
    rng = np.random.default_rng(seed)
    s = atoms[rng.integers(0, atoms.shape[0], n)] * np.exp(1j * rng.uniform(0, 6.28, n))[:, None]
    s = s + 0.02 * (rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape))
    return s.astype(np.complex64), rng.uniform(0.7, 1.35, n).astype(np.float32)


def test_noalloc_matches_ordinary_entry_point_on_consecutive_calls(snap):
    import torch
    T, params, NATOMS, natoms, d_params, d_atoms, atoms = _inputs(snap, torch)
    calls = [(_voxels(atoms, 700, 1), True), (_voxels(atoms, 333, 2), False),
             (_voxels(atoms, 1500, 3), True)]
    for (img, b1map), use_map in calls:
        nvox = img.shape[0]
        d_img = torch.from_numpy(img.view(np.float32)).cuda()
        d_b1 = torch.from_numpy(b1map).cuda() if use_map else None
        # the ordinary entry point
        ref_maps = torch.empty((nvox, 5), device="cuda")
        ref_idx = torch.empty(nvox, dtype=torch.int64, device="cuda")
        snap.MRF_match(ref_maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, nvox, in_b1map=d_b1,
                       d_index=ref_idx)
        # the allocation-free one, called through the C ABI
        maps = torch.full((nvox, 5), -1.0, device="cuda")
        idx = torch.full((nvox,), -1, dtype=torch.int64, device="cuda")
        snap.MRF_match_noalloc(maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, nvox,
                               d_b1map=d_b1, d_index=idx)
        torch.cuda.synchronize()
        m, r = maps.cpu().numpy(), ref_maps.cpu().numpy()
        np.testing.assert_array_equal(idx.cpu().numpy(), ref_idx.cpu().numpy())
        np.testing.assert_array_equal(m[:, :4], r[:, :4])
        np.testing.assert_allclose(m[:, 4], r[:, 4], rtol=1e-5)


def test_noalloc_rejects_requests_beyond_its_fixed_scratch(snap):
    import torch
    T, params, NATOMS, natoms, d_params, d_atoms, atoms = _inputs(snap, torch)
    n = snap.NOALLOC_MAX_VOXELS + 1
    d_img = torch.zeros((n, T, 2), device="cuda")
    maps = torch.empty((n, 5), device="cuda")
    with pytest.raises(snap.SnapMRFError, match="exceed the fixed scratch limit"):
        snap.MRF_match_noalloc(maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, n)
