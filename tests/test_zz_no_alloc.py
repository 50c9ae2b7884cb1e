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


def test_noalloc_strided_inputs_and_no_allocation(snap):
    """A padded image (img_stride > nreps), atoms with more time points than
    are matched (atom_stride > nreps), with and without a B1 map over the
    four-block dictionary: the same maps as the ordinary entry point, and no
    device scratch allocated by the allocation-free calls."""
    import torch
    T, params, NATOMS, natoms, d_params, d_atoms, atoms = _inputs(snap, torch)
    nreps, istride = 100, 131
    img, b1map = _voxels(atoms, 900, 4)
    pad = np.zeros((img.shape[0], istride), np.complex64)
    pad[:, :T] = img
    d_img = torch.from_numpy(pad.view(np.float32)).cuda()
    d_b1 = torch.from_numpy(b1map).cuda()
    nvox = img.shape[0]
    for b1 in (d_b1, None):
        ref_maps = torch.empty((nvox, 5), device="cuda")
        ref_idx = torch.empty(nvox, dtype=torch.int64, device="cuda")
        snap.MRF_match(ref_maps, d_img, d_atoms, d_params, T, nreps, NATOMS, natoms, nvox, in_b1map=b1,
                       d_index=ref_idx, img_stride=istride)
        maps = torch.full((nvox, 5), -1.0, device="cuda")
        idx = torch.full((nvox,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        before = snap.scratch_allocations()
        for _ in range(2):
            snap.MRF_match_noalloc(maps, d_img, d_atoms, d_params, T, nreps, NATOMS, natoms, nvox,
                                   d_b1map=b1, d_index=idx, img_stride=istride)
        torch.cuda.synchronize()
        assert snap.scratch_allocations() == before
        m, r = maps.cpu().numpy(), ref_maps.cpu().numpy()
        np.testing.assert_array_equal(idx.cpu().numpy(), ref_idx.cpu().numpy())
        np.testing.assert_array_equal(m[:, :4], r[:, :4])
        np.testing.assert_allclose(m[:, 4], r[:, 4], rtol=1e-5)
    # the ordinary entry point does allocate (the counter counts)
    snap.MRF_match(ref_maps, d_img, d_atoms, d_params, T, nreps, NATOMS, natoms, nvox, in_b1map=d_b1,
                   img_stride=istride)
    torch.cuda.synchronize()
    assert snap.scratch_allocations() > before


def test_noalloc_flags_a_mixed_b1_block(snap):
    """With a B1 map, a block holding two B1 values cannot be matched by
    nearest-B1 bins: the call's maps are NaN, its indices -1, and the device
    error word reads 9; the next correct call is unaffected."""
    import torch
    T, params, NATOMS, natoms, d_params, d_atoms, atoms = _inputs(snap, torch)
    bad = params.copy()
    bad[natoms + 3, 3] += 0.05           # one atom of block 1 with another B1
    d_bad = torch.from_numpy(bad).cuda()
    img, b1map = _voxels(atoms, 300, 5)
    d_img = torch.from_numpy(img.view(np.float32)).cuda()
    d_b1 = torch.from_numpy(b1map).cuda()
    maps = torch.zeros((300, 5), device="cuda")
    idx = torch.zeros(300, dtype=torch.int64, device="cuda")
    assert snap.device_error(reset=True) == 0
    snap.MRF_match_noalloc(maps, d_img, d_atoms, d_bad, T, T, NATOMS, natoms, 300, d_b1map=d_b1, d_index=idx)
    assert snap.device_error(reset=True) == 9
    assert np.isnan(maps.cpu().numpy()).all() and (idx.cpu().numpy() == -1).all()
    snap.MRF_match_noalloc(maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, 300, d_b1map=d_b1, d_index=idx)
    assert snap.device_error(reset=True) == 0
    assert np.isfinite(maps.cpu().numpy()).all() and (idx.cpu().numpy() >= 0).all()


def test_noalloc_rejects_requests_beyond_its_fixed_scratch(snap):
    import torch
    T, params, NATOMS, natoms, d_params, d_atoms, atoms = _inputs(snap, torch)
    n = snap.NOALLOC_MAX_VOXELS + 1
    d_img = torch.zeros((n, T, 2), device="cuda")
    maps = torch.empty((n, 5), device="cuda")
    with pytest.raises(snap.SnapMRFError, match="exceed the fixed scratch limit"):
        snap.MRF_match_noalloc(maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, n)
