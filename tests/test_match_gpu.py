"""Matching on the GPU vs the oracle and the reference's matching self-test.

Index parity: the chosen atom must equal the oracle's (FP64 scores, the
reference's first-argmax and merge rules) wherever the FP64 score of the
oracle's winner beats the GPU's pick by more than 1e-6 relative; where it
does not, the two scores must agree to 1e-6 (a near-tie either may win).
Maps T1/T2/B0/B1 are then bit-identical params; PD within 1e-5 relative.
"""
import numpy as np
import pytest

from cases import MATCH_SELFTEST_INDICES, mrf_schedule
from gpu_util import run_dict, run_match

pytestmark = pytest.mark.gpu


def scores64(img, atoms, idx):
    return np.abs(np.einsum("vt,vt->v", np.conj(atoms[idx].astype(np.complex128)), img.astype(np.complex128)))


def check_parity(img, atoms, params, maps, got, ref_maps, ref_idx):
    s_ref = scores64(img, atoms, ref_idx)
    s_got = scores64(img, atoms, got)
    diff = got != ref_idx
    gap = (s_ref - s_got) / np.maximum(s_ref, 1e-30)
    print(f"index mismatches: {diff.sum()} / {len(got)}, max gap at mismatches "
          f"{gap[diff].max() if diff.any() else 0:.2e}")
    assert np.all(np.abs(gap[diff]) <= 1e-6)
    np.testing.assert_array_equal(maps[:, :4], params[got])
    ok = ref_maps[:, 4] > 0
    np.testing.assert_allclose(maps[ok, 4], s_got[ok], rtol=1e-5)


def test_reference_matching_selftest(snap, golden):
    atoms = golden["atoms_mrf"]
    params = golden["params_mrf"].reshape(-1, 4)
    idx = MATCH_SELFTEST_INDICES
    maps, got = run_match(snap, atoms[idx], atoms, params)
    np.testing.assert_array_equal(got, idx)
    assert np.abs(maps[:, :4] - params[idx]).sum() < 1e-6


def _dictionary(snap, oracle, T=300, nb1=1, b1s=None, seed=0):
    h = mrf_schedule(T, seed=seed)
    t1 = np.geomspace(100, 3000, 14)
    t2 = np.geomspace(10, 800, 12)
    b1s = b1s if b1s is not None else np.linspace(0.8, 1.2, nb1)
    rows = [(a, b, 0.0, d) for d in b1s for b in t2 for a in t1 if a > b]
    params = np.array(rows, np.float32)
    natoms = params.shape[0] // len(b1s)
    atoms = run_dict(snap, "epg_fisp", params, h, T, natoms=natoms, nstates=20,
                     flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    return atoms, params, natoms


def _voxels(atoms, n, seed, snr=30.0):
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, atoms.shape[0], n)
    mix = rng.integers(0, atoms.shape[0], n)
    s = atoms[pick] + 0.3 * atoms[mix]
    s = s * (rng.uniform(0.5, 1, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n)))[:, None]
    sig = np.linalg.norm(s, axis=1, keepdims=True) / np.sqrt(s.shape[1]) / snr
    s = s + sig / np.sqrt(2) * (rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape))
    return s.astype(np.complex64)


@pytest.mark.parametrize("device_img", [False, True])
def test_global_match_vs_oracle(snap, oracle, device_img):
    atoms, params, natoms = _dictionary(snap, oracle, nb1=3)
    img = _voxels(atoms, 700, 1)
    maps, got = run_match(snap, img, atoms, params, natoms=natoms, device_img=device_img)
    ref_maps, ref_idx = oracle.match(img, atoms, params, atoms.shape[1], natoms=natoms, nthreads=8)
    check_parity(img, atoms, params, maps, got, ref_maps, ref_idx)


@pytest.mark.parametrize("b1_device", [False, True])
def test_b1_map_match_vs_oracle(snap, oracle, b1_device):
    b1s = np.float32([0.6, 0.75, 0.9, 1.05, 1.2, 1.35])
    atoms, params, natoms = _dictionary(snap, oracle, b1s=b1s, T=200)
    nvox = 1000
    img = _voxels(atoms, nvox, 2)
    rng = np.random.default_rng(3)
    b1map = rng.uniform(0.5, 1.5, nvox).astype(np.float32)
    b1map[:6] = [0.0, 0.675, 11.0, np.nan, 1.35, -20.0]  # background, exact tie, far away, NaN
    b1map[6:40] = 0.675  # a tie between blocks 0 and 1 goes to block 0
    maps, got = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map, b1_device=b1_device)
    ref_maps, ref_idx = oracle.match(img, atoms, params, atoms.shape[1], natoms=natoms, b1map=b1map,
                                     nthreads=8)
    assert np.all(got // natoms == ref_idx // natoms), "B1 block choice"
    check_parity(img, atoms, params, maps, got, ref_maps, ref_idx)


def test_b1_map_with_mixed_blocks_uses_general_merge(snap, oracle):
    """A block holding several B1 values: every block is matched and merged
    by the B1 of its matched atom (src/functions.cu:1351-1384)."""
    atoms, params, natoms = _dictionary(snap, oracle, nb1=4, T=120)
    params = params.copy()
    params[1::3, 3] += 0.07
    nvox = 300
    img = _voxels(atoms, nvox, 5)
    b1map = np.random.default_rng(6).uniform(0.7, 1.3, nvox).astype(np.float32)
    maps, got = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map)
    ref_maps, ref_idx = oracle.match(img, atoms, params, atoms.shape[1], natoms=natoms, b1map=b1map)
    check_parity(img, atoms, params, maps, got, ref_maps, ref_idx)


def test_ties_zero_and_nan_voxels(snap, oracle):
    atoms, params, natoms = _dictionary(snap, oracle, nb1=1, T=64)
    atoms = atoms.copy()
    atoms[7] = atoms[3]          # exact duplicate: the lower index must win
    img = np.zeros((5, atoms.shape[1]), np.complex64)
    img[0] = atoms[3] * (0.5 - 0.2j)
    img[2] = np.nan
    img[3] = atoms[7]
    img[4, :] = 1e-20
    maps, got = run_match(snap, img, atoms, params)
    assert got[0] == 3 and got[3] == 3
    assert got[1] == 0 and maps[1, 4] == 0       # all-zero voxel: atom 0, PD 0
    assert got[2] == 0 and maps[2, 4] == 0       # NaN never beats the initial 0
    ref_maps, ref_idx = oracle.match(img, atoms, params, atoms.shape[1])
    np.testing.assert_array_equal(got[[0, 1, 2, 3]], ref_idx[[0, 1, 2, 3]])


def test_ragged_sizes_and_time_subset(snap, oracle):
    """Atom and voxel counts off the tile sizes, matching a prefix of the
    time points (nreps < stride)."""
    atoms, params, natoms = _dictionary(snap, oracle, nb1=1, T=90)
    atoms = atoms[:131]
    params = params[:131]
    img = _voxels(atoms, 67, 8)
    maps, got = run_match(snap, img, atoms, params, nreps=77)
    ref_maps, ref_idx = oracle.match(img[:, :77], np.ascontiguousarray(atoms[:, :77]), params, 77)
    check_parity(img[:, :77], atoms[:, :77], params, maps, got, ref_maps, ref_idx)


def test_pipeline_config0_like(snap, oracle):
    """EPG-FISP with inversion (T = 1000, w = 20), T1 100:100:3000 x T2
    20:10:300, noisy off-grid voxels: the map equals the oracle's."""
    T = 1000
    h = mrf_schedule(T, seed=0)
    params, NATOMS, natoms = snap.grid_params("100:100:3000", "20:10:300")
    assert NATOMS == 837
    atoms = run_dict(snap, "epg_fisp", params, h, T, nstates=20, flags=snap.DICT_NORMALIZE)
    ref_atoms = oracle.dict_atoms("epg_fisp", params, h, T, nstates=20, flags=oracle.NORMALIZE,
                                  nthreads=8)
    assert np.abs(atoms - ref_atoms).max() < 1e-4
    rng = np.random.default_rng(0)
    nvox = 512
    vp = np.stack([rng.uniform(100, 3000, nvox), rng.uniform(20, 300, nvox)], 1)
    vp = vp[vp[:, 0] > vp[:, 1]]
    vparams = np.concatenate([vp, np.zeros((len(vp), 1)), np.ones((len(vp), 1))], 1).astype(np.float32)
    sig = oracle.dict_atoms("epg_fisp", vparams, h, T, nstates=20, nthreads=8)
    img = _voxels(sig.astype(np.complex64), len(vp), 4)
    maps, got = run_match(snap, img, atoms, params)
    ref_maps, ref_idx = oracle.match(img, atoms, params, T, nthreads=8)
    check_parity(img, atoms, params, maps, got, ref_maps, ref_idx)


@pytest.mark.parametrize("use_map,nreps,stride_pad", [(False, 300, 0), (True, 300, 0), (True, 213, 5),
                                                      (False, 77, 3)])
def test_fp32_imaginary_atom_form_equals_complex_form(snap, oracle, use_map, nreps, stride_pad):
    """FISP atoms with every RF phase 0 are purely imaginary; with
    SNAPMRF_MATCH_IMAG_ATOMS the FP32 form multiplies only their imaginary
    parts (half the products), and its sums equal the complex form's
    exactly (the real parts' products add exact zeros): same maps, indices
    and PD bit for bit, for whole and partial time ranges, padded image
    rows (odd strides take the 8-byte load path) and ragged tiles."""
    b1s = np.float32([0.7, 0.85, 1.0, 1.15, 1.3])
    atoms, params, natoms = _dictionary(snap, oracle, b1s=b1s, T=300)
    assert np.abs(atoms.real).max() == 0
    nvox = 777
    img = _voxels(atoms, nvox, 11)
    if stride_pad:
        pad = np.zeros((nvox, 300 + stride_pad), np.complex64)
        pad[:, :300] = img
        img = pad
    b1map = np.random.default_rng(12).uniform(0.6, 1.4, nvox).astype(np.float32) if use_map else None
    a = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map, nreps=nreps, device_img=True)
    b = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map, nreps=nreps, device_img=True,
                  flags=snap.MATCH_IMAG_ATOMS)
    assert snap.device_error(reset=True) == 0
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[0], b[0])
    ref_maps, ref_idx = oracle.match(img[:, :nreps], np.ascontiguousarray(atoms[:, :nreps]), params, nreps,
                                     natoms=natoms, b1map=b1map, nthreads=8)
    check_parity(img[:, :nreps], atoms[:, :nreps], params, b[0], b[1], ref_maps, ref_idx)


def test_fp32_imaginary_atom_form_rejects_complex_atoms(snap, oracle):
    """Atoms with a real part under SNAPMRF_MATCH_IMAG_ATOMS: NaN maps,
    indices -1 and device error 7, as in the tensor-core forms."""
    atoms, params, natoms = _dictionary(snap, oracle, nb1=1, T=100)
    atoms = atoms.copy()
    atoms[5] += 0.01
    img = _voxels(atoms, 100, 13)
    assert snap.device_error(reset=True) == 0
    maps, got = run_match(snap, img, atoms, params, flags=snap.MATCH_IMAG_ATOMS)
    assert snap.device_error(reset=True) == 7
    assert np.isnan(maps).all() and (got == -1).all()


@pytest.mark.parametrize("prec", [0, 2])
def test_host_image_streamed_in_chunks(snap, oracle, prec):
    """A host image of 72 MB (four chunks of 18 MB) with padded rows: the
    library streams it to the device chunk by chunk on its copy stream and
    (FP32) matches each chunk as it arrives, (tensor cores) the first two
    chunks' voxels once they have arrived and the rest at the end; maps and
    indices equal the device-image call's bit for bit, with and without a B1
    map, pageable and page-locked, and img_device_copy keeps the uploaded
    rows.  The tensor-core form with SNAPMRF_MATCH_UPLOAD_EARLY (the upload
    overlapping the work already queued) gives the same maps too."""
    import torch
    T = 600
    b1s = np.float32([0.8, 1.0, 1.2])
    atoms, params, natoms = _dictionary(snap, oracle, b1s=b1s, T=T)
    nvox = 15000
    img = np.zeros((nvox, T + 3), np.complex64)
    img[:, :T] = _voxels(atoms, nvox, 21)
    b1map = np.random.default_rng(22).uniform(0.7, 1.3, nvox).astype(np.float32)
    d_atoms = torch.from_numpy(atoms.view(np.float32)).cuda()
    d_params = torch.from_numpy(params).cuda()
    d_img = torch.from_numpy(np.ascontiguousarray(img).view(np.float32)).cuda()
    h_pinned = torch.from_numpy(np.ascontiguousarray(img).view(np.float32)).pin_memory()
    flags = snap.MATCH_IMAG_ATOMS | snap.MATCH_ASSUME_UNIFORM_B1
    for b1 in (None, torch.from_numpy(b1map).cuda()):
        out = {}
        for name, src in (("device", d_img), ("pageable", img), ("pinned", h_pinned)):
            maps = torch.full((nvox, 5), -1.0, device="cuda")
            idx = torch.full((nvox,), -1, dtype=torch.int64, device="cuda")
            copy = torch.zeros((nvox, T, 2), device="cuda") if name != "device" else None
            snap.MRF_match(maps, src, d_atoms, d_params, T, T, params.shape[0], natoms, nvox, in_b1map=b1,
                           precision=prec, flags=flags, d_index=idx, img_stride=T + 3, img_device_copy=copy,
                           upload_early=(prec != 0 and copy is not None))
            torch.cuda.synchronize()
            out[name] = (maps.cpu().numpy(), idx.cpu().numpy())
            if copy is not None:
                c = copy.cpu().numpy()
                np.testing.assert_array_equal(c[..., 0] + 1j * c[..., 1], img[:, :T])
        assert snap.device_error(reset=True) == 0
        for name in ("pageable", "pinned"):
            np.testing.assert_array_equal(out[name][1], out["device"][1])
            np.testing.assert_array_equal(out[name][0][:, :4], out["device"][0][:, :4])
            # the FP32 form's PD is bit-equal; the tensor-core rescoring sums
            # two samples per load when rows are 16-byte aligned (the dense
            # uploaded copy, not the padded device rows): last-bit changes
            np.testing.assert_allclose(out[name][0][:, 4], out["device"][0][:, 4], rtol=0 if prec == 0 else 1e-6)


def test_streamed_upload_options_are_checked(snap, oracle):
    import torch
    atoms, params, natoms = _dictionary(snap, oracle, nb1=1, T=64)
    img = _voxels(atoms, 10, 23)
    d_atoms = torch.from_numpy(atoms.view(np.float32)).cuda()
    d_params = torch.from_numpy(params).cuda()
    maps = torch.empty((10, 5), device="cuda")
    with pytest.raises(snap.SnapMRFError, match="UPLOAD_EARLY needs img_device_copy"):
        snap.MRF_match(maps, img, d_atoms, d_params, 64, 64, params.shape[0], natoms, 10, upload_early=True)
    with pytest.raises(snap.SnapMRFError, match="applies to a host image"):
        snap.MRF_match(maps, torch.from_numpy(img.view(np.float32)).cuda(), d_atoms, d_params, 64, 64,
                       params.shape[0], natoms, 10, img_device_copy=torch.empty((10, 64, 2), device="cuda"))
