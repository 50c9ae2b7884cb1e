"""Tensor-core matching (BF16, FP16 or FP8-E4M3 scores, top-k, exact FP32
rescoring) against the FP32 path.  Criteria (FP8: the looser bounds of
LIMITS, its 3-bit mantissa):
  - the reference's noiseless self-test recovers every parameter exactly;
  - at least 99 % of voxels get the FP32 path's atom, and every voxel that
    does not has an atom whose FP64 score is within 1e-3 (relative) of the
    FP32 path's pick: the BF16 pre-selection only ever swaps near-ties;
  - T1/T2/B0/B1 are the chosen atom's parameters; PD within 1e-5 of the
    FP32 path's where both pick the same atom;
  - no bounded wait ran out (snapmrf_device_error() == 0).
"""
import numpy as np
import pytest

from cases import MATCH_SELFTEST_INDICES, mrf_schedule
from gpu_util import run_dict, run_match

pytestmark = pytest.mark.gpu
BF16, FP16, FP8 = 1, 2, 3
PRECS = pytest.mark.parametrize("prec", [BF16, FP16, FP8], ids=["bf16", "fp16", "fp8"])
# (least argmax agreement with the FP32 path, largest relative score loss of
# a differing pick) per precision
LIMITS = {BF16: (0.99, 1e-3), FP16: (0.99, 1e-3), FP8: (0.97, 5e-3)}


def _dictionary(snap, T, b1s, nt1=14, nt2=12, seed=0):
    h = mrf_schedule(T, seed=seed)
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 800, nt2)
            for a in np.geomspace(100, 3000, nt1) if a > b]
    params = np.array(rows, np.float32)
    natoms = params.shape[0] // len(b1s)
    atoms = run_dict(snap, "epg_fisp", params, h, T, natoms=natoms, nstates=20,
                     flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    return atoms, params, natoms


def _voxels(atoms, n, seed, snr=30.0):
    rng = np.random.default_rng(seed)
    s = atoms[rng.integers(0, atoms.shape[0], n)] + 0.3 * atoms[rng.integers(0, atoms.shape[0], n)]
    s = s * (rng.uniform(0.5, 1, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n)))[:, None]
    sig = np.linalg.norm(s, axis=1, keepdims=True) / np.sqrt(s.shape[1]) / snr
    s = s + sig / np.sqrt(2) * (rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape))
    return s.astype(np.complex64)


def compare(img, atoms, params, m32, i32, m16, i16, min_agree=0.99, max_loss=1e-3):
    agree = np.mean(i16 == i32)
    s = lambda idx: np.abs(np.einsum("vt,vt->v", np.conj(atoms[idx].astype(np.complex128)),
                                     img.astype(np.complex128)))
    diff = i16 != i32
    rel = (s(i32) - s(i16)) / np.maximum(s(i32), 1e-30)
    print(f"agreement {agree:.5f} ({diff.sum()} of {len(i32)} differ), max rel score loss "
          f"{rel[diff].max() if diff.any() else 0:.2e}")
    assert agree >= min_agree
    assert np.all(rel[diff] <= max_loss)
    np.testing.assert_array_equal(m16[:, :4], params[i16])
    same = ~diff & (m32[:, 4] > 0)
    np.testing.assert_allclose(m16[same, 4], m32[same, 4], rtol=1e-5)


@PRECS
def test_tc_reference_selftest(snap, golden, prec):
    """The reference's noiseless self-test dictionary (T = 100, 10 ms grid
    steps) is nearly degenerate: the exact atom's runner-ups score 0.99997 and
    0.99999, below BF16 resolution, so the BF16 pre-selection can miss the
    exact atom.  Every pick must score within 1e-3 of the exact one."""
    atoms = golden["atoms_mrf"]
    params = golden["params_mrf"].reshape(-1, 4)
    idx = MATCH_SELFTEST_INDICES
    maps, got = run_match(snap, atoms[idx], atoms, params, precision=prec)
    a = atoms.astype(np.complex128)
    score = np.abs(np.einsum("vt,vt->v", np.conj(a[got]), a[idx]))
    print(f"exact picks {np.sum(got == idx)} of {len(idx)}, min score {score.min():.6f}")
    assert np.all(score >= 1 - LIMITS[prec][1])
    np.testing.assert_array_equal(maps[:, :4], params[got])
    assert snap.device_error(reset=True) == 0


IMAG = pytest.mark.parametrize("imag", [False, True], ids=["complex", "imag"])


def _flags(snap, imag):
    return snap.MATCH_IMAG_ATOMS if imag else 0


@PRECS
@IMAG
@pytest.mark.parametrize("T", [200, 1000])
def test_tc_global_vs_fp32(snap, T, prec, imag):
    atoms, params, natoms = _dictionary(snap, T, (0.8, 1.0, 1.2))
    img = _voxels(atoms, 900, 1)
    m32, i32 = run_match(snap, img, atoms, params, natoms=natoms)
    m16, i16 = run_match(snap, img, atoms, params, natoms=natoms, precision=prec, flags=_flags(snap, imag))
    compare(img, atoms, params, m32, i32, m16, i16, *LIMITS[prec])
    assert snap.device_error(reset=True) == 0


@PRECS
@IMAG
def test_tc_b1map_vs_fp32(snap, prec, imag):
    b1s = np.float32([0.6, 0.75, 0.9, 1.05, 1.2, 1.35])
    atoms, params, natoms = _dictionary(snap, 300, b1s, nt1=16, nt2=14)
    nvox = 1500
    img = _voxels(atoms, nvox, 2)
    b1map = np.random.default_rng(3).uniform(0.5, 1.5, nvox).astype(np.float32)
    b1map[:4] = [0.0, 0.675, 11.0, np.nan]
    m32, i32 = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map)
    m16, i16 = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1map, precision=prec,
                         flags=_flags(snap, imag))
    assert np.all(i16 // natoms == i32 // natoms)
    compare(img, atoms, params, m32, i32, m16, i16, *LIMITS[prec])
    assert snap.device_error(reset=True) == 0


@PRECS
@IMAG
def test_tc_ragged_tiles(snap, prec, imag):
    """Atom and voxel counts off the 128- and 256-wide tiles, K not a multiple of 64."""
    atoms, params, natoms = _dictionary(snap, 77, (1.0,))
    atoms, params = atoms[:131], params[:131]
    img = _voxels(atoms, 67, 8)
    m32, i32 = run_match(snap, img, atoms, params)
    m16, i16 = run_match(snap, img, atoms, params, precision=prec, flags=_flags(snap, imag))
    compare(img, atoms, params, m32, i32, m16, i16, min_agree=min(0.97, LIMITS[prec][0]),
            max_loss=LIMITS[prec][1])
    assert snap.device_error(reset=True) == 0


@PRECS
def test_tc_zero_nan_and_duplicate_atoms(snap, prec):
    atoms, params, natoms = _dictionary(snap, 64, (1.0,))
    atoms = atoms.copy()
    atoms[7] = atoms[3]
    img = np.zeros((5, atoms.shape[1]), np.complex64)
    img[0] = atoms[3] * (0.5 - 0.2j)
    img[2] = np.nan
    img[3] = atoms[7]
    maps, got = run_match(snap, img, atoms, params, precision=prec)
    assert got[0] == 3 and got[3] == 3
    assert got[1] == 0 and maps[1, 4] == 0
    assert got[2] == 0 and maps[2, 4] == 0
    assert snap.device_error(reset=True) == 0


@pytest.mark.parametrize("prec", [BF16, FP16], ids=["bf16", "fp16"])
def test_tc_imag_flag_on_complex_atoms_fails_loudly(snap, prec):
    """SNAPMRF_MATCH_IMAG_ATOMS asserts Re d = 0; atoms with a real part turn
    the maps to NaN and set the device error word (7) instead of matching
    against half of each atom."""
    atoms, params, natoms = _dictionary(snap, 64, (1.0,))
    atoms = atoms.copy()
    atoms[5] = atoms[5] + 0.01
    img = _voxels(atoms, 40, 9)
    maps, _ = run_match(snap, img, atoms, params, precision=prec, flags=snap.MATCH_IMAG_ATOMS)
    assert np.all(np.isnan(maps))
    assert snap.device_error(reset=True) == 7
    assert snap.device_error() == 0
    maps, _ = run_match(snap, img, atoms, params, precision=prec)
    assert np.all(np.isfinite(maps))


@pytest.mark.parametrize("prec", [BF16, FP16], ids=["bf16", "fp16"])
@pytest.mark.parametrize("normalize", [False, True])
def test_dictionary_packs_atoms_for_matching(snap, prec, normalize):
    """MRF_dict(d_packed=...) writes each atom's imaginary part as one 16-bit
    row (the matching operand); MRF_match(packed_atoms=...) then skips its own
    packing and gives identical maps and indices."""
    import torch
    T = 300
    h = mrf_schedule(T, seed=21)
    b1s = (0.9, 1.0, 1.1)
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 800, 12)
            for a in np.geomspace(100, 3000, 14) if a > b]
    params = np.array(rows, np.float32)
    NATOMS = params.shape[0]
    natoms = NATOMS // len(b1s)
    pitch = snap.packed_pitch(T)
    assert pitch % 64 == 0 and pitch >= T
    flags = snap.DICT_ALL_B1_BLOCKS | (snap.DICT_NORMALIZE if normalize else 0)
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.empty((NATOMS, T, 2), device="cuda")
    d_packed = torch.full((NATOMS, pitch), 12345, dtype=torch.int16, device="cuda")
    snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, 20, "epg_fisp", flags=flags,
                  d_packed=d_packed, packed_precision=prec)
    torch.cuda.synchronize()
    a = d_atoms.cpu().numpy()
    assert np.all(a[..., 0] == 0)
    dt = torch.float16 if prec == FP16 else torch.bfloat16
    want = torch.zeros((NATOMS, pitch), dtype=dt)
    want[:, :T] = torch.from_numpy(a[..., 1]).to(dt)
    assert torch.equal(d_packed.cpu().view(dt), want)
    atoms = (a[..., 0] + 1j * a[..., 1]).astype(np.complex64)
    img = _voxels(atoms, 700, 22)
    b1map = np.random.default_rng(23).uniform(0.85, 1.15, 700).astype(np.float32)
    runs = []
    for packed in (None, d_packed):
        d_maps = torch.full((700, 5), -7.0, device="cuda")
        d_index = torch.full((700,), -1, dtype=torch.int64, device="cuda")
        snap.MRF_match(d_maps, img, d_atoms, d_params, T, T, NATOMS, natoms, 700, in_b1map=b1map,
                       precision=prec, flags=snap.MATCH_IMAG_ATOMS, d_index=d_index, img_stride=T,
                       packed_atoms=packed)
        torch.cuda.synchronize()
        runs.append((d_maps.cpu().numpy(), d_index.cpu().numpy()))
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert snap.device_error(reset=True) == 0


def test_packed_atoms_are_rejected_where_they_do_not_apply(snap):
    import torch
    T = 40
    h = mrf_schedule(T, seed=24)
    params = np.array([(500.0, 50.0, 0.0, 1.0), (900.0, 80.0, 0.0, 1.0)], np.float32)
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.empty((2, T, 2), device="cuda")
    d_packed = torch.empty((2, snap.packed_pitch(T)), dtype=torch.int16, device="cuda")
    with pytest.raises(snap.SnapMRFError):   # complex recursion: atoms not purely imaginary
        snap.MRF_dict(d_atoms, d_params, h, T, T, 2, 2, 4, 10, "epg_ssfp", d_packed=d_packed,
                      packed_precision=FP16)
    with pytest.raises(snap.SnapMRFError):   # FP8 has no packed form
        snap.MRF_dict(d_atoms, d_params, h, T, T, 2, 2, 4, 10, "epg_fisp", d_packed=d_packed,
                      packed_precision=FP8)
    snap.MRF_dict(d_atoms, d_params, h, T, T, 2, 2, 4, 10, "epg_fisp", d_packed=d_packed, packed_precision=FP16)
    img = np.ones((3, T), np.complex64)
    d_maps = torch.empty((3, 5), device="cuda")
    with pytest.raises(snap.SnapMRFError):   # packed atoms need the imaginary-atom form
        snap.MRF_match(d_maps, img, d_atoms, d_params, T, T, 2, 2, 3, precision=FP16, packed_atoms=d_packed)


def test_bounded_wait_runs_out_and_reports(snap):
    """The wait primitive of the tensor-core kernels (an mbarrier wait bounded
    by %globaltimer) made to run out: one warp waits 2 ms on an mbarrier that
    nothing arrives on, gives up, returns, and the device error word reads
    10; the device keeps working (a tensor-core match afterwards runs clean
    and agrees with FP32)."""
    import time
    import torch
    assert snap.device_error(reset=True) == 0
    t0 = time.perf_counter()
    snap.selftest_bounded_wait(2000)
    torch.cuda.synchronize()
    took = time.perf_counter() - t0
    assert snap.device_error(reset=True) == 10
    assert took < 5.0
    assert snap.device_error(reset=True) == 0
    with pytest.raises(snap.SnapMRFError, match="limit must be"):
        snap.selftest_bounded_wait(0)
    atoms, params, natoms = _dictionary(snap, 128, [1.0])
    img = _voxels(atoms, 300, 31)
    m32, i32 = run_match(snap, img, atoms, params)
    m16, i16 = run_match(snap, img, atoms, params, precision=FP16)
    assert snap.device_error(reset=True) == 0
    compare(img, atoms, params, m32, i32, m16, i16)
