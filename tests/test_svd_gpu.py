"""Low-rank compression (snapmrf_svd_compress) and compressed matching against
the FP64 restatement of matlab/MRF_dict_B1.m:127-159 (oracle.svd_compress,
LAPACK's SVD per B1 block).  Criteria:
  - the sfrac rule gives the oracle's rank (energy fractions chosen midway
    between two cumulative values);
  - the singular values of every block within 1e-5 (relative) of LAPACK's
    for i < r;
  - the r-dimensional subspaces: ||U U^H - U_ref U_ref^H||_2 <= 1e-7 s_1 / s_r
    (the passes over the atoms are FP32: a direction is resolved to about
    1e-8 of the largest singular value);
  - the basis orthonormal to 1e-5 and the coordinates equal to U^H d
    (FP64, with the returned basis) to 1e-5 of the atom norm; rows / columns
    beyond r zero;
  - purely imaginary atoms: basis imaginary parts and coordinate real parts
    exactly 0;
  - compressed FP32 matching gives the oracle's compressed pick (same basis)
    wherever the FP64 compressed scores of the two picks differ by more than
    1e-5 (relative), else a pick within that of the best; PD within 1e-5;
  - compressed BF16 / FP16 (hi + lo split operands) with FP32 rescoring
    against the full atoms: >= 99 % argmax agreement with uncompressed FP32
    matching, every differing pick within 1e-3 of the best exact score; FP8
    (plain E4M3 coordinates) >= 95 % and 5e-3;
  - two calls with one seed give bit-identical bases.
"""
import numpy as np
import pytest

from cases import mrf_schedule
from gpu_util import run_dict, run_match, torch_cuda

pytestmark = pytest.mark.gpu
ERR_INVALID, ERR_UNSUPPORTED = 1, 7


@pytest.fixture(scope="module")
def oracle_mod():
    from oracle import oracle as o
    return o


def _dictionary(snap, T=400, b1s=(0.8, 1.0, 1.2), nt1=16, nt2=14, seed=3):
    h = mrf_schedule(T, seed=seed)
    rows = [(a, b, 0.0, d) for d in b1s for b in np.geomspace(10, 800, nt2)
            for a in np.geomspace(100, 3000, nt1) if a > b]
    params = np.array(rows, np.float32)
    natoms = params.shape[0] // len(b1s)
    atoms = run_dict(snap, "epg_fisp", params, h, T, natoms=natoms, nstates=20,
                     flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    return atoms, params, natoms


def _complexify(atoms, natoms, seed=5):
    """A general complex dictionary: per-atom phases and per-block phase ramps."""
    rng = np.random.default_rng(seed)
    T = atoms.shape[1]
    nb = atoms.shape[0] // natoms
    ph = rng.uniform(0, 2 * np.pi, atoms.shape[0])[:, None]
    ramp = np.repeat(rng.uniform(-0.02, 0.02, nb), natoms)[:, None] * np.arange(T)[None, :]
    c = np.abs(atoms) * np.exp(1j * (ph + ramp + 0.3 * np.sin(np.arange(T) / 17.0)))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    return c.astype(np.complex64)


def _voxels(atoms, params, natoms, n, seed, snr=40.0):
    rng = np.random.default_rng(seed)
    j = rng.integers(0, atoms.shape[0], n)
    s = atoms[j] * (rng.uniform(0.5, 1, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n)))[:, None]
    sig = np.linalg.norm(s, axis=1, keepdims=True) / np.sqrt(s.shape[1]) / snr
    s = s + sig / np.sqrt(2) * (rng.standard_normal(s.shape) + 1j * rng.standard_normal(s.shape))
    b1 = params[j, 3] + rng.uniform(-0.04, 0.04, n).astype(np.float32)
    return s.astype(np.complex64), b1.astype(np.float32)


def _sfrac_for(sv0, r):
    f = np.cumsum(sv0.astype(np.float64) ** 2) / np.sum(sv0.astype(np.float64) ** 2)
    return float(0.5 * (f[r - 1] + f[r]))


def _compress(snap, atoms, natoms, **kw):
    torch = torch_cuda()
    d = torch.from_numpy(np.ascontiguousarray(atoms, np.complex64).view(np.float32)).cuda()
    c = snap.svd_compress(d, atoms.shape[1], atoms.shape[0], natoms, **kw)
    torch.cuda.synchronize()
    B = c.basis.cpu().numpy()
    basis = (B[..., 0] + 1j * B[..., 1]).astype(np.complex128)
    Cf = c.coeffs.cpu().numpy()
    coeffs = (Cf[..., 0] + 1j * Cf[..., 1]).astype(np.complex128)
    return c, d, basis, coeffs


def _check_basis(atoms, natoms, c, basis, coeffs, ref_basis, ref_sv):
    r = c.rank
    nb = basis.shape[0]
    T = atoms.shape[1]
    assert np.all(basis[:, r:] == 0) and np.all(coeffs[:, r:] == 0)
    for b in range(nb):
        U = basis[b, :r, :T]
        np.testing.assert_allclose(U @ np.conj(U).T, np.eye(r), atol=1e-5)
        np.testing.assert_allclose(c.sv[b, :r], ref_sv[b, :r], rtol=1e-5)
        Pr = ref_basis[b].T @ np.conj(ref_basis[b])
        Pg = U.T @ np.conj(U)
        dist = np.linalg.norm(Pr - Pg, 2)
        print(f"block {b}: rank {r}, projector distance {dist:.2e}, sv {c.sv[b, :3]}")
        assert dist <= 1e-7 * ref_sv[b, 0] / ref_sv[b, r - 1]
        A = atoms[b * natoms:(b + 1) * natoms].astype(np.complex128)
        want = A @ np.conj(U).T
        got = coeffs[b * natoms:(b + 1) * natoms, :r]
        assert np.max(np.abs(got - want)) <= 1e-5


@pytest.mark.parametrize("target", [6, 12, 24])
def test_svd_imag_atoms_vs_lapack(snap, oracle_mod, target):
    atoms, params, natoms = _dictionary(snap)
    _, _, _, sv = oracle_mod.svd_compress(atoms, natoms, rank=1)
    sfrac = _sfrac_for(sv[0], target)
    ref_basis, ref_coeffs, r_ref, ref_sv = oracle_mod.svd_compress(atoms, natoms, sfrac=sfrac)
    assert r_ref == target
    c, _, basis, coeffs = _compress(snap, atoms, natoms, sfrac=sfrac, max_rank=32, imag_atoms=True)
    assert c.rank == r_ref
    B = c.basis.cpu().numpy()
    Cf = c.coeffs.cpu().numpy()
    assert np.all(B[..., 1] == 0) and np.all(Cf[..., 0] == 0)
    _check_basis(atoms, natoms, c, basis, coeffs, ref_basis, ref_sv)


@pytest.mark.parametrize("target", [8, 20])
def test_svd_complex_atoms_vs_lapack(snap, oracle_mod, target):
    atoms, params, natoms = _dictionary(snap)
    atoms = _complexify(atoms, natoms)
    _, _, _, sv = oracle_mod.svd_compress(atoms, natoms, rank=1)
    sfrac = _sfrac_for(sv[0], target)
    ref_basis, ref_coeffs, r_ref, ref_sv = oracle_mod.svd_compress(atoms, natoms, sfrac=sfrac)
    c, _, basis, coeffs = _compress(snap, atoms, natoms, sfrac=sfrac, max_rank=40)
    assert c.rank == r_ref == target
    _check_basis(atoms, natoms, c, basis, coeffs, ref_basis, ref_sv)


def test_svd_fixed_rank_deterministic(snap, oracle_mod):
    atoms, params, natoms = _dictionary(snap)
    c1, _, b1, k1 = _compress(snap, atoms, natoms, rank=10, max_rank=16, imag_atoms=True, seed=7)
    c2, _, b2, k2 = _compress(snap, atoms, natoms, rank=10, max_rank=16, imag_atoms=True, seed=7)
    assert c1.rank == c2.rank == 10
    assert np.array_equal(b1, b2) and np.array_equal(k1, k2)
    ref_basis, _, _, ref_sv = oracle_mod.svd_compress(atoms, natoms, rank=10)
    _check_basis(atoms, natoms, c1, b1, k1, ref_basis, ref_sv)


def test_svd_errors(snap):
    torch = torch_cuda()
    atoms, params, natoms = _dictionary(snap, T=120)
    d = torch.from_numpy(atoms.view(np.float32)).cuda()
    with pytest.raises(snap.SnapMRFError) as e:     # keeps no vector
        snap.svd_compress(d, 120, atoms.shape[0], natoms, sfrac=1e-6, max_rank=8)
    assert e.value.status == ERR_INVALID
    with pytest.raises(snap.SnapMRFError) as e:     # more than max_rank
        snap.svd_compress(d, 120, atoms.shape[0], natoms, sfrac=0.999999, max_rank=4)
    assert e.value.status == ERR_INVALID
    with pytest.raises(snap.SnapMRFError) as e:     # subspace above the bound
        snap.svd_compress(d, 120, atoms.shape[0], natoms, rank=4, max_rank=snap.SVD_MAX_SUBSPACE)
    assert e.value.status == ERR_INVALID


def _match(snap, img, d_atoms, params, T, NATOMS, natoms, b1, cmp, precision=0, flags=0, atoms_given=True):
    torch = torch_cuda()
    nvox = img.shape[0]
    d_maps = torch.full((nvox, 5), -7.0, dtype=torch.float32, device="cuda")
    d_index = torch.full((nvox,), -1, dtype=torch.int64, device="cuda")
    d_params = torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda()
    snap.MRF_match(d_maps, img, d_atoms if atoms_given else None, d_params, T, T, NATOMS, natoms, nvox,
                   in_b1map=b1, flags=flags | snap.MATCH_ASSUME_UNIFORM_B1, d_index=d_index,
                   precision=precision, compressed=cmp)
    torch.cuda.synchronize()
    assert snap.device_error(reset=True) == 0
    return d_maps.cpu().numpy(), d_index.cpu().numpy()


@pytest.mark.parametrize("imag", [True, False], ids=["imag", "complex"])
def test_compressed_fp32_vs_oracle(snap, oracle_mod, imag):
    atoms, params, natoms = _dictionary(snap)
    if not imag:
        atoms = _complexify(atoms, natoms)
    T = atoms.shape[1]
    img, b1 = _voxels(atoms, params, natoms, 3000, seed=11)
    c, d, basis, coeffs = _compress(snap, atoms, natoms, rank=12, max_rank=16, imag_atoms=imag)
    m, i = _match(snap, img, d, params, T, atoms.shape[0], natoms, b1, c,
                  flags=snap.MATCH_IMAG_ATOMS if imag else 0)
    r = c.rank
    mo, io = oracle_mod.match_compressed(img, basis[:, :r], coeffs[:, :r], params, natoms, b1map=b1)
    # FP64 compressed scores of both picks, in the bin each voxel was matched in
    bins = io // natoms
    assert np.all(i // natoms == bins)
    xc = np.einsum("vit,vt->vi", np.conj(basis[bins, :r]), img.astype(np.complex128))
    s = lambda g: np.abs(np.einsum("vi,vi->v", np.conj(coeffs[g, :r]), xc))
    s_o, s_g = s(io), s(i)
    rel = (s_o - s_g) / s_o
    diff = i != io
    print(f"compressed FP32: {diff.sum()} of {len(i)} picks differ, max rel gap {rel[diff].max() if diff.any() else 0:.2e}")
    assert np.all(rel[diff] <= 1e-5)
    np.testing.assert_array_equal(m[:, :4], params[i])
    np.testing.assert_allclose(m[:, 4], s_g, rtol=1e-5)


@pytest.mark.parametrize("prec", [1, 2, 3], ids=["bf16", "fp16", "fp8"])
def test_compressed_tc_rescored_vs_fp32(snap, prec):
    atoms, params, natoms = _dictionary(snap)
    T = atoms.shape[1]
    img, b1 = _voxels(atoms, params, natoms, 4000, seed=13)
    m32, i32 = run_match(snap, img, atoms, params, natoms=natoms, b1map=b1)
    c, d, basis, coeffs = _compress(snap, atoms, natoms, sfrac=0.99999, max_rank=48, imag_atoms=True)
    print("rank", c.rank)
    m, i = _match(snap, img, d, params, T, atoms.shape[0], natoms, b1, c, precision=prec,
                  flags=snap.MATCH_IMAG_ATOMS)
    sc = lambda g: np.abs(np.einsum("vt,vt->v", np.conj(atoms[g].astype(np.complex128)),
                                    img.astype(np.complex128)))
    agree = np.mean(i == i32)
    diff = i != i32
    rel = (sc(i32) - sc(i)) / sc(i32)
    print(f"compressed prec {prec}, rank {c.rank}: agreement {agree:.5f}, "
          f"max rel loss {rel[diff].max() if diff.any() else 0:.2e}")
    min_agree, max_loss = (0.95, 5e-3) if prec == 3 else (0.99, 1e-3)
    assert agree >= min_agree
    assert np.all(rel[diff] <= max_loss)
    np.testing.assert_array_equal(m[:, :4], params[i])
    same = ~diff
    np.testing.assert_allclose(m[same, 4], m32[same, 4], rtol=1e-5)


def test_compressed_tc_without_atoms(snap, oracle_mod):
    """No full atoms: the candidates are rescored in FP32 in the compressed
    space, so the picks follow the compressed FP32 form."""
    atoms, params, natoms = _dictionary(snap)
    T = atoms.shape[1]
    img, b1 = _voxels(atoms, params, natoms, 3000, seed=17)
    c, d, basis, coeffs = _compress(snap, atoms, natoms, rank=16, max_rank=16, imag_atoms=True)
    m32, i32 = _match(snap, img, d, params, T, atoms.shape[0], natoms, b1, c, flags=snap.MATCH_IMAG_ATOMS)
    m16, i16 = _match(snap, img, d, params, T, atoms.shape[0], natoms, b1, c, precision=2,
                      flags=snap.MATCH_IMAG_ATOMS, atoms_given=False)
    agree = np.mean(i16 == i32)
    print(f"compressed FP16 without atoms vs compressed FP32: {agree:.5f}")
    assert agree >= 0.99
    same = i16 == i32
    np.testing.assert_allclose(m16[same, 4], m32[same, 4], rtol=1e-5)


def test_compressed_match_errors(snap):
    torch = torch_cuda()
    atoms, params, natoms = _dictionary(snap, T=120)
    img, b1 = _voxels(atoms, params, natoms, 100, seed=3)
    c, d, _, _ = _compress(snap, atoms, natoms, rank=6, max_rank=8, imag_atoms=True)
    with pytest.raises(snap.SnapMRFError) as e:     # several blocks, no B1 map
        _match(snap, img, d, params, 120, atoms.shape[0], natoms, None, c)
    assert e.value.status == ERR_UNSUPPORTED
    d_params = torch.from_numpy(params).cuda()
    d_maps = torch.empty((100, 5), dtype=torch.float32, device="cuda")
    packed = torch.empty((atoms.shape[0], snap.packed_pitch(120)), dtype=torch.int16, device="cuda")
    with pytest.raises(snap.SnapMRFError) as e:     # packed operand and a basis
        snap.MRF_match(d_maps, img, d, d_params, 120, 120, atoms.shape[0], natoms, 100, in_b1map=b1,
                       precision=2, flags=snap.MATCH_IMAG_ATOMS, packed_atoms=packed, compressed=c)
    assert e.value.status == ERR_INVALID


def test_svd_blocks_smaller_than_subspace(snap, oracle_mod):
    """Blocks of 6 atoms with a subspace of 16 vectors (and 40 samples): the
    Gram matrices are rank-deficient, the directions beyond 6 drop out, and a
    fixed rank of 4 still matches LAPACK."""
    torch = torch_cuda()
    rng = np.random.default_rng(21)
    T, natoms, nb = 40, 6, 3
    atoms = rng.standard_normal((nb * natoms, T)) + 1j * rng.standard_normal((nb * natoms, T))
    atoms = (atoms / np.linalg.norm(atoms, axis=1, keepdims=True)).astype(np.complex64)
    c, _, basis, coeffs = _compress(snap, atoms, natoms, rank=4, max_rank=8)
    assert c.rank == 4
    ref_basis, _, _, ref_sv = oracle_mod.svd_compress(atoms, natoms, rank=4)
    assert np.all(np.isfinite(basis)) and np.all(np.isfinite(coeffs))
    np.testing.assert_allclose(c.sv[:, 6:], 0.0, atol=1e-3)
    _check_basis(atoms, natoms, c, basis, coeffs, ref_basis, ref_sv)
