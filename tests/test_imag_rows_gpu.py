"""Imaginary rows (DICT_IMAG_ROWS, MATCH_IMAG_ROWS, START_IMAG_ROWS): the
zero-phase FISP dictionary stored as FP32 rows of Im(atom) instead of complex
rows whose real parts are zeros.  Criteria, each bit for bit:
  - the rows equal the imaginary parts of the complex dictionary, with the
    same norms and the same 16-bit operand, as generated and normalised;
  - BF16 / FP16 matching with the packed operand (the rows read only by the
    FP32 rescoring) gives the same atom indices and (T1, T2, B0, B1), PD
    within 1e-6 (the rescoring's sums run in another order);
  - the sub-grid start gives the same (T1, T2) and moves the same voxels;
and the forms that would read the rows as complex atoms refuse them.
"""
import numpy as np
import pytest

from cases import mrf_schedule
from gpu_util import torch_cuda

pytestmark = pytest.mark.gpu


def _inputs(T=300, b1s=(0.9, 0.95, 1.0, 1.05, 1.1), seed=43):
    h = mrf_schedule(T, seed=seed)
    t1 = np.array([150 * 1.05 ** k for k in range(60)], np.float32)
    t2 = np.array([15 * 1.05 ** k for k in range(60)], np.float32)
    rows = [(a, b, 0.0, d) for d in b1s for b in t2 for a in t1 if a > b]
    params = np.array(rows, np.float32)
    return h, params, params.shape[0] // len(b1s)


def _dict(snap, torch, h, params, natoms, flags, prec, rows):
    T = h.shape[1]
    NATOMS = params.shape[0]
    d_params = torch.from_numpy(params).cuda()
    shape = (NATOMS, T) if rows else (NATOMS, T, 2)
    d_atoms = torch.full(shape, 5.0, dtype=torch.float32, device="cuda")
    d_norms = torch.full((NATOMS,), -1.0, dtype=torch.float32, device="cuda")
    d_packed = torch.full((NATOMS, snap.packed_pitch(T)), 3, dtype=torch.int16, device="cuda")
    snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, 30, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS | flags | (snap.DICT_IMAG_ROWS if rows else 0),
                  d_norms=d_norms, d_packed=d_packed, packed_precision=prec)
    return d_params, d_atoms, d_norms, d_packed


@pytest.mark.parametrize("mode", ["operand", "normalize", "raw"])
def test_imag_rows_equal_the_complex_dictionary(snap, mode):
    torch = torch_cuda()
    h, params, natoms = _inputs()
    flags = {"operand": snap.DICT_NORMALIZE_OPERAND, "normalize": snap.DICT_NORMALIZE, "raw": 0}[mode]
    _, a_c, n_c, p_c = _dict(snap, torch, h, params, natoms, flags, snap.PREC_BF16, rows=False)
    _, a_r, n_r, p_r = _dict(snap, torch, h, params, natoms, flags, snap.PREC_BF16, rows=True)
    torch.cuda.synchronize()
    assert torch.all(a_c[..., 0] == 0)
    assert torch.equal(a_r, a_c[..., 1])
    assert torch.equal(n_r, n_c)
    assert torch.equal(p_r, p_c)


def test_imag_rows_refused_where_the_atoms_are_complex(snap):
    torch = torch_cuda()
    h, params, natoms = _inputs(T=64, b1s=(1.0,))
    T = h.shape[1]
    NATOMS = params.shape[0]
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.empty((NATOMS, T, 2), dtype=torch.float32, device="cuda")
    for echo in ("epg_ssfp", "roa_ssfp", "epg_se"):
        with pytest.raises(snap.SnapMRFError, match="IMAG_ROWS"):
            snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, 20, echo,
                          flags=snap.DICT_IMAG_ROWS)
    d_maps = torch.empty((16, 5), dtype=torch.float32, device="cuda")
    d_img = torch.zeros((16, T, 2), dtype=torch.float32, device="cuda")
    for prec in (snap.PREC_FP32, snap.PREC_BF16):
        # FP32 reads the atoms themselves; BF16 without the packed operand packs them
        with pytest.raises(snap.SnapMRFError, match="IMAG_ROWS"):
            snap.MRF_match(d_maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, 16, precision=prec,
                           flags=snap.MATCH_IMAG_ATOMS | snap.MATCH_IMAG_ROWS)


@pytest.mark.parametrize("prec_name", ["bf16", "fp16"])
def test_imag_rows_match_and_start_like_complex_rows(snap, prec_name):
    torch = torch_cuda()
    prec = snap.PREC_FP16 if prec_name == "fp16" else snap.PREC_BF16
    h, params, natoms = _inputs()
    T = h.shape[1]
    NATOMS = params.shape[0]
    d_params, a_c, n_c, p_c = _dict(snap, torch, h, params, natoms, snap.DICT_NORMALIZE_OPERAND, prec, rows=False)
    _, a_r, n_r, p_r = _dict(snap, torch, h, params, natoms, snap.DICT_NORMALIZE_OPERAND, prec, rows=True)
    rng = np.random.default_rng(44)
    nvox = 4000
    # voxels off the grid: the atoms between grid points, by the product's own recursion
    vp = np.stack([rng.uniform(250, 3000, nvox), rng.uniform(25, 250, nvox), np.zeros(nvox),
                   rng.uniform(0.92, 1.08, nvox)], 1).astype(np.float32)
    vp[:, 1] = np.minimum(vp[:, 1], vp[:, 0] / 3)
    d_sig = torch.empty((nvox, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_sig, torch.from_numpy(vp).cuda(), h, T, T, nvox, 1, 4, 30, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS)
    sig = d_sig.cpu().numpy()
    x = (sig[..., 0] + 1j * sig[..., 1]) * (rng.uniform(0.5, 1, nvox) * np.exp(1j * rng.uniform(0, 6.28, nvox)))[:, None]
    sd = 0.02 * np.linalg.norm(x, axis=1, keepdims=True) / np.sqrt(T)
    x = x + sd / np.sqrt(2) * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    d_img = torch.from_numpy(x.astype(np.complex64).view(np.float32)).cuda().reshape(nvox, T, 2)
    d_b1 = torch.from_numpy(vp[:, 3].copy()).cuda()
    out = {}
    for rows, atoms in ((False, a_c), (True, a_r)):
        d_maps = torch.full((nvox, 5), -1.0, dtype=torch.float32, device="cuda")
        d_index = torch.full((nvox,), -2, dtype=torch.int64, device="cuda")
        snap.MRF_match(d_maps, d_img, atoms, d_params, T, T, NATOMS, natoms, nvox, in_b1map=d_b1,
                       precision=prec, d_index=d_index, packed_atoms=p_c if not rows else p_r,
                       atom_norms=n_c if not rows else n_r,
                       flags=snap.MATCH_IMAG_ATOMS | snap.MATCH_ASSUME_UNIFORM_B1 | (snap.MATCH_IMAG_ROWS if rows else 0))
        matched = d_maps.clone()
        count = torch.zeros(1, dtype=torch.int32, device="cuda")
        snap.refine_start(d_maps, d_img, atoms, d_params, d_index, T, NATOMS, natoms, nvox, d_b1map=d_b1,
                          imag_atoms=True, imag_rows=rows, d_count=count)
        torch.cuda.synchronize()
        out[rows] = (matched.cpu().numpy(), d_index.cpu().numpy(), d_maps.cpu().numpy(), int(count.item()))
    (m_c, i_c, s_c, c_c), (m_r, i_r, s_r, c_r) = out[False], out[True]
    np.testing.assert_array_equal(i_r, i_c)
    np.testing.assert_array_equal(m_r[:, :4], m_c[:, :4])
    # PD: the rescoring's inner products summed four samples per load from
    # the rows (two from complex rows), so rounding only
    np.testing.assert_allclose(m_r[:, 4], m_c[:, 4], rtol=1e-6)
    np.testing.assert_array_equal(s_r[:, :4], s_c[:, :4])
    assert c_r == c_c and c_c > 0.7 * nvox  # (voxels next to the small grid's edges keep their grid point)
