"""The oracle itself, pinned to the reference's golden vectors (CPU only)."""
import numpy as np
import pytest

from cases import MATCH_SELFTEST_INDICES, REFERENCE_DICT_CASES, reference_case_inputs


@pytest.mark.parametrize("name", list(REFERENCE_DICT_CASES))
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_oracle_reproduces_reference_goldens(oracle, golden, name, precision):
    echo, h_mrf, params, NATOMS, natoms, nreps = reference_case_inputs(name, golden)
    atoms = oracle.dict_atoms(echo, params, h_mrf, nreps, natoms=natoms, nstates=101,
                              precision=precision)
    ref = golden["atoms_" + name].astype(np.complex128)
    assert atoms.shape == ref.shape
    d = np.abs(atoms - ref)
    # the goldens hold the reference's FP32 GPU results (__sincosf, cuBLAS):
    # the restatement agrees to better than 1e-6 in every element
    assert d.max() < 1e-6, (name, d.max())


def test_oracle_grid_restatement_matches_reference_parser(golden):
    from cases import GRID_CASES, reference_grid
    for i, (a, b, c, d) in enumerate(GRID_CASES):
        p, _ = reference_grid(a, b, c, d)
        np.testing.assert_array_equal(p, golden[f"grid_{i}"].reshape(-1, 4))


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_oracle_matching_selftest(oracle, golden, precision):
    """src/functions.cu:1720-1824: noiseless voxels copied from atoms_mrf.ra
    are matched back to exactly their own parameters."""
    atoms = golden["atoms_mrf"]
    params = golden["params_mrf"].reshape(-1, 4)
    idx = MATCH_SELFTEST_INDICES
    img = atoms[idx]
    maps, got = oracle.match(img, atoms, params, atoms.shape[1], precision=precision)
    np.testing.assert_array_equal(got, idx)
    diff = np.abs(maps[:, :4] - params[idx]).sum()
    assert diff < 1e-6


def test_oracle_f32_tracks_f64(oracle):
    """FP32 restatement vs FP64 on a long FISP schedule: the recursion is
    contractive, so FP32 stays close."""
    from cases import mrf_schedule
    h = mrf_schedule(300, seed=3)
    params = np.array([[t1, t2, 0, 1] for t1 in (300.0, 1000.0, 2500.0) for t2 in (30.0, 100.0)],
                      np.float32)
    a64 = oracle.dict_atoms("epg_fisp", params, h, 300, nstates=20, precision="f64")
    a32 = oracle.dict_atoms("epg_fisp", params, h, 300, nstates=20, precision="f32")
    rel = np.abs(a32 - a64).max(axis=1) / np.abs(a64).max(axis=1)
    assert rel.max() < 1e-5


def test_oracle_b1_blocks_and_normalize(oracle):
    """ALL_B1_BLOCKS generates block j with alpha * b1_j; NORMALIZE gives unit norms."""
    from cases import mrf_schedule
    h = mrf_schedule(50, seed=1)
    base = np.array([[800.0, 80.0, 0, 0]], np.float32)
    params = np.concatenate([base.copy() for _ in range(3)])
    params[:, 3] = [0.8, 1.0, 1.2]
    atoms, norms = oracle.dict_atoms("epg_fisp", params, h, 50, natoms=1, nstates=20,
                                     flags=oracle.ALL_B1_BLOCKS | oracle.NORMALIZE, return_norms=True)
    assert atoms.shape == (3, 50)
    np.testing.assert_allclose(np.linalg.norm(atoms, axis=1), 1.0, rtol=1e-12)
    h2 = h.copy()
    h2[0] = (h[0] * np.float32(0.8)).astype(np.float32)
    single = oracle.dict_atoms("epg_fisp", base[:, :] + [0, 0, 0, 1], h2, 50, nstates=20)
    np.testing.assert_allclose(atoms[0] * norms[0], single[0], rtol=1e-12, atol=1e-15)
