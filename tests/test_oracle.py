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


@pytest.mark.parametrize("echo", ["epg_fisp", "epg_sr"])
def test_oracle_forward_mode_matches_dictionary_and_differences(oracle, echo):
    """The FP64 dual-number recursion (the derivative oracle) gives the
    dictionary oracle's atoms, and its tangents agree with central
    differences of itself."""
    rng = np.random.default_rng(0)
    T, w = 300, 30
    a = np.deg2rad(10 + 50 * np.abs(np.sin(np.pi * np.arange(T) / 250)))
    tr = rng.uniform(11, 15, T)
    h = np.array([a, np.zeros(T), tr, tr / 2], np.float32)
    th = (900.0, 60.0, 0.95)
    s, _, _, _ = oracle.fisp_jvp(th, (0, 0, 0), h, nstates=w, echo=echo)
    params = np.array([[th[0], th[1], 0, th[2]]], np.float32)
    at = oracle.dict_atoms(echo, params, h, T, nstates=w, flags=oracle.ALL_B1_BLOCKS)[0]
    assert np.abs(at.real).max() == 0
    assert np.abs(at.imag - s).max() < 1e-6 * np.abs(s).max()
    y = s * 0.8j + 0.01 * rng.standard_normal(T)
    for i, step in ((0, 1.0), (1, 0.1), (2, 1e-4)):
        tg = [0.0, 0.0, 0.0]
        tg[i] = 1.0
        _, ds, L, dL = oracle.fisp_jvp(th, tg, h, nstates=w, echo=echo, y=y)
        tp, tm = list(th), list(th)
        tp[i] += step
        tm[i] -= step
        sp, _, Lp, _ = oracle.fisp_jvp(tp, (0, 0, 0), h, nstates=w, echo=echo, y=y)
        sm, _, Lm, _ = oracle.fisp_jvp(tm, (0, 0, 0), h, nstates=w, echo=echo, y=y)
        assert np.abs(ds - (sp - sm) / (2 * step)).max() < 1e-5 * np.abs(ds).max()
        assert abs(dL - (Lp - Lm) / (2 * step)) < 1e-5 * abs(dL) + 1e-9
    v = rng.standard_normal(T)
    _, ds, _, _ = oracle.fisp_jvp(th, (0, 0, 0), h, nstates=w, echo=echo, dalpha=v)
    hp, hm = h.astype(np.float64).copy(), h.astype(np.float64).copy()
    # alpha is read as float32: difference along v with a step float32 resolves
    e = 1e-3
    hp[0] += e * v
    hm[0] -= e * v
    sp, _, _, _ = oracle.fisp_jvp(th, (0, 0, 0), hp.astype(np.float32), nstates=w, echo=echo)
    sm, _, _, _ = oracle.fisp_jvp(th, (0, 0, 0), hm.astype(np.float32), nstates=w, echo=echo)
    dv = (hp[0].astype(np.float32).astype(np.float64) - hm[0].astype(np.float32)) / (2 * e)
    # the float32 rounding of the perturbed angles changes the effective direction
    _, ds2, _, _ = oracle.fisp_jvp(th, (0, 0, 0), h, nstates=w, echo=echo, dalpha=dv)
    assert np.abs(ds2 - (sp - sm) / (2 * e)).max() < 1e-4 * np.abs(ds2).max()
    assert np.abs(ds2 - ds).max() < 1e-3 * np.abs(ds).max()


def _with_spectrum(rng, T, n, s):
    """A T x n complex matrix with singular values s (returned as n atoms)."""
    qa, _ = np.linalg.qr(rng.standard_normal((T, len(s))) + 1j * rng.standard_normal((T, len(s))))
    qb, _ = np.linalg.qr(rng.standard_normal((n, len(s))) + 1j * rng.standard_normal((n, len(s))))
    return ((qa * s) @ np.conj(qb).T).T


def test_oracle_svd_rank_rule(oracle):
    """nDictSpace = sum(cumsum(s.^2)./sum(s.^2) <= sfrac) on block 0, kept for
    every block (matlab/MRF_dict_B1.m:143-150)."""
    rng = np.random.default_rng(0)
    s0 = np.sqrt([0.5, 0.3, 0.15, 0.05])          # cumulative energy 0.5 0.8 0.95 1.0
    s1 = np.sqrt([0.9, 0.06, 0.03, 0.01])
    atoms = np.concatenate([_with_spectrum(rng, 12, 9, s0), _with_spectrum(rng, 12, 9, s1)])
    for sfrac, r in [(0.49, 0), (0.6, 1), (0.9, 2), (0.97, 3), (0.9999, 3)]:
        basis, coeffs, rank, sv = oracle.svd_compress(atoms, 9, sfrac=sfrac)
        assert rank == r, (sfrac, rank)
        assert basis.shape == (2, r, 12) and coeffs.shape == (18, r)
    np.testing.assert_allclose(sv[0, :4], s0, rtol=1e-12)
    np.testing.assert_allclose(sv[1, :4], s1, rtol=1e-12)
    # the coordinates hold the kept energy of each block
    basis, coeffs, rank, sv = oracle.svd_compress(atoms, 9, sfrac=0.9)
    for b in range(2):
        np.testing.assert_allclose(np.sum(np.abs(coeffs[9 * b:9 * b + 9]) ** 2), np.sum(sv[b, :2] ** 2),
                                   rtol=1e-12)


def test_oracle_compressed_match_full_rank_is_exact(oracle):
    """At full rank the projection is exact, so compressed matching equals
    the oracle's MRF_match (picks and PD)."""
    rng = np.random.default_rng(1)
    T, natoms, nb, nvox = 40, 16, 3, 50
    atoms = rng.standard_normal((nb * natoms, T)) + 1j * rng.standard_normal((nb * natoms, T))
    atoms /= np.linalg.norm(atoms, axis=1, keepdims=True)
    params = np.array([(100.0 + i, 10.0 + i % 7, 0.0, 0.8 + 0.2 * (i // natoms)) for i in range(nb * natoms)],
                      np.float32)
    img = (atoms[rng.integers(0, nb * natoms, nvox)] * 2.0
           + 0.05 * (rng.standard_normal((nvox, T)) + 1j * rng.standard_normal((nvox, T))))
    b1 = params[rng.integers(0, nb * natoms, nvox), 3] + rng.uniform(-0.05, 0.05, nvox).astype(np.float32)
    basis, coeffs, rank, _ = oracle.svd_compress(atoms, natoms, rank=natoms)
    mc, ic = oracle.match_compressed(img, basis, coeffs, params, natoms, b1map=b1)
    m, i = oracle.match(img.astype(np.complex64), atoms.astype(np.complex64), params, T, natoms=natoms,
                        b1map=b1)
    np.testing.assert_array_equal(ic, i)
    np.testing.assert_allclose(mc[:, 4], m[:, 4], rtol=1e-5)


def test_trans_params_restatement_matches_the_product_table(snap):
    """The oracle's numpy trans_params (used by the CPU arm so that it loads
    no product code) gives the table of the product's host code, which is
    bit-identical to the reference's own (test_host)."""
    from oracle import oracle as orc
    for t1, t2, b0, b1 in [(np.arange(100, 3001, 100), np.arange(20, 301, 10), [0], [1]),
                           ([100 * 1.05 ** k for k in range(81)], [10 * 1.05 ** k for k in range(109)], [0],
                            [0.6 + 0.02 * k for k in range(41)]),
                           ([300, 200, 100], [150, 50], [-5, 0, 5], [0.9, 1.1])]:
        t1, t2, b0, b1 = (np.asarray(v, np.float32) for v in (t1, t2, b0, b1))
        np.testing.assert_array_equal(orc.trans_params(t1, t2, b0, b1), snap.trans_params(t1, t2, b0, b1))


def test_fp64_gauss_newton_converges_to_the_noiseless_truth(oracle):
    """The FP64 refinement (the checker of the GPU refinement's maps) walks
    from a 5 % grid offset to the parameters a noiseless voxel was made with."""
    from cases import mrf_schedule
    T, w = 200, 20
    h = mrf_schedule(T, seed=3)
    for t1, t2, b1 in [(900.0, 60.0, 1.0), (1500.0, 200.0, 0.85)]:
        s, _, _, _ = oracle.fisp_jvp((t1, t2, b1), (0, 0, 0), h, nstates=w)
        x = (0.7 - 0.4j) * 1j * s
        g1, g2, pd = oracle.refine_gn_f64((t1 * 1.05, t2 / 1.05, b1), x, h, nstates=w)
        assert abs(g1 - t1) < 1e-6 * t1 and abs(g2 - t2) < 1e-6 * t2
        assert abs(pd - abs(0.7 - 0.4j) * np.linalg.norm(s)) < 1e-9 * pd


def test_ssfp_forward_mode_matches_dictionary_and_differences(oracle):
    """The FP64 forward mode of the bSSFP recursion: its signal equals the
    oracle's epg_ssfp atoms (one B1 block, before normalisation) and each
    tangent equals central differences of the signal (T1, T2, B0, B1)."""
    from cases import c4_ssfp_csv
    T, w = 80, 20
    h = c4_ssfp_csv(T, seed=9)
    th = (900.0, 70.0, 13.0, 1.1)
    s, _ = oracle.ssfp_jvp(th, (0, 0, 0, 0), h, nstates=w)
    params = np.array([[th[0], th[1], th[2], th[3]]], np.float32)
    ref, norms = oracle.dict_atoms("epg_ssfp", params, h, T, nstates=w, return_norms=True)
    np.testing.assert_allclose(s / np.linalg.norm(s), ref[0], atol=2e-6)
    for j, step in enumerate((1e-3 * th[0], 1e-3 * th[1], 1e-2, 1e-4)):
        tg = [0.0] * 4
        tg[j] = 1.0
        _, ds = oracle.ssfp_jvp(th, tg, h, nstates=w)
        tp, tm = list(th), list(th)
        tp[j] += step
        tm[j] -= step
        fd = (oracle.ssfp_jvp(tp, (0, 0, 0, 0), h, nstates=w)[0] -
              oracle.ssfp_jvp(tm, (0, 0, 0, 0), h, nstates=w)[0]) / (2 * step)
        err = np.abs(ds - fd).max() / np.abs(fd).max()
        assert err < 1e-5, (j, err)
