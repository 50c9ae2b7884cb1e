"""Sub-grid start of the refinement (snapmrf_refine_start): the FP64
restatement checked against the recursion itself on the CPU, the CUDA kernel
against the restatement on the GPU, and the start followed by one refinement
pass against FP64 Gauss-Newton to convergence."""
import numpy as np
import pytest


def schedule(T, seed=0):
    rng = np.random.default_rng(seed)
    a = np.deg2rad(5 + 55 * np.abs(np.sin(np.pi * np.arange(T) / 230)) + rng.uniform(0, 3, T))
    a[0] = np.pi
    tr = rng.uniform(11, 15, T)
    return np.array([a, np.zeros(T), tr, tr / 2], np.float32)


def geometric(lo, hi):
    return np.array([lo * 1.05 ** k for k in range(400) if lo * 1.05 ** k <= hi], np.float32)


B1_BLOCKS = np.array([0.96, 0.98, 1.00, 1.02, 1.04], np.float32)


def make_case(orc, T, w, n, seed, with_map, noise=0.0, b1_blocks=B1_BLOCKS):
    """(h, params, natoms, unit-norm FP64 atoms, img, b1map or None, truth
    [n][3], rho): voxels at random off-grid (T1, T2) inside the grid; with a
    map, B1 off the block values too."""
    h = schedule(T, seed)
    t1, t2 = geometric(200.0, 3000.0), geometric(20.0, 400.0)
    b1 = b1_blocks if with_map else np.array([1.0], np.float32)
    params = orc.trans_params(t1, t2, [0.0], b1)
    natoms = params.shape[0] // len(b1)
    nthr = orc.max_threads()
    atoms = orc.dict_atoms("epg_fisp", params, h, T, natoms=natoms, nstates=w, precision="f64",
                           flags=orc.ALL_B1_BLOCKS | orc.NORMALIZE, nthreads=nthr)
    rng = np.random.default_rng(100 + seed)
    vt1 = rng.uniform(300.0, 2000.0, n)
    vt2 = np.minimum(rng.uniform(30.0, 250.0, n), vt1 / 3)
    vb1 = rng.uniform(0.965, 1.035, n) if with_map else np.ones(n)
    vp = np.stack([vt1, vt2, np.zeros(n), vb1], 1).astype(np.float32)
    # one block per voxel: each voxel's signal at its own B1
    sig = orc.dict_atoms("epg_fisp", vp, h, T, natoms=1, nstates=w, precision="f64",
                         flags=orc.ALL_B1_BLOCKS, nthreads=nthr)
    rho = rng.uniform(0.5, 2.0, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    img = sig * rho[:, None]
    if noise:
        sd = noise * np.linalg.norm(img, axis=1, keepdims=True) / np.sqrt(T)
        img = img + sd / np.sqrt(2) * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape))
    truth = vp[:, [0, 1, 3]].astype(np.float64)
    return h, params, natoms, atoms, img.astype(np.complex64), (vp[:, 3].copy() if with_map else None), truth, rho


def match_f64(orc, img, atoms, params, natoms, b1map):
    maps, idx = orc.match(img, atoms, params, atoms.shape[1], natoms=natoms, b1map=b1map,
                          nthreads=orc.max_threads())
    return maps, idx


@pytest.mark.parametrize("with_map", [False, True])
def test_start_oracle_lands_near_the_truth(oracle, with_map):
    """Noise-free voxels: where the true (T1, T2) lies within a grid step of
    the matched atom, the surrogate's optimum is within 1e-4 of it (5e-4 with
    the quadratic in B1 across blocks 0.02 apart; the grid point is up to
    2.5 % away); where the match landed more than a grid step
    from the truth (a correlated T1-T2 valley, or the B1 of the block away
    from the voxel's), the start may leave the stencil by up to half a step
    and is still nearer than the grid point."""
    T, w, n = 200, 20, 40
    h, params, natoms, atoms, img, b1map, truth, _ = make_case(oracle, T, w, n, seed=1, with_map=with_map)
    maps, idx = match_f64(oracle, img, atoms, params, natoms, b1map)
    grid_err = np.abs(maps[:, :2] / truth[:, :2] - 1)
    start, moved = oracle.refine_start_f64(maps, idx, atoms, params, img, natoms, b1map=b1map)
    assert moved.all()
    err = np.abs(start[:, :2] / truth[:, :2] - 1)
    steps = np.abs(np.log(maps[:, :2] / truth[:, :2]) / np.log(1.05))
    inside = (steps < 0.95).all(1)
    assert np.median(grid_err) > 5e-3 and inside.mean() >= 0.7
    assert err[inside].max() < (5e-4 if with_map else 1e-4), err[inside].max()
    assert (err.max(1) < grid_err.max(1)).all()
    np.testing.assert_array_equal(start[:, 2:], maps[:, 2:])


def test_start_oracle_leaves_edges_and_foreign_maps(oracle):
    """Voxels matched on the grid's edge (smallest T2, largest T1), with no
    index, or whose maps no longer hold the matched atom stay as they are."""
    T, w, n = 200, 20, 12
    h, params, natoms, atoms, img, _, truth, _ = make_case(oracle, T, w, n, seed=2, with_map=False)
    maps, idx = match_f64(oracle, img, atoms, params, natoms, None)
    t1, t2 = params[:natoms, 0], params[:natoms, 1]
    idx = idx.copy()
    maps = maps.copy()
    edge_t2 = int(np.flatnonzero(t2 == t2.min())[5])
    edge_t1 = int(np.flatnonzero((t1 == t1.max()) & (t2 == np.unique(t2)[10]))[0])
    for v, k in ((0, edge_t2), (1, edge_t1)):
        idx[v] = k
        maps[v, :4] = params[k]
    idx[2] = -1
    idx[3] = params.shape[0]
    maps[4, 0] *= 1.01
    start, moved = oracle.refine_start_f64(maps, idx, atoms, params, img, natoms)
    assert not moved[:5].any() and moved[5:].all()
    np.testing.assert_array_equal(start[:5], maps[:5])


def _device_case(snap, oracle, T, w, n, seed, with_map, noise):
    """The case with the dictionary, matching and signals of the product on
    the GPU; returns host copies of everything the start reads."""
    import torch
    h, params, natoms, _, img, b1map, truth, rho = make_case(oracle, T, w, 4, seed, with_map)
    NATOMS = params.shape[0]
    d_params = torch.from_numpy(params).cuda()
    d_atoms = torch.empty((NATOMS, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_atoms, d_params, h, T, T, NATOMS, natoms, 4, w, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE)
    rng = np.random.default_rng(200 + seed)
    vt1 = rng.uniform(300.0, 2000.0, n)
    vt2 = np.minimum(rng.uniform(30.0, 250.0, n), vt1 / 3)
    vb1 = rng.uniform(0.965, 1.035, n) if with_map else np.ones(n)
    vp = np.stack([vt1, vt2, np.zeros(n), vb1], 1).astype(np.float32)
    d_sig = torch.empty((n, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_sig, torch.from_numpy(vp).cuda(), h, T, T, n, 1, 4, w, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS)
    sig = d_sig.cpu().numpy()
    sig = sig[..., 0] + 1j * sig[..., 1]
    rho = rng.uniform(0.5, 2.0, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    x = sig * rho[:, None]
    if noise:
        sd = noise * np.linalg.norm(x, axis=1, keepdims=True) / np.sqrt(T)
        x = x + sd / np.sqrt(2) * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    x = x.astype(np.complex64)
    d_img = torch.from_numpy(x.view(np.float32).reshape(n, T, 2)).cuda()
    d_b1 = torch.from_numpy(vp[:, 3].copy()).cuda() if with_map else None
    d_maps = torch.empty((n, 5), dtype=torch.float32, device="cuda")
    d_index = torch.empty(n, dtype=torch.int64, device="cuda")
    snap.MRF_match(d_maps, d_img, d_atoms, d_params, T, T, NATOMS, natoms, n, in_b1map=d_b1,
                   d_index=d_index, flags=snap.MATCH_IMAG_ATOMS)
    torch.cuda.synchronize()
    return dict(h=h, params=params, natoms=natoms, NATOMS=NATOMS, d_params=d_params, d_atoms=d_atoms,
                d_img=d_img, d_b1=d_b1, d_maps=d_maps, d_index=d_index, img=x, truth=vp[:, [0, 1, 3]],
                b1map=None if d_b1 is None else vp[:, 3].copy())


@pytest.mark.gpu
@pytest.mark.parametrize("with_map", [False, True])
@pytest.mark.parametrize("imag", [True, False])
def test_start_kernel_matches_fp64_restatement(snap, oracle, with_map, imag):
    """Same FP32 atoms, maps and index: the CUDA start equals the FP64
    restatement to 2e-5 (relative) and moves exactly the same voxels; the
    complex-Gram form (imag=False) gives the imaginary-atom form's result."""
    import torch
    T, w, n = 400, 30, 300
    c = _device_case(snap, oracle, T, w, n, seed=3, with_map=with_map, noise=0.02)
    maps0 = c["d_maps"].cpu().numpy()
    idx = c["d_index"].cpu().numpy()
    atoms = c["d_atoms"].cpu().numpy()
    atoms = atoms[..., 0] + 1j * atoms[..., 1]
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    snap.refine_start(c["d_maps"], c["d_img"], c["d_atoms"], c["d_params"], c["d_index"], T, c["NATOMS"],
                      c["natoms"], n, d_b1map=c["d_b1"], imag_atoms=imag, d_count=count)
    got = c["d_maps"].cpu().numpy()
    want, moved = oracle.refine_start_f64(maps0, idx, atoms, c["params"], c["img"], c["natoms"],
                                          b1map=c["b1map"])
    assert moved.mean() > 0.9
    assert int(count.item()) == int(moved.sum())
    np.testing.assert_array_equal(got[~moved], maps0[~moved])
    np.testing.assert_allclose(got[moved, :2], want[moved, :2], rtol=2e-5)
    np.testing.assert_array_equal(got[:, 2:], maps0[:, 2:])


@pytest.mark.gpu
@pytest.mark.parametrize("T", [400, 401])
def test_start_from_imaginary_rows_equals_complex_rows(snap, oracle, T):
    """The start read from the FP32 Im rows (SNAPMRF_START_IMAG_ROWS: with an
    even T and row stride each lane copies its two samples of a row at once,
    with an odd T one at a time) equals the start read from the complex
    rows, bit for bit, and moves the voxels."""
    import torch
    w, n = 30, 300
    c = _device_case(snap, oracle, T, w, n, seed=5, with_map=True, noise=0.02)
    d_rows = torch.empty((c["NATOMS"], T), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_rows, c["d_params"], c["h"], T, T, c["NATOMS"], c["natoms"], 4, w, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS | snap.DICT_NORMALIZE | snap.DICT_IMAG_ROWS)
    maps0 = c["d_maps"].clone()
    out = []
    for atoms, rows in ((c["d_atoms"], False), (d_rows, True)):
        c["d_maps"].copy_(maps0)
        snap.refine_start(c["d_maps"], c["d_img"], atoms, c["d_params"], c["d_index"], T, c["NATOMS"],
                          c["natoms"], n, d_b1map=c["d_b1"], imag_atoms=True, imag_rows=rows)
        out.append(c["d_maps"].cpu().numpy())
    m0 = maps0.cpu().numpy()
    assert np.any(out[0][:, :2] != m0[:, :2], axis=1).mean() > 0.9
    np.testing.assert_array_equal(out[1], out[0])


@pytest.mark.gpu
def test_start_then_one_pass_reaches_the_converged_fit(snap, oracle):
    """Matched grid point -> start -> one refinement pass lands where FP64
    Gauss-Newton run to convergence from the grid point lands (median 2e-5,
    every voxel 5e-4), and a second pass moves no voxel by more than 1e-3."""
    import torch
    T, w, n = 400, 30, 200
    c = _device_case(snap, oracle, T, w, n, seed=4, with_map=True, noise=0.02)
    maps0 = c["d_maps"].cpu().numpy()
    snap.refine_start(c["d_maps"], c["d_img"], c["d_atoms"], c["d_params"], c["d_index"], T, c["NATOMS"],
                      c["natoms"], n, d_b1map=c["d_b1"], imag_atoms=True)
    snap.refine_gn(c["d_maps"], c["d_img"], c["h"], T, T, n, w, "epg_fisp", iterations=1, tol=0.0,
                   d_b1map=c["d_b1"])
    one = c["d_maps"].cpu().numpy()
    snap.refine_gn(c["d_maps"], c["d_img"], c["h"], T, T, n, w, "epg_fisp", iterations=1, tol=0.0,
                   d_b1map=c["d_b1"])
    two = c["d_maps"].cpu().numpy()
    assert np.abs(two[:, :2] / one[:, :2] - 1).max() < 1e-3
    ref = np.array([oracle.refine_gn_f64((maps0[v, 0], maps0[v, 1], c["b1map"][v]), c["img"][v].astype(np.complex128),
                                         c["h"], nstates=w)[:2] for v in range(n)])
    err = np.abs(one[:, :2] / ref - 1)
    assert np.median(err) < 2e-5 and err.max() < 5e-4, (np.median(err), err.max())
