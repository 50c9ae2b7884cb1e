"""The benchmark definition's other configurations as parity cases on the GPU:
C0 (EPG-FISP, T = 1000, w = 20, 837 atoms, 64x64 voxels) at full size, C3
(adjoint of 4096 atoms) against the FP64 forward-mode oracle, and C4 (SSFP
with B0 and B1 blocks, ROA with 100 isochromats, max-PD matching without a
B1 map) at reduced grid sizes.  Inputs are seeded synthetic stand-ins with
the configurations' shapes and distributions."""
import numpy as np
import pytest

from cases import c4_ssfp_csv, mrf_schedule, rel_err_per_atom
from gpu_util import run_dict, run_match

pytestmark = pytest.mark.gpu


def _grid(t1s, t2s, b0s=(0.0,), b1s=(1.0,)):
    rows = [(a, b, c, d) for d in b1s for c in b0s for b in t2s for a in t1s if a > b]
    return np.array(rows, np.float32)


def _scores(atoms, img):
    """|<atom, voxel>| for every pair, FP64: [nvox][natoms]."""
    return np.abs(img.astype(np.complex128) @ atoms.astype(np.complex128).conj().T)


def _assert_indices_equal_where_separated(idx, ref_idx, scores, gap=2e-5):
    """The FP32 matching against the FP64 oracle: every pick scores within
    `gap` (relative) of the exact best, a margin above the rounding of a
    1000-term FP32 dot product, and the picks are equal wherever the exact
    best leads the runner-up by more than that."""
    n = scores.shape[0]
    best = scores.max(axis=1)
    assert np.all(scores[np.arange(n), idx] >= best * (1 - gap))
    srt = np.sort(scores, axis=1)
    sure = (srt[:, -1] - srt[:, -2]) > gap * srt[:, -1]
    assert sure.mean() > 0.5
    np.testing.assert_array_equal(idx[sure], ref_idx[sure])


# --------------------------------------------------------------------------
# C0
# --------------------------------------------------------------------------

def test_c0_fisp_dictionary_and_matching(snap, oracle):
    T, w = 1000, 20
    h = mrf_schedule(T, seed=0)
    t1 = np.arange(100, 3001, 100, dtype=np.float32)
    t2 = np.arange(20, 301, 10, dtype=np.float32)
    params = snap.trans_params(t1, t2, np.zeros(1, np.float32), np.ones(1, np.float32))
    assert params.shape[0] == 837
    flags = snap.DICT_NORMALIZE
    atoms = run_dict(snap, "epg_fisp", params, h, T, nstates=w, flags=flags)
    ref = oracle.dict_atoms("epg_fisp", params, h, T, nstates=w, flags=oracle.NORMALIZE, nthreads=8)
    rel = rel_err_per_atom(atoms, ref)
    print(f"C0 dictionary: max rel vs FP64 oracle {rel.max():.2e}")
    assert rel.max() < 2e-5

    # 64 x 64 voxels at off-grid (T1, T2), M0 ~ U[0.5, 1], random phase, SNR 30
    rng = np.random.default_rng(0)
    n = 64 * 64
    vt1 = rng.uniform(100, 3000, n)
    vt2 = rng.uniform(20, 300, n)
    bad = vt2 >= vt1
    while bad.any():
        vt2[bad] = rng.uniform(20, 300, bad.sum())
        bad = vt2 >= vt1
    vp = np.stack([vt1, vt2, np.zeros(n), np.ones(n)], 1).astype(np.float32)
    sig = oracle.dict_atoms("epg_fisp", vp, h, T, nstates=w, nthreads=8)
    sig = sig * (rng.uniform(0.5, 1.0, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n)))[:, None]
    sigma = np.linalg.norm(sig, axis=1, keepdims=True) / np.sqrt(T) / 30.0
    img = (sig + sigma / np.sqrt(2) * (rng.standard_normal(sig.shape) + 1j * rng.standard_normal(sig.shape)))
    img = img.astype(np.complex64)

    maps, idx = run_match(snap, img, atoms, params)
    ref_maps, ref_idx = oracle.match(img, atoms, params, T, precision="f64", nthreads=8)
    scores = _scores(atoms, img)
    _assert_indices_equal_where_separated(idx, ref_idx, scores)
    np.testing.assert_allclose(maps[:, 4], ref_maps[:, 4], rtol=2e-5)
    for prec in (snap.PREC_BF16, snap.PREC_FP16):
        m2, i2 = run_match(snap, img, atoms, params, precision=prec)
        best = scores[np.arange(n), idx]
        picked = scores[np.arange(n), i2]
        agree = np.mean((i2 == idx) | (picked >= best * (1 - 1e-6)))
        print(f"C0 precision {prec}: agreement {agree:.5f}")
        assert agree >= 0.999


# --------------------------------------------------------------------------
# C3
# --------------------------------------------------------------------------

def test_c3_adjoint_4096_atoms(snap, oracle):
    import torch
    T, w, n = 1000, 50, 4096
    h = mrf_schedule(T, seed=3)
    rng = np.random.default_rng(3)
    t1 = np.exp(rng.uniform(np.log(200), np.log(4000), n))
    t2 = np.exp(rng.uniform(np.log(20), np.log(400), n))
    t2 = np.minimum(t2, 0.9 * t1)
    b1 = rng.uniform(0.7, 1.3, n)
    params = np.stack([t1, t2, np.zeros(n), b1], 1).astype(np.float32)
    d_p = torch.from_numpy(params).cuda()
    d_sig = torch.empty((n, T, 2), device="cuda")
    d_gp = torch.empty((n, 3), device="cuda")
    zeros = torch.zeros((n, T, 2), device="cuda")
    snap.epg_adjoint(d_p, h, T, T, n, zeros, d_gp, 4, w, "epg_fisp", d_signal=d_sig, checkpoint_every=32)
    y = (0.05 * (rng.standard_normal((n, T)) + 1j * rng.standard_normal((n, T)))).astype(np.complex64)
    d_y = torch.from_numpy(y.view(np.float32).reshape(n, T, 2)).cuda()
    d_g = 2 * (d_sig - d_y)                       # dL/ds of L = sum |s - y|^2
    d_ga = torch.empty((T,), device="cuda")
    snap.epg_adjoint(d_p, h, T, T, n, d_g, d_gp, 4, w, "epg_fisp", d_grad_alpha=d_ga, checkpoint_every=32)
    torch.cuda.synchronize()
    gp = d_gp.cpu().numpy()
    assert np.isfinite(gp).all() and np.isfinite(d_ga.cpu().numpy()).all()
    for i in rng.choice(n, 24, replace=False):
        th = (params[i, 0], params[i, 1], params[i, 3])
        for k, tg in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
            _, ds, _, want = oracle.fisp_jvp(th, tg, h, nstates=w, y=y[i])
            g = 2 * (oracle.fisp_jvp(th, (0, 0, 0), h, nstates=w)[0] - y[i].imag)
            scale = float(np.abs(g) @ np.abs(ds))
            assert abs(gp[i, k] - want) <= 1e-3 * abs(want) + 1e-4 * scale, (i, k, gp[i, k], want)
    # central differences of the FP64 loss at h = 1e-3 relative
    for i in rng.choice(n, 4, replace=False):
        th = np.array([params[i, 0], params[i, 1], params[i, 3]], np.float64)
        for k in range(3):
            step = 1e-3 * th[k]
            tp, tm = th.copy(), th.copy()
            tp[k] += step
            tm[k] -= step
            lp = oracle.fisp_jvp(tuple(tp), (0, 0, 0), h, nstates=w, y=y[i])[2]
            lm = oracle.fisp_jvp(tuple(tm), (0, 0, 0), h, nstates=w, y=y[i])[2]
            fd = (lp - lm) / (2 * step)
            tg = [0.0, 0.0, 0.0]
            tg[k] = 1.0
            _, ds, _, _ = oracle.fisp_jvp(tuple(th), tuple(tg), h, nstates=w)
            g = 2 * (oracle.fisp_jvp(tuple(th), (0, 0, 0), h, nstates=w)[0] - y[i].imag)
            scale = float(np.abs(g) @ np.abs(ds))
            assert abs(gp[i, k] - fd) <= 2e-3 * abs(fd) + 1e-4 * scale, (i, k, gp[i, k], fd)


# --------------------------------------------------------------------------
# C4
# --------------------------------------------------------------------------

def _c4_csv(T=500, seed=4):
    return c4_ssfp_csv(T, seed)


def test_c4_ssfp_b0_b1_grid_and_max_pd_matching(snap, oracle):
    T, w = 500, 50
    h = _c4_csv(T)
    t1 = np.array([100.0 * 1.05 ** k for k in range(0, 81, 16)], np.float32)
    t2 = np.array([10.0 * 1.05 ** k for k in range(0, 109, 27)], np.float32)
    b0 = np.arange(-100.0, 100.1, 20.0, dtype=np.float32)
    b1 = np.array([0.8, 0.9, 1.0, 1.1, 1.2], np.float32)
    params = snap.trans_params(t1, t2, b0, b1)
    natoms = params.shape[0] // len(b1)
    atoms = run_dict(snap, "epg_ssfp", params, h, T, natoms=natoms, nstates=w)
    ref = oracle.dict_atoms("epg_ssfp", params, h, T, natoms=natoms, nstates=w, nthreads=8)
    rel = rel_err_per_atom(atoms, ref)
    print(f"C4 SSFP ({params.shape[0]} atoms): max rel vs FP64 oracle {rel.max():.2e}")
    assert rel.max() < 1e-4
    # voxels from dictionary atoms with noise, no B1 map: max-PD merge = global MIP
    rng = np.random.default_rng(5)
    pick = rng.integers(0, params.shape[0], 512)
    img = atoms[pick] * (rng.uniform(0.5, 1, 512) * np.exp(1j * rng.uniform(0, 6.28, 512)))[:, None]
    img = (img + 0.01 * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape)))
    img = img.astype(np.complex64)
    maps, idx = run_match(snap, img, atoms, params, natoms=natoms)
    ref_maps, ref_idx = oracle.match(img, atoms, params, T, natoms=natoms, precision="f64", nthreads=8)
    _assert_indices_equal_where_separated(idx, ref_idx, _scores(atoms, img))
    np.testing.assert_allclose(maps[:, 4], ref_maps[:, 4], rtol=2e-5)


def test_c4_roa_100_isochromats(snap, oracle):
    T = 500
    h = _c4_csv(T, seed=6)
    params = _grid(np.geomspace(200, 3000, 4), np.geomspace(20, 300, 3), b0s=(-100.0, -36.0, 0.0, 52.0, 100.0),
                   b1s=(0.8, 1.0, 1.2))
    natoms = params.shape[0] // 3
    got = run_dict(snap, "roa_ssfp", params, h, T, natoms=natoms, n_iso=100, flags=snap.DICT_ALL_B1_BLOCKS)
    ref = oracle.dict_atoms("roa_ssfp", params, h, T, natoms=natoms, n_iso=100, flags=oracle.ALL_B1_BLOCKS,
                            nthreads=8)
    rel = rel_err_per_atom(got[:ref.shape[0]], ref)
    print(f"C4 ROA n_iso=100: max rel vs FP64 oracle {rel.max():.2e}")
    assert rel.max() < 1e-4


def _crb_loss_fp64(oracle, tissues, h, w):
    """sum_i [M^-1]_00 / T1^2 + [M^-1]_11 / T2^2 from the FP64 forward mode."""
    total, per, sig = 0.0, [], []
    for (t1, t2, b1) in tissues:
        f, f1, _, _ = oracle.fisp_jvp((t1, t2, b1), (1, 0, 0), h, nstates=w)
        _, f2, _, _ = oracle.fisp_jvp((t1, t2, b1), (0, 1, 0), h, nstates=w)
        V = np.stack([f1, f2, f], 1)
        Mi = np.linalg.inv(V.T @ V)
        li = Mi[0, 0] / t1 ** 2 + Mi[1, 1] / t2 ** 2
        per.append(li)
        sig.append(np.stack([f, f1, f2]))
        total += li
    return total, np.array(per), np.array(sig)


def test_c3_crb_schedule_gradient_three_tissues(snap, oracle):
    """The CRB loss of three tissues and its gradient with respect to every
    flip angle (T = 1000, w = 50, checkpoints every 32 steps) against the
    FP64 forward-mode oracle and central differences of its loss along
    random directions."""
    import torch
    T, w = 1000, 50
    h = mrf_schedule(T, seed=30, inversion=False)
    tissues = [(1000.0, 80.0, 1.0), (1500.0, 150.0, 0.9), (800.0, 50.0, 1.1)]
    params = np.array([(a, b, 0.0, c) for a, b, c in tissues], np.float32)
    d_p = torch.from_numpy(params).cuda()
    d_loss = torch.empty(3, device="cuda")
    d_ga = torch.empty(T, device="cuda")
    d_sig = torch.empty((3, 3, T), device="cuda")
    snap.crb_gradient(d_p, h, T, T, 3, d_loss, d_ga, 4, w, "epg_fisp", d_signals=d_sig, checkpoint_every=32)
    torch.cuda.synchronize()
    total, per, sig = _crb_loss_fp64(oracle, [tuple(map(float, p[[0, 1, 3]])) for p in params], h, w)
    err = np.abs(d_sig.cpu().numpy() - sig).max(axis=2) / np.abs(sig).max(axis=2)
    print(f"f, df/dT1, df/dT2 vs FP64: max rel {err.max():.2e}; loss {d_loss.cpu().numpy()} vs {per}")
    assert err.max() < 1e-4
    np.testing.assert_allclose(d_loss.cpu().numpy(), per, rtol=2e-3)
    g = d_ga.cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(31)
    for trial in range(3):
        v = rng.standard_normal(T)
        e = 2e-3
        hp, hm = h.copy(), h.copy()
        hp[0] = (h[0].astype(np.float64) + e * v).astype(np.float32)
        hm[0] = (h[0].astype(np.float64) - e * v).astype(np.float32)
        dv = (hp[0].astype(np.float64) - hm[0]) / (2 * e)   # the direction the float32 angles take
        tl = [tuple(map(float, p[[0, 1, 3]])) for p in params]
        lp, _, _ = _crb_loss_fp64(oracle, tl, hp, w)
        lm, _, _ = _crb_loss_fp64(oracle, tl, hm, w)
        fd = (lp - lm) / (2 * e)
        got = float(g @ dv)
        print(f"CRB gradient along a random direction: adjoint {got:.6e}, FP64 difference {fd:.6e}")
        assert abs(got - fd) <= 5e-3 * abs(fd) + 1e-3 * float(np.abs(g) @ np.abs(dv))


def test_epg_jvp_matches_fp64_forward_mode(snap, oracle):
    """snapmrf_epg_jvp: f, df/dT1 and df/dT2 of three atoms against the FP64
    forward mode (1e-4 of each row's peak), equal to the CRB gradient's
    forward pass on the same inputs, and a Jacobian-vector product along a
    mixed direction against the FP64 one."""
    import torch
    T, w = 400, 30
    h = mrf_schedule(T, seed=32, inversion=False)
    tissues = [(1000.0, 80.0, 1.0), (1500.0, 150.0, 0.9), (800.0, 50.0, 1.1)]
    params = np.array([(a, b, 0.0, c) for a, b, c in tissues], np.float32)
    d_p = torch.from_numpy(params).cuda()
    d_out = torch.full((3, 3, T), float("nan"), device="cuda")
    snap.epg_jvp(d_p, h, T, T, 3, d_out, 4, w, "epg_fisp")
    d_sig = torch.empty((3, 3, T), device="cuda")
    d_loss = torch.empty(3, device="cuda")
    d_ga = torch.empty(T, device="cuda")
    snap.crb_gradient(d_p, h, T, T, 3, d_loss, d_ga, 4, w, "epg_fisp", d_signals=d_sig)
    torch.cuda.synchronize()
    got = d_out.cpu().numpy()
    np.testing.assert_array_equal(got, d_sig.cpu().numpy())
    for i, (t1, t2, b1) in enumerate(tissues):
        f, f1, _, _ = oracle.fisp_jvp((t1, t2, b1), (1, 0, 0), h, nstates=w)
        _, f2, _, _ = oracle.fisp_jvp((t1, t2, b1), (0, 1, 0), h, nstates=w)
        for row, ref in zip(got[i], (f, f1, f2)):
            assert np.abs(row - ref).max() <= 1e-4 * np.abs(ref).max()
        _, fv, _, _ = oracle.fisp_jvp((t1, t2, b1), (3.0, -0.5, 0), h, nstates=w)
        jv = 3.0 * got[i, 1].astype(np.float64) - 0.5 * got[i, 2]
        assert np.abs(jv - fv).max() <= 1e-4 * np.abs(fv).max()


def test_crb_loss_autograd_descends(snap):
    """A few gradient steps on the flip angles through CRBLoss lower the CRB
    loss of three tissues."""
    import torch
    from snapmrf_b200.autograd import CRBLoss
    T, w = 400, 30
    h = mrf_schedule(T, seed=32, inversion=False)
    tissues = torch.tensor([(1000.0, 80.0, 0.0, 1.0), (1500.0, 150.0, 0.0, 0.9), (800.0, 50.0, 0.0, 1.1)],
                           device="cuda")
    alpha = torch.tensor(h[0], device="cuda", requires_grad=True)
    opt = torch.optim.Adam([alpha], lr=5e-3)
    losses = []
    for _ in range(15):
        opt.zero_grad()
        loss = CRBLoss.apply(tissues, alpha, h, w, "epg_fisp")
        loss.backward()
        assert torch.isfinite(alpha.grad).all()
        opt.step()
        losses.append(loss.item())
    print("CRB loss during descent:", [round(v, 4) for v in losses])
    assert losses[-1] < 0.95 * losses[0]
    assert sum(b < a for a, b in zip(losses, losses[1:])) >= 12
