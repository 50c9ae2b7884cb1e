"""Derivative kernels on the GPU (snapmrf_epg_adjoint, snapmrf_refine_gn)
against the FP64 forward-mode oracle, central differences and
torch.autograd.gradcheck."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def schedule(T, seed=0, sr=False):
    rng = np.random.default_rng(seed)
    a = np.deg2rad(5 + 55 * np.abs(np.sin(np.pi * np.arange(T) / 230)) + rng.uniform(0, 3, T))
    if sr:
        a[::50] = np.deg2rad(90)
    tr = rng.uniform(11, 15, T)
    te = tr * rng.uniform(0.3, 0.6, T)
    return np.array([a, np.zeros(T), tr, te], np.float32)


def atoms_params(n, seed=1):
    rng = np.random.default_rng(seed)
    t1 = rng.uniform(300, 2500, n)
    t2 = rng.uniform(20, 250, n)
    b1 = rng.uniform(0.7, 1.2, n)
    return np.stack([t1, t2, np.zeros(n), b1], 1).astype(np.float32)


def run_adjoint(snap, params, h, nstates, echo, gsig, checkpoint_every=0, per_atom=True):
    import torch
    n, T = params.shape[0], h.shape[1]
    d_params = torch.from_numpy(params).cuda()
    d_g = torch.from_numpy(np.ascontiguousarray(gsig.astype(np.complex64)).view(np.float32)).cuda()
    d_sig = torch.full((n, T, 2), 7.0, device="cuda")
    d_gp = torch.full((n, 3), 7.0, device="cuda")
    d_ga = torch.full((T,), 7.0, device="cuda")
    d_gaa = torch.full((n, T), 7.0, device="cuda") if per_atom else None
    snap.epg_adjoint(d_params, h, T, T, n, d_g, d_gp, 4, nstates, echo, d_signal=d_sig, d_grad_alpha=d_ga,
                     d_grad_alpha_atoms=d_gaa, checkpoint_every=checkpoint_every)
    torch.cuda.synchronize()
    s = d_sig.cpu().numpy()
    return (s[..., 0] + 1j * s[..., 1], d_gp.cpu().numpy(), d_ga.cpu().numpy(),
            None if d_gaa is None else d_gaa.cpu().numpy())


@pytest.mark.parametrize("echo", ["epg_fisp", "epg_sr"])
@pytest.mark.parametrize("nstates", [1, 2, 7, 30, 50])
def test_adjoint_matches_fp64_forward_mode(snap, oracle, echo, nstates):
    """dL/dT1, dL/dT2, dL/dB1 and dL/dalpha (along a random direction) of
    L = sum |s - y|^2 agree with the FP64 dual-number oracle to 1e-3 of the
    gradient's scale."""
    T = 400
    h = schedule(T, seed=nstates, sr=echo == "epg_sr")
    params = atoms_params(5, seed=nstates)
    rng = np.random.default_rng(7)
    ys, ref_sig = [], []
    for p in params:
        s, _, _, _ = oracle.fisp_jvp((p[0], p[1], p[3]), (0, 0, 0), h, nstates=nstates, echo=echo)
        ref_sig.append(s)
        ys.append(1j * s * rng.uniform(0.5, 1.5) + 0.02 * (rng.standard_normal(T) + 1j * rng.standard_normal(T)))
    ys = np.array(ys)
    ref_sig = np.array(ref_sig)
    # dL/ds = 2 (s - y), with s the oracle's signal
    gsig = 2 * (1j * ref_sig - ys)
    sig, gp, ga, gaa = run_adjoint(snap, params, h, nstates, echo, gsig)
    assert np.abs(sig.real).max() == 0
    np.testing.assert_allclose(sig.imag, ref_sig, rtol=0, atol=2e-5 * np.abs(ref_sig).max())
    v = rng.standard_normal(T)
    for i, p in enumerate(params):
        th = (p[0], p[1], p[3])
        for k, tg in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
            _, ds, _, w = oracle.fisp_jvp(th, tg, h, nstates=nstates, echo=echo, y=ys[i])
            # scale of the sum's terms, for gradients that cancel to near 0
            scale = float(np.abs(gsig[i].imag) @ np.abs(ds))
            assert abs(gp[i, k] - w) <= 1e-3 * abs(w) + 1e-4 * scale, (i, k, gp[i, k], w, scale)
        wa = oracle.fisp_jvp(th, (0, 0, 0), h, nstates=nstates, echo=echo, dalpha=v, y=ys[i])[3]
        got = float(np.dot(gaa[i].astype(np.float64), v))
        scale = float(np.abs(gaa[i]).astype(np.float64) @ np.abs(v))
        assert abs(got - wa) <= 1e-3 * scale, (i, got, wa, scale)
    np.testing.assert_allclose(ga, gaa.astype(np.float64).sum(0), rtol=1e-5, atol=1e-5 * np.abs(gaa).max())


def test_adjoint_checkpoint_interval_does_not_change_results(snap):
    T, w = 257, 20
    h = schedule(T, seed=3)
    params = atoms_params(37, seed=3)
    rng = np.random.default_rng(3)
    gsig = rng.standard_normal((37, T)) + 1j * rng.standard_normal((37, T))
    base = run_adjoint(snap, params, h, w, "epg_fisp", gsig, checkpoint_every=0)
    for c in (1, 5, 64, T, 10 * T):
        other = run_adjoint(snap, params, h, w, "epg_fisp", gsig, checkpoint_every=c)
        for a, b in zip(base, other):
            np.testing.assert_array_equal(a, b)


def test_adjoint_signal_equals_dictionary(snap):
    """The adjoint's forward sweep gives the atoms snapmrf_mrf_dict gives
    (one B1 block per atom)."""
    from gpu_util import run_dict
    T, w = 300, 40
    h = schedule(T, seed=4)
    params = atoms_params(50, seed=4)
    sig, _, _, _ = run_adjoint(snap, params, h, w, "epg_fisp", np.zeros((50, T)))
    ref = run_dict(snap, "epg_fisp", params, h, T, natoms=1, nstates=w, flags=snap.DICT_ALL_B1_BLOCKS)
    rel = np.abs(sig - ref).max(axis=1) / np.abs(ref).max(axis=1)
    assert rel.max() < 2e-6


def test_adjoint_vs_central_differences_of_the_dictionary(snap):
    """Gradient of L = sum_t w_t Im s_t against central differences of
    snapmrf_mrf_dict itself (FP32)."""
    from gpu_util import run_dict
    T, w = 300, 25
    h = schedule(T, seed=5)
    params = atoms_params(4, seed=5)
    rng = np.random.default_rng(5)
    wt = rng.standard_normal(T)
    _, gp, _, _ = run_adjoint(snap, params, h, w, "epg_fisp", np.broadcast_to(1j * wt, (4, T)))
    # relative steps large enough for FP32 differences of ~1e-5 gradients
    for k, (col, rel) in enumerate(((0, 1e-2), (1, 1e-2), (3, 1e-3))):
        hp, hm = params.copy(), params.copy()
        step = rel * params[:, col]
        hp[:, col] += step
        hm[:, col] -= step
        sp = run_dict(snap, "epg_fisp", hp, h, T, natoms=1, nstates=w, flags=snap.DICT_ALL_B1_BLOCKS)
        sm = run_dict(snap, "epg_fisp", hm, h, T, natoms=1, nstates=w, flags=snap.DICT_ALL_B1_BLOCKS)
        fd = ((sp.imag.astype(np.float64) - sm.imag) @ wt) / (hp[:, col].astype(np.float64) - hm[:, col])
        np.testing.assert_allclose(gp[:, k], fd, rtol=1e-2, atol=1e-2 * np.abs(fd).max())


def test_autograd_gradcheck(snap):
    import torch
    from snapmrf_b200.autograd import EPGSignal
    T, w = 48, 12
    h = schedule(T, seed=6)
    base = torch.tensor(atoms_params(2, seed=6), device="cuda")
    scale = torch.tensor([1000.0, 100.0, 1.0, 1.0], device="cuda")
    u = (base / scale).clone().requires_grad_(True)
    alpha = torch.tensor(h[0], device="cuda").requires_grad_(True)

    def f(u_, a_):
        return EPGSignal.apply(u_ * scale, a_, h, w, "epg_fisp")

    assert torch.autograd.gradcheck(f, (u, alpha), eps=1e-3, atol=2e-3, rtol=2e-2, check_undefined_grad=False)
    # and the same through a scalar loss, against the oracle
    from oracle import oracle as orc
    y = torch.randn((2, T, 2), device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    loss = ((f(u, alpha) - y) ** 2).sum()
    loss.backward()
    p = (u.detach() * scale).cpu().numpy()
    yc = y.cpu().numpy()
    yc = yc[..., 0] + 1j * yc[..., 1]
    for i in range(2):
        want = orc.fisp_jvp((p[i, 0], p[i, 1], p[i, 3]), (1000.0, 0, 0), h, nstates=w, y=yc[i])[3]
        assert abs(u.grad[i, 0].item() - want) <= 1e-3 * abs(want) + 1e-4


def test_adjoint_rejects_unsupported_inputs(snap):
    import torch
    T = 20
    h = schedule(T)
    d_params = torch.from_numpy(atoms_params(2)).cuda()
    g = torch.zeros((2, T, 2), device="cuda")
    gp = torch.zeros((2, 3), device="cuda")
    with pytest.raises(snap.SnapMRFError, match="epg_fisp, epg_sr or epg_ssfp"):
        snap.epg_adjoint(d_params, h, T, T, 2, g, gp, 4, 10, "epg_se")
    hp = h.copy()
    hp[1, 3] = 0.5
    with pytest.raises(snap.SnapMRFError):
        snap.epg_adjoint(d_params, hp, T, T, 2, g, gp, 4, 10, "epg_fisp")
    with pytest.raises(snap.SnapMRFError):
        snap.epg_adjoint(d_params, h, T, T, 2, g, gp, 4, 300, "epg_fisp")


# --------------------------------------------------------------------------
# Gauss-Newton refinement
# --------------------------------------------------------------------------

def gn_step_fp64(orc, theta, x, h, w, echo="epg_fisp"):
    """One projected Gauss-Newton step in FP64 from the oracle's tangents."""
    return orc.gn_step_f64(theta, x, h, nstates=w, echo=echo)


def run_gn(snap, theta, img, h, w, iterations, echo="epg_fisp", max_rel_step=0.2, b1map=None, tol=1e-4):
    """theta [n][3] = (T1, T2, B1) -> (T1, T2, B1) [n][3], PD, M0."""
    import torch
    n = theta.shape[0]
    maps = np.zeros((n, 5), np.float32)
    maps[:, 0], maps[:, 1], maps[:, 3], maps[:, 4] = theta[:, 0], theta[:, 1], theta[:, 2], -1
    d_maps = torch.from_numpy(maps).cuda()
    d_img = torch.from_numpy(np.ascontiguousarray(img.astype(np.complex64)).view(np.float32)).cuda()
    d_m0 = torch.full((n,), -1.0, device="cuda")
    d_b1 = None if b1map is None else torch.from_numpy(np.ascontiguousarray(b1map, np.float32)).cuda()
    snap.refine_gn(d_maps, d_img, h, h.shape[1], h.shape[1], n, w, echo, iterations=iterations,
                   max_rel_step=max_rel_step, tol=tol, d_b1map=d_b1, d_m0=d_m0)
    torch.cuda.synchronize()
    out = d_maps.cpu().numpy()
    assert np.all(out[:, 2] == 0)
    return out[:, [0, 1, 3]], out[:, 4], d_m0.cpu().numpy()


def synthetic_voxels(orc, n, h, w, seed, echo="epg_fisp", noise=0.0):
    rng = np.random.default_rng(seed)
    truth = atoms_params(n, seed=seed)
    rho = rng.uniform(0.5, 2, n) * np.exp(1j * rng.uniform(0, 6.28, n))
    x = []
    for p, r in zip(truth, rho):
        s, _, _, _ = orc.fisp_jvp((p[0], p[1], p[3]), (0, 0, 0), h, nstates=w, echo=echo)
        x.append(r * 1j * s + noise * (rng.standard_normal(len(s)) + 1j * rng.standard_normal(len(s))))
    return truth, rho, np.array(x)


@pytest.mark.parametrize("echo", ["epg_fisp", "epg_sr"])
def test_gn_step_matches_fp64_step(snap, oracle, echo):
    T, w = 300, 30
    h = schedule(T, seed=8, sr=echo == "epg_sr")
    truth, rho, x = synthetic_voxels(oracle, 6, h, w, seed=8, echo=echo, noise=0.01)
    rng = np.random.default_rng(9)
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.95, 1.05, 6), truth[:, 1] * rng.uniform(0.95, 1.05, 6),
                       truth[:, 3]], 1).astype(np.float32)
    got, _, _ = run_gn(snap, theta0, x, h, w, 1, echo=echo, max_rel_step=1e6)
    for i in range(6):
        d, _, _ = gn_step_fp64(oracle, tuple(theta0[i].astype(np.float64)), x[i], h, w, echo)
        step = got[i, :2].astype(np.float64) - theta0[i, :2]
        np.testing.assert_allclose(step, d, rtol=2e-3, atol=2e-3 * np.abs(d).max() + 1e-3)
        assert got[i, 2] == theta0[i, 2]


def test_gn_recovers_off_grid_parameters(snap, oracle):
    T, w = 500, 40
    h = schedule(T, seed=10)
    truth, rho, x = synthetic_voxels(oracle, 64, h, w, seed=10)
    rng = np.random.default_rng(11)
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.9, 1.1, 64), truth[:, 1] * rng.uniform(0.9, 1.1, 64),
                       truth[:, 3]], 1).astype(np.float32)
    got, pd, m0 = run_gn(snap, theta0, x, h, w, 5)
    np.testing.assert_allclose(got[:, 0], truth[:, 0], rtol=2e-3)
    np.testing.assert_allclose(got[:, 1], truth[:, 1], rtol=2e-3)
    np.testing.assert_allclose(m0, np.abs(rho), rtol=2e-3)
    for i in range(64):
        s, _, _, _ = oracle.fisp_jvp((truth[i, 0], truth[i, 1], truth[i, 3]), (0, 0, 0), h, nstates=w)
        assert abs(pd[i] - abs(rho[i]) * np.linalg.norm(s)) <= 2e-3 * pd[i]


def test_gn_zero_iterations_only_evaluates(snap, oracle):
    T, w = 200, 20
    h = schedule(T, seed=12)
    truth, rho, x = synthetic_voxels(oracle, 10, h, w, seed=12)
    theta0 = np.stack([truth[:, 0], truth[:, 1], truth[:, 3]], 1).astype(np.float32)
    got, pd, m0 = run_gn(snap, theta0, x, h, w, 0)
    np.testing.assert_array_equal(got, theta0)
    np.testing.assert_allclose(m0, np.abs(rho), rtol=1e-4)


def test_gn_leaves_unusable_voxels(snap, oracle):
    T, w = 100, 10
    h = schedule(T, seed=13)
    truth, rho, x = synthetic_voxels(oracle, 5, h, w, seed=13)
    theta0 = np.stack([truth[:, 0], truth[:, 1], truth[:, 3]], 1).astype(np.float32)
    theta0[0, 0] = np.nan
    theta0[1, 1] = 0
    theta0[2, 0] = theta0[2, 1]  # T1 == T2
    got, pd, m0 = run_gn(snap, theta0, x, h, w, 2)
    np.testing.assert_array_equal(got[:3], theta0[:3])
    assert np.all(pd[:3] == -1) and np.all(m0[:3] == -1)
    assert np.all(pd[3:] > 0)


def test_gn_uses_the_b1_map(snap, oracle):
    """Maps matched at a quantised B1 block value, refined at the measured B1."""
    T, w = 400, 30
    h = schedule(T, seed=14)
    truth, rho, x = synthetic_voxels(oracle, 32, h, w, seed=14)
    rng = np.random.default_rng(15)
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.95, 1.05, 32), truth[:, 1] * rng.uniform(0.95, 1.05, 32),
                       np.round(truth[:, 3] / 0.05) * 0.05], 1).astype(np.float32)
    got, _, _ = run_gn(snap, theta0, x, h, w, 4, b1map=truth[:, 3])
    np.testing.assert_array_equal(got[:, 2], truth[:, 3])
    np.testing.assert_allclose(got[:, 0], truth[:, 0], rtol=2e-3)
    np.testing.assert_allclose(got[:, 1], truth[:, 1], rtol=2e-3)


def test_gn_early_exit_agrees_with_full_iterations(snap, oracle):
    """Voxels that stop once their step is below tol end where running every
    iteration on every voxel ends (to well within tol's effect); 333 voxels
    exercise partly filled blocks of the compacted voxel lists."""
    T, w = 300, 25
    h = schedule(T, seed=16)
    truth, rho, x = synthetic_voxels(oracle, 333, h, w, seed=16, noise=0.003)
    rng = np.random.default_rng(17)
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.9, 1.1, 333), truth[:, 1] * rng.uniform(0.9, 1.1, 333),
                       truth[:, 3]], 1).astype(np.float32)
    full, pd_f, _ = run_gn(snap, theta0, x, h, w, 4, tol=0.0)
    early, pd_e, _ = run_gn(snap, theta0, x, h, w, 4, tol=1e-4)
    np.testing.assert_allclose(early[:, :2], full[:, :2], rtol=5e-4)
    np.testing.assert_allclose(pd_e, pd_f, rtol=1e-5)
    one, _, _ = run_gn(snap, theta0, x, h, w, 1, tol=1e-4)
    assert not np.allclose(one[:, :2], full[:, :2], rtol=5e-4)


# --------------------------------------------------------------------------
# Gauss-Newton on the complex bSSFP recursion
# --------------------------------------------------------------------------

def _ssfp_voxels(orc, n, h, w, seed, noise=0.0):
    rng = np.random.default_rng(seed)
    t1 = np.exp(rng.uniform(np.log(300), np.log(2500), n))
    t2 = np.minimum(np.exp(rng.uniform(np.log(30), np.log(300), n)), 0.5 * t1)
    b0 = rng.uniform(-60, 60, n)
    b1 = rng.uniform(0.85, 1.15, n)
    truth = np.stack([t1, t2, b0, b1], 1)
    rho = rng.uniform(0.5, 2, n) * np.exp(1j * rng.uniform(0, 6.28, n))
    x = []
    for p, r in zip(truth, rho):
        s, _ = orc.ssfp_jvp(tuple(p), (0, 0, 0, 0), h, nstates=w)
        x.append(r * s + noise * (rng.standard_normal(len(s)) + 1j * rng.standard_normal(len(s))))
    return truth, rho, np.array(x)


def _run_gn_ssfp(snap, start, img, h, w, iterations, b1map=None, tol=0.0, max_rel_step=0.2):
    import torch
    n = start.shape[0]
    maps = np.zeros((n, 5), np.float32)
    maps[:, :4] = start
    maps[:, 4] = -1
    d_maps = torch.from_numpy(maps).cuda()
    d_img = torch.from_numpy(np.ascontiguousarray(img.astype(np.complex64)).view(np.float32)).cuda()
    d_m0 = torch.full((n,), -1.0, device="cuda")
    d_b1 = None if b1map is None else torch.from_numpy(np.ascontiguousarray(b1map, np.float32)).cuda()
    snap.refine_gn(d_maps, d_img, h, h.shape[1], h.shape[1], n, w, "epg_ssfp", iterations=iterations,
                   max_rel_step=max_rel_step, tol=tol, d_b1map=d_b1, d_m0=d_m0)
    torch.cuda.synchronize()
    return d_maps.cpu().numpy(), d_m0.cpu().numpy()


def test_gn_ssfp_step_matches_fp64_step(snap, oracle):
    """One Gauss-Newton step of (T1, T2, B0, B1) on the complex bSSFP
    recursion against the FP64 projected step from the oracle's forward
    mode (noisy voxels, starts off by a few percent, no trust region)."""
    from cases import c4_ssfp_csv
    T, w = 200, 30
    h = c4_ssfp_csv(T, seed=41)
    truth, rho, x = _ssfp_voxels(oracle, 6, h, w, seed=42, noise=0.002)
    rng = np.random.default_rng(43)
    start = (truth * np.stack([rng.uniform(0.97, 1.03, 6), rng.uniform(0.97, 1.03, 6), np.ones(6),
                               rng.uniform(0.98, 1.02, 6)], 1)).astype(np.float32)
    start[:, 2] += rng.uniform(-1.5, 1.5, 6).astype(np.float32)
    got, _ = _run_gn_ssfp(snap, start, x, h, w, 1, max_rel_step=1e6)
    for i in range(6):
        d, _, _ = oracle.ssfp_gn_step_f64(tuple(start[i].astype(np.float64)), x[i], h, nstates=w)
        step = got[i, :4].astype(np.float64) - start[i].astype(np.float64)
        print(i, step, d)
        np.testing.assert_allclose(step, d, rtol=5e-3, atol=5e-3 * np.abs(d).max() + 1e-4)


@pytest.mark.parametrize("with_map", [False, True])
def test_gn_ssfp_recovers_off_grid_parameters(snap, oracle, with_map):
    """Noiseless bSSFP voxels from off-grid (T1, T2, B0, B1), started a grid
    step away (5 % in T1 and T2, 2 Hz, 0.04 in B1; with a B1 map, B1 exact
    and kept): six iterations recover the parameters, and PD / M0 are those
    of the exact fit."""
    from cases import c4_ssfp_csv
    T, w = 300, 40
    h = c4_ssfp_csv(T, seed=44)
    n = 24
    truth, rho, x = _ssfp_voxels(oracle, n, h, w, seed=45)
    sign = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    start = truth.copy()
    start[:, 0] *= 1.05 ** sign
    start[:, 1] /= 1.05 ** sign
    start[:, 2] += 2.0 * sign
    if not with_map:
        start[:, 3] += 0.04 * sign
    b1map = truth[:, 3] if with_map else None
    got, m0 = _run_gn_ssfp(snap, start.astype(np.float32), x, h, w, 6, b1map=b1map)
    err = np.abs(got[:, :4] - truth) / np.array([truth[:, 0], truth[:, 1], np.full(n, 100.0), truth[:, 3]]).T
    print("max relative errors (T1, T2, B0/100 Hz, B1):", err.max(axis=0))
    assert err[:, :2].max() < 1e-3 and err[:, 2].max() < 1e-3 and err[:, 3].max() < 1e-3
    for i in range(n):
        s, _ = oracle.ssfp_jvp(tuple(truth[i]), (0, 0, 0, 0), h, nstates=w)
        assert abs(m0[i] - abs(rho[i])) < 2e-3 * abs(rho[i])
        assert abs(got[i, 4] - abs(rho[i]) * np.linalg.norm(s)) < 2e-3 * abs(rho[i]) * np.linalg.norm(s)


def test_ssfp_adjoint_matches_fp64_forward_mode_and_differences(snap, oracle):
    """Reverse mode through the complex bSSFP recursion (B0 precession,
    alternating RF phase, the inversion) with checkpoints: for a loss linear
    in the signal, L = sum_t Re(conj(g_t) s_t), the gradients by (T1, T2, B0,
    B1) equal the FP64 forward mode's, the schedule gradient equals FP64
    central differences along random directions, the signal equals the FP64
    recursion's, and the checkpoint interval changes nothing."""
    import torch
    from cases import c4_ssfp_csv
    T, w, n = 150, 30, 8
    h = c4_ssfp_csv(T, seed=47)
    rng = np.random.default_rng(48)
    t1 = np.exp(rng.uniform(np.log(300), np.log(2500), n))
    t2 = np.minimum(np.exp(rng.uniform(np.log(30), np.log(300), n)), 0.5 * t1)
    params = np.stack([t1, t2, rng.uniform(-60, 60, n), rng.uniform(0.85, 1.15, n)], 1).astype(np.float32)
    g = (rng.standard_normal((n, T)) + 1j * rng.standard_normal((n, T))).astype(np.complex64)
    d_p = torch.from_numpy(params).cuda()
    d_g = torch.from_numpy(g.view(np.float32).reshape(n, T, 2)).cuda()
    out = {}
    for C in (7, 1, T):
        d_sig = torch.empty((n, T, 2), device="cuda")
        d_gp = torch.empty((n, 4), device="cuda")
        d_ga = torch.empty(T, device="cuda")
        d_gaa = torch.empty((n, T), device="cuda")
        snap.epg_adjoint(d_p, h, T, T, n, d_g, d_gp, 4, w, "epg_ssfp", d_signal=d_sig, d_grad_alpha=d_ga,
                         d_grad_alpha_atoms=d_gaa, checkpoint_every=C)
        torch.cuda.synchronize()
        out[C] = (d_sig.cpu().numpy(), d_gp.cpu().numpy(), d_ga.cpu().numpy(), d_gaa.cpu().numpy())
    for C in (1, T):
        for a, b in zip(out[7], out[C]):
            np.testing.assert_array_equal(a, b)
    sig, gp, ga, gaa = out[7]
    sig = sig[..., 0] + 1j * sig[..., 1]
    np.testing.assert_allclose(ga, gaa.sum(axis=0), rtol=1e-4, atol=1e-4 * np.abs(gaa).sum(axis=0).max())
    for i in range(n):
        th = tuple(params[i].astype(np.float64))
        s, _ = oracle.ssfp_jvp(th, (0, 0, 0, 0), h, nstates=w)
        assert np.abs(sig[i] - s).max() <= 1e-5 * np.abs(s).max()
        for j in range(4):
            tg = [0.0] * 4
            tg[j] = 1.0
            _, ds = oracle.ssfp_jvp(th, tg, h, nstates=w)
            want = float(np.sum((np.conj(g[i]) * ds).real))
            scale = float(np.sum(np.abs(g[i]) * np.abs(ds)))
            assert abs(gp[i, j] - want) <= 1e-3 * abs(want) + 1e-4 * scale, (i, j, gp[i, j], want)
    # the schedule's flip entries: central differences of the FP64 loss
    def loss(hh):
        total = 0.0
        for i in range(n):
            s, _ = oracle.ssfp_jvp(tuple(params[i].astype(np.float64)), (0, 0, 0, 0), hh, nstates=w)
            total += float(np.sum((np.conj(g[i]) * s).real))
        return total
    for trial in range(2):
        v = rng.standard_normal(T)
        e = 1e-3
        hp, hm = h.copy(), h.copy()
        hp[0] = (h[0].astype(np.float64) + e * v).astype(np.float32)
        hm[0] = (h[0].astype(np.float64) - e * v).astype(np.float32)
        dv = (hp[0].astype(np.float64) - hm[0]) / (2 * e)
        fd = (loss(hp) - loss(hm)) / (2 * e)
        got = float(ga.astype(np.float64) @ dv)
        print(f"bSSFP schedule gradient along a random direction: adjoint {got:.6e}, FP64 difference {fd:.6e}")
        assert abs(got - fd) <= 5e-3 * abs(fd) + 1e-3 * float(np.abs(ga) @ np.abs(dv))


@pytest.mark.parametrize("tol", [0.0, 1e-4])
def test_gn_tail_launch_gives_identical_maps(snap, monkeypatch, tol):
    """The refinement splits its voxel list into whole rounds of resident
    blocks (4 lanes per voxel at w = 50) and a tail with 16 lanes per voxel;
    every state sees the same operations in both layouts, so the maps equal
    those of one launch over the whole list bit for bit.  30,001 voxels are
    three whole rounds on a 148-SM part and a ragged tail; with tol > 0 the
    compacted lists of later iterations split again."""
    import torch
    T, w, n = 200, 50, 30001
    h = schedule(T, seed=21)
    rng = np.random.default_rng(21)
    truth = atoms_params(n, seed=21)
    d_sig = torch.empty((n, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_sig, torch.from_numpy(truth).cuda(), h, T, T, n, 1, 4, w, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS)
    sig = d_sig.cpu().numpy()
    rho = rng.uniform(0.5, 2, n) * np.exp(1j * rng.uniform(0, 6.28, n))
    x = (sig[..., 0] + 1j * sig[..., 1]) * rho[:, None]
    x = x + 0.003 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.9, 1.1, n), truth[:, 1] * rng.uniform(0.9, 1.1, n),
                       truth[:, 3]], 1).astype(np.float32)
    split, pd_s, m0_s = run_gn(snap, theta0, x, h, w, 3, tol=tol)
    monkeypatch.setenv("SNAPMRF_GN_TAIL", "0")
    whole, pd_w, m0_w = run_gn(snap, theta0, x, h, w, 3, tol=tol)
    np.testing.assert_array_equal(split, whole)
    np.testing.assert_array_equal(pd_s, pd_w)
    np.testing.assert_array_equal(m0_s, m0_w)
    # and the refinement did its work: the start was 5 % off on the median
    assert np.median(np.abs(split[:, 0] / truth[:, 0] - 1)) < 0.4 * np.median(np.abs(theta0[:, 0] / truth[:, 0] - 1))


@pytest.mark.parametrize("layout", ["4,7", "7,4", "13,2"])
def test_gn_layouts_give_identical_maps(snap, monkeypatch, layout):
    """Lane groups of any width (the default at w = 50 is 5 lanes x 5 pairs;
    4, 7 or 13 lanes per voxel here, the warp's last lanes idle where the
    width does not divide 32) perform the same operations on every state, so
    the maps are the same bit for bit; 3,001 voxels leave partly filled
    CTAs."""
    import torch
    T, w, n = 200, 50, 3001
    h = schedule(T, seed=23)
    rng = np.random.default_rng(23)
    truth = atoms_params(n, seed=23)
    d_sig = torch.empty((n, T, 2), dtype=torch.float32, device="cuda")
    snap.MRF_dict(d_sig, torch.from_numpy(truth).cuda(), h, T, T, n, 1, 4, w, "epg_fisp",
                  flags=snap.DICT_ALL_B1_BLOCKS)
    sig = d_sig.cpu().numpy()
    x = (sig[..., 0] + 1j * sig[..., 1]) * (rng.uniform(0.5, 2, n) * np.exp(1j * rng.uniform(0, 6.28, n)))[:, None]
    theta0 = np.stack([truth[:, 0] * rng.uniform(0.95, 1.05, n), truth[:, 1] * rng.uniform(0.95, 1.05, n),
                       truth[:, 3]], 1).astype(np.float32)
    want, pd_w, m0_w = run_gn(snap, theta0, x, h, w, 2, tol=1e-4)
    monkeypatch.setenv("SNAPMRF_GN_LAYOUT", layout)
    got, pd_g, m0_g = run_gn(snap, theta0, x, h, w, 2, tol=1e-4)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(pd_g, pd_w)
    np.testing.assert_array_equal(m0_g, m0_w)
