"""ctypes wrapper of liboracle.so, the CPU restatement of snapMRF's path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product (snapmrf_b200/)
never imports it.  Built by `make -C oracle` (or build() below).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_HARNESS = HERE / "_ref" / "ref_harness"

ALL_B1_BLOCKS = 1
NORMALIZE = 2

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        sz, vp = C.c_size_t, C.c_void_p
        for suf in ("f64", "f32"):
            f = getattr(L, "oracle_dict_" + suf)
            f.restype = C.c_int
            f.argtypes = [vp, vp, vp, vp, sz, sz, sz, sz, C.c_int, C.c_int, C.c_char_p, C.c_uint,
                          C.c_int, C.c_int]
            g = getattr(L, "oracle_match_" + suf)
            g.restype = C.c_int
            g.argtypes = [vp, vp, vp, vp, vp, sz, sz, sz, sz, sz, sz, C.c_int, vp, C.c_int]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def max_threads() -> int:
    return lib().oracle_max_threads()


def dict_atoms(echo: str, params, h_mrf, nreps: int, natoms: int | None = None, nstates: int = 101,
               flags: int = 0, n_iso: int = 1, precision: str = "f64", nthreads: int = 1,
               return_norms: bool = False):
    """MRF_dict restated on the CPU.  Returns complex128 [gen_atoms][nreps]
    for the blocks the echo type generates (block 0 only for the non-SSFP
    types unless ALL_B1_BLOCKS)."""
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 4)
    h_mrf = np.ascontiguousarray(h_mrf, np.float32)
    NREPS = h_mrf.shape[-1]
    NATOMS = params.shape[0]
    natoms = natoms or NATOMS
    out = np.zeros((NATOMS, nreps, 2), np.float64)
    norms = np.zeros(NATOMS, np.float64)
    f = getattr(lib(), "oracle_dict_" + precision)
    r = f(out.ctypes.data, norms.ctypes.data, params.ctypes.data, h_mrf.ctypes.data, nreps, NREPS,
          NATOMS, natoms, 4, nstates, echo.encode(), flags, n_iso, nthreads)
    if r <= 0:
        raise RuntimeError(f"oracle_dict failed: {r}")
    gen = r * natoms
    atoms = out[:gen, :, 0] + 1j * out[:gen, :, 1]
    return (atoms, norms[:gen]) if return_norms else atoms


def match(img, atoms, params, nreps: int, natoms: int | None = None, b1map=None,
          precision: str = "f64", nthreads: int = 1):
    """MRF_match restated: returns (maps [nvox][5] float32, index [nvox])."""
    img = np.ascontiguousarray(img, np.complex64)
    atoms = np.ascontiguousarray(atoms, np.complex64)
    params = np.ascontiguousarray(params, np.float32).reshape(-1, 4)
    nvox = img.shape[0]
    NATOMS = atoms.shape[0]
    natoms = natoms or NATOMS
    maps = np.zeros((nvox, 5), np.float32)
    idx = np.zeros(nvox, np.int64)
    b1 = None if b1map is None else np.ascontiguousarray(b1map, np.float32).reshape(-1)
    f = getattr(lib(), "oracle_match_" + precision)
    r = f(maps.ctypes.data, idx.ctypes.data, img.ctypes.data, atoms.ctypes.data, params.ctypes.data,
          nreps, img.shape[1], atoms.shape[1], NATOMS, natoms, nvox, 4,
          None if b1 is None else b1.ctypes.data, nthreads)
    if r != 0:
        raise RuntimeError(f"oracle_match failed: {r}")
    return maps, idx


def fisp_jvp(theta, tangent, h_mrf, nstates: int = 101, echo: str = "epg_fisp", dalpha=None, y=None):
    """FP64 forward-mode derivative of the real FISP / SR recursion (every
    RF phase 0) along one direction.

    theta = (T1, T2, B1), tangent = (dT1, dT2, dB1), optional dalpha [T]
    (direction in the flip-angle schedule), optional targets y complex [T].
    Returns (Im s [T], d Im s [T], loss, dloss) with loss = sum |s - y|^2
    (0, 0 without y)."""
    h_mrf = np.ascontiguousarray(h_mrf, np.float32)
    T = h_mrf.shape[-1]
    sig = np.zeros(T, np.float64)
    dsig = np.zeros(T, np.float64)
    loss = C.c_double(0)
    dloss = C.c_double(0)
    da = None if dalpha is None else np.ascontiguousarray(dalpha, np.float64)
    yy = None if y is None else np.ascontiguousarray(np.stack([np.real(y), np.imag(y)], -1), np.float64)
    if echo not in ("epg_fisp", "epg_sr"):
        raise ValueError("fisp_jvp covers epg_fisp and epg_sr")
    f = lib().oracle_fisp_jvp_f64
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_double] * 6 + \
        [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p]
    r = f(sig.ctypes.data, dsig.ctypes.data, C.byref(loss), C.byref(dloss), *map(float, theta),
          *map(float, tangent), h_mrf.ctypes.data, None if da is None else da.ctypes.data, T, nstates,
          1 if echo == "epg_fisp" else 0, None if yy is None else yy.ctypes.data)
    if r != 0:
        raise RuntimeError(f"oracle_fisp_jvp failed: {r}")
    return sig, dsig, loss.value, dloss.value


def ssfp_schedule(h_csv, nreps: int | None = None) -> np.ndarray:
    """The epg_ssfp conversion of a CSV schedule as MRF_dict does it
    (src/functions.cu:1240-1261): flip fraction x 60 deg in rad, phase deg
    -> rad, TR + 16 ms, TE + 3.5 ms, in float32."""
    h = np.asarray(h_csv, np.float32)
    n = nreps or h.shape[1]
    fa_scale = np.float32(60.0 * np.pi / 180.0)
    ph_scale = np.float32(np.pi / 180.0)
    return np.array([h[0, :n] * fa_scale, h[1, :n] * ph_scale, h[2, :n] + np.float32(16.0),
                     h[3, :n] + np.float32(3.5)], np.float32)


def ssfp_jvp(theta, tangent, h_csv, nstates: int = 101, TI: float = 40.0):
    """FP64 forward mode of the complex bSSFP recursion (epg_ssfp, no
    normalisation) along one direction: theta = (T1, T2, B0, B1), tangent =
    (dT1, dT2, dB0, dB1), h_csv the schedule in the CSV convention.
    Returns (s [T] complex, ds [T] complex)."""
    mrf = np.ascontiguousarray(ssfp_schedule(h_csv))
    T = mrf.shape[1]
    sig = np.zeros(2 * T, np.float64)
    dsig = np.zeros(2 * T, np.float64)
    f = lib().oracle_ssfp_jvp_f64
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p] + [C.c_double] * 8 + [C.c_void_p, C.c_size_t, C.c_int, C.c_double]
    r = f(sig.ctypes.data, dsig.ctypes.data, *map(float, theta), *map(float, tangent), mrf.ctypes.data, T,
          nstates, TI)
    if r != 0:
        raise RuntimeError(f"oracle_ssfp_jvp failed: {r}")
    return sig[0::2] + 1j * sig[1::2], dsig[0::2] + 1j * dsig[1::2]


def ssfp_gn_step_f64(theta, x, h_csv, nstates: int = 101, refine_b1: bool = True):
    """One projected Gauss-Newton step of (T1, T2, B0[, B1]) in FP64 for one
    voxel under x = rho * s(theta), s the bSSFP signal, rho complex and
    eliminated by variable projection.  Returns (step, |rho|, |<s,x>|/||s||)."""
    n = 4 if refine_b1 else 3
    cols, s = [], None
    for j in range(n):
        tg = [0.0] * 4
        tg[j] = 1.0
        s, ds = ssfp_jvp(theta, tg, h_csv, nstates)
        cols.append(ds)
    J = np.stack(cols, 1)
    x = np.asarray(x, np.complex128)
    ss = np.vdot(s, s).real
    rho = np.vdot(s, x) / ss
    Pj = J - np.outer(s, (s.conj() @ J) / ss)
    A = (abs(rho) ** 2) * (Pj.conj().T @ Pj).real
    b = (np.conj(rho) * (Pj.conj().T @ x)).real
    return np.linalg.solve(A, b), abs(rho), abs(np.vdot(s, x)) / np.sqrt(ss)


def trans_params(t1, t2, b0, b1) -> np.ndarray:
    """params[NATOMS][4] = {T1, T2, B0, B1} restated from trans_params
    (src/functions.cu:355-391): B1 outermost, then B0, then T2, T1
    innermost, keeping T1 > T2 strictly (compute_natoms, :393-414)."""
    t1, t2, b0, b1 = (np.asarray(v, np.float32).reshape(-1) for v in (t1, t2, b0, b1))
    rows = [(a, b, c, d) for d in b1 for c in b0 for b in t2 for a in t1 if a > b]
    return np.array(rows, np.float32).reshape(-1, 4)


def gn_step_f64(theta, x, h_mrf, nstates: int = 101, echo: str = "epg_fisp"):
    """One projected Gauss-Newton step of (T1, T2) in FP64 for one voxel x
    (complex [T]) under the model x = rho * s(T1, T2, B1), s = i f the real
    FISP / SR signal, rho complex and eliminated by variable projection.  The
    refinement has no counterpart in the reference; this is the checker's
    FP64 statement of it, built on the forward-mode derivatives above.
    theta = (T1, T2, B1).  Returns (step [2], |rho|, |<s, x>| / ||s||)."""
    s, d1, _, _ = fisp_jvp(theta, (1, 0, 0), h_mrf, nstates=nstates, echo=echo)
    _, d2, _, _ = fisp_jvp(theta, (0, 1, 0), h_mrf, nstates=nstates, echo=echo)
    s, J = 1j * s, np.stack([1j * d1, 1j * d2], 1)
    x = np.asarray(x, np.complex128)
    rho = np.vdot(s, x) / np.vdot(s, s)
    ss = np.vdot(s, s).real
    Pj = J - np.outer(s, (s.conj() @ J) / ss)
    A = (abs(rho) ** 2) * (Pj.conj().T @ Pj).real
    b = (np.conj(rho) * (Pj.conj().T @ x)).real
    return np.linalg.solve(A, b), abs(rho), abs(np.vdot(s, x)) / np.sqrt(ss)


def refine_gn_f64(theta, x, h_mrf, nstates: int = 101, echo: str = "epg_fisp", iterations: int = 40,
                  tol: float = 1e-12, max_rel_step: float = 0.2):
    """FP64 Gauss-Newton of (T1, T2) from theta = (T1, T2, B1) iterated to
    convergence (every step at most max_rel_step of each value, T1 > T2 > 0
    kept): the least-squares fit of one voxel.  Returns (T1, T2, PD) with PD =
    |<s, x>| / ||s|| at the result."""
    t1, t2, b1 = (float(v) for v in theta)
    for _ in range(iterations):
        d, _, _ = gn_step_f64((t1, t2, b1), x, h_mrf, nstates, echo)
        d = np.clip(d, [-max_rel_step * t1, -max_rel_step * t2], [max_rel_step * t1, max_rel_step * t2])
        n2 = max(t2 + d[1], 1e-3)
        n1 = max(t1 + d[0], n2 * (1 + 1e-4))
        done = abs(n1 - t1) <= tol * t1 and abs(n2 - t2) <= tol * t2
        t1, t2 = n1, n2
        if done:
            break
    _, _, pd = gn_step_f64((t1, t2, b1), x, h_mrf, nstates, echo)
    return t1, t2, pd


START_C, START_UM, START_UP, START_VM, START_VP, START_D = range(6)


def _stencil_f64(params, base: int, n: int, j: int):
    """Six-point stencil of block-local row j in the block starting at
    `base`, or None: [matched, T1 below, T1 above, T2 below, T2 above,
    diagonal] as block-local rows, and whether the diagonal is (T1 above, T2
    above) (else T1 below, T2 below).  T1 neighbours are the adjacent table
    rows in the matched T2 row; the T2 neighbours are the rows holding the
    matched T1 in the adjacent T2 rows of the table (trans_params order,
    src/functions.cu:355-391)."""
    P = params[base:base + n]
    t1, t2, b0 = P[:, 0], P[:, 1], P[:, 2]
    if j < 1 or j + 1 >= n:
        return None
    T1m, T1c, T1p, T2c, B0c = t1[j - 1], t1[j], t1[j + 1], t2[j], b0[j]
    if t2[j - 1] != T2c or t2[j + 1] != T2c or b0[j - 1] != B0c or b0[j + 1] != B0c:
        return None
    if not ((T1m < T1c < T1p) or (T1m > T1c > T1p)):
        return None
    T2n, rcs = [], []
    for d in (-1, 1):
        r = j + 2 * d
        while 0 <= r < n and t2[r] == T2c and b0[r] == B0c:
            r += d
        if not 0 <= r < n:
            return None
        T2r = t2[r]
        if b0[r] != B0c or not T2r != T2c or not np.isfinite(T2r):
            return None
        while 0 <= r < n and t2[r] == T2r and b0[r] == B0c and t1[r] != T1c:
            r += d
        if not 0 <= r < n:
            return None
        if not (t1[r] == T1c and t2[r] == T2r and b0[r] == B0c):
            return None
        T2n.append(T2r)
        rcs.append(r)
    if not (T2n[0] != T2n[1] and (T2n[0] < T2c) == (T2c < T2n[1])):
        return None
    st = [j, j - 1, j + 1, rcs[0], rcs[1], None]
    du, dm = rcs[1] + 1, rcs[0] - 1
    if du < n and t1[du] == T1p and t2[du] == T2n[1] and b0[du] == B0c:
        st[START_D] = du
        return st, True
    if dm >= 0 and t1[dm] == T1m and t2[dm] == T2n[0] and b0[dm] == B0c:
        st[START_D] = dm
        return st, False
    return None


def refine_start_f64(maps, index, atoms, params, img, natoms: int, b1map=None, iterations: int = 10):
    """Sub-grid start of the refinement (snapmrf_refine_start) in FP64.  No
    counterpart in the reference; this is the checker's statement of it.

    Per voxel: the matched atom's six-point stencil (_stencil_f64); with a B1
    map, the stencil of the three B1 blocks around the match (clamped to the
    table) interpolated quadratically (Lagrange) to the voxel's B1.  In
    (U, V) = (log T1 / T1c, log T2 / T2c) the six signals give the quadratic
    surrogate s = c + a U + b V + d U^2 + e V^2 + f U V (a, d through the
    three nodes along T1; b, e along T2; f from the diagonal node's residual).
    `iterations` Gauss-Newton steps with variable projection on it (each step
    clipped to half the stencil's width, the point kept within 1.5 times the
    stencil's extent on each side) from U = V = 0.  Returns (maps with the
    new T1, T2 as float32, mask of the voxels moved)."""
    maps = np.array(maps, np.float32, copy=True)
    atoms = np.asarray(atoms)
    params = np.asarray(params, np.float32)
    NATOMS = params.shape[0]
    nb = NATOMS // natoms
    moved = np.zeros(maps.shape[0], bool)

    def quad(sm, s0, sp, hm, hp):
        q = ((sp - s0) / hp - (sm - s0) / hm) / (hp - hm)
        return (sp - s0) / hp - q * hp, q

    for v in range(maps.shape[0]):
        k = int(index[v])
        if k < 0 or k >= NATOMS:
            continue
        b, j = divmod(k, natoms)
        T1c, T2c = params[k, 0], params[k, 1]
        if maps[v, 0] != T1c or maps[v, 1] != T2c or not (T1c > T2c) or not (T2c > 0):
            continue
        found = _stencil_f64(params, b * natoms, natoms, j)
        if found is None:
            continue
        st, diag_up = found
        bb = b * natoms
        qbase, qw = [bb], [1.0]
        if b1map is not None and nb >= 3:
            bs = min(max(b - 1, 0), nb - 3)
            qbase = [(bs + q) * natoms for q in range(3)]
            nodes = [float(params[qb + j, 3]) for qb in qbase]
            ok = all(params[bb + r, m] == params[qb + r, m] for qb in qbase for r in st for m in range(3))
            ok = ok and all(params[qb + r, 3] == nd for qb, nd in zip(qbase, nodes) for r in st)
            if not ok or len(set(nodes)) < 3:
                continue
            bv = float(b1map[v])
            if not np.isfinite(bv):
                continue
            n0, n1, n2 = nodes
            qw = [(bv - n1) * (bv - n2) / ((n0 - n1) * (n0 - n2)), (bv - n0) * (bv - n2) / ((n1 - n0) * (n1 - n2)),
                  (bv - n0) * (bv - n1) / ((n2 - n0) * (n2 - n1))]
        S = [sum(w * atoms[qb + r].astype(np.complex128) for w, qb in zip(qw, qbase)) for r in st]
        hum = np.log(params[bb + st[START_UM], 0] / np.float64(T1c))
        hup = np.log(params[bb + st[START_UP], 0] / np.float64(T1c))
        hvm = np.log(params[bb + st[START_VM], 1] / np.float64(T2c))
        hvp = np.log(params[bb + st[START_VP], 1] / np.float64(T2c))
        hud, hvd = (hup, hvp) if diag_up else (hum, hvm)
        c = S[START_C]
        a_, d_ = quad(S[START_UM], c, S[START_UP], hum, hup)
        b_, e_ = quad(S[START_VM], c, S[START_VP], hvm, hvp)
        f_ = (S[START_D] - c - a_ * hud - b_ * hvd - d_ * hud ** 2 - e_ * hvd ** 2) / (hud * hvd)
        M = np.array([c, a_, b_, d_, e_, f_])
        Gh = M.conj() @ M.T
        pv = M.conj() @ np.asarray(img[v], np.complex128)
        ulo, uhi = 1.5 * min(hum, hup), 1.5 * max(hum, hup)
        vlo, vhi = 1.5 * min(hvm, hvp), 1.5 * max(hvm, hvp)
        lu, lv = 0.5 * (max(hum, hup) - min(hum, hup)), 0.5 * (max(hvm, hvp) - min(hvm, hvp))
        U = V = 0.0
        for _ in range(iterations):
            c0 = np.array([1.0, U, V, U * U, V * V, U * V])
            c1 = np.array([0.0, 1.0, 0.0, 2 * U, 0.0, V])
            c2 = np.array([0.0, 0.0, 1.0, 0.0, 2 * V, U])
            Ss = (c0 @ Gh @ c0).real
            g1, g2 = c0 @ Gh @ c1, c0 @ Gh @ c2
            H11, H12, H22 = (c1 @ Gh @ c1).real, (c1 @ Gh @ c2).real, (c2 @ Gh @ c2).real
            P, Q1, Q2 = c0 @ pv, c1 @ pv, c2 @ pv
            if not Ss > 0:
                break
            rho = P / Ss
            r2 = abs(rho) ** 2
            A11 = r2 * (H11 - abs(g1) ** 2 / Ss)
            A12 = r2 * (H12 - (np.conj(g1) * g2).real / Ss)
            A22 = r2 * (H22 - abs(g2) ** 2 / Ss)
            b1 = (np.conj(rho) * (Q1 - np.conj(g1) * P / Ss)).real
            b2 = (np.conj(rho) * (Q2 - np.conj(g2) * P / Ss)).real
            det = A11 * A22 - A12 * A12
            if not det > 0 or not A11 > 0 or not np.isfinite(det):
                break
            d1, d2 = (A22 * b1 - A12 * b2) / det, (A11 * b2 - A12 * b1) / det
            if not (np.isfinite(d1) and np.isfinite(d2)):
                break
            U = min(max(U + min(max(d1, -lu), lu), ulo), uhi)
            V = min(max(V + min(max(d2, -lv), lv), vlo), vhi)
        T1, T2 = float(T1c) * np.exp(U), float(T2c) * np.exp(V)
        if not (np.isfinite(T1) and np.isfinite(T2) and T2 > 0 and T1 > T2 * (1 + 1e-4)):
            continue
        maps[v, 0], maps[v, 1] = T1, T2
        moved[v] = True
    return maps, moved


def svd_compress(atoms, natoms: int, sfrac: float | None = None, rank: int | None = None):
    """Low-rank compression per B1 block, restated from matlab/MRF_dict_B1.m:127-159
    (input.reduce = 1) in FP64 numpy:

      per block b (ii = 1..numel(B1_v)): [U, S, ~] = svd(dict_norm_b, 'econ');
      block 0 only: fNRG_v = cumsum(s.^2) ./ sum(s.^2),
                    nDictSpace = sum(fNRG_v <= sfrac)              (:143-147)
      U_r = U(:, 1:nDictSpace); dict_compress = U_r' * dict_norm_b   (:149-150)

    atoms: [NATOMS][nreps] complex, block b = rows [b*natoms, (b+1)*natoms)
    (the columns of MATLAB's nreps x natoms dict_norm).  A fixed `rank`
    replaces the sfrac rule.  Returns (basis [nb][r][nreps] with row i = u_i,
    coeffs [NATOMS][r] = U_r^H d_j, r, singular values [nb][min(nreps, natoms)]).
    """
    atoms = np.asarray(atoms, np.complex128)
    nb = atoms.shape[0] // natoms
    us, ss = [], []
    for b in range(nb):
        D = atoms[b * natoms:(b + 1) * natoms].T
        U, s, _ = np.linalg.svd(D, full_matrices=False)
        us.append(U)
        ss.append(s)
    if rank is None:
        f = np.cumsum(ss[0] ** 2) / np.sum(ss[0] ** 2)
        rank = int(np.sum(f <= sfrac))
    basis = np.stack([U[:, :rank].T for U in us])
    coeffs = np.concatenate([atoms[b * natoms:(b + 1) * natoms] @ np.conj(us[b][:, :rank])
                             for b in range(nb)])
    return basis, coeffs, rank, np.stack(ss)


def match_compressed(img, basis, coeffs, params, natoms: int, b1map=None):
    """Matching in the compressed space (FP64): each voxel is projected onto
    the basis of the B1 block nearest its B1 (the reference's merge rule,
    src/functions.cu:1351-1384: strict '<' from 10, ties to the lower block;
    block 0 without a map) and the first atom of that block with the largest
    |c_j^H U^H x| wins; PD = that modulus.  Returns (maps [nvox][5], index)."""
    img = np.asarray(img, np.complex128)
    coeffs = np.asarray(coeffs, np.complex128)
    params = np.asarray(params, np.float32).reshape(-1, 4)
    nb = coeffs.shape[0] // natoms
    nvox = img.shape[0]
    bins = np.zeros(nvox, np.int64)
    if b1map is not None:
        b1 = np.asarray(b1map, np.float32).reshape(-1)
        heads = params[np.arange(nb) * natoms, 3]
        for v in range(nvox):
            best, dist = 0, np.float32(10.0)
            for k in range(nb):
                d = np.float32(abs(b1[v] - heads[k]))
                if d < dist:
                    best, dist = k, d
            bins[v] = best
    maps = np.zeros((nvox, 5), np.float32)
    idx = np.zeros(nvox, np.int64)
    r = basis.shape[1]
    for b in range(nb):
        sel = np.nonzero(bins == b)[0]
        if sel.size == 0:
            continue
        xc = img[sel, :basis.shape[2]] @ np.conj(np.asarray(basis[b], np.complex128)).T
        C = coeffs[b * natoms:(b + 1) * natoms, :r]
        s = np.abs(xc @ np.conj(C).T)
        j = np.argmax(s, axis=1)
        g = b * natoms + j
        maps[sel, :4] = params[g]
        maps[sel, 4] = s[np.arange(sel.size), j]
        idx[sel] = g
    return maps, idx
