"""The mrf CLI of this package: matching against a saved dictionary
(--load-atoms / --load-params) gives the maps of the run that generated it,
and --refine refines them."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CLI = ROOT / "snapmrf_b200" / "mrf"
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not CLI.exists(), reason="mrf CLI not built")]

HEADER = "flip_angle_(fraction_of_nominal),rf_phase_(deg),extension_of_base_TR_(ms),extension_of_base_TE_(ms)"


def _run(args, cwd):
    r = subprocess.run([str(CLI), *args], cwd=cwd, stdin=subprocess.DEVNULL, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_cli_saved_dictionary_and_refinement(snap, tmp_path):
    T = 200
    rng = np.random.default_rng(40)
    a = np.deg2rad(10 + 50 * np.abs(np.sin(np.pi * np.arange(T) / 70)))
    tr = rng.uniform(11, 15, T)
    sched = np.array([a, np.zeros(T), tr, tr / 2], np.float32)     # raw epg_fisp schedule
    rows = "\n".join(",".join(repr(float(v)) for v in sched[:, t]) for t in range(T))
    (tmp_path / "sched.csv").write_text(HEADER + "\n" + rows + "\n")
    grid = ["-e", "epg_fisp", "-t", "300:100:2000", "-s", "30:10:200", "-b", "0", "-r", "0.9:0.1:1.1",
            "-w", "20", "-T", str(T), "--all-b1-blocks", "--normalize"]
    _run(grid + ["sched.csv", "-a", "atoms.ra", "-p", "params.ra"], tmp_path)
    atoms = snap.ra_read(str(tmp_path / "atoms.ra"))
    params = snap.ra_read(str(tmp_path / "params.ra"))
    n = 60
    pick = rng.integers(0, atoms.shape[0], n)
    img = atoms[pick] * (rng.uniform(0.5, 1, n) * np.exp(1j * rng.uniform(0, 6.28, n)))[:, None]
    img = (img + 0.003 * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape))).astype(np.complex64)
    snap.ra_write(str(tmp_path / "img.ra"), img.reshape(6, 10, T))
    snap.ra_write(str(tmp_path / "b1.ra"), params[pick, 3].astype(np.float32).reshape(6, 10))
    _run(grid + ["sched.csv", "img.ra", "-M", "b1.ra", "-m", "maps_gen.ra"], tmp_path)
    out = _run(["-e", "epg_fisp", "-w", "20", "-T", str(T), "sched.csv", "img.ra", "-M", "b1.ra",
                "--load-atoms", "atoms.ra", "--load-params", "params.ra", "-m", "maps_load.ra"], tmp_path)
    assert "Constructing dictionary" not in out
    m_gen = snap.ra_read(str(tmp_path / "maps_gen.ra"))
    m_load = snap.ra_read(str(tmp_path / "maps_load.ra"))
    np.testing.assert_array_equal(m_gen, m_load)
    # refinement keeps B1 from the map, moves T1 / T2 off the grid, keeps them positive
    _run(grid + ["sched.csv", "img.ra", "-M", "b1.ra", "-m", "maps_ref.ra", "--refine", "3"], tmp_path)
    m_ref = snap.ra_read(str(tmp_path / "maps_ref.ra")).reshape(-1, 5)
    m_gen = m_gen.reshape(-1, 5)
    assert np.all(m_ref[:, 1] > 0) and np.all(m_ref[:, 0] > m_ref[:, 1])
    np.testing.assert_allclose(m_ref[:, 0], m_gen[:, 0], rtol=0.2)
    assert np.mean(m_ref[:, 0] != m_gen[:, 0]) > 0.5


def test_cli_compressed_matching(snap, tmp_path):
    """--compress: the bases and compressed atoms written in MATLAB's layouts
    (U_r as (nreps, r x blocks), dict_compress as (r, NATOMS)), orthonormal
    bases, coordinates U_r^H d, and FP16 compressed matching (rescored in
    FP32) picking the uncompressed FP32 run's atoms."""
    T = 200
    rng = np.random.default_rng(41)
    a = np.deg2rad(10 + 50 * np.abs(np.sin(np.pi * np.arange(T) / 70)))
    tr = rng.uniform(11, 15, T)
    sched = np.array([a, np.zeros(T), tr, tr / 2], np.float32)
    rows = "\n".join(",".join(repr(float(v)) for v in sched[:, t]) for t in range(T))
    (tmp_path / "sched.csv").write_text(HEADER + "\n" + rows + "\n")
    grid = ["-e", "epg_fisp", "-t", "300:100:2000", "-s", "30:10:200", "-b", "0", "-r", "0.9:0.1:1.1",
            "-w", "20", "-T", str(T), "--all-b1-blocks", "--normalize"]
    _run(grid + ["sched.csv", "-a", "atoms.ra", "-p", "params.ra"], tmp_path)
    atoms = snap.ra_read(str(tmp_path / "atoms.ra")).astype(np.complex128)
    params = snap.ra_read(str(tmp_path / "params.ra"))
    n = 200
    pick = rng.integers(0, atoms.shape[0], n)
    img = atoms[pick] * (rng.uniform(0.5, 1, n) * np.exp(1j * rng.uniform(0, 6.28, n)))[:, None]
    img = (img + 0.003 * (rng.standard_normal(img.shape) + 1j * rng.standard_normal(img.shape))).astype(np.complex64)
    snap.ra_write(str(tmp_path / "img.ra"), img.reshape(10, 20, T))
    snap.ra_write(str(tmp_path / "b1.ra"), params[pick, 3].astype(np.float32).reshape(10, 20))
    _run(grid + ["sched.csv", "img.ra", "-M", "b1.ra", "-m", "maps32.ra"], tmp_path)
    out = _run(grid + ["sched.csv", "img.ra", "-M", "b1.ra", "-m", "maps_c.ra", "--precision", "fp16",
                       "--compress", "0.99999", "--max-rank", "32", "--out-basis", "basis.ra",
                       "--out-compressed", "comp.ra"], tmp_path)
    r = int(out.split("Rank: ")[1].split()[0])
    nb = 3
    natoms = atoms.shape[0] // nb
    basis = snap.ra_read(str(tmp_path / "basis.ra")).astype(np.complex128)
    comp = snap.ra_read(str(tmp_path / "comp.ra")).astype(np.complex128)
    assert 1 <= r <= 32 and basis.shape == (nb * r, T) and comp.shape == (atoms.shape[0], r)
    for b in range(nb):
        U = basis[b * r:(b + 1) * r]
        np.testing.assert_allclose(U @ np.conj(U).T, np.eye(r), atol=1e-5)
        want = atoms[b * natoms:(b + 1) * natoms] @ np.conj(U).T
        assert np.max(np.abs(comp[b * natoms:(b + 1) * natoms] - want)) <= 1e-5
    m32 = snap.ra_read(str(tmp_path / "maps32.ra")).reshape(-1, 5)
    mc = snap.ra_read(str(tmp_path / "maps_c.ra")).reshape(-1, 5)
    same = np.all(m32[:, :4] == mc[:, :4], axis=1)
    print(f"rank {r}: {same.mean():.4f} of the picks equal the FP32 run's")
    assert same.mean() >= 0.97
    np.testing.assert_allclose(mc[same, 4], m32[same, 4], rtol=1e-5)
