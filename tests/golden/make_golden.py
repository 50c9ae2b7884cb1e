"""Regenerates tests/golden/golden.npz from the reference.

Run in a container that has the reference tree (REF_ROOT, default: a
checkout named "reference" beside this repository) and the reference harness built (`make -C oracle ref`):

    python tests/golden/make_golden.py

Contents:
  atoms_<echo>      the reference's golden dictionaries (data/atoms_*.ra),
                    produced by the inputs of src/test.cu:43-203
  atoms_mrf, params_mrf  the matching self-test dictionary (data/atoms_mrf.ra,
                    data/params_mrf.ra, src/functions.cu:1720-1824)
  mrf5              data/MRF_5.csv as read by the reference's csv_read
  grid_<i>          params tables from the reference's own parse_length /
                    parse_params / compute_natoms / trans_params for the grid
                    strings in GRID_CASES (run through oracle/_ref/ref_harness)
  logspace_<i>      the reference's logspace for LOGSPACE_CASES
  gridN_<n>         the -N hard-coded grids (src/mrf.cu:179-203)
  csv_<name>        csv_read of the small CSV texts in CSV_CASES
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REF = Path(os.environ.get("REF_ROOT", str(Path(__file__).resolve().parents[3] / "reference")))
HARNESS = REPO / "oracle" / "_ref" / "ref_harness"

sys.path.insert(0, str(HERE.parent))
from cases import CSV_CASES, GRID_CASES, GRIDN_CASES, LOGSPACE_CASES  # noqa: E402


def ra_read(path: Path) -> np.ndarray:
    b = path.read_bytes()
    hdr = np.frombuffer(b[:48], dtype="<u8")
    _, _, eltype, elbyte, size, ndims = (int(x) for x in hdr)
    dims = [int(d) for d in np.frombuffer(b[48:48 + 8 * ndims], dtype="<u8")]
    dt = {(3, 4): "<f4", (4, 8): "<c8"}[(eltype, elbyte)]
    off = 48 + 8 * ndims
    return np.frombuffer(b[off:off + size], dtype=dt).reshape(tuple(reversed(dims))).copy()


def harness(*args: str) -> str:
    r = subprocess.run([str(HARNESS), *args], stdin=subprocess.DEVNULL, capture_output=True,
                       text=True, check=True)
    return r.stdout


def main() -> None:
    if not HARNESS.exists():
        sys.exit("build the reference harness first: make -C oracle ref")
    out: dict[str, np.ndarray] = {}
    for name in ["epg_se", "epg_sr", "epg_tse1", "epg_tse2", "epg_fisp", "epg_ssfp", "roa_ssfp"]:
        out["atoms_" + name] = ra_read(REF / "data" / f"atoms_{name}.ra")
    out["atoms_mrf"] = ra_read(REF / "data" / "atoms_mrf.ra")
    out["params_mrf"] = ra_read(REF / "data" / "params_mrf.ra")
    with tempfile.TemporaryDirectory() as td:
        t = Path(td)
        harness("csv", str(REF / "data" / "MRF_5.csv"), str(t / "m5.f32"))
        out["mrf5"] = np.fromfile(t / "m5.f32", np.float32).reshape(4, -1)
        for i, (a, b, c, d) in enumerate(GRID_CASES):
            line = harness("grid", a, b, c, d, str(t / "g.f32")).split()
            p = np.fromfile(t / "g.f32", np.float32).reshape(-1, 4)
            out[f"grid_{i}"] = p
            out[f"grid_{i}_dims"] = np.array([int(x) for x in line], np.int64)
        for i, (mn, mx, n) in enumerate(LOGSPACE_CASES):
            harness("logspace", repr(mn), repr(mx), str(n), str(t / "l.f32"))
            out[f"logspace_{i}"] = np.fromfile(t / "l.f32", np.float32)
        for n in GRIDN_CASES:
            line = harness("gridN", str(n), str(t / "n.f32")).split()
            out[f"gridN_{n}"] = np.fromfile(t / "n.f32", np.float32).reshape(-1, 4)
            out[f"gridN_{n}_dims"] = np.array([int(x) for x in line], np.int64)
        for name, text in CSV_CASES.items():
            (t / f"{name}.csv").write_text(text)
            rows = int(harness("csv", str(t / f"{name}.csv"), str(t / "c.f32")).split()[0])
            out[f"csv_{name}"] = np.fromfile(t / "c.f32", np.float32).reshape(4, rows)
    np.savez_compressed(HERE / "golden.npz", **out)
    print(f"wrote {HERE / 'golden.npz'} ({len(out)} arrays)")


if __name__ == "__main__":
    main()
