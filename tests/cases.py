"""Test cases shared by the CPU and GPU suites.

REFERENCE_DICT_CASES restates the inputs of the reference's own dictionary
unit tests (src/test.cu:43-203): schedule built by generate_echo
(src/functions.cu:1588-1598, constant rows) or read from data/MRF_5.csv,
grid strings for T1/T2/B0/B1, 101 EPG states.  The expected outputs are the
golden atoms in tests/golden/golden.npz.
"""
from __future__ import annotations

import math

import numpy as np


def generate_echo(nreps: int, alpha: float, phi: float, TR: float, TE: float) -> np.ndarray:
    """Constant schedule h_echo[4][nreps] (generate_echo)."""
    return np.array([[alpha] * nreps, [phi] * nreps, [TR] * nreps, [TE] * nreps], np.float32)


# name -> (echo_type, schedule or "mrf5", T1, T2, B0, B1)
REFERENCE_DICT_CASES = {
    "epg_se": ("epg_se", generate_echo(1, math.pi, 0.0, 1000.0, 25.0),
               "600:600:600", "100:100:100", "0:1:0", "1"),
    "epg_sr": ("epg_sr", generate_echo(10, math.pi / 3, math.pi / 2, 500.0, 1.0),
               "600", "100", "0", "1"),
    "epg_tse1": ("epg_tse1", generate_echo(3, 2 * math.pi / 3, 0.0, 0.0, 0.0),
                 "1000:1000:1000", "100:100:100", "0:1:0", "1"),
    "epg_tse2": ("epg_tse2", generate_echo(10, math.pi, 0.0, 50.0, 25.0),
                 "600:600:600", "100:100:100", "0:1:0", "1"),
    "epg_fisp": ("epg_fisp", generate_echo(3, math.pi / 6, 0.0, 10.0, 5.0),
                 "1000:1000", "100:100", "0:0", "1"),
    "epg_ssfp": ("epg_ssfp", "mrf5", "100:100:200", "20+20:20:40+1000", "0", "1"),
    "roa_ssfp": ("roa_ssfp", "mrf5", "100:100:200", "20+20:20:40+1000", "0", "1"),
}

# The reference's matching self-test picks 10 atoms of atoms_mrf.ra with
# glibc rand() % 109 (unseeded): these are those indices.
MATCH_SELFTEST_INDICES = [66, 14, 11, 98, 101, 89, 9, 39, 88, 52]


def reference_grid(T1: str, T2: str, B0: str, B1: str) -> np.ndarray:
    """params table for grid strings, restated in numpy (used to build
    inputs; the product's parser is tested against the reference's own
    output separately)."""
    def parse(s):
        vals = []
        tmp = None
        for count, rng in enumerate(s.split("+"), 1):
            parts = rng.split(":")
            mn = np.float32(float(parts[0]))
            if len(parts) == 1:
                st, mx, n = np.float32(0), mn, 1
            elif len(parts) == 2:
                st, mx = np.float32(1), np.float32(float(parts[1]))
                n = int(np.float32(np.float32(mx - mn) / np.float32(1)) + np.float32(1))
            else:
                st, mx = np.float32(float(parts[1])), np.float32(float(parts[2]))
                n = int(np.float32(np.float32(mx - mn) / st) + np.float32(1))
            start = mn
            if count == 1:
                tmp = np.float32(mn + np.float32(n - 1) * st)
            else:
                if abs(np.float32(tmp - mn)) < 1e-7:
                    n -= 1
                    start = np.float32(mn + st)
                tmp = np.float32(mn + np.float32(n) * st)
            vals += [np.float32(start + np.float32(i) * st) for i in range(n)]
        return np.array(vals, np.float32)

    t1, t2, b0, b1 = parse(T1), parse(T2), parse(B0), parse(B1)
    rows = [(a, b, c, d) for d in b1 for c in b0 for b in t2 for a in t1 if a > b]
    return np.array(rows, np.float32).reshape(-1, 4), len(b1)


def reference_case_inputs(name: str, golden) -> tuple:
    """(echo, h_mrf, params, NATOMS, natoms, nreps) for a reference test case."""
    echo, sched, T1, T2, B0, B1 = REFERENCE_DICT_CASES[name]
    h_mrf = golden["mrf5"] if isinstance(sched, str) else sched
    params, l_b1 = reference_grid(T1, T2, B0, B1)
    NATOMS = params.shape[0]
    return echo, np.ascontiguousarray(h_mrf, np.float32), params, NATOMS, NATOMS // l_b1, h_mrf.shape[1]


def mrf_schedule(T: int, seed: int, fa_deg=lambda t: 10.0 + 50.0 * abs(math.sin(math.pi * t / 250.0)),
                 tr=(11.0, 15.0), inversion: bool = True, phase_deg=None) -> np.ndarray:
    """A raw (radian / ms) FISP schedule: flip alpha_t, phase, TR_t ~ U[tr],
    TE = TR/2; alpha_0 = 180 deg when inversion."""
    rng = np.random.default_rng(seed)
    a = np.array([fa_deg(t) for t in range(T)], np.float64)
    if inversion:
        a[0] = 180.0
    TR = rng.uniform(tr[0], tr[1], T)
    ph = np.zeros(T) if phase_deg is None else np.array([phase_deg(t) for t in range(T)], np.float64)
    return np.array([np.deg2rad(a), np.deg2rad(ph), TR, TR / 2], np.float32)


def c4_ssfp_csv(T: int = 500, seed: int = 4) -> np.ndarray:
    """The bSSFP schedule of the large off-resonance configuration:
    alpha_t = 5 + 55 |sin(pi t / 200)| deg, phase alternating 0 / 180 deg,
    TR ~ U[10, 14] ms, TE = TR / 2, written in the epg_ssfp / roa_ssfp CSV
    convention (fraction of 60 deg, deg, TR - 16, TE - 3.5;
    src/functions.cu:1240-1261)."""
    rng = np.random.default_rng(seed)
    t = np.arange(T)
    fa = (5.0 + 55.0 * np.abs(np.sin(np.pi * t / 200.0))) / 60.0
    ph = np.where(t % 2 == 0, 0.0, 180.0)
    tr = rng.uniform(10.0, 14.0, T)
    return np.array([fa, ph, tr - 16.0, tr / 2 - 3.5], np.float32)


def geometric_grid(lo: float, hi: float, ratio: float = 1.05) -> np.ndarray:
    """lo * ratio^k <= hi (the 5 % relaxation-time grids)."""
    return np.array([lo * ratio ** k for k in range(400) if lo * ratio ** k <= hi], np.float32)


def rel_err_per_atom(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """max_t |a - b| / max_t |b| per atom (rows)."""
    num = np.abs(a - b).max(axis=-1)
    den = np.abs(b).max(axis=-1)
    return num / np.maximum(den, 1e-30)


# Inputs whose reference outputs are recorded in tests/golden/golden.npz by
# tests/golden/make_golden.py (run through the reference's own host code).
GRID_CASES = [
    ("600:600:600", "100:100:100", "0:1:0", "1"),
    ("600", "100", "0", "1"),
    ("1000:1000:1000", "100:100:100", "0:1:0", "1"),
    ("1000:1000", "100:100", "0:0", "1"),
    ("100:100:200", "20+20:20:40+1000", "0", "1"),
    ("20:20:3000", "20:10:1000", "0", "1"),
    ("100:10:200", "10:10:100", "0", "1"),
    ("100:100:3000", "20:10:300", "0", "1"),
    ("100:100:1000", "20:20:200", "-50:25:50", "0.6:0.2:1.4"),
    ("0:1:2+2.5:1:4", "0.5", "0", "1"),
    ("20:10:100+110:10:200", "5", "0", "1"),
    ("1:0.1:2", "0.05:0.05:0.5", "0", "0.6:0.02:1.4"),
    ("300+100:50:500+500:100:900", "10:5:60", "-3:1.5:3", "0.9:0.05:1.1"),
]
LOGSPACE_CASES = [(100.0, 3000.0, 7), (20.0, 1000.0, 5), (-150.0, 150.0, 21), (-150.0, 150.0, 20),
                  (0.5, 1.5, 11), (3.0, 3.0, 1), (5.0, 1.0, 4), (0.0, 100.0, 9)]
GRIDN_CASES = [2000, 23100, 100000]
CSV_CASES = {
    # header of exactly 99 characters: only the header is skipped
    "hdr99": "h" * 99 + "\n" + "0.5,0,1.5,0\n0.25,90,1.25,0.5\n1,180,0,0\n",
    # short header: the first data row is skipped as well (two fgets chunks)
    "hdr10": "flip,phase\n" + "0.5,0,1.5,0\n0.25,90,1.25,0.5\n1,180,0,0\n",
    # long header: three chunks, the tail of the header row is read as data
    "hdr150": "x" * 150 + "\n" + "0.5,0,1.5,0\n0.25,90,1.25,0.5\n",
}
