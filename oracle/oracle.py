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
