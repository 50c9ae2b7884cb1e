"""Python mirror of the reference's host interface (src/functions.h,
src/ra.h) over the C ABI of libsnapmrf.so (include/snapmrf.h).

Function names and argument meaning follow the reference: MRF_dict,
MRF_match, csv_dim, csv_read, parse_length, parse_params, logspace,
compute_natoms, trans_params, ra_read, ra_write.  Device buffers are passed
as torch CUDA tensors (or raw device addresses); torch is used only for
device memory and streams.  Where the reference prints and exits, these
raise SnapMRFError with the library's message.  There is no CPU fallback:
every compute entry point runs the CUDA kernels of libsnapmrf.so and fails
loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libsnapmrf.so"

NPARAMS = 4  # src/mrf.cu:58
NMAPS = 5    # src/mrf.cu:59

# dictionary flags (include/snapmrf.h)
DICT_ALL_B1_BLOCKS = 0x1
DICT_NORMALIZE = 0x2
DICT_REFERENCE_ORDER = 0x4
DICT_SEPARATE_RELAX = 0x8
DICT_NORMALIZE_OPERAND = 0x10
DICT_IMAG_ROWS = 0x20
# matching
PREC_FP32 = 0
PREC_BF16 = 1
PREC_FP16 = 2
PREC_FP8 = 3
MATCH_ASSUME_UNIFORM_B1 = 0x1
MATCH_IMAG_ATOMS = 0x2
MATCH_UPLOAD_EARLY = 0x4
MATCH_IMAG_ROWS = 0x8
START_IMAG_ATOMS = 0x1
START_IMAG_ROWS = 0x2

ECHO_TYPES = ("epg_ssfp", "roa_ssfp", "epg_sr", "epg_se", "epg_tse1", "epg_tse2", "epg_fisp")

RA_MAGIC = 0x7961727261776172
RA_TYPES = {(1, 4): np.int32, (1, 8): np.int64, (2, 4): np.uint32, (2, 8): np.uint64,
            (3, 4): np.float32, (3, 8): np.float64, (4, 8): np.complex64, (4, 16): np.complex128}


class SnapMRFError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"snapmrf status {status}: {msg}")
        self.status = status


class DictOpts(C.Structure):
    _fields_ = [("flags", C.c_uint), ("n_iso", C.c_int), ("d_norms", C.c_void_p), ("d_packed", C.c_void_p),
                ("packed_precision", C.c_int)]


class MatchOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("flags", C.c_uint), ("img_stride", C.c_size_t),
                ("atom_stride", C.c_size_t), ("b1map", C.c_void_p), ("b1map_on_host", C.c_int),
                ("d_index", C.c_void_p), ("topk", C.c_int), ("packed_atoms", C.c_void_p),
                ("packed_nreps", C.c_size_t), ("basis", C.c_void_p), ("basis_rows", C.c_size_t),
                ("basis_stride", C.c_size_t), ("coeffs", C.c_void_p), ("coeff_stride", C.c_size_t),
                ("rank", C.c_int), ("atom_norms", C.c_void_p), ("img_device_copy", C.c_void_p)]


class SvdOpts(C.Structure):
    _fields_ = [("flags", C.c_uint), ("atom_stride", C.c_size_t), ("sfrac", C.c_double), ("rank", C.c_int),
                ("oversample", C.c_int), ("power_iters", C.c_int), ("seed", C.c_ulonglong)]


class RA(C.Structure):
    _fields_ = [("flags", C.c_uint64), ("eltype", C.c_uint64), ("elbyte", C.c_uint64),
                ("size", C.c_uint64), ("ndims", C.c_uint64), ("dims", C.POINTER(C.c_uint64)),
                ("data", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    """Loads libsnapmrf.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise SnapMRFError(-1, f"{LIB_PATH} is not built; run __graft_entry__.build() first")
        L = C.CDLL(str(LIB_PATH))
        sz, vp, fp = C.c_size_t, C.c_void_p, C.POINTER(C.c_float)
        L.snapmrf_last_error.restype = C.c_char_p
        L.snapmrf_version.restype = C.c_char_p
        L.snapmrf_kernel_launches.restype = C.c_uint64
        L.snapmrf_scratch_allocations.restype = C.c_uint64
        L.snapmrf_device_error.argtypes = [C.c_int]
        L.snapmrf_selftest_bounded_wait.argtypes = [C.c_uint, C.c_void_p]
        L.snapmrf_csv_dim.restype = sz
        L.snapmrf_csv_dim.argtypes = [C.c_char_p]
        L.snapmrf_csv_read.argtypes = [vp, sz, C.c_char_p]
        L.snapmrf_parse_range.argtypes = [C.c_char_p, fp, fp, fp, C.POINTER(sz)]
        L.snapmrf_parse_length.restype = sz
        L.snapmrf_parse_length.argtypes = [C.c_char_p]
        L.snapmrf_parse_params.argtypes = [vp, C.c_char_p, sz]
        L.snapmrf_linspace.argtypes = [vp, C.c_float, C.c_float, sz]
        L.snapmrf_logspace.argtypes = [vp, C.c_float, C.c_float, sz]
        L.snapmrf_compute_natoms.restype = sz
        L.snapmrf_compute_natoms.argtypes = [vp, vp, sz, sz, sz, sz]
        L.snapmrf_trans_params.argtypes = [vp, vp, vp, vp, vp, sz, sz, sz, sz, sz, C.c_int]
        L.snapmrf_ra_read.argtypes = [C.POINTER(RA), C.c_char_p, C.c_int]
        L.snapmrf_ra_write.argtypes = [C.POINTER(RA), C.c_char_p]
        L.snapmrf_ra_free.argtypes = [C.POINTER(RA)]
        L.snapmrf_ra_free.restype = None
        L.snapmrf_mrf_dict.argtypes = [vp, vp, vp, sz, sz, sz, sz, C.c_int, C.c_int, C.c_char_p,
                                       C.POINTER(DictOpts), vp]
        L.snapmrf_normalize.argtypes = [vp, sz, sz, vp, vp]
        L.snapmrf_packed_pitch.restype = sz
        L.snapmrf_packed_pitch.argtypes = [sz]
        L.snapmrf_mrf_match.argtypes = [vp, vp, C.c_int, vp, vp, sz, sz, sz, sz, C.c_int, C.c_int,
                                        C.POINTER(MatchOpts), vp]
        L.snapmrf_svd_compress.argtypes = [vp, sz, sz, sz, C.c_int, vp, sz, vp, sz, C.POINTER(C.c_int),
                                           vp, C.POINTER(SvdOpts), vp]
        L.snapmrf_mrf_match_noalloc.argtypes = [vp, vp, sz, vp, sz, vp, sz, sz, sz, sz, C.c_int, C.c_int,
                                                vp, vp, vp]
        L.snapmrf_epg_adjoint.argtypes = [vp, C.c_int, vp, sz, sz, sz, C.c_int, C.c_char_p, vp, vp, vp,
                                          vp, vp, C.c_int, vp]
        L.snapmrf_epg_jvp.argtypes = [vp, C.c_int, vp, sz, sz, sz, C.c_int, C.c_char_p, vp, vp]
        L.snapmrf_crb_gradient.argtypes = [vp, C.c_int, vp, sz, sz, sz, C.c_int, C.c_char_p, vp, vp, vp,
                                           C.c_int, vp]
        L.snapmrf_refine_gn.argtypes = [vp, C.c_int, vp, sz, vp, vp, sz, sz, sz, C.c_int, C.c_char_p, C.c_int,
                                        C.c_float, C.c_float, vp, vp]
        L.snapmrf_refine_start.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, sz, sz, sz, vp, sz, sz, vp,
                                           C.c_uint, vp, vp]
        _lib = L
    return _lib


def device_error(reset: bool = False) -> int:
    """Error word of the tensor-core kernels (0 = none); synchronises the device."""
    return lib().snapmrf_device_error(1 if reset else 0)


def selftest_bounded_wait(limit_us: int = 1000, stream=None) -> None:
    """Runs one warp that waits with a limit of limit_us on an mbarrier
    nothing arrives on (the tensor-core kernels' wait primitive): the wait
    gives up and device_error() then reads 10."""
    _check(lib().snapmrf_selftest_bounded_wait(limit_us, _stream_ptr(stream)))


def kernel_launches() -> int:
    """Kernels launched by libsnapmrf.so so far in this process."""
    return lib().snapmrf_kernel_launches()


def scratch_allocations() -> int:
    """Device scratch allocations libsnapmrf.so has made so far in this process."""
    return lib().snapmrf_scratch_allocations()


def _check(rc: int) -> None:
    if rc != 0:
        raise SnapMRFError(rc, lib().snapmrf_last_error().decode(errors="replace"))


def _ptr(x) -> int | None:
    """Device/host address of a torch tensor, numpy array or raw int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except Exception:
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---------------------------------------------------------------------------
# host: CSV, grids, params (src/functions.cu:100-414)
# ---------------------------------------------------------------------------

def csv_dim(path: str) -> int:
    n = lib().snapmrf_csv_dim(str(path).encode())
    if n == C.c_size_t(-1).value:
        raise SnapMRFError(5, lib().snapmrf_last_error().decode())
    return n


def csv_read(path: str, nreps: int) -> np.ndarray:
    """Schedule h_mrf[4][nreps] (flip, phase, TR, TE columns)."""
    out = np.zeros((4, nreps), np.float32)
    _check(lib().snapmrf_csv_read(out.ctypes.data, nreps, str(path).encode()))
    return out


def parse_range(s: str):
    mn, st, mx = C.c_float(), C.c_float(), C.c_float()
    n = C.c_size_t()
    _check(lib().snapmrf_parse_range(s.encode(), C.byref(mn), C.byref(st), C.byref(mx), C.byref(n)))
    return mn.value, st.value, mx.value, n.value


def parse_length(s: str) -> int:
    n = lib().snapmrf_parse_length(s.encode())
    if n == 0:
        raise SnapMRFError(6, lib().snapmrf_last_error().decode())
    return n


def parse_params(s: str) -> np.ndarray:
    n = parse_length(s)
    out = np.zeros(n, np.float32)
    _check(lib().snapmrf_parse_params(out.ctypes.data, s.encode(), n))
    return out


def linspace(mn: float, step: float, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().snapmrf_linspace(out.ctypes.data, mn, step, n)
    return out


def logspace(mn: float, mx: float, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().snapmrf_logspace(out.ctypes.data, mn, mx, n)
    return out


def compute_natoms(t1, t2, l_b0: int, l_b1: int) -> int:
    t1 = np.ascontiguousarray(t1, np.float32)
    t2 = np.ascontiguousarray(t2, np.float32)
    return lib().snapmrf_compute_natoms(t1.ctypes.data, t2.ctypes.data, len(t1), len(t2), l_b0, l_b1)


def trans_params(t1, t2, b0, b1) -> np.ndarray:
    """params[NATOMS][4] = {T1, T2, B0, B1}, B1 > B0 > T2 > T1 order, T1 > T2."""
    t1, t2, b0, b1 = (np.ascontiguousarray(v, np.float32) for v in (t1, t2, b0, b1))
    n = compute_natoms(t1, t2, len(b0), len(b1))
    out = np.zeros((n, NPARAMS), np.float32)
    if n:
        _check(lib().snapmrf_trans_params(out.ctypes.data, t1.ctypes.data, t2.ctypes.data,
                                          b0.ctypes.data, b1.ctypes.data, len(t1), len(t2),
                                          len(b0), len(b1), n, NPARAMS))
    return out


def grid_params(T1: str, T2: str, B0: str = "0", B1: str = "1"):
    """The mrf CLI's grid pipeline (src/mrf.cu:205-253): returns
    (params [NATOMS][4], NATOMS, natoms)."""
    t1, t2, b0, b1 = (parse_params(s) for s in (T1, T2, B0, B1))
    p = trans_params(t1, t2, b0, b1)
    return p, p.shape[0], p.shape[0] // len(b1)


# ---------------------------------------------------------------------------
# RA files (src/ra.cu)
# ---------------------------------------------------------------------------

def ra_read(path: str) -> np.ndarray:
    """Reads an RA file into an array of shape dims[::-1] (dims[0] fastest)."""
    a = RA()
    _check(lib().snapmrf_ra_read(C.byref(a), str(path).encode(), 0))
    try:
        dims = [a.dims[i] for i in range(a.ndims)]
        dt = RA_TYPES.get((a.eltype, a.elbyte))
        if dt is None:
            raise SnapMRFError(7, f"{path}: RA eltype {a.eltype}/{a.elbyte} not supported")
        buf = (C.c_uint8 * a.size).from_address(a.data) if a.size else b""
        arr = np.frombuffer(bytes(buf), dtype=dt).reshape(tuple(reversed(dims)))
        return arr.copy()
    finally:
        lib().snapmrf_ra_free(C.byref(a))


def ra_write(path: str, arr: np.ndarray) -> None:
    """Writes arr (shape dims[::-1]) as RA: complex64 -> complex, float32 -> float."""
    arr = np.ascontiguousarray(arr)
    code = {np.dtype(np.complex64): (4, 8), np.dtype(np.complex128): (4, 16),
            np.dtype(np.float32): (3, 4), np.dtype(np.float64): (3, 8),
            np.dtype(np.int32): (1, 4), np.dtype(np.int64): (1, 8)}.get(arr.dtype)
    if code is None:
        raise SnapMRFError(7, f"dtype {arr.dtype} not supported")
    dims = (C.c_uint64 * arr.ndim)(*reversed(arr.shape))
    a = RA(0, code[0], code[1], arr.nbytes, arr.ndim, C.cast(dims, C.POINTER(C.c_uint64)),
           arr.ctypes.data)
    _check(lib().snapmrf_ra_write(C.byref(a), str(path).encode()))


# ---------------------------------------------------------------------------
# device entry points
# ---------------------------------------------------------------------------

def MRF_dict(d_atoms, d_params, h_mrf, nreps: int, NREPS: int, NATOMS: int, natoms: int,
             nparams: int = NPARAMS, nstates: int = 101, echo_type: str = "epg_ssfp", *,
             flags: int = 0, n_iso: int = 1, d_norms=None, d_packed=None, packed_precision: int = 0,
             stream=None) -> None:
    """Dictionary generation (src/functions.cu:1224-1315).

    d_atoms: device complex64 [NATOMS][nreps] (out); d_params: device float32
    [NATOMS][nparams]; h_mrf: host float32 [4][NREPS] schedule."""
    h_mrf = np.ascontiguousarray(h_mrf, np.float32)
    if h_mrf.size < 4 * NREPS:
        raise SnapMRFError(1, "h_mrf must hold 4*NREPS values")
    opts = DictOpts(flags, n_iso, _ptr(d_norms), _ptr(d_packed), packed_precision)
    _check(lib().snapmrf_mrf_dict(_ptr(d_atoms), _ptr(d_params), h_mrf.ctypes.data, nreps, NREPS,
                                  NATOMS, natoms, nparams, nstates, echo_type.encode(),
                                  C.byref(opts), _stream_ptr(stream)))


def normalize(d_atoms, nreps: int, NATOMS: int, d_norms=None, stream=None) -> None:
    """Unit-l2 normalisation of atoms in place (src/functions.cu:670-685)."""
    _check(lib().snapmrf_normalize(_ptr(d_atoms), nreps, NATOMS, _ptr(d_norms), _stream_ptr(stream)))


def MRF_match(d_maps, img, d_atoms, d_params, NREPS: int, nreps: int, NATOMS: int, natoms: int,
              nvoxels: int, nparams: int = NPARAMS, nmaps: int = NMAPS, in_b1map=None, *,
              precision: int = PREC_FP32, flags: int = 0, img_stride: int = 0,
              d_index=None, topk: int = 0, packed_atoms=None, compressed=None, atom_norms=None,
              img_device_copy=None, upload_early: bool = False, stream=None) -> None:
    """Template matching (src/functions.cu:1493-1584).

    img: host numpy complex64 [nvoxels][stride] or a device tensor; NREPS is
    the dictionary's time points (atom stride), nreps the matched time points.
    in_b1map: None, a path to an RA B1 map, a host array or a device tensor.
    compressed: a Compressed from svd_compress: match in its rank-r space
    (d_atoms may then be None; with atoms the tensor-core forms rescore
    their candidates against them).
    atom_norms: device float32 [NATOMS], the norms of d_atoms when they are
    not normalised (MRF_dict with DICT_NORMALIZE_OPERAND); BF16 / FP16 with
    packed_atoms only.
    img_device_copy: with a host image, a device complex64 [nvoxels][nreps]
    buffer that receives the uploaded image and keeps it (e.g. for
    refine_gn); upload_early (needs it) lets the upload overlap the work
    already queued on the stream, which must not use that buffer."""
    on_host = isinstance(img, np.ndarray) or (hasattr(img, "device") and img.device.type == "cpu")
    if isinstance(img, np.ndarray):
        img = np.ascontiguousarray(img, np.complex64)
        if not img_stride:
            img_stride = img.shape[-1] if img.ndim > 1 else nreps
    b1 = None
    b1_host = 0
    if in_b1map is not None:
        if isinstance(in_b1map, (str, os.PathLike)):
            in_b1map = ra_read(in_b1map).astype(np.float32).reshape(-1)
        if isinstance(in_b1map, np.ndarray):
            in_b1map = np.ascontiguousarray(in_b1map, np.float32).reshape(-1)
            if in_b1map.size < nvoxels:
                raise SnapMRFError(1, "B1 map has fewer values than voxels")
            b1_host = 1
        elif hasattr(in_b1map, "device") and in_b1map.device.type == "cpu":
            b1_host = 1
        b1 = in_b1map
    cb = compressed
    opts = MatchOpts(precision, flags, img_stride, NREPS, _ptr(b1), b1_host, _ptr(d_index), topk,
                     _ptr(packed_atoms), nreps if packed_atoms is not None else 0,
                     _ptr(cb.basis) if cb else None, cb.max_rank if cb else 0, cb.basis_stride if cb else 0,
                     _ptr(cb.coeffs) if cb else None, cb.coeff_stride if cb else 0, cb.rank if cb else 0,
                     _ptr(atom_norms), _ptr(img_device_copy))
    if upload_early:
        opts.flags |= MATCH_UPLOAD_EARLY
    _check(lib().snapmrf_mrf_match(_ptr(d_maps), _ptr(img), 1 if on_host else 0, _ptr(d_atoms),
                                   _ptr(d_params), nreps, NATOMS, natoms, nvoxels, nparams, nmaps,
                                   C.byref(opts), _stream_ptr(stream)))


SVD_MAX_SUBSPACE = 80
SVD_IMAG_ATOMS = 0x2


class Compressed:
    """A dictionary compressed per B1 block by svd_compress: the bases
    (device complex64 [nblocks][max_rank][basis_stride]), the atoms'
    coordinates (device complex64 [NATOMS][coeff_stride]), the rank r and
    the singular values (numpy [nblocks][max_rank])."""

    def __init__(self, basis, coeffs, rank: int, max_rank: int, basis_stride: int, coeff_stride: int, sv):
        self.basis, self.coeffs, self.rank, self.max_rank = basis, coeffs, rank, max_rank
        self.basis_stride, self.coeff_stride, self.sv = basis_stride, coeff_stride, sv


def svd_compress(d_atoms, nreps: int, NATOMS: int, natoms: int, *, sfrac: float = 0.0, rank: int = 0,
                 max_rank: int = 64, imag_atoms: bool = False, oversample: int = 0, power_iters: int = 0,
                 seed: int = 0, atom_stride: int = 0, stream=None) -> Compressed:
    """Low-rank compression of each B1 block (matlab/MRF_dict_B1.m:127-159):
    the rank from block 0's energy fraction sfrac (or a fixed rank), the
    r leading left singular vectors of each block and the atoms'
    coordinates in them.  d_atoms: device complex64 [NATOMS][atom_stride]."""
    import torch
    nb = NATOMS // natoms
    dev = d_atoms.device if hasattr(d_atoms, "device") else torch.device("cuda")
    bstride = nreps
    basis = torch.empty((nb, max_rank, bstride, 2), dtype=torch.float32, device=dev)
    coeffs = torch.empty((NATOMS, max_rank, 2), dtype=torch.float32, device=dev)
    sv = np.zeros((nb, max_rank), np.float64)
    r = C.c_int(0)
    o = SvdOpts(SVD_IMAG_ATOMS if imag_atoms else 0, atom_stride, sfrac, rank, oversample, power_iters, seed)
    _check(lib().snapmrf_svd_compress(_ptr(d_atoms), nreps, NATOMS, natoms, max_rank, _ptr(basis), bstride,
                                      _ptr(coeffs), max_rank, C.byref(r), sv.ctypes.data, C.byref(o),
                                      _stream_ptr(stream)))
    return Compressed(basis, coeffs, r.value, max_rank, bstride, max_rank, sv)


NOALLOC_MAX_VOXELS = 65536
NOALLOC_MAX_B1_BLOCKS = 1024


def MRF_match_noalloc(d_maps, d_img, d_atoms, d_params, NREPS: int, nreps: int, NATOMS: int,
                      natoms: int, nvoxels: int, nparams: int = NPARAMS, nmaps: int = NMAPS,
                      d_b1map=None, *, img_stride: int = 0, d_index=None, stream=None) -> None:
    """MRF_match for callers that cannot allocate device memory while they
    run (a framework whose caching allocator already holds the GPU's free
    memory, or a reconstruction pipeline that must not allocate after
    start-up).  Every input and output is a device buffer; the working
    arrays come from a fixed ~1.3 MiB array the library reserves per GPU, so
    at most NOALLOC_MAX_VOXELS voxels (and NOALLOC_MAX_B1_BLOCKS B1 blocks
    with a B1 map) per call.  Calls share that array: do not let two calls
    run on the GPU at the same time.  Each call looks up the array's device
    address on the current device; the first call on a device also makes
    the runtime load the array and should precede any stream capture.  With
    a B1 map, a B1 block holding several B1 values gives NaN maps, indices
    -1 and device_error() == 9."""
    _check(lib().snapmrf_mrf_match_noalloc(_ptr(d_maps), _ptr(d_img), img_stride, _ptr(d_atoms), NREPS,
                                           _ptr(d_params), nreps, NATOMS, natoms, nvoxels, nparams, nmaps,
                                           _ptr(d_b1map), _ptr(d_index), _stream_ptr(stream)))


# ---------------------------------------------------------------------------
# derivatives (no counterpart in the reference)
# ---------------------------------------------------------------------------

def _schedule(h_mrf, NREPS: int) -> np.ndarray:
    h_mrf = np.ascontiguousarray(h_mrf, np.float32)
    if h_mrf.size < 4 * NREPS:
        raise SnapMRFError(1, "h_mrf must hold 4*NREPS values")
    return h_mrf


def epg_adjoint(d_params, h_mrf, nreps: int, NREPS: int, natoms: int, d_grad_signal, d_grad_params,
                nparams: int = NPARAMS, nstates: int = 101, echo_type: str = "epg_fisp", *,
                d_signal=None, d_grad_alpha=None, d_grad_alpha_atoms=None, checkpoint_every: int = 0,
                stream=None) -> None:
    """Reverse-mode derivative of the real FISP / SR recursion: given
    dL/ds (device complex64 [natoms][nreps]) writes dL/d(T1, T2, B1) into
    d_grad_params [natoms][3] and, optionally, dL/dalpha_t."""
    h_mrf = _schedule(h_mrf, NREPS)
    _check(lib().snapmrf_epg_adjoint(_ptr(d_params), nparams, h_mrf.ctypes.data, nreps, NREPS, natoms,
                                     nstates, echo_type.encode(), _ptr(d_grad_signal), _ptr(d_signal),
                                     _ptr(d_grad_params), _ptr(d_grad_alpha), _ptr(d_grad_alpha_atoms),
                                     checkpoint_every, _stream_ptr(stream)))


def refine_gn(d_maps, d_img, h_mrf, nreps: int, NREPS: int, nvoxels: int, nstates: int = 101,
              echo_type: str = "epg_fisp", *, nmaps: int = NMAPS, iterations: int = 3,
              max_rel_step: float = 0.2, tol: float = 1e-4, img_stride: int = 0, d_b1map=None,
              d_m0=None, stream=None) -> None:
    """Gauss-Newton refinement of matched (T1, T2) in place: d_maps device
    float32 [nvoxels][nmaps] (T1, T2, B0, B1, PD) as MRF_match writes them;
    d_img device complex64 voxels; d_b1map optional device B1 map (else the
    maps' B1 column).  At most `iterations` steps per voxel; a voxel stops
    once a step moved T1 and T2 by at most tol (relative; 0: never early)."""
    h_mrf = _schedule(h_mrf, NREPS)
    _check(lib().snapmrf_refine_gn(_ptr(d_maps), nmaps, _ptr(d_img), img_stride, _ptr(d_b1map),
                                   h_mrf.ctypes.data, nreps,
                                   NREPS, nvoxels, nstates, echo_type.encode(), iterations, max_rel_step,
                                   tol, _ptr(d_m0), _stream_ptr(stream)))


def refine_start(d_maps, d_img, d_atoms, d_params, d_index, nreps: int, NATOMS: int, natoms: int,
                 nvoxels: int, *, nmaps: int = NMAPS, nparams: int = NPARAMS, img_stride: int = 0,
                 d_b1map=None, imag_atoms: bool = False, imag_rows: bool = False, d_count=None,
                 stream=None) -> None:
    """Sub-grid start for refine_gn, in place: each voxel's matched atom
    (d_index, int64, as MRF_match writes it) and its six-point (T1, T2)
    neighbourhood of the dictionary (d_atoms complex [NATOMS][nreps]; with
    d_b1map, three B1 blocks interpolated to the voxel's B1) give a quadratic
    surrogate in (log T1, log T2); the fit of the voxel maximised over that
    surrogate replaces (T1, T2) in d_maps.  Voxels on the grid's edge are
    left as they are.  imag_atoms: every atom is purely imaginary (zero-phase
    FISP / SR); imag_rows (with imag_atoms): d_atoms holds their Im rows as
    MRF_dict(flags=DICT_IMAG_ROWS) writes them.  d_count: optional device
    int32 counter of voxels moved."""
    _check(lib().snapmrf_refine_start(_ptr(d_maps), nmaps, _ptr(d_index), _ptr(d_atoms), _ptr(d_params),
                                      nparams, nreps, NATOMS, natoms, _ptr(d_img), img_stride, nvoxels,
                                      _ptr(d_b1map),
                                      (START_IMAG_ATOMS if imag_atoms else 0) | (START_IMAG_ROWS if imag_rows else 0),
                                      _ptr(d_count),
                                      _stream_ptr(stream)))


def packed_pitch(nreps: int) -> int:
    """Row pitch (elements) of atoms packed by MRF_dict(d_packed=...)."""
    return int(lib().snapmrf_packed_pitch(nreps))


def epg_jvp(d_params, h_mrf, nreps: int, NREPS: int, natoms: int, d_out, nparams: int = NPARAMS,
            nstates: int = 101, echo_type: str = "epg_fisp", stream=None) -> None:
    """Forward mode of the real FISP / SR recursion: d_out [natoms][3][nreps]
    = f, df/dT1, df/dT2 of each atom s = i f as generated (d_params rows T1,
    T2, B0, B1; flip angle alpha_t * B1).  A Jacobian-vector product along
    (dT1, dT2) is dT1 * d_out[:, 1] + dT2 * d_out[:, 2]."""
    h_mrf = _schedule(h_mrf, NREPS)
    _check(lib().snapmrf_epg_jvp(_ptr(d_params), nparams, h_mrf.ctypes.data, nreps, NREPS, natoms, nstates,
                                 echo_type.encode(), _ptr(d_out), _stream_ptr(stream)))


def crb_gradient(d_params, h_mrf, nreps: int, NREPS: int, ntissues: int, d_loss, d_grad_alpha,
                 nparams: int = NPARAMS, nstates: int = 101, echo_type: str = "epg_fisp", *,
                 d_signals=None, checkpoint_every: int = 0, stream=None) -> None:
    """Normalised Cramer-Rao bounds of (T1, T2) per tissue (d_loss [ntissues])
    and the gradient of their sum with respect to the flip angles
    (d_grad_alpha [nreps]); d_signals optional [ntissues][3][nreps] = f,
    df/dT1, df/dT2 of the real FISP / SR signal s = i f."""
    h_mrf = _schedule(h_mrf, NREPS)
    _check(lib().snapmrf_crb_gradient(_ptr(d_params), nparams, h_mrf.ctypes.data, nreps, NREPS, ntissues,
                                      nstates, echo_type.encode(), _ptr(d_loss), _ptr(d_grad_alpha),
                                      _ptr(d_signals), checkpoint_every, _stream_ptr(stream)))
