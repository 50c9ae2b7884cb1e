"""Host side of the product (C++ in libsnapmrf.so): grid parser, parameter
table, CSV reader and RA files, checked against the reference's own host
code outputs recorded in tests/golden/golden.npz.  CPU only."""
import ctypes as C
import struct

import numpy as np
import pytest

from cases import CSV_CASES, GRID_CASES, GRIDN_CASES, LOGSPACE_CASES


@pytest.mark.parametrize("i", range(len(GRID_CASES)))
def test_grid_pipeline_bit_identical(snap, golden, i):
    T1, T2, B0, B1 = GRID_CASES[i]
    l1, l2, l0, lb, N, n = golden[f"grid_{i}_dims"]
    assert snap.parse_length(T1) == l1 and snap.parse_length(T2) == l2
    assert snap.parse_length(B0) == l0 and snap.parse_length(B1) == lb
    params, NATOMS, natoms = snap.grid_params(T1, T2, B0, B1)
    assert (NATOMS, natoms) == (N, n)
    ref = golden[f"grid_{i}"].reshape(-1, 4)
    assert params.tobytes() == ref.tobytes()


@pytest.mark.parametrize("i", range(len(LOGSPACE_CASES)))
def test_logspace_bit_identical(snap, golden, i):
    mn, mx, n = LOGSPACE_CASES[i]
    got = snap.logspace(mn, mx, n)
    assert got.tobytes() == golden[f"logspace_{i}"].tobytes()


@pytest.mark.parametrize("N", GRIDN_CASES)
def test_hard_coded_N_grids(snap, golden, N):
    """-N grids of src/mrf.cu:179-203: l_b1 = 11, l_b0 = 21, l_t1 = l_t2 =
    round(sqrt(N / 21 / 11)), logspace ranges."""
    import math
    l_b1, l_b0 = 11, 21
    l_t = max(1, int(round(math.sqrt(N // l_b0 // l_b1))))
    t1 = snap.logspace(100.0, 3000.0, l_t)
    t2 = snap.logspace(20.0, 1000.0, l_t)
    b0 = snap.logspace(-150.0, 150.0, l_b0)
    b1 = snap.logspace(0.5, 1.5, l_b1)
    p = snap.trans_params(t1, t2, b0, b1)
    assert p.tobytes() == golden[f"gridN_{N}"].reshape(-1, 4).tobytes()


@pytest.mark.parametrize("name", list(CSV_CASES))
def test_csv_reader_quirks(snap, golden, tmp_path, name):
    """csv_read skips two 100-byte fgets chunks (src/functions.cu:122-158)."""
    f = tmp_path / f"{name}.csv"
    f.write_text(CSV_CASES[name])
    nreps = snap.csv_dim(str(f)) - 1
    got = snap.csv_read(str(f), nreps)
    ref = golden[f"csv_{name}"]
    assert got.shape == ref.shape
    assert got.tobytes() == ref.tobytes()


def test_csv_mrf5(snap, golden, tmp_path):
    ref = golden["mrf5"]
    hdr = "flip_angle_(fraction_of_nominal),rf_phase_(deg),extension_of_base_TR_(ms),extension_of_base_TE_(ms)"
    assert len(hdr) == 99
    rows = "\n".join(",".join(repr(float(v)) for v in ref[:, t]) for t in range(ref.shape[1]))
    f = tmp_path / "m.csv"
    f.write_text(hdr + "\n" + rows + "\n")
    assert snap.csv_dim(str(f)) - 1 == ref.shape[1]
    np.testing.assert_array_equal(snap.csv_read(str(f), ref.shape[1]), ref)


def test_csv_errors(snap, tmp_path):
    with pytest.raises(snap.SnapMRFError):
        snap.csv_dim(str(tmp_path / "missing.csv"))
    f = tmp_path / "short.csv"
    f.write_text("h" * 99 + "\n1,2\n")
    with pytest.raises(snap.SnapMRFError, match="fewer than 4 columns"):
        snap.csv_read(str(f), 1)


@pytest.mark.parametrize("bad", ["5:1", "5:1:1", "1:0:3", "1:-1:3", "x" * 1100])
def test_grid_errors(snap, bad):
    """max < min asserts in the reference; a non-positive step has no length."""
    with pytest.raises(snap.SnapMRFError):
        snap.parse_params(bad)


def test_trans_params_order(snap):
    p = snap.trans_params([100, 200, 300], [150, 250], [0, 5], [0.9, 1.1])
    # B1 outermost, then B0, T2, T1; only T1 > T2
    assert p.shape == (3 * 2 * 2, 4)
    np.testing.assert_array_equal(p[:3], np.float32([[200, 150, 0, 0.9], [300, 150, 0, 0.9], [300, 250, 0, 0.9]]))
    np.testing.assert_array_equal(p[3:6, 2], [5, 5, 5])
    np.testing.assert_array_equal(p[6:, 3], np.float32([1.1] * 6))


def test_ra_roundtrip(snap, tmp_path):
    rng = np.random.default_rng(0)
    for arr in [rng.standard_normal((3, 7)).astype(np.float32),
                (rng.standard_normal((5, 4)) + 1j * rng.standard_normal((5, 4))).astype(np.complex64),
                np.arange(12, dtype=np.int32).reshape(2, 2, 3)]:
        p = tmp_path / "x.ra"
        snap.ra_write(str(p), arr)
        b = p.read_bytes()
        magic, flags, eltype, elbyte, size, ndims = struct.unpack("<6Q", b[:48])
        assert magic == 0x7961727261776172 and flags == 0 and size == arr.nbytes
        assert list(struct.unpack(f"<{ndims}Q", b[48:48 + 8 * ndims])) == list(reversed(arr.shape))
        back = snap.ra_read(str(p))
        assert back.dtype == arr.dtype
        np.testing.assert_array_equal(back, arr)


def test_ra_reads_reference_goldens_layout(snap, golden, tmp_path):
    """An RA file laid out like the reference's data/atoms_*.ra reads back."""
    a = golden["atoms_epg_ssfp"]
    p = tmp_path / "a.ra"
    hdr = struct.pack("<6Q", 0x7961727261776172, 0, 4, 8, a.nbytes, 2) + struct.pack("<2Q", a.shape[1], a.shape[0])
    p.write_bytes(hdr + a.tobytes())
    np.testing.assert_array_equal(snap.ra_read(str(p)), a)


def test_ra_errors(snap, tmp_path):
    p = tmp_path / "bad.ra"
    p.write_bytes(b"\0" * 48)
    with pytest.raises(snap.SnapMRFError, match="bad magic"):
        snap.ra_read(str(p))
    p.write_bytes(struct.pack("<6Q", 0x7961727261776172, 0, 3, 4, 400, 1) + struct.pack("<Q", 100) + b"\0" * 40)
    with pytest.raises(snap.SnapMRFError, match="fewer than"):
        snap.ra_read(str(p))
    p.write_bytes(struct.pack("<3Q", 0x7961727261776172, 0, 3))
    with pytest.raises(snap.SnapMRFError, match="truncated"):
        snap.ra_read(str(p))
    p.write_bytes(struct.pack("<6Q", 0x7961727261776172, 1, 3, 4, 4, 1) + struct.pack("<Q", 1) + b"\0" * 4)
    with pytest.raises(snap.SnapMRFError, match="big-endian"):
        snap.ra_read(str(p))
    with pytest.raises(snap.SnapMRFError):
        snap.ra_read(str(tmp_path / "nope.ra"))


def test_dict_argument_errors_without_gpu(snap):
    """Argument validation happens before any device work."""
    h = np.zeros((4, 10), np.float32)
    with pytest.raises(snap.SnapMRFError, match="echo types"):
        snap.MRF_dict(1, 1, h, 10, 10, 4, 4, echo_type="epg_nope", stream=0)
    with pytest.raises(snap.SnapMRFError, match="multiple of natoms"):
        snap.MRF_dict(1, 1, h, 10, 10, 5, 4, echo_type="epg_fisp", stream=0)
    with pytest.raises(snap.SnapMRFError, match="nreps"):
        snap.MRF_dict(1, 1, h, 11, 10, 4, 4, echo_type="epg_fisp", stream=0)
    with pytest.raises(snap.SnapMRFError, match="nstates"):
        snap.MRF_dict(1, 1, h, 10, 10, 4, 4, nstates=0, echo_type="epg_fisp", stream=0)
    assert snap.lib().snapmrf_last_error().decode().startswith("MRF_dict")


def test_match_argument_errors_without_gpu(snap):
    img = np.zeros((4, 10), np.complex64)
    with pytest.raises(snap.SnapMRFError, match="nmaps"):
        snap.MRF_match(1, img, 1, 1, 10, 10, 4, 4, 4, nmaps=4, stream=0)
    with pytest.raises(snap.SnapMRFError, match="precision"):
        snap.MRF_match(1, img, 1, 1, 10, 10, 4, 4, 4, precision=9, stream=0)


def test_normalize_operand_argument_errors_without_gpu(snap):
    """DICT_NORMALIZE_OPERAND needs the packed operand and atoms that are not
    normalised; atom_norms needs BF16 / FP16 matching of packed atoms.  Both
    are checked before any device work."""
    h = np.zeros((4, 10), np.float32)
    with pytest.raises(snap.SnapMRFError, match="NORMALIZE_OPERAND"):
        snap.MRF_dict(1, 1, h, 10, 10, 4, 4, echo_type="epg_fisp", flags=snap.DICT_NORMALIZE_OPERAND, stream=0)
    with pytest.raises(snap.SnapMRFError, match="NORMALIZE_OPERAND"):
        snap.MRF_dict(1, 1, h, 10, 10, 4, 4, echo_type="epg_fisp", d_packed=1,
                      flags=snap.DICT_NORMALIZE_OPERAND | snap.DICT_NORMALIZE, stream=0)
    with pytest.raises(snap.SnapMRFError, match="NORMALIZE_OPERAND"):
        snap.MRF_dict(1, 1, h, 10, 10, 4, 4, echo_type="epg_ssfp", d_packed=1,
                      flags=snap.DICT_NORMALIZE_OPERAND, stream=0)
    img = np.zeros((4, 10), np.complex64)
    for kw in (dict(precision=snap.PREC_FP32, packed_atoms=1), dict(precision=snap.PREC_FP8, packed_atoms=1),
               dict(precision=snap.PREC_FP16)):
        with pytest.raises(snap.SnapMRFError, match="atom_norms"):
            snap.MRF_match(1, img, 1, 1, 10, 10, 4, 4, 4, atom_norms=1, stream=0, **kw)


def test_epg_jvp_refuses_bad_arguments_before_any_device_work(snap):
    """The forward-mode entry point checks its pointers, sizes and echo type
    before it touches the device (no GPU needed)."""
    h = np.zeros((4, 8), np.float32)
    with pytest.raises(snap.SnapMRFError, match="null pointer"):
        snap.epg_jvp(None, h, 8, 8, 1, None)
    with pytest.raises(snap.SnapMRFError, match="bad sizes"):
        snap.epg_jvp(1, h, 8, 8, 0, 1)
    with pytest.raises(snap.SnapMRFError, match="echo type"):
        snap.epg_jvp(1, h, 8, 8, 1, 1, echo_type="epg_ssfp")
