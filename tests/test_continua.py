"""Restart files (include/afid_continua.h) on the CPU: the native HDF5 writer and reader against
the oracle's restatement of the file format (oracle/afid_h5.py) and against a file written by the
HDF5 library itself, and the continua file set of WriteFlowField.F90 / ReadFlowInterp.F90."""
import os

import numpy as np
import pytest

import afid_gpu as ag
from helpers import bou_text
from oracle import afid_h5 as h5

SCIPY_DATA = None
try:
    import scipy.io.matlab as _m
    SCIPY_DATA = os.path.join(os.path.dirname(_m.__file__), "tests", "data")
except Exception:  # pragma: no cover
    pass


def _library_file():
    if SCIPY_DATA is None:
        pytest.skip("scipy test data not present")
    path = os.path.join(SCIPY_DATA, "testhdf5_7.4_GLNX86.mat")
    twin = os.path.join(SCIPY_DATA, "testdouble_7.1_GLNX86.mat")
    if not (os.path.exists(path) and os.path.exists(twin)):
        pytest.skip("scipy test data not present")
    return path, twin


def test_lookup3_known_answers():
    """The self-test values of Bob Jenkins' lookup3.c (driver5)."""
    assert h5.lookup3(b"") == 0xDEADBEEF
    assert h5.lookup3(b"Four score and seven years ago") == 0x17770551
    assert h5.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def test_readers_match_a_file_written_by_the_hdf5_library():
    """scipy's MATLAB 7.3 test file is an HDF5 file (512-byte user block, version-0 superblock)
    written by the HDF5 library; its variable also ships in a MATLAB 5 file that scipy reads."""
    from scipy.io import loadmat
    path, twin = _library_file()
    want = loadmat(twin)["testdouble"].astype(np.float64)        # (1, 9) in MATLAB's view
    assert np.allclose(want.ravel(), np.pi / 4 * np.arange(9))
    assert h5.names(path) == ["testdouble"]
    got_oracle = h5.read(path, "testdouble")
    assert got_oracle.shape == (9, 1)                             # column-major on disk
    np.testing.assert_array_equal(got_oracle.ravel(), want.ravel())
    assert ag.h5_info(path, "testdouble") == (ag.H5_F64, (9, 1))
    np.testing.assert_array_equal(ag.h5_read(path, "testdouble").ravel(), want.ravel())
    with pytest.raises(ag.AfidError) as e:
        ag.h5_read(path, "nothere")
    assert e.value.status == ag.AFID_E_IO


def _datasets(rng):
    d = {f"scalar_{c}": np.array([rng.integers(-2**31, 2**31 - 1)], dtype=np.int32) for c in "abcdefgh"}
    d["time"] = np.array([0.125])
    d["r1"] = rng.standard_normal(17)
    d["r2"] = rng.standard_normal((5, 3))
    d["r3"] = rng.standard_normal((4, 3, 9))
    d["r4"] = rng.integers(-1000, 1000, (2, 3, 4, 5)).astype(np.int32)
    d["empty"] = np.zeros((0, 4))
    d["a_name_that_is_rather_long_for_a_dataset_" + "x" * 60] = np.array([1.0, -0.0, np.inf, np.nan])
    return d


def test_native_writer_output_reads_with_the_oracle(tmp_path):
    """Sixteen datasets (two symbol table nodes under the B-tree), ranks 1-4, both types, an empty
    dataset, special values; layout facts of the default HDF5 format checked on the bytes."""
    rng = np.random.default_rng(3)
    d = _datasets(rng)
    path = str(tmp_path / "many.h5")
    ag.h5_write(path, d)
    f = h5.H5File(path)
    assert (f.base, f.sb_version, f.so, f.sl) == (0, 0, 8, 8)
    raw = open(path, "rb").read()
    assert int.from_bytes(raw[40:48], "little") == len(raw)      # end-of-file address
    assert sorted(f.root()) == sorted(d)
    for k, v in d.items():
        got = f.read(k)
        assert got.dtype == v.dtype and got.shape == v.shape, k
        np.testing.assert_array_equal(got, v)
        nat = ag.h5_read(path, k)
        assert nat.shape == v.shape
        np.testing.assert_array_equal(nat, v.astype(np.float64))
    # every dataset header is version 1 with dataspace, datatype, fill value and layout messages
    for k, addr in f.root().items():
        types = [t for t, _, _ in f.messages(addr)]
        assert types == [0x01, 0x03, 0x05, 0x08], k


def test_native_reader_takes_the_newer_layout(tmp_path):
    """Superblock version 2, version-2 object headers, link-message root group, compact and
    contiguous storage, big-endian and 32-bit types."""
    rng = np.random.default_rng(4)
    d = {"var": rng.standard_normal((3, 4, 5)), "small": np.arange(6, dtype=np.int32).reshape(2, 3),
         "be": rng.standard_normal(7).astype(">f8"), "f32": rng.standard_normal(5).astype(np.float32),
         "u16": np.arange(9, dtype=np.uint16), "i64": np.array([-3, 2**40], dtype=np.int64)}
    path = str(tmp_path / "v2.h5")
    h5.write_v2(path, d, compact=("small", "u16"))
    f = h5.H5File(path)
    assert f.sb_version == 2
    for k, v in d.items():
        np.testing.assert_array_equal(f.read(k), v)
        np.testing.assert_array_equal(ag.h5_read(path, k), v.astype(np.float64))
    assert ag.h5_info(path, "small") == (ag.H5_I32, (2, 3))


def test_reader_refuses_damaged_files(tmp_path):
    rng = np.random.default_rng(5)
    path = str(tmp_path / "ok.h5")
    ag.h5_write(path, {"var": rng.standard_normal((8, 8, 8))})
    raw = open(path, "rb").read()
    cases = {"truncated_meta": raw[:300], "truncated_data": raw[:len(raw) - 8], "garbage": bytes(rng.integers(0, 256, 4096, dtype=np.uint8)),
             "empty": b""}
    for name, blob in cases.items():
        p = str(tmp_path / f"{name}.h5")
        open(p, "wb").write(blob)
        with pytest.raises(ag.AfidError) as e:
            ag.h5_read(p, "var")
        assert e.value.status == ag.AFID_E_IO, name
    with pytest.raises(ag.AfidError) as e:
        ag.h5_read(str(tmp_path / "missing.h5"), "var")
    assert e.value.status == ag.AFID_E_IO
    for bad in ({"a//b": np.zeros(2)}, {"/a": np.zeros(2)}, {"a/": np.zeros(2)},
                {"a": np.zeros(2), "a/b": np.zeros(2)}):   # empty path components; a dataset used as a group
        with pytest.raises(ag.AfidError) as e:
            ag.h5_write(str(tmp_path / "bad.h5"), bad)
        assert e.value.status == ag.AFID_E_INVALID


def _input(**kw):
    return ag.parse_bou_in(bou_text(16, 12, 8, **kw))


def _fields(inp, rng, sal=False):
    nx, nym, nzm = inp.nxm + 1, inp.nym, inp.nzm
    f = {k: rng.standard_normal((nzm, nym, nx)) for k in ("vx", "vy", "vz", "temp", "pr")}
    for k in ("vy", "vz", "temp", "pr"):
        f[k][..., -1] = 0.0
    if sal:
        f["sal"] = rng.standard_normal((inp.nzmr, inp.nymr, inp.nxmr))
    return f


def test_continua_file_set_matches_the_reference_layout(tmp_path):
    """WriteFlowField.F90(final=.true.): continua_{temp,vx,vy,vz,pr}.h5 with 'var' of dims
    (nzm, nym, nx) and continua_master.h5 with the grid description; read back unchanged."""
    inp = _input(multires=0)
    rng = np.random.default_rng(6)
    f = _fields(inp, rng)
    m = ag.continua_master(inp, 1.25)
    d = str(tmp_path / "outputdir")
    ag.write_flow_field(d, m, f, final=True)
    assert sorted(os.listdir(d)) == sorted(f"continua_{k}.h5" for k in ("master", "temp", "vx", "vy", "vz", "pr"))
    for k in ("vx", "vy", "vz", "temp", "pr"):
        p = os.path.join(d, f"continua_{k}.h5")
        assert h5.names(p) == ["var"]
        ds = h5.H5File(p).dataset("var")
        assert ds.shape == (inp.nzm, inp.nym, inp.nxm + 1) and ds.dtype == np.dtype("<f8")
        np.testing.assert_array_equal(h5.read(p, "var"), f[k])
    mp = os.path.join(d, "continua_master.h5")
    assert h5.names(mp) == sorted(["nx", "ny", "nz", "ylen", "zlen", "time", "istr3", "str3"])
    want = dict(nx=inp.nxm + 1, ny=inp.nym + 1, nz=inp.nzm + 1, istr3=inp.istr3)
    for k, v in want.items():
        a = h5.read(mp, k)
        assert a.dtype == np.dtype("<i4") and a.shape == (1,) and int(a[0]) == v, k
    for k, v in dict(ylen=inp.ylen, zlen=inp.zlen, time=1.25, str3=inp.str3).items():
        a = h5.read(mp, k)
        assert a.dtype == np.dtype("<f8") and a.shape == (1,) and a[0] == v, k
    back = ag.read_flow_field(d, ag.continua_master(inp))
    assert back["time"] == 1.25
    for k in ("vx", "vy", "vz", "temp", "pr"):
        np.testing.assert_array_equal(back[k], f[k])


def test_continua_with_refined_salinity(tmp_path):
    """MULTIRES = 1: continua_sal.h5 on the refined grid with dims (nzmr, nymr, nxmr + 1), the
    extra x node zero; nxr, nyr, nzr, istr3r in the master file."""
    inp = _input(multires=1, nxmr=24, nymr=24, nzmr=16, flagsal=1, istr3r=4)
    rng = np.random.default_rng(7)
    f = _fields(inp, rng, sal=True)
    m = ag.continua_master(inp, 0.5)
    d = str(tmp_path / "out")
    ag.write_flow_field(d, m, f, final=True)
    sp = os.path.join(d, "continua_sal.h5")
    s = h5.read(sp, "var")
    assert s.shape == (16, 24, 25)
    np.testing.assert_array_equal(s[..., :24], f["sal"])
    assert np.all(s[..., 24] == 0.0)
    mp = os.path.join(d, "continua_master.h5")
    for k, v in dict(nxr=25, nyr=25, nzr=17, istr3r=4).items():
        assert int(h5.read(mp, k)[0]) == v
    back = ag.read_flow_field(d, ag.continua_master(inp), with_sal=True)
    np.testing.assert_array_equal(back["sal"], f["sal"])
    mm = ag.read_continua_master(d, multires=True)
    assert (mm.nxr, mm.nyr, mm.nzr, mm.istr3r, mm.time) == (25, 25, 17, 4, 0.5)


def test_frames_and_optional_pressure(tmp_path):
    """final = .false. writes fields/NNNNN_* (NNNNN = nint(time/SAVE_3D)) without pr and without a
    master; a restart without continua_pr.h5 leaves pr unread."""
    inp = _input(multires=0)
    rng = np.random.default_rng(8)
    f = _fields(inp, rng)
    d = str(tmp_path / "o")
    m = ag.continua_master(inp, 2.6)
    ag.write_flow_field(d, m, {k: f[k] for k in ("vx", "vy", "vz", "temp")}, final=False, save_3d=0.5)
    assert sorted(os.listdir(os.path.join(d, "fields"))) == sorted(f"00005_{k}.h5" for k in ("temp", "vx", "vy", "vz"))
    np.testing.assert_array_equal(h5.read(os.path.join(d, "fields", "00005_vz.h5"), "var"), f["vz"])
    # nint rounds halves away from zero: time / SAVE_3D = 2.5 is frame 00003, 4.5 is 00005
    for t, frame in ((1.25, "00003"), (2.25, "00005")):
        ag.write_flow_field(d, ag.continua_master(inp, t), {k: f[k] for k in ("vx", "vy", "vz", "temp")},
                            final=False, save_3d=0.5)
        assert os.path.exists(os.path.join(d, "fields", f"{frame}_temp.h5")), (t, frame)
    ag.write_flow_field(d, m, f, final=True)
    os.remove(os.path.join(d, "continua_pr.h5"))
    back = ag.read_flow_field(d, ag.continua_master(inp))
    assert back["pr"] is None
    np.testing.assert_array_equal(back["temp"], f["temp"])


def test_restart_refuses_other_grids_and_domains(tmp_path):
    """ReadFlowInterp.F90:76-89: a different Ly/Lz aborts; a different grid needs interpolation,
    which this library does not provide (AFID_E_INVALID); no files: AFID_E_IO."""
    inp = _input(multires=0)
    rng = np.random.default_rng(9)
    d = str(tmp_path / "o")
    ag.write_flow_field(d, ag.continua_master(inp), _fields(inp, rng), final=True)
    for kw in (dict(ylen=1.5), dict(zlen=0.5), dict(str3=3.0), dict(istr3=0)):
        other = ag.parse_bou_in(bou_text(16, 12, 8, multires=0, **kw))
        with pytest.raises(ag.AfidError) as e:
            ag.read_flow_field(d, ag.continua_master(other))
        assert e.value.status == ag.AFID_E_INVALID, kw
    other = ag.parse_bou_in(bou_text(20, 12, 8, multires=0))
    with pytest.raises(ag.AfidError) as e:
        ag.read_flow_field(d, ag.continua_master(other))
    assert e.value.status == ag.AFID_E_INVALID
    with pytest.raises(ag.AfidError) as e:
        ag.read_flow_field(str(tmp_path / "nothing"), ag.continua_master(inp))
    assert e.value.status == ag.AFID_E_IO


# ---- the interpolating restart (ReadFlowInterp.F90:85-136) --------------------------------------
from oracle import afid_oracle as o  # noqa: E402
from oracle import afid_restart as rs  # noqa: E402
from oracle import afid_salinity as sa  # noqa: E402


def _old_files(tmp_path, old_kw, rng, sal=False, fields=None):
    text = bou_text(*old_kw.pop("dims"), **old_kw)
    inp = ag.parse_bou_in(text)
    f = fields if fields is not None else _fields(inp, rng, sal=sal)
    d = str(tmp_path / "old")
    ag.write_flow_field(d, ag.continua_master(inp, 0.75), f, final=True)
    return d, f


INTERP_CASES = [
    # (old grid, new grid): finer, coarser, other stretching, 2-D, other wall conditions
    (dict(dims=(16, 12, 8)), dict(dims=(24, 18, 12), str3=3.0)),
    (dict(dims=(24, 16, 12), istr3=0), dict(dims=(16, 12, 8))),
    (dict(dims=(32, 24, 1)), dict(dims=(48, 16, 1), istr3=1, str3=1.5)),
    (dict(dims=(16, 12, 8)), dict(dims=(20, 24, 6), inslwn=0, tfixn=0, rayt=-1e6)),
    (dict(dims=(16, 12, 8)), dict(dims=(20, 12, 8), inslws=0, tfixs=0)),
]


@pytest.mark.parametrize("old_kw,new_kw", INTERP_CASES)
def test_interpolating_restart_matches_oracle(tmp_path, old_kw, new_kw):
    """InterpInputVel on another grid: native C++ against the NumPy restatement, 1e-13 of each
    field's scale; the pressure is zero and the time comes from the master file."""
    rng = np.random.default_rng(10)
    d, _ = _old_files(tmp_path, dict(old_kw), rng)
    new_text = bou_text(*new_kw["dims"], **{k: v for k, v in new_kw.items() if k != "dims"})
    inp = ag.parse_bou_in(new_text)
    got = ag.read_flow_interp(d, inp)
    assert got["interpolated"] and not got["pr_read"] and got["time"] == 0.75
    assert np.all(got["pr"] == 0.0)
    g = o.create_grid(o.parse_bou_in(new_text))
    m = rs.read_master(d, False)
    old = {k: h5.read(os.path.join(d, f"continua_{k}.h5"), "var") for k in ("vx", "vy", "vz", "temp")}
    want = rs.interp_input_vel(old, m, g)
    for k in ("vx", "vy", "vz", "temp"):
        scale = max(np.abs(want[k]).max(), 1e-300)
        assert np.abs(got[k] - want[k]).max() < 1e-13 * scale, k


def test_interpolating_restart_of_refined_salinity(tmp_path):
    """InterpInputSal: the refined salinity from another refined grid (and another coarse grid)."""
    rng = np.random.default_rng(11)
    old_kw = dict(dims=(16, 12, 8), multires=1, nxmr=32, nymr=24, nzmr=16, flagsal=1, istr3r=4, rays=1e6)
    d, f = _old_files(tmp_path, dict(old_kw), rng, sal=True)
    new_text = bou_text(16, 12, 8, multires=1, nxmr=40, nymr=36, nzmr=12, flagsal=1, istr3r=0, rays=-1e6,
                        sfixn=0)
    inp = ag.parse_bou_in(new_text)
    got = ag.read_flow_interp(d, inp)
    assert got["interpolated"]
    g = o.create_grid(o.parse_bou_in(new_text))
    mg = sa.create_mgrd(g)
    m = rs.read_master(d, True)
    salo = h5.read(os.path.join(d, "continua_sal.h5"), "var")[..., :m.nxr - 1]
    want = rs.interp_input_sal(salo, m, g, mg)
    assert got["sal"].shape == want.shape == (12, 36, 40)
    assert np.abs(got["sal"] - want).max() < 1e-13 * np.abs(want).max()
    # the coarse grid did not change: the flow fields come through the same interpolation as
    # the identity map (Hermite weights (0, 1, 0, 0) on coinciding points)
    for k in ("temp",):
        np.testing.assert_allclose(got[k][..., :16], f[k][..., :16], rtol=0, atol=1e-14)


def _solenoidal(inp, rng):
    """vx, vy from a stream function at the cell corners (discrete divergence zero), vz = 0."""
    g = o.create_grid(o.parse_bou_in(bou_text(inp.nxm, inp.nym, inp.nzm, istr3=inp.istr3, str3=inp.str3)))
    nxm, nym, nzm = inp.nxm, inp.nym, inp.nzm
    nx = nxm + 1
    xc = g.xc[:nx]
    yc = np.arange(nym) / nym * inp.ylen
    zz = np.arange(nzm)[:, None, None]
    X, Y = xc[None, None, :], yc[None, :, None]
    psi = np.sin(np.pi * X) ** 2 * (np.cos(2 * np.pi * Y / inp.ylen) + 0.3 * np.sin(4 * np.pi * Y / inp.ylen)) \
        * (1.0 + 0.2 * np.cos(2 * np.pi * zz / max(nzm, 1)))
    psi = psi + 0.01 * rng.standard_normal(psi.shape) * np.sin(np.pi * X) ** 2
    dy = nym / inp.ylen
    vx = (np.roll(psi, -1, axis=1) - psi) * dy                         # at (xc_k, ym_j)
    vy = np.zeros_like(vx)
    vy[..., :nxm] = -(psi[..., 1:] - psi[..., :nxm]) / (xc[1:] - xc[:nxm])   # at (xm_k, yc_j)
    return dict(vx=vx, vy=vy, vz=np.zeros_like(vx), temp=np.zeros_like(vx), pr=np.zeros_like(vx))


def _divergence(f, inp, xc):
    nxm = inp.nxm
    dy, dz = inp.nym / inp.ylen, inp.nzm / inp.zlen
    dvx = (f["vx"][..., 1:nxm + 1] - f["vx"][..., :nxm]) / (xc[1:] - xc[:nxm])
    dvy = (np.roll(f["vy"], -1, axis=1) - f["vy"])[..., :nxm] * dy
    dvz = (np.roll(f["vz"], -1, axis=0) - f["vz"])[..., :nxm] * dz
    return dvx + dvy + dvz, np.abs(dvx).max()


@pytest.mark.parametrize("dims_old,dims_new", [((16, 24, 4), (24, 36, 6)), ((32, 32, 1), (20, 48, 1))])
def test_interpolating_restart_keeps_a_solenoidal_field_solenoidal(tmp_path, dims_old, dims_new):
    """The velocity is rebuilt from interpolated gradients, so a discretely divergence-free field
    stays divergence-free on the new grid away from the periodic seams (the last y row and z plane
    close through the first one), to round-off of the gradient scale."""
    rng = np.random.default_rng(12)
    old_inp = ag.parse_bou_in(bou_text(*dims_old))
    f = _solenoidal(old_inp, rng)
    div_old, _ = _divergence(f, old_inp, o.create_grid(o.parse_bou_in(bou_text(*dims_old))).xc[:dims_old[0] + 1])
    assert np.abs(div_old).max() < 1e-10
    d = str(tmp_path / "old")
    ag.write_flow_field(d, ag.continua_master(old_inp, 0.0), f, final=True)
    new_inp = ag.parse_bou_in(bou_text(*dims_new))
    got = ag.read_flow_interp(d, new_inp)
    xc = o.create_grid(o.parse_bou_in(bou_text(*dims_new))).xc[:dims_new[0] + 1]
    div, scale = _divergence(got, new_inp, xc)
    inner = div[:max(dims_new[2] - 1, 1), :dims_new[1] - 1, :]
    assert np.abs(inner).max() < 1e-11 * scale


def test_interpolating_restart_resolves_smooth_fields(tmp_path):
    """A smooth temperature onto a finer, differently stretched grid: cubic Hermite accuracy."""
    old_inp = ag.parse_bou_in(bou_text(32, 32, 16))
    g0 = o.create_grid(o.parse_bou_in(bou_text(32, 32, 16)))
    new_text = bou_text(48, 40, 24, istr3=0)
    g1 = o.create_grid(o.parse_bou_in(new_text))

    def field(g, nxm, nym, nzm):
        x = np.append(g.xm[:nxm], 0.0)[None, None, :]
        y = g.ym[None, :, None]
        z = g.zm[:, None, None]
        t = 0.5 - x + 0.1 * np.sin(np.pi * x) * np.cos(2 * np.pi * y) * np.cos(2 * np.pi * z)
        t[..., -1] = 0.0
        return np.broadcast_to(t, (nzm, nym, nxm + 1)).copy()
    rng = np.random.default_rng(13)
    f = _fields(old_inp, rng)
    f["temp"] = field(g0, 32, 32, 16)
    d = str(tmp_path / "old")
    ag.write_flow_field(d, ag.continua_master(old_inp, 0.0), f, final=True)
    got = ag.read_flow_interp(d, ag.parse_bou_in(new_text))
    want = field(g1, 48, 40, 24)
    assert np.abs(got["temp"][..., :48] - want[..., :48]).max() < 2e-4


def test_interpolating_restart_refusals(tmp_path):
    rng = np.random.default_rng(14)
    d, f = _old_files(tmp_path, dict(dims=(16, 12, 8)), rng)
    same = ag.read_flow_interp(d, ag.parse_bou_in(bou_text(16, 12, 8)))
    assert not same["interpolated"] and same["pr_read"]
    for k in ("vx", "vy", "vz", "temp", "pr"):
        np.testing.assert_array_equal(same[k], f[k])
    for text in (bou_text(16, 12, 1), bou_text(16, 12, 8, ylen=2.0)):
        with pytest.raises(ag.AfidError) as e:
            ag.read_flow_interp(d, ag.parse_bou_in(text))
        assert e.value.status == ag.AFID_E_INVALID


def test_allocation_failure_is_a_status_not_a_crash(tmp_path):
    """No C++ exception crosses the C ABI: the padded copy the refined salinity file needs
    (x extent nxmr + 1) cannot be allocated for an absurd refined grid, and the call answers
    AFID_E_ALLOC (the caller's salinity array is never read, the allocation comes first)."""
    inp = _input(multires=0)
    rng = np.random.default_rng(15)
    f = _fields(inp, rng)
    m = ag.continua_master(inp, 0.0)
    m.multires, m.nxr, m.nyr, m.nzr, m.istr3r = 1, 1 << 20, 1 << 20, 1 << 12, 0
    f["sal"] = np.zeros(4)
    with pytest.raises(ag.AfidError) as e:
        ag.write_flow_field(str(tmp_path / "o"), m, f, final=True)
    assert e.value.status == ag.AFID_E_ALLOC


def test_native_writer_matches_the_golden_restart_set(tmp_path):
    """tests/golden/continua/ holds a restart set written by the oracle's own version-0 writer
    (tests/golden/make_continua_golden.py); the native writer must produce the same bytes from the
    same arrays, and both readers must read the set back."""
    gold = os.path.join(os.path.dirname(__file__), "golden", "continua")
    inp = ag.parse_bou_in(bou_text(4, 3, 2, multires=1, nxmr=8, nymr=6, nzmr=4, flagsal=1, istr3r=4))
    m = ag.continua_master(inp, 0.625)
    f = {k: h5.read(os.path.join(gold, f"continua_{k}.h5"), "var") for k in ("vx", "vy", "vz", "temp", "pr")}
    f["sal"] = h5.read(os.path.join(gold, "continua_sal.h5"), "var")[..., :8]
    d = str(tmp_path / "out")
    ag.write_flow_field(d, m, f, final=True)
    names = sorted(os.listdir(gold))
    assert sorted(os.listdir(d)) == names
    for n in names:
        assert open(os.path.join(d, n), "rb").read() == open(os.path.join(gold, n), "rb").read(), n
    back = ag.read_flow_field(gold, m, with_sal=True)
    assert back["time"] == 0.625
    for k in ("vx", "vy", "vz", "temp", "pr", "sal"):
        np.testing.assert_array_equal(back[k], f[k])


def test_nested_groups_and_large_groups(tmp_path):
    """Groups nest through '/' paths; an empty group is an entry of its own; a group of 600
    members needs a two-level group B-tree (75 symbol table nodes over three leaf nodes).  The
    oracle reader and the native reader both find every dataset."""
    rng = np.random.default_rng(16)
    d = {f"big/{k:05d}": rng.standard_normal(3) for k in range(600)}
    d.update({"g/a": np.arange(4, dtype=np.int32), "g/b/c": rng.standard_normal((2, 3)), "empty": None,
              "top": np.array([2.5])})
    path = str(tmp_path / "nested.h5")
    ag.h5_write(path, d)
    f = h5.H5File(path)
    assert sorted(f.root()) == ["big", "empty", "g", "top"]
    assert f.is_group("empty") and f.links(f.resolve("empty")) == {}
    assert sorted(f.links(f.resolve("g"))) == ["a", "b"]
    btree = [int.from_bytes(b[:8], "little") for t, _, b in f.messages(f.resolve("big")) if t == 0x11][0]
    assert f.buf[f._abs(btree) + 5] == 1                       # root node one level above the leaves
    assert len(f.links(f.resolve("big"))) == 600
    for k, v in d.items():
        if v is None:
            continue
        np.testing.assert_array_equal(f.read(k), v)
        np.testing.assert_array_equal(ag.h5_read(path, k), v.astype(np.float64))
    with pytest.raises(ag.AfidError) as e:
        ag.h5_read(path, "g")                                    # a group is not a dataset
    assert e.value.status == ag.AFID_E_IO


def test_means_file_layout(tmp_path):
    """means.h5 as CalcMeanProfiles / CalcSalStats lay it out: one group per profile, one dataset
    per sample named nint(time / TOUT) as five digits."""
    rng = np.random.default_rng(17)
    times = np.array([0.5, 1.0, 1.5000000001])
    prof = rng.standard_normal((3, 15, 16))
    sal = rng.standard_normal((3, 6, 24))
    d = str(tmp_path / "outputdir")
    ag.write_means(d, 0.5, times, prof, sal)
    p = os.path.join(d, "means.h5")
    groups = list(ag.PROFILE_NAMES) + list(ag.SAL_PROFILE_NAMES)
    assert sorted(h5.names(p)) == sorted(groups)
    f = h5.H5File(p)
    for q, g in enumerate(groups):
        assert sorted(f.links(f.resolve(g))) == ["00001", "00002", "00003"], g
        for s in range(3):
            want = prof[s, q] if q < 15 else sal[s, q - 15]
            np.testing.assert_array_equal(f.read(f"{g}/{s + 1:05d}"), want)
            np.testing.assert_array_equal(ag.h5_read(p, f"{g}/{s + 1:05d}"), want)
    # no samples yet: the empty groups HdfCreateMeansFile makes
    ag.write_means(str(tmp_path / "empty"), 0.5, np.zeros(0), np.zeros((0, 15, 16)))
    f0 = h5.H5File(str(tmp_path / "empty" / "means.h5"))
    assert sorted(f0.root()) == sorted(ag.PROFILE_NAMES)
    assert all(f0.links(f0.resolve(g)) == {} for g in ag.PROFILE_NAMES)
    # two samples with the same NNNNN: the later one is stored, as HdfSerialWriteReal1D deletes
    # the existing dataset before it writes (h5tools/HdfRoutines.F90:159-161)
    ag.write_means(str(tmp_path / "twice"), 0.5, np.array([0.5, 0.52, 1.0]), prof)
    f2 = h5.H5File(str(tmp_path / "twice" / "means.h5"))
    for q, g in enumerate(ag.PROFILE_NAMES):
        assert sorted(f2.links(f2.resolve(g))) == ["00001", "00002"], g
        np.testing.assert_array_equal(f2.read(f"{g}/00001"), prof[1, q])
        np.testing.assert_array_equal(f2.read(f"{g}/00002"), prof[2, q])


def test_means_samples_closer_than_half_tout_keep_the_later(tmp_path):
    """With dt > TOUT/2 two main-loop sample points can round to the same nint(time / TOUT); the
    reference's writer then replaces the first profile by the second.  The Recorder (and
    afid_run_io's sample list, which goes through the same afid_write_means) store the later one."""
    text = bou_text(6, 8, 4, tout=0.5, tframe=0.0)
    inp = ag.parse_bou_in(text)
    fake = _FakeSolver(6, 8, 4)
    d = str(tmp_path / "outputdir")
    rec = ag.Recorder(fake, inp, d, ag.Tables(inp))
    for t in (0.0, 0.3, 0.7, 1.0):            # numbers 0, 1, 1, 2: the 0.7 sample replaces 0.3
        rec.profiles(t)
    rec.flush()
    m = h5.H5File(os.path.join(d, "means.h5"))
    assert sorted(m.links(m.resolve("Tbar"))) == ["00000", "00001", "00002"]
    np.testing.assert_array_equal(m.read("Tbar/00000"), np.full(6, 100.0))
    np.testing.assert_array_equal(m.read("Tbar/00001"), np.full(6, 300.0))   # the third call
    np.testing.assert_array_equal(m.read("vxT/00002"), np.full(6, 403.0))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_movie_file_layout(tmp_path, axis):
    """flowmov/movie_{x,y,z}cut.h5 as MakeMovie*Cut.F90 / h5_tools.F90 lay them out: groups vx, vy,
    vz, temp, sal; one plane per frame named nint(time / TFRAME); the y and z cuts keep nx rows for
    vx and nxm for the cell-centred fields; a later frame with the same number replaces the
    earlier one."""
    rng = np.random.default_rng(18 + axis)
    nxm, nym, nzm, nxmr, nymr, nzmr = 6, 8, 4, 12, 16, 8
    nx = nxm + 1
    rows, cols = [(nzm, nym), (nzm, nx), (nym, nx)][axis]
    rrows, rcols = [(nzmr, nymr), (nzmr, nxmr), (nymr, nxmr)][axis]
    times = np.array([0.1, 0.2, 0.2 + 1e-9, 0.4])          # frames 1, 2, 2 (replaces), 4
    planes = rng.standard_normal((4, 4, rows, cols))
    sal = rng.standard_normal((4, rrows, rcols))
    d = str(tmp_path / "outputdir")
    ag.write_movie(d, axis, 0.1, times, planes, nxm, nym, nzm, sal, (nxmr, nymr, nzmr))
    p = os.path.join(d, "flowmov", ["movie_xcut.h5", "movie_ycut.h5", "movie_zcut.h5"][axis])
    f = h5.H5File(p)
    assert sorted(f.root()) == sorted(["vx", "vy", "vz", "temp", "sal"])
    for v, g in enumerate(("vx", "vy", "vz", "temp", "sal")):
        assert sorted(f.links(f.resolve(g))) == ["00001", "00002", "00004"], g
        for frame, src in (("00001", 0), ("00002", 2), ("00004", 3)):
            got = f.read(f"{g}/{frame}")
            if g == "sal":
                want = sal[src]
            elif axis == 0 or g == "vx":
                want = planes[src, v]
            else:
                want = planes[src, v][:, :nxm]
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("axis", [1, 2])
def test_movie_mean_file_layout(tmp_path, axis):
    """flowmov/movie_ymean.h5 and movie_zmean.h5 (mean_zplane.F90 through write_H5_plane): the
    layout of the y and z cuts, under the plane-mean file names."""
    rng = np.random.default_rng(28 + axis)
    nxm, nym, nzm, nxmr, nymr, nzmr = 6, 8, 4, 12, 16, 8
    nx = nxm + 1
    rows = nzm if axis == 1 else nym
    rrows = nzmr if axis == 1 else nymr
    times = np.array([0.0, 0.1, 0.2])
    planes = rng.standard_normal((3, 4, rows, nx))
    sal = rng.standard_normal((3, rrows, nxmr))
    d = str(tmp_path / "outputdir")
    ag.write_movie_mean(d, axis, 0.1, times, planes, nxm, nym, nzm, sal, (nxmr, nymr, nzmr))
    p = os.path.join(d, "flowmov", "movie_ymean.h5" if axis == 1 else "movie_zmean.h5")
    f = h5.H5File(p)
    assert sorted(f.root()) == sorted(["vx", "vy", "vz", "temp", "sal"])
    for v, g in enumerate(("vx", "vy", "vz", "temp")):
        assert sorted(f.links(f.resolve(g))) == ["00000", "00001", "00002"]
        for fr in range(3):
            want = planes[fr, v] if g == "vx" else planes[fr, v][:, :nxm]
            np.testing.assert_array_equal(f.read(f"{g}/{fr:05d}"), want)
    np.testing.assert_array_equal(f.read("sal/00002"), sal[2])
    with pytest.raises(ag.AfidError):
        ag.write_movie_mean(d, 0, 0.1, times, planes, nxm, nym, nzm)   # no x-mean file


def test_spectrum_file_layout(tmp_path):
    """{vx,vy,vz,te}_spectrum.h5 (write_3D_spectrum, h5_tools.F90:229-302): dataset 'var' with the
    declared (nxm, nym, nzm) extent, the nym/2 + 1 computed wavenumber rows first, zeros after."""
    rng = np.random.default_rng(30)
    nxm, nym, nzm = 5, 12, 4
    half = rng.random((nzm, nym // 2 + 1, nxm))
    p = str(tmp_path / "vx_spectrum.h5")
    ag.write_spectrum_file(p, half, nym)
    assert h5.names(p) == ["var"]
    got = h5.read(p, "var")
    assert got.shape == (nzm, nym, nxm)
    np.testing.assert_array_equal(got[:, :nym // 2 + 1, :], half)
    assert np.all(got[:, nym // 2 + 1:, :] == 0.0)
    with pytest.raises(ValueError):
        ag.write_spectrum_file(p, half, nym + 4)


def test_oracle_mean_plane_is_the_loop_sum():
    """The oracle's ymean / zmean: ascending-order sums divided once (checked against an
    explicit triple loop) on a small field."""
    rng = np.random.default_rng(31)
    f = rng.standard_normal((3, 4, 5))
    y = np.zeros((3, 5))
    z = np.zeros((4, 5))
    for i in range(3):
        for j in range(4):
            for k in range(5):
                y[i, k] += f[i, j, k]
                z[j, k] += f[i, j, k]
    np.testing.assert_array_equal(o.mean_plane(f, 1), y / 4.0)
    np.testing.assert_array_equal(o.mean_plane(f, 2), z / 3.0)


def test_grid_info_file(tmp_path):
    """cordin_info.h5 as WriteGridInfo.F90 writes it, against the oracle's grids."""
    text = bou_text(16, 12, 8, multires=1, nxmr=24, nymr=18, nzmr=16, flagsal=1, istr3r=4)
    tables = ag.Tables(ag.parse_bou_in(text))
    mgrd = ag.Mgrd(tables)
    d = str(tmp_path / "outputdir")
    ag.write_grid_info(d, tables, mgrd)
    g = o.create_grid(o.parse_bou_in(text))
    m = sa.create_mgrd(g)
    p = os.path.join(d, "cordin_info.h5")
    assert sorted(h5.names(p)) == sorted(["xm", "xc", "ym", "zm", "xmr", "xcr", "ymr", "zmr"])
    want = dict(xm=g.xm[:16], xc=g.xc[:17], ym=g.ym, zm=g.zm, xmr=m.xmr[1:25], xcr=m.xcr, ymr=m.ymr, zmr=m.zmr)
    for k, v in want.items():
        got = h5.read(p, k)
        assert got.shape == v.shape, k
        np.testing.assert_allclose(got, v, rtol=0, atol=1e-15, err_msg=k)
    ag.write_grid_info(str(tmp_path / "flat"), ag.Tables(ag.parse_bou_in(bou_text(16, 12, 8))))
    assert sorted(h5.names(str(tmp_path / "flat" / "cordin_info.h5"))) == ["xc", "xm", "ym", "zm"]


class _FakeSolver:
    """Stands in for ag.Solver on the CPU: every array it returns encodes what was asked for."""

    def __init__(self, nxm, nym, nzm, refined=None):
        self.nxm, self.nym, self.nzm, self.nx = nxm, nym, nzm, nxm + 1
        self.refined = refined
        self.calls = 0

    def mean_profiles(self):
        self.calls += 1
        return {n: np.full(self.nxm, 100.0 * self.calls + q) for q, n in enumerate(ag.PROFILE_NAMES)}

    def sal_profiles(self):
        return {n: np.full(self.refined[0], -100.0 * self.calls - q) for q, n in enumerate(ag.SAL_PROFILE_NAMES)}

    def mean_plane(self, which, axis):
        shape = {1: (self.nzm, self.nx), 2: (self.nym, self.nx)}[axis]
        return np.full(shape, -(1000.0 * which + 10.0 * axis))

    def sal_mean_plane(self, axis):
        nxmr, nymr, nzmr = self.refined
        return np.full((nzmr, nxmr) if axis == 1 else (nymr, nxmr), -7.0 * axis)

    def slice(self, which, axis, index):
        shape = {0: (self.nzm, self.nym), 1: (self.nzm, self.nx), 2: (self.nym, self.nx)}[axis]
        return np.full(shape, 1000.0 * which + 100.0 * axis + index)

    def sal_download(self):
        nxmr, nymr, nzmr = self.refined
        k = np.arange(nxmr)[None, None, :]
        j = np.arange(nymr)[None, :, None]
        i = np.arange(nzmr)[:, None, None]
        return (1e4 * i + 1e2 * j + k).astype(np.float64)


def test_recorder_writes_the_reference_outputs(tmp_path):
    """ag.Recorder: cordin_info.h5 at start, a means.h5 sample per TOUT call, the three movie cuts
    per TFRAME call at the reference's cut positions (0-based: x at 0 and vx at 1, y at nym/2,
    z at nzm/2; salinity on its own grid)."""
    text = bou_text(6, 8, 4, multires=1, nxmr=12, nymr=16, nzmr=8, flagsal=1, istr3r=4, tout=0.5, tframe=0.25)
    inp = ag.parse_bou_in(text)
    tables = ag.Tables(inp)
    mgrd = ag.Mgrd(tables)
    fake = _FakeSolver(6, 8, 4, refined=(12, 16, 8))
    d = str(tmp_path / "outputdir")
    rec = ag.Recorder(fake, inp, d, tables, mgrd)
    assert os.path.exists(os.path.join(d, "cordin_info.h5"))
    for t in (0.0, 0.5):
        rec.profiles(t)
    for t in (0.25, 0.5):
        rec.frame(t)
    rec.flush()
    m = h5.H5File(os.path.join(d, "means.h5"))
    assert sorted(m.links(m.resolve("Tbar"))) == ["00000", "00001"]
    np.testing.assert_array_equal(m.read("vxT/00001"), np.full(6, 203.0))
    np.testing.assert_array_equal(m.read("chiS/00000"), np.full(12, -105.0))
    x = h5.H5File(os.path.join(d, "flowmov", "movie_xcut.h5"))
    assert sorted(x.links(x.resolve("vx"))) == ["00001", "00002"]
    assert x.read("vx/00001")[0, 0] == 0 * 1000 + 0 * 100 + 1          # vx at x index 1
    assert x.read("temp/00002")[0, 0] == 3 * 1000 + 0 * 100 + 0        # the others at 0
    y = h5.H5File(os.path.join(d, "flowmov", "movie_ycut.h5"))
    assert y.read("vy/00001").shape == (4, 6) and y.read("vx/00001").shape == (4, 7)
    assert y.read("vz/00001")[0, 0] == 2 * 1000 + 1 * 100 + 4          # y index nym/2 = 4
    for name, axis in (("movie_ymean.h5", 1), ("movie_zmean.h5", 2)):   # mean_yplane / mean_zplane
        mf = h5.H5File(os.path.join(d, "flowmov", name))
        assert sorted(mf.links(mf.resolve("temp"))) == ["00001", "00002"]
        assert mf.read("vx/00001").shape == ((4, 7) if axis == 1 else (8, 7))
        assert mf.read("vy/00002")[0, 0] == -(1000 * 1 + 10 * axis)
        assert mf.read("sal/00001").shape == ((8, 12) if axis == 1 else (16, 12))
    z = h5.H5File(os.path.join(d, "flowmov", "movie_zcut.h5"))
    assert z.read("vx/00002")[0, 0] == 0 * 1000 + 2 * 100 + 2          # z index nzm/2 = 2
    np.testing.assert_array_equal(x.read("sal/00001"), fake.sal_download()[:, :, 0])
    np.testing.assert_array_equal(y.read("sal/00001"), fake.sal_download()[:, 8, :])
    np.testing.assert_array_equal(z.read("sal/00001"), fake.sal_download()[4, :, :])


def test_nested_layout_matches_the_oracle_writer_byte_for_byte(tmp_path):
    """The oracle's own nested-group writer (oracle/afid_h5.py write_v0_tree) and the native
    writer produce the same bytes: a two-level group B-tree, nested and empty groups, and the
    means.h5 written by afid_write_means."""
    rng = np.random.default_rng(19)
    tree = {f"big/{k:05d}": rng.standard_normal(3) for k in range(600)}
    tree.update({"g/a": np.arange(4, dtype=np.int32), "g/b/c": rng.standard_normal((2, 3)), "empty": None,
                 "top": np.array([2.5])})
    a, b = str(tmp_path / "oracle.h5"), str(tmp_path / "native.h5")
    h5.write_v0_tree(a, tree)
    ag.h5_write(b, tree)
    assert open(a, "rb").read() == open(b, "rb").read()
    # means.h5: groups in the library's order, each followed by its samples
    times, prof = np.array([0.5, 1.0]), rng.standard_normal((2, 15, 8))
    ag.write_means(str(tmp_path / "m"), 0.5, times, prof)
    want = {}
    for q, g in enumerate(ag.PROFILE_NAMES):
        want[g] = None
        for s in range(2):
            want[f"{g}/{s + 1:05d}"] = prof[s, q]
    h5.write_v0_tree(str(tmp_path / "means_oracle.h5"), want)
    assert open(tmp_path / "m" / "means.h5", "rb").read() == open(tmp_path / "means_oracle.h5", "rb").read()
