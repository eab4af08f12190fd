"""HDF5 output in the reference's layout (nedyson_b200/h5io.py, nedyson_b200/checkpoint.py).

* round trips of every datatype the simulation files use (complex128 as the compound
  {r, i} of float64, float64, int32 / int64, fixed-length strings, scalars, groups with
  more members than one symbol-table node holds);
* the complex datatype message is byte-for-byte the one in the reference's own files
  (written by HighFive / the HDF5 library, e.g. tests/data/Gfree_const.h5 /GL);
* green_func::print_to_file / read_from_file (reference src/greens.cpp:202-307) of a
  HostGF, reading the Matsubara component under either name (M or GM);
* the free propagator G0_from_h0 against the reference's golden file (free-test.cpp).
"""
import json
import os

import numpy as np

from nedyson_b200.checkpoint import _green_to, read_green
from nedyson_b200.greens import HostGF
from nedyson_b200.h5io import H5File, H5Writer, _dtype_message
from nedyson_b200.inputs import g0_from_h0
from oracle import pyoracle as po

GOLD = os.path.join(os.path.dirname(__file__), "golden")
# datatype message of a std::complex<double> dataset in the reference's files
HIGHFIVE_COMPLEX = bytes.fromhex(
    "16020000100000007200000000000000000000000000000000000000000000000000000000000000"
    "000000000000000011203f000800000000004000340b0034ff030000690000000000000008000000"
    "0000000000000000000000000000000000000000000000000000000011203f000800000000004000"
    "340b0034ff030000")


def test_complex_datatype_matches_reference_files():
    body, _, size = _dtype_message(np.zeros(1, np.complex128))
    assert size == 16
    assert body == HIGHFIVE_COMPLEX


def test_round_trip_all_kinds(tmp_path):
    rng = np.random.default_rng(3)
    w = H5Writer()
    z = rng.normal(size=(5, 4)) + 1j * rng.normal(size=(5, 4))
    w["/G/GL"] = z
    w["/G/nt"] = np.int32(20)
    w["/x/i64"] = np.arange(7, dtype=np.int64)
    w["/x/f"] = rng.normal(size=(2, 3, 4))
    w["/beta"] = 9.5
    w["/solve/params/mode"] = "GF2"
    for i in range(70):
        w[f"/many/m{i:03d}"] = np.float64(i)
    p = str(tmp_path / "f.h5")
    w.save(p)
    f = H5File(p)
    assert f.keys("/") == ["G", "beta", "many", "solve", "x"]
    assert np.array_equal(f["/G/GL"], z) and f["/G/nt"] == 20
    assert np.array_equal(f["/x/i64"], np.arange(7)) and f["/x/f"].shape == (2, 3, 4)
    assert f["/beta"] == 9.5 and f["/solve/params/mode"] == "GF2"
    assert len(f.keys("/many")) == 70 and f["/many/m069"] == 69.0 and f["/many/m000"] == 0.0


def test_green_round_trip_and_matsubara_name(tmp_path):
    rng = np.random.default_rng(4)
    g = HostGF(6, 5, 3, -1)
    for a in (g.les, g.ret, g.tv, g.mat):
        a[:] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    w = H5Writer()
    _green_to(w, "/G", g)
    w["/H/GM"] = g.mat.reshape(-1)  # the name read_from_file looks for
    for k in ("GR", "GL", "GTV"):
        w["/H/" + k] = getattr(g, {"GR": "ret", "GL": "les", "GTV": "tv"}[k]).reshape(-1)
    for k, v in (("nt", 6), ("ntau", 5), ("sig", -1), ("nao", 3)):
        w["/H/" + k] = np.int32(v)
    p = str(tmp_path / "g.h5")
    w.save(p)
    f = H5File(p)
    for grp in ("/G", "/H"):
        h = read_green(f, grp)
        for c in ("les", "ret", "tv", "mat"):
            assert np.array_equal(getattr(h, c), getattr(g, c)), (grp, c)


def test_free_propagator_golden():
    """G0_from_h0 against the reference's fixture.  The fixture's imaginary-time points are
    equidistant (tau_m = m beta / ntau: it predates the Legendre collocation grid), so the
    closed forms are checked on that grid; the time components do not depend on it and are
    also checked for the oracle's restatement."""
    gold = json.load(open(os.path.join(GOLD, "gfree_const.json")))
    nt, ntau, nao, k = gold["Nt"], gold["Ntau"], gold["nao"], gold["k"]
    h0 = np.array(gold["h0"])
    ref = {key: np.array([complex(a, b) for a, b in gold[key]]) for key in ("GR", "GL", "GTV", "GM")}
    x_uniform = np.linspace(-1.0, 1.0, ntau + 1)
    G = HostGF(nt, ntau, nao, -1)
    g0_from_h0(G, x_uniform, gold["mu"], h0, gold["beta"], gold["dt"], k)
    got = {"GR": G.ret.reshape(-1), "GL": G.les.reshape(-1), "GTV": G.tv.reshape(-1), "GM": G.mat.reshape(-1)}
    for key, r in ref.items():
        err = np.linalg.norm(got[key][:len(r)] - r)
        assert err < gold["tol_norm"], ("inputs", key, err)
    Go = HostGF(nt, ntau, nao, -1)
    po.Dyson(nt, ntau, nao, k).g0_from_h0(Go, gold["mu"], h0, gold["beta"], gold["dt"])
    for key, arr in (("GR", Go.ret.reshape(-1)), ("GL", Go.les.reshape(-1))):
        err = np.linalg.norm(arr[:len(ref[key])] - ref[key])
        assert err < gold["tol_norm"], ("oracle", key, err)
