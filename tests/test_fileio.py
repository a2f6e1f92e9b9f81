"""File formats at either side of the solver (specfwat_b200.fileio).

Pinned against the reference's own example files: the CMTSOLUTION and
STATIONS copies in tests/golden/reference_files/, and, when
SPECFWAT_REFERENCE_ROOT names a SpecFWAT source tree, a model file (Fortran unformatted record) and a SAC trace
whose structure tests/golden/make_reference_fixtures.py recorded.
"""
import json
import os
import struct

import numpy as np
import pytest

from specfwat_b200 import fileio as F

HERE = os.path.join(os.path.dirname(__file__), "golden", "reference_files")
# root of a SpecFWAT source tree, for the checks against its binary example
# files; skipped when unset
REF = os.environ.get("SPECFWAT_REFERENCE_ROOT", "")
SUMMARY = json.load(open(os.path.join(HERE, "summary.json")))


def test_cmtsolution_and_stations():
    c = F.read_cmtsolution(os.path.join(HERE, "CMTSOLUTION"))
    assert c["name"] == "hom_explosion"
    assert (c["time_shift"], c["hdur"], c["lat"], c["lon"], c["depth"]) == (0.0, 5.0, 36.0, -120.0, 1.0)
    assert c["mt"] == (1e23, 1e23, 1e23, 0.0, 0.0, 0.0)
    x, y, z, mt, f0, ts = F.cmt_to_source(c)
    assert (x, y, z, f0, ts) == (-120.0, 36.0, -1000.0, 5.0, 0.0)
    assert mt[0] == pytest.approx(1e16)
    st = F.read_stations(os.path.join(HERE, "STATIONS"))
    assert st[0]["name"] == "ST001" and st[0]["network"] == "MX"
    assert st[0]["lat"] == pytest.approx(-0.8209138629358446)
    xyz = F.stations_xyz(st)
    assert xyz.shape == (len(st), 3) and xyz[0, 0] == pytest.approx(st[0]["lon"])


@pytest.mark.skipif(not REF or not os.path.isdir(REF),
                    reason="SPECFWAT_REFERENCE_ROOT not set to a SpecFWAT source tree")
def test_reference_model_file_and_sac():
    m = SUMMARY["model_bin"]
    k = F.read_kernel_bin(os.path.join(REF, m["file"]))
    assert k.shape == (m["nspec"], 5, 5, 5)
    assert list(k.reshape(-1)[:5]) == m["first"]
    assert float(k.min()) == m["min"] and float(k.max()) == m["max"]
    assert float(k.astype(np.float64).sum()) == pytest.approx(m["sum"], rel=1e-12)
    s = SUMMARY["sac"]
    hdr, d = F.read_sac(os.path.join(REF, s["file"]))
    assert hdr["npts"] == s["npts"] == d.size and hdr["nvhdr"] == 6
    assert hdr["delta"] == pytest.approx(s["delta"]) and hdr["b"] == s["b"]
    assert float(d.astype(np.float64).sum()) == pytest.approx(s["sum"], rel=1e-12)


def test_kernel_bin_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    k = rng.standard_normal((6, 7, 5, 5, 5)).astype(np.float32)
    paths = F.write_event_kernels(tmp_path, 3, k)
    assert [os.path.basename(p) for p in paths] == [
        f"proc000003_{n}_kernel.bin" for n in ("rho", "mu", "kappa", "rhop", "beta", "alpha")]
    for p, kk in zip(paths, k):
        raw = open(p, "rb").read()
        assert len(raw) == 8 + 7 * 500
        assert struct.unpack("<i", raw[:4])[0] == 7 * 500 == struct.unpack("<i", raw[-4:])[0]
        assert np.array_equal(F.read_kernel_bin(p, nspec=7), kk)
    bad = bytearray(open(paths[0], "rb").read())
    bad[-1] ^= 1
    open(tmp_path / "bad.bin", "wb").write(bytes(bad))
    with pytest.raises(ValueError):
        F.read_kernel_bin(tmp_path / "bad.bin")
    with pytest.raises(ValueError):
        F.read_kernel_bin(paths[0], nspec=8)


def test_adj_ascii_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    adj = rng.standard_normal((2, 3, 50))
    st = [{"name": "ST001", "network": "MX"}, {"name": "ST002", "network": "MX"}]
    F.write_adjoint_sources(tmp_path, st, adj, t0=1.2, dt=0.02)
    t, v = F.read_adj_ascii(tmp_path / "MX.ST002.BXZ.adj")
    assert np.allclose(t, -1.2 + 0.02 * np.arange(50), atol=1e-14)
    assert np.array_equal(v, adj[1, 2])


def test_sac_round_trip(tmp_path):
    d = np.sin(np.arange(300) * 0.1).astype(np.float32)
    F.write_sac(tmp_path / "a.sac", d, 0.05, b=-2.0, baz=123.5, dist=4.2e4)
    hdr, r = F.read_sac(tmp_path / "a.sac")
    assert np.array_equal(r, d)
    assert hdr["npts"] == 300 and hdr["delta"] == pytest.approx(0.05)
    assert hdr["b"] == -2.0 and hdr["baz"] == 123.5 and hdr["dist"] == pytest.approx(4.2e4)
    assert hdr["e"] == pytest.approx(-2.0 + 0.05 * 299)
