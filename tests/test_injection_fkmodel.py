"""FKmodel files (the reference's ``src_rec/FKmodel_<event>``, read by
``read_fk_model``, src/shared/fk_coupling.f90:12-59) into the layered
incident field of the FK injection.

The fixture ``tests/golden/FKmodel_example`` is written in that keyword
format with values chosen here.  Checked: the parsed values; the azimuth
convention (a wave from back azimuth 120 degrees travels toward 300
degrees); the incident wavefront passing ORIGIN_WAVEFRONT at ORIGIN_TIME
with the AMPLITUDE given; zero free-surface traction and continuity at both
interfaces; malformed files rejected.
"""
import os

import numpy as np
import pytest

from specfwat_b200.injection import plane_wave_from_fkmodel, read_fkmodel

FIX = os.path.join(os.path.dirname(__file__), "golden", "FKmodel_example")


def test_parse():
    fk = read_fkmodel(FIX)
    assert fk["nlayer"] == 3 and fk["wave"] == "SV"
    assert np.allclose(fk["vp"], [4500.0, 6000.0, 8000.0])
    assert np.allclose(fk["vs"], [2600.0, 3464.0, 4600.0])
    assert np.allclose(fk["rho"], [2400.0, 2700.0, 3300.0])
    assert np.allclose(fk["ztop"], [0.0, -4000.0, -25000.0])
    assert fk["back_azimuth"] == 120.0 and fk["take_off"] == 18.5
    assert fk["frequency_max"] == 0.25 and fk["amplitude"] == 2.0
    assert fk["origin_wavefront"] == (12000.0, 8000.0, -40000.0) and fk["origin_time"] == 3.0


def test_field_geometry_and_boundary_conditions():
    w = plane_wave_from_fkmodel(read_fkmodel(FIX))
    # propagation toward azimuth 300 (clockwise from north): east -0.866, north 0.5
    assert np.allclose(w.eh[:2], [np.sin(np.deg2rad(300.0)), np.cos(np.deg2rad(300.0))])
    assert w.p == pytest.approx(np.sin(np.deg2rad(18.5)) / 4600.0)
    assert np.allclose(w.h, [4000.0, 21000.0])
    t = np.arange(1500) * 0.02
    # the incident wave alone passes the origin point first: peak at ORIGIN_TIME
    # with the AMPLITUDE given (interface reflections come ~6.5 s later)
    u0 = w.displacement(np.array([[12000.0, 8000.0, -40000.0]]), t)[:, 0]
    early = t < 6.0
    k = np.argmax(np.linalg.norm(u0[early], axis=1))
    assert abs(t[k] - 3.0) < 0.03
    assert np.linalg.norm(u0[k]) == pytest.approx(2.0, rel=1e-3)
    up = np.array([[0.0, 0.0, 1.0]])
    side = np.array([[1.0, 0.0, 0.0]])
    top = np.array([[5000.0, 3000.0, 0.0]])
    assert np.abs(w.traction(top, up, t)).max() < 1e-9 * np.abs(w.traction(top, side, t)).max()
    for zi in (-4000.0, -25000.0):
        a = np.array([[2000.0, -1000.0, zi + 1e-3]])
        b = np.array([[2000.0, -1000.0, zi - 1e-3]])
        ua, ub = w.displacement(a, t), w.displacement(b, t)
        assert np.abs(ua - ub).max() < 1e-6 * np.abs(ua).max(), zi
        ta, tb = w.traction(a, up, t), w.traction(b, up, t)
        assert np.abs(ta - tb).max() < 1e-6 * np.abs(ta).max(), zi


def test_malformed_files(tmp_path):
    text = open(FIX).read()
    bad = tmp_path / "FKmodel_bad"
    bad.write_text(text.replace("LAYER 2 ", "LAYER 5 "))
    with pytest.raises(ValueError, match="LAYER"):
        read_fkmodel(bad)
    bad.write_text(text.replace("-25000.", "1000."))
    with pytest.raises(ValueError, match="tops"):
        read_fkmodel(bad)
    bad.write_text(text.replace("INCIDENT_WAVE      sv", "INCIDENT_WAVE      sh"))
    with pytest.raises(ValueError, match="INCIDENT_WAVE"):
        read_fkmodel(bad)
    bad.write_text(text.replace("ORIGIN_WAVEFRONT", "# ORIGIN_WAVEFRONT"))
    with pytest.raises(ValueError, match="x0"):
        plane_wave_from_fkmodel(read_fkmodel(bad))
    w = plane_wave_from_fkmodel(read_fkmodel(bad), x0=(0.0, 0.0, -30000.0))
    assert w.x0[2] == -30000.0
