"""Particle-state CSV reader and writer against text the reference solver
wrote (tests/golden/particle_state_00500_sub8.csv, cut from its resume file)."""
import os

import numpy as np
import pytest

from lsmps_vpm_v2_b200.state import _stod, read_particle_state, write_particle_state

FIX = os.path.join(os.path.dirname(__file__), "golden", "particle_state_00500_sub8.csv")


def test_reads_the_reference_state():
    p = read_particle_state(FIX)
    n = p["x"].size
    assert n == 2716
    assert p["x"][0] == 2.05 and p["y"][0] == 0.65
    assert p["gz"][0] == -0.000386427 and p["vorticity"][0] == -0.966067
    assert p["u"][0] == 1.01056 and p["v"][0] == -0.455162 and p["s"][0] == 0.02
    assert p["active"].dtype == np.uint8 and set(np.unique(p["active"])) <= {0, 1}
    assert 0 < int(p["active"].sum()) < n          # the state has inactive particles
    assert np.all((p["chi"] >= 0.0) & (p["chi"] <= 1.0)) and np.any(p["chi"] == 1.0)   # body mask
    assert "pressure" not in p
    assert len(np.unique(p["s"])) > 1               # several particle sizes


def test_writer_reproduces_the_reference_text():
    # the resume file was written with the stream's default 6 significant digits
    p = read_particle_state(FIX)
    out = FIX + ".tmp"
    try:
        write_particle_state(out, p, precision=6)
        with open(out) as a, open(FIX) as b:
            assert a.read() == b.read()
    finally:
        os.remove(out)


def test_round_trip_at_twelve_digits(tmp_path):
    rng = np.random.default_rng(3)
    n = 500
    p = dict(x=rng.normal(size=n), y=rng.normal(size=n) * 1e-7, gz=rng.normal(size=n) * 1e5,
             vorticity=rng.normal(size=n), u=rng.normal(size=n), v=rng.normal(size=n),
             s=rng.uniform(0.01, 0.1, n), active=(rng.random(n) < 0.7).astype(np.uint8), chi=rng.random(n))
    pres = rng.normal(size=n)
    f = tmp_path / "state.csv"
    write_particle_state(str(f), p, ubody=0.25, vbody=-0.5, pressure=pres, ngh_num=np.arange(n),
                         ngh_ids=[[i, i + 1, i + 2] for i in range(n)])
    header = f.read_text().split("\n", 1)[0]
    assert header == "xp,yp,gpz,vor,up,vp,sp,active,chi,pressure,ngh_num,ngh_ID"
    r = read_particle_state(str(f))
    for k in ("x", "y", "gz", "vorticity", "s", "chi"):
        np.testing.assert_allclose(r[k], p[k], rtol=1e-11, atol=0)
    np.testing.assert_allclose(r["u"], p["u"] - 0.25, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(r["v"], p["v"] + 0.5, rtol=1e-11, atol=1e-15)
    np.testing.assert_allclose(r["pressure"], pres, rtol=1e-11, atol=0)
    assert np.array_equal(r["active"], p["active"])


def test_stod_semantics():
    assert _stod("12|13|14") == 12.0        # a neighbour list reads as its first entry
    assert _stod(" -1.5e-3abc") == -1.5e-3
    assert _stod("1") == 1.0 and _stod(".5") == 0.5
    with pytest.raises(ValueError):
        _stod("")
    with pytest.raises(ValueError):
        _stod("|3")


def test_particle_level(tmp_path):
    p = read_particle_state(FIX, sigma=0.02, max_level=4)
    s = p["s"]
    # size sigma * 2^k sits k levels above max_level
    for sz, lvl in ((0.02, 4), (0.04, 3), (0.08, 2)):
        if np.any(np.isclose(s, sz)):
            assert np.all(p["level"][np.isclose(s, sz)] == lvl)
