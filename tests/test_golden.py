"""Regression fixtures (tests/golden/, written by tests/golden/make_golden.py from
the FP64 oracle; the reference has no golden vectors of its own).

CPU: the oracle still reproduces them.  GPU: the library matches them to the
parity bars (force 1e-11 relative, sums 1e-12 relative, Delta H 1e-9, same
accept, NERSC files load with their header checksum and plaquette, demon sweeps
with the same hit counts and energies within 1e-9).
"""
import os

import numpy as np
import pytest

import mag_b200 as M
import oracle as O
from mag_b200.field_hmc import read_nersc_header
from oracle import nersc as N

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DIMS = (4, 4, 4, 4)
NERSC_DIMS = (2, 2, 2, 4)


@pytest.fixture(scope="module")
def g():
    return dict(np.load(os.path.join(HERE, "hmc_4x4x4x4.npz")))


def _rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def test_oracle_reproduces_hmc_fixture(g):
    U = O.gen_hot(DIMS, 3)
    assert np.array_equal(U, g["U"])
    p_thin = O.make_params(DIMS, mag=2, action=1, beta=2.25, n_stout=0, n_steps=8)
    p_st = O.make_params(DIMS, mag=2, action=1, beta=2.25, n_stout=3, rho=0.1, n_steps=8)
    assert _rel(O.force(p_thin, U), g["F"]) < 1e-14
    assert _rel(O.force(p_st, U), g["F_stout3"]) < 1e-14
    plaq, rect = O.plaq_rect(DIMS, U)
    assert abs(plaq - g["plaq"]) <= 1e-13 * abs(g["plaq"]) and abs(rect - g["rect"]) <= 1e-13 * abs(g["rect"])
    assert np.array_equal(O.gen_momenta(DIMS, 11, 0), g["P"])
    U1, rec = O.trajectory(p_thin, 0, U, g["P"], float(g["uniform"]), [0.0, 0.0])
    assert abs(rec["delta_h"] - g["delta_h"]) < 1e-10 and rec["accept"] == int(g["accept"])
    assert np.abs(U1 - g["U_after"]).max() < 1e-12


@pytest.mark.parametrize("name,two_row", [("unit_2x2x2x4.nersc", False), ("hot_2x2x2x4.nersc", True)])
def test_nersc_fixtures_oracle_and_header_reader(tmp_path, name, two_row):
    path = os.path.join(HERE, name)
    U, info = N.import_config(path, NERSC_DIMS)
    assert info["checksum"] == info["checksum_header"]
    h = read_nersc_header(path)
    assert h["dims"] == list(NERSC_DIMS) and h["two_row"] == int(two_row) and h["checksum_header"] == info["checksum"]
    # re-export: identical bytes except the ARCHIVE_DATE line (local time zone)
    out = tmp_path / "re"
    seq = 2 if two_row else 1
    N.export_config(out, NERSC_DIMS, U, two_row=two_row, beta=2.25, seq=seq, label="golden", unix_time=1735689600)
    if not two_row:
        a = [ln for ln in open(path, "rb").read().split(b"\n") if not ln.startswith(b"ARCHIVE_DATE")]
        b = [ln for ln in open(out, "rb").read().split(b"\n") if not ln.startswith(b"ARCHIVE_DATE")]
        assert a == b
    else:
        # the import rebuilt the third row with reunitarize, which also renormalises rows 0, 1
        pa = np.frombuffer(open(path, "rb").read()[h["payload_offset"]:], ">f8")
        pb = np.frombuffer(open(out, "rb").read()[read_nersc_header(out)["payload_offset"]:], ">f8")
        assert pa.shape == pb.shape and np.abs(pa - pb).max() < 1e-15


DEMON_DIMS, DEMON_HOT, DEMON_SEED, DEMON_SWEEPS, DEMON_EMAX = (4, 4, 4, 4), 5, 9, 2, 50.0


@pytest.fixture(scope="module")
def gd():
    return dict(np.load(os.path.join(HERE, "demon_4x4x4x4.npz")))


def test_oracle_reproduces_demon_fixture(gd):
    U1, E, acc, rej, dev = O.demon_sweeps(DEMON_DIMS, O.gen_hot(DEMON_DIMS, DEMON_HOT), seed=DEMON_SEED,
                                          n_sweeps=DEMON_SWEEPS, e_max=DEMON_EMAX)
    assert acc == int(gd["accepted"]) and rej == int(gd["rejected"])
    assert np.abs(E - gd["E"]).max() < 1e-12
    assert np.abs(U1[::7] - gd["U_after_every7"]).max() < 1e-14
    assert np.all(dev < 1e-13)


@pytest.mark.gpu
def test_gpu_matches_demon_fixture(gd):
    with M.Chmc(DEMON_DIMS, mag=0) as c:
        c.set_gauge(O.gen_hot(DEMON_DIMS, DEMON_HOT))
        res = c.demon_microcanonical(DEMON_SWEEPS, DEMON_EMAX, seed=DEMON_SEED, update_links=True)
        Ug = c.get_gauge()
    assert res["accepted"] == int(gd["accepted"]) and res["rejected"] == int(gd["rejected"])
    assert np.abs(res["demon_energy"] - gd["E"]).max() < 1e-9
    assert np.abs(Ug[::7] - gd["U_after_every7"]).max() < 1e-12


@pytest.mark.gpu
def test_gpu_matches_hmc_fixture(g):
    with M.Chmc(DIMS, mag=2, action="iwasaki", beta=2.25, n_stout=0, n_steps=8, seed=11) as c:
        c.set_gauge(g["U"])
        assert _rel(c.get_force(), g["F"]) < 1e-11
        p, r, _ = c.gauge_action()
        assert abs(p - g["plaq"]) <= 1e-12 * abs(g["plaq"]) and abs(r - g["rect"]) <= 1e-12 * abs(g["rect"])
        c.init_momentum(g["P"])
        c.set_uniforms([float(g["uniform"])])
        (rec,) = c.trajectory(refresh_momenta=False)
        assert abs(rec["delta_h"] - g["delta_h"]) < 1e-9 and rec["accept"] == int(g["accept"])
        assert np.abs(c.get_gauge() - g["U_after"]).max() < 1e-10
    with M.Chmc(DIMS, mag=2, action="iwasaki", beta=2.25, n_stout=3, rho=0.1) as c:
        c.set_gauge(g["U"])
        assert _rel(c.get_force(), g["F_stout3"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["unit_2x2x2x4.nersc", "hot_2x2x2x4.nersc"])
def test_gpu_loads_nersc_fixtures(name):
    path = os.path.join(HERE, name)
    Uo, _ = N.import_config(path, NERSC_DIMS)
    with M.Chmc(NERSC_DIMS, mag=0) as c:
        info = c.import_config_nersc(path)
        assert info["checksum"] == info["checksum_header"]
        assert np.abs(c.get_gauge() - Uo).max() < 1e-15
