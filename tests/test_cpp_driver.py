"""The C++ drop-in header (include/mag_field.hpp) compiles and links against
libmag_b200.so; on a GPU the driver's trajectories equal the Python API's."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "hmc_driver")


def build_driver() -> str:
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
           "hmc_driver.cpp"), "-L", os.path.join(ROOT, "mag_b200"), "-lmag_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "mag_b200"), "-o", BIN]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return BIN


def test_cpp_driver_compiles_and_links():
    build_driver()
    assert os.path.exists(BIN)


@pytest.mark.gpu
def test_cpp_driver_matches_python_api(tmp_path):
    import mag_b200 as M

    out = subprocess.run([build_driver(), "4", str(tmp_path / "cfg.nersc")], check=True, capture_output=True,
                         text=True)
    res = json.loads(out.stdout.strip().splitlines()[-1])
    with M.Chmc((4, 4, 4, 8), mag=2, n_stout=1, rho=0.1, n_steps=4, tau=1.0, seed=5) as c:
        c.hot_start(3)
        H, parts = c.get_hamiltonian()
        recs = c.run_chmc(3)
    assert res["h0"] == H and res["kin0"] == parts[0]
    assert res["dh"] == [r[0]["delta_h"] for r in recs]
    assert abs(res["cplaq_after"] - res["cplaq_before"]) < 1e-12
    # export_config_nersc -> import_config_nersc (two-row file, third row rebuilt) resumes the same field
    assert abs(res["plaq_reload"] - res["plaq"]) < 1e-13
    # init_momentum(L, traj, m = 4) draws exactly twice the m = 1 momenta (width sqrt(m));
    # evolve_momentum(L, dt = 0.1, m = 2.5) adds F dt m = 0.25 F to every component
    assert res["sqrt_m_exact"] == 1
    assert res["fmax"] > 0.1 and res["kick_err"] < 1e-14 * max(1.0, res["fmax"])
