"""The C ABI from C: tests/c/host_abi.c includes include/canard_gpu.h as a
C11 translation unit, links libcanard_b200.so and calls the host-only entry
points (coefficients, LU factors, exchange plans, restart files) with no GPU
and no Python in between; its values equal the Python binding's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from canard_b200 import api, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_caller(tmp_path):
    exe = str(tmp_path / "host_abi")
    libdir = os.path.dirname(api.LIBPATH)
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "host_abi.c"), "-o", exe, "-L", libdir, "-lcanard_b200",
                    "-Wl,-rpath," + libdir], check=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    vals = dict(line.split(" ", 1) for line in r.stdout.splitlines() if " " in line)
    assert r.stdout.splitlines()[-1] == "ok"
    assert float(vals["coeffs0"]) == api.coeffs(0.85, 0.85)[0]
    assert float(vals["penta_xu0"]) == api.penta(0.85, 0.85, 33, 0, 0, 0)[0].reshape(-1)[0]
    cs = cases.decompose(cases.tgv(nx=16, ny=16, nz=30), [(1, 1, 2)])
    links = api.plan_export(cs, api.PLAN_FACES)
    assert int(vals["links"]) == len(links)
    assert int(vals["cross"]) == int(np.sum(links[:, 0] != links[:, 3]))
    t6, q = api.read_restart_file(str(tmp_path / "restart_c.da"), 40)
    assert list(t6) == [12, 3, 0.25, 0.5, 0.75, 1.5]
