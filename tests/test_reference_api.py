"""The reference-signature C++ API (include/lt_reference_api.hpp): a C++ caller written
against the reference's function names, linked against liblt_b200.so, gives the
reference's results (golden fixture of Benchmarks/ConfigFiles/90Pot81.par)."""
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, catalog_from_npz, golden, grid_from_npz, max_rel_err

import lenstool_hpc_b200 as lt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    lib = build.build()
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cuda = pathlib.Path("/usr/local/cuda")
    exe = tmp_path_factory.mktemp("refapi") / "driver"
    cmd = [cxx, "-std=c++17", "-O1", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}",
           str(ROOT / "tests" / "reference_api_driver.cpp"), "-o", str(exe), f"-L{lib.parent}", "-llt_b200",
           f"-Wl,-rpath,{lib.parent}", f"-L{cuda / 'lib64'}", "-lcudart", f"-Wl,-rpath,{cuda / 'lib64'}"]
    subprocess.run(cmd, check=True)
    return exe


def test_reference_signatures_on_90pot81(driver, tmp_path, oracle_lib):
    z = golden("par_90Pot81.npz")
    cat, g = catalog_from_npz(z), grid_from_npz(z)
    cat.dlsds = np.full(cat.n, 0.7)
    n = cat.n
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(cat.type.astype(np.int32).tobytes())
        for a in (cat.position_x, cat.position_y, cat.b0, cat.ellipticity_angle, cat.anglecos, cat.anglesin,
                  cat.ellipticity_potential, cat.rcore, cat.rcut, cat.dlsds):
            f.write(np.ascontiguousarray(a, np.float64).tobytes())
        f.write(np.array([g.xmin, g.xmax, g.ymin, g.ymax], np.float64).tobytes())
        f.write(np.int32(g.nx).tobytes())
    out = tmp_path / "out.bin"
    r = subprocess.run([str(driver), str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    o = np.fromfile(out, dtype=np.float64).reshape(14, g.ny, g.nx)
    dls, dos, dol = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos
    TOL = 1e-12
    assert max_rel_err(o[0], z["grad"][0]) <= TOL and max_rel_err(o[1], z["grad"][1]) <= TOL
    for k in range(4):
        assert max_rel_err(o[2 + k], z["hess"][k]) <= TOL
    a, b, c = z["hess"][0], z["hess"][1], z["hess"][2]
    assert max_rel_err(o[6], oracle_lib.map("ampli1", a, b, c, D).reshape(g.ny, g.nx)) <= 1e-10
    assert max_rel_err(o[7], z["amplif5"]) <= TOL
    assert max_rel_err(o[8], b * D) <= TOL
    h = 70. / 50.
    mult = lt.CH4PIG * h / dol / dls * dos
    assert max_rel_err(o[9], (a + c) * 0.5 * 0.7 * mult) <= 1e-12
    assert max_rel_err(o[10], z["pot"] * D) <= TOL
    assert max_rel_err(o[11], z["grad"][0] * D) <= TOL and max_rel_err(o[12], z["grad"][1] * D) <= TOL
    assert max_rel_err(o[13], z["hess"][0]) <= TOL
