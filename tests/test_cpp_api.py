"""The C++ mirror of OFELI's API (include/ofeli_b200/OFELI.h): an
OFELI-style demo program compiles against it, and on the GPU reproduces the
reference's golden solution."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_err
from ofeli_b200 import fields
from oracle import oracle as O

LIBDIR = os.path.join(ROOT, "ofeli_b200")


def build_demo(tmp_path, name="laplace_demo"):
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L", LIBDIR,
                    "-lofeli_gpu", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("name", ["laplace_demo", "mesh_file_demo"])
def test_demo_compiles_and_links(tmp_path, name):
    assert os.path.exists(build_demo(tmp_path, name))


@pytest.mark.gpu
def test_demo_reproduces_reference(cuda, tmp_path):
    g, info = load_golden("p2d_65")
    exe = build_demo(tmp_path)
    f = fields.uniform_pm1(1234, 65 * 65)
    fpath, upath = str(tmp_path / "f.f64"), str(tmp_path / "u.f64")
    f.tofile(fpath)
    out = subprocess.run([exe, "64", "DILU", fpath, upath], check=True, capture_output=True,
                         text=True).stdout
    words = out.split()
    assert int(words[words.index("iterations") + 1]) == info["runs"]["CG_DILU"]["iters"]
    u = np.fromfile(upath)
    _, _, code = O.mesh2d(64, 64)
    assert rel_err(u, O.insert_bc(code, g["x_CG_DILU"])) <= 1e-12
    assert float(out.split("residual")[1].split()[0]) <= 1e-10


@pytest.mark.gpu
def test_mesh_file_demo_reproduces_reference(cuda, tmp_path):
    """Mesh(file, true) + DC3DT4 + CG/D-ILU on the Kuhn-cube file, and
    Mesh::put of the mesh read."""
    g, info = load_golden("meshio")
    exe = build_demo(tmp_path, "mesh_file_demo")
    f = fields.uniform_pm1(info["tet"]["seed_f"], info["files"]["tet"]["nodes"])
    fpath, upath, mpath = str(tmp_path / "f.f64"), str(tmp_path / "u.f64"), str(tmp_path / "p.m")
    f.tofile(fpath)
    out = subprocess.run([exe, os.path.join(ROOT, "tests", "golden", "meshio_tet.m"), fpath,
                          upath, mpath], check=True, capture_output=True, text=True).stdout
    words = out.split()
    assert abs(int(words[words.index("iterations") + 1])
               - info["runs"]["tet_CG_DILU"]["iters"]) <= 2
    assert rel_err(np.fromfile(upath), g["tet_u_CG_DILU"]) <= 1e-12
    assert open(mpath, "rb").read() == g["tet_put"].tobytes()
