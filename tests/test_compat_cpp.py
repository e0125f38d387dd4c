"""The libbuff-compatible C++ layer (buff-em_b200/compat/libbuff_b200.hpp)
compiles against the C-ABI and drives the path like buff-scatter does."""
import os
import subprocess

import numpy as np
import pytest

import buffem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "scatter_driver")
    lib = os.path.join(ROOT, "buff-em_b200")
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", os.path.join(ROOT, "tests", "cpp", "scatter_driver.cpp"),
                    "-L", lib, "-lbuffem_b200", f"-Wl,-rpath,{lib}", "-o", out], check=True)
    return out


def geo(tmp_path, mesh, eps="4+0.2i"):
    p = tmp_path / "g.buffgeo"
    p.write_text(f"OBJECT S\n MESHFILE {mesh}\n MATERIAL CONST_EPS_{eps}\nENDOBJECT\n")
    return str(p)


def test_compat_geometry(driver, sphere, tmp_path):
    r = subprocess.run([driver, geo(tmp_path, sphere(2)), "1.0", "geometry-only"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "bfs 72" in r.stdout


def test_compat_objects_carry_transformed_vertices(driver, sphere, tmp_path):
    """Objects[no]->Vertices / Origin after ROTATED and DISPLACED lines, as the
    Python binding reads them."""
    mesh = sphere(2)
    p = tmp_path / "t.buffgeo"
    p.write_text(f"MATERIAL Drude\n wp = 3e14\n Eps(w) = 1 - wp^2/(w*(w + 1e13*i))\nENDMATERIAL\n"
                 f"OBJECT A\n MESHFILE {mesh}\n MATERIAL VACUUM\nENDOBJECT\n"
                 f"OBJECT B\n MESHFILE {mesh}\n MATERIAL drude\n DISPLACED 0 0 3\n"
                 f" ROTATED 30 ABOUT 1 0 0\nENDOBJECT\n")
    r = subprocess.run([driver, str(p), "0.5", "geometry-only"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "label B 1" in r.stdout
    eps = complex(*map(float, [ln for ln in r.stdout.splitlines() if ln.startswith("eps ")][0].split()[1:]))
    w = 0.5 * 3e14
    assert abs(eps - (1 - 9e28 / (w * (w + 1e13j)))) <= 1e-14 * abs(eps)
    qzz = complex(*map(float, [ln for ln in r.stdout.splitlines() if ln.startswith("qzz ")][0].split()[1:]))
    assert qzz == eps
    last = [ln for ln in r.stdout.splitlines() if ln.startswith("last ")][0].split()[1:]
    xyz, origin = buffem.SWGGeometry(str(p)).vertices(1)
    assert int(last[0]) == len(xyz) and int(last[1]) == 72
    assert np.array_equal(np.array(last[2:5], float), origin)
    assert np.array_equal(np.array(last[5:8], float), xyz[0])
    assert np.allclose(origin, [0, -3 * np.sin(np.pi / 6), 3 * np.cos(np.pi / 6)], atol=1e-15)


@pytest.mark.gpu
def test_compat_drive_matches_python(driver, sphere, tmp_path):
    g = geo(tmp_path, sphere(3))
    r = subprocess.run([driver, g, "1.0"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    vals = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())
    j0 = complex(*map(float, vals["J0"].split()))
    pabs = float(vals["PAbs"].split()[0])
    G = buffem.SWGGeometry(g)
    M = G.AssembleVIEMatrix(1.0)
    M.LUFactorize()
    pw = buffem.PlaneWave([1, 0, 0], [0, 0, 1])
    J = G.AssembleRHSVector(1.0, pw)
    M.LUSolve(J)
    assert abs(J[0] - j0) <= 1e-12 * abs(J[0])
    assert abs(G.GetPFTMatrix(J, 1.0, pw)[0, 0] - pabs) <= 1e-10 * abs(pabs)


@pytest.mark.gpu
def test_compat_extras_match_python(driver, sphere, tmp_path):
    """The C++ layer's full PFT, GetFields and buff-neq flux give the Python
    binding's numbers (both sit on the same C-ABI)."""
    g = geo(tmp_path, sphere(3))
    r = subprocess.run([driver, g, "0.8", "extras"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    vals = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())
    G = buffem.SWGGeometry(g)
    M = G.AssembleVIEMatrix(0.8)
    M.LUFactorize()
    pw = buffem.PlaneWave([1, 0, 0], [0, 0, 1])
    J = G.AssembleRHSVector(0.8, pw)
    M.LUSolve(J)
    assert abs(G.GetPFTMatrix(J, 0.8, pw, full=True)[0, 4] - float(vals["Fz"])) <= 1e-10 * abs(float(vals["Fz"]))
    F = G.GetFields(pw, J, 0.8, np.array([[0.3, -0.2, 2.5]]))[0]
    ex = complex(*map(float, vals["Ex"].split()))
    hy = complex(*map(float, vals["Hy"].split()))
    assert abs(F[0] - ex) <= 1e-10 * abs(ex) and abs(F[4] - hy) <= 1e-10 * abs(hy)
    prad = buffem.NEQ(G).GetFlux(0.8)[0, 0, 1]
    assert abs(prad - float(vals["PRad"])) <= 1e-9 * abs(prad)
