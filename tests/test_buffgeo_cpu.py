""".buffgeo parsing on the host (SWGGeometry.cc:52-383): one-time DISPLACED /
ROTATED transformations composed in order and applied before the vertex
merge, MESHPATH and BUFF_MESH_PATH lookup, the MESH__ special names and the
reference's error cases, checked through bg_geometry_vertices without a GPU."""
import math
import shutil

import numpy as np
import pytest

import buffem


def read_nodes(path):
    lines = open(path).read().splitlines()
    i = lines.index("$Nodes")
    n = int(lines[i + 1])
    return np.array([[float(v) for v in lines[i + 2 + k].split()[1:4]] for k in range(n)])


def geo(tmp_path, body, name="g.buffgeo"):
    p = tmp_path / name
    p.write_text(body)
    return str(p)


def obj(mesh, *lines, label="A", mat="CONST_EPS_4+0.2i"):
    inner = "".join(f" {ln}\n" for ln in lines)
    return f"OBJECT {label}\n MESHFILE {mesh}\n MATERIAL {mat}\n{inner}ENDOBJECT\n"


def rot(theta_deg, axis):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    c, s = math.cos(math.radians(theta_deg)), math.sin(math.radians(theta_deg))
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return c * np.eye(3) + s * K + (1 - c) * np.outer(a, a)


def test_untransformed_vertices_are_the_file_nodes(buffem_lib, sphere, tmp_path):
    mesh = sphere(2)
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh)))
    xyz, origin = G.vertices(0)
    assert np.array_equal(xyz, read_nodes(mesh)) and np.array_equal(origin, np.zeros(3))


def test_displacements_compose_exactly(buffem_lib, sphere, tmp_path):
    mesh = sphere(2)
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "DISPLACED 0.5 0 1", "DISPLACED 0 -2 0.25")))
    xyz, origin = G.vertices(0)
    d = np.array([0.5, 0.0, 1.0]) + np.array([0.0, -2.0, 0.25])
    assert np.array_equal(xyz, read_nodes(mesh) + d) and np.array_equal(origin, d)
    # the displacement form of bg_geometry_create_objects gives the same vertices
    H = buffem.SWGGeometry(meshfiles=mesh, materials=buffem.Material(eps=4 + 0.2j), displacements=[d])
    assert np.array_equal(H.vertices(0)[0], xyz)


def test_rotation_and_order_of_composition(buffem_lib, sphere, tmp_path):
    mesh = sphere(2)
    X = read_nodes(mesh)
    R = rot(90, [0, 0, 1])
    d = np.array([1.0, 0.0, 0.0])
    # displaced, then rotated: XP = R (X + d); the origin goes to R d
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "DISPLACED 1 0 0", "ROTATED 90 ABOUT 0 0 1")))
    xyz, origin = G.vertices(0)
    assert np.allclose(xyz, (X + d) @ R.T, atol=1e-14, rtol=0)
    assert np.allclose(origin, [0, 1, 0], atol=1e-15, rtol=0)
    # both on one line, in the same order: the same transformation
    G1 = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "DISPLACED 1 0 0 ROTATED 90 ABOUT 0 0 1"), "one.buffgeo"))
    assert np.array_equal(G1.vertices(0)[0], xyz)
    # rotated, then displaced: XP = R X + d
    G2 = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "ROTATED 90 ABOUT 0 0 2", "DISPLACED 1 0 0"), "two.buffgeo"))
    xyz2, origin2 = G2.vertices(0)
    assert np.allclose(xyz2, X @ R.T + d, atol=1e-14, rtol=0) and np.array_equal(origin2, d)
    # a rigid motion leaves the numbering alone
    G0 = buffem.SWGGeometry(geo(tmp_path, obj(mesh), "zero.buffgeo"))
    assert np.array_equal(G.faces(0), G0.faces(0)) and np.array_equal(G2.faces(0), G0.faces(0))


def test_general_rotation_is_right_handed_and_rigid(buffem_lib, sphere, tmp_path):
    mesh = sphere(2)
    X = read_nodes(mesh)
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "ROTATED 37.5 ABOUT 1 -2 0.5", "DISPLACED 0.1 0.2 0.3")))
    xyz, origin = G.vertices(0)
    R = rot(37.5, [1, -2, 0.5])
    assert np.allclose(xyz, X @ R.T + [0.1, 0.2, 0.3], atol=1e-14, rtol=0)
    assert np.allclose(R @ R.T, np.eye(3), atol=1e-15) and np.linalg.det(R) > 0
    # right-handed: a quarter turn about +z takes +x to +y
    assert np.allclose(rot(90, [0, 0, 1]) @ [1, 0, 0], [0, 1, 0], atol=1e-15)


def test_two_objects_keep_their_own_transformations(buffem_lib, sphere, tmp_path):
    mesh = sphere(2)
    X = read_nodes(mesh)
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh, "ROTATED 45 ABOUT 0 1 0", label="A")
                               + obj(mesh, "DISPLACED 0 0 3", label="B", mat="VACUUM")))
    assert G.NumObjects == 2 and G.BFIndexOffset == [0, 72, 144]
    assert np.allclose(G.vertices(0)[0], X @ rot(45, [0, 1, 0]).T, atol=1e-14, rtol=0)
    assert np.array_equal(G.vertices(1)[0], X + [0, 0, 3]) and np.array_equal(G.vertices(1)[1], [0, 0, 3])


def test_object_labels(buffem_lib, sphere, tmp_path):
    """GetObjectByLabel matches ignoring case, first match wins, -1 if none;
    objects made from mesh files are labelled by the file name."""
    mesh = sphere(2)
    G = buffem.SWGGeometry(geo(tmp_path, obj(mesh, label="Sphere_A") + obj(mesh, "DISPLACED 0 0 3", label="b")
                               + obj(mesh, "DISPLACED 0 0 6", label="SPHERE_a")))
    assert [G.label(i) for i in range(3)] == ["Sphere_A", "b", "SPHERE_a"]
    assert G.GetObjectByLabel("sphere_a") == 0 and G.GetObjectByLabel("B") == 1
    assert G.GetObjectByLabel("c") == -1
    H = buffem.SWGGeometry(meshfiles=mesh, materials=buffem.Material(eps=2.0))
    assert H.label(0) == mesh and H.GetObjectByLabel(mesh.upper()) == 0
    L = buffem.lib()
    buf = buffem.C.create_string_buffer(4)
    assert L.bg_geometry_object_label(G.h, 0, buf, 4) == 8 and buf.value == b"Sph"
    assert L.bg_geometry_object_label(G.h, 3, None, 0) == buffem.BG_ERR_ARG
    assert L.bg_geometry_object_label(G.h, 0, None, 4) == buffem.BG_ERR_ARG
    assert L.bg_geometry_object_index(G.h, None) == buffem.BG_ERR_ARG


def test_mesh_lookup(buffem_lib, sphere, tmp_path, monkeypatch):
    mesh = sphere(2)
    sub = tmp_path / "meshes"
    sub.mkdir()
    shutil.copy(mesh, sub / "ball.vmsh")
    # MESHPATH relative to the .buffgeo file's directory
    G = buffem.SWGGeometry(geo(tmp_path, "MESHPATH meshes\n" + obj("ball.vmsh")))
    assert G.TotalBFs == 72
    # BUFF_MESH_PATH, colon-separated
    other = tmp_path / "elsewhere"
    other.mkdir()
    monkeypatch.setenv("BUFF_MESH_PATH", f"{tmp_path / 'none'}:{sub}")
    G = buffem.SWGGeometry(geo(other, obj("ball.vmsh")))
    assert G.TotalBFs == 72
    monkeypatch.delenv("BUFF_MESH_PATH")
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(geo(other, obj("ball.vmsh"), "n.buffgeo"))
    assert e.value.status == -2 and "ball.vmsh" in str(e.value)


def test_special_mesh_names(buffem_lib, sphere, tmp_path, monkeypatch):
    shutil.copy(sphere(2), tmp_path / "ball.vmsh")
    monkeypatch.chdir(tmp_path)
    G = buffem.SWGGeometry("MESH__ball__MAT__CONST_EPS_4+0.2i")
    assert G.NumObjects == 1 and G.TotalBFs == 72
    assert buffem.SWGGeometry("MESH__ball.vmsh__MAT__VACUUM").TotalBFs == 72
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry("MESH__ball")
    assert "no MATERIAL" in str(e.value)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry("MESH__ball__SVT__eps")
    assert "could not find file" in str(e.value) and "eps.SVTensor" in str(e.value)


@pytest.mark.parametrize("body,line,words", [
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n DISPLACED 1 2 3 4\nENDOBJECT\n", 4, "junk at end of line"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n ROTATED 30 0 0 1\nENDOBJECT\n", 4, "ABOUT"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n ROTATED 30 ABOUT 0 0 0\nENDOBJECT\n", 4, "axis"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n DISPLACED 1 x 3\nENDOBJECT\n", 4, "bad number"),
    ("OBJECT A\n MESHFILE m.vmsh\nENDOBJECT\n", 3, "no MATERIAL"),
    ("OBJECT A\n MATERIAL CONST_EPS_2\nENDOBJECT\n", 3, "no MESHFILE"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_4+0.2ix\nENDOBJECT\n", 3, "bad permittivity"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL Gold\nENDOBJECT\n", 3, "unknown material Gold"),
    ("OBJECT A\n MESHFILE m.vmsh a\n MATERIAL CONST_EPS_2\nENDOBJECT\n", 2, "one argument"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n LABEL x\nENDOBJECT\n", 4, "syntax error"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n ROT 9 ABOUT 0 0 1\nENDOBJECT\n", 4, "syntax error"),
    ("# comment\n\nOBJECT\n MESHFILE m.vmsh\nENDOBJECT\n", 3, "invalid OBJECT"),
    ("MESHPATH\n", 1, "invalid MESHPATH"),
    ("ENDOBJECT\n", 1, "syntax error"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL CONST_EPS_2\n", 1, "without ENDOBJECT"),
])
def test_reference_error_cases(buffem_lib, tmp_path, body, line, words):
    path = geo(tmp_path, body)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(path)
    assert e.value.status == -2
    msg = str(e.value)
    assert f"{path}:{line}:" in msg and words in msg, msg


def test_empty_file_and_bad_vertex_queries(buffem_lib, sphere, tmp_path):
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(geo(tmp_path, "# nothing\n"))
    assert "no objects" in str(e.value)
    G = buffem.SWGGeometry(geo(tmp_path, obj(sphere(2)), "ok.buffgeo"))
    L = buffem.lib()
    assert L.bg_geometry_vertices(G.h, 1, None, None) == buffem.BG_ERR_ARG
    assert L.bg_geometry_vertices(G.h, -1, None, None) == buffem.BG_ERR_ARG
    assert L.bg_geometry_vertices(None, 0, None, None) == buffem.BG_ERR_ARG
    assert L.bg_geometry_vertices(G.h, 0, None, None) == len(read_nodes(sphere(2)))


DRUDE = """MATERIAL Metal
  # Drude model, w in rad/s
  wp = 1.2e16;   gam = 4.0e13
  Eps(w) = 1 - wp^2 / (w * (w + i*gam));
ENDMATERIAL
"""
LORENTZ = """material Polar
  Eps(w) = EpsInf * (w^2 + a1*i*w + a0) / (w^2 + b1*i*w + b0)
  EpsInf = 6.5
  a0 = -3.3e28
  a1 = +8.9e11
  b0 = -2.2e28; b1 = 8.9e11
  Mu(w) = 1
ENDMATERIAL
"""


def drude(w):
    return 1 - 1.2e16 ** 2 / (w * (w + 1j * 4.0e13))


def lorentz(w):
    return 6.5 * (w * w + 8.9e11j * w - 3.3e28) / (w * w + 8.9e11j * w - 2.2e28)


def test_material_sections(buffem_lib, sphere, tmp_path):
    """MATERIAL ... ENDMATERIAL sections: Eps(w) with w = Omega x 3e14 rad/s,
    constants in any order before use by Eps(w), semicolons, comments, names
    matched ignoring case, Mu(w) ignored."""
    mesh = sphere(2)
    G = buffem.SWGGeometry(geo(tmp_path, DRUDE + LORENTZ + obj(mesh, label="A", mat="METAL")
                               + obj(mesh, "DISPLACED 0 0 3", label="B", mat="polar")
                               + obj(mesh, "DISPLACED 0 0 6", label="C", mat="CONST_EPS_2+0.1i")))
    for omega in (0.1, 0.7, 1.3, 2.0 + 0.05j, 0.3j):
        w = complex(omega) * 3e14
        for obj_, ref in ((0, drude(w)), (1, lorentz(w))):
            got = G.material_eps(obj_, omega)
            assert abs(got - ref) <= 1e-13 * abs(ref), (obj_, omega, got, ref)
        assert G.material_eps(2, omega) == 2 + 0.1j
    L = buffem.lib()
    e = np.zeros(2)
    assert L.bg_geometry_material_eps(G.h, 0, 1.0, 0.0, buffem._ptr(e)) == 1
    assert L.bg_geometry_material_eps(G.h, 2, 1.0, 0.0, buffem._ptr(e)) == 0
    assert L.bg_geometry_material_eps(G.h, 3, 1.0, 0.0, buffem._ptr(e)) == buffem.BG_ERR_ARG
    T = buffem.SWGGeometry(meshfiles=mesh, materials=buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR,
                                                                     tensor=np.diag([2.0, 3.0, 4.0])))
    assert L.bg_geometry_material_eps(T.h, 0, 1.0, 0.0, buffem._ptr(e)) == buffem.BG_ERR_ARG


@pytest.mark.parametrize("expr,value", [
    ("-2^2", -4), ("2^3^2", 512), ("(1+2)*3-4/8", 8.5), ("2*-3", -6), ("-(1-3)", 2),
    ("exp(i*pi)", -1), ("sqrt(-4)", 2j), ("abs(3+4*i)", 5), ("cosh(0) + sinh(0) + tanh(0)", 1),
    ("log(e) + sin(0) + cos(0) + tan(0) + atan(0) + asin(0) + acos(1)", 2), ("1.5e3 + .5", 1500.5),
    ("2^-1", 0.5), ("(1+i)^2", 2j), ("4^0.5", 2), ("step(-0.5) + 2*step(0) + 4*step(3)", 6),
])
def test_material_expressions(buffem_lib, sphere, tmp_path, expr, value):
    G = buffem.SWGGeometry(geo(tmp_path, f"MATERIAL X\n Eps(w) = {expr}\nENDMATERIAL\n" + obj(sphere(2), mat="x")))
    assert abs(G.material_eps(0, 1.0) - value) < 1e-14 * max(1.0, abs(value))


def test_material_constants_chain(buffem_lib, sphere, tmp_path):
    body = "MATERIAL X\n a = 2; b = a*a + i\n c = b / a\n Eps(w) = c + w/3e14\nENDMATERIAL\n"
    G = buffem.SWGGeometry(geo(tmp_path, body + obj(sphere(2), mat="X")))
    assert abs(G.material_eps(0, 0.25) - ((4 + 1j) / 2 + 0.25)) < 1e-15


@pytest.mark.parametrize("body,line,words", [
    ("MATERIAL X\n a = 1\nENDMATERIAL\n", 2, "no Eps(w)"),
    ("MATERIAL X\n Eps(w) = 1 + q\nENDMATERIAL\n", 2, "unknown name q"),
    ("MATERIAL X\n a = w\n Eps(w) = a\nENDMATERIAL\n", 2, "w may only appear"),
    ("MATERIAL X\n Eps(w) = foo(w)\nENDMATERIAL\n", 2, "unknown function foo"),
    ("MATERIAL X\n Eps(w) = (1 + w\nENDMATERIAL\n", 2, "missing )"),
    ("MATERIAL X\n Eps(w) = 1 w\nENDMATERIAL\n", 2, "junk after expression"),
    ("MATERIAL X\n 2a = 1\n Eps(w) = 1\nENDMATERIAL\n", 2, "bad name"),
    ("MATERIAL X\n Eps(w) 1\nENDMATERIAL\n", 2, "NAME = EXPRESSION"),
    ("MATERIAL X\n Eps(w) = 1\n", 1, "without ENDMATERIAL"),
    ("MATERIAL\n", 1, "no name given"),
    ("MATERIAL X Y\n", 1, "syntax error"),
    ("OBJECT A\n MESHFILE m.vmsh\n MATERIAL Later\nENDOBJECT\nMATERIAL Later\n Eps(w) = 2\nENDMATERIAL\n", 3,
     "unknown material Later"),
])
def test_material_section_errors(buffem_lib, tmp_path, body, line, words):
    path = geo(tmp_path, body)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(path)
    assert e.value.status == -2
    msg = str(e.value)
    assert f"{path}:{line}:" in msg and words in msg, msg


def test_dispersive_geometry_is_refused_by_batched_sweeps(buffem_lib, sphere, tmp_path):
    G = buffem.SWGGeometry(geo(tmp_path, DRUDE + obj(sphere(2), mat="Metal")))
    L = buffem.lib()
    geoms = (buffem.C.c_void_p * 1)(G.h)
    w = np.array([1.0, 0.0])
    E0 = np.array([1.0, 0, 0, 0, 0, 0])
    nh = np.array([0, 0, 1.0])
    out = np.zeros(64)
    st = L.bg_batch_sweep(geoms, 1, buffem._ptr(w), 1, buffem._ptr(E0), buffem._ptr(nh), 1, 0, buffem._ptr(out), None)
    assert st == buffem.BG_ERR_ARG and "frequency-dependent" in L.bg_last_error().decode()


def two_spheres(tmp_path, mesh):
    return geo(tmp_path, obj(mesh, label="Upper") + obj(mesh, "DISPLACED 0 0 -0.5", label="Lower"), "two.buffgeo")


def test_trans_files(buffem_lib, sphere, tmp_path):
    """TRANS lines (one-line and TRANS ... ENDTRANS forms): each
    transformation follows the object's own DISPLACED lines; objects not
    named stay in place."""
    mesh = sphere(2)
    X = read_nodes(mesh)
    g = two_spheres(tmp_path, mesh)
    t = tmp_path / "s.trans"
    t.write_text("# separations\n"
                 "TRANS 4.0 OBJECT Upper DISP 0 0 4.0\n"
                 "TRANS  tilt\n  OBJECT lower ROT 90 ABOUT 0 0 1\n  OBJECT UPPER DISP 1 0 0 DISP 0 1 0\nENDTRANS\n"
                 "TRANS 6 OBJECT Upper DISP 0 0 6 OBJECT Lower DISP 0 0 -1\n")
    assert buffem.ReadTransFile(str(t)) == ["4.0", "tilt", "6"]
    G = buffem.SWGGeometry(g, TransFile=str(t), Transformation=0)
    assert np.array_equal(G.vertices(0)[0], X + [0, 0, 4.0]) and np.array_equal(G.vertices(0)[1], [0, 0, 4.0])
    assert np.array_equal(G.vertices(1)[0], X + [0, 0, -0.5])
    G = buffem.SWGGeometry(g, TransFile=str(t), Transformation=1)
    assert np.array_equal(G.vertices(0)[0], X + [1.0, 1.0, 0])
    R = rot(90, [0, 0, 1])
    assert np.allclose(G.vertices(1)[0], (X + [0, 0, -0.5]) @ R.T, atol=1e-14, rtol=0)
    G = buffem.SWGGeometry(g, TransFile=str(t), Transformation=2)
    assert np.array_equal(G.vertices(1)[1], [0, 0, -1.5])
    assert G.TotalBFs == 144 and G.label(0) == "Upper"


@pytest.mark.parametrize("body,line,words", [
    ("TRANS\n", 1, "needs a tag"),
    ("TRANS a OBJECT\n", 1, "needs a label"),
    ("TRANS a OBJECT Upper\n", 1, "no transformation given"),
    ("TRANS a OBJECT Upper DISP 1 2\n", 1, "three numbers"),
    ("TRANS a Upper DISP 1 2 3\n", 1, "expected OBJECT"),
    ("TRANS a\n OBJECT Upper DISP 1 2 3\n", 1, "without ENDTRANS"),
    ("SHIFT a\n", 1, "syntax error"),
    ("TRANS a\n OBJECT Upper SPIN 3\nENDTRANS\n", 2, "unknown transformation SPIN"),
])
def test_trans_file_errors(buffem_lib, sphere, tmp_path, body, line, words):
    t = tmp_path / "bad.trans"
    t.write_text(body)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(two_spheres(tmp_path, sphere(2)), TransFile=str(t))
    msg = str(e.value)
    assert f"{t}:{line}:" in msg and words in msg, msg


def test_trans_file_selection_errors(buffem_lib, sphere, tmp_path):
    g = two_spheres(tmp_path, sphere(2))
    t = tmp_path / "s.trans"
    t.write_text("TRANS 1 OBJECT Middle DISP 0 0 1\n")
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(g, TransFile=str(t))
    assert "no object labelled Middle" in str(e.value)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(g, TransFile=str(t), Transformation=1)
    assert "has 1 transformations" in str(e.value)
    (tmp_path / "empty.trans").write_text("# nothing\n")
    with pytest.raises(buffem.BuffError) as e:
        buffem.ReadTransFile(str(tmp_path / "empty.trans"))
    assert "no transformations" in str(e.value)


def test_long_lines(buffem_lib, sphere, tmp_path):
    """Lines of any length (a 5000-character Eps(w) expression)."""
    terms = " + ".join(["0.001"] * 1000)
    G = buffem.SWGGeometry(geo(tmp_path, f"MATERIAL Long\n Eps(w) = 1 + {terms}\nENDMATERIAL\n" + obj(sphere(2), mat="Long")))
    assert abs(G.material_eps(0, 1.0) - 2.0) < 1e-12


SVT = """# uniaxial crystal with a Drude-like ordinary axis
MATERIAL Ordinary
  wp = 6e14
  Eps(w) = 4 - wp^2/(w*(w + 1e13*i))
ENDMATERIAL
EpsE = 2.5;
Qxx = MP_Ordinary
Qyy = MP_ordinary
Qzz = EpsE + 0.5*i
Qxy = 0.1*MP_CONST_EPS_2+1i
EpsYX = 0.3
Eps13 = w/3e14
"""


def svt_expected(omega):
    w = complex(omega) * 3e14
    eo = 4 - 36e28 / (w * (w + 1e13j))
    q = np.zeros((3, 3), complex)
    q[0, 0] = q[1, 1] = eo
    q[2, 2] = 2.5 + 0.5j
    q[0, 1] = q[1, 0] = 0.5 * (0.1 * (2 + 1j) + 0.3)
    q[0, 2] = q[2, 0] = 0.5 * (w / 3e14 + 0.0)
    return q


def test_svtensor_files(buffem_lib, sphere, tmp_path):
    """SVTENSOR files: MATERIAL sections and MP_ names, numeric constants,
    the Q/Eps component spellings, identity defaults, averaged off-diagonal
    pairs; the tensor at each frequency is what the device receives."""
    (tmp_path / "uni.SVTensor").write_text(SVT)
    G = buffem.SWGGeometry(geo(tmp_path, f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR uni.SVTensor\nENDOBJECT\n"))
    for omega in (0.3, 1.0, 1.7 + 0.02j):
        got = G.material_tensor(0, omega, (0.3, -0.2, 0.1))
        assert np.allclose(got, svt_expected(omega), rtol=1e-14, atol=0), omega
    # the scalar query is the xx component (SVTensor::Evaluate(Omega, x),
    # SVTensor.cc:375-380)
    for omega in (0.3, 1.7 + 0.02j):
        assert G.material_eps(0, omega) == pytest.approx(svt_expected(omega)[0, 0], rel=1e-14)


def test_svtensor_reads_the_whole_file_first(buffem_lib, sphere, tmp_path):
    """Constants and MATERIAL sections may follow the expressions that use
    them (the reference parses the whole file, then sets every constant on
    every expression: SVTensor.cc:88-113); a constant whose name contains
    'Eps2' (MyEps2) is an ordinary constant."""
    body = ("Qzz = A + 1\nQxx = MyEps2 * MP_Late\nA = 3\nMyEps2 = 0.5\n"
            "MATERIAL Late\n Eps(w) = 4 + 2*i\nENDMATERIAL\n")
    (tmp_path / "late.SVTensor").write_text(body)
    G = buffem.SWGGeometry(geo(tmp_path, f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR late.SVTensor\nENDOBJECT\n"))
    q = G.material_tensor(0, 1.0)
    assert np.allclose(q, np.diag([2 + 1j, 2 + 1j, 4]), rtol=0, atol=1e-15)


@pytest.mark.parametrize("body,defaults", [
    ("Eps = 3 + w/3e14\n", "iso"),
    ("Q = 3 + w/3e14\n", "iso"),
    ("Qxx = 3 + w/3e14\n", "iso"),
    ("Qyy = 5\n", "yy"),
])
def test_svtensor_defaults(buffem_lib, sphere, tmp_path, body, defaults):
    (tmp_path / "t.SVTensor").write_text(body)
    G = buffem.SWGGeometry(geo(tmp_path, f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR t.SVTensor\nENDOBJECT\n"))
    q = G.material_tensor(0, 0.5)
    if defaults == "iso":
        assert np.allclose(q, 3.5 * np.eye(3), rtol=0, atol=1e-15)
    else:
        assert np.allclose(q, np.diag([1, 5, 1]), rtol=0, atol=1e-15)


@pytest.mark.parametrize("body,x,want", [
    ("Eps = 2 + x\n", (0.25, 0, 0), 2.25 * np.eye(3)),
    # the given Qxy and the identity's Qyx = 0 are averaged (SVTensor.cc:362-367)
    ("Qxy = r*Theta\n", (0, 0.5, 0), np.array([[1, 0.125 * np.pi, 0], [0.125 * np.pi, 1, 0], [0, 0, 1]])),
    ("MATERIAL In\n Eps(w) = 2\nENDMATERIAL\nEps = step(1.0-r)*MP_In + step(r-1.0)*MP_VACUUM\n", (0.3, 0.2, 0.1),
     2 * np.eye(3)),
])
def test_svtensor_of_position(buffem_lib, sphere, tmp_path, body, x, want):
    """SVTENSOR expressions of position (SVTensor.cc:96-102: x, y, z, r,
    Theta, Phi) load and evaluate at a point on the host; the assembly
    compiles them for the device at each frequency (tests/test_gpu_ref_pins)."""
    (tmp_path / "p.SVTensor").write_text(body)
    G = buffem.SWGGeometry(geo(tmp_path, f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR p.SVTensor\nENDOBJECT\n"))
    assert np.allclose(G.material_tensor(0, 1.0, x), want, rtol=0, atol=1e-14)


@pytest.mark.parametrize("body,words", [
    ("Qxw = 1\n", "invalid component"),
    ("Eps = MP_Nothing\n", "unknown material MP_Nothing"),
    ("c = two\nEps = 1\n", "invalid constant value"),
    ("just words\n", "syntax error"),
    ("Eps = 1 +\n", "unexpected end"),
    ("MATERIAL M\n Eps(w) = 2\n", "without ENDMATERIAL"),
    ("Eps = MP_CONST_EPS_1 + MP_CONST_EPS_2 + MP_CONST_EPS_3 + MP_CONST_EPS_4\n", "too many MP_"),
    ("Eps = MP_CONST_EPS_2 + Eps2\n", "Eps2 is not defined"),
])
def test_svtensor_errors(buffem_lib, sphere, tmp_path, body, words):
    (tmp_path / "bad.SVTensor").write_text(body)
    with pytest.raises(buffem.BuffError) as e:
        buffem.SWGGeometry(geo(tmp_path, f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR bad.SVTensor\nENDOBJECT\n"))
    assert words in str(e.value), str(e.value)


def test_svtensor_lookup_path_and_shared_materials(buffem_lib, sphere, tmp_path, monkeypatch):
    """SVTENSOR files are found along BUFF_SVTENSOR_PATH and may use MATERIAL
    sections of the .buffgeo file (one material database, as MatProp's)."""
    sub = tmp_path / "tensors"
    sub.mkdir()
    (sub / "m.SVTensor").write_text("Eps = 2*MP_Host\n")
    monkeypatch.setenv("BUFF_SVTENSOR_PATH", str(sub))
    body = "MATERIAL Host\n Eps(w) = 1.5 + 0.25*i\nENDMATERIAL\n" + \
        f"OBJECT A\n MESHFILE {sphere(2)}\n SVTENSOR m.SVTensor\nENDOBJECT\n"
    G = buffem.SWGGeometry(geo(tmp_path, body))
    assert np.allclose(G.material_tensor(0, 1.0), (3 + 0.5j) * np.eye(3), rtol=0, atol=1e-15)


def test_material_tensor_of_functor_materials(buffem_lib, sphere):
    """bg_geometry_material_tensor restates the device's functors on the host."""
    mesh = sphere(2)
    T = np.array([[2, 0.4, 0], [0.2, 3, 0.1j], [0, 0.3j, 4]], complex)
    cases = [
        (buffem.Material(eps=4 + 0.2j), (0, 0, 0), (4 + 0.2j) * np.eye(3)),
        (buffem.Material(kind=buffem.BG_MAT_CONST_TENSOR, tensor=T), (0, 0, 0), None),
        (buffem.Material(kind=buffem.BG_MAT_JANUS_Z, eps=4, eps2=12 + 1j), (0, 0, 0.2), 4 * np.eye(3)),
        (buffem.Material(kind=buffem.BG_MAT_JANUS_Z, eps=4, eps2=12 + 1j), (0, 0, -0.2), (12 + 1j) * np.eye(3)),
        (buffem.Material(kind=buffem.BG_MAT_GAUSSIAN, eps=3 + 0.1j, amp=1.5, width=0.7, center=(0.1, 0, 0)),
         (0.4, 0.2, -0.1), (3 + 0.1j + 1.5 * np.exp(-(0.09 + 0.04 + 0.01) / 0.49)) * np.eye(3)),
    ]
    for mat, x, ref in cases:
        G = buffem.SWGGeometry(meshfiles=mesh, materials=mat)
        q = G.material_tensor(0, 1.0, x)
        if ref is None:
            ref = T.copy()
            for a in range(3):
                b = (a + 1) % 3
                ref[a, b] = ref[b, a] = 0.5 * (T[a, b] + T[b, a])
        assert np.allclose(q, ref, rtol=1e-15, atol=1e-15), (mat.kind, q, ref)
