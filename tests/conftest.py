import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "buff-em_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def meshdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("meshes"))


@pytest.fixture(scope="session")
def sphere(meshdir):
    import meshgen

    def make(n, radius=1.0, jitter=0.0, seed=0):
        return meshgen.cached_sphere(meshdir, n, radius, jitter, seed)

    return make


@pytest.fixture(scope="session")
def ref_mesh(meshdir):
    """Writes one of the reference's own test meshes (tests/golden/ref_meshes.npz)
    back to gmsh 2.2 text and returns the path."""
    data = np.load(os.path.join(ROOT, "tests", "golden", "ref_meshes.npz"))

    def make(name):
        path = os.path.join(meshdir, name + ".vmsh")
        if not os.path.exists(path):
            ids, xyz, tets = data[name + "_ids"], data[name + "_xyz"], data[name + "_tets"]
            with open(path, "w") as f:
                f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(ids))
                for i, (x, y, z) in zip(ids, xyz):
                    f.write("%d %.17g %.17g %.17g\n" % (i, x, y, z))
                f.write("$EndNodes\n$Elements\n%d\n" % len(tets))
                for k, t in enumerate(tets):
                    f.write("%d 4 2 0 1 %d %d %d %d\n" % (k + 1, *t))
                f.write("$EndElements\n")
        return path

    return make


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def buffem_lib():
    import buffem
    buffem.lib()
    return buffem
