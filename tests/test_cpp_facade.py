"""C++ facade (include/vx_octree.hpp): compiles against vx.h and links libvx.so
(CPU); casts through the C ABI on a GPU (gpu)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "castray_demo.cpp")
LIBDIR = os.path.join(ROOT, "vbvs--vixen_b200")


def _build(tmp_path):
    exe = str(tmp_path / "castray_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lvx", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_facade_compiles_and_links(vx, tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_facade_cast_ray(vx, cuda, tmp_path):
    out = subprocess.run([_build(tmp_path)], check=True, capture_output=True, text=True).stdout.splitlines()
    # Expected values are the oracle's (the restated reference castRay): the -y
    # ray enters the voxel's top face at y = 4 (t = 36, normal +y); the +x and
    # diagonal rays miss because the reference's POP (SVOTraversal.cpp:437-504,
    # MAX_RES = 2^22) resumes one scale too fine after crossing a parent cell.
    assert out[0].startswith("hit=0")
    assert out[1] == "hit=1 t=36.000000 pos=17,3,10 normal=0,1,0 scale=5"
    assert out[2].startswith("hit=0")
    assert out[3] == "batch hits=1000"


def test_demo_expectations_come_from_the_oracle(vo):
    s = vo.OracleScene.from_keys([(17, 3, 10), (0, 0, 0), (63, 63, 63)], (0, 0, 0), (64, 64, 64), 6)
    h = [s.castRay(o, d, 0.0, 1000.0) for o, d in [((-5, 3.5, 10.5), (1, 0, 0)), ((17.5, 40, 10.5), (0, -1, 0)),
                                                    ((10.5, 3.5, 3.5), (1, 0, 1))]]
    assert [int(x["flags"] & 1) for x in h] == [0, 1, 0]
    assert h[1]["t"] == 36.0 and tuple(h[1]["key"]) == (17, 3, 10) and tuple(h[1]["normal"]) == (0, 1, 0)
