"""The C++ host side (include/kf_gfusion.hpp over the C ABI) builds, links and, on a GPU,
drives the same frames to the same poses as the Python binding."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "oglfusionkinectv2_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "frame_loop.cpp")


def build_frame_loop(tmp_path):
    exe = str(tmp_path / "frame_loop")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", PKG, "-lkf", "-Wl,-rpath," + PKG, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_host_builds_and_links(tmp_path):
    exe = build_frame_loop(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_cpp_host_matches_python_binding(tmp_path):
    from oglfusionkinectv2_b200 import GFusion, synth
    exe = build_frame_loop(tmp_path)
    w = synth.plain_c1(8)
    frames = [w.frame(k) for k in range(8)]
    path = tmp_path / "frames.u16"
    np.stack(frames).astype(np.uint16).tofile(path)
    pose0 = w.poses[0].flatten(order="F")
    args = [exe, str(path), "8", "128", "1.5", "0.03"] + [repr(float(v)) for v in pose0]
    r = subprocess.run(args, capture_output=True, text=True, check=True)
    lines = r.stdout.strip().splitlines()
    cpp = [np.array(l.split()[1:], float).reshape(4, 4, order="F") for l in lines[:8]]
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    for k in range(8):
        g.frameStep(frames[k])
        np.testing.assert_array_equal(g.getPose(), cpp[k])
    assert lines[8].startswith("triangles ") and int(lines[8].split()[1]) > 0
