"""The header-only C++ front (include/vlsgAdvect.hpp) compiles against the
C ABI, and on a GPU gives the same result as the Python front."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "front_sphere.cpp")
LIBDIR = os.path.join(ROOT, "viennals_b200")


def build_front(out):
    from viennals_b200 import _lib

    _lib.load()  # make sure libvlsgpu.so is built
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
                           "-L", LIBDIR, "-lvlsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out])


def test_cpp_front_compiles(tmp_path):
    build_front(str(tmp_path / "front_sphere"))
    assert os.path.exists(tmp_path / "front_sphere")


@pytest.mark.gpu
def test_cpp_front_matches_python_front(tmp_path):
    exe = str(tmp_path / "front_sphere")
    build_front(exe)
    out = subprocess.check_output([exe, "2.0"], text=True).split()
    vals = dict(zip(out[0::2], out[1::2]))
    from parity_cases import sphere_growth_eo1, run_gpu

    g, lss, v, p = sphere_growth_eo1()
    ctx, res = run_gpu(g, lss, v, p)
    idx, val, w = ctx.download(0)
    s = float(np.sum(val * (1.0 + 1e-3 * (idx[:, 0] + 7 * idx[:, 1] + 13 * idx[:, 2]))))
    assert int(vals["steps"]) == res.number_of_time_steps
    assert float(vals["time"]) == res.advected_time
    assert int(vals["points"]) == len(val)
    assert int(vals["width"]) == w
    assert abs(float(vals["checksum"]) - s) <= 1e-9 * abs(s)


@pytest.mark.gpu
def test_cpp_front_host_velocity_field(tmp_path):
    """The same run with the velocity as a C++ VelocityField (host callback)."""
    exe = str(tmp_path / "front_sphere")
    build_front(exe)
    a = subprocess.check_output([exe, "2.0"], text=True)
    b = subprocess.check_output([exe, "2.0", "callback"], text=True)
    assert a == b


@pytest.mark.gpu
def test_cpp_front_keeps_level_sets_resident(tmp_path):
    """Five single-step applies through the C++ front: the first uploads, the
    next four find the device copy current (version stamps) and skip the
    upload; the results equal five single steps of a context.  A touch()ed
    level set is uploaded again."""
    exe = str(tmp_path / "front_sphere")
    build_front(exe)
    out = subprocess.check_output([exe, "5", "loop"], text=True).split()
    vals = dict(zip(out[0::2], out[1::2]))
    assert int(vals["skipped"]) == 4
    assert int(vals["after_touch"]) == 4  # the touched object was uploaded
