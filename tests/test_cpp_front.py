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


BATCH_SRC = os.path.join(ROOT, "tests", "cpp", "front_batch.cpp")


def build_batch_front(out):
    from viennals_b200 import _lib

    _lib.load()
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           BATCH_SRC, "-L", LIBDIR, "-lvlsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", out])


def test_cpp_batch_front_compiles(tmp_path):
    build_batch_front(str(tmp_path / "front_batch"))
    assert os.path.exists(tmp_path / "front_batch")


@pytest.mark.gpu
def test_cpp_batch_front_matches_batch_context(tmp_path):
    """vlsg::AdvectBatch (C++) over 5 domains, two steps, against the Python
    batch context: the same points, bit-identical values, the same runs and
    advected times; the second apply finds the domains resident."""
    from parity_cases import params
    from viennals_b200.advect import BatchContext
    from viennals_b200.synth import batch_domains

    items = batch_domains(5, seed=13, points_range=(2e3, 2e4))
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(src, "wb") as f:
        np.array([len(items)], np.int32).tofile(f)
        for grid, dom, vel in items:
            np.array(grid.min, np.int64).tofile(f)
            np.array(grid.max, np.int64).tofile(f)
            np.array(grid.bc, np.int32).tofile(f)
            np.array([grid.delta, vel.descriptor().rate[0]], np.float64).tofile(f)
            np.array([len(dom.values)], np.int64).tofile(f)
            np.ascontiguousarray(dom.idx, np.int32).tofile(f)
            np.ascontiguousarray(dom.values, np.float64).tofile(f)
            np.array([len(dom.run_sign)], np.int64).tofile(f)
            np.ascontiguousarray(dom.run_start, np.int32).tofile(f)
            np.ascontiguousarray(dom.run_sign, np.int8).tofile(f)
            np.array([dom.width], np.int32).tofile(f)
    exe = str(tmp_path / "front_batch")
    build_batch_front(exe)
    out = subprocess.check_output([exe, src, dst, "2"], text=True)
    assert "skipped 1" in out
    b = BatchContext(0, 1)
    b.set_domains(items)
    p = params(7, 1, 0.0)
    times = np.zeros(len(items))
    for _ in range(2):
        times += [r.advected_time for r in b.advect(p)]
    with open(dst, "rb") as f:
        buf = f.read()
    off = 4
    for d in range(len(items)):
        ref = b.download_domain(d)
        n = int(np.frombuffer(buf, np.int64, 1, off)[0]); off += 8
        idx = np.frombuffer(buf, np.int32, 3 * n, off).reshape(n, 3); off += 12 * n
        val = np.frombuffer(buf, np.float64, n, off); off += 8 * n
        m = int(np.frombuffer(buf, np.int64, 1, off)[0]); off += 8
        rs = np.frombuffer(buf, np.int32, 3 * m, off).reshape(m, 3); off += 12 * m
        sg = np.frombuffer(buf, np.int8, m, off); off += m
        w = int(np.frombuffer(buf, np.int32, 1, off)[0]); off += 4
        t = float(np.frombuffer(buf, np.float64, 1, off)[0]); off += 8
        assert np.array_equal(idx, ref.idx) and np.array_equal(val.view(np.int64), ref.values.view(np.int64))
        assert np.array_equal(rs, ref.run_start) and np.array_equal(sg, ref.run_sign)
        assert w == ref.width and t == times[d]
    b.close()
