"""include/vlsgViennaLS.hpp (viennals::Domain <-> vlsg::LevelSet) compiled
against stand-ins with the reference's call signatures (tests/cpp/
viennals_stub): a 3D sphere and a 2D circle go through toVlsg and fromVlsg
unchanged (points in HRLE order, values, width, a point-data array), and on
a GPU a Domain advanced through vlsg::Advect comes back with the points and
values the C ABI gives for the same step, its point data gathered by the
source ids."""
import os
import subprocess

import numpy as np
import pytest

from parity_cases import params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "domain_convert.cpp")
STUB = os.path.join(ROOT, "tests", "cpp", "viennals_stub")
LIBDIR = os.path.join(ROOT, "viennals_b200")


def _build(out):
    from viennals_b200 import _lib

    _lib.load()
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I",
                           os.path.join(ROOT, "include"), "-I", STUB, SRC, "-L", LIBDIR, "-lvlsgpu",
                           f"-Wl,-rpath,{LIBDIR}", "-o", out])


def _write(path, grid, dom, rate=1.0):
    d = grid.dim
    with open(path, "wb") as f:
        np.array([d], np.int32).tofile(f)
        np.array(grid.min[:d], np.int64).tofile(f)
        np.array(grid.max[:d], np.int64).tofile(f)
        np.array(grid.bc[:d], np.int32).tofile(f)
        np.array([grid.delta, rate], np.float64).tofile(f)
        idx = np.asarray(dom.idx, np.int32)
        rs = np.asarray(dom.run_start, np.int32)
        if d == 2:
            idx = np.concatenate([idx, np.zeros((len(idx), 1), np.int32)], 1)
            rs = np.concatenate([rs, np.zeros((len(rs), 1), np.int32)], 1)
        np.array([len(dom.values)], np.int64).tofile(f)
        np.ascontiguousarray(idx).tofile(f)
        np.ascontiguousarray(dom.values, np.float64).tofile(f)
        np.array([len(dom.run_sign)], np.int64).tofile(f)
        np.ascontiguousarray(rs).tofile(f)
        np.ascontiguousarray(dom.run_sign, np.int8).tofile(f)
        np.array([dom.width], np.int32).tofile(f)


def _read(path):
    buf = open(path, "rb").read()
    n = int(np.frombuffer(buf, np.int64, 1, 0)[0])
    off = 8
    idx = np.frombuffer(buf, np.int32, 3 * n, off).reshape(n, 3)
    off += 12 * n
    val = np.frombuffer(buf, np.float64, n, off)
    off += 8 * n
    w = int(np.frombuffer(buf, np.int32, 1, off)[0])
    off += 4
    ids = np.frombuffer(buf, np.float64, n, off)
    off += 8 * n
    seg = int(np.frombuffer(buf, np.int32, 1, off)[0])
    return idx, val, w, ids, seg


def _cases():
    from viennals_b200 import BoundaryConditionEnum as BC, Grid
    from viennals_b200.geometry import make_circle, make_sphere

    g3 = Grid([-3, 3, -3, 3, -3, 3], [BC.INFINITE_BOUNDARY] * 3, 0.25)
    g2 = Grid([-20, 20, -20, 20], [BC.REFLECTIVE_BOUNDARY] * 2, 0.5, dim=2)
    return [(g3, make_sphere(g3, [0.1, 0.0, -0.2], 1.7)), (g2, make_circle(g2, [5.0, 0.0], 7.3))]


@pytest.mark.parametrize("case", [0, 1], ids=["3D sphere", "2D circle"])
def test_round_trip(tmp_path, case):
    grid, dom = _cases()[case]
    exe = str(tmp_path / "domain_convert")
    _build(exe)
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write(src, grid, dom)
    subprocess.check_call([exe, src, dst, "roundtrip"])
    idx, val, w, ids, seg = _read(dst)
    assert np.array_equal(idx[:, :grid.dim], dom.idx)
    assert np.array_equal(val.view(np.int64), np.asarray(dom.values).view(np.int64))
    assert w == dom.width and seg == 1
    assert np.array_equal(ids, np.arange(len(dom.values), dtype=np.float64))


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1], ids=["3D sphere", "2D circle"])
def test_advect_through_domain_conversions(tmp_path, case):
    from viennals_b200.advect import Context
    from viennals_b200.velocity import constant_scalar

    grid, dom = _cases()[case]
    exe = str(tmp_path / "domain_convert")
    _build(exe)
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write(src, grid, dom, rate=1.0)
    subprocess.check_call([exe, src, dst, "advect", "1"])
    idx, val, w, ids, _ = _read(dst)
    ctx = Context(0, 0)
    ctx.set_grid(grid)
    ctx.set_level_set_count(1)
    ctx.upload(0, dom)
    ctx.set_velocity(constant_scalar(1.0).descriptor())
    scheme = 2 if grid.dim == 2 else 0  # LAX_FRIEDRICHS_1ST_ORDER / ENGQUIST_OSHER_1ST_ORDER
    ctx.advect(params(scheme, 0, 0.0, track_point_data=1, update_point_data=1))
    gi, gv, gw = ctx.download(0)
    src_ids, _, _ = ctx.download_point_data(0)
    ctx.close()
    assert np.array_equal(idx[:, :grid.dim], gi)
    assert np.array_equal(val.view(np.int64), gv.view(np.int64))
    assert w == gw
    assert np.array_equal(ids, np.where(src_ids >= 0, src_ids, 0).astype(np.float64))


def test_header_instantiates_for_float_and_both_dimensions(tmp_path):
    # toVlsg / fromVlsg for Domain<float, 2>, Domain<float, 3> and Domain<double, 2>
    # (Advect<float, D> callers) compile against the stand-ins too
    src = tmp_path / "inst.cpp"
    src.write_text(
        '#include "vlsgViennaLS.hpp"\n'
        "template <class T, int D> int roundTrip() {\n"
        "  viennals::Domain<T, D> a, b;\n"
        "  typename viennals::Domain<T, D>::DomainType::Entry e;\n"
        "  for (int k = 0; k < D; ++k) e.start[k] = k;\n"
        "  e.value = T(0.25);\n"
        "  e.defined = true;\n"
        "  a.domain.entries.push_back(e);\n"
        "  vlsg::LevelSet ls = vlsg::toVlsg(a);\n"
        "  vlsg::fromVlsg(ls, b);\n"
        "  return ls.grid.dim == D && b.getDomain().getNumberOfPoints() == 1 ? 0 : 1;\n"
        "}\n"
        "int main() { return roundTrip<float, 2>() + roundTrip<float, 3>() + roundTrip<double, 2>(); }\n")
    exe = str(tmp_path / "inst")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                           os.path.join(ROOT, "include"), "-I", STUB, str(src), "-L", LIBDIR,
                           "-lvlsgpu", f"-Wl,-rpath,{LIBDIR}", "-o", exe])
    assert subprocess.call([exe]) == 0
