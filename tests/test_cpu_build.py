"""The incremental build's staleness rule (jax_alfa_b200/build.py): an object
is rebuilt when it is missing, when its recorded nvcc command line differs,
or when a file nvcc listed as its dependency is newer than it."""
import os
import time

from jax_alfa_b200 import build


def _touch(path, t):
    with open(path, "a"):
        pass
    os.utime(path, (t, t))


def test_object_is_stale_only_when_a_listed_dependency_is_newer(tmp_path):
    src, hdr, other = tmp_path / "unit.cu", tmp_path / "unit.cuh", tmp_path / "unrelated.cuh"
    obj = tmp_path / "unit.o"
    now = time.time()
    for p in (src, hdr, other):
        _touch(p, now - 100)
    _touch(obj, now - 50)
    cmd = ["nvcc", "-c", str(src), "-o", str(obj)]
    (tmp_path / "unit.o.cmd").write_text(" ".join(cmd))
    (tmp_path / "unit.o.d").write_text(f"{obj} : {src} \\\n    {hdr}\n")
    assert not build._unit_stale("unit.cu", str(obj), cmd)
    _touch(other, now)  # not a dependency of this object
    assert not build._unit_stale("unit.cu", str(obj), cmd)
    _touch(hdr, now)  # a listed header changed
    assert build._unit_stale("unit.cu", str(obj), cmd)


def test_object_is_stale_when_its_command_line_changes(tmp_path):
    src, obj = tmp_path / "unit.cu", tmp_path / "unit.o"
    now = time.time()
    _touch(src, now - 100)
    _touch(obj, now - 50)
    cmd = ["nvcc", "-O3", "-c", str(src), "-o", str(obj)]
    (tmp_path / "unit.o.cmd").write_text(" ".join(cmd))
    (tmp_path / "unit.o.d").write_text(f"{obj} : {src}\n")
    assert not build._unit_stale("unit.cu", str(obj), cmd)
    assert build._unit_stale("unit.cu", str(obj), cmd + ["-DALFA_BUILD_FP32"])
    assert build._unit_stale("unit.cu", str(tmp_path / "missing.o"), cmd)


def test_every_engine_source_builds_in_both_precisions():
    units = {(s, tuple(x), suf) for s, x, suf in build.UNITS}
    for s in build.ENGINE:
        assert (s, (), "") in units and (s, ("-DALFA_BUILD_FP32",), "_f32") in units
    for s in build.ONCE:
        assert (s, (), "") in units
    assert all(os.path.exists(os.path.join(build.CSRC, s)) for s in build.SOURCES)
