"""The resident 128^3 stencil's brick geometry, checked on the CPU: the row
map of a brick's warps, the tiling of the mesh, the staged halo rows and the
neighbour counters the kernel waits on (tests/wave_bricks_check.cpp includes
khrr-nbody_b200/csrc/wave_bricks.h, the header the kernel is built from; no
device work)."""
import subprocess

from conftest import PKG, ROOT


def test_wave_brick_geometry(tmp_path):
    exe = tmp_path / "wave_bricks_check"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(PKG / "csrc"),
                        str(ROOT / "tests" / "wave_bricks_check.cpp"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
