"""The symmetric pair kernel's work plan, checked on the CPU: every ordered
pair of 128-body tiles of a system evaluated exactly once (none across
systems), sums accumulated for every real body and for no ghost, and
(equal-mass runs) every block of one mass, at most 1024 bodies
(tests/pair_plan_check.cpp replays the items against plan_pair_items in
libkhrr.so; no device work)."""
import os
import subprocess

import pytest

from conftest import PKG, ROOT

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def checker(libkhrr, tmp_path_factory):
    exe = tmp_path_factory.mktemp("plan") / "pair_plan_check"
    build = PKG / "build"
    cmd = ["g++", "-std=c++20", "-O2", "-I", str(ROOT / "include"), "-I", str(PKG / "csrc"),
           "-I", f"{CUDA}/include", str(ROOT / "tests" / "pair_plan_check.cpp"), "-o", str(exe),
           "-L", str(build), "-lkhrr", f"-Wl,-rpath,{build}", "-L", f"{CUDA}/lib64", "-lcudart",
           f"-Wl,-rpath,{CUDA}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


LAYOUTS = [
    ("the 786k galaxy, 444 CTAs, automatic chunks", "fixed", 444, 0, [786432]),
    ("131k, automatic chunks (1 block per item)", "fixed", 444, 0, [131072]),
    ("131k, chunks of 5 blocks", "fixed", 444, 5, [131072]),
    ("131k, chunks of 32 blocks", "fixed", 16, 0, [131072]),
    ("ragged sizes: ghosts, short last blocks", "fixed", 444, 3, [1000, 2000, 77, 1, 3000, 1025]),
    ("single bodies and single blocks", "fixed", 444, 0, [1, 1024, 128, 129]),
    ("an uneven ensemble", "fixed", 444, 0, [4096, 121856, 86016, 11264, 1024 * 37 + 512, 9000]),
    ("equal-mass runs: the 786k galaxy", "mass", 444, 0, [786432]),
    ("equal-mass runs: components off the 1024 grid", "mass", 444, 0, [62464, 27648, 9216, 13824, 1536]),
    ("equal-mass runs, chunks of 3", "mass", 444, 3, [62464, 4096, 128 * 41]),
]


@pytest.mark.parametrize("label,blocks,ctas,chunk,sizes", LAYOUTS, ids=[x[0] for x in LAYOUTS])
def test_pair_plan_covers_every_pair_once(checker, label, blocks, ctas, chunk, sizes):
    r = subprocess.run([str(checker), blocks, str(ctas), str(chunk)] + [str(n) for n in sizes],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
