"""The reference-compatible program khrr_nbody end to end on a small
two-galaxy encounter (analytic halo on): output files and their layouts, the
trajectory against the same run through the Python API, and a restart from
the it = 10 snapshots that continues the same trajectory (max |dx| <= 1e-12)."""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu

DRIVER = PKG / "build" / "khrr_nbody"


def write_inputs(d: pathlib.Path, i_cont: int, tmax: float):
    import khrr
    from khrr.galaxy import make_galaxy
    ini = d / "ini"
    ini.mkdir(parents=True, exist_ok=True)
    L = khrr.lib()
    for k, seed in enumerate((41, 42)):
        g = make_galaxy(512, 1024, seed)
        for comp, (p, v) in (("S", (g.star_pos, g.star_vel)), ("DM", (g.dm_pos, g.dm_vel))):
            L.khrr_write_start_txt(str(ini / f"start_{comp}{k}.txt").encode(), len(p),
                                   np.ascontiguousarray(p).ctypes.data, np.ascontiguousarray(v).ctypes.data, 0.0)
    (ini / "__start_galaxies.ini").write_text(
        "2\t--- M_glx\n0\t--- k_glx\n512,1024\t--- N\n1.0,6.699356\t--- M\n0.004,0.004\t--- eps\n0.0\t--- alpha\n"
        "1.5,0.0,0.0\t--- X\n-0.3,0.1,0.0\t--- V\n"
        "1\t--- k_glx\n512,1024\t--- N\n1.0,6.699356\t--- M\n0.004,0.004\t--- eps\n30.0\t--- alpha\n"
        "-1.5,0.0,0.0\t--- X\n0.3,-0.1,0.0\t--- V\n")
    (ini / "__gr_par.ini").write_text(
        "1.0 \t--- Mh\n0.3333 \t--- a\n1.0000 \t--- Rh\n0.0 \t--- Mb\n0.0431 \t--- b\n0.2000 \t--- Rb\n"
        "0.004 \t--- eps\n0.002 \t--- dtgrav\n3.720 \t--- K_m\n0.900 \t--- K_r\n")
    (ini / "__GPUs.ini").write_text("1\t--- nGPU\n0\t--- deviceId[0]\n")
    (ini / "__start_nbody.ini").write_text(f"{i_cont} \t--- i_cont\n{tmax} \t--- tmax\n0.010 \t--- dt_save\n")


def run_driver(d, kernel="one-sided"):
    # the API runs below use the library's default (one-sided) kernel, so the
    # driver is pinned to it for the bit-for-bit comparisons
    r = subprocess.run([str(DRIVER), "--data", str(d), "--quiet", "--mesh-nx", "32", "--mesh-dx", "0.25",
                        "--kernel", kernel], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def read_snapshot(path, n):
    raw = path.read_bytes()
    cnt = np.frombuffer(raw[:4], "<i4")[0]
    t = np.frombuffer(raw[4:12], "<f8")[0]
    rec = np.frombuffer(raw[12:], "<f8").reshape(cnt, 6)
    assert cnt == n
    return t, rec[:, :3], rec[:, 3:]


def api_run(d, nsteps, flags=0):
    """The same simulation through the Python API (flags: KHRR_FP64 or 0)."""
    import khrr
    from test_io import Galaxy
    L = khrr.lib()
    gals = (Galaxy * 4)()
    cnt = C.c_int()
    assert L.khrr_read_galaxies_ini(str(d / "ini" / "__start_galaxies.ini").encode(), gals, 4, C.byref(cnt)) == 0
    nmax = 4000
    pos, vel, mass, eps2 = np.zeros((nmax, 3)), np.zeros((nmax, 3)), np.zeros(nmax), np.zeros(nmax)
    n, ns = C.c_int64(), C.c_int64()
    assert L.khrr_load_initial_conditions(str(d / "ini").encode(), gals, cnt.value, nmax, pos.ctypes.data,
                                          vel.ctypes.data, mass.ctypes.data, eps2.ctypes.data, C.byref(n),
                                          C.byref(ns)) == 0
    n = n.value
    ctx = khrr.Context(0)
    try:
        ctx.set_external_field(Mh=1.0, a=0.3333, Rh=1.0, Mb=0.0, b=0.0431, Rb=0.2)
        ctx.upload(pos[:n], vel[:n], mass[:n], eps2[:n])
        ctx.forces(khrr.ACC | khrr.PHI | flags)
        e0 = ctx.conservation()
        ctx.step(0.002, nsteps, flags)
        return n, ns.value, ctx.download(), e0
    finally:
        ctx.close()


def test_driver_run_outputs_and_restart(libkhrr, tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    assert DRIVER.exists(), "build khrr-nbody_b200 first"
    d = tmp_path / "nbody"
    write_inputs(d, 0, 0.1)
    run_driver(d)
    out, bins = d / "out", d / "bin"

    # Conservation logs: header + t = 0 + one row per save (10 saves).
    for name, header in (("E(t).csv", "it, t, E, E_rel_err, E_rel_err_magnitude, Ek, Ep"),
                         ("Lz(t).csv", "it, t, Lz, Lz_rel_err, Lz_rel_err_magnitude"),
                         ("LL(t).csv", "it, t, LL, LL_rel_err, LL_rel_err_magnitude"),
                         ("Imp(t).csv", "it, t, Imp, Imp_abs_err, Imp_rel_err, Imp_rel_err_magnitude")):
        lines = (out / name).read_text().splitlines()
        assert lines[0] == header and len(lines) == 12, name
    e_rows = [l.split(", ") for l in (out / "E(t).csv").read_text().splitlines()[1:]]
    assert [int(r[0]) for r in e_rows] == [0] + [5 * k for k in range(1, 11)]
    assert e_rows[0][1] == "0" and e_rows[0][3] == "0"
    for name in ("E(t).dat", "imp(t).dat", "LL(t).dat", "Lz(t).dat"):
        assert len((out / name).read_text().splitlines()) == 11
    assert len((out / "sample.csv").read_text().splitlines()) == 11
    assert len((out / "time_frame.dat").read_text().splitlines()) == 10
    phi_files = sorted((out / "phi").glob("phi_*.csv"))
    assert len(phi_files) == 10 and len(phi_files[0].read_text().splitlines()) == 33
    assert (bins / "LIE_0.bin").stat().st_size == 72

    # Trajectory equals the same run through the API (50 steps to t = 0.1).
    n, ns, state, e0 = api_run(d, 50)
    t, ps, vs = read_snapshot(bins / "S_   10.bin", ns)
    _, pd, vd = read_snapshot(bins / "DM_   10.bin", n - ns)
    assert abs(t - 0.1) < 1e-12
    assert np.abs(np.concatenate([ps, pd]) - state["pos"]).max() <= 1e-12
    assert np.abs(np.concatenate([vs, vd]) - state["vel"]).max() <= 1e-12
    assert float(e_rows[0][2]) == pytest.approx(e0["E"], rel=1e-14, abs=1e-15)

    # Restart from the it = 10 snapshots and continue to t = 0.2.
    write_inputs(d, 10, 0.2)
    run_driver(d)
    lines = (out / "E(t).csv").read_text().splitlines()
    assert len(lines) == 22  # appended, no new header
    _, _, state2, _ = api_run(d, 100)
    t2, ps2, vs2 = read_snapshot(bins / "S_   20.bin", ns)
    _, pd2, _ = read_snapshot(bins / "DM_   20.bin", n - ns)
    assert abs(t2 - 0.2) < 1e-12
    assert np.abs(np.concatenate([ps2, pd2]) - state2["pos"]).max() <= 1e-12


@pytest.mark.parametrize("kernel", ["pair", "auto"])
def test_driver_kernel_choice(libkhrr, tmp_path, kernel):
    """--kernel pair (the symmetric kernel) and auto (the autotuner) follow
    the one-sided trajectory over the same 50 steps.  The kernels sum each
    body's terms in different orders (both within 1e-6 of FP64 per force
    evaluation), and close encounters amplify those differences along the
    trajectory: max |dx| <= 1e-5 here (measured 1.2e-6), between the
    suite's 1e-7 after 10 steps and 1e-4 after 100 steps."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = tmp_path / "nbody"
    write_inputs(d, 0, 0.1)
    run_driver(d, kernel)
    n, ns, state, _ = api_run(d, 50)
    _, ps, _ = read_snapshot(d / "bin" / "S_   10.bin", ns)
    _, pd, _ = read_snapshot(d / "bin" / "DM_   10.bin", n - ns)
    assert np.abs(np.concatenate([ps, pd]) - state["pos"]).max() <= 1e-5


def test_driver_fp64_kernel(libkhrr, tmp_path):
    """--kernel fp64: the reference's own precision through the driver; its
    snapshot equals the API run with KHRR_FP64 (the same calls), and differs
    from the FP32 one-sided run by the FP32 rounding only."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    d = tmp_path / "nbody"
    write_inputs(d, 0, 0.1)
    run_driver(d, "fp64")
    n, ns, state, _ = api_run(d, 50, khrr.FP64)
    _, ps, _ = read_snapshot(d / "bin" / "S_   10.bin", ns)
    _, pd, _ = read_snapshot(d / "bin" / "DM_   10.bin", n - ns)
    assert np.abs(np.concatenate([ps, pd]) - state["pos"]).max() <= 1e-12
    _, _, state32, _ = api_run(d, 50)
    assert np.abs(state32["pos"] - state["pos"]).max() <= 1e-5


def test_driver_wave_mode(libkhrr, tmp_path):
    """--wave: the reference's Wave solver; the trajectory equals the API
    run with the same mesh solver, and the phi/ cuts show the wave field from
    the setup (frame 0) on."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    d = tmp_path / "nbody"
    write_inputs(d, 0, 0.02)
    r = subprocess.run([str(DRIVER), "--data", str(d), "--quiet", "--mesh-nx", "32", "--mesh-dx", "0.25", "--wave",
                        "--wave-setup", "300"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    iters = int(0.002 / (0.5 * 0.25 / (4574.337022617616 * np.sqrt(3.0))))
    assert f"Wave eq iterations: {iters}" in r.stdout
    out, bins = d / "out", d / "bin"
    phi_files = sorted((out / "phi").glob("phi_*.csv"))
    assert len(phi_files) == 3 and (out / "phi" / "phi_    0.csv").exists()
    assert len((out / "E(t).csv").read_text().splitlines()) == 4
    # the same run through the API
    from test_io import Galaxy
    L = khrr.lib()
    gals = (Galaxy * 4)()
    cnt = C.c_int()
    assert L.khrr_read_galaxies_ini(str(d / "ini" / "__start_galaxies.ini").encode(), gals, 4, C.byref(cnt)) == 0
    nmax = 4000
    pos, vel, mass, eps2 = np.zeros((nmax, 3)), np.zeros((nmax, 3)), np.zeros(nmax), np.zeros(nmax)
    n, ns = C.c_int64(), C.c_int64()
    assert L.khrr_load_initial_conditions(str(d / "ini").encode(), gals, cnt.value, nmax, pos.ctypes.data,
                                          vel.ctypes.data, mass.ctypes.data, eps2.ctypes.data, C.byref(n),
                                          C.byref(ns)) == 0
    n = n.value
    ctx = khrr.Context(0)
    try:
        ctx.set_external_field(Mh=1.0, a=0.3333, Rh=1.0, Mb=0.0, b=0.0431, Rb=0.2)
        ctx.upload(pos[:n], vel[:n], mass[:n], eps2[:n])
        ctx.set_mesh_solver(khrr.WaveParams.make(32, 0.25), assign=khrr.ASSIGN_NGP, fp64=True,
                            iters_per_step=iters, setup_iters=300)
        ctx.forces(khrr.ACC | khrr.PHI | khrr.MESH)
        ctx.step(0.002, 10, khrr.MESH | khrr.PHI)
        st = ctx.download()
        field = ctx.mesh_solver_phi(32)
    finally:
        ctx.close()
    last = (out / "phi" / "phi_   10.csv").read_text().splitlines()[1:]
    cut = np.array([float(l.split(", ")[1]) for l in last])
    want = field.reshape(32, 32, 32)[16, 16, :]
    assert np.abs(cut - want).max() <= 1e-7 * max(1.0, np.abs(want).max())
    rows = [l.split(", ") for l in (out / "E(t).csv").read_text().splitlines()[1:]]
    assert int(rows[-1][0]) == 10
    # body 1 of sample.csv (6 significant digits) is the API run's body 1
    srow = (out / "sample.csv").read_text().splitlines()[-1].split(", ")
    assert abs(float(srow[5]) - st["pos"][1, 2]) <= 1e-5 * abs(st["pos"][1, 2]) + 1e-12
    # and the final snapshot-free state: phi of body 1 is the gathered field
    assert abs(float(srow[7]) - st["phi"][1]) <= 1e-5 * abs(st["phi"][1])
