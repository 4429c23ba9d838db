"""The FP64 direct sum (KHRR_FP64): the reference's own precision behind the
state API, and the comparator of the FP32 path's precision contract.

  * forces and potentials equal the FP64 oracle and the reference's own FP64
    kernel (the _ref-generated fixture) to relative RMS 1e-12 (the FP64 kernel
    takes r^-1 from rsqrt, the reference from sqrt and a division: the sums
    differ in the last bits only);
  * time steps follow the reference's 10-step corrected trajectory
    (max |dx| <= 1e-12) and the oracle's 20-step run with its energy;
  * batched systems, ragged sizes (ghosts) and per-body softenings;
  * the BASELINE configuration's small galaxy (16,384 stars + 32,768 DM,
    dt 0.002, 100 steps): the FP32 pair kernel's trajectory stays within
    max |dx| <= 1e-6 of the FP64 run's (measured 6e-8), and its relative
    energy drift is within 1.1 times the FP64 run's (the precision contract;
    measured 1.001), L_z to 1e-9.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PAIR = (128, 8, 128)


def rel_rms(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


@pytest.fixture(scope="module")
def ctx(libkhrr):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    c = khrr.Context(0)
    yield c
    c.close()


def galaxy(ns, nd, seed, eps_d=0.004):
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(ns, nd, seed, eps_dm=eps_d).arrays()
    return pos, vel, mass, eps * eps


def test_fp64_forces_match_reference_fixture(ctx, golden):
    import khrr
    g = golden("forces_n1536.npz")
    vel = np.zeros_like(g["pos"])
    ctx.upload(g["pos"], vel, g["mass"], g["eps2"])
    ctx.forces(khrr.ACC | khrr.PHI | khrr.FP64)
    out = ctx.download()
    assert rel_rms(out["acc"], g["acc_f64"]) <= 1e-12
    assert rel_rms(out["phi"], g["phi"]) <= 1e-12


@pytest.mark.parametrize("n_s,n_d,eps_d", [(1024, 2048, 0.004), (1000, 2001, 0.006), (130, 0, 0.004)])
def test_fp64_forces_match_oracle(ctx, oracle, n_s, n_d, eps_d):
    import khrr
    pos, vel, mass, eps2 = galaxy(n_s, n_d, seed=61, eps_d=eps_d)
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PHI | khrr.FP64)
    out = ctx.download()
    assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= 1e-12
    assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= 1e-12


def test_fp64_batched_systems(ctx, oracle):
    import khrr
    parts = [galaxy(200, 500, seed=62), galaxy(1024, 2048, seed=63), galaxy(700, 1500, seed=64, eps_d=0.008)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    ctx.upload(pos, vel, mass, eps2, offsets=off)
    ctx.forces(khrr.ACC | khrr.PHI | khrr.FP64)
    out = ctx.download()
    for k, (ps, vs, ms, es) in enumerate(parts):
        s = slice(off[k], off[k + 1])
        assert rel_rms(out["acc"][s], oracle.accel_f64(ps, ms, es)) <= 1e-12
        assert rel_rms(out["phi"][s], oracle.phi_f64(ps, ms, es)) <= 1e-12


def test_fp64_steps_follow_the_reference_trajectory(ctx, golden):
    import khrr
    g = golden("steps_n1024.npz")
    ctx.upload(g["pos"], g["vel"], g["mass"], g["eps2"])
    ctx.forces(khrr.ACC | khrr.FP64)
    ctx.step(float(g["dt"]), int(g["nsteps"]), khrr.FP64)
    out = ctx.download()
    assert np.abs(out["pos"].reshape(-1) - g["corrected_pos"]).max() <= 1e-12
    assert np.abs(out["vel"].reshape(-1) - g["corrected_vel"]).max() <= 1e-10
    assert rel_rms(out["acc"], g["corrected_acc"]) <= 1e-12


def test_fp64_steps_and_energy_match_oracle(ctx, oracle):
    import khrr
    pos, vel, mass, eps2 = galaxy(1024, 2048, seed=65)
    dt, nsteps = 0.002, 20
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.FP64)
    ctx.step(dt, nsteps, khrr.PHI | khrr.FP64)
    e1 = ctx.conservation()
    out = ctx.download()
    p_or, v_or, _, _ = oracle.run_steps(pos, vel, mass, eps2, dt, nsteps)
    assert np.abs(out["pos"] - p_or).max() <= 1e-11
    c1 = oracle.conservation(p_or, v_or, mass, oracle.phi_f64(p_or, mass, eps2))
    assert abs(e1["E"] / c1["E"] - 1.0) <= 1e-11


def test_fp64_flag_validation(ctx):
    import khrr
    pos, vel, mass, eps2 = galaxy(128, 128, seed=66)
    ctx.upload(pos, vel, mass, eps2)
    with pytest.raises(khrr.KhrrError):
        ctx.forces(khrr.ACC | khrr.FP64 | khrr.PLAIN)
    with pytest.raises(khrr.KhrrError):
        ctx.step(0.002, 1, khrr.FP64 | khrr.PLAIN)


def run(ctx, pos, vel, mass, eps2, dt, nsteps, flags, every=10):
    """nsteps steps from the uploaded state with E and L_z every `every` steps."""
    import khrr
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PHI | (flags & khrr.FP64))
    log = [ctx.conservation()]
    for _ in range(nsteps // every):
        ctx.step(dt, every, flags | khrr.PHI)
        log.append(ctx.conservation())
    return ctx.download(), log


def test_small_galaxy_precision_contract(ctx):
    """16,384 stars + 32,768 DM (the configuration run on the reference's CPU
    and on the GPU), 100 steps at dt 0.002: the FP32 pair kernel against the
    FP64 direct sum from the same initial state."""
    import khrr
    pos, vel, mass, eps2 = galaxy(16384, 32768, seed=1000)
    dt, nsteps = 0.002, 100
    ref, log64 = run(ctx, pos, vel, mass, eps2, dt, nsteps, khrr.FP64)
    ctx.set_tuning(*PAIR, 0, 2)
    try:
        got, log32 = run(ctx, pos, vel, mass, eps2, dt, nsteps, 0)
    finally:
        ctx.set_tuning()
    assert np.abs(got["pos"] - ref["pos"]).max() <= 1e-6
    d64 = abs(log64[-1]["E"] / log64[0]["E"] - 1.0)
    d32 = abs(log32[-1]["E"] / log32[0]["E"] - 1.0)
    assert d64 > 0.0
    assert d32 <= 1.1 * d64, (d32, d64)
    assert abs(log32[-1]["Lz"] / log64[-1]["Lz"] - 1.0) <= 1e-9


def test_fp64_symmetric_and_one_sided_forms_agree(ctx, monkeypatch):
    """The symmetric FP64 pass (default: each unordered pair once, FP64
    atomics) and the one-sided one (KHRR_FP64_ONESIDED=1, every ordered pair,
    the reference's loop) give the same forces and potentials to FP64
    rounding, over several 1024-body blocks, ragged systems (ghosts, short
    last blocks) and per-body softenings, and the same 5-step trajectory."""
    import khrr
    parts = [galaxy(3000, 6001, seed=65, eps_d=0.006), galaxy(128, 0, seed=66), galaxy(1500, 2600, seed=67)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("KHRR_FP64_ONESIDED", mode)
        ctx.upload(pos, vel, mass, eps2, offsets=off)
        ctx.forces(khrr.ACC | khrr.PHI | khrr.FP64)
        f = ctx.download()
        ctx.step(0.002, 5, khrr.FP64)
        out[mode] = (f, ctx.download())
    (f0, s0), (f1, s1) = out["0"], out["1"]
    assert rel_rms(f0["acc"], f1["acc"]) <= 1e-13
    assert rel_rms(f0["phi"], f1["phi"]) <= 1e-13
    assert np.abs(s0["pos"] - s1["pos"]).max() <= 1e-12
