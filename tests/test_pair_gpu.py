"""GPU parity of the symmetric pair kernel (tuning packed = 2) against the oracle.

The pair kernel evaluates each unordered pair once and applies it to both
bodies; its FP32 partials are added into 64-bit fixed-point sums per body
(integer atomics), so they must meet the same bounds as the one-sided kernel:
  * accelerations and potentials: relative RMS <= 1e-6 vs the FP64 oracle
    (SMALL_N_TOL = 2e-6 for the small generated systems, as in
    test_forces_gpu.py), whatever the mass and softening scales (the
    fixed-point scales follow them per 128-body tile);
  * every pass is bitwise reproducible (integer addition does not depend on
    the order in which partials arrive);
  * graph time steps follow the reference's golden trajectory as closely as
    the one-sided kernel does (max |dx| <= 1e-7 after 10 steps).
Layouts cover the block-mass form (component counts multiples of 1024), the
general form (ragged counts, ghosts, per-body masses), per-component
softening, several systems, forced chunk sizes and a system of 48 blocks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL_N_TOL = 2e-6
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


def galaxy(ns, nd, seed, eps_s=0.004, eps_d=0.004):
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(ns, nd, seed, eps_stars=eps_s, eps_dm=eps_d).arrays()
    return pos, vel, mass, eps * eps


def pair_forces(ctx, pos, vel, mass, eps2, flags, split=0, offsets=None):
    ctx.set_tuning(*PAIR, split, 2)
    try:
        ctx.upload(pos, vel, mass, eps2, offsets=offsets)
        ctx.forces(flags)
        return ctx.download()
    finally:
        ctx.set_tuning()


@pytest.mark.parametrize("split", [0, 1, 2, 5])
@pytest.mark.parametrize("eps_d", [0.004, 0.007])
def test_block_mass_galaxy(ctx, oracle, split, eps_d):
    """2048 stars + 4096 DM: whole 1024 blocks of one mass (the factored
    form), uniform or per-component softening, several chunk sizes."""
    import khrr
    pos, vel, mass, eps2 = galaxy(2048, 4096, seed=31, eps_d=eps_d)
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI, split)
    assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= 1e-6
    assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= 1e-6


@pytest.mark.parametrize("sizes", [[(1536, 2560)], [(640, 1408)], [(1536, 2560), (512, 1024), (2048, 4096)]])
def test_block_mass_with_short_blocks(ctx, oracle, sizes):
    """Component counts that are whole 128-body tiles but not whole 1024
    blocks: the blocks are runs of equal-mass tiles (some shorter than 1024),
    so the factored-mass form still applies; single and several systems."""
    import khrr
    parts = [galaxy(ns, nd, seed=44 + k) for k, (ns, nd) in enumerate(sizes)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI, offsets=off)
    for k, (ps, vs, ms, es) in enumerate(parts):
        s = slice(off[k], off[k + 1])
        assert rel_rms(out["acc"][s], oracle.accel_f64(ps, ms, es)) <= 1e-6
        assert rel_rms(out["phi"][s], oracle.phi_f64(ps, ms, es)) <= 1e-6


@pytest.mark.parametrize("n_s,n_d", [(1000, 2000), (130, 0), (1, 0), (1023, 1025), (3000, 77)])
def test_general_form_ragged_sizes(ctx, oracle, n_s, n_d):
    """Counts that are not multiples of 1024 (or 128): ghosts, a short last
    block, per-body masses."""
    import khrr
    pos, vel, mass, eps2 = galaxy(n_s, n_d, seed=32, eps_d=0.006)
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI)
    if len(mass) == 1:
        assert np.all(out["acc"] == 0.0)
        return
    assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= SMALL_N_TOL
    assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= SMALL_N_TOL


def test_random_masses(ctx, oracle):
    import khrr
    pos, vel, mass, eps2 = galaxy(2048, 2048, seed=33)
    rng = np.random.default_rng(33)
    mass = mass * rng.uniform(0.5, 1.5, size=mass.shape)
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI)
    assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= 1e-6
    assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= 1e-6


@pytest.mark.parametrize("flags_name", ["ACC", "PHI"])
def test_single_output_sets(ctx, oracle, flags_name):
    import khrr
    pos, vel, mass, eps2 = galaxy(1024, 3072, seed=34)
    out = pair_forces(ctx, pos, vel, mass, eps2, getattr(khrr, flags_name))
    if flags_name == "ACC":
        assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= 1e-6
    else:
        assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= 1e-6


def test_pair_passes_are_bitwise_reproducible(ctx):
    import khrr
    pos, vel, mass, eps2 = galaxy(2048, 4096, seed=35)
    ctx.set_tuning(*PAIR, 0, 2)
    try:
        ctx.upload(pos, vel, mass, eps2)
        ctx.forces(khrr.ACC | khrr.PHI)
        a = ctx.download()
        ctx.forces(khrr.ACC | khrr.PHI)
        b = ctx.download()
    finally:
        ctx.set_tuning()
    assert np.array_equal(a["acc"], b["acc"]) and np.array_equal(a["phi"], b["phi"])


@pytest.mark.parametrize("mass_scale,eps_s", [(1e-20, 0.004), (1e20, 0.004), (1.0, 1e-5), (3e-8, 2e-4)])
def test_fixed_point_scales(ctx, oracle, mass_scale, eps_s):
    """The fixed-point scales follow the system: masses in units 1e-20 and
    1e20 of the generator's, and stars with a softening 400 times smaller
    than the dark matter's (star and dark-matter tiles then take scales 2^16
    apart).  Against the one-sided kernel (FP64 partial sums, the same FP32
    pair terms) in every case; against the FP64 oracle where the softening
    keeps close pairs from amplifying the FP32 rounding of the positions."""
    import khrr
    pos, vel, mass, eps2 = galaxy(2048, 4096, seed=46, eps_s=eps_s, eps_d=0.004)
    mass = mass * mass_scale
    ctx.set_tuning()
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PHI)
    one = ctx.download()
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI)
    assert rel_rms(out["acc"], one["acc"]) <= 1e-6
    assert rel_rms(out["phi"], one["phi"]) <= 1e-6
    if eps_s >= 0.004:
        assert rel_rms(out["acc"], oracle.accel_f64(pos, mass, eps2)) <= 1e-6
        assert rel_rms(out["phi"], oracle.phi_f64(pos, mass, eps2)) <= 1e-6


def test_pair_agrees_with_one_sided_kernel(ctx):
    import khrr
    pos, vel, mass, eps2 = galaxy(3072, 6144, seed=36, eps_d=0.006)
    ctx.set_tuning()
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PHI)
    one = ctx.download()
    two = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI)
    assert rel_rms(two["acc"], one["acc"]) <= 1e-6
    assert rel_rms(two["phi"], one["phi"]) <= 1e-6


def test_batched_systems(ctx, oracle):
    import khrr
    parts = [galaxy(200, 500, seed=37), galaxy(1024, 2048, seed=38),
             galaxy(700, 1500, seed=39, eps_d=0.008), galaxy(3000, 1, seed=40)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI, offsets=off)
    for k, (ps, vs, ms, es) in enumerate(parts):
        s = slice(off[k], off[k + 1])
        assert rel_rms(out["acc"][s], oracle.accel_f64(ps, ms, es)) <= SMALL_N_TOL
        assert rel_rms(out["phi"][s], oracle.phi_f64(ps, ms, es)) <= SMALL_N_TOL


def test_forty_eight_blocks_against_fp64_samples(ctx, oracle):
    """16384 + 32768 bodies (48 blocks, rows cut into several chunks):
    sampled targets against the FP64 oracle."""
    import khrr
    pos, vel, mass, eps2 = galaxy(16384, 32768, seed=41)
    out = pair_forces(ctx, pos, vel, mass, eps2, khrr.ACC | khrr.PHI)
    tgt = np.random.default_rng(41).choice(len(mass), 512, replace=False)
    assert rel_rms(out["acc"][tgt], oracle.accel_f64(pos, mass, eps2, targets=tgt)) <= 1e-6
    assert rel_rms(out["phi"][tgt], oracle.phi_f64(pos, mass, eps2, targets=tgt)) <= 1e-6


def test_time_steps_follow_the_golden_trajectory(ctx, golden):
    """The reference's 10-step trajectory with the pair kernel in the step
    graphs, the potential fused into the last pass."""
    import khrr
    g = golden("steps_n1024.npz")
    ctx.set_tuning(*PAIR, 0, 2)
    try:
        ctx.upload(g["pos"], g["vel"], g["mass"], g["eps2"])
        ctx.forces(khrr.ACC)
        ctx.step(float(g["dt"]), int(g["nsteps"]), khrr.PHI)
        out = ctx.download()
    finally:
        ctx.set_tuning()
    assert np.abs(out["pos"].reshape(-1) - g["corrected_pos"]).max() <= 1e-7
    assert rel_rms(out["acc"], g["corrected_acc"]) <= 1e-5


def test_multi_block_steps_match_one_sided_steps(ctx):
    import khrr
    pos, vel, mass, eps2 = galaxy(2048, 4096, seed=42)
    res = []
    for tuning in (None, (*PAIR, 0, 2)):
        if tuning:
            ctx.set_tuning(*tuning)
        try:
            ctx.upload(pos, vel, mass, eps2)
            ctx.forces(khrr.ACC)
            ctx.step(0.002, 5, khrr.PHI)
            res.append(ctx.download())
        finally:
            ctx.set_tuning()
    assert np.abs(res[0]["pos"] - res[1]["pos"]).max() <= 1e-8
    assert rel_rms(res[1]["acc"], res[0]["acc"]) <= 1e-6


def test_tuning_validation(ctx):
    import khrr
    with pytest.raises(khrr.KhrrError):
        ctx.set_tuning(128, 4, 128, 0, 2)      # the pair kernel has one shape
    with pytest.raises(khrr.KhrrError):
        ctx.set_tuning(128, 4, 128, 0, 3)
    ctx.set_tuning(*PAIR, 0, 2)
    assert ctx.get_tuning()["packed"] == 2
    ctx.set_tuning()


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")


def test_kernel_level_entry_points_under_the_pair_tuning(ctx, golden, oracle):
    """khrr_accel / khrr_phi (the reference's call sites) with pos_i == pos_j
    take the pair kernel under the pair tuning, in the form the caller's
    arrays admit (classified on the device): overwrite and accumulate modes,
    the potential, ragged and whole-block sizes, equal and per-component
    softenings; a distinct target set still runs the one-sided kernel."""
    import torch
    import khrr
    g = golden("forces_n1536.npz")
    cases = [(g["pos"], g["mass"], g["eps2"], g["acc_f64"], g["phi"], 1e-6)]
    # ragged (general form); whole 1024 blocks with equal softenings (the
    # block-mass uniform form); whole blocks with two softenings
    for ns, nd, eps_d, tol in ((2500, 4321, 0.006, SMALL_N_TOL), (2048, 4096, 0.004, 1e-6),
                               (2048, 4096, 0.006, 1e-6)):
        p_, _, m_, e_ = galaxy(ns, nd, seed=43, eps_d=eps_d)
        cases.append((p_, m_, e_, oracle.accel_f64(p_, m_, e_), oracle.phi_f64(p_, m_, e_), tol))
    ctx.set_tuning(*PAIR, 0, 2)
    try:
        for pos, mass, eps2, acc_ref, phi_ref, tol in cases:
            n = len(mass)
            P, M, E = _dev(torch, pos), _dev(torch, mass), _dev(torch, eps2)
            A = torch.full((n, 3), 0.25, dtype=torch.float64, device="cuda")
            F = torch.full((n,), 2.0, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            ctx.accel(A.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n, 0)
            ctx.phi(F.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n, 0)
            ctx.synchronize()
            assert rel_rms(A.cpu().numpy() - 0.25, acc_ref) <= tol
            assert rel_rms(F.cpu().numpy() - 2.0, phi_ref) <= tol
            ctx.accel(A.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n, khrr.OVERWRITE)
            ctx.synchronize()
            assert rel_rms(A.cpu().numpy(), acc_ref) <= tol
        pos, vel, mass, eps2 = galaxy(256, 512, seed=4)
        pos_i = np.random.default_rng(9).uniform(-1, 1, pos.shape)
        P, Pi, M, E = _dev(torch, pos), _dev(torch, pos_i), _dev(torch, mass), _dev(torch, eps2)
        A = torch.zeros((len(mass), 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ctx.accel(A.data_ptr(), Pi.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), len(mass), khrr.OVERWRITE)
        ctx.synchronize()
    finally:
        ctx.set_tuning()
    d = pos[None, :, :] - pos_i[:, None, :]
    r2 = (d ** 2).sum(-1) + 0.5 * (eps2[:, None] + eps2[None, :])
    ref = (d * (mass[None, :] / r2 ** 1.5)[:, :, None]).sum(1)
    assert rel_rms(A.cpu().numpy(), ref) <= SMALL_N_TOL


def test_kernel_level_zero_softening_takes_the_one_sided_kernel(ctx):
    """A softening of zero leaves no bound for the fixed-point sums: under the
    pair tuning khrr_accel then runs the one-sided kernel, so its result is
    that kernel's bit for bit (the zero-softened body's self term is NaN, as
    the reference's 0/0 is)."""
    import torch
    import khrr
    pos, vel, mass, eps2 = galaxy(1024, 2048, seed=47)
    eps2 = eps2.copy()
    eps2[5] = 0.0
    n = len(mass)
    P, M, E = _dev(torch, pos), _dev(torch, mass), _dev(torch, eps2)
    res = []
    for tuning in (None, (*PAIR, 0, 2)):
        A = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        if tuning:
            ctx.set_tuning(*tuning)
        try:
            ctx.accel(A.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n, khrr.OVERWRITE)
            ctx.synchronize()
        finally:
            ctx.set_tuning()
        res.append(A.cpu().numpy())
    assert np.array_equal(res[0], res[1], equal_nan=True)
    assert np.isfinite(np.delete(res[1], 5, axis=0)).all()


def test_two_million_bodies_in_linear_memory(ctx, oracle):
    """The 2,097,152-body system of the large-mesh configuration (698,368
    stars + 1,398,784 DM, eps 0.002, 2,048 blocks): the pair kernel's sums
    take 32 bytes per body (67 MB), so the whole context stays within about
    half a gigabyte of device memory, and sampled targets meet the FP64
    oracle."""
    import torch
    import khrr
    pos, vel, mass, eps2 = galaxy(698368, 1398784, seed=45, eps_s=0.002, eps_d=0.002)
    n = len(mass)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    ctx.set_tuning(*PAIR, 0, 2)
    try:
        ctx.upload(pos, vel, mass, eps2)
        ctx.forces(khrr.ACC)
        free1, _ = torch.cuda.mem_get_info()
        out = ctx.download(pos=False, vel=False, phi=False)
    finally:
        ctx.set_tuning()
    # state (9 FP64 arrays of 24 or 8 B), shadow (20 B) and sums (32 B) per body
    assert free0 - free1 <= 1.5e9
    tgt = np.random.default_rng(45).choice(n, 256, replace=False)
    assert rel_rms(out["acc"][tgt], oracle.accel_f64(pos, mass, eps2, targets=tgt)) <= 1e-6
