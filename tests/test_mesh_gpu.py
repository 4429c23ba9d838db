"""GPU parity of the p2mesh path (binning, prefix sums, deposits, wave
stencil, gradient, gather) against the reference fixtures and the oracle.

Tolerances: cell ids, counts, the reference start_id view, maxPBC and the
exclusive scan are bit-exact; id_in_cell is checked as a per-cell permutation
of 0..count-1 (slots come from atomics, as in the reference); FP64 cell
masses and cell potentials <= 1e-12 relative (atomic summation order); the
FP64 wave iteration, gradient and gather are bit-exact (IEEE double, no FMA
contraction); the FP32 stencil equals the oracle's FP32 restatement exactly
on the same FP32 inputs and tracks the FP64 reference to <= 1e-5 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ctx(libkhrr, torch_cuda):
    import khrr
    c = khrr.Context(0)
    yield c
    c.close()


def dev(torch, a, dtype=None):
    a = np.ascontiguousarray(a)
    return torch.as_tensor(a, device="cuda")


def check_slots(cell_id, slot, count):
    """id_in_cell of every cell is a permutation of 0..count-1."""
    order = np.lexsort((slot, cell_id))
    c, s = cell_id[order], slot[order]
    first = np.r_[True, c[1:] != c[:-1]]
    start = np.maximum.accumulate(np.where(first, np.arange(len(c)), 0))
    assert np.array_equal(s, np.arange(len(c)) - start)
    assert np.array_equal(np.bincount(cell_id, minlength=len(count)), count)


@pytest.mark.parametrize("nx", [16, 24])
def test_kernel_level_binning_matches_reference(ctx, torch_cuda, golden, nx):
    import khrr
    torch = torch_cuda
    g = golden("bin_n3072.npz")
    k = f"nx{nx}_"
    n, C = len(g["mass"]), nx ** 3
    mesh = khrr.Mesh.make(g[k + "lo"], g[k + "cs"], (nx, nx, nx))
    P, M = dev(torch, g["pos"]), dev(torch, g["mass"])
    pci = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(2 * C, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(C, dtype=torch.int32, device="cuda")
    cm = torch.zeros(C, dtype=torch.float64, device="cuda")
    maxpbc = torch.zeros((C + 511) // 512, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.assign_particles_to_cells(P.data_ptr(), n, mesh, pci.data_ptr(), info.data_ptr(), cnt.data_ptr(),
                                  M.data_ptr(), cm.data_ptr())
    ctx.compute_prefix_sums(info.data_ptr(), maxpbc.data_ptr(), C, khrr.SCAN_REFERENCE)
    ctx.synchronize()
    p, inf = pci.cpu().numpy(), info.cpu().numpy()
    assert np.array_equal(p[0::2], g[k + "cell_id"])
    assert np.array_equal(inf[0::2], g[k + "count"])
    assert np.array_equal(cnt.cpu().numpy(), g[k + "count"])
    check_slots(p[0::2], p[1::2], g[k + "count"])
    assert np.array_equal(inf[1::2], g[k + "start_id"])
    assert np.array_equal(maxpbc.cpu().numpy(), g[k + "maxpbc"])
    assert np.allclose(cm.cpu().numpy(), g[k + "cell_mass"], rtol=1e-12, atol=0)
    # true exclusive scan
    ctx.compute_prefix_sums(info.data_ptr(), maxpbc.data_ptr(), C, khrr.SCAN_EXCLUSIVE)
    ctx.synchronize()
    cnt_ref = g[k + "count"]
    assert np.array_equal(info.cpu().numpy()[1::2], np.r_[0, np.cumsum(cnt_ref)[:-1]])
    # cell potential deposit
    phi = dev(torch, g["phi"])
    cp = torch.zeros(C, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.cell_phi(phi.data_ptr(), pci.data_ptr(), info.data_ptr(), n, cp.data_ptr())
    ctx.synchronize()
    assert np.allclose(cp.cpu().numpy(), g[k + "cell_phi"], rtol=1e-12, atol=1e-300)


def test_binning_without_separate_counter(ctx, torch_cuda, golden):
    """cell_count NULL: the slots come from cell_info.count itself."""
    import khrr
    torch = torch_cuda
    g = golden("bin_n3072.npz")
    nx, n = 16, len(g["mass"])
    mesh = khrr.Mesh.make(g["nx16_lo"], g["nx16_cs"], (nx, nx, nx))
    P = dev(torch, g["pos"])
    pci = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(2 * nx ** 3, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.assign_particles_to_cells(P.data_ptr(), n, mesh, pci.data_ptr(), info.data_ptr())
    ctx.synchronize()
    p = pci.cpu().numpy()
    assert np.array_equal(info.cpu().numpy()[0::2], g["nx16_count"])
    check_slots(p[0::2], p[1::2], g["nx16_count"])


def test_wave_iterations_gradient_and_gather(ctx, torch_cuda, golden, oracle):
    import khrr
    torch = torch_cuda
    g = golden("wave_nx16.npz")
    nx, dx = int(g["nx"]), float(g["dx"])
    W = khrr.WaveParams.make(nx, dx, c=float(g["c"]), dt=float(g["dt"]))
    bufs = [torch.zeros(nx ** 3, dtype=torch.float64, device="cuda") for _ in range(3)]
    mass = dev(torch, g["cell_mass"])
    torch.cuda.synchronize()
    old, cur, nxt = bufs
    for _ in range(5):
        ctx.wave_iteration(nxt.data_ptr(), cur.data_ptr(), old.data_ptr(), mass.data_ptr(), W)
        old, cur, nxt = cur, nxt, old
    ctx.synchronize()
    assert np.array_equal(cur.cpu().numpy(), g["phi"])
    assert np.array_equal(old.cpu().numpy(), g["phi_prev"])
    acc = torch.zeros(3 * nx ** 3, dtype=torch.float64, device="cuda")
    acc_abs = torch.zeros(nx ** 3, dtype=torch.float64, device="cuda")
    ctx.acc_field(acc.data_ptr(), acc_abs.data_ptr(), cur.data_ptr(), nx, dx)
    ctx.synchronize()
    a = acc.cpu().numpy().reshape(-1, 3)
    assert np.array_equal(a, g["cell_acc"])
    assert np.allclose(acc_abs.cpu().numpy(), np.sqrt((a ** 2).sum(1)), rtol=1e-15, atol=0)
    # gather to bodies through their cells
    rng = np.random.default_rng(4)
    cid = rng.integers(0, nx ** 3, 1000).astype(np.int32)
    pci = dev(torch, np.stack([cid, np.zeros_like(cid)], 1).reshape(-1))
    pacc = torch.zeros(3000, dtype=torch.float64, device="cuda")
    pval = torch.zeros(1000, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.apply_cells_to_particles(pacc.data_ptr(), pval.data_ptr(), acc.data_ptr(), cur.data_ptr(),
                                 pci.data_ptr(), 1000)
    ctx.synchronize()
    ga, gp = oracle.gather(cid, a, g["phi"])
    assert np.array_equal(pacc.cpu().numpy().reshape(-1, 3), ga)
    assert np.array_equal(pval.cpu().numpy(), gp)


def galaxy_state(ns, nd, seed):
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(ns, nd, seed).arrays()
    return pos, vel, mass, eps * eps


@pytest.mark.parametrize("ns,nd,nx,L", [(1000, 2001, 24, 1.2), (43008, 88064, 64, 2.0)])
def test_context_binning_matches_oracle(ctx, oracle, ns, nd, nx, L):
    pos, vel, mass, eps2 = galaxy_state(ns, nd, seed=14)
    pos[:17] *= 3.0  # a few bodies outside the mesh
    ctx.upload(pos, vel, mass, eps2)
    lo, cs = (-L,) * 3, (2 * L / nx,) * 3
    b = ctx.bin(lo, cs, (nx, nx, nx))
    cid, slot, cnt = oracle.assign(pos, lo, cs, (nx, nx, nx))
    st, sr, mp = oracle.scan(cnt)
    assert np.array_equal(b["cell_id"], cid)
    assert np.array_equal(b["count"], cnt)
    check_slots(b["cell_id"], b["id_in_cell"], cnt)
    assert np.array_equal(b["start"], st)
    assert np.array_equal(b["start_ref"], sr)
    assert np.allclose(b["cell_mass"], oracle.cell_masses(mass, cid, nx ** 3), rtol=1e-12, atol=0)


def test_context_binning_of_several_systems(ctx, oracle):
    parts = [galaxy_state(300, 600, 15), galaxy_state(512, 1024, 16)]
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    eps2 = np.concatenate([p[3] for p in parts])
    off = np.cumsum([0] + [len(p[2]) for p in parts])
    ctx.upload(pos, vel, mass, eps2, offsets=off)
    lo, cs, nx = (-1.0,) * 3, (2.0 / 16,) * 3, 16
    b = ctx.bin(lo, cs, (nx, nx, nx))
    cid, slot, cnt = oracle.assign(pos, lo, cs, (nx, nx, nx))
    assert np.array_equal(b["cell_id"], cid) and np.array_equal(b["count"], cnt)
    check_slots(b["cell_id"], b["id_in_cell"], cnt)


def test_binning_at_full_size_properties(ctx, oracle):
    """786,432 bodies on 128^3 cells over [-4,4]^3: ids exact vs the oracle,
    and the size-independent scan properties."""
    pos, vel, mass, eps2 = galaxy_state(262144, 524288, 1000)
    ctx.upload(pos, vel, mass, eps2)
    nx = 128
    lo, cs = (-4.0,) * 3, (8.0 / nx,) * 3
    b = ctx.bin(lo, cs, (nx, nx, nx))
    cid, slot, cnt = oracle.assign(pos, lo, cs, (nx, nx, nx))
    assert np.array_equal(b["cell_id"], cid)
    assert np.array_equal(b["count"], cnt)
    assert b["count"].sum() == len(mass)
    assert b["start"][0] == 0 and np.array_equal(np.diff(b["start"]), b["count"][:-1])
    blocks = np.arange(nx ** 3) // 512
    assert np.array_equal(b["start_ref"], b["start"][blocks * 512])
    assert abs(b["cell_mass"].sum() / mass.sum() - 1.0) < 1e-12


def test_wave_solve_fp32_matches_restatement_and_converges(ctx, oracle):
    import khrr
    pos, vel, mass, eps2 = galaxy_state(4096, 8192, 17)
    nx, L = 32, 4.0
    dx = 2 * L / nx
    ctx.upload(pos, vel, mass, eps2)
    b = ctx.bin((-L,) * 3, (dx,) * 3, (nx, nx, nx))
    W = khrr.WaveParams.make(nx, dx)
    it, res, phi = ctx.wave_solve(W, tol=0.0, max_iter=12, check_every=4, cold=True)
    assert it == 12
    Wo = oracle.wave_params(nx, dx)
    m32 = b["cell_mass"].astype(np.float32)
    prev, cur = np.zeros(nx ** 3, np.float32), np.zeros(nx ** 3, np.float32)
    for _ in range(12):
        prev, cur = cur, oracle.wave_iter_f32(Wo, cur, prev, m32)
    assert np.array_equal(phi, cur)
    # tracks the FP64 reference iteration
    p64, c64 = np.zeros(nx ** 3), np.zeros(nx ** 3)
    for _ in range(12):
        p64, c64 = c64, oracle.wave_iter_f64(Wo, c64, p64, b["cell_mass"])
    assert np.abs(phi - c64).max() <= 1e-5 * np.abs(c64).max()
    # residual shrinks as the field relaxes; a warm start continues from it
    it2, res2, _ = ctx.wave_solve(W, tol=0.0, max_iter=300, check_every=50)
    it3, res3, _ = ctx.wave_solve(W, tol=0.0, max_iter=300, check_every=50)
    assert res3 < res2
    it4, res4, _ = ctx.wave_solve(W, tol=res3 * 1.5, max_iter=100000, check_every=10)
    assert res4 < res3 * 1.5 and it4 < 100000


@pytest.mark.parametrize("kernel", ["0", "1", "2"])
@pytest.mark.parametrize("nx,max_iter,check_every", [(37, 7, 3), (40, 6, 6), (200, 5, 5)])
def test_wave_solve_pairs_and_singles_bit_exact(ctx, oracle, nx, max_iter, check_every, kernel, monkeypatch):
    """Every FP32 stencil kernel (KHRR_WAVE_TMA: 0 the cache-fed one-step
    kernel, 1 the tensor-copy one-step kernel, 2 pairs through the
    tensor-copy two-step kernel; meshes the tensor-copy kernels cannot take,
    nx = 37, fall back to the cache-fed one) and odd counts: the field equals
    the oracle's FP32 restatement bit for bit (meshes that are not multiples
    of the 32 x 8 x TZ tile, and the TZ = 32 shape from nx = 192 up), and the
    residual of the last iteration matches the FP64 norm of the oracle's last
    step."""
    import khrr
    monkeypatch.setenv("KHRR_WAVE_TMA", kernel)
    pos, vel, mass, eps2 = galaxy_state(2048, 4096, 18)
    L = 3.0
    dx = 2 * L / nx
    ctx.upload(pos, vel, mass, eps2)
    b = ctx.bin((-L,) * 3, (dx,) * 3, (nx, nx, nx))
    W = khrr.WaveParams.make(nx, dx)
    it, res, phi = ctx.wave_solve(W, tol=0.0, max_iter=max_iter, check_every=check_every, cold=True)
    assert it == max_iter
    Wo = oracle.wave_params(nx, dx)
    m32 = b["cell_mass"].astype(np.float32)
    prev, cur = np.zeros(nx ** 3, np.float32), np.zeros(nx ** 3, np.float32)
    for _ in range(max_iter):
        prev, cur = cur, oracle.wave_iter_f32(Wo, cur, prev, m32)
    assert np.array_equal(phi, cur)
    d = cur.astype(np.float64) - prev.astype(np.float64)
    want = np.sqrt((d * d).sum() / (cur.astype(np.float64) ** 2).sum())
    assert abs(res - want) <= 1e-12 * want


@pytest.mark.parametrize("nx", [37, 96])
def test_fp64_wave_iteration_bit_exact_on_random_fields(ctx, torch_cuda, oracle, nx):
    """The FP64 stencil (the reference's wave_diss_iteration expressions, its
    divisions through shared correctly rounded reciprocals) equals the
    oracle's IEEE-division restatement bit for bit on random fields, three
    iterations in a row, on a mesh that is not a multiple of the thread tile."""
    import khrr
    torch = torch_cuda
    rng = np.random.default_rng(nx)
    C = nx ** 3
    dx = 8.0 / nx
    W = khrr.WaveParams.make(nx, dx)
    Wo = oracle.wave_params(nx, dx)
    mass = rng.uniform(0.0, 1e-3, C)
    prev, cur = rng.normal(0.0, 1.0, C), rng.normal(0.0, 1.0, C)
    bufs = [torch.as_tensor(prev, device="cuda"), torch.as_tensor(cur, device="cuda"),
            torch.zeros(C, dtype=torch.float64, device="cuda")]
    M = torch.as_tensor(mass, device="cuda")
    torch.cuda.synchronize()
    for k in range(3):
        o, c, n = bufs[k % 3], bufs[(k + 1) % 3], bufs[(k + 2) % 3]
        ctx.wave_iteration(n.data_ptr(), c.data_ptr(), o.data_ptr(), M.data_ptr(), W)
        prev, cur = cur, oracle.wave_iter_f64(Wo, cur, prev, mass)
    ctx.synchronize()
    assert np.array_equal(bufs[(3 + 1) % 3].cpu().numpy(), cur)


@pytest.mark.parametrize("max_iter,check_every", [(7, 3), (6, 6), (1, 1), (4, 2)])
def test_resident_stencil_128_bit_exact(ctx, oracle, max_iter, check_every):
    """The shared-memory-resident FP32 stencil (128^3: one CTA per z plane,
    all iterations of a chunk in one cooperative launch, neighbour planes
    exchanged through counters): the field equals the oracle's FP32
    restatement bit for bit, for odd and even chunks and single iterations,
    and the residual of the last iteration matches the FP64 norm of the
    oracle's last step."""
    import khrr
    pos, vel, mass, eps2 = galaxy_state(8192, 16384, 19)
    nx, L = 128, 4.0
    dx = 2 * L / nx
    ctx.upload(pos, vel, mass, eps2)
    b = ctx.bin((-L,) * 3, (dx,) * 3, (nx, nx, nx))
    W = khrr.WaveParams.make(nx, dx)
    it, res, phi = ctx.wave_solve(W, tol=0.0, max_iter=max_iter, check_every=check_every, cold=True)
    assert it == max_iter
    Wo = oracle.wave_params(nx, dx)
    m32 = b["cell_mass"].astype(np.float32)
    prev, cur = np.zeros(nx ** 3, np.float32), np.zeros(nx ** 3, np.float32)
    for _ in range(max_iter):
        prev, cur = cur, oracle.wave_iter_f32(Wo, cur, prev, m32)
    assert np.array_equal(phi, cur)
    d = cur.astype(np.float64) - prev.astype(np.float64)
    want = np.sqrt((d * d).sum() / (cur.astype(np.float64) ** 2).sum())
    assert abs(res - want) <= 1e-12 * want


def test_resident_stencil_matches_per_iteration_launches(ctx, monkeypatch):
    """Long runs at 128^3 (warm continuation over several calls, chunks of 50
    with residual checks): the resident kernel and one launch per iteration
    (KHRR_WAVE_RESIDENT=0) give the same field bits and residuals."""
    import khrr
    pos, vel, mass, eps2 = galaxy_state(8192, 16384, 20)
    nx, L = 128, 4.0
    dx = 2 * L / nx
    ctx.upload(pos, vel, mass, eps2)
    ctx.bin((-L,) * 3, (dx,) * 3, (nx, nx, nx))
    W = khrr.WaveParams.make(nx, dx)
    runs = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("KHRR_WAVE_RESIDENT", mode)
        out = [ctx.wave_solve(W, tol=0.0, max_iter=101, check_every=50, cold=True)]
        out.append(ctx.wave_solve(W, tol=0.0, max_iter=203, check_every=50))
        runs[mode] = out
    for (i1, r1, p1), (i0, r0, p0) in zip(runs["1"], runs["0"]):
        assert i1 == i0
        assert np.array_equal(p1, p0)
        assert abs(r1 - r0) <= 1e-12 * r0


def test_call_timing_of_mesh_calls(ctx):
    """khrr_call_timing: the device time of the last timed khrr_bin /
    khrr_sort_by_cell is positive and no longer than the call measured from
    outside (which adds the downloads and the closing host synchronisation);
    without a timed call it reports KHRR_ERR_STATE."""
    import time
    import khrr
    pos, vel, mass, eps2 = galaxy_state(8192, 16384, 41)
    ctx.upload(pos, vel, mass, eps2)
    nx, L = 64, 4.0
    ctx.enable_timing(False)
    ctx.bin((-L,) * 3, (2 * L / nx,) * 3, (nx, nx, nx))
    with pytest.raises(khrr.KhrrError) as e:
        ctx.call_timing()
    assert e.value.status == 6  # KHRR_ERR_STATE
    ctx.enable_timing(True)
    try:
        t0 = time.perf_counter()
        b = ctx.bin((-L,) * 3, (2 * L / nx,) * 3, (nx, nx, nx))
        wall = (time.perf_counter() - t0) * 1e3
        ms = ctx.call_timing()
        assert 0.0 < ms <= wall
        assert b["count"].sum() == len(mass)
        t0 = time.perf_counter()
        order = ctx.sort_by_cell()
        wall = (time.perf_counter() - t0) * 1e3
        ms2 = ctx.call_timing()
        assert 0.0 < ms2 <= wall
        assert np.array_equal(np.sort(order), np.arange(len(mass)))
    finally:
        ctx.enable_timing(False)
