"""GPU parity of the p2mesh pieces beyond the reference's NGP path and of the
mesh-force solver (the reference's Wave mode) against the oracle.

Tolerances: the counting-sort order equals the oracle's scatter of the GPU's
own cell ids, slots and starts exactly; the CIC deposit <= 1e-12 relative
(FP64 atomic order); the CIC gather is bit-exact (fixed corner order, IEEE
double, no FMA contraction); the mesh-force setup evaluation with the FP64
stencil and NGP deposit equals the reference-composed fixture to <= 1e-12
relative (only the deposit's summation order differs); Wave-mode trajectories
(setup + steps) against the oracle run: FP64 stencil max|dx| <= 1e-12 and
max|dv| <= 1e-10, FP32 stencil with CIC max|dx| <= 1e-9 and potentials
<= 1e-6 relative (an ulp of a cell mass rounded to FP32 can differ).
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


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def galaxy(ns, nd, seed):
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(ns, nd, seed).arrays()
    return pos, vel, mass, eps * eps


def test_cic_deposit_and_gather(ctx, torch_cuda, oracle):
    import khrr
    torch = torch_cuda
    rng = np.random.default_rng(8)
    nx, L = 24, 1.5
    cs = 2 * L / nx
    mesh = khrr.Mesh.make((-L,) * 3, (cs,) * 3, (nx,) * 3)
    pos, _, mass, _ = galaxy(1024, 2048, 31)
    pos[:50] = rng.uniform(-3, 3, (50, 3))   # some clouds partly or wholly outside
    C = nx ** 3
    P, M = dev(torch, pos), dev(torch, mass)
    cm = torch.zeros(C, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()   # torch's fill runs on its own stream, the deposit on the context's
    ctx.cic_deposit(P.data_ptr(), M.data_ptr(), len(mass), mesh, cm.data_ptr())
    ctx.synchronize()
    want = oracle.cic_deposit(pos, mass, (-L,) * 3, (cs,) * 3, (nx,) * 3)
    got = cm.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # gather a smooth field and a gradient back
    cacc = rng.normal(size=(C, 3))
    cval = rng.normal(size=C)
    A = torch.zeros((len(mass), 3), dtype=torch.float64, device="cuda")
    V = torch.zeros(len(mass), dtype=torch.float64, device="cuda")
    CA, CV = dev(torch, cacc), dev(torch, cval)   # held until the kernel has run
    torch.cuda.synchronize()
    ctx.cic_gather(P.data_ptr(), len(mass), mesh, CA.data_ptr(), CV.data_ptr(), A.data_ptr(), V.data_ptr())
    ctx.synchronize()
    wa, wv = oracle.cic_gather(pos, (-L,) * 3, (cs,) * 3, (nx,) * 3, cacc, cval)
    assert np.array_equal(A.cpu().numpy(), wa)
    assert np.array_equal(V.cpu().numpy(), wv)


def test_cic_refuses_non_cubic(ctx, torch_cuda):
    import khrr
    torch = torch_cuda
    mesh = khrr.Mesh.make((-1,) * 3, (0.1,) * 3, (16, 16, 8))
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(khrr.KhrrError):
        ctx.cic_deposit(buf.data_ptr(), buf.data_ptr(), 1, mesh, buf.data_ptr())


def test_counting_sort(ctx, torch_cuda, oracle):
    pos, vel, mass, eps2 = galaxy(2048, 4096, 32)
    ctx.upload(pos, vel, mass, eps2)
    nx, L = 32, 2.0
    b = ctx.bin((-L,) * 3, (2 * L / nx,) * 3, (nx,) * 3)
    order = ctx.sort_by_cell()
    assert np.array_equal(np.sort(order), np.arange(len(mass)))
    assert (np.diff(b["cell_id"][order]) >= 0).all()
    assert np.array_equal(order, oracle.scatter_order(b["cell_id"], b["id_in_cell"], b["start"]))


def test_counting_sort_two_systems(ctx, torch_cuda):
    """Bodies of every system are numbered as uploaded (global indices)."""
    p1, v1, m1, e1 = galaxy(300, 600, 33)
    p2, v2, m2, e2 = galaxy(500, 200, 34)
    pos, vel = np.concatenate([p1, p2]), np.concatenate([v1, v2])
    mass, eps2 = np.concatenate([m1, m2]), np.concatenate([e1, e2])
    ctx.upload(pos, vel, mass, eps2, offsets=[0, 900, 1600])
    b = ctx.bin((-2.0,) * 3, (0.125,) * 3, (32,) * 3)
    order = ctx.sort_by_cell()
    assert np.array_equal(np.sort(order), np.arange(1600))
    assert (np.diff(b["cell_id"][order]) >= 0).all()


def test_mesh_force_setup_matches_reference(ctx, torch_cuda, golden):
    import khrr
    g = golden("meshforce_n3072.npz")
    nx, dx = int(g["nx"]), float(g["dx"])
    pos, mass = g["pos"], g["mass"]
    n = len(mass)
    ctx.upload(pos, np.zeros_like(pos), mass, np.full(n, 0.004 ** 2))
    W = khrr.WaveParams.make(nx, dx, c=float(g["c"]), dt=float(g["dt"]))
    ctx.set_mesh_solver(W, assign=khrr.ASSIGN_NGP, fp64=True, iters_per_step=10, setup_iters=int(g["iters"]))
    try:
        ctx.forces(khrr.ACC | khrr.PHI | khrr.MESH)
        st = ctx.download()
        scale = np.abs(g["acc"]).max()
        assert np.abs(st["acc"] - g["acc"]).max() <= 1e-12 * scale
        assert np.abs(st["phi"] - g["phi"]).max() <= 1e-12 * np.abs(g["phi"]).max()
        assert np.abs(ctx.mesh_solver_phi(nx) - g["cell_phi"]).max() <= 1e-12 * np.abs(g["cell_phi"]).max()
    finally:
        ctx.set_mesh_solver(None)


@pytest.mark.parametrize("cic,fp64", [(False, True), (True, True), (True, False), (False, False)])
def test_mesh_steps_match_oracle(ctx, torch_cuda, oracle, cic, fp64):
    import khrr
    pos, vel, mass, eps2 = galaxy(1024, 2048, 35)
    nx, dx, dt, nsteps, iters, setup = 32, 0.25, 0.002, 4, 60, 600
    ctx.upload(pos, vel, mass, eps2)
    W = khrr.WaveParams.make(nx, dx)
    ctx.set_mesh_solver(W, assign=khrr.ASSIGN_CIC if cic else khrr.ASSIGN_NGP, fp64=fp64, iters_per_step=iters,
                        setup_iters=setup)
    try:
        ctx.forces(khrr.ACC | khrr.PHI | khrr.MESH)
        ctx.step(dt, nsteps - 1, khrr.MESH)
        ctx.step(dt, 1, khrr.MESH | khrr.PHI)     # graphs of other ring rotations, the phi variant
        st = ctx.download()
    finally:
        ctx.set_mesh_solver(None)
    OW = oracle.wave_params(nx, dx)
    p, v, a, phi = oracle.mesh_steps(OW, pos, vel, mass, dt, nsteps, iters=iters, setup_iters=setup,
                                     cic=cic, fp64=fp64)
    if fp64:
        assert np.abs(st["pos"] - p).max() <= 1e-12
        assert np.abs(st["vel"] - v).max() <= 1e-10
        assert np.abs(st["phi"] - phi).max() <= 1e-10 * np.abs(phi).max()
    else:
        assert np.abs(st["pos"] - p).max() <= 1e-9
        assert np.abs(st["phi"] - phi).max() <= 1e-6 * np.abs(phi).max()
    assert np.isfinite(st["acc"]).all()


def test_mesh_steps_resident_stencil_128(ctx, torch_cuda, monkeypatch):
    """Wave-mode steps on the encounter's 128^3 mesh (CIC, FP32 stencil): with
    the shared-memory-resident stencil (all iterations of a force evaluation
    in one launch) the trajectory, accelerations and potentials equal those
    of one launch per iteration (KHRR_WAVE_RESIDENT=0) bit for bit; odd
    iteration counts per step exercise the ring's single-iteration tail."""
    import khrr
    pos, vel, mass, eps2 = galaxy(8192, 16384, 37)
    nx, dx, dt = 128, 0.0625, 0.002
    W = khrr.WaveParams.make(nx, dx)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("KHRR_WAVE_RESIDENT", mode)
        ctx.upload(pos, vel, mass, eps2)
        ctx.set_mesh_solver(W, assign=khrr.ASSIGN_CIC, fp64=False, iters_per_step=37, setup_iters=101)
        try:
            ctx.forces(khrr.ACC | khrr.PHI | khrr.MESH)
            ctx.step(dt, 2, khrr.MESH)
            ctx.step(dt, 1, khrr.MESH | khrr.PHI)
            out[mode] = ctx.download()
        finally:
            ctx.set_mesh_solver(None)
    for key in ("pos", "vel", "acc", "phi"):
        assert np.array_equal(out["1"][key], out["0"][key]), key
    assert np.isfinite(out["1"]["acc"]).all()


def test_mesh_solver_rejects_bad_use(ctx, torch_cuda):
    import khrr
    pos, vel, mass, eps2 = galaxy(256, 256, 36)
    ctx.upload(pos, vel, mass, eps2)
    with pytest.raises(khrr.KhrrError):
        ctx.forces(khrr.ACC | khrr.MESH)             # no solver set
    W = khrr.WaveParams.make(16, 0.25)
    with pytest.raises(khrr.KhrrError):
        ctx.set_mesh_solver(W, assign=7)
    ctx.upload(np.concatenate([pos, pos]), np.concatenate([vel, vel]), np.concatenate([mass, mass]),
               np.concatenate([eps2, eps2]), offsets=[0, 512, 1024])
    ctx.set_mesh_solver(W, setup_iters=10, iters_per_step=5)
    try:
        with pytest.raises(khrr.KhrrError):
            ctx.forces(khrr.ACC | khrr.MESH)         # two systems on one mesh
    finally:
        ctx.set_mesh_solver(None)
