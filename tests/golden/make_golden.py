"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own kernels compiled for the host (oracle/_ref, built by
oracle/Makefile from the reference tree) on small seeded inputs and stores
inputs + outputs as compressed .npz files.  The reference has no tests or
golden vectors of its own, so these fixtures are the pin for the oracle
restatement (oracle/oracle.c) and, through it, for the CUDA path.

Usage:  python tests/golden/make_golden.py [meshforce]   (needs the reference tree;
        with "meshforce" only that fixture is written)
"""
from __future__ import annotations

import json
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "khrr-nbody_b200"))

from pyoracle import Reference, build  # noqa: E402
from khrr.galaxy import make_galaxy  # noqa: E402

OUT = ROOT / "tests" / "golden"


def galaxy_inputs(ns, nd, seed, eps_s=0.004, eps_d=0.004):
    g = make_galaxy(ns, nd, seed, eps_stars=eps_s, eps_dm=eps_d)
    pos, vel, mass, eps = g.arrays()
    return pos, vel, mass, eps * eps


def main() -> None:
    build()
    R = Reference()

    # --- forces: FP64 (block-exact launch), FP32, potential ------------------
    pos, vel, mass, eps2 = galaxy_inputs(512, 1024, seed=11, eps_s=0.004, eps_d=0.008)
    np.savez_compressed(
        OUT / "forces_n1536.npz", pos=pos, vel=vel, mass=mass, eps2=eps2,
        acc_f64=R.accel_team(pos, mass, eps2), acc_f32=R.accel_f32(pos, mass, eps2),
        phi=R.phi_team(pos, mass, eps2))

    # --- external field and one predictor + corrector -----------------------
    fields = [(0.0, 0.0), (1.0, 0.0), (1.0, 0.5)]
    fex = []
    consts = []
    for Mh, Mb in fields:
        consts.append(list(R.set_field(Mh=Mh, Mb=Mb, ns=512, nn=1536).values()))
        fex.append(R.fex(pos))
    R.set_field(Mh=1.0, Mb=0.5, ns=512, nn=1536)
    n = len(mass)
    acc = R.accel_team(pos, mass, eps2).reshape(-1)
    P, V = pos.reshape(-1).copy(), vel.reshape(-1).copy()
    post, velt, a0 = np.zeros(3 * n), np.zeros(3 * n), acc.copy()
    R.integ(acc, post, velt, P, V, 0.002, 0, 0.0, a0)
    acct = R.accel_team(post, mass, eps2).reshape(-1)
    P2, V2, a1 = P.copy(), V.copy(), acc.copy()
    R.integ(acct, P2, V2, post, velt, 0.002, 1, 0.002, a1)
    np.savez_compressed(
        OUT / "integ_n1536.npz", fields=np.array(fields), consts=np.array(consts),
        fex=np.array(fex), post=post, velt=velt, pos1=P2, vel1=V2, acc1=a1)

    # --- 10 reference time steps (literal: force accumulates, D1) and the
    #     corrected form (force overwritten), no external field --------------
    pos, vel, mass, eps2 = galaxy_inputs(512, 512, seed=12)
    n = len(mass)
    R.set_field(ns=512, nn=n)
    traj = {}
    for label, accumulate in (("literal", True), ("corrected", False)):
        P, V = pos.reshape(-1).copy(), vel.reshape(-1).copy()
        acc = R.accel_team(P, mass, eps2).reshape(-1)
        acct = np.zeros(3 * n)
        post, velt = np.zeros(3 * n), np.zeros(3 * n)
        for _ in range(10):
            R.integ(acc, post, velt, P, V, 0.002, 0, 0.0, acc)
            f = R.accel_team(post, mass, eps2).reshape(-1)
            acct = acct + f if accumulate else f
            R.integ(acct, P, V, post, velt, 0.002, 1, 0.0, acc)
        traj[label + "_pos"] = P.copy()
        traj[label + "_vel"] = V.copy()
        traj[label + "_acc"] = acc.copy()
    np.savez_compressed(OUT / "steps_n1024.npz", pos=pos, vel=vel, mass=mass, eps2=eps2,
                        dt=0.002, nsteps=10, **traj)

    # --- p2mesh binning on two meshes, with bodies outside the domain -------
    pos, vel, mass, eps2 = galaxy_inputs(1024, 2048, seed=13)
    rng = np.random.default_rng(5)
    pos[:64] = rng.uniform(-3.0, 3.0, (64, 3))   # some bodies outside [-1,1]^3 / [-1.2,1.2]^3
    phi = R.phi_team(pos, mass, eps2)
    bins = {}
    for nx, L in ((16, 1.0), (24, 1.2)):
        lo = (-L, -L, -L)
        cs = (2 * L / nx,) * 3
        R.set_mesh(lo, cs, (nx, nx, nx))
        b = R.bin(pos, mass, nx ** 3)
        cp = R.cell_phi(phi, b["pci"], b["cell_info"], nx ** 3)
        for k in ("cell_id", "id_in_cell", "count", "start_id", "maxpbc", "cell_mass"):
            bins[f"nx{nx}_{k}"] = b[k]
        bins[f"nx{nx}_cell_phi"] = cp
        bins[f"nx{nx}_lo"] = np.array(lo)
        bins[f"nx{nx}_cs"] = np.array(cs)
    np.savez_compressed(OUT / "bin_n3072.npz", pos=pos, mass=mass, phi=phi, **bins)

    # --- damped-wave iterations + gradient + gather on a 16^3 mesh ----------
    nx, dx = 16, 0.2
    c = 4574.337022617616
    dt = 0.5 * dx / (c * np.sqrt(3.0))
    sim_l = 0.5 * nx * dx
    R.set_mesh((-sim_l,) * 3, (dx,) * 3, (nx, nx, nx), nx_wave=nx, dx_wave=dx, dt_wave=dt,
               c_wave=c, diss_base=0.1, diss_extra=0.01, sim_l=sim_l, bc_l=sim_l / 10.0)
    cm = rng.uniform(0.0, 1e-3, nx ** 3)
    prev, cur = np.zeros(nx ** 3), np.zeros(nx ** 3)
    for _ in range(5):
        nxt = R.wave(cur, prev, cm)
        prev, cur = cur, nxt
    cell_acc = R.acc_field(nx, dx, cur)
    np.savez_compressed(OUT / "wave_nx16.npz", cell_mass=cm, phi_prev=prev, phi=cur,
                        cell_acc=cell_acc, nx=nx, dx=dx, dt=dt, c=c, sim_l=sim_l)

    meshforce(R)

    # --- the reference's .ini reader on two galaxy files ---------------------
    parsed = {}
    with tempfile.TemporaryDirectory() as td:
        two = pathlib.Path(td) / "__start_galaxies.ini"
        two.write_text(
            "2\t\t\t---- M_glx\n"
            "0\t\t\t---- k_glx\n131072,262144 \t\t---- N_s,N_dm\n1.0,6.699356 \t\t---- M\n"
            "0.004,0.004 \t\t---- eps\n0.0\t\t\t---- alpha\n-1.5,0.0,0.0\t\t---- X\n0.3,-0.1,0.0\t\t---- V\n"
            "1\t\t\t---- k_glx\n131072,262144 \t\t---- N_s,N_dm\n1.0,0.0 \t\t---- M\n"
            "0.004,0.002 \t\t---- eps\n30.0\t\t\t---- alpha\n1.5,0.0,0.0\t\t---- X\n-0.3,0.1,0.0\t\t---- V\n")
        parsed["two_galaxies"] = {"text": two.read_text(), "parsed": R.read_galaxies(two)}
    (OUT / "galaxies_ini.json").write_text(json.dumps(parsed, indent=1))
    print("golden fixtures written to", OUT)


def meshforce(R) -> None:
    """The reference's Wave-mode force (calc_acceleration_by_grid,
    nbody/src/nbody.cu:183-285) composed from its own kernels: bin + NGP
    deposit, 40 wave iterations from a zero field, acc_field, the two
    gathers.  A 16^3 mesh of dx = 0.2 over [-1.6, 1.6]^3 (some bodies outside,
    clamped into the faces)."""
    pos, vel, mass, eps2 = galaxy_inputs(1024, 2048, seed=17)
    nx, dx, iters = 16, 0.2, 40
    c = 4574.337022617616
    dt = 0.5 * dx / (c * np.sqrt(3.0))
    sim_l = 0.5 * nx * dx
    R.set_mesh((-sim_l,) * 3, (dx,) * 3, (nx, nx, nx), nx_wave=nx, dx_wave=dx, dt_wave=dt,
               c_wave=c, diss_base=0.1, diss_extra=0.01, sim_l=sim_l, bc_l=sim_l / 10.0)
    b = R.bin(pos, mass, nx ** 3)
    prev, cur = np.zeros(nx ** 3), np.zeros(nx ** 3)
    for _ in range(iters):
        nxt = R.wave(cur, prev, b["cell_mass"])
        prev, cur = cur, nxt
    cell_acc = R.acc_field(nx, dx, cur)
    acc, phi = R.apply(b["pci"], cell_acc, cur)
    np.savez_compressed(OUT / "meshforce_n3072.npz", pos=pos, mass=mass, acc=acc, phi=phi, cell_phi=cur,
                        nx=nx, dx=dx, dt=dt, c=c, sim_l=sim_l, iters=iters)


if __name__ == "__main__":
    if sys.argv[1:] == ["meshforce"]:
        build()
        meshforce(Reference())
    else:
        main()
