"""numpy bindings for the oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle.so`` (the CPU restatement, oracle.c) and,
when present, ``oracle/_ref/libkhrr_ref.so`` (the reference's own kernel
headers compiled for the host).  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libkhrr_ref.so"

_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_d = C.c_double
_vp = C.c_void_p


def build(quiet: bool = True) -> None:
    """Run the oracle Makefile (builds _ref too when the reference tree exists)."""
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


class OrcField(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "Mh", "a", "Rh", "Mb", "b", "Rb", "Rh2", "con", "const1", "Mh_inf", "c_phi_h", "c_phi_b")]


class OrcWave(C.Structure):
    _fields_ = [("nx", C.c_int)] + [(k, C.c_double) for k in (
        "dx", "dt", "c", "diss_base", "diss_extra", "sim_l", "bc_l")]


def _c3(a):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


def _tg(targets):
    if targets is None:
        return None, 0
    t = np.ascontiguousarray(targets, dtype=np.int64)
    return t, t.size


class Oracle:
    """The CPU restatement (oracle.c)."""

    def __init__(self, path: os.PathLike | None = None):
        p = pathlib.Path(path) if path else ORACLE_SO
        if not p.exists():
            build()
        L = C.CDLL(str(p))
        self.L = L
        L.orc_field_init.argtypes = [C.POINTER(OrcField)] + [_d] * 6
        for name in ("orc_accel_f64", "orc_accel_f32"):
            getattr(L, name).argtypes = [_i64, _f64p, _f64p, _f64p, _i64, _vp, _f64p]
        L.orc_phi_f64.argtypes = [_i64, _f64p, _f64p, _f64p, _i64, _vp, _f64p]
        L.orc_fex.argtypes = [C.POINTER(OrcField), _i64, _f64p, _f64p]
        L.orc_integ.argtypes = [_i64, C.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, _d, C.c_int, _f64p]
        L.orc_run_steps.argtypes = [_i64, C.c_void_p, _f64p, _f64p, _f64p, _f64p, _d, C.c_int,
                                    C.c_int, _f64p, _f64p]
        L.orc_conservation.argtypes = [_i64, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_assign.argtypes = [_i64, _f64p, _f64p, _f64p, _i32p, _i32p, _i32p, _i32p, _i64]
        L.orc_scan.argtypes = [_i64, _i32p, _i32p, _i32p, _i32p]
        L.orc_cell_masses.argtypes = [_i64, _f64p, _i32p, _f64p, _i64]
        L.orc_cell_phi.argtypes = [_i64, _f64p, _i32p, _i32p, _f64p]
        L.orc_wave_iter_f64.argtypes = [C.POINTER(OrcWave), _f64p, _f64p, _f64p, _f64p]
        L.orc_wave_iter_f32.argtypes = [C.POINTER(OrcWave), _f32p, _f32p, _f32p, _f32p]
        L.orc_acc_field.argtypes = [C.c_int, _d, _f64p, _f64p]
        L.orc_gather.argtypes = [_i64, _i32p, _vp, _vp, _vp, _vp]
        L.orc_cic_deposit.argtypes = [_i64, _f64p, _f64p, _f64p, _f64p, _i32p, _f64p]
        L.orc_cic_gather.argtypes = [_i64, _f64p, _f64p, _f64p, _i32p, _vp, _vp, _vp, _vp]
        L.orc_scatter_order.argtypes = [_i64, _i32p, _i32p, _i32p, _i32p]
        L.orc_mesh_force.argtypes = [C.POINTER(OrcWave), C.c_int, C.c_int, C.c_int, _i64, _f64p, _f64p,
                                     _vp, _vp, C.POINTER(C.c_int), _f64p, _f64p]
        L.orc_max_threads.restype = C.c_int

    # -- field ------------------------------------------------------------
    def field(self, Mh=0.0, a=0.3333, Rh=1.0, Mb=0.0, b=0.0431, Rb=0.2) -> OrcField:
        f = OrcField()
        self.L.orc_field_init(C.byref(f), Mh, a, Rh, Mb, b, Rb)
        return f

    def fex(self, field: OrcField, pos):
        p = _c3(pos)
        out = np.zeros_like(p)
        self.L.orc_fex(C.byref(field), p.size // 3, p, out)
        return out.reshape(-1, 3)

    # -- direct sums --------------------------------------------------------
    def _sum(self, fn, pos, mass, eps2, targets, width):
        p = _c3(pos)
        n = p.size // 3
        t, nt = _tg(targets)
        cnt = nt if t is not None else n
        out = np.zeros(cnt * width)
        fn(n, p, np.ascontiguousarray(mass, np.float64), np.ascontiguousarray(eps2, np.float64),
           nt, t.ctypes.data if t is not None else None, out)
        return out.reshape(cnt, width) if width > 1 else out

    def accel_f64(self, pos, mass, eps2, targets=None):
        return self._sum(self.L.orc_accel_f64, pos, mass, eps2, targets, 3)

    def accel_f32(self, pos, mass, eps2, targets=None):
        return self._sum(self.L.orc_accel_f32, pos, mass, eps2, targets, 3)

    def phi_f64(self, pos, mass, eps2, targets=None):
        return self._sum(self.L.orc_phi_f64, pos, mass, eps2, targets, 1)

    # -- integrator ---------------------------------------------------------
    def integ(self, field, acc, pos_t, vel_t, pos, vel, dt, istep, acc0):
        n = pos.size // 3
        self.L.orc_integ(n, C.byref(field) if field is not None else None, acc, pos_t, vel_t,
                         pos, vel, dt, istep, acc0)

    def run_steps(self, pos, vel, mass, eps2, dt, nsteps, field=None, compat_accumulate=False,
                  acc=None, acct=None):
        """Reference time loop (nbody.cu:1525-1582); returns (pos, vel, acc, acct)."""
        p = _c3(pos).copy()
        v = _c3(vel).copy()
        n = p.size // 3
        m = np.ascontiguousarray(mass, np.float64)
        e = np.ascontiguousarray(eps2, np.float64)
        if acc is None:
            acc = self.accel_f64(p, m, e).reshape(-1)
        acc = _c3(acc).copy()
        acct = np.zeros(3 * n) if acct is None else _c3(acct).copy()
        self.L.orc_run_steps(n, C.byref(field) if field is not None else None, p, v, m, e, dt,
                             nsteps, int(compat_accumulate), acc, acct)
        return p.reshape(-1, 3), v.reshape(-1, 3), acc.reshape(-1, 3), acct.reshape(-1, 3)

    def conservation(self, pos, vel, mass, psi):
        out = np.zeros(16)
        n = _c3(pos).size // 3
        self.L.orc_conservation(n, _c3(pos), _c3(vel), np.ascontiguousarray(mass, np.float64),
                                np.ascontiguousarray(psi, np.float64), out)
        keys = ("Lx", "Ly", "Lz", "Ix", "Iy", "Iz", "Ek", "Ep", "E", "R_max", "Z_max",
                "Vr_max", "Vfi_max", "Vz_max")
        return dict(zip(keys, out[:14].tolist()))

    # -- p2mesh ---------------------------------------------------------------
    def assign(self, pos, lo, cs, grid):
        p = _c3(pos)
        n = p.size // 3
        g = np.ascontiguousarray(grid, np.int32)
        ncells = int(g[0]) * int(g[1]) * int(g[2])
        cell_id = np.zeros(n, np.int32)
        slot = np.zeros(n, np.int32)
        count = np.zeros(ncells, np.int32)
        self.L.orc_assign(n, p, np.ascontiguousarray(lo, np.float64),
                          np.ascontiguousarray(cs, np.float64), g, cell_id, slot, count, ncells)
        return cell_id, slot, count

    def scan(self, count):
        c = np.ascontiguousarray(count, np.int32)
        nb = (c.size + 511) // 512
        st = np.zeros(c.size, np.int32)
        sr = np.zeros(c.size, np.int32)
        mp = np.zeros(nb, np.int32)
        self.L.orc_scan(c.size, c, st, sr, mp)
        return st, sr, mp

    def cell_masses(self, mass, cell_id, ncells):
        out = np.zeros(ncells)
        self.L.orc_cell_masses(len(cell_id), np.ascontiguousarray(mass, np.float64),
                               np.ascontiguousarray(cell_id, np.int32), out, ncells)
        return out

    def cell_phi(self, phi, cell_id, count, cell_phi=None):
        out = np.zeros(len(count)) if cell_phi is None else np.ascontiguousarray(cell_phi, np.float64).copy()
        self.L.orc_cell_phi(len(cell_id), np.ascontiguousarray(phi, np.float64),
                            np.ascontiguousarray(cell_id, np.int32),
                            np.ascontiguousarray(count, np.int32), out)
        return out

    @staticmethod
    def wave_params(nx, dx, c=4574.337022617616, dt=None, diss_base=0.1, diss_extra=0.01,
                    sim_l=None, bc_l=None) -> OrcWave:
        """Mesh constants as nbody/src/nbody.cu:1134-1143 derives them."""
        if dt is None:
            dt = 0.5 * dx / (c * np.sqrt(3.0))
        if sim_l is None:
            sim_l = 0.5 * nx * dx
        if bc_l is None:
            bc_l = sim_l / 10.0
        return OrcWave(nx, dx, dt, c, diss_base, diss_extra, sim_l, bc_l)

    def wave_iter_f64(self, W: OrcWave, phi, phi_old, mass):
        out = np.zeros_like(phi, dtype=np.float64)
        self.L.orc_wave_iter_f64(C.byref(W), out, np.ascontiguousarray(phi, np.float64),
                                 np.ascontiguousarray(phi_old, np.float64),
                                 np.ascontiguousarray(mass, np.float64))
        return out

    def wave_iter_f32(self, W: OrcWave, phi, phi_old, mass):
        out = np.zeros(np.asarray(phi).shape, dtype=np.float32)
        self.L.orc_wave_iter_f32(C.byref(W), out, np.ascontiguousarray(phi, np.float32),
                                 np.ascontiguousarray(phi_old, np.float32),
                                 np.ascontiguousarray(mass, np.float32))
        return out

    def acc_field(self, nx, dx, phi):
        out = np.zeros(nx * nx * nx * 3)
        self.L.orc_acc_field(nx, dx, np.ascontiguousarray(phi, np.float64), out)
        return out.reshape(-1, 3)

    def gather(self, cell_id, cell_acc, cell_phi):
        n = len(cell_id)
        acc = np.zeros(3 * n)
        phi = np.zeros(n)
        ca = _c3(cell_acc)
        cp = np.ascontiguousarray(cell_phi, np.float64)
        self.L.orc_gather(n, np.ascontiguousarray(cell_id, np.int32), ca.ctypes.data,
                          cp.ctypes.data, acc.ctypes.data, phi.ctypes.data)
        return acc.reshape(-1, 3), phi

    # -- beyond the reference's NGP path -----------------------------------------
    def cic_deposit(self, pos, mass, lo, cs, grid, cell_mass=None):
        g = np.ascontiguousarray(grid, np.int32)
        ncells = int(g[0]) * int(g[1]) * int(g[2])
        out = np.zeros(ncells) if cell_mass is None else np.ascontiguousarray(cell_mass, np.float64).copy()
        p = _c3(pos)
        self.L.orc_cic_deposit(p.size // 3, p, np.ascontiguousarray(mass, np.float64),
                               np.ascontiguousarray(lo, np.float64), np.ascontiguousarray(cs, np.float64), g, out)
        return out

    def cic_gather(self, pos, lo, cs, grid, cell_acc, cell_val):
        p = _c3(pos)
        n = p.size // 3
        acc = np.zeros(3 * n)
        val = np.zeros(n)
        ca = _c3(cell_acc)
        cv = np.ascontiguousarray(cell_val, np.float64)
        self.L.orc_cic_gather(n, p, np.ascontiguousarray(lo, np.float64), np.ascontiguousarray(cs, np.float64),
                              np.ascontiguousarray(grid, np.int32), ca.ctypes.data, cv.ctypes.data,
                              acc.ctypes.data, val.ctypes.data)
        return acc.reshape(-1, 3), val

    def scatter_order(self, cell_id, slot, start):
        n = len(cell_id)
        order = np.full(n, -1, np.int32)
        self.L.orc_scatter_order(n, np.ascontiguousarray(cell_id, np.int32), np.ascontiguousarray(slot, np.int32),
                                 np.ascontiguousarray(start, np.int32), order)
        return order

    def mesh_force(self, W: OrcWave, pos, mass, iters, cic=False, fp64=True):
        """One mesh-force evaluation from a zero field (orc_mesh_force)."""
        ncells = W.nx ** 3
        ring64 = np.zeros(3 * ncells)
        ring32 = np.zeros(3 * ncells, np.float32)
        rot = C.c_int(0)
        p = _c3(pos)
        n = p.size // 3
        acc = np.zeros(3 * n)
        phi = np.zeros(n)
        self.L.orc_mesh_force(C.byref(W), int(cic), int(fp64), int(iters), n, p,
                              np.ascontiguousarray(mass, np.float64), ring64.ctypes.data, ring32.ctypes.data,
                              C.byref(rot), acc, phi)
        return acc.reshape(-1, 3), phi

    def mesh_steps(self, W: OrcWave, pos, vel, mass, dt, nsteps, iters, setup_iters, cic=False, fp64=True,
                   field=None):
        """The reference's Wave-mode run (nbody/src/nbody.cu:1449-1472 setup,
        1521-1589 per step) with the mesh force of orc_mesh_force: setup from a
        zero field, then per step predictor, acct = mesh force at the predicted
        positions, corrector.  Returns pos, vel, acc, phi after nsteps."""
        nx = W.nx
        ncells = nx ** 3
        ring64 = np.zeros(3 * ncells)
        ring32 = np.zeros(3 * ncells, np.float32)
        rot = C.c_int(0)
        pos = _c3(pos).copy()
        vel = _c3(vel).copy()
        m = np.ascontiguousarray(mass, np.float64)
        n = pos.size // 3
        acc = np.zeros(3 * n)
        phi = np.zeros(n)

        self.L.orc_mesh_force(C.byref(W), int(cic), int(fp64), setup_iters, n, pos, m, ring64.ctypes.data,
                              ring32.ctypes.data, C.byref(rot), acc, phi)
        fref = C.byref(field) if field is not None else None
        post = np.zeros_like(pos)
        velt = np.zeros_like(vel)
        acct = np.zeros(3 * n)
        for _ in range(nsteps):
            self.L.orc_integ(n, fref, acc, post, velt, pos, vel, dt, 0, acc)
            self.L.orc_mesh_force(C.byref(W), int(cic), int(fp64), iters, n, post, m, ring64.ctypes.data,
                                  ring32.ctypes.data, C.byref(rot), acct, phi)
            self.L.orc_integ(n, fref, acct, pos, vel, post, velt, dt, 1, acc)
        return pos.reshape(-1, 3), vel.reshape(-1, 3), acc.reshape(-1, 3), phi

    def max_threads(self) -> int:
        return int(self.L.orc_max_threads())


class Reference:
    """The reference's own kernels compiled for the host (oracle/_ref)."""

    def __init__(self, path: os.PathLike | None = None):
        p = pathlib.Path(path) if path else REF_SO
        if not p.exists():
            raise FileNotFoundError(f"{p} not built (needs the reference source tree)")
        L = C.CDLL(str(p))
        self.L = L
        L.ref_set_field.argtypes = [_d] * 6 + [C.c_int, C.c_int]
        L.ref_get_field_consts.argtypes = [_f64p]
        L.ref_fex.argtypes = [_i64, _f64p, _f64p]
        L.ref_accel.argtypes = [_i64, _f64p, _f64p, _f64p, _i64, _vp, _f64p]
        L.ref_accel_f32.argtypes = [_i64, _f64p, _f64p, _f64p, _i64, _vp, _f64p]
        L.ref_accel_team.argtypes = [_i64, _f64p, _f64p, _f64p, _f64p]
        L.ref_accel_team.restype = C.c_int
        L.ref_phi_team.argtypes = [_i64, _f64p, _f64p, _f64p, _f64p]
        L.ref_phi_team.restype = C.c_int
        L.ref_integ.argtypes = [_i64, _f64p, _f64p, _f64p, _f64p, _f64p, _d, C.c_int, _d, _f64p]
        L.ref_set_mesh.argtypes = [_d] * 6 + [C.c_int] * 4 + [_d] * 7
        L.ref_assign.argtypes = [_i64, _f64p, _i32p, _i32p, _i32p]
        L.ref_adjust.argtypes = [_i64, _i32p, _i32p]
        L.ref_prefix_team.argtypes = [_i64, _i32p, _i32p]
        L.ref_cell_masses.argtypes = [_i64, _f64p, _i32p, _f64p]
        L.ref_cell_phi.argtypes = [_i64, _f64p, _i32p, _i32p, _f64p]
        L.ref_wave.argtypes = [_f64p, _f64p, _f64p, _f64p]
        L.ref_acc_field.argtypes = [C.c_int, _d, _f64p, _f64p, _vp]
        L.ref_apply_acc.argtypes = [_i64, _f64p, _f64p, _i32p]
        L.ref_apply_cell.argtypes = [_i64, _f64p, _f64p, _i32p]
        L.ref_read_galaxies.argtypes = [C.c_char_p, C.c_int, _i32p, _i32p] + [_f64p] * 9
        L.ref_read_galaxies.restype = C.c_int
        L.ref_max_threads.restype = C.c_int

    def set_field(self, Mh=0.0, a=0.3333, Rh=1.0, Mb=0.0, b=0.0431, Rb=0.2, ns=0, nn=0):
        self.L.ref_set_field(Mh, a, Rh, Mb, b, Rb, ns, nn)
        out = np.zeros(4)
        self.L.ref_get_field_consts(out)
        return dict(zip(("Rh2", "con", "const1", "Mh_inf"), out.tolist()))

    def fex(self, pos):
        p = _c3(pos)
        out = np.zeros_like(p)
        self.L.ref_fex(p.size // 3, p, out)
        return out.reshape(-1, 3)

    def accel(self, pos, mass, eps2, targets=None):
        """ACCEL_kernel FP64 (blockDim 1); returns the targets' accelerations."""
        p = _c3(pos)
        n = p.size // 3
        t, nt = _tg(targets)
        acc = np.zeros(3 * n)
        self.L.ref_accel(n, p, np.ascontiguousarray(mass, np.float64),
                         np.ascontiguousarray(eps2, np.float64), nt,
                         t.ctypes.data if t is not None else None, acc)
        acc = acc.reshape(-1, 3)
        return acc[t] if t is not None else acc

    def accel_f32(self, pos, mass, eps2, targets=None):
        p = _c3(pos)
        n = p.size // 3
        t, nt = _tg(targets)
        out = np.zeros(3 * (nt if t is not None else n))
        self.L.ref_accel_f32(n, p, np.ascontiguousarray(mass, np.float64),
                             np.ascontiguousarray(eps2, np.float64), nt,
                             t.ctypes.data if t is not None else None, out)
        return out.reshape(-1, 3)

    def accel_team(self, pos, mass, eps2):
        p = _c3(pos)
        acc = np.zeros_like(p)
        if self.L.ref_accel_team(p.size // 3, p, np.ascontiguousarray(mass, np.float64),
                                 np.ascontiguousarray(eps2, np.float64), acc):
            raise ValueError("n must be a multiple of 512")
        return acc.reshape(-1, 3)

    def phi_team(self, pos, mass, eps2):
        p = _c3(pos)
        phi = np.zeros(p.size // 3)
        if self.L.ref_phi_team(p.size // 3, p, np.ascontiguousarray(mass, np.float64),
                               np.ascontiguousarray(eps2, np.float64), phi):
            raise ValueError("n must be a multiple of 512")
        return phi

    def integ(self, acc, pos_t, vel_t, pos, vel, dt, istep, t, acc0):
        self.L.ref_integ(pos.size // 3, acc, pos_t, vel_t, pos, vel, dt, istep, t, acc0)

    def set_mesh(self, lo, cs, grid, nx_wave=0, dx_wave=0.0, dt_wave=0.0, c_wave=0.0,
                 diss_base=0.0, diss_extra=0.0, sim_l=0.0, bc_l=0.0):
        self.L.ref_set_mesh(lo[0], lo[1], lo[2], cs[0], cs[1], cs[2], int(grid[0]), int(grid[1]),
                            int(grid[2]), nx_wave, dx_wave, dt_wave, c_wave, diss_base,
                            diss_extra, sim_l, bc_l)

    def bin(self, pos, mass, ncells):
        """assign + computePrefixSums + adjustGlobalPrefixSums + cell masses,
        with the arrays zeroed first, as convert_particles_to_grid does
        (nbody/src/nbody.cu:139-181)."""
        p = _c3(pos)
        n = p.size // 3
        pci = np.zeros(2 * n, np.int32)
        ci = np.zeros(2 * ncells, np.int32)
        cnt = np.zeros(ncells, np.int32)
        nb = (ncells + 511) // 512
        maxpbc = np.zeros(nb, np.int32)
        cm = np.zeros(ncells)
        self.L.ref_assign(n, p, pci, ci, cnt)
        self.L.ref_prefix_team(ncells, ci, maxpbc)
        self.L.ref_adjust(ncells, ci, maxpbc)
        self.L.ref_cell_masses(n, np.ascontiguousarray(mass, np.float64), pci, cm)
        return dict(cell_id=pci[0::2].copy(), id_in_cell=pci[1::2].copy(), count=ci[0::2].copy(),
                    start_id=ci[1::2].copy(), slot_count=cnt, maxpbc=maxpbc, cell_mass=cm,
                    pci=pci, cell_info=ci)

    def cell_phi(self, phi, pci, cell_info, ncells):
        out = np.zeros(ncells)
        self.L.ref_cell_phi(len(phi), np.ascontiguousarray(phi, np.float64), pci, cell_info, out)
        return out

    def wave(self, phi, phi_old, mass):
        out = np.zeros_like(phi, dtype=np.float64)
        self.L.ref_wave(out, np.ascontiguousarray(phi, np.float64),
                        np.ascontiguousarray(phi_old, np.float64),
                        np.ascontiguousarray(mass, np.float64))
        return out

    def acc_field(self, nx, dx, phi):
        out = np.zeros(nx ** 3 * 3)
        self.L.ref_acc_field(nx, dx, np.ascontiguousarray(phi, np.float64), out, None)
        return out.reshape(-1, 3)

    def apply(self, pci, cell_acc, cell_phi):
        n = len(pci) // 2
        acc = np.zeros(3 * n)
        phi = np.zeros(n)
        self.L.ref_apply_acc(n, acc, _c3(cell_acc), pci)
        self.L.ref_apply_cell(n, phi, np.ascontiguousarray(cell_phi, np.float64), pci)
        return acc.reshape(-1, 3), phi

    def read_galaxies(self, path, maxg=64):
        ns = np.zeros(maxg, np.int32)
        nd = np.zeros(maxg, np.int32)
        arrs = [np.zeros(maxg) for _ in range(5)] + [np.zeros(3 * maxg), np.zeros(3 * maxg)] + \
               [np.zeros(maxg), np.zeros(maxg)]
        k = self.L.ref_read_galaxies(str(path).encode(), maxg, ns, nd, *arrs)
        if k < 0:
            raise OSError(f"reference reader failed on {path}")
        ms, md, es, ed, ang, cen, vel, mbs, mbd = arrs
        return [dict(n_star=int(ns[i]), n_dark=int(nd[i]), m_star=ms[i], m_dark=md[i],
                     eps_star=es[i], eps_dark=ed[i], angle=ang[i], centre=tuple(cen[3 * i:3 * i + 3]),
                     vel=tuple(vel[3 * i:3 * i + 3]), m_star_body=mbs[i], m_dark_body=mbd[i])
                for i in range(min(k, maxg))]

    def max_threads(self) -> int:
        return int(self.L.ref_max_threads())
