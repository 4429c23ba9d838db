"""Python binding of libkhrr (include/khrr.h) over ctypes.

This is the host-side mirror of the reference's time loop for tests and
benchmarks: numpy arrays in the reference's layouts (AoS xyz float64
positions/velocities, float64 masses and eps^2) go through the C ABI; all
compute runs in the library's CUDA kernels.  There is no CPU fallback: if
``build/libkhrr.so`` is missing or cannot create a context, calls raise.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parents[1]
LIB_PATH = PKG_DIR / "build" / "libkhrr.so"

ACC = 1
PHI = 2
COMPAT_ACCUMULATE = 4
PLAIN = 8
OVERWRITE = 16
MESH = 32
FP64 = 64
ASSIGN_NGP = 0
ASSIGN_CIC = 1

STATUS = {0: "KHRR_OK", 1: "KHRR_ERR_INVALID_ARG", 2: "KHRR_ERR_NOT_MULTIPLE", 3: "KHRR_ERR_CUDA",
          4: "KHRR_ERR_IO", 5: "KHRR_ERR_TIMEOUT", 6: "KHRR_ERR_STATE", 7: "KHRR_ERR_OOM",
          8: "KHRR_ERR_UNSUPPORTED", 9: "KHRR_ERR_TOO_LARGE"}


class KhrrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class FieldParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("Mh", "a", "Rh", "Mb", "b", "Rb")]


class Lie(C.Structure):
    _fields_ = [("L", C.c_double * 3), ("Imp", C.c_double * 3)] + [
        (k, C.c_double) for k in ("Ek", "Ep", "E", "R_max", "Z_max", "Vr_max", "Vfi_max", "Vz_max")]

    def as_dict(self):
        d = {"Lx": self.L[0], "Ly": self.L[1], "Lz": self.L[2],
             "Ix": self.Imp[0], "Iy": self.Imp[1], "Iz": self.Imp[2]}
        for k in ("Ek", "Ep", "E", "R_max", "Z_max", "Vr_max", "Vfi_max", "Vz_max"):
            d[k] = getattr(self, k)
        return d


class Tuning(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("threads", "i_per_thread", "j_tile", "j_split", "packed")]


class Mesh(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("cell", C.c_double * 3), ("grid", C.c_int * 3)]

    @classmethod
    def make(cls, lo, cell, grid):
        m = cls()
        for k in range(3):
            m.lo[k], m.cell[k], m.grid[k] = float(lo[k]), float(cell[k]), int(grid[k])
        return m


class WaveParams(C.Structure):
    _fields_ = [("nx", C.c_int)] + [(k, C.c_double) for k in (
        "dx", "dt", "c", "diss_base", "diss_extra", "sim_l", "bc_l")]

    @classmethod
    def make(cls, nx, dx, c=4574.337022617616, dt=None, diss_base=0.1, diss_extra=0.01,
             sim_l=None, bc_l=None):
        """Constants as the reference derives them (nbody/src/nbody.cu:1134-1143)."""
        if dt is None:
            dt = 0.5 * dx / (c * np.sqrt(3.0))
        if sim_l is None:
            sim_l = 0.5 * nx * dx
        if bc_l is None:
            bc_l = sim_l / 10.0
        return cls(int(nx), dx, dt, c, diss_base, diss_extra, sim_l, bc_l)


class MeshSolver(C.Structure):
    _fields_ = [("wave", WaveParams), ("assign", C.c_int), ("fp64", C.c_int), ("iters_per_step", C.c_int),
                ("setup_iters", C.c_int)]


SCAN_REFERENCE = 0
SCAN_EXCLUSIVE = 1


_lib = None


def lib(path: pathlib.Path | str | None = None) -> C.CDLL:
    """Load libkhrr (the in-tree build) once."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run `make -C {PKG_DIR}` (or __graft_entry__.build())")
    L = C.CDLL(str(p))
    vp, i64, d, i = C.c_void_p, C.c_int64, C.c_double, C.c_int
    sigs = {
        "khrr_abi_version": ([], i),
        "khrr_status_name": ([i], C.c_char_p),
        "khrr_create": ([i, C.POINTER(vp)], i),
        "khrr_destroy": ([vp], None),
        "khrr_last_error": ([vp], C.c_char_p),
        "khrr_get_stream": ([vp], vp),
        "khrr_set_stream": ([vp, vp], i),
        "khrr_synchronize": ([vp], i),
        "khrr_accel": ([vp, vp, vp, vp, vp, vp, i64, i], i),
        "khrr_phi": ([vp, vp, vp, vp, vp, vp, i64, i], i),
        "khrr_integ_time": ([vp, vp, vp, vp, vp, vp, d, i, d, vp, i64], i),
        "khrr_set_external_field": ([vp, C.POINTER(FieldParams)], i),
        "khrr_upload_state": ([vp, i64, vp, vp, vp, vp, i, vp], i),
        "khrr_download_state": ([vp, vp, vp, vp, vp], i),
        "khrr_forces": ([vp, i], i),
        "khrr_step": ([vp, d, i, i], i),
        "khrr_conservation": ([vp, C.POINTER(Lie)], i),
        "khrr_set_tuning": ([vp, C.POINTER(Tuning)], i),
        "khrr_get_tuning": ([vp, C.POINTER(Tuning)], i),
        "khrr_autotune": ([vp, C.c_char_p], i),
        "khrr_call_timing": ([vp, C.POINTER(C.c_double)], i),
        "khrr_enable_timing": ([vp, i], i),
        "khrr_force_timing": ([vp, C.POINTER(d), C.POINTER(i64), C.POINTER(d)], i),
        "khrr_pair_count": ([vp, C.POINTER(d)], i),
        "khrr_fp32_probe": ([vp, C.POINTER(d)], i),
        "khrr_set_accelerations": ([vp, vp], i),
        "khrr_accel_fp64_sample": ([vp, vp, i64, vp, vp], i),
        "khrr_assign_particles_to_cells": ([vp, vp, i64, C.POINTER(Mesh), vp, vp, vp, vp, vp], i),
        "khrr_compute_prefix_sums": ([vp, vp, vp, i64, i], i),
        "khrr_cell_phi": ([vp, vp, vp, vp, i64, vp], i),
        "khrr_wave_iteration": ([vp, vp, vp, vp, vp, C.POINTER(WaveParams)], i),
        "khrr_acc_field": ([vp, vp, vp, vp, i, d], i),
        "khrr_apply_cells_to_particles": ([vp, vp, vp, vp, vp, vp, i64], i),
        "khrr_bin": ([vp, C.POINTER(Mesh), vp, vp, vp, vp, vp, vp], i),
        "khrr_wave_solve": ([vp, C.POINTER(WaveParams), d, i, i, i, C.POINTER(i), C.POINTER(d), vp], i),
        "khrr_bin_cell_phi": ([vp, i, vp], i),
        "khrr_accel_noalloc": ([vp, vp, vp, vp, vp, i64, i, vp], i),
        "khrr_probe_bounded_wait": ([vp, d], i),
        "khrr_probe_resident_wave": ([vp, d], i),
        "khrr_cic_deposit": ([vp, vp, vp, i64, C.POINTER(Mesh), vp], i),
        "khrr_cic_gather": ([vp, vp, i64, C.POINTER(Mesh), vp, vp, vp, vp], i),
        "khrr_sort_by_cell": ([vp, vp], i),
        "khrr_set_mesh_solver": ([vp, C.POINTER(MeshSolver)], i),
        "khrr_mesh_solver_phi": ([vp, vp], i),
        # host-only file surface
        "khrr_read_galaxies_ini": ([C.c_char_p, vp, i, C.POINTER(i)], i),
        "khrr_read_start_nbody_ini": ([C.c_char_p, C.POINTER(i), C.POINTER(d), C.POINTER(d)], i),
        "khrr_read_gr_par_ini": ([C.c_char_p, vp, C.POINTER(d), C.POINTER(d), C.POINTER(d), C.POINTER(d)], i),
        "khrr_read_gpus_ini": ([C.c_char_p, C.POINTER(i), vp, i], i),
        "khrr_read_start_txt": ([C.c_char_p, i64, vp, vp, C.POINTER(i64), C.POINTER(d)], i),
        "khrr_write_start_txt": ([C.c_char_p, i64, vp, vp, d], i),
        "khrr_write_snapshot": ([C.c_char_p, C.c_int32, d, vp, vp], i),
        "khrr_read_snapshot": ([C.c_char_p, i64, vp, vp, C.POINTER(C.c_int32), C.POINTER(d)], i),
        "khrr_write_lie0": ([C.c_char_p, vp], i),
        "khrr_read_lie0": ([C.c_char_p, vp], i),
        "khrr_load_initial_conditions": ([C.c_char_p, vp, i, i64, vp, vp, vp, vp, C.POINTER(i64),
                                          C.POINTER(i64)], i),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _f64(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def _ptr(a):
    """numpy array -> its data pointer; raw integer addresses pass through."""
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """One libkhrr context on one CUDA device (its own stream)."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = C.c_void_p()
        st = self.L.khrr_create(device, C.byref(h))
        if st != 0:
            raise KhrrError(st, f"khrr_create(device={device}) failed")
        self.h = h
        self.n = 0
        self.offsets = None

    # -- plumbing -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.khrr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            raise KhrrError(st, (self.L.khrr_last_error(self.h) or b"").decode())

    @property
    def stream(self) -> int:
        return int(self.L.khrr_get_stream(self.h) or 0)

    def set_stream(self, stream_ptr: int | None):
        self._check(self.L.khrr_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self):
        self._check(self.L.khrr_synchronize(self.h))

    # -- kernel-level (device pointers as integers) ---------------------------
    def accel(self, acc_ptr, pos_i_ptr, pos_j_ptr, mass_ptr, eps2_ptr, n, flags=0):
        self._check(self.L.khrr_accel(self.h, acc_ptr, pos_i_ptr, pos_j_ptr, mass_ptr, eps2_ptr, n, flags))

    def phi(self, phi_ptr, pos_i_ptr, pos_j_ptr, mass_ptr, eps2_ptr, n, flags=0):
        self._check(self.L.khrr_phi(self.h, phi_ptr, pos_i_ptr, pos_j_ptr, mass_ptr, eps2_ptr, n, flags))

    def integ_time(self, acc, pos_t, vel_t, pos, vel, dt, istep, t, acc0, n):
        self._check(self.L.khrr_integ_time(self.h, acc, pos_t, vel_t, pos, vel, dt, istep, t, acc0, n))

    # -- simulation-level -------------------------------------------------------
    def set_external_field(self, Mh=0.0, a=0.3333, Rh=1.0, Mb=0.0, b=0.0431, Rb=0.2, enable=True):
        if not enable:
            self._check(self.L.khrr_set_external_field(self.h, None))
            return
        p = FieldParams(Mh, a, Rh, Mb, b, Rb)
        self._check(self.L.khrr_set_external_field(self.h, C.byref(p)))

    def upload(self, pos, vel, mass, eps2, offsets=None):
        pos = _f64(pos).reshape(-1)
        vel = _f64(vel).reshape(-1)
        mass = _f64(mass)
        eps2 = _f64(eps2)
        n = mass.size
        if pos.size != 3 * n or vel.size != 3 * n or eps2.size != n:
            raise ValueError("pos/vel must be n x 3 and mass/eps2 n")
        off = None
        nsys = 1
        if offsets is not None:
            off = np.ascontiguousarray(offsets, dtype=np.int64)
            nsys = off.size - 1
        self._check(self.L.khrr_upload_state(self.h, n, _ptr(pos), _ptr(vel), _ptr(mass), _ptr(eps2),
                                             nsys, _ptr(off)))
        self.n = n
        self.offsets = off

    def download(self, pos=True, vel=True, acc=True, phi=True):
        n = self.n
        out = {}
        P = np.empty((n, 3)) if pos else None
        V = np.empty((n, 3)) if vel else None
        A = np.empty((n, 3)) if acc else None
        F = np.empty(n) if phi else None
        self._check(self.L.khrr_download_state(self.h, _ptr(P), _ptr(V), _ptr(A), _ptr(F)))
        for k, v in (("pos", P), ("vel", V), ("acc", A), ("phi", F)):
            if v is not None:
                out[k] = v
        return out

    def download_into(self, pos=None, vel=None, acc=None, phi=None):
        """Download into caller-provided (e.g. pinned) float64 buffers."""
        self._check(self.L.khrr_download_state(self.h, _ptr(pos), _ptr(vel), _ptr(acc), _ptr(phi)))

    def upload_ptrs(self, n, pos, vel, mass, eps2, nsys=1, offsets_ptr=None):
        """Upload from raw host pointers (pinned buffers in the e2e benchmark)."""
        self._check(self.L.khrr_upload_state(self.h, n, pos, vel, mass, eps2, nsys, offsets_ptr))
        self.n = n

    def set_accelerations(self, acc):
        a = _f64(acc).reshape(-1)
        self._check(self.L.khrr_set_accelerations(self.h, _ptr(a)))

    def set_accelerations_ptr(self, acc_ptr):
        self._check(self.L.khrr_set_accelerations(self.h, acc_ptr))

    def accel_fp64_sample(self, targets):
        """FP64 direct sum on the GPU for the given body indices -> (acc, phi)."""
        t = np.ascontiguousarray(targets, dtype=np.int64)
        acc = np.empty((t.size, 3))
        phi = np.empty(t.size)
        self._check(self.L.khrr_accel_fp64_sample(self.h, _ptr(t), t.size, _ptr(acc), _ptr(phi)))
        return acc, phi

    def forces(self, flags=ACC):
        self._check(self.L.khrr_forces(self.h, flags))

    def step(self, dt, nsteps=1, flags=0):
        self._check(self.L.khrr_step(self.h, dt, nsteps, flags))

    def conservation(self) -> dict:
        out = Lie()
        self._check(self.L.khrr_conservation(self.h, C.byref(out)))
        return out.as_dict()

    def set_tuning(self, threads=128, i_per_thread=4, j_tile=128, j_split=0, packed=1):
        t = Tuning(threads, i_per_thread, j_tile, j_split, packed)
        self._check(self.L.khrr_set_tuning(self.h, C.byref(t)))

    def get_tuning(self) -> dict:
        t = Tuning()
        self._check(self.L.khrr_get_tuning(self.h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def autotune(self, cache_path=None):
        self._check(self.L.khrr_autotune(self.h, str(cache_path).encode() if cache_path else None))

    def enable_timing(self, on=True):
        self._check(self.L.khrr_enable_timing(self.h, 1 if on else 0))

    def force_timing(self):
        ms = C.c_double()
        launches = C.c_int64()
        pairs = C.c_double()
        self._check(self.L.khrr_force_timing(self.h, C.byref(ms), C.byref(launches), C.byref(pairs)))
        return ms.value, launches.value, pairs.value

    def call_timing(self) -> float:
        """Device milliseconds of the last timed khrr_bin / khrr_bin_cell_phi /
        khrr_sort_by_cell (timing enabled), without its downloads and host sync."""
        ms = C.c_double()
        self._check(self.L.khrr_call_timing(self.h, C.byref(ms)))
        return ms.value

    def pair_count(self) -> float:
        p = C.c_double()
        self._check(self.L.khrr_pair_count(self.h, C.byref(p)))
        return p.value

    def fp32_probe(self) -> float:
        t = C.c_double()
        self._check(self.L.khrr_fp32_probe(self.h, C.byref(t)))
        return t.value

    # -- p2mesh ----------------------------------------------------------------
    def assign_particles_to_cells(self, pos_ptr, n, mesh: Mesh, pci_ptr, cell_info_ptr,
                                  cell_count_ptr=None, mass_ptr=None, cell_mass_ptr=None):
        self._check(self.L.khrr_assign_particles_to_cells(self.h, pos_ptr, n, C.byref(mesh), pci_ptr,
                                                          cell_info_ptr, cell_count_ptr, mass_ptr,
                                                          cell_mass_ptr))

    def compute_prefix_sums(self, cell_info_ptr, max_pbc_ptr, ncells, mode=SCAN_REFERENCE):
        self._check(self.L.khrr_compute_prefix_sums(self.h, cell_info_ptr, max_pbc_ptr, ncells, mode))

    def cell_phi(self, phi_ptr, pci_ptr, cell_info_ptr, n, cell_phi_ptr):
        self._check(self.L.khrr_cell_phi(self.h, phi_ptr, pci_ptr, cell_info_ptr, n, cell_phi_ptr))

    def wave_iteration(self, phi_new_ptr, phi_ptr, phi_old_ptr, mass_ptr, params: WaveParams):
        self._check(self.L.khrr_wave_iteration(self.h, phi_new_ptr, phi_ptr, phi_old_ptr, mass_ptr,
                                               C.byref(params)))

    def acc_field(self, cell_acc_ptr, cell_acc_abs_ptr, cell_phi_ptr, nx, dx):
        self._check(self.L.khrr_acc_field(self.h, cell_acc_ptr, cell_acc_abs_ptr, cell_phi_ptr, nx, dx))

    def apply_cells_to_particles(self, pacc_ptr, pval_ptr, cacc_ptr, cval_ptr, pci_ptr, n):
        self._check(self.L.khrr_apply_cells_to_particles(self.h, pacc_ptr, pval_ptr, cacc_ptr, cval_ptr,
                                                         pci_ptr, n))

    def bin(self, lo, cell, grid):
        """Bin the uploaded bodies -> dict(cell_id, id_in_cell, count, start, start_ref, cell_mass)."""
        m = Mesh.make(lo, cell, grid)
        ncells = int(grid[0]) * int(grid[1]) * int(grid[2])
        out = {"cell_id": np.empty(self.n, np.int32), "id_in_cell": np.empty(self.n, np.int32),
               "count": np.empty(ncells, np.int32), "start": np.empty(ncells, np.int32),
               "start_ref": np.empty(ncells, np.int32), "cell_mass": np.empty(ncells)}
        self._check(self.L.khrr_bin(self.h, C.byref(m), *[_ptr(out[k]) for k in (
            "cell_id", "id_in_cell", "count", "start", "start_ref", "cell_mass")]))
        return out

    def cic_deposit(self, pos_ptr, mass_ptr, n, mesh: Mesh, cell_mass_ptr):
        self._check(self.L.khrr_cic_deposit(self.h, _ptr(pos_ptr), _ptr(mass_ptr), n, C.byref(mesh),
                                            _ptr(cell_mass_ptr)))

    def cic_gather(self, pos_ptr, n, mesh: Mesh, cell_acc_ptr, cell_val_ptr, pacc_ptr, pval_ptr):
        self._check(self.L.khrr_cic_gather(self.h, _ptr(pos_ptr), n, C.byref(mesh), _ptr(cell_acc_ptr),
                                           _ptr(cell_val_ptr), _ptr(pacc_ptr), _ptr(pval_ptr)))

    def sort_by_cell(self, want=True):
        """Counting-sort order of the last bin (body indices by cell)."""
        order = np.empty(self.n, np.int32) if want else None
        self._check(self.L.khrr_sort_by_cell(self.h, _ptr(order)))
        return order

    def set_mesh_solver(self, params: WaveParams | None, assign=ASSIGN_NGP, fp64=False, iters_per_step=None,
                        setup_iters=20000, dt=0.002):
        """The reference's Wave mode; iters_per_step defaults to (int)(dt / params.dt)."""
        if params is None:
            self._check(self.L.khrr_set_mesh_solver(self.h, None))
            return
        if iters_per_step is None:
            iters_per_step = int(dt / params.dt)
        ms = MeshSolver(params, int(assign), 1 if fp64 else 0, int(iters_per_step), int(setup_iters))
        self._check(self.L.khrr_set_mesh_solver(self.h, C.byref(ms)))

    def probe_bounded_wait(self, seconds=0.2) -> int:
        """Status of the library's bounded-wait failure path (KHRR_ERR_TIMEOUT
        = 5 when it works); raises nothing."""
        return int(self.L.khrr_probe_bounded_wait(self.h, float(seconds)))

    def probe_resident_wave(self, seconds=0.2) -> int:
        """khrr_probe_resident_wave: the cooperative 128^3 stencil with one brick
        withholding its counter; returns the status (KHRR_ERR_TIMEOUT expected)."""
        return int(self.L.khrr_probe_resident_wave(self.h, float(seconds)))

    def mesh_solver_phi(self, nx):
        out = np.empty(nx ** 3)
        self._check(self.L.khrr_mesh_solver_phi(self.h, _ptr(out)))
        return out

    def wave_solve(self, params: WaveParams, tol=1e-5, max_iter=1000, check_every=30, cold=False,
                   want_phi=True):
        it = C.c_int()
        res = C.c_double()
        phi = np.empty(params.nx ** 3, np.float32) if want_phi else None
        self._check(self.L.khrr_wave_solve(self.h, C.byref(params), tol, max_iter, check_every,
                                           1 if cold else 0, C.byref(it), C.byref(res), _ptr(phi)))
        return it.value, res.value, phi
