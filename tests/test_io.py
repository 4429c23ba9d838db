"""The drop-in file surface (no GPU): the .ini readers against the reference's
own parser, start_*.txt / snapshot / LIE_0.bin layouts and round trips, and
the initial-condition load (tilt, shift, masses, reference body order)."""
import ctypes as C
import json
import math
import os
import pathlib
import struct

import numpy as np
import pytest

from conftest import GOLDEN

# The reference project's own .ini files, when its tree is given by
# KHRR_REFERENCE (the project root, as oracle/Makefile's REF); the tests that
# read them are skipped without it.
_REF = os.environ.get("KHRR_REFERENCE")
REF_INI = pathlib.Path(_REF) / "data" / "nbody" / "ini" if _REF else None


class Galaxy(C.Structure):
    _fields_ = [("n_star", C.c_int), ("n_dark", C.c_int), ("m_star", C.c_double), ("m_dark", C.c_double),
                ("eps_star", C.c_double), ("eps_dark", C.c_double), ("angle_deg", C.c_double),
                ("centre", C.c_double * 3), ("vel", C.c_double * 3)]


class Lie(C.Structure):
    _fields_ = [("L", C.c_double * 3), ("Imp", C.c_double * 3)] + [
        (k, C.c_double) for k in ("Ek", "Ep", "E", "R_max", "Z_max", "Vr_max", "Vfi_max", "Vz_max")]


@pytest.fixture(scope="module")
def L(libkhrr):
    import khrr
    return khrr.lib()  # with the C signatures (64-bit pointers)


def read_galaxies(L, path):
    out = (Galaxy * 64)()
    cnt = C.c_int()
    st = L.khrr_read_galaxies_ini(str(path).encode(), out, 64, C.byref(cnt))
    return st, [out[i] for i in range(min(cnt.value, 64))]


def test_galaxies_ini_matches_reference_parser(L, tmp_path):
    d = json.loads((GOLDEN / "galaxies_ini.json").read_text())["two_galaxies"]
    p = tmp_path / "__start_galaxies.ini"
    p.write_text(d["text"])
    st, gals = read_galaxies(L, p)
    assert st == 0 and len(gals) == len(d["parsed"])
    for g, r in zip(gals, d["parsed"]):
        assert g.n_star == r["n_star"] and g.n_dark == r["n_dark"]
        assert g.m_star == r["m_star"] and g.m_dark == r["m_dark"]
        assert g.eps_star == r["eps_star"] and g.eps_dark == r["eps_dark"]
        assert g.angle_deg == r["angle"]
        assert tuple(g.centre) == tuple(r["centre"]) and tuple(g.vel) == tuple(r["vel"])
        if g.n_star:
            assert g.m_star / g.n_star == r["m_star_body"]
        if g.n_dark:
            assert g.m_dark / g.n_dark == r["m_dark_body"]


@pytest.mark.skipif(REF_INI is None or not REF_INI.exists(),
                    reason="KHRR_REFERENCE does not name the reference tree")
def test_shipped_ini_files(L):
    import pyoracle
    st, gals = read_galaxies(L, REF_INI / "__start_galaxies.ini")
    assert st == 0
    try:
        ref = pyoracle.Reference().read_galaxies(REF_INI / "__start_galaxies.ini")
    except FileNotFoundError:
        ref = None
    if ref is not None:
        assert [(g.n_star, g.n_dark, g.m_star, g.m_dark) for g in gals] == \
               [(r["n_star"], r["n_dark"], r["m_star"], r["m_dark"]) for r in ref]
    i_cont, tmax, dts = C.c_int(), C.c_double(), C.c_double()
    assert L.khrr_read_start_nbody_ini(str(REF_INI / "__start_nbody.ini").encode(), C.byref(i_cont),
                                       C.byref(tmax), C.byref(dts)) == 0
    assert (i_cont.value, tmax.value, dts.value) == (0, 30.0, 0.01)
    field = (C.c_double * 6)()
    eps, dtg, km, kr = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    assert L.khrr_read_gr_par_ini(str(REF_INI / "__gr_par.ini").encode(), field, C.byref(eps), C.byref(dtg),
                                  C.byref(km), C.byref(kr)) == 0
    assert list(field) == [0.0, 0.3333, 1.0, 0.0, 0.0431, 0.2]
    assert (eps.value, dtg.value, km.value, kr.value) == (0.004, 0.002, 3.72, 0.9)
    ngpu = C.c_int()
    devs = (C.c_int * 4)()
    assert L.khrr_read_gpus_ini(str(REF_INI / "__GPUs.ini").encode(), C.byref(ngpu), devs, 4) == 0
    assert ngpu.value == 1 and devs[0] == 0


def test_missing_and_malformed_files(L, tmp_path):
    st, _ = read_galaxies(L, tmp_path / "nope.ini")
    assert st == 4  # KHRR_ERR_IO
    bad = tmp_path / "bad.ini"
    bad.write_text("2\t--- M_glx\n0\t--- k\n100,200\t--- N\n")
    st, _ = read_galaxies(L, bad)
    assert st == 4
    n, t = C.c_int64(), C.c_double()
    pos = np.zeros(30)
    vel = np.zeros(30)
    trunc = tmp_path / "start.txt"
    trunc.write_text("10 0.0\n0 0 0 1 1 1\n")
    assert L.khrr_read_start_txt(str(trunc).encode(), 10, pos.ctypes.data, vel.ctypes.data, C.byref(n),
                                 C.byref(t)) == 4


def test_start_txt_round_trip(L, tmp_path):
    rng = np.random.default_rng(1)
    pos, vel = rng.normal(size=(100, 3)), rng.normal(size=(100, 3))
    p = tmp_path / "start_S0.txt"
    assert L.khrr_write_start_txt(str(p).encode(), 100, pos.ctypes.data, vel.ctypes.data, C.c_double(0.0)) == 0
    assert p.read_text().splitlines()[0] == "100 0.000000"
    P, V = np.zeros((100, 3)), np.zeros((100, 3))
    n, t = C.c_int64(), C.c_double()
    assert L.khrr_read_start_txt(str(p).encode(), 100, P.ctypes.data, V.ctypes.data, C.byref(n), C.byref(t)) == 0
    assert n.value == 100 and np.array_equal(P, pos) and np.array_equal(V, vel)
    # The shipped format ("N t", six columns with 6 decimals) reads the same way.
    q = tmp_path / "ref.txt"
    q.write_text("2 0.000000\n0.000035 0.000047 0.001940 -0.436802 1.265211 0.188578\n"
                 "0.004109 -0.032145 -0.000168 0.709329 -0.256181 0.276377\n")
    assert L.khrr_read_start_txt(str(q).encode(), 2, P.ctypes.data, V.ctypes.data, C.byref(n), C.byref(t)) == 0
    assert P[0, 2] == 0.001940 and V[1, 0] == 0.709329


def test_snapshot_layout_and_round_trip(L, tmp_path):
    rng = np.random.default_rng(2)
    pos, vel = rng.normal(size=(7, 3)), rng.normal(size=(7, 3))
    p = tmp_path / "S_   10.bin"
    assert L.khrr_write_snapshot(str(p).encode(), 7, C.c_double(0.25), pos.ctypes.data, vel.ctypes.data) == 0
    raw = p.read_bytes()
    assert len(raw) == 4 + 8 + 7 * 48
    assert struct.unpack("<i", raw[:4])[0] == 7 and struct.unpack("<d", raw[4:12])[0] == 0.25
    rec = np.frombuffer(raw[12:], dtype="<f8").reshape(7, 6)
    assert np.array_equal(rec[:, :3], pos) and np.array_equal(rec[:, 3:], vel)
    P, V = np.zeros((7, 3)), np.zeros((7, 3))
    cnt, t = C.c_int32(), C.c_double()
    assert L.khrr_read_snapshot(str(p).encode(), 7, P.ctypes.data, V.ctypes.data, C.byref(cnt), C.byref(t)) == 0
    assert cnt.value == 7 and t.value == 0.25 and np.array_equal(P, pos) and np.array_equal(V, vel)


def test_lie0_layout(L, tmp_path):
    lie = Lie()
    lie.L[0], lie.L[1], lie.L[2] = 1.0, 2.0, 3.0
    lie.Imp[0], lie.Imp[1], lie.Imp[2] = 4.0, 5.0, 6.0
    lie.E = -7.5
    p = tmp_path / "LIE_0.bin"
    assert L.khrr_write_lie0(str(p).encode(), C.byref(lie)) == 0
    raw = p.read_bytes()
    assert len(raw) == 72  # L0, Imp0 and E0 written with sizeof(double3)
    assert struct.unpack("<7d", raw[:56]) == (1.0, 2.0, 3.0, 4.0, 5.0, 6.0, -7.5)
    back = Lie()
    assert L.khrr_read_lie0(str(p).encode(), C.byref(back)) == 0
    assert list(back.L) == [1.0, 2.0, 3.0] and back.E == -7.5


def test_initial_conditions_load(L, tmp_path):
    """Two galaxies (the second tilted 30 degrees, one without dark matter):
    the reference body order and its tilt/shift formula."""
    from khrr.galaxy import make_galaxy, place
    g1 = make_galaxy(256, 512, 31)
    g2 = make_galaxy(128, 0, 32, eps_stars=0.002)
    for k, g in enumerate((g1, g2)):
        for comp, (p, v) in (("S", (g.star_pos, g.star_vel)), ("DM", (g.dm_pos, g.dm_vel))):
            if len(p):
                L.khrr_write_start_txt(str(tmp_path / f"start_{comp}{k}.txt").encode(), len(p),
                                       np.ascontiguousarray(p).ctypes.data, np.ascontiguousarray(v).ctypes.data,
                                       C.c_double(0.0))
    (tmp_path / "__start_galaxies.ini").write_text(
        "2 --- M\n0 --- k\n256,512 --- N\n1.0,6.699356 --- M\n0.004,0.004 --- eps\n0.0 --- a\n"
        "1.5,0.0,0.0 --- X\n-0.3,0.1,0.0 --- V\n"
        "1 --- k\n128,64 --- N\n1.0,0.0 --- M\n0.002,0.004 --- eps\n30.0 --- a\n"
        "-1.5,0.0,0.0 --- X\n0.3,-0.1,0.0 --- V\n")
    st, gals = read_galaxies(L, tmp_path / "__start_galaxies.ini")
    assert st == 0 and gals[1].n_dark == 0  # massless component has no bodies
    arr = (Galaxy * 2)(*gals)
    nmax = 1000
    pos, vel = np.zeros((nmax, 3)), np.zeros((nmax, 3))
    mass, eps2 = np.zeros(nmax), np.zeros(nmax)
    n, ns = C.c_int64(), C.c_int64()
    assert L.khrr_load_initial_conditions(str(tmp_path).encode(), arr, 2, nmax, pos.ctypes.data, vel.ctypes.data,
                                          mass.ctypes.data, eps2.ctypes.data, C.byref(n), C.byref(ns)) == 0
    assert n.value == 256 + 512 + 128 and ns.value == 384
    p1, v1 = place(g1.star_pos, g1.star_vel, 0.0, (1.5, 0, 0), (-0.3, 0.1, 0))
    p2, v2 = place(g2.star_pos, g2.star_vel, 30.0, (-1.5, 0, 0), (0.3, -0.1, 0))
    pd, vd = place(g1.dm_pos, g1.dm_vel, 0.0, (1.5, 0, 0), (-0.3, 0.1, 0))
    assert np.array_equal(pos[:896], np.concatenate([p1, p2, pd]))
    assert np.array_equal(vel[:896], np.concatenate([v1, v2, vd]))
    assert np.all(mass[:256] == 1.0 / 256) and np.all(mass[256:384] == 1.0 / 128)
    assert np.all(mass[384:896] == 6.699356 / 512)
    assert np.all(eps2[256:384] == 0.002 ** 2) and np.all(eps2[:256] == 0.004 ** 2)
    # the tilt is the reference's shear: z uses the already rotated x
    c, s = math.cos(30 * 3.14159265358979 / 180), math.sin(30 * 3.14159265358979 / 180)
    x0, z0 = g2.star_pos[0, 0], g2.star_pos[0, 2]
    xn = -1.5 + x0 * c + z0 * s
    assert pos[256, 2] == 0.0 + z0 * c - xn * s
