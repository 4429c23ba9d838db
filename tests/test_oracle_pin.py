"""Pin the oracle restatement (oracle/oracle.c) to the reference's own output.

The fixtures in tests/golden/ were produced by tests/golden/make_golden.py
running the reference's kernels compiled for the host (oracle/_ref).  Both
sides are built without FMA contraction and follow the same operation order,
so the comparisons are exact.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN


def test_accel_f64_matches_reference(oracle, golden):
    g = golden("forces_n1536.npz")
    a = oracle.accel_f64(g["pos"], g["mass"], g["eps2"])
    assert np.array_equal(a, g["acc_f64"])


def test_accel_f32_matches_reference(oracle, golden):
    g = golden("forces_n1536.npz")
    a = oracle.accel_f32(g["pos"], g["mass"], g["eps2"])
    assert np.array_equal(a, g["acc_f32"])


def test_phi_matches_reference(oracle, golden):
    g = golden("forces_n1536.npz")
    assert np.array_equal(oracle.phi_f64(g["pos"], g["mass"], g["eps2"]), g["phi"])


def test_targets_subset(oracle, golden):
    g = golden("forces_n1536.npz")
    t = np.array([0, 7, 511, 512, 1535])
    assert np.array_equal(oracle.accel_f64(g["pos"], g["mass"], g["eps2"], t), g["acc_f64"][t])
    assert np.array_equal(oracle.phi_f64(g["pos"], g["mass"], g["eps2"], t), g["phi"][t])


def test_field_and_integrator(oracle, golden):
    f = golden("forces_n1536.npz")
    g = golden("integ_n1536.npz")
    for (Mh, Mb), consts, fex in zip(g["fields"], g["consts"], g["fex"]):
        F = oracle.field(Mh=Mh, Mb=Mb)
        assert [F.Rh2, F.con, F.const1, F.Mh_inf] == list(consts)
        assert np.array_equal(oracle.fex(F, f["pos"]), fex)
    F = oracle.field(Mh=1.0, Mb=0.5)
    n = len(f["mass"])
    acc = oracle.accel_f64(f["pos"], f["mass"], f["eps2"]).reshape(-1)
    P, V = f["pos"].reshape(-1).copy(), f["vel"].reshape(-1).copy()
    post, velt, a0 = np.zeros(3 * n), np.zeros(3 * n), acc.copy()
    oracle.integ(F, acc, post, velt, P, V, 0.002, 0, a0)
    assert np.array_equal(post, g["post"]) and np.array_equal(velt, g["velt"])
    acct = oracle.accel_f64(post, f["mass"], f["eps2"]).reshape(-1)
    a1 = acc.copy()
    oracle.integ(F, acct, P, V, post, velt, 0.002, 1, a1)
    assert np.array_equal(P, g["pos1"]) and np.array_equal(V, g["vel1"])
    assert np.array_equal(a1, g["acc1"])


@pytest.mark.parametrize("label,accumulate", [("literal", True), ("corrected", False)])
def test_time_steps(oracle, golden, label, accumulate):
    g = golden("steps_n1024.npz")
    p, v, acc, _ = oracle.run_steps(g["pos"], g["vel"], g["mass"], g["eps2"], float(g["dt"]),
                                    int(g["nsteps"]), compat_accumulate=accumulate)
    assert np.array_equal(p.reshape(-1), g[label + "_pos"])
    assert np.array_equal(v.reshape(-1), g[label + "_vel"])
    assert np.array_equal(acc.reshape(-1), g[label + "_acc"])


@pytest.mark.parametrize("nx", [16, 24])
def test_binning_scan_deposit(oracle, golden, nx):
    g = golden("bin_n3072.npz")
    k = f"nx{nx}_"
    cid, slot, cnt = oracle.assign(g["pos"], g[k + "lo"], g[k + "cs"], (nx, nx, nx))
    assert np.array_equal(cid, g[k + "cell_id"])
    assert np.array_equal(slot, g[k + "id_in_cell"])
    assert np.array_equal(cnt, g[k + "count"])
    st, sr, mp = oracle.scan(cnt)
    assert np.array_equal(sr, g[k + "start_id"])
    assert np.array_equal(mp, g[k + "maxpbc"])
    assert st[0] == 0 and np.array_equal(np.diff(st), cnt[:-1])
    assert np.array_equal(oracle.cell_masses(g["mass"], cid, nx ** 3), g[k + "cell_mass"])
    assert np.array_equal(oracle.cell_phi(g["phi"], cid, cnt), g[k + "cell_phi"])


def test_wave_and_gradient(oracle, golden):
    g = golden("wave_nx16.npz")
    nx, dx = int(g["nx"]), float(g["dx"])
    W = oracle.wave_params(nx, dx, c=float(g["c"]), dt=float(g["dt"]))
    prev, cur = np.zeros(nx ** 3), np.zeros(nx ** 3)
    for _ in range(5):
        prev, cur = cur, oracle.wave_iter_f64(W, cur, prev, g["cell_mass"])
    assert np.array_equal(cur, g["phi"]) and np.array_equal(prev, g["phi_prev"])
    assert np.array_equal(oracle.acc_field(nx, dx, cur), g["cell_acc"])


def test_wave_f32_tracks_f64(oracle, golden):
    g = golden("wave_nx16.npz")
    nx, dx = int(g["nx"]), float(g["dx"])
    W = oracle.wave_params(nx, dx, c=float(g["c"]), dt=float(g["dt"]))
    prev, cur = np.zeros(nx ** 3, np.float32), np.zeros(nx ** 3, np.float32)
    for _ in range(5):
        prev, cur = cur, oracle.wave_iter_f32(W, cur, prev, g["cell_mass"])
    scale = np.abs(g["phi"]).max()
    assert np.abs(cur - g["phi"]).max() <= 1e-5 * scale


def test_galaxies_fixture_is_consistent():
    d = json.loads((GOLDEN / "galaxies_ini.json").read_text())["two_galaxies"]
    p = d["parsed"]
    assert len(p) == 2 and p[1]["n_dark"] == 0 and p[1]["angle"] == 30.0
