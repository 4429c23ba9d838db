"""khrr_accel_noalloc: the force pass for callers that cannot allocate device
memory on their call path (a host program whose device-memory budget is fixed
at start-up, or a plugin host that only passes in buffers it owns).

Checked through the C ABI, with the acceleration tolerance of the other GPU
tests for small systems (relative RMS 2e-6 against FP64; FP32 pair terms):
  * against the FP64 oracle (oracle.c) and against the context entry point
    khrr_accel, on two calls in a row of different sizes and positions, so the
    second call runs on scratch the first one left behind;
  * in accumulate mode (acc += sum) on top of a known array;
  * with a distinct set of target positions pos_i (the i shadow of the scratch
    array), against an FP64 direct sum written out here and against
    khrr_accel given the same pos_i;
  * sizes above KHRR_NOALLOC_MAX_BODIES are refused before any device work.
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_BODIES = 32768  # KHRR_NOALLOC_MAX_BODIES in include/khrr.h
TOL = 2e-6


def rel_rms(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def direct_sum_f64(pos_i, pos_j, mass, eps2):
    """ACCEL_kernel's sum (nbody-kernel.cuh:89-142) in FP64 with distinct
    target positions: a_i = sum_j m_j d / (d^2 + (eps2_i + eps2_j)/2)^{3/2},
    d = pos_j[j] - pos_i[i], the softening of i read from eps2[i]."""
    out = np.zeros_like(pos_i)
    for s in range(0, len(pos_i), 256):
        d = pos_j[None, :, :] - pos_i[s:s + 256, None, :]
        r2 = (d * d).sum(-1) + 0.5 * (eps2[s:s + 256, None] + eps2[None, :])
        k = mass[None, :] / (r2 * np.sqrt(r2))
        out[s:s + 256] = (d * k[:, :, None]).sum(1)
    return out


@pytest.fixture(scope="module")
def noalloc(libkhrr):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    fn = khrr.lib().khrr_accel_noalloc
    fn.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_int, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")


def test_noalloc_matches_oracle_and_context_entry_point(noalloc, oracle):
    import torch
    import khrr
    from khrr.galaxy import make_galaxy

    ctx = khrr.Context(0)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        for ns, nd, seed in ((3000, 6000, 21), (1000, 2001, 22)):
            pos, vel, mass, eps = make_galaxy(ns, nd, seed, eps_dm=0.006).arrays()
            n = len(mass)
            eps2 = eps * eps
            P, M, E = _dev(torch, pos), _dev(torch, mass), _dev(torch, eps2)
            ref = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
            got = torch.full((n, 3), 7.0, dtype=torch.float64, device="cuda")  # overwritten
            torch.cuda.synchronize()
            ctx.accel(ref.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n,
                      khrr.OVERWRITE)
            ctx.synchronize()
            st = noalloc(got.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n,
                         khrr.OVERWRITE, stream)
            assert st == 0, khrr.STATUS.get(st, st)
            torch.cuda.synchronize()
            g = got.cpu().numpy()
            f64 = oracle.accel_f64(pos, mass, eps2).reshape(n, 3)
            assert np.isfinite(g).all()
            assert rel_rms(g, f64) <= TOL
            assert rel_rms(g, ref.cpu().numpy()) <= TOL

        # accumulate mode: acc += sum on top of a known array
        base = np.random.default_rng(5).standard_normal((n, 3))
        acc = _dev(torch, base)
        torch.cuda.synchronize()
        st = noalloc(acc.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n, 0, stream)
        assert st == 0, khrr.STATUS.get(st, st)
        torch.cuda.synchronize()
        assert rel_rms(acc.cpu().numpy() - base, f64) <= TOL

        st = noalloc(got.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), MAX_BODIES + 1,
                     khrr.OVERWRITE, stream)
        assert st == 9  # KHRR_ERR_TOO_LARGE
    finally:
        ctx.close()


def test_noalloc_distinct_targets(noalloc):
    import torch
    import khrr
    from khrr.galaxy import make_galaxy

    pos, vel, mass, eps = make_galaxy(1000, 2001, 23, eps_dm=0.006).arrays()
    n = len(mass)
    eps2 = eps * eps
    pos_i = pos + 0.01 * np.random.default_rng(9).standard_normal(pos.shape)
    Pi, Pj, M, E = _dev(torch, pos_i), _dev(torch, pos), _dev(torch, mass), _dev(torch, eps2)
    got = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    ref = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    st = noalloc(got.data_ptr(), Pi.data_ptr(), Pj.data_ptr(), M.data_ptr(), E.data_ptr(), n,
                 khrr.OVERWRITE, stream)
    assert st == 0, khrr.STATUS.get(st, st)
    torch.cuda.synchronize()
    ctx = khrr.Context(0)
    try:
        ctx.accel(ref.data_ptr(), Pi.data_ptr(), Pj.data_ptr(), M.data_ptr(), E.data_ptr(), n, khrr.OVERWRITE)
        ctx.synchronize()
    finally:
        ctx.close()
    g = got.cpu().numpy()
    f64 = direct_sum_f64(pos_i, pos, mass, eps2)
    assert np.isfinite(g).all()
    assert rel_rms(g, f64) <= TOL
    assert rel_rms(g, ref.cpu().numpy()) <= TOL
