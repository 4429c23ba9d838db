"""khrr_accel_noalloc: the force pass for callers that cannot allocate device
memory on their call path (a host program whose device-memory budget is fixed
at start-up, or a plugin host that only passes in buffers it owns).

It is checked through the C ABI against the context entry point khrr_accel on
two calls in a row (different sizes and positions, so the second call runs on
scratch the first one left behind), with the acceleration tolerance of the
other GPU tests for small systems (relative RMS 2e-6; the two paths split the
j sum differently, so they agree to FP32 rounding, not bit for bit).  Sizes
above KHRR_NOALLOC_MAX_BODIES must be refused before any device work.
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


def test_noalloc_matches_context_entry_point(libkhrr):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    from khrr.galaxy import make_galaxy

    fn = khrr.lib().khrr_accel_noalloc
    fn.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_int, C.c_void_p]
    fn.restype = C.c_int

    ctx = khrr.Context(0)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        for ns, nd, seed in ((3000, 6000, 21), (1000, 2001, 22)):
            pos, vel, mass, eps = make_galaxy(ns, nd, seed, eps_dm=0.006).arrays()
            n = len(mass)
            dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")
            P, M, E = dev(pos), dev(mass), dev(eps * eps)
            ref = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
            got = torch.full((n, 3), 7.0, dtype=torch.float64, device="cuda")  # overwritten
            torch.cuda.synchronize()
            ctx.accel(ref.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n,
                      khrr.OVERWRITE)
            ctx.synchronize()
            st = fn(got.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), n,
                    khrr.OVERWRITE, stream)
            assert st == 0, khrr.STATUS.get(st, st)
            torch.cuda.synchronize()
            assert rel_rms(got.cpu().numpy(), ref.cpu().numpy()) <= TOL

        st = fn(got.data_ptr(), P.data_ptr(), P.data_ptr(), M.data_ptr(), E.data_ptr(), MAX_BODIES + 1,
                khrr.OVERWRITE, stream)
        assert st == 9  # KHRR_ERR_TOO_LARGE
    finally:
        ctx.close()
