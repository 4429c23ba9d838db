"""Failure detection without a GPU fault: a kernel's bounded wait on a
barrier that nothing completes gives up after a short limit, the host reads
KHRR_ERR_TIMEOUT through the context's error flag, and the context keeps
working (the next force evaluation equals one from a fresh context)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(libkhrr):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import khrr
    c = khrr.Context(0)
    yield c
    c.close()


def galaxy():
    from khrr.galaxy import make_galaxy
    pos, vel, mass, eps = make_galaxy(512, 1024, 51).arrays()
    return pos, vel, mass, eps * eps


def test_bounded_wait_times_out_and_reports(ctx):
    import khrr
    t0 = time.perf_counter()
    st = ctx.probe_bounded_wait(0.25)
    dt = time.perf_counter() - t0
    assert khrr.STATUS[st] == "KHRR_ERR_TIMEOUT"
    assert b"bounded wait" in ctx.L.khrr_last_error(ctx.h)
    assert 0.25 <= dt < 5.0
    # the flag was cleared: a second probe times out again on its own
    assert khrr.STATUS[ctx.probe_bounded_wait(0.05)] == "KHRR_ERR_TIMEOUT"


def test_context_usable_after_timeout(ctx):
    import khrr
    pos, vel, mass, eps2 = galaxy()
    assert khrr.STATUS[ctx.probe_bounded_wait(0.1)] == "KHRR_ERR_TIMEOUT"
    ctx.upload(pos, vel, mass, eps2)
    ctx.forces(khrr.ACC | khrr.PHI)
    ctx.step(0.002, 2, khrr.PHI)
    after = ctx.download()
    fresh = khrr.Context(0)
    try:
        fresh.upload(pos, vel, mass, eps2)
        fresh.forces(khrr.ACC | khrr.PHI)
        fresh.step(0.002, 2, khrr.PHI)
        want = fresh.download()
    finally:
        fresh.close()
    for k in ("pos", "vel", "acc", "phi"):
        assert np.array_equal(after[k], want[k]), k


def test_probe_rejects_bad_limits(ctx):
    import khrr
    assert khrr.STATUS[ctx.probe_bounded_wait(0.0)] == "KHRR_ERR_INVALID_ARG"
    assert khrr.STATUS[ctx.probe_bounded_wait(60.0)] == "KHRR_ERR_INVALID_ARG"


def test_resident_stencil_wait_times_out_and_context_recovers(ctx):
    """The cooperative 128^3 stencil's CTAs wait on one another's counters:
    with one brick withholding its counter, its neighbours' bounded waits give
    up, the abort word ends every other wait, the call reports
    KHRR_ERR_TIMEOUT, and the next resident wave solve on the same context
    equals one on a fresh context bit for bit."""
    import khrr
    t0 = time.perf_counter()
    st = ctx.probe_resident_wave(0.25)
    dt = time.perf_counter() - t0
    if khrr.STATUS[st] == "KHRR_ERR_UNSUPPORTED":
        pytest.skip("the resident stencil does not run on this device")
    assert khrr.STATUS[st] == "KHRR_ERR_TIMEOUT"
    assert 0.25 <= dt < 5.0
    assert khrr.STATUS[ctx.probe_resident_wave(0.0)] == "KHRR_ERR_INVALID_ARG"
    pos, vel, mass, eps2 = galaxy()
    nx, L = 128, 4.0
    W = khrr.WaveParams.make(nx, 2 * L / nx)
    out = []
    for c in (ctx, khrr.Context(0)):
        try:
            c.upload(pos, vel, mass, eps2)
            c.bin((-L,) * 3, (2 * L / nx,) * 3, (nx, nx, nx))
            out.append(c.wave_solve(W, tol=0.0, max_iter=60, check_every=30, cold=True))
        finally:
            if c is not ctx:
                c.close()
    (i1, r1, p1), (i2, r2, p2) = out
    assert i1 == i2 == 60
    assert np.array_equal(p1, p2)
    assert r1 == r2 or abs(r1 - r2) <= 1e-12 * r2
