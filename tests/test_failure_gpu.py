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
