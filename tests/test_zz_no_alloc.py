"""p6_pt_costs_static (the allocation-free cost call) against p6_pt_costs.

Collected last so that it also runs after every other GPU test has used the
device; it passes alone as well.  Two calls in a row with different vectors
check that nothing carries over in the shared static scratch, and a fresh
session that only ever makes static calls must leave the device's free memory
and its own allocating scratch untouched."""
import numpy as np
import pytest

from powder6_b200._lib import P6Error
from powder6_b200.pt_gpu import PTContext, PTSession, nacl_problem, pt_scales, reflection_dmin, start_vectors, synthesise

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 4 << 20


@pytest.fixture(scope='module')
def session(oracle):
    P = nacl_problem(seed=1)
    truth = synthesise(P, oracle.PtModel(P).pattern, seed=1)
    ctx = PTContext(P, truth, {'chains': 8, 'sweeps': 1, 'maxTemp': 10.0, 'seed': 1, 'scales': pt_scales(P, truth)})
    with PTSession(ctx) as s:
        yield P, truth, s


def test_static_costs_equal_allocating_costs_twice_in_a_row(session):
    P, truth, s = session
    first = [truth] + start_vectors(P, truth, 5, seed=21)
    second = start_vectors(P, truth, 9, seed=22)
    c1, y1 = s.costs_static(first, with_pattern=True)
    c2 = s.costs_static(second)
    r1, ry1 = s.costs(first, with_pattern=True)
    r2 = s.costs(second)
    assert np.array_equal(c1, r1) and np.array_equal(y1, ry1)
    assert np.array_equal(c2, r2)


def test_static_costs_reject_oversize_requests(session):
    P, truth, s = session
    n = SCRATCH_BYTES // (len(P.tth) * 4) + 1          # patterns alone exceed the scratch
    with pytest.raises(P6Error, match='static scratch'):
        s.costs_static([truth] * n, with_pattern=True)
    # the same count without patterns fits, and the session still works
    c = s.costs_static([truth] * n)
    assert np.all(c == c[0]) and np.isfinite(c[0])


def test_static_costs_allocate_no_device_memory(oracle):
    torch = pytest.importorskip('torch')
    P = nacl_problem(seed=1)
    truth = synthesise(P, oracle.PtModel(P).pattern, seed=1)
    ctx = PTContext(P, truth, {'chains': 8, 'sweeps': 1, 'maxTemp': 10.0, 'seed': 1, 'scales': pt_scales(P, truth)})
    with PTSession(ctx) as s:
        s.costs_static([truth])                      # first call on the device: address look-up
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        for n in (1, 7, 64, 300):                    # growing, the last larger than any costs() call here
            c = s.costs_static(start_vectors(P, truth, n, seed=30 + n))
            assert c.shape == (n,) and np.all(np.isfinite(c))
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(0)[0] == free0
        assert s.vector_capacity() == 0              # the allocating scratch was never grown
        s.costs([truth])                             # the allocating call does grow it
        assert s.vector_capacity() >= 1
