"""GPU tests of the serving form, in both execution forms (resident handles on streams, and
batched kernels): results are bitwise the same alone and among requests of mixed sizes, match
the single-request path and the oracle, respect the memory budget, and cancellation frees a
request."""
import numpy as np
import pytest

from tests.helpers import KH_TOL, oracle_solution, random_k, rel_c

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16, 16), (24, 24, 24), (32, 32, 32), (8, 8, 8), (32, 16, 16), (48, 48, 48)]
FORMS = [pytest.param(False, id="handles"), pytest.param(True, id="batched")]
RING = 64 << 20  # pinned staging per server: ample for these sizes, quick to allocate


def _solve_alone(k, batched):
    from opentm_b200 import Server
    s = Server(max_active=4, batched=batched, host_stage_bytes=RING)
    rid = s.submit(k)
    s.run_until_idle()
    return s.poll(rid)


@pytest.mark.parametrize("batched", FORMS)
def test_batch_equals_alone_bitwise_and_oracle(batched):
    from opentm_b200 import Server
    # repeated sizes: the handle form reuses a resident handle for them
    shapes = SHAPES + [(32, 32, 32), (24, 24, 24), (32, 32, 32)]
    ks = [random_k(sh, seed=60 + i)[0] for i, sh in enumerate(shapes)]
    s = Server(max_active=16, iters_per_step=2, batched=batched, streams=3, host_stage_bytes=RING)
    ids = [s.submit(k) for k in ks]
    s.run_until_idle()
    for k, rid in zip(ks, ids):
        C, info = s.poll(rid)
        C1, info1 = _solve_alone(k, batched)
        assert np.array_equal(C, C1), (C, C1)
        assert info.stats.iterations == info1.stats.iterations
        assert max(info.stats.rel_res) <= 1e-6
        assert rel_c(C, oracle_solution(k)["C"]) <= KH_TOL


@pytest.mark.parametrize("batched", FORMS)
def test_server_matches_single_request_path(batched):
    from opentm_b200 import HomoConfig, Homogenization_H
    k, _ = random_k((32, 32, 32), seed=70)
    C, _ = _solve_alone(k, batched)
    H = Homogenization_H(HomoConfig(reso=32, femRelThres=1e-6, pre_smooth=2, post_smooth=2, warm_start=False))
    H.update(torch.from_numpy(k).cuda())
    if batched:
        # same algorithm, separately compiled kernels: equal to the solver tolerance
        assert rel_c(C, H.heatMatrix()) <= 1e-7
    else:
        # the handle form runs the single-request solver itself
        assert np.array_equal(C, H.heatMatrix())


@pytest.mark.parametrize("batched", FORMS)
def test_budget_admission_and_rejection(batched):
    from opentm_b200 import OtmError, Server
    b32 = Server.request_bytes((32, 32, 32))
    budget = int(b32 * 1.5)
    s = Server(hbm_budget_bytes=budget, max_active=8, batched=batched, host_stage_bytes=RING)
    ks = [random_k((32, 32, 32), seed=80 + i)[0] for i in range(3)]
    ids = [s.submit(k) for k in ks]
    nr, nq = s.step()
    assert nr <= 1 and s.bytes_in_use() <= budget and s.bytes_resident() <= budget
    s.run_until_idle()
    for rid in ids:
        assert s.poll(rid) is not None
    assert s.bytes_resident() <= budget
    with pytest.raises(OtmError) as ei:
        s.submit(random_k((64, 64, 64), seed=1)[0])
    assert ei.value.status == 8  # OTM_ERR_BUDGET


def test_handles_evicted_for_other_sizes():
    """A budget with room for one 32^3 and one 24^3 handle: alternating sizes force idle handles
    out (least recently used first); every result still equals the request solved alone."""
    from opentm_b200 import Server
    sizes = [(32, 32, 32), (24, 24, 24), (16, 16, 16), (32, 32, 32), (24, 24, 24), (16, 16, 16)]
    budget = Server.request_bytes((32, 32, 32)) + Server.request_bytes((24, 24, 24))
    s = Server(hbm_budget_bytes=budget, streams=2, host_stage_bytes=0)  # fields in pageable memory
    ks = [random_k(sh, seed=120 + i)[0] for i, sh in enumerate(sizes)]
    ids = []
    for k in ks:
        ids.append(s.submit(k))
        s.step()
        assert s.bytes_resident() <= budget
    s.run_until_idle()
    assert s.bytes_resident() <= budget and s.bytes_in_use() == 0
    for k, rid in zip(ks, ids):
        C, _ = s.poll(rid)
        assert np.array_equal(C, _solve_alone(k, False)[0])


def test_failed_request_leaves_handle_usable():
    """A field with a NaN fails with OTM_ERR_NAN; the next request of that size, on the same
    resident handle, solves normally."""
    from opentm_b200 import OtmError, Server
    bad = np.ones((16, 16, 16), dtype=np.float32)
    bad[3, 3, 3] = np.nan
    good, _ = random_k((16, 16, 16), seed=130)
    s = Server(streams=1, host_stage_bytes=RING)
    a = s.submit(bad)
    s.run_until_idle()
    with pytest.raises(OtmError) as ei:
        s.poll(a)
    assert ei.value.status == 7  # OTM_ERR_NAN
    b = s.submit(good)
    s.run_until_idle()
    C, info = s.poll(b)
    assert np.array_equal(C, _solve_alone(good, False)[0])
    assert max(info.stats.rel_res) <= 1e-6


@pytest.mark.parametrize("batched", FORMS)
def test_cancel_running_and_queued(batched):
    from opentm_b200 import OtmError, Server
    s = Server(max_active=1, iters_per_step=1, batched=batched, host_stage_bytes=RING)
    a = s.submit(random_k((32, 32, 32), seed=90)[0])
    b = s.submit(random_k((32, 32, 32), seed=91)[0])
    s.step()
    s.cancel(a)
    s.cancel(b)
    s.run_until_idle()
    for rid in (a, b):
        with pytest.raises(OtmError) as ei:
            s.poll(rid)
        assert ei.value.status == 11  # OTM_ERR_CANCELLED
    assert s.bytes_in_use() == 0


@pytest.mark.parametrize("batched", FORMS)
def test_requests_arriving_while_others_run(batched):
    from opentm_b200 import Server
    s = Server(max_active=8, iters_per_step=1, batched=batched, host_stage_bytes=RING)
    first = [s.submit(random_k((32, 32, 32), seed=100 + i)[0]) for i in range(3)]
    s.step()
    late_k = [random_k((24, 24, 24), seed=110 + i)[0] for i in range(3)]
    late = [s.submit(k) for k in late_k]  # admitted while the first ones run
    s.run_until_idle()
    for k, rid in zip(late_k, late):
        C, info = s.poll(rid)
        assert np.array_equal(C, _solve_alone(k, batched)[0])
    assert all(s.poll(r) is not None for r in first)
