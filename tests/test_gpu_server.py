"""GPU tests of the serving form: results are bitwise the same alone and in a batch of mixed
sizes, match the single-request path and the oracle, respect the memory budget, and
cancellation frees a request."""
import numpy as np
import pytest

from tests.helpers import KH_TOL, oracle_solution, random_k, rel_c

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16, 16), (24, 24, 24), (32, 32, 32), (8, 8, 8), (32, 16, 16), (48, 48, 48)]


def _solve_alone(k):
    from opentm_b200 import Server
    s = Server(max_active=4)
    rid = s.submit(k)
    s.run_until_idle()
    return s.poll(rid)


def test_batch_equals_alone_bitwise_and_oracle():
    from opentm_b200 import Server
    ks = [random_k(sh, seed=60 + i)[0] for i, sh in enumerate(SHAPES)]
    s = Server(max_active=16, iters_per_step=2)
    ids = [s.submit(k) for k in ks]
    s.run_until_idle()
    for k, rid in zip(ks, ids):
        C, info = s.poll(rid)
        C1, info1 = _solve_alone(k)
        assert np.array_equal(C, C1), (C, C1)
        assert info.stats.iterations == info1.stats.iterations
        assert max(info.stats.rel_res) <= 1e-6
        assert rel_c(C, oracle_solution(k)["C"]) <= KH_TOL


def test_server_matches_single_request_path():
    from opentm_b200 import HomoConfig, Homogenization_H
    k, _ = random_k((32, 32, 32), seed=70)
    C, _ = _solve_alone(k)
    H = Homogenization_H(HomoConfig(reso=32, femRelThres=1e-6, pre_smooth=2, post_smooth=2, warm_start=False))
    H.update(torch.from_numpy(k).cuda())
    # same algorithm, separately compiled kernels: equal to the solver tolerance
    assert rel_c(C, H.heatMatrix()) <= 1e-7


def test_budget_admission_and_rejection():
    from opentm_b200 import OtmError, Server
    b32 = Server.request_bytes((32, 32, 32))
    s = Server(hbm_budget_bytes=int(b32 * 1.5), max_active=8)
    ks = [random_k((32, 32, 32), seed=80 + i)[0] for i in range(3)]
    ids = [s.submit(k) for k in ks]
    nr, nq = s.step()
    assert nr <= 1 and s.bytes_in_use() <= int(b32 * 1.5)
    s.run_until_idle()
    for rid in ids:
        assert s.poll(rid) is not None
    with pytest.raises(OtmError) as ei:
        s.submit(random_k((64, 64, 64), seed=1)[0])
    assert ei.value.status == 8  # OTM_ERR_BUDGET


def test_cancel_running_and_queued():
    from opentm_b200 import OtmError, Server
    s = Server(max_active=1, iters_per_step=1)
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


def test_requests_arriving_while_others_run():
    from opentm_b200 import Server
    s = Server(max_active=8, iters_per_step=1)
    first = [s.submit(random_k((32, 32, 32), seed=100 + i)[0]) for i in range(3)]
    s.step()
    late_k = [random_k((24, 24, 24), seed=110 + i)[0] for i in range(3)]
    late = [s.submit(k) for k in late_k]  # admitted while the first ones run
    s.run_until_idle()
    for k, rid in zip(late_k, late):
        C, info = s.poll(rid)
        assert np.array_equal(C, _solve_alone(k)[0])
    assert all(s.poll(r) is not None for r in first)
