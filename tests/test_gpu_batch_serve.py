"""The continuous-batching server (lbfgsb_b200_batch_server_*).

Requests arrive while others are running: they are admitted as memory frees up, their
rounds run in the same launches as the running solves, and each result must equal the same
solve run alone through lbfgsb_b200_minimize_batch_device_f32 (bit for bit: an instance's
launches do not depend on the others).  A budget that holds one solve at a time serialises
the server without changing any result; a request larger than the whole budget is refused.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIDES = [24, 64, 40, 16, 90, 33, 52, 70]
SEEDS = [400 + k for k in range(len(SIDES))]


@pytest.fixture(scope="module")
def LB():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lbfgsb_b200
    lbfgsb_b200.load()
    return lbfgsb_b200


def _opt(LB):
    o = LB.default_option(np.float32)
    o.eps_g = 1e-6
    o.max_iteration = 300
    return o


def _alone(LB, bt, p, form):
    import torch
    x = torch.zeros(bt.n[p], dtype=torch.float32, device="cuda")
    rc, stat, summ, _ = LB.solve_batch_device(bt, [x], _opt(LB), form=form, ids=[p])
    torch.cuda.synchronize()
    assert rc == 0 and stat == [0]
    return x.cpu().numpy(), summ[0]


@pytest.mark.parametrize("budget_solves", [None, 1])
def test_served_results_equal_solves_alone(LB, budget_solves):
    import torch
    form = LB.FORM_MIXED
    sides = SIDES if budget_solves is None else [48] * 6
    bt = LB.SynthBatch(sides, SEEDS[:len(sides)], single_precision_fields=True, dtype=np.float32)
    budget = 150 * 10**9
    if budget_solves == 1:
        # room for one request at a time: admitted one after another
        one = LB.load().lbfgsb_b200_batch_request_bytes(bt.n[0], form, 8)
        assert one > 0
        budget = int(one * 1.5)
    sv = LB.BatchServer(bt, _opt(LB), hbm_budget_bytes=budget, form=form, rounds_per_loop=2)
    xs = [torch.zeros(n, dtype=torch.float32, device="cuda") for n in bt.n]
    torch.cuda.synchronize()
    tickets = []
    for p in range(len(sides)):
        rc, t = sv.submit(p, xs[p])
        assert rc == 0
        tickets.append(t)
        time.sleep(0.003)  # later requests arrive while earlier ones run
    outs = [sv.wait(t) for t in tickets]
    peak_bytes, peak_live = sv.peak()
    sv.close()
    torch.cuda.synchronize()
    assert peak_bytes <= budget
    if budget_solves == 1:
        assert peak_live == 1
    else:
        assert peak_live > 1
    for p, (st, summ, lat, q) in enumerate(outs):
        assert st == 0
        xa, sa = _alone(LB, bt, p, form)
        assert (summ.info, summ.num_iteration) == (sa.info, sa.num_iteration)
        assert summ.residual_g == sa.residual_g
        np.testing.assert_array_equal(xs[p].cpu().numpy(), xa)
        assert lat >= q >= 0.0
    bt.close()


def test_request_over_budget_is_refused(LB):
    import torch
    bt = LB.SynthBatch([64], [1], single_precision_fields=True, dtype=np.float32)
    sv = LB.BatchServer(bt, _opt(LB), hbm_budget_bytes=1 << 16, form=LB.FORM_MIXED)
    x = torch.zeros(bt.n[0], dtype=torch.float32, device="cuda")
    rc, _ = sv.submit(0, x)
    assert rc == 1
    sv.close()
    bt.close()


def test_submit_from_threads(LB):
    """Submissions from several host threads while the server runs."""
    import torch
    bt = LB.SynthBatch(SIDES, SEEDS, single_precision_fields=True, dtype=np.float32)
    sv = LB.BatchServer(bt, _opt(LB), form=LB.FORM_MIXED)
    xs = [torch.zeros(n, dtype=torch.float32, device="cuda") for n in bt.n]
    torch.cuda.synchronize()
    tickets = [None] * len(SIDES)

    def worker(ps):
        for p in ps:
            rc, t = sv.submit(p, xs[p])
            assert rc == 0
            tickets[p] = t

    th = [threading.Thread(target=worker, args=(list(range(k, len(SIDES), 3)),)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    outs = [sv.wait(t) for t in tickets]
    sv.close()
    assert all(o[0] == 0 and o[1].info in (1, 2, 4, 5) for o in outs)
    bt.close()
