"""Serving (fast-gpr-fwi_b200/serve.py): a mixed stream of forward and
gradient requests of different sizes, admitted by an HBM budget and run
concurrently, gives every request the result it gets alone, bit for bit."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests(fg):
    serve = __import__("importlib").import_module("fast-gpr-fwi_b200.serve")
    out = []
    shapes = [(48, 40, 3, 120, 6), (64, 56, 9, 90, 6), (40, 56, 2, 150, 5), (56, 48, 12, 100, 6),
              (48, 40, 1, 200, 6), (72, 64, 5, 80, 8)]
    for n, (nx, ny, shots, nt, pml) in enumerate(shapes):
        wl = fg.workloads.small(seed=10 + n, nx=nx, ny=ny, shots=shots, nt=nt, pml=pml, fixed=True)
        wl.source_step = [0.03, 0.01, 0.0]
        kw = wl.kwargs("cuda")
        for k in ("er", "se", "mr", "device", "tv"):
            kw.pop(k)
        rng = np.random.default_rng(n)
        resid = None
        if n % 2 == 0:
            resid = torch.tensor(rng.standard_normal((shots, nt, wl.nrx)).astype(np.float32) * 1e-3)
        out.append(serve.Request(kw, torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr), resid))
    return serve, out


def _arrays(res):
    return [None if t is None else t.cpu().numpy() for t in (res.traces, res.grad_eps, res.grad_sig)]


def test_results_same_alone_and_in_the_mix(fg):
    serve, reqs = _requests(fg)
    alone = []
    for r in reqs:
        srv = serve.Server("cuda:0", max_active=1)
        alone.append(_arrays(srv.submit(r).result()))
        srv.close()
    srv = serve.Server("cuda:0", max_active=4)
    futs = [srv.submit(r) for r in reqs + reqs]
    mixed = [f.result() for f in futs]
    st = srv.stats()
    srv.close()
    assert st["requests"] == 2 * len(reqs) and st["peak_active"] >= 2
    assert st["p99_s"] >= st["p50_s"] > 0
    for k, res in enumerate(mixed):
        for a, b in zip(alone[k % len(reqs)], _arrays(res)):
            if a is None:
                assert b is None
            else:
                assert np.array_equal(a, b)


def test_budget_admission_and_checkpoint_fallback(fg):
    serve, reqs = _requests(fg)
    grad = reqs[2]                    # a gradient request
    srv = serve.Server("cuda:0", max_active=2)
    full = srv.submit(grad).result()
    srv.close()
    # a budget below the full-history footprint: the gradient takes the checkpointed solve, same bits
    tight = serve.Server("cuda:0", hbm_budget=int(full.bytes_reserved * 0.6), max_active=2)
    ck = tight.submit(grad).result()
    tight.close()
    assert full.checkpoint is None and ck.checkpoint is not None and ck.bytes_reserved < full.bytes_reserved
    for a, b in zip(_arrays(full), _arrays(ck)):
        assert np.array_equal(a, b)
    # a budget too small for any form of the request is refused
    tiny = serve.Server("cuda:0", hbm_budget=1 << 20, max_active=1)
    with pytest.raises(MemoryError):
        tiny.submit(grad).result()
    tiny.close()


def _survey_requests(fg, serve, n=3, shots=(3, 5, 2)):
    """Forward requests of one survey: same grid, model and waveform, each
    with its own shot positions."""
    out = []
    for k in range(n):
        wl = fg.workloads.small(seed=77, nx=64, ny=56, shots=shots[k], nt=110, pml=6, fixed=True)
        wl.source_location = [0.3 + 0.6 + 0.2 * k, 0.25 + 0.3, 0.0]
        wl.source_step = [0.05, 0.01, 0.0]
        kw = wl.kwargs("cuda")
        for key in ("er", "se", "mr", "device", "tv"):
            kw.pop(key)
        out.append(serve.Request(kw, torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr), None,
                                 merge_key="survey-77"))
    return out


def test_merged_forward_requests_equal_alone(fg):
    """Forward requests of one survey queued behind a running request are
    merged into one solve; each gets the traces it gets alone."""
    serve, _ = _requests(fg)
    survey = _survey_requests(fg, serve)
    alone = []
    for r in survey:
        srv = serve.Server("cuda:0", max_active=1)
        alone.append(srv.submit(r).result().traces.cpu().numpy())
        srv.close()
    big = fg.workloads.small(seed=5, nx=200, ny=200, shots=16, nt=2500, pml=10, fixed=True)
    big.source_step = [0.05, 0.01, 0.0]
    kw = big.kwargs("cuda")
    for key in ("er", "se", "mr", "device", "tv"):
        kw.pop(key)
    hold = serve.Request(kw, torch.tensor(big.er), torch.tensor(big.se), torch.tensor(big.mr),
                         torch.zeros((16, 2500, big.nrx)))
    srv = serve.Server("cuda:0", max_active=1)
    first = srv.submit(hold)                     # a gradient request holds the one slot for ~0.1 s
    futs = [srv.submit(r) for r in survey]       # these queue up behind it and are merged
    first.result()
    got = [f.result() for f in futs]
    st = srv.stats()
    srv.close()
    assert st["merged"] == len(survey)
    for a, res in zip(alone, got):
        assert res.traces.shape[0] == a.shape[0]
        assert np.array_equal(a, res.traces.cpu().numpy())


def test_shortest_job_first_and_fifo(fg):
    """Behind a running request, 'sjf' admits the queued request with the least
    work first and 'fifo' the oldest; every result is the same either way."""
    serve, reqs = _requests(fg)
    big = fg.workloads.small(seed=6, nx=200, ny=200, shots=16, nt=6000, pml=10, fixed=True)
    big.source_step = [0.05, 0.01, 0.0]
    kw = big.kwargs("cuda")
    for key in ("er", "se", "mr", "device", "tv"):
        kw.pop(key)
    hold = serve.Request(kw, torch.tensor(big.er), torch.tensor(big.se), torch.tensor(big.mr),
                         torch.zeros((16, 6000, big.nrx)))   # holds the one slot while the others queue
    queued = [reqs[3], reqs[4], reqs[0]]   # forward 56x48x12x100; gradients 48x40x1x200, 48x40x3x120
    order = {}
    results = {}
    for policy in ("sjf", "fifo"):
        srv = serve.Server("cuda:0", max_active=1, policy=policy, max_wait=60.0)
        first = srv.submit(hold)
        futs = [srv.submit(r) for r in queued]
        first.result()
        got = [f.result() for f in futs]
        srv.close()
        order[policy] = [k for k, _ in sorted(enumerate(got), key=lambda kv: kv[1].started)]
        results[policy] = [r.traces.cpu().numpy() for r in got]
    # work (nx * ny * shots * nt, gradients x 2.5): 3.2e6 (forward), 0.96e6, 1.73e6
    assert order["fifo"] == [0, 1, 2]
    assert order["sjf"] == [1, 2, 0]
    for a, b in zip(results["sjf"], results["fifo"]):
        assert np.array_equal(a, b)


def test_batched_small_requests_equal_alone(fg):
    """Small shot-lane requests of different grids, models and step counts
    queued behind a running request are solved together in one persistent
    launch per direction; each gets the bits it gets alone."""
    serve = __import__("importlib").import_module("fast-gpr-fwi_b200.serve")
    reqs = []
    for n, (nx, ny, shots, nt) in enumerate([(56, 48, 12, 100), (64, 40, 9, 130), (48, 64, 20, 90)]):
        wl = fg.workloads.small(seed=30 + n, nx=nx, ny=ny, shots=shots, nt=nt, pml=6, fixed=True)
        wl.source_step = [0.02, 0.01, 0.0]
        kw = wl.kwargs("cuda")
        for key in ("er", "se", "mr", "device", "tv"):
            kw.pop(key)
        resid = None
        if n != 1:
            rng = np.random.default_rng(n)
            resid = torch.tensor(rng.standard_normal((shots, nt, wl.nrx)).astype(np.float32) * 1e-3)
        reqs.append(serve.Request(kw, torch.tensor(wl.er), torch.tensor(wl.se), torch.tensor(wl.mr), resid))
    alone = []
    for r in reqs:
        srv = serve.Server("cuda:0", max_active=1)
        alone.append(_arrays(srv.submit(r).result()))
        srv.close()
    big = fg.workloads.small(seed=5, nx=200, ny=200, shots=4, nt=6000, pml=10, fixed=True)
    big.source_step = [0.05, 0.01, 0.0]
    kw = big.kwargs("cuda")
    for key in ("er", "se", "mr", "device", "tv"):
        kw.pop(key)
    hold = serve.Request(kw, torch.tensor(big.er), torch.tensor(big.se), torch.tensor(big.mr), None)
    srv = serve.Server("cuda:0", max_active=1)
    first = srv.submit(hold)                     # holds the one slot while the small ones queue
    futs = [srv.submit(r) for r in reqs]
    first.result()
    got = [_arrays(f.result()) for f in futs]
    st = srv.stats()
    srv.close()
    assert st["batched"] == len(reqs)
    for a, b in zip(alone, got):
        for x, y in zip(a, b):
            if x is None:
                assert y is None
            else:
                assert np.array_equal(x, y)
