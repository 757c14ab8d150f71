"""GPU tests of the serving loop: results of batched requests of mixed sizes
against the single-request path and the FP64 oracle; the same result alone
and in the mix; memory-based admission; errors."""
import threading
import time

import numpy as np
import pytest

import vqcb200 as V
from helpers import rel
from oracle import oracle as O
from vqcb200 import workloads as W
from vqcb200.serve import Server

pytestmark = pytest.mark.gpu


def make_request(rng, n, layers):
    th = rng.uniform(0, 2 * np.pi, layers * 2 * n)
    spec = W.hea_spec(n, layers, th)
    g = float(rng.uniform(0.2, 1.5))
    return spec, W.tfim_spec(n, g)


def test_serve_matches_single_path_and_oracle():
    rng = np.random.default_rng(50)
    reqs = []
    for i in range(24):
        n = int(rng.integers(9, 17))
        layers = int(rng.integers(2, 6))
        spec, hspec = make_request(rng, n, layers)
        reqs.append((n, spec, hspec, bool(i % 2)))
    with Server(dtype=np.complex64, memory_bytes=1 << 30, max_active=64) as srv:
        tickets = [srv.submit(n, W.to_circuit(spec), W.to_operator(h), want_grad=g) for n, spec, h, g in reqs]
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
        lt = srv.loop_timing()
    assert st["completed"] == len(reqs)
    # batching happened: fewer launches than request-steps
    assert st["launches"] < st["request_steps"]
    # every iteration that launched work is timed, in non-negative phases
    assert 0 < lt["iterations"] <= st["iterations"]
    assert min(lt["build_s"], lt["device_wait_s"], lt["retire_s"]) >= 0
    for (n, spec, hspec, g), (e, grads, lat) in zip(reqs, results):
        e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=4)
        assert abs(e - e_ref) / max(abs(e_ref), 1.0) < 1e-5
        if g:
            assert rel(grads, g_ref) < 1e-5
        else:
            assert grads is None
        assert lat >= 0


def test_same_result_alone_and_in_the_mix():
    """A request's result does not depend on what it is batched with: within
    the FP32 bound (1e-5) on an FP32 server (a request of 2^18+ amplitudes may
    run on the generic or on a compiled kernel, depending on whether its pass
    structure was compiled when it was planned), and bit for bit on an FP64
    server (one kernel for every request)."""
    rng = np.random.default_rng(51)
    mix = []
    for i in range(16):
        n = int(rng.integers(9, 19))
        spec, hspec = make_request(rng, n, int(rng.integers(2, 7)))
        mix.append((n, spec, hspec))
    for dtype in (np.complex64, np.complex128):
        for probe_i in (5, max(range(16), key=lambda i: mix[i][0])):
            probe = mix[probe_i]
            with Server(dtype=dtype, memory_bytes=2 << 30, max_active=64) as srv:
                t = srv.submit(probe[0], W.to_circuit(probe[1]), W.to_operator(probe[2]), want_grad=True)
                alone = srv.wait(t)
                ts = [srv.submit(n, W.to_circuit(s), W.to_operator(h), want_grad=True) for n, s, h in mix]
                in_mix = [srv.wait(x) for x in ts][probe_i]
            if dtype == np.complex128:
                assert alone[0] == in_mix[0]
                assert np.array_equal(alone[1], in_mix[1])
            else:
                assert abs(alone[0] - in_mix[0]) <= 1e-5 * abs(in_mix[0])
                assert rel(alone[1], in_mix[1]) < 1e-5


def test_compiled_batch_kernels_match_oracle():
    """Requests of 2^18 or more amplitudes run on batch kernels compiled for
    their pass structure once it has been compiled (by a planner thread, after
    the first request of that structure was handed on to run on the generic
    kernel).  A cold and a warm round of one structure both match the oracle."""
    rng = np.random.default_rng(59)
    n = 18
    reqs = [make_request(rng, n, 3) for _ in range(4)]
    with Server(dtype=np.complex64, memory_bytes=1 << 30, max_active=8) as srv:
        cold = srv.wait(srv.submit(n, W.to_circuit(reqs[0][0]), W.to_operator(reqs[0][1])))
        time.sleep(10)  # the structure's kernels compile meanwhile
        ts = [srv.submit(n, W.to_circuit(sp), W.to_operator(h), want_grad=bool(i % 2 == 0)) for i, (sp, h) in
              enumerate(reqs)]
        warm = [srv.wait(t) for t in ts]
    for (sp, h), (e, g, _), want in [(reqs[0], cold, True)] + [(r, o, i % 2 == 0) for i, (r, o) in
                                                              enumerate(zip(reqs, warm))]:
        e_ref, g_ref = O.energy_and_gradient(O.from_spec(sp), O.terms_from_spec(h), O.zero_state(n), nthreads=8)
        assert abs(e - e_ref) / max(abs(e_ref), 1.0) < 1e-5
        if want:
            assert rel(g, g_ref) < 1e-5
        else:
            assert g is None


def test_requests_arriving_while_others_run():
    """Continuous batching: a second wave submitted from another thread while
    the first runs is admitted and finishes; everything completes."""
    rng = np.random.default_rng(52)
    reqs = []
    for _ in range(40):
        n = int(rng.integers(10, 20))
        reqs.append((n,) + make_request(rng, n, int(rng.integers(2, 10))))
    out = {}
    with Server(dtype=np.complex64, memory_bytes=256 << 20, max_active=8) as srv:
        def client(lo, hi, delay):
            time.sleep(delay)
            ts = [(i, srv.submit(reqs[i][0], W.to_circuit(reqs[i][1]), W.to_operator(reqs[i][2]))) for i in range(lo, hi)]
            for i, t in ts:
                out[i] = srv.wait(t)
        th = [threading.Thread(target=client, args=(0, 20, 0.0)), threading.Thread(target=client, args=(20, 40, 0.05))]
        for x in th:
            x.start()
        for x in th:
            x.join()
        st = srv.stats()
    assert len(out) == 40 and st["completed"] == 40
    # the memory budget (256 MiB) and 8 slots forced waiting: more iterations than the longest request's steps
    assert st["iterations"] > 0
    for i in (0, 25, 39):
        n, spec, hspec = reqs[i]
        e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=4)
        assert abs(out[i][0] - e_ref) / max(abs(e_ref), 1.0) < 1e-5
        assert rel(out[i][1], g_ref) < 1e-5


def test_fp64_server():
    rng = np.random.default_rng(53)
    n = 12
    spec, hspec = make_request(rng, n, 3)
    with Server(dtype=np.complex128, memory_bytes=1 << 28, max_active=4) as srv:
        e, g, _ = srv.wait(srv.submit(n, W.to_circuit(spec), W.to_operator(hspec)))
    e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=4)
    assert abs(e - e_ref) < 1e-12
    assert rel(g, g_ref) < 1e-12


def test_admission_rejects_oversized_and_bad_requests():
    rng = np.random.default_rng(54)
    spec, hspec = make_request(rng, 20, 2)
    with Server(dtype=np.complex64, memory_bytes=1 << 20, max_active=4) as srv:
        t = srv.submit(20, W.to_circuit(spec), W.to_operator(hspec))
        with pytest.raises(BlockingIOError):
            srv.wait(t)
        # three-target dense gates are not served
        from oracle import gates_ref as GR
        bad = V.QCircuit([V.QuantumGate((1, 2, 3), GR.random_unitary(3, rng))])
        t = srv.submit(9, bad, V.QubitsOperator(V.pauli({1: "Z"})))
        with pytest.raises(NotImplementedError):
            srv.wait(t)
        # a tiny request still works after the failures
        spec, hspec = make_request(rng, 9, 1)
        e, g, _ = srv.wait(srv.submit(9, W.to_circuit(spec), W.to_operator(hspec)))
        assert np.isfinite(e.real)


def test_wait_timeout():
    rng = np.random.default_rng(55)
    spec, hspec = make_request(rng, 22, 12)
    with Server(dtype=np.complex64, memory_bytes=1 << 30, max_active=4) as srv:
        t = srv.submit(22, W.to_circuit(spec), W.to_operator(hspec))
        with pytest.raises(TimeoutError):
            srv.wait(t, timeout=0.0)
        srv.wait(t)


def test_cancel_queued_and_running_requests():
    """vqc_serve_cancel: a request still waiting for admission (one slot, the
    slot taken) is dropped at once; a running one is retired at the next
    iteration with its memory back in the budget; the others finish with the
    same results as alone."""
    from vqcb200._lib import Cancelled
    rng = np.random.default_rng(56)
    big = make_request(rng, 22, 12)
    small = [make_request(rng, 10, 2) for _ in range(3)]
    with Server(dtype=np.complex64, memory_bytes=1 << 30, max_active=1) as srv:
        t_run = srv.submit(22, W.to_circuit(big[0]), W.to_operator(big[1]))
        ts = [srv.submit(10, W.to_circuit(s), W.to_operator(h)) for s, h in small]
        t_queued = ts[1]
        assert srv.cancel(t_queued) is True
        assert srv.cancel(t_run) is True
        with pytest.raises(Cancelled):
            srv.wait(t_run)
        with pytest.raises(Cancelled):
            srv.wait(t_queued)
        for i in (0, 2):
            e, g, _ = srv.wait(ts[i])
            e_ref, g_ref = O.energy_and_gradient(O.from_spec(small[i][0]), O.terms_from_spec(small[i][1]),
                                                 O.zero_state(10), nthreads=4)
            assert abs(e - e_ref) / max(abs(e_ref), 1.0) < 1e-5
            assert rel(g, g_ref) < 1e-5
        # a finished request cannot be cancelled; its result is still collected
        t_done = srv.submit(10, W.to_circuit(small[0][0]), W.to_operator(small[0][1]))
        while srv.stats()["completed"] < 3:
            time.sleep(0.01)
        assert srv.cancel(t_done) is False
        srv.wait(t_done)
        st = srv.stats()
    assert st["completed"] == 3 and st["bytes_admitted"] == 0


def test_poisoned_request_is_rejected_and_isolated():
    """A request carrying a NaN gate entry (or an infinite Pauli coefficient)
    is refused at submission; requests submitted around it, batched together,
    give the oracle's results."""
    rng = np.random.default_rng(57)
    reqs = [(int(n),) + make_request(rng, int(n), 3) for n in rng.integers(9, 15, 6)]
    with Server(dtype=np.complex64, memory_bytes=1 << 30, max_active=16) as srv:
        ts = [srv.submit(n, W.to_circuit(s), W.to_operator(h)) for n, s, h in reqs[:3]]
        poisoned = V.QCircuit([V.RxGate(1, float("nan"), isparas=True), V.CNOTGate(1, 2)])
        with pytest.raises(ValueError):
            srv.submit(9, poisoned, V.QubitsOperator(V.pauli({1: "Z"})))
        with pytest.raises(ValueError):
            srv.submit(9, W.to_circuit(reqs[0][1][:4]),
                       V.QubitsOperator(V.QubitsTerm({1: "Z"}, coeff=float("inf"))))
        ts += [srv.submit(n, W.to_circuit(s), W.to_operator(h)) for n, s, h in reqs[3:]]
        out = [srv.wait(t) for t in ts]
    for (n, spec, hspec), (e, g, _) in zip(reqs, out):
        e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=4)
        assert abs(e - e_ref) / max(abs(e_ref), 1.0) < 1e-5
        assert rel(g, g_ref) < 1e-5


def test_slow_client_does_not_hold_the_server():
    """A client that never collects its results: the loop still finishes every
    request and returns its device memory to the budget; the results stay
    available until collected (or the server closes)."""
    rng = np.random.default_rng(58)
    reqs = [make_request(rng, 12, 3) for _ in range(8)]
    with Server(dtype=np.complex64, memory_bytes=64 << 20, max_active=2) as srv:
        ts = [srv.submit(12, W.to_circuit(s), W.to_operator(h)) for s, h in reqs]
        # collect only the last one; the others are left waiting for a client
        srv.wait(ts[-1])
        deadline = time.time() + 60
        while srv.stats()["completed"] < len(reqs) and time.time() < deadline:
            time.sleep(0.01)
        st = srv.stats()
        assert st["completed"] == len(reqs)
        assert st["bytes_admitted"] == 0 and st["running"] == 0
        e, g, _ = srv.wait(ts[0], timeout=0.0)  # finished long ago: no wait needed
        assert np.isfinite(e.real) and g.shape == (36 * 2,)
