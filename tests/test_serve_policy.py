"""Host logic of the serving loop (no GPU): batch formation and the
admission arithmetic of wvlh.serve."""
from types import SimpleNamespace

from wvlh.serve import Request, client_bytes, form_launch, request_scratch
from wvlh.workloads import free_sphere, full_periodic, poisson_arrivals, serving_clients


def _req(cid, kind, t, scratch=10, norb=4):
    c = SimpleNamespace(id=cid, norb=norb, scratch_bytes=scratch)
    return Request(client=c, kind=kind, t_arrival=t)


def test_form_launch_first_fit_in_arrival_order():
    q = [_req(0, "H", 0), _req(1, "H", 1), _req(0, "H", 2), _req(2, "rho", 3), _req(3, "H", 4, scratch=100),
         _req(4, "H", 5)]
    p = form_launch(q, busy=set(), scratch_cap=35, max_orbitals=100)
    # client 0's second H waits for its first; client 3 does not fit the cap
    assert [r.t_arrival for r in p["H"]] == [0, 1, 5]
    assert [r.t_arrival for r in p["rho"]] == [3]


def test_form_launch_busy_and_oldest_always_taken():
    q = [_req(0, "H", 0, scratch=500), _req(1, "rho", 1), _req(1, "H", 2)]
    p = form_launch(q, busy={(1, "rho")}, scratch_cap=35, max_orbitals=100)
    assert [r.t_arrival for r in p["H"]] == [0]       # the oldest, even above the cap
    assert p["rho"] == []                             # (1, rho) is in flight
    p = form_launch(q, busy=set(), scratch_cap=1000, max_orbitals=6)
    assert [r.t_arrival for r in p["H"]] == [0]       # orbital cap: 4 + 4 > 6
    assert [r.t_arrival for r in p["rho"]] == [1]


def test_resident_and_scratch_bytes():
    lr = full_periodic((16, 12, 10))
    assert client_bytes(lr, 3, 8) == 2 * 3 * lr.ncoeff * 8 + lr.nisf * 16
    F, I = lr.fine, lr.isf
    assert request_scratch(lr, 2, 4) == 2 * 4 * (2 * 20 * F[1] * F[0] + 20 * I[1] * I[0])
    fr = free_sphere((11, 13, 9))
    assert fr.fine == (36, 40, 32) and fr.isf == (51, 55, 47)


def test_serving_workload_shapes():
    cl = serving_clients(nclient=16, seed=9)
    assert len(cl) == 16
    for lr, norb, seed in cl:
        assert all(16 <= n <= 64 for n in lr.n) and 4 <= norb <= 128
        assert lr.periodic in ((1, 1, 1), (0, 0, 0))
    arr = poisson_arrivals(100.0, 500, 16, seed=1)
    t = [a[0] for a in arr]
    assert t == sorted(t) and 3.0 < t[-1] < 7.5   # mean 5 s for 500 arrivals at 100/s
    assert 150 < sum(a[2] == "rho" for a in arr) < 350
