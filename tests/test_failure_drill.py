"""Failure drill of the multi-rank path on CPU ranks (gloo, no GPU): a rank
leaves between steps, the others find out on the host and report it, and a
collective already waiting for the dead rank ends with the process group's
short timeout instead of hanging.  Nothing here faults or waits on a GPU."""
import datetime
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _step(rank, k):
    """one step's exchange: the energy sums of the step (all-reduce)"""
    import torch.distributed as dist
    from wvlh.shard import allreduce_energies
    e = torch.full((3,), float(rank + k), dtype=torch.float64)
    return allreduce_energies(e, -e, torch.ones(3, dtype=torch.float64))


def _worker(rank, world, port, sport, leaver, mode, out):
    import torch.distributed as dist
    from wvlh.shard import RankFailure, StepMonitor
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=4))
    # the store is served by the test process, so it outlives every rank
    store = dist.TCPStore("127.0.0.1", sport, is_master=False, timeout=datetime.timedelta(seconds=30))
    mon = StepMonitor(store, rank, world)
    log = []
    try:
        for k in range(3):
            if rank == leaver and k == 1:
                log.append("left")
                out[rank] = log
                return          # leaves between steps, with nothing in flight
            if mode == "monitor":
                mon.barrier(k, timeout=3.0)
            log.append(_step(rank, k))
    except RankFailure as e:
        log.append(("failure", e.step, e.missing))
    except RuntimeError as e:          # the collective's own timeout
        log.append(("timeout", type(e).__name__))
    out[rank] = log
    # no destroy_process_group on a broken group: the process exits


@pytest.mark.parametrize("world,leaver", [(2, 1), (3, 2)])
def test_rank_leaving_between_steps_is_reported(world, leaver):
    import torch.distributed as dist
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    sport = _free_port()
    server = dist.TCPStore("127.0.0.1", sport, is_master=True, wait_for_workers=False,
                           timeout=datetime.timedelta(seconds=30))
    mp.spawn(_worker, args=(world, _free_port(), sport, leaver, "monitor", out), nprocs=world, join=True)
    del server
    assert out[leaver][-1] == "left"
    for r in range(world):
        if r == leaver:
            continue
        log = out[r]
        assert len(log) == 2
        assert abs(log[0][0] - sum(3.0 * q for q in range(world))) < 1e-12   # step 0 completed
        assert log[1] == ("failure", 1, [leaver])


def test_collective_waiting_for_a_dead_rank_times_out():
    """Without the monitor the survivor enters the step's all-reduce; the
    process group's 4 s timeout ends it with an error on the host."""
    import torch.distributed as dist
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    sport = _free_port()
    server = dist.TCPStore("127.0.0.1", sport, is_master=True, wait_for_workers=False,
                           timeout=datetime.timedelta(seconds=30))
    mp.spawn(_worker, args=(2, _free_port(), sport, 1, "bare", out), nprocs=2, join=True)
    del server
    assert out[1][-1] == "left"
    assert out[0][-1][0] == "timeout"
