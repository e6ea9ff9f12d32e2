"""Admission policy of the serving loop (host logic, no GPU): FIFO order, slot limit, HBM budget, head-of-line
waiting, release, requests that can never fit; and the size estimate's scaling."""
import pytest

from diffractom_b200.serving import Scheduler, estimate_request_bytes


def test_fifo_slots_and_budget():
    s = Scheduler(max_slots=2, budget_bytes=100)
    for rid, nb in [(0, 40), (1, 50), (2, 30), (3, 10)]:
        s.enqueue(rid, nb)
    assert s.admit() == [0, 1]                 # two slots
    assert s.admit() == []                     # slots full
    s.release(0)
    assert s.admit() == [2]                    # 50 + 30 <= 100
    s.release(1)
    assert s.admit() == [3]
    assert s.used() == 40 and s.queue == []


def test_head_of_line_waits_for_memory():
    s = Scheduler(max_slots=4, budget_bytes=100)
    s.enqueue(0, 70)
    s.enqueue(1, 60)
    s.enqueue(2, 10)
    assert s.admit() == [0]                    # 1 does not fit next to 0; 2 waits behind it (FIFO)
    s.release(0)
    assert s.admit() == [1, 2]
    s2 = Scheduler(max_slots=4, budget_bytes=100)
    s2.enqueue(0, 30)
    assert s2.admit(free_bytes=20) == []       # the device's free memory also bounds admission
    assert s2.admit(free_bytes=40) == [0]


def test_oversized_and_bad_arguments():
    s = Scheduler(max_slots=1, budget_bytes=100)
    with pytest.raises(MemoryError):
        s.enqueue(0, 101)
    with pytest.raises(ValueError):
        Scheduler(max_slots=0, budget_bytes=1)


def test_estimate_grows_with_the_request():
    cfg = dict(Nx=64, Ny=64, My=67, N_Omega=90, N_eta=90)
    small = estimate_request_bytes(cfg, 500, 3)
    assert estimate_request_bytes(cfg, 1000, 3) > small
    assert estimate_request_bytes({**cfg, "Nx": 128, "Ny": 128}, 500, 3) > small
    assert estimate_request_bytes(cfg, 500, 8) > small
    assert estimate_request_bytes(cfg, 500, 3, precision="bf16") > small      # + the dense BF16 PF
