"""Admission control of cumm.serve (CPU): HBM budget and slots."""
import threading

import pytest

from cumm.serve import Admission, SparseEncoder


def test_admission_budget_and_slots():
    a = Admission(budget_bytes=100, slots=2)
    assert a.try_admit(60)
    assert not a.try_admit(50)          # over budget
    assert a.try_admit(40)
    assert not a.try_admit(1)           # no slot
    a.release(60)
    assert a.try_admit(50)
    assert a.used == 90 and a.active == 2
    with pytest.raises(ValueError):
        a.try_admit(200)                # can never fit


def test_admission_release_wakes_waiter():
    a = Admission(budget_bytes=10, slots=1)
    assert a.try_admit(10)
    got = []

    def waiter():
        while not a.try_admit(5):
            a.wait_change(0.05)
        got.append(True)

    t = threading.Thread(target=waiter)
    t.start()
    a.release(10)
    t.join(5)
    assert got == [True]


def test_footprint_monotone():
    assert SparseEncoder.footprint_bytes(10_000) < SparseEncoder.footprint_bytes(400_000)
