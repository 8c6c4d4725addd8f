"""Host-side pieces of bench.py on CPU: the one-server queue that turns the
plain driver's measured per-job times into served latencies (_fifo)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_fifo_serves_in_arrival_order():
    # jobs arrive at 0, 1, 1.5 and 10 s and take 2, 1, 1 and 0.5 s: the
    # second and third wait behind the first, the fourth finds the server idle
    arrivals = np.array([0.0, 1.0, 1.5, 10.0])
    service = np.array([2.0, 1.0, 1.0, 0.5])
    lat, finish = bench._fifo(arrivals, service)
    assert np.allclose(finish, [2.0, 3.0, 4.0, 10.5])
    assert np.allclose(lat, [2.0, 2.0, 2.5, 0.5])


def test_fifo_takes_arrival_order_not_index_order():
    arrivals = np.array([5.0, 0.0, 1.0])
    service = np.array([1.0, 3.0, 1.0])
    lat, finish = bench._fifo(arrivals, service)
    # served as job 1 (0..3), job 2 (3..4), job 0 (5..6)
    assert np.allclose(finish, [6.0, 3.0, 4.0])
    assert np.allclose(lat, [1.0, 3.0, 3.0])
