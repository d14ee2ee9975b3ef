"""The byte models behind bench.py's roofline fractions (no GPU): the DO-BFS
level formula and the build formula's pass count, checked on hand-worked
cases."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_bfs_level_bytes_by_hand():
    bench = _bench()
    V = 1000
    trace = [
        {"direction": 0, "frontier": 1, "edges": 10, "discovered": 10},    # TD: 12*1 + 8*10 + 12*10
        {"direction": 1, "frontier": 10, "edges": 500, "discovered": 600},  # BU: 4V + 8U + 4*500 + 12*600
        {"direction": 0, "frontier": 50, "edges": 80, "discovered": 5},     # TD: 12*50 + 8*80 + 12*5
    ]
    total, per = bench.bfs_bytes(trace, V)
    td = (12 * 1 + 8 * 10 + 12 * 10) + (12 * 50 + 8 * 80 + 12 * 5)
    U = V - 1 - 10                      # unvisited entering the bottom-up level
    bu = 4 * V + 8 * U + 4 * 500 + 12 * 600
    assert per == {"td": td, "bu": bu}
    assert total == td + bu


def test_sort_pass_count_follows_the_id_width():
    bench = _bench()
    # P = ceil(ceil(log2 V) / 8): 3 passes for 22-bit ids, 4 for 26-bit ones
    for V, P in ((1 << 22, 3), (1 << 26, 4), (1 << 24, 3), (1 << 16, 2), (2, 1)):
        assert bench.sort_passes(V) == P
