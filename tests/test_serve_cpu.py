"""Host logic of the serving loop: the table store's LRU order, byte budget
and table-count limit (CPU tensors stand in for device arrays)."""
import torch

from hashgraph_b200.serve import TableStore


class _T:
    def __init__(self, nbytes):
        self.offsets = torch.empty(1, dtype=torch.int32)
        self.keys = torch.empty(nbytes // 8, dtype=torch.int64)
        self.idx = None


def _bytes(t):
    return TableStore.table_bytes(t)


def test_lru_order_and_count_limit():
    s = TableStore(budget_bytes=1 << 40, max_tables=3)
    for i in range(3):
        s.make_room(80)
        s.put(i, _T(80))
    s.get(0)                       # 0 is now the most recent
    s.make_room(80)
    s.put(3, _T(80))
    assert list(s.tables) == [2, 0, 3]  # 1 was least recently used and went first
    assert s.evictions == 1


def test_byte_budget():
    t = _T(800)
    s = TableStore(budget_bytes=3 * _bytes(t), max_tables=100)
    for i in range(5):
        s.make_room(_bytes(t))
        s.put(i, _T(800))
        assert s.bytes <= s.budget
    assert set(s.tables) == {2, 3, 4}
    assert s.evictions == 2


def test_replacing_a_table_keeps_the_byte_count():
    s = TableStore(budget_bytes=1 << 40, max_tables=10)
    s.put(7, _T(800))
    b = s.bytes
    s.put(7, _T(800))
    assert s.bytes == b and len(s.tables) == 1
