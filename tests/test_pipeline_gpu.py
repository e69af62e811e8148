"""HostPipeline (hashgraph_b200.pipeline): batches in pinned host memory,
uploaded, built, probed and downloaded on overlapping streams.  Every batch's
count and pairs must equal one plain build + intersect of the same keys
(the oracle's pairs; a_ref compared through the key it names, since a table
without an index reports CSR positions)."""
import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = from_np_u(a, device="cpu")
    return t.pin_memory()


@pytest.mark.parametrize("kb,with_index", [(8, False), (4, True)])
def test_pipeline_matches_oracle(hg, kb, with_index):
    import torch
    from hashgraph_b200.pipeline import HostPipeline
    n, nq, B = 300_000, 250_000, 262_144
    sizes = [(n, nq), (n // 3, nq), (n, 17), (0, 1000), (n - 5, nq // 2)]
    batches, ref = [], []
    for i, (na, nqi) in enumerate(sizes):
        a = oracle.gen_uniform(na, kb, 10 + i)
        q = oracle.gen_overlap(nqi, a, 0.4, 20 + i) if na else oracle.gen_uniform(nqi, kb, 20 + i)
        batches.append((_pinned(a), _pinned(q)))
        off, k, idx = oracle.build(a, B, True)
        c, pairs = oracle.intersect(off, k, idx, q, pair_cap=4 * max(nqi, 1))
        ref.append((a, q, c, pairs))
    pipe = HostPipeline(n, nq, B, key_bytes=kb, with_index=with_index, pair_cap=nq)
    outs = [torch.zeros((nq, 2), dtype=torch.int32).pin_memory() for _ in sizes]
    for rep in range(2):  # the same pipeline twice: buffers are reused
        counts = pipe.run(batches, outs)
        assert hg.device_error() == 0
        for i, (a, q, c, pairs) in enumerate(ref):
            assert counts[i] == c, (rep, i)
            got = outs[i][:c].numpy().view(np.uint32)
            np.testing.assert_array_equal(np.sort(got[:, 1]), np.sort(pairs[:, 1]))
            if with_index:
                key = lambda p: np.sort(p[:, 0].astype(np.uint64) << np.uint64(32) | p[:, 1])  # noqa: E731
                np.testing.assert_array_equal(key(got), key(pairs.astype(np.uint32)))
            elif i == len(ref) - 1:  # a_ref is a CSR position: the last table is still there
                tk = pipe.table.keys[: a.size].cpu().numpy().view(a.dtype)
                np.testing.assert_array_equal(tk[got[:, 0]], q[got[:, 1]])
            else:
                assert got[:, 0].max(initial=0) < max(a.size, 1)


def test_pipeline_rejects_unpinned_and_oversized(hg):
    import torch
    from hashgraph_b200 import HGError
    from hashgraph_b200.pipeline import HostPipeline
    pipe = HostPipeline(1000, 1000, 1024)
    a = torch.zeros(1000, dtype=torch.int64)
    with pytest.raises(HGError):
        pipe.run([(a, a.pin_memory())])
    big = torch.zeros(1001, dtype=torch.int64).pin_memory()
    with pytest.raises(HGError):
        pipe.run([(big, a.pin_memory())])
