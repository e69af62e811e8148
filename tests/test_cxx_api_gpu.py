"""The C++ classes that keep the reference's API (SingleHashGraph,
MultiHashGraph), exercised through the reference's own test mains rewritten
over them (hashgraph_b200/_lib/multi-hash, sing-hash): same arguments, same
sequential inputs, with `check` -- buildSingle() cross-checks the exported
reference-layout table against the plain build, and the intersect output is
compared with a CPU multiset join.  A mismatch exits non-zero."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "hashgraph_b200", "_lib")

pytestmark = pytest.mark.gpu


def _run(exe, *args):
    path = os.path.join(LIB, exe)
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hashgraph_b200", "csrc")], check=True)
    r = subprocess.run([path, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "error" not in r.stderr.lower(), r.stderr[:2000]
    return r.stdout


@pytest.mark.parametrize("n_a,n_b,table", [(100_000, 60_000, 100_000), (1 << 22, 3 << 20, 1 << 22),
                                           (5000, 9000, 4099)])
def test_multi_hash_intersect_check(hg, n_a, n_b, table):
    # argv: size maxkey binCount gpuCount lrbBins check countSizeB intersect (tableSize = maxkey)
    out = _run("multi-hash", n_a, table, 16000, 1, 16000, "check", n_b, "intersect")
    assert "multi intersect() time:" in out
    assert f"intersect check ok: {min(n_a, n_b)} matches" in out


@pytest.mark.parametrize("n,table", [(1_000_000, 1_000_000), (1 << 22, 1 << 21), (777, 1)])
def test_multi_hash_build_check(hg, n, table):
    out = _run("multi-hash", n, table, 16000, 1, 16000, "check", 1, "build")
    assert "multi buildTable() time:" in out


def test_single_hash_build(hg):
    out = _run("sing-hash", 1 << 22, 1 << 23, 16000)
    assert "single buildTable() time:" in out


@pytest.mark.parametrize("gpus,n_a,n_b,table", [(2, 1_000_000, 700_000, 1_000_000), (3, 100_000, 60_000, 99_991),
                                                (8, 1 << 22, 3 << 20, 1 << 22), (8, 5, 9, 1), (4, 7, 3, 10)])
def test_multi_hash_several_gpus_intersect_check(hg, gpus, n_a, n_b, table):
    """gpuCount > 1: the OpenMP team builds A (finding the splits), B on A's
    splits, and intersects shard by shard; every GPU's output together must
    be the multiset join, and each shard's exported table must equal the
    single table's range.  With one device all shards share it (their
    kernels never wait on each other; the threads meet on the host)."""
    out = _run("multi-hash", n_a, table, 16000, gpus, 16000, "check", n_b, "intersect")
    assert "multi intersect() time:" in out
    assert f"intersect check ok: {min(n_a, n_b)} matches" in out


@pytest.mark.parametrize("gpus,n,table", [(2, 1_000_000, 1_000_000), (5, 1 << 21, 1 << 21), (8, 3, 100)])
def test_multi_hash_several_gpus_build_check(hg, gpus, n, table):
    out = _run("multi-hash", n, table, 1000, gpus, 16000, "check", 1, "build")
    assert "multi buildTable() time:" in out


def test_multi_hash_rejects_bad_gpu_count(hg):
    path = os.path.join(LIB, "multi-hash")
    r = subprocess.run([path, "1000", "1000", "16000", "65", "16000", "nocheck", "1000", "build"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "gpuCount" in r.stderr
