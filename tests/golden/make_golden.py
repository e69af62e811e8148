"""Generates the golden fixtures in tests/golden/ from the reference itself.

Part `hash` (runs anywhere the reference sources are present): compiles the
reference's own hash_murmur on the host (oracle/ref_hash_driver.cu, built by
`make -C oracle ref` from the reference headers where they lie) and records
its output on edge keys and seeded random keys -> murmur_ref.npz.

Part `multi` (needs a CUDA GPU; the reference's build and intersect only run
on the device): runs the unmodified reference MultiHashGraph with gpuCount = 1
(oracle/_ref/ref_multi, ref_multi32) on small seeded inputs and records the
canonical CSR, the match count and the sorted matched keys -> ref_multi_*.npz,
plus digests of the 2^20-key workload -> ref_multi_digest.json.

    python tests/golden/make_golden.py hash  [--out DIR]
    python tests/golden/make_golden.py multi [--out DIR]
    python tests/golden/make_golden.py timing [--n LOG2] [--key-bytes 8|4]

Part `timing` (GPU): times the reference MultiHashGraph (gpuCount = 1,
sm_100a) on the seeded build + intersect workload -- A = 2^n uniform keys
(seed 3), B = 2^n keys with 25% drawn from A (seed 30), tableSize = 2^n --
with CUDA events as its own test main does, and prints its JSON timing line.

The fixtures only depend on the oracle's generators (oracle/hg_oracle.c), so
the inputs are regenerated from the parameters stored next to each result.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# Small reference runs: (name, key_bytes, n_a, n_b, n_buckets, kind, seed_a, seed_b, frac)
MULTI_CASES = [
    ("u64_uniform", 8, 4096, 4096, 4096, "uniform", 11, 12, 0.5),
    ("u32_uniform_np2", 4, 3000, 5000, 2999, "uniform", 13, 14, 0.25),
    ("u64_dups", 8, 2048, 3072, 1024, "dups", 15, 16, 0.5),
]
DIGEST_CASE = ("u32_config1", 4, 1 << 20, 1 << 20, 1 << 20, "uniform", 1, 2, 0.5)


def make_inputs(key_bytes, n_a, n_b, kind, seed_a, seed_b, frac):
    a = oracle.gen_uniform(n_a, key_bytes, seed_a)
    if kind == "dups":
        a = (a % np.array(97, dtype=a.dtype)).astype(a.dtype)
    b = oracle.gen_overlap(n_b, a, frac, seed_b)
    return a, b


def canonical_csr(offsets, keys):
    keys = keys.copy()
    oracle.canonicalize(offsets.astype(np.uint32), keys, None)
    return keys


def part_hash(out):
    single, multi = oracle.ref_binary("ref_hash_single"), oracle.ref_binary("ref_hash_multi")
    if not single or not multi:
        ref_root = os.environ.get("REF_ROOT", "/root/reference")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF_ROOT={ref_root}"], check=True)
        single, multi = oracle.ref_binary("ref_hash_single"), oracle.ref_binary("ref_hash_multi")
    edge = np.array([0, 1, 2, 42, 0xFFFFFFFF, 1 << 32, (1 << 32) + 5, 0xFFFFFFFFFFFFFFFF,
                     0x8000000000000000, 0x7FFFFFFF, 0x80000000, 0xDEADBEEFCAFEBABE], dtype=np.uint64)
    rand = oracle.gen_uniform(4096, 8, 2024)
    keys = np.concatenate([edge, rand])
    res = {}
    with tempfile.TemporaryDirectory() as td:
        kf, hf = os.path.join(td, "k.u64"), os.path.join(td, "h.u32")
        keys.tofile(kf)
        for name, exe in (("single", single), ("multi", multi)):
            subprocess.run([exe, kf, hf], check=True)
            res[name] = np.fromfile(hf, dtype=np.uint32)
    np.savez_compressed(os.path.join(out, "murmur_ref.npz"), keys=keys, hash_single=res["single"],
                        hash_multi=res["multi"])
    print("murmur_ref.npz:", keys.size, "keys")


def run_ref(exe, a, b, n_buckets, workdir):
    fa, fb = os.path.join(workdir, "a.bin"), os.path.join(workdir, "b.bin")
    a.astype(np.int64 if a.dtype == np.uint64 else np.uint32).tofile(fa)
    b.astype(np.int64 if b.dtype == np.uint64 else np.uint32).tofile(fb)
    r = subprocess.run([exe, fa, str(a.size), fb, str(b.size), str(n_buckets), workdir, "1"],
                       check=True, capture_output=True, text=True)
    timing = json.loads(r.stdout.strip().splitlines()[-1])
    off = np.fromfile(os.path.join(workdir, "A_offsets.i64"), dtype=np.int64)
    kv = np.fromfile(os.path.join(workdir, "A_edges.kv"), dtype=np.uint8)
    # keyval_ind {hkey_t key; int64 ind}: 16 bytes for both key widths (padding)
    rec = kv.reshape(-1, 16)
    if a.dtype == np.uint64:
        ekeys = rec[:, :8].copy().view(np.uint64).ravel()
    else:
        ekeys = rec[:, :4].copy().view(np.uint32).ravel()
    eind = rec[:, 8:].copy().view(np.int64).ravel()
    common = int(np.fromfile(os.path.join(workdir, "common.i64"), dtype=np.int64)[0])
    pk = np.fromfile(os.path.join(workdir, "pairs.key"),
                     dtype=np.uint64 if a.dtype == np.uint64 else np.uint32)
    return off, ekeys, eind, common, np.sort(pk), timing


def part_multi(out):
    cases = []
    with tempfile.TemporaryDirectory() as td:
        for (name, kb, na, nb, nbk, kind, sa, sb, frac) in MULTI_CASES:
            exe = oracle.ref_binary("ref_multi" if kb == 8 else "ref_multi32")
            a, b = make_inputs(kb, na, nb, kind, sa, sb, frac)
            off, ekeys, eind, common, pk, timing = run_ref(exe, a, b, nbk, td)
            ck = canonical_csr(off.astype(np.uint32), ekeys)
            np.savez_compressed(os.path.join(out, f"ref_multi_{name}.npz"),
                                offsets=off.astype(np.uint32), keys=ck, ind=eind, common=common,
                                matched_keys=pk)
            cases.append({"name": name, "key_bytes": kb, "n_a": na, "n_b": nb, "n_buckets": nbk,
                          "kind": kind, "seed_a": sa, "seed_b": sb, "frac": frac, "common": common})
            print(name, "common", common, timing)
        (name, kb, na, nb, nbk, kind, sa, sb, frac) = DIGEST_CASE
        exe = oracle.ref_binary("ref_multi32")
        a, b = make_inputs(kb, na, nb, kind, sa, sb, frac)
        off, ekeys, eind, common, pk, timing = run_ref(exe, a, b, nbk, td)
        ck = canonical_csr(off.astype(np.uint32), ekeys)
        digest = {"name": name, "key_bytes": kb, "n_a": na, "n_b": nb, "n_buckets": nbk, "kind": kind,
                  "seed_a": sa, "seed_b": sb, "frac": frac, "common": common,
                  "offsets_sha256": hashlib.sha256(off.astype(np.uint32).tobytes()).hexdigest(),
                  "canonical_keys_sha256": hashlib.sha256(ck.tobytes()).hexdigest(),
                  "matched_keys_sha256": hashlib.sha256(pk.tobytes()).hexdigest(),
                  "reference_timing": timing}
    with open(os.path.join(out, "ref_multi_cases.json"), "w") as f:
        json.dump({"cases": cases, "digest": digest}, f, indent=1)
    print("digest", digest)


def part_timing(log2n, key_bytes):
    n = 1 << log2n
    exe = oracle.ref_binary("ref_multi" if key_bytes == 8 else "ref_multi32")
    a = oracle.gen_uniform(n, key_bytes, 3)
    b = oracle.gen_overlap(n, a, 0.25, 30)
    with tempfile.TemporaryDirectory() as td:
        fa, fb = os.path.join(td, "a.bin"), os.path.join(td, "b.bin")
        a.astype(np.int64 if key_bytes == 8 else np.uint32).tofile(fa)
        b.astype(np.int64 if key_bytes == 8 else np.uint32).tofile(fb)
        del a, b
        r = subprocess.run([exe, fa, str(n), fb, str(n), str(n), "-", "1"], check=True,
                           capture_output=True, text=True)
    timing = json.loads(r.stdout.strip().splitlines()[-1])
    timing["build_keys_per_s"] = n / timing["build_a_s"]
    timing["build_and_intersect_keys_per_s"] = n / (timing["build_a_s"] + timing["intersect_s"])
    timing["published_composite_keys_per_s"] = n / timing["total_s"]
    print(json.dumps(timing))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("part", choices=["hash", "multi", "timing"])
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--n", type=int, default=28)
    ap.add_argument("--key-bytes", type=int, default=8)
    args = ap.parse_args()
    if args.part == "hash":
        os.makedirs(args.out, exist_ok=True)
        part_hash(args.out)
    elif args.part == "multi":
        os.makedirs(args.out, exist_ok=True)
        part_multi(args.out)
    else:
        part_timing(args.n, args.key_bytes)


if __name__ == "__main__":
    main()
