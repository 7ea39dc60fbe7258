"""Subtree keys, detection and cache marking of libsr_eval.so (host side, no
GPU) against the reference's outputs (tests/golden)."""
import numpy as np

from conftest import load_golden
import symbolic_regression_gpu_b200 as sg


def test_flat_keys_bit_exact():
    pop, d = load_golden("hash_kat.npz")
    keys = []
    for t, v in pop:
        sizes, _ = sg.subtree_hashes(t, v)
        for i in range(t.size):
            keys.append(sg.subtree_key(t[i:i + sizes[i]], v[i:i + sizes[i]]))
    assert (np.array(keys, np.uint64) == d["flat_keys"]).all()


def test_merkle_hashes_bit_exact():
    pop, d = load_golden("hash_kat.npz")
    sizes, hashes = zip(*(sg.subtree_hashes(t, v) for t, v in pop))
    assert (np.concatenate(sizes) == d["sizes"]).all()
    assert (np.concatenate(hashes) == d["merkle"]).all()


def test_detection_matches_reference():
    pop, d = load_golden("detect.npz")
    stats, groups = sg.detect_subtrees(pop, 3, 10)
    assert stats["num_subtrees"] == int(d["num_subtrees"])
    assert stats["covered_tokens"] == int(d["covered_tokens"])
    assert stats["coverage"] == float(d["coverage"])
    assert stats["avg_subtree_size"] == float(d["avg_subtree_size"])
    # Identical key set; each key with the same size and occurrence count.
    ref = {int(k): (int(s), int(c)) for k, s, c in
           zip(d["group_key"], d["group_size"], d["group_count"])}
    ours = {int(k): (int(s), int(c)) for k, s, c in
            zip(groups["key"], groups["size"], groups["count"])}
    assert ours == ref
    # Largest first, as the reference orders groups.
    assert (np.diff(groups["size"]) <= 0).all()


def test_cache_marking_bit_exact():
    pop, d = load_golden("detect.npz")
    hints = sg.mark_cached(pop, d["mark_keys"], d["mark_slots"])
    assert (hints == d["mark_hints"]).all()
    hints_half = sg.mark_cached(pop, d["mark_keys"][::2], d["mark_slots"][::2])
    assert (hints_half == d["mark_half_hints"]).all()


def test_empty_cache_marks_nothing():
    pop, _ = load_golden("detect.npz")
    hints = sg.mark_cached(pop, np.zeros(0, np.uint64), np.zeros(0, np.int32))
    assert (hints == -1).all()
