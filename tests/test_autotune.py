"""Autotuner plumbing on the host: explicit symbolic options reach the
analysis, and the cache lookup picks this device's entry for the shape and
precision at the nearest tuned batch width (defaults otherwise)."""
import json

from orbit_b200 import autotune
from orbit_b200.symbolic import Symbolic


def test_options_reach_the_analysis():
    base = Symbolic(6, 10, 12, leaf_cells=16, chunk_elems=2048, tc_min_n=32, subtree_div=0)
    small_leaf = Symbolic(6, 10, 12, leaf_cells=8, chunk_elems=2048, tc_min_n=32, subtree_div=0)
    big_chunk = Symbolic(6, 10, 12, leaf_cells=16, chunk_elems=8192, tc_min_n=32, subtree_div=0)
    assert small_leaf.info["nsuper"] > base.info["nsuper"]
    assert big_chunk.info["solve_items_per_bin"] < base.info["solve_items_per_bin"]
    assert base.info["leaf_cells"] == 16
    # a lower tensor-core threshold puts more supernodes on the tensor-core path (larger packs)
    lo = Symbolic(15, 24, 28, leaf_cells=32, tc_min_n=16)
    hi = Symbolic(15, 24, 28, leaf_cells=32, tc_min_n=200)
    assert lo.info["tc_pack_floats"] > hi.info["tc_pack_floats"]


def test_cache_lookup(tmp_path):
    path = tmp_path / "tuned.json"
    opts12 = {"leaf_cells": 48, "chunk_elems": 16384, "tc_min_n": 32, "subtree_div": 0}
    opts4 = {"leaf_cells": 64, "chunk_elems": 4096, "tc_min_n": 48, "subtree_div": 1024}
    cache = {
        autotune._key("devA", (15, 72, 80), 32, 12): {"options": opts12, "ms_per_batch": 1.0},
        autotune._key("devA", (15, 72, 80), 32, 4): {"options": opts4, "ms_per_batch": 1.0},
        autotune._key("devB", (15, 72, 80), 32, 12): {"options": opts4, "ms_per_batch": 1.0},
    }
    path.write_text(json.dumps(cache))
    assert autotune.tuned_options((15, 72, 80), 32, 12, device="devA", path=str(path)) == opts12
    assert autotune.tuned_options((15, 72, 80), 32, 10, device="devA", path=str(path)) == opts12
    assert autotune.tuned_options((15, 72, 80), 32, 3, device="devA", path=str(path)) == opts4
    assert autotune.tuned_options((15, 72, 80), 64, 12, device="devA", path=str(path)) == autotune.DEFAULTS
    assert autotune.tuned_options((15, 40, 80), 32, 12, device="devA", path=str(path)) == autotune.DEFAULTS
    assert autotune.tuned_options((15, 72, 80), 32, 12, device="devC", path=str(path)) == autotune.DEFAULTS
