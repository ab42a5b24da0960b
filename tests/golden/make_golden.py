"""Writes reference_kats.json: the known-answer tests of the diskann-rs test
suite that pin the search path, transcribed by hand from the reference test
sources (cited per case).  The reference publishes no numeric golden outputs
and its Rust toolchain is absent, so these assertions are what pins the
oracle and the GPU path to the reference's behaviour.

Run: python tests/golden/make_golden.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

FIVE_NODE_POSITIONS = [[0.0, 0.0], [1.0, 0.0], [2.0, 0.0], [0.0, 2.0], [2.0, 1.0]]
FIVE_NODE_NEIGHBORS = [[1, 3], [0, 2], [1, 4], [0, 4], [2, 3]]

KATS = {
    # src/lib.rs:1349-1398 test_beam_search_small_graph (DistL2 = euclidean)
    "beam_search_small_graph": {
        "positions": FIVE_NODE_POSITIONS,
        "neighbors": FIVE_NODE_NEIGHBORS,
        "query": [2.1, 0.9],
        "start": [0],
        "beam_width": 5,
        "k": 3,
        "metric": "euclidean",
        "expect_len": 3,
        "expect_prefix": [4, 2],
    },
    # src/lib.rs:1400-1436 test_beam_search_with_filter (odd ids only)
    "beam_search_with_filter": {
        "positions": FIVE_NODE_POSITIONS,
        "neighbors": FIVE_NODE_NEIGHBORS,
        "query": [2.1, 0.9],
        "start": [0],
        "beam_width": 5,
        "k": 3,
        "expanded_beam": 10,
        "max_iterations": 20,
        "early_term_factor": 1.5,
        "allowed": [1, 3],
        "expect_contains": [1, 3],
        "metric": "euclidean",
    },
    # src/lib.rs:1319-1346 test_candidate_ordering
    "candidate_ordering": {"cands": [[1.0, 0], [2.0, 1], [0.5, 2]], "min_order": [2, 0, 1], "max_top": 1},
    # src/lib.rs:1439-1469 test_prune_neighbors_alpha (DistL2)
    "prune_alpha": {
        "vectors": [[0.0, 0.0], [1.0, 0.0], [1.2, 0.0], [0.0, 2.0]],
        "node": 0,
        "cands": [1, 2, 3],
        "max_degree": 3,
        "alpha": 1.0,
        "metric": "euclidean",
        "expect_contains": [1, 3],
    },
    # src/lib.rs:1472-1496 test_prune_neighbors_max_degree (DistL2)
    "prune_max_degree": {
        "vectors": [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [2.0, 0.0], [0.0, 2.0]],
        "node": 0,
        "cands": [1, 2, 3, 4, 5],
        "alpha": 1.2,
        "metric": "euclidean",
        "degree_to_len": [[2, 2], [5, 5], [1, 1]],
    },
    # src/lib.rs:1163-1187 test_persistence_and_open / :1290-1312 from_shared_bytes
    "square_best": {
        "vectors": [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]],
        "query": [0.9, 0.9],
        "k": 2,
        "beam_width": 8,
        "metric": "euclidean",
        "expect_first": 3,
    },
    # src/lib.rs:1090-1111 test_small_index_l2
    "small_index_l2": {
        "vectors": [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [0.5, 0.5]],
        "query": [0.1, 0.1],
        "k": 3,
        "beam_width": 8,
        "metric": "euclidean",
        "expect_len": 3,
        "first_within": 1.0,
    },
    # src/lib.rs:1114-1140 test_cosine
    "cosine_direction": {
        "vectors": [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 1.0, 0.0], [1.0, 0.0, 1.0]],
        "query": [2.0, 0.0, 0.0],
        "k": 2,
        "beam_width": 8,
        "metric": "cosine",
        "min_cos_first": 0.7,
    },
    # src/lib.rs:1190-1232 test_grid_connectivity (5x5 grid, R=4, L_build=64, alpha=1.5)
    "grid_connectivity": {
        "grid": 5,
        "max_degree": 4,
        "build_beam_width": 64,
        "alpha": 1.5,
        "k": 10,
        "beam_width": 32,
        "metric": "euclidean",
        "miss_first_within": 2.0,
        "top5_within": 5.0,
    },
    # tests/correctness.rs:294-317 test_single_vector_index
    "single_vector": {"vectors": [[1.0, 2.0, 3.0]], "queries": [[1.0, 2.0, 3.0], [0.0, 0.0, 0.0]],
                      "ks": [1, 10], "beam_width": 8, "metric": "euclidean", "expect": [[0], [0]]},
    # tests/correctness.rs:320-342 test_two_vector_index
    "two_vectors": {"vectors": [[0.0, 0.0], [10.0, 10.0]], "queries": [[0.1, 0.1], [9.9, 9.9]], "k": 2,
                    "beam_width": 8, "metric": "euclidean", "expect": [[0, 1], [1, 0]]},
    # tests/correctness.rs:380-402 test_identical_vectors
    "identical_vectors": {"vectors": [[1.0, 2.0, 3.0]] * 10, "query": [1.0, 2.0, 3.0], "k": 5,
                          "beam_width": 8, "metric": "euclidean", "expect_len": 5, "max_dist": 1e-6},
    # src/filtered.rs:519-560 and python/tests/tests.py:74-94: Filter truth tables
    "filters": [
        {"filter": ["eq", 0, 5], "true": [[5, 10]], "false": [[4, 10], []]},
        {"filter": ["in", 0, [1, 3, 5]], "true": [[1], [3], [5]], "false": [[2]]},
        {"filter": ["range", 0, 10, 20], "true": [[10], [15], [20]], "false": [[9], [21]]},
        {"filter": ["and", [["eq", 0, 5], ["gt", 1, 10]]], "true": [[5, 15]], "false": [[5, 5], [4, 15]]},
        {"filter": ["or", [["eq", 0, 5], ["eq", 0, 10]]], "true": [[5], [10]], "false": [[7]]},
        {"filter": ["and", [["eq", 0, 3], ["range", 1, 10, 20], ["in", 2, [7, 8, 9]]]],
         "true": [[3, 10, 7], [3, 20, 9]], "false": [[2, 10, 7], [3, 21, 7], [3, 15, 99]]},
        {"filter": ["or", [["lt", 0, 2], ["gt", 0, 8]]], "true": [[1], [9]], "false": [[5]]},
        {"filter": ["none"], "true": [[]], "false": []},
    ],
    # src/rabitq.rs:296,314: padded dim and code size
    "rabitq_sizes": {"padded": [[100, 128], [128, 128], [768, 1024], [1, 64]], "code_size": [[128, 24], [1024, 136]]},
}


def main():
    path = os.path.join(HERE, "reference_kats.json")
    with open(path, "w") as f:
        json.dump(KATS, f, indent=1, sort_keys=True)
    print(path)


if __name__ == "__main__":
    main()
