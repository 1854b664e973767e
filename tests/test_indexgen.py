"""Index-set generator: Python twin, C oracle and the library agree bit for bit,
and the streams match the committed SHA-256 fixtures."""
import json
import os

import numpy as np

from oracle import oracle as O
from paralanczos_b200 import api, indexgen as IG

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_splitmix_known_values():
    # SplitMix64 reference values (Steele, Lea & Flood, OOPSLA 2014) for state 0
    assert IG.splitmix64(0) == 0xE220A8397B1DCDAF
    assert O.lib().orc_splitmix64(0) == 0xE220A8397B1DCDAF


def test_streams_match_golden_sha256():
    gold = json.load(open(os.path.join(GOLD, "indexgen.json")))
    for name, g in gold.items():
        o, i = IG.gen_stream(*g["args"])
        assert IG.stream_sha256(o, i) == g["sha256"], name
        o2, i2 = O.gen_stream(*g["args"])
        assert np.array_equal(o, o2) and np.array_equal(i, i2), name
        o3, i3 = api.gen_stream_host(*g["args"])
        assert np.array_equal(o, o3) and np.array_equal(i, i3), name
        assert i[:o[1]].tolist() == g["first_set"]


def test_sets_distinct_and_in_range():
    o, i = O.gen_stream(11, 0, 2000, 300, 2, 2, 300)
    for s in range(2000):
        S = i[o[s]:o[s + 1]]
        assert len(set(S.tolist())) == len(S)
        assert S.min() >= 0 and S.max() < 300
    # k == n gives a permutation
    S = O.gen_set(4, 9, 64, 64)
    assert sorted(S.tolist()) == list(range(64))


def test_inverse_k_distribution():
    ks = np.array([IG.gen_k(3, s, IG.KDIST_INV_K) for s in range(20000)])
    w = np.array([96, 48, 32, 24, 16, 12, 8, 6, 4, 3]) / 249.0
    freq = np.array([(ks == k).mean() for k in IG.INV_K_VALUES])
    assert np.abs(freq - w).max() < 0.01
    # E[k] of the 1/k mix over {8..256}: 10 values / H, H = sum 1/k = 0.32422
    assert abs(ks.mean() - 10 / 0.3242187) < 0.6


def test_counter_based_resume():
    # set s depends only on (seed, s): a stream split in two equals the whole
    o, i = O.gen_stream(21, 0, 100, 1000, 1, 8, 256)
    o1, i1 = O.gen_stream(21, 0, 37, 1000, 1, 8, 256)
    o2, i2 = O.gen_stream(21, 37, 63, 1000, 1, 8, 256)
    assert np.array_equal(i, np.r_[i1, i2])
