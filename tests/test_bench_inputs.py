"""The benchmark's committed input permutation equals what the library computes
today (tests/golden/bench/make_bench_inputs.py regenerates it), and is a permutation."""
from __future__ import annotations

import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _maker():
    spec = importlib.util.spec_from_file_location("make_bench_inputs", os.path.join(HERE, "golden", "bench", "make_bench_inputs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_permutation_fixture_is_current():
    mk = _maker()
    fixed = mk.load()
    assert len(fixed) == 64 ** 3
    assert np.array_equal(np.sort(fixed), np.arange(64 ** 3, dtype=np.int32))
    assert np.array_equal(fixed, mk.compute())
