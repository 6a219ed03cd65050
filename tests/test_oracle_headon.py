"""The checker's numpy head-on builder (oracle/headon.py) makes the same model,
array for array, as the engine's scenario builder, so the benchmark's
reference arm runs the same crash without loading the engine library."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import headon as H  # noqa: E402

from crushrs_b200 import scenarios as S  # noqa: E402


def _same(a, b):
    ka, kb = H.desc_arrays(a), H.desc_arrays(b)
    assert sorted(ka) == sorted(kb)
    for k in ka:
        if ka[k] is None or kb[k] is None:
            assert ka[k] is None and kb[k] is None, k
            continue
        assert ka[k].shape == kb[k].shape, k
        assert np.array_equal(ka[k], kb[k]), k


@pytest.mark.parametrize("which", ["plain", "refined"])
def test_numpy_headon_equals_engine_builder(which):
    if which == "plain":
        ours, eng = H.plain_headon(), S.Model.build(S.plain_headon())
    else:
        ours, eng = H.refined_headon(max_steps=5000), S.Model.build(S.refined_headon(max_steps=5000))
    _same(ours.desc, eng.desc)


def test_refined_headon_sizes():
    m = H.refined_headon()
    # two blocks of 0.05 m (36x30x138 and 36x24x150) and the road slab
    assert (m.hex_part == 0).sum() == 36 * 30 * 138
    assert (m.hex_part == 1).sum() == 36 * 24 * 150
    assert m.desc.n_contacts == 4 and m.desc.n_vehicles == 2
