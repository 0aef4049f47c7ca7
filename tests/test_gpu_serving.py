"""Serving loop on the device: each result is the same alone and in the
mix, and the batched form reproduces the single-excitation form."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BATCH_TOL = 1e-6  # relative to the largest |V| / |I|: batched vs one excitation per handle


def _stream():
    from magnelio_b200 import serving

    return serving.request_stream(6, seed=11, mean_gap=0.001, cells=(16**3, 28**3), steps=(300, 600),
                                  ports=(2, 4), n_freq=7)


def test_results_are_the_same_alone_and_in_the_mix():
    from magnelio_b200 import serving

    reqs = _stream()
    loop = serving.ServingLoop(max_slots=4, slice_steps=128)
    mixed = loop.run(reqs)
    assert mixed.n == len(reqs)
    assert mixed.mean_active > 1.0
    for req, res in zip(reqs, mixed.results):
        alone = serving.ServingLoop(max_slots=1, slice_steps=97).run([req])
        a = alone.results[0]
        assert np.array_equal(a.V, res.V) and np.array_equal(a.I, res.I)
        assert np.array_equal(a.S, res.S)
        assert res.footprint >= res.device_bytes  # the admission estimate covers what the handle held


def test_batched_form_matches_one_excitation_per_handle():
    from magnelio_b200 import serving

    reqs = _stream()[:3]
    batched = serving.ServingLoop(max_slots=4, slice_steps=128).run(reqs)
    plain = serving.ServingLoop(slice_steps=128).run(reqs, plain=True)
    for a, b in zip(batched.results, plain.results):
        assert a.rid == b.rid
        sv = float(np.max(np.abs(b.V)))
        si = float(np.max(np.abs(b.I)))
        assert float(np.max(np.abs(a.V - b.V))) <= BATCH_TOL * sv
        assert float(np.max(np.abs(a.I - b.I))) <= BATCH_TOL * si
