"""Serving loop on the device: each result is the same alone and in the
mix, the batched form reproduces the single-excitation form, and a served
S-matrix (waveguide ports with their modes solved on the device, or lumped
ports) meets the float64 oracle's."""

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


S_TOL = 1e-3      # |S_gpu - S_oracle|, linear
PHASE_TOL = 0.1   # degrees, where |S| > 0.05


def test_served_s_matrix_meets_the_fp64_oracle():
    """Float32 batched serving vs the float64 CPU oracle on the same
    request: the S-matrix agrees to |dS| <= 1e-3 and 0.1 degree."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import serving, workloads

    reqs = serving.request_stream(1, seed=5, mean_gap=0.0, cells=(14**3, 14**3), steps=(900, 900), ports=(2, 2),
                                  n_freq=9, port_kind="lumped")
    req = reqs[0]
    res = serving.ServingLoop(max_slots=1, slice_steps=300).run([req]).results[0]
    prob = req.build(None).materialize()  # host arrays for the oracle
    Vs, Is = [], []
    for b in range(req.n_ports):
        r = OracleRun(prob, b=b).run(req.steps)
        Vs.append(np.array(r.V))
        Is.append(np.array(r.I))
    S_ref = workloads.s_matrix(np.stack(Vs), np.stack(Is), prob.dt, req.freqs, req.z0, req.n_ports)
    dS = np.abs(res.S - S_ref)
    assert float(dS.max()) <= S_TOL, float(dS.max())
    big = np.abs(S_ref) > 0.05
    dphi = np.degrees(np.abs(np.angle(res.S[big] / S_ref[big])))
    assert float(dphi.max()) <= PHASE_TOL, float(dphi.max())


@pytest.mark.parametrize("plain", [False, True])
def test_device_s_matrix_equals_the_host_assembly_of_the_records(plain):
    """With the V/I histories left on the device (records=False) the served
    S-matrices come from the device post-step; they equal the host assembly
    of the same runs' records to float64 round-off, in the batched and the
    single-excitation forms."""
    from magnelio_b200 import serving

    reqs = _stream()[:3]
    host = serving.ServingLoop(max_slots=4, slice_steps=128).run(reqs, plain=plain)
    dev = serving.ServingLoop(max_slots=4, slice_steps=128, records=False).run(reqs, plain=plain)
    for a, b in zip(host.results, dev.results):
        assert a.rid == b.rid and b.V is None and b.S.shape == a.S.shape
        assert float(np.max(np.abs(a.S - b.S) / np.maximum(1.0, np.abs(a.S)))) < 1e-9


@pytest.mark.parametrize("records", [True, False])
def test_served_modal_s_matrix_meets_the_fp64_oracle(records):
    """A request with two waveguide ports (two TE modes each, ports built
    here with the modes solved on the device) and one lumped port, served
    in float32 with the S-matrix from the host records or the device
    post-step, against the float64 oracle's records through the same
    power-wave maps: |dS| <= 1e-3 and 0.1 degree."""
    from oracle.fit_oracle import OracleRun
    from magnelio_b200 import serving, sparams

    req = serving.request_stream(1, seed=5, mean_gap=0.0, cells=(16**3, 16**3), steps=(900, 900), ports=(3, 3),
                                 modes=(2, 2), n_freq=9)[0]
    res = serving.ServingLoop(max_slots=1, slice_steps=300, records=records).run([req]).results[0]
    prob = req.build(None).materialize()
    n = req.n_ports
    assert n == len(prob.channels) and sum(m.n_modes for m in prob.modal) >= 3
    Vs, Is = [], []
    for b in range(n):
        r = OracleRun(prob, b=b).run(req.steps)
        Vs.append(np.array(r.V))
        Is.append(np.array(r.I))
    maps, icot = serving.ServingLoop.channel_maps(req, prob, n)
    S_ref = sparams.s_matrix(Vs, Is, prob.dt, req.freqs, list(maps), [bool(c) for c in icot], list(range(n)),
                             a_threshold=0.0)
    assert res.S.shape == S_ref.shape
    dS = np.abs(res.S - S_ref)
    assert float(dS.max()) <= S_TOL, float(dS.max())
    big = np.abs(S_ref) > 0.05
    dphi = np.degrees(np.abs(np.angle(res.S[big] / S_ref[big])))
    assert float(dphi.max()) <= PHASE_TOL, float(dphi.max())


def test_device_built_materials_equal_the_host_build():
    """A serving request's material matrices and coefficients built on the
    device (fitb_build_materials) march exactly like the same constants
    built on the host and uploaded: identical fields and V/I."""
    from magnelio_b200 import workloads

    outs = []
    for dev in (True, False):
        p = workloads.waveguide_section(np.random.default_rng(21), cells=22**3, n_inserts=3, ridged=True, n_ports=3,
                                        steps=150, device_setup=dev)
        assert (p.alpha_E is None) == dev
        with p.build_engine("single") as eng:
            eng.step(150)
            outs.append([eng.read_fields(b) for b in range(p.batch)] + [eng.read_vi(b) for b in range(p.batch)])
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
