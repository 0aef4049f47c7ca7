"""Serving loop mechanics on a scripted engine and a virtual clock (no GPU):
admission by footprint and slots, arrival order, continuous joining,
latency accounting, batched vs single-excitation results, S-matrix
extraction."""

from __future__ import annotations

import math

import numpy as np
import pytest

from magnelio_b200 import serving, workloads
from oracle.fit_oracle import dense_lowest_eigs


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class ScriptedEngine:
    """Steps cost virtual time; V/I of field set b depend only on the
    problem and the excitation that field set carries."""

    live = []

    def __init__(self, prob, clock, cost_per_cell_step=1e-9):
        self.p = prob
        self.clock = clock
        self.cost = cost_per_cell_step * prob.nx * prob.ny * prob.nz * prob.batch
        self.n = 0
        self.cap = 0
        ScriptedEngine.live.append(self)
        self.closed = False

    def reserve_steps(self, n):
        self.cap = n

    def step(self, k):
        self.n += k
        self.clock.t += self.cost * k

    def sync(self):
        pass

    def query(self):
        return True  # a step costs virtual time when it is issued

    @property
    def n_channels(self):
        return sum(m.n_modes for m in self.p.modal) + len(self.p.lumped)

    def _sources(self, b):
        """Per channel the source series field set b carries."""
        out = []
        for mp in self.p.modal:
            exc = mp.excitation[b] if b < len(mp.excitation) else None
            for m in range(mp.n_modes):
                out.append(exc[1][: self.n] if exc is not None and exc[0] == m else np.zeros(self.n))
        for lp in self.p.lumped:
            out.append(lp.v_src[b][: self.n] if len(lp.v_src[b]) else np.zeros(self.n))
        return out

    def read_vi(self, b):
        P = self.n_channels
        V = np.zeros((self.n, P))
        I = np.zeros((self.n, P))
        rng = np.random.default_rng(self.p.nx * 1000 + self.p.nz)
        coup = rng.uniform(-0.5, 0.5, (P, P)) + np.eye(P)
        for q, src in enumerate(self._sources(b)):
            for j in range(P):
                V[:, j] += coup[j, q] * src
                I[:, j] += 0.01 * coup[q, j] * src
        return V, I

    @property
    def device_bytes(self):
        return serving.estimate_footprint(self.p.nx, self.p.ny, self.p.nz, self.p.batch, self.cap,
                                          len(self.p.lumped)) // 2

    def close(self):
        self.closed = True


def _loop(clock, **kw):
    return serving.ServingLoop(engine_factory=lambda p, prec, dev: ScriptedEngine(p, clock), clock=clock,
                               sleep=clock.sleep, **kw)


def _stream(n=10, steps=(200, 400), port_kind="lumped"):
    kw = {} if port_kind == "lumped" else {"lowest": dense_lowest_eigs, "device_tables": False}
    return serving.request_stream(n, seed=3, mean_gap=0.002, cells=(12**3, 20**3), steps=steps, ports=(2, 4),
                                  n_freq=5, port_kind=port_kind, **kw)


def test_every_request_completes_with_its_own_s_matrix():
    clock = Clock()
    ScriptedEngine.live = []
    stats = _loop(clock, hbm_budget=1 << 40, max_slots=4, slice_steps=64).run(_stream())
    assert stats.n == 10 and [r.rid for r in stats.results] == list(range(10))
    assert all(e.closed for e in ScriptedEngine.live)
    for r in stats.results:
        P = r.S.shape[1]
        assert r.S.shape == (5, P, P) and r.V.shape[0] == P
        assert r.finished >= r.admitted >= r.arrival
    assert 0 < stats.p50 <= stats.p99
    assert stats.mean_active > 1.0  # requests overlapped


def test_slots_and_memory_budget_bound_the_running_set():
    clock = Clock()
    reqs = _stream(8)
    fps = [serving._footprint_of(serving.ServingLoop._problem(r, None), r.steps, "single") for r in reqs]
    budget = int(2.5 * max(fps))
    loop = _loop(clock, hbm_budget=budget, max_slots=8, slice_steps=32)
    seen = []
    orig = loop.engine_factory

    def factory(p, prec, dev):
        e = orig(p, prec, dev)
        seen.append(sum(1 for x in ScriptedEngine.live if not x.closed))
        return e

    ScriptedEngine.live = []
    loop.engine_factory = factory
    stats = loop.run(reqs)
    assert stats.n == 8
    assert stats.peak_bytes <= budget
    assert max(seen) <= 3


def test_batched_and_single_excitation_forms_agree():
    clock = Clock()
    reqs = _stream(5)
    batched = _loop(clock, hbm_budget=1 << 40, max_slots=4, slice_steps=50).run(reqs)
    clock2 = Clock()
    plain = _loop(clock2, hbm_budget=1 << 40, slice_steps=50).run(reqs, plain=True)
    assert plain.n == batched.n == 5
    for a, b in zip(batched.results, plain.results):
        np.testing.assert_allclose(a.V, b.V, rtol=0, atol=0)
        np.testing.assert_allclose(a.S, b.S, rtol=1e-12, atol=0)


def test_s_matrix_of_a_matched_two_port_line():
    """Two ports joined by an ideal delay line of Z0: S11 = S22 = 0,
    |S21| = |S12| = 1."""
    dt, n, z0, d = 1e-12, 4000, 50.0, 25
    t = (np.arange(n) + 1) * dt
    inc = np.exp(-((t - 200e-12) / 40e-12) ** 2)
    V = np.zeros((2, n, 2))
    I = np.zeros((2, n, 2))
    for i in range(2):
        j = 1 - i
        V[i, :, i] = inc
        I[i, :, i] = inc / z0
        out = np.concatenate([np.zeros(d), inc[:-d]])
        V[i, :, j] = out
        I[i, :, j] = -out / z0
    S = workloads.s_matrix(V, I, dt, [2e9, 4e9], z0)
    assert np.max(np.abs(S[:, 0, 0])) < 1e-12 and np.max(np.abs(S[:, 1, 1])) < 1e-12
    np.testing.assert_allclose(np.abs(S[:, 1, 0]), 1.0, rtol=1e-9)
    np.testing.assert_allclose(np.angle(S[:, 1, 0]), np.angle(np.exp(-2j * math.pi * np.array([2e9, 4e9]) * d * dt)),
                               atol=1e-9)


def test_footprint_estimate_counts_the_big_buffers():
    fp = serving.estimate_footprint(64, 64, 64, 4, 1000, 4, [(2, 8), (2, 8)])
    vol = 68 * 66 * 72 + 8 * 72  # rows of nz + 2 rounded up to 8 entries
    assert fp > 2 * 4 * 3 * vol * 4 + 6 * 3 * vol * 4
    # the fused step's second buffer set: fields and psi once more
    fpf = serving.estimate_footprint(64, 64, 64, 4, 1000, 4, [(2, 8), (2, 8)], fused=True)
    assert fpf - fp == 2 * 4 * 3 * vol * 4 + 2 * 4 * 4 * (65 * 65 * 16) * 4  # psi rows padded to 16
    with pytest.raises(TypeError):
        serving.estimate_footprint(64, 64)


def test_each_form_gets_its_stencil_and_a_refusal_keeps_the_default():
    """Single-excitation handles go on the slab step, batched ones keep the
    default kernels; a handle that refuses the form keeps its default."""
    from magnelio_b200._lib import FitbError

    assert serving.serving_stencil(1) == ("fused", 16)
    assert serving.serving_stencil(3) is None

    class Eng:
        def __init__(self, refuse):
            self.refuse = refuse
            self.form = None

        def configure_stencil(self, kind, variant):
            if self.refuse:
                raise FitbError(-4, "dispersive materials need an in-place stencil mode")
            self.form = (kind, variant)

    ok, no = Eng(False), Eng(True)
    serving.ServingLoop._configure(ok, ("fused", 16))
    serving.ServingLoop._configure(no, ("fused", 16))
    serving.ServingLoop._configure(Eng(False), None)
    assert ok.form == ("fused", 16) and no.form is None


class AsyncEngine(ScriptedEngine):
    """Steps run in the background of the virtual clock: a slice issued at
    t finishes at t + cost (handles overlap fully), query() polls it."""

    def __init__(self, prob, clock, cost_per_cell_step=1e-9):
        super().__init__(prob, clock, cost_per_cell_step)
        self.ready_at = 0.0

    def step(self, k):
        self.n += k
        self.ready_at = max(self.ready_at, self.clock.t) + self.cost * k

    def query(self):
        return self.clock.t >= self.ready_at


def test_overlapping_handles_finish_independently_and_arrivals_start_on_time():
    """With slices that overlap on the device, a small request completes
    while a large one is still running, and a request arriving while every
    resident handle is busy starts at its arrival, not at the next slice
    end."""
    clock = Clock()
    loop = serving.ServingLoop(engine_factory=lambda p, prec, dev: AsyncEngine(p, clock), clock=clock,
                               sleep=clock.sleep, max_slots=4, slice_steps=50, hbm_budget=1 << 40,
                               stencil=None)
    big = serving.request_stream(1, seed=3, mean_gap=1e-6, cells=(20**3, 20**3), steps=(400, 400), ports=(2, 2),
                                 n_freq=5, port_kind="lumped")[0]
    small = serving.request_stream(1, seed=4, mean_gap=1e-6, cells=(8**3, 8**3), steps=(100, 100), ports=(2, 2),
                                   n_freq=5, port_kind="lumped")[0]
    small.rid = 1
    small.arrival = 0.5 * (big.steps * 2 * 20**3 * 1e-9) / 8  # during the big request's first slices
    stats = loop.run([big, small])
    res = {r.rid: r for r in stats.results}
    assert set(res) == {big.rid, 1}
    assert res[1].admitted - small.arrival < 5e-5          # started on arrival (a slice lasts 8e-4 s)
    assert res[1].finished < res[big.rid].finished          # did not wait for the big one
    for r in res.values():
        assert r.V.shape[0] == 2 and r.V.shape[1] == (400 if r.rid == big.rid else 100)
        assert np.isfinite(r.S).all()


@pytest.mark.timeout(30)
def test_a_request_waiting_for_memory_does_not_spin_the_loop():
    """An arrived request that the memory budget holds back waits for a
    slice to end.  A loop that polled without sleeping here would never
    advance the virtual clock the slices finish on, and the test would run
    into its timeout."""
    clock = Clock()
    reqs = serving.request_stream(3, seed=5, mean_gap=1e-6, cells=(16**3, 16**3), steps=(300, 300), ports=(2, 2),
                                  n_freq=5, port_kind="lumped")
    one = serving._footprint_of(reqs[0].build(None), 300, "single")
    loop = serving.ServingLoop(engine_factory=lambda p, prec, dev: AsyncEngine(p, clock), clock=clock,
                               sleep=clock.sleep, max_slots=4, slice_steps=50, hbm_budget=int(1.5 * one),
                               stencil=None)
    stats = loop.run(reqs)
    assert stats.n == 3 and stats.peak_bytes <= int(1.5 * one)
    assert stats.mean_active <= 1.0 + 1e-9  # the budget admits one request at a time


def test_modal_requests_carry_waveguide_ports_with_one_to_three_modes():
    """The default stream: both end faces are waveguide ports (1-3 TE modes
    each), the ports beyond two are lumped; every channel is driven by its
    own field set and the request's channel count is the problem's."""
    reqs = _stream(6, port_kind="modal")
    seen = set()
    for r in reqs:
        p = r.build(None)
        assert len(p.modal) == 2 and len(p.channels) == r.n_ports
        n_modal = sum(m.n_modes for m in p.modal)
        assert all(1 <= m.n_modes <= 3 for m in p.modal) and len(p.lumped) == r.n_ports - n_modal
        seen.update(m.n_modes for m in p.modal)
        c = 0
        for mp in p.modal:
            for m in range(mp.n_modes):
                assert mp.excitation[c][0] == m and np.max(np.abs(mp.excitation[c][1])) > 0
                assert all(e is None for q, e in enumerate(mp.excitation) if q != c and q < p.batch
                           and not (e is not None and e[0] != m))
                c += 1
        serving.ServingLoop._problem(r, None)  # the request takes the problem's band
        assert r.freqs[0] >= 7e9 and r.freqs[-1] == p.f_band[1]
        for kind, info in p.channels:
            if kind == "modal":
                assert info.omega_c / (2 * np.pi) < r.freqs[0]  # every mode propagates over the band
    assert len(seen) >= 2


def test_modal_requests_agree_between_the_batched_and_single_excitation_forms():
    clock = Clock()
    reqs = _stream(4, port_kind="modal")
    batched = _loop(clock, hbm_budget=1 << 40, max_slots=4, slice_steps=50).run(reqs)
    clock2 = Clock()
    plain = _loop(clock2, hbm_budget=1 << 40, slice_steps=50).run(_stream(4, port_kind="modal"), plain=True)
    assert plain.n == batched.n == 4
    for a, b in zip(batched.results, plain.results):
        assert a.S.shape == b.S.shape and a.S.shape[1] == a.S.shape[2]
        np.testing.assert_allclose(a.V, b.V, rtol=0, atol=0)
        np.testing.assert_allclose(a.S, b.S, rtol=1e-12, atol=0)


def test_a_modal_request_refuses_fewer_field_sets_than_channels():
    import numpy as np

    with pytest.raises(ValueError, match="driven channels"):
        workloads.waveguide_section_modal(np.random.default_rng(2), cells=12**3, n_modes=(2, 2), steps=50,
                                          batch=2, lowest=dense_lowest_eigs, device_tables=False)
