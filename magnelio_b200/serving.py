"""Continuous-batching serving loop for S-parameter solves on one GPU.

A request is one mesh with its ports; every driven channel of the request
(a mode of a waveguide port, or a lumped port) is one field set of a single
engine handle, so the excitations of one mesh
advance together in every launch and read the coefficients once per cell
(the batch dimension).  The loop:

* admits requests in arrival order as soon as a slot and enough device
  memory are free (footprint estimated from the grid before the handle is
  built, checked against the handle's own count after);
* keeps every admitted mesh, its fields and its histories resident on the
  device until its last step;
* advances all admitted handles in slices of steps, each handle on its own
  CUDA stream, so the work of different requests overlaps on the GPU; a
  handle gets its next slice as soon as its last one has finished (polled,
  non-blocking), and new arrivals are admitted whenever a slice ends
  (requests join and leave the running set continuously);
* on completion forms the S-matrix (on the device by default, from the
  recorded port voltages and currents and each channel's power-wave map)
  and releases the device memory.

Latency is measured from a request's arrival to its S-matrix; throughput is
solves per second of wall time.  ``plain=True`` serves the same stream one
excitation at a time (one field set per handle, one handle at a time), the
single-excitation form the batched loop is compared with.
"""

from __future__ import annotations

import copy
import dataclasses
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float              # seconds after the stream starts
    build: object               # callable(batch: int | None) -> FitProblem
    n_ports: int                # driven channels (set from the built problem)
    steps: int
    freqs: np.ndarray
    z0: float = 50.0
    # the built problem of a request served one excitation at a time,
    # shared by its single-excitation handles
    cache: dict = field(default_factory=dict, repr=False)


@dataclass
class Result:
    rid: int
    S: np.ndarray               # (n_freq, P, P)
    V: np.ndarray               # (P, steps, P) port voltages per excitation
    I: np.ndarray
    arrival: float
    admitted: float
    finished: float
    footprint: int              # estimated device bytes
    device_bytes: int           # what the handle held

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServingStats:
    n: int
    wall: float
    solves_per_s: float
    p50: float
    p99: float
    mean_active: float
    peak_bytes: int
    results: list = field(default_factory=list)

    def summary(self) -> dict:
        return {"requests": self.n, "wall_s": self.wall, "solves_per_s": self.solves_per_s,
                "p50_s": self.p50, "p99_s": self.p99, "mean_active": self.mean_active,
                "peak_device_bytes": self.peak_bytes}


def estimate_footprint(nx, ny, nz, batch, steps, n_channels, cpml_layers=(), precision="single",
                       n_dispersive_states=0, fused=False) -> int:
    """Device bytes a handle for this problem holds, from the engine's
    padded layout: fields (B sets), coefficients and mass diagonals, the
    staging buffer, CPML psi slabs, the V/I recorder sized for ``steps``;
    ``fused``: the fused step's second set of fields and psi."""
    esz = 4 if precision == "single" else 8
    sets = 2 if fused else 1
    njp, nkp = ny + 2, -(-(nz + 2) // 8) * 8
    si = njp * nkp
    vol = (nx + 4) * si + 8 * nkp
    n_e = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    total = sets * 2 * batch * 3 * vol * esz   # E, H
    total += 6 * 3 * vol * esz                 # alpha/beta E/H, M_eps, M_mu
    total += n_e * esz                         # staging
    for axis, n in cpml_layers:
        dims = [nx + 1, ny + 1, nz + 1]
        dims[axis] = n
        slab = dims[0] * dims[1] * (-(-dims[2] // 16) * 16)  # rows padded to 16 entries
        total += sets * batch * 4 * slab * esz + 4 * slab + 3 * n * esz
    cap = max(int(steps), 1024)
    total += 2 * batch * cap * max(n_channels, 1) * 8
    total += n_dispersive_states * batch * 8 * esz
    return int(total + (4 << 20))              # small tables and counters


def _footprint_of(prob, steps, precision, fused=False):
    layers = [("xyz".index(f.face[0]), len(f.b)) for f in prob.cpml]
    n_modal = sum(m.n_modes for m in prob.modal)
    nch = len(prob.lumped) + n_modal
    fp = estimate_footprint(prob.nx, prob.ny, prob.nz, prob.batch, steps, nch, layers, precision, fused=fused)
    # DTBC histories (scattered and incident) and the kernel tables
    cap = max(int(steps), 1024)
    return fp + n_modal * (2 * prob.batch * cap + 4 * cap) * 8


def serving_stencil(batch: int):
    """Stencil form of a served handle with ``batch`` field sets, each form
    on the kernels measured fastest for it in the served mix: one field set
    on the slab step (the TMA tile march with the CPML inside it: 0.636
    solves/s on the full stream against 0.48-0.51 on the tile step),
    several on the batched two-pass kernels (with eight requests resident
    the TMA forms' shared memory per CTA limits how many CTAs of different
    requests share an SM: 10.64 vs 9.98 solves/s on the quarter-scale
    stream)."""
    return ("fused", 16) if batch == 1 else None


class ServingLoop:
    """See the module docstring.  ``engine_factory(problem, precision,
    device)`` builds the engine of an admitted problem (the default builds a
    :class:`~magnelio_b200.engine.FitEngine` through
    ``FitProblem.build_engine``)."""

    def __init__(self, device: int = 0, precision: str = "single", hbm_budget: int | None = None,
                 max_slots: int = 8, slice_steps: int = 512, engine_factory=None, tune=None,
                 clock=time.perf_counter, sleep=time.sleep, stencil=serving_stencil, records: bool = True,
                 coef: str | None = None):
        self.device = device
        # coefficient storage of every handle ("f16": 16-bit with per-component
        # scales, in the forms that take it; None: the field dtype)
        self.coef = coef
        # records=False: S-matrices come from the device post-step
        # (FitEngine.s_parameters) and the V/I histories stay on the device
        # (Result.V / Result.I are None)
        self.records = records
        self.precision = precision
        self.stencil = stencil        # callable(batch) -> (kind, variant) or None (the engine default)
        self.max_slots = max_slots
        self.slice_steps = slice_steps
        self.engine_factory = engine_factory or (lambda p, prec, dev: p.build_engine(prec, device=dev))
        self.tune = tune              # callable(problem, engine) or None
        self.clock = clock
        self.sleep = sleep
        self.hbm_budget = hbm_budget if hbm_budget is not None else self._default_budget()

    def _default_budget(self) -> int:
        try:
            import torch

            free, _total = torch.cuda.mem_get_info(self.device)
            return int(0.85 * free)
        except Exception:
            return 16 << 30

    def run(self, requests, plain: bool = False) -> ServingStats:
        reqs = sorted(requests, key=lambda r: r.arrival)
        if plain:
            # one excitation per handle, one handle at a time
            units = [(r, p) for r in reqs for p in range(r.n_ports)]
            slots = 1
        else:
            units = [(r, None) for r in reqs]
            slots = self.max_slots
        pending = deque([list(u) + [None] for u in units])  # [request, port, built problem]
        active = []                   # dicts: req, port, eng, prob, done, admitted, fp
        partial = {}                  # plain mode: rid -> per-port (V, I)
        results = []
        used = 0
        peak = 0
        active_samples = []
        t0 = self.clock()
        while pending or active:
            now = self.clock() - t0
            while pending and len(active) < slots and pending[0][0].arrival <= now:
                req, port, prob = pending[0]
                if port is not None and port >= req.n_ports:
                    pending.popleft()             # the request kept fewer channels
                    req.cache.clear()
                    continue
                if prob is None:
                    prob = pending[0][2] = self._problem(req, port)
                form = self.stencil(prob.batch) if self.stencil is not None else None
                fp = _footprint_of(prob, req.steps, self.precision, form is not None and form[0] == "fused")
                if active and used + fp > self.hbm_budget:
                    break                         # wait for memory (arrival order kept)
                pending.popleft()
                if port is not None and port == req.n_ports - 1:
                    req.cache.clear()
                eng = self.engine_factory(prob, self.precision, self.device)
                self._configure(eng, form)
                self._storage(eng, self.coef)
                if self.tune is not None:
                    self.tune(prob, eng)
                eng.reserve_steps(req.steps)
                used += fp
                peak = max(peak, used)
                active.append({"req": req, "port": port, "eng": eng, "prob": prob, "done": 0,
                               "admitted": self.clock() - t0, "fp": fp})
            if not active:
                nxt = pending[0][0].arrival
                self.sleep(max(0.0, nxt - (self.clock() - t0)))
                continue
            active_samples.append(len(active))
            # a slice on every idle handle (asynchronous, own streams), then
            # wait until at least one handle has finished its slice: a small
            # request does not wait for the largest one's slice
            for a in active:
                if not a.get("busy"):
                    k = min(self.slice_steps, a["req"].steps - a["done"])
                    a["eng"].step(k)
                    a["k"] = k
                    a["busy"] = True
            # with a slot free, a future arrival also ends the wait (its
            # handle starts then, not when some slice ends); one that has
            # arrived but waits for memory waits for a slice to end
            due = None
            if pending and len(active) < slots and pending[0][0].arrival > self.clock() - t0:
                due = pending[0][0].arrival
            finished = {id(a) for a in self._wait_any(active, None if due is None else t0 + due)}
            still = []
            for a in active:
                if id(a) not in finished:
                    still.append(a)
                    continue
                a["busy"] = False
                a["done"] += a["k"]
                if a["done"] < a["req"].steps:
                    still.append(a)
                    continue
                req = a["req"]
                eng = a["eng"]
                nset = a["prob"].batch
                on_device = not self.records and hasattr(eng, "s_parameters")
                if on_device:
                    VI = None
                    cols = self._device_columns(eng, req, a["port"], a["prob"])
                else:
                    VI = [eng.read_vi(b) for b in range(nset)]
                dev_bytes = eng.device_bytes
                eng.close()
                used -= a["fp"]
                fin = self.clock() - t0
                if on_device:
                    got = partial.setdefault(req.rid, {})
                    got.update(cols)
                    if len(got) == req.n_ports:
                        S = np.stack([got[p] for p in range(req.n_ports)], axis=2)
                        results.append(Result(rid=req.rid, S=S, V=None, I=None, arrival=req.arrival,
                                              admitted=a["admitted"], finished=fin, footprint=a["fp"],
                                              device_bytes=dev_bytes))
                        del partial[req.rid]
                elif a["port"] is None:
                    V = np.stack([v for v, _ in VI[:req.n_ports]])
                    I = np.stack([i for _, i in VI[:req.n_ports]])
                    results.append(self._result(req, V, I, a, fin, dev_bytes))
                else:
                    got = partial.setdefault(req.rid, {})
                    got[a["port"]] = VI[0]
                    if len(got) == req.n_ports:
                        V = np.stack([got[p][0] for p in range(req.n_ports)])
                        I = np.stack([got[p][1] for p in range(req.n_ports)])
                        results.append(self._result(req, V, I, a, fin, dev_bytes))
                        del partial[req.rid]
            active = still
        wall = self.clock() - t0
        lat = np.array([r.latency for r in results]) if results else np.zeros(1)
        return ServingStats(n=len(results), wall=wall, solves_per_s=len(results) / max(wall, 1e-9),
                            p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                            mean_active=float(np.mean(active_samples)) if active_samples else 0.0,
                            peak_bytes=int(peak), results=sorted(results, key=lambda r: r.rid))

    def _wait_any(self, active, until=None):
        """The handles whose slice has finished, waiting for at least one or
        until the clock reaches ``until`` (then possibly none); engines
        without a non-blocking query are synchronised in turn."""
        while True:
            done = []
            for a in active:
                if not a.get("busy"):
                    continue
                query = getattr(a["eng"], "query", None)
                if query is None:
                    a["eng"].sync()
                    done.append(a)
                elif query():
                    done.append(a)
            if done or (until is not None and self.clock() >= until):
                return done
            self.sleep(2e-5)

    @staticmethod
    def _storage(eng, coef):
        """16-bit coefficient storage on a new handle whose stencil form takes
        it; others keep the field dtype."""
        setter = getattr(eng, "set_coefficient_storage", None)
        if coef is None or setter is None:
            return
        from magnelio_b200._lib import FitbError

        try:
            setter(coef)
        except FitbError:
            pass

    @staticmethod
    def _configure(eng, form):
        """The stencil form on a new handle; a handle that does not take it
        (dispersive materials need the in-place forms) keeps the engine's
        default kernels."""
        configure = getattr(eng, "configure_stencil", None)
        if form is None or configure is None:
            return
        from magnelio_b200._lib import FitbError

        try:
            configure(*form)
        except FitbError:
            pass

    @staticmethod
    def _problem(req, port):
        """The request's problem; for the single-excitation form the copy
        whose one field set drives channel ``port`` (built once per
        request)."""
        if port is None:
            prob = req.build(None)
        else:
            proto = req.cache.get("problem")
            if proto is None:
                proto = req.cache["problem"] = req.build(None)
            prob = copy.copy(proto)
            prob.batch = 1
            prob.lumped = [dataclasses.replace(lp, v_src=[lp.v_src[port]]) for lp in proto.lumped]
            prob.modal = [dataclasses.replace(mp, excitation=[mp.excitation[port]] if mp.excitation else [])
                          for mp in proto.modal]
            prob.e0 = proto.e0[:1]
            prob.h0 = proto.h0[:1]
        if prob.channels:
            req.n_ports = len(prob.channels)
        if prob.f_band is not None:
            req.freqs = np.linspace(prob.f_band[0], prob.f_band[1], len(req.freqs))
        return prob

    @staticmethod
    def channel_maps(req, prob, n_channels):
        """Power-wave maps ``(n_channels, 4, F)`` and the co-temporal flags of
        a request's channels: a modal channel's from its port
        (``waveguide_ports.power_wave_maps``: discrete impedance and half-cell
        de-stagger, I shifted by the Yee half step), a lumped port's
        ``a = (V + Z0 I) / (2 sqrt Z0)``, ``b = (V - Z0 I) / (2 sqrt Z0)``
        with I taken with V."""
        from magnelio_b200 import waveguide_ports as wp

        F = len(req.freqs)
        maps = np.zeros((n_channels, 4, F), complex)
        icot = np.ones(n_channels, np.int32)
        chans = prob.channels or [("lumped", req.z0)] * n_channels
        for c in range(n_channels):
            kind, info = chans[c] if c < len(chans) else ("lumped", req.z0)
            if kind == "modal":
                maps[c] = wp.power_wave_maps(info, req.freqs, prob.dt)
                icot[c] = 0
            else:
                rz = np.sqrt(info)
                maps[c, 0], maps[c, 1] = 1.0 / (2 * rz), info / (2 * rz)
                maps[c, 2], maps[c, 3] = 1.0 / (2 * rz), -info / (2 * rz)
        return maps, icot

    @classmethod
    def _device_columns(cls, eng, req, port, prob):
        """S-matrix columns of a finished handle from the device post-step:
        {driven channel: S[:, :, channel]}, with each channel's power-wave
        map (:meth:`channel_maps`; for lumped ports the time origin and dt
        factor of :func:`magnelio_b200.workloads.s_matrix` are common to a
        and b and cancel in b / a)."""
        P = req.n_ports
        maps, icot = cls.channel_maps(req, prob, eng.n_channels)
        driven = list(range(P)) if port is None else [port]
        S = eng.s_parameters(req.freqs, maps, icot, driven, a_threshold=0.0)
        return {p: S[:, :P, b] for b, p in enumerate(driven)}

    def _result(self, req, V, I, a, fin, dev_bytes):
        from magnelio_b200.workloads import s_matrix

        prob = a["prob"]
        dt = prob.dt
        if prob.channels:
            from magnelio_b200 import sparams

            maps, icot = self.channel_maps(req, prob, V.shape[2])
            S = sparams.s_matrix(list(V), list(I), dt, req.freqs, list(maps), [bool(c) for c in icot],
                                 list(range(req.n_ports)), a_threshold=0.0)
        else:
            S = s_matrix(V, I, dt, req.freqs, req.z0, req.n_ports)
        return Result(rid=req.rid, S=S, V=V, I=I, arrival=req.arrival, admitted=a["admitted"], finished=fin,
                      footprint=a["fp"], device_bytes=dev_bytes)


def request_stream(n: int, seed: int = 7, mean_gap: float = 0.020, cells=(32**3, 192**3), steps=(6000, 12000),
                   ports=(2, 4), n_freq: int = 101, device_setup: bool = True, port_kind: str = "modal",
                   modes=(1, 3), lowest=None, device_tables: bool = True):
    """The serving workload: ``n`` requests with Poisson arrivals (mean gap
    ``mean_gap`` s), each a rectangular or single-ridge waveguide section
    with dimensions ``U[0.7, 1.3]`` x (22.86, 10.16, 40) mm, 0-4 dielectric
    inserts (``eps_r ~ U[2, 10]``), a log-uniform cell count in ``cells``,
    a port count in ``ports`` and a step count in ``steps``.

    ``port_kind="modal"`` (the default): the two end faces are waveguide
    ports with a mode count in ``modes`` each (TE modes below the empty
    guide's TM11 cut-off; ports built by
    :func:`magnelio_b200.workloads.waveguide_section_modal`, mode solve and
    DTBC tables on the GPU unless ``lowest`` / ``device_tables`` say
    otherwise), the ports beyond two are lumped; the S-matrix band is the
    built problem's ``f_band`` (every kept mode propagates over it; the
    request holds an estimate from the empty guide's cut-offs until then).  ``port_kind="lumped"``: every port is a
    50 Ohm lumped port, CPML terminates both ends, band 7-13 GHz.

    With ``device_setup`` (the default) a request's material matrices and
    coefficients are built on the device when its handle is created: the
    host prepares the grid and the cell materials only."""
    from magnelio_b200.workloads import te_cutoffs, te_mode_count, waveguide_section, waveguide_section_modal

    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += float(rng.exponential(mean_gap))
        dims = np.array([22.86e-3, 10.16e-3, 40e-3]) * rng.uniform(0.7, 1.3, 3)
        c = int(np.exp(rng.uniform(np.log(cells[0]), np.log(cells[1]))))
        P = int(rng.integers(ports[0], ports[1] + 1))
        st = int(rng.integers(steps[0], steps[1] + 1))
        ins = int(rng.integers(0, 5))
        ridged = bool(rng.integers(0, 2))
        sub = int(rng.integers(0, 2**31 - 1))
        if port_kind == "lumped":
            def build(batch, dims=dims, c=c, P=P, st=st, ins=ins, ridged=ridged, sub=sub):
                return waveguide_section(np.random.default_rng(sub), a=dims[0], b=dims[1], length=dims[2], cells=c,
                                         n_inserts=ins, ridged=ridged, n_ports=P, steps=st, batch=batch,
                                         device_setup=device_setup)

            out.append(Request(rid=rid, arrival=t, build=build, n_ports=P, steps=st,
                               freqs=np.linspace(7.0e9, 13.0e9, n_freq)))
            continue
        nm = [te_mode_count(dims[0], dims[1], int(rng.integers(modes[0], modes[1] + 1))) for _ in range(2)]
        fc = te_cutoffs(dims[0], dims[1], max(nm))[0]
        f_hi = max(13.0e9, 1.25 * float(fc[-1]))
        f_lo = max(7.0e9, 1.05 * float(fc[-1]))

        def build(batch, dims=dims, c=c, P=P, st=st, ins=ins, ridged=ridged, sub=sub, nm=tuple(nm)):
            return waveguide_section_modal(np.random.default_rng(sub), a=dims[0], b=dims[1], length=dims[2],
                                           cells=c, n_inserts=ins, ridged=ridged, n_modes=nm, n_lumped=P - 2,
                                           steps=st, batch=batch, device_setup=device_setup,
                                           lowest=lowest, device_tables=device_tables)

        out.append(Request(rid=rid, arrival=t, build=build, n_ports=sum(nm) + P - 2, steps=st,
                           freqs=np.linspace(f_lo, f_hi, n_freq)))
    return out
