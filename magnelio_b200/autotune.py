"""Autotuner for the stencil kernels: kernel form (tile shape), march depth
(i planes per CTA) and batch width.

The reference has fixed kernels; this engine has several stencil forms
(``stream``, ``vec``, ``fused``, ``bulk``, ``simple``), each with variants
and a chunk length along the march axis, and the best choice depends on the
grid, the batch width, the precision and the GPU.  :func:`tune_problem`
builds a scratch handle with a problem's coefficients and CPML faces (no
ports, sources or monitors: the stencil is the part that depends on the
choice), times every candidate with the engine's own CUDA-event stencil
timer, and returns the fastest; results are cached per (grid, batch,
precision, coefficient storage, CPML faces, GPU) in a JSON file
(``$FITB_TUNE_CACHE``, default ``~/.cache/magnelio_b200/autotune.json``).
:func:`apply` configures a live engine with a result.  Tuning never touches
a live engine's fields: the timer advances the fields it times.
"""

from __future__ import annotations

import json
import os
from dataclasses import asdict, dataclass, field
from pathlib import Path

from magnelio_b200._lib import FitbError

# (kind, variant, i planes per CTA; 0 = the form's own plan)
DEFAULT_CANDIDATES = (
    ("stream", 0, 0),
    ("stream", 1, 0),
    ("stream", 2, 0),
    ("stream", 3, 0),
    ("stream", 0, 8),
    ("stream", 0, 16),
    ("stream", 0, 32),
    ("stream", 0, 64),
    ("stream", 0, 128),
    ("vec", 3, 0),
    ("vec", 2, 0),
    ("fused", 7, 0),
    ("fused", 7, 16),
    ("fused", 8, 0),
    ("fused", 9, 0),
    ("fused", 0, 0),
    ("fused", 16, 0),
    ("fused", 17, 0),
    ("fused", 18, 0),
    ("fused", 19, 0),
    ("fused", 20, 0),
    ("fused", 21, 0),
    ("fused", 22, 0),
    ("fused", 23, 0),
    ("fused", 24, 0),
    ("fused", 25, 0),
    ("bulk", 0, 0),
)
CANDIDATE_SET = 6  # bump when the candidates change: cached results of another set are not reused


@dataclass
class TuneResult:
    kind: str
    variant: int
    ichunk: int
    batch: int
    ms: float  # one E + H stencil pass, all field sets
    gcells: float  # cell-updates per second / 1e9 at that time
    table: list = field(default_factory=list)  # [(kind, variant, ichunk, batch, ms)]

    def config(self) -> tuple:
        return self.kind, self.variant, self.ichunk


def _cache_path() -> Path:
    p = os.environ.get("FITB_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "magnelio_b200" / "autotune.json"


def _device_name(device: int) -> str:
    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.get_device_name(device)
    except Exception:  # pragma: no cover - torch is optional here
        pass
    return "unknown"


def cache_key(nx, ny, nz, batch, precision, coef, n_cpml, device_name) -> str:
    return f"{nx}x{ny}x{nz}|B{batch}|{precision}|{coef}|cpml{n_cpml}|{device_name}|c{CANDIDATE_SET}"


def _load_cache(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store_cache(path: Path, key: str, res: TuneResult) -> None:
    data = _load_cache(path)
    data[key] = asdict(res)
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1))
        tmp.replace(path)
    except OSError:
        pass  # a read-only home: tuning still works, it is just not remembered


def tune_engine(eng, candidates=DEFAULT_CANDIDATES, iters: int = 10, warmup: int = 2):
    """Time each candidate (kind, variant, ichunk) on ``eng`` and leave the
    fastest configured.  Candidates the handle refuses (a form that does not
    take this batch width, a variant that does not fit) are skipped.  The
    engine's fields advance: pass a scratch engine.  Returns (best, table)
    with per-candidate milliseconds for one E + H pass."""
    table = []
    for kind, variant, ichunk in candidates:
        try:
            eng.configure_stencil(kind, variant, ichunk)
            eng.time_stencil(warmup)
            t_e, t_h = eng.time_stencil(iters)
        except FitbError:
            continue
        table.append((kind, int(variant), int(ichunk), float(t_e + t_h)))
    if not table:
        raise RuntimeError("no stencil candidate ran on this handle")
    best = min(table, key=lambda r: r[3])
    eng.configure_stencil(best[0], best[1], best[2])
    return best, table


def _scratch_engine(prob, batch: int, precision: str, device: int, coef: str):
    from magnelio_b200.engine import FitEngine

    eng = FitEngine(prob.nx, prob.ny, prob.nz, prob.dt, batch=batch, precision=precision, device=device)
    try:
        if coef != "native":
            eng.set_coefficient_storage(coef)
        prob.put_coefficients(eng)
        for f in prob.cpml:
            eng.add_cpml(f.face, f.b, f.c, f.ck, f.air)
    except Exception:
        eng.close()
        raise
    return eng


def tune_problem(prob, precision: str = "single", batch_widths=(1,), device: int = 0, coef: str = "native",
                 candidates=DEFAULT_CANDIDATES, iters: int = 10, use_cache: bool = True) -> TuneResult:
    """Fastest stencil configuration for ``prob``'s grid at each batch width
    in ``batch_widths``; the result is the one with the most cell-updates
    per second.  Cached unless ``use_cache`` is false."""
    if getattr(prob, "dispersion", None):
        # the ADE update needs an in-place stencil form
        candidates = [c for c in candidates if c[0] != "fused"]
    path = _cache_path()
    dev = _device_name(device)
    cache = _load_cache(path) if use_cache else {}
    cells = prob.nx * prob.ny * prob.nz
    results = []
    for B in batch_widths:
        key = cache_key(prob.nx, prob.ny, prob.nz, B, precision, coef, len(prob.cpml), dev)
        if getattr(prob, "dispersion", None):
            key += "|ade"
        if key in cache:
            results.append(TuneResult(**cache[key]))
            continue
        eng = _scratch_engine(prob, B, precision, device, coef)
        try:
            best, table = tune_engine(eng, candidates, iters=iters)
        finally:
            eng.close()
        res = TuneResult(kind=best[0], variant=best[1], ichunk=best[2], batch=B, ms=best[3],
                         gcells=cells * B / (best[3] * 1e-3) / 1e9,
                         table=[(k, v, c, B, ms) for k, v, c, ms in table])
        if use_cache:
            _store_cache(path, key, res)
        results.append(res)
    return max(results, key=lambda r: r.gcells)


def apply(eng, res: TuneResult) -> None:
    """Configure a live engine with a tuning result (between steps)."""
    eng.configure_stencil(res.kind, res.variant, res.ichunk)


def best_batch(results) -> int:
    """Batch width with the highest throughput among tuning results."""
    return int(max(results, key=lambda r: r.gcells).batch)


__all__ = ["TuneResult", "DEFAULT_CANDIDATES", "tune_engine", "tune_problem", "apply", "cache_key", "best_batch"]
