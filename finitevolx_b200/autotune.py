"""Autotuner for the fused kernels' launch choices.

Each tuner times the candidates on the device (CUDA events, warm, the median
of several launches) through the library's own entry points and applies the
fastest:

* ``tune_qg_stage``: the fused QG stage kernel's tile shape (64x16, 32x16,
  128x8, 64x32, 128x16 cells; the halo follows the scheme) for one scheme
  and dtype.
* ``tune_qg_split``: whether the stage kernel writes the next DST operand
  split itself (fused) or a separate split pass does (unfused).
* ``tune_dst_kernel``: the even/odd DST product on single CTAs with 64- or
  32-element K blocks (3 or 6 ring stages) or on CTA pairs (cta_group::2,
  each pair sharing its B blocks).
* ``tune_ensemble``: the persistent work-queue grid (CTAs per SM).

Results are cached in a JSON file keyed by device name and workload
(``FVX_AUTOTUNE_CACHE``, default ``~/.cache/finitevolx_b200/autotune.json``)
so later runs reuse them without timing.
"""

from __future__ import annotations

import json
import os
import pathlib
import statistics

import torch

from finitevolx_b200._lib import I, SCHEMES, check, fn

_TILES = ("64x16", "32x16", "128x8", "64x32", "128x16", "16x16")


def _cache_path() -> pathlib.Path:
    p = os.environ.get("FVX_AUTOTUNE_CACHE")
    return pathlib.Path(p) if p else pathlib.Path.home() / ".cache" / "finitevolx_b200" / "autotune.json"


def _load() -> dict:
    try:
        return json.loads(_cache_path().read_text())
    except Exception:
        return {}


def _store(key: str, value) -> None:
    data = _load()
    data[key] = value
    try:
        path = _cache_path()
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(data, indent=1, sort_keys=True))
    except OSError:
        pass  # a read-only home only costs re-tuning


def _device_key() -> str:
    return torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")


def _time(fn_call, reps: int = 7, warm: int = 2, batch: int = 5) -> float:
    """Median over ``reps`` of the device time of ``batch`` back-to-back
    calls between two events, per call: the calls queue behind each other,
    so the host's launch latency does not enter the window."""
    for _ in range(warm):
        fn_call()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(batch):
            fn_call()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / batch)
    return statistics.median(ts)


def _time_graph(fn_call, reps: int = 7, warm: int = 2, batch: int = 10) -> float:
    """Like _time, but the ``batch`` calls are captured once in a CUDA graph
    and the graph is replayed between the events: for kernels of a few
    microseconds, whose back-to-back host calls would otherwise pace the
    window."""
    for _ in range(warm):
        fn_call()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(batch):
            fn_call()
    g.replay()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / batch)
    del g
    return statistics.median(ts)


def set_stage_tile(method: str, dtype: torch.dtype, cfg: int) -> None:
    check(fn("fvx_qg_tile_config")(I(SCHEMES[method]), I(1 if dtype == torch.float64 else 0), I(cfg)),
          "tile config")


def tune_qg_stage(model, q, dt: float, use_cache: bool = True) -> dict:
    """Pick the stage kernel's tile shape for ``model`` (a QGModel) on
    state ``q``; returns {"tile": name, "ms": {name: median ms per step}}.
    Candidates are timed as whole steps (graph-replayed): inside a step the
    stage reads inputs the DST products just wrote, which the stage timed
    alone does not reproduce (at 2048^2 the two orderings of 64x16 and
    64x32 disagree)."""
    g = model.grid
    key = f"{_device_key()}/qg_stage/{model.method}/{model.dtype}/{g.Ny}x{g.Nx}"
    if use_cache:
        hit = _load().get(key)
        if hit:
            set_stage_tile(model.method, model.dtype, _TILES.index(hit["tile"]))
            return hit
    n_cfg = fn("fvx_qg_tile_config")(I(0), I(0), I(-1))
    out = torch.empty_like(q)
    ms = {}
    for cfg in range(n_cfg):
        set_stage_tile(model.method, model.dtype, cfg)
        ms[_TILES[cfg]] = _time_graph(lambda: model.step(q, dt, out=out), batch=4)
    best = min(ms, key=ms.get)
    set_stage_tile(model.method, model.dtype, _TILES.index(best))
    res = {"tile": best, "ms": ms}
    _store(key, res)
    return res


def tune_qg_split(model, q, dt: float, use_cache: bool = True) -> dict:
    """Fused (the stage kernel writes the DST operand split) against unfused
    (a separate split pass before each DST) for whole steps; sets
    ``model.fuse_split`` and returns {"fused": bool, "ms": {...}}."""
    g = model.grid
    key = f"{_device_key()}/qg_split/{model.method}/{model.dtype}/{g.Ny}x{g.Nx}"
    if use_cache:
        hit = _load().get(key)
        if hit:
            model.fuse_split = bool(hit["fused"])
            return hit
    out = torch.empty_like(q)
    ms = {}
    model.step(q, dt, out=out)  # leaves split(out) in the workspace for the fused chain
    ms["fused"] = _time_graph(lambda: model.step(out, dt, out=out, presplit=True), batch=4)
    ms["unfused"] = _time_graph(lambda: model.step(q, dt, out=out, presplit=False), batch=4)
    fused = ms["fused"] <= ms["unfused"]
    model.fuse_split = fused
    res = {"fused": fused, "ms": ms}
    _store(key, res)
    return res


DST_KERNELS = ("single64", "pair", "single32")


def set_dst_kernel(kind) -> None:
    """``kind``: one of DST_KERNELS (or its index)."""
    k = DST_KERNELS.index(kind) if isinstance(kind, str) else int(kind)
    check(fn("fvx_dst_kernel_config")(I(k)), "dst kernel config")


def tune_dst_kernel(model, q, dt: float, use_cache: bool = True) -> dict:
    """The even/odd DST product forms timed over whole QG steps of ``model``
    (a QGModel); returns {"kernel": name, "ms": {name: median ms}}."""
    g = model.grid
    key = f"{_device_key()}/dst_kernel/{model.dtype}/{g.Ny}x{g.Nx}"
    if use_cache:
        hit = _load().get(key)
        if hit and hit.get("kernel") in DST_KERNELS:
            set_dst_kernel(hit["kernel"])
            return hit
    out = torch.empty_like(q)

    ms = {}
    for name in DST_KERNELS:
        set_dst_kernel(name)
        ms[name] = _time_graph(lambda: model.step(q, dt, out=out), batch=4)
    best = min(ms, key=ms.get)
    set_dst_kernel(best)
    res = {"kernel": best, "ms": ms}
    _store(key, res)
    return res


def tune_ensemble(ens, candidates=(0, 1, 2, 4), steps: int = 3, use_cache: bool = True) -> dict:
    """Persistent-grid occupancy for a QGEnsemble (0 = as many CTAs as fit)."""
    sig = ",".join(f"{n}:{nl}" for n, nl in ens.members)
    key = f"{_device_key()}/ensemble/{ens.method}/{hash(sig) & 0xffffffff:08x}"
    if use_cache:
        hit = _load().get(key)
        if hit:
            ens.set_blocks_per_sm(int(hit["blocks_per_sm"]))
            return hit
    ms = {}
    for c in candidates:
        ens.set_blocks_per_sm(c)
        ms[str(c)] = _time(lambda: ens.step(steps), reps=3, warm=1, batch=1)
    best = min(ms, key=ms.get)
    ens.set_blocks_per_sm(int(best))
    res = {"blocks_per_sm": int(best), "ms": ms}
    _store(key, res)
    return res
