"""QG snapshot output (scripts/qg_1p5_layer.py:514-638): the sampled state's
fields computed on the device and written as a Zarr v3 store.

The reference gathers each snapshot to the host (``record_snapshot``), keeps
every snapshot in host lists and writes an ``xarray.Dataset`` with
``to_zarr`` at the end.  Here ``QGSnapshotRecorder.record`` computes the
seven planes (q, psi, eta, u and v at T points, speed, relative vorticity at
T points) with one fused kernel after the library's velocity and vorticity
kernels, copies them on a side stream into a pinned host slot, and a writer
thread stores each plane as one chunk of a Zarr v3 array as soon as its copy
has landed: output overlaps the following steps and no run-length list of
snapshots is held in memory.

Format: a Zarr v3 group (``zarr.json``) with one array per variable (shape
[time, y, x], chunks [1, y, x], little-endian ``bytes`` codec, no
compression -- the image has no compression codecs), ``dimension_names`` and
the reference's variable attributes; coordinates ``time``, ``x``, ``y`` as
1-D arrays, the static ``wind_curl`` field and the ``pv_enstrophy`` series
(0.5 mean(q^2), computed from the downloaded plane as the reference does).
``read_zarr_v3`` reads such a store back (tests, users without zarr).
"""

from __future__ import annotations

import json
import pathlib
import queue
import threading

import numpy as np
import torch

from finitevolx_b200._lib import D, I, P, check, fn, sfx, stream_ptr

VARIABLES = (
    ("q", "potential_vorticity_anomaly", "s-1"),
    ("psi", "streamfunction", "m2 s-1"),
    ("eta", "free_surface_anomaly", "m"),
    ("u", "zonal_velocity_at_t_points", "m s-1"),
    ("v", "meridional_velocity_at_t_points", "m s-1"),
    ("speed", "speed_at_t_points", "m s-1"),
    ("relative_vorticity", "relative_vorticity_at_t_points", "s-1"),
)


def _dtype_name(dt: np.dtype) -> str:
    return {np.dtype("float32"): "float32", np.dtype("float64"): "float64"}[np.dtype(dt)]


def _array_meta(shape, chunks, dtype, dims, attrs) -> dict:
    return {
        "zarr_format": 3,
        "node_type": "array",
        "shape": list(shape),
        "data_type": _dtype_name(dtype),
        "chunk_grid": {"name": "regular", "configuration": {"chunk_shape": list(chunks)}},
        "chunk_key_encoding": {"name": "default", "configuration": {"separator": "/"}},
        "fill_value": "NaN",
        "codecs": [{"name": "bytes", "configuration": {"endian": "little"}}],
        "attributes": attrs,
        "dimension_names": list(dims),
    }


def _write_json(path: pathlib.Path, obj) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(obj, indent=1))


def _write_chunk(root: pathlib.Path, name: str, index, data: np.ndarray) -> None:
    p = root / name / "c" / "/".join(str(i) for i in index)
    p.parent.mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(data).astype(data.dtype.newbyteorder("<"), copy=False).tofile(p)


def write_array(root, name, data: np.ndarray, dims, attrs=None) -> None:
    """A whole array as one chunk (coordinates, static fields)."""
    root = pathlib.Path(root)
    data = np.asarray(data)
    _write_json(root / name / "zarr.json", _array_meta(data.shape, data.shape, data.dtype, dims, attrs or {}))
    _write_chunk(root, name, (0,) * data.ndim, data)


def read_zarr_v3(path) -> dict:
    """{name: (array, dimension_names, attributes)} of an uncompressed Zarr v3
    group written by this module, plus "__attrs__": the group attributes."""
    root = pathlib.Path(path)
    out = {"__attrs__": json.loads((root / "zarr.json").read_text())["attributes"]}
    for child in sorted(p for p in root.iterdir() if (p / "zarr.json").exists()):
        meta = json.loads((child / "zarr.json").read_text())
        shape, chunks = meta["shape"], meta["chunk_grid"]["configuration"]["chunk_shape"]
        dt = np.dtype(meta["data_type"]).newbyteorder("<")
        arr = np.full(shape, np.nan, dtype=dt)
        grid = [range((s + c - 1) // c) for s, c in zip(shape, chunks)]
        for idx in np.ndindex(*[len(g) for g in grid]):
            f = child / "c" / "/".join(str(i) for i in idx)
            if f.exists():
                block = np.fromfile(f, dtype=dt).reshape(chunks)
                sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, shape))
                arr[sl] = block[tuple(slice(0, x.stop - x.start) for x in sl)]
        out[child.name] = (arr, meta["dimension_names"], meta["attributes"])
    return out


class QGSnapshotRecorder:
    """Records snapshots of a QGModel run into a Zarr v3 store at ``path``.

    ``record(q, step_index)`` enqueues the snapshot of state ``q`` (full
    [Ny, Nx] array with its ghost ring) on the current stream and returns at
    once; ``close()`` waits for the writes and writes the metadata.
    ``eta_scale`` = f0 / g (eta = eta_scale psi); ``wind_curl`` optional
    static [Ny-2, Nx-2] field; ``attrs`` the dataset attributes.
    """

    def __init__(self, model, path, dt: float, eta_scale: float, x=None, y=None, wind_curl=None,
                 attrs=None, slots: int = 2):
        from finitevolx_b200.solvers.spectral import DSTHelmholtzPlan
        from finitevolx_b200.swm import Vorticity2D
        g = model.grid
        self.model, self.dt, self.eta_scale = model, float(dt), float(eta_scale)
        self.root = pathlib.Path(path)
        self.root.mkdir(parents=True, exist_ok=True)
        self.ny, self.nx = g.Ny - 2, g.Nx - 2
        self.np_dtype = np.float32 if model.dtype == torch.float32 else np.float64
        self._vort = Vorticity2D(g)
        # its own plan: the model's DST workspace may hold the next step's
        # pre-split operand
        self._plan = DSTHelmholtzPlan(self.ny, self.nx, g.dx, g.dy, (model.lam,),
                                      fp64=model.dtype == torch.float64 or not model.plan.split_ok)
        self._dev = [torch.empty((7, self.ny, self.nx), dtype=model.dtype, device="cuda") for _ in range(slots)]
        self._psi = torch.zeros((g.Ny, g.Nx), dtype=model.dtype, device="cuda")
        self._host = [torch.empty((7, self.ny, self.nx), dtype=model.dtype, pin_memory=True) for _ in range(slots)]
        self._free = [threading.Event() for _ in range(slots)]
        for e in self._free:
            e.set()
        self._ready = [torch.cuda.Event() for _ in range(slots)]
        self._packed = torch.cuda.Event()
        self._side = torch.cuda.Stream()
        self._q: queue.Queue = queue.Queue()
        self._err: list = []
        self.times: list = []
        self.pv_enstrophy: dict = {}
        self._slot = 0
        self.x = np.asarray(x if x is not None else (np.arange(self.nx) + 0.5) * g.dx)
        self.y = np.asarray(y if y is not None else (np.arange(self.ny) + 0.5) * g.dy)
        self.wind_curl = None if wind_curl is None else np.asarray(wind_curl)
        self.attrs = dict(attrs or {})
        self._thread = threading.Thread(target=self._writer, daemon=True)
        self._thread.start()

    # -- device side -----------------------------------------------------------
    def record(self, q, step_index: int) -> None:
        from finitevolx_b200.qg import geostrophic_velocity
        if self._err:
            raise self._err[0]
        m = self.model
        s = self._slot
        self._slot = (s + 1) % len(self._host)
        # the writer is done with slot s, so its copy (and the device planes
        # it read) finished: slot s can be refilled
        self._free[s].wait()
        self._free[s].clear()
        self._psi[1:-1, 1:-1] = self._plan.solve(q[1:-1, 1:-1].contiguous())
        u, v = geostrophic_velocity(self._psi, m.grid)
        z = self._vort.relative_vorticity(u, v)
        check(fn(f"fvx_qg_snapshot_pack_{sfx(q)}")(P(q), P(self._psi), P(u), P(v), P(z), I(m.grid.Ny),
                                                    I(m.grid.Nx), D(self.eta_scale), P(self._dev[s]), stream_ptr()),
              "snapshot pack")
        self._packed.record()
        self._side.wait_event(self._packed)
        with torch.cuda.stream(self._side):
            self._host[s].copy_(self._dev[s], non_blocking=True)
            self._ready[s].record(self._side)
        t = len(self.times)
        self.times.append(step_index * self.dt)
        self._q.put((t, s))

    # -- host side -------------------------------------------------------------
    def _writer(self) -> None:
        while True:
            item = self._q.get()
            if item is None:
                return
            t, s = item
            try:
                self._ready[s].synchronize()
                planes = self._host[s].numpy()
                for k, (name, _, _) in enumerate(VARIABLES):
                    _write_chunk(self.root, name, (t, 0, 0), planes[k])
                self.pv_enstrophy[t] = float(0.5 * np.mean(planes[0].astype(np.float64) ** 2))
            except Exception as e:  # reported by the next record / close
                self._err.append(e)
            finally:
                self._free[s].set()

    def close(self) -> None:
        self._q.put(None)
        self._thread.join()
        if self._err:
            raise self._err[0]
        T = len(self.times)
        _write_json(self.root / "zarr.json", {"zarr_format": 3, "node_type": "group", "attributes": self.attrs})
        for name, long_name, units in VARIABLES:
            _write_json(self.root / name / "zarr.json",
                        _array_meta((T, self.ny, self.nx), (1, self.ny, self.nx), self.np_dtype, ("time", "y", "x"),
                                    {"long_name": long_name, "units": units}))
        write_array(self.root, "time", np.asarray(self.times, np.float64), ("time",),
                    {"long_name": "time", "units": "s"})
        write_array(self.root, "x", self.x, ("x",))
        write_array(self.root, "y", self.y, ("y",))
        write_array(self.root, "pv_enstrophy", np.asarray([self.pv_enstrophy[t] for t in range(T)]), ("time",),
                    {"long_name": "domain_mean_pv_enstrophy", "units": "s-2"})
        if self.wind_curl is not None:
            write_array(self.root, "wind_curl", self.wind_curl, ("y", "x"),
                        {"long_name": "double_gyre_pv_forcing", "units": "s-2"})

    def __del__(self):
        t = getattr(self, "_thread", None)
        if t is not None and t.is_alive():
            self._q.put(None)
