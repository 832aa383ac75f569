"""Node-field snapshots of a solve: the reference's Zarr v3 ``fv-fields`` groups, written
behind the device.

A snapshot is the group the reference's ``write_node_fields`` writes
(``zvcfd/io/node_fields.py:1-64``): arrays in the mesh's node order — ``velocity`` ``(N, 3)``,
``pressure`` ``(N,)``, optionally ``wall_nodes`` ``(W,)`` with ``wss`` ``(W, 3)`` and any other
array a caller adds — chunked along the node axis, floats cast to ``dtype`` (``float32`` by
default), and the group attribute ``zvcfd`` = ``{"kind": "fv-fields", "step", "time_s",
"nodes", "mesh", "fields"}``. The reference writes it with the ``zarr`` package and the zstd
codec; neither is in this build's environment, so this module writes the Zarr v3 storage format
itself, from the published specification (Zarr storage specification 3.0):

- ``<group>/zarr.json``: ``{"zarr_format": 3, "node_type": "group", "attributes": {...}}``;
- ``<group>/<name>/zarr.json``: ``node_type`` ``"array"``, ``shape``, ``data_type``, a
  ``regular`` chunk grid, the ``default`` chunk-key encoding with ``/`` separators, the fill
  value, and the codec chain ``bytes`` (little-endian) then ``gzip`` (a core Zarr v3 codec,
  from the standard library's zlib) when ``compress``;
- ``<group>/<name>/c/<i>/<j>...``: one file per chunk, C order.

Any Zarr v3 reader, the reference's ``read_node_fields`` included, reads these groups.
:func:`read_node_fields` reads the ``bytes``, ``gzip`` and (when the ``zstandard`` module is
importable) ``zstd`` codecs, so the reference's own snapshots open too where zstd is present.

:class:`SnapshotWriter` is the transient solve's callback that takes a snapshot every
``every`` steps without stalling the host: the velocity and pressure are copied into device
buffers on the solve's stream (HBM to HBM, microseconds, ordered between the step that made them
and the next one), then from there into pinned host buffers on a side stream, and a worker
thread waits for that copy, casts and writes the group while the next steps run. A small pool
of buffer sets bounds the memory; when every set is still being written, the next snapshot
waits for the oldest.
"""

from __future__ import annotations

import gzip
import json
import queue
import threading
from pathlib import Path

import numpy as np

KIND = "fv-fields"
ZARR_TYPES = {np.dtype(t): t for t in ("bool", "int8", "int16", "int32", "int64", "uint8",
                                       "uint16", "uint32", "uint64", "float32", "float64")}


def _json(path: Path, doc: dict) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(doc, indent=1))


def _fill(dt: np.dtype):
    return False if dt.kind == "b" else 0 if dt.kind in "iu" else 0.0


def write_array(path, a: np.ndarray, *, chunk: int, compress: bool = True, level: int = 1):
    """One Zarr v3 array: chunks of ``chunk`` rows (whole trailing axes) under ``path``."""
    path = Path(path)
    a = np.ascontiguousarray(a)
    if a.dtype not in ZARR_TYPES:
        raise TypeError(f"dtype {a.dtype} has no Zarr v3 name here")
    rows = min(chunk, max(len(a), 1))
    cshape = [rows] + list(a.shape[1:])
    codecs = [{"name": "bytes", "configuration": {"endian": "little"}}]
    if compress:
        codecs.append({"name": "gzip", "configuration": {"level": level}})
    _json(path / "zarr.json", {
        "zarr_format": 3, "node_type": "array", "shape": list(a.shape),
        "data_type": ZARR_TYPES[a.dtype],
        "chunk_grid": {"name": "regular", "configuration": {"chunk_shape": cshape}},
        "chunk_key_encoding": {"name": "default", "configuration": {"separator": "/"}},
        "fill_value": _fill(a.dtype), "codecs": codecs, "attributes": {}})
    le = a.astype(a.dtype.newbyteorder("<"), copy=False)
    trailing = "/".join("0" for _ in a.shape[1:])
    for i, start in enumerate(range(0, len(a), rows)):
        block = np.zeros(cshape, le.dtype)                 # the last chunk is padded whole
        part = le[start:start + rows]
        block[:len(part)] = part
        raw = block.tobytes(order="C")
        if compress:
            raw = gzip.compress(raw, compresslevel=level, mtime=0)
        key = f"c/{i}" + (f"/{trailing}" if trailing else "")
        f = path / key
        f.parent.mkdir(parents=True, exist_ok=True)
        f.write_bytes(raw)


def _decode(raw: bytes, codecs: list) -> bytes:
    for c in reversed(codecs):
        name = c["name"]
        if name == "bytes":
            continue
        if name == "gzip":
            raw = gzip.decompress(raw)
        elif name == "zstd":
            try:
                import zstandard
            except ImportError as e:
                raise RuntimeError("a zstd-compressed snapshot needs the zstandard module") from e
            raw = zstandard.ZstdDecompressor().decompress(raw)
        else:
            raise ValueError(f"codec {name!r} is not read here")
    return raw


def read_array(path) -> np.ndarray:
    """A Zarr v3 array written by :func:`write_array` (or any regular-grid array chunked along
    its first axis only, with the codecs :func:`_decode` reads)."""
    path = Path(path)
    meta = json.loads((path / "zarr.json").read_text())
    if meta.get("zarr_format") != 3 or meta.get("node_type") != "array":
        raise ValueError(f"{path}: not a Zarr v3 array")
    shape = tuple(meta["shape"])
    cshape = tuple(meta["chunk_grid"]["configuration"]["chunk_shape"])
    if cshape[1:] != shape[1:]:
        raise ValueError(f"{path}: chunks must hold whole rows")
    endian = next((c.get("configuration", {}).get("endian", "little")
                   for c in meta["codecs"] if c["name"] == "bytes"), "little")
    dt = np.dtype(meta["data_type"]).newbyteorder("<" if endian == "little" else ">")
    sep = meta["chunk_key_encoding"].get("configuration", {}).get("separator", "/")
    out = np.full(shape, meta["fill_value"], dt.newbyteorder("="))
    rows = cshape[0] if cshape else 1
    trailing = sep.join("0" for _ in shape[1:])
    for i, start in enumerate(range(0, shape[0] if shape else 0, rows)):
        key = f"c{sep}{i}" + (f"{sep}{trailing}" if trailing else "")
        f = path / key
        if not f.exists():
            continue                                      # a missing chunk is all fill value
        block = np.frombuffer(_decode(f.read_bytes(), meta["codecs"]), dt).reshape(cshape)
        n = min(rows, shape[0] - start)
        out[start:start + n] = block[:n]
    return out


def write_node_fields(path, fields: dict, *, step: int, time_s: float | None,
                      mesh: str | None = None, chunk: int = 1 << 18,
                      dtype: str | None = "float32", compress: bool = True) -> Path:
    """Write one snapshot group (the reference's ``write_node_fields``,
    ``zvcfd/io/node_fields.py:26-51``); float arrays are cast to ``dtype`` (``None`` keeps
    them)."""
    path = Path(path)
    n = None
    for name, a in fields.items():
        a = np.asarray(a)
        if dtype is not None and a.dtype.kind == "f":
            a = a.astype(dtype)
        write_array(path / name, a, chunk=chunk, compress=compress)
        if name in ("velocity", "pressure"):
            n = len(a)
    _json(path / "zarr.json", {
        "zarr_format": 3, "node_type": "group",
        "attributes": {"zvcfd": {"kind": KIND, "step": int(step),
                                 "time_s": None if time_s is None else float(time_s),
                                 "nodes": n, "mesh": mesh, "fields": sorted(fields)}}})
    return path


def read_node_fields(path) -> tuple:
    """``(fields, attributes)`` of a snapshot group (``zvcfd/io/node_fields.py:54-61``)."""
    path = Path(path)
    doc = json.loads((path / "zarr.json").read_text())
    meta = dict(doc.get("attributes", {}).get("zvcfd", {}))
    if meta.get("kind") != KIND:
        raise ValueError(f"{path}: not a {KIND} group")
    return {k: read_array(path / k) for k in meta["fields"]}, meta


class SnapshotWriter:
    """A transient solve's callback writing a snapshot group every ``every`` steps behind the
    device (see the module docstring).

    Args:
        directory: snapshots go to ``directory/step-<step:09d>.zarr``.
        every: steps between snapshots.
        wss: add ``wall_nodes`` and ``wss`` (the solver's ``wall_shear()``).
        dtype, compress, chunk, mesh: as :func:`write_node_fields`.
        buffers: pinned buffer sets in flight (the depth of the write-behind).

    Use ``solver.solve_transient(..., callback=writer)`` and ``writer.close()`` (or a ``with``
    block) to wait for the last writes; an error of the worker is raised there, or at the next
    snapshot. ``paths`` lists the groups written, in order.
    """

    def __init__(self, directory, *, every: int = 1, wss: bool = False,
                 dtype: str | None = "float32", compress: bool = True, chunk: int = 1 << 18,
                 mesh: str | None = None, buffers: int = 2):
        self.directory = Path(directory)
        self.every, self.wss = max(int(every), 1), bool(wss)
        self.options = {"dtype": dtype, "compress": compress, "chunk": chunk, "mesh": mesh}
        self.step = 0
        self.paths = []
        self._free = queue.Queue()
        for _ in range(max(int(buffers), 1)):
            self._free.put(None)                         # a slot; its buffers come on first use
        self._work = queue.Queue()
        self._error = None
        self._stream = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _stage(self, slot, tensors: dict):
        """This slot's copy of the tensors: on the device, first a copy into the slot's device
        buffers on the current stream (ordered after the step that made the values and before
        the next step that overwrites them), then, on a side stream, the copy of those buffers
        into the slot's pinned host buffers; returns ``(slot, event of the host copy)``."""
        import torch

        if slot is None:
            slot = {"dev": {}, "host": {}}
        if not any(t.is_cuda for t in tensors.values()):
            for k, t in tensors.items():
                slot["host"][k] = t.detach().cpu().numpy().copy()
            return slot, None
        if self._stream is None:
            self._stream = torch.cuda.Stream()
        for k, t in tensors.items():
            d = slot["dev"].get(k)
            if d is None or d.shape != t.shape or d.dtype != t.dtype:
                d = torch.empty_like(t)
                slot["dev"][k] = d
            d.copy_(t)
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream())
        done = torch.cuda.Event()
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ready)
            for k, d in slot["dev"].items():
                h = slot["host"].get(k)
                if h is None or h.shape != d.shape or h.dtype != d.dtype:
                    h = torch.empty(d.shape, dtype=d.dtype, pin_memory=True)
                    slot["host"][k] = h
                h.copy_(d, non_blocking=True)
            done.record(self._stream)
        return slot, done

    def __call__(self, solver, dt=None) -> None:
        self.step += 1
        if self.step % self.every:
            return
        if self._error is not None:
            raise RuntimeError("a snapshot write failed") from self._error
        slot = self._free.get()                          # waits while every slot is in flight
        U, P = getattr(solver, "U", None), getattr(solver, "P", None)
        if U is not None and P is not None and hasattr(U, "is_cuda"):
            slot, event = self._stage(slot, {"velocity": U, "pressure": P})
        else:                                            # a solver that gathers on the host
            f = solver.fields()
            slot, event = {"dev": {}, "host": {"velocity": f["U"], "pressure": f["P"]}}, None
        extra = {}
        if self.wss:
            nodes, tau = solver.wall_shear()
            extra = {"wall_nodes": np.asarray(nodes), "wss": np.asarray(tau)}
        path = self.directory / f"step-{self.step:09d}.zarr"
        self.paths.append(path)
        self._work.put((slot, event, extra, path, self.step, float(solver.t)))

    def _run(self):
        while True:
            item = self._work.get()
            if item is None:
                return
            slot, event, extra, path, step, t = item
            try:
                if event is not None:
                    event.synchronize()
                fields = {k: (v.numpy() if hasattr(v, "numpy") else v)
                          for k, v in slot["host"].items()}
                write_node_fields(path, fields | extra, step=step, time_s=t, **self.options)
            except Exception as e:                       # reported at the next call or close
                self._error = e
            finally:
                self._free.put(slot)

    def close(self) -> None:
        """Wait for every snapshot in flight; raise the first write error, if any."""
        if self._thread.is_alive():
            self._work.put(None)
            self._thread.join()
        if self._error is not None:
            raise RuntimeError("a snapshot write failed") from self._error


__all__ = ["KIND", "SnapshotWriter", "read_array", "read_node_fields", "write_array",
           "write_node_fields"]
