"""Node-field snapshots (``zvcfd_b200.snapshots``): the reference's ``fv-fields`` groups in the
Zarr v3 storage format, and the write-behind callback.

- write then read: float arrays cast to ``float32`` by default (``None`` keeps them), integer
  arrays untouched, several chunks with a ragged last one, the group attributes of the
  reference's ``write_node_fields`` (``zvcfd/io/node_fields.py:47-50``);
- the stored layout is the specification's: group and array ``zarr.json`` documents, chunk
  keys ``c/<i>/<j>`` holding C-order little-endian bytes, raw or gzip;
- a group of another kind is refused; an empty array round-trips;
- the callback on a stand-in solver (host tensors): one group per ``every`` steps with that
  step's fields, and a write error surfaces at ``close``.
"""

import gzip
import json

import numpy as np
import pytest
import torch

from zvcfd_b200.snapshots import (SnapshotWriter, read_array, read_node_fields, write_array,
                                  write_node_fields)


def _fields(n=50, w=9):
    rng = np.random.default_rng(0)
    return {"velocity": rng.normal(size=(n, 3)), "pressure": rng.normal(size=n),
            "wall_nodes": np.sort(rng.choice(n, w, replace=False)).astype(np.int64),
            "wss": rng.normal(size=(w, 3))}


def test_round_trip_casts_floats_only(tmp_path):
    f = _fields()
    p = write_node_fields(tmp_path / "s.zarr", f, step=7, time_s=0.25, mesh="../m.zarrvectors",
                          chunk=16)
    got, meta = read_node_fields(p)
    assert meta == {"kind": "fv-fields", "step": 7, "time_s": 0.25, "nodes": 50,
                    "mesh": "../m.zarrvectors", "fields": sorted(f)}
    for k in ("velocity", "pressure", "wss"):
        assert got[k].dtype == np.float32
        np.testing.assert_array_equal(got[k], f[k].astype(np.float32))
    assert got["wall_nodes"].dtype == np.int64
    np.testing.assert_array_equal(got["wall_nodes"], f["wall_nodes"])
    p2 = write_node_fields(tmp_path / "d.zarr", f, step=0, time_s=None, dtype=None,
                           compress=False, chunk=7)
    got2, meta2 = read_node_fields(p2)
    assert meta2["time_s"] is None
    for k in f:
        np.testing.assert_array_equal(got2[k], f[k])
        assert got2[k].dtype == f[k].dtype


def test_layout_is_zarr_v3(tmp_path):
    a = np.arange(30, dtype=np.float64).reshape(10, 3)
    write_array(tmp_path / "raw", a, chunk=4, compress=False)
    meta = json.loads((tmp_path / "raw" / "zarr.json").read_text())
    assert meta["zarr_format"] == 3 and meta["node_type"] == "array"
    assert meta["shape"] == [10, 3] and meta["data_type"] == "float64"
    assert meta["chunk_grid"] == {"name": "regular", "configuration": {"chunk_shape": [4, 3]}}
    assert meta["chunk_key_encoding"] == {"name": "default", "configuration": {"separator": "/"}}
    assert meta["codecs"] == [{"name": "bytes", "configuration": {"endian": "little"}}]
    assert meta["fill_value"] == 0.0
    keys = sorted(p.relative_to(tmp_path / "raw").as_posix()
                  for p in (tmp_path / "raw" / "c").rglob("*") if p.is_file())
    assert keys == ["c/0/0", "c/1/0", "c/2/0"]
    last = np.frombuffer((tmp_path / "raw" / "c" / "2" / "0").read_bytes(), "<f8").reshape(4, 3)
    np.testing.assert_array_equal(last[:2], a[8:])           # the ragged chunk, padded
    assert (last[2:] == 0).all()
    write_array(tmp_path / "gz", a.astype(np.float32), chunk=4, compress=True)
    meta = json.loads((tmp_path / "gz" / "zarr.json").read_text())
    assert [c["name"] for c in meta["codecs"]] == ["bytes", "gzip"]
    first = gzip.decompress((tmp_path / "gz" / "c" / "0" / "0").read_bytes())
    np.testing.assert_array_equal(np.frombuffer(first, "<f4").reshape(4, 3), a[:4])
    group = json.loads((write_node_fields(tmp_path / "g", {"pressure": a[:, 0]}, step=1,
                                          time_s=0.0) / "zarr.json").read_text())
    assert group["zarr_format"] == 3 and group["node_type"] == "group"


def test_other_kinds_and_empty_arrays(tmp_path):
    (tmp_path / "x").mkdir()
    (tmp_path / "x" / "zarr.json").write_text(json.dumps(
        {"zarr_format": 3, "node_type": "group", "attributes": {"zvcfd": {"kind": "lbm"}}}))
    with pytest.raises(ValueError, match="fv-fields"):
        read_node_fields(tmp_path / "x")
    write_array(tmp_path / "e", np.zeros((0, 3)), chunk=8)
    assert read_array(tmp_path / "e").shape == (0, 3)
    with pytest.raises(TypeError):
        write_array(tmp_path / "c", np.zeros(3, complex), chunk=8)


class _Stand:
    """A solver's surface as the callback sees it: device-or-host ``U``, ``P`` and ``t``."""

    def __init__(self, n):
        self.U = torch.zeros((n, 3), dtype=torch.float64)
        self.P = torch.zeros(n, dtype=torch.float64)
        self.t = 0.0

    def step(self, k):
        self.t += 0.1
        self.U += k
        self.P -= k

    def wall_shear(self):
        return np.array([0, 2]), self.U[[0, 2]].numpy()


def test_callback_writes_every_nth_step(tmp_path):
    s = _Stand(20)
    seen = {}
    with SnapshotWriter(tmp_path, every=2, wss=True, dtype=None, buffers=1) as w:
        for k in range(1, 6):
            s.step(k)
            w(s, 0.1)
            seen[w.step] = (s.U.clone().numpy(), s.P.clone().numpy(), s.t)
    assert [p.name for p in w.paths] == ["step-000000002.zarr", "step-000000004.zarr"]
    for p in w.paths:
        f, meta = read_node_fields(p)
        U, P, t = seen[meta["step"]]
        np.testing.assert_array_equal(f["velocity"], U)
        np.testing.assert_array_equal(f["pressure"], P)
        np.testing.assert_array_equal(f["wall_nodes"], [0, 2])
        assert meta["time_s"] == pytest.approx(t) and meta["nodes"] == 20


def test_a_write_error_surfaces_at_close(tmp_path):
    blocker = tmp_path / "file"
    blocker.write_text("not a directory")
    w = SnapshotWriter(blocker / "below")
    w(_Stand(4))
    with pytest.raises(RuntimeError, match="snapshot write failed"):
        w.close()
