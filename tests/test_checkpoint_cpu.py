"""Checkpoint file format (raw SoA planes + JSON metadata) on the CPU: round
trips in both precisions, and every kind of damaged or mismatched file is
refused with a clear error."""
import dataclasses
import json
import os

import numpy as np
import pytest

from aeromhd_cuda_b200 import checkpoint as ck
from aeromhd_cuda_b200.config import Config


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_state_round_trip_is_exact(tmp_path, dtype):
    rng = np.random.default_rng(3)
    U = rng.standard_normal((10, 14, 9)).astype(dtype)
    U[8, 0, 0] = np.nan          # non-finite values survive as they are
    U[1, 2, 3] = -np.inf
    cfg = Config(nx=10, ny=5, precision="fp32" if dtype == np.float32 else "fp64")
    meta = {"config": dataclasses.asdict(cfg), "t": 0.125, "step": 7, "arr": np.arange(3)}
    m = ck.write_state(str(tmp_path / "a"), U, meta)
    assert m["dtype"] == ("float32" if dtype == np.float32 else "float64")
    V, m2 = ck.read_state(str(tmp_path / "a"))
    assert V.dtype == dtype and V.shape == U.shape
    assert np.array_equal(V, U, equal_nan=True)
    assert m2["t"] == 0.125 and m2["step"] == 7 and m2["arr"] == [0, 1, 2]
    assert ck.config_from_meta(m2) == cfg
    # the .bin is plain little-endian C-order planes: readable without this module
    raw = np.fromfile(str(tmp_path / "a.bin"), dtype=np.dtype(dtype).newbyteorder("<")).reshape(U.shape)
    assert np.array_equal(raw, U, equal_nan=True)


def test_damaged_or_mismatched_files_are_refused(tmp_path):
    U = np.zeros((10, 6, 6))
    p = str(tmp_path / "s")
    ck.write_state(p, U, {"config": dataclasses.asdict(Config(nx=2, ny=2))})
    # flipped byte: checksum
    with open(p + ".bin", "r+b") as f:
        f.seek(17)
        f.write(b"\x01")
    with pytest.raises(ck.CheckpointError, match="checksum"):
        ck.read_state(p)
    ck.read_state(p, verify=False)           # the caller may skip the checksum
    # truncated payload
    with open(p + ".bin", "r+b") as f:
        f.truncate(100)
    with pytest.raises(ck.CheckpointError, match="bytes"):
        ck.read_state(p, verify=False)
    # wrong format tag, wrong dtype, missing file
    ck.write_state(p, U, {})
    m = json.load(open(p + ".json"))
    for key, val, msg in (("format", "other/9", "format"), ("dtype", "int8", "dtype")):
        bad = dict(m, **{key: val})
        json.dump(bad, open(p + ".json", "w"))
        with pytest.raises(ck.CheckpointError, match=msg):
            ck.read_state(p)
    os.remove(p + ".json")
    with pytest.raises(ck.CheckpointError, match="cannot read"):
        ck.read_state(p)
    # shapes and types the writer refuses
    with pytest.raises(ck.CheckpointError):
        ck.write_state(p, np.zeros((9, 4, 4)))
    with pytest.raises(ck.CheckpointError):
        ck.write_state(p, np.zeros((10, 4, 4), dtype=np.int32))
    with pytest.raises(ck.CheckpointError, match="unknown fields"):
        ck.config_from_meta({"config": {"nx": 4, "not_a_field": 1}})


def test_cli_prints_metadata(tmp_path, capsys):
    p = str(tmp_path / "c")
    ck.write_state(p, np.ones((10, 5, 5), dtype=np.float32), {"t": 1.5, "diagnostics": {"diag_times": [0.0]}})
    assert ck.main([p]) == 0
    out = json.loads(capsys.readouterr().out)
    assert out["t"] == 1.5 and "diagnostics" not in out
