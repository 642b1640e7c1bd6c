"""Checkpoint / resume of solver and ensemble states: raw SoA planes + JSON metadata.

A state file pair ``<prefix>.bin`` / ``<prefix>.json``:

* ``.bin``: the conserved planes ``U[10][nx+4][ny+4]`` (ghost cells included,
  slot order rho, mx, my, mz, Bx, By, Bz, E, psi, rhoC of config.py), C order,
  little-endian float32 or float64 -- the layout of ``MHDSolver.U`` and of the
  reference's ``self.U`` (solver.py:87), readable with
  ``numpy.fromfile(path, dtype).reshape(shape)`` from any language;
* ``.json``: format tag, dtype, shape, SHA-256 of the ``.bin``, the ``Config``
  fields, and the loop state needed to continue the run exactly: ``t``,
  ``step``, ``dt``, ``glm_ch`` (solver.py:221), the cumulative boundary energy
  (solver.py:316-317) and the diagnostic histories (solver.py:335-444).

Resuming a saved solver continues with the same dt, ch and states as the
uninterrupted run (the device loop recomputes dt and ch from the state, as the
reference's loop head does, solver.py:476-479).  An ensemble checkpoint is one
state pair per instance plus an index file.  The same pair format stores the
corrector's training snapshots (``write_state`` / ``read_state``).

The reference writes no checkpoints (its snapshots, solver.py:446-463, are
primitive interior fields kept in memory).
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os
import sys
from typing import Dict, List, Tuple

import numpy as np

from .config import NVAR, Config

FORMAT = "aeromhd-b200-state/1"
_DTYPES = {"float32": np.dtype("<f4"), "float64": np.dtype("<f8")}
_DIAG_LISTS = ("diag_times", "diag_mixing_width_integral", "diag_mixing_width_thresh", "diag_mixedness",
               "diag_enstrophy", "diag_enstrophy_local", "diag_perturbation_amp", "diag_mode_amps",
               "diag_stag_pressure", "diag_divB_max", "diag_divB_L2", "diag_energy_total", "diag_mass_total",
               "diag_boundary_flux_cumulative")


class CheckpointError(ValueError):
    pass


def _sha256(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def _jsonable(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, (np.floating, np.integer)):
        return v.item()
    if isinstance(v, (list, tuple)):
        return [_jsonable(x) for x in v]
    if isinstance(v, dict):
        return {k: _jsonable(x) for k, x in v.items()}
    return v


def write_state(prefix: str, U: np.ndarray, meta: Dict | None = None) -> Dict:
    """Write U (a [10][nx+4][ny+4] float32/float64 array) and its metadata; returns the metadata."""
    U = np.asarray(U)
    if U.ndim != 3 or U.shape[0] != NVAR:
        raise CheckpointError(f"state must be [{NVAR}][nx+4][ny+4], got shape {U.shape}")
    name = {np.dtype("float32"): "float32", np.dtype("float64"): "float64"}.get(U.dtype.newbyteorder("="))
    if name is None:
        raise CheckpointError(f"state dtype must be float32 or float64, got {U.dtype}")
    d = os.path.dirname(os.path.abspath(prefix))
    os.makedirs(d, exist_ok=True)
    binp, jsp = prefix + ".bin", prefix + ".json"
    tmp = binp + ".tmp"
    np.ascontiguousarray(U, dtype=_DTYPES[name]).tofile(tmp)
    os.replace(tmp, binp)
    m = {"format": FORMAT, "dtype": name, "shape": list(U.shape), "byte_order": "little",
         "sha256": _sha256(binp)}
    m.update(_jsonable(meta or {}))
    tmp = jsp + ".tmp"
    with open(tmp, "w") as f:
        json.dump(m, f, indent=1, allow_nan=True)
    os.replace(tmp, jsp)
    return m


def read_state(prefix: str, verify: bool = True) -> Tuple[np.ndarray, Dict]:
    """Read a state pair written by write_state; checks format, size and (verify) the checksum."""
    binp, jsp = prefix + ".bin", prefix + ".json"
    try:
        with open(jsp) as f:
            m = json.load(f)
    except (OSError, ValueError) as e:
        raise CheckpointError(f"cannot read {jsp}: {e}") from e
    if m.get("format") != FORMAT:
        raise CheckpointError(f"{jsp}: unknown format {m.get('format')!r} (expected {FORMAT!r})")
    if m.get("dtype") not in _DTYPES or m.get("byte_order") != "little":
        raise CheckpointError(f"{jsp}: unsupported dtype/byte order {m.get('dtype')!r}/{m.get('byte_order')!r}")
    shape = tuple(int(x) for x in m["shape"])
    if len(shape) != 3 or shape[0] != NVAR:
        raise CheckpointError(f"{jsp}: bad shape {shape}")
    dt = _DTYPES[m["dtype"]]
    want = int(np.prod(shape)) * dt.itemsize
    have = os.path.getsize(binp) if os.path.exists(binp) else -1
    if have != want:
        raise CheckpointError(f"{binp}: {have} bytes, expected {want}")
    if verify and _sha256(binp) != m.get("sha256"):
        raise CheckpointError(f"{binp}: checksum mismatch")
    U = np.fromfile(binp, dtype=dt).reshape(shape)
    return U, m


def config_from_meta(m: Dict) -> Config:
    fields = {f.name for f in dataclasses.fields(Config)}
    c = m.get("config")
    if not isinstance(c, dict):
        raise CheckpointError("metadata holds no config")
    unknown = set(c) - fields
    if unknown:
        raise CheckpointError(f"config has unknown fields {sorted(unknown)}")
    return Config(**c)


# ------------------------------------------------------------------ solver
def solver_meta(solver) -> Dict:
    m = {"config": dataclasses.asdict(solver.cfg), "t": float(solver.t), "step": int(solver.step),
         "dt": float(solver.dt), "glm_ch": float(solver.cfg.glm_ch),
         "glm_ch_frozen": float(getattr(solver, "_glm_ch_frozen", 0.0)),
         "cumulative_boundary_energy": float(solver._cumulative_boundary_energy),
         "rh_results": getattr(solver, "_rh_results", None),
         "rho_light": float(getattr(solver, "_rho_light", 1.0)), "rho_heavy": float(getattr(solver, "_rho_heavy", 1.0))}
    m["diagnostics"] = {k: _jsonable(list(getattr(solver, k, []))) for k in _DIAG_LISTS}
    return m


def save_checkpoint(solver, prefix: str) -> Dict:
    """Write the solver's state (device -> host once) and loop state."""
    from .solver import to_numpy
    return write_state(prefix, to_numpy(solver.U), solver_meta(solver))


def restore(solver, U: np.ndarray, m: Dict) -> None:
    """Put a read state into an existing solver of the same grid."""
    expect = (NVAR, solver.nx_tot, solver.ny_tot)
    if tuple(U.shape) != expect:
        raise CheckpointError(f"checkpoint grid {tuple(U.shape)} does not match the solver's {expect}")
    solver.U = U
    solver.t = float(m["t"])
    solver.step = int(m["step"])
    solver.dt = float(m.get("dt", 0.0))
    solver.cfg.glm_ch = float(m.get("glm_ch", solver.cfg.glm_ch))
    solver._glm_ch_frozen = float(m.get("glm_ch_frozen", 0.0))
    solver._cumulative_boundary_energy = float(m.get("cumulative_boundary_energy", 0.0))
    solver._rh_results = m.get("rh_results")
    solver._rho_light = float(m.get("rho_light", 1.0))
    solver._rho_heavy = float(m.get("rho_heavy", 1.0))
    for k, v in (m.get("diagnostics") or {}).items():
        if k in _DIAG_LISTS:
            setattr(solver, k, [np.asarray(x) for x in v] if k == "diag_mode_amps" else list(v))


def load_checkpoint(prefix: str, verify: bool = True):
    """A new MHDSolver continuing the saved run (needs a CUDA device)."""
    from .solver import MHDSolver
    U, m = read_state(prefix, verify)
    s = MHDSolver(config_from_meta(m))
    restore(s, U, m)
    return s


# ---------------------------------------------------------------- ensemble
def save_ensemble(ens, directory: str) -> Dict:
    """One state pair per instance (inst_00000.bin/.json ...) plus index.json with
    each instance's loop state from its control block."""
    os.makedirs(directory, exist_ok=True)
    ctl = ens.controls()
    entries: List[Dict] = []
    for k, c in enumerate(ens.configs):
        name = f"inst_{k:05d}"
        meta = {"config": dataclasses.asdict(c), "t": float(ctl[k].t), "step": int(ctl[k].step),
                "dt": float(ctl[k].last_dt), "glm_ch": float(ctl[k].ch),
                "cumulative_boundary_energy": float(ctl[k].e_bnd), "instance": k}
        from .solver import to_numpy
        write_state(os.path.join(directory, name), to_numpy(ens.state(k)), meta)
        entries.append({"name": name, "t": meta["t"], "step": meta["step"]})
    index = {"format": FORMAT + "+ensemble", "instances": entries, "tile_x": int(ens.tile_x)}
    with open(os.path.join(directory, "index.json"), "w") as f:
        json.dump(index, f, indent=1)
    return index


def read_ensemble(directory: str, verify: bool = True) -> List[Tuple[np.ndarray, Dict]]:
    try:
        with open(os.path.join(directory, "index.json")) as f:
            index = json.load(f)
    except (OSError, ValueError) as e:
        raise CheckpointError(f"cannot read {directory}/index.json: {e}") from e
    if index.get("format") != FORMAT + "+ensemble":
        raise CheckpointError(f"{directory}: unknown ensemble format {index.get('format')!r}")
    return [read_state(os.path.join(directory, e["name"]), verify) for e in index["instances"]]


def load_ensemble(directory: str, t_end: float | None = None, verify: bool = True, **kw):
    """A new Ensemble holding the saved states, each instance set to continue from
    its saved t, step and boundary energy toward t_end (default: the first
    instance's configured t_end).  Returns (ensemble, per-instance metadata)."""
    from .ensemble import Ensemble
    items = read_ensemble(directory, verify)
    cfgs = [config_from_meta(m) for _, m in items]
    ens = Ensemble(cfgs, **kw)
    for k, (U, m) in enumerate(items):
        ens.set_state(k, U)
    metas = [m for _, m in items]
    ens.resume([m["t"] for m in metas], [m["step"] for m in metas],
               [m.get("cumulative_boundary_energy", 0.0) for m in metas],
               cfgs[0].t_end if t_end is None else float(t_end))
    return ens, metas


def main(argv=None) -> int:
    """python -m aeromhd_cuda_b200.checkpoint <prefix>: print a checkpoint's metadata after verifying it."""
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m aeromhd_cuda_b200.checkpoint <prefix>", file=sys.stderr)
        return 2
    U, m = read_state(argv[0])
    m = dict(m)
    m.pop("diagnostics", None)
    print(json.dumps(m, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
