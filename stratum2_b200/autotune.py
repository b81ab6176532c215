"""Autotuner front end: runs s2_autotune (a coordinate search over the wavefront renderer's wave
size, traversal triangle batch, triangle-step vote and lane-refill threshold, timed on the caller's
own scene, view and render parameters; whether to shade in material-sorted or queue order, to
sort continuation rays, and to trace each bounce's shadow rays in the next bounce's traversal
launch) and keeps the results in a JSON file keyed by GPU and workload, so later runs of the same
workload apply them without searching."""
from __future__ import annotations

import json
import os
from pathlib import Path

from . import _abi

FIELDS = ("wave_paths", "trav_tris_per_step", "trav_vote8", "refill_min", "shade_order", "trace_order", "shadow_merge")


def default_path() -> Path:
    return Path(os.environ.get("S2_TUNING_FILE", Path.home() / ".cache" / "stratum2_b200" / "tuning.json"))


def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:  # pragma: no cover - no torch / no device
        return "unknown-gpu"


def workload_key(device, view, params: _abi.S2RenderParams) -> str:
    w = view.image_max[0] - view.image_min[0]
    h = view.image_max[1] - view.image_min[1]
    tris = int(device.bvh_stats.triangle_count) if device.bvh_stats is not None else 0
    return (f"{gpu_name()}|tris={tris}|{w}x{h}|spp={params.spp}|len={params.min_path_length}-{params.max_path_length}"
            f"|flags={params.flags}")


def to_dict(t: _abi.S2Tuning) -> dict:
    return {f: int(getattr(t, f)) for f in FIELDS}


def from_dict(d: dict) -> _abi.S2Tuning:
    t = _abi.S2Tuning()
    for f in FIELDS:
        setattr(t, f, int(d.get(f, 0)))
    return t


def load(path: Path | None = None) -> dict:
    p = Path(path) if path else default_path()
    if not p.exists():
        return {}
    try:
        return json.loads(p.read_text())
    except (OSError, json.JSONDecodeError):
        return {}


def save(table: dict, path: Path | None = None):
    p = Path(path) if path else default_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(table, indent=1, sort_keys=True))
    tmp.replace(p)


def autotune(device, view, params: _abi.S2RenderParams, path: Path | None = None, force: bool = False) -> dict:
    """Applies the stored tuning of this workload, or searches for one (and stores it).  Returns
    {"tuning": {...}, "key": ..., "searched": bool, "trials": n}."""
    key = workload_key(device, view, params)
    table = load(path)
    if not force and key in table:
        device.set_tuning(from_dict(table[key]))
        return {"tuning": table[key], "key": key, "searched": False, "trials": 0}
    t, trials = device.autotune(view, params)
    table[key] = to_dict(t)
    save(table, path)
    return {"tuning": table[key], "key": key, "searched": True, "trials": trials}
