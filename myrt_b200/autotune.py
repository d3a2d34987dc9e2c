"""Autotuner for the wavefront's launch shape: paths in flight per wave (the
queue size) and resident blocks per SM of the grid-stride kernels (the tile
of work per SM), chosen by timing the actual batch on the device.

Each candidate renders the batch once untimed (which also captures its CUDA
graph) and then `reps` times between CUDA events on the batch's stream; the
fastest candidate is applied and, when `cache` is given, stored in a JSON file
keyed by the device name and a digest of the batch's jobs, so later runs of
the same batch on the same kind of device skip the search.
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

WAVE_CANDIDATES = (1 << 20, 2 << 20, 4 << 20, 8 << 20, 16 << 20)
BLOCK_CANDIDATES = (4, 8, 12, 16)


def _signature(batch) -> str:
    h = hashlib.sha256(json.dumps([{k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in sorted(j.items())}
                                   for j in batch._jobs], sort_keys=True).encode())
    return h.hexdigest()[:16]


def time_frame(batch, reps: int = 2) -> float:
    """Milliseconds per myrt_batch_render (CUDA events on the batch's stream)."""
    import torch

    st = torch.cuda.ExternalStream(batch.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        e0.record(st)
    for _ in range(reps):
        batch.render()
    with torch.cuda.stream(st):
        e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_batch(batch, waves=WAVE_CANDIDATES, blocks=BLOCK_CANDIDATES, reps: int = 2, cache: str | None = None,
               device_name: str | None = None) -> dict:
    """Returns {"wave_paths", "blocks_per_sm", "ms", "results"} and leaves the
    best setting applied; the batch's accumulation is reset afterwards."""
    key = None
    if cache:
        if device_name is None:
            import torch

            device_name = torch.cuda.get_device_name()
        key = f"{device_name}|{_signature(batch)}"
        path = Path(cache)
        if path.exists():
            known = json.loads(path.read_text()).get(key)
            if known:
                batch.set_tuning(known["wave_paths"], known["blocks_per_sm"])
                return dict(known, cached=True)
    results = []
    for w in waves:
        for b in blocks:
            batch.set_tuning(w, b)
            batch.render()  # capture + warm-up
            ms = time_frame(batch, reps)
            results.append({"wave_paths": w, "blocks_per_sm": b, "ms": ms})
            batch.reset()
    best = min(results, key=lambda r: r["ms"])
    batch.set_tuning(best["wave_paths"], best["blocks_per_sm"])
    batch.reset()
    out = {"wave_paths": best["wave_paths"], "blocks_per_sm": best["blocks_per_sm"], "ms": best["ms"],
           "results": results}
    if cache and key:
        path = Path(cache)
        path.parent.mkdir(parents=True, exist_ok=True)
        data = json.loads(path.read_text()) if path.exists() else {}
        data[key] = {"wave_paths": best["wave_paths"], "blocks_per_sm": best["blocks_per_sm"], "ms": best["ms"]}
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1))
        os.replace(tmp, path)
    return out
