"""Batched ensembles: many independent SNAC models advanced together.

The reference runs one model per process; a batch holds hundreds of models
of uneven mesh size and material parameters and advances all of them with
one launch per kernel type per step (snac_gpu_batch_* in include/snac_gpu.h).
Per-model results are bit-identical to stepping each model alone.

    b = SnacBatch(cfgs)           # cfgs: list of SnacConfig
    b.time_step_zero()
    autotune(b)                   # optional: pick the launch shape (cached)
    b.step(2000)
    s = b.models[7].state()       # any model, as a SnacContext view

The autotuner times candidate launch shapes (threads per node tile,
persistent-grid sizes, steps per CUDA graph, tile order) on a scratch batch
built from the same configurations, by coordinate descent from the
default, and caches the winner per (GPU, batch signature) in a JSON file.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
from typing import Dict, List, Optional, Sequence

from .abi import BatchTuning, Desc, SnacConfig
from .context import SnacContext, SnacError, load_library

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tuning_cache.json")


class SnacBatch:
    """n models on one GPU, one launch per kernel type per step."""

    def __init__(self, cfgs: Sequence[SnacConfig]):
        if not cfgs:
            raise ValueError("a batch needs at least one model")
        self.lib = load_library()
        self.cfgs = list(cfgs)
        descs = [c.desc() for c in self.cfgs]  # each config keeps its arrays alive
        self._descs = (Desc * len(descs))(*descs)
        self.h = C.c_void_p()
        rc = self.lib.snac_gpu_batch_create(self._descs, len(descs), C.byref(self.h))
        if rc != 0:
            msg = self.lib.snac_gpu_batch_last_error(self.h).decode() if self.h else ""
            if self.h:
                self.lib.snac_gpu_batch_destroy(self.h)
                self.h = C.c_void_p()
            raise SnacError(rc, msg or "snac_gpu_batch_create failed")
        self.models: List[SnacContext] = [
            SnacContext.borrowed(cfg, self.lib.snac_gpu_batch_model(self.h, i), self) for i, cfg in enumerate(self.cfgs)
        ]

    def __len__(self):
        return len(self.cfgs)

    def close(self):
        if self.h:
            for m in self.models:
                m.close()
            self.lib.snac_gpu_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> int:
        if rc != 0:
            m = self.lib.snac_gpu_batch_error_model(self.h)
            raise SnacError(rc, self.lib.snac_gpu_batch_last_error(self.h).decode(), m)
        return rc

    # -- stepping ----------------------------------------------------------------------
    def time_step_zero(self):
        return self._check(self.lib.snac_gpu_batch_time_step_zero(self.h))

    def step(self, n: int = 1):
        """n steps of every model, one launch per kernel type per step."""
        return self._check(self.lib.snac_gpu_batch_step(self.h, int(n)))

    def step_each(self, n: int = 1):
        """n steps of every model, model after model with each model's own launches."""
        return self._check(self.lib.snac_gpu_batch_step_each(self.h, int(n)))

    def time_steps(self, n: int, each: bool = False) -> float:
        """Device time (ms, CUDA events on the batch stream) of n steps."""
        ms = C.c_double()
        self._check(self.lib.snac_gpu_batch_time_steps(self.h, int(n), int(bool(each)), C.byref(ms)))
        return ms.value

    # -- launch shape -------------------------------------------------------------------
    @property
    def tuning(self) -> Dict[str, int]:
        t = BatchTuning()
        self._check(self.lib.snac_gpu_batch_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    @tuning.setter
    def tuning(self, d: Dict[str, int]):
        t = BatchTuning.from_dict({**self.tuning, **d})
        self._check(self.lib.snac_gpu_batch_set_tuning(self.h, C.byref(t)))

    @property
    def launches(self) -> int:
        return int(self.lib.snac_gpu_batch_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.snac_gpu_batch_stream(self.h) or 0)

    @property
    def n_elements(self) -> int:
        return sum(c.n_elements for c in self.cfgs)


# ---- autotuner -------------------------------------------------------------------------

# candidate values per knob, searched one knob at a time from the default
SEARCH_SPACE: Dict[str, List[int]] = {
    "steps_per_graph": [1, 4, 16, 64, 256],  # 256: the largest graph the library captures
    "elem_blocks_per_sm": [0, 4, 8, 16],
    "node_threads": [64, 128, 256],
    "node_blocks_per_sm": [0, 8, 16],
    "minls_threads": [64, 128, 256],
    "order": [0, 1],
    "split_classes": [1, 0],
}


def batch_signature(cfgs: Sequence[SnacConfig]) -> str:
    """Hash of what decides the launch shape: mesh sizes, rheology, temperature, dt type."""
    h = hashlib.sha1()
    for c in cfgs:
        h.update(f"{c.nx},{c.ny},{c.nz},{c.plugin},{int(bool(c.temperature))},{c.dtType};".encode())
    return f"{len(cfgs)}:{h.hexdigest()[:16]}"


def gpu_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        pass
    return "unknown-gpu"


def _load_cache(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def search(measure, start: Dict[str, int], space: Dict[str, List[int]] = SEARCH_SPACE, passes: int = 1):
    """Coordinate descent: for each knob, try its candidates with the others
    fixed and keep the fastest.  `measure(tuning) -> ms` (lower is better).
    Returns (best tuning, best ms, [(tuning, ms) tried])."""
    seen = {}

    def timed(t):
        key = tuple(sorted(t.items()))
        if key not in seen:
            seen[key] = measure(t)
            tried.append((dict(t), seen[key]))
        return seen[key]

    tried = []
    best = dict(start)
    best_ms = timed(best)
    for _ in range(passes):
        for knob, values in space.items():
            for v in values:
                cand = {**best, knob: v}
                ms = timed(cand)
                if ms < best_ms:
                    best, best_ms = cand, ms
    return best, best_ms, tried


def autotune(batch: SnacBatch, steps: int = 20, cache_path: Optional[str] = DEFAULT_CACHE,
             in_place: bool = False, force: bool = False, verbose: bool = False) -> Dict[str, int]:
    """Choose and apply the launch shape of `batch`.

    The search runs on a scratch batch built from the same configurations
    (so the batch's own models do not advance) unless in_place=True.  Each
    candidate is timed over `steps` steps after one untimed run that
    captures its graphs.  The result is cached per (GPU, batch signature)."""
    key = f"{gpu_name()}|{batch_signature(batch.cfgs)}"
    cache = _load_cache(cache_path) if cache_path else {}
    if not force and key in cache:
        batch.tuning = cache[key]["tuning"]
        return batch.tuning

    scratch = batch if in_place else SnacBatch(batch.cfgs)
    try:
        if not in_place:
            scratch.time_step_zero()
            scratch.step(1)  # leave step zero's unfused first step out of the timings

        def measure(t):
            scratch.tuning = t
            scratch.time_steps(max(t["steps_per_graph"], 2))  # capture this shape's graphs
            ms = scratch.time_steps(steps) / steps
            if verbose:
                print(f"  {t} -> {ms:.4f} ms/step", flush=True)
            return ms

        best, best_ms, tried = search(measure, scratch.tuning)
    finally:
        if not in_place:
            scratch.close()
    batch.tuning = best
    if cache_path:
        cache = _load_cache(cache_path)
        cache[key] = {"tuning": best, "ms_per_step": best_ms, "candidates": len(tried)}
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    return batch.tuning
