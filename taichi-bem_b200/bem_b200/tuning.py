"""Launch-shape autotuner for the context tuning keys (bem_ctx_set_tuning).

For a workload key (device, operation, problem size, precision) each
candidate value of a tuning key is set on the engine, the caller's `run`
is timed with CUDA events on the current stream (one untimed call first, then
the median of `repeats`), and the fastest value is kept on the engine and
written to a JSON cache, so later processes on the same kind of GPU take the
cached choice without timing.  The cache file is
$BEM_B200_TUNING_CACHE, else ~/.cache/bem_b200/tuning.json.

Only keys that change the launch shape and not the result's accuracy are
tuned this way (the Calderon sweep's form, the normal matrix's tile order,
the Cholesky panel width, the wavenumbers per k-batched launch); the
normal matrix's accumulation segment (BEM_TUNE_GRAM_KSEG) trades accuracy
for speed and keeps its built-in default.
"""
from __future__ import annotations

import json
import os
import statistics

from . import _lib as L

CACHE_ENV = "BEM_B200_TUNING_CACHE"
KEY_NAMES = {L.TUNE_CALDERON_GROUP: "calderon_group", L.TUNE_GRAM_KSEG: "gram_kseg", L.TUNE_CHOL_NB: "chol_nb",
             L.TUNE_GRAM_BAND: "gram_band", L.TUNE_KBATCH_GROUP: "kbatch_group",
             L.TUNE_GRAM_PAIR: "gram_pair", L.TUNE_LU_UPDATE: "lu_update"}


def cache_path() -> str:
    return os.environ.get(CACHE_ENV) or os.path.join(os.path.expanduser("~"), ".cache", "bem_b200", "tuning.json")


def device_key(device=None) -> str:
    """'<name>/sm<major><minor>/<SMs>' of the CUDA device."""
    import torch
    p = torch.cuda.get_device_properties(device if device is not None else torch.cuda.current_device())
    return f"{p.name}/sm{p.major}{p.minor}/{p.multi_processor_count}"


def cuda_timer(run, repeats: int) -> float:
    """Median milliseconds of `run()` over `repeats` calls after one untimed
    call, CUDA events on the current stream."""
    import torch
    run()
    ts = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


class Autotuner:
    """Chooses tuning-key values per workload key and caches them.

    engine: an object with set_tuning(key, value) (bem_b200.engine.Engine);
    timer(run, repeats) -> ms (default: CUDA events); path: the JSON cache
    (default: cache_path()); device: the device part of the workload key
    (default: device_key())."""

    def __init__(self, engine, path: str | None = None, timer=None, device: str | None = None):
        self.engine = engine
        self.path = path or cache_path()
        self.timer = timer or cuda_timer
        self._device = device
        self.last = {}

    @property
    def device(self) -> str:
        if self._device is None:
            self._device = device_key()
        return self._device

    def load(self) -> dict:
        try:
            with open(self.path) as fh:
                d = json.load(fh)
            return d if isinstance(d, dict) else {}
        except (OSError, ValueError):
            return {}

    def _save(self, entry_key: str, entry: dict):
        d = self.load()
        d[entry_key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        tmp = self.path + f".tmp{os.getpid()}"
        with open(tmp, "w") as fh:
            json.dump(d, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def entry_key(self, workload: str, knob: int) -> str:
        return f"{self.device}|{workload}|{KEY_NAMES.get(knob, str(knob))}"

    def cached(self, workload: str, knob: int, candidates) -> int | None:
        """The cached choice for `workload` if it is one of `candidates`, set
        on the engine; else None (nothing set)."""
        c = self.load().get(self.entry_key(workload, knob))
        if isinstance(c, dict) and c.get("value") in [int(x) for x in candidates]:
            self.engine.set_tuning(knob, int(c["value"]))
            return int(c["value"])
        return None

    def tune(self, workload: str, knob: int, candidates, run, repeats: int = 1, retune: bool = False) -> int:
        """The value of tuning key `knob` for `workload`: the cached choice if
        it is one of `candidates` (and not `retune`), else the fastest
        candidate by timing `run`.  The chosen value is left set on the
        engine.  self.last records the timings ({} for a cached choice)."""
        candidates = [int(c) for c in candidates]
        ek = self.entry_key(workload, knob)
        if not retune:
            c = self.cached(workload, knob, candidates)
            if c is not None:
                self.last = {}
                return c
        times = {}
        for c in candidates:
            self.engine.set_tuning(knob, c)
            times[c] = float(self.timer(run, repeats))
        best = min(candidates, key=lambda c: times[c])
        self.engine.set_tuning(knob, best)
        self.last = times
        self._save(ek, {"value": best, "ms": {str(c): t for c, t in times.items()}})
        return best
