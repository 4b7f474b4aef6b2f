"""Persisted autotuning table, one JSON file per device.

The reference specialises its kernels per call through NVRTC macros
(search/gpu_bls.py:33-36: dtype, N_TILE, bin and duration counts).  Here the
kernels are compiled once, and the launch-time knobs that do not change any
result -- periods per work-queue tile, the staged order of the points -- are
chosen per kind of batch by timing (``BLSEngine.autotune``) and remembered in
this table, so that later processes on the same kind of device start with the
tuned settings.

File: ``<dir>/tuning-<device name>-sm<major><minor>.json``, where ``dir`` is
``$ATB_TUNING_DIR`` or ``~/.cache/astro_transit_gpu_b200``.  Entries are keyed
by ``BLSEngine.tune_key`` (method, and the powers of two of the curve count,
mean points and mean periods), written as a string.  A file written by another
library version or device is ignored.
"""
from __future__ import annotations

import json
import os
import re
import tempfile
import threading
from typing import Any, Dict, Optional

FORMAT = 1


def default_dir() -> str:
    return os.environ.get("ATB_TUNING_DIR") or os.path.join(
        os.path.expanduser("~"), ".cache", "astro_transit_gpu_b200")


def table_path(device_name: str, capability, directory: Optional[str] = None) -> str:
    slug = re.sub(r"[^A-Za-z0-9]+", "_", device_name).strip("_") or "device"
    return os.path.join(directory or default_dir(),
                        f"tuning-{slug}-sm{capability[0]}{capability[1]}.json")


def key_str(key) -> str:
    return "|".join(str(k) for k in key)


class TuningTable:
    """Tuned knob settings per kind of batch for one device (thread-safe)."""

    def __init__(self, path: str, device_name: str, library: str):
        self.path = path
        self.device_name = device_name
        self.library = library
        self.entries: Dict[str, Dict[str, Any]] = {}
        self._lock = threading.Lock()

    def load(self) -> "TuningTable":
        """Read the file if it exists and was written for this device and
        library version; anything else leaves the table empty."""
        try:
            with open(self.path) as f:
                doc = json.load(f)
        except (OSError, ValueError):
            return self
        if (doc.get("format") == FORMAT and doc.get("device") == self.device_name
                and doc.get("library") == self.library and isinstance(doc.get("entries"), dict)):
            with self._lock:
                self.entries = {str(k): dict(v) for k, v in doc["entries"].items()
                                if isinstance(v, dict)}
        return self

    def save(self) -> None:
        """Write the table atomically (a temporary file renamed into place)."""
        with self._lock:
            doc = {"format": FORMAT, "device": self.device_name, "library": self.library,
                   "entries": self.entries}
        d = os.path.dirname(self.path)
        os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=d, prefix=".tuning-", suffix=".json")
        try:
            with os.fdopen(fd, "w") as f:
                json.dump(doc, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except BaseException:
            try:
                os.unlink(tmp)
            except OSError:
                pass
            raise

    def get(self, key) -> Optional[Dict[str, Any]]:
        with self._lock:
            e = self.entries.get(key_str(key))
            return dict(e) if e is not None else None

    def put(self, key, settings: Dict[str, Any]) -> None:
        with self._lock:
            self.entries[key_str(key)] = dict(settings)
