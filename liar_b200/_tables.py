"""Access to the spectral data tables in liar_b200/data/tables.json (CIE 1931 observer, metal n, k,
Meng-Simon recovery spectra, the Cornell box's measured spectra)."""
from __future__ import annotations

import functools
import json
from pathlib import Path

import numpy as np

_PATH = Path(__file__).resolve().parent / "data" / "tables.json"


@functools.lru_cache(maxsize=None)
def _load() -> dict:
    return json.loads(_PATH.read_text())


def observer() -> np.ndarray:
    """(n, 4) float32: wavelength (m), xbar, ybar, zbar."""
    return np.asarray(_load()["observer"], dtype=np.float32)


@functools.lru_cache(maxsize=None)
def observer_y_weights() -> tuple[np.ndarray, np.ndarray]:
    """Wavelengths and trapezoid weights whose dot product with a spectrum gives its Y, normalised so
    that the unit spectrum has Y = 1 (Observer::Observer / tristimulus, kernel/observer.cpp:57-188)."""
    o = observer().astype(np.float64)
    w = o[:, 0]
    n = len(w)
    dY = np.zeros(n)
    prev = w[0]
    for k in range(n - 1):
        dY[k] = o[k, 2] * ((w[k + 1] - prev) / 2)
        prev = w[k]
    dY[n - 1] = o[n - 1, 2] * ((w[n - 1] - prev) / 2)
    return w, dY / dY.sum()


def spd(name: str) -> list:
    return _load()["spd"][name]


def recovery() -> dict:
    """{"wavelengths": [m], "xy": [[x, y]], "spectra": [[values]]}."""
    return _load()["recovery"]


def cornell_box() -> dict:
    """{"wavelengths": [m], "white", "red", "green", "light": [values]}: the measured Cornell box
    spectra (the table of the reference's src/liar/tools/cornell_box.py)."""
    return _load()["cornell_box"]
