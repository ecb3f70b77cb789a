"""Spectral power distribution files (the reference's liar.tools.spd, src/liar/tools/spd.py).

A file is whitespace-separated columns: the wavelength, then one column per spectrum. Lines that
are empty or start with '#' or ';' are skipped. Wavelengths above 1 are taken as nanometres and
converted to metres.
"""
from __future__ import annotations

import io

from liar_b200 import _tables
from liar_b200.spectra import Sampled


def _records(lines):
    for raw in lines:
        line = raw.strip()
        if line and not line.startswith(("#", ";")):
            yield [float(v) for v in line.split()]


def load(fp) -> list:
    """The spectra of an open text file, one Sampled per value column."""
    rows = list(_records(fp))
    if not rows:
        raise ValueError("no spectral data")
    width = len(rows[0])
    if width < 2 or any(len(r) != width for r in rows):
        raise ValueError("every line needs the wavelength and the same number of values")
    wavelengths = [r[0] for r in rows]
    if any(w > 1 for w in wavelengths):
        wavelengths = [w * 1e-9 for w in wavelengths]
    return [Sampled(wavelengths, [r[c] for r in rows]) for c in range(1, width)]


def loads(s: str) -> list:
    """load() of a string."""
    return load(io.StringIO(s))


def load_builtin_refractive_index(material: str) -> tuple[Sampled, Sampled]:
    """(n, k) of a built-in metal: Ag, Al, Au or Cu (the reference's data/spd/*.spd)."""
    try:
        rows = _tables.spd(material)
    except KeyError:
        raise ValueError(f"Material '{material}' not found in built-in data.") from None
    ws = [r[0] for r in rows]
    return Sampled(ws, [r[1] for r in rows]), Sampled(ws, [r[2] for r in rows])


def dump(obj, fp) -> None:
    """Writes one or more spectra sampled at the same wavelengths (nanometres when given in metres)."""
    spectra = [obj] if isinstance(obj, Sampled) else list(obj)
    if not spectra:
        raise ValueError("Must have a list of at least one spectrum")
    if not all(hasattr(s, "wavelengths") and hasattr(s, "values") for s in spectra):
        raise ValueError("All spectra must have 'wavelengths' and 'values' attributes (like Sampled)")
    ws = tuple(spectra[0].wavelengths)
    if any(tuple(s.wavelengths) != ws for s in spectra[1:]):
        raise ValueError("All spectra must be sampled on the same wavelengths. Resample before dumping.")
    if all(w < 1 for w in ws):
        ws = tuple(w * 1e9 for w in ws)
    for k, w in enumerate(ws):
        fp.write(" ".join(str(v) for v in (w, *(s.values[k] for s in spectra))) + "\n")
