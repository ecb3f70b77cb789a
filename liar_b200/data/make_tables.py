"""Regenerates ``liar_b200/data/tables.json`` from the reference's data files.

The tables are public physical data, kept identical to the reference's so that spectral results
can be compared with it:
* ``observer``: the CIE 1931 2-degree colour matching functions (CVRL database), as shipped in the
  reference's data/observer.tsv (loaded by src/liar/__init__.py:51-66, wavelengths in nm there,
  stored here in metres like the reference's Observer).
* ``spd``: complex refractive index n + ik of Ag, Al, Au, Cu (Hagemann, Gudat, Kunz 1974 and the
  other sources named in each reference data/spd/*.spd header), wavelengths in metres.
* ``recovery``: the spectra of the tristimulus-to-spectrum recovery of Meng, Simon, Hanika and
  Dachsbacher, "Physically Meaningful Rendering using Tristimulus Colours" (EGSR 2015), sampled
  at chromaticities xy, as shipped in the reference's data/recovery_meng_simon.json (loaded by
  src/liar/__init__.py:72-79); wavelengths in metres.
* ``cornell_box``: the measured spectra of the Cornell box (Cornell University Program of Computer
  Graphics, "The Cornell Box" data): white, red and green wall reflectances and the light's
  emission, 400-700 nm in 4 nm steps, as embedded in the reference's src/liar/tools/cornell_box.py
  (the table passed to spd.loads there); wavelengths in metres.

Run in a container that has the reference mounted: ``python liar_b200/data/make_tables.py
/path/to/reference``. The product reads only the generated JSON.
"""
import json
import sys
from pathlib import Path


def read_columns(path: Path):
    rows = []
    for line in path.read_text().splitlines():
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        rows.append(line.split())
    return rows


def main(ref: Path) -> None:
    rows = read_columns(ref / "data" / "observer.tsv")
    header, body = rows[0], rows[1:]
    assert header == ["w", "xbar", "ybar", "zbar"], header
    observer = [[float(r[0]) * 1e-9, float(r[1]), float(r[2]), float(r[3])] for r in body]
    spd = {}
    for name in ("Ag", "Al", "Au", "Cu"):
        body = read_columns(ref / "data" / "spd" / f"{name}.spd")
        spd[name] = [[float(r[0]) * 1e-9, float(r[1]), float(r[2])] for r in body]
    rec = json.loads((ref / "data" / "recovery_meng_simon.json").read_text())
    recovery = {"wavelengths": [float(w) * 1e-9 for w in rec["wavelengths"]],
                "xy": [[float(v) for v in s["xy"]] for s in rec["spectra"]],
                "spectra": [[float(v) for v in s["spectrum"]] for s in rec["spectra"]]}
    # the numeric table of the spd.loads("""...""") literal in tools/cornell_box.py
    text = (ref / "src" / "liar" / "tools" / "cornell_box.py").read_text()
    body = text.split('spd.loads("""', 1)[1].split('"""', 1)[0]
    cols = [[float(v) for v in line.split()] for line in body.splitlines() if line.strip()]
    assert all(len(c) == 5 for c in cols), "expected wavelength, white, red, green, light columns"
    cornell = {"wavelengths": [c[0] * 1e-9 for c in cols], "white": [c[1] for c in cols],
               "red": [c[2] for c in cols], "green": [c[3] for c in cols], "light": [c[4] for c in cols]}
    out = Path(__file__).resolve().parent / "tables.json"
    out.write_text(json.dumps({"observer": observer, "spd": spd, "recovery": recovery, "cornell_box": cornell},
                              indent=None, separators=(",", ":")))
    print(out, len(observer), {k: len(v) for k, v in spd.items()}, len(recovery["xy"]), len(cols))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} REFERENCE_CHECKOUT")
    main(Path(sys.argv[1]))
