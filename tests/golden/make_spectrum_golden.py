"""Writes tests/golden/sampled_resample.json from the reference's own known-answer test.

Source: test/test_spectrum.cpp:256-278 (TEST(Spectrum, Sampled)) evaluates
liar.spectra.Sampled([400e-9, 500e-9, 600e-9], [0.1, 0.2, 0.]).resample(ws) and expects vs (to
1e-6). The reference cannot be built here, so the vectors are read from the test source as text.
Run: python tests/golden/make_spectrum_golden.py /path/to/reference
"""
import json
import re
import sys
from pathlib import Path


def floats(text):
    return [float(x.rstrip("f")) for x in re.findall(r"[-+]?\d*\.?\d+(?:e[-+]?\d+)?f?", text)]


def main(ref: Path):
    src = (ref / "test" / "test_spectrum.cpp").read_text()
    block = src[src.index("TEST(Spectrum, Sampled)"):]
    call = re.search(r'evaluate\("liar\.spectra\.Sampled\(\[(.*?)\], \[(.*?)\]\)"\)', block)
    ws = re.search(r"TWavelengths ws = \{(.*?)\};", block, re.S)
    vs = re.search(r"TValues vs =\s*\{(.*?)\};", block, re.S)
    out = {
        "source": "test/test_spectrum.cpp TEST(Spectrum, Sampled)",
        "sampled_wavelengths": floats(call.group(1)),
        "sampled_values": floats(call.group(2)),
        "resample_wavelengths": floats(ws.group(1)),
        "expected_values": floats(vs.group(1)),
        "tolerance": 1e-6,
    }
    path = Path(__file__).resolve().parent / "sampled_resample.json"
    path.write_text(json.dumps(out, indent=1))
    print(path, out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} REFERENCE_CHECKOUT")
    main(Path(sys.argv[1]))
