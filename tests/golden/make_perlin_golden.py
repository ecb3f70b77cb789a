"""Writes tests/golden/perlin_tables.json: outputs of pcg-cpp's pcg32_k2_fast and the permutation
tables that the reference's Perlin texture builds from a seed (src/liar/textures/perlin.cpp:
140-151: `pcg32_k2_fast rng(seed); std::shuffle(table, table + 256, rng)` per axis).

The reference pins pcg-cpp cci.20220409 (conanfile.py:93). Its generator is compiled here from
the copy of pcg-cpp that pyarrow vendors (pyarrow/include/arrow/vendored/pcg, the same generator
definitions), and std::shuffle is this machine's libstdc++ (g++), the standard library of a Linux
build of the reference. liar_b200/textures.py restates both; tests/test_textures.py checks the
restatement against these vectors.

Usage: python tests/golden/make_perlin_golden.py
"""
from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
SEEDS = [0, 1, 7, 42, 1234567, 4294967295]

SOURCE = r"""
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>
#include "arrow/vendored/pcg/pcg_random.hpp"
using arrow_vendored::pcg32_k2_fast;
int main() {
    const uint32_t seeds[] = {@SEEDS@};
    std::printf("{");
    for (size_t s = 0; s < sizeof(seeds) / sizeof(seeds[0]); ++s) {
        std::printf("%s\"%u\": {\"outputs\": [", s ? ", " : "", seeds[s]);
        pcg32_k2_fast g(seeds[s]);
        for (int i = 0; i < 20; ++i) std::printf("%s%u", i ? ", " : "", (unsigned)g());
        std::printf("], \"tables\": [");
        pcg32_k2_fast rng(seeds[s]);
        for (int k = 0; k < 3; ++k) {
            size_t table[256];
            for (size_t i = 0; i < 256; ++i) table[i] = i;
            std::shuffle(table, table + 256, rng);
            std::printf("%s[", k ? ", " : "");
            for (size_t i = 0; i < 256; ++i) std::printf("%s%zu", i ? ", " : "", table[i]);
            std::printf("]");
        }
        std::printf("], \"shuffles\": {");
        for (int n : {2, 3, 10, 11}) {  // both parities of std::shuffle's paired draws
            pcg32_k2_fast r2(seeds[s]);
            std::vector<size_t> v(n);
            for (int i = 0; i < n; ++i) v[i] = (size_t)i;
            std::shuffle(v.begin(), v.end(), r2);
            std::printf("%s\"%d\": [", n == 2 ? "" : ", ", n);
            for (int i = 0; i < n; ++i) std::printf("%s%zu", i ? ", " : "", v[i]);
            std::printf("]");
        }
        std::printf("}}");
    }
    std::printf("}\n");
    return 0;
}
"""


def main() -> None:
    import pyarrow
    inc = pyarrow.get_include()
    with tempfile.TemporaryDirectory() as tmp:
        src = Path(tmp) / "gen.cpp"
        src.write_text(SOURCE.replace("@SEEDS@", ", ".join(f"{s}u" for s in SEEDS)))
        exe = Path(tmp) / "gen"
        subprocess.run(["g++", "-O1", "-std=c++17", "-I", inc, str(src), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
        gxx = subprocess.run(["g++", "-dumpfullversion"], capture_output=True, text=True).stdout.strip()
    data = json.loads(out)
    data = {"generator": "pcg32_k2_fast (pcg-cpp as vendored by pyarrow)", "shuffle": f"libstdc++ of g++ {gxx}",
            "seeds": data}
    (HERE / "perlin_tables.json").write_text(json.dumps(data, separators=(",", ":")))
    print(HERE / "perlin_tables.json", len(SEEDS), "seeds")


if __name__ == "__main__":
    main()
