"""``liar.tools``: the reference's scripting helpers (src/liar/tools/): ``spd`` (spectral data
files), ``cornell_box`` (the Cornell box scene), ``scripting`` (render options and targets) and
``rgb_spaces`` (named RGB spaces)."""
