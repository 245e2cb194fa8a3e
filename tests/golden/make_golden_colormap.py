"""Generate the colour-image golden fixture from the reference's own renderer code.

Loads oracle/_ref/libcmap_ref.so, which oracle/ref_colormap.py builds from the
reference's src/renderer.cpp (the five `Renderer::generate*Colormap` table
generators, src/renderer.cpp:672-800, and the body of FIELD_FRAGMENT_SHADER,
src/renderer.cpp:47-77, under a GLSL shim whose 1-D lookup follows the OpenGL
GL_LINEAR / GL_CLAMP_TO_EDGE rule), and stores into
tests/golden/ref_colormap.npz:

* `tables`  (5, 256, 3) float32: the generators' RGB32F textures;
* `field`, `cell_type` (N,): a seeded sample of field values that covers the
  normalisation range, both clamped ends, every texel centre and texel edge of
  the first range, and every cell class 0..4 of the reference's CellType;
* `ranges`  (R, 2): the (minVal, maxVal) uniforms, one degenerate;
* `rgba`    (R, 5, N, 4) float32: the shader's FragColor per range, colormap
  and sample.

Runs on the host (no GPU).  Usage: python tests/golden/make_golden_colormap.py
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(REPO, "oracle", "_ref", "libcmap_ref.so")
OUT = os.path.join(HERE, "ref_colormap.npz")

RANGES = np.array([[0.0, 1.0], [-3.5, 12.25], [2.0, 2.0], [101325.0, 101375.0]], np.float32)


def sample():
    rng = np.random.default_rng(20261204)
    lo, hi = RANGES[0]
    span = hi - lo + np.float32(1e-4)
    k = np.arange(257, dtype=np.float32)
    centres = lo + (k[:256] + np.float32(0.5)) / np.float32(256.0) * span  # texel centres
    edges = lo + k / np.float32(256.0) * span                              # texel edges
    wide = rng.uniform(-0.5, 1.5, 600).astype(np.float32)                  # both clamped ends
    others = np.concatenate([rng.uniform(lo_, hi_, 40) for lo_, hi_ in RANGES[1:]]).astype(np.float32)
    ends = np.array([lo, hi, -1.0, 2.0, 0.0, 12.25, -3.5, 101325.0, 101375.0, 2.0], np.float32)
    field = np.concatenate([centres, edges, wide, others, ends]).astype(np.float32)
    cell_type = np.zeros(field.size, np.uint8)
    cell_type[rng.choice(field.size, field.size // 5, replace=False)] = rng.integers(1, 5, field.size // 5)
    return field, cell_type


def main():
    lib = C.CDLL(LIB)
    lib.ref_colormap_table.argtypes = [C.c_int, C.c_void_p]
    lib.ref_colormap.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_float, C.c_float, C.c_void_p]
    tables = np.zeros((5, 256, 3), np.float32)
    for c in range(5):
        lib.ref_colormap_table(c, tables[c].ctypes.data)
    field, cell_type = sample()
    ct_f = cell_type.astype(np.float32)  # the cell-type texture holds floats
    rgba = np.zeros((len(RANGES), 5, field.size, 4), np.float32)
    for r, (lo, hi) in enumerate(RANGES):
        for c in range(5):
            lib.ref_colormap(field.ctypes.data, ct_f.ctypes.data, field.size, c, float(lo), float(hi),
                             rgba[r, c].ctypes.data)
    np.savez_compressed(OUT, tables=tables, field=field, cell_type=cell_type, ranges=RANGES, rgba=rgba)
    print("wrote", OUT, field.size, "samples")


if __name__ == "__main__":
    main()
