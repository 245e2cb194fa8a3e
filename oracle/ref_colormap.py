"""Builds the reference renderer's colour path as a host library (test
infrastructure only, like the rest of oracle/).

The reference draws its field image with OpenGL: `Renderer::generate*Colormap`
(src/renderer.cpp:672-800) fill a 256-texel RGB32F 1-D texture, and the
fragment shader `FIELD_FRAGMENT_SHADER` (src/renderer.cpp:47-77) greys wall
cells, normalises the field value and looks it up in that texture.  This
script reads both from the reference's own source where it lies and writes
one C++ translation unit into oracle/_ref/:

* the five generators, verbatim except that `Renderer::` is dropped (they use
  no member state);
* the shader's `main()` body, verbatim except that GLSL float literals get the
  `f` suffix they need to stay single precision in C++, under a small shim:
  vec2 / vec3 / vec4, `clamp`, the uniforms and in / out variables as
  globals, and `texture()`.  The shim's 1-D lookup is the OpenGL rule for
  GL_LINEAR + GL_CLAMP_TO_EDGE (u = s * 256 - 1/2, texels floor(u) and
  floor(u) + 1 clamped to [0, 255], weights 1 - frac(u) and frac(u)) in exact
  FP32; a GPU's texture unit quantises the weight, which this does not model.
  The 2-D lookups return the fragment's own texel (one fragment per cell).

It then compiles that unit with g++ into oracle/_ref/libcmap_ref.so, which
exports `ref_colormap_table` and `ref_colormap`.  Nothing here is shipped or
linked by the product; tests/golden/make_golden_colormap.py turns the
library's outputs into committed fixtures.

Usage: python oracle/ref_colormap.py <reference checkout> <output dir>
"""
import os
import re
import subprocess
import sys

GENERATORS = ["Jet", "Hot", "Plasma", "Inferno", "Viridis"]  # colormap ids 0..4


def _braced(text, start):
    """Return the text of the brace block opening at or after `start`."""
    i = text.index("{", start)
    depth = 0
    for k in range(i, len(text)):
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[i:k + 1]
    raise ValueError("unbalanced braces")


def extract(renderer_src):
    """The generator functions (as free functions) and the shader's main body."""
    gens = []
    for name in GENERATORS:
        m = re.search(r"void\s+Renderer::(generate%sColormap)\s*\(\s*std::vector<float>\s*&\s*colors\s*\)" % name,
                      renderer_src)
        if not m:
            raise ValueError(f"generate{name}Colormap not found")
        gens.append(f"static void {m.group(1)}(std::vector<float> &colors)\n" + _braced(renderer_src, m.end()))
    m = re.search(r'FIELD_FRAGMENT_SHADER\s*=\s*R"\((.*?)\)";', renderer_src, re.S)
    if not m:
        raise ValueError("FIELD_FRAGMENT_SHADER not found")
    glsl = m.group(1)
    mm = re.search(r"void\s+main\s*\(\s*\)", glsl)
    body = _braced(glsl, mm.end())
    # GLSL float literals are single precision; in C++ they need the suffix
    body = re.sub(r"(?<![\w.])(\d+\.\d+)(?![\w.])", r"\1f", body)
    return gens, body


SHIM = r"""// Generated by oracle/ref_colormap.py from the reference's src/renderer.cpp.
// Test infrastructure only: the reference's colour-table generators and the
// body of its field fragment shader under a minimal GLSL shim.
#include <algorithm>
#include <cmath>
#include <vector>

struct vec2 { float x, y; };
struct vec3 { float r, g, b; };
struct vec4 {
    float r, g, b, a;
    vec4() : r(0), g(0), b(0), a(0) {}
    vec4(float R, float G, float B, float A) : r(R), g(G), b(B), a(A) {}
    vec4(vec3 c, float A) : r(c.r), g(c.g), b(c.b), a(A) {}
};
struct Texel { float r; vec3 rgb; };
static float clamp(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
struct sampler1D { const float *rgb; };  // 256 RGB texels
struct sampler2D { float v; };           // the fragment's own texel
static Texel texture(sampler2D s, vec2) { Texel t; t.r = s.v; t.rgb = vec3{s.v, s.v, s.v}; return t; }
// GL_LINEAR, GL_CLAMP_TO_EDGE, 256 texels, exact FP32 weights
static Texel texture(sampler1D s, float c) {
    const float u = c * 256.0f - 0.5f;
    const float fl = std::floor(u);
    const float w = u - fl;
    int i0 = (int)fl, i1 = (int)fl + 1;
    i0 = i0 < 0 ? 0 : (i0 > 255 ? 255 : i0);
    i1 = i1 < 0 ? 0 : (i1 > 255 ? 255 : i1);
    float o[3];
    for (int k = 0; k < 3; k++) o[k] = (1.0f - w) * s.rgb[3 * i0 + k] + w * s.rgb[3 * i1 + k];
    Texel t; t.r = o[0]; t.rgb = vec3{o[0], o[1], o[2]}; return t;
}

// ---- the reference's colour-table generators
@GENERATORS@

// ---- the reference's field fragment shader: uniforms and in / out as globals
static vec2 TexCoord;
static vec4 FragColor;
static sampler2D fieldTexture, cellTypeTexture;
static sampler1D colormapTexture;
static float minVal, maxVal;
static void shader_main()
@SHADER@

static void table(int cmap, std::vector<float> &colors) {
    switch (cmap) {
    case 0: generateJetColormap(colors); break;
    case 1: generateHotColormap(colors); break;
    case 2: generatePlasmaColormap(colors); break;
    case 3: generateInfernoColormap(colors); break;
    default: generateViridisColormap(colors); break;
    }
}

extern "C" void ref_colormap_table(int cmap, float *rgb) {
    std::vector<float> c;
    table(cmap, c);
    std::copy(c.begin(), c.begin() + 768, rgb);
}

// One fragment per cell: field value and cell class (as the float the
// cell-type texture holds) in, RGBA out.
extern "C" void ref_colormap(const float *field, const float *cell_type, long n, int cmap, float lo, float hi,
                             float *rgba) {
    std::vector<float> c;
    table(cmap, c);
    colormapTexture.rgb = c.data();
    minVal = lo;
    maxVal = hi;
    for (long e = 0; e < n; e++) {
        fieldTexture.v = field[e];
        cellTypeTexture.v = cell_type[e];
        TexCoord = vec2{0.5f, 0.5f};
        shader_main();
        rgba[4 * e + 0] = FragColor.r;
        rgba[4 * e + 1] = FragColor.g;
        rgba[4 * e + 2] = FragColor.b;
        rgba[4 * e + 3] = FragColor.a;
    }
}
"""


def main(ref_root, out_dir):
    src_path = os.path.join(ref_root, "src", "renderer.cpp")
    with open(src_path, encoding="utf-8") as f:
        gens, body = extract(f.read())
    unit = SHIM.replace("@GENERATORS@", "\n\n".join(gens)).replace("@SHADER@", body)
    os.makedirs(out_dir, exist_ok=True)
    cpp = os.path.join(out_dir, "colormap_ref.cpp")
    with open(cpp, "w", encoding="utf-8") as f:
        f.write(unit)
    so = os.path.join(out_dir, "libcmap_ref.so")
    # plain IEEE single precision: no fast-math, no FMA contraction
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", cpp, "-o", so], check=True)
    return so


if __name__ == "__main__":
    if len(sys.argv) != 3:
        sys.exit(__doc__)
    print("ref_colormap: built", main(sys.argv[1], sys.argv[2]))
