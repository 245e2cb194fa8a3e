"""Colour images (fvm_colormap_*): the renderer's colour tables (CPU) and the
field pass on the GPU against the oracle's CPU restatement of the fragment
shader on the same derived field.  The restatement and the library's tables
are pinned to the reference's own renderer code: tests/golden/ref_colormap.npz
holds the outputs of its colour-table generators and of its field fragment
shader compiled for the host (tests/golden/make_golden_colormap.py)."""
import os

import numpy as np
import pytest

from helpers import small
import fvm_b200
from fvm_b200 import abi
from oracle import oracle


@pytest.mark.parametrize("cmap", range(5))
def test_library_tables_equal_the_oracle_tables(cmap):
    assert np.array_equal(fvm_b200.colormap_table(cmap), oracle.colormap_table(cmap))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_colormap.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("cmap", range(5))
def test_tables_equal_the_reference_generators(golden, cmap):
    """Renderer::generate*Colormap (src/renderer.cpp:672-800): bit-exact."""
    ref = golden["tables"][cmap]
    assert np.array_equal(oracle.colormap_table(cmap), ref)
    assert np.array_equal(fvm_b200.colormap_table(cmap), ref)


@pytest.mark.parametrize("cmap", range(5))
def test_oracle_shader_equals_the_reference_shader(golden, cmap):
    """FIELD_FRAGMENT_SHADER (src/renderer.cpp:47-77) on every golden sample
    (texel centres and edges, both clamped ends, a degenerate range, every
    cell class 0..4): bit-exact in FP32."""
    field, ct = golden["field"], golden["cell_type"]
    assert set(np.unique(ct)) == {0, 1, 2, 3, 4}
    for r, (lo, hi) in enumerate(golden["ranges"]):
        got = oracle.colormap(field, ct, cmap, float(lo), float(hi), fmt=0)
        assert np.array_equal(got, golden["rgba"][r, cmap]), (r, cmap)


def test_reference_extraction_on_a_synthetic_renderer():
    """oracle/ref_colormap.py takes the generators as free functions and the
    shader's main body with single-precision literals."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "ref_colormap", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                                     "ref_colormap.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    gens = "".join(f"void Renderer::generate{n}Colormap(std::vector<float> &colors)\n{{\n    if (1) {{ colors[0] = 0.5f; }}\n}}\n"
                   for n in mod.GENERATORS)
    shader = ('const char *FIELD_FRAGMENT_SHADER = R"(\n#version 330 core\nuniform float minVal;\n'
              'void main() {\n    float a = clamp(x / (y + 0.0001), 0.0, 1.0);\n    vec4 c = vec4(0.3, 0.3, 0.3, 1.0);\n}\n)";\n')
    out_gens, body = mod.extract(gens + shader)
    assert len(out_gens) == 5 and all(g.startswith("static void generate") for g in out_gens)
    assert all("Renderer::" not in g and g.rstrip().endswith("}") for g in out_gens)
    assert "0.0001f" in body and "clamp(x / (y + 0.0001f), 0.0f, 1.0f)" in body
    assert "vec4(0.3f, 0.3f, 0.3f, 1.0f)" in body and "uniform" not in body


def test_table_end_points():
    jet, hot = fvm_b200.colormap_table(abi.CMAP_JET), fvm_b200.colormap_table(abi.CMAP_HOT)
    assert tuple(jet[0]) == (0.0, 0.0, 0.5) and tuple(jet[255]) == (0.5, 0.0, 0.0)
    assert tuple(hot[0]) == (0.0, 0.0, 0.0) and np.allclose(hot[255], 1.0, atol=1e-6)
    for c in range(5):
        t = fvm_b200.colormap_table(c)
        assert t.min() >= 0.0 and t.max() <= 1.0


def test_oracle_shader_masks_walls_and_clamps():
    field = np.array([[-1.0, 0.0, 0.5, 2.0, 3.0, 0.5]], np.float32)
    ct = np.array([[0, 0, 0, 0, 0, 1]], np.uint8)
    img = oracle.colormap(field, ct, abi.CMAP_HOT, 0.0, 1.0, fmt=0)
    assert np.allclose(img[0, 5], (0.3, 0.3, 0.3, 1.0))
    assert np.array_equal(img[0, 0], img[0, 1])  # below range clamps to the first texel
    assert np.array_equal(img[0, 3], img[0, 4])  # above range clamps to the last texel
    assert np.allclose(img[0, 3, :3], oracle.colormap_table(abi.CMAP_HOT)[255])
    u8 = oracle.colormap(field, ct, abi.CMAP_HOT, 0.0, 1.0, fmt=1)
    assert u8.dtype == np.uint8 and (u8[..., 3] == 255).all()


def test_errors_and_ppm(tmp_path):
    with pytest.raises(fvm_b200.FvmError):
        fvm_b200.colormap_table(7)
    img = np.zeros((3, 5, 4), np.uint8)
    img[0, :, 0] = 255  # bottom row red
    path = tmp_path / "f.ppm"
    fvm_b200.write_ppm(path, img)
    data = path.read_bytes()
    assert data.startswith(b"P6\n5 3\n255\n") and len(data) == len(b"P6\n5 3\n255\n") + 45
    assert data[-15] == 255  # last row written is the bottom grid row


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [abi.FIELD_TEMPERATURE, abi.FIELD_MACH, abi.FIELD_PRESSURE])
def test_gpu_image_matches_oracle_shader(kind):
    import torch
    p, e = small("euler_m3_circle", 320, 160)
    s = fvm_b200.Solver(p, e)
    p.dt = s.compute_dt()
    s.step(60)
    n = p.nx * p.ny
    field = torch.empty(n, dtype=torch.float32, device="cuda")
    s.field_to_device(kind, field.data_ptr())
    s.synchronize()
    f = field.cpu().numpy().reshape(p.ny, p.nx)
    ct = s.cell_types().reshape(p.ny, p.nx)
    fluid = (ct != abi.CELL_SOLID) & (ct != abi.CELL_GHOST)
    lo, hi = float(f[fluid].min()), float(f[fluid].max())
    for cmap in range(5):
        rgba = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        s.colormap_to_device(kind, cmap, lo, hi, rgba.data_ptr(), abi.RGBA_F32)
        u8 = torch.empty((n, 4), dtype=torch.uint8, device="cuda")
        s.colormap_to_device(kind, cmap, lo, hi, u8.data_ptr(), abi.RGBA_U8)
        s.synchronize()
        g32 = rgba.cpu().numpy().reshape(p.ny, p.nx, 4)
        g8 = u8.cpu().numpy().reshape(p.ny, p.nx, 4)
        r32 = oracle.colormap(f, ct, cmap, lo, hi, fmt=0)
        r8 = oracle.colormap(f, ct, cmap, lo, hi, fmt=1)
        # float: the GPU's normalising division is the fast approximate one
        assert np.abs(g32 - r32).max() <= 2e-5, cmap
        d8 = np.abs(g8.astype(int) - r8.astype(int))
        assert d8.max() <= 1 and (d8 > 0).mean() <= 1e-3, cmap
        assert np.array_equal(g8[~fluid], r8[~fluid])
