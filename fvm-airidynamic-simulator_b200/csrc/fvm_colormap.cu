// fvm_colormap.cu -- headless counterpart of the renderer's field pass:
// colour tables and the C ABI entry fvm_colormap_to_device.  The reference
// draws the field with an OpenGL fragment shader (src/renderer.cpp:47-77)
// sampling a 256-entry RGB table built on the CPU (src/renderer.cpp:672-799);
// here the same arithmetic runs as a CUDA kernel (k_colormap, fvm_aux.cu)
// into a caller device buffer, one RGBA pixel per cell, with no graphics API.
#include <algorithm>

#include "fvm_handle.h"

// The five 256-entry tables, t = i/255, in the reference generators'
// expressions: jet (piecewise linear, :672-716), hot (:719-734), and the
// polynomial plasma (:737-754), inferno (:757-779) and viridis (:782-799).
static void build_lut(int cmap, ColormapLUT &L) {
    for (int i = 0; i < 256; i++) {
        const float t = i / 255.0f;
        float r, g, b;
        switch (cmap) {
        case FVM_CMAP_JET:
            if (t < 0.125f) {
                r = 0.0f, g = 0.0f, b = 0.5f + 4.0f * t;
            } else if (t < 0.375f) {
                r = 0.0f, g = 4.0f * (t - 0.125f), b = 1.0f;
            } else if (t < 0.625f) {
                r = 4.0f * (t - 0.375f), g = 1.0f, b = 1.0f - 4.0f * (t - 0.375f);
            } else if (t < 0.875f) {
                r = 1.0f, g = 1.0f - 4.0f * (t - 0.625f), b = 0.0f;
            } else {
                r = 1.0f - 4.0f * (t - 0.875f), g = 0.0f, b = 0.0f;
            }
            break;
        case FVM_CMAP_HOT:
            r = std::min(1.0f, t * 2.5f);
            g = std::max(0.0f, std::min(1.0f, (t - 0.4f) * 2.5f));
            b = std::max(0.0f, (t - 0.8f) * 5.0f);
            break;
        case FVM_CMAP_PLASMA:
            r = 0.050383f + t * (2.028462f + t * (-1.312035f + t * 0.233106f));
            g = 0.029803f + t * (0.192182f + t * (1.429032f + t * (-1.651143f + t * 0.500000f)));
            b = 0.527975f + t * (1.573141f + t * (-2.481592f + t * 0.880392f));
            r = std::clamp(r, 0.0f, 1.0f), g = std::clamp(g, 0.0f, 1.0f), b = std::clamp(b, 0.0f, 1.0f);
            break;
        case FVM_CMAP_INFERNO:
            r = std::clamp(1.5f * t, 0.0f, 1.0f);
            g = std::clamp(2.0f * (t - 0.25f), 0.0f, 1.0f);
            b = std::clamp(0.6f - 1.2f * t, 0.0f, 0.6f);
            break;
        default:  // FVM_CMAP_VIRIDIS
            r = 0.267004f + t * (0.003991f + t * (0.494266f + t * 0.234652f));
            g = 0.004874f + t * (1.014627f + t * (-0.531556f + t * 0.512042f));
            b = 0.329415f + t * (1.423671f + t * (-2.252694f + t * 0.499477f));
            r = std::clamp(r, 0.0f, 1.0f), g = std::clamp(g, 0.0f, 1.0f), b = std::clamp(b, 0.0f, 1.0f);
            break;
        }
        L.rgb[3 * i] = r;
        L.rgb[3 * i + 1] = g;
        L.rgb[3 * i + 2] = b;
    }
}

extern "C" int fvm_colormap_table(int colormap, float *rgb_out) {
    if (!rgb_out) return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_table: null output");
    if (colormap < FVM_CMAP_JET || colormap > FVM_CMAP_VIRIDIS)
        return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_table: unknown colormap");
    ColormapLUT L;
    build_lut(colormap, L);
    std::copy(L.rgb, L.rgb + 256 * 3, rgb_out);
    return FVM_OK;
}

extern "C" int fvm_colormap_to_device(fvm_handle *h, int field_kind, int colormap, float min_val, float max_val,
                                      void *dev_rgba, int format) {
    if (!h) return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_to_device: null handle");
    if (!h->Un) return fvm_internal_set_error(FVM_ERR_STATE, "fvm_colormap_to_device: solver not initialized");
    if (!dev_rgba) return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_to_device: null destination");
    if (field_kind < 0 || field_kind > 4)
        return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_to_device: unknown field kind");
    if (colormap < FVM_CMAP_JET || colormap > FVM_CMAP_VIRIDIS)
        return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_to_device: unknown colormap");
    if (format != FVM_RGBA_F32 && format != FVM_RGBA_U8)
        return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_colormap_to_device: unknown pixel format");
    ColormapLUT L;
    build_lut(colormap, L);
    cudaError_t e = launch_colormap(field_kind, h->g, h->Un, h->ct, L, min_val, max_val, dev_rgba, format, h->stream);
    if (e != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    h->launches++;
    return FVM_OK;
}
