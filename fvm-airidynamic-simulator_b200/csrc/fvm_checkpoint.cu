// fvm_checkpoint.cu -- checkpoint / restore files (C ABI fvm_save_checkpoint,
// fvm_load_checkpoint).  No reference counterpart: the reference keeps its
// state only in device memory.
//
// File layout (little endian):
//   fvm_ckpt_header (256 bytes: magic "FVMB200C", version, grid, the solve's
//   parameters and extension knobs, the device time-step state)
//   payload: rho, rho*u, rho*v, E, rho*e as nx*ny float32 planes, row-major
//   (idx = j*nx + i), the layout of fvm_read_fields
// The header's CRC-32 (IEEE 802.3, reflected, polynomial 0xEDB88320) covers
// the payload.  Restoring reproduces the saved solve bit for bit: besides the
// fields, the header carries the time step the next step will use, the
// device-side simulated time and the CFL maxima of the last step, which
// otherwise would be recomputed from the state by a different reduction.
#include <cstdio>
#include <cstring>
#include <vector>

#include "fvm_handle.h"

namespace {

constexpr char kMagic[8] = {'F', 'V', 'M', 'B', '2', '0', '0', 'C'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kFlagDtReady = 1u, kFlagCflValid = 2u;

struct fvm_ckpt_header {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    int32_t nx, ny;
    uint32_t fields;  // 5
    uint32_t flags;   // kFlagDtReady, kFlagCflValid
    float next_dt, t_device, cfl_speed, cfl_nu;
    uint64_t payload_bytes;
    uint32_t payload_crc32;
    uint32_t reserved0;
    fvm_sim_params params;
    fvm_ext ext;
    unsigned char pad[256 - 64 - sizeof(fvm_sim_params) - sizeof(fvm_ext)];
};
static_assert(sizeof(fvm_ckpt_header) == 256, "checkpoint header is 256 bytes");

struct Crc32 {
    uint32_t table[256];
    Crc32() {
        for (uint32_t n = 0; n < 256; n++) {
            uint32_t c = n;
            for (int k = 0; k < 8; k++) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[n] = c;
        }
    }
    uint32_t update(uint32_t crc, const unsigned char *p, size_t n) const {
        crc = ~crc;
        for (size_t i = 0; i < n; i++) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
        return ~crc;
    }
};
const Crc32 &crc_table() {
    static const Crc32 t;
    return t;
}

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

int ckerr(int code, const char *msg) { return fvm_internal_set_error(code, msg); }

}  // namespace

extern "C" int fvm_save_checkpoint(fvm_handle *h, const fvm_sim_params *p, const char *path) {
    if (!h || !p || !path) return ckerr(FVM_ERR_INVALID, "fvm_save_checkpoint: null argument");
    if (!h->Un) return ckerr(FVM_ERR_STATE, "fvm_save_checkpoint: solver not initialized");
    const int nx = h->g.nx, ny = h->g.ny;
    const size_t plane = (size_t)nx * ny;
    std::vector<float> data(plane * 5);
    if (int r = fvm_read_fields(h, data.data(), data.data() + plane, data.data() + 2 * plane, data.data() + 3 * plane,
                                data.data() + 4 * plane))
        return r;
    cudaError_t e = cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return ckerr(FVM_ERR_CUDA, cudaGetErrorString(e));
    fvm_ckpt_header hd;
    memset(&hd, 0, sizeof hd);
    memcpy(hd.magic, kMagic, 8);
    hd.version = kVersion;
    hd.header_bytes = sizeof hd;
    hd.nx = nx;
    hd.ny = ny;
    hd.fields = 5;
    hd.flags = (h->dt_ready ? kFlagDtReady : 0u) | (h->cfl_valid ? kFlagCflValid : 0u);
    hd.next_dt = h->h_sc->dt;
    hd.t_device = h->h_sc->t;
    hd.cfl_speed = h->h_sc->cfl[0];
    hd.cfl_nu = h->h_sc->cfl[1];
    hd.payload_bytes = plane * 5 * sizeof(float);
    hd.payload_crc32 =
        crc_table().update(0u, reinterpret_cast<const unsigned char *>(data.data()), (size_t)hd.payload_bytes);
    hd.params = *p;
    hd.ext = h->ext;
    File f;
    f.f = fopen(path, "wb");
    if (!f.f) return ckerr(FVM_ERR_INVALID, "fvm_save_checkpoint: cannot open the file for writing");
    if (fwrite(&hd, sizeof hd, 1, f.f) != 1 || fwrite(data.data(), sizeof(float), plane * 5, f.f) != plane * 5)
        return ckerr(FVM_ERR_INVALID, "fvm_save_checkpoint: short write");
    if (fclose(f.f) != 0) {
        f.f = nullptr;
        return ckerr(FVM_ERR_INVALID, "fvm_save_checkpoint: close failed");
    }
    f.f = nullptr;
    return FVM_OK;
}

// Read and validate a checkpoint file: header fields and the payload CRC.
static int read_checkpoint(const char *path, fvm_ckpt_header &hd, std::vector<float> *data) {
    if (!path) return ckerr(FVM_ERR_INVALID, "checkpoint: null path");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return ckerr(FVM_ERR_INVALID, "checkpoint: cannot open the file");
    if (fread(&hd, sizeof hd, 1, f.f) != 1) return ckerr(FVM_ERR_INVALID, "checkpoint: short header");
    if (memcmp(hd.magic, kMagic, 8) != 0) return ckerr(FVM_ERR_INVALID, "checkpoint: not a checkpoint file");
    if (hd.version != kVersion || hd.header_bytes != sizeof hd || hd.fields != 5)
        return ckerr(FVM_ERR_UNSUPPORTED, "checkpoint: unsupported checkpoint version or layout");
    if (hd.nx <= 0 || hd.ny <= 0 || hd.params.nx != hd.nx || hd.params.ny != hd.ny ||
        hd.payload_bytes != (uint64_t)hd.nx * (uint64_t)hd.ny * 5u * sizeof(float))
        return ckerr(FVM_ERR_INVALID, "checkpoint: inconsistent header");
    const size_t n = (size_t)hd.nx * hd.ny * 5;
    std::vector<float> local;
    std::vector<float> &buf = data ? *data : local;
    buf.resize(n);
    if (fread(buf.data(), sizeof(float), n, f.f) != n) return ckerr(FVM_ERR_INVALID, "checkpoint: short payload");
    if (crc_table().update(0u, reinterpret_cast<const unsigned char *>(buf.data()), (size_t)hd.payload_bytes) !=
        hd.payload_crc32)
        return ckerr(FVM_ERR_INVALID, "checkpoint: payload checksum mismatch");
    return FVM_OK;
}

extern "C" int fvm_checkpoint_info(const char *path, fvm_sim_params *p_out, fvm_ext *ext_out) {
    fvm_ckpt_header hd;
    if (int r = read_checkpoint(path, hd, nullptr)) return r;
    if (p_out) *p_out = hd.params;
    if (ext_out) *ext_out = hd.ext;
    return FVM_OK;
}

extern "C" int fvm_load_checkpoint(fvm_handle *h, const char *path, fvm_sim_params *p_out) {
    if (!h) return ckerr(FVM_ERR_INVALID, "fvm_load_checkpoint: null handle");
    fvm_ckpt_header hd;
    std::vector<float> data;
    if (int r = read_checkpoint(path, hd, &data)) return r;
    const size_t plane = (size_t)hd.nx * hd.ny;
    // geometry, buffers and launch shapes from the saved parameters, then the state
    if (int r = fvm_initialize(h, &hd.params, &hd.ext)) return r;
    if (int r = fvm_write_fields(h, data.data(), data.data() + plane, data.data() + 2 * plane, data.data() + 3 * plane,
                                 data.data() + 4 * plane))
        return r;
    cudaError_t e = cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return ckerr(FVM_ERR_CUDA, cudaGetErrorString(e));
    h->h_sc->dt = hd.next_dt;
    h->h_sc->t = hd.t_device;
    h->h_sc->cfl[0] = hd.cfl_speed;
    h->h_sc->cfl[1] = hd.cfl_nu;
    e = cudaMemcpyAsync(h->sc, h->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice, h->stream);
    h->launches_at_sc_copy = -1;
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return ckerr(FVM_ERR_CUDA, cudaGetErrorString(e));
    h->dt_ready = (hd.flags & kFlagDtReady) != 0;
    h->fixed_dt = hd.next_dt;
    h->cfl_valid = (hd.flags & kFlagCflValid) != 0;
    h->disp_fresh = false;
    if (p_out) *p_out = hd.params;
    return FVM_OK;
}
