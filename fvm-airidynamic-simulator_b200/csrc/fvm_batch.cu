// fvm_batch.cu -- many independent solves advanced together (C ABI
// fvm_batch_*).  No reference counterpart: the reference runs one solve.
//
// Each instance is a full solve handle (own buffers, geometry, ghost table,
// device scalars, own CFL time step).  A batched step is six launches for the
// whole batch (viscous pre-pass, stage 1, ghost pass, stage 2, viscous
// post-pass, ghost pass + per-instance finalize); each launch is a persistent
// grid walking a tile list that spans every instance.  Which ping-pong buffer
// holds U^n is kept per instance on the device, so one captured CUDA graph of
// a step replays for any number of steps and any mix of instance parities.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "fvm_handle.h"
#include "fvm_tma.cuh"

struct fvm_batch {
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t admit = nullptr;     // set-up of instances being added (overlaps running steps)
    fvm_ext ext{};
    StageTune tune{128, 6, 32};
    bool tune_fixed = false;          // FVM_BATCH_TUNE pins the launch shape
    std::vector<fvm_handle *> slots;  // instance id -> handle (nullptr when free)
    std::vector<long long> steps;     // steps taken per instance
    std::vector<fvm_handle *> parked; // retired instances kept for reuse at the same grid size
    // device descriptors of the active instances
    BatchInst *d_insts = nullptr;
    TileDesc *d_stage_tiles = nullptr, *d_visc_tiles = nullptr;
    GhostChunk *d_chunks = nullptr;
    int n_active = 0, n_stage_tiles = 0, n_visc_tiles = 0, n_chunks = 0;
    size_t cap_insts = 0, cap_stage = 0, cap_visc = 0, cap_chunks = 0;
    bool dirty = true;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
};

static int berr(int code, const char *msg) { return fvm_internal_set_error(code, msg); }

#define BCK(call)                                                                  \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) return berr(FVM_ERR_CUDA, cudaGetErrorString(_e));  \
    } while (0)

static void drop_graph(fvm_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

template <class T>
static int ensure(T **ptr, size_t *cap, size_t n) {
    if (n <= *cap && *ptr) return FVM_OK;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    size_t c = std::max<size_t>(n, 16);
    if (cudaMalloc(ptr, c * sizeof(T)) != cudaSuccess) return berr(FVM_ERR_ALLOC, "batch descriptor allocation");
    *cap = c;
    return FVM_OK;
}

// Rows per tile for the current set of instances: the tallest tile in
// {64, 32, 16} that still gives about 2000 tiles, so the persistent grid
// (148 SMs x resident CTAs) stays fed with work while tall tiles keep the
// per-tile halo rows cheap.  Measured on B200: 48M cells over 256 solves run
// best at 64, ~10M cells at 32, ~2.7M cells at 16 (64 loses 16 % there).
static int batch_rows(const fvm_batch *b) {
    const int W = stage_cols_per_cta(b->tune);
    for (int rows : {64, 32}) {
        long long tiles = 0;
        for (const fvm_handle *h : b->slots)
            if (h) tiles += (long long)((h->g.nx + W - 1) / W) * ((h->g.ny + rows - 1) / rows);
        if (tiles >= 2000) return rows;
    }
    return 16;
}

// Rebuild the device descriptors and tile lists after the set of instances changed.
static int rebuild(fvm_batch *b) {
    std::vector<BatchInst> insts;
    std::vector<TileDesc> stiles, vtiles;
    std::vector<GhostChunk> chunks;
    if (!b->tune_fixed) b->tune.rows = batch_rows(b);
    const int W = stage_cols_per_cta(b->tune), rows = b->tune.rows;
    for (size_t id = 0; id < b->slots.size(); id++) {
        fvm_handle *h = b->slots[id];
        if (!h) continue;
        BatchInst I;
        memset(&I, 0, sizeof I);
        for (int k = 0; k < 4; k++) {
            I.tm_in[k] = h->tm_in[k];
            I.tm_ctr[k] = h->tm_ctr[k];
            I.buf[k] = h->buf[k];
        }
        I.g = h->g;
        I.mask = h->mask;
        I.sc = h->sc;
        I.fs = Freestream{h->prm.rho_inf, h->prm.u_inf, h->prm.v_inf, h->prm.p_inf};
        I.wall = WallParams{h->prm.enable_viscosity, h->prm.adiabatic_wall, h->prm.T_wall};
        I.prandtl = h->ext.prandtl;
        I.ref_prandtl = (h->ext.prandtl == PRANDTL_REF) ? 1 : 0;
        I.viscous = h->prm.enable_viscosity ? 1 : 0;
        I.ghosts = h->ghosts;
        I.n_ghost = h->n_ghost;
        I.n_gchunks = std::max(1, (h->n_ghost + 127) / 128);
        I.recompute_dt = h->ext.dt_policy == FVM_DT_RECOMPUTE;
        I.cfl_num = h->prm.cfl;
        I.cfl_visc = h->prm.cfl_visc;
        I.min_dx = fminf(h->prm.dx, h->prm.dy);
        const int inst = (int)insts.size();
        insts.push_back(I);
        for (int j0 = 0; j0 < h->g.ny; j0 += rows)
            for (int i0 = 0; i0 < h->g.nx; i0 += W) {
                stiles.push_back(TileDesc{inst, i0, j0, 0});
                if (I.viscous) vtiles.push_back(TileDesc{inst, i0, j0, 0});
            }
        for (int c = 0; c < I.n_gchunks; c++) chunks.push_back(GhostChunk{inst, c * 128, 128, 0});
    }
    if (int r = ensure(&b->d_insts, &b->cap_insts, insts.size())) return r;
    if (int r = ensure(&b->d_stage_tiles, &b->cap_stage, stiles.size())) return r;
    if (int r = ensure(&b->d_visc_tiles, &b->cap_visc, vtiles.size())) return r;
    if (int r = ensure(&b->d_chunks, &b->cap_chunks, chunks.size())) return r;
    if (!insts.empty())
        BCK(cudaMemcpyAsync(b->d_insts, insts.data(), insts.size() * sizeof(BatchInst), cudaMemcpyHostToDevice,
                            b->stream));
    if (!stiles.empty())
        BCK(cudaMemcpyAsync(b->d_stage_tiles, stiles.data(), stiles.size() * sizeof(TileDesc),
                            cudaMemcpyHostToDevice, b->stream));
    if (!vtiles.empty())
        BCK(cudaMemcpyAsync(b->d_visc_tiles, vtiles.data(), vtiles.size() * sizeof(TileDesc),
                            cudaMemcpyHostToDevice, b->stream));
    if (!chunks.empty())
        BCK(cudaMemcpyAsync(b->d_chunks, chunks.data(), chunks.size() * sizeof(GhostChunk), cudaMemcpyHostToDevice,
                            b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    b->n_active = (int)insts.size();
    b->n_stage_tiles = (int)stiles.size();
    b->n_visc_tiles = (int)vtiles.size();
    b->n_chunks = (int)chunks.size();
    b->dirty = false;
    drop_graph(b);
    return FVM_OK;
}

static int enqueue_batch_step(fvm_batch *b) {
    const int sch = b->ext.flux_scheme, lim = b->ext.limiter;
    const StageTune &tn = b->tune;
    cudaStream_t st = b->stream;
    if (b->n_visc_tiles) {
        BCK(launch_viscous_batch(tn, b->d_insts, b->d_visc_tiles, b->n_visc_tiles, 0, st));
        b->launches++;
    }
    // launches as in a single solve's step: stage 1 and an Euler-only stage 2
    // let the ghost pass after them launch early; with viscous instances the
    // post half step follows stage 2, which then launches plainly
    const bool visc = b->n_visc_tiles > 0;
    BCK(launch_stage_batch(1, sch, lim, tn, b->d_insts, b->d_stage_tiles, b->n_stage_tiles, 1, true, st));
    BCK(launch_ghost_batch(b->d_insts, b->d_chunks, b->n_chunks, 1, st));
    BCK(launch_stage_batch(2, sch, lim, tn, b->d_insts, b->d_stage_tiles, b->n_stage_tiles, visc ? 0 : 1, !visc, st));
    b->launches += 3;
    if (b->n_visc_tiles) {
        BCK(launch_viscous_batch(tn, b->d_insts, b->d_visc_tiles, b->n_visc_tiles, 1, st));
        b->launches++;
    }
    BCK(launch_ghost_batch(b->d_insts, b->d_chunks, b->n_chunks, 2, st));
    b->launches++;
    return FVM_OK;
}

#define CHECK_BATCH(b)                                                     \
    do {                                                                   \
        if (!(b)) return berr(FVM_ERR_INVALID, "null batch");              \
    } while (0)

static fvm_handle *inst_of(fvm_batch *b, int id) {
    if (!b || id < 0 || id >= (int)b->slots.size()) return nullptr;
    return b->slots[id];
}

extern "C" int fvm_batch_create(fvm_batch **out, const fvm_ext *ext) {
    if (!out) return berr(FVM_ERR_INVALID, "null out");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return berr(FVM_ERR_CUDA, "no CUDA device");
    fvm_batch *b = new fvm_batch();
    if (ext)
        b->ext = *ext;
    else
        fvm_ext_default(&b->ext);
    if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->admit, cudaStreamNonBlocking) != cudaSuccess) {
        if (b->own) cudaStreamDestroy(b->own);
        delete b;
        return berr(FVM_ERR_CUDA, "stream creation failed");
    }
    b->stream = b->own;
    if (const char *env = getenv("FVM_BATCH_TUNE")) {
        int x = 0, y = 0, z = 0;
        if (sscanf(env, "%d,%d,%d", &x, &y, &z) == 3 && (x == 128 || x == 256) && (y == 4 || y == 6) && z >= 4) {
            b->tune = StageTune{x, y, z};
            b->tune_fixed = true;
        }
    }
    *out = b;
    return FVM_OK;
}

extern "C" int fvm_batch_destroy(fvm_batch *b) {
    if (!b) return FVM_OK;
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (fvm_handle *h : b->slots)
        if (h) fvm_destroy(h);
    for (fvm_handle *h : b->parked) fvm_destroy(h);
    cudaFree(b->d_insts);
    cudaFree(b->d_stage_tiles);
    cudaFree(b->d_visc_tiles);
    cudaFree(b->d_chunks);
    if (b->own) cudaStreamDestroy(b->own);
    if (b->admit) cudaStreamDestroy(b->admit);
    delete b;
    return FVM_OK;
}

extern "C" int fvm_batch_set_stream(fvm_batch *b, void *stream) {
    CHECK_BATCH(b);
    cudaStreamSynchronize(b->stream);
    b->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : b->own;
    for (fvm_handle *h : b->slots)
        if (h) fvm_set_stream(h, b->stream);
    drop_graph(b);
    return FVM_OK;
}

// HBM bytes one instance of this size holds (admission estimate).
extern "C" size_t fvm_batch_instance_bytes(int nx, int ny) {
    const size_t pitch = ((size_t)nx + 31) / 32 * 32;
    const size_t plane = pitch * (size_t)ny;
    // 4 states of 5 float planes, SDF plane, mask plane, dense cell classes,
    // a generous ghost-table bound and the fixed-size scalars/partials
    return plane * 5 * 4 * 4 + plane * 4 + plane + (size_t)nx * ny + (size_t)(nx + ny) * 16 * 28 + 64 * 1024;
}

extern "C" int fvm_batch_add(fvm_batch *b, const fvm_sim_params *p, int *id_out) {
    CHECK_BATCH(b);
    if (!p || !id_out) return berr(FVM_ERR_INVALID, "null argument");
    // The instance is set up on the admission stream, so adding does not wait
    // for batched steps already queued on the batch stream (the new instance
    // joins the tile list at the next fvm_batch_step).
    fvm_handle *h = nullptr;
    // a retired instance of the same grid size keeps its buffers: reset it in place
    for (size_t k = 0; k < b->parked.size(); k++) {
        fvm_handle *c = b->parked[k];
        if (c->g.nx == p->nx && c->g.ny == p->ny) {
            b->parked.erase(b->parked.begin() + (long)k);
            c->stream = b->admit;  // parked: no work of its own pending
            if (int r = fvm_reset(c, p)) {
                fvm_destroy(c);
                return r;
            }
            h = c;
            break;
        }
    }
    if (!h) {
        if (int r = fvm_create(&h)) return r;
        h->stream = b->admit;
        if (int r = fvm_initialize(h, p, &b->ext)) {
            fvm_destroy(h);
            return r;
        }
    }
    // the batch launches one kernel shape for every instance (threads and
    // ring depth fix the tensor maps; rows per tile is chosen at rebuild)
    if (h->tune.nt != b->tune.nt || h->tune.ring != b->tune.ring) {
        h->tune = b->tune;
        if (int r = fvm_internal_build_maps(h)) {
            fvm_destroy(h);
            return r;
        }
    }
    // first time step of this solve (recompute policy) or the given one
    float dt = p->dt;
    if (b->ext.dt_policy == FVM_DT_RECOMPUTE) {
        if (int r = fvm_internal_compute_dt(h, p, &dt)) {
            fvm_destroy(h);
            return r;
        }
    }
    // device scalars of the fresh solve; on a CUDA error the instance is
    // destroyed here, so its memory never stays outside the batch's accounting
    auto fail = [&](cudaError_t e) {
        fvm_destroy(h);
        return berr(FVM_ERR_CUDA, cudaGetErrorString(e));
    };
    DevScalars init;
    cudaError_t ce;
    if ((ce = cudaMemcpyAsync(&init, h->sc, sizeof init, cudaMemcpyDeviceToHost, b->admit)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(b->admit)) != cudaSuccess)
        return fail(ce);
    init.dt = dt;
    init.t = p->t_current;
    init.parity = 0;
    init.counter = 0;
    init.red[0] = init.red[1] = 0.0f;
    if ((ce = cudaMemcpyAsync(h->sc, &init, sizeof init, cudaMemcpyHostToDevice, b->admit)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(b->admit)) != cudaSuccess)
        return fail(ce);
    h->stream = b->stream;
    int id = -1;
    for (size_t k = 0; k < b->slots.size(); k++)
        if (!b->slots[k]) {
            id = (int)k;
            break;
        }
    if (id < 0) {
        id = (int)b->slots.size();
        b->slots.push_back(nullptr);
        b->steps.push_back(0);
    }
    b->slots[id] = h;
    b->steps[id] = 0;
    b->dirty = true;
    *id_out = id;
    return FVM_OK;
}

extern "C" int fvm_batch_remove(fvm_batch *b, int id) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h) return berr(FVM_ERR_INVALID, "unknown instance id");
    cudaStreamSynchronize(b->stream);
    fvm_destroy(h);
    b->slots[id] = nullptr;
    b->dirty = true;
    return FVM_OK;
}

extern "C" int fvm_batch_retire(fvm_batch *b, int id) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h) return berr(FVM_ERR_INVALID, "unknown instance id");
    b->parked.push_back(h);
    b->slots[id] = nullptr;
    b->dirty = true;
    return FVM_OK;
}

extern "C" int fvm_batch_trim(fvm_batch *b, size_t keep_bytes, size_t *parked_bytes_out) {
    CHECK_BATCH(b);
    auto held = [](fvm_handle *h) {
        size_t x = 0;
        fvm_memory_usage(h, &x);
        return x;
    };
    size_t total = 0;
    for (fvm_handle *h : b->parked) total += held(h);
    if (total > keep_bytes) BCK(cudaStreamSynchronize(b->stream));
    // oldest first
    while (total > keep_bytes && !b->parked.empty()) {
        fvm_handle *h = b->parked.front();
        total -= held(h);
        b->parked.erase(b->parked.begin());
        fvm_destroy(h);
    }
    if (parked_bytes_out) *parked_bytes_out = total;
    return FVM_OK;
}

bool fvm_internal_batch_has_parked(fvm_batch *b, int nx, int ny) {
    for (fvm_handle *h : b->parked)
        if (h->g.nx == nx && h->g.ny == ny) return true;
    return false;
}

extern "C" int fvm_batch_count(fvm_batch *b, int *n) {
    CHECK_BATCH(b);
    if (!n) return berr(FVM_ERR_INVALID, "null output");
    int c = 0;
    for (fvm_handle *h : b->slots) c += h != nullptr;
    *n = c;
    return FVM_OK;
}

extern "C" int fvm_batch_step(fvm_batch *b, int n) {
    CHECK_BATCH(b);
    if (n < 0) return berr(FVM_ERR_INVALID, "negative step count");
    if (b->dirty)
        if (int r = rebuild(b)) return r;
    if (b->n_active == 0 || n == 0) return FVM_OK;
    const bool graphs = getenv("FVM_NO_GRAPH") == nullptr && b->stream != cudaStreamLegacy &&
                        b->stream != cudaStreamPerThread && b->stream != nullptr;
    if (graphs && !b->graph) {
        cudaGraph_t g;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        long long before = b->launches;
        int r = enqueue_batch_step(b);
        cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
        b->launches = before;
        if (r) return r;
        BCK(ec);
        cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        BCK(ei);
    }
    const int per = 4 + (b->n_visc_tiles ? 2 : 0);
    for (int k = 0; k < n; k++) {
        if (graphs) {
            BCK(cudaGraphLaunch(b->graph, b->stream));
            b->launches += per;
        } else if (int r = enqueue_batch_step(b)) {
            return r;
        }
    }
    for (size_t id = 0; id < b->slots.size(); id++)
        if (b->slots[id]) b->steps[id] += n;
    return FVM_OK;
}

extern "C" int fvm_batch_synchronize(fvm_batch *b) {
    CHECK_BATCH(b);
    BCK(cudaStreamSynchronize(b->stream));
    for (fvm_handle *h : b->slots) {
        if (!h) continue;
        DevScalars s;
        BCK(cudaMemcpy(&s, h->sc, sizeof s, cudaMemcpyDeviceToHost));
        if (s.err & kErrTimeout) return berr(FVM_ERR_TIMEOUT, "a bounded device wait expired in a batched step");
        if (s.err & kErrSmemAlign)
            return berr(FVM_ERR_CUDA, "shared-memory staging area not 128-byte aligned; batched step skipped");
    }
    return FVM_OK;
}

// Current parameters of an instance: t_current, step and the dt of its last
// step (recompute policy) are read from the device.
extern "C" int fvm_batch_instance(fvm_batch *b, int id, fvm_sim_params *p_out) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h || !p_out) return berr(FVM_ERR_INVALID, "unknown instance id or null output");
    BCK(cudaStreamSynchronize(b->stream));
    DevScalars s;
    BCK(cudaMemcpy(&s, h->sc, sizeof s, cudaMemcpyDeviceToHost));
    *p_out = h->prm;
    p_out->step = (int)b->steps[id];
    if (b->ext.dt_policy == FVM_DT_RECOMPUTE) {
        p_out->t_current = s.t;
        p_out->dt = b->steps[id] > 0 ? s.dt_last : s.dt;
    } else {
        p_out->t_current = h->prm.t_current + (float)b->steps[id] * h->prm.dt;
    }
    return FVM_OK;
}

extern "C" int fvm_batch_read_fields(fvm_batch *b, int id, float *rho, float *rho_u, float *rho_v, float *E,
                                     float *rho_e) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h) return berr(FVM_ERR_INVALID, "unknown instance id");
    BCK(cudaStreamSynchronize(b->stream));
    unsigned parity = 0;
    BCK(cudaMemcpy(&parity, &h->sc->parity, sizeof parity, cudaMemcpyDeviceToHost));
    const float *src = h->buf[parity ? BUF_X : BUF_N];
    float *dst[5] = {rho, rho_u, rho_v, E, rho_e};
    for (int k = 0; k < 5; k++)
        if (dst[k])
            BCK(cudaMemcpy2D(dst[k], (size_t)h->g.nx * 4, src + (size_t)k * h->g.plane, (size_t)h->g.pitch * 4,
                             (size_t)h->g.nx * 4, h->g.ny, cudaMemcpyDeviceToHost));
    return FVM_OK;
}

extern "C" int fvm_batch_nonfinite_count(fvm_batch *b, int id, unsigned long long *count) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h || !count) return berr(FVM_ERR_INVALID, "unknown instance id or null output");
    BCK(cudaStreamSynchronize(b->stream));
    return fvm_nonfinite_count(h, count, 0);
}

extern "C" int fvm_batch_diagnostics(fvm_batch *b, int id, fvm_diag *out) {
    CHECK_BATCH(b);
    fvm_handle *h = inst_of(b, id);
    if (!h || !out) return berr(FVM_ERR_INVALID, "unknown instance id or null output");
    BCK(cudaStreamSynchronize(b->stream));
    unsigned parity = 0;
    BCK(cudaMemcpy(&parity, &h->sc->parity, sizeof parity, cudaMemcpyDeviceToHost));
    // point the handle's current-state slot at the buffer holding U^n
    float *saved = h->buf[BUF_N];
    h->buf[BUF_N] = parity ? h->buf[BUF_X] : saved;
    int r = fvm_diagnostics(h, out);
    h->buf[BUF_N] = saved;
    return r;
}

extern "C" int fvm_batch_memory_usage(fvm_batch *b, size_t *bytes) {
    CHECK_BATCH(b);
    if (!bytes) return berr(FVM_ERR_INVALID, "null output");
    size_t t = 0;
    for (fvm_handle *h : b->slots) {
        if (!h) continue;
        size_t x = 0;
        fvm_memory_usage(h, &x);
        t += x;
    }
    *bytes = t;
    return FVM_OK;
}

extern "C" int fvm_batch_launch_count(fvm_batch *b, long long *count_out) {
    CHECK_BATCH(b);
    if (!count_out) return berr(FVM_ERR_INVALID, "null output");
    *count_out = b->launches;
    return FVM_OK;
}
