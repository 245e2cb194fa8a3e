// fvm_api.cu -- the C ABI (include/fvm_b200.h): solve handle, device buffers,
// TMA descriptors, step orchestration, CUDA-graph replay, readback and
// measurement hooks.  Host C++ only launches kernels; there is no CPU
// compute path for anything the reference runs on the GPU.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fvm_b200.h"
#include "fvm_kernels.cuh"
#include "fvm_tma.cuh"

using namespace fvm;

#define FVM_STR2(x) #x
#define FVM_STR(x) FVM_STR2(x)

// ------------------------------------------------------------ error text
static thread_local std::string g_last_error = "";

static int set_err(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

extern "C" const char *fvm_last_error(void) { return g_last_error.c_str(); }

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess)                                                                         \
            return set_err(FVM_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
    } while (0)

#define CKA(call)                                                                                      \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess)                                                                         \
            return set_err(FVM_ERR_ALLOC, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
    } while (0)

#define CHECK_HANDLE(h)                                                                 \
    do {                                                                                \
        if (!(h)) return set_err(FVM_ERR_INVALID, "%s: null handle", __func__);         \
    } while (0)

#define CHECK_INIT(h)                                                                   \
    do {                                                                                \
        CHECK_HANDLE(h);                                                                \
        if (!(h)->Un) return set_err(FVM_ERR_STATE, "%s: solver not initialized", __func__); \
    } while (0)

// ------------------------------------------------------ parameter helpers
extern "C" void fvm_params_default(fvm_sim_params *p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->nx = 512;
    p->ny = 256;
    p->dx = 1.0f;
    p->dy = 1.0f;
    p->domain_width = 10.0f;
    p->domain_height = 5.0f;
    p->mach = 3.0f;
    p->T_inf = 300.0f;
    p->p_inf = 101325.0f;
    p->obstacle_x = 2.5f;
    p->obstacle_y = 2.5f;
    p->obstacle_r = 0.5f;
    p->obstacle_shape = FVM_SHAPE_CIRCLE;
    p->cfl = 0.5f;
    p->dt = 1e-6f;
    p->enable_viscosity = false;
    p->cfl_visc = 0.4f;
    p->adiabatic_wall = true;
    p->T_wall = 300.0f;
    p->paused = true;
}

// SimParams::computeDerived (src/include/common.h:93-101)
extern "C" void fvm_params_compute_derived(fvm_sim_params *p) {
    if (!p) return;
    p->rho_inf = p->p_inf / (R_GAS * p->T_inf);
    p->c_inf = sqrtf(GAMMA * R_GAS * p->T_inf);
    p->u_inf = p->mach * p->c_inf;
    p->dx = p->domain_width / (float)p->nx;
    p->dy = p->domain_height / (float)p->ny;
    p->obstacle_y = p->domain_height / 2.0f;
}

extern "C" void fvm_ext_default(fvm_ext *e) {
    if (!e) return;
    memset(e, 0, sizeof(*e));
    e->flux_scheme = FVM_FLUX_HLLC;
    e->limiter = FVM_LIMITER_MINMOD;
    e->prandtl = PRANDTL_REF;
    e->dt_policy = FVM_DT_FIXED;
    e->cone_half_angle = 0.2617993877991494f;
    e->cone_length = 0.3f;
    e->ref_length = 0.0f;
}

// ------------------------------------------------------------ TMA encode
typedef CUresult (*PFN_encodeTiled_t)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                      CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                      CUtensorMapFloatOOBfill);

static PFN_encodeTiled_t get_encode() {
    static PFN_encodeTiled_t fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled_t>(p);
    }
    return fn;
}

// 3-D map over (x, y, field) of one 5-plane state; box = (box_w, 1, 5).
static int encode_state_map(CUtensorMap *m, float *base, const GridDesc &g, int box_w) {
    PFN_encodeTiled_t enc = get_encode();
    if (!enc) return set_err(FVM_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, 5};
    cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 4, (cuuint64_t)g.plane * 4};
    cuuint32_t box[3] = {(cuuint32_t)box_w, 1, 5};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(FVM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FVM_OK;
}

#include "fvm_handle.h"

static const char *kKernelNames[] = {"stage1", "stage2", "viscous_pre", "viscous_post", "ghost1", "ghost2",
                                     "set_scalars"};

static cudaEvent_t take_event(fvm_handle *h) {
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

static void resolve_timing(fvm_handle *h) {
    if (h->pending.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto &t : h->pending) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        auto &slot = h->ktimes[kKernelNames[t.kernel]];
        slot.first += 1;
        slot.second += ms;
        h->event_pool.push_back(t.a);
        h->event_pool.push_back(t.b);
    }
    h->pending.clear();
}

// Runs `fn` (one kernel launch) bracketed by events when timing is on.
template <class F>
static cudaError_t timed(fvm_handle *h, int kernel, F fn) {
    if (!h->timing) {
        h->launches++;
        return fn();
    }
    TimedLaunch t{kernel, take_event(h), take_event(h)};
    cudaEventRecord(t.a, h->stream);
    cudaError_t e = fn();
    cudaEventRecord(t.b, h->stream);
    h->pending.push_back(t);
    h->launches++;
    return e;
}

static void drop_graphs(fvm_handle *h) {
    for (int k = 0; k < 2; k++) {
        if (h->graph[k]) cudaGraphExecDestroy(h->graph[k]);
        h->graph[k] = nullptr;
        h->graph_key[k] = 0;
        if (h->graph1[k]) cudaGraphExecDestroy(h->graph1[k]);
        h->graph1[k] = nullptr;
        h->graph1_key[k] = 0;
    }
}

static void free_buffers(fvm_handle *h) {
    drop_graphs(h);
    for (int k = 0; k < NBUF; k++) {
        if (h->buf[k]) cudaFree(h->buf[k]);
        h->buf[k] = nullptr;
    }
    if (h->sdf) cudaFree(h->sdf);
    if (h->ct) cudaFree(h->ct);
    if (h->mask) cudaFree(h->mask);
    if (h->ghosts) cudaFree(h->ghosts);
    if (h->d_diag) cudaFree(h->d_diag);
    h->sdf = nullptr;
    h->ct = nullptr;
    h->mask = nullptr;
    h->ghosts = nullptr;
    h->d_diag = nullptr;
    h->n_ghost = h->ghost_cap = 0;
    h->bytes = 0;
    h->parity_base = nullptr;
}

// Launch tuning of the marching kernels per grid class: threads per CTA,
// input ring depth (rows) and rows per CTA.  The default comes from
// heuristic_tune below; FVM_TUNE="nt,ring,rows" overrides it; fvm_autotune
// measures the candidates and caches the winner per grid class for the
// process.
struct TuneKey {
    int nx, ny, viscous, scheme, limiter;
    bool operator<(const TuneKey &o) const {
        return std::tie(nx, ny, viscous, scheme, limiter) < std::tie(o.nx, o.ny, o.viscous, o.scheme, o.limiter);
    }
};
static std::map<TuneKey, StageTune> g_tune_cache;

// Default launch shape before (or without) autotuning: 128 threads, a 4-row
// input ring and about 48 row bands: the tile height in {4, 8, 16, ..., 64}
// nearest ny / 48.  Measured on B200 (NS step): 1024x512 fastest at 8 rows
// (0.071 ms; 10 and 12 rows 0.080 / 0.077), 2048x1024 at 24 (0.181 ms; 32 rows
// 0.197), 4096x2048 at 40-48 (0.614 ms; 64 rows 0.661), 8192x4096 at 64;
// 512x256 wants 4.  Small grids are latency-bound and want many short tiles,
// large ones tall tiles, which keep the per-tile halo rows cheap.
static StageTune heuristic_tune(int, int ny) {
    StageTune t{128, 4, 4};
    const double want = ny / 48.0;
    double best = 1e30;
    for (int rows : {4, 8, 16, 24, 32, 40, 48, 56, 64}) {
        const double d = rows > want ? rows - want : want - rows;
        if (d < best) {
            best = d;
            t.rows = rows;
        }
    }
    return t;
}

static StageTune pick_tune(const fvm_handle *h, int nx, int ny);

static StageTune pick_tune(const fvm_handle *h, int nx, int ny) {
    const char *env = getenv("FVM_TUNE");
    if (env) {
        int x = 0, y = 0, z = 0;
        if (sscanf(env, "%d,%d,%d", &x, &y, &z) == 3 && (x == 128 || x == 256) && (y == 4 || y == 6) && z >= 4 &&
            (z & 1) == 0)
            return StageTune{x, y, z};
    }
    TuneKey k{nx, ny, h->prm.enable_viscosity ? 1 : 0, h->ext.flux_scheme, h->ext.limiter};
    auto it = g_tune_cache.find(k);
    if (it != g_tune_cache.end()) return it->second;
    return heuristic_tune(nx, ny);
}

static int alloc_buffers(fvm_handle *h, int nx, int ny) {
    free_buffers(h);
    GridDesc g;
    g.nx = nx;
    g.ny = ny;
    g.pitch = (nx + 31) / 32 * 32;
    g.plane = (long long)g.pitch * ny;
    g.dx = h->prm.dx;
    g.dy = h->prm.dy;
    h->g = g;
    const size_t state_bytes = (size_t)g.plane * 5 * sizeof(float);
    for (int k = 0; k < NBUF; k++) {
        CKA(cudaMalloc(&h->buf[k], state_bytes));
        CK(cudaMemsetAsync(h->buf[k], 0, state_bytes, h->stream));
    }
    CKA(cudaMalloc(&h->sdf, (size_t)g.plane * sizeof(float)));
    CKA(cudaMalloc(&h->ct, (size_t)nx * ny));
    CKA(cudaMalloc(&h->mask, (size_t)g.plane));
    CK(cudaMemsetAsync(h->ct, 0, (size_t)nx * ny, h->stream));
    h->diag_parts = diagnostics_parts(g);
    CKA(cudaMalloc(&h->d_diag, (size_t)(h->diag_parts * 8 + 16) * sizeof(double)));
    h->bytes = state_bytes * NBUF + (size_t)g.plane * 5 + (size_t)nx * ny + (size_t)(h->diag_parts * 8 + 16) * 8;
    h->tune = pick_tune(h, nx, ny);
    return FVM_OK;
}

static int build_maps(fvm_handle *h) {
    CK(prepare_step_kernels(h->tune));
    for (int k = 0; k < NBUF; k++) {
        int r = encode_state_map(&h->tm_in[k], h->buf[k], h->g, stage_box_in(h->tune));
        if (r) return r;
        r = encode_state_map(&h->tm_ctr[k], h->buf[k], h->g, stage_box_blend(h->tune));
        if (r) return r;
    }
    return FVM_OK;
}

static Freestream freestream(const fvm_sim_params &p) { return Freestream{p.rho_inf, p.u_inf, p.v_inf, p.p_inf}; }
static WallParams wall(const fvm_sim_params &p) {
    return WallParams{p.enable_viscosity, p.adiabatic_wall, p.T_wall};
}

__global__ void k_set_scalars(DevScalars *sc, float dt, float t, int set_t) {
    sc->dt = dt;
    if (set_t) sc->t = t;
}

__global__ void k_zero_scalars(DevScalars *sc) {
    sc->red[0] = sc->red[1] = 0.0f;
    sc->cfl[0] = sc->cfl[1] = 0.0f;
    sc->counter = 0;
    sc->err = 0;
    sc->nonfinite = 0;
}

// Geometry from the current parameters: SDF + classes (optionally with the
// zero-state fix-up of newly exposed cells), masks and the ghost table.
static int build_geometry(fvm_handle *h, bool fixup) {
    const fvm_sim_params &p = h->prm;
    ShapeParamsHost s{p.obstacle_x, p.obstacle_y, p.obstacle_r, p.obstacle_rotation, p.wing_rotation,
                      h->ext.cone_half_angle, h->ext.cone_length, p.obstacle_shape};
    launch_sdf(h->g, s, h->sdf, h->ct, fixup ? h->Un : nullptr, h->stream);
    CK(cudaGetLastError());
    launch_mask(h->g, h->ct, h->mask, h->stream);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(h->d_count, 0, sizeof(int), h->stream));
    launch_ghost_table(h->g, h->sdf, h->ct, nullptr, 0, h->d_count, h->stream);
    CK(cudaGetLastError());
    int n = 0;
    CK(cudaMemcpyAsync(&n, h->d_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (n > h->ghost_cap) {
        if (h->ghosts) cudaFree(h->ghosts);
        h->ghosts = nullptr;
        h->ghost_cap = std::max(n, 64);
        CKA(cudaMalloc(&h->ghosts, (size_t)h->ghost_cap * sizeof(GhostInfo)));
    }
    CK(cudaMemsetAsync(h->d_count, 0, sizeof(int), h->stream));
    if (n > 0) launch_ghost_table(h->g, h->sdf, h->ct, h->ghosts, h->ghost_cap, h->d_count, h->stream);
    CK(cudaGetLastError());
    h->n_ghost = n;
    drop_graphs(h);
    return FVM_OK;
}

// Boundary conditions on the current state (both phases), set-up path.
static int apply_bc_full(fvm_handle *h) {
    CK(launch_bc_phase1(h->g, h->Un, h->mask, freestream(h->prm), h->stream));
    if (h->n_ghost > 0) {
        CK(cudaMemcpyAsync(h->buf[BUF_S], h->Un, (size_t)h->g.plane * 5 * sizeof(float), cudaMemcpyDeviceToDevice,
                           h->stream));
        GhostArgs ga{};
        ga.g = h->g;
        ga.list = h->ghosts;
        ga.n = h->n_ghost;
        ga.A = h->Un;
        ga.B1 = h->buf[BUF_S];
        ga.B2 = nullptr;
        ga.sc = h->sc;
        ga.fs = freestream(h->prm);
        ga.wall = wall(h->prm);
        CK(launch_ghost(ga, h->stream));
    }
    return FVM_OK;
}

// ------------------------------------------------------------- lifecycle
extern "C" int fvm_create(fvm_handle **out) {
    if (!out) return set_err(FVM_ERR_INVALID, "fvm_create: null out");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return set_err(FVM_ERR_CUDA, "fvm_create: no CUDA device");
    fvm_handle *h = new fvm_handle();
    cudaGetDevice(&h->device);
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, h->device);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, h->device);
    if (major != 10) {
        delete h;
        return set_err(FVM_ERR_UNSUPPORTED, "fvm_create: device sm_%d%d, this build targets sm_100a", major, minor);
    }
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return set_err(FVM_ERR_CUDA, "fvm_create: stream creation failed");
    }
    h->stream = h->own;
    fvm_params_default(&h->prm);
    fvm_ext_default(&h->ext);
    if (cudaMalloc(&h->sc, sizeof(DevScalars)) != cudaSuccess || cudaMalloc(&h->d_count, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->d_tmp, 16) != cudaSuccess || cudaMalloc(&h->d_counter, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->d_disp, sizeof(DisplayDesc)) != cudaSuccess ||
        cudaMallocHost(&h->h_sc, sizeof(DevScalars)) != cudaSuccess) {
        delete h;
        return set_err(FVM_ERR_ALLOC, "fvm_create: allocation failed");
    }
    cudaMemsetAsync(h->sc, 0, sizeof(DevScalars), h->stream);
    cudaMemsetAsync(h->d_disp, 0, sizeof(DisplayDesc), h->stream);
    cudaStreamSynchronize(h->stream);
    *out = h;
    return FVM_OK;
}

extern "C" int fvm_destroy(fvm_handle *h) {
    if (!h) return FVM_OK;
    cudaStreamSynchronize(h->stream);
    resolve_timing(h);
    free_buffers(h);
    for (auto e : h->event_pool) cudaEventDestroy(e);
    if (h->sc) cudaFree(h->sc);
    if (h->d_count) cudaFree(h->d_count);
    if (h->d_tmp) cudaFree(h->d_tmp);
    if (h->d_counter) cudaFree(h->d_counter);
    if (h->d_disp) cudaFree(h->d_disp);
    if (h->h_sc) cudaFreeHost(h->h_sc);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return FVM_OK;
}

extern "C" int fvm_set_stream(fvm_handle *h, void *stream) {
    CHECK_HANDLE(h);
    cudaStreamSynchronize(h->stream);
    h->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : h->own;
    drop_graphs(h);
    return FVM_OK;
}

static int validate(const fvm_sim_params *p, const fvm_ext *e) {
    if (!p) return set_err(FVM_ERR_INVALID, "null params");
    if (p->nx <= 0 || p->ny <= 0) return set_err(FVM_ERR_INVALID, "nx, ny must be positive (got %d, %d)", p->nx, p->ny);
    if ((long long)p->nx * p->ny > (1LL << 31) - 1) return set_err(FVM_ERR_INVALID, "grid too large");
    if (!(p->dx > 0.0f) || !(p->dy > 0.0f)) return set_err(FVM_ERR_INVALID, "dx, dy must be positive");
    if (p->obstacle_shape < 0 || p->obstacle_shape > 6) return set_err(FVM_ERR_INVALID, "unknown obstacle shape");
    if (e) {
        if (e->flux_scheme < 0 || e->flux_scheme > 1) return set_err(FVM_ERR_INVALID, "unknown flux scheme");
        if (e->limiter < 0 || e->limiter > 1) return set_err(FVM_ERR_INVALID, "unknown limiter");
        if (e->dt_policy < 0 || e->dt_policy > 1) return set_err(FVM_ERR_INVALID, "unknown dt policy");
        if (!(e->prandtl > 0.0f)) return set_err(FVM_ERR_INVALID, "prandtl must be positive");
    }
    return FVM_OK;
}

extern "C" int fvm_reset(fvm_handle *h, const fvm_sim_params *p) {
    CHECK_INIT(h);
    if (int r = validate(p, nullptr)) return r;
    if (p->nx != h->g.nx || p->ny != h->g.ny)
        return set_err(FVM_ERR_INVALID, "fvm_reset: grid %dx%d differs from the allocated %dx%d (use fvm_initialize)",
                       p->nx, p->ny, h->g.nx, h->g.ny);
    h->disp_fresh = false;
    h->prm = *p;
    h->g.dx = p->dx;
    h->g.dy = p->dy;
    k_zero_scalars<<<1, 1, 0, h->stream>>>(h->sc);
    h->launches_at_sc_copy = -1;  // the host copy of the scalars is out of date
    CK(cudaGetLastError());
    launch_init(h->g, h->Un, freestream(h->prm), h->stream);
    CK(cudaGetLastError());
    if (int r = build_geometry(h, false)) return r;
    if (int r = apply_bc_full(h)) return r;
    CK(cudaStreamSynchronize(h->stream));
    h->dt_ready = false;
    h->cfl_valid = false;
    return FVM_OK;
}

extern "C" int fvm_initialize(fvm_handle *h, const fvm_sim_params *p, const fvm_ext *ext) {
    CHECK_HANDLE(h);
    if (int r = validate(p, ext)) return r;
    if (h->disp) {  // a registered display field is sized for the old grid
        CK(launch_set_display(h->d_disp, nullptr, 0, h->stream));
        h->disp = nullptr;
    }
    h->disp_fresh = false;
    h->prm = *p;
    if (ext) h->ext = *ext;
    if (int r = alloc_buffers(h, p->nx, p->ny)) return r;
    if (int r = build_maps(h)) return r;
    return fvm_reset(h, p);
}

extern "C" int fvm_resize(fvm_handle *h, int nx, int ny) {
    CHECK_HANDLE(h);
    if (nx <= 0 || ny <= 0) return set_err(FVM_ERR_INVALID, "fvm_resize: nx, ny must be positive");
    if (h->Un && nx == h->g.nx && ny == h->g.ny) return FVM_OK;
    if (h->disp) {  // a registered display field is sized for the old grid
        CK(launch_set_display(h->d_disp, nullptr, 0, h->stream));
        h->disp = nullptr;
    }
    h->disp_fresh = false;
    h->prm.nx = nx;
    h->prm.ny = ny;
    if (int r = alloc_buffers(h, nx, ny)) return r;
    return build_maps(h);
}

extern "C" int fvm_set_ext(fvm_handle *h, const fvm_ext *ext) {
    CHECK_HANDLE(h);
    if (int r = validate(&h->prm, ext)) return r;
    if (!ext) return set_err(FVM_ERR_INVALID, "null ext");
    h->ext = *ext;
    drop_graphs(h);
    h->dt_ready = false;
    return FVM_OK;
}

extern "C" int fvm_update_obstacle(fvm_handle *h, const fvm_sim_params *p) {
    CHECK_INIT(h);
    if (int r = validate(p, nullptr)) return r;
    h->disp_fresh = false;
    h->prm = *p;
    if (int r = build_geometry(h, true)) return r;
    if (int r = apply_bc_full(h)) return r;
    h->cfl_valid = false;
    h->dt_ready = false;
    return FVM_OK;
}

// --------------------------------------------------------------- stepping
static StepArgs step_args(fvm_handle *h, float *out, int apply_bc, int cfl, float dt_scale) {
    StepArgs a{};
    a.g = h->g;
    a.out = out;
    a.mask = h->mask;
    a.sc = h->sc;
    a.fs = freestream(h->prm);
    a.wall = wall(h->prm);
    a.prandtl = h->ext.prandtl;
    a.ref_prandtl = (h->ext.prandtl == PRANDTL_REF) ? 1 : 0;
    a.rows_per_cta = h->tune.rows;
    a.apply_bc = apply_bc;
    a.cfl = cfl;
    a.dt_scale = dt_scale;
    a.pdl = 1;
    return a;
}

static GhostArgs ghost_args(fvm_handle *h, float *A, const float *B1, const float *B2, int cfl, int finalize) {
    GhostArgs ga{};
    ga.g = h->g;
    ga.list = h->ghosts;
    ga.n = h->n_ghost;
    ga.A = A;
    ga.B1 = B1;
    ga.B2 = B2;
    ga.sc = h->sc;
    ga.fs = freestream(h->prm);
    ga.wall = wall(h->prm);
    ga.cfl = cfl;
    ga.finalize = finalize;
    ga.recompute_dt = h->ext.dt_policy == FVM_DT_RECOMPUTE;
    ga.cfl_num = h->prm.cfl;
    ga.cfl_visc = h->prm.cfl_visc;
    ga.min_dx = fminf(h->prm.dx, h->prm.dy);
    ga.viscous = h->prm.enable_viscosity ? 1 : 0;
    return ga;
}

// One step's launches; leaves U^{n+1} in buf[BUF_X] (the caller swaps).
static int enqueue_step(fvm_handle *h) {
    const int sch = h->ext.flux_scheme, lim = h->ext.limiter;
    const StageTune &tn = h->tune;
    cudaStream_t st = h->stream;
    float *Un = h->buf[BUF_N], *Us = h->buf[BUF_S], *Ux = h->buf[BUF_X], *Ud = h->buf[BUF_D];
    const CUtensorMap &inN = h->tm_in[BUF_N], &inS = h->tm_in[BUF_S], &inD = h->tm_in[BUF_D];
    const CUtensorMap &ctrN = h->tm_ctr[BUF_N], &ctrD = h->tm_ctr[BUF_D];
    if (!h->prm.enable_viscosity) {
        // a marching pass followed by a ghost pass lets it launch early (its
        // few CTAs then wait on the device); a marching successor is not
        // launched early, its CTAs would spread unevenly over the SMs that
        // free up first
        StepArgs a1 = step_args(h, Us, 1, 0, 1.0f);
        a1.early_launch = 1;
        CK(timed(h, 0, [&] { return launch_stage(1, sch, lim, tn, inN, ctrN, a1, st); }));
        GhostArgs g1 = ghost_args(h, Us, Un, nullptr, 0, 0);
        CK(timed(h, 4, [&] { return launch_ghost(g1, st); }));
        StepArgs a2 = step_args(h, Ux, 1, 1, 1.0f);
        a2.disp = h->disp ? h->d_disp : nullptr;
        a2.early_launch = 1;
        CK(timed(h, 1, [&] { return launch_stage(2, sch, lim, tn, inS, ctrN, a2, st); }));
        GhostArgs g2 = ghost_args(h, Ux, Un, Us, 1, 1);
        g2.disp = h->disp ? h->d_disp : nullptr;
        CK(timed(h, 5, [&] { return launch_ghost(g2, st); }));
    } else {
        StepArgs v1 = step_args(h, Ud, 0, 0, 0.5f);
        CK(timed(h, 2, [&] { return launch_viscous(tn, inN, v1, st); }));
        StepArgs a1 = step_args(h, Us, 1, 0, 1.0f);
        a1.early_launch = 1;
        CK(timed(h, 0, [&] { return launch_stage(1, sch, lim, tn, inD, ctrD, a1, st); }));
        GhostArgs g1 = ghost_args(h, Us, Ud, nullptr, 0, 0);
        CK(timed(h, 4, [&] { return launch_ghost(g1, st); }));
        // stage 2 blends with the diffused U^n and overwrites it in place;
        // launched plainly: with programmatic serialization behind the ghost
        // pass this step ran 4 % slower at 1024x512 (the Euler stage 2 gains)
        StepArgs a2 = step_args(h, Ud, 0, 0, 1.0f);
        a2.pdl = 0;
        CK(timed(h, 1, [&] { return launch_stage(2, sch, lim, tn, inS, ctrD, a2, st); }));
        StepArgs v2 = step_args(h, Ux, 1, 2, 0.5f);
        v2.disp = h->disp ? h->d_disp : nullptr;
        v2.early_launch = 1;
        CK(timed(h, 3, [&] { return launch_viscous(tn, inD, v2, st); }));
        GhostArgs g2 = ghost_args(h, Ux, Ud, nullptr, 2, 1);
        g2.disp = h->disp ? h->d_disp : nullptr;
        CK(timed(h, 5, [&] { return launch_ghost(g2, st); }));
    }
    return FVM_OK;
}

static void swap_state(fvm_handle *h) {
    std::swap(h->buf[BUF_N], h->buf[BUF_X]);
    std::swap(h->tm_in[BUF_N], h->tm_in[BUF_X]);
    std::swap(h->tm_ctr[BUF_N], h->tm_ctr[BUF_X]);
}

// Make sc->dt hold the dt of the next step.
static int prepare_dt(fvm_handle *h, fvm_sim_params *p) {
    if (h->ext.dt_policy == FVM_DT_FIXED) {
        // the step kernels never change sc->dt under this policy: write it
        // only when the caller's dt differs from the one already there
        if (h->dt_ready && h->fixed_dt == p->dt) return FVM_OK;
        k_set_scalars<<<1, 1, 0, h->stream>>>(h->sc, p->dt, p->t_current, 0);
        CK(cudaGetLastError());
        h->launches++;
        h->fixed_dt = p->dt;
        h->dt_ready = true;
        return FVM_OK;
    }
    if (!h->dt_ready) {
        float dt = 0.0f;
        if (int r = fvm_compute_dt(h, p, &dt)) return r;
        k_set_scalars<<<1, 1, 0, h->stream>>>(h->sc, dt, p->t_current, 1);
        CK(cudaGetLastError());
        h->launches++;
        h->dt_ready = true;
    }
    return FVM_OK;
}

static unsigned long long graph_key(fvm_handle *h) {
    unsigned long long k = (unsigned long long)h->prm.enable_viscosity;
    k = k * 31 + h->ext.flux_scheme;
    k = k * 31 + h->ext.limiter;
    k = k * 131 + h->tune.nt;
    k = k * 131 + h->tune.ring;
    k = k * 1031 + h->tune.rows;
    k = k * 1000003ULL + (unsigned long long)h->n_ghost;
    k = k * 7 + h->ext.dt_policy;
    k = k * 1000003ULL + (unsigned long long)(uintptr_t)h->stream;
    k = k * 3 + (h->disp != nullptr ? 1 : 0);  // display-field variants of the last passes
    uint32_t c1, c2;
    memcpy(&c1, &h->prm.cfl, 4);
    memcpy(&c2, &h->prm.cfl_visc, 4);
    k = k * 1000003ULL + c1;
    k = k * 1000003ULL + c2;
    return k;
}

// Status of the error word in the host copy of the device scalars.
static int device_error_status(fvm_handle *h) {
    if (h->h_sc->err & kErrTimeout)
        return set_err(FVM_ERR_TIMEOUT, "a bounded device wait expired (error word 0x%x)", h->h_sc->err);
    if (h->h_sc->err & kErrSmemAlign)
        return set_err(FVM_ERR_CUDA, "shared-memory staging area not 128-byte aligned; step skipped (error word 0x%x)",
                       h->h_sc->err);
    return FVM_OK;
}

static int check_device_error(fvm_handle *h) {
    CK(cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return device_error_status(h);
}

static int finish_steps(fvm_handle *h, fvm_sim_params *p, int n) {
    if (h->ext.dt_policy == FVM_DT_FIXED) {
        for (int k = 0; k < n; k++) p->t_current += p->dt;
        p->step += n;
    } else {
        if (int r = check_device_error(h)) return r;
        p->dt = h->h_sc->dt_last;
        p->t_current = h->h_sc->t;
        p->step += n;
    }
    h->cfl_valid = true;
    return FVM_OK;
}

// Which ping-pong buffer holds U^n (0: the one that held it at the first
// captured step); the captured pointers depend on it.
static int state_parity(fvm_handle *h) {
    if (!h->parity_base) h->parity_base = h->buf[BUF_N];
    return (h->buf[BUF_N] == h->parity_base) ? 0 : 1;
}

// Captured graphs of `nsteps` steps (2 or 1) for both buffer parities, built
// together the first time either is needed (and again after a change of
// their key), so no later call pays for a capture and an instantiation.  The
// other parity's graph is captured with the state pointers swapped and
// restored afterwards; capture launches nothing.
static int ensure_graphs(fvm_handle *h, int nsteps, cudaGraphExec_t *graphs, unsigned long long *keys) {
    const int cur = state_parity(h);
    const unsigned long long key = graph_key(h);
    for (int par = 0; par < 2; par++) {
        if (graphs[par] && keys[par] == key) continue;
        if (graphs[par]) {
            cudaGraphExecDestroy(graphs[par]);
            graphs[par] = nullptr;
        }
        const bool other = par != cur;
        if (other) swap_state(h);
        cudaGraph_t gr;
        cudaError_t eb = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (eb != cudaSuccess) {
            if (other) swap_state(h);
            CK(eb);
        }
        long long before = h->launches;
        // two steps swap the state twice (also when a step fails to enqueue),
        // one step not at all: the pointers end as they began
        int r = enqueue_step(h);
        if (nsteps == 2) {
            swap_state(h);
            if (!r) r = enqueue_step(h);
            swap_state(h);
        }
        cudaError_t ec = cudaStreamEndCapture(h->stream, &gr);
        h->launches = before;
        if (other) swap_state(h);
        if (r) {
            if (ec == cudaSuccess) cudaGraphDestroy(gr);
            return r;
        }
        CK(ec);
        cudaError_t ei = cudaGraphInstantiate(&graphs[par], gr, 0);
        cudaGraphDestroy(gr);
        CK(ei);
        keys[par] = key;
    }
    return FVM_OK;
}

extern "C" int fvm_step(fvm_handle *h, fvm_sim_params *p) { return fvm_steps(h, p, 1); }

extern "C" int fvm_steps(fvm_handle *h, fvm_sim_params *p, int n) {
    CHECK_INIT(h);
    if (!p) return set_err(FVM_ERR_INVALID, "null params");
    if (n < 0) return set_err(FVM_ERR_INVALID, "negative step count");
    if (n == 0) return FVM_OK;
    h->disp_fresh = false;  // until every step is queued
    // per-step knobs the reference reads from params on every call
    h->prm.cfl = p->cfl;
    h->prm.cfl_visc = p->cfl_visc;
    h->prm.dt = p->dt;
    if (p->enable_viscosity != h->prm.enable_viscosity || p->adiabatic_wall != h->prm.adiabatic_wall ||
        p->T_wall != h->prm.T_wall) {
        h->prm.enable_viscosity = p->enable_viscosity;
        h->prm.adiabatic_wall = p->adiabatic_wall;
        h->prm.T_wall = p->T_wall;
        drop_graphs(h);
    }
    if (int r = prepare_dt(h, p)) return r;
    const bool use_graph = !h->timing && h->stream != nullptr && h->stream != cudaStreamLegacy &&
                           h->stream != cudaStreamPerThread && getenv("FVM_NO_GRAPH") == nullptr;
    int done = 0;
    if (use_graph && n >= 2) {
        const int par = state_parity(h);
        if (int r = ensure_graphs(h, 2, h->graph, h->graph_key)) return r;
        const int per_step = h->prm.enable_viscosity ? 6 : 4;
        for (; done + 2 <= n; done += 2) {
            CK(cudaGraphLaunch(h->graph[par], h->stream));
            h->launches += 2 * per_step;
        }
    }
    if (use_graph && done < n) {
        // one remaining step: a captured single step for this buffer parity
        const int par = state_parity(h);
        if (int r = ensure_graphs(h, 1, h->graph1, h->graph1_key)) return r;
        CK(cudaGraphLaunch(h->graph1[par], h->stream));
        h->launches += h->prm.enable_viscosity ? 6 : 4;
        swap_state(h);
        done++;
    }
    for (; done < n; done++) {
        if (int r = enqueue_step(h)) return r;
        swap_state(h);
    }
    const int rf = finish_steps(h, p, n);
    h->disp_fresh = rf == FVM_OK && h->disp != nullptr;
    return rf;
}

extern "C" int fvm_synchronize(fvm_handle *h) {
    CHECK_HANDLE(h);
    CK(cudaStreamSynchronize(h->stream));
    resolve_timing(h);
    // only kernels set the error word: when none was launched since
    // fvm_queue_dt copied the device scalars (the reference's per-frame
    // queue / synchronize / read sequence), that copy, complete now, holds it
    if (h->launches == h->launches_at_sc_copy) return device_error_status(h);
    return check_device_error(h);
}

// CFL maxima of the current state: after a step they come from the fused
// reduction (mu of the last viscous half step, as the reference's d_mu_);
// otherwise from a standalone pass over the state.
static int cfl_maxima(fvm_handle *h, float *ms, float *mn) {
    if (!h->cfl_valid) {
        CK(launch_cfl_state(h->g, h->Un, h->mask, h->sc, h->stream));
        h->launches += 2;
        h->cfl_valid = true;
    }
    CK(cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *ms = h->h_sc->cfl[0];
    *mn = h->h_sc->cfl[1];
    return FVM_OK;
}

// readTimeStepResult (src/solver.cu:3250-3265)
static float dt_from_maxima(const fvm_sim_params *p, float max_speed, float max_nu) {
    float min_dx = fminf(p->dx, p->dy);
    float dt = p->cfl * min_dx / (max_speed + 1e-10f);
    if (p->enable_viscosity) {
        float dt_visc = p->cfl_visc * min_dx * min_dx / (max_nu + 1e-10f);
        dt = fminf(dt, dt_visc);
    }
    return dt;
}

extern "C" int fvm_compute_dt(fvm_handle *h, const fvm_sim_params *p, float *dt_out) {
    CHECK_INIT(h);
    if (!p || !dt_out) return set_err(FVM_ERR_INVALID, "null argument");
    float ms = 0.0f, mn = 0.0f;
    if (int r = cfl_maxima(h, &ms, &mn)) return r;
    *dt_out = dt_from_maxima(p, ms, mn);
    return FVM_OK;
}

extern "C" int fvm_queue_dt(fvm_handle *h, const fvm_sim_params *p) {
    CHECK_INIT(h);
    if (!p) return set_err(FVM_ERR_INVALID, "null params");
    if (!h->cfl_valid) {
        CK(launch_cfl_state(h->g, h->Un, h->mask, h->sc, h->stream));
        h->launches += 2;
        h->cfl_valid = true;
    }
    CK(cudaMemcpyAsync(h->h_sc, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->stream));
    h->launches_at_sc_copy = h->launches;
    return FVM_OK;
}

extern "C" int fvm_read_dt(fvm_handle *h, const fvm_sim_params *p, float *dt_out) {
    CHECK_INIT(h);
    if (!p || !dt_out) return set_err(FVM_ERR_INVALID, "null argument");
    *dt_out = dt_from_maxima(p, h->h_sc->cfl[0], h->h_sc->cfl[1]);
    return FVM_OK;
}

// --------------------------------------------------------------- readback
extern "C" int fvm_get_cell_types(fvm_handle *h, uint8_t *host_types) {
    CHECK_INIT(h);
    if (!host_types) return set_err(FVM_ERR_INVALID, "null buffer");
    CK(cudaMemcpyAsync(host_types, h->ct, (size_t)h->g.nx * h->g.ny, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

extern "C" int fvm_get_sdf(fvm_handle *h, float *host_sdf) {
    CHECK_INIT(h);
    if (!host_sdf) return set_err(FVM_ERR_INVALID, "null buffer");
    CK(cudaMemcpy2DAsync(host_sdf, (size_t)h->g.nx * 4, h->sdf, (size_t)h->g.pitch * 4, (size_t)h->g.nx * 4, h->g.ny,
                         cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

extern "C" int fvm_read_fields(fvm_handle *h, float *rho, float *rho_u, float *rho_v, float *E, float *rho_e) {
    CHECK_INIT(h);
    float *dst[5] = {rho, rho_u, rho_v, E, rho_e};
    for (int k = 0; k < 5; k++) {
        if (!dst[k]) continue;
        CK(cudaMemcpy2DAsync(dst[k], (size_t)h->g.nx * 4, h->Un + (size_t)k * h->g.plane, (size_t)h->g.pitch * 4,
                             (size_t)h->g.nx * 4, h->g.ny, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

static int check_region(const fvm_handle *h, int i0, int j0, int w, int hgt) {
    if (i0 < 0 || j0 < 0 || w <= 0 || hgt <= 0 || (long long)i0 + w > h->g.nx || (long long)j0 + hgt > h->g.ny)
        return set_err(FVM_ERR_INVALID, "region [%d, %d) x [%d, %d) outside the %d x %d grid", i0, i0 + w, j0, j0 + hgt,
                       h->g.nx, h->g.ny);
    return FVM_OK;
}

extern "C" int fvm_read_region(fvm_handle *h, int i0, int j0, int w, int hgt, float *rho, float *rho_u,
                               float *rho_v, float *E, float *rho_e) {
    CHECK_INIT(h);
    if (int r = check_region(h, i0, j0, w, hgt)) return r;
    float *dst[5] = {rho, rho_u, rho_v, E, rho_e};
    const size_t off = (size_t)j0 * h->g.pitch + i0;
    for (int k = 0; k < 5; k++) {
        if (!dst[k]) continue;
        CK(cudaMemcpy2DAsync(dst[k], (size_t)w * 4, h->Un + (size_t)k * h->g.plane + off, (size_t)h->g.pitch * 4,
                             (size_t)w * 4, hgt, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

extern "C" int fvm_read_region_geometry(fvm_handle *h, int i0, int j0, int w, int hgt, float *sdf,
                                        uint8_t *cell_types) {
    CHECK_INIT(h);
    if (int r = check_region(h, i0, j0, w, hgt)) return r;
    if (sdf)
        CK(cudaMemcpy2DAsync(sdf, (size_t)w * 4, h->sdf + (size_t)j0 * h->g.pitch + i0, (size_t)h->g.pitch * 4,
                             (size_t)w * 4, hgt, cudaMemcpyDeviceToHost, h->stream));
    if (cell_types)
        CK(cudaMemcpy2DAsync(cell_types, (size_t)w, h->ct + (size_t)j0 * h->g.nx + i0, (size_t)h->g.nx, (size_t)w,
                             hgt, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

extern "C" int fvm_write_fields(fvm_handle *h, const float *rho, const float *rho_u, const float *rho_v,
                                const float *E, const float *rho_e) {
    CHECK_INIT(h);
    h->disp_fresh = false;
    const float *src[5] = {rho, rho_u, rho_v, E, rho_e};
    for (int k = 0; k < 5; k++) {
        if (!src[k]) continue;
        CK(cudaMemcpy2DAsync(h->Un + (size_t)k * h->g.plane, (size_t)h->g.pitch * 4, src[k], (size_t)h->g.nx * 4,
                             (size_t)h->g.nx * 4, h->g.ny, cudaMemcpyHostToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    h->cfl_valid = false;
    h->dt_ready = false;
    return FVM_OK;
}

extern "C" int fvm_read_primitives(fvm_handle *h, float *u, float *v, float *p, float *T) {
    CHECK_INIT(h);
    const size_t n = (size_t)h->g.nx * h->g.ny;
    float *d = nullptr;
    CKA(cudaMallocAsync(&d, n * 4 * sizeof(float), h->stream));
    CK(launch_primitives(h->g, h->Un, d, d + n, d + 2 * n, d + 3 * n, h->stream));
    h->launches++;
    float *dst[4] = {u, v, p, T};
    for (int k = 0; k < 4; k++)
        if (dst[k]) CK(cudaMemcpyAsync(dst[k], d + k * n, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaFreeAsync(d, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

extern "C" int fvm_field_to_device(fvm_handle *h, int kind, float *dev_dst) {
    CHECK_INIT(h);
    if (!dev_dst) return set_err(FVM_ERR_INVALID, "null destination");
    if (kind < 0 || kind > 4) return set_err(FVM_ERR_INVALID, "unknown field kind %d", kind);
    const bool into_display = h->disp && dev_dst == h->disp;
    // the registered display field, already written by the last step
    if (into_display && kind == h->disp_kind && h->disp_fresh) return FVM_OK;
    CK(launch_derived(kind, h->g, h->Un, dev_dst, h->stream));
    h->launches++;
    if (into_display) h->disp_fresh = kind == h->disp_kind;
    return FVM_OK;
}

extern "C" int fvm_set_display_field(fvm_handle *h, int kind, float *dev_dst) {
    CHECK_INIT(h);
    if (dev_dst && (kind < 0 || kind > 4)) return set_err(FVM_ERR_INVALID, "unknown field kind %d", kind);
    if (dev_dst == h->disp && (!dev_dst || kind == h->disp_kind)) return FVM_OK;
    // the descriptor is updated in stream order, before the next step reads it
    CK(launch_set_display(h->d_disp, dev_dst, dev_dst ? kind : 0, h->stream));
    h->launches++;
    h->disp = dev_dst;
    h->disp_kind = dev_dst ? kind : 0;
    h->disp_fresh = false;
    return FVM_OK;
}

extern "C" int fvm_cell_types_to_device(fvm_handle *h, float *dev_dst) {
    CHECK_INIT(h);
    if (!dev_dst) return set_err(FVM_ERR_INVALID, "null destination");
    CK(launch_ct_to_float(h->g, h->ct, dev_dst, h->stream));
    h->launches++;
    return FVM_OK;
}

extern "C" int fvm_vector_arrows(fvm_handle *h, float *dev_vertex_data, int max_vertices, int step, float u_inf,
                                 float max_arrow_length, float arrow_head_angle, float arrow_head_length,
                                 int *n_vertices_out) {
    CHECK_INIT(h);
    if (!dev_vertex_data || !n_vertices_out || step <= 0 || max_vertices < 0)
        return set_err(FVM_ERR_INVALID, "fvm_vector_arrows: bad argument");
    CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), h->stream));
    CK(launch_arrows_cap(h->g, h->Un, dev_vertex_data, max_vertices, h->d_counter, step, u_inf, max_arrow_length,
                         arrow_head_angle, arrow_head_length, h->stream));
    h->launches++;
    int n = 0;
    CK(cudaMemcpyAsync(&n, h->d_counter, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n_vertices_out = n;
    return FVM_OK;
}

// ------------------------------------------------------------------ stats
static int max_reduce(fvm_handle *h, int what, float *out) {
    CHECK_INIT(h);
    if (!out) return set_err(FVM_ERR_INVALID, "null output");
    CK(cudaMemsetAsync(h->d_tmp, 0, sizeof(float), h->stream));
    CK(launch_max_reduce(what, h->g, h->Un, h->d_tmp, h->stream));
    h->launches++;
    CK(cudaMemcpyAsync(out, h->d_tmp, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}
extern "C" int fvm_max_temperature(fvm_handle *h, float *out) { return max_reduce(h, 0, out); }
extern "C" int fvm_max_mach(fvm_handle *h, float *out) { return max_reduce(h, 1, out); }

extern "C" int fvm_memory_usage(fvm_handle *h, size_t *bytes) {
    CHECK_HANDLE(h);
    if (!bytes) return set_err(FVM_ERR_INVALID, "null output");
    *bytes = h->bytes + (size_t)h->ghost_cap * sizeof(GhostInfo) + sizeof(DevScalars);
    return FVM_OK;
}

extern "C" int fvm_gpu_mem_info(size_t *free_bytes, size_t *total_bytes) {
    if (!free_bytes || !total_bytes) return set_err(FVM_ERR_INVALID, "null output");
    CK(cudaMemGetInfo(free_bytes, total_bytes));
    return FVM_OK;
}

extern "C" int fvm_diagnostics(fvm_handle *h, fvm_diag *out) {
    CHECK_INIT(h);
    if (!out) return set_err(FVM_ERR_INVALID, "null output");
    double *parts = h->d_diag, *fin = h->d_diag + (size_t)h->diag_parts * 8;
    CK(launch_diagnostics(h->g, h->Un, h->ct, h->mask, h->prm.enable_viscosity ? 1 : 0, h->ext.prandtl,
                          h->ext.prandtl == PRANDTL_REF, parts, h->diag_parts, fin, h->stream));
    h->launches += 2;
    double r[8];
    CK(cudaMemcpyAsync(r, fin, sizeof r, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    memset(out, 0, sizeof(*out));
    out->force_x = r[0];
    out->force_y = r[1];
    const double q_inf = 0.5 * (double)h->prm.rho_inf * (double)h->prm.u_inf * (double)h->prm.u_inf;
    const double L = h->ext.ref_length > 0 ? (double)h->ext.ref_length : 2.0 * (double)h->prm.obstacle_r;
    out->cd = (q_inf > 0 && L > 0) ? r[0] / (q_inf * L) : 0.0;
    out->cl = (q_inf > 0 && L > 0) ? r[1] / (q_inf * L) : 0.0;
    out->mass = r[2];
    out->mom_x = r[3];
    out->mom_y = r[4];
    out->energy = r[5];
    out->wall_heat = r[6];
    out->wall_heat_max = r[7];
    return FVM_OK;
}

extern "C" int fvm_shock_standoff(fvm_handle *h, double *standoff_out) {
    CHECK_INIT(h);
    if (!standoff_out) return set_err(FVM_ERR_INVALID, "null output");
    const double g = 1.4, pinf = h->prm.p_inf;
    const double cinf = std::sqrt(g * pinf / (double)h->prm.rho_inf);
    const double M = (double)h->prm.u_inf / cinf;
    if (!(M > 1.0)) {
        *standoff_out = NAN;
        return FVM_OK;
    }
    const double p2 = pinf * (1.0 + 2.0 * g / (g + 1.0) * (M * M - 1.0));
    double *dout = h->d_diag + (size_t)h->diag_parts * 8 + 8;
    CK(launch_standoff(h->g, h->Un, h->sdf, pinf + 0.5 * (p2 - pinf), dout, h->stream));
    h->launches++;
    CK(cudaMemcpyAsync(standoff_out, dout, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return FVM_OK;
}

// ------------------------------------------------------------ measurement
extern "C" int fvm_set_kernel_timing(fvm_handle *h, int enable) {
    CHECK_HANDLE(h);
    resolve_timing(h);
    h->timing = enable != 0;
    h->ktimes.clear();
    return FVM_OK;
}

extern "C" int fvm_kernel_times(fvm_handle *h, fvm_kernel_time *out, int cap, int *count_out) {
    CHECK_HANDLE(h);
    resolve_timing(h);
    int n = 0;
    for (auto &kv : h->ktimes) {
        if (out && n < cap) {
            memset(&out[n], 0, sizeof(out[n]));
            snprintf(out[n].name, sizeof(out[n].name), "%s", kv.first.c_str());
            out[n].launches = kv.second.first;
            out[n].total_ms = kv.second.second;
        }
        n++;
    }
    if (count_out) *count_out = n;
    return FVM_OK;
}

extern "C" int fvm_launch_count(fvm_handle *h, long long *count_out) {
    CHECK_HANDLE(h);
    if (!count_out) return set_err(FVM_ERR_INVALID, "null output");
    *count_out = h->launches;
    return FVM_OK;
}

// Time each candidate tuning over `steps` steps from a snapshot of the
// current state (restored after every candidate) and keep the fastest.
extern "C" int fvm_autotune(fvm_handle *h, const fvm_sim_params *p, int steps, float *best_ms_out) {
    CHECK_INIT(h);
    if (!p || steps < 2) return set_err(FVM_ERR_INVALID, "fvm_autotune: need params and steps >= 2");
    const size_t bytes = (size_t)h->g.plane * 5 * sizeof(float);
    float *snap = nullptr;
    CKA(cudaMalloc(&snap, bytes));
    CK(cudaMemcpyAsync(snap, h->buf[BUF_N], bytes, cudaMemcpyDeviceToDevice, h->stream));
    const StageTune before = h->tune;
    const bool timing = h->timing;
    h->timing = false;
    fvm_sim_params q = *p;
    StageTune best = before;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = FVM_OK;
    // tile heights between the powers of two let the tuner fill the last
    // wave of CTAs (e.g. 8192x4096: 64-row tiles are 4.83 waves on 148 SMs)
    constexpr int kRows = 13;
    const int nts[2] = {128, 256}, rings[2] = {4, 6},
              rows[kRows] = {4, 8, 16, 24, 32, 40, 48, 56, 64, 80, 96, 128, 256};
    for (int a1 = 0; a1 < 2 && rc == FVM_OK; a1++)
        for (int a2 = 0; a2 < 2 && rc == FVM_OK; a2++)
            for (int a3 = 0; a3 < kRows && rc == FVM_OK; a3++) {
                StageTune cand{nts[a1], rings[a2], rows[a3]};
                if (rows[a3] > std::max(16, h->g.ny)) continue;
                h->tune = cand;
                drop_graphs(h);
                if ((rc = build_maps(h)) != FVM_OK) break;
                fvm_sim_params w = q;
                if ((rc = fvm_steps(h, &w, 3)) != FVM_OK) break;  // warm (captures both graph kinds)
                cudaEventRecord(e0, h->stream);
                if ((rc = fvm_steps(h, &w, steps)) != FVM_OK) break;
                cudaEventRecord(e1, h->stream);
                cudaEventSynchronize(e1);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= steps;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = cand;
                }
                // restore the state for the next candidate (buffer roles may have swapped)
                cudaMemcpyAsync(h->buf[BUF_N], snap, bytes, cudaMemcpyDeviceToDevice, h->stream);
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->tune = (rc == FVM_OK) ? best : before;
    drop_graphs(h);
    int r2 = build_maps(h);
    cudaMemcpyAsync(h->buf[BUF_N], snap, bytes, cudaMemcpyDeviceToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaFree(snap);
    h->timing = timing;
    h->cfl_valid = false;
    h->dt_ready = false;
    h->disp_fresh = false;  // the tuning steps wrote it; the state is restored
    if (rc != FVM_OK) return rc;
    if (r2 != FVM_OK) return r2;
    g_tune_cache[TuneKey{h->g.nx, h->g.ny, h->prm.enable_viscosity ? 1 : 0, h->ext.flux_scheme, h->ext.limiter}] =
        best;
    if (best_ms_out) *best_ms_out = best_ms;
    return FVM_OK;
}

extern "C" int fvm_set_tune(fvm_handle *h, int nt, int ring, int rows) {
    CHECK_INIT(h);
    if (!(nt == 128 || nt == 256) || !(ring == 4 || ring == 6) || rows < 4 || rows > 65536 || (rows & 1))
        return set_err(FVM_ERR_INVALID,
                       "fvm_set_tune: threads 128 or 256, ring 4 or 6, even rows 4..65536 (got %d, %d, %d)", nt, ring,
                       rows);
    h->tune = StageTune{nt, ring, rows};
    drop_graphs(h);
    return build_maps(h);
}

extern "C" int fvm_nonfinite_count(fvm_handle *h, unsigned long long *count, int reset) {
    CHECK_INIT(h);
    unsigned v = 0;
    CK(cudaMemcpyAsync(&v, &h->sc->nonfinite, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    if (reset) CK(cudaMemsetAsync(&h->sc->nonfinite, 0, sizeof(unsigned), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (count) *count = v;
    return FVM_OK;
}

extern "C" int fvm_get_tune(fvm_handle *h, int *nt, int *ring, int *rows) {
    CHECK_INIT(h);
    if (nt) *nt = h->tune.nt;
    if (ring) *ring = h->tune.ring;
    if (rows) *rows = h->tune.rows;
    return FVM_OK;
}

extern "C" int fvm_debug_stage1(fvm_handle *h, float dt, int with_ghost, float *rho, float *rho_u, float *rho_v,
                                float *E, float *rho_e) {
    CHECK_INIT(h);
    k_set_scalars<<<1, 1, 0, h->stream>>>(h->sc, dt, 0.0f, 0);
    h->launches_at_sc_copy = -1;
    CK(cudaGetLastError());
    float *Un = h->buf[BUF_N], *Us = h->buf[BUF_S];
    StepArgs a1 = step_args(h, Us, 1, 0, 1.0f);
    CK(launch_stage(1, h->ext.flux_scheme, h->ext.limiter, h->tune, h->tm_in[BUF_N], h->tm_ctr[BUF_N], a1, h->stream));
    if (with_ghost && h->n_ghost > 0) {
        GhostArgs g1 = ghost_args(h, Us, Un, nullptr, 0, 0);
        CK(launch_ghost(g1, h->stream));
    }
    float *dst[5] = {rho, rho_u, rho_v, E, rho_e};
    for (int k = 0; k < 5; k++)
        if (dst[k])
            CK(cudaMemcpy2DAsync(dst[k], (size_t)h->g.nx * 4, Us + (size_t)k * h->g.plane, (size_t)h->g.pitch * 4,
                                 (size_t)h->g.nx * 4, h->g.ny, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->dt_ready = false;
    return check_device_error(h);
}

int fvm_internal_build_maps(fvm_handle *h) { return build_maps(h); }
int fvm_internal_compute_dt(fvm_handle *h, const fvm_sim_params *p, float *dt) { return fvm_compute_dt(h, p, dt); }
int fvm_internal_set_error(int code, const char *msg) { return set_err(code, "%s", msg); }

extern "C" int fvm_debug_wait_timeout(fvm_handle *h, long long limit_cycles) {
    CHECK_INIT(h);
    if (limit_cycles <= 0 || limit_cycles > kWaitCycles)
        return set_err(FVM_ERR_INVALID, "fvm_debug_wait_timeout: limit must be in 1..%lld cycles", kWaitCycles);
    CK(cudaStreamSynchronize(h->stream));
    CK(launch_wait_probe(h->sc, limit_cycles, h->stream));
    const int r = check_device_error(h);
    // clear the error word the probe set, so the solve goes on
    unsigned zero = 0;
    CK(cudaMemcpyAsync(&h->sc->err, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->launches_at_sc_copy = -1;
    return r;
}

extern "C" int fvm_debug_ghost_table(fvm_handle *h, int *out, int cap, int *count_out) {
    CHECK_INIT(h);
    static_assert(sizeof(GhostInfo) == 6 * sizeof(int), "GhostInfo layout");
    if (count_out) *count_out = h->n_ghost;
    int n = std::min(cap, h->n_ghost);
    if (out && n > 0) {
        std::vector<GhostInfo> t((size_t)n);
        CK(cudaMemcpy(t.data(), h->ghosts, (size_t)n * sizeof(GhostInfo), cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; k++) {
            int *o = out + (size_t)k * 7;
            o[0] = (int)((long long)t[k].j * h->g.pitch + t[k].i);
            memcpy(o + 1, &t[k], sizeof(GhostInfo));
        }
    }
    return FVM_OK;
}

extern "C" const char *fvm_build_info(void) {
    return "fvm_b200: sm_100a, nvcc " FVM_STR(__CUDACC_VER_MAJOR__) "." FVM_STR(__CUDACC_VER_MINOR__)
           ", --use_fast_math, marching TMA stage kernels";
}
