// The batched ensemble behind glz_ens_* in include/glazier_gpu.h.
//
// Independent replicas of the plain sweep (contact, volume and surface terms;
// lattices of any even sides, each with its own parameters and seed) share
// flat device arrays and run as one persistent launch per colour over every
// replica's tiles. One Monte Carlo step (the colour launches and a one-thread
// clock advance) is captured once into a CUDA graph and replayed; the kernels
// read the step and pass counters from the device clock, so the same graph
// serves every step. A replica's results are bit-identical to a plain
// glz_gpu_* run of the same start, whatever the schedule, so the autotuner
// chooses the persistent grid and the order replicas' tiles are dealt in by
// time alone.
//
// Replicas whose models state other terms (fields, length, connectivity,
// division, death, motility, drift, nematic) are engines of their own. When
// their steps replay from captured graphs (the direct kernel's engines: the
// engine clock makes one captured step serve every step), the batch's step
// and every engine's step are child graphs of one graph, replayed once per
// MCS; otherwise each engine steps on its own stream from a host thread.
//
// No reference counterpart: glazier runs one lattice per GpuSimulation.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/glazier_gpu.h"
#include "device.cuh"
#include "engine.h"

namespace glz {
int sweep_box(int dim, uint32_t box[3]);
}

namespace {

int fail(int code, const std::string &msg) {
    glz::set_last_error(msg);
    return code;
}

#define CU(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return fail(GLZ_DRIVER, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

double at(const double *p, size_t i) { return p ? p[i] : 0.0; }

int offsets_for(int order, int depth, int out[26][3]) {
    static const int O1[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    static const int O2[18][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                                  {1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1}, {1, 0, -1},
                                  {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
    int all[26][3];
    int k = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (dx || dy || dz) {
                    all[k][0] = dx;
                    all[k][1] = dy;
                    all[k][2] = dz;
                    ++k;
                }
    int n = 0;
    if (depth > 1) {
        if (order == 1) {
            std::memcpy(out, O1, sizeof O1);
            return 6;
        }
        if (order == 2) {
            std::memcpy(out, O2, sizeof O2);
            return 18;
        }
        std::memcpy(out, all, sizeof all);
        return 26;
    }
    if (order >= 2) {
        for (int i = 0; i < 26; ++i)
            if (all[i][2] == 0) std::memcpy(out[n++], all[i], sizeof all[i]);
        return n;
    }
    for (int i = 0; i < 6; ++i)
        if (O1[i][2] == 0) std::memcpy(out[n++], O1[i], sizeof O1[i]);
    return n;
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

struct Replica {
    glz::Geometry g{};
    long long label_off = 0, cell_off = 0;
    size_t n_labels = 0;
    int tiles = 0;
    uint64_t seed = 0;
    std::vector<uint8_t> cell_type;
};

template <typename T>
int dev_alloc(T **p, size_t n) {
    CU(cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)));
    return GLZ_OK;
}

}  // namespace

struct glz_ens {
    int n = 0, dim = 2, n_off = 8, ncol = 4;
    bool uniform = false;
    cudaStream_t stream = nullptr;
    std::vector<Replica> reps;
    long long total_sites = 0, total_cells = 0;
    uint32_t *labels = nullptr;
    uint8_t *cell_type = nullptr;
    int2 *vs_base[2] = {};
    long long *vs_delta[3] = {};
    int *volc = nullptr;
    int *anchor = nullptr;
    float *tables = nullptr;  // per replica: contact, tv, lv, ts, ls
    uint8_t *connected = nullptr;
    glz::EnsembleReplica *d_reps = nullptr;
    CUtensorMap *d_maps = nullptr;
    int *d_prefix = nullptr, *d_order = nullptr;
    glz::EnsembleClock *d_clock = nullptr;
    int *error_flag = nullptr;
    unsigned long long *medium = nullptr;
    bool use_tma = false;
    int total_tiles = 0;
    long long step = 0, pass = 0;
    int max_ctas = 0;  // 0: one full wave
    int schedule = 0;  // 0: replicas in their own order; 1: largest first
    int tile_shape = 0;  // EnsembleLaunch::tile_shape
    int one_launch = 0;  // EnsembleLaunch::one_launch
    unsigned *d_barrier = nullptr;
    int window_tiles = 0;  // all replicas' tiles of the windowed kernel
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // Replicas as the caller numbered them: slot[i] >= 0 is replica i's index
    // in the batch above (n of them), slot[i] < 0 engine -slot[i] - 1, a
    // replica whose model states more than contact, volume and surface,
    // stepped as its own engine beside the batch.
    int all = 0, device = 0;
    std::vector<int> slot;
    std::vector<glz_gpu *> engines;
    // The batch's step and every engine replica's clocked step as child
    // graphs of one graph, replayed once per MCS; the array versions of the
    // engines' steps it holds.
    cudaGraphExec_t mixed = nullptr;
    std::vector<uint64_t> versions;
};

namespace {

void drop_mixed(glz_ens *h) {
    if (h->mixed) cudaGraphExecDestroy(h->mixed);
    h->mixed = nullptr;
}

void drop_graph(glz_ens *h) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->exec = nullptr;
    h->graph = nullptr;
    drop_mixed(h);
}

// A replica's tiles under a tile shape: the windowed kernel's, or the
// direct blocks' over its targets.
int tiles_of(const glz_ens *h, const Replica &rep, int shape) {
    if (shape == 0) return rep.tiles;
    int bx, by;
    glz::ensemble_tile(shape, bx, by);
    return ((rep.g.w / 2 + bx - 1) / bx) * ((rep.g.h / 2 + by - 1) / by);
}

// Lay the replicas' tiles out in schedule order (`schedule` bit 0: largest
// first; bits 1-2: the tile shape) and upload the order.
int set_schedule(glz_ens *h, int schedule, int max_ctas) {
    const int shape = (schedule >> 1) & 3, one = (schedule >> 3) & 1;
    if (shape > 0 && h->dim != 2) return fail(GLZ_INVALID, "the direct tile shapes are for planes");
    if (one && shape == 0) return fail(GLZ_INVALID, "one launch per step is a schedule of the direct tile shapes");
    std::vector<int> order(h->n);
    std::iota(order.begin(), order.end(), 0);
    if (schedule & 1)
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return h->reps[a].tiles > h->reps[b].tiles; });
    std::vector<int> prefix(h->n + 1, 0);
    for (int i = 0; i < h->n; ++i) prefix[i + 1] = prefix[i] + tiles_of(h, h->reps[order[i]], shape);
    h->total_tiles = prefix[h->n];
    h->tile_shape = shape;
    h->one_launch = one;
    CU(cudaMemcpyAsync(h->d_order, order.data(), h->n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->d_prefix, prefix.data(), (h->n + 1) * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->schedule = schedule;
    h->max_ctas = max_ctas;
    drop_graph(h);
    return GLZ_OK;
}

glz::EnsembleLaunch launch_of(glz_ens *h, int colour) {
    glz::EnsembleLaunch e{};
    e.n = h->n;
    e.total_tiles = h->total_tiles;
    e.tile_shape = h->tile_shape;
    e.one_launch = h->one_launch;
    e.barrier = h->d_barrier;
    e.colour = colour;
    e.max_ctas = h->max_ctas;
    e.replicas = h->d_reps;
    e.maps = h->use_tma ? h->d_maps : nullptr;
    e.tile_prefix = h->d_prefix;
    e.order = h->d_order;
    e.clock = h->d_clock;
    for (int k = 0; k < 2; ++k) e.vs_base[k] = h->vs_base[k];
    for (int k = 0; k < 3; ++k) e.vs_delta[k] = h->vs_delta[k];
    e.total_cells = h->total_cells;
    e.ncol = h->ncol;
    e.error_flag = h->error_flag;
    return e;
}

// One Monte Carlo step of every replica: the colour launches and the clock.
int enqueue_step(glz_ens *h) {
    if (h->one_launch)
        CU(glz::launch_ensemble_sweep(launch_of(h, 0), h->dim, h->n_off, h->uniform, h->stream));
    else
        for (int c = 0; c < h->ncol; ++c)
            CU(glz::launch_ensemble_sweep(launch_of(h, c), h->dim, h->n_off, h->uniform, h->stream));
    CU(glz::launch_clock_advance(h->d_clock, h->ncol, h->stream));
    return GLZ_OK;
}

int build_graph(glz_ens *h) {
    if (h->exec) return GLZ_OK;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(h);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("graph capture: ") + cudaGetErrorString(e));
    h->graph = g;
    CU(cudaGraphInstantiate(&h->exec, g, 0));
    return GLZ_OK;
}

int run(glz_ens *h, uint64_t steps, bool graph, double *ms) {
    if (graph)
        if (int rc = build_graph(h)) return rc;
    cudaEvent_t a = nullptr, b = nullptr;
    if (ms) {
        CU(cudaEventCreate(&a));
        CU(cudaEventCreate(&b));
        CU(cudaEventRecord(a, h->stream));
    }
    for (uint64_t s = 0; s < steps; ++s) {
        if (graph)
            CU(cudaGraphLaunch(h->exec, h->stream));
        else if (int rc = enqueue_step(h))
            return rc;
        h->step += 1;
        h->pass += h->ncol;
    }
    if (ms) {
        CU(cudaEventRecord(b, h->stream));
        CU(cudaEventSynchronize(b));
        float t = 0.0f;
        CU(cudaEventElapsedTime(&t, a, b));
        *ms = t;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    CU(cudaStreamSynchronize(h->stream));
    int flag = 0;
    CU(cudaMemcpy(&flag, h->error_flag, sizeof flag, cudaMemcpyDeviceToHost));
    if (flag) return fail(GLZ_DRIVER, "an ensemble sweep tile reported an error (flag " + std::to_string(flag) + ")");
    return GLZ_OK;
}

int settle_all(glz_ens *h) {
    const long long p = h->pass;
    CU(glz::launch_settle(h->vs_base[p % 2], h->vs_delta[(p + 2) % 3], nullptr, nullptr, 0, (int)h->total_cells, 0, nullptr,
                          h->stream));
    return GLZ_OK;
}

}  // namespace

extern "C" {

// The batch: replicas whose models price contact, volume and surface only.
static int create_batched(int n, const glz_model *models, const uint32_t *const *labels,
                          const uint8_t *const *cell_types, const size_t *n_labels, glz_ens **out) {
    if (!out) return fail(GLZ_INVALID, "null output handle");
    *out = nullptr;
    if (n < 1 || !models || !labels || !cell_types || !n_labels) return fail(GLZ_INVALID, "no replicas or a null array");
    glz_ens *h = new glz_ens();
    auto bail = [&](int rc) {
        glz_ens_destroy(h);
        return rc;
    };
    h->n = n;
    h->reps.resize(n);
    bool uniform = true, exact = true;
    for (int r = 0; r < n; ++r) {
        const glz_model &m = models[r];
        const int w = m.width, hh = m.height, d = m.depth;
        if (w <= 0 || hh <= 0 || d <= 0) return bail(fail(GLZ_INVALID, "a replica has a zero dimension"));
        if (w % 2 || hh % 2 || (d > 1 && d % 2)) {
            char msg[160];
            std::snprintf(msg, sizeof msg,
                          "the checkerboard split needs even sides; replica %d is %d by %d by %d", r, w, hh, d);
            return bail(fail(GLZ_ODD_LATTICE, msg));
        }
        if (!labels[r] || !cell_types[r] || n_labels[r] < 1 || !m.contact || m.n_types < 1 || m.n_types > 255)
            return bail(fail(GLZ_INVALID, "replica " + std::to_string(r) + ": missing start or contact matrix"));
        if (!(m.temperature > 0.0)) return bail(fail(GLZ_INVALID, "the temperature must be positive"));
        bool extra = m.n_species > 0;
        for (int k = 0; k < m.n_types; ++k) {
            extra |= at(m.lambda_length, k) != 0.0 || at(m.division_volume, k) > 0.0 || at(m.death_rate, k) > 0.0;
            extra |= m.connected && m.connected[k];
            extra |= at(m.lambda_activity, k) != 0.0 || (m.nematic && at(m.lambda_nematic, k) != 0.0);
            for (int a = 0; a < 3; ++a) extra |= at(m.external, 3 * (size_t)k + a) != 0.0;
        }
        if (extra)
            return bail(fail(GLZ_UNSUPPORTED, "the ensemble runs contact, volume and surface terms only; replica " +
                                                  std::to_string(r) + " states more"));
        Replica &rep = h->reps[r];
        glz::Geometry &g = rep.g;
        g.w = w;
        g.h = hh;
        g.d = d;
        g.dim = d > 1 ? 3 : 2;
        g.ncol = g.dim == 3 ? 8 : 4;
        g.sites = w * hh * d;
        g.nm = g.dim == 3 ? 9 : 5;
        glz::set_dividers(g);
        g.n_off = offsets_for(m.neighbour_order, d, g.off);
        if (r == 0) {
            h->dim = g.dim;
            h->n_off = g.n_off;
            h->ncol = g.ncol;
        } else if (g.dim != h->dim || g.n_off != h->n_off) {
            return bail(fail(GLZ_INVALID, "every replica of an ensemble shares one neighbourhood"));
        }
        rep.n_labels = n_labels[r];
        rep.seed = m.seed;
        rep.cell_type.assign(cell_types[r], cell_types[r] + n_labels[r]);
        for (long long i = 0; i < g.sites; ++i)
            if (labels[r][i] >= n_labels[r])
                return bail(fail(GLZ_INVALID, "replica " + std::to_string(r) + ": a label past its type table"));
        for (size_t l = 0; l < n_labels[r]; ++l) {
            if (rep.cell_type[l] >= m.n_types) return bail(fail(GLZ_INVALID, "a cell type past the type count"));
            uniform &= rep.cell_type[l] == rep.cell_type[0];
        }
        const int t = rep.cell_type[0];
        const float j = (float)m.contact[t * m.n_types + t];
        for (int k = -26; k <= 26; ++k)
            if ((double)(float)((double)j * k) != (double)j * k) exact = false;
        const uint32_t TX = h->dim == 2 ? 128 : 64, TY = h->dim == 2 ? 32 : 8, TZ = h->dim == 2 ? 1 : 8;
        rep.tiles = (int)(((w + TX - 1) / TX) * ((hh + TY - 1) / TY) * (h->dim == 3 ? (d + TZ - 1) / TZ : 1));
        rep.label_off = h->total_sites;
        rep.cell_off = h->total_cells;
        h->total_sites += g.sites;
        h->total_cells += (long long)n_labels[r];
        h->total_tiles += rep.tiles;
    }
    h->uniform = uniform && exact;
    if (h->total_sites >= (1LL << 31) || h->total_cells >= (1LL << 31))
        return bail(fail(GLZ_INVALID, "the ensemble holds 2^31 sites or labels or more"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(GLZ_DRIVER, "cannot create a stream"));

    int rc;
    const size_t cells = (size_t)h->total_cells;
    if ((rc = dev_alloc(&h->labels, (size_t)h->total_sites)) || (rc = dev_alloc(&h->cell_type, cells)) ||
        (rc = dev_alloc(&h->vs_base[0], cells)) || (rc = dev_alloc(&h->vs_base[1], cells)) ||
        (rc = dev_alloc(&h->vs_delta[0], cells)) || (rc = dev_alloc(&h->vs_delta[1], cells)) ||
        (rc = dev_alloc(&h->vs_delta[2], cells)) || (rc = dev_alloc(&h->volc, cells * h->ncol)) ||
        (rc = dev_alloc(&h->anchor, cells * 4)) || (rc = dev_alloc(&h->d_reps, (size_t)n)) ||
        (rc = dev_alloc(&h->d_maps, (size_t)n)) || (rc = dev_alloc(&h->d_prefix, (size_t)n + 1)) ||
        (rc = dev_alloc(&h->d_order, (size_t)n)) || (rc = dev_alloc(&h->d_clock, 1)) ||
        (rc = dev_alloc(&h->d_barrier, 2)) ||
        (rc = dev_alloc(&h->error_flag, 1)) || (rc = dev_alloc(&h->medium, 2)))
        return bail(rc);
    // per-type tables, one block per replica: contact (n_types^2), tv, lv, ts, ls
    size_t table_floats = 0, conn_bytes = 0;
    for (int r = 0; r < n; ++r) {
        table_floats += (size_t)models[r].n_types * models[r].n_types + 4 * (size_t)models[r].n_types;
        conn_bytes += models[r].n_types;
    }
    if ((rc = dev_alloc(&h->tables, table_floats)) || (rc = dev_alloc(&h->connected, conn_bytes))) return bail(rc);

    bool tma = true;
    for (int r = 0; r < n; ++r) tma &= models[r].width % 4 == 0;
    const char *env = std::getenv("GLAZIER_SWEEP_TMA");
    h->use_tma = tma && !(env && env[0] == '0');
    EncodeTiled encode = nullptr;
    if (h->use_tma) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
            q != cudaDriverEntryPointSuccess)
            h->use_tma = false;
        else
            encode = reinterpret_cast<EncodeTiled>(fn);
    }

    std::vector<glz::EnsembleReplica> descs(n);
    std::vector<CUtensorMap> maps(n);
    std::vector<float> tables(table_floats);
    std::vector<uint8_t> conn(conn_bytes, 0);
    size_t toff = 0, coff = 0;
    for (int r = 0; r < n; ++r) {
        const glz_model &m = models[r];
        Replica &rep = h->reps[r];
        const int nt = m.n_types;
        float *tc = tables.data() + toff;
        for (int i = 0; i < nt * nt; ++i) tc[i] = (float)m.contact[i];
        for (int k = 0; k < nt; ++k) {
            tc[nt * nt + k] = (float)at(m.target_volume, k);
            tc[nt * nt + nt + k] = (float)at(m.lambda_volume, k);
            tc[nt * nt + 2 * nt + k] = (float)at(m.target_surface, k);
            tc[nt * nt + 3 * nt + k] = (float)at(m.lambda_surface, k);
        }
        float *dt = h->tables + toff;
        glz::SweepLaunch &a = descs[r].a;
        a = glz::SweepLaunch{};
        a.g = rep.g;
        a.t.contact = dt;
        a.t.target_volume = dt + nt * nt;
        a.t.lambda_volume = dt + nt * nt + nt;
        a.t.target_surface = dt + nt * nt + 2 * nt;
        a.t.lambda_surface = dt + nt * nt + 3 * nt;
        a.t.connected = h->connected + coff;
        a.n_types = nt;
        a.n_species = 0;
        a.beta = (float)(1.0 / m.temperature);
        a.labels = h->labels + rep.label_off;
        a.cell_type = h->cell_type + rep.cell_off;
        a.vol_by_colour = h->volc + rep.cell_off * h->ncol;
        a.anchor = h->anchor + rep.cell_off * 4;
        a.n_labels = (int)rep.n_labels;
        const int t = rep.cell_type[0];
        a.uniform_type = h->uniform ? t : -1;
        a.uniform_contact_exact = h->uniform;
        a.uniform_contact = (float)m.contact[t * nt + t];
        a.u_target_volume = (float)at(m.target_volume, t);
        a.u_lambda_volume = (float)at(m.lambda_volume, t);
        a.u_target_surface = (float)at(m.target_surface, t);
        a.u_lambda_surface = (float)at(m.lambda_surface, t);
        a.use_tma = h->use_tma;
        a.error_flag = h->error_flag;
        descs[r].cell_off = rep.cell_off;
        descs[r].seed = rep.seed;
        toff += (size_t)nt * nt + 4 * (size_t)nt;
        coff += nt;

        if (cudaMemcpyAsync(h->labels + rep.label_off, labels[r], rep.g.sites * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, h->stream) ||
            cudaMemcpyAsync(h->cell_type + rep.cell_off, rep.cell_type.data(), rep.n_labels, cudaMemcpyHostToDevice,
                            h->stream))
            return bail(fail(GLZ_DRIVER, "replica upload failed"));
        std::memset(&maps[r], 0, sizeof maps[r]);
        if (h->use_tma) {
            uint32_t box[3];
            glz::sweep_box(h->dim, box);
            cuuint64_t dims[3] = {(cuuint64_t)rep.g.w, (cuuint64_t)rep.g.h, (cuuint64_t)rep.g.d};
            cuuint64_t strides[2] = {(cuuint64_t)rep.g.w * 4, (cuuint64_t)rep.g.w * rep.g.h * 4};
            cuuint32_t boxd[3] = {box[0], box[1], box[2]};
            cuuint32_t elem[3] = {1, 1, 1};
            if (encode(&maps[r], CU_TENSOR_MAP_DATA_TYPE_UINT32, h->dim, h->labels + rep.label_off, dims, strides, boxd,
                       elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return bail(fail(GLZ_DRIVER, "cuTensorMapEncodeTiled failed"));
        }
    }
    if (cudaMemcpyAsync(h->tables, tables.data(), table_floats * sizeof(float), cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(h->connected, conn.data(), conn_bytes, cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(h->d_reps, descs.data(), n * sizeof(glz::EnsembleReplica), cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(h->d_maps, maps.data(), n * sizeof(CUtensorMap), cudaMemcpyHostToDevice, h->stream) ||
        cudaMemsetAsync(h->d_clock, 0, sizeof(glz::EnsembleClock), h->stream) ||
        cudaMemsetAsync(h->error_flag, 0, sizeof(int), h->stream))
        return bail(fail(GLZ_DRIVER, "ensemble upload failed"));
    // Every replica's tallies from its lattice, into base slot 0.
    for (int r = 0; r < n; ++r) {
        Replica &rep = h->reps[r];
        glz::RecountLaunch rl{};
        rl.g = rep.g;
        rl.labels = h->labels + rep.label_off;
        rl.n_labels = (int)rep.n_labels;
        rl.vs_base = h->vs_base[0] + rep.cell_off;
        for (int k = 0; k < 3; ++k) rl.vs_delta[k] = h->vs_delta[k] + rep.cell_off;
        rl.vol_by_colour = h->volc + rep.cell_off * h->ncol;
        rl.anchor = h->anchor + rep.cell_off * 4;
        rl.tracks = 0;
        rl.error_flag = h->error_flag;
        if (glz::launch_recount(rl, h->stream) != cudaSuccess) return bail(fail(GLZ_DRIVER, "recount failed"));
    }
    if (!glz::ensemble_grid_cap(h->dim, h->n_off, h->uniform)) return bail(fail(GLZ_DRIVER, "kernel setup failed"));
    if ((rc = set_schedule(h, 0, 0))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bail(fail(GLZ_DRIVER, std::string("ensemble setup: ") + cudaGetErrorString(cudaGetLastError())));
    *out = h;
    return GLZ_OK;
}

// Whether a model states a term the batch does not price: fields, length,
// connectivity, division, death, motility, drift or nematic.
static bool needs_engine(const glz_model &m) {
    bool extra = m.n_species > 0;
    for (int k = 0; k < m.n_types; ++k) {
        extra |= at(m.lambda_length, k) != 0.0 || at(m.division_volume, k) > 0.0 || at(m.death_rate, k) > 0.0;
        extra |= m.connected && m.connected[k];
        extra |= at(m.lambda_activity, k) != 0.0 || (m.nematic && at(m.lambda_nematic, k) != 0.0);
        for (int a = 0; a < 3; ++a) extra |= at(m.external, 3 * (size_t)k + a) != 0.0;
    }
    return extra;
}

int glz_ens_create(int n, const glz_model *models, const uint32_t *const *labels, const uint8_t *const *cell_types,
                   const size_t *n_labels, glz_ens **out) {
    if (!out) return fail(GLZ_INVALID, "null output handle");
    *out = nullptr;
    if (n < 1 || !models || !labels || !cell_types || !n_labels) return fail(GLZ_INVALID, "no replicas or a null array");
    std::vector<int> batch, alone;
    for (int r = 0; r < n; ++r) (needs_engine(models[r]) ? alone : batch).push_back(r);
    glz_ens *h = nullptr;
    if (!batch.empty()) {
        std::vector<glz_model> bm;
        std::vector<const uint32_t *> bl;
        std::vector<const uint8_t *> bt;
        std::vector<size_t> bn;
        for (int r : batch) {
            bm.push_back(models[r]);
            bl.push_back(labels[r]);
            bt.push_back(cell_types[r]);
            bn.push_back(n_labels[r]);
        }
        if (int rc = create_batched((int)batch.size(), bm.data(), bl.data(), bt.data(), bn.data(), &h)) return rc;
    } else {
        h = new glz_ens();
        h->n = 0;
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            glz_ens_destroy(h);
            return fail(GLZ_DRIVER, "cannot create a stream");
        }
    }
    h->all = n;
    h->slot.assign(n, 0);
    cudaGetDevice(&h->device);
    for (size_t b = 0; b < batch.size(); ++b) h->slot[batch[b]] = (int)b;
    for (int r : alone) {
        glz_gpu *g = nullptr;
        if (int rc = glz_gpu_create(&models[r], labels[r], cell_types[r], n_labels[r], nullptr, nullptr, &g)) {
            const std::string why = glz_last_error();
            glz_ens_destroy(h);
            return fail(rc, "replica " + std::to_string(r) + ": " + why);
        }
        h->engines.push_back(g);
        h->slot[r] = -(int)h->engines.size();
    }
    *out = h;
    return GLZ_OK;
}

// Replica i: its batch index (>= 0) or its engine, GLZ_INVALID when there is none.
static int which(glz_ens *h, int replica, int *batched, glz_gpu **engine) {
    if (replica < 0 || replica >= h->all) return fail(GLZ_INVALID, "no such replica");
    const int s = h->slot[replica];
    *batched = s >= 0 ? s : -1;
    *engine = s < 0 ? h->engines[-s - 1] : nullptr;
    return GLZ_OK;
}

// The batch's step and each engine replica's clocked step side by side in
// one graph.
static int build_mixed(glz_ens *h) {
    drop_mixed(h);
    if (h->n > 0)
        if (int rc = build_graph(h)) return rc;
    cudaGraph_t g = nullptr;
    CU(cudaGraphCreate(&g, 0));
    const auto done = [&](int rc) {
        cudaGraphDestroy(g);
        return rc;
    };
    cudaGraphNode_t node = nullptr;
    if (h->n > 0 && cudaGraphAddChildGraphNode(&node, g, nullptr, 0, h->graph) != cudaSuccess)
        return done(fail(GLZ_DRIVER, "cannot add the batch to the ensemble graph"));
    h->versions.assign(h->engines.size(), 0);
    for (size_t k = 0; k < h->engines.size(); ++k) {
        cudaGraph_t eg = nullptr;
        if (int rc = glz::engine_step_graph(h->engines[k], &eg, &h->versions[k])) return done(rc);
        const cudaError_t e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, eg);
        cudaGraphDestroy(eg);
        if (e != cudaSuccess) return done(fail(GLZ_DRIVER, "cannot add an engine replica to the ensemble graph"));
    }
    if (cudaGraphInstantiate(&h->mixed, g, 0) != cudaSuccess)
        return done(fail(GLZ_DRIVER, "cannot instantiate the ensemble graph"));
    return done(GLZ_OK);
}

// `steps` MCS of a batch and engine replicas that all replay from graphs:
// one replay of the mixed graph per MCS on the ensemble's stream. Before
// each, every engine makes room for its next divisions; one whose arrays
// grew makes the graph be captured anew.
static int step_mixed(glz_ens *h, uint64_t steps, double *ms) {
    for (glz_gpu *g : h->engines)
        if (int rc = glz::engine_begin_replays(g)) return rc;
    cudaEvent_t a = nullptr, b = nullptr;
    if (ms) {
        CU(cudaEventCreate(&a));
        CU(cudaEventCreate(&b));
        CU(cudaEventRecord(a, h->stream));
    }
    int rc = GLZ_OK;
    for (uint64_t s = 0; s < steps && rc == GLZ_OK; ++s) {
        bool stale = h->mixed == nullptr || h->versions.size() != h->engines.size();
        for (size_t k = 0; k < h->engines.size() && rc == GLZ_OK; ++k) {
            uint64_t v = 0;
            rc = glz::engine_before_replay(h->engines[k], h->stream, &v);
            stale |= rc == GLZ_OK && (k >= h->versions.size() || v != h->versions[k]);
        }
        if (rc == GLZ_OK && stale) rc = build_mixed(h);
        if (rc == GLZ_OK && cudaGraphLaunch(h->mixed, h->stream) != cudaSuccess)
            rc = fail(GLZ_DRIVER, "ensemble graph launch failed");
        if (rc != GLZ_OK) break;
        h->step += 1;
        h->pass += h->ncol;
        for (glz_gpu *g : h->engines) glz::engine_after_replay(g);
    }
    if (ms && rc == GLZ_OK) {
        CU(cudaEventRecord(b, h->stream));
        CU(cudaEventSynchronize(b));
        float t = 0.0f;
        CU(cudaEventElapsedTime(&t, a, b));
        *ms = t;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (rc) return rc;
    CU(cudaStreamSynchronize(h->stream));
    if (h->n > 0) {
        int flag = 0;
        CU(cudaMemcpy(&flag, h->error_flag, sizeof flag, cudaMemcpyDeviceToHost));
        if (flag) return fail(GLZ_DRIVER, "an ensemble sweep tile reported an error (flag " + std::to_string(flag) + ")");
    }
    for (size_t k = 0; k < h->engines.size(); ++k)
        if (int r = glz::engine_end_replays(h->engines[k])) return r;
    return GLZ_OK;
}

// `steps` MCS of every replica. With engine replicas that all replay from
// graphs, one mixed graph per MCS; otherwise the batch on the ensemble's
// stream and each engine on its own stream from a host thread of its own,
// all at once.
static int step_all(glz_ens *h, uint64_t steps, double *ms) {
    if (h->engines.empty()) return run(h, steps, true, ms);
    bool replays = true;
    for (glz_gpu *g : h->engines) replays &= glz::engine_replays(g);
    if (replays) return step_mixed(h, steps, ms);
    const auto t0 = std::chrono::steady_clock::now();
    const size_t e = h->engines.size();
    std::vector<int> rcs(e, GLZ_OK);
    std::vector<std::string> why(e);
    std::vector<std::thread> threads;
    threads.reserve(e);
    for (size_t k = 0; k < e; ++k)
        threads.emplace_back([h, k, steps, &rcs, &why] {
            if (cudaSetDevice(h->device) != cudaSuccess) {
                rcs[k] = GLZ_DRIVER;
                why[k] = "cannot select the ensemble's device";
                return;
            }
            rcs[k] = glz_gpu_step(h->engines[k], steps);
            if (rcs[k]) why[k] = glz_last_error();
        });
    int rc = GLZ_OK;
    if (h->n > 0)
        rc = run(h, steps, true, nullptr);
    else
        h->step += (long long)steps;
    for (auto &t : threads) t.join();
    if (ms) *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (rc) return rc;
    for (int r = 0; r < h->all; ++r)
        if (h->slot[r] < 0 && rcs[-h->slot[r] - 1])
            return fail(rcs[-h->slot[r] - 1], "replica " + std::to_string(r) + ": " + why[-h->slot[r] - 1]);
    return GLZ_OK;
}

int glz_ens_step(glz_ens *h, uint64_t steps) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    return step_all(h, steps, nullptr);
}

int glz_ens_step_timed(glz_ens *h, uint64_t steps, double *ms) {
    if (!h || !ms) return fail(GLZ_INVALID, "null handle or output");
    return step_all(h, steps, ms);
}

size_t glz_ens_n_labels(glz_ens *h, int replica) {
    int b = -1;
    glz_gpu *g = nullptr;
    if (!h || which(h, replica, &b, &g)) return 0;
    return g ? glz_gpu_n_labels(g) : h->reps[b].n_labels;
}

int glz_ens_set_infection(glz_ens *h, int replica, int species, int from_type, int to_type, double threshold) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    int b = -1;
    glz_gpu *g = nullptr;
    if (int rc = which(h, replica, &b, &g)) return rc;
    if (!g) return fail(GLZ_UNSUPPORTED, "replica " + std::to_string(replica) + " is batched and has no fields");
    drop_mixed(h);  // the engine's captured step carries the rule
    return glz_gpu_set_infection(g, species, from_type, to_type, threshold);
}

int glz_ens_autotune(glz_ens *h, uint64_t trial_steps, int *choice) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    if (h->n == 0) {  // nothing batched: no schedule to choose
        if (choice) *choice = 0;
        return GLZ_OK;
    }
    if (trial_steps < 1) trial_steps = 1;
    // Snapshot the state, time each candidate on it, put the state back: the
    // candidates give identical results, so only the time decides.
    const size_t cells = (size_t)h->total_cells, sites = (size_t)h->total_sites;
    std::vector<void *> keep;
    auto backup = [&](const void *src, size_t bytes) -> void * {
        void *dst = nullptr;
        if (cudaMalloc(&dst, bytes ? bytes : 1) != cudaSuccess) return nullptr;
        cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream);
        keep.push_back(dst);
        return dst;
    };
    struct Saved { void *dev; const void *src; size_t bytes; };
    std::vector<Saved> saved = {
        {nullptr, h->labels, sites * 4}, {nullptr, h->vs_base[0], cells * 8}, {nullptr, h->vs_base[1], cells * 8},
        {nullptr, h->vs_delta[0], cells * 8}, {nullptr, h->vs_delta[1], cells * 8}, {nullptr, h->vs_delta[2], cells * 8},
        {nullptr, h->volc, cells * h->ncol * 4}, {nullptr, h->d_clock, sizeof(glz::EnsembleClock)}};
    for (auto &s : saved)
        if (!(s.dev = backup(s.src, s.bytes))) {
            for (void *p : keep) cudaFree(p);
            return fail(GLZ_DRIVER, "autotune snapshot allocation failed");
        }
    const long long step0 = h->step, pass0 = h->pass;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int cap = glz::ensemble_grid_cap(h->dim, h->n_off, h->uniform);
    const int grids[3] = {0, cap > 2 * sms ? cap - sms : 0, sms};
    double best = 1e30;
    int best_i = 0, i = 0, rc = GLZ_OK;
    // (schedule, grid cap): replica order x tile shape, the windowed kernel
    // at three grid sizes, the direct shapes at one block per tile
    std::vector<std::pair<int, int>> cands;
    for (int shape = 0; shape < (h->dim == 2 ? 4 : 1); ++shape)
        for (int order = 0; order < 2; ++order) {
            if (shape == 0) {
                for (int g : grids) cands.push_back({order, g});
            } else {
                cands.push_back({order + 2 * shape, 0});      // a launch per colour pass
                cands.push_back({order + 2 * shape + 8, 0});  // the step's passes in one launch
            }
        }
    for (auto [sch, g] : cands) {
        if ((rc = set_schedule(h, sch, g))) break;
        double ms = 0.0;
        if ((rc = run(h, 1, true, nullptr))) break;  // warm the graph
        if ((rc = run(h, trial_steps, true, &ms))) break;
        if (ms < best) {
            best = ms;
            best_i = i;
        }
        for (auto &s : saved) cudaMemcpyAsync(const_cast<void *>(s.src), s.dev, s.bytes, cudaMemcpyDeviceToDevice, h->stream);
        h->step = step0;
        h->pass = pass0;
        ++i;
    }
    cudaStreamSynchronize(h->stream);
    for (void *p : keep) cudaFree(p);
    if (rc) return rc;
    if (choice) *choice = best_i;
    return set_schedule(h, cands[best_i].first, cands[best_i].second);
}

int glz_ens_set_schedule(glz_ens *h, int schedule, int max_ctas) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    if (schedule < 0 || schedule > 15 || max_ctas < 0) return fail(GLZ_INVALID, "no such schedule");
    return h->n > 0 ? set_schedule(h, schedule, max_ctas) : GLZ_OK;
}

int glz_ens_labels(glz_ens *h, int replica, uint32_t *out, size_t sites) {
    if (!h || !out) return fail(GLZ_INVALID, "null handle or buffer");
    glz_gpu *g = nullptr;
    if (int rc = which(h, replica, &replica, &g)) return rc;
    if (g) return glz_gpu_labels(g, out, sites);
    const Replica &rep = h->reps[replica];
    if (sites != (size_t)rep.g.sites) return fail(GLZ_INVALID, "the buffer is not one label per site");
    CU(cudaMemcpyAsync(out, h->labels + rep.label_off, sites * 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

static int ens_tallies(glz_ens *h, int replica, std::vector<int2> &vs, unsigned long long medium[2]) {
    if (replica < 0 || replica >= h->n) return fail(GLZ_INVALID, "no such replica");
    if (int rc = settle_all(h)) return rc;
    const Replica &rep = h->reps[replica];
    vs.resize(rep.n_labels);
    CU(cudaMemcpyAsync(vs.data(), h->vs_base[h->pass % 2] + rep.cell_off, rep.n_labels * sizeof(int2),
                       cudaMemcpyDeviceToHost, h->stream));
    CU(glz::launch_medium_count(rep.g, h->labels + rep.label_off, h->medium, h->stream));
    CU(cudaMemcpyAsync(medium, h->medium, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int glz_ens_volumes(glz_ens *h, int replica, uint32_t *out, size_t *count) {
    if (!h || !count) return fail(GLZ_INVALID, "null handle or count");
    glz_gpu *g = nullptr;
    if (int rc = which(h, replica, &replica, &g)) return rc;
    if (g) return glz_gpu_volumes(g, out, count);
    const size_t n = h->reps[replica].n_labels;
    if (!out || *count < n) {
        *count = n;
        return fail(GLZ_INVALID, "the buffer is shorter than the label count");
    }
    std::vector<int2> vs;
    unsigned long long medium[2];
    if (int rc = ens_tallies(h, replica, vs, medium)) return rc;
    out[0] = (uint32_t)medium[0];
    for (size_t l = 1; l < n; ++l) out[l] = vs[l].x > 0 ? (uint32_t)vs[l].x : 0u;
    *count = n;
    return GLZ_OK;
}

int glz_ens_surfaces(glz_ens *h, int replica, int64_t *out, size_t *count) {
    if (!h || !count) return fail(GLZ_INVALID, "null handle or count");
    glz_gpu *g = nullptr;
    if (int rc = which(h, replica, &replica, &g)) return rc;
    if (g) return glz_gpu_surfaces(g, out, count);
    const size_t n = h->reps[replica].n_labels;
    if (!out || *count < n) {
        *count = n;
        return fail(GLZ_INVALID, "the buffer is shorter than the label count");
    }
    std::vector<int2> vs;
    unsigned long long medium[2];
    if (int rc = ens_tallies(h, replica, vs, medium)) return rc;
    out[0] = (int64_t)medium[1];
    for (size_t l = 1; l < n; ++l) out[l] = vs[l].y;
    *count = n;
    return GLZ_OK;
}

uint64_t glz_ens_mcs(const glz_ens *h) { return h ? (uint64_t)h->step : 0; }

void *glz_ens_stream(glz_ens *h) { return h ? (void *)h->stream : nullptr; }

void glz_ens_destroy(glz_ens *h) {
    if (!h) return;
    for (glz_gpu *g : h->engines) glz_gpu_destroy(g);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graph(h);
    cudaFree(h->labels); cudaFree(h->cell_type);
    for (auto *p : h->vs_base) cudaFree(p);
    for (auto *p : h->vs_delta) cudaFree(p);
    cudaFree(h->volc); cudaFree(h->anchor); cudaFree(h->tables); cudaFree(h->connected);
    cudaFree(h->d_reps); cudaFree(h->d_maps); cudaFree(h->d_prefix); cudaFree(h->d_order);
    cudaFree(h->d_clock); cudaFree(h->d_barrier); cudaFree(h->error_flag); cudaFree(h->medium);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
