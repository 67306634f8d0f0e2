// The host engine behind the C ABI in include/glazier_gpu.h.
//
// Replaces `GpuSimulation` (glazier-cuda/src/lib.rs:748-1533): it owns the
// device copy of a run, one CUDA stream, and the per-step schedule
//   sweep colour 0 .. ncol-1  ->  field rounds  ->  division and death
// (lib.rs:1075-1141). Kernels are compiled ahead of time for sm_100a; there
// is no run-time compilation and no CPU path: a call that cannot run on the
// device fails with a status.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/glazier_gpu.h"
#include "device.cuh"
#include "engine.h"

namespace glz {
int sweep_box(int dim, uint32_t box[3]);
}

namespace {
thread_local std::string g_error = "no error";
}

namespace glz {
void set_last_error(const std::string &msg) { g_error = msg; }
}

namespace {

int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}

#define CU(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return fail(GLZ_DRIVER, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// lattice.rs:8-88: the neighbour offsets of an order, in the reference's
// order (the sweep's pick and the contact sum both follow it).
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

// field.rs:155-160
int substeps_for(double diffusion, int dimensions) {
    if (diffusion <= 0.0) return 1;
    double k = std::ceil(diffusion / (1.0 / (2.0 * (double)dimensions)));
    return k < 1.0 ? 1 : (int)k;
}

double at(const double *p, size_t i) { return p ? p[i] : 0.0; }

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct glz_gpu {
    int device = 0;
    cudaStream_t stream = nullptr;
    glz::Geometry g{};
    int n_types = 0, n_species = 0;
    float beta = 0.0f;
    uint64_t seed = 0;
    bool has_length = false, tracks = false, has_chemotaxis = false, has_pop = false, has_external = false;
    bool has_motility = false, has_nematic = false;
    float *nematic = nullptr;  // 2 per site, with the nematic term
    float *activity = nullptr;  // sites, with motility
    uint2 *pending = nullptr;   // a motility pass's accepted copies
    int *pending_count = nullptr;
    int substeps[glz::kMaxSpecies] = {};
    float fd[glz::kMaxSpecies] = {}, fdecay[glz::kMaxSpecies] = {};

    // per-type tables
    float *contact = nullptr, *tv = nullptr, *lv = nullptr, *ts = nullptr, *ls = nullptr;
    float *chemo = nullptr, *sec = nullptr, *upt = nullptr, *ext = nullptr, *maxact = nullptr, *lamact = nullptr;
    double *tl = nullptr, *ll = nullptr, *divv = nullptr, *death = nullptr, *lnem = nullptr;
    uint8_t *connected = nullptr;

    // state
    uint32_t *labels = nullptr;
    uint8_t *cell_type = nullptr;
    std::vector<uint8_t> cell_type_host;
    size_t n_labels = 0, cap = 0;
    glz::Tallies t{};
    float *field_buf = nullptr;  // 2 * n_species * sites: two buffers per species
    int field_cur[glz::kMaxSpecies] = {};
    uint64_t pass_no = 0, mcs = 0;
    bool use_tma = false;
    bool lean = false;    // the sweep prices contact, volume and surface only
    bool direct = false;  // ... on a lattice small enough for the direct kernel
    int compact = 0;      // ... queueing a warp's unlike copies (1, large passes) or a block's (2)
    bool resident = false;  // ... with nothing between passes: every MCS in one launch
    bool cluster = false;   // ... a plane, in one thread-block cluster's shared memory
    bool band = false;      // ... a large plane, streamed by row bands in one launch per call
    unsigned *barrier = nullptr;  // the resident sweep's grid barrier
    int max_ctas = 0;
    int uniform = -1;
    bool uniform_exact = false;
    // the infection rule (glz_gpu_set_infection); dose per label, cap entries
    int infect_species = -1, infect_from = 0, infect_to = 0;
    long long infect_threshold = 0;
    unsigned long long *dose = nullptr;
    float uniform_j = 0.0f;
    std::vector<float> host_tv, host_lv, host_ts, host_ls;
    CUtensorMap tmap{};
    int *error_flag = nullptr;
    unsigned long long *medium = nullptr;

    // Population models keep the live label count on the device (divisions
    // add to it there). The host holds an upper bound of it for the work it
    // has queued, and after each population step the count is copied into a
    // pinned slot and marked by an event, so the bound tightens without
    // waiting for the stream whenever a copy has landed.
    static constexpr int kCountSlots = 4;
    int *n_live = nullptr;
    int *n_seen = nullptr;  // pinned, kCountSlots entries
    cudaEvent_t n_event[kCountSlots] = {};
    uint64_t n_step[kCountSlots] = {};  // the population step each slot's copy follows
    uint64_t pop_steps = 0;             // population steps queued
    size_t n_bound = 0;
    // The most cells one step can add: cells at or past their division
    // volume hold disjoint sites, so at most sites / (the least division
    // volume, and at least 4 sites, cpu.rs:681) of them divide.
    size_t born_most = 0;

    // Steps of a direct-kernel engine replay from one captured graph: its
    // kernels read the step, pass and field buffers from `clock`, so the
    // same graph serves every step. GLAZIER_ENGINE_GRAPH=0 queues every
    // launch from the host instead.
    glz::EngineClock *clock = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    bool graph_on = true;
    uint64_t records_from = 0;  // count records older than this step predate graph replays
    uint64_t arrays_version = 0;  // bumped when the per-label arrays move (a captured step then is stale)

    // population scratch, `cap` entries each
    unsigned char *mode = nullptr;
    double *plan = nullptr;
    int *moved = nullptr;
    uint32_t *daughter = nullptr;
    int *counters = nullptr;

    float *field_ptr(int s, int which) { return field_buf + ((size_t)2 * s + which) * (size_t)g.sites; }

    glz::TypeTables tables() const {
        glz::TypeTables tt{};
        tt.contact = contact;
        tt.target_volume = tv;
        tt.lambda_volume = lv;
        tt.target_surface = ts;
        tt.lambda_surface = ls;
        tt.target_length = tl;
        tt.lambda_length = ll;
        tt.division_volume = divv;
        tt.death_rate = death;
        tt.connected = connected;
        tt.chemotaxis = chemo;
        tt.external = ext;
        tt.max_activity = maxact;
        tt.lambda_activity = lamact;
        tt.lambda_nematic = lnem;
        tt.secretion = sec;
        tt.uptake = upt;
        return tt;
    }
};

namespace {

template <typename T>
int dev_alloc(T **p, size_t n) {
    CU(cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)));
    return GLZ_OK;
}

template <typename T>
int upload(glz_gpu *h, T **p, const std::vector<T> &host) {
    int rc = dev_alloc(p, host.size());
    if (rc) return rc;
    if (!host.empty()) CU(cudaMemcpyAsync(*p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    return GLZ_OK;
}

void free_tallies(glz::Tallies &t) {
    for (auto *p : t.vs_base) cudaFree(p);
    for (auto *p : t.vs_delta) cudaFree(p);
    for (auto *p : t.mom_base) cudaFree(p);
    for (auto *p : t.mom_delta) cudaFree(p);
    cudaFree(t.vol_by_colour);
    cudaFree(t.anchor);
    t = glz::Tallies{};
}

void free_population(glz_gpu *h) {
    cudaFree(h->mode);
    cudaFree(h->plan);
    cudaFree(h->moved);
    cudaFree(h->daughter);
    h->mode = nullptr;
    h->plan = nullptr;
    h->moved = nullptr;
    h->daughter = nullptr;
}

void drop_step_graph(glz_gpu *h) {
    if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
}

// Per-label arrays sized for `cap` labels. The settled tallies, anchors,
// per-colour volumes and cell types of the first n_labels entries carry over
// exactly, so growing never changes a run; every delta word starts at zero.
int alloc_labels(glz_gpu *h, size_t cap) {
    const int nm = h->g.nm;
    const size_t n = h->n_labels;
    const uint64_t p = h->pass_no;
    glz::Tallies fresh{};
    for (int k = 0; k < 2; ++k) {
        if (int rc = dev_alloc(&fresh.vs_base[k], cap)) return rc;
        if (h->tracks)
            if (int rc = dev_alloc(&fresh.mom_base[k], cap * nm)) return rc;
    }
    for (int k = 0; k < 3; ++k) {
        if (int rc = dev_alloc(&fresh.vs_delta[k], cap)) return rc;
        CU(cudaMemsetAsync(fresh.vs_delta[k], 0, cap * sizeof(long long), h->stream));
        if (h->tracks) {
            if (int rc = dev_alloc(&fresh.mom_delta[k], cap * nm)) return rc;
            CU(cudaMemsetAsync(fresh.mom_delta[k], 0, cap * nm * sizeof(long long), h->stream));
        }
    }
    if (int rc = dev_alloc(&fresh.vol_by_colour, cap * h->g.ncol)) return rc;
    if (int rc = dev_alloc(&fresh.anchor, cap * 4)) return rc;
    uint8_t *types = nullptr;
    if (int rc = dev_alloc(&types, cap)) return rc;
    unsigned long long *dose = nullptr;
    if (int rc = dev_alloc(&dose, cap)) return rc;
    CU(cudaMemsetAsync(dose, 0, cap * sizeof(unsigned long long), h->stream));
    // the device holds the live types (an infection may have switched some)
    if (n && h->cap)
        CU(cudaMemcpyAsync(types, h->cell_type, n, cudaMemcpyDeviceToDevice, h->stream));
    else if (n)
        CU(cudaMemcpyAsync(types, h->cell_type_host.data(), n, cudaMemcpyHostToDevice, h->stream));
    if (h->cap) {
        CU(cudaMemcpyAsync(dose, h->dose, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, h->stream));
        // the caller has settled: base slot p % 2 holds every tally
        CU(cudaMemcpyAsync(fresh.vs_base[p % 2], h->t.vs_base[p % 2], n * sizeof(int2), cudaMemcpyDeviceToDevice,
                           h->stream));
        if (h->tracks)
            CU(cudaMemcpyAsync(fresh.mom_base[p % 2], h->t.mom_base[p % 2], n * nm * sizeof(long long),
                               cudaMemcpyDeviceToDevice, h->stream));
        CU(cudaMemcpyAsync(fresh.vol_by_colour, h->t.vol_by_colour, n * h->g.ncol * sizeof(int),
                           cudaMemcpyDeviceToDevice, h->stream));
        CU(cudaMemcpyAsync(fresh.anchor, h->t.anchor, n * 4 * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
    }
    CU(cudaStreamSynchronize(h->stream));
    free_tallies(h->t);
    h->t = fresh;
    free_population(h);
    if (h->has_pop) {
        if (int rc = dev_alloc(&h->mode, cap)) return rc;
        if (int rc = dev_alloc(&h->plan, cap * 6)) return rc;
        if (int rc = dev_alloc(&h->moved, cap)) return rc;
        if (int rc = dev_alloc(&h->daughter, cap)) return rc;
    }
    cudaFree(h->cell_type);
    h->cell_type = types;
    cudaFree(h->dose);
    h->dose = dose;
    h->cap = cap;
    drop_step_graph(h);  // its kernels hold the old arrays
    h->arrays_version += 1;
    return GLZ_OK;
}

// Recount every tally from the lattice; with `when` (a device flag) only if
// it is nonzero when the recount runs.
int recount(glz_gpu *h, const int *when = nullptr) {
    const uint64_t p = h->pass_no;
    glz::RecountLaunch r{};
    r.g = h->g;
    r.labels = h->labels;
    r.n_labels = (int)(h->n_live ? h->cap : h->n_labels);
    r.n_live = h->n_live;
    r.when = when;
    r.vs_base = h->t.vs_base[p % 2];
    r.mom_base = h->t.mom_base[p % 2];
    for (int k = 0; k < 3; ++k) {
        r.vs_delta[k] = h->t.vs_delta[k];
        r.mom_delta[k] = h->t.mom_delta[k];
    }
    r.vol_by_colour = h->t.vol_by_colour;
    r.anchor = h->t.anchor;
    r.tracks = h->tracks;
    r.nematic = h->has_nematic ? h->nematic : nullptr;
    r.error_flag = h->error_flag;
    CU(glz::launch_recount(r, h->stream));
    return GLZ_OK;
}

int settle(glz_gpu *h) {
    const uint64_t p = h->pass_no;
    CU(glz::launch_settle(h->t.vs_base[p % 2], h->t.vs_delta[(p + 2) % 3], h->t.mom_base[p % 2],
                          h->t.mom_delta[(p + 2) % 3], h->g.nm, (int)(h->n_live ? h->cap : h->n_labels), h->tracks,
                          h->n_live, h->stream));
    return GLZ_OK;
}

// The exact live label count of a population model, read after the stream
// drains; the types of labels born since the last read join the host copy.
int sync_count(glz_gpu *h) {
    if (!h->n_live) return GLZ_OK;
    int n = 0;
    CU(cudaMemcpyAsync(&n, h->n_live, sizeof n, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if ((size_t)n > h->n_labels) {
        h->cell_type_host.resize((size_t)n);
        CU(cudaMemcpy(h->cell_type_host.data() + h->n_labels, h->cell_type + h->n_labels, (size_t)n - h->n_labels,
                      cudaMemcpyDeviceToHost));
    }
    h->n_labels = (size_t)n;
    h->n_bound = (size_t)n;
    return GLZ_OK;
}

// The one type every label carries, or -1 when labels differ in type. The
// reference gives the medium's entry the first cell type (cpu.rs:203), so a
// single-type tissue is uniform medium included. Set at creation; a daughter
// takes its mother's type, so division keeps it.
void find_uniform_type(glz_gpu *h, const double *contact, int n_types) {
    h->uniform = -1;
    if (h->n_labels == 0) return;
    const uint8_t t = h->cell_type_host[0];
    for (size_t l = 1; l < h->n_labels; ++l)
        if (h->cell_type_host[l] != t) return;
    h->uniform = t;
    // The sweep then sums contact energies as J times a count m, |m| <=
    // n_off, which equals the neighbour-by-neighbour f32 sum when every J m
    // is exactly representable in f32.
    const float j = (float)contact[t * n_types + t];
    h->uniform_j = j;
    h->uniform_exact = true;
    for (int m = -26; m <= 26; ++m) {
        const double exact = (double)j * (double)m;
        if ((double)(float)exact != exact) h->uniform_exact = false;
    }
}

// The launch of the colour pass `colour` at the engine's current step and
// pass number.
glz::SweepLaunch pass_launch(glz_gpu *h, int colour) {
    const uint64_t p = h->pass_no;
    glz::SweepLaunch a{};
    a.g = h->g;
    a.t = h->tables();
    a.n_types = h->n_types;
    a.n_species = h->n_species;
    a.beta = h->beta;
    a.colour = colour;
    a.step = (int32_t)h->mcs;
    a.key_pick = glz::stream_key(h->seed, a.step, colour, 0);
    a.key_accept = glz::stream_key(h->seed, a.step, colour, 1);
    a.labels = h->labels;
    a.cell_type = h->cell_type;
    a.vs_base = h->t.vs_base[p % 2];
    a.vs_prev = h->t.vs_delta[(p + 2) % 3];
    a.vs_cur = reinterpret_cast<unsigned long long *>(h->t.vs_delta[p % 3]);
    a.vs_next_base = h->t.vs_base[(p + 1) % 2];
    a.vs_clear = h->t.vs_delta[(p + 1) % 3];
    a.mom_base = h->t.mom_base[p % 2];
    a.mom_prev = h->t.mom_delta[(p + 2) % 3];
    a.mom_cur = reinterpret_cast<unsigned long long *>(h->t.mom_delta[p % 3]);
    a.mom_next_base = h->t.mom_base[(p + 1) % 2];
    a.mom_clear = h->t.mom_delta[(p + 1) % 3];
    a.vol_by_colour = h->t.vol_by_colour;
    a.anchor = h->t.anchor;
    a.n_labels = (int)h->n_labels;
    a.n_live = h->n_live;
    a.uniform_type = h->uniform;
    a.uniform_contact_exact = h->uniform_exact;
    a.uniform_contact = h->uniform_j;
    if (h->uniform >= 0) {
        a.u_target_volume = h->host_tv[h->uniform];
        a.u_lambda_volume = h->host_lv[h->uniform];
        a.u_target_surface = h->host_ts[h->uniform];
        a.u_lambda_surface = h->host_ls[h->uniform];
    }
    a.has_length = h->has_length;
    a.tracks = h->tracks;
    a.has_chemotaxis = h->has_chemotaxis;
    a.has_external = h->has_external;
    a.has_motility = h->has_motility;
    a.has_nematic = h->has_nematic;
    a.nematic = h->nematic;
    a.activity = h->activity;
    a.pending = h->pending;
    a.pending_count = h->pending_count;
    for (int s = 0; s < h->n_species; ++s) a.fields[s] = h->field_ptr(s, h->field_cur[s]);
    a.use_tma = h->use_tma;
    a.lean = h->lean;
    a.direct = h->direct;
    a.compact = h->compact;
    a.max_ctas = h->max_ctas;
    a.tensor_map = h->use_tma ? &h->tmap : nullptr;
    a.error_flag = h->error_flag;
    return a;
}

int sweep_pass(glz_gpu *h, int colour) {
    const glz::SweepLaunch a = pass_launch(h, colour);
    CU(glz::launch_sweep(a, h->stream));
    if (h->has_motility) CU(glz::launch_apply_copies(a, h->activity, h->stream));
    h->pass_no += 1;
    return GLZ_OK;
}

int field_step(glz_gpu *h) {
    int rounds = 0;
    for (int s = 0; s < h->n_species; ++s) rounds = h->substeps[s] > rounds ? h->substeps[s] : rounds;
    for (int r = 0; r < rounds; ++r) {
        glz::FieldLaunch f{};
        f.g = h->g;
        f.n_species = h->n_species;
        f.round = r;
        f.labels = h->labels;
        f.cell_type = h->cell_type;
        f.secretion = h->sec;
        f.uptake = h->upt;
        f.infect_species = h->infect_species;
        f.infect_from = h->infect_from;
        f.dose = h->dose;
        for (int s = 0; s < h->n_species; ++s) {
            f.active[s] = r < h->substeps[s];
            f.last[s] = r == h->substeps[s] - 1;
            f.d[s] = h->fd[s];
            f.decay[s] = h->fdecay[s];
            f.in[s] = h->field_ptr(s, h->field_cur[s]);
            f.out[s] = h->field_ptr(s, 1 - h->field_cur[s]);
        }
        CU(glz::launch_field_round(f, h->stream));
        for (int s = 0; s < h->n_species; ++s)
            if (f.active[s]) h->field_cur[s] = 1 - h->field_cur[s];
    }
    return GLZ_OK;
}

// The most labels a population model can hold after one more step from a
// count of n: each live cell divides at most once, and at most born_most
// cells divide.
size_t after_step(const glz_gpu *h, size_t n) { return n + (h->born_most < n ? h->born_most : n); }

// The label capacity a population model grows to from a count of n: room
// for at least 16 steps of the most divisions, or 16 times the count when
// that is less.
size_t capacity_for(const glz_gpu *h, size_t n) {
    size_t room = 16 * h->born_most;
    if (room > 16 * n) room = 16 * n;
    if (room < n) room = n;
    return n + room + 64;
}

// Keep room for the next step's divisions. The host's bound of the count
// comes from the newest count copy that has landed (each step queued after
// it adds at most its most divisions); only when that is not enough does the
// host wait for the exact count, and grow when that is not.
int ensure_capacity(glz_gpu *h) {
    if (after_step(h, h->n_bound) <= h->cap) return GLZ_OK;
    for (int back = 0; back < glz_gpu::kCountSlots && (uint64_t)back < h->pop_steps; ++back) {
        const int slot = (int)((h->pop_steps - 1 - (uint64_t)back) % glz_gpu::kCountSlots);
        if (h->n_step[slot] < h->records_from) break;
        const cudaError_t q = cudaEventQuery(h->n_event[slot]);
        if (q == cudaErrorNotReady) {
            cudaGetLastError();
            continue;
        }
        CU(q);
        size_t bound = (size_t)h->n_seen[slot];
        for (uint64_t k = h->n_step[slot] + 1; k < h->pop_steps && bound <= h->cap; ++k) bound = after_step(h, bound);
        if (bound < h->n_bound) h->n_bound = bound;
        break;
    }
    if (after_step(h, h->n_bound) <= h->cap) return GLZ_OK;
    if (int rc = sync_count(h)) return rc;
    if (after_step(h, h->n_labels) <= h->cap) return GLZ_OK;
    if (int rc = settle(h)) return rc;
    return alloc_labels(h, capacity_for(h, h->n_labels));
}

// The population step's launches; `clocked` for a captured step (the settle
// slots and the death draws' step from the clock).
int population_launches(glz_gpu *h, bool clocked) {
    if (clocked)
        CU(glz::launch_settle_clocked(h->t, h->g.nm, (int)h->cap, h->tracks, h->n_live, h->clock, h->g.ncol,
                                      h->stream));
    else if (int rc = settle(h))
        return rc;
    // The pass count at the step's end has the parity of its start (ncol is
    // even), so the base slot below is the same for every step of a graph.
    const uint64_t p = h->pass_no;
    glz::PopulationLaunch a{};
    a.g = h->g;
    a.t = h->tables();
    a.labels = h->labels;
    a.cell_type_in = h->cell_type;
    a.cell_type_out = h->cell_type;
    a.n_labels = (int)h->n_labels;
    a.cap = (int)h->cap;
    a.n_live = h->n_live;
    a.vs_base = h->t.vs_base[p % 2];
    a.mom_base = h->t.mom_base[p % 2];
    a.anchor = h->t.anchor;
    a.key_death = glz::stream_key(h->seed, (int32_t)h->mcs, glz::kPopulationStream, 0);
    a.mode = h->mode;
    a.plan = h->plan;
    a.moved = h->moved;
    a.daughter = h->daughter;
    a.counters = h->counters;
    a.clock = clocked ? h->clock : nullptr;
    a.seed = h->seed;
    // plan, count, decide (the count grows on the device), apply; a step
    // without an event changes nothing and its recount returns at once
    CU(glz::launch_population_plan(a, h->stream));
    CU(glz::launch_population_apply(a, h->stream));
    return recount(h, h->counters + 1);
}

int population(glz_gpu *h) {
    if (int rc = ensure_capacity(h)) return rc;
    if (int rc = population_launches(h, false)) return rc;
    const int slot = (int)(h->pop_steps % glz_gpu::kCountSlots);
    CU(cudaMemcpyAsync(&h->n_seen[slot], h->n_live, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaEventRecord(h->n_event[slot], h->stream));
    h->n_step[slot] = h->pop_steps++;
    h->n_bound = after_step(h, h->n_bound);
    return GLZ_OK;
}

int check_error_flag(glz_gpu *h) {
    int flag = 0;
    CU(cudaMemcpyAsync(&flag, h->error_flag, sizeof flag, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (flag == 1) return fail(GLZ_DRIVER, "a sweep tile's tensor copy did not complete within its wait limit");
    if (flag == 2) return fail(GLZ_INVALID, "a label is not below the cell type count");
    if (flag == 3) return fail(GLZ_DRIVER, "the sweep's shared-memory window was not 128-byte aligned");
    if (flag == 4) return fail(GLZ_DRIVER, "a resident sweep's grid barrier did not complete within its wait limit");
    return GLZ_OK;
}

// The step schedule, with each phase bracketed by events when `ms` is given.
// Every MCS of the call in one cooperative launch. GLZ_OK with *done false
// when the blocks cannot all be resident (nothing launched; the caller runs
// the passes one by one, and later calls do too).
int run_resident(glz_gpu *h, uint64_t steps, double *ms, bool *done) {
    *done = false;
    glz::ResidentLaunch r{};
    r.a = pass_launch(h, 0);
    r.seed = h->seed;
    r.step0 = (int32_t)h->mcs;
    r.mcs = (int)steps;
    r.pass0 = (long long)h->pass_no;
    for (int k = 0; k < 2; ++k) r.vs_base[k] = h->t.vs_base[k];
    for (int k = 0; k < 3; ++k) r.vs_delta[k] = h->t.vs_delta[k];
    r.barrier = h->barrier;
    cudaEvent_t ev[2] = {};
    if (ms) {
        for (auto &e : ev) CU(cudaEventCreate(&e));
        ms[0] = ms[1] = ms[2] = 0.0;
    }
    CU(cudaMemsetAsync(h->barrier, 0, 2 * sizeof(unsigned), h->stream));
    if (ms) CU(cudaEventRecord(ev[0], h->stream));
    cudaError_t e = cudaErrorNotSupported;
    if (h->cluster) {
        e = glz::launch_cluster_sweep(r, h->stream);
        if (e == cudaErrorNotSupported) {
            cudaGetLastError();
            h->cluster = false;  // and later calls: the plane does not fit a cluster
        }
    }
    if (!h->cluster) e = glz::launch_resident_sweep(r, h->stream);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();
        h->resident = false;
        for (auto &x : ev)
            if (x) cudaEventDestroy(x);
        return GLZ_OK;
    }
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("resident sweep: ") + cudaGetErrorString(e));
    if (ms) {
        CU(cudaEventRecord(ev[1], h->stream));
        CU(cudaEventSynchronize(ev[1]));
        float t = 0.0f;
        CU(cudaEventElapsedTime(&t, ev[0], ev[1]));
        ms[0] = t;
        for (auto &x : ev) cudaEventDestroy(x);
    }
    h->pass_no += steps * (uint64_t)h->g.ncol;
    h->mcs += steps;
    *done = true;
    CU(cudaStreamSynchronize(h->stream));
    return check_error_flag(h);
}

// One step with clocked launches, for capture: the direct passes (and the
// motility copies), the activity decay, the field rounds, the infection rule,
// the population step, then the clock's advance. Host state is left as it is.
int queue_clocked_step(glz_gpu *h) {
    for (int c = 0; c < h->g.ncol; ++c) {
        glz::SweepLaunch a = pass_launch(h, c);
        a.clock = h->clock;
        a.seed = h->seed;
        a.tal = h->t;
        a.field_buf = h->field_buf;
        CU(glz::launch_sweep(a, h->stream));
        if (h->has_motility) CU(glz::launch_apply_copies(a, h->activity, h->stream));
    }
    if (h->has_motility) CU(glz::launch_activity_decay(h->activity, h->g.sites, h->stream));
    int rounds = 0;
    for (int s = 0; s < h->n_species; ++s) rounds = h->substeps[s] > rounds ? h->substeps[s] : rounds;
    for (int r = 0; r < rounds; ++r) {
        glz::FieldLaunch f{};
        f.g = h->g;
        f.n_species = h->n_species;
        f.round = r;
        f.labels = h->labels;
        f.cell_type = h->cell_type;
        f.secretion = h->sec;
        f.uptake = h->upt;
        f.infect_species = h->infect_species;
        f.infect_from = h->infect_from;
        f.dose = h->dose;
        f.clock = h->clock;
        f.field_buf = h->field_buf;
        for (int s = 0; s < h->n_species; ++s) {
            f.active[s] = r < h->substeps[s];
            f.last[s] = r == h->substeps[s] - 1;
            f.d[s] = h->fd[s];
            f.decay[s] = h->fdecay[s];
        }
        CU(glz::launch_field_round(f, h->stream));
    }
    if (h->infect_species >= 0)
        CU(glz::launch_infection(h->cell_type, h->dose, (int)(h->n_live ? h->cap : h->n_labels), h->infect_from,
                                 h->infect_to, h->infect_threshold, h->n_live, h->stream));
    if (h->has_pop)
        if (int rc = population_launches(h, true)) return rc;
    CU(glz::launch_engine_clock_advance(h->clock, h->g.ncol, h->stream));
    return GLZ_OK;
}

// One clocked step as a graph (not instantiated).
int capture_step_graph(glz_gpu *h, cudaGraph_t *out) {
    *out = nullptr;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = queue_clocked_step(h);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("step capture: ") + cudaGetErrorString(e));
    *out = graph;
    return GLZ_OK;
}

int capture_step(glz_gpu *h) {
    cudaGraph_t graph = nullptr;
    if (int rc = capture_step_graph(h, &graph)) return rc;
    const cudaError_t ei = cudaGraphInstantiate(&h->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(GLZ_DRIVER, std::string("step graph: ") + cudaGetErrorString(ei));
    return GLZ_OK;
}

// The clock from the host's counters, on the engine's stream.
int upload_clock(glz_gpu *h) {
    glz::EngineClock c{(long long)h->mcs, (long long)h->pass_no, 0u, 0u};
    for (int s = 0; s < h->n_species; ++s) {
        c.field_cur |= (unsigned)(h->field_cur[s] & 1) << s;
        c.field_flip |= (unsigned)(h->substeps[s] & 1) << s;
    }
    CU(cudaMemcpyAsync(h->clock, &c, sizeof c, cudaMemcpyHostToDevice, h->stream));
    return GLZ_OK;
}

// The host's counters after one replayed step.
void advance_host(glz_gpu *h) {
    h->pass_no += (uint64_t)h->g.ncol;
    h->mcs += 1;
    for (int s = 0; s < h->n_species; ++s)
        if (h->substeps[s] & 1) h->field_cur[s] = 1 - h->field_cur[s];
    if (h->has_pop) h->n_bound = after_step(h, h->n_bound);
}

// Steps of a direct-kernel engine, one graph replay each. The clock starts
// from the host's counters; the host keeps them in step with every replay,
// and checks label room before each (a growth drops the graph, whose kernels
// hold the old arrays, and the next replay captures it anew).
int run_graph(glz_gpu *h, uint64_t steps) {
    if (int rc = upload_clock(h)) return rc;
    h->records_from = h->pop_steps;  // count records from before the replays say nothing of them
    for (uint64_t r = 0; r < steps; ++r) {
        if (h->has_pop)
            if (int rc = ensure_capacity(h)) return rc;
        if (!h->step_exec)
            if (int rc = capture_step(h)) return rc;
        CU(cudaGraphLaunch(h->step_exec, h->stream));
        advance_host(h);
    }
    CU(cudaStreamSynchronize(h->stream));
    if (int rc = sync_count(h)) return rc;
    return check_error_flag(h);
}

// The band sweep's step schedule: every MCS of the call in one launch when
// nothing runs between steps, else one launch per MCS followed by the field
// step (and the infection rule). Phases are bracketed by events when `ms` is
// given. A plane the band sweep turns down goes back to the per-pass kernels.
int run_steps(glz_gpu *h, uint64_t steps, double *ms);

int run_band(glz_gpu *h, uint64_t steps, double *ms) {
    const bool between = h->n_species > 0 || h->infect_species >= 0;
    cudaEvent_t ev[3] = {};
    if (ms) {
        for (auto &e : ev) CU(cudaEventCreate(&e));
        ms[0] = ms[1] = ms[2] = 0.0;
    }
    const auto done = [&](int rc) {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        return rc;
    };
    while (steps > 0) {
        // launches of at most 65536 MCS keep the barrier's arrival count
        // (blocks x passes) far inside 32 bits
        const uint64_t chunk = between ? 1 : (steps < 65536 ? steps : 65536);
        glz::ResidentLaunch r{};
        r.a = pass_launch(h, 0);
        r.seed = h->seed;
        r.step0 = (int32_t)h->mcs;
        r.mcs = (int)chunk;
        r.pass0 = (long long)h->pass_no;
        for (int k = 0; k < 2; ++k) r.vs_base[k] = h->t.vs_base[k];
        for (int k = 0; k < 3; ++k) r.vs_delta[k] = h->t.vs_delta[k];
        r.barrier = h->barrier;
        if (cudaMemsetAsync(h->barrier, 0, 2 * sizeof(unsigned), h->stream) != cudaSuccess)
            return done(fail(GLZ_DRIVER, "barrier reset failed"));
        if (ms && cudaEventRecord(ev[0], h->stream) != cudaSuccess) return done(fail(GLZ_DRIVER, "event record failed"));
        const cudaError_t e = glz::launch_band_sweep(r, h->stream);
        if (e == cudaErrorNotSupported) {
            cudaGetLastError();
            h->band = false;  // and later calls: the per-pass kernels take this plane
            done(GLZ_OK);
            return run_steps(h, steps, ms);
        }
        if (e != cudaSuccess) return done(fail(GLZ_DRIVER, std::string("band sweep: ") + cudaGetErrorString(e)));
        h->pass_no += chunk * (uint64_t)h->g.ncol;
        h->mcs += chunk;
        if (ms && cudaEventRecord(ev[1], h->stream) != cudaSuccess) return done(fail(GLZ_DRIVER, "event record failed"));
        if (h->n_species > 0)
            if (int rc = field_step(h)) return done(rc);
        if (h->infect_species >= 0) {
            const cudaError_t ei = glz::launch_infection(h->cell_type, h->dose, (int)(h->n_live ? h->cap : h->n_labels), h->infect_from,
                                                         h->infect_to, h->infect_threshold, h->n_live, h->stream);
            if (ei != cudaSuccess) return done(fail(GLZ_DRIVER, std::string("infection: ") + cudaGetErrorString(ei)));
        }
        if (ms) {
            if (cudaEventRecord(ev[2], h->stream) != cudaSuccess || cudaEventSynchronize(ev[2]) != cudaSuccess)
                return done(fail(GLZ_DRIVER, "event record failed"));
            float t0 = 0.0f, t1 = 0.0f;
            cudaEventElapsedTime(&t0, ev[0], ev[1]);
            cudaEventElapsedTime(&t1, ev[1], ev[2]);
            ms[0] += t0;
            ms[1] += t1;
        }
        steps -= chunk;
    }
    done(GLZ_OK);
    CU(cudaStreamSynchronize(h->stream));
    return check_error_flag(h);
}

int run_steps(glz_gpu *h, uint64_t steps, double *ms) {
    if (h->band) return run_band(h, steps, ms);
    if (!ms && h->graph_on && h->direct && !h->resident && steps > 0) return run_graph(h, steps);
    // resident launches of at most 65536 MCS, so the barrier's arrival count
    // (blocks x passes) stays far inside 32 bits
    double total[3] = {0.0, 0.0, 0.0};
    while (h->resident && steps > 0) {
        const uint64_t chunk = steps < 65536 ? steps : 65536;
        bool done = false;
        double part[3];
        if (int rc = run_resident(h, chunk, ms ? part : nullptr, &done)) return rc;
        if (!done) break;
        if (ms)
            for (int k = 0; k < 3; ++k) total[k] += part[k];
        steps -= chunk;
    }
    if (ms && steps == 0) {
        for (int k = 0; k < 3; ++k) ms[k] = total[k];
        return GLZ_OK;
    }
    if (steps == 0) return GLZ_OK;
    cudaEvent_t ev[6] = {};
    if (ms) {
        for (auto &e : ev) CU(cudaEventCreate(&e));
        ms[0] = ms[1] = ms[2] = 0.0;
    }
    int rc = GLZ_OK;
    for (uint64_t r = 0; r < steps && rc == GLZ_OK; ++r) {
        if (ms) CU(cudaEventRecord(ev[0], h->stream));
        for (int c = 0; c < h->g.ncol && rc == GLZ_OK; ++c) rc = sweep_pass(h, c);
        if (rc == GLZ_OK && h->has_motility) {
            const cudaError_t e = glz::launch_activity_decay(h->activity, h->g.sites, h->stream);
            if (e != cudaSuccess) rc = fail(GLZ_DRIVER, std::string("activity decay: ") + cudaGetErrorString(e));
        }
        if (ms) CU(cudaEventRecord(ev[1], h->stream));
        if (rc == GLZ_OK && h->n_species > 0) rc = field_step(h);
        if (rc == GLZ_OK && h->infect_species >= 0) {
            const cudaError_t e = glz::launch_infection(h->cell_type, h->dose, (int)(h->n_live ? h->cap : h->n_labels), h->infect_from,
                                                        h->infect_to, h->infect_threshold, h->n_live, h->stream);
            if (e != cudaSuccess) rc = fail(GLZ_DRIVER, std::string("infection: ") + cudaGetErrorString(e));
        }
        if (ms) CU(cudaEventRecord(ev[2], h->stream));
        if (rc == GLZ_OK && h->has_pop) rc = population(h);
        if (ms) CU(cudaEventRecord(ev[3], h->stream));
        h->mcs += 1;
        if (ms && rc == GLZ_OK) {
            CU(cudaEventSynchronize(ev[3]));
            for (int k = 0; k < 3; ++k) {
                float t = 0.0f;
                CU(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
                ms[k] += t;
            }
        }
    }
    if (ms)
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    if (rc != GLZ_OK) return rc;
    CU(cudaStreamSynchronize(h->stream));
    if (int rc2 = sync_count(h)) return rc2;
    return check_error_flag(h);
}

}  // namespace

namespace glz {

bool engine_replays(const glz_gpu *h) { return h->graph_on && h->direct && !h->resident && !h->band; }

int engine_begin_replays(glz_gpu *h) {
    if (int rc = upload_clock(h)) return rc;
    h->records_from = h->pop_steps;
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int engine_step_graph(glz_gpu *h, cudaGraph_t *out, uint64_t *version) {
    *version = h->arrays_version;
    return capture_step_graph(h, out);
}

int engine_before_replay(glz_gpu *h, cudaStream_t replays, uint64_t *version) {
    if (h->has_pop && after_step(h, h->n_bound) > h->cap) {
        // the replays so far ran on the caller's stream: let them finish
        // before the engine reads its count (and grows, settling on its own)
        CU(cudaStreamSynchronize(replays));
        if (int rc = ensure_capacity(h)) return rc;
    }
    *version = h->arrays_version;
    return GLZ_OK;
}

void engine_after_replay(glz_gpu *h) { advance_host(h); }

int engine_end_replays(glz_gpu *h) {
    CU(cudaStreamSynchronize(h->stream));
    if (int rc = sync_count(h)) return rc;
    return check_error_flag(h);
}

}  // namespace glz

extern "C" {

const char *glz_last_error(void) { return g_error.c_str(); }

int glz_gpu_create(const glz_model *m, const uint32_t *labels, const uint8_t *cell_type, size_t n_labels,
                   const double *fields, const double *activity, glz_gpu **out) {
    if (!out) return fail(GLZ_INVALID, "null output handle");
    *out = nullptr;
    if (!m || !labels || !cell_type) return fail(GLZ_INVALID, "null model, labels or cell types");
    const int w = m->width, hh = m->height, d = m->depth;
    if (w <= 0 || hh <= 0 || d <= 0) return fail(GLZ_INVALID, "the lattice has a zero dimension");
    if (w % 2 != 0 || hh % 2 != 0 || (d > 1 && d % 2 != 0)) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "the checkerboard split needs even sides; the lattice is %d by %d by %d", w, hh,
                      d);
        return fail(GLZ_ODD_LATTICE, msg);
    }
    const long long sites = (long long)w * hh * d;
    if (sites >= (1LL << 31)) return fail(GLZ_INVALID, "the lattice has 2^31 sites or more");
    const int nt = m->n_types, ns = m->n_species;
    if (nt < 1 || nt > 255 || !m->contact) return fail(GLZ_INVALID, "the model needs 1 to 255 types and a contact matrix");
    if (ns < 0 || ns > glz::kMaxSpecies) return fail(GLZ_INVALID, "the device engine runs at most 8 species");
    if (m->neighbour_order < 1 || m->neighbour_order > 3)
        return fail(GLZ_INVALID, "neighbour order is outside the range one to three");
    if (!(m->temperature > 0.0)) return fail(GLZ_INVALID, "the temperature must be positive");
    if (n_labels < 1) return fail(GLZ_INVALID, "the cell type table is empty");

    bool nematic = false, motility = false, drift = false;
    for (int k = 0; k < nt; ++k) {
        nematic |= m->nematic && at(m->lambda_nematic, k) != 0.0;
        motility |= at(m->lambda_activity, k) != 0.0 && at(m->max_activity, k) > 0.0;
        for (int a = 0; a < 3; ++a) drift |= at(m->external, 3 * (size_t)k + a) != 0.0;
    }
    if (activity && !motility)
        for (long long i = 0; i < sites; ++i)
            if (activity[i] != 0.0) return fail(GLZ_UNSUPPORTED, "a nonzero activity needs the motility term");
    for (long long i = 0; i < sites; ++i)
        if (labels[i] >= n_labels) return fail(GLZ_INVALID, "a label is not below the cell type count");
    for (size_t l = 0; l < n_labels; ++l)
        if (cell_type[l] >= nt) return fail(GLZ_INVALID, "a cell type is not below the type count");

    glz_gpu *h = new glz_gpu();
    auto bail = [&](int rc) {
        glz_gpu_destroy(h);
        return rc;
    };
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return bail(fail(GLZ_DRIVER, "no CUDA device"));
    h->device = dev;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(GLZ_DRIVER, "cannot create a stream"));

    glz::Geometry &g = h->g;
    g.w = w;
    g.h = hh;
    g.d = d;
    g.dim = d > 1 ? 3 : 2;
    g.ncol = g.dim == 3 ? 8 : 4;
    g.sites = (int)sites;
    glz::set_dividers(g);
    // the moment words: the geometric sums, then the nematic field's two
    h->has_nematic = nematic;
    g.nm = (g.dim == 3 ? 9 : 5) + (nematic ? 2 : 0);
    g.n_off = offsets_for(m->neighbour_order, d, g.off);
    h->n_types = nt;
    h->n_species = ns;
    h->beta = (float)(1.0 / m->temperature);
    h->seed = m->seed;

    std::vector<float> contact(nt * nt), tv(nt), lv(nt), ts(nt), ls(nt);
    std::vector<double> tl(nt), ll(nt), divv(nt), death(nt);
    std::vector<uint8_t> conn(nt);
    bool has_conn = false;
    for (int a = 0; a < nt * nt; ++a) contact[a] = (float)m->contact[a];
    for (int k = 0; k < nt; ++k) {
        tv[k] = (float)at(m->target_volume, k);
        lv[k] = (float)at(m->lambda_volume, k);
        ts[k] = (float)at(m->target_surface, k);
        ls[k] = (float)at(m->lambda_surface, k);
        tl[k] = at(m->target_length, k);
        ll[k] = at(m->lambda_length, k);
        divv[k] = at(m->division_volume, k);
        death[k] = at(m->death_rate, k);
        conn[k] = m->connected ? (m->connected[k] != 0) : 0;
        has_conn |= conn[k] != 0;
        h->has_length |= ll[k] != 0.0;
        h->has_pop |= divv[k] > 0.0 || death[k] > 0.0;
    }
    h->tracks = h->has_length || h->has_pop || h->has_nematic;
    std::vector<double> lnem(nt);
    for (int k = 0; k < nt; ++k) lnem[k] = at(m->lambda_nematic, k);
    std::vector<float> maxact(nt), lamact(nt);
    for (int k = 0; k < nt; ++k) {
        maxact[k] = (float)at(m->max_activity, k);
        lamact[k] = (float)at(m->lambda_activity, k);
    }
    h->has_motility = motility;
    std::vector<float> ext(3 * (size_t)nt);
    for (size_t i = 0; i < ext.size(); ++i) ext[i] = (float)at(m->external, i);
    h->has_external = drift;
    std::vector<float> chemo(nt * (size_t)ns), sec(nt * (size_t)ns), upt(nt * (size_t)ns);
    for (size_t i = 0; i < chemo.size(); ++i) {
        chemo[i] = (float)at(m->chemotaxis, i);
        sec[i] = (float)at(m->secretion, i);
        upt[i] = (float)at(m->uptake, i);
        h->has_chemotaxis |= chemo[i] != 0.0f;
    }
    for (int s = 0; s < ns; ++s) {
        h->substeps[s] = substeps_for(at(m->diffusion, s), g.dim);
        h->fd[s] = (float)(at(m->diffusion, s) / (double)h->substeps[s]);
        h->fdecay[s] = (float)(at(m->decay, s) / (double)h->substeps[s]);
    }
    if (has_conn) {
        int all[26][3];
        int n = offsets_for(3, d, all);  // the full Moore / 26 ring (connectivity.rs:23-29)
        g.ring_n = n;
        std::memcpy(g.ring, all, sizeof all);
        for (int a = 0; a < n; ++a) {
            uint32_t mask = 0;
            for (int b = 0; b < n; ++b)
                if (std::abs(all[a][0] - all[b][0]) <= 1 && std::abs(all[a][1] - all[b][1]) <= 1 &&
                    std::abs(all[a][2] - all[b][2]) <= 1)
                    mask |= 1u << b;
            g.adjacency[a] = mask;
        }
    }

    // GLAZIER_SWEEP_LEAN=0 keeps every model on the general sweep kernel.
    const char *lean_env = std::getenv("GLAZIER_SWEEP_LEAN");
    h->lean = !h->has_length && !h->tracks && !h->has_chemotaxis && !h->has_external && !h->has_motility && !has_conn &&
              !(lean_env && lean_env[0] == '0');
    // A lean plane of at most 1024^2 sites, or a lean volume of any size,
    // takes the direct kernel: one thread per target reading the lattice
    // through the caches beats the lean kernel's window ring there (per MCS,
    // L2 flushed: 0.035 against 0.040 ms at 1024^2; 0.37 against 0.91 ms at
    // 256^3 and 0.64 against 1.07 ms at 320^3, a lattice past L2; at 2048^2
    // and 4096^2 the lean kernel leads: 100 MCS back to back at 2048^2 take
    // 5.8 ms on it against 7.8 ms on the warp-queued direct kernel, though a
    // single MCS after an L2 flush is 6 % faster on the latter).
    // GLAZIER_SWEEP_DIRECT=0: never, =1: at any size.
    const char *direct_env = std::getenv("GLAZIER_SWEEP_DIRECT");
    const int direct_mode = direct_env ? (direct_env[0] == '0' ? 0 : 1) : -1;
    const long long direct_most = g.dim == 2 ? 1024LL * 1024LL : sites;
    // Models with other terms (length, chemotaxis, connectivity, motility,
    // drift, nematic, division and death) take the direct kernel on planes up
    // to 1024^2 and volumes up to 128^3, where the tiled kernel's window
    // staging costs more than it saves.
    const long long direct_most_general = g.dim == 2 ? 1024LL * 1024LL : 128LL * 128LL * 128LL;
    h->direct = direct_mode == 1 || (direct_mode == -1 && sites <= (h->lean ? direct_most : direct_most_general));
    // From 2^18 targets a pass the direct kernel gathers each block's unlike
    // copies into one queue priced by whole warps, and from a million it
    // queues each warp's (GLAZIER_SWEEP_COMPACT=0: neither, =1: the warp's,
    // =2: the block's, at any size).
    const char *compact_env = std::getenv("GLAZIER_SWEEP_COMPACT");
    const int compact_mode = compact_env ? (compact_env[0] == '0' ? 0 : (compact_env[0] == '2' ? 2 : 1)) : -1;
    const long long targets = sites / g.ncol;
    h->compact = compact_mode >= 0 ? compact_mode
                                   : (targets >= glz::kDirectCompactFrom ? 1 : (targets >= glz::kDirectGatherFrom ? 2 : 0));
    // With no fields, division or death there is nothing between colour
    // passes: a direct plane of at most 512^2 sites runs every MCS of a call
    // in one cooperative launch, which saves more launch time than its grid
    // barrier costs (in a volume the barrier and its L2 reads lose to a
    // launch per pass). GLAZIER_SWEEP_RESIDENT=0: a launch per pass, =1: one
    // launch at any size or dimension.
    const char *resident_env = std::getenv("GLAZIER_SWEEP_RESIDENT");
    const int resident_mode = resident_env ? (resident_env[0] == '0' ? 0 : 1) : -1;
    h->resident = h->lean && h->direct && ns == 0 && !h->has_pop &&
                  (resident_mode == 1 || (resident_mode == -1 && g.dim == 2 && sites <= 512LL * 512LL));
    // A resident plane runs in one thread-block cluster when it fits one
    // (GLAZIER_SWEEP_CLUSTER=0: the cooperative grid instead).
    const char *cluster_env = std::getenv("GLAZIER_SWEEP_CLUSTER");
    h->cluster = h->resident && g.dim == 2 && !(cluster_env && cluster_env[0] == '0');
    // The band sweep (every colour pass of a call in one launch, rows
    // streamed by bands) runs a lean plane only when asked
    // (GLAZIER_SWEEP_BAND=1) and its rows are whole 16-byte units: at 2048^2,
    // 4096^2 and 8192^2 it measured slower than the windowed lean kernel
    // (0.169 against 0.145 ms per MCS at 4096^2, L2 flushed).
    const char *band_env = std::getenv("GLAZIER_SWEEP_BAND");
    h->band = h->lean && g.dim == 2 && band_env && band_env[0] == '1' && glz::band_sweep_fits(w, hh);
    if (h->band) h->direct = h->resident = h->cluster = false;
    h->host_tv = tv;
    h->host_lv = lv;
    h->host_ts = ts;
    h->host_ls = ls;
    int rc;
    if ((rc = upload(h, &h->contact, contact)) || (rc = upload(h, &h->tv, tv)) || (rc = upload(h, &h->lv, lv)) ||
        (rc = upload(h, &h->ts, ts)) || (rc = upload(h, &h->ls, ls)) || (rc = upload(h, &h->tl, tl)) ||
        (rc = upload(h, &h->ll, ll)) || (rc = upload(h, &h->divv, divv)) || (rc = upload(h, &h->death, death)) ||
        (rc = upload(h, &h->connected, conn)) || (rc = upload(h, &h->chemo, chemo)) || (rc = upload(h, &h->sec, sec)) ||
        (rc = upload(h, &h->upt, upt)) || (rc = upload(h, &h->ext, ext)) || (rc = upload(h, &h->maxact, maxact)) ||
        (rc = upload(h, &h->lamact, lamact)) || (rc = upload(h, &h->lnem, lnem)))
        return bail(rc);

    if ((rc = dev_alloc(&h->labels, (size_t)sites))) return bail(rc);
    if (cudaMemcpyAsync(h->labels, labels, sites * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream))
        return bail(fail(GLZ_DRIVER, "label upload failed"));
    h->cell_type_host.assign(cell_type, cell_type + n_labels);
    h->n_labels = n_labels;
    find_uniform_type(h, m->contact, nt);
    if (h->has_pop) {
        double least = 0.0;  // the least division volume, at least the 4 sites a division needs
        for (int k = 0; k < nt; ++k)
            if (divv[k] > 0.0) {
                const double v = divv[k] < 4.0 ? 4.0 : std::ceil(divv[k]);
                least = least == 0.0 || v < least ? v : least;
            }
        h->born_most = least > 0.0 ? (size_t)((double)sites / least) : 0;
    }
    if ((rc = alloc_labels(h, h->has_pop ? capacity_for(h, n_labels) : n_labels))) return bail(rc);
    if (h->has_pop) {
        const int n = (int)n_labels;
        if ((rc = dev_alloc(&h->n_live, 1))) return bail(rc);
        if (cudaMemcpy(h->n_live, &n, sizeof n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaHostAlloc((void **)&h->n_seen, glz_gpu::kCountSlots * sizeof(int), cudaHostAllocDefault) != cudaSuccess)
            return bail(fail(GLZ_DRIVER, "label count set-up failed"));
        for (auto &e : h->n_event)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                return bail(fail(GLZ_DRIVER, "cannot create an event"));
        h->n_bound = n_labels;
    }

    if (ns > 0) {
        if ((rc = dev_alloc(&h->field_buf, (size_t)2 * ns * sites))) return bail(rc);
        std::vector<float> f((size_t)sites);
        for (int s = 0; s < ns; ++s) {
            for (long long i = 0; i < sites; ++i) f[i] = (float)(fields ? fields[(size_t)s * sites + i] : at(m->initial, s));
            if (cudaMemcpy(h->field_ptr(s, 0), f.data(), sites * sizeof(float), cudaMemcpyHostToDevice))
                return bail(fail(GLZ_DRIVER, "field upload failed"));
        }
    }
    if (h->has_nematic) {
        std::vector<float> q(2 * (size_t)sites);
        for (size_t i = 0; i < q.size(); ++i) q[i] = (float)m->nematic[i];
        if ((rc = dev_alloc(&h->nematic, q.size()))) return bail(rc);
        if (cudaMemcpy(h->nematic, q.data(), q.size() * sizeof(float), cudaMemcpyHostToDevice))
            return bail(fail(GLZ_DRIVER, "nematic field upload failed"));
    }
    if (h->has_motility) {
        std::vector<float> act((size_t)sites);
        for (long long i = 0; i < sites; ++i) act[i] = activity ? (float)activity[i] : 0.0f;
        if ((rc = dev_alloc(&h->activity, (size_t)sites))) return bail(rc);
        if (cudaMemcpy(h->activity, act.data(), sites * sizeof(float), cudaMemcpyHostToDevice))
            return bail(fail(GLZ_DRIVER, "activity upload failed"));
        if ((rc = dev_alloc(&h->pending, (size_t)(sites / g.ncol + 1)))) return bail(rc);
        if ((rc = dev_alloc(&h->pending_count, 1))) return bail(rc);
        if (cudaMemset(h->pending_count, 0, sizeof(int))) return bail(fail(GLZ_DRIVER, "memset failed"));
    }
    if ((rc = dev_alloc(&h->error_flag, 1))) return bail(rc);
    if ((rc = dev_alloc(&h->clock, 1))) return bail(rc);
    if (const char *graph_env = std::getenv("GLAZIER_ENGINE_GRAPH")) h->graph_on = graph_env[0] != '0';
    if ((rc = dev_alloc(&h->barrier, 2))) return bail(rc);
    if ((rc = dev_alloc(&h->medium, 2))) return bail(rc);
    if ((rc = dev_alloc(&h->counters, 2))) return bail(rc);
    if (cudaMemsetAsync(h->error_flag, 0, sizeof(int), h->stream)) return bail(fail(GLZ_DRIVER, "memset failed"));

    // The tensor copy needs rows that are a whole number of 16-byte units.
    const char *env = std::getenv("GLAZIER_SWEEP_TMA");
    h->use_tma = (w % 4 == 0) && !(env && env[0] == '0');
    // GLAZIER_SWEEP_CTAS caps the sweep's persistent grid; the default is one
    // full wave of resident CTAs.
    if (const char *cap = std::getenv("GLAZIER_SWEEP_CTAS")) h->max_ctas = std::atoi(cap);
    if (h->use_tma) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
            q != cudaDriverEntryPointSuccess) {
            h->use_tma = false;
        } else {
            uint32_t box[3];
            glz::sweep_box(g.dim, box);
            const cuuint32_t rank = g.dim;
            cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)hh, (cuuint64_t)d};
            cuuint64_t strides[2] = {(cuuint64_t)w * 4, (cuuint64_t)w * hh * 4};
            cuuint32_t boxd[3] = {box[0], box[1], box[2]};
            cuuint32_t elem[3] = {1, 1, 1};
            CUresult r = reinterpret_cast<EncodeTiled>(fn)(
                &h->tmap, CU_TENSOR_MAP_DATA_TYPE_UINT32, rank, h->labels, dims, strides, boxd, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return bail(fail(GLZ_DRIVER, "cuTensorMapEncodeTiled failed"));
        }
    }
    if ((rc = recount(h))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bail(fail(GLZ_DRIVER, std::string("setup: ") + cudaGetErrorString(cudaGetLastError())));
    *out = h;
    return GLZ_OK;
}

int glz_set_device(int ordinal) {
    CU(cudaSetDevice(ordinal));
    return GLZ_OK;
}

int glz_gpu_step(glz_gpu *h, uint64_t steps) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    return run_steps(h, steps, nullptr);
}

int glz_gpu_step_profiled(glz_gpu *h, uint64_t steps, double ms[3]) {
    if (!h || !ms) return fail(GLZ_INVALID, "null handle or output");
    return run_steps(h, steps, ms);
}

int glz_gpu_set_labels(glz_gpu *h, const uint32_t *labels, size_t sites) {
    if (!h || !labels) return fail(GLZ_INVALID, "null handle or labels");
    if (sites != (size_t)h->g.sites) return fail(GLZ_INVALID, "the lattice is not one label per site");
    CU(cudaMemcpyAsync(h->labels, labels, sites * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    return recount(h);
}

// Whether `p` is device memory of the handle's device (plain or managed).
static bool on_device(const glz_gpu *h, const void *p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == h->device;
}

int glz_gpu_set_labels_device(glz_gpu *h, const uint32_t *labels, size_t sites) {
    if (!h || !labels) return fail(GLZ_INVALID, "null handle or labels");
    if (sites != (size_t)h->g.sites) return fail(GLZ_INVALID, "the lattice is not one label per site");
    if (!on_device(h, labels)) return fail(GLZ_INVALID, "the labels are not device memory of the engine's device");
    CU(cudaMemcpyAsync(h->labels, labels, sites * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
    if (int rc = recount(h)) return rc;
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int glz_gpu_labels(glz_gpu *h, uint32_t *out, size_t sites) {
    if (!h || !out) return fail(GLZ_INVALID, "null handle or buffer");
    if (sites != (size_t)h->g.sites) return fail(GLZ_INVALID, "the buffer is not one label per site");
    CU(cudaMemcpyAsync(out, h->labels, sites * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int glz_gpu_field(glz_gpu *h, int index, double *out, size_t sites) {
    if (!h || !out) return fail(GLZ_INVALID, "null handle or buffer");
    if (index < 0 || index >= h->n_species) return fail(GLZ_INVALID, "no such species");
    if (sites != (size_t)h->g.sites) return fail(GLZ_INVALID, "the buffer is not one value per site");
    std::vector<float> f(sites);
    CU(cudaMemcpyAsync(f.data(), h->field_ptr(index, h->field_cur[index]), sites * sizeof(float),
                       cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < sites; ++i) out[i] = (double)f[i];
    return GLZ_OK;
}

static int read_tallies(glz_gpu *h, std::vector<int2> &vs, unsigned long long medium[2]) {
    if (int rc = settle(h)) return rc;
    vs.resize(h->n_labels);
    CU(cudaMemcpyAsync(vs.data(), h->t.vs_base[h->pass_no % 2], h->n_labels * sizeof(int2), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(glz::launch_medium_count(h->g, h->labels, h->medium, h->stream));
    CU(cudaMemcpyAsync(medium, h->medium, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int glz_gpu_volumes(glz_gpu *h, uint32_t *out, size_t *count) {
    if (!h || !count) return fail(GLZ_INVALID, "null handle or count");
    if (!out || *count < h->n_labels) {
        *count = h->n_labels;
        return fail(GLZ_INVALID, "the buffer is shorter than the label count");
    }
    std::vector<int2> vs;
    unsigned long long medium[2];
    if (int rc = read_tallies(h, vs, medium)) return rc;
    out[0] = (uint32_t)medium[0];
    for (size_t l = 1; l < h->n_labels; ++l) out[l] = vs[l].x > 0 ? (uint32_t)vs[l].x : 0u;
    *count = h->n_labels;
    return GLZ_OK;
}

int glz_gpu_surfaces(glz_gpu *h, int64_t *out, size_t *count) {
    if (!h || !count) return fail(GLZ_INVALID, "null handle or count");
    if (!out || *count < h->n_labels) {
        *count = h->n_labels;
        return fail(GLZ_INVALID, "the buffer is shorter than the label count");
    }
    std::vector<int2> vs;
    unsigned long long medium[2];
    if (int rc = read_tallies(h, vs, medium)) return rc;
    out[0] = (int64_t)medium[1];
    for (size_t l = 1; l < h->n_labels; ++l) out[l] = (int64_t)vs[l].y;
    *count = h->n_labels;
    return GLZ_OK;
}

int glz_gpu_cell_types(glz_gpu *h, uint8_t *out, size_t *count) {
    if (!h || !count) return fail(GLZ_INVALID, "null handle or count");
    if (!out || *count < h->n_labels) {
        *count = h->n_labels;
        return fail(GLZ_INVALID, "the buffer is shorter than the label count");
    }
    CU(cudaMemcpyAsync(out, h->cell_type, h->n_labels, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    *count = h->n_labels;
    return GLZ_OK;
}

int glz_gpu_set_infection(glz_gpu *h, int species, int from_type, int to_type, double threshold) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    if (species < 0 || species >= h->n_species) return fail(GLZ_INVALID, "the infection names no species of the model");
    if (from_type < 1 || from_type >= h->n_types || to_type < 1 || to_type >= h->n_types || from_type == to_type)
        return fail(GLZ_INVALID, "the infection switches between two distinct cell types (not the medium)");
    if (!(threshold >= 0.0) || !(threshold * (double)glz::kDoseScale < 9.0e18))
        return fail(GLZ_INVALID, "the infection threshold must be finite and >= 0");
    h->infect_species = species;
    h->infect_from = from_type;
    h->infect_to = to_type;
    h->infect_threshold = std::llround(threshold * (double)glz::kDoseScale);
    // types now change during a run: the sweep reads them per copy
    h->uniform = -1;
    drop_step_graph(h);  // its launches carry the rule and the uniform-type pricing
    return GLZ_OK;
}

int glz_gpu_set_nematic_field(glz_gpu *h, const double *field, size_t len) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    drop_step_graph(h);
    if (len != 2 * (size_t)h->g.sites) {
        char msg[128];
        std::snprintf(msg, sizeof msg, "nematic field has %zu sites, the lattice %d", len / 2, h->g.sites);
        return fail(GLZ_INVALID, msg);
    }
    // lib.rs:1207-1210
    if (!h->has_nematic) return fail(GLZ_DRIVER, "the model has no nematic coupling to update");
    if (!field) return fail(GLZ_INVALID, "null field");
    std::vector<float> q(len);
    for (size_t i = 0; i < len; ++i) q[i] = (float)field[i];
    CU(cudaMemcpyAsync(h->nematic, q.data(), len * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    // the per-cell sums follow the new field: settle, then recount every tally
    if (int rc = settle(h)) return rc;
    if (int rc = recount(h)) return rc;
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

int glz_gpu_set_nematic_field_device(glz_gpu *h, const float *field, size_t len) {
    if (!h) return fail(GLZ_INVALID, "null handle");
    drop_step_graph(h);
    if (len != 2 * (size_t)h->g.sites) {
        char msg[128];
        std::snprintf(msg, sizeof msg, "nematic field has %zu sites, the lattice %d", len / 2, h->g.sites);
        return fail(GLZ_INVALID, msg);
    }
    if (!h->has_nematic) return fail(GLZ_DRIVER, "the model has no nematic coupling to update");
    if (!field) return fail(GLZ_INVALID, "null field");
    if (!on_device(h, field)) return fail(GLZ_INVALID, "the field is not device memory of the engine's device");
    CU(cudaMemcpyAsync(h->nematic, field, len * sizeof(float), cudaMemcpyDeviceToDevice, h->stream));
    if (int rc = settle(h)) return rc;
    if (int rc = recount(h)) return rc;
    CU(cudaStreamSynchronize(h->stream));
    return GLZ_OK;
}

uint64_t glz_gpu_mcs(const glz_gpu *h) { return h ? h->mcs : 0; }

size_t glz_gpu_n_labels(const glz_gpu *h) { return h ? h->n_labels : 0; }

const char *glz_gpu_sweep_kernel(const glz_gpu *h) {
    if (!h) return "";
    if (h->band) return "band";
    if (h->cluster) return "cluster";
    if (h->resident) return "resident";
    if (h->direct) return h->compact == 1 ? "compact" : (h->compact == 2 ? "gathered" : "direct");
    return h->lean ? "lean" : "general";
}

void *glz_gpu_stream(glz_gpu *h) { return h ? (void *)h->stream : nullptr; }

int glz_gpu_device_labels(glz_gpu *h, void **labels) {
    if (!h || !labels) return fail(GLZ_INVALID, "null handle or output");
    *labels = h->labels;
    return GLZ_OK;
}

int glz_gpu_device_field(glz_gpu *h, int index, void **field) {
    if (!h || !field) return fail(GLZ_INVALID, "null handle or output");
    if (index < 0 || index >= h->n_species) return fail(GLZ_INVALID, "no such species");
    *field = h->field_ptr(index, h->field_cur[index]);
    return GLZ_OK;
}

void glz_gpu_destroy(glz_gpu *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->contact); cudaFree(h->tv); cudaFree(h->lv); cudaFree(h->ts); cudaFree(h->ls);
    cudaFree(h->chemo); cudaFree(h->sec); cudaFree(h->upt); cudaFree(h->ext); cudaFree(h->maxact); cudaFree(h->lamact);
    cudaFree(h->activity); cudaFree(h->pending); cudaFree(h->pending_count); cudaFree(h->nematic); cudaFree(h->lnem);
    cudaFree(h->tl); cudaFree(h->ll); cudaFree(h->divv); cudaFree(h->death); cudaFree(h->connected);
    cudaFree(h->labels); cudaFree(h->cell_type); cudaFree(h->field_buf); cudaFree(h->dose);
    cudaFree(h->error_flag); cudaFree(h->medium); cudaFree(h->barrier); cudaFree(h->counters);
    free_tallies(h->t);
    free_population(h);
    drop_step_graph(h);
    cudaFree(h->clock);
    cudaFree(h->n_live);
    if (h->n_seen) cudaFreeHost(h->n_seen);
    for (auto &e : h->n_event)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
