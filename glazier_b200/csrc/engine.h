// Internal interface between the host engine (engine.cu) and the kernel
// files. Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "device.cuh"

namespace glz {

constexpr int kMaxSpecies = 8;
constexpr int kMaxTypes = 64;

// Lattice geometry. A plane has d == 1, dim == 2, four colours; a volume has
// dim == 3 and eight.
struct Geometry {
    int w, h, d, dim, ncol, sites;
    int n_off;          // energy neighbourhood (lattice.rs:69-88)
    int off[26][3];
    int ring_n;         // connectivity ring (connectivity.rs:23-29), 0 when off
    int ring[26][3];
    uint32_t adjacency[26];
    int nm;             // exact moment sums per cell: 5 in a plane, 9 in a volume
    // w, h and their halves (a colour's targets per row and rows per plane)
    // as multiply-shift dividers; set_dividers fills them from w and h
    Divider div_w, div_h, div_hw, div_hh;
};

inline void set_dividers(Geometry &g) {
    g.div_w = make_divider((uint32_t)g.w);
    g.div_h = make_divider((uint32_t)g.h);
    g.div_hw = make_divider((uint32_t)(g.w / 2 > 0 ? g.w / 2 : 1));
    g.div_hh = make_divider((uint32_t)(g.h / 2 > 0 ? g.h / 2 : 1));
}

// Per-type tables in device memory, row-major [type][...], index 0 the medium.
struct TypeTables {
    const float *contact;       // n_types * n_types
    const float *target_volume, *lambda_volume, *target_surface, *lambda_surface;
    const double *target_length, *lambda_length, *division_volume, *death_rate;
    const uint8_t *connected;
    const float *chemotaxis, *secretion, *uptake;  // n_types * n_species
    const float *external;                         // n_types * 3: the drift vector
    const float *max_activity, *lambda_activity;   // the motility (Act) term
    const double *lambda_nematic;
};

// The per-cell tallies a colour pass reads, in the rotation that gives every
// pass a snapshot without an extra launch:
//   the value at the start of pass p is B[p % 2] + D[(p + 2) % 3];
//   pass p adds its changes into D[p % 3], and on the way writes
//   B[(p + 1) % 2] = B[p % 2] + D[(p + 2) % 3] and clears D[(p + 1) % 3],
//   none of which any thread of pass p reads.
// `vol_surf` words hold (volume, surface); `mom` holds nm int64 sums per cell.
struct Tallies {
    int2 *vs_base[2];
    long long *vs_delta[3];
    long long *mom_base[2];
    long long *mom_delta[3];
    int *vol_by_colour;  // ncol per cell: only the current colour's entry changes in a pass
    int *anchor;         // 4 per cell (x, y, z, unused): the integer origin of the moment sums
};

// The device clock of an engine whose steps replay from one captured CUDA
// graph: the kernels of a step read the step's number, its first pass's
// number and each species' current field buffer here, so the same graph
// serves every step; the graph's last node advances it.
struct EngineClock {
    long long step;       // Monte Carlo steps completed
    long long pass;       // colour passes completed
    unsigned field_cur;   // bit s: the buffer (0 or 1) holding species s
    unsigned field_flip;  // bit s: species s takes an odd number of sub-steps, so its buffer flips each step
};

struct SweepLaunch {
    Geometry g;
    TypeTables t;
    int n_types, n_species;
    float beta;  // (float)(1 / T), rounded once on the host
    int colour;
    int32_t step;
    uint64_t key_pick, key_accept;  // stream_key(seed, step, colour, 0 / 1)
    uint32_t *labels;
    const uint8_t *cell_type;
    // this pass's view of the tallies
    const int2 *vs_base;
    const long long *vs_prev;
    unsigned long long *vs_cur;
    int2 *vs_next_base;
    long long *vs_clear;
    const long long *mom_base;
    const long long *mom_prev;
    unsigned long long *mom_cur;
    long long *mom_next_base;
    long long *mom_clear;
    int *vol_by_colour;
    const int *anchor;
    int n_labels;
    // Population models keep their live label count in device memory (it
    // changes on the device when cells divide); n_labels is then the
    // capacity and kernels read the count here. Null otherwise.
    const int *n_live;
    int uniform_type;  // the type of every label when they share one, else -1
    int uniform_contact_exact;  // J m is exact in f32 for every |m| <= n_off (see sweep.cu)
    float uniform_contact;      // J[type][type] when uniform
    float u_target_volume, u_lambda_volume, u_target_surface, u_lambda_surface;
    int has_length, tracks, has_chemotaxis, has_external, has_motility, has_nematic;
    // the nematic field, (Q_xx, Q_xy) per site; its per-cell sums ride in the
    // moment words after the geometric ones (g.nm counts both)
    const float *nematic;
    // Motility reads labels and activity two sites from the target, where
    // same-colour targets change during the pass, so a pass with it leaves
    // both as they were and lists its accepted copies (target, new label)
    // for launch_apply_copies.
    const float *activity;
    uint2 *pending;
    int *pending_count;
    const float *fields[kMaxSpecies];
    int use_tma;
    int lean;                // take the lean kernel: no length, chemotaxis, connectivity or moment tracking
    int direct;              // a lean model small enough for the direct kernel (one thread per target)
    int compact;             // the direct kernel queues unlike copies before pricing them: 1 per warp, 2 per block
    int direct_span;         // targets a block of the block-queued direct kernel takes (0: 256 a thread-row)
    int max_ctas;            // > 0 caps the persistent grid (each CTA then walks more tiles)
    const void *tensor_map;  // CUtensorMap in device-visible memory, or null
    int *error_flag;
    // A clocked launch (the direct kernel only) takes its step, draws, tally
    // slots and field buffers from `clock` at run time: from this pass's
    // colour, the seed, every tally array and the field buffers.
    const EngineClock *clock;
    uint64_t seed;
    Tallies tal;
    float *field_buf;  // two buffers per species, species-major
};

cudaError_t launch_sweep(const SweepLaunch &a, cudaStream_t stream);

// Every requested MCS of a small lean model with nothing between its passes
// in one cooperative launch (sweep.cu, the resident sweep).
struct ResidentLaunch {
    SweepLaunch a;           // static fields; the pass fields are set per pass
    uint64_t seed;
    int32_t step0;           // the first MCS's step number
    int mcs;                 // MCS to run
    long long pass0;         // the first pass's number (the tally rotation's phase)
    int2 *vs_base[2];
    long long *vs_delta[3];
    unsigned *barrier;       // [0] arrivals, [1] barriers completed; zero at launch
};

// cudaErrorCooperativeLaunchTooLarge (and nothing launched) when the blocks
// cannot all be resident at once.
// Targets a pass from which the direct kernel queues a block's unlike copies
// (kDirectGatherFrom) and from which a warp's (kDirectCompactFrom).
constexpr int kDirectGatherFrom = 1 << 18;
constexpr int kDirectCompactFrom = 1 << 20;

cudaError_t launch_resident_sweep(const ResidentLaunch &r, cudaStream_t stream);
// The same MCS in one thread-block cluster holding a small plane in shared
// memory; cudaErrorNotSupported (nothing launched) when it does not fit one.
cudaError_t launch_cluster_sweep(const ResidentLaunch &r, cudaStream_t stream);

// Every MCS of a call (or one MCS, when fields run between steps) of a large
// lean plane in one cooperative launch: one CTA per SM streams its band of
// rows through shared memory, a grid barrier between passes (band.cu).
// cudaErrorNotSupported (nothing launched) when the plane does not suit it.
cudaError_t launch_band_sweep(const ResidentLaunch &r, cudaStream_t stream);
// Whether a plane of this width and height suits the band sweep on the
// current device (rows whole 16-byte units, a ring of enough rows).
bool band_sweep_fits(int w, int h);

// Apply a motility pass's listed copies: the label, and the activity of a
// type with a maximum (lib.rs:696-698); then clear the list.
cudaError_t launch_apply_copies(const SweepLaunch &a, float *activity, cudaStream_t stream);

// The activity's memory runs down by one each Monte Carlo step
// (lib.rs:426-432, motility.rs).
cudaError_t launch_activity_decay(float *activity, int sites, cudaStream_t stream);

// The batched ensemble: independent replicas of one neighbourhood, all their
// tiles in one persistent launch per colour. Replica state lives in flat
// arrays; each replica's SweepLaunch holds its static fields (geometry,
// tables, absolute label/type/colour-count pointers) and the kernel patches
// the per-pass ones from the clock.
struct EnsembleClock {
    long long step;  // Monte Carlo steps completed
    long long pass;  // colour passes completed
};

struct EnsembleReplica {
    SweepLaunch a;
    long long cell_off;  // first entry of this replica in the flat per-cell arrays
    uint64_t seed;
};

struct EnsembleLaunch {
    int n;             // replicas
    int total_tiles;
    int colour;
    int max_ctas;
    const EnsembleReplica *replicas;
    const void *maps;        // one CUtensorMap per replica (64-byte aligned), or null
    const int *tile_prefix;  // n + 1 entries, in schedule order
    const int *order;        // schedule position -> replica
    const EnsembleClock *clock;
    int2 *vs_base[2];
    long long *vs_delta[3];
    long long total_cells;
    int ncol;
    int uniform_contact_exact;
    int *error_flag;
    // 0: the windowed persistent kernel (128 x 32 tiles); 1, 2, 3: one block
    // per tile of 32 x 8, 16 x 16 or 64 x 4 targets of a plane, priced where
    // they lie (tile_prefix and total_tiles then count those tiles)
    int tile_shape;
    // The colour schedule of the direct shapes: 0 a launch per colour pass;
    // 1 every pass of the step in one cooperative launch, blocks striding
    // over the tiles, a grid barrier (bounded, error flag 4) between passes.
    int one_launch;
    unsigned *barrier;  // [0] arrivals, [1] barriers completed; zero at launch
};

// Targets per tile along x and y of ensemble tile shape `shape` (1, 2, 3).
inline void ensemble_tile(int shape, int &bx, int &by) {
    bx = shape == 1 ? 32 : (shape == 2 ? 16 : 64);
    by = 256 / bx;
}

cudaError_t launch_ensemble_sweep(const EnsembleLaunch &e, int dim, int n_off, bool uniform, cudaStream_t stream);
cudaError_t launch_clock_advance(EnsembleClock *clock, int ncol, cudaStream_t stream);
int ensemble_grid_cap(int dim, int n_off, bool uniform);

struct FieldLaunch {
    Geometry g;
    int n_species;
    int round;
    const float *in[kMaxSpecies];
    float *out[kMaxSpecies];
    float d[kMaxSpecies], decay[kMaxSpecies];
    int active[kMaxSpecies], last[kMaxSpecies];
    const uint32_t *labels;
    const uint8_t *cell_type;
    const float *secretion, *uptake;
    // the infection rule (an extension): the uptake of species infect_species
    // by cells of type infect_from adds into dose[label], in units of 2^-24
    int infect_species = -1;  // -1: no rule
    int infect_from;
    unsigned long long *dose;
    // Clocked: each species' buffers from the clock's current bit and the
    // round (`in`, `out` unused), two per species in field_buf.
    const EngineClock *clock = nullptr;
    float *field_buf = nullptr;
};

cudaError_t launch_field_round(const FieldLaunch &a, cudaStream_t stream);

// A cell of type `from` whose dose has reached `threshold` (units of 2^-24)
// turns to type `to`.
// With `n_live` (device memory) the count is read there and n_labels is the
// capacity.
cudaError_t launch_infection(uint8_t *cell_type, const unsigned long long *dose, int n_labels, int from, int to,
                             long long threshold, const int *n_live, cudaStream_t stream);

// Fixed-point scale of the infection dose: an uptake amount u adds
// rint(u * 2^24), so the sum is exact and its order does not matter.
constexpr float kDoseScale = 16777216.0f;

// Recount every tally from the lattice into base slot `slot`, clearing every
// delta word: volume, per-colour volume, surface, anchor (first site in scan
// order) and the exact moment sums.
struct RecountLaunch {
    Geometry g;
    const uint32_t *labels;
    int n_labels;
    int2 *vs_base;
    long long *mom_base;
    long long *vs_delta[3];
    long long *mom_delta[3];
    int *vol_by_colour;
    int *anchor;
    int tracks;
    const float *nematic;  // with the nematic term: its sums follow the moments
    int *error_flag;  // set to 2 when a label is not below n_labels
    // Population models: the live count in device memory (n_labels is then
    // the capacity), and a device flag the recount runs only when nonzero
    // (the population step's event flag). Null: n_labels, and always.
    const int *n_live;
    const int *when;
};

cudaError_t launch_recount(const RecountLaunch &a, cudaStream_t stream);

// Fold the pending deltas into the base: B[s] += D[pd]; D[pd] = 0.
// With `n_live` (device memory) the count is read there and n_labels is the
// capacity.
cudaError_t launch_settle(int2 *vs_base, long long *vs_delta, long long *mom_base, long long *mom_delta, int nm,
                          int n_labels, int tracks, const int *n_live, cudaStream_t stream);
// The same settle at the end of a clocked step: the slots follow from the
// clock's pass count after the step's `ncol` passes.
cudaError_t launch_settle_clocked(const Tallies &t, int nm, int n_labels, int tracks, const int *n_live,
                                  const EngineClock *clock, int ncol, cudaStream_t stream);
// Advance an engine's clock by one step of `ncol` passes.
cudaError_t launch_engine_clock_advance(EngineClock *clock, int ncol, cudaStream_t stream);

// The medium's volume and unlike-bond surface, counted from the lattice
// (the sweep keeps no tally for label 0).
cudaError_t launch_medium_count(const Geometry &g, const uint32_t *labels, unsigned long long *out,
                                cudaStream_t stream);

struct PopulationLaunch {
    Geometry g;
    TypeTables t;
    uint32_t *labels;
    const uint8_t *cell_type_in;
    uint8_t *cell_type_out;  // may alias cell_type_in
    int n_labels;            // unused: the count lives in n_live
    int cap;
    int *n_live;             // the live label count; decide adds the daughters to it
    const int2 *vs_base;     // settled tallies
    const long long *mom_base;
    const int *anchor;
    uint64_t key_death;      // stream_key(seed, step, kPopulationStream, 0)
    const EngineClock *clock;  // clocked: the step (for the death draws) from here, with `seed`
    uint64_t seed;
    // scratch, n_labels entries each
    unsigned char *mode;
    double *plan;            // 6 per cell: centroid, axis
    int *moved;
    uint32_t *daughter;
    int *counters;           // [0] daughters issued, [1] events (the recount's `when`)
};

// Record the message glz_last_error() returns on this thread.
void set_last_error(const std::string &msg);

}  // namespace glz

struct glz_gpu;

namespace glz {

// An engine's steps replayed inside another graph (the batched ensemble):
// whether its steps replay from a captured graph at all; the clock set from
// its counters before a run of replays; its clocked step as a graph, with the
// version of its per-label arrays the graph holds; before each replay, room
// for that step's divisions (syncing `replays` first when it must read its
// count; a growth changes the version and the graph must be captured anew);
// after each replay, its counters; after the run, its count and error flag.
bool engine_replays(const glz_gpu *h);
int engine_begin_replays(glz_gpu *h);
int engine_step_graph(glz_gpu *h, cudaGraph_t *out, uint64_t *version);
int engine_before_replay(glz_gpu *h, cudaStream_t replays, uint64_t *version);
void engine_after_replay(glz_gpu *h);
int engine_end_replays(glz_gpu *h);

cudaError_t launch_population_plan(const PopulationLaunch &a, cudaStream_t stream);
cudaError_t launch_population_apply(const PopulationLaunch &a, cudaStream_t stream);

}  // namespace glz
