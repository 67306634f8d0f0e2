/*
 * glazier_gpu.h — the C ABI of the B200 Cellular Potts device engine.
 *
 * Every entry point replaces one item of the reference device backend,
 * glazier-cuda/src/lib.rs (`GpuSimulation`, `GpuError`), and the glazier-py
 * `GpuSession` built on it (glazier-py/src/lib.rs:184-241). The citations
 * beside each declaration name the reference item it stands in for.
 *
 * Conventions
 *   - Plain pointers and sizes; the caller owns every buffer it passes.
 *   - Every call returns a status: GLZ_OK, or a code with a message that
 *     glz_last_error() returns for the calling thread.
 *   - One handle owns one CUDA stream on one device. A handle is not safe to
 *     use from two threads at once (the reference `GpuSession` is
 *     `unsendable`); distinct handles are independent and may be driven
 *     from host threads of their own at the same time.
 *   - A model input the device engine would not use (an activity field with
 *     no motility term) is refused at creation with GLZ_UNSUPPORTED, never
 *     dropped silently (lib.rs:819-821).
 */
#ifndef GLAZIER_GPU_H
#define GLAZIER_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. GpuError::OddLattice and GpuError::Driver (lib.rs:723-746)
 * are GLZ_ODD_LATTICE and GLZ_DRIVER; the other two are refusals the
 * reference raises as Driver strings or does not need. */
enum {
    GLZ_OK = 0,
    GLZ_ODD_LATTICE = 1, /* message contains "even sides" (gpu_matches_cpu.rs:146) */
    GLZ_DRIVER = 2,      /* a CUDA call failed */
    GLZ_UNSUPPORTED = 3, /* a model term this engine does not run */
    GLZ_INVALID = 4      /* a bad argument: null pointer, wrong length, bad index */
};

/*
 * The model, as glazier-core/src/model.rs:9-76 states it, flattened.
 * Per-type arrays hold n_types entries with index 0 the medium; the
 * per-type-per-species tables are row-major [type][species]. Pointers the
 * model does not need may be NULL (read as zeros). `nematic` is NULL or
 * 2 * sites values (Q_xx, Q_xy) per site.
 */
typedef struct glz_model {
    int32_t width, height, depth, neighbour_order;
    int32_t n_types, n_species;
    double temperature;
    uint64_t seed;
    const double *contact; /* n_types * n_types, symmetric */
    const double *target_volume, *lambda_volume, *target_surface, *lambda_surface;
    const double *division_volume, *death_rate, *target_length, *lambda_length;
    const uint8_t *connected;
    const double *max_activity, *lambda_activity, *external /* 3 per type */, *lambda_nematic;
    const double *diffusion, *decay, *initial; /* n_species */
    const double *secretion, *uptake, *chemotaxis; /* n_types * n_species */
    const double *nematic;
} glz_model;

typedef struct glz_gpu glz_gpu;

/* Make CUDA device `ordinal` current for this thread's later calls (the
 * reference always takes device 0, lib.rs:823; one process per GPU picks its
 * own). */
int glz_set_device(int ordinal);

/* The message of the last failed call on this thread (`GpuError` Display,
 * lib.rs:730-740). Never NULL. */
const char *glz_last_error(void);

/*
 * Upload a start and build the device state: GpuSimulation::from_cpu
 * (lib.rs:814-1049).
 *   labels     sites = width*height*depth labels, x fastest, 0 the medium
 *   cell_type  n_labels types, index 0 the medium; n_labels > max label
 *   fields     NULL (each species starts at its `initial`) or
 *              n_species * sites concentrations, species-major
 *   activity   NULL (every site starts with none) or sites values, the
 *              motility term's memory; a nonzero one for a model without
 *              the motility term is refused (GLZ_UNSUPPORTED)
 * Refuses odd sides (GLZ_ODD_LATTICE, lib.rs:816-818). Every term of the
 * model runs: contact, volume, surface, length, connectivity, chemotaxis,
 * nematic, motility (Act) and drift, fields, division and death.
 */
int glz_gpu_create(const glz_model *model, const uint32_t *labels, const uint8_t *cell_type, size_t n_labels,
                   const double *fields, const double *activity, glz_gpu **out);

/* Run `steps` Monte Carlo steps and wait for them: GpuSimulation::step
 * (lib.rs:1055-1144). */
int glz_gpu_step(glz_gpu *h, uint64_t steps);

/* Replace the lattice and recount every tally from it, keeping the cell
 * types, fields and step count: a restart from a label field
 * (Simulation::from_labels, glazier-core/src/cpu.rs:151-175, as the
 * Blueprint's `initial.labels` uses it). Labels are checked on the device;
 * one not below the label count fails the next glz_gpu_step. */
int glz_gpu_set_labels(glz_gpu *h, const uint32_t *labels, size_t sites);

/* glz_gpu_set_labels from device memory of the handle's device (uint32 per
 * site): the zero-copy restart for a solver that keeps the lattice on the
 * device. No reference counterpart: the reference restarts from host labels
 * only (Simulation::from_labels, glazier-core/src/cpu.rs:151-175). The caller's writes to `labels` must be complete before the call
 * (its stream synchronized, or the handle's stream made to wait on it); the
 * copy and the recount run on the handle's stream and are done when the call
 * returns. Memory of another device or of the host: GLZ_INVALID. */
int glz_gpu_set_labels_device(glz_gpu *h, const uint32_t *labels, size_t sites);

/* Run `steps` Monte Carlo steps like glz_gpu_step and report the device time
 * of each phase in milliseconds: ms[0] the colour sweeps, ms[1] the field
 * step, ms[2] division and death. No reference counterpart. */
int glz_gpu_step_profiled(glz_gpu *h, uint64_t steps, double ms[3]);

/* Copy the lattice back, `sites` labels: GpuSimulation::labels (lib.rs:1227). */
int glz_gpu_labels(glz_gpu *h, uint32_t *out, size_t sites);

/* Copy species `index` back as f64, `sites` values: GpuSimulation::field
 * (lib.rs:1235-1242). */
int glz_gpu_field(glz_gpu *h, int index, double *out, size_t sites);

/* Per-label volumes, index 0 the medium, clamped at zero:
 * GpuSimulation::volumes (lib.rs:1262-1270). `*count` holds the capacity of
 * `out` on entry and the label count on return; a short buffer is
 * GLZ_INVALID with the needed count in `*count`. */
int glz_gpu_volumes(glz_gpu *h, uint32_t *out, size_t *count);

/* Per-label unlike-bond surfaces: GpuSimulation::surfaces (lib.rs:1248-1256).
 * `*count` as for glz_gpu_volumes. */
int glz_gpu_surfaces(glz_gpu *h, int64_t *out, size_t *count);

/* Per-label cell types (the host mirror `cell_type_host`, lib.rs:799).
 * `*count` as for glz_gpu_volumes. */
int glz_gpu_cell_types(glz_gpu *h, uint8_t *out, size_t *count);

/* The infection rule of the two-field infection model, an extension with no
 * reference counterpart (glazier's types only change by division): after
 * each step's field update, a cell of type `from_type` whose summed uptake of
 * species `species` has reached `threshold` turns to type `to_type`. The
 * uptake is the exchange's upt * v per site (field.rs:133-149), summed per
 * cell in fixed point (units of 2^-24, rounded to nearest per site), so the
 * sum is exact and independent of order. Daughters start at zero. Set it
 * before stepping; it stays for the handle's life. */
int glz_gpu_set_infection(glz_gpu *h, int species, int from_type, int to_type, double threshold);

/* Replace the nematic field, 2 * sites values: GpuSimulation::set_nematic_field
 * (lib.rs:1199-1221); the per-cell field sums are recounted. A field of the
 * wrong length is GLZ_INVALID; a model without a nematic coupling is refused
 * with the reference's message (GLZ_DRIVER, as the reference's Driver). */
int glz_gpu_set_nematic_field(glz_gpu *h, const double *field, size_t len);

/* glz_gpu_set_nematic_field from device memory: 2 f32 per site (q_xx, q_xy),
 * with the same checks, recount and ordering rule as
 * glz_gpu_set_labels_device. The device form of set_nematic_field
 * (glazier-cuda/src/lib.rs:1199-1221), which takes host f64 pairs. The host form rounds its f64 values to f32, so
 * equal f32 values make the same run. */
int glz_gpu_set_nematic_field_device(glz_gpu *h, const float *field, size_t len);

/* Monte Carlo steps completed: `pub mcs` (lib.rs:805). */
uint64_t glz_gpu_mcs(const glz_gpu *h);

/* Labels ever issued, the medium included (`cell_type_host.len()`,
 * lib.rs:1365). */
size_t glz_gpu_n_labels(const glz_gpu *h);

/* The sweep kernel the handle's next step takes: "band", "lean", "direct",
 * "gathered", "compact", "resident", "cluster" or "general" (the engine picks
 * it from the model's terms and the lattice's size; "direct", "gathered" and
 * "compact" take every term, "band", "lean", "resident" and "cluster"
 * contact, volume and surface only, "general" every term through tiles). A diagnostic with no reference
 * counterpart: the reference has one kernel (lib.rs:436-716). Never NULL. */
const char *glz_gpu_sweep_kernel(const glz_gpu *h);

/* The handle's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the engine's. No reference counterpart: the
 * reference keeps its stream private (lib.rs:751). */
void *glz_gpu_stream(glz_gpu *h);

/* Device addresses of the lattice (uint32 per site) and of species `index`
 * (f32 per site), valid until the next glz_gpu_step or glz_gpu_destroy; for
 * a caller that couples another solver on the device (the zero-copy form of
 * GpuSession.labels, glazier-py/src/lib.rs:215-219). */
int glz_gpu_device_labels(glz_gpu *h, void **labels);
int glz_gpu_device_field(glz_gpu *h, int index, void **field);

/* Release the device state: Drop for GpuSimulation. NULL is a no-op. */
void glz_gpu_destroy(glz_gpu *h);

/* ---------------------------------------------------------------- ensemble
 *
 * A batch of independent replicas run as one: every replica whose model
 * prices contact, volume and surface only has its tiles in one persistent
 * launch per colour, one Monte Carlo step replayed from a CUDA graph; a
 * replica whose model states more (fields, length, connectivity, division,
 * death, motility, drift, nematic) runs as its own engine beside the batch,
 * on its own stream from a host thread of its own, over the same steps. No
 * reference counterpart (glazier runs one lattice per GpuSimulation); each
 * replica's results are bit-identical to a glz_gpu_* run of the same start.
 * Replicas may differ in size, parameters and seed; the batched ones share
 * one neighbourhood.
 */
typedef struct glz_ens glz_ens;

/* n replicas: models[i], labels[i] (sites_i labels), cell_types[i]
 * (n_labels[i] types). */
int glz_ens_create(int n, const glz_model *models, const uint32_t *const *labels, const uint8_t *const *cell_types,
                   const size_t *n_labels, glz_ens **out);
/* Run `steps` Monte Carlo steps of every replica and wait. */
int glz_ens_step(glz_ens *h, uint64_t steps);
/* The same, reporting the milliseconds the steps took: the batch's device
 * time, or the call's elapsed time when engine replicas run beside it. */
int glz_ens_step_timed(glz_ens *h, uint64_t steps, double *ms);
/* Labels replica `replica` has issued so far, the medium included (an engine
 * replica's count grows with its divisions); 0 for no such replica. */
size_t glz_ens_n_labels(glz_ens *h, int replica);
/* glz_gpu_set_infection for an engine replica; a batched replica has no
 * fields (GLZ_UNSUPPORTED). */
int glz_ens_set_infection(glz_ens *h, int replica, int species, int from_type, int to_type, double threshold);
/* Time each schedule on a snapshot of the state for `trial_steps` steps,
 * restore the state, keep the fastest: replica order x tile shape (the
 * windowed persistent kernel's 128 x 32 tiles at three grid sizes, and for
 * planes blocks of 32 x 8, 16 x 16 or 64 x 4 targets priced where they lie)
 * x colour schedule for those blocks (a launch per colour pass, or a step's
 * passes in one cooperative launch with a grid barrier between them).
 * `choice` gets the index of the candidate kept. */
int glz_ens_autotune(glz_ens *h, uint64_t trial_steps, int *choice);
/* Choose a schedule directly: bit 0 the replica order (0 as given, 1 largest
 * first), bits 1-2 the tile shape (0 windowed, 1 32 x 8, 2 16 x 16, 3 64 x 4;
 * 1-3 for planes only), bit 3 the step's passes in one launch (shapes 1-3
 * only); max_ctas caps the windowed kernel's grid (0 for one full wave).
 * Results do not depend on it. */
int glz_ens_set_schedule(glz_ens *h, int schedule, int max_ctas);
int glz_ens_labels(glz_ens *h, int replica, uint32_t *out, size_t sites);
int glz_ens_volumes(glz_ens *h, int replica, uint32_t *out, size_t *count);
int glz_ens_surfaces(glz_ens *h, int replica, int64_t *out, size_t *count);
uint64_t glz_ens_mcs(const glz_ens *h);
void *glz_ens_stream(glz_ens *h);
void glz_ens_destroy(glz_ens *h);

/* ---------------------------------------------------------------- field adjoint
 *
 * The chemical-field step differentiated with respect to its parameters,
 * conditioned on a recorded lattice trajectory (the Metropolis sweep itself is
 * never differentiated). No reference counterpart. The forward is the
 * engine's own field step in f32 (one MCS per trajectory step); the backward
 * is its hand-written adjoint, recomputing each segment of `checkpoint_every`
 * steps from a saved state.
 *
 * Parameters, f64, 2 S + 2 T S values: D[S], decay[S], secretion[T][S],
 * uptake[T][S] (S species, T types, row-major). A trajectory is steps * sites
 * owner types, 255 for the medium.
 */
typedef struct glz_adj glz_adj;

int glz_adj_create(int width, int height, int depth, int n_species, int n_types, int steps, int checkpoint_every,
                   glz_adj **out);
/* owner_types: host, steps * sites. */
int glz_adj_set_trajectory(glz_adj *h, const uint8_t *owner_types);
/* fields0, fields_final: device, n_species * sites f32, species-major,
 * distinct buffers. Returns once the fields are written. */
int glz_adj_forward(glz_adj *h, const double *params, const float *fields0, float *fields_final);
/* grad_final: device, the loss gradient at the final fields; grad_params:
 * host, 2 S + 2 T S values; grad_fields0: device or NULL. Uses the
 * parameters of the last forward. Gradients are summed in an order fixed by
 * the lattice, so they are the same bits for every checkpoint interval and
 * every run. */
int glz_adj_backward(glz_adj *h, const float *grad_final, double *grad_params, float *grad_fields0);
/* The CUDA stream (a cudaStream_t) all of the handle's work runs on. */
void *glz_adj_stream(glz_adj *h);
void glz_adj_destroy(glz_adj *h);

/* The most f32 values of intermediate fields glz_field_step_noalloc holds:
 * 4,194,304 (16 MiB), beside a 256-byte status line. */
#define GLZ_NOALLOC_FIELD_SCRATCH (1u << 22)

/*
 * One Monte Carlo step of the chemical-field solver on buffers the caller
 * owns, allocating nothing. No counterpart in the reference: it serves callers
 * that cannot call cudaMalloc, such as a host application that fixes its
 * device-memory budget at start-up and forbids allocation afterwards, or a
 * coupled solver that hands this library only buffers it owns.
 *
 * The arithmetic is the engine's own field step (glz_gpu_step's): per species
 * ceil(D / (1/(2 dim))) sub-steps of FTCS diffusion and decay, secretion and
 * uptake by each site's owner folded into the species' last sub-step. The
 * engine's infection rule (glz_gpu_set_infection) is not part of it: a caller
 * that needs it keeps an engine handle.
 *   width, height, depth   the lattice; n_species 1..8, n_types 1..64
 *   diffusion, decay       host, n_species values each
 *   secretion, uptake      host, n_types * n_species values, [type][species]
 *   labels, cell_type      device: one label per site; n_labels types
 *   fields_in, fields_out  device, n_species * sites f32, species-major;
 *                          two buffers that share no byte (else GLZ_INVALID)
 *   stream                 a cudaStream_t, or NULL for the default stream
 * The work runs on `stream` and the call waits for it. A label at or past
 * n_labels, or a cell type at or past n_types, gets diffusion and decay only
 * and the call returns GLZ_INVALID with the reason, as glz_gpu_step does.
 *
 * The scratch (a status word and up to GLZ_NOALLOC_FIELD_SCRATCH values of
 * intermediate fields: none for one sub-step, one buffer per species for
 * two, two for three or more) lives in one fixed array in device memory that
 * every GPU loading this library holds until the process exits; the rate
 * tables travel in the kernel's parameters. A step needing more scratch is
 * refused with GLZ_INVALID. The first call on a device looks up that array's
 * device address and keeps it for the life of the process (a context that
 * cudaDeviceReset replaces is not followed); make that first call before any
 * stream capture. Every call shares the array, and each clears its status
 * word first; two calls whose work overlaps on the GPU race on it: order them
 * on one stream or wait between them.
 */
int glz_field_step_noalloc(int width, int height, int depth, int n_species, int n_types, const double *diffusion,
                           const double *decay, const double *secretion, const double *uptake,
                           const uint32_t *labels, const uint8_t *cell_type, size_t n_labels,
                           const float *fields_in, float *fields_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GLAZIER_GPU_H */
