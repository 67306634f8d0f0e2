/*
 * ORACLE — test infrastructure, not the product.
 *
 * A plain-C restatement of glazier's serial f64 Cellular Potts engine, the
 * reference's own correctness baseline. Only the tests, the smoke check and
 * the CPU-baseline leg of the benchmark load this file's library; nothing in
 * the glazier_b200 package calls it.
 *
 * Each function names the reference source it follows (paths are inside the
 * glazier repository):
 *   glazier-core/src/rng.rs          xoshiro256++ with SplitMix64 seeding
 *   glazier-core/src/lattice.rs      offsets, wrap, index, coords, tiling
 *   glazier-core/src/moments.rs      running second moments, power iteration
 *   glazier-core/src/connectivity.rs local one-piece test
 *   glazier-core/src/field.rs        FTCS diffusion, decay, exchange
 *   glazier-core/src/motility.rs     Act memory
 *   glazier-core/src/cpu.rs          attempt, step, energy, divide_and_die
 *
 * Arithmetic is IEEE f64 in the reference's operation order, compiled with
 * -ffp-contract=off so no multiply-add is fused, and `exp`/`log`/`sqrt` come
 * from the C library the reference links, so a run reproduces the reference
 * engine bit for bit on the same inputs.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- rng.rs */

typedef struct {
    uint64_t s[4];
} xoshiro;

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* rng.rs:17-29 */
static void xo_seed(xoshiro *r, uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; ++i) {
        z += 0x9E3779B97F4A7C15ULL;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
        r->s[i] = x ^ (x >> 31);
    }
}

/* rng.rs:32-45 */
static uint64_t xo_next(xoshiro *r) {
    uint64_t *s = r->s;
    uint64_t result = rotl(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
}

/* rng.rs:48-50 */
static double xo_f64(xoshiro *r) {
    return (double)(xo_next(r) >> 11) * (1.0 / 9007199254740992.0);
}

/* rng.rs:53-62 */
static uint64_t xo_below(xoshiro *r, uint64_t n) {
    uint64_t zone = UINT64_MAX - (UINT64_MAX % n);
    for (;;) {
        uint64_t v = xo_next(r);
        if (v < zone) return v % n;
    }
}

/* ---------------------------------------------------------------- lattice.rs */

/* lattice.rs:8-60 : ORDER1, ORDER2, ORDER3 */
static const int ORDER1[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
static const int ORDER2[18][3] = {
    {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},   {0, 0, -1},
    {1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1},  {1, 0, -1},
    {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};

static void order3(int out[26][3]) {
    int k = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
                if (dx || dy || dz) {
                    out[k][0] = dx;
                    out[k][1] = dy;
                    out[k][2] = dz;
                    ++k;
                }
}

/* lattice.rs:69-88 */
static int offsets_for(int order, int depth, int out[26][3]) {
    int all3[26][3];
    order3(all3);
    int n = 0;
    if (depth > 1) {
        if (order == 1) {
            memcpy(out, ORDER1, sizeof ORDER1);
            return 6;
        }
        if (order == 2) {
            memcpy(out, ORDER2, sizeof ORDER2);
            return 18;
        }
        memcpy(out, all3, sizeof all3);
        return 26;
    }
    if (order >= 2) {
        for (int k = 0; k < 26; ++k)
            if (all3[k][2] == 0) {
                memcpy(out[n], all3[k], sizeof all3[k]);
                ++n;
            }
        return n;
    }
    for (int k = 0; k < 6; ++k)
        if (ORDER1[k][2] == 0) {
            memcpy(out[n], ORDER1[k], sizeof ORDER1[k]);
            ++n;
        }
    return n;
}

/* lattice.rs:96-111 */
static inline long wrapi(long v, long span) {
    long r = v % span;
    return r < 0 ? r + span : r;
}

typedef struct {
    long w, h, d;
} dims;

/* lattice.rs:205-208 */
static inline long idx(const dims *g, long x, long y, long z) {
    return (wrapi(z, g->d) * g->h + wrapi(y, g->h)) * g->w + wrapi(x, g->w);
}

/* lattice.rs:212-221 */
static inline void coords(const dims *g, long index, long *x, long *y, long *z) {
    long plane = g->w * g->h;
    *z = index / plane;
    long rest = index % plane;
    *x = rest % g->w;
    *y = rest / g->w;
}

/* ---------------------------------------------------------------- moments.rs */

typedef struct {
    double n;
    double s[3];
    double p[6];
    int has_anchor;
    double anchor[3];
} moments;

/* moments.rs:32-52 */
static double fold_about(double v, double a, double span) {
    double out = v;
    if (span > 1.0) {
        if (out - a > span / 2.0)
            out -= span;
        else if (a - out > span / 2.0)
            out += span;
    }
    return out;
}

static void mo_unwrap(const moments *m, double x, double y, double z, const double ext[3], double out[3]) {
    if (!m->has_anchor) {
        out[0] = x;
        out[1] = y;
        out[2] = z;
        return;
    }
    out[0] = fold_about(x, m->anchor[0], ext[0]);
    out[1] = fold_about(y, m->anchor[1], ext[1]);
    out[2] = fold_about(z, m->anchor[2], ext[2]);
}

/* moments.rs:74-88 */
static moments mo_with(const moments *m, const double site[3], double sign) {
    double x = site[0], y = site[1], z = site[2];
    moments out = *m;
    out.n += sign;
    out.s[0] += sign * x;
    out.s[1] += sign * y;
    out.s[2] += sign * z;
    out.p[0] += sign * x * x;
    out.p[1] += sign * y * y;
    out.p[2] += sign * z * z;
    out.p[3] += sign * x * y;
    out.p[4] += sign * x * z;
    out.p[5] += sign * y * z;
    return out;
}

/* moments.rs:55-60 */
static void mo_add(moments *m, const double site[3]) {
    if (!m->has_anchor) {
        m->has_anchor = 1;
        memcpy(m->anchor, site, sizeof m->anchor);
    }
    *m = mo_with(m, site, 1.0);
}

/* moments.rs:63-70 */
static void mo_remove(moments *m, const double site[3]) {
    int had = m->has_anchor;
    double a[3];
    memcpy(a, m->anchor, sizeof a);
    *m = mo_with(m, site, -1.0);
    m->has_anchor = had;
    memcpy(m->anchor, a, sizeof a);
    if (m->n <= 0.0) memset(m, 0, sizeof *m);
}

/* moments.rs:92-104 */
static void mo_cov(const moments *m, double c[3][3]) {
    if (m->n <= 0.0) {
        memset(c, 0, sizeof(double) * 9);
        return;
    }
    double mm[3] = {m->s[0] / m->n, m->s[1] / m->n, m->s[2] / m->n};
    double xx = m->p[0] / m->n - mm[0] * mm[0];
    double yy = m->p[1] / m->n - mm[1] * mm[1];
    double zz = m->p[2] / m->n - mm[2] * mm[2];
    double xy = m->p[3] / m->n - mm[0] * mm[1];
    double xz = m->p[4] / m->n - mm[0] * mm[2];
    double yz = m->p[5] / m->n - mm[1] * mm[2];
    c[0][0] = xx; c[0][1] = xy; c[0][2] = xz;
    c[1][0] = xy; c[1][1] = yy; c[1][2] = yz;
    c[2][0] = xz; c[2][1] = yz; c[2][2] = zz;
}

/* moments.rs:165-186 */
static double principal_axis(double c[3][3], double v[3]) {
    v[0] = 1.0; v[1] = 0.7; v[2] = 0.3;
    double w[3];
    for (int round = 0; round < 20; ++round) {
        for (int i = 0; i < 3; ++i) w[i] = c[i][0] * v[0] + c[i][1] * v[1] + c[i][2] * v[2];
        double norm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (norm < 1e-15) {
            v[0] = 1.0; v[1] = 0.0; v[2] = 0.0;
            return 0.0;
        }
        v[0] = w[0] / norm; v[1] = w[1] / norm; v[2] = w[2] / norm;
    }
    for (int i = 0; i < 3; ++i) w[i] = c[i][0] * v[0] + c[i][1] * v[1] + c[i][2] * v[2];
    double lambda = v[0] * w[0] + v[1] * w[1] + v[2] * w[2];
    return lambda > 0.0 ? lambda : 0.0;
}

/* moments.rs:150-155 */
static double mo_length(const moments *m) {
    if (m->n < 2.0) return 0.0;
    double c[3][3], v[3];
    mo_cov(m, c);
    return 4.0 * sqrt(principal_axis(c, v));
}

/* moments.rs:131-141 */
static void mo_anisotropy(const moments *m, double *a0, double *a1) {
    *a0 = 0.0;
    *a1 = 0.0;
    if (m->n < 2.0) return;
    double c[3][3];
    mo_cov(m, c);
    double trace = c[0][0] + c[1][1];
    if (trace <= 1e-12) return;
    *a0 = (c[0][0] - c[1][1]) / trace;
    *a1 = 2.0 * c[0][1] / trace;
}

/* ---------------------------------------------------------------- model */

/* The model as glazier-core/src/model.rs:9-76 states it, flattened. Per-type
 * arrays have n_types entries with index 0 the medium; per-type-per-species
 * arrays are row-major [type][species]. */
typedef struct {
    int32_t width, height, depth, neighbour_order;
    int32_t n_types, n_species;
    double temperature;
    uint64_t seed;
    const double *contact;
    const double *target_volume, *lambda_volume, *target_surface, *lambda_surface;
    const double *division_volume, *death_rate, *target_length, *lambda_length;
    const uint8_t *connected;
    const double *max_activity, *lambda_activity, *external, *lambda_nematic;
    const double *diffusion, *decay, *initial;
    const double *secretion, *uptake, *chemotaxis;
    const double *nematic; /* 2 per site, or NULL */
} orc_model;

typedef struct {
    double target_volume, lambda_volume, target_surface, lambda_surface;
    double division_volume, death_rate, target_length, lambda_length;
    int connected;
    double max_activity, lambda_activity, external[3], lambda_nematic;
} ctype;

typedef struct {
    dims g;
    long sites;
    int n_types, n_species, order;
    double temperature;
    uint64_t seed;
    double *contact;
    ctype *types;
    double *diffusion, *decay;
    double *secretion, *uptake, *chemotaxis;
    double *nematic;
    int n_off;
    int off[26][3];
    int ring_n;
    int ring[26][3];
    int tracks_moments, has_nematic, has_motility, has_population, has_chemotaxis_rows;

    uint32_t *labels;
    size_t n_labels, cap;
    uint32_t *volume;
    int64_t *surface;
    uint8_t *cell_type;
    moments *mom;
    double (*nsum)[2];
    double *activity;
    double *fields; /* species-major */
    int *substeps;
    double *scratch;
    xoshiro rng;
    uint64_t mcs, accepted, attempted;
} osim;

static char last_error[512];

EXPORT const char *orc_last_error(void) { return last_error; }

static double *dupd(const double *src, size_t n) {
    double *out = (double *)calloc(n ? n : 1, sizeof(double));
    if (src && n) memcpy(out, src, n * sizeof(double));
    return out;
}

/* field.rs:155-160 */
EXPORT int orc_substeps_for(double diffusion, int dimensions) {
    if (diffusion <= 0.0) return 1;
    double limit = 1.0 / (2.0 * (double)(dimensions > 1 ? dimensions : 1));
    double k = ceil(diffusion / limit);
    return k < 1.0 ? 1 : (int)k;
}

static inline double contact_energy(const osim *s, int a, int b) { return s->contact[a * s->n_types + b]; }
static inline const ctype *type_of(const osim *s, uint32_t label) { return &s->types[s->cell_type[label]]; }

static void reserve(osim *s, size_t want) {
    if (want <= s->cap) return;
    size_t cap = s->cap ? s->cap : 16;
    while (cap < want) cap *= 2;
    s->volume = (uint32_t *)realloc(s->volume, cap * sizeof *s->volume);
    s->surface = (int64_t *)realloc(s->surface, cap * sizeof *s->surface);
    s->cell_type = (uint8_t *)realloc(s->cell_type, cap * sizeof *s->cell_type);
    s->mom = (moments *)realloc(s->mom, cap * sizeof *s->mom);
    s->nsum = (double(*)[2])realloc(s->nsum, cap * sizeof *s->nsum);
    s->cap = cap;
}

static void extent(const osim *s, double ext[3]) {
    ext[0] = (double)s->g.w;
    ext[1] = (double)s->g.h;
    ext[2] = (double)s->g.d;
}

/* cpu.rs:46-59 */
static void count_surface(const osim *s, int64_t *out, size_t labels) {
    memset(out, 0, labels * sizeof *out);
    for (long i = 0; i < s->sites; ++i) {
        long x, y, z;
        coords(&s->g, i, &x, &y, &z);
        uint32_t l = s->labels[i];
        for (int k = 0; k < s->n_off; ++k) {
            long n = idx(&s->g, x + s->off[k][0], y + s->off[k][1], z + s->off[k][2]);
            if (n != i && s->labels[n] != l) out[l] += 1;
        }
    }
}

/* cpu.rs:11-21 */
static void count_moments(const osim *s, moments *out, size_t labels) {
    memset(out, 0, labels * sizeof *out);
    double ext[3];
    extent(s, ext);
    for (long i = 0; i < s->sites; ++i) {
        uint32_t l = s->labels[i];
        long x, y, z;
        coords(&s->g, i, &x, &y, &z);
        double site[3];
        mo_unwrap(&out[l], (double)x, (double)y, (double)z, ext, site);
        mo_add(&out[l], site);
    }
}

/* cpu.rs:24-34 */
static void count_nematic(const osim *s, double (*out)[2], size_t labels) {
    memset(out, 0, labels * sizeof *out);
    if (!s->nematic) return;
    for (long i = 0; i < s->sites; ++i) {
        out[s->labels[i]][0] += s->nematic[2 * i];
        out[s->labels[i]][1] += s->nematic[2 * i + 1];
    }
}

/* model.rs:160-232, only the checks an engine relies on */
static int validate(const orc_model *m) {
    int n = m->n_types;
    if (n == 0) {
        snprintf(last_error, sizeof last_error, "a model needs at least the medium type");
        return 0;
    }
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            if (fabs(m->contact[a * n + b] - m->contact[b * n + a]) > 1e-12) {
                snprintf(last_error, sizeof last_error, "contact matrix is asymmetric at (%d, %d)", a, b);
                return 0;
            }
    if (m->width <= 0 || m->height <= 0 || m->depth <= 0) {
        snprintf(last_error, sizeof last_error, "the lattice has a zero dimension");
        return 0;
    }
    if (m->neighbour_order < 1 || m->neighbour_order > 3) {
        snprintf(last_error, sizeof last_error, "neighbour order %d is outside the range one to three", m->neighbour_order);
        return 0;
    }
    if (m->temperature <= 0.0) {
        snprintf(last_error, sizeof last_error, "the temperature must be positive");
        return 0;
    }
    return 1;
}

/* lattice.rs:169-196 */
static uint32_t tile_grid(osim *s, long side, long nx, long ny, long nz) {
    uint32_t next = 1;
    if (nx > s->g.w / side) nx = s->g.w / side;
    if (ny > s->g.h / side) ny = s->g.h / side;
    if (s->g.d == 1)
        nz = 1;
    else if (nz > s->g.d / side)
        nz = s->g.d / side;
    long side_z = s->g.d == 1 ? 1 : side;
    for (long bz = 0; bz < nz; ++bz)
        for (long by = 0; by < ny; ++by)
            for (long bx = 0; bx < nx; ++bx) {
                for (long z = bz * side_z; z < (bz + 1) * side_z; ++z)
                    for (long y = by * side; y < (by + 1) * side; ++y)
                        for (long x = bx * side; x < (bx + 1) * side; ++x) s->labels[idx(&s->g, x, y, z)] = next;
                ++next;
            }
    return next - 1;
}

/*
 * cpu.rs:122-217: build a run from the model and either a label field
 * (from_labels) or a grid of squares (tiled_grid, when labels is NULL).
 */
EXPORT osim *orc_create(const orc_model *m, const uint32_t *labels, long side, long nx, long ny, long nz) {
    if (!validate(m)) return NULL;
    if (m->n_types < 2) {
        snprintf(last_error, sizeof last_error, "a start needs a cell type beside the medium");
        return NULL;
    }
    osim *s = (osim *)calloc(1, sizeof *s);
    s->g.w = m->width;
    s->g.h = m->height;
    s->g.d = m->depth;
    s->sites = s->g.w * s->g.h * s->g.d;
    s->n_types = m->n_types;
    s->n_species = m->n_species;
    s->order = m->neighbour_order;
    s->temperature = m->temperature;
    s->seed = m->seed;
    int nt = m->n_types, ns = m->n_species;
    s->contact = dupd(m->contact, (size_t)nt * nt);
    s->types = (ctype *)calloc(nt, sizeof *s->types);
    for (int t = 0; t < nt; ++t) {
        ctype *c = &s->types[t];
#define TAKE(f) c->f = m->f ? m->f[t] : 0.0
        TAKE(target_volume); TAKE(lambda_volume); TAKE(target_surface); TAKE(lambda_surface);
        TAKE(division_volume); TAKE(death_rate); TAKE(target_length); TAKE(lambda_length);
        TAKE(max_activity); TAKE(lambda_activity); TAKE(lambda_nematic);
#undef TAKE
        c->connected = m->connected ? m->connected[t] != 0 : 0;
        for (int a = 0; a < 3; ++a) c->external[a] = m->external ? m->external[3 * t + a] : 0.0;
    }
    s->diffusion = dupd(m->diffusion, ns);
    s->decay = dupd(m->decay, ns);
    s->secretion = dupd(m->secretion, (size_t)nt * ns);
    s->uptake = dupd(m->uptake, (size_t)nt * ns);
    s->chemotaxis = dupd(m->chemotaxis, (size_t)nt * ns);
    s->nematic = m->nematic ? dupd(m->nematic, 2 * (size_t)s->sites) : NULL;
    s->n_off = offsets_for(m->neighbour_order, m->depth, s->off);

    int has_conn = 0, has_len = 0, has_nem_type = 0, has_mot = 0, has_pop = 0;
    for (int t = 0; t < nt; ++t) {
        has_conn |= s->types[t].connected;
        has_len |= s->types[t].lambda_length != 0.0;
        has_nem_type |= s->types[t].lambda_nematic != 0.0;
        has_mot |= s->types[t].lambda_activity != 0.0 && s->types[t].max_activity > 0.0;
        has_pop |= s->types[t].division_volume > 0.0 || s->types[t].death_rate > 0.0;
    }
    s->has_nematic = s->nematic != NULL && has_nem_type;   /* model.rs:122-124 */
    s->tracks_moments = has_len || s->has_nematic;         /* model.rs:129-131 */
    s->has_motility = has_mot;                             /* model.rs:93-97 */
    s->has_population = has_pop;                           /* model.rs:144-148 */
    s->ring_n = 0;
    if (has_conn) { /* connectivity.rs:23-29 */
        int all3[26][3];
        order3(all3);
        for (int k = 0; k < 26; ++k)
            if (m->depth > 1 || all3[k][2] == 0) {
                memcpy(s->ring[s->ring_n], all3[k], sizeof all3[k]);
                ++s->ring_n;
            }
    }

    s->labels = (uint32_t *)calloc(s->sites, sizeof *s->labels);
    size_t n;
    if (labels) {
        memcpy(s->labels, labels, s->sites * sizeof *labels);
        uint32_t mx = 0;
        for (long i = 0; i < s->sites; ++i)
            if (labels[i] > mx) mx = labels[i];
        if (mx == 0) {
            snprintf(last_error, sizeof last_error, "the label field holds no cells");
            free(s->labels);
            free(s);
            return NULL;
        }
        n = mx;
    } else {
        n = tile_grid(s, side, nx, ny, nz);
    }
    /* cpu.rs:178-217 assemble */
    s->n_labels = n + 1;
    reserve(s, s->n_labels);
    memset(s->volume, 0, s->n_labels * sizeof *s->volume);
    for (long i = 0; i < s->sites; ++i) s->volume[s->labels[i]] += 1;
    count_surface(s, s->surface, s->n_labels);
    count_moments(s, s->mom, s->n_labels);
    count_nematic(s, s->nsum, s->n_labels);
    memset(s->cell_type, 1, s->n_labels);
    s->activity = (double *)calloc(s->sites, sizeof(double));
    s->fields = (double *)calloc((size_t)(ns ? ns : 1) * s->sites, sizeof(double));
    s->substeps = (int *)calloc(ns ? ns : 1, sizeof(int));
    int dimensions = s->g.d > 1 ? 3 : 2;
    for (int k = 0; k < ns; ++k) {
        double init = m->initial ? m->initial[k] : 0.0;
        for (long i = 0; i < s->sites; ++i) s->fields[(size_t)k * s->sites + i] = init;
        s->substeps[k] = orc_substeps_for(s->diffusion[k], dimensions);
    }
    s->scratch = (double *)calloc(s->sites, sizeof(double));
    xo_seed(&s->rng, m->seed);
    return s;
}

EXPORT void orc_destroy(osim *s) {
    if (!s) return;
    free(s->contact); free(s->types); free(s->diffusion); free(s->decay);
    free(s->secretion); free(s->uptake); free(s->chemotaxis); free(s->nematic);
    free(s->labels); free(s->volume); free(s->surface); free(s->cell_type);
    free(s->mom); free(s->nsum); free(s->activity); free(s->fields);
    free(s->substeps); free(s->scratch);
    free(s);
}

/* cpu.rs:220-224 */
EXPORT void orc_set_cell_types(osim *s, const uint8_t *types, size_t n) {
    for (size_t i = 0; i < n && i + 1 < s->n_labels; ++i) s->cell_type[i + 1] = types[i];
}

/* ---------------------------------------------------------------- connectivity.rs */

/* connectivity.rs:43-84 */
static int locally_connected(const osim *s, long target, uint32_t label) {
    long x, y, z;
    coords(&s->g, target, &x, &y, &z);
    int members[26][3];
    int count = 0;
    for (int k = 0; k < s->ring_n; ++k) {
        long site = idx(&s->g, x + s->ring[k][0], y + s->ring[k][1], z + s->ring[k][2]);
        if (site != target && s->labels[site] == label) {
            memcpy(members[count], s->ring[k], sizeof members[count]);
            ++count;
        }
    }
    if (count <= 1) return 1;
    int seen[26] = {0};
    int stack[26];
    int top = 1, reached = 1;
    stack[0] = 0;
    seen[0] = 1;
    while (top > 0) {
        --top;
        int here = stack[top];
        for (int other = 0; other < count; ++other) {
            if (seen[other]) continue;
            int dx = members[here][0] - members[other][0];
            int dy = members[here][1] - members[other][1];
            int dz = members[here][2] - members[other][2];
            if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) {
                seen[other] = 1;
                stack[top] = other;
                ++top;
                ++reached;
            }
        }
    }
    return reached == count;
}

/* ---------------------------------------------------------------- energy terms, cpu.rs */

static inline double sq(double v) { return v * v; }

/* cpu.rs:413-425 */
static double volume_term(const osim *s, uint32_t label, long change) {
    if (label == 0) return 0.0;
    const ctype *t = type_of(s, label);
    if (t->lambda_volume == 0.0) return 0.0;
    double v = (double)s->volume[label];
    double after = v + (double)change;
    return t->lambda_volume * (sq(after - t->target_volume) - sq(v - t->target_volume));
}

/* cpu.rs:399-411 */
static double surface_term(const osim *s, uint32_t label, long change) {
    if (label == 0 || change == 0) return 0.0;
    const ctype *t = type_of(s, label);
    if (t->lambda_surface == 0.0) return 0.0;
    double sv = (double)s->surface[label];
    double after = sv + (double)change;
    return t->lambda_surface * (sq(after - t->target_surface) - sq(sv - t->target_surface));
}

/* cpu.rs:291-305 */
static double length_term(const osim *s, uint32_t label, const double site[3], double sign) {
    if (label == 0) return 0.0;
    const ctype *t = type_of(s, label);
    if (t->lambda_length == 0.0) return 0.0;
    const moments *m = &s->mom[label];
    double ext[3], u[3];
    extent(s, ext);
    mo_unwrap(m, site[0], site[1], site[2], ext, u);
    double before = mo_length(m);
    moments w = mo_with(m, u, sign);
    double after = mo_length(&w);
    return t->lambda_length * (sq(after - t->target_length) - sq(before - t->target_length));
}

/* cpu.rs:315-332 */
static double nematic_term(const osim *s, uint32_t label, long index, const double site[3], double sign) {
    if (label == 0) return 0.0;
    const ctype *t = type_of(s, label);
    if (t->lambda_nematic == 0.0) return 0.0;
    const moments *m = &s->mom[label];
    double ext[3], u[3];
    extent(s, ext);
    mo_unwrap(m, site[0], site[1], site[2], ext, u);
    double a0, a1, b0, b1;
    mo_anisotropy(m, &a0, &a1);
    moments w = mo_with(m, u, sign);
    mo_anisotropy(&w, &b0, &b1);
    const double *f = s->nsum[label];
    const double *q = &s->nematic[2 * index];
    double before = f[0] * a0 + f[1] * a1;
    double after = (f[0] + sign * q[0]) * b0 + (f[1] + sign * q[1]) * b1;
    return -t->lambda_nematic * (after - before);
}

/* cpu.rs:242-288 */
EXPORT double orc_delta_energy(const osim *s, long target, uint32_t newl) {
    uint32_t old = s->labels[target];
    if (old == newl) return 0.0;
    long tx, ty, tz;
    coords(&s->g, target, &tx, &ty, &tz);
    int told = s->cell_type[old], tnew = s->cell_type[newl];
    double delta = 0.0;
    long like_old = 0, like_new = 0, bonds = 0;
    for (int k = 0; k < s->n_off; ++k) {
        long n = idx(&s->g, tx + s->off[k][0], ty + s->off[k][1], tz + s->off[k][2]);
        if (n == target) continue;
        bonds += 1;
        uint32_t ln = s->labels[n];
        int tn = s->cell_type[ln];
        if (ln != old)
            delta -= contact_energy(s, told, tn);
        else
            like_old += 1;
        if (ln != newl)
            delta += contact_energy(s, tnew, tn);
        else
            like_new += 1;
    }
    delta += volume_term(s, old, -1);
    delta += volume_term(s, newl, 1);
    if (s->tracks_moments) {
        double site[3] = {(double)tx, (double)ty, (double)tz};
        delta += length_term(s, old, site, -1.0);
        delta += length_term(s, newl, site, 1.0);
        if (s->has_nematic) {
            delta += nematic_term(s, old, target, site, -1.0);
            delta += nematic_term(s, newl, target, site, 1.0);
        }
    }
    delta += surface_term(s, old, 2 * like_old - bonds);
    delta += surface_term(s, newl, bonds - 2 * like_new);
    return delta;
}

/* motility.rs:58-79 */
static double neighbourhood_mean(const osim *s, long site, uint32_t label) {
    long x, y, z;
    coords(&s->g, site, &x, &y, &z);
    double here = s->activity[site];
    double log_sum = log(here > 0.0 ? here : 0.0);
    double count = 1.0;
    for (int k = 0; k < s->n_off; ++k) {
        long n = idx(&s->g, x + s->off[k][0], y + s->off[k][1], z + s->off[k][2]);
        if (n == site || s->labels[n] != label) continue;
        double value = s->activity[n];
        if (value <= 0.0) return 0.0;
        log_sum += log(value);
        count += 1.0;
    }
    if (!isfinite(log_sum)) return 0.0;
    return exp(log_sum / count);
}

/* cpu.rs:341-371 */
static double move_work(const osim *s, uint32_t newl, uint32_t old, long target, long source) {
    double work = 0.0;
    if (newl != 0) {
        const ctype *t = type_of(s, newl);
        if (t->lambda_activity != 0.0 && t->max_activity > 0.0) {
            double into = neighbourhood_mean(s, source, newl);
            double out_of = neighbourhood_mean(s, target, old);
            work -= t->lambda_activity / t->max_activity * (into - out_of);
        }
        if (t->external[0] != 0.0 || t->external[1] != 0.0 || t->external[2] != 0.0) {
            long tx, ty, tz, sx, sy, sz;
            coords(&s->g, target, &tx, &ty, &tz);
            coords(&s->g, source, &sx, &sy, &sz);
            double spans[3] = {(double)s->g.w, (double)s->g.h, (double)s->g.d};
            long a[3] = {tx, ty, tz}, b[3] = {sx, sy, sz};
            double st[3];
            for (int i = 0; i < 3; ++i) {
                double raw = (double)(a[i] - b[i]);
                if (raw > spans[i] / 2.0)
                    st[i] = raw - spans[i];
                else if (raw < -spans[i] / 2.0)
                    st[i] = raw + spans[i];
                else
                    st[i] = raw;
            }
            work -= t->external[0] * st[0] + t->external[1] * st[1] + t->external[2] * st[2];
        }
    }
    return work;
}

/* cpu.rs:381-395 */
static double chemotaxis_work(const osim *s, uint32_t newl, long target, long source) {
    if (newl == 0 || s->n_species == 0) return 0.0;
    const double *row = &s->chemotaxis[(size_t)s->cell_type[newl] * s->n_species];
    double work = 0.0;
    for (int k = 0; k < s->n_species; ++k) {
        double lambda = row[k];
        if (lambda == 0.0) continue;
        const double *values = &s->fields[(size_t)k * s->sites];
        work -= lambda * (values[target] - values[source]);
    }
    return work;
}

/* cpu.rs:432-517 */
EXPORT int orc_attempt(osim *s) {
    uint64_t sites = (uint64_t)s->sites;
    long target = (long)xo_below(&s->rng, sites);
    int pick = (int)xo_below(&s->rng, (uint64_t)s->n_off);
    long tx, ty, tz;
    coords(&s->g, target, &tx, &ty, &tz);
    long source = idx(&s->g, tx + s->off[pick][0], ty + s->off[pick][1], tz + s->off[pick][2]);
    uint32_t old = s->labels[target], newl = s->labels[source];
    s->attempted += 1;
    if (old == newl) return 0;
    if (old != 0 && s->volume[old] <= 1) return 0;
    if (old != 0 && s->ring_n > 0 && type_of(s, old)->connected && !locally_connected(s, target, old)) return 0;

    double delta = orc_delta_energy(s, target, newl) + chemotaxis_work(s, newl, target, source) +
                   move_work(s, newl, old, target, source);
    int accept = delta <= 0.0 || xo_f64(&s->rng) < exp(-delta / s->temperature);
    if (!accept) return 0;

    long like_old = 0, like_new = 0, bonds = 0;
    for (int k = 0; k < s->n_off; ++k) {
        long n = idx(&s->g, tx + s->off[k][0], ty + s->off[k][1], tz + s->off[k][2]);
        if (n == target) continue;
        bonds += 1;
        uint32_t ln = s->labels[n];
        if (ln == old) like_old += 1;
        if (ln == newl) like_new += 1;
    }
    s->surface[old] += 2 * like_old - bonds;
    s->surface[newl] += bonds - 2 * like_new;
    if (s->has_nematic) {
        const double *q = &s->nematic[2 * target];
        s->nsum[old][0] -= q[0];
        s->nsum[old][1] -= q[1];
        s->nsum[newl][0] += q[0];
        s->nsum[newl][1] += q[1];
    }
    if (s->tracks_moments) {
        double ext[3], leaving[3], joining[3];
        extent(s, ext);
        mo_unwrap(&s->mom[old], (double)tx, (double)ty, (double)tz, ext, leaving);
        mo_remove(&s->mom[old], leaving);
        mo_unwrap(&s->mom[newl], (double)tx, (double)ty, (double)tz, ext, joining);
        mo_add(&s->mom[newl], joining);
    }
    if (newl != 0) {
        const ctype *t = type_of(s, newl);
        if (t->max_activity > 0.0) s->activity[target] = t->max_activity;
    }
    s->labels[target] = newl;
    s->volume[old] -= 1;
    s->volume[newl] += 1;
    s->accepted += 1;
    return 1;
}

/* field.rs:99-130 */
static void fields_diffuse(osim *s) {
    int n_faces = s->g.d > 1 ? 6 : 4;
    for (int k = 0; k < s->n_species; ++k) {
        int steps = s->substeps[k];
        double d = s->diffusion[k] / (double)steps;
        double decay = s->decay[k] / (double)steps;
        double *values = &s->fields[(size_t)k * s->sites];
        for (int r = 0; r < steps; ++r) {
            for (long here = 0; here < s->sites; ++here) {
                long x, y, z;
                coords(&s->g, here, &x, &y, &z);
                double laplacian = -(double)n_faces * values[here];
                for (int f = 0; f < n_faces; ++f)
                    laplacian += values[idx(&s->g, x + ORDER1[f][0], y + ORDER1[f][1], z + ORDER1[f][2])];
                s->scratch[here] = values[here] + d * laplacian - decay * values[here];
            }
            memcpy(values, s->scratch, s->sites * sizeof(double));
        }
    }
}

/* field.rs:133-149 */
static void fields_exchange(osim *s) {
    for (int k = 0; k < s->n_species; ++k) {
        double *values = &s->fields[(size_t)k * s->sites];
        for (long site = 0; site < s->sites; ++site) {
            uint32_t label = s->labels[site];
            if (label == 0) continue;
            int t = s->cell_type[label];
            double secreted = s->secretion[(size_t)t * s->n_species + k];
            double taken = s->uptake[(size_t)t * s->n_species + k];
            values[site] += secreted;
            values[site] -= taken * values[site];
            if (values[site] < 0.0) values[site] = 0.0;
        }
    }
}

/* cpu.rs:659-673 and 679-712 */
static int divide(osim *s, uint32_t label) {
    double ext[3];
    extent(s, ext);
    moments m;
    memset(&m, 0, sizeof m);
    long count = 0;
    for (long i = 0; i < s->sites; ++i)
        if (s->labels[i] == label) ++count;
    if (count < 4) return 0;
    long *where = (long *)malloc(count * sizeof(long));
    double(*u)[3] = (double(*)[3])malloc(count * sizeof *u);
    long j = 0;
    for (long i = 0; i < s->sites; ++i) {
        if (s->labels[i] != label) continue;
        long x, y, z;
        coords(&s->g, i, &x, &y, &z);
        mo_unwrap(&m, (double)x, (double)y, (double)z, ext, u[j]);
        mo_add(&m, u[j]);
        where[j] = i;
        ++j;
    }
    double centre[3] = {m.s[0] / m.n, m.s[1] / m.n, m.s[2] / m.n};
    double c[3][3], axis[3];
    mo_cov(&m, c);
    principal_axis(c, axis);
    uint32_t daughter = (uint32_t)s->n_labels;
    uint32_t moved = 0;
    for (long k = 0; k < count; ++k) {
        double along = (u[k][0] - centre[0]) * axis[0] + (u[k][1] - centre[1]) * axis[1] + (u[k][2] - centre[2]) * axis[2];
        if (along > 0.0) {
            s->labels[where[k]] = daughter;
            ++moved;
        }
    }
    int ok = 1;
    if (moved == 0 || (long)moved == count) {
        for (long k = 0; k < count; ++k) s->labels[where[k]] = label;
        ok = 0;
    } else {
        reserve(s, s->n_labels + 1);
        s->volume[label] -= moved;
        s->volume[s->n_labels] = moved;
        s->surface[s->n_labels] = 0;
        memset(&s->mom[s->n_labels], 0, sizeof(moments));
        s->nsum[s->n_labels][0] = 0.0;
        s->nsum[s->n_labels][1] = 0.0;
        s->cell_type[s->n_labels] = s->cell_type[label];
        s->n_labels += 1;
    }
    free(where);
    free(u);
    return ok;
}

/* cpu.rs:715-725 */
static void kill(osim *s, uint32_t label) {
    for (long i = 0; i < s->sites; ++i)
        if (s->labels[i] == label) s->labels[i] = 0;
    uint32_t gone = s->volume[label];
    s->volume[label] = 0;
    s->volume[0] += gone;
    s->surface[label] = 0;
}

/* cpu.rs:620-655 */
EXPORT void orc_divide_and_die(osim *s, int *divided_out, int *died_out) {
    int divided = 0, died = 0;
    size_t n = s->n_labels;
    uint32_t *live = (uint32_t *)malloc(n * sizeof(uint32_t));
    size_t nl = 0;
    for (uint32_t l = 1; l < n; ++l)
        if (s->volume[l] > 0) live[nl++] = l;
    for (size_t k = 0; k < nl; ++k) {
        uint32_t l = live[k];
        const ctype *t = type_of(s, l);
        if (t->division_volume > 0.0 && (double)s->volume[l] >= t->division_volume && divide(s, l)) ++divided;
    }
    n = s->n_labels;
    live = (uint32_t *)realloc(live, n * sizeof(uint32_t));
    nl = 0;
    for (uint32_t l = 1; l < n; ++l)
        if (s->volume[l] > 0) live[nl++] = l;
    for (size_t k = 0; k < nl; ++k) {
        uint32_t l = live[k];
        const ctype *t = type_of(s, l);
        if (t->death_rate > 0.0 && xo_f64(&s->rng) < t->death_rate) {
            kill(s, l);
            ++died;
        }
    }
    free(live);
    if (divided > 0 || died > 0) {
        count_surface(s, s->surface, s->n_labels);
        count_moments(s, s->mom, s->n_labels);
        count_nematic(s, s->nsum, s->n_labels);
    }
    if (divided_out) *divided_out = divided;
    if (died_out) *died_out = died;
}

/* cpu.rs:522-538 */
EXPORT void orc_step(osim *s, uint64_t steps) {
    for (uint64_t r = 0; r < steps; ++r) {
        for (long i = 0; i < s->sites; ++i) orc_attempt(s);
        if (s->n_species > 0) {
            fields_diffuse(s);
            fields_exchange(s);
        }
        if (s->has_motility)
            for (long i = 0; i < s->sites; ++i)
                if (s->activity[i] > 0.0) s->activity[i] -= 1.0;
        if (s->has_population) orc_divide_and_die(s, NULL, NULL);
        s->mcs += 1;
    }
}

/* Copy-in attempts with a budget, for a bounded timing sample. */
EXPORT void orc_attempts(osim *s, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) orc_attempt(s);
}

/* cpu.rs:545-581 */
EXPORT double orc_energy(const osim *s) {
    double contact = 0.0;
    for (long i = 0; i < s->sites; ++i) {
        long x, y, z;
        coords(&s->g, i, &x, &y, &z);
        uint32_t l = s->labels[i];
        for (int k = 0; k < s->n_off; ++k) {
            long n = idx(&s->g, x + s->off[k][0], y + s->off[k][1], z + s->off[k][2]);
            uint32_t ln = s->labels[n];
            if (ln != l) contact += contact_energy(s, s->cell_type[l], s->cell_type[ln]);
        }
    }
    contact /= 2.0;
    double volume = 0.0, surface = 0.0, length = 0.0, nematic = 0.0;
    int64_t *counted = (int64_t *)malloc(s->n_labels * sizeof(int64_t));
    count_surface(s, counted, s->n_labels);
    for (size_t l = 1; l < s->n_labels; ++l) {
        const ctype *t = type_of(s, (uint32_t)l);
        volume += t->lambda_volume * sq((double)s->volume[l] - t->target_volume);
        if (t->lambda_length != 0.0) length += t->lambda_length * sq(mo_length(&s->mom[l]) - t->target_length);
        surface += t->lambda_surface * sq((double)counted[l] - t->target_surface);
        if (s->has_nematic && t->lambda_nematic != 0.0) {
            double a0, a1;
            mo_anisotropy(&s->mom[l], &a0, &a1);
            nematic -= t->lambda_nematic * (s->nsum[l][0] * a0 + s->nsum[l][1] * a1);
        }
    }
    free(counted);
    return contact + volume + surface + length + nematic;
}

/* ---------------------------------------------------------------- accessors */

EXPORT long orc_sites(const osim *s) { return s->sites; }
EXPORT size_t orc_n_labels(const osim *s) { return s->n_labels; }
EXPORT uint64_t orc_mcs(const osim *s) { return s->mcs; }
EXPORT uint64_t orc_accepted(const osim *s) { return s->accepted; }
EXPORT uint64_t orc_attempted(const osim *s) { return s->attempted; }
EXPORT void orc_labels(const osim *s, uint32_t *out) { memcpy(out, s->labels, s->sites * sizeof *out); }
EXPORT void orc_volumes(const osim *s, uint32_t *out) { memcpy(out, s->volume, s->n_labels * sizeof *out); }
EXPORT void orc_surfaces(const osim *s, int64_t *out) { memcpy(out, s->surface, s->n_labels * sizeof *out); }
EXPORT void orc_cell_types(const osim *s, uint8_t *out) { memcpy(out, s->cell_type, s->n_labels); }
EXPORT void orc_field(const osim *s, int k, double *out) {
    memcpy(out, &s->fields[(size_t)k * s->sites], s->sites * sizeof(double));
}
EXPORT void orc_set_field(osim *s, int k, const double *in) {
    memcpy(&s->fields[(size_t)k * s->sites], in, s->sites * sizeof(double));
}
EXPORT void orc_lengths(const osim *s, double *out) {
    for (size_t l = 0; l < s->n_labels; ++l) out[l] = mo_length(&s->mom[l]);
}

/* Replace the lattice and recount volume, surface, moments and nematic sums,
 * as a test that paints a lattice by hand does (gpu_matches_cpu.rs:308-309). */
EXPORT void orc_set_labels(osim *s, const uint32_t *labels) {
    memcpy(s->labels, labels, s->sites * sizeof *labels);
    memset(s->volume, 0, s->n_labels * sizeof *s->volume);
    for (long i = 0; i < s->sites; ++i) s->volume[labels[i]] += 1;
    count_surface(s, s->surface, s->n_labels);
    count_moments(s, s->mom, s->n_labels);
    count_nematic(s, s->nsum, s->n_labels);
}

/* Recounts from the lattice, for checking bookkeeping (cpu.rs:583-609). */
EXPORT void orc_recounted_surfaces(const osim *s, int64_t *out) { count_surface(s, out, s->n_labels); }

/* ---------------------------------------------------------------- unit hooks */

EXPORT void orc_xoshiro_stream(uint64_t seed, size_t n, uint64_t *out) {
    xoshiro r;
    xo_seed(&r, seed);
    for (size_t i = 0; i < n; ++i) out[i] = xo_next(&r);
}

EXPORT void orc_xoshiro_below(uint64_t seed, uint64_t bound, size_t n, uint64_t *out) {
    xoshiro r;
    xo_seed(&r, seed);
    for (size_t i = 0; i < n; ++i) out[i] = xo_below(&r, bound);
}

/* A moments record filled with the listed sites, then its length, the
 * anisotropy and the principal axis: moments.rs tests 204-285 use this. */
EXPORT void orc_moments_of(const double *sites, size_t n, double *length, double *aniso, double *axis) {
    moments m;
    memset(&m, 0, sizeof m);
    for (size_t i = 0; i < n; ++i) mo_add(&m, &sites[3 * i]);
    *length = mo_length(&m);
    mo_anisotropy(&m, &aniso[0], &aniso[1]);
    double c[3][3];
    mo_cov(&m, c);
    principal_axis(c, axis);
}

EXPORT void orc_unwrap_about(const double *anchor, const double *site, const double *ext, double *out) {
    moments m;
    memset(&m, 0, sizeof m);
    mo_add(&m, anchor);
    mo_unwrap(&m, site[0], site[1], site[2], ext, out);
}

EXPORT int orc_offsets(int order, int depth, int *out) {
    int o[26][3];
    int n = offsets_for(order, depth, o);
    memcpy(out, o, n * 3 * sizeof(int));
    return n;
}

EXPORT int orc_locally_connected(const uint32_t *labels, long w, long h, long d, long target, uint32_t label) {
    osim s;
    memset(&s, 0, sizeof s);
    s.g.w = w;
    s.g.h = h;
    s.g.d = d;
    s.sites = w * h * d;
    s.labels = (uint32_t *)labels;
    int all3[26][3];
    order3(all3);
    for (int k = 0; k < 26; ++k)
        if (d > 1 || all3[k][2] == 0) {
            memcpy(s.ring[s.ring_n], all3[k], sizeof all3[k]);
            ++s.ring_n;
        }
    return locally_connected(&s, target, label);
}
