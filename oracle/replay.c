/*
 * ORACLE — test infrastructure, not the product.
 *
 * A serial host replay of the device engine's schedule, written
 * independently of the CUDA source: the same colour order, the same counter
 * hash, the same per-colour snapshots of every per-cell tally and the same
 * f32/f64 operation order, so a device run must reproduce it bit for bit.
 * The tests load it through ctypes; nothing in the glazier_b200 package
 * does.
 *
 * What it replays, with the reference items each part restates:
 *   draw / mix / to_f32     the counter hash of glazier-cuda/src/lib.rs:33-50
 *   colour -> site map      lib.rs:476-493 (4 colours in a plane, 8 in a volume)
 *   copy guards             lib.rs:501-504, with the per-colour guard below
 *   connectivity veto       lib.rs:365-389, 511-521 (connectivity.rs:23-84)
 *   contact, volume,        lib.rs:523-576 (cpu.rs:242-288, 399-425)
 *   surface terms
 *   length term             cpu.rs:291-305, moments.rs:92-155, from exact
 *                           int64 sums about an integer anchor
 *   chemotaxis              lib.rs:644-651 (cpu.rs:381-395)
 *   Metropolis              lib.rs:676-679, with a project-written expf
 *   field step              lib.rs:314-363 (field.rs:99-160)
 *   division and death      lib.rs:1362-1461 (cpu.rs:620-725), planned per
 *                           cell from exact moments and a counter-hash draw
 *
 * Two rules differ from the reference device kernel, which reads per-cell
 * counters live while other threads change them (lib.rs:9-15):
 *   - every per-cell tally a colour pass reads is the value at the start of
 *     the pass (its snapshot), so the pass is order-free and deterministic;
 *   - a copy may not take a site from a cell that has no site outside the
 *     current colour. Under snapshots the reference's `volume <= 1` guard no
 *     longer stops a cell made only of same-colour sites from losing them all
 *     in one pass; this rule does, and it refuses every copy the reference
 *     guard refuses.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/glazier_gpu.h"

#define EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- hash */

static inline uint64_t mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline uint64_t draw(uint64_t seed, uint32_t site, int32_t step, int colour, int index) {
    return mix(seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)site) ^ (0xA0761D6478BD642FULL * (uint64_t)(int64_t)step) ^
               (0xE7037ED1A0B428DBULL * (uint64_t)(int64_t)(4 * colour + index)));
}

static inline float to_f32(uint64_t bits) { return (float)(bits >> 11) * 0x1p-53f; }
static inline double to_f64(uint64_t bits) { return (double)(bits >> 11) * 0x1p-53; }

/* The population draws take their own stream index, clear of the sweep's. */
#define POPULATION_STREAM 16

/*
 * exp for the Metropolis test: Cody and Waite's argument reduction
 * (W. J. Cody and W. Waite, "Software Manual for the Elementary Functions",
 * 1980) with ln 2 split in two, then the degree-7 Taylor polynomial of e^r on
 * |r| <= ln2/2 by Horner's rule in fused multiply-adds, then a scale by 2^k
 * through the exponent field. Every step is a correctly rounded IEEE
 * operation, so the host and the device agree bit for bit. Below -87 the
 * result is taken as zero, which no draw in [0, 1) can fall under.
 */
EXPORT float rp_expf(float x) {
    if (x < -87.0f) return 0.0f;
    if (x > 88.0f) return INFINITY;
    float k = rintf(x * 1.44269504088896341f);
    float r = fmaf(k, -0.693145751953125f, x);
    r = fmaf(k, -1.428606765330187e-06f, r);
    float p = 1.98412698e-04f;      /* 1/7! */
    p = fmaf(p, r, 1.38888889e-03f); /* 1/6! */
    p = fmaf(p, r, 8.33333333e-03f); /* 1/5! */
    p = fmaf(p, r, 4.16666667e-02f); /* 1/4! */
    p = fmaf(p, r, 1.66666667e-01f); /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    uint32_t bits = (uint32_t)(ki + 127) << 23;
    float scale;
    memcpy(&scale, &bits, sizeof scale);
    return p * scale;
}

/* ln x for the motility term: 2 atanh((m - 1) / (m + 1)) as the series
 * s + s^3/3 + ... + s^9/9 (Abramowitz and Stegun 4.1.27) on the mantissa m
 * reduced to [sqrt(1/2), sqrt(2)], plus e ln 2 split hi + lo; the device's
 * operations in the same order. */
EXPORT float rp_logf(float x) {
    int e = 0;
    if (x < 1.17549435e-38f) {
        x = x * 16777216.0f;
        e = -24;
    }
    uint32_t bits;
    memcpy(&bits, &x, sizeof bits);
    e += (int)((bits >> 23) & 0xff) - 127;
    uint32_t mb = (bits & 0x007fffffu) | 0x3f800000u;
    float m;
    memcpy(&m, &mb, sizeof m);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 0.111111111f;
    p = fmaf(p, s2, 0.142857143f);
    p = fmaf(p, s2, 0.2f);
    p = fmaf(p, s2, 0.333333333f);
    p = p * s2;
    float lm = (2.0f * s) * (1.0f + p);
    float fe = (float)e;
    return fmaf(fe, 0.693145751953125f, lm) + fe * 1.428606765330187e-06f;
}

/* ---------------------------------------------------------------- geometry */

static inline int wrapi(int v, int n) {
    int r = v % n;
    return r < 0 ? r + n : r;
}

/* Minimum image of an integer offset on a periodic axis (moments.rs:36-46). */
static inline int fold_int(int d, int span) {
    if (2 * d > span) return d - span;
    if (2 * d < -span) return d + span;
    return d;
}

static int order3(int out[26][3]) {
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
    return k;
}

/* lattice.rs:69-88 */
static int offsets_for(int order, int depth, int out[26][3]) {
    static const int O1[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    static const int O2[18][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                                  {1, 1, 0},  {1, -1, 0}, {-1, 1, 0},  {-1, -1, 0}, {1, 0, 1}, {1, 0, -1},
                                  {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
    int all[26][3];
    order3(all);
    int n = 0;
    if (depth > 1) {
        if (order == 1) {
            memcpy(out, O1, sizeof O1);
            return 6;
        }
        if (order == 2) {
            memcpy(out, O2, sizeof O2);
            return 18;
        }
        memcpy(out, all, sizeof all);
        return 26;
    }
    if (order >= 2) {
        for (int k = 0; k < 26; ++k)
            if (all[k][2] == 0) memcpy(out[n++], all[k], sizeof all[k]);
        return n;
    }
    for (int k = 0; k < 6; ++k)
        if (O1[k][2] == 0) memcpy(out[n++], O1[k], sizeof O1[k]);
    return n;
}

/* ---------------------------------------------------------------- state */

typedef struct {
    int w, h, d, dim, ncol, sites;
    int n_off, off[26][3];
    int ring_n, ring[26][3];
    uint32_t adjacency[26];
    int n_types, n_species;
    float beta; /* (float)(1 / T), rounded once on the host */
    uint64_t seed;
    float *contact, *tv, *lv, *ts, *ls, *chemo, *sec, *upt;
    float *ext; /* 3 per type: the drift vector */
    int has_external;
    /* motility (Act): activity per site, per-type maximum and strength; a
     * pass with it lists its copies and applies them at its end */
    float *maxact, *lamact, *act;
    int has_motility;
    uint32_t *pending; /* 2 per copy: target, new label */
    /* the nematic field (2 per site) and its per-cell sums, carried in the
     * moment words after the geometric ones in units of 2^-32 */
    float *nem;
    double *lnem;
    int has_nematic, nmg; /* nmg: the geometric moment words, 5 or 9 */
    double *tl, *ll, *div_vol, *death;
    uint8_t *connected;
    float *fd, *fdecay; /* per species per sub-step */
    int *substeps;
    int has_conn, has_length, has_pop, tracks;
    int nm; /* moment sums per cell: 5 in a plane, 9 in a volume */

    uint32_t *labels;
    size_t n_labels, cap;
    uint8_t *cell_type;
    int32_t *vol, *surf, *volc, *anchor;
    int64_t *mom;
    float *fields, *scratch;
    uint64_t mcs;
    uint64_t accepted;
    /* the infection rule (glz_gpu_set_infection): species -1 is none; dose per
     * label in units of 2^-24 */
    int inf_species, inf_from, inf_to;
    int64_t inf_threshold;
    int64_t *dose;
} rsim;

static char rp_error[256];
EXPORT const char *rp_last_error(void) { return rp_error; }

static void reserve(rsim *s, size_t want) {
    if (want <= s->cap) return;
    size_t cap = s->cap ? s->cap : 16;
    while (cap < want) cap *= 2;
    s->cell_type = (uint8_t *)realloc(s->cell_type, cap);
    s->vol = (int32_t *)realloc(s->vol, cap * sizeof(int32_t));
    s->surf = (int32_t *)realloc(s->surf, cap * sizeof(int32_t));
    s->volc = (int32_t *)realloc(s->volc, cap * s->ncol * sizeof(int32_t));
    s->anchor = (int32_t *)realloc(s->anchor, cap * 3 * sizeof(int32_t));
    s->mom = (int64_t *)realloc(s->mom, cap * s->nm * sizeof(int64_t));
    s->dose = (int64_t *)realloc(s->dose, cap * sizeof(int64_t));
    memset(s->dose + s->cap, 0, (cap - s->cap) * sizeof(int64_t));
    s->cap = cap;
}

static inline int colour_of(const rsim *s, int x, int y, int z) {
    return (x & 1) | ((y & 1) << 1) | (s->dim == 3 ? ((z & 1) << 2) : 0);
}

/* The tallies a device recount builds from the lattice: volume, volume per
 * colour, unlike-bond surface, anchor (the cell's first site in scan order)
 * and the exact moment sums about it. The medium's entries are kept too. */
/* A nematic field component in the per-cell sums: units of 2^-32, rounded
 * to nearest. */
static int64_t nematic_fixed(float q) { return (int64_t)llrint((double)q * 4294967296.0); }

static void recount(rsim *s) {
    size_t n = s->n_labels;
    memset(s->vol, 0, n * sizeof(int32_t));
    memset(s->surf, 0, n * sizeof(int32_t));
    memset(s->volc, 0, n * s->ncol * sizeof(int32_t));
    memset(s->mom, 0, n * s->nm * sizeof(int64_t));
    for (size_t l = 0; l < n; ++l) s->anchor[3 * l] = s->anchor[3 * l + 1] = s->anchor[3 * l + 2] = -1;
    for (int i = 0; i < s->sites; ++i) {
        uint32_t l = s->labels[i];
        int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
        if (s->anchor[3 * l] < 0) {
            s->anchor[3 * l] = x;
            s->anchor[3 * l + 1] = y;
            s->anchor[3 * l + 2] = z;
        }
        s->vol[l] += 1;
        s->volc[l * s->ncol + colour_of(s, x, y, z)] += 1;
        int bonds = 0;
        for (int k = 0; k < s->n_off; ++k) {
            int nb = (wrapi(z + s->off[k][2], s->d) * s->h + wrapi(y + s->off[k][1], s->h)) * s->w +
                     wrapi(x + s->off[k][0], s->w);
            if (nb != i && s->labels[nb] != l) ++bonds;
        }
        s->surf[l] += bonds;
    }
    for (int i = 0; i < s->sites; ++i) {
        uint32_t l = s->labels[i];
        if (l == 0) continue;
        int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
        int64_t ux = fold_int(x - s->anchor[3 * l], s->w);
        int64_t uy = fold_int(y - s->anchor[3 * l + 1], s->h);
        int64_t uz = fold_int(z - s->anchor[3 * l + 2], s->d);
        int64_t *m = &s->mom[l * s->nm];
        if (s->dim == 2) {
            m[0] += ux; m[1] += uy; m[2] += ux * ux; m[3] += uy * uy; m[4] += ux * uy;
        } else {
            m[0] += ux; m[1] += uy; m[2] += uz;
            m[3] += ux * ux; m[4] += uy * uy; m[5] += uz * uz;
            m[6] += ux * uy; m[7] += ux * uz; m[8] += uy * uz;
        }
        if (s->has_nematic) {
            m[s->nmg] += nematic_fixed(s->nem[2 * i]);
            m[s->nmg + 1] += nematic_fixed(s->nem[2 * i + 1]);
        }
    }
}

static float *f32_copy(const double *src, size_t n) {
    float *out = (float *)calloc(n ? n : 1, sizeof(float));
    for (size_t i = 0; src && i < n; ++i) out[i] = (float)src[i];
    return out;
}

static double *f64_copy(const double *src, size_t n) {
    double *out = (double *)calloc(n ? n : 1, sizeof(double));
    if (src && n) memcpy(out, src, n * sizeof(double));
    return out;
}

/* field.rs:155-160 */
static int substeps_for(double diffusion, int dimensions) {
    if (diffusion <= 0.0) return 1;
    double k = ceil(diffusion / (1.0 / (2.0 * (double)dimensions)));
    return k < 1.0 ? 1 : (int)k;
}

EXPORT rsim *rp_create(const glz_model *m, const uint32_t *labels, const uint8_t *cell_type, size_t n_labels,
                       const double *fields) {
    if (m->width % 2 || m->height % 2 || (m->depth > 1 && m->depth % 2)) {
        snprintf(rp_error, sizeof rp_error, "the checkerboard split needs even sides; the lattice is %d by %d by %d",
                 m->width, m->height, m->depth);
        return NULL;
    }
    rsim *s = (rsim *)calloc(1, sizeof *s);
    s->inf_species = -1;
    s->w = m->width;
    s->h = m->height;
    s->d = m->depth;
    s->dim = s->d > 1 ? 3 : 2;
    s->ncol = s->dim == 3 ? 8 : 4;
    s->nmg = s->dim == 3 ? 9 : 5;
    s->nm = s->nmg;
    s->sites = s->w * s->h * s->d;
    s->n_off = offsets_for(m->neighbour_order, m->depth, s->off);
    int nt = m->n_types, ns = m->n_species;
    s->n_types = nt;
    s->n_species = ns;
    s->beta = (float)(1.0 / m->temperature);
    s->seed = m->seed;
    s->contact = f32_copy(m->contact, (size_t)nt * nt);
    s->tv = f32_copy(m->target_volume, nt);
    s->lv = f32_copy(m->lambda_volume, nt);
    s->ts = f32_copy(m->target_surface, nt);
    s->ls = f32_copy(m->lambda_surface, nt);
    s->tl = f64_copy(m->target_length, nt);
    s->ll = f64_copy(m->lambda_length, nt);
    s->div_vol = f64_copy(m->division_volume, nt);
    s->death = f64_copy(m->death_rate, nt);
    s->chemo = f32_copy(m->chemotaxis, (size_t)nt * ns);
    s->ext = f32_copy(m->external, 3 * (size_t)nt);
    s->maxact = f32_copy(m->max_activity, (size_t)nt);
    s->lamact = f32_copy(m->lambda_activity, (size_t)nt);
    for (int t = 0; t < nt; ++t) s->has_motility |= s->lamact[t] != 0.0f && s->maxact[t] > 0.0f;
    s->lnem = (double *)calloc((size_t)nt, sizeof(double));
    for (int t = 0; t < nt; ++t) {
        s->lnem[t] = m->lambda_nematic ? m->lambda_nematic[t] : 0.0;
        s->has_nematic |= m->nematic != NULL && s->lnem[t] != 0.0;
    }
    if (s->has_nematic) {
        s->nm = s->nmg + 2;
        s->nem = f32_copy(m->nematic, 2 * (size_t)s->sites);
    }
    for (int i = 0; i < 3 * nt; ++i) s->has_external |= s->ext[i] != 0.0f;
    s->sec = f32_copy(m->secretion, (size_t)nt * ns);
    s->upt = f32_copy(m->uptake, (size_t)nt * ns);
    s->connected = (uint8_t *)calloc(nt, 1);
    for (int t = 0; t < nt; ++t) {
        s->connected[t] = m->connected ? m->connected[t] != 0 : 0;
        s->has_conn |= s->connected[t];
        s->has_length |= s->ll[t] != 0.0;
        s->has_pop |= s->div_vol[t] > 0.0 || s->death[t] > 0.0;
    }
    s->tracks = s->has_length || s->has_pop || s->has_nematic;
    s->fd = (float *)calloc(ns ? ns : 1, sizeof(float));
    s->fdecay = (float *)calloc(ns ? ns : 1, sizeof(float));
    s->substeps = (int *)calloc(ns ? ns : 1, sizeof(int));
    for (int k = 0; k < ns; ++k) {
        double D = m->diffusion ? m->diffusion[k] : 0.0, dec = m->decay ? m->decay[k] : 0.0;
        s->substeps[k] = substeps_for(D, s->dim);
        s->fd[k] = (float)(D / (double)s->substeps[k]);
        s->fdecay[k] = (float)(dec / (double)s->substeps[k]);
    }
    if (s->has_conn) {
        int all[26][3];
        order3(all);
        for (int k = 0; k < 26; ++k)
            if (s->d > 1 || all[k][2] == 0) memcpy(s->ring[s->ring_n++], all[k], sizeof all[k]);
        for (int a = 0; a < s->ring_n; ++a) {
            uint32_t mask = 0;
            for (int b = 0; b < s->ring_n; ++b)
                if (abs(s->ring[a][0] - s->ring[b][0]) <= 1 && abs(s->ring[a][1] - s->ring[b][1]) <= 1 &&
                    abs(s->ring[a][2] - s->ring[b][2]) <= 1)
                    mask |= 1u << b;
            s->adjacency[a] = mask;
        }
    }
    s->labels = (uint32_t *)malloc(s->sites * sizeof(uint32_t));
    memcpy(s->labels, labels, s->sites * sizeof(uint32_t));
    s->n_labels = n_labels;
    reserve(s, n_labels);
    memcpy(s->cell_type, cell_type, n_labels);
    s->act = (float *)calloc((size_t)s->sites, sizeof(float));
    s->pending = (uint32_t *)malloc(2 * (size_t)s->sites * sizeof(uint32_t));
    s->fields = (float *)calloc((size_t)(ns ? ns : 1) * s->sites, sizeof(float));
    s->scratch = (float *)calloc((size_t)(ns ? ns : 1) * s->sites, sizeof(float));
    for (int k = 0; k < ns; ++k)
        for (int i = 0; i < s->sites; ++i)
            s->fields[(size_t)k * s->sites + i] =
                fields ? (float)fields[(size_t)k * s->sites + i] : (float)(m->initial ? m->initial[k] : 0.0);
    recount(s);
    return s;
}

EXPORT void rp_destroy(rsim *s) {
    if (!s) return;
    free(s->contact); free(s->tv); free(s->lv); free(s->ts); free(s->ls); free(s->tl); free(s->ll);
    free(s->div_vol); free(s->death); free(s->chemo); free(s->sec); free(s->upt); free(s->ext); free(s->connected);
    free(s->maxact); free(s->lamact); free(s->act); free(s->pending); free(s->nem); free(s->lnem);
    free(s->fd); free(s->fdecay); free(s->substeps);
    free(s->dose);
    free(s->labels); free(s->cell_type); free(s->vol); free(s->surf); free(s->volc); free(s->anchor);
    free(s->mom); free(s->fields); free(s->scratch);
    free(s);
}

/* ---------------------------------------------------------------- energies */

/* lib.rs:371-389 */
static int one_piece(uint32_t present, const uint32_t *adjacency) {
    if (present == 0u || (present & (present - 1u)) == 0u) return 1;
    uint32_t reached = present & (~present + 1u);
    for (int round = 0; round < 26; ++round) {
        uint32_t grown = reached, rest = reached;
        while (rest) {
            int k = __builtin_ctz(rest);
            grown |= adjacency[k];
            rest &= rest - 1u;
        }
        grown &= present;
        if (grown == reached) break;
        reached = grown;
    }
    return reached == present;
}

/* The dominant eigenvalue of a symmetric 3x3 by twenty rounds of power
 * iteration and a Rayleigh quotient (moments.rs:165-186). */
static double power_lambda(const double c[3][3]) {
    double v[3] = {1.0, 0.7, 0.3}, w[3];
    for (int round = 0; round < 20; ++round) {
        for (int i = 0; i < 3; ++i) w[i] = c[i][0] * v[0] + c[i][1] * v[1] + c[i][2] * v[2];
        double norm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (norm < 1e-15) return 0.0;
        v[0] = w[0] / norm;
        v[1] = w[1] / norm;
        v[2] = w[2] / norm;
    }
    for (int i = 0; i < 3; ++i) w[i] = c[i][0] * v[0] + c[i][1] * v[1] + c[i][2] * v[2];
    double lambda = v[0] * w[0] + v[1] * w[1] + v[2] * w[2];
    return lambda > 0.0 ? lambda : 0.0;
}

/* The major axis 4 sqrt(lambda_max) of a cell of n sites with exact sums m
 * (moments.rs:150-155). A plane takes the 2x2 closed form. */
static double axis_length(int dim, int64_t n, const int64_t *m) {
    if (n < 2) return 0.0;
    double dn = (double)n;
    if (dim == 2) {
        double mx = (double)m[0] / dn, my = (double)m[1] / dn;
        double cxx = (double)m[2] / dn - mx * mx;
        double cyy = (double)m[3] / dn - my * my;
        double cxy = (double)m[4] / dn - mx * my;
        double half = 0.5 * (cxx + cyy), diff = 0.5 * (cxx - cyy);
        double lambda = half + sqrt(diff * diff + cxy * cxy);
        return 4.0 * sqrt(lambda > 0.0 ? lambda : 0.0);
    }
    double mx = (double)m[0] / dn, my = (double)m[1] / dn, mz = (double)m[2] / dn;
    double c[3][3];
    c[0][0] = (double)m[3] / dn - mx * mx;
    c[1][1] = (double)m[4] / dn - my * my;
    c[2][2] = (double)m[5] / dn - mz * mz;
    c[0][1] = c[1][0] = (double)m[6] / dn - mx * my;
    c[0][2] = c[2][0] = (double)m[7] / dn - mx * mz;
    c[1][2] = c[2][1] = (double)m[8] / dn - my * mz;
    return 4.0 * sqrt(power_lambda(c));
}

static void site_terms(int dim, int64_t ux, int64_t uy, int64_t uz, int64_t *t) {
    if (dim == 2) {
        t[0] = ux; t[1] = uy; t[2] = ux * ux; t[3] = uy * uy; t[4] = ux * uy;
    } else {
        t[0] = ux; t[1] = uy; t[2] = uz; t[3] = ux * ux; t[4] = uy * uy; t[5] = uz * uz;
        t[6] = ux * uy; t[7] = ux * uz; t[8] = uy * uz;
    }
}

/* Change in a cell's length energy when the site at offset u (in its own
 * frame) leaves (sign -1) or joins (+1) it (cpu.rs:291-305). */
static double length_delta(const rsim *s, int t, int64_t n, const int64_t *m, const int64_t *terms, int sign) {
    int64_t after[11];
    for (int k = 0; k < s->nm; ++k) after[k] = m[k] + sign * terms[k];
    double before = axis_length(s->dim, n, m) - s->tl[t];
    double now = axis_length(s->dim, n + sign, after) - s->tl[t];
    return s->ll[t] * (now * now - before * before);
}

/* In-plane anisotropy of a cell from its exact sums (moments.rs), as the
 * device takes it. */
static void anisotropy(const rsim *s, int64_t n, const int64_t *m, double *a0, double *a1) {
    *a0 = 0.0;
    *a1 = 0.0;
    if (n < 2) return;
    double dn = (double)n;
    double mx = (double)m[0] / dn, my = (double)m[1] / dn;
    double cxx = (double)m[s->dim == 2 ? 2 : 3] / dn - mx * mx;
    double cyy = (double)m[s->dim == 2 ? 3 : 4] / dn - my * my;
    double cxy = (double)m[s->dim == 2 ? 4 : 6] / dn - mx * my;
    double trace = cxx + cyy;
    if (!(trace > 1e-12)) return;
    *a0 = (cxx - cyy) / trace;
    *a1 = 2.0 * cxy / trace;
}

/* Change in a cell's nematic energy (cpu.rs:315-332) when the site with sum
 * terms `terms` (moment terms, then the field in fixed point) leaves (-1) or
 * joins (+1) it. */
static double nematic_delta(const rsim *s, int t, int64_t n, const int64_t *m, const int64_t *terms, int sign) {
    int64_t after[11];
    for (int k = 0; k < s->nm; ++k) after[k] = m[k] + sign * terms[k];
    double a0, a1, b0, b1;
    anisotropy(s, n, m, &a0, &a1);
    anisotropy(s, n + sign, after, &b0, &b1);
    double scale = 1.0 / 4294967296.0;
    double before = (double)m[s->nmg] * scale * a0 + (double)m[s->nmg + 1] * scale * a1;
    double now = (double)after[s->nmg] * scale * b0 + (double)after[s->nmg + 1] * scale * b1;
    return -s->lnem[t] * (now - before);
}

/* One colour pass over the lattice: every target of the colour, each priced
 * against the tallies at the start of the pass. */
/* The geometric mean of the activity over the sites of `label` around `site`,
 * the site itself included; zero once one of them has none left
 * (lib.rs:391-424, motility.rs:58-79). */
static float activity_mean(const rsim *s, int site, int x, int y, int z, uint32_t label) {
    float here = s->act[site];
    if (!(here > 0.0f)) return 0.0f;
    float log_sum = rp_logf(here), count = 1.0f;
    for (int k = 0; k < s->n_off; ++k) {
        int n = (wrapi(z + s->off[k][2], s->d) * s->h + wrapi(y + s->off[k][1], s->h)) * s->w +
                wrapi(x + s->off[k][0], s->w);
        if (n == site || s->labels[n] != label) continue;
        float v = s->act[n];
        if (!(v > 0.0f)) return 0.0f;
        log_sum = log_sum + rp_logf(v);
        count = count + 1.0f;
    }
    return rp_expf(log_sum / count);
}

static void pass(rsim *s, int colour) {
    size_t n = s->n_labels;
    int32_t *snap_vol = (int32_t *)malloc(n * sizeof(int32_t));
    int32_t *snap_surf = (int32_t *)malloc(n * sizeof(int32_t));
    int64_t *snap_mom = (int64_t *)malloc(n * s->nm * sizeof(int64_t));
    memcpy(snap_vol, s->vol, n * sizeof(int32_t));
    memcpy(snap_surf, s->surf, n * sizeof(int32_t));
    memcpy(snap_mom, s->mom, n * s->nm * sizeof(int64_t));

    int32_t step = (int32_t)s->mcs;
    size_t np = 0; /* copies listed for the end of the pass (motility) */
    int hw = s->w / 2, hh = s->h / 2, hd = s->dim == 3 ? s->d / 2 : 1;
    int cx = colour & 1, cy = (colour >> 1) & 1, cz = (colour >> 2) & 1;
    for (int iz = 0; iz < hd; ++iz)
        for (int iy = 0; iy < hh; ++iy)
            for (int ix = 0; ix < hw; ++ix) {
                int x = 2 * ix + cx, y = 2 * iy + cy, z = s->dim == 3 ? 2 * iz + cz : 0;
                uint32_t target = (uint32_t)((z * s->h + y) * s->w + x);
                uint64_t h0 = draw(s->seed, target, step, colour, 0);
                int pick = (int)(h0 % (uint64_t)s->n_off);
                int sx = wrapi(x + s->off[pick][0], s->w);
                int sy = wrapi(y + s->off[pick][1], s->h);
                int sz = wrapi(z + s->off[pick][2], s->d);
                uint32_t source = (uint32_t)((sz * s->h + sy) * s->w + sx);
                uint32_t old = s->labels[target], nw = s->labels[source];
                if (old == nw) continue;
                int t_old = s->cell_type[old], t_new = s->cell_type[nw];

                if (old != 0) {
                    /* The per-colour guard: the cell must keep a site of
                     * another colour, which no copy in this pass can take. */
                    int32_t other = 0;
                    for (int c = 0; c < s->ncol; ++c)
                        if (c != colour) other += s->volc[old * s->ncol + c];
                    if (other == 0) continue;
                }
                if (old != 0 && s->ring_n > 0 && s->connected[t_old]) {
                    uint32_t present = 0;
                    for (int k = 0; k < s->ring_n; ++k) {
                        int nb = (wrapi(z + s->ring[k][2], s->d) * s->h + wrapi(y + s->ring[k][1], s->h)) * s->w +
                                 wrapi(x + s->ring[k][0], s->w);
                        if ((uint32_t)nb != target && s->labels[nb] == old) present |= 1u << k;
                    }
                    if (!one_piece(present, s->adjacency)) continue;
                }

                float delta = 0.0f;
                int like_old = 0, like_new = 0, bonds = 0;
                for (int k = 0; k < s->n_off; ++k) {
                    int nb = (wrapi(z + s->off[k][2], s->d) * s->h + wrapi(y + s->off[k][1], s->h)) * s->w +
                             wrapi(x + s->off[k][0], s->w);
                    if ((uint32_t)nb == target) continue;
                    ++bonds;
                    uint32_t ln = s->labels[nb];
                    int tn = s->cell_type[ln];
                    if (ln != old)
                        delta = delta - s->contact[t_old * s->n_types + tn];
                    else
                        ++like_old;
                    if (ln != nw)
                        delta = delta + s->contact[t_new * s->n_types + tn];
                    else
                        ++like_new;
                }
                int ds_old = 2 * like_old - bonds;
                int ds_new = bonds - 2 * like_new;

                /* lambda ((v -/+ 1 - V_t)^2 - (v - V_t)^2) = lambda (1 -/+ 2 (v - V_t)) */
                if (old != 0 && s->lv[t_old] != 0.0f) {
                    float dv = (float)snap_vol[old] - s->tv[t_old];
                    delta = delta + s->lv[t_old] * (1.0f - 2.0f * dv);
                }
                if (nw != 0 && s->lv[t_new] != 0.0f) {
                    float dv = (float)snap_vol[nw] - s->tv[t_new];
                    delta = delta + s->lv[t_new] * (2.0f * dv + 1.0f);
                }
                /* lambda ((s + ds - S_t)^2 - (s - S_t)^2) = lambda ds (2 (s - S_t) + ds) */
                if (old != 0 && s->ls[t_old] != 0.0f) {
                    float e = (float)snap_surf[old] - s->ts[t_old], dsf = (float)ds_old;
                    delta = delta + s->ls[t_old] * (dsf * (2.0f * e + dsf));
                }
                if (nw != 0 && s->ls[t_new] != 0.0f) {
                    float e = (float)snap_surf[nw] - s->ts[t_new], dsf = (float)ds_new;
                    delta = delta + s->ls[t_new] * (dsf * (2.0f * e + dsf));
                }
                int64_t terms_old[11], terms_new[11];
                if (s->has_nematic) {
                    int64_t q0 = nematic_fixed(s->nem[2 * (size_t)target]);
                    int64_t q1 = nematic_fixed(s->nem[2 * (size_t)target + 1]);
                    terms_old[s->nmg] = terms_new[s->nmg] = q0;
                    terms_old[s->nmg + 1] = terms_new[s->nmg + 1] = q1;
                }
                if (s->tracks) {
                    if (old != 0) {
                        const int32_t *an = &s->anchor[3 * old];
                        site_terms(s->dim, fold_int(x - an[0], s->w), fold_int(y - an[1], s->h),
                                   fold_int(z - an[2], s->d), terms_old);
                    }
                    if (nw != 0) {
                        const int32_t *an = &s->anchor[3 * nw];
                        site_terms(s->dim, fold_int(x - an[0], s->w), fold_int(y - an[1], s->h),
                                   fold_int(z - an[2], s->d), terms_new);
                    }
                }
                /* length then nematic, leaving cell first (lib.rs:578-639) */
                if (old != 0) {
                    if (s->has_length && s->ll[t_old] != 0.0)
                        delta = delta + (float)length_delta(s, t_old, snap_vol[old], &snap_mom[old * s->nm], terms_old, -1);
                    if (s->has_nematic && s->lnem[t_old] != 0.0)
                        delta = delta + (float)nematic_delta(s, t_old, snap_vol[old], &snap_mom[old * s->nm], terms_old, -1);
                }
                if (nw != 0) {
                    if (s->has_length && s->ll[t_new] != 0.0)
                        delta = delta + (float)length_delta(s, t_new, snap_vol[nw], &snap_mom[nw * s->nm], terms_new, 1);
                    if (s->has_nematic && s->lnem[t_new] != 0.0)
                        delta = delta + (float)nematic_delta(s, t_new, snap_vol[nw], &snap_mom[nw * s->nm], terms_new, 1);
                }
                if (nw != 0) {
                    for (int k = 0; k < s->n_species; ++k) {
                        float lam = s->chemo[t_new * s->n_species + k];
                        if (lam == 0.0f) continue;
                        const float *f = &s->fields[(size_t)k * s->sites];
                        delta = delta - lam * (f[target] - f[source]);
                    }
                }
                /* motility, cpu.rs:346-352 */
                if (nw != 0 && s->has_motility && s->lamact[t_new] != 0.0f && s->maxact[t_new] > 0.0f) {
                    float into = activity_mean(s, (int)source, sx, sy, sz, nw);
                    float out_of = activity_mean(s, (int)target, x, y, z, old);
                    delta = delta - (s->lamact[t_new] / s->maxact[t_new]) * (into - out_of);
                }
                /* the drift, cpu.rs:360-369: work e . (target - source), folded */
                if (nw != 0 && s->has_external) {
                    float ex = s->ext[3 * t_new], ey = s->ext[3 * t_new + 1], ez = s->ext[3 * t_new + 2];
                    if (ex != 0.0f || ey != 0.0f || ez != 0.0f) {
                        float fx = (float)fold_int(x - sx, s->w), fy = (float)fold_int(y - sy, s->h),
                              fz = (float)fold_int(z - sz, s->d);
                        delta = delta - (ex * fx + ey * fy + ez * fz);
                    }
                }

                int accept = delta <= 0.0f;
                if (!accept) {
                    float u = to_f32(draw(s->seed, target, step, colour, 1));
                    accept = u < rp_expf(-delta * s->beta);
                }
                if (!accept) continue;
                s->accepted += 1;
                if (s->has_motility) {
                    /* motility reads two sites out: the pass's writes wait */
                    s->pending[2 * np] = target;
                    s->pending[2 * np + 1] = nw;
                    ++np;
                } else {
                    s->labels[target] = nw;
                }
                if (old != 0) {
                    s->vol[old] -= 1;
                    s->surf[old] += ds_old;
                    s->volc[old * s->ncol + colour] -= 1;
                    if (s->tracks)
                        for (int k = 0; k < s->nm; ++k) s->mom[old * s->nm + k] -= terms_old[k];
                }
                if (nw != 0) {
                    s->vol[nw] += 1;
                    s->surf[nw] += ds_new;
                    s->volc[nw * s->ncol + colour] += 1;
                    if (s->tracks)
                        for (int k = 0; k < s->nm; ++k) s->mom[nw * s->nm + k] += terms_new[k];
                }
            }
    for (size_t k = 0; k < np; ++k) {
        uint32_t target = s->pending[2 * k], nw = s->pending[2 * k + 1];
        s->labels[target] = nw;
        if (nw != 0 && s->maxact[s->cell_type[nw]] > 0.0f) s->act[target] = s->maxact[s->cell_type[nw]];
    }
    free(snap_vol);
    free(snap_surf);
    free(snap_mom);
}

/* ---------------------------------------------------------------- fields */

/* One MCS of the field solver: sub-step rounds of FTCS diffusion and decay
 * (lib.rs:314-341), each species' secretion and uptake folded into its last
 * sub-step (lib.rs:343-363). */
static void field_step(rsim *s) {
    int rounds = 0;
    for (int k = 0; k < s->n_species; ++k)
        if (s->substeps[k] > rounds) rounds = s->substeps[k];
    float faces = s->dim == 3 ? 6.0f : 4.0f;
    for (int r = 0; r < rounds; ++r) {
        for (int k = 0; k < s->n_species; ++k) {
            if (r >= s->substeps[k]) continue;
            const float *u = &s->fields[(size_t)k * s->sites];
            float *out = &s->scratch[(size_t)k * s->sites];
            float d = s->fd[k], decay = s->fdecay[k];
            int last = r == s->substeps[k] - 1;
            for (int i = 0; i < s->sites; ++i) {
                int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
                float here = u[i];
                float sum = u[(z * s->h + y) * s->w + wrapi(x - 1, s->w)];
                sum = sum + u[(z * s->h + y) * s->w + wrapi(x + 1, s->w)];
                sum = sum + u[(z * s->h + wrapi(y - 1, s->h)) * s->w + x];
                sum = sum + u[(z * s->h + wrapi(y + 1, s->h)) * s->w + x];
                if (s->dim == 3) {
                    sum = sum + u[(wrapi(z - 1, s->d) * s->h + y) * s->w + x];
                    sum = sum + u[(wrapi(z + 1, s->d) * s->h + y) * s->w + x];
                }
                float v = here + d * (sum - faces * here) - decay * here;
                if (last) {
                    uint32_t l = s->labels[i];
                    if (l != 0) {
                        int t = s->cell_type[l];
                        v = v + s->sec[t * s->n_species + k];
                        float amount = s->upt[t * s->n_species + k] * v;
                        if (k == s->inf_species && t == s->inf_from)
                            s->dose[l] += (int64_t)llrintf(amount * 16777216.0f);
                        v = v - amount;
                        v = v < 0.0f ? 0.0f : v;
                    }
                }
                out[i] = v;
            }
            memcpy((void *)u, out, s->sites * sizeof(float));
        }
    }
}

/* ---------------------------------------------------------------- population */

/* Division and death for one MCS, planned per cell (lib.rs:1362-1461):
 *   - a live cell of volume >= its type's division volume (and >= 4 sites,
 *     cpu.rs:681) is cut by the plane through its centroid perpendicular to
 *     its major axis, from its exact moments; sites with (r - c).axis > 0 go
 *     to the daughter, and a cut that moves nothing or everything is no
 *     division (cpu.rs:697-703). Daughters take labels n_labels, n_labels+1,
 *     ... in the mothers' label order.
 *   - any other live cell of a type with a death rate dies when its
 *     counter-hash draw falls under the rate; its sites become medium.
 * Then every tally is recounted from the lattice (cpu.rs:649-653). */
static void population(rsim *s) {
    size_t n = s->n_labels;
    int32_t step = (int32_t)s->mcs;
    uint8_t *mode = (uint8_t *)calloc(n, 1);
    double (*plan)[6] = (double(*)[6])calloc(n, sizeof *plan);
    int32_t *moved = (int32_t *)calloc(n, sizeof(int32_t));
    for (size_t l = 1; l < n; ++l) {
        int32_t v = s->vol[l];
        if (v <= 0) continue;
        int t = s->cell_type[l];
        if (s->div_vol[t] > 0.0 && (double)v >= s->div_vol[t] && v >= 4) {
            const int64_t *m = &s->mom[l * s->nm];
            double dn = (double)v, c[3][3], mean[3];
            if (s->dim == 2) {
                mean[0] = (double)m[0] / dn; mean[1] = (double)m[1] / dn; mean[2] = 0.0;
                c[0][0] = (double)m[2] / dn - mean[0] * mean[0];
                c[1][1] = (double)m[3] / dn - mean[1] * mean[1];
                c[0][1] = c[1][0] = (double)m[4] / dn - mean[0] * mean[1];
                c[2][2] = c[0][2] = c[2][0] = c[1][2] = c[2][1] = 0.0;
            } else {
                mean[0] = (double)m[0] / dn; mean[1] = (double)m[1] / dn; mean[2] = (double)m[2] / dn;
                c[0][0] = (double)m[3] / dn - mean[0] * mean[0];
                c[1][1] = (double)m[4] / dn - mean[1] * mean[1];
                c[2][2] = (double)m[5] / dn - mean[2] * mean[2];
                c[0][1] = c[1][0] = (double)m[6] / dn - mean[0] * mean[1];
                c[0][2] = c[2][0] = (double)m[7] / dn - mean[0] * mean[2];
                c[1][2] = c[2][1] = (double)m[8] / dn - mean[1] * mean[2];
            }
            double v3[3] = {1.0, 0.7, 0.3}, w[3];
            int degenerate = 0;
            for (int round = 0; round < 20; ++round) {
                for (int i = 0; i < 3; ++i) w[i] = c[i][0] * v3[0] + c[i][1] * v3[1] + c[i][2] * v3[2];
                double norm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
                if (norm < 1e-15) {
                    degenerate = 1;
                    break;
                }
                v3[0] = w[0] / norm; v3[1] = w[1] / norm; v3[2] = w[2] / norm;
            }
            if (degenerate) { v3[0] = 1.0; v3[1] = 0.0; v3[2] = 0.0; }
            mode[l] = 1;
            for (int i = 0; i < 3; ++i) {
                plan[l][i] = mean[i];
                plan[l][3 + i] = v3[i];
            }
        } else if (s->death[t] > 0.0) {
            double u = to_f64(draw(s->seed, (uint32_t)l, step, POPULATION_STREAM, 0));
            if (u < s->death[t]) mode[l] = 2;
        }
    }
    /* Count what each cut would move. */
    for (int i = 0; i < s->sites; ++i) {
        uint32_t l = s->labels[i];
        if (l == 0 || mode[l] != 1) continue;
        int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
        double ux = (double)fold_int(x - s->anchor[3 * l], s->w);
        double uy = (double)fold_int(y - s->anchor[3 * l + 1], s->h);
        double uz = (double)fold_int(z - s->anchor[3 * l + 2], s->d);
        double along = (ux - plan[l][0]) * plan[l][3] + (uy - plan[l][1]) * plan[l][4] + (uz - plan[l][2]) * plan[l][5];
        if (along > 0.0) moved[l] += 1;
    }
    uint32_t *daughter = (uint32_t *)calloc(n, sizeof(uint32_t));
    size_t next = n;
    int acted = 0;
    for (size_t l = 1; l < n; ++l) {
        if (mode[l] == 1) {
            if (moved[l] > 0 && moved[l] < s->vol[l]) {
                daughter[l] = (uint32_t)next++;
                acted = 1;
            } else {
                mode[l] = 0;
            }
        } else if (mode[l] == 2) {
            acted = 1;
        }
    }
    if (acted) {
        for (int i = 0; i < s->sites; ++i) {
            uint32_t l = s->labels[i];
            if (l == 0 || mode[l] == 0) continue;
            if (mode[l] == 2) {
                s->labels[i] = 0;
                continue;
            }
            int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
            double ux = (double)fold_int(x - s->anchor[3 * l], s->w);
            double uy = (double)fold_int(y - s->anchor[3 * l + 1], s->h);
            double uz = (double)fold_int(z - s->anchor[3 * l + 2], s->d);
            double along =
                (ux - plan[l][0]) * plan[l][3] + (uy - plan[l][1]) * plan[l][4] + (uz - plan[l][2]) * plan[l][5];
            if (along > 0.0) s->labels[i] = daughter[l];
        }
        size_t old_n = s->n_labels;
        reserve(s, next);
        for (size_t l = 1; l < old_n; ++l)
            if (mode[l] == 1) s->cell_type[daughter[l]] = s->cell_type[l];
        s->n_labels = next;
        recount(s);
    }
    free(mode);
    free(plan);
    free(moved);
    free(daughter);
}

/* One Monte Carlo step: the colour passes in order, the field step, then
 * division and death (lib.rs:1075-1141). */
/* The infection rule, as glz_gpu_set_infection states it. */
EXPORT int rp_set_infection(rsim *s, int species, int from_type, int to_type, double threshold) {
    if (species < 0 || species >= s->n_species || from_type < 1 || from_type >= s->n_types || to_type < 1 ||
        to_type >= s->n_types || from_type == to_type || !(threshold >= 0.0) || !(threshold * 16777216.0 < 9.0e18))
        return 4;
    s->inf_species = species;
    s->inf_from = from_type;
    s->inf_to = to_type;
    s->inf_threshold = llround(threshold * 16777216.0);
    return 0;
}

/* Replace the nematic field (2 per site) and recount its per-cell sums, as
 * glz_gpu_set_nematic_field does. */
EXPORT int rp_set_nematic_field(rsim *s, const double *field) {
    if (!s->has_nematic) return 2;
    for (int i = 0; i < 2 * s->sites; ++i) s->nem[i] = (float)field[i];
    recount(s);
    return 0;
}

EXPORT void rp_step(rsim *s, uint64_t steps) {
    for (uint64_t r = 0; r < steps; ++r) {
        for (int c = 0; c < s->ncol; ++c) pass(s, c);
        if (s->has_motility)
            for (int i = 0; i < s->sites; ++i) s->act[i] = s->act[i] > 0.0f ? s->act[i] - 1.0f : 0.0f;
        if (s->n_species > 0) field_step(s);
        if (s->inf_species >= 0)
            for (size_t l = 1; l < s->n_labels; ++l)
                if (s->cell_type[l] == s->inf_from && s->dose[l] >= s->inf_threshold) s->cell_type[l] = (uint8_t)s->inf_to;
        if (s->has_pop) population(s);
        s->mcs += 1;
    }
}

/* ---------------------------------------------------------------- accessors */

EXPORT size_t rp_n_labels(const rsim *s) { return s->n_labels; }
EXPORT uint64_t rp_mcs(const rsim *s) { return s->mcs; }
EXPORT uint64_t rp_accepted(const rsim *s) { return s->accepted; }
EXPORT void rp_labels(const rsim *s, uint32_t *out) { memcpy(out, s->labels, s->sites * sizeof(uint32_t)); }
EXPORT void rp_cell_types(const rsim *s, uint8_t *out) { memcpy(out, s->cell_type, s->n_labels); }

/* Volumes and surfaces with the medium's entries recounted from the lattice,
 * as the device reads them back. */
EXPORT void rp_volumes(const rsim *s, uint32_t *out) {
    out[0] = 0;
    for (int i = 0; i < s->sites; ++i)
        if (s->labels[i] == 0) out[0] += 1;
    for (size_t l = 1; l < s->n_labels; ++l) out[l] = s->vol[l] > 0 ? (uint32_t)s->vol[l] : 0;
}

EXPORT void rp_surfaces(const rsim *s, int64_t *out) {
    int64_t medium = 0;
    for (int i = 0; i < s->sites; ++i) {
        if (s->labels[i] != 0) continue;
        int x = i % s->w, y = (i / s->w) % s->h, z = i / (s->w * s->h);
        for (int k = 0; k < s->n_off; ++k) {
            int nb = (wrapi(z + s->off[k][2], s->d) * s->h + wrapi(y + s->off[k][1], s->h)) * s->w +
                     wrapi(x + s->off[k][0], s->w);
            if (nb != i && s->labels[nb] != 0) ++medium;
        }
    }
    out[0] = medium;
    for (size_t l = 1; l < s->n_labels; ++l) out[l] = s->surf[l];
}

EXPORT void rp_volumes_by_colour(const rsim *s, int32_t *out) {
    memcpy(out, s->volc, s->n_labels * s->ncol * sizeof(int32_t));
}

EXPORT void rp_moments(const rsim *s, int64_t *out) { memcpy(out, s->mom, s->n_labels * s->nm * sizeof(int64_t)); }

EXPORT void rp_field(const rsim *s, int k, float *out) {
    memcpy(out, &s->fields[(size_t)k * s->sites], s->sites * sizeof(float));
}

EXPORT void rp_lengths(const rsim *s, double *out) {
    for (size_t l = 0; l < s->n_labels; ++l) out[l] = l ? axis_length(s->dim, s->vol[l], &s->mom[l * s->nm]) : 0.0;
}

/* Unit hooks for the hash, so tests can check the device's draws directly. */
EXPORT uint64_t rp_draw(uint64_t seed, uint32_t site, int32_t step, int colour, int index) {
    return draw(seed, site, step, colour, index);
}
EXPORT float rp_to_f32(uint64_t bits) { return to_f32(bits); }
