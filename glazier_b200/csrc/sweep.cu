// The checkerboard Metropolis copy sweep: one launch per colour.
//
// Replaces `cpm_sweep` of the reference device engine (glazier-cuda/src/
// lib.rs:436-716). Same-colour targets are two apart on every axis, outside
// any neighbourhood, so a pass's copies are independent and the labels a
// target reads do not change during the pass.
//
// Layout of the work:
//   - Persistent CTAs walk the lattice tile by tile. A tile and its one-site
//     halo are staged in shared memory; tiles clear of the periodic edge
//     arrive by a TMA tensor copy issued one tile ahead into the other of two
//     buffers, so the copy of tile i+1 overlaps the work on tile i. Edge
//     tiles, and lattices whose rows are not whole 16-byte units, take
//     wrapped plain loads.
//   - The CTA first draws every target's neighbour pick (one counter-hash
//     draw per target) and keeps only the targets whose neighbour carries
//     another label, about a fifth of them in a tissue, in a shared queue;
//     warps then take the queue 32 copies at a time and price them densely.
//     The expensive path never runs with idle lanes that a light target left
//     behind, and no warp waits on another's share.
//
// Per-cell tallies (volume, surface, exact moment sums) are read from the
// snapshot the rotation in engine.h gives each pass and changed by integer
// atomics whose order does not matter; a pass is therefore deterministic and
// a host replay of the same schedule reproduces it bit for bit.

#include <cooperative_groups.h>
#include <atomic>
#include <cuda.h>

#include <cstdlib>

#include "device.cuh"
#include "engine.h"
#include "neighbours.cuh"
#include "pricing.cuh"

namespace glz {

template <int DIM>
struct Tile;

// A plane's tile height (rows of targets and their window), a build-time knob.
#ifndef GLZ_TILE2_TY
#define GLZ_TILE2_TY 32
#endif

template <>
struct Tile<2> {
    static constexpr int TX = 128, TY = GLZ_TILE2_TY, TZ = 1;
    static constexpr int HX = 4;  // x halo rounded up to 16 bytes for the tensor copy
    static constexpr int PX = TX + 2 * HX, PY = TY + 2, PZ = 1;
    static constexpr int HZ = 0;
    static constexpr int NT = (TX / 2) * (TY / 2);
};

template <>
struct Tile<3> {
    static constexpr int TX = 64, TY = 8, TZ = 8;
    static constexpr int HX = 4;
    static constexpr int PX = TX + 2 * HX, PY = TY + 2, PZ = TZ + 2;
    static constexpr int HZ = 1;
    static constexpr int NT = (TX / 2) * (TY / 2) * (TZ / 2);
};

template <int DIM, int NOFF>
__host__ __device__ constexpr int window_offset(int k) {
    return (neighbour_offset<DIM, NOFF>(k, 2) * Tile<DIM>::PY + neighbour_offset<DIM, NOFF>(k, 1)) * Tile<DIM>::PX +
           neighbour_offset<DIM, NOFF>(k, 0);
}

#ifndef GLZ_SWEEP_MIN_BLOCKS
#define GLZ_SWEEP_MIN_BLOCKS 3
#endif

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemTypes = 16;  // contact tables up to 16 types live in shared memory
constexpr long long kWaitLimit = 1LL << 24;

template <int DIM>
struct SweepSmem {
    static constexpr int WIN = Tile<DIM>::PX * Tile<DIM>::PY * Tile<DIM>::PZ;
    // A tensor copy's shared-memory destination must sit on a 128-byte
    // boundary, so each window buffer is padded to a multiple of 32 labels.
    static constexpr int WIN_STRIDE = (WIN + 31) / 32 * 32;
    static constexpr int TPW = Tile<DIM>::NT / kWarps;  // targets per warp per tile
    alignas(128) uint32_t win[2][WIN_STRIDE];
    uint32_t queue[Tile<DIM>::NT];  // the tile's targets whose neighbour carries another label
    int queued, taken;
    float contact[kSmemTypes * kSmemTypes];
    int woff[26];
    int wring[26];
    alignas(8) unsigned long long mbar[2];
};

// The dominant eigenvalue of a symmetric 3x3 by twenty rounds of power
// iteration and a Rayleigh quotient, as the serial engine takes it
// (moments.rs:165-186).
__device__ double power_lambda(const double c[3][3]) {
    double v0 = 1.0, v1 = 0.7, v2 = 0.3;
    for (int round = 0; round < 20; ++round) {
        double w0 = c[0][0] * v0 + c[0][1] * v1 + c[0][2] * v2;
        double w1 = c[1][0] * v0 + c[1][1] * v1 + c[1][2] * v2;
        double w2 = c[2][0] * v0 + c[2][1] * v1 + c[2][2] * v2;
        double norm = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
        if (norm < 1e-15) return 0.0;
        v0 = w0 / norm;
        v1 = w1 / norm;
        v2 = w2 / norm;
    }
    double w0 = c[0][0] * v0 + c[0][1] * v1 + c[0][2] * v2;
    double w1 = c[1][0] * v0 + c[1][1] * v1 + c[1][2] * v2;
    double w2 = c[2][0] * v0 + c[2][1] * v1 + c[2][2] * v2;
    double lambda = v0 * w0 + v1 * w1 + v2 * w2;
    return lambda > 0.0 ? lambda : 0.0;
}

// 4 sqrt(lambda_max) of a cell's covariance from its n sites and exact sums
// (moments.rs:150-155); a plane takes the 2x2 closed form.
template <int DIM>
__device__ double axis_length(long long n, const long long *m) {
    if (n < 2) return 0.0;
    double dn = (double)n;
    if (DIM == 2) {
        double mx = (double)m[0] / dn, my = (double)m[1] / dn;
        double cxx = (double)m[2] / dn - mx * mx;
        double cyy = (double)m[3] / dn - my * my;
        double cxy = (double)m[4] / dn - mx * my;
        double half = 0.5 * (cxx + cyy), diff = 0.5 * (cxx - cyy);
        double lambda = half + sqrt(diff * diff + cxy * cxy);
        return 4.0 * sqrt(lambda > 0.0 ? lambda : 0.0);
    } else {
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
}

template <int DIM>
__device__ __forceinline__ void site_terms(int ux, int uy, int uz, long long *t) {
    if (DIM == 2) {
        t[0] = ux; t[1] = uy; t[2] = (long long)ux * ux; t[3] = (long long)uy * uy; t[4] = (long long)ux * uy;
    } else {
        t[0] = ux; t[1] = uy; t[2] = uz;
        t[3] = (long long)ux * ux; t[4] = (long long)uy * uy; t[5] = (long long)uz * uz;
        t[6] = (long long)ux * uy; t[7] = (long long)ux * uz; t[8] = (long long)uy * uz;
    }
}

// Change in a cell's length energy (cpu.rs:291-305) when the site with sum
// terms `terms` leaves (sign -1) or joins (+1) it, from the pass snapshot.
template <int DIM>
__device__ __noinline__ double length_delta(const SweepLaunch &a, int type, int label, long long n,
                                            const long long *terms, int sign) {
    constexpr int NM = DIM == 2 ? 5 : 9;
    const size_t at = (size_t)label * a.g.nm;  // the moment words of a cell: NM, then the nematic sums
    long long m[NM], after[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        m[k] = a.mom_base[at + k] + a.mom_prev[at + k];
        after[k] = m[k] + sign * terms[k];
    }
    double tl = a.t.target_length[type];
    double before = axis_length<DIM>(n, m) - tl;
    double now = axis_length<DIM>(n + sign, after) - tl;
    return a.t.lambda_length[type] * (now * now - before * before);
}

// Change in a cell's nematic energy (cpu.rs:315-332, lib.rs:603-637) when the
// site with sum terms `terms` (its moment terms, then its field components in
// fixed point) leaves (sign -1) or joins (+1) it: -lambda (f' . a' - f . a),
// f the cell's field sum and a its anisotropy, from the pass snapshot.
template <int DIM>
__device__ __noinline__ double nematic_delta(const SweepLaunch &a, int type, int label, long long n,
                                             const long long *terms, int sign) {
    constexpr int NM = DIM == 2 ? 5 : 9;
    const size_t at = (size_t)label * a.g.nm;
    long long m[NM + 2], after[NM + 2];
#pragma unroll
    for (int k = 0; k < NM + 2; ++k) {
        m[k] = a.mom_base[at + k] + a.mom_prev[at + k];
        after[k] = m[k] + sign * terms[k];
    }
    double a0, a1, b0, b1;
    anisotropy<DIM>(n, m, a0, a1);
    anisotropy<DIM>(n + sign, after, b0, b1);
    const double scale = 1.0 / 4294967296.0;
    const double before = (double)m[NM] * scale * a0 + (double)m[NM + 1] * scale * a1;
    const double now = (double)after[NM] * scale * b0 + (double)after[NM + 1] * scale * b1;
    return -a.t.lambda_nematic[type] * (now - before);
}

// lib.rs:371-389: whether the ring positions in `present` are one piece.
__device__ __forceinline__ bool one_piece(uint32_t present, const uint32_t *adjacency) {
    if (present == 0u || (present & (present - 1u)) == 0u) return true;
    uint32_t reached = present & (~present + 1u);
    for (int round = 0; round < 26; ++round) {
        uint32_t grown = reached, rest = reached;
        while (rest) {
            int k = __ffs(rest) - 1;
            grown |= adjacency[k];
            rest &= rest - 1u;
        }
        grown &= present;
        if (grown == reached) break;
        reached = grown;
    }
    return reached == present;
}

// Position of target j of a tile: local coordinates in the tile.
template <int DIM>
__device__ __forceinline__ void target_of(int j, int colour, int &lx, int &ly, int &lz) {
    using T = Tile<DIM>;
    const int jx = j % (T::TX / 2);
    const int jy = (j / (T::TX / 2)) % (T::TY / 2);
    const int jz = DIM == 3 ? j / ((T::TX / 2) * (T::TY / 2)) : 0;
    lx = 2 * jx + (colour & 1);
    ly = 2 * jy + ((colour >> 1) & 1);
    lz = DIM == 3 ? 2 * jz + ((colour >> 2) & 1) : 0;
}

// The rare parts of pricing live out of line, so the registers they need do
// not weigh on the common path.

// The per-colour guard: whether cell `old` keeps a site of a colour other than
// the pass's own, which no copy in this pass can take.
__device__ __noinline__ bool keeps_other_colour(const SweepLaunch &a, uint32_t old) {
    int other = 0;
    for (int c = 0; c < a.g.ncol; ++c)
        if (c != a.colour) other += a.vol_by_colour[(size_t)old * a.g.ncol + c];
    return other != 0;
}

// The connectivity veto (lib.rs:511-521): the ring positions of `old` around
// the target must be one piece.
__device__ __noinline__ bool ring_one_piece(const SweepLaunch &a, const int *wring, const uint32_t *win, int wc,
                                            uint32_t old) {
    uint32_t present = 0;
    for (int k = 0; k < a.g.ring_n; ++k)
        if (win[wc + wring[k]] == old) present |= 1u << k;
    return one_piece(present, a.g.adjacency);
}

// The moment-sum terms of the target site in a cell's own frame.
template <int DIM>
__device__ __forceinline__ void terms_of(const SweepLaunch &a, uint32_t label, int x, int y, int z, long long *t) {
    const int *an = &a.anchor[(size_t)label * 4];
    site_terms<DIM>(fold_int(x - an[0], a.g.w), fold_int(y - an[1], a.g.h), fold_int(z - an[2], a.g.d), t);
}

// The geometric mean of the activity over the sites of `label` around `site`
// (x, y, z), the site itself included; zero as soon as one of them has none
// left (lib.rs:391-424, motility.rs:58-79). Labels and activity are the
// pass's starting values: a pass with motility defers its writes.
template <int DIM>
__device__ __noinline__ float activity_mean(const SweepLaunch &a, uint32_t site, int x, int y, int z,
                                            uint32_t label) {
    const float here = a.activity[site];
    if (!(here > 0.0f)) return 0.0f;
    float log_sum = motility_log(here), count = 1.0f;
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    for (int k = 0; k < a.g.n_off; ++k) {
        const uint32_t n = (uint32_t)(((size_t)wrap(z + a.g.off[k][2], D) * H + wrap(y + a.g.off[k][1], H)) * W +
                                      wrap(x + a.g.off[k][0], W));
        if (n == site || a.labels[n] != label) continue;
        const float v = a.activity[n];
        if (!(v > 0.0f)) return 0.0f;
        log_sum = __fadd_rn(log_sum, motility_log(v));
        count = __fadd_rn(count, 1.0f);
    }
    return metropolis_exp(__fdiv_rn(log_sum, count));
}

// The length, chemotaxis, motility and drift terms of a copy (cpu.rs:291-305,
// 341-395).
template <int DIM>
__device__ __noinline__ float extra_terms(const SweepLaunch &a, uint32_t old, uint32_t nw, int t_old, int t_new,
                                          int vol_old, int vol_new, int x, int y, int z, int pick, uint32_t target,
                                          float delta) {
    constexpr int NM = DIM == 2 ? 5 : 9;
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    // the length and nematic terms, leaving cell first (lib.rs:578-639)
    if (a.has_length || a.has_nematic) {
        long long terms[NM + 2];
        if (a.has_nematic) {
            terms[NM] = nematic_fixed(a.nematic[2 * (size_t)target]);
            terms[NM + 1] = nematic_fixed(a.nematic[2 * (size_t)target + 1]);
        }
        const bool len_old = a.has_length && a.t.lambda_length[t_old] != 0.0;
        const bool nem_old = a.has_nematic && a.t.lambda_nematic[t_old] != 0.0;
        if (old != 0 && (len_old || nem_old)) {
            terms_of<DIM>(a, old, x, y, z, terms);
            if (len_old) delta = __fadd_rn(delta, (float)length_delta<DIM>(a, t_old, old, vol_old, terms, -1));
            if (nem_old) delta = __fadd_rn(delta, (float)nematic_delta<DIM>(a, t_old, old, vol_old, terms, -1));
        }
        const bool len_new = a.has_length && a.t.lambda_length[t_new] != 0.0;
        const bool nem_new = a.has_nematic && a.t.lambda_nematic[t_new] != 0.0;
        if (nw != 0 && (len_new || nem_new)) {
            terms_of<DIM>(a, nw, x, y, z, terms);
            if (len_new) delta = __fadd_rn(delta, (float)length_delta<DIM>(a, t_new, nw, vol_new, terms, 1));
            if (nem_new) delta = __fadd_rn(delta, (float)nematic_delta<DIM>(a, t_new, nw, vol_new, terms, 1));
        }
    }
    const int ox = a.g.off[pick][0], oy = a.g.off[pick][1], oz = a.g.off[pick][2];
    const int sx = wrap(x + ox, W), sy = wrap(y + oy, H), sz = wrap(z + oz, D);
    if (a.has_chemotaxis && nw != 0) {
        const uint32_t source = (uint32_t)(((size_t)sz * H + sy) * W + sx);
        for (int s = 0; s < a.n_species; ++s) {
            const float lam = a.t.chemotaxis[t_new * a.n_species + s];
            if (lam == 0.0f) continue;
            const float *f = a.fields[s];
            delta = __fsub_rn(delta, __fmul_rn(lam, __fsub_rn(f[target], f[source])));
        }
    }
    // Motility (cpu.rs:346-352, lib.rs:656-663): the cell's memory pulls it
    // where it has been.
    if (a.has_motility && nw != 0) {
        const float lam = a.t.lambda_activity[t_new], top = a.t.max_activity[t_new];
        if (lam != 0.0f && top > 0.0f) {
            const uint32_t source = (uint32_t)(((size_t)sz * H + sy) * W + sx);
            const float into = activity_mean<DIM>(a, source, sx, sy, sz, nw);
            const float out_of = activity_mean<DIM>(a, target, x, y, z, old);
            delta = __fsub_rn(delta, __fmul_rn(__fdiv_rn(lam, top), __fsub_rn(into, out_of)));
        }
    }
    // The drift (cpu.rs:360-369, lib.rs:664-673): work e . (target - source),
    // the step folded onto the lattice.
    if (a.has_external && nw != 0) {
        const float ex = a.t.external[3 * t_new], ey = a.t.external[3 * t_new + 1], ez = a.t.external[3 * t_new + 2];
        if (ex != 0.0f || ey != 0.0f || ez != 0.0f) {
            const float fx = (float)fold_int(x - sx, W), fy = (float)fold_int(y - sy, H), fz = (float)fold_int(z - sz, D);
            delta = __fsub_rn(delta, __fadd_rn(__fadd_rn(__fmul_rn(ex, fx), __fmul_rn(ey, fy)), __fmul_rn(ez, fz)));
        }
    }
    return delta;
}

// The moment sums follow an accepted copy: the site leaves `old` and joins `nw`.
template <int DIM>
__device__ __noinline__ void commit_moments(const SweepLaunch &a, uint32_t old, uint32_t nw, int x, int y, int z) {
    constexpr int NM = DIM == 2 ? 5 : 9;
    const int nm = a.g.nm;
    long long terms[NM], q[2] = {0, 0};
    if (a.has_nematic) {
        const size_t site = ((size_t)z * a.g.h + y) * a.g.w + x;
        q[0] = nematic_fixed(a.nematic[2 * site]);
        q[1] = nematic_fixed(a.nematic[2 * site + 1]);
    }
    if (old != 0) {
        terms_of<DIM>(a, old, x, y, z, terms);
#pragma unroll
        for (int k = 0; k < NM; ++k) atomicAdd(&a.mom_cur[(size_t)old * nm + k], (unsigned long long)(-terms[k]));
        if (a.has_nematic)
            for (int k = 0; k < 2; ++k) atomicAdd(&a.mom_cur[(size_t)old * nm + NM + k], (unsigned long long)(-q[k]));
    }
    if (nw != 0) {
        terms_of<DIM>(a, nw, x, y, z, terms);
#pragma unroll
        for (int k = 0; k < NM; ++k) atomicAdd(&a.mom_cur[(size_t)nw * nm + k], (unsigned long long)terms[k]);
        if (a.has_nematic)
            for (int k = 0; k < 2; ++k) atomicAdd(&a.mom_cur[(size_t)nw * nm + NM + k], (unsigned long long)q[k]);
    }
}

// Price one copy attempt whose neighbour pick is known to carry another label
// and commit it if the Metropolis test takes it. UNIFORM: every label carries
// one type, so the contact sum is J times a difference of like-neighbour
// counts (the host has checked that J m is exact in f32 for every count m,
// which makes it the same number the neighbour-by-neighbour sum rounds to)
// and the per-type constants come from the launch parameters.
//
// EXTRAS false compiles out the length, chemotaxis, connectivity and moment
// parts, for launches whose model has none of them. `woff`, `contact` and
// `wring` are the shared-memory tables: window offset of each pick, the
// contact matrix when `small_types`, the connectivity ring.
template <int DIM, int NOFF, bool UNIFORM, bool EXTRAS>
__device__ __forceinline__ void price_and_commit(const SweepLaunch &a, const int *woff, const float *contact,
                                                 const int *wring, const uint32_t *win, uint32_t entry, int x0,
                                                 int y0, int z0, bool small_types) {
    using T = Tile<DIM>;
    const int W = a.g.w, H = a.g.h;
    const int j = (int)(entry & 0xffffu);
    const int pick = (int)(entry >> 16);
    int lx, ly, lz;
    target_of<DIM>(j, a.colour, lx, ly, lz);
    const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
    const uint32_t target = (uint32_t)((z * H + y) * W + x);
    const int wc = ((lz + T::HZ) * T::PY + (ly + 1)) * T::PX + (lx + T::HX);
    const uint32_t old = win[wc];
    const uint32_t nw = win[wc + woff[pick]];

    // The snapshot tallies of both cells, requested before the neighbour loop
    // so their latency hides behind it.
    long long prev_old = 0, prev_new = 0;
    int2 base_old = make_int2(0, 0), base_new = make_int2(0, 0);
    if (old != 0) {
        base_old = a.vs_base[old];
        prev_old = a.vs_prev[old];
    }
    if (nw != 0) {
        base_new = a.vs_base[nw];
        prev_new = a.vs_prev[nw];
    }
    const int t_old = UNIFORM ? a.uniform_type : a.cell_type[old];
    const int t_new = UNIFORM ? a.uniform_type : a.cell_type[nw];

    float delta = 0.0f;
    int like_old = 0, like_new = 0;
    if (UNIFORM) {
#pragma unroll
        for (int k = 0; k < NOFF; ++k) {
            const uint32_t ln = win[wc + window_offset<DIM, NOFF>(k)];
            like_old += ln == old;
            like_new += ln == nw;
        }
        delta = __fmul_rn(a.uniform_contact, (float)(like_old - like_new));
    } else {
#pragma unroll
        for (int k = 0; k < NOFF; ++k) {
            const uint32_t ln = win[wc + window_offset<DIM, NOFF>(k)];
            const int tn = ln == old ? t_old : (ln == nw ? t_new : (int)a.cell_type[ln]);
            if (ln != old) {
                const float j_old =
                    small_types ? contact[t_old * a.n_types + tn] : a.t.contact[t_old * a.n_types + tn];
                delta = __fsub_rn(delta, j_old);
            } else {
                ++like_old;
            }
            if (ln != nw) {
                const float j_new =
                    small_types ? contact[t_new * a.n_types + tn] : a.t.contact[t_new * a.n_types + tn];
                delta = __fadd_rn(delta, j_new);
            } else {
                ++like_new;
            }
        }
    }

    if (old != 0) {
        // A like neighbour is a site of another colour, since every neighbour
        // of a target is; only a target with none needs the per-colour count.
        if (like_old == 0 && !keeps_other_colour(a, old)) return;
        if (EXTRAS && a.g.ring_n > 0 && a.t.connected[t_old] && !ring_one_piece(a, wring, win, wc, old)) return;
    }
    const int ds_old = 2 * like_old - NOFF;
    const int ds_new = NOFF - 2 * like_new;

    int vol_old, surf_old, vol_new, surf_new;
    {
        int dv, ds;
        unpack_delta(prev_old, dv, ds);
        vol_old = base_old.x + dv;
        surf_old = base_old.y + ds;
        unpack_delta(prev_new, dv, ds);
        vol_new = base_new.x + dv;
        surf_new = base_new.y + ds;
    }
    delta = size_terms<UNIFORM>(a, old, nw, t_old, t_new, vol_old, vol_new, surf_old, surf_new, ds_old, ds_new, delta);
    if (EXTRAS && (a.has_length || a.has_chemotaxis || a.has_external || a.has_motility || a.has_nematic))
        delta = extra_terms<DIM>(a, old, nw, t_old, t_new, vol_old, vol_new, x, y, z, pick, target, delta);

    // Metropolis: a copy that lowers the energy (or keeps it) is taken, else
    // with probability exp(-delta / T). The draw and the exponential are
    // computed on every lane, so the test needs no branch; a lane whose delta
    // is not positive takes the copy whatever they say.
    {
        const float u = to_f32(draw(a.key_accept, target));
        if (!(delta <= 0.0f || u < metropolis_exp(__fmul_rn(-delta, a.beta)))) return;
    }

    if (EXTRAS && a.has_motility) {
        const int k = atomicAdd(a.pending_count, 1);
        a.pending[k] = make_uint2(target, nw);
    } else {
        a.labels[target] = nw;
    }
    if (old != 0) {
        atomicAdd(&a.vs_cur[old], pack_delta(-1, ds_old));
        atomicSub(&a.vol_by_colour[(size_t)old * a.g.ncol + a.colour], 1);
    }
    if (nw != 0) {
        atomicAdd(&a.vs_cur[nw], pack_delta(1, ds_new));
        atomicAdd(&a.vol_by_colour[(size_t)nw * a.g.ncol + a.colour], 1);
    }
    if (EXTRAS && a.tracks) commit_moments<DIM>(a, old, nw, x, y, z);
}

template <int DIM>
__device__ __forceinline__ void tile_origin(int t, int W, int H, int &x0, int &y0, int &z0) {
    using T = Tile<DIM>;
    const int tiles_x = (W + T::TX - 1) / T::TX;
    const int tiles_y = (H + T::TY - 1) / T::TY;
    x0 = (t % tiles_x) * T::TX;
    y0 = ((t / tiles_x) % tiles_y) * T::TY;
    z0 = DIM == 3 ? (t / (tiles_x * tiles_y)) * T::TZ : 0;
}

template <int DIM>
__device__ __forceinline__ bool tile_interior(const SweepLaunch &a, int x0, int y0, int z0) {
    using T = Tile<DIM>;
    return a.use_tma && x0 >= T::HX && x0 + T::TX + T::HX <= a.g.w && y0 >= 1 && y0 + T::TY + 1 <= a.g.h &&
           (DIM == 2 || (z0 >= 1 && z0 + T::TZ + 1 <= a.g.d));
}

// One thread issues the tensor copy of a tile's window into `dst`, arriving
// on `bar` with the byte count the copy will deliver.
template <int DIM>
__device__ __forceinline__ void issue_window(const CUtensorMap &tmap, uint32_t *dst, unsigned long long *bar, int x0,
                                             int y0, int z0) {
    using T = Tile<DIM>;
    const uint32_t b = smem_addr(bar);
    const uint32_t bytes = SweepSmem<DIM>::WIN * sizeof(uint32_t);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    const uint64_t map = reinterpret_cast<uint64_t>(&tmap);
    // x0 - HX is a multiple of 4 labels, i.e. of 16 bytes, as a tensor copy's
    // inner coordinate must be.
    if (DIM == 2) {
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
                "r"(smem_addr(dst)),
            "l"(map), "r"(x0 - T::HX), "r"(y0 - 1), "r"(b)
            : "memory");
    } else {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];" ::"r"(smem_addr(dst)),
            "l"(map), "r"(x0 - T::HX), "r"(y0 - 1), "r"(z0 - 1), "r"(b)
            : "memory");
    }
}

// Wrapped plain loads of a tile's window, for tiles on the periodic edge and
// lattices whose rows are not whole 16-byte units.
template <int DIM>
__device__ __forceinline__ void load_window_plain(const SweepLaunch &a, uint32_t *win, int x0, int y0, int z0) {
    using T = Tile<DIM>;
    using Smem = SweepSmem<DIM>;
    const int tid = threadIdx.x;
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    // Where every window coordinate lies within one lattice span of it (the
    // halo reaches back no further than a span, the last tile's window no
    // further than one span past the end) a compare wraps it; otherwise the
    // remainder does.
    const auto reach = [](int n, int t, int h) { return h <= n && ((n - 1) / t) * t + t + h <= 2 * n; };
    const bool once = reach(W, T::TX, T::HX) && reach(H, T::TY, 1) && (DIM == 2 || reach(D, T::TZ, T::HZ));
    for (int i = tid; i < Smem::WIN; i += blockDim.x) {
        const int px = i % T::PX;
        const int py = (i / T::PX) % T::PY;
        const int pz = i / (T::PX * T::PY);
        int gx = x0 - T::HX + px, gy = y0 - 1 + py, gz = DIM == 3 ? z0 - 1 + pz : 0;
        if (once) {
            gx += gx < 0 ? W : (gx >= W ? -W : 0);
            gy += gy < 0 ? H : (gy >= H ? -H : 0);
            if (DIM == 3) gz += gz < 0 ? D : (gz >= D ? -D : 0);
        } else {
            gx = wrap(gx, W);
            gy = wrap(gy, H);
            gz = DIM == 3 ? wrap(gz, D) : 0;
        }
        win[i] = a.labels[((size_t)gz * H + gy) * W + gx];
    }
    // generic writes to a buffer a later tensor copy will overwrite
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
}

// Price every target of the pass's colour in one tile whose window is in
// shared memory: the light pass queues the targets whose neighbour pick
// carries another label, the heavy pass prices and commits the queue.
template <int DIM, int NOFF, bool UNIFORM>
__device__ __forceinline__ void price_tile(const SweepLaunch &a, SweepSmem<DIM> &S, const uint32_t *win, int x0,
                                           int y0, int z0, bool small_types) {
    using T = Tile<DIM>;
    using Smem = SweepSmem<DIM>;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    // Light pass: every target's pick; only targets whose neighbour
    // carries another label go into the tile's queue. A warp keeps its
    // entries in registers and reserves queue room once per tile.
    constexpr int PER_LANE = Smem::TPW / 32;
    const bool full = x0 + T::TX <= W && y0 + T::TY <= H && (DIM == 2 || z0 + T::TZ <= D);
    const int tile_base = (z0 * H + y0) * W + x0;
    uint32_t entries[PER_LANE];
    unsigned masks[PER_LANE];
    int total = 0;
#pragma unroll
    for (int k = 0; k < PER_LANE; ++k) {
        const int j = warp * Smem::TPW + k * 32 + lane;
        int lx, ly, lz;
        target_of<DIM>(j, a.colour, lx, ly, lz);
        bool active = false;
        if (full || (x0 + lx < W && y0 + ly < H && (DIM == 2 || z0 + lz < D))) {
            const uint32_t target = (uint32_t)(tile_base + (lz * H + ly) * W + lx);
            const int wc = ((lz + T::HZ) * T::PY + (ly + 1)) * T::PX + (lx + T::HX);
            const int pick = pick_of<NOFF>(draw(a.key_pick, target));
            active = win[wc] != win[wc + S.woff[pick]];
            entries[k] = (uint32_t)j | ((uint32_t)pick << 16);
        }
        masks[k] = __ballot_sync(0xffffffffu, active);
        total += __popc(masks[k]);
    }
    int base = 0;
    if (lane == 0 && total) base = atomicAdd(&S.queued, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < PER_LANE; ++k) {
        if (masks[k] & (1u << lane)) S.queue[base + __popc(masks[k] & below)] = entries[k];
        base += __popc(masks[k]);
    }
    __syncthreads();
    // Heavy pass: warps take the queue 32 copies at a time.
    const int queued = S.queued;
    for (;;) {
        int first = 0;
        if (lane == 0) first = atomicAdd(&S.taken, 32);
        first = __shfl_sync(0xffffffffu, first, 0);
        if (first >= queued) break;
        if (first + lane < queued)
            price_and_commit<DIM, NOFF, UNIFORM, true>(a, S.woff, S.contact, S.wring, win, S.queue[first + lane], x0,
                                                       y0, z0, small_types);
    }
    __syncthreads();
    if (tid == 0) {
        S.queued = 0;
        S.taken = 0;
    }
}

// Wait for phase `parity` of an mbarrier, giving up after kWaitLimit polls.
__device__ __forceinline__ uint32_t wait_parity(unsigned long long *bar, uint32_t parity) {
    const uint32_t b = smem_addr(bar);
    uint32_t done = 0;
    for (long long spin = 0; spin < kWaitLimit && !done; ++spin) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
    }
    return done;
}

// Tally rotation for the next pass, spread over the whole grid: no thread of
// this pass reads what is written here (engine.h).
template <int DIM>
__device__ __forceinline__ void rotate_tallies(const SweepLaunch &a) {
    const int NM = a.g.nm;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t n = a.n_live ? (size_t)*a.n_live : (size_t)a.n_labels;
    for (size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
        int dv, ds;
        unpack_delta(a.vs_prev[l], dv, ds);
        const int2 b = a.vs_base[l];
        a.vs_next_base[l] = make_int2(b.x + dv, b.y + ds);
        a.vs_clear[l] = 0;
        if (a.tracks) {
#pragma unroll
            for (int k = 0; k < NM; ++k) {
                a.mom_next_base[l * NM + k] = a.mom_base[l * NM + k] + a.mom_prev[l * NM + k];
                a.mom_clear[l * NM + k] = 0;
            }
        }
    }
}

template <int DIM, int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kThreads, GLZ_SWEEP_MIN_BLOCKS) sweep_kernel(const __grid_constant__ SweepLaunch a,
                                                         const __grid_constant__ CUtensorMap tmap) {
    using T = Tile<DIM>;
    using Smem = SweepSmem<DIM>;
    static_assert(Smem::WIN_STRIDE * sizeof(uint32_t) % 128 == 0, "window buffers must stay 128-byte aligned");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // The launch asks for 128 spare bytes so the layout can start on a
    // 128-byte boundary whatever the dynamic region's own alignment.
    const uint32_t raw = smem_addr(smem_raw);
    Smem &S = *reinterpret_cast<Smem *>(smem_raw + ((128u - (raw & 127u)) & 127u));

    const int tid = threadIdx.x;
    if (smem_addr(S.win[0]) & 127u) {  // never true by construction; refuse rather than copy misaligned
        if (tid == 0) atomicExch(a.error_flag, 3);
        return;
    }
    const int W = a.g.w, H = a.g.h, D = a.g.d;

    const bool small_types = a.n_types <= kSmemTypes;
    if (small_types)
        for (int i = tid; i < a.n_types * a.n_types; i += blockDim.x) S.contact[i] = a.t.contact[i];
    if (tid < NOFF) S.woff[tid] = (a.g.off[tid][2] * T::PY + a.g.off[tid][1]) * T::PX + a.g.off[tid][0];
    if (tid < a.g.ring_n) S.wring[tid] = (a.g.ring[tid][2] * T::PY + a.g.ring[tid][1]) * T::PX + a.g.ring[tid][0];
    if (tid == 0) {
        S.queued = 0;
        S.taken = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Nothing above reads what the previous pass writes; a programmatic launch
    // may have started this grid before it ended (see launch_lean).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    rotate_tallies<DIM>(a);
    __syncthreads();

    const int tiles = ((W + T::TX - 1) / T::TX) * ((H + T::TY - 1) / T::TY) * (DIM == 3 ? (D + T::TZ - 1) / T::TZ : 1);
    int waited[2] = {0, 0};
    bool pending[2] = {false, false};  // a copy issued into the buffer and not yet waited for
    int t = blockIdx.x;
    if (t < tiles) {
        int x0, y0, z0;
        tile_origin<DIM>(t, W, H, x0, y0, z0);
        if (tile_interior<DIM>(a, x0, y0, z0)) {
            if (tid == 0) issue_window<DIM>(tmap, S.win[0], &S.mbar[0], x0, y0, z0);
            pending[0] = true;
        }
    }
    for (int it = 0; t < tiles; t += gridDim.x, ++it) {
        const int buf = it & 1;
        int x0, y0, z0;
        tile_origin<DIM>(t, W, H, x0, y0, z0);
        const int next = t + gridDim.x;
        if (next < tiles) {
            int nx0, ny0, nz0;
            tile_origin<DIM>(next, W, H, nx0, ny0, nz0);
            if (tile_interior<DIM>(a, nx0, ny0, nz0)) {
                if (tid == 0) issue_window<DIM>(tmap, S.win[buf ^ 1], &S.mbar[buf ^ 1], nx0, ny0, nz0);
                pending[buf ^ 1] = true;
            }
        }
        uint32_t *win = S.win[buf];
        if (tile_interior<DIM>(a, x0, y0, z0)) {
            // Bounded wait: a copy that never lands sets the error flag and the
            // CTA stops rather than spinning for ever.
            const uint32_t done = wait_parity(&S.mbar[buf], waited[buf] & 1);
            waited[buf] += 1;
            pending[buf] = false;
            if (!__syncthreads_and(done)) {
                // Before leaving, give a copy still in flight into the other
                // buffer its own bounded wait, so no copy lands after exit.
                if (pending[buf ^ 1]) wait_parity(&S.mbar[buf ^ 1], waited[buf ^ 1] & 1);
                if (tid == 0) atomicExch(a.error_flag, 1);
                return;
            }
        } else {
            load_window_plain<DIM>(a, win, x0, y0, z0);
        }
        price_tile<DIM, NOFF, UNIFORM>(a, S, win, x0, y0, z0, small_types);
    }
}

// ---------------------------------------------------------------- the lean sweep
//
// Models whose copies price only contact, volume and surface terms (no
// length, chemotaxis, connectivity veto or moment tracking) take this kernel:
// the same draws, copies and commits as sweep_kernel, with the work laid out
// so that no CTA-wide barrier stands between tiles.
//   - Each warp owns a fixed share of every tile's targets (two rows of them
//     in a plane) and prices it alone: light pass, its own queue, heavy pass.
//     Warps drift apart by up to the depth of the window ring.
//   - Windows arrive through a ring of kLeanStages buffers, by tensor copies
//     issued up to kLeanStages tiles ahead; the last warp to finish with a
//     buffer issues the next copy into it.
//   - A tile on the periodic edge takes the copy with its out-of-lattice
//     cells filled, then the warps overwrite those cells with the wrapped
//     labels, each a disjoint share of window rows, and meet on an mbarrier
//     (a bounded wait) before pricing. Without tensor copies (rows that are
//     not whole 16-byte units, or a lattice smaller than a window) every cell
//     of every window is loaded that way.
#ifndef GLZ_LEAN_STAGES
#define GLZ_LEAN_STAGES 3
#endif
constexpr int kLeanStages = GLZ_LEAN_STAGES;
#ifndef GLZ_LEAN_WARPS
#define GLZ_LEAN_WARPS 8
#endif
#ifndef GLZ_LEAN_MIN_BLOCKS
#define GLZ_LEAN_MIN_BLOCKS 3
#endif
constexpr int kLeanWarps = GLZ_LEAN_WARPS;
constexpr int kLeanThreads = 32 * kLeanWarps;
constexpr int kRotate = 2;  // labels per thread whose rotation reads are copied in ahead

template <int DIM>
struct LeanSmem {
    static constexpr int WIN = SweepSmem<DIM>::WIN;
    static constexpr int WIN_STRIDE = SweepSmem<DIM>::WIN_STRIDE;
    static constexpr int TPW = Tile<DIM>::NT / kLeanWarps;  // targets per warp per tile
    alignas(128) uint32_t win[kLeanStages][WIN_STRIDE];
    uint32_t queue[kLeanWarps][TPW + 32];  // a tile's entries after fewer than 32 held from the tile before
    float contact[kSmemTypes * kSmemTypes];
    int woff[26];
    int done[kLeanStages];    // warps finished with the buffer's current tile
    int issued[kLeanStages];  // copies issued into the buffer
    alignas(8) unsigned long long full[kLeanStages];     // the buffer's copy has landed
    alignas(8) unsigned long long patched[kLeanStages];  // every warp has patched its rows
    // the tally rotation's first kRotate labels per thread, copied in while the tiles run
    alignas(16) int2 rot_base[2 * kLeanThreads];
    alignas(16) long long rot_prev[2 * kLeanThreads];
};

// Tensor copies for every tile, edge tiles included: the lattice's rows are
// whole 16-byte units and the lattice is at least a window on every axis, so
// an edge window wraps at most once per axis.
template <int DIM>
__device__ __forceinline__ bool lean_copies(const SweepLaunch &a) {
    using T = Tile<DIM>;
    return a.use_tma && a.g.w >= T::PX && a.g.h >= T::PY && (DIM == 2 || a.g.d >= T::PZ);
}

// Start tile i of this CTA's list into its buffer: a tensor copy, or a bare
// arrival when copies are off, so the buffer's phase completes either way.
template <int DIM>
__device__ __forceinline__ void lean_issue(const SweepLaunch &a, const CUtensorMap &tmap, LeanSmem<DIM> &S, int i,
                                           bool copies) {
    const int slot = i % kLeanStages;
    S.issued[slot] += 1;
    if (copies) {
        int x0, y0, z0;
        tile_origin<DIM>((int)blockIdx.x + i * (int)gridDim.x, a.g.w, a.g.h, x0, y0, z0);
        issue_window<DIM>(tmap, S.win[slot], &S.full[slot], x0, y0, z0);
    } else {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&S.full[slot])) : "memory");
    }
}

// The warp's rows of an edge tile's window (rows warp, warp + kLeanWarps, ...):
// in a row whose y (and z) lie in the lattice only the cells the copy left
// filled, else every cell, from the wrapped labels.
template <int DIM>
__device__ __forceinline__ void lean_patch(const SweepLaunch &a, uint32_t *win, int x0, int y0, int z0, bool copies) {
    using T = Tile<DIM>;
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Whether every window coordinate is at most one lattice span outside it
    // (the halo reaches back no further than a span, the last tile's window
    // no further than one span past the end), so one step wraps it.
    const auto reach = [](int n, int t, int h) { return h <= n && ((n - 1) / t) * t + t + h <= 2 * n; };
    const bool once = reach(W, T::TX, T::HX) && reach(H, T::TY, 1) && (DIM == 2 || reach(D, T::TZ, T::HZ));
    int lo = 0, hi = 0;  // window columns [lo, hi) lie inside the lattice
    if (copies) {
        lo = T::HX - x0 > 0 ? T::HX - x0 : 0;
        hi = W - x0 + T::HX < T::PX ? W - x0 + T::HX : T::PX;
    }
    for (int r = warp; r < T::PY * T::PZ; r += kLeanWarps) {
        const int py = r % T::PY, pz = r / T::PY;
        const int gy = y0 - 1 + py, gz = DIM == 3 ? z0 - T::HZ + pz : 0;
        const bool inside = copies && gy >= 0 && gy < H && gz >= 0 && gz < D;
        const auto wr = [once](int v, int n) { return once ? (v < 0 ? v + n : (v >= n ? v - n : v)) : wrap(v, n); };
        const uint32_t *row = a.labels + ((size_t)(DIM == 3 ? wr(gz, D) : 0) * H + wr(gy, H)) * W;
        uint32_t *dst = win + r * T::PX;
        const int n = inside ? lo + (T::PX - hi) : T::PX;
        for (int c = lane; c < n; c += 32) {
            const int px = inside && c >= lo ? hi + (c - lo) : c;
            dst[px] = row[wr(x0 - T::HX + px, W)];
        }
    }
}

// The warp is done with tile i's buffer (lane 0 acts); the last warp out
// refills it with tile i + kLeanStages.
template <int DIM>
__device__ __forceinline__ void lean_release(const SweepLaunch &a, const CUtensorMap &tmap, LeanSmem<DIM> &S, int i,
                                             int mine, bool copies) {
    if ((threadIdx.x & 31) != 0) return;
    const int slot = i % kLeanStages;
    __threadfence_block();
    if (atomicAdd(&S.done[slot], 1) == kLeanWarps - 1) {
        S.done[slot] = 0;
        if (i + kLeanStages < mine) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            lean_issue<DIM>(a, tmap, S, i + kLeanStages, copies);
        }
    }
}

template <int DIM, int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kLeanThreads, GLZ_LEAN_MIN_BLOCKS)
    lean_sweep_kernel(const __grid_constant__ SweepLaunch a, const __grid_constant__ CUtensorMap tmap) {
    using T = Tile<DIM>;
    using Smem = LeanSmem<DIM>;
    constexpr int PER_LANE = Smem::TPW / 32;
    static_assert(Smem::TPW % 32 == 0, "a warp's targets fill whole lanes");
    static_assert(Smem::WIN_STRIDE * sizeof(uint32_t) % 128 == 0, "window buffers must stay 128-byte aligned");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    Smem &S = *reinterpret_cast<Smem *>(smem_raw + ((128u - (raw & 127u)) & 127u));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (smem_addr(S.win[0]) & 127u) {  // never true by construction; refuse rather than copy misaligned
        if (tid == 0) atomicExch(a.error_flag, 3);
        return;
    }
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const int tiles = ((W + T::TX - 1) / T::TX) * ((H + T::TY - 1) / T::TY) * (DIM == 3 ? (D + T::TZ - 1) / T::TZ : 1);
    const int mine = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const bool copies = lean_copies<DIM>(a);

    if (tid == 0) {
        for (int k = 0; k < kLeanStages; ++k) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.full[k])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&S.patched[k])), "r"(kLeanWarps));
            S.done[k] = 0;
            S.issued[k] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const bool small_types = a.n_types <= kSmemTypes;
    if (!UNIFORM && small_types)
        for (int k = tid; k < a.n_types * a.n_types; k += blockDim.x) S.contact[k] = a.t.contact[k];
#pragma unroll
    for (int k = 0; k < NOFF; ++k)
        if (tid == k) S.woff[k] = window_offset<DIM, NOFF>(k);
    // Everything above reads nothing the previous pass writes. Launched
    // programmatically, this grid may have started before that pass ended:
    // wait here for it to finish (its labels and tallies visible), then let
    // the next pass's grid start its own prologue.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tid == 0)
        for (int i = 0; i < kLeanStages && i < mine; ++i) lean_issue<DIM>(a, tmap, S, i, copies);
    // Tally rotation (no thread of this pass reads what it writes): the reads
    // of each thread's first kRotate labels are copied into shared memory now
    // and finished after the tiles, so their latency hides behind pricing.
    const size_t rot_stride = (size_t)gridDim.x * blockDim.x;
    const size_t rot_first = (size_t)blockIdx.x * blockDim.x + tid;
#pragma unroll
    for (int k = 0; k < kRotate; ++k) {
        const size_t l = rot_first + k * rot_stride;
        if (l < (size_t)a.n_labels) {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(&S.rot_base[k * kLeanThreads + tid])),
                         "l"(a.vs_base + l)
                         : "memory");
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(&S.rot_prev[k * kLeanThreads + tid])),
                         "l"(a.vs_prev + l)
                         : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    __syncthreads();

    // this lane's targets: offset from the tile's first site, window cell
    int rel[PER_LANE], cell[PER_LANE];
#pragma unroll
    for (int k = 0; k < PER_LANE; ++k) {
        int lx, ly, lz;
        target_of<DIM>(warp * Smem::TPW + k * 32 + lane, a.colour, lx, ly, lz);
        rel[k] = (lz * H + ly) * W + lx;
        cell[k] = ((lz + T::HZ) * T::PY + (ly + 1)) * T::PX + (lx + T::HX);
    }
    uint32_t *queue = S.queue[warp];
    const unsigned below = (1u << lane) - 1u;
    uint32_t patch_parity = 0;  // bit k: parity of the next phase of patched[k]
    // entries held over from the previous tile: queue[0, held), its buffer and origin
    int held = 0, held_slot = -1, hx0 = 0, hy0 = 0, hz0 = 0;
    // The CTA's tiles are blockIdx.x + i gridDim.x; their tile coordinates
    // advance by the grid's own decomposition, so the loop divides nothing.
    const int tiles_x = (W + T::TX - 1) / T::TX, tiles_y = (H + T::TY - 1) / T::TY;
    const int step_x = (int)gridDim.x % tiles_x, step_y = ((int)gridDim.x / tiles_x) % tiles_y;
    const int step_z = (int)gridDim.x / (tiles_x * tiles_y);
    int tx = (int)blockIdx.x % tiles_x, ty = ((int)blockIdx.x / tiles_x) % tiles_y;
    int tz = (int)blockIdx.x / (tiles_x * tiles_y);

    for (int i = 0; i < mine; ++i) {
        const int slot = i % kLeanStages;
        if (i > 0) {
            tx += step_x;
            const int cx = tx >= tiles_x;
            tx -= cx ? tiles_x : 0;
            ty += step_y + cx;
            const int cy = ty >= tiles_y;
            ty -= cy ? tiles_y : 0;
            tz += step_z + cy;
        }
        const int x0 = tx * T::TX, y0 = ty * T::TY, z0 = DIM == 3 ? tz * T::TZ : 0;
        uint32_t *win = S.win[slot];
        bool ok = wait_parity(&S.full[slot], (uint32_t)(i / kLeanStages) & 1u) != 0;
        const bool edge = !copies || !(x0 >= T::HX && x0 + T::TX + T::HX <= W && y0 >= 1 && y0 + T::TY + 1 <= H &&
                                       (DIM == 2 || (z0 >= 1 && z0 + T::TZ + 1 <= D)));
        if (edge && __all_sync(0xffffffffu, ok)) {
            lean_patch<DIM>(a, win, x0, y0, z0, copies);
            // generic writes to a buffer a later tensor copy will overwrite
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&S.patched[slot])) : "memory");
            ok = wait_parity(&S.patched[slot], (patch_parity >> slot) & 1u) != 0;
            patch_parity ^= 1u << slot;
        }
        if (!__all_sync(0xffffffffu, ok)) {
            // A copy or a warp that never came: flag it, give each buffer's
            // latest copy its own bounded wait so none lands after exit, stop.
            if (lane == 0) {
                atomicExch(a.error_flag, 1);
                for (int k = 0; k < kLeanStages; ++k)
                    if (S.issued[k] > 0) wait_parity(&S.full[k], (uint32_t)(S.issued[k] - 1) & 1u);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            return;
        }

        // Light pass: this warp's targets; those whose neighbour pick carries
        // another label go into the warp's queue, behind the entries held
        // from the previous tile.
        const bool full = x0 + T::TX <= W && y0 + T::TY <= H && (DIM == 2 || z0 + T::TZ <= D);
        const uint32_t tile_base = (uint32_t)((z0 * H + y0) * W + x0);
        uint32_t entries[PER_LANE];
        unsigned masks[PER_LANE];
#pragma unroll
        for (int k = 0; k < PER_LANE; ++k) {
            const int j = warp * Smem::TPW + k * 32 + lane;
            bool in = full;
            if (!full) {
                int lx, ly, lz;
                target_of<DIM>(j, a.colour, lx, ly, lz);
                in = x0 + lx < W && y0 + ly < H && (DIM == 2 || z0 + lz < D);
            }
            bool active = false;
            int pick = 0;
            if (in) {
                pick = pick_of<NOFF>(draw(a.key_pick, tile_base + (uint32_t)rel[k]));
                active = win[cell[k]] != win[cell[k] + S.woff[pick]];
            }
            entries[k] = (uint32_t)j | ((uint32_t)pick << 16);
            masks[k] = __ballot_sync(0xffffffffu, active);
        }
        int total = held;
#pragma unroll
        for (int k = 0; k < PER_LANE; ++k) {
            if (masks[k] & (1u << lane)) queue[total + __popc(masks[k] & below)] = entries[k];
            total += __popc(masks[k]);
        }
        __syncwarp();
        // Heavy pass: whole rounds of 32 copies, oldest first; entry e is the
        // previous tile's when e < held. Whatever of the previous tile is still
        // queued after them goes in one last short round, so that tile's
        // buffer can be let go; fewer than 32 of this tile's stay held.
        int taken = 0;
        for (;;) {
            const int n = total - taken;
            if (n < 32 && taken >= held) break;
            const int e = taken + lane;
            if (e < total) {
                const bool before = e < held;
                price_and_commit<DIM, NOFF, UNIFORM, false>(a, S.woff, S.contact, nullptr,
                                                            before ? S.win[held_slot] : win, queue[e],
                                                            before ? hx0 : x0, before ? hy0 : y0,
                                                            before ? hz0 : z0, small_types);
            }
            taken += n < 32 ? n : 32;
        }
        __syncwarp();
        if (held_slot >= 0) lean_release<DIM>(a, tmap, S, i - 1, mine, copies);
        // move what this tile keeps to the front of the queue (a full round
        // came first, so the source lies past the first 32 entries)
        const int keep = total - taken;
        if (taken > 0 && keep > 0) {
            const uint32_t v = lane < keep ? queue[taken + lane] : 0u;
            __syncwarp();
            if (lane < keep) queue[lane] = v;
            __syncwarp();
        }
        held = keep;
        held_slot = slot;
        hx0 = x0;
        hy0 = y0;
        hz0 = z0;
    }
    // the last tile's held entries, then its buffer
    if (mine > 0) {
        if (lane < held)
            price_and_commit<DIM, NOFF, UNIFORM, false>(a, S.woff, S.contact, nullptr, S.win[held_slot], queue[lane],
                                                        hx0, hy0, hz0, small_types);
        __syncwarp();
        lean_release<DIM>(a, tmap, S, mine - 1, mine, copies);
    }
    // finish the rotation: this thread's copied labels, then any past them
    asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
    for (int k = 0; k < kRotate; ++k) {
        const size_t l = rot_first + k * rot_stride;
        if (l < (size_t)a.n_labels) {
            int dv, ds;
            unpack_delta(S.rot_prev[k * kLeanThreads + tid], dv, ds);
            const int2 b = S.rot_base[k * kLeanThreads + tid];
            a.vs_next_base[l] = make_int2(b.x + dv, b.y + ds);
            a.vs_clear[l] = 0;
        }
    }
    for (size_t l = rot_first + kRotate * rot_stride; l < (size_t)a.n_labels; l += rot_stride) {
        int dv, ds;
        unpack_delta(a.vs_prev[l], dv, ds);
        const int2 b = a.vs_base[l];
        a.vs_next_base[l] = make_int2(b.x + dv, b.y + ds);
        a.vs_clear[l] = 0;
    }
}

// ---------------------------------------------------------------- the direct sweep
//
// Small lattices of the lean models take a kernel with no staging at all:
// one thread per target, the labels read where they lie (a target's
// neighbours are other colours, which no copy in the pass changes), priced
// with price_and_commit's arithmetic operation for operation. The lean
// kernel's window ring, patches and queues cost more latency than they save
// when a pass is a few tiles.
// The per-pass view of the tallies and draws a direct pass reads.
struct PassView {
    int colour;
    uint64_t key_pick, key_accept;
    const int2 *vs_base;
    const long long *vs_prev;
    unsigned long long *vs_cur;
};

// The per-colour guard of keeps_other_colour, for a direct pass.
__device__ __noinline__ bool direct_keeps_other_colour(const SweepLaunch &a, int colour, uint32_t old) {
    int other = 0;
    for (int c = 0; c < a.g.ncol; ++c)
        if (c != colour) other += a.vol_by_colour[(size_t)old * a.g.ncol + c];
    return other != 0;
}

// Where a direct pass finds and puts labels and tallies: global memory.
struct GlobalPass {
    const SweepLaunch &a;
    const PassView &v;
    __device__ __forceinline__ uint32_t label(int x, int y, int z) const {
        return a.labels[(z * a.g.h + y) * a.g.w + x];
    }
    __device__ __forceinline__ int2 base(uint32_t l) const { return v.vs_base[l]; }
    __device__ __forceinline__ long long prev(uint32_t l) const { return v.vs_prev[l]; }
    __device__ __forceinline__ bool keeps_other_colour(uint32_t old) const {
        return direct_keeps_other_colour(a, v.colour, old);
    }
    __device__ __forceinline__ void put(uint32_t target, int, int, int, uint32_t nw) const { a.labels[target] = nw; }
    __device__ __forceinline__ void tally(uint32_t l, int dv, int ds) const {
        atomicAdd(&v.vs_cur[l], pack_delta(dv, ds));
        atomicAdd(&a.vol_by_colour[(size_t)l * a.g.ncol + v.colour], dv);
    }
};

// Site (x, y, z) of target j of colour `colour` in a direct pass.
template <int DIM>
__device__ __forceinline__ void direct_site(const SweepLaunch &a, int colour, int j, int &x, int &y, int &z) {
    const uint32_t row = udiv(a.g.div_hw, (uint32_t)j), plane = udiv(a.g.div_hh, row);
    x = 2 * (int)((uint32_t)j - row * (uint32_t)(a.g.w / 2)) + (colour & 1);
    y = 2 * (int)(row - plane * (uint32_t)(a.g.h / 2)) + ((colour >> 1) & 1);
    z = DIM == 3 ? 2 * (int)plane + ((colour >> 2) & 1) : 0;
}

// The connectivity veto (lib.rs:511-521) for a direct pass: the ring
// positions of `old` around target (x, y, z), read where they lie, must be
// one piece.
__device__ __noinline__ bool direct_ring_one_piece(const SweepLaunch &a, int x, int y, int z, uint32_t old) {
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    uint32_t present = 0;
    for (int k = 0; k < a.g.ring_n; ++k) {
        const int nx = wrap(x + a.g.ring[k][0], W), ny = wrap(y + a.g.ring[k][1], H), nz = wrap(z + a.g.ring[k][2], D);
        if (a.labels[((size_t)nz * H + ny) * W + nx] == old) present |= 1u << k;
    }
    return one_piece(present, a.g.adjacency);
}

// The offset of neighbour `pick`, chosen among compile-time constants (the
// 26-neighbourhood has a closed form) rather than read from a table.
template <int DIM, int NOFF>
__device__ __forceinline__ void pick_offset(int pick, int &dx, int &dy, int &dz) {
    if constexpr (DIM == 3 && NOFF == 26) {
        dx = neighbour_offset<3, 26>(pick, 0);
        dy = neighbour_offset<3, 26>(pick, 1);
        dz = neighbour_offset<3, 26>(pick, 2);
    } else {
        dx = dy = dz = 0;
#pragma unroll
        for (int k = 0; k < NOFF; ++k)
            if (k == pick) {
                dx = neighbour_offset<DIM, NOFF>(k, 0);
                dy = neighbour_offset<DIM, NOFF>(k, 1);
                dz = neighbour_offset<DIM, NOFF>(k, 2);
            }
    }
}

// The copy attempt at target (x, y, z) of a direct pass, its labels and
// tallies found through `acc`: a target's neighbours are other colours, which
// no copy in the pass changes. Priced with price_and_commit's arithmetic
// operation for operation.
template <int DIM, int NOFF, bool UNIFORM, class Access, bool EXTRAS = false>
__device__ __forceinline__ void direct_target(const SweepLaunch &a, const Access &acc, uint64_t key_pick,
                                              uint64_t key_accept, int x, int y, int z, int known_pick = -1,
                                              bool known_labels = false, uint32_t known_old = 0,
                                              uint32_t known_new = 0) {
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const int xm = x == 0 ? W - 1 : x - 1, xp = x == W - 1 ? 0 : x + 1;
    const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
    const int zm = z == 0 ? D - 1 : z - 1, zp = z == D - 1 ? 0 : z + 1;
    const auto at = [&](int k) -> uint32_t {
        const int dx = neighbour_offset<DIM, NOFF>(k, 0), dy = neighbour_offset<DIM, NOFF>(k, 1),
                  dz = neighbour_offset<DIM, NOFF>(k, 2);
        const int nx = dx < 0 ? xm : (dx > 0 ? xp : x), ny = dy < 0 ? ym : (dy > 0 ? yp : y),
                  nz = dz < 0 ? zm : (dz > 0 ? zp : z);
        return acc.label(nx, ny, nz);
    };
    const uint32_t target = (uint32_t)((z * H + y) * W + x);
    const int pick = known_pick >= 0 ? known_pick : pick_of<NOFF>(draw(key_pick, target));
    int dx, dy, dz;
    pick_offset<DIM, NOFF>(pick, dx, dy, dz);
    // A caller that read the two labels earlier in the pass passes them: the
    // target's changes only by its own commit and the neighbour is another
    // colour, so they are still the pass's.
    const uint32_t nw = known_labels ? known_new
                                     : acc.label(dx < 0 ? xm : (dx > 0 ? xp : x), dy < 0 ? ym : (dy > 0 ? yp : y),
                                                 dz < 0 ? zm : (dz > 0 ? zp : z));
    const uint32_t old = known_labels ? known_old : acc.label(x, y, z);
    if (old == nw) return;
    const int2 base_old = acc.base(old), base_new = acc.base(nw);
    const long long prev_old = acc.prev(old), prev_new = acc.prev(nw);
    const int t_old = UNIFORM ? a.uniform_type : a.cell_type[old];
    const int t_new = UNIFORM ? a.uniform_type : a.cell_type[nw];
    float delta = 0.0f;
    int like_old = 0, like_new = 0;
    if (UNIFORM) {
#pragma unroll
        for (int k = 0; k < NOFF; ++k) {
            const uint32_t ln = at(k);
            like_old += ln == old;
            like_new += ln == nw;
        }
        delta = __fmul_rn(a.uniform_contact, (float)(like_old - like_new));
    } else {
#pragma unroll
        for (int k = 0; k < NOFF; ++k) {
            const uint32_t ln = at(k);
            const int tn = ln == old ? t_old : (ln == nw ? t_new : (int)a.cell_type[ln]);
            if (ln != old)
                delta = __fsub_rn(delta, a.t.contact[t_old * a.n_types + tn]);
            else
                ++like_old;
            if (ln != nw)
                delta = __fadd_rn(delta, a.t.contact[t_new * a.n_types + tn]);
            else
                ++like_new;
        }
    }
    if (old != 0 && like_old == 0 && !acc.keeps_other_colour(old)) return;
    if (EXTRAS && old != 0 && a.g.ring_n > 0 && a.t.connected[t_old] && !direct_ring_one_piece(a, x, y, z, old))
        return;
    const int ds_old = 2 * like_old - NOFF;
    const int ds_new = NOFF - 2 * like_new;
    int dv, ds;
    unpack_delta(prev_old, dv, ds);
    const int vol_old = base_old.x + dv, surf_old = base_old.y + ds;
    unpack_delta(prev_new, dv, ds);
    const int vol_new = base_new.x + dv, surf_new = base_new.y + ds;
    delta = size_terms<UNIFORM>(a, old, nw, t_old, t_new, vol_old, vol_new, surf_old, surf_new, ds_old, ds_new, delta);
    if (EXTRAS && (a.has_length || a.has_chemotaxis || a.has_external || a.has_motility || a.has_nematic))
        delta = extra_terms<DIM>(a, old, nw, t_old, t_new, vol_old, vol_new, x, y, z, pick, target, delta);
    const float u = to_f32(draw(key_accept, target));
    if (!(delta <= 0.0f || u < metropolis_exp(__fmul_rn(-delta, a.beta)))) return;
    if (EXTRAS && a.has_motility) {
        const int k = atomicAdd(a.pending_count, 1);
        a.pending[k] = make_uint2(target, nw);
    } else {
        acc.put(target, x, y, z, nw);
    }
    if (old != 0) acc.tally(old, -1, ds_old);
    if (nw != 0) acc.tally(nw, 1, ds_new);
    if (EXTRAS && a.tracks) commit_moments<DIM>(a, old, nw, x, y, z);
}

// K 0: one target per thread, priced where it lies. K > 0: each warp takes
// 32 K consecutive targets; every lane draws its targets' picks and compares
// the two labels, the targets whose pick carries another label go into the
// warp's queue, and the warp prices the queue in full rounds, so that a
// round's lanes all have a copy to price. The queue pays on large passes
// (0.37 against 0.51 ms per MCS at 256^3 with K 4); below a million targets
// a pass (kDirectCompactFrom, engine.h) the block-queued form below, with its
// wider grid, hides more latency.
constexpr int kDirectCompactK = 4;
// K < 0: the block's 256 |K| consecutive targets are drawn and compared by
// all its threads, the unlike ones gathered into one block-wide queue, and
// the queue priced from its front by as many whole warps as it needs: the
// plain form's wide grid, with a warp's lanes busy in the pricing rounds.
// Two targets a thread (per MCS at 1024^2: 37.3 us with two, 52.0 with one;
// at 128^3, with the register cap below, 0.060 ms with two, 0.062 with one).
template <int DIM>
constexpr int kDirectBlockK = -2;

// Direct passes of the lean models are held to 64 registers, four blocks of
// 256 per SM, so that a 2^18-target pass of two targets a thread is one wave
// (at 128^3: 0.060 ms per MCS against 0.073 uncapped, 0.065 at 48 registers);
// the every-term passes keep their registers (capped, they spill and slow).
template <bool EXTRAS>
constexpr int kDirectMinBlocks = EXTRAS ? 1 : 4;

template <int DIM, int NOFF, bool UNIFORM, int K, bool EXTRAS>
__device__ __forceinline__ void direct_sweep_body(const SweepLaunch &a) {
    const int targets = (a.g.w / 2) * (a.g.h / 2) * (DIM == 3 ? a.g.d / 2 : 1);
    const PassView v{a.colour, a.key_pick, a.key_accept, a.vs_base, a.vs_prev, a.vs_cur};
    const GlobalPass acc{a, v};
    if constexpr (K == 0) {
        const int j = blockIdx.x * blockDim.x + threadIdx.x;
        if (j < targets) {
            int x, y, z;
            direct_site<DIM>(a, a.colour, j, x, y, z);
            direct_target<DIM, NOFF, UNIFORM, GlobalPass, EXTRAS>(a, acc, v.key_pick, v.key_accept, x, y, z);
        }
    } else if constexpr (K < 0) {
        constexpr int KB = -K;
        __shared__ int queue[256 * KB];
        __shared__ uint8_t picks[256 * KB];
        __shared__ uint2 pair[256 * KB];  // (old, new) labels of each queued copy, as the light step read them
        __shared__ int counts[8];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const unsigned below = (1u << lane) - 1u;
        // The block's targets [first, last): direct_span of them (at most 256 KB)
        // when the launch spreads the pass evenly over the SMs' resident
        // blocks, else 256 KB.
        const int span = a.direct_span > 0 ? a.direct_span : 256 * KB;
        const int first = (int)blockIdx.x * span;
        const int last = min(first + span, targets);
        unsigned masks[KB];
        int picked[KB];
        uint2 labels[KB];
        int mine = 0;
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            const int j = first + k * 256 + (int)threadIdx.x;
            bool unlike = false;
            int pick = 0;
            labels[k] = make_uint2(0u, 0u);
            if (j < last) {
                int x, y, z;
                direct_site<DIM>(a, a.colour, j, x, y, z);
                pick = pick_of<NOFF>(draw(v.key_pick, (uint32_t)((z * a.g.h + y) * a.g.w + x)));
                int dx, dy, dz;
                pick_offset<DIM, NOFF>(pick, dx, dy, dz);
                const int nx = x + dx < 0 ? a.g.w - 1 : (x + dx >= a.g.w ? 0 : x + dx);
                const int ny = y + dy < 0 ? a.g.h - 1 : (y + dy >= a.g.h ? 0 : y + dy);
                const int nz = z + dz < 0 ? a.g.d - 1 : (z + dz >= a.g.d ? 0 : z + dz);
                labels[k] = make_uint2(acc.label(x, y, z), acc.label(nx, ny, nz));
                unlike = labels[k].x != labels[k].y;
            }
            masks[k] = __ballot_sync(0xffffffffu, unlike);
            picked[k] = pick;
            mine += __popc(masks[k]);
        }
        if (lane == 0) counts[warp] = mine;
        __syncthreads();
        int at = 0, total = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            at += w < warp ? counts[w] : 0;
            total += counts[w];
        }
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            if (masks[k] & (1u << lane)) {
                queue[at + __popc(masks[k] & below)] = first + k * 256 + (int)threadIdx.x;
                picks[at + __popc(masks[k] & below)] = (uint8_t)picked[k];
                pair[at + __popc(masks[k] & below)] = labels[k];
            }
            at += __popc(masks[k]);
        }
        __syncthreads();
        for (int e = (int)threadIdx.x; e < total; e += 256) {
            int x, y, z;
            direct_site<DIM>(a, a.colour, queue[e], x, y, z);
            const uint2 ln = pair[e];
            direct_target<DIM, NOFF, UNIFORM, GlobalPass, EXTRAS>(a, acc, v.key_pick, v.key_accept, x, y, z, picks[e],
                                                                  true, ln.x, ln.y);
        }
    } else {
        __shared__ int queue[8][32 * K];
        __shared__ uint8_t picks[8][32 * K];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const unsigned below = (1u << lane) - 1u;
        const int first = (blockIdx.x * 8 + warp) * 32 * K;
        int total = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int j = first + k * 32 + lane;
            bool unlike = false;
            int pick = 0;
            if (j < targets) {
                int x, y, z;
                direct_site<DIM>(a, a.colour, j, x, y, z);
                pick = pick_of<NOFF>(draw(v.key_pick, (uint32_t)((z * a.g.h + y) * a.g.w + x)));
                int dx, dy, dz;
                pick_offset<DIM, NOFF>(pick, dx, dy, dz);
                const int nx = x + dx < 0 ? a.g.w - 1 : (x + dx >= a.g.w ? 0 : x + dx);
                const int ny = y + dy < 0 ? a.g.h - 1 : (y + dy >= a.g.h ? 0 : y + dy);
                const int nz = z + dz < 0 ? a.g.d - 1 : (z + dz >= a.g.d ? 0 : z + dz);
                unlike = acc.label(x, y, z) != acc.label(nx, ny, nz);
            }
            const unsigned m = __ballot_sync(0xffffffffu, unlike);
            if (unlike) {
                queue[warp][total + __popc(m & below)] = j;
                picks[warp][total + __popc(m & below)] = (uint8_t)pick;
            }
            total += __popc(m);
        }
        __syncwarp();
        for (int e = lane; e < total; e += 32) {
            int x, y, z;
            direct_site<DIM>(a, a.colour, queue[warp][e], x, y, z);
            direct_target<DIM, NOFF, UNIFORM, GlobalPass, EXTRAS>(a, acc, v.key_pick, v.key_accept, x, y, z,
                                                                  picks[warp][e]);
        }
    }
    rotate_tallies<DIM>(a);
}

template <int DIM, int NOFF, bool UNIFORM, int K, bool EXTRAS>
__global__ void __launch_bounds__(256, kDirectMinBlocks<EXTRAS>) direct_sweep_kernel(const __grid_constant__ SweepLaunch a) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    direct_sweep_body<DIM, NOFF, UNIFORM, K, EXTRAS>(a);
}

// A clocked launch's pass fields from the engine clock, as pass_launch
// (engine.cu) sets them on the host: the step and its draws, the tally slots
// of the pass's number, each species' current field buffer.
__device__ __forceinline__ void clock_patch(SweepLaunch &d) {
    const EngineClock c = *d.clock;
    const long long p = c.pass + d.colour;
    d.step = (int32_t)c.step;
    d.key_pick = stream_key(d.seed, d.step, d.colour, 0);
    d.key_accept = stream_key(d.seed, d.step, d.colour, 1);
    d.vs_base = d.tal.vs_base[p % 2];
    d.vs_prev = d.tal.vs_delta[(p + 2) % 3];
    d.vs_cur = reinterpret_cast<unsigned long long *>(d.tal.vs_delta[p % 3]);
    d.vs_next_base = d.tal.vs_base[(p + 1) % 2];
    d.vs_clear = d.tal.vs_delta[(p + 1) % 3];
    d.mom_base = d.tal.mom_base[p % 2];
    d.mom_prev = d.tal.mom_delta[(p + 2) % 3];
    d.mom_cur = reinterpret_cast<unsigned long long *>(d.tal.mom_delta[p % 3]);
    d.mom_next_base = d.tal.mom_base[(p + 1) % 2];
    d.mom_clear = d.tal.mom_delta[(p + 1) % 3];
    for (int s = 0; s < d.n_species; ++s)
        d.fields[s] = d.field_buf + ((size_t)2 * s + ((c.field_cur >> s) & 1u)) * (size_t)d.g.sites;
}

// The direct pass of a step replayed from a graph: the block copies the
// launch into shared memory, patches it from the clock and prices from there.
template <int DIM, int NOFF, bool UNIFORM, int K, bool EXTRAS>
__global__ void __launch_bounds__(256, kDirectMinBlocks<EXTRAS>) direct_sweep_clocked(const __grid_constant__ SweepLaunch a) {
    __shared__ SweepLaunch d;
    static_assert(sizeof(SweepLaunch) % sizeof(int) == 0, "the launch copies as words");
    const int *src = reinterpret_cast<const int *>(&a);
    int *dst = reinterpret_cast<int *>(&d);
    for (int i = threadIdx.x; i < (int)(sizeof(SweepLaunch) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) clock_patch(d);
    __syncthreads();
    direct_sweep_body<DIM, NOFF, UNIFORM, K, EXTRAS>(d);
}

// ---------------------------------------------------------------- the resident sweep
//
// A small lean model with nothing between its colour passes but the passes
// (no fields, division, death or infection) runs every requested MCS in one
// cooperative launch: the direct pass's work per target, the tally rotation,
// then a grid barrier, pass after pass. Each pass's draws and tally slots
// follow from its number as the host would set them. Reads of what other
// blocks wrote in earlier passes are plain loads: the barrier's gpu-scope
// release (each block's fence and arrival) and acquire (the waiting thread's
// acquire load and fence, then the block barrier) order them after those
// writes, whatever an SM's L1 held before. The barrier's wait is bounded: a
// block that gives up sets error flag 4 and returns, and the others then
// give up at their next barrier.

// polls of the barrier word (each an L2 round trip, so the limit is seconds)
constexpr long long kBarrierLimit = 1LL << 22;

// Barrier number k of the launch (k = 0, 1, ...): false if it timed out.
__device__ __forceinline__ bool resident_barrier(unsigned *bar, unsigned k) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        if (atomicAdd(&bar[0], 1u) + 1u == gridDim.x * (k + 1u)) {
            __threadfence();
            atomicExch(&bar[1], k + 1u);
        } else {
            long long spin = 0;
            for (;;) {
                unsigned g;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(&bar[1]) : "memory");
                if (g >= k + 1u || ++spin > kBarrierLimit) {
                    ok = g >= k + 1u;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

template <int DIM, int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(256) resident_sweep_kernel(const __grid_constant__ ResidentLaunch r) {
    const SweepLaunch &a = r.a;
    const int targets = (a.g.w / 2) * (a.g.h / 2) * (DIM == 3 ? a.g.d / 2 : 1);
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    unsigned k = 0;
    for (int m = 0; m < r.mcs; ++m) {
        const int32_t step = (int32_t)((uint32_t)r.step0 + (uint32_t)m);
        for (int c = 0; c < a.g.ncol; ++c) {
            const long long p = r.pass0 + (long long)m * a.g.ncol + c;
            const PassView v{c, stream_key(r.seed, step, c, 0), stream_key(r.seed, step, c, 1), r.vs_base[p % 2],
                             r.vs_delta[(p + 2) % 3], reinterpret_cast<unsigned long long *>(r.vs_delta[p % 3])};
            if (j < targets) {
                int x, y, z;
                direct_site<DIM>(a, c, j, x, y, z);
                direct_target<DIM, NOFF, UNIFORM>(a, GlobalPass{a, v}, v.key_pick, v.key_accept, x, y, z);
            }
            // the rotation for the next pass, which no thread of this one reads
            int2 *next_base = r.vs_base[(p + 1) % 2];
            long long *clear = r.vs_delta[(p + 1) % 3];
            for (size_t l = j; l < (size_t)a.n_labels; l += stride) {
                int dv, ds;
                unpack_delta(v.vs_prev[l], dv, ds);
                const int2 b = v.vs_base[l];
                next_base[l] = make_int2(b.x + dv, b.y + ds);
                clear[l] = 0;
            }
            if (!resident_barrier(r.barrier, k++)) {
                if (threadIdx.x == 0) atomicExch(a.error_flag, 4);
                return;
            }
        }
    }
}

// Run `mcs` MCS of a small lean model in one cooperative launch, or return
// cudaErrorCooperativeLaunchTooLarge (nothing launched) when its blocks
// cannot all be resident.
template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t launch_resident(const ResidentLaunch &r, cudaStream_t stream) {
    const int targets = (r.a.g.w / 2) * (r.a.g.h / 2) * (DIM == 3 ? r.a.g.d / 2 : 1);
    const int blocks = (targets + 255) / 256;
    static std::atomic<int> most_once{0};  // handles on other host threads may launch too
    if (!most_once.load(std::memory_order_acquire)) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaError_t e = cudaGetDevice(&dev)) return e;
        if (cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return e;
        if (cudaError_t e =
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resident_sweep_kernel<DIM, NOFF, UNIFORM>, 256, 0))
            return e;
        most_once.store(sms * per_sm, std::memory_order_release);
    }
    const int most = most_once.load(std::memory_order_acquire);
    if (blocks > most) return cudaErrorCooperativeLaunchTooLarge;
    void *args[] = {const_cast<ResidentLaunch *>(&r)};
    return cudaLaunchCooperativeKernel((const void *)resident_sweep_kernel<DIM, NOFF, UNIFORM>, dim3(blocks), dim3(256),
                                       args, 0, stream);
}

template <bool UNIFORM>
static cudaError_t resident_any(const ResidentLaunch &r, cudaStream_t stream) {
    if (r.a.g.dim == 2) {
        if (r.a.g.n_off == 4) return launch_resident<2, 4, UNIFORM>(r, stream);
        if (r.a.g.n_off == 8) return launch_resident<2, 8, UNIFORM>(r, stream);
    } else {
        if (r.a.g.n_off == 6) return launch_resident<3, 6, UNIFORM>(r, stream);
        if (r.a.g.n_off == 18) return launch_resident<3, 18, UNIFORM>(r, stream);
        if (r.a.g.n_off == 26) return launch_resident<3, 26, UNIFORM>(r, stream);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_resident_sweep(const ResidentLaunch &r, cudaStream_t stream) {
    for (int k = 0; k < r.a.g.n_off; ++k)
        for (int axis = 0; axis < 3; ++axis) {
            const int want = r.a.g.dim == 2 ? (r.a.g.n_off == 4 ? neighbour_offset<2, 4>(k, axis)
                                                                 : neighbour_offset<2, 8>(k, axis))
                                            : (r.a.g.n_off == 6    ? neighbour_offset<3, 6>(k, axis)
                                               : r.a.g.n_off == 18 ? neighbour_offset<3, 18>(k, axis)
                                                                   : neighbour_offset<3, 26>(k, axis));
            if (r.a.g.off[k][axis] != want) return cudaErrorInvalidValue;
        }
    return r.a.uniform_type >= 0 && r.a.uniform_contact_exact ? resident_any<true>(r, stream)
                                                              : resident_any<false>(r, stream);
}

// ---------------------------------------------------------------- the cluster sweep
//
// A small plane of a model the resident sweep takes runs every MCS of a call
// in ONE thread-block cluster: the lattice split by rows over the cluster's
// CTAs and held in their shared memory, the tallies dealt by label (label l
// in CTA l mod C), every read or atomic on another CTA's part through
// distributed shared memory, and the cluster's hardware barrier between
// passes. The copies, draws and tally rotation are the resident sweep's;
// the lattice and tallies go back to global memory at the end.

constexpr int kClusterThreads = 1024;
#ifndef GLZ_CLUSTER_MAX
#define GLZ_CLUSTER_MAX 16
#endif
constexpr int kClusterMax = GLZ_CLUSTER_MAX;  // CTAs of a cluster at most (16 is the non-portable limit)
// A plane takes a cluster of at least kClusterMin CTAs (fewer only when it
// has fewer rows), more while a CTA would hold more targets than threads:
// a pass's work per CTA is what bounds it, so spreading a 128^2 plane over
// 8 SMs rather than 4 cuts its 100 MCS from 1.17 to 0.99 ms.
#ifndef GLZ_CLUSTER_MIN
#define GLZ_CLUSTER_MIN 8
#endif
constexpr int kClusterMin = GLZ_CLUSTER_MIN;  // a power of two
constexpr int kClusterSmem = 200 * 1024;
#ifndef GLZ_CLUSTER_PER_THREAD
#define GLZ_CLUSTER_PER_THREAD 1
#endif
constexpr int kClusterPerThread = GLZ_CLUSTER_PER_THREAD;  // a pass's targets a thread draws at most

// Shared-memory layout of one CTA of a C-CTA cluster sweep (bytes from the
// start): delta[3][Lc] (i64), base[2][Lc] (int2), the pointer tables
// (delta 3C, base 2C, volc C), rows[H], slab[R W] (u32), volc[Lc][4] (i32),
// the pass's queue of unlike copies (target index, pick) with room for every
// target of the CTA's rows, and the queue's two fill counters.
struct ClusterLayout {
    int C, R, Lc, qcap;
    size_t delta, base, dptr, bptr, vptr, rows, slab, volc, queue, picks, qn, bytes;
    __host__ __device__ ClusterLayout(int w, int h, int n_labels, int c) : C(c) {
        R = (h + c - 1) / c;
        Lc = (n_labels + c - 1) / c;
        qcap = (R + 1) / 2 * (w / 2);
        delta = 0;
        base = delta + 3 * (size_t)Lc * 8;
        dptr = base + 2 * (size_t)Lc * 8;
        bptr = dptr + 3 * (size_t)c * 8;
        vptr = bptr + 2 * (size_t)c * 8;
        rows = vptr + (size_t)c * 8;
        slab = rows + (size_t)h * 8;
        volc = slab + ((size_t)R * w * 4 + 15) / 16 * 16;
        queue = volc + (size_t)Lc * 16;
        picks = queue + (size_t)qcap * 4;
        qn = picks + ((size_t)qcap + 15) / 16 * 16;
        bytes = qn + 16;
    }
};

// Labels and tallies of a cluster pass: `rows[y]` is row y in whichever CTA
// holds it; a label's tallies sit in CTA l & mask at index l >> shift.
struct ClusterPass {
    uint32_t *const *rows;
    int2 *const *bptr;         // [slot * C + rank]
    long long *const *dptr;    // [slot * C + rank]
    int *const *vptr;          // [rank]
    int C, shift, mask, colour, bslot, pslot, cslot;
    __device__ __forceinline__ uint32_t label(int x, int y, int) const { return rows[y][x]; }
    __device__ __forceinline__ int2 base(uint32_t l) const { return bptr[bslot * C + (l & mask)][l >> shift]; }
    __device__ __forceinline__ long long prev(uint32_t l) const { return dptr[pslot * C + (l & mask)][l >> shift]; }
    __device__ __forceinline__ bool keeps_other_colour(uint32_t old) const {
        const int *v = vptr[old & mask] + (size_t)(old >> shift) * 4;
        int other = 0;
        for (int c = 0; c < 4; ++c)
            if (c != colour) other += v[c];
        return other != 0;
    }
    __device__ __forceinline__ void put(uint32_t, int x, int y, int, uint32_t nw) const { rows[y][x] = nw; }
    __device__ __forceinline__ void tally(uint32_t l, int dv, int ds) const {
        atomicAdd(reinterpret_cast<unsigned long long *>(&dptr[cslot * C + (l & mask)][l >> shift]),
                  pack_delta(dv, ds));
        atomicAdd(&vptr[l & mask][(size_t)(l >> shift) * 4 + colour], dv);
    }
};

template <int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kClusterThreads, 1) cluster_sweep_kernel(const __grid_constant__ ResidentLaunch r) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const SweepLaunch &a = r.a;
    const int C = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
    const int W = a.g.w, H = a.g.h, n_labels = a.n_labels;
    const ClusterLayout L(W, H, n_labels, C);
    const int tid = threadIdx.x, nth = blockDim.x;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    long long *delta = reinterpret_cast<long long *>(smem_raw + L.delta);
    int2 *base = reinterpret_cast<int2 *>(smem_raw + L.base);
    long long **dptr = reinterpret_cast<long long **>(smem_raw + L.dptr);
    int2 **bptr = reinterpret_cast<int2 **>(smem_raw + L.bptr);
    int **vptr = reinterpret_cast<int **>(smem_raw + L.vptr);
    uint32_t **rows = reinterpret_cast<uint32_t **>(smem_raw + L.rows);
    uint32_t *slab = reinterpret_cast<uint32_t *>(smem_raw + L.slab);
    int *volc = reinterpret_cast<int *>(smem_raw + L.volc);
    int *queue = reinterpret_cast<int *>(smem_raw + L.queue);
    uint8_t *picks = reinterpret_cast<uint8_t *>(smem_raw + L.picks);
    int *qn = reinterpret_cast<int *>(smem_raw + L.qn);
    const int y0 = rank * L.R, y1 = min(H, y0 + L.R);
    const int lane = tid & 31;
    if (tid < 2) qn[tid] = 0;

    // this CTA's rows and labels, and where every CTA's parts lie
    for (int i = tid; i < (y1 - y0) * W; i += nth) slab[i] = a.labels[(size_t)y0 * W + i];
    for (int i = tid; i < L.Lc; i += nth) {
        const int l = i * C + rank;
        const bool in = l < n_labels;
        for (int k = 0; k < 2; ++k) base[k * L.Lc + i] = in ? r.vs_base[k][l] : make_int2(0, 0);
        for (int k = 0; k < 3; ++k) delta[k * L.Lc + i] = in ? r.vs_delta[k][l] : 0;
        for (int c = 0; c < 4; ++c) volc[i * 4 + c] = in ? a.vol_by_colour[(size_t)l * 4 + c] : 0;
    }
    for (int y = tid; y < H; y += nth) {
        const int o = y / L.R;
        rows[y] = cluster.map_shared_rank(slab, o) + (size_t)(y - o * L.R) * W;
    }
    for (int i = tid; i < C; i += nth) {
        for (int k = 0; k < 3; ++k) dptr[k * C + i] = cluster.map_shared_rank(delta + k * L.Lc, i);
        for (int k = 0; k < 2; ++k) bptr[k * C + i] = cluster.map_shared_rank(base + k * L.Lc, i);
        vptr[i] = cluster.map_shared_rank(volc, i);
    }
    cluster.sync();  // every CTA's part in place before any is read

    const int hw = W / 2;
    for (int m = 0; m < r.mcs; ++m) {
        const int32_t step = (int32_t)((uint32_t)r.step0 + (uint32_t)m);
        for (int c = 0; c < 4; ++c) {
            const long long p = r.pass0 + (long long)m * 4 + c;
            const ClusterPass acc{rows, bptr, dptr, vptr, C, __ffs(C) - 1, C - 1, c,
                                  (int)(p % 2), (int)((p + 2) % 3), (int)(p % 3)};
            const uint64_t key_pick = stream_key(r.seed, step, c, 0), key_accept = stream_key(r.seed, step, c, 1);
            // this CTA's targets of colour c: rows of its slab of the colour's
            // parity. Every thread draws its targets' picks and compares the
            // two labels; the unlike ones go into the CTA's queue (a warp's
            // slots reserved at once), which whole warps then price from its
            // front. A pass's copies read only its snapshot and other
            // colours' labels and commit by atomics, so the queue's order
            // changes nothing.
            const int yf = y0 + ((y0 & 1) != ((c >> 1) & 1));
            const int count = yf < y1 ? (y1 - yf + 1) / 2 * hw : 0;
            int *fill = qn + (p & 1);
            for (int t0 = 0; t0 < count; t0 += nth) {
                const int t = t0 + tid;
                bool unlike = false;
                int pick = 0;
                if (t < count) {
                    const int y = yf + 2 * (t / hw), x = 2 * (t % hw) + (c & 1);
                    pick = pick_of<NOFF>(draw(key_pick, (uint32_t)(y * W + x)));
                    int dx, dy, dz;
                    pick_offset<2, NOFF>(pick, dx, dy, dz);
                    const int nx = x + dx < 0 ? W - 1 : (x + dx >= W ? 0 : x + dx);
                    const int ny = y + dy < 0 ? H - 1 : (y + dy >= H ? 0 : y + dy);
                    unlike = acc.label(x, y, 0) != acc.label(nx, ny, 0);
                }
                const unsigned m = __ballot_sync(0xffffffffu, unlike);
                int slot = 0;
                if (lane == 0 && m) slot = atomicAdd(fill, __popc(m));
                slot = __shfl_sync(0xffffffffu, slot, 0) + __popc(m & ((1u << lane) - 1u));
                if (unlike) {
                    queue[slot] = t;
                    picks[slot] = (uint8_t)pick;
                }
            }
            __syncthreads();
            const int total = *fill;
            if (tid == 0) qn[(p + 1) & 1] = 0;  // the next pass's counter; no thread reads it before the cluster barrier
            for (int e = tid; e < total; e += nth) {
                const int t = queue[e];
                const int y = yf + 2 * (t / hw), x = 2 * (t % hw) + (c & 1);
                direct_target<2, NOFF, UNIFORM>(a, acc, key_pick, key_accept, x, y, 0, (int)picks[e]);
            }
            // this CTA's labels' rotation for the next pass, which no thread of this one reads
            int2 *next_base = base + ((p + 1) % 2) * L.Lc;
            long long *clear = delta + ((p + 1) % 3) * L.Lc;
            for (int i = tid; i < L.Lc; i += nth) {
                int dv, ds;
                unpack_delta(delta[acc.pslot * L.Lc + i], dv, ds);
                const int2 b = base[acc.bslot * L.Lc + i];
                next_base[i] = make_int2(b.x + dv, b.y + ds);
                clear[i] = 0;
            }
            cluster.sync();
        }
    }

    // back to global memory: this CTA's rows and labels
    for (int i = tid; i < (y1 - y0) * W; i += nth) a.labels[(size_t)y0 * W + i] = slab[i];
    for (int i = tid; i < L.Lc; i += nth) {
        const int l = i * C + rank;
        if (l >= n_labels) continue;
        for (int k = 0; k < 2; ++k) r.vs_base[k][l] = base[k * L.Lc + i];
        for (int k = 0; k < 3; ++k) r.vs_delta[k][l] = delta[k * L.Lc + i];
        for (int c = 0; c < 4; ++c) a.vol_by_colour[(size_t)l * 4 + c] = volc[i * 4 + c];
    }
}

// Run `mcs` MCS of a small 2D lean model in one cluster; cudaErrorNotSupported
// (nothing launched) when the plane or its labels do not fit one.
template <int NOFF, bool UNIFORM>
static cudaError_t launch_cluster(const ResidentLaunch &r, cudaStream_t stream) {
    const SweepLaunch &a = r.a;
    const long long targets = (long long)a.g.w * a.g.h / 4;
    int want = kClusterMin;
    while (want < kClusterMax && (long long)want * kClusterThreads < targets) want *= 2;
    // past kClusterPerThread targets a thread the cooperative grid's wider
    // spread is faster
    if ((long long)want * kClusterThreads * kClusterPerThread < targets) return cudaErrorNotSupported;
    auto kernel = cluster_sweep_kernel<NOFF, UNIFORM>;
    static std::atomic<bool> ready{false};  // handles on other host threads may launch too
    if (!ready.load(std::memory_order_acquire)) {
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmem) ||
            cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
        ready.store(true, std::memory_order_release);
    }
    // the widest cluster up to `want` CTAs that the device schedules and whose parts fit
    for (int C = want; C >= 1; C /= 2) {
        if (C > a.g.h) continue;
        const ClusterLayout L(a.g.w, a.g.h, a.n_labels, C);
        if (L.bytes > (size_t)kClusterSmem) break;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = L.bytes;
        cfg.stream = stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            continue;
        }
        return cudaLaunchKernelEx(&cfg, kernel, r);
    }
    return cudaErrorNotSupported;
}

cudaError_t launch_cluster_sweep(const ResidentLaunch &r, cudaStream_t stream) {
    const SweepLaunch &a = r.a;
    if (a.g.dim != 2 || a.g.ncol != 4) return cudaErrorNotSupported;
    for (int k = 0; k < a.g.n_off; ++k)
        for (int axis = 0; axis < 3; ++axis) {
            const int want = a.g.n_off == 4 ? neighbour_offset<2, 4>(k, axis) : neighbour_offset<2, 8>(k, axis);
            if (a.g.off[k][axis] != want) return cudaErrorInvalidValue;
        }
    const bool uniform = a.uniform_type >= 0 && a.uniform_contact_exact;
    if (a.g.n_off == 4) return uniform ? launch_cluster<4, true>(r, stream) : launch_cluster<4, false>(r, stream);
    if (a.g.n_off == 8) return uniform ? launch_cluster<8, true>(r, stream) : launch_cluster<8, false>(r, stream);
    return cudaErrorNotSupported;
}

template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t launch_direct(const SweepLaunch &a, cudaStream_t stream);

// Whether sweeps launch programmatically (GLAZIER_SWEEP_PDL=0: plainly).
static int programmatic_launch() {
    static const int on = [] {
        const char *env = std::getenv("GLAZIER_SWEEP_PDL");
        return env && env[0] == '0' ? 0 : 1;
    }();
    return on;
}

// Blocks of the block-queued direct kernel that the device holds at once by
// its launch bounds (SMs x kDirectMinBlocks blocks of 256 threads; the lean
// form's 64-register cap makes that exactly four per SM); 0 if the SM count
// cannot be read. A device attribute only, so a launch being captured into
// a graph may ask.
static int gathered_slots(bool extras) {
    static std::atomic<int> sms_once{0};  // handles on other host threads may launch too
    int sms = sms_once.load(std::memory_order_acquire);
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) {
            cudaGetLastError();
            return 0;
        }
        sms_once.store(sms, std::memory_order_release);
    }
    return sms * (extras ? kDirectMinBlocks<true> : kDirectMinBlocks<false>);
}

template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t launch_direct(const SweepLaunch &a, cudaStream_t stream) {
    const int targets = (a.g.w / 2) * (a.g.h / 2) * (DIM == 3 ? a.g.d / 2 : 1);
    const bool compact = a.compact == 1, gathered = a.compact == 2;
    const int per_block = 256 * (compact ? kDirectCompactK : (gathered ? -kDirectBlockK<DIM> : 1));
    int grid = (targets + per_block - 1) / per_block;
    SweepLaunch b = a;
    b.direct_span = 0;
    if (gathered) {
        // Spread the pass evenly over whole waves of resident blocks, so that
        // no SM holds more of its targets than another (at 128^3 and 1024^2:
        // 592 blocks of 443 targets instead of 512 of 512 on 148 SMs).
        const int slots = gathered_slots(!a.lean);
        if (slots > 0) {
            const int waves = (grid + slots - 1) / slots;
            const int spread = waves * slots;
            b.direct_span = (targets + spread - 1) / spread;
            grid = (targets + b.direct_span - 1) / b.direct_span;
        }
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(256);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    // a motility pass follows its predecessor's copy list and a memset, not a kernel
    attr[0].val.programmaticStreamSerializationAllowed = programmatic_launch() && !a.has_motility;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (a.clock) {  // a step captured into a graph: plain launches, pass fields from the clock
        cfg.numAttrs = 0;
        if (!a.lean)
            return compact    ? cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, kDirectCompactK, true>, b)
                   : gathered ? cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, kDirectBlockK<DIM>, true>, b)
                              : cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, 0, true>, b);
        return compact    ? cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, kDirectCompactK, false>, b)
               : gathered ? cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, kDirectBlockK<DIM>, false>, b)
                          : cudaLaunchKernelEx(&cfg, direct_sweep_clocked<DIM, NOFF, UNIFORM, 0, false>, b);
    }
    if (!a.lean)  // every term: length, chemotaxis, connectivity, motility, drift, nematic, moments
        return compact    ? cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, kDirectCompactK, true>, b)
               : gathered ? cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, kDirectBlockK<DIM>, true>, b)
                          : cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, 0, true>, b);
    return compact    ? cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, kDirectCompactK, false>, b)
           : gathered ? cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, kDirectBlockK<DIM>, false>, b)
                      : cudaLaunchKernelEx(&cfg, direct_sweep_kernel<DIM, NOFF, UNIFORM, 0, false>, b);
}

template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t launch_lean(const SweepLaunch &a, const CUtensorMap &tmap, cudaStream_t stream) {
    using T = Tile<DIM>;
    static std::atomic<int> grid_cap_once{0};  // handles on other host threads may launch too
    const size_t smem = sizeof(LeanSmem<DIM>) + 128;
    if (!grid_cap_once.load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(lean_sweep_kernel<DIM, NOFF, UNIFORM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e) return e;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev))) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lean_sweep_kernel<DIM, NOFF, UNIFORM>,
                                                               kLeanThreads, smem)))
            return e;
        grid_cap_once.store(sms * (per_sm > 0 ? per_sm : 1), std::memory_order_release);
    }
    const int tiles = ((a.g.w + T::TX - 1) / T::TX) * ((a.g.h + T::TY - 1) / T::TY) *
                      (DIM == 3 ? (a.g.d + T::TZ - 1) / T::TZ : 1);
    const int grid_cap = grid_cap_once.load(std::memory_order_acquire);
    int grid = tiles < grid_cap ? tiles : grid_cap;
    if (a.max_ctas > 0 && grid > a.max_ctas) grid = a.max_ctas;
    // Programmatic launch: the grid may start its prologue while the previous
    // kernel on the stream ends (the kernel waits before it reads pass data).
    // GLAZIER_SWEEP_PDL=0 launches it plainly.
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kLeanThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = programmatic_launch();
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, lean_sweep_kernel<DIM, NOFF, UNIFORM>, a, tmap);
}

template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t launch(const SweepLaunch &a, cudaStream_t stream) {
    // the compile-time neighbourhood must be the one the host built
    for (int k = 0; k < NOFF; ++k)
        for (int axis = 0; axis < 3; ++axis)
            if (a.g.off[k][axis] != neighbour_offset<DIM, NOFF>(k, axis)) return cudaErrorInvalidValue;
    CUtensorMap tmap;
    if (a.use_tma && a.tensor_map)
        tmap = *static_cast<const CUtensorMap *>(a.tensor_map);
    else
        memset(&tmap, 0, sizeof tmap);
    if (a.direct) return launch_direct<DIM, NOFF, UNIFORM>(a, stream);
    if (a.lean) return launch_lean<DIM, NOFF, UNIFORM>(a, tmap, stream);
    using T = Tile<DIM>;
    static std::atomic<int> grid_cap_once{0};  // handles on other host threads may launch too
    const size_t smem = sizeof(SweepSmem<DIM>) + 128;
    if (!grid_cap_once.load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(sweep_kernel<DIM, NOFF, UNIFORM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e) return e;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev))) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<DIM, NOFF, UNIFORM>, kThreads, smem)))
            return e;
        grid_cap_once.store(sms * (per_sm > 0 ? per_sm : 1), std::memory_order_release);
    }
    const int tiles = ((a.g.w + T::TX - 1) / T::TX) * ((a.g.h + T::TY - 1) / T::TY) *
                      (DIM == 3 ? (a.g.d + T::TZ - 1) / T::TZ : 1);
    const int grid_cap = grid_cap_once.load(std::memory_order_acquire);
    int grid = tiles < grid_cap ? tiles : grid_cap;
    if (a.max_ctas > 0 && grid > a.max_ctas) grid = a.max_ctas;
    // programmatic launch as the lean kernel's, except for a motility pass,
    // which follows its predecessor's copy list and a memset, not a kernel
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = programmatic_launch() && !a.has_motility;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, sweep_kernel<DIM, NOFF, UNIFORM>, a, tmap);
}

template <bool UNIFORM>
static cudaError_t launch_any(const SweepLaunch &a, cudaStream_t stream) {
    if (a.g.dim == 2) {
        if (a.g.n_off == 4) return launch<2, 4, UNIFORM>(a, stream);
        if (a.g.n_off == 8) return launch<2, 8, UNIFORM>(a, stream);
    } else {
        if (a.g.n_off == 6) return launch<3, 6, UNIFORM>(a, stream);
        if (a.g.n_off == 18) return launch<3, 18, UNIFORM>(a, stream);
        if (a.g.n_off == 26) return launch<3, 26, UNIFORM>(a, stream);
    }
    return cudaErrorInvalidValue;
}

__global__ void apply_copies_kernel(const __grid_constant__ SweepLaunch a, float *activity) {
    const int count = *a.pending_count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint2 p = a.pending[k];
        a.labels[p.x] = p.y;
        if (p.y != 0) {
            const float top = a.t.max_activity[a.cell_type[p.y]];
            if (top > 0.0f) activity[p.x] = top;
        }
    }
}

cudaError_t launch_apply_copies(const SweepLaunch &a, float *activity, cudaStream_t stream) {
    // at most one copy per target, and a pass has sites / colours targets
    const int most = a.g.sites / a.g.ncol + 1;
    apply_copies_kernel<<<(most + 255) / 256, 256, 0, stream>>>(a, activity);
    if (cudaError_t e = cudaGetLastError()) return e;
    return cudaMemsetAsync(a.pending_count, 0, sizeof(int), stream);
}

__global__ void activity_decay_kernel(float *activity, int sites) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sites) return;
    const float v = activity[i];
    activity[i] = v > 0.0f ? __fsub_rn(v, 1.0f) : 0.0f;
}

cudaError_t launch_activity_decay(float *activity, int sites, cudaStream_t stream) {
    activity_decay_kernel<<<(sites + 255) / 256, 256, 0, stream>>>(activity, sites);
    return cudaGetLastError();
}

cudaError_t launch_sweep(const SweepLaunch &a, cudaStream_t stream) {
    return a.uniform_type >= 0 && a.uniform_contact_exact ? launch_any<true>(a, stream) : launch_any<false>(a, stream);
}


// ---------------------------------------------------------------- the ensemble

template <int DIM>
struct EnsembleSmem {
    SweepSmem<DIM> s;
    SweepLaunch desc;  // the current replica's launch, per-pass fields patched
    int replica;       // the replica `desc` holds, -1 before the first tile
    int next_replica;
};

// The schedule position of tile t: the last prefix entry at or below it.
__device__ __forceinline__ int replica_of_tile(const int *prefix, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int DIM, int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kThreads, GLZ_SWEEP_MIN_BLOCKS)
    ensemble_sweep_kernel(const __grid_constant__ EnsembleLaunch e) {
    using T = Tile<DIM>;
    using Smem = SweepSmem<DIM>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    EnsembleSmem<DIM> &E = *reinterpret_cast<EnsembleSmem<DIM> *>(smem_raw + ((128u - (raw & 127u)) & 127u));
    Smem &S = E.s;
    const int tid = threadIdx.x;
    if (smem_addr(S.win[0]) & 127u) {
        if (tid == 0) atomicExch(e.error_flag, 3);
        return;
    }
    const long long step = e.clock->step;
    const long long pass = e.clock->pass + e.colour;

    // Tally rotation for the next pass over every replica's cells at once.
    {
        const size_t stride = (size_t)gridDim.x * blockDim.x;
        int2 *const base = e.vs_base[pass % 2];
        const long long *const prev = e.vs_delta[(pass + 2) % 3];
        int2 *const next_base = e.vs_base[(pass + 1) % 2];
        long long *const clear = e.vs_delta[(pass + 1) % 3];
        for (size_t l = (size_t)blockIdx.x * blockDim.x + tid; l < (size_t)e.total_cells; l += stride) {
            int dv, ds;
            unpack_delta(prev[l], dv, ds);
            const int2 b = base[l];
            next_base[l] = make_int2(b.x + dv, b.y + ds);
            clear[l] = 0;
        }
    }
    if (tid < NOFF) S.woff[tid] = window_offset<DIM, NOFF>(tid);
    if (tid == 0) {
        S.queued = 0;
        S.taken = 0;
        E.replica = -1;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const CUtensorMap *maps = static_cast<const CUtensorMap *>(e.maps);
    int waited[2] = {0, 0};
    bool pending[2] = {false, false};
    // The position, origin and tensor-copy eligibility of global tile t.
    auto locate = [&](int t, int &pos, int &x0, int &y0, int &z0) -> bool {
        pos = replica_of_tile(e.tile_prefix, e.n, t);
        const SweepLaunch &ra = e.replicas[e.order[pos]].a;
        tile_origin<DIM>(t - e.tile_prefix[pos], ra.g.w, ra.g.h, x0, y0, z0);
        return maps != nullptr && tile_interior<DIM>(ra, x0, y0, z0);
    };
    // Each CTA takes a contiguous run of the schedule's tiles (runs differ by
    // at most one tile), so consecutive tiles mostly share a replica and its
    // launch stays in shared memory.
    const int per = e.total_tiles / (int)gridDim.x, extra = e.total_tiles % (int)gridDim.x;
    const int first = (int)blockIdx.x * per + ((int)blockIdx.x < extra ? (int)blockIdx.x : extra);
    const int last = first + per + ((int)blockIdx.x < extra ? 1 : 0);
    int t = first;
    if (t < last) {
        int pos, x0, y0, z0;
        if (locate(t, pos, x0, y0, z0)) {
            if (tid == 0) issue_window<DIM>(maps[e.order[pos]], S.win[0], &S.mbar[0], x0, y0, z0);
            pending[0] = true;
        }
    }
    for (int it = 0; t < last; ++t, ++it) {
        const int buf = it & 1;
        int pos, x0, y0, z0;
        const bool interior = locate(t, pos, x0, y0, z0);
        const int r = e.order[pos];
        const int next = t + 1;
        if (next < last) {
            int npos, nx0, ny0, nz0;
            if (locate(next, npos, nx0, ny0, nz0)) {
                if (tid == 0) issue_window<DIM>(maps[e.order[npos]], S.win[buf ^ 1], &S.mbar[buf ^ 1], nx0, ny0, nz0);
                pending[buf ^ 1] = true;
            }
        }
        if (r != E.replica) {
            // Bring this replica's launch into shared memory and patch the
            // per-pass fields: keys, tally rotation, colour, step.
            __syncthreads();
            const EnsembleReplica &rep = e.replicas[r];
            const int *src = reinterpret_cast<const int *>(&rep.a);
            int *dst = reinterpret_cast<int *>(&E.desc);
            for (int i = tid; i < (int)(sizeof(SweepLaunch) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            if (tid == 0) {
                SweepLaunch &d = E.desc;
                d.colour = e.colour;
                d.step = (int32_t)step;
                d.key_pick = stream_key(rep.seed, d.step, e.colour, 0);
                d.key_accept = stream_key(rep.seed, d.step, e.colour, 1);
                d.vs_base = e.vs_base[pass % 2] + rep.cell_off;
                d.vs_prev = e.vs_delta[(pass + 2) % 3] + rep.cell_off;
                d.vs_cur = reinterpret_cast<unsigned long long *>(e.vs_delta[pass % 3] + rep.cell_off);
                E.replica = r;
            }
            const bool small = rep.a.n_types <= kSmemTypes;
            if (small)
                for (int i = tid; i < rep.a.n_types * rep.a.n_types; i += blockDim.x) S.contact[i] = rep.a.t.contact[i];
            __syncthreads();
        }
        const SweepLaunch &a = E.desc;
        uint32_t *win = S.win[buf];
        if (interior) {
            const uint32_t done = wait_parity(&S.mbar[buf], waited[buf] & 1);
            waited[buf] += 1;
            pending[buf] = false;
            if (!__syncthreads_and(done)) {
                if (pending[buf ^ 1]) wait_parity(&S.mbar[buf ^ 1], waited[buf ^ 1] & 1);
                if (tid == 0) atomicExch(e.error_flag, 1);
                return;
            }
        } else {
            load_window_plain<DIM>(a, win, x0, y0, z0);
        }
        price_tile<DIM, NOFF, UNIFORM>(a, S, win, x0, y0, z0, a.n_types <= kSmemTypes);
    }
}

// ---------------------------------------------------------------- the lean ensemble
//
// The lean kernel's layout over an ensemble: warp-owned target shares, the
// window ring refilled by the last warp out, queue entries carried into the
// warp's next tile. Warps may be on different tiles, so each ring slot holds
// its own copy of the tile's replica launch, with the pass's fields patched
// in; the warp that refills a slot copies the next tile's launch in first.
// Each CTA takes a contiguous run of the schedule's tiles.
template <int DIM>
struct LeanEnsembleSmem {
    LeanSmem<DIM> s;
    SweepLaunch desc[kLeanStages];  // the slot's tile's replica launch
    int org[kLeanStages][4];        // the slot's tile: origin x, y, z, replica
};

// The schedule's tile t: its replica's launch (pass fields patched) and
// origin into slot `slot`, by the whole warp; lane 0 then starts its window
// (a tensor copy, or a bare arrival when the replica's window takes plain
// loads).
template <int DIM>
__device__ __forceinline__ void lean_ens_fill(const EnsembleLaunch &e, LeanEnsembleSmem<DIM> &E, int t, int slot,
                                              long long step, long long pass) {
    using T = Tile<DIM>;
    const int lane = threadIdx.x & 31;
    const int pos = replica_of_tile(e.tile_prefix, e.n, t);
    const int r = e.order[pos];
    const EnsembleReplica &rep = e.replicas[r];
    const int *src = reinterpret_cast<const int *>(&rep.a);
    int *dst = reinterpret_cast<int *>(&E.desc[slot]);
    for (int i = lane; i < (int)(sizeof(SweepLaunch) / sizeof(int)); i += 32) dst[i] = src[i];
    __syncwarp();
    if (lane == 0) {
        SweepLaunch &d = E.desc[slot];
        d.colour = e.colour;
        d.step = (int32_t)step;
        d.key_pick = stream_key(rep.seed, d.step, e.colour, 0);
        d.key_accept = stream_key(rep.seed, d.step, e.colour, 1);
        d.vs_base = e.vs_base[pass % 2] + rep.cell_off;
        d.vs_prev = e.vs_delta[(pass + 2) % 3] + rep.cell_off;
        d.vs_cur = reinterpret_cast<unsigned long long *>(e.vs_delta[pass % 3] + rep.cell_off);
        int x0, y0, z0;
        tile_origin<DIM>(t - e.tile_prefix[pos], d.g.w, d.g.h, x0, y0, z0);
        E.org[slot][0] = x0;
        E.org[slot][1] = y0;
        E.org[slot][2] = z0;
        E.org[slot][3] = r;
        E.s.issued[slot] += 1;
        const CUtensorMap *maps = static_cast<const CUtensorMap *>(e.maps);
        if (maps && lean_copies<DIM>(d))
            issue_window<DIM>(maps[r], E.s.win[slot], &E.s.full[slot], x0, y0, z0);
        else
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&E.s.full[slot])) : "memory");
    }
}

template <int DIM, int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kLeanThreads, GLZ_LEAN_MIN_BLOCKS)
    lean_ensemble_kernel(const __grid_constant__ EnsembleLaunch e) {
    using T = Tile<DIM>;
    using Smem = LeanSmem<DIM>;
    constexpr int PER_LANE = Smem::TPW / 32;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    LeanEnsembleSmem<DIM> &E = *reinterpret_cast<LeanEnsembleSmem<DIM> *>(smem_raw + ((128u - (raw & 127u)) & 127u));
    Smem &S = E.s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (smem_addr(S.win[0]) & 127u) {
        if (tid == 0) atomicExch(e.error_flag, 3);
        return;
    }
    const long long step = e.clock->step;
    const long long pass = e.clock->pass + e.colour;
    const int per = e.total_tiles / (int)gridDim.x, extra = e.total_tiles % (int)gridDim.x;
    const int first = (int)blockIdx.x * per + ((int)blockIdx.x < extra ? (int)blockIdx.x : extra);
    const int mine = per + ((int)blockIdx.x < extra ? 1 : 0);

    if (tid == 0) {
        for (int k = 0; k < kLeanStages; ++k) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.full[k])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&S.patched[k])), "r"(kLeanWarps));
            S.done[k] = 0;
            S.issued[k] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
#pragma unroll
    for (int k = 0; k < NOFF; ++k)
        if (tid == k) S.woff[k] = window_offset<DIM, NOFF>(k);
    __syncthreads();
    if (warp == 0)
        for (int i = 0; i < kLeanStages && i < mine; ++i) lean_ens_fill<DIM>(e, E, first + i, i, step, pass);
    // the tally rotation over every replica's cells, its reads copied in ahead
    const size_t rot_stride = (size_t)gridDim.x * blockDim.x;
    const size_t rot_first = (size_t)blockIdx.x * blockDim.x + tid;
    const int2 *rot_base = e.vs_base[pass % 2];
    const long long *rot_prev = e.vs_delta[(pass + 2) % 3];
#pragma unroll
    for (int k = 0; k < kRotate; ++k) {
        const size_t l = rot_first + k * rot_stride;
        if (l < (size_t)e.total_cells) {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(&S.rot_base[k * kLeanThreads + tid])),
                         "l"(rot_base + l)
                         : "memory");
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(&S.rot_prev[k * kLeanThreads + tid])),
                         "l"(rot_prev + l)
                         : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");

    uint32_t *queue = S.queue[warp];
    const unsigned below = (1u << lane) - 1u;
    uint32_t patch_parity = 0;
    int held = 0, held_slot = -1;

    for (int i = 0; i < mine; ++i) {
        const int slot = i % kLeanStages;
        uint32_t *win = S.win[slot];
        bool ok = wait_parity(&S.full[slot], (uint32_t)(i / kLeanStages) & 1u) != 0;
        const SweepLaunch &a = E.desc[slot];
        const int x0 = E.org[slot][0], y0 = E.org[slot][1], z0 = E.org[slot][2];
        const int W = a.g.w, H = a.g.h, D = a.g.d;
        const bool copies = e.maps != nullptr && lean_copies<DIM>(a);
        const bool edge = !copies || !(x0 >= T::HX && x0 + T::TX + T::HX <= W && y0 >= 1 && y0 + T::TY + 1 <= H &&
                                       (DIM == 2 || (z0 >= 1 && z0 + T::TZ + 1 <= D)));
        if (edge && __all_sync(0xffffffffu, ok)) {
            lean_patch<DIM>(a, win, x0, y0, z0, copies);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&S.patched[slot])) : "memory");
            ok = wait_parity(&S.patched[slot], (patch_parity >> slot) & 1u) != 0;
            patch_parity ^= 1u << slot;
        }
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) {
                atomicExch(e.error_flag, 1);
                for (int k = 0; k < kLeanStages; ++k)
                    if (S.issued[k] > 0) wait_parity(&S.full[k], (uint32_t)(S.issued[k] - 1) & 1u);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            return;
        }

        // light pass over this warp's share, behind the entries held over
        const bool full = x0 + T::TX <= W && y0 + T::TY <= H && (DIM == 2 || z0 + T::TZ <= D);
        const uint32_t tile_base = (uint32_t)((z0 * H + y0) * W + x0);
        uint32_t entries[PER_LANE];
        unsigned masks[PER_LANE];
#pragma unroll
        for (int k = 0; k < PER_LANE; ++k) {
            const int j = warp * Smem::TPW + k * 32 + lane;
            int lx, ly, lz;
            target_of<DIM>(j, e.colour, lx, ly, lz);
            const bool in = full || (x0 + lx < W && y0 + ly < H && (DIM == 2 || z0 + lz < D));
            bool active = false;
            int pick = 0;
            if (in) {
                const int wc = ((lz + T::HZ) * T::PY + (ly + 1)) * T::PX + (lx + T::HX);
                pick = pick_of<NOFF>(draw(a.key_pick, tile_base + (uint32_t)((lz * H + ly) * W + lx)));
                active = win[wc] != win[wc + S.woff[pick]];
            }
            entries[k] = (uint32_t)j | ((uint32_t)pick << 16);
            masks[k] = __ballot_sync(0xffffffffu, active);
        }
        int total = held;
#pragma unroll
        for (int k = 0; k < PER_LANE; ++k) {
            if (masks[k] & (1u << lane)) queue[total + __popc(masks[k] & below)] = entries[k];
            total += __popc(masks[k]);
        }
        __syncwarp();
        int taken = 0;
        for (;;) {
            const int n = total - taken;
            if (n < 32 && taken >= held) break;
            const int q = taken + lane;
            if (q < total) {
                const int s_ = q < held ? held_slot : slot;
                price_and_commit<DIM, NOFF, UNIFORM, false>(E.desc[s_], S.woff, nullptr, nullptr, S.win[s_], queue[q],
                                                            E.org[s_][0], E.org[s_][1], E.org[s_][2], false);
            }
            taken += n < 32 ? n : 32;
        }
        __syncwarp();
        if (held_slot >= 0) {
            // release the previous tile's slot; the last warp out refills it
            int last_out = 0;
            if (lane == 0) {
                __threadfence_block();
                last_out = atomicAdd(&S.done[held_slot], 1) == kLeanWarps - 1;
                if (last_out) S.done[held_slot] = 0;
            }
            last_out = __shfl_sync(0xffffffffu, last_out, 0);
            if (last_out && i - 1 + kLeanStages < mine) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                lean_ens_fill<DIM>(e, E, first + i - 1 + kLeanStages, held_slot, step, pass);
            }
        }
        const int keep = total - taken;
        if (taken > 0 && keep > 0) {
            const uint32_t v = lane < keep ? queue[taken + lane] : 0u;
            __syncwarp();
            if (lane < keep) queue[lane] = v;
            __syncwarp();
        }
        held = keep;
        held_slot = slot;
    }
    if (mine > 0) {
        if (lane < held)
            price_and_commit<DIM, NOFF, UNIFORM, false>(E.desc[held_slot], S.woff, nullptr, nullptr, S.win[held_slot],
                                                        queue[lane], E.org[held_slot][0], E.org[held_slot][1],
                                                        E.org[held_slot][2], false);
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            atomicAdd(&S.done[held_slot], 1);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    int2 *next_base = e.vs_base[(pass + 1) % 2];
    long long *clear = e.vs_delta[(pass + 1) % 3];
#pragma unroll
    for (int k = 0; k < kRotate; ++k) {
        const size_t l = rot_first + k * rot_stride;
        if (l < (size_t)e.total_cells) {
            int dv, ds;
            unpack_delta(S.rot_prev[k * kLeanThreads + tid], dv, ds);
            const int2 b = S.rot_base[k * kLeanThreads + tid];
            next_base[l] = make_int2(b.x + dv, b.y + ds);
            clear[l] = 0;
        }
    }
    for (size_t l = rot_first + kRotate * rot_stride; l < (size_t)e.total_cells; l += rot_stride) {
        int dv, ds;
        unpack_delta(rot_prev[l], dv, ds);
        const int2 b = rot_base[l];
        next_base[l] = make_int2(b.x + dv, b.y + ds);
        clear[l] = 0;
    }
}

// ---------------------------------------------------------------- the direct ensemble
//
// A plane ensemble's pass with one block per tile of BX x BY targets of one
// replica: the block finds its replica, copies the replica's launch into
// shared memory with the pass's fields patched from the clock, and prices
// every target of its tile where it lies (direct_target, as the direct
// kernel does). The tile shape sets which sites a block's loads share; the
// autotuner picks it by time, since the results do not depend on it.
// Tile t of colour pass `colour` (pass number `pass`, step `step`): the
// block finds the tile's replica, patches the replica's launch into `d` and
// prices the tile's targets.
template <int NOFF, bool UNIFORM, int BX, int BY>
__device__ __forceinline__ void direct_ensemble_tile(const EnsembleLaunch &e, SweepLaunch &d, int *where, int t,
                                                     int colour, long long step, long long pass) {
    if (threadIdx.x == 0) {
        const int pos = replica_of_tile(e.tile_prefix, e.n, t);
        where[0] = pos;
        where[1] = e.order[pos];
    }
    __syncthreads();
    const int pos = where[0];
    const EnsembleReplica &rep = e.replicas[where[1]];
    {
        const int *src = reinterpret_cast<const int *>(&rep.a);
        int *dst = reinterpret_cast<int *>(&d);
        for (int i = threadIdx.x; i < (int)(sizeof(SweepLaunch) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        d.colour = colour;
        d.step = (int32_t)step;
        d.key_pick = stream_key(rep.seed, d.step, colour, 0);
        d.key_accept = stream_key(rep.seed, d.step, colour, 1);
        d.vs_base = e.vs_base[pass % 2] + rep.cell_off;
        d.vs_prev = e.vs_delta[(pass + 2) % 3] + rep.cell_off;
        d.vs_cur = reinterpret_cast<unsigned long long *>(e.vs_delta[pass % 3] + rep.cell_off);
    }
    __syncthreads();
    const int lt = t - e.tile_prefix[pos];
    const int hw = d.g.w / 2, hh = d.g.h / 2;
    const int tiles_x = (hw + BX - 1) / BX;
    const int jx = (lt % tiles_x) * BX + (int)threadIdx.x % BX;
    const int jy = (lt / tiles_x) * BY + (int)threadIdx.x / BX;
    if (jx < hw && jy < hh) {
        const PassView v{colour, d.key_pick, d.key_accept, d.vs_base, d.vs_prev, d.vs_cur};
        direct_target<2, NOFF, UNIFORM, GlobalPass, false>(d, GlobalPass{d, v}, v.key_pick, v.key_accept,
                                                           2 * jx + (colour & 1), 2 * jy + ((colour >> 1) & 1), 0);
    }
    __syncthreads();  // `d` and `where` serve the block's next tile
}

// The tally rotation over every replica's cells for the pass numbered `pass`,
// which no thread of that pass reads, spread over the grid.
__device__ __forceinline__ void ensemble_rotate(const EnsembleLaunch &e, long long pass) {
    int2 *next_base = e.vs_base[(pass + 1) % 2];
    long long *clear = e.vs_delta[(pass + 1) % 3];
    const int2 *base = e.vs_base[pass % 2];
    const long long *prev = e.vs_delta[(pass + 2) % 3];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x; l < (size_t)e.total_cells; l += stride) {
        int dv, ds;
        unpack_delta(prev[l], dv, ds);
        const int2 b = base[l];
        next_base[l] = make_int2(b.x + dv, b.y + ds);
        clear[l] = 0;
    }
}

// A plane ensemble's pass with one block per tile of BX x BY targets of one
// replica, priced where they lie (direct_target, as the direct kernel does).
// The tile shape sets which sites a block's loads share; the autotuner picks
// it by time, since the results do not depend on it.
template <int NOFF, bool UNIFORM, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) direct_ensemble_kernel(const __grid_constant__ EnsembleLaunch e) {
    __shared__ SweepLaunch d;
    __shared__ int where[2];  // the tile's place in the schedule, its replica
    const long long step = e.clock->step;
    const long long pass = e.clock->pass + e.colour;
    direct_ensemble_tile<NOFF, UNIFORM, BX, BY>(e, d, where, (int)blockIdx.x, e.colour, step, pass);
    ensemble_rotate(e, pass);
}

// Every colour pass of a step in one cooperative launch: blocks stride over
// the tiles, a grid barrier between passes (the tallies a pass reads are its
// snapshot, complete once every block has finished the pass before).
template <int NOFF, bool UNIFORM, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) direct_ensemble_step_kernel(const __grid_constant__ EnsembleLaunch e) {
    __shared__ SweepLaunch d;
    __shared__ int where[2];
    const long long step = e.clock->step;
    for (int c = 0; c < e.ncol; ++c) {
        const long long pass = e.clock->pass + c;
        for (int t = (int)blockIdx.x; t < e.total_tiles; t += (int)gridDim.x)
            direct_ensemble_tile<NOFF, UNIFORM, BX, BY>(e, d, where, t, c, step, pass);
        ensemble_rotate(e, pass);
        if (c + 1 < e.ncol && !resident_barrier(e.barrier, (unsigned)c)) {
            if (threadIdx.x == 0) atomicExch(e.error_flag, 4);
            return;
        }
    }
}

template <int NOFF, bool UNIFORM, int BX, int BY>
static cudaError_t direct_ensemble_shape(const EnsembleLaunch &e, cudaStream_t stream) {
    if (!e.one_launch) {
        direct_ensemble_kernel<NOFF, UNIFORM, BX, BY><<<e.total_tiles, BX * BY, 0, stream>>>(e);
        return cudaGetLastError();
    }
    static std::atomic<int> most_once{0};  // blocks that can all be resident at once
    if (!most_once.load(std::memory_order_acquire)) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaError_t x = cudaGetDevice(&dev)) return x;
        if (cudaError_t x = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return x;
        if (cudaError_t x = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, direct_ensemble_step_kernel<NOFF, UNIFORM, BX, BY>, BX * BY, 0))
            return x;
        most_once.store(sms * per_sm, std::memory_order_release);
    }
    const int most = most_once.load(std::memory_order_acquire);
    if (most < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int grid = e.total_tiles < most ? e.total_tiles : most;
    if (cudaError_t x = cudaMemsetAsync(e.barrier, 0, 2 * sizeof(unsigned), stream)) return x;
    void *args[] = {const_cast<EnsembleLaunch *>(&e)};
    return cudaLaunchCooperativeKernel((const void *)direct_ensemble_step_kernel<NOFF, UNIFORM, BX, BY>, dim3(grid),
                                       dim3(BX * BY), args, 0, stream);
}

template <int NOFF, bool UNIFORM>
static cudaError_t direct_ensemble_launch(const EnsembleLaunch &e, cudaStream_t stream) {
    if (e.total_tiles <= 0) return cudaSuccess;
    if (e.tile_shape == 1) return direct_ensemble_shape<NOFF, UNIFORM, 32, 8>(e, stream);
    if (e.tile_shape == 2) return direct_ensemble_shape<NOFF, UNIFORM, 16, 16>(e, stream);
    return direct_ensemble_shape<NOFF, UNIFORM, 64, 4>(e, stream);
}

__global__ void clock_advance_kernel(EnsembleClock *clock, int ncol) {
    clock->step += 1;
    clock->pass += ncol;
}

template <int DIM, int NOFF, bool UNIFORM>
static int ensemble_cap() {
    static std::atomic<int> cap{0};  // handles on other host threads may launch too
    if (!cap.load(std::memory_order_acquire)) {
        const size_t smem = sizeof(EnsembleSmem<DIM>) + 128;
        if (cudaFuncSetAttribute(ensemble_sweep_kernel<DIM, NOFF, UNIFORM>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
            return 0;
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ensemble_sweep_kernel<DIM, NOFF, UNIFORM>, kThreads,
                                                          smem))
            return 0;
        cap.store(sms * (per_sm > 0 ? per_sm : 1), std::memory_order_release);
    }
    return cap.load(std::memory_order_acquire);
}

// Whether ensembles take the lean kernel (GLAZIER_ENSEMBLE_LEAN=0: the
// barrier-per-tile one).
static bool lean_ensemble() {
    static const bool on = [] {
        const char *env = std::getenv("GLAZIER_ENSEMBLE_LEAN");
        return !(env && env[0] == '0');
    }();
    return on;
}

template <int DIM, int NOFF, bool UNIFORM>
static int lean_ensemble_cap() {
    static std::atomic<int> cap{0};  // handles on other host threads may launch too
    if (!cap.load(std::memory_order_acquire)) {
        const size_t smem = sizeof(LeanEnsembleSmem<DIM>) + 128;
        if (cudaFuncSetAttribute(lean_ensemble_kernel<DIM, NOFF, UNIFORM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem))
            return 0;
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lean_ensemble_kernel<DIM, NOFF, UNIFORM>,
                                                          kLeanThreads, smem))
            return 0;
        cap.store(sms * (per_sm > 0 ? per_sm : 1), std::memory_order_release);
    }
    return cap.load(std::memory_order_acquire);
}

template <int DIM, int NOFF, bool UNIFORM>
static cudaError_t ensemble_launch(const EnsembleLaunch &e, cudaStream_t stream) {
    if (lean_ensemble()) {
        const int cap = lean_ensemble_cap<DIM, NOFF, UNIFORM>();
        if (!cap) return cudaErrorInvalidConfiguration;
        int grid = e.total_tiles < cap ? e.total_tiles : cap;
        if (e.max_ctas > 0 && grid > e.max_ctas) grid = e.max_ctas;
        const size_t smem = sizeof(LeanEnsembleSmem<DIM>) + 128;
        lean_ensemble_kernel<DIM, NOFF, UNIFORM><<<grid, kLeanThreads, smem, stream>>>(e);
        return cudaGetLastError();
    }
    const int cap = ensemble_cap<DIM, NOFF, UNIFORM>();
    if (!cap) return cudaErrorInvalidConfiguration;
    int grid = e.total_tiles < cap ? e.total_tiles : cap;
    if (e.max_ctas > 0 && grid > e.max_ctas) grid = e.max_ctas;
    const size_t smem = sizeof(EnsembleSmem<DIM>) + 128;
    ensemble_sweep_kernel<DIM, NOFF, UNIFORM><<<grid, kThreads, smem, stream>>>(e);
    return cudaGetLastError();
}

template <bool UNIFORM>
static cudaError_t ensemble_any(const EnsembleLaunch &e, int dim, int n_off, cudaStream_t stream) {
    if (e.tile_shape > 0) {
        if (dim != 2 || e.tile_shape > 3) return cudaErrorInvalidValue;
        return n_off == 4 ? direct_ensemble_launch<4, UNIFORM>(e, stream) : direct_ensemble_launch<8, UNIFORM>(e, stream);
    }
    if (dim == 2) {
        if (n_off == 4) return ensemble_launch<2, 4, UNIFORM>(e, stream);
        if (n_off == 8) return ensemble_launch<2, 8, UNIFORM>(e, stream);
    } else {
        if (n_off == 6) return ensemble_launch<3, 6, UNIFORM>(e, stream);
        if (n_off == 18) return ensemble_launch<3, 18, UNIFORM>(e, stream);
        if (n_off == 26) return ensemble_launch<3, 26, UNIFORM>(e, stream);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_ensemble_sweep(const EnsembleLaunch &e, int dim, int n_off, bool uniform, cudaStream_t stream) {
    return uniform ? ensemble_any<true>(e, dim, n_off, stream) : ensemble_any<false>(e, dim, n_off, stream);
}

cudaError_t launch_clock_advance(EnsembleClock *clock, int ncol, cudaStream_t stream) {
    clock_advance_kernel<<<1, 1, 0, stream>>>(clock, ncol);
    return cudaGetLastError();
}

template <int DIM, int NOFF, bool UNIFORM>
static int grid_cap_of() {
    return lean_ensemble() ? lean_ensemble_cap<DIM, NOFF, UNIFORM>() : ensemble_cap<DIM, NOFF, UNIFORM>();
}

template <bool UNIFORM>
static int cap_any(int dim, int n_off) {
    if (dim == 2) return n_off == 4 ? grid_cap_of<2, 4, UNIFORM>() : grid_cap_of<2, 8, UNIFORM>();
    if (n_off == 6) return grid_cap_of<3, 6, UNIFORM>();
    if (n_off == 18) return grid_cap_of<3, 18, UNIFORM>();
    return grid_cap_of<3, 26, UNIFORM>();
}

int ensemble_grid_cap(int dim, int n_off, bool uniform) { return uniform ? cap_any<true>(dim, n_off) : cap_any<false>(dim, n_off); }

// The box a sweep tile's tensor copy moves: the tile plus its halo.
int sweep_box(int dim, uint32_t box[3]) {
    if (dim == 2) {
        box[0] = Tile<2>::PX;
        box[1] = Tile<2>::PY;
        box[2] = 1;
    } else {
        box[0] = Tile<3>::PX;
        box[1] = Tile<3>::PY;
        box[2] = Tile<3>::PZ;
    }
    return 0;
}

}  // namespace glz
