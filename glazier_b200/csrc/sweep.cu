// The checkerboard Metropolis copy sweep: one launch per colour.
//
// Replaces `cpm_sweep` of the reference device engine (glazier-cuda/src/
// lib.rs:436-716). Each CTA owns a tile of the lattice, stages the tile and a
// one-site halo of labels in shared memory (a TMA tensor copy for tiles away
// from the periodic edge, wrapped plain loads elsewhere), and prices every
// target of the pass's colour in it. Same-colour targets are two apart on
// every axis, outside any neighbourhood, so a pass's copies are independent
// and the labels a target reads do not change during the pass.
//
// Per-cell tallies (volume, surface, exact moment sums) are read from the
// snapshot the rotation in engine.h gives each pass, and changed by integer
// atomics whose order does not matter; a pass is therefore deterministic and
// a host replay of the same schedule reproduces it bit for bit.

#include <cuda.h>

#include "device.cuh"
#include "engine.h"

namespace glz {

template <int DIM>
struct Tile;

template <>
struct Tile<2> {
    static constexpr int TX = 64, TY = 32, TZ = 1;
    static constexpr int HX = 4;  // x halo rounded up to 16 bytes for the tensor copy
    static constexpr int PX = TX + 2 * HX, PY = TY + 2, PZ = 1;
    static constexpr int HZ = 0;
    static constexpr int NT = (TX / 2) * (TY / 2);
};

template <>
struct Tile<3> {
    static constexpr int TX = 32, TY = 8, TZ = 8;
    static constexpr int HX = 4;
    static constexpr int PX = TX + 2 * HX, PY = TY + 2, PZ = TZ + 2;
    static constexpr int HZ = 1;
    static constexpr int NT = (TX / 2) * (TY / 2) * (TZ / 2);
};

constexpr int kSweepThreads = 256;
constexpr int kSmemTypes = 16;  // contact tables up to 16 types live in shared memory
constexpr long long kWaitLimit = 1LL << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

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
__device__ double length_delta(const SweepLaunch &a, int type, int label, long long n, const long long *terms,
                               int sign) {
    constexpr int NM = DIM == 2 ? 5 : 9;
    long long m[NM], after[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        m[k] = a.mom_base[(size_t)label * NM + k] + a.mom_prev[(size_t)label * NM + k];
        after[k] = m[k] + sign * terms[k];
    }
    double tl = a.t.target_length[type];
    double before = axis_length<DIM>(n, m) - tl;
    double now = axis_length<DIM>(n + sign, after) - tl;
    return a.t.lambda_length[type] * (now * now - before * before);
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

template <int DIM, int NOFF>
__global__ void __launch_bounds__(kSweepThreads) sweep_kernel(const __grid_constant__ SweepLaunch a,
                                                              const __grid_constant__ CUtensorMap tmap) {
    using T = Tile<DIM>;
    constexpr int NM = DIM == 2 ? 5 : 9;
    __shared__ alignas(128) uint32_t win[T::PX * T::PY * T::PZ];
    __shared__ float s_contact[kSmemTypes * kSmemTypes];
    __shared__ alignas(8) unsigned long long mbar;
    __shared__ int s_woff[26];
    __shared__ int s_wring[26];

    const int tid = threadIdx.x;
    const int W = a.g.w, H = a.g.h, D = a.g.d;

    // Tally rotation for the next pass: no thread of this pass reads what is
    // written here (engine.h).
    {
        const size_t stride = (size_t)gridDim.x * blockDim.x;
        for (size_t l = (size_t)blockIdx.x * blockDim.x + tid; l < (size_t)a.n_labels; l += stride) {
            int dv, ds;
            unpack_delta(a.vs_prev[l], dv, ds);
            int2 b = a.vs_base[l];
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

    const int tiles_x = (W + T::TX - 1) / T::TX;
    const int tiles_y = (H + T::TY - 1) / T::TY;
    const int bx = blockIdx.x % tiles_x;
    const int by = (blockIdx.x / tiles_x) % tiles_y;
    const int bz = blockIdx.x / (tiles_x * tiles_y);
    const int x0 = bx * T::TX, y0 = by * T::TY, z0 = bz * T::TZ;

    const bool small_types = a.n_types <= kSmemTypes;
    if (small_types)
        for (int i = tid; i < a.n_types * a.n_types; i += blockDim.x) s_contact[i] = a.t.contact[i];
    if (tid < NOFF) s_woff[tid] = (a.g.off[tid][2] * T::PY + a.g.off[tid][1]) * T::PX + a.g.off[tid][0];
    if (tid < a.g.ring_n) s_wring[tid] = (a.g.ring[tid][2] * T::PY + a.g.ring[tid][1]) * T::PX + a.g.ring[tid][0];

    const bool interior = a.use_tma && x0 >= T::HX && x0 + T::TX + T::HX <= W && y0 >= 1 && y0 + T::TY + 1 <= H &&
                          (DIM == 2 || (z0 >= 1 && z0 + T::TZ + 1 <= D));
    bool loaded = true;
    if (interior) {
        // One tensor copy of the window. x0 - HX is a multiple of 4 labels,
        // i.e. of 16 bytes, as every tensor copy's inner coordinate must be.
        const uint32_t bar = smem_addr(&mbar);
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0) {
            const uint32_t bytes = sizeof(win);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
            const uint64_t map = reinterpret_cast<uint64_t>(&tmap);
            if (DIM == 2) {
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                    "[%4];" ::"r"(smem_addr(win)),
                    "l"(map), "r"(x0 - T::HX), "r"(y0 - 1), "r"(bar)
                    : "memory");
            } else {
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
                    "%4}], [%5];" ::"r"(smem_addr(win)),
                    "l"(map), "r"(x0 - T::HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
                    : "memory");
            }
        }
        // Bounded wait: a copy that never lands sets the error flag and the
        // tile is skipped rather than spinning for ever.
        uint32_t done = 0;
        for (long long spin = 0; spin < kWaitLimit && !done; ++spin) {
            asm volatile(
                "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                : "=r"(done)
                : "r"(bar)
                : "memory");
        }
        if (!done) {
            loaded = false;
            if (tid == 0) atomicExch(a.error_flag, 1);
        }
    } else {
        for (int i = tid; i < T::PX * T::PY * T::PZ; i += blockDim.x) {
            const int px = i % T::PX;
            const int py = (i / T::PX) % T::PY;
            const int pz = i / (T::PX * T::PY);
            const int gx = wrap(x0 - T::HX + px, W);
            const int gy = wrap(y0 - 1 + py, H);
            const int gz = DIM == 3 ? wrap(z0 - 1 + pz, D) : 0;
            win[i] = a.labels[((size_t)gz * H + gy) * W + gx];
        }
    }
    __syncthreads();
    if (!__syncthreads_and(loaded)) return;

    const int cx = a.colour & 1, cy = (a.colour >> 1) & 1, cz = (a.colour >> 2) & 1;
    for (int j = tid; j < T::NT; j += blockDim.x) {
        const int jx = j % (T::TX / 2);
        const int jy = (j / (T::TX / 2)) % (T::TY / 2);
        const int jz = DIM == 3 ? j / ((T::TX / 2) * (T::TY / 2)) : 0;
        const int lx = 2 * jx + cx, ly = 2 * jy + cy, lz = DIM == 3 ? 2 * jz + cz : 0;
        const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
        if (x >= W || y >= H || (DIM == 3 && z >= D)) continue;
        const uint32_t target = (uint32_t)(((size_t)z * H + y) * W + x);
        const int wc = ((lz + T::HZ) * T::PY + (ly + 1)) * T::PX + (lx + T::HX);

        const uint32_t old = win[wc];
        const int pick = (int)(draw(a.key_pick, target) % (uint64_t)NOFF);
        const uint32_t nw = win[wc + s_woff[pick]];
        if (old == nw) continue;

        const int t_old = a.cell_type[old], t_new = a.cell_type[nw];
        float delta = 0.0f;
        int like_old = 0, like_new = 0;
#pragma unroll
        for (int k = 0; k < NOFF; ++k) {
            const uint32_t ln = win[wc + s_woff[k]];
            const int tn = ln == old ? t_old : (ln == nw ? t_new : (int)a.cell_type[ln]);
            if (ln != old) {
                const float j_old = small_types ? s_contact[t_old * a.n_types + tn] : a.t.contact[t_old * a.n_types + tn];
                delta = __fsub_rn(delta, j_old);
            } else {
                ++like_old;
            }
            if (ln != nw) {
                const float j_new = small_types ? s_contact[t_new * a.n_types + tn] : a.t.contact[t_new * a.n_types + tn];
                delta = __fadd_rn(delta, j_new);
            } else {
                ++like_new;
            }
        }

        if (old != 0) {
            // The per-colour guard: the losing cell must keep a site of
            // another colour. A like neighbour is one, since every neighbour
            // of a target is of another colour.
            if (like_old == 0) {
                int other = 0;
                for (int c = 0; c < a.g.ncol; ++c)
                    if (c != a.colour) other += a.vol_by_colour[(size_t)old * a.g.ncol + c];
                if (other == 0) continue;
            }
            if (a.g.ring_n > 0 && a.t.connected[t_old]) {
                uint32_t present = 0;
                for (int k = 0; k < a.g.ring_n; ++k)
                    if (win[wc + s_wring[k]] == old) present |= 1u << k;
                if (!one_piece(present, a.g.adjacency)) continue;
            }
        }
        const int ds_old = 2 * like_old - NOFF;
        const int ds_new = NOFF - 2 * like_new;

        int vol_old = 0, surf_old = 0, vol_new = 0, surf_new = 0;
        if (old != 0) {
            int dv, ds;
            unpack_delta(a.vs_prev[old], dv, ds);
            const int2 b = a.vs_base[old];
            vol_old = b.x + dv;
            surf_old = b.y + ds;
        }
        if (nw != 0) {
            int dv, ds;
            unpack_delta(a.vs_prev[nw], dv, ds);
            const int2 b = a.vs_base[nw];
            vol_new = b.x + dv;
            surf_new = b.y + ds;
        }
        if (old != 0) {
            const float lam = a.t.lambda_volume[t_old];
            if (lam != 0.0f) {
                const float v = (float)vol_old, tv = a.t.target_volume[t_old];
                const float p = __fsub_rn(__fsub_rn(v, 1.0f), tv), q = __fsub_rn(v, tv);
                delta = __fadd_rn(delta, __fmul_rn(lam, __fsub_rn(__fmul_rn(p, p), __fmul_rn(q, q))));
            }
        }
        if (nw != 0) {
            const float lam = a.t.lambda_volume[t_new];
            if (lam != 0.0f) {
                const float v = (float)vol_new, tv = a.t.target_volume[t_new];
                const float p = __fsub_rn(__fadd_rn(v, 1.0f), tv), q = __fsub_rn(v, tv);
                delta = __fadd_rn(delta, __fmul_rn(lam, __fsub_rn(__fmul_rn(p, p), __fmul_rn(q, q))));
            }
        }
        if (old != 0) {
            const float lam = a.t.lambda_surface[t_old];
            if (lam != 0.0f) {
                const float sv = (float)surf_old, ts = a.t.target_surface[t_old];
                const float after = __fadd_rn(sv, (float)ds_old);
                const float p = __fsub_rn(after, ts), q = __fsub_rn(sv, ts);
                delta = __fadd_rn(delta, __fmul_rn(lam, __fsub_rn(__fmul_rn(p, p), __fmul_rn(q, q))));
            }
        }
        if (nw != 0) {
            const float lam = a.t.lambda_surface[t_new];
            if (lam != 0.0f) {
                const float sv = (float)surf_new, ts = a.t.target_surface[t_new];
                const float after = __fadd_rn(sv, (float)ds_new);
                const float p = __fsub_rn(after, ts), q = __fsub_rn(sv, ts);
                delta = __fadd_rn(delta, __fmul_rn(lam, __fsub_rn(__fmul_rn(p, p), __fmul_rn(q, q))));
            }
        }

        long long terms_old[NM], terms_new[NM];
        if (a.tracks) {
            if (old != 0) {
                const int *an = &a.anchor[(size_t)old * 4];
                site_terms<DIM>(fold_int(x - an[0], W), fold_int(y - an[1], H), fold_int(z - an[2], D), terms_old);
            }
            if (nw != 0) {
                const int *an = &a.anchor[(size_t)nw * 4];
                site_terms<DIM>(fold_int(x - an[0], W), fold_int(y - an[1], H), fold_int(z - an[2], D), terms_new);
            }
            if (a.has_length) {
                if (old != 0 && a.t.lambda_length[t_old] != 0.0)
                    delta = __fadd_rn(delta, (float)length_delta<DIM>(a, t_old, old, vol_old, terms_old, -1));
                if (nw != 0 && a.t.lambda_length[t_new] != 0.0)
                    delta = __fadd_rn(delta, (float)length_delta<DIM>(a, t_new, nw, vol_new, terms_new, 1));
            }
        }

        if (a.has_chemotaxis && nw != 0) {
            const int ox = a.g.off[pick][0], oy = a.g.off[pick][1], oz = a.g.off[pick][2];
            const uint32_t source =
                (uint32_t)(((size_t)wrap(z + oz, D) * H + wrap(y + oy, H)) * W + wrap(x + ox, W));
            for (int s = 0; s < a.n_species; ++s) {
                const float lam = a.t.chemotaxis[t_new * a.n_species + s];
                if (lam == 0.0f) continue;
                const float *f = a.fields[s];
                delta = __fsub_rn(delta, __fmul_rn(lam, __fsub_rn(f[target], f[source])));
            }
        }

        bool accept = delta <= 0.0f;
        if (!accept) {
            const float u = to_f32(draw(a.key_accept, target));
            accept = u < metropolis_exp(__fdiv_rn(-delta, a.temperature));
        }
        if (!accept) continue;

        a.labels[target] = nw;
        if (old != 0) {
            atomicAdd(&a.vs_cur[old], pack_delta(-1, ds_old));
            atomicSub(&a.vol_by_colour[(size_t)old * a.g.ncol + a.colour], 1);
            if (a.tracks)
#pragma unroll
                for (int k = 0; k < NM; ++k)
                    atomicAdd(&a.mom_cur[(size_t)old * NM + k], (unsigned long long)(-terms_old[k]));
        }
        if (nw != 0) {
            atomicAdd(&a.vs_cur[nw], pack_delta(1, ds_new));
            atomicAdd(&a.vol_by_colour[(size_t)nw * a.g.ncol + a.colour], 1);
            if (a.tracks)
#pragma unroll
                for (int k = 0; k < NM; ++k)
                    atomicAdd(&a.mom_cur[(size_t)nw * NM + k], (unsigned long long)terms_new[k]);
        }
    }
}

template <int DIM, int NOFF>
static cudaError_t launch(const SweepLaunch &a, cudaStream_t stream) {
    using T = Tile<DIM>;
    const int tiles = ((a.g.w + T::TX - 1) / T::TX) * ((a.g.h + T::TY - 1) / T::TY) *
                      (DIM == 3 ? (a.g.d + T::TZ - 1) / T::TZ : 1);
    CUtensorMap tmap;
    if (a.use_tma && a.tensor_map)
        tmap = *static_cast<const CUtensorMap *>(a.tensor_map);
    else
        memset(&tmap, 0, sizeof tmap);
    sweep_kernel<DIM, NOFF><<<tiles, kSweepThreads, 0, stream>>>(a, tmap);
    return cudaGetLastError();
}

cudaError_t launch_sweep(const SweepLaunch &a, cudaStream_t stream) {
    if (a.g.dim == 2) {
        if (a.g.n_off == 4) return launch<2, 4>(a, stream);
        if (a.g.n_off == 8) return launch<2, 8>(a, stream);
    } else {
        if (a.g.n_off == 6) return launch<3, 6>(a, stream);
        if (a.g.n_off == 18) return launch<3, 18>(a, stream);
        if (a.g.n_off == 26) return launch<3, 26>(a, stream);
    }
    return cudaErrorInvalidValue;
}

// The tensor map a sweep's interior tiles copy their window with: the
// lattice as a 2D or 3D uint32 array, a box of the tile plus its halo.
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
