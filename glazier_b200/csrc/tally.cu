// Per-cell tallies from the lattice: the recount, the settle that folds the
// pending deltas into the base, and the medium's own counts.
//
// The recount replaces `recount` (glazier-cuda/src/lib.rs:144-172) and the
// host-side `assemble` (glazier-core/src/cpu.rs:178-217) that seeds every
// counter before a run. Besides volume and surface it counts each cell's
// sites per checkerboard colour (the sweep's guard reads these), fixes each
// cell's anchor at its first site in scan order (the frame moments.rs
// unwraps a cell in), and accumulates the exact int64 moment sums about it.

#include <climits>

#include "device.cuh"
#include "engine.h"
#include "neighbours.cuh"

namespace glz {

// A lattice holds fewer than 2^31 sites, so 32-bit division suffices.
__device__ __forceinline__ void coords_of(const Geometry &g, size_t i, int &x, int &y, int &z) {
    const uint32_t s = (uint32_t)i;
    const uint32_t row = udiv(g.div_w, s);
    const uint32_t plane = udiv(g.div_h, row);
    x = (int)(s - row * (uint32_t)g.w);
    y = (int)(row - plane * (uint32_t)g.h);
    z = (int)plane;
}

// The label count a recount covers: the live count in device memory for a
// population model, else the launch's.
__device__ __forceinline__ int recount_labels(const RecountLaunch &a) { return a.n_live ? *a.n_live : a.n_labels; }

// Whether a conditional recount runs (the population step's event flag).
__device__ __forceinline__ bool recount_runs(const RecountLaunch &a) { return !a.when || *a.when != 0; }

// The tallies a recount rebuilds, zeroed for the live labels (a conditional
// recount's stand-in for its memsets).
__global__ void clear_tallies_kernel(const __grid_constant__ RecountLaunch a) {
    if (!recount_runs(a)) return;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= recount_labels(a)) return;
    a.vs_base[l] = make_int2(0, 0);
    for (int c = 0; c < a.g.ncol; ++c) a.vol_by_colour[(size_t)l * a.g.ncol + c] = 0;
    for (int k = 0; k < 3; ++k) a.vs_delta[k][l] = 0;
    if (a.tracks)
        for (int j = 0; j < a.g.nm; ++j) {
            a.mom_base[(size_t)l * a.g.nm + j] = 0;
            for (int k = 0; k < 3; ++k) a.mom_delta[k][(size_t)l * a.g.nm + j] = 0;
        }
}

__global__ void fill_anchor_kernel(const __grid_constant__ RecountLaunch a) {
    if (!recount_runs(a)) return;
    int *anchor = a.anchor;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= recount_labels(a)) return;
    anchor[4 * l + 0] = 0;
    anchor[4 * l + 1] = 0;
    anchor[4 * l + 2] = 0;
    anchor[4 * l + 3] = INT_MAX;
}

// Unlike-label neighbours of site i (label l) at (x, y, z), in 32-bit index
// arithmetic: the wrapped coordinates one step either side are formed once
// and each offset picks among them. A neighbour that wraps onto the site
// itself is not a bond.
__device__ __forceinline__ int unlike_neighbours(const Geometry &g, const uint32_t *labels, uint32_t i, uint32_t l,
                                                 int x, int y, int z) {
    const int W = g.w, H = g.h, D = g.d;
    const int xm = x == 0 ? W - 1 : x - 1, xp = x == W - 1 ? 0 : x + 1;
    const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
    const int zm = z == 0 ? D - 1 : z - 1, zp = z == D - 1 ? 0 : z + 1;
    int bonds = 0;
    for (int k = 0; k < g.n_off; ++k) {
        const int dx = g.off[k][0], dy = g.off[k][1], dz = g.off[k][2];
        const uint32_t nx = (uint32_t)(dx < 0 ? xm : (dx > 0 ? xp : x));
        const uint32_t ny = (uint32_t)(dy < 0 ? ym : (dy > 0 ? yp : y));
        const uint32_t nz = (uint32_t)(dz < 0 ? zm : (dz > 0 ? zp : z));
        const uint32_t n = (nz * (uint32_t)H + ny) * (uint32_t)W + nx;
        bonds += n != i && labels[n] != l;
    }
    return bonds;
}

// Volume, unlike-bond surface, per-colour volume and first site of every
// label. Blocks run along lattice rows (x across threads, one row per block
// row), so a warp holds 32 consecutive sites of one row and a cell usually
// covers a run of lanes: each run adds its counts through its first lane
// (whose site is also the run's first), one atomic per run, not per site.
// Along a row only x changes, so a run's sites alternate between two
// colours, starting with its first lane's. A label that comes back later in
// the warp starts another run. Neighbour addresses are the compile-time
// neighbourhood's offsets over the wrapped rows and columns either side.
template <int DIM, int NOFF>
__global__ void recount_counts_kernel(const __grid_constant__ RecountLaunch a) {
    constexpr uint32_t kNone = 0xffffffffu;
    if (!recount_runs(a)) return;
    const uint32_t n_labels = (uint32_t)recount_labels(a);
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const int lane = threadIdx.x & 31;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int xm = x == 0 ? W - 1 : x - 1, xp = x == W - 1 ? 0 : x + 1;
    for (int row = blockIdx.y; row < H * D; row += gridDim.y) {
        const int y = row % H, z = row / H;
        const uint32_t i = (uint32_t)row * (uint32_t)W + (uint32_t)x;
        uint32_t l = x < W ? a.labels[i] : kNone;
        if (l != kNone && l >= n_labels) {
            atomicExch(a.error_flag, 2);
            l = kNone;
        }
        int bonds = 0;
        if (l != kNone) {
            const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
            const int zm = z == 0 ? D - 1 : z - 1, zp = z == D - 1 ? 0 : z + 1;
#pragma unroll
            for (int k = 0; k < NOFF; ++k) {
                const int dx = neighbour_offset<DIM, NOFF>(k, 0), dy = neighbour_offset<DIM, NOFF>(k, 1),
                          dz = neighbour_offset<DIM, NOFF>(k, 2);
                const uint32_t nx = (uint32_t)(dx < 0 ? xm : (dx > 0 ? xp : x));
                const uint32_t ny = (uint32_t)(dy < 0 ? ym : (dy > 0 ? yp : y));
                const uint32_t nz = (uint32_t)(dz < 0 ? zm : (dz > 0 ? zp : z));
                const uint32_t n = (nz * (uint32_t)H + ny) * (uint32_t)W + nx;
                // a neighbour that wraps onto the site itself is not a bond
                bonds += n != i && a.labels[n] != l;
            }
        }
        const int colour = (x & 1) | ((y & 1) << 1) | (DIM == 3 ? ((z & 1) << 2) : 0);
        const unsigned full = 0xffffffffu;
        const uint32_t before = __shfl_up_sync(full, l, 1);
        const bool head = lane == 0 || l != before;
        const unsigned heads = __ballot_sync(full, head);
        // inclusive prefix sum of the bond counts over the warp
        int scan = bonds;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(full, scan, o);
            if (lane >= o) scan += v;
        }
        const unsigned later = heads & ~(full >> (31 - lane));  // heads after this lane
        const int last = later ? __ffs(later) - 2 : 31;          // this lane's run ends here
        const int scan_last = __shfl_sync(full, scan, last);
        if (head && l != kNone) {
            const int len = last - lane + 1;
            const int run_bonds = scan_last - scan + bonds;
            atomicAdd(&a.vs_base[l].x, len);
            if (run_bonds) atomicAdd(&a.vs_base[l].y, run_bonds);
            atomicMin(&a.anchor[4 * (size_t)l + 3], (int)i);
            int *by_colour = &a.vol_by_colour[(size_t)l * a.g.ncol];
            atomicAdd(&by_colour[colour], (len + 1) / 2);
            if (len > 1) atomicAdd(&by_colour[colour ^ 1], len / 2);
        }
    }
}

template <int DIM, int NOFF>
static cudaError_t launch_counts(const RecountLaunch &a, cudaStream_t stream) {
    for (int k = 0; k < NOFF; ++k)
        for (int axis = 0; axis < 3; ++axis)
            if (a.g.off[k][axis] != neighbour_offset<DIM, NOFF>(k, axis)) return cudaErrorInvalidValue;
    const int bx = a.g.w >= 256 ? 256 : (a.g.w + 31) / 32 * 32;
    const int rows = a.g.h * a.g.d;
    const dim3 grid((unsigned)((a.g.w + bx - 1) / bx), (unsigned)(rows < 65535 ? rows : 65535));
    recount_counts_kernel<DIM, NOFF><<<grid, bx, 0, stream>>>(a);
    return cudaGetLastError();
}

static cudaError_t launch_counts_any(const RecountLaunch &a, cudaStream_t stream) {
    if (a.g.dim == 2) {
        if (a.g.n_off == 4) return launch_counts<2, 4>(a, stream);
        if (a.g.n_off == 8) return launch_counts<2, 8>(a, stream);
    } else {
        if (a.g.n_off == 6) return launch_counts<3, 6>(a, stream);
        if (a.g.n_off == 18) return launch_counts<3, 18>(a, stream);
        if (a.g.n_off == 26) return launch_counts<3, 26>(a, stream);
    }
    return cudaErrorInvalidValue;
}

__global__ void recount_anchor_kernel(const __grid_constant__ RecountLaunch a) {
    if (!recount_runs(a)) return;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= recount_labels(a)) return;
    const int first = a.anchor[4 * l + 3];
    if (first == INT_MAX) return;
    int x, y, z;
    coords_of(a.g, (size_t)first, x, y, z);
    a.anchor[4 * l + 0] = x;
    a.anchor[4 * l + 1] = y;
    a.anchor[4 * l + 2] = z;
}

__global__ void recount_moments_kernel(const __grid_constant__ RecountLaunch a) {
    if (!recount_runs(a)) return;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const uint32_t l = a.labels[i];
    if (l == 0 || l >= (uint32_t)recount_labels(a)) return;
    int x, y, z;
    coords_of(a.g, i, x, y, z);
    const int *an = &a.anchor[4 * (size_t)l];
    const long long ux = fold_int(x - an[0], a.g.w);
    const long long uy = fold_int(y - an[1], a.g.h);
    const long long uz = fold_int(z - an[2], a.g.d);
    unsigned long long *m = reinterpret_cast<unsigned long long *>(&a.mom_base[(size_t)l * a.g.nm]);
    if (a.g.dim == 2) {
        atomicAdd(&m[0], (unsigned long long)ux);
        atomicAdd(&m[1], (unsigned long long)uy);
        atomicAdd(&m[2], (unsigned long long)(ux * ux));
        atomicAdd(&m[3], (unsigned long long)(uy * uy));
        atomicAdd(&m[4], (unsigned long long)(ux * uy));
    } else {
        atomicAdd(&m[0], (unsigned long long)ux);
        atomicAdd(&m[1], (unsigned long long)uy);
        atomicAdd(&m[2], (unsigned long long)uz);
        atomicAdd(&m[3], (unsigned long long)(ux * ux));
        atomicAdd(&m[4], (unsigned long long)(uy * uy));
        atomicAdd(&m[5], (unsigned long long)(uz * uz));
        atomicAdd(&m[6], (unsigned long long)(ux * uy));
        atomicAdd(&m[7], (unsigned long long)(ux * uz));
        atomicAdd(&m[8], (unsigned long long)(uy * uz));
    }
    if (a.nematic) {
        const int g = a.g.dim == 2 ? 5 : 9;
        atomicAdd(&m[g], (unsigned long long)nematic_fixed(a.nematic[2 * i]));
        atomicAdd(&m[g + 1], (unsigned long long)nematic_fixed(a.nematic[2 * i + 1]));
    }
}

cudaError_t launch_recount(const RecountLaunch &a, cudaStream_t stream) {
    const size_t n = (size_t)a.n_labels;  // the count, or the capacity with n_live
    const int lb = (int)((n + 255) / 256);
    const int sb = (a.g.sites + 255) / 256;
    if (a.n_live || a.when) {
        clear_tallies_kernel<<<lb, 256, 0, stream>>>(a);
    } else {
        cudaError_t e;
        if ((e = cudaMemsetAsync(a.vs_base, 0, n * sizeof(int2), stream))) return e;
        if ((e = cudaMemsetAsync(a.vol_by_colour, 0, n * a.g.ncol * sizeof(int), stream))) return e;
        for (int k = 0; k < 3; ++k)
            if ((e = cudaMemsetAsync(a.vs_delta[k], 0, n * sizeof(long long), stream))) return e;
        if (a.tracks) {
            if ((e = cudaMemsetAsync(a.mom_base, 0, n * a.g.nm * sizeof(long long), stream))) return e;
            for (int k = 0; k < 3; ++k)
                if ((e = cudaMemsetAsync(a.mom_delta[k], 0, n * a.g.nm * sizeof(long long), stream))) return e;
        }
    }
    fill_anchor_kernel<<<lb, 256, 0, stream>>>(a);
    if (cudaError_t e = launch_counts_any(a, stream)) return e;
    recount_anchor_kernel<<<lb, 256, 0, stream>>>(a);
    if (a.tracks) recount_moments_kernel<<<sb, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

__device__ __forceinline__ void settle_one(int l, int2 *vs_base, long long *vs_delta, long long *mom_base,
                                           long long *mom_delta, int nm, int tracks);

__global__ void settle_kernel(int2 *vs_base, long long *vs_delta, long long *mom_base, long long *mom_delta, int nm,
                              int n, int tracks, const int *n_live) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (n_live ? *n_live : n)) return;
    settle_one(l, vs_base, vs_delta, mom_base, mom_delta, nm, tracks);
}

// The slots at the end of a clocked step: pass number clock->pass + ncol.
__global__ void settle_clocked_kernel(const Tallies t, int nm, int n, int tracks, const int *n_live,
                                      const EngineClock *clock, int ncol) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (n_live ? *n_live : n)) return;
    const long long p = clock->pass + ncol;
    settle_one(l, t.vs_base[p % 2], t.vs_delta[(p + 2) % 3], t.mom_base[p % 2], t.mom_delta[(p + 2) % 3], nm, tracks);
}

__global__ void engine_clock_kernel(EngineClock *clock, int ncol) {
    clock->step += 1;
    clock->pass += ncol;
    clock->field_cur ^= clock->field_flip;
}

cudaError_t launch_settle_clocked(const Tallies &t, int nm, int n_labels, int tracks, const int *n_live,
                                  const EngineClock *clock, int ncol, cudaStream_t stream) {
    if (n_labels <= 0) return cudaSuccess;
    settle_clocked_kernel<<<(n_labels + 255) / 256, 256, 0, stream>>>(t, nm, n_labels, tracks, n_live, clock, ncol);
    return cudaGetLastError();
}

cudaError_t launch_engine_clock_advance(EngineClock *clock, int ncol, cudaStream_t stream) {
    engine_clock_kernel<<<1, 1, 0, stream>>>(clock, ncol);
    return cudaGetLastError();
}

__device__ __forceinline__ void settle_one(int l, int2 *vs_base, long long *vs_delta, long long *mom_base,
                                           long long *mom_delta, int nm, int tracks) {
    int dv, ds;
    unpack_delta(vs_delta[l], dv, ds);
    int2 b = vs_base[l];
    vs_base[l] = make_int2(b.x + dv, b.y + ds);
    vs_delta[l] = 0;
    if (tracks)
        for (int k = 0; k < nm; ++k) {
            mom_base[(size_t)l * nm + k] += mom_delta[(size_t)l * nm + k];
            mom_delta[(size_t)l * nm + k] = 0;
        }
}

cudaError_t launch_settle(int2 *vs_base, long long *vs_delta, long long *mom_base, long long *mom_delta, int nm,
                          int n_labels, int tracks, const int *n_live, cudaStream_t stream) {
    if (n_labels <= 0) return cudaSuccess;
    settle_kernel<<<(n_labels + 255) / 256, 256, 0, stream>>>(vs_base, vs_delta, mom_base, mom_delta, nm, n_labels,
                                                              tracks, n_live);
    return cudaGetLastError();
}

__global__ void medium_count_kernel(const __grid_constant__ Geometry g, const uint32_t *labels,
                                    unsigned long long *out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long sites = 0, bonds = 0;
    if (i < (size_t)g.sites && labels[i] == 0) {
        int x, y, z;
        coords_of(g, i, x, y, z);
        sites = 1;
        bonds = (unsigned long long)unlike_neighbours(g, labels, (uint32_t)i, 0u, x, y, z);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sites += __shfl_down_sync(0xffffffffu, sites, o);
        bonds += __shfl_down_sync(0xffffffffu, bonds, o);
    }
    if ((threadIdx.x & 31) == 0 && (sites || bonds)) {
        atomicAdd(&out[0], sites);
        atomicAdd(&out[1], bonds);
    }
}

cudaError_t launch_medium_count(const Geometry &g, const uint32_t *labels, unsigned long long *out,
                                cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), stream);
    if (e) return e;
    medium_count_kernel<<<(g.sites + 255) / 256, 256, 0, stream>>>(g, labels, out);
    return cudaGetLastError();
}

}  // namespace glz
