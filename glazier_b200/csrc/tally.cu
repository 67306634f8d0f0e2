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

namespace glz {

__device__ __forceinline__ void coords_of(const Geometry &g, size_t i, int &x, int &y, int &z) {
    x = (int)(i % g.w);
    y = (int)((i / g.w) % g.h);
    z = (int)(i / ((size_t)g.w * g.h));
}

__global__ void fill_anchor_kernel(int *anchor, int n) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    anchor[4 * l + 0] = 0;
    anchor[4 * l + 1] = 0;
    anchor[4 * l + 2] = 0;
    anchor[4 * l + 3] = INT_MAX;
}

__global__ void recount_counts_kernel(const __grid_constant__ RecountLaunch a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const uint32_t l = a.labels[i];
    if (l >= (uint32_t)a.n_labels) {
        atomicExch(a.error_flag, 2);
        return;
    }
    int x, y, z;
    coords_of(a.g, i, x, y, z);
    int bonds = 0;
    for (int k = 0; k < a.g.n_off; ++k) {
        const size_t n = ((size_t)wrap(z + a.g.off[k][2], a.g.d) * a.g.h + wrap(y + a.g.off[k][1], a.g.h)) * a.g.w +
                         wrap(x + a.g.off[k][0], a.g.w);
        if (n != i && a.labels[n] != l) ++bonds;
    }
    const int colour = (x & 1) | ((y & 1) << 1) | (a.g.dim == 3 ? ((z & 1) << 2) : 0);
    atomicAdd(&a.vs_base[l].x, 1);
    if (bonds) atomicAdd(&a.vs_base[l].y, bonds);
    atomicAdd(&a.vol_by_colour[(size_t)l * a.g.ncol + colour], 1);
    atomicMin(&a.anchor[4 * (size_t)l + 3], (int)i);
}

__global__ void recount_anchor_kernel(const __grid_constant__ RecountLaunch a) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.n_labels) return;
    const int first = a.anchor[4 * l + 3];
    if (first == INT_MAX) return;
    int x, y, z;
    coords_of(a.g, (size_t)first, x, y, z);
    a.anchor[4 * l + 0] = x;
    a.anchor[4 * l + 1] = y;
    a.anchor[4 * l + 2] = z;
}

__global__ void recount_moments_kernel(const __grid_constant__ RecountLaunch a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const uint32_t l = a.labels[i];
    if (l == 0 || l >= (uint32_t)a.n_labels) return;
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
}

cudaError_t launch_recount(const RecountLaunch &a, cudaStream_t stream) {
    const size_t n = (size_t)a.n_labels;
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
    const int lb = (int)((n + 255) / 256);
    const int sb = (a.g.sites + 255) / 256;
    fill_anchor_kernel<<<lb, 256, 0, stream>>>(a.anchor, (int)n);
    recount_counts_kernel<<<sb, 256, 0, stream>>>(a);
    recount_anchor_kernel<<<lb, 256, 0, stream>>>(a);
    if (a.tracks) recount_moments_kernel<<<sb, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

__global__ void settle_kernel(int2 *vs_base, long long *vs_delta, long long *mom_base, long long *mom_delta, int nm,
                              int n, int tracks) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
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
                          int n_labels, int tracks, cudaStream_t stream) {
    if (n_labels <= 0) return cudaSuccess;
    settle_kernel<<<(n_labels + 255) / 256, 256, 0, stream>>>(vs_base, vs_delta, mom_base, mom_delta, nm, n_labels,
                                                              tracks);
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
        for (int k = 0; k < g.n_off; ++k) {
            const size_t n =
                ((size_t)wrap(z + g.off[k][2], g.d) * g.h + wrap(y + g.off[k][1], g.h)) * g.w + wrap(x + g.off[k][0], g.w);
            if (n != i && labels[n] != 0) ++bonds;
        }
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
