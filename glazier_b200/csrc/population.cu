// Division and death, planned per cell on the device.
//
// Replaces `run_population` (glazier-cuda/src/lib.rs:1362-1461) and its
// kernels `cell_circular_sums`, `cell_moments` and `apply_population`
// (lib.rs:66-142), which took five host round trips every Monte Carlo step.
// Here every decision is made on the device from the exact moment sums:
//   plan    per cell: a live cell at or past its division volume (and of at
//           least four sites, cpu.rs:681) plans a cut through its centroid
//           perpendicular to its major axis (power iteration on the
//           covariance, moments.rs:165-186); any other live cell of a type
//           with a death rate dies when its counter-hash draw falls under the
//           rate (the reference's `else if`, lib.rs:1406-1423).
//   count   per site: how many sites each planned cut would move.
//   decide  one CTA, in label order: a cut that moves nothing or everything
//           is no division (cpu.rs:697-703); the rest take daughter labels
//           n_labels, n_labels + 1, ... in their mothers' order, a prefix sum
//           over the compacted list of dividing cells. The live label count
//           stays in device memory: decide reads it and adds the daughters,
//           so no host read stands between steps.
//   apply   per site: death to medium, the far side of a cut to the daughter.
// The engine then recounts every tally from the lattice (cpu.rs:649-653),
// a recount whose kernels return at once when decide found no event.

#include "device.cuh"
#include "engine.h"

namespace glz {

__device__ __forceinline__ double along_cut(const Geometry &g, const int *anchor, const double *plan, uint32_t l,
                                            size_t i) {
    const int x = (int)(i % g.w), y = (int)((i / g.w) % g.h), z = (int)(i / ((size_t)g.w * g.h));
    const int *an = &anchor[4 * (size_t)l];
    const double ux = (double)fold_int(x - an[0], g.w);
    const double uy = (double)fold_int(y - an[1], g.h);
    const double uz = (double)fold_int(z - an[2], g.d);
    const double *p = &plan[6 * (size_t)l];
    return (ux - p[0]) * p[3] + (uy - p[1]) * p[4] + (uz - p[2]) * p[5];
}

__global__ void plan_kernel(const __grid_constant__ PopulationLaunch a) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= *a.n_live) return;
    a.moved[l] = 0;
    a.mode[l] = 0;
    if (l == 0) return;
    const int v = a.vs_base[l].x;
    if (v <= 0) return;
    const int t = a.cell_type_in[l];
    const double div_vol = a.t.division_volume[t];
    if (div_vol > 0.0 && (double)v >= div_vol && v >= 4) {
        const long long *m = &a.mom_base[(size_t)l * a.g.nm];
        const double dn = (double)v;
        double c[3][3], mean[3];
        if (a.g.dim == 2) {
            mean[0] = (double)m[0] / dn;
            mean[1] = (double)m[1] / dn;
            mean[2] = 0.0;
            c[0][0] = (double)m[2] / dn - mean[0] * mean[0];
            c[1][1] = (double)m[3] / dn - mean[1] * mean[1];
            c[0][1] = c[1][0] = (double)m[4] / dn - mean[0] * mean[1];
            c[2][2] = c[0][2] = c[2][0] = c[1][2] = c[2][1] = 0.0;
        } else {
            mean[0] = (double)m[0] / dn;
            mean[1] = (double)m[1] / dn;
            mean[2] = (double)m[2] / dn;
            c[0][0] = (double)m[3] / dn - mean[0] * mean[0];
            c[1][1] = (double)m[4] / dn - mean[1] * mean[1];
            c[2][2] = (double)m[5] / dn - mean[2] * mean[2];
            c[0][1] = c[1][0] = (double)m[6] / dn - mean[0] * mean[1];
            c[0][2] = c[2][0] = (double)m[7] / dn - mean[0] * mean[2];
            c[1][2] = c[2][1] = (double)m[8] / dn - mean[1] * mean[2];
        }
        double v0 = 1.0, v1 = 0.7, v2 = 0.3;
        bool degenerate = false;
        for (int round = 0; round < 20; ++round) {
            const double w0 = c[0][0] * v0 + c[0][1] * v1 + c[0][2] * v2;
            const double w1 = c[1][0] * v0 + c[1][1] * v1 + c[1][2] * v2;
            const double w2 = c[2][0] * v0 + c[2][1] * v1 + c[2][2] * v2;
            const double norm = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
            if (norm < 1e-15) {
                degenerate = true;
                break;
            }
            v0 = w0 / norm;
            v1 = w1 / norm;
            v2 = w2 / norm;
        }
        if (degenerate) {
            v0 = 1.0;
            v1 = 0.0;
            v2 = 0.0;
        }
        double *p = &a.plan[6 * (size_t)l];
        p[0] = mean[0];
        p[1] = mean[1];
        p[2] = mean[2];
        p[3] = v0;
        p[4] = v1;
        p[5] = v2;
        a.mode[l] = 1;
    } else if (a.t.death_rate[t] > 0.0) {
        const uint64_t key =
            a.clock ? stream_key(a.seed, (int32_t)a.clock->step, kPopulationStream, 0) : a.key_death;
        if (to_f64(draw(key, (uint32_t)l)) < a.t.death_rate[t]) a.mode[l] = 2;
    }
}

__global__ void count_cut_kernel(const __grid_constant__ PopulationLaunch a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const uint32_t l = a.labels[i];
    if (l == 0 || a.mode[l] != 1) return;
    if (along_cut(a.g, a.anchor, a.plan, l, i) > 0.0) atomicAdd(&a.moved[l], 1);
}

// One CTA walks the labels in order and hands each kept division the next
// daughter label: a block-wide prefix sum over the flags of each chunk.
__global__ void __launch_bounds__(1024) decide_kernel(const __grid_constant__ PopulationLaunch a) {
    __shared__ int warp_total[32];
    __shared__ int running;
    __shared__ int any_event;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n_labels = *a.n_live;
    if (tid == 0) {
        running = 0;
        any_event = 0;
    }
    __syncthreads();
    for (int base = 0; base < n_labels; base += blockDim.x) {
        const int l = base + tid;
        int keep = 0;
        if (l < n_labels && l > 0) {
            const unsigned char m = a.mode[l];
            if (m == 1) {
                const int moved = a.moved[l];
                if (moved > 0 && moved < a.vs_base[l].x)
                    keep = 1;
                else
                    a.mode[l] = 0;
            }
            if (keep || m == 2) any_event = 1;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        const int before_in_warp = __popc(ballot & ((1u << lane) - 1u));
        if (lane == 0) warp_total[wid] = __popc(ballot);
        __syncthreads();
        if (wid == 0) {
            int v = lane < (int)(blockDim.x >> 5) ? warp_total[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int up = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += up;
            }
            warp_total[lane] = v;  // inclusive prefix over warps
        }
        __syncthreads();
        const int warp_before = wid == 0 ? 0 : warp_total[wid - 1];
        if (keep) {
            const uint32_t d = (uint32_t)(n_labels + running + warp_before + before_in_warp);
            a.daughter[l] = d;
            a.cell_type_out[d] = a.cell_type_in[l];
        }
        __syncthreads();
        if (tid == 0) running += warp_total[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (tid == 0) {
        a.counters[0] = running;
        a.counters[1] = any_event;
        *a.n_live = n_labels + running;  // every thread read the count before the first barrier
    }
}

__global__ void apply_kernel(const __grid_constant__ PopulationLaunch a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const uint32_t l = a.labels[i];
    if (l == 0) return;
    const unsigned char m = a.mode[l];
    if (m == 2) {
        a.labels[i] = 0;
    } else if (m == 1) {
        if (along_cut(a.g, a.anchor, a.plan, l, i) > 0.0) a.labels[i] = a.daughter[l];
    }
}

cudaError_t launch_population_plan(const PopulationLaunch &a, cudaStream_t stream) {
    plan_kernel<<<(a.cap + 255) / 256, 256, 0, stream>>>(a);
    count_cut_kernel<<<(a.g.sites + 255) / 256, 256, 0, stream>>>(a);
    decide_kernel<<<1, 1024, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_population_apply(const PopulationLaunch &a, cudaStream_t stream) {
    apply_kernel<<<(a.g.sites + 255) / 256, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace glz
