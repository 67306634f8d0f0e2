// The chemical-field step: FTCS diffusion and decay, with secretion and
// uptake by the cell that owns each site folded into each species' last
// sub-step.
//
// Replaces `field_diffuse` and `field_exchange` (glazier-cuda/src/lib.rs
// 314-363) and their driver `run_fields` (lib.rs:1147-1189). One launch runs
// one sub-step round for every species that still has a sub-step left, so a
// model whose species all take one sub-step (the common case) reads its
// labels and every species once per Monte Carlo step:
//   out = u + d (sum of faces - faces u) - decay u          (field.rs:110-130)
//   on owned sites: v = out + sec; v -= upt v; v = max(v, 0) (field.rs:133-149)
// With an infection rule set (glz_gpu_set_infection, an extension), the
// uptake upt v of the rule's species by cells of the rule's type is summed
// per cell in fixed point, and infection_kernel switches the cells whose sum
// has reached the threshold.
// Exchange reads only its own species, so running it right after that
// species' last sub-step is the reference's order.

#include "device.cuh"
#include "engine.h"

namespace glz {

// Add each lane's `amount` into dose[label] through the first lane of each
// run of equal labels in the warp: one atomic per run. Every lane of the warp
// takes part; a lane with nothing to add passes label kNoDose.
constexpr uint32_t kNoDose = 0xffffffffu;

__device__ __forceinline__ void add_dose(unsigned long long *dose, uint32_t label, long long amount) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t before = __shfl_up_sync(full, label, 1);
    const bool head = lane == 0 || label != before;
    const unsigned heads = __ballot_sync(full, head);
    long long scan = amount;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(full, scan, o);
        if (lane >= o) scan += v;
    }
    const unsigned later = heads & ~(full >> (31 - lane));
    const int last = later ? __ffs(later) - 2 : 31;
    const long long scan_last = __shfl_sync(full, scan, last);
    if (head && label != kNoDose) {
        const long long run = scan_last - scan + amount;
        if (run != 0) atomicAdd(&dose[label], (unsigned long long)run);
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) field_round_kernel(const __grid_constant__ FieldLaunch a) {
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < (size_t)a.g.sites;
    // with an infection rule every lane stays for the warp's dose sums
    if (!in && a.infect_species < 0) return;
    const size_t c = in ? i : 0;
    // fewer than 2^31 sites: 32-bit quotients by the geometry's dividers
    const uint32_t qw = udiv(a.g.div_w, (uint32_t)c), plane = udiv(a.g.div_h, qw);
    const int x = (int)((uint32_t)c - qw * (uint32_t)W);
    const int y = (int)(qw - plane * (uint32_t)H);
    const int z = DIM == 3 ? (int)plane : 0;
    const size_t row = ((size_t)z * H + y) * W;
    const size_t xm = row + (x == 0 ? W - 1 : x - 1);
    const size_t xp = row + (x == W - 1 ? 0 : x + 1);
    const size_t ym = ((size_t)z * H + (y == 0 ? H - 1 : y - 1)) * W + x;
    const size_t yp = ((size_t)z * H + (y == H - 1 ? 0 : y + 1)) * W + x;
    size_t zm = 0, zp = 0;
    if (DIM == 3) {
        zm = ((size_t)(z == 0 ? D - 1 : z - 1) * H + y) * W + x;
        zp = ((size_t)(z == D - 1 ? 0 : z + 1) * H + y) * W + x;
    }
    const float faces = DIM == 3 ? 6.0f : 4.0f;
    int type = -1;
    uint32_t label = 0;
    const unsigned cur = a.clock ? a.clock->field_cur : 0u;
    for (int s = 0; s < a.n_species; ++s) {
        if (!a.active[s]) continue;
        long long taken = 0;  // this site's uptake of the infection species, fixed point
        // clocked: a species active in this round has flipped once a round before it
        const unsigned from = ((cur >> s) & 1u) ^ ((unsigned)a.round & 1u);
        float *const out = a.clock ? a.field_buf + ((size_t)2 * s + (from ^ 1u)) * (size_t)a.g.sites : a.out[s];
        if (in) {
            const float *__restrict__ u =
                a.clock ? a.field_buf + ((size_t)2 * s + from) * (size_t)a.g.sites : a.in[s];
            const float here = u[i];
            float sum = u[xm];
            sum = __fadd_rn(sum, u[xp]);
            sum = __fadd_rn(sum, u[ym]);
            sum = __fadd_rn(sum, u[yp]);
            if (DIM == 3) {
                sum = __fadd_rn(sum, u[zm]);
                sum = __fadd_rn(sum, u[zp]);
            }
            float v = __fsub_rn(__fadd_rn(here, __fmul_rn(a.d[s], __fsub_rn(sum, __fmul_rn(faces, here)))),
                                __fmul_rn(a.decay[s], here));
            if (a.last[s]) {
                if (type < 0) {
                    label = a.labels[i];
                    type = label == 0 ? 0x7fffffff : a.cell_type[label];
                }
                if (type != 0x7fffffff) {
                    v = __fadd_rn(v, a.secretion[type * a.n_species + s]);
                    const float amount = __fmul_rn(a.uptake[type * a.n_species + s], v);
                    if (s == a.infect_species && type == a.infect_from)
                        taken = __float2ll_rn(__fmul_rn(amount, kDoseScale));
                    v = __fsub_rn(v, amount);
                    v = v < 0.0f ? 0.0f : v;
                }
            }
            out[i] = v;
        }
        if (s == a.infect_species && a.last[s])
            add_dose(a.dose, in && type == a.infect_from ? label : kNoDose, taken);
    }
}

__global__ void infection_kernel(uint8_t *cell_type, const unsigned long long *dose, int n_labels, int from, int to,
                                 long long threshold, const int *n_live) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = n_live ? *n_live : n_labels;
    if (l == 0 || l >= n) return;
    if (cell_type[l] == from && (long long)dose[l] >= threshold) cell_type[l] = (uint8_t)to;
}

cudaError_t launch_infection(uint8_t *cell_type, const unsigned long long *dose, int n_labels, int from, int to,
                             long long threshold, const int *n_live, cudaStream_t stream) {
    infection_kernel<<<(n_labels + 255) / 256, 256, 0, stream>>>(cell_type, dose, n_labels, from, to, threshold,
                                                                 n_live);
    return cudaGetLastError();
}

cudaError_t launch_field_round(const FieldLaunch &a, cudaStream_t stream) {
    const int blocks = (a.g.sites + 255) / 256;
    if (a.g.dim == 2)
        field_round_kernel<2><<<blocks, 256, 0, stream>>>(a);
    else
        field_round_kernel<3><<<blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace glz
