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
// Exchange reads only its own species, so running it right after that
// species' last sub-step is the reference's order.

#include "device.cuh"
#include "engine.h"

namespace glz {

template <int DIM>
__global__ void __launch_bounds__(256) field_round_kernel(const __grid_constant__ FieldLaunch a) {
    const int W = a.g.w, H = a.g.h, D = a.g.d;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    const int x = (int)(i % W);
    const int y = (int)((i / W) % H);
    const int z = DIM == 3 ? (int)(i / ((size_t)W * H)) : 0;
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
    for (int s = 0; s < a.n_species; ++s) {
        if (!a.active[s]) continue;
        const float *__restrict__ u = a.in[s];
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
                const uint32_t l = a.labels[i];
                type = l == 0 ? 0x7fffffff : a.cell_type[l];
            }
            if (type != 0x7fffffff) {
                v = __fadd_rn(v, a.secretion[type * a.n_species + s]);
                v = __fsub_rn(v, __fmul_rn(a.uptake[type * a.n_species + s], v));
                v = v < 0.0f ? 0.0f : v;
            }
        }
        a.out[s][i] = v;
    }
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
