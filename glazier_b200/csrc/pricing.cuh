// Pricing pieces shared by the sweep kernels (sweep.cu, band.cu): the
// volume and surface energy terms, and the shared-memory address helper.
#pragma once

#include <cstdint>

#include "engine.h"

namespace glz {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// The volume and surface parts of a copy's energy change, added to `delta`
// in a fixed order (old cell's volume, new cell's volume, old cell's
// surface, new cell's surface), correctly rounded f32 throughout so a host
// replay gets the same bits; the medium (label 0) has neither term.
//   volume:  lambda ((v -/+ 1 - V_t)^2 - (v - V_t)^2) = lambda (1 -/+ 2 (v - V_t))
//   surface: lambda ((s + ds - S_t)^2 - (s - S_t)^2) = lambda ds (2 (s - S_t) + ds)
template <bool UNIFORM>
__device__ __forceinline__ float size_terms(const SweepLaunch &a, uint32_t old, uint32_t nw, int t_old, int t_new,
                                            int vol_old, int vol_new, int surf_old, int surf_new, int ds_old,
                                            int ds_new, float delta) {
    if (old != 0) {
        const float lam = UNIFORM ? a.u_lambda_volume : a.t.lambda_volume[t_old];
        if (lam != 0.0f) {
            const float e = __fsub_rn((float)vol_old, UNIFORM ? a.u_target_volume : a.t.target_volume[t_old]);
            delta = __fadd_rn(delta, __fmul_rn(lam, __fsub_rn(1.0f, __fmul_rn(2.0f, e))));
        }
    }
    if (nw != 0) {
        const float lam = UNIFORM ? a.u_lambda_volume : a.t.lambda_volume[t_new];
        if (lam != 0.0f) {
            const float e = __fsub_rn((float)vol_new, UNIFORM ? a.u_target_volume : a.t.target_volume[t_new]);
            delta = __fadd_rn(delta, __fmul_rn(lam, __fadd_rn(__fmul_rn(2.0f, e), 1.0f)));
        }
    }
    if (old != 0) {
        const float lam = UNIFORM ? a.u_lambda_surface : a.t.lambda_surface[t_old];
        if (lam != 0.0f) {
            const float e = __fsub_rn((float)surf_old, UNIFORM ? a.u_target_surface : a.t.target_surface[t_old]);
            const float d = (float)ds_old;
            delta = __fadd_rn(delta, __fmul_rn(lam, __fmul_rn(d, __fadd_rn(__fmul_rn(2.0f, e), d))));
        }
    }
    if (nw != 0) {
        const float lam = UNIFORM ? a.u_lambda_surface : a.t.lambda_surface[t_new];
        if (lam != 0.0f) {
            const float e = __fsub_rn((float)surf_new, UNIFORM ? a.u_target_surface : a.t.target_surface[t_new]);
            const float d = (float)ds_new;
            delta = __fadd_rn(delta, __fmul_rn(lam, __fmul_rn(d, __fadd_rn(__fmul_rn(2.0f, e), d))));
        }
    }
    return delta;
}

}  // namespace glz
