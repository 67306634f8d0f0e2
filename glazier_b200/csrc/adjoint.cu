// The adjoint of the chemical-field step, conditioned on a recorded lattice
// trajectory, behind glz_adj_* in include/glazier_gpu.h.
//
// Forward, one Monte Carlo step per species s (the engine's field step,
// field.rs:99-149, in its f32 operation order):
//   k_s sub-steps   u' = u + d (sum of faces - faces u) - e u,  d = D/k, e = decay/k
//   exchange        v1 = u + sec[t];  v2 = v1 - upt[t] v1;  v = max(v2, 0)
// on sites owned by a cell of type t (owner 255 is the medium: no exchange).
// The discrete Metropolis sweep itself is never differentiated: the owners of
// every step come from a trajectory the caller recorded.
//
// Backward, per step in reverse, per species:
//   exchange        lambda_v1 = lambda_v [v2 >= 0] (1 - upt);  d/dsec += lambda_v1;
//                   d/dupt += -lambda_v [v2 >= 0] v1
//   sub-step        lambda_u = lambda' + d (sum of faces of lambda' - faces lambda') - e lambda'
//                   (the periodic Laplacian is its own transpose);
//                   d/dd += lambda' (sum of faces of u - faces u);  d/de += -lambda' u
// and dD = dd / k, d(decay) = de / k. The forward state is kept at every
// `checkpoint_every`-th step; the backward recomputes each segment's sub-step
// inputs from its checkpoint, but for the last segment, whose sub-step states
// the forward keeps as it goes. Adjoint fields are f32; parameter gradients are
// summed in f64 in an order fixed by the lattice alone.
//
// One launch runs one sub-step round of every species that has a sub-step
// left (the engine's round structure), so with one sub-step per species a
// step is one launch forward and one backward. The backward of a species'
// last round applies the exchange adjoint on the fly at the site and its
// faces (it is pointwise), so it needs no launch of its own.
//
// No reference counterpart: glazier has no differentiable field step.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/glazier_gpu.h"
#include "device.cuh"
#include "engine.h"

namespace {

int fail(int code, const std::string &msg) {
    glz::set_last_error(msg);
    return code;
}

#define CU(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return fail(GLZ_DRIVER, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kThreads = 256;
constexpr uint8_t kMedium = 255;

struct Grid {
    int w, h, d, dim, sites;
    glz::Divider div_w, div_h;  // w and h as multiply-shift dividers
};

__device__ __forceinline__ void faces_of(const Grid &g, size_t i, size_t nb[6]) {
    const int W = g.w, H = g.h, D = g.d;
    // fewer than 2^31 sites: 32-bit quotients
    const uint32_t r = glz::udiv(g.div_w, (uint32_t)i), pl = glz::udiv(g.div_h, r);
    const int x = (int)((uint32_t)i - r * (uint32_t)W), y = (int)(r - pl * (uint32_t)H), z = (int)pl;
    const size_t row = ((size_t)z * H + y) * W;
    nb[0] = row + (x == 0 ? W - 1 : x - 1);
    nb[1] = row + (x == W - 1 ? 0 : x + 1);
    nb[2] = ((size_t)z * H + (y == 0 ? H - 1 : y - 1)) * W + x;
    nb[3] = ((size_t)z * H + (y == H - 1 ? 0 : y + 1)) * W + x;
    if (g.dim == 3) {
        nb[4] = ((size_t)(z == 0 ? D - 1 : z - 1) * H + y) * W + x;
        nb[5] = ((size_t)(z == D - 1 ? 0 : z + 1) * H + y) * W + x;
    }
}

__device__ __forceinline__ float face_sum(const Grid &g, const float *u, const size_t nb[6]) {
    float sum = u[nb[0]];
    sum = __fadd_rn(sum, u[nb[1]]);
    sum = __fadd_rn(sum, u[nb[2]]);
    sum = __fadd_rn(sum, u[nb[3]]);
    if (g.dim == 3) {
        sum = __fadd_rn(sum, u[nb[4]]);
        sum = __fadd_rn(sum, u[nb[5]]);
    }
    return sum;
}

// Every kernel here may be launched before the one ahead of it on the stream
// has finished (programmatic dependent launch, `launch_after`): it waits for
// that grid and its memory first, then lets the next launch start.
__device__ __forceinline__ void grid_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class Kernel, class... Args>
cudaError_t launch_after(Kernel kernel, int grid, size_t smem, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

struct Species {
    const float *in;    // the sub-step's input
    float *out;         // its output (after the exchange in the last round); may be null
    float *keep;        // last round: where to keep the exchange input; may be null
    int active, last;
};

// The per-sub-step diffusion and decay of each species live in device
// memory (`de`: d for every species, then e), like the rate tables, so a
// captured sequence of rounds serves any parameters with the same sub-step
// counts.
struct ForwardRound {
    Grid g;
    int n_species;
    const uint8_t *owner;  // this step's owner types
    const float *sec, *upt, *de;
    Species sp[glz::kMaxSpecies];
};

// One sub-step round of the field step; the exchange on a species' last round.
__global__ void __launch_bounds__(kThreads) forward_round(const __grid_constant__ ForwardRound a) {
    grid_wait();
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.g.sites) return;
    size_t nb[6];
    faces_of(a.g, i, nb);
    const float faces = a.g.dim == 3 ? 6.0f : 4.0f;
    int t = -1;
    for (int s = 0; s < a.n_species; ++s) {
        const Species &p = a.sp[s];
        if (!p.active) continue;
        const float here = p.in[i];
        const float sum = face_sum(a.g, p.in, nb);
        const float d = a.de[s], e = a.de[a.n_species + s];
        float v = __fsub_rn(__fadd_rn(here, __fmul_rn(d, __fsub_rn(sum, __fmul_rn(faces, here)))), __fmul_rn(e, here));
        if (p.last) {
            if (p.keep) p.keep[i] = v;
            if (t < 0) t = a.owner[i];
            if (t != kMedium) {
                v = __fadd_rn(v, a.sec[t * a.n_species + s]);
                v = __fsub_rn(v, __fmul_rn(a.upt[t * a.n_species + s], v));
                v = v < 0.0f ? 0.0f : v;
            }
        }
        if (p.out) p.out[i] = v;
    }
}

// Lattices whose rows are whole multiples of four sites take the round
// kernels in four-site form: a thread takes sites x0 .. x0 + 3 of a row (x0
// a multiple of 4), reads the row and the rows across its y (and z) faces as
// float4 and the two x neighbours past its ends as scalars, so neighbouring
// sites share their loads. Each site's arithmetic is the one-site kernel's,
// operation for operation, so both forms give the same field bits.
struct Quad {
    size_t c;     // the first of the four sites
    size_t l, r;  // the x neighbour before the first and after the last
    size_t f[4];  // the same four x in the rows across the y-1, y+1, z-1 and z+1 faces
};

__device__ __forceinline__ Quad quad_of(const Grid &g, size_t q) {
    const int W = g.w, H = g.h, D = g.d;
    const uint32_t i = (uint32_t)(4 * q);  // fewer than 2^31 sites
    const uint32_t rw = glz::udiv(g.div_w, i), pl = glz::udiv(g.div_h, rw);
    const int x0 = (int)(i - rw * (uint32_t)W), y = (int)(rw - pl * (uint32_t)H), z = (int)pl;
    const size_t row = ((size_t)z * H + y) * W;
    Quad o;
    o.c = row + x0;
    o.l = row + (x0 == 0 ? W - 1 : x0 - 1);
    o.r = row + (x0 + 4 == W ? 0 : x0 + 4);
    o.f[0] = ((size_t)z * H + (y == 0 ? H - 1 : y - 1)) * W + x0;
    o.f[1] = ((size_t)z * H + (y == H - 1 ? 0 : y + 1)) * W + x0;
    o.f[2] = g.dim == 3 ? ((size_t)(z == 0 ? D - 1 : z - 1) * H + y) * W + x0 : 0;
    o.f[3] = g.dim == 3 ? ((size_t)(z == D - 1 ? 0 : z + 1) * H + y) * W + x0 : 0;
    return o;
}

__device__ __forceinline__ void ld4(const float *p, float v[4]) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
}

__device__ __forceinline__ void st4(float *p, const float v[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

__device__ __forceinline__ void ld4(const uint8_t *p, int v[4]) {
    const uchar4 t = *reinterpret_cast<const uchar4 *>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
}

// The four sites' face sums, in face_sum's order, from their own values h,
// the x neighbours past the ends xl and xr, and the rows across the faces.
__device__ __forceinline__ void quad_sums(bool volume, const float h[4], float xl, float xr, const float fy0[4],
                                          const float fy1[4], const float fz0[4], const float fz1[4], float sum[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float v = __fadd_rn(k == 0 ? xl : h[k - 1], k == 3 ? xr : h[k + 1]);
        v = __fadd_rn(v, fy0[k]);
        v = __fadd_rn(v, fy1[k]);
        if (volume) {
            v = __fadd_rn(v, fz0[k]);
            v = __fadd_rn(v, fz1[k]);
        }
        sum[k] = v;
    }
}

__global__ void __launch_bounds__(kThreads) forward_quads(const __grid_constant__ ForwardRound a) {
    grid_wait();
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)a.g.sites / 4) return;
    const Quad o = quad_of(a.g, q);
    const bool volume = a.g.dim == 3;
    const float faces = volume ? 6.0f : 4.0f;
    int own[4];
    bool have_own = false;
    for (int s = 0; s < a.n_species; ++s) {
        const Species &p = a.sp[s];
        if (!p.active) continue;
        float h[4], fy0[4], fy1[4], fz0[4] = {}, fz1[4] = {}, sum[4], v[4];
        ld4(p.in + o.c, h);
        ld4(p.in + o.f[0], fy0);
        ld4(p.in + o.f[1], fy1);
        if (volume) {
            ld4(p.in + o.f[2], fz0);
            ld4(p.in + o.f[3], fz1);
        }
        quad_sums(volume, h, p.in[o.l], p.in[o.r], fy0, fy1, fz0, fz1, sum);
        const float d = a.de[s], e = a.de[a.n_species + s];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] = __fsub_rn(__fadd_rn(h[k], __fmul_rn(d, __fsub_rn(sum[k], __fmul_rn(faces, h[k])))), __fmul_rn(e, h[k]));
        if (p.last) {
            if (p.keep) st4(p.keep + o.c, v);
            if (!have_own) {
                ld4(a.owner + o.c, own);
                have_own = true;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int t = own[k];
                if (t != kMedium) {
                    v[k] = __fadd_rn(v[k], a.sec[t * a.n_species + s]);
                    v[k] = __fsub_rn(v[k], __fmul_rn(a.upt[t * a.n_species + s], v[k]));
                    v[k] = v[k] < 0.0f ? 0.0f : v[k];
                }
            }
        }
        if (p.out) st4(p.out + o.c, v);
    }
}

// Parameter gradients are summed without atomics, in an order fixed by the
// lattice alone, so a backward is bit-reproducible and independent of the
// checkpoint interval: the backward kernel runs on a fixed grid of at most
// `kBlocks` blocks striding over the sites, each block adds its own totals
// into its own row of `partial` (blocks x n_grads f64; a row is touched by
// one block only and launches are ordered on one stream), and
// `reduce_partials` sums the rows in block order at the end.
constexpr int kBlocks = 148 * 8;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// The block's sum of one f64 per thread, in a fixed order, on thread 0.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kWarps; ++w) total += scratch[w];
    __syncthreads();
    return total;
}

struct Adjoint {
    const float *u;     // the sub-step's input
    const float *exch;  // last round: the exchange input
    const float *lam;   // the adjoint of the round's output (of the step's output in the last round)
    float *lam_in;      // the adjoint of the sub-step's input
    int active, last;
};

struct BackwardRound {
    Grid g;
    int n_species, n_types, n_grads;
    const uint8_t *owner;
    const float *sec, *upt, *de;
    double *partial;
    Adjoint sp[glz::kMaxSpecies];
};

// The exchange adjoint at site j: the adjoint of the exchange input from the
// adjoint `l` of its output, with v1 and the clamp gate for the gradients.
__device__ __forceinline__ float exchange_adjoint(const BackwardRound &a, const Adjoint &p, int s, size_t j, float l,
                                                  float *v1_out, float *lv_out) {
    const uint8_t t = a.owner[j];
    if (t == kMedium) return l;
    const float q = a.upt[t * a.n_species + s];
    const float v1 = __fadd_rn(p.exch[j], a.sec[t * a.n_species + s]);
    const float v2 = __fsub_rn(v1, __fmul_rn(q, v1));
    const float lv = v2 < 0.0f ? 0.0f : l;
    if (v1_out) {
        *v1_out = v1;
        *lv_out = lv;
    }
    return __fmul_rn(lv, __fsub_rn(1.0f, q));
}

// One sub-step round backward, last rounds first: lambda of every active
// species through its exchange (last round) and sub-step, and the gradients.
// Each warp reduces the exchange gradients of one owner type at a time (the
// types present in its 32 sites, in lane order of first appearance); lane 0
// adds them to the warp's own shared row. The block's row of `partial` is
// copied into shared memory as the launch starts, summed into there, and
// written back at the end, so no read of it waits at the tail.
__global__ void __launch_bounds__(kThreads) backward_round(const __grid_constant__ BackwardRound a) {
    grid_wait();
    extern __shared__ double acc[];  // kWarps rows of 2 * n_types (sec then upt), then the block's n_grads row
    __shared__ double scratch[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int T = a.n_types, S = a.n_species;
    const float faces = a.g.dim == 3 ? 6.0f : 4.0f;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double *global_row = a.partial + (size_t)blockIdx.x * a.n_grads;
    double *row = acc + (size_t)kWarps * 2 * T;
    for (int k = threadIdx.x; k < a.n_grads; k += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(row + k)), "l"(global_row + k)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    double *mine = acc + (size_t)warp * 2 * T;
    for (int s = 0; s < S; ++s) {
        const Adjoint &p = a.sp[s];
        if (!p.active) continue;
        if (p.last) {
            for (int k = threadIdx.x; k < kWarps * 2 * T; k += blockDim.x) acc[k] = 0.0;
            __syncthreads();
        }
        double gd = 0.0, ge = 0.0;
        // every lane of a warp takes the same number of trips
        for (size_t base = (size_t)blockIdx.x * blockDim.x; base < (size_t)a.g.sites; base += stride) {
            const size_t i = base + threadIdx.x;
            const bool in = i < (size_t)a.g.sites;
            float l1 = 0.0f, dupt = 0.0f;
            int t = kMedium;
            if (in) {
                size_t nb[6];
                faces_of(a.g, i, nb);
                float l = p.lam[i];
                float ls;
                if (p.last) {
                    float v1 = 0.0f, lv = 0.0f;
                    t = a.owner[i];
                    l = exchange_adjoint(a, p, s, i, l, &v1, &lv);
                    if (t != kMedium) {
                        l1 = l;
                        dupt = -__fmul_rn(lv, v1);
                    }
                    ls = exchange_adjoint(a, p, s, nb[0], p.lam[nb[0]], nullptr, nullptr);
                    const int nf = a.g.dim == 3 ? 6 : 4;
                    for (int f = 1; f < nf; ++f)
                        ls = __fadd_rn(ls, exchange_adjoint(a, p, s, nb[f], p.lam[nb[f]], nullptr, nullptr));
                } else {
                    ls = face_sum(a.g, p.lam, nb);
                }
                const float d = a.de[s], e = a.de[S + s];
                p.lam_in[i] = __fsub_rn(__fadd_rn(l, __fmul_rn(d, __fsub_rn(ls, __fmul_rn(faces, l)))), __fmul_rn(e, l));
                const float here = p.u[i];
                const float us = face_sum(a.g, p.u, nb);
                gd += (double)__fmul_rn(l, __fsub_rn(us, __fmul_rn(faces, here)));
                ge -= (double)__fmul_rn(l, here);
            }
            if (p.last) {
                unsigned todo = __ballot_sync(0xffffffffu, t != kMedium);
                while (todo) {
                    const int leader = __ffs(todo) - 1;
                    const int tt = __shfl_sync(0xffffffffu, t, leader);
                    const bool same = t == tt;
                    const double x = warp_sum(same ? (double)l1 : 0.0);
                    const double y = warp_sum(same ? (double)dupt : 0.0);
                    if (lane == 0) {
                        mine[tt] += x;
                        mine[T + tt] += y;
                    }
                    todo &= ~__ballot_sync(0xffffffffu, same);
                }
            }
        }
        // gradient layout: d, e per species, then sec, upt per (type, species);
        // the row's copy has landed once every thread has waited for its own
        // part and block_sum's barrier has passed
        asm volatile("cp.async.wait_all;" ::: "memory");
        const double td = block_sum(gd, scratch);
        const double te = block_sum(ge, scratch);
        if (threadIdx.x == 0) {
            row[s] += td;
            row[S + s] += te;
        }
        if (p.last) {
            __syncthreads();
            for (int k = threadIdx.x; k < 2 * T; k += blockDim.x) {
                double v = 0.0;
                for (int w = 0; w < kWarps; ++w) v += acc[(size_t)w * 2 * T + k];
                const int tt = k % T;
                row[(k < T ? 2 * S : 2 * S + T * S) + tt * S + s] += v;
            }
            __syncthreads();
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (int k = threadIdx.x; k < a.n_grads; k += blockDim.x) global_row[k] = row[k];
}

// A species' rates for owner type t: from registers holding the first TMAX
// types (TMAX > 0, every type below TMAX), else from the tables.
template <int TMAX>
struct Rates {
    float sec[TMAX > 0 ? TMAX : 1], upt[TMAX > 0 ? TMAX : 1];
    const float *gsec, *gupt;  // the tables at the species, stride n_species
    int stride;
    __device__ __forceinline__ void load(const float *sec_table, const float *upt_table, int s, int n_species,
                                         int n_types) {
        gsec = sec_table + s;
        gupt = upt_table + s;
        stride = n_species;
#pragma unroll
        for (int tt = 0; tt < (TMAX > 0 ? TMAX : 1); ++tt) {
            sec[tt] = TMAX > 0 && tt < n_types ? gsec[tt * stride] : 0.0f;
            upt[tt] = TMAX > 0 && tt < n_types ? gupt[tt * stride] : 0.0f;
        }
    }
    __device__ __forceinline__ void of(int t, float &s_out, float &u_out) const {
        if (TMAX > 0) {
            s_out = sec[0];
            u_out = upt[0];
#pragma unroll
            for (int tt = 1; tt < (TMAX > 0 ? TMAX : 1); ++tt)
                if (t == tt) {
                    s_out = sec[tt];
                    u_out = upt[tt];
                }
        } else {
            s_out = gsec[t * stride];
            u_out = gupt[t * stride];
        }
    }
};

// The exchange adjoint of one site of type t (kMedium: none) whose exchange
// input was x: exchange_adjoint with the owner, the input and the rates
// already read.
template <int TMAX>
__device__ __forceinline__ float exchange_adjoint_at(const Rates<TMAX> &r, int t, float x, float l, float *v1_out,
                                                     float *lv_out) {
    if (t == kMedium) return l;
    float sec, q;
    r.of(t, sec, q);
    const float v1 = __fadd_rn(x, sec);
    const float v2 = __fsub_rn(v1, __fmul_rn(q, v1));
    const float lv = v2 < 0.0f ? 0.0f : l;
    *v1_out = v1;
    *lv_out = lv;
    return __fmul_rn(lv, __fsub_rn(1.0f, q));
}

// backward_round in four-site form. Each thread adds its four sites'
// gradient terms in x order. With TMAX > 0 (every owner type below TMAX)
// each thread also keeps its exchange gradients per owner type in registers
// across its trips, and each warp sums them once at the end of a species;
// with TMAX 0 the warps reduce them type by type on every trip, as
// backward_round does. Either way the order is fixed by the lattice.
template <int TMAX>
__global__ void __launch_bounds__(kThreads) backward_quads(const __grid_constant__ BackwardRound a) {
    grid_wait();
    extern __shared__ double acc[];  // kWarps rows of 2 * n_types (sec then upt), then the block's n_grads row
    __shared__ double scratch[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int T = a.n_types, S = a.n_species;
    const bool volume = a.g.dim == 3;
    const float faces = volume ? 6.0f : 4.0f;
    const size_t quads = (size_t)a.g.sites / 4, stride = (size_t)gridDim.x * blockDim.x;
    double *global_row = a.partial + (size_t)blockIdx.x * a.n_grads;
    double *row = acc + (size_t)kWarps * 2 * T;
    for (int k = threadIdx.x; k < a.n_grads; k += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(row + k)),
                     "l"(global_row + k)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    double *mine = acc + (size_t)warp * 2 * T;
    for (int s = 0; s < S; ++s) {
        const Adjoint &p = a.sp[s];
        if (!p.active) continue;
        if (p.last) {
            for (int k = threadIdx.x; k < kWarps * 2 * T; k += blockDim.x) acc[k] = 0.0;
            __syncthreads();
        }
        double gd = 0.0, ge = 0.0;
        double tsec[TMAX > 0 ? TMAX : 1] = {}, tupt[TMAX > 0 ? TMAX : 1] = {};  // per owner type, TMAX > 0
        const float d = a.de[s], e = a.de[S + s];
        Rates<TMAX> rates;
        rates.load(a.sec, a.upt, s, S, T);
        // every lane of a warp takes the same number of trips
        for (size_t base = (size_t)blockIdx.x * blockDim.x; base < quads; base += stride) {
            const size_t q = base + threadIdx.x;
            const bool in = q < quads;
            float l1[4] = {}, dupt[4] = {};
            int t[4] = {kMedium, kMedium, kMedium, kMedium};
            if (in) {
                const Quad o = quad_of(a.g, q);
                float l[4], fy0[4], fy1[4], fz0[4] = {}, fz1[4] = {}, ls[4];
                ld4(p.lam + o.c, l);
                ld4(p.lam + o.f[0], fy0);
                ld4(p.lam + o.f[1], fy1);
                if (volume) {
                    ld4(p.lam + o.f[2], fz0);
                    ld4(p.lam + o.f[3], fz1);
                }
                float xl = p.lam[o.l], xr = p.lam[o.r];
                // the sub-step input, read before anything is written
                float u[4], uy0[4], uy1[4], uz0[4] = {}, uz1[4] = {}, us[4];
                ld4(p.u + o.c, u);
                ld4(p.u + o.f[0], uy0);
                ld4(p.u + o.f[1], uy1);
                if (volume) {
                    ld4(p.u + o.f[2], uz0);
                    ld4(p.u + o.f[3], uz1);
                }
                const float ul = p.u[o.l], ur = p.u[o.r];
                if (p.last) {
                    float x[4], v1, lv;
                    ld4(a.owner + o.c, t);
                    ld4(p.exch + o.c, x);
                    int ty0[4], ty1[4], tz0[4] = {}, tz1[4] = {};
                    float xy0[4], xy1[4], xz0[4] = {}, xz1[4] = {};
                    ld4(a.owner + o.f[0], ty0);
                    ld4(p.exch + o.f[0], xy0);
                    ld4(a.owner + o.f[1], ty1);
                    ld4(p.exch + o.f[1], xy1);
                    if (volume) {
                        ld4(a.owner + o.f[2], tz0);
                        ld4(p.exch + o.f[2], xz0);
                        ld4(a.owner + o.f[3], tz1);
                        ld4(p.exch + o.f[3], xz1);
                    }
                    const int tl = a.owner[o.l], tr = a.owner[o.r];
                    const float xxl = p.exch[o.l], xxr = p.exch[o.r];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        l[k] = exchange_adjoint_at(rates, t[k], x[k], l[k], &v1, &lv);
                        if (t[k] != kMedium) {
                            l1[k] = l[k];
                            dupt[k] = -__fmul_rn(lv, v1);
                        }
                        fy0[k] = exchange_adjoint_at(rates, ty0[k], xy0[k], fy0[k], &v1, &lv);
                        fy1[k] = exchange_adjoint_at(rates, ty1[k], xy1[k], fy1[k], &v1, &lv);
                        if (volume) {
                            fz0[k] = exchange_adjoint_at(rates, tz0[k], xz0[k], fz0[k], &v1, &lv);
                            fz1[k] = exchange_adjoint_at(rates, tz1[k], xz1[k], fz1[k], &v1, &lv);
                        }
                    }
                    xl = exchange_adjoint_at(rates, tl, xxl, xl, &v1, &lv);
                    xr = exchange_adjoint_at(rates, tr, xxr, xr, &v1, &lv);
                }
                quad_sums(volume, l, xl, xr, fy0, fy1, fz0, fz1, ls);
                float li[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    li[k] = __fsub_rn(__fadd_rn(l[k], __fmul_rn(d, __fsub_rn(ls[k], __fmul_rn(faces, l[k])))),
                                      __fmul_rn(e, l[k]));
                st4(p.lam_in + o.c, li);
                quad_sums(volume, u, ul, ur, uy0, uy1, uz0, uz1, us);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    gd += (double)__fmul_rn(l[k], __fsub_rn(us[k], __fmul_rn(faces, u[k])));
                    ge -= (double)__fmul_rn(l[k], u[k]);
                }
            }
            if (TMAX > 0 && p.last) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int tt = 0; tt < (TMAX > 0 ? TMAX : 1); ++tt) {
                        tsec[tt] += t[k] == tt ? (double)l1[k] : 0.0;
                        tupt[tt] += t[k] == tt ? (double)dupt[k] : 0.0;
                    }
            } else if (p.last) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    unsigned todo = __ballot_sync(0xffffffffu, t[k] != kMedium);
                    while (todo) {
                        const int leader = __ffs(todo) - 1;
                        const int tt = __shfl_sync(0xffffffffu, t[k], leader);
                        const bool same = t[k] == tt;
                        const double x = warp_sum(same ? (double)l1[k] : 0.0);
                        const double y = warp_sum(same ? (double)dupt[k] : 0.0);
                        if (lane == 0) {
                            mine[tt] += x;
                            mine[T + tt] += y;
                        }
                        todo &= ~__ballot_sync(0xffffffffu, same);
                    }
                }
            }
        }
        if (TMAX > 0 && p.last) {
#pragma unroll
            for (int tt = 0; tt < (TMAX > 0 ? TMAX : 1); ++tt) {
                const double x = warp_sum(tsec[tt]), y = warp_sum(tupt[tt]);
                if (lane == 0 && tt < T) {
                    mine[tt] = x;
                    mine[T + tt] = y;
                }
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        const double td = block_sum(gd, scratch);
        const double te = block_sum(ge, scratch);
        if (threadIdx.x == 0) {
            row[s] += td;
            row[S + s] += te;
        }
        if (p.last) {
            __syncthreads();
            for (int k = threadIdx.x; k < 2 * T; k += blockDim.x) {
                double v = 0.0;
                for (int w = 0; w < kWarps; ++w) v += acc[(size_t)w * 2 * T + k];
                const int tt = k % T;
                row[(k < T ? 2 * S : 2 * S + T * S) + tt * S + s] += v;
            }
            __syncthreads();
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (int k = threadIdx.x; k < a.n_grads; k += blockDim.x) global_row[k] = row[k];
}

// grads[k] = the sum over blocks of partial[b][k], one warp per k: lane l
// adds rows l, l + 32, ... in order, then the warp's lanes are summed by the
// fixed shuffle tree, so the order depends on the block count alone.
__global__ void __launch_bounds__(kThreads) reduce_partials(const double *__restrict__ partial, int blocks, int n_grads,
                                                            double *__restrict__ grads) {
    grid_wait();
    const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (k >= n_grads) return;  // whole warps leave together
    double v = 0.0;
#pragma unroll 8
    for (int b = lane; b < blocks; b += 32) v += partial[(size_t)b * n_grads + k];
    v = warp_sum(v);
    if (lane == 0) grads[k] = v;
}

// field.rs:155-160
int substeps(double diffusion, int dimensions) {
    if (diffusion <= 0.0) return 1;
    double k = std::ceil(diffusion / (1.0 / (2.0 * (double)dimensions)));
    return k < 1.0 ? 1 : (int)k;
}

}  // namespace

struct glz_adj {
    Grid g{};
    int n_species = 0, n_types = 0, steps = 0, every = 1;
    cudaStream_t stream = nullptr;
    uint8_t *owner = nullptr;  // steps * sites
    bool have_trajectory = false;
    float *ckpt = nullptr;     // ceil(steps / every) checkpoints of n_species * sites
    float *seg = nullptr;      // a segment's sub-step states: every * (kmax + 1) * n_species * sites
    float *tmp[2] = {};        // n_species * sites each: sub-step outputs inside a step
    float *work[2] = {};       // step outputs between checkpoints
    float *lam[2] = {};        // the adjoint fields
    float *d_sec = nullptr, *d_upt = nullptr;  // d_sec starts the one allocation of the rate tables
    float *staging = nullptr;                  // pinned: the rate tables on their way in
    float *d_de = nullptr;      // per-sub-step d then e per species
    float *final_out = nullptr; // n_species * sites: the forward's last step, copied to the caller
    double *partial = nullptr;  // kBlocks rows of n_grads
    double *d_grads = nullptr;  // n_grads: d, e per species, then sec, upt per (type, species)
    std::vector<double> params;
    std::vector<int> k;
    int kmax = 0;
    int seg_kmax = -1;          // the kmax `seg` was sized for
    bool forward_done = false;
    // The forward and backward sequences as CUDA graphs, captured for the
    // sub-step counts in `graph_k` and replayed for any parameters with them.
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
    std::vector<int> graph_k;
    int bwd_cur[glz::kMaxSpecies] = {};  // after a backward: which lam buffer holds each species
};

namespace {

size_t field_floats(const glz_adj *h) { return (size_t)h->n_species * h->g.sites; }
int n_grads(const glz_adj *h) { return 2 * h->n_species + 2 * h->n_types * h->n_species; }
// Rows of whole multiples of four sites take the four-site kernels.
bool quads(const glz_adj *h) { return h->g.w % 4 == 0; }
int blocks_for(const glz_adj *h) {
    const long long items = quads(h) ? h->g.sites / 4 : h->g.sites;
    return (int)((items + kThreads - 1) / kThreads);
}

int launch_forward(glz_adj *h, const ForwardRound &a) {
    CU(quads(h) ? launch_after(forward_quads, blocks_for(h), 0, h->stream, a)
                : launch_after(forward_round, blocks_for(h), 0, h->stream, a));
    return GLZ_OK;
}
// the rate tables in one run: sec and upt per (type, species), d and e per species
size_t table_floats(const glz_adj *h) { return (size_t)2 * h->n_types * h->n_species + 2 * h->n_species; }

// The sub-step state j of species s at step `local` of the segment starting
// at checkpoint `sg`: j < k[s] the input of sub-step j, j = k[s] the exchange
// input. State 0 of the segment's first step is the checkpoint itself.
float *seg_state(glz_adj *h, int sg, int local, int j, int s) {
    if (local == 0 && j == 0) return h->ckpt + ((size_t)sg * h->n_species + s) * (size_t)h->g.sites;
    return h->seg + (((size_t)local * (h->kmax + 1) + j) * h->n_species + s) * (size_t)h->g.sites;
}

int set_params(glz_adj *h, const double *params) {
    const int S = h->n_species, T = h->n_types;
    for (int s = 0; s < S; ++s)
        if (!(params[s] >= 0.0) || !(params[S + s] >= 0.0) || !std::isfinite(params[s]) ||
            !std::isfinite(params[S + s]))
            return fail(GLZ_INVALID, "diffusion and decay must be finite and >= 0");
    h->params.assign(params, params + n_grads(h));
    h->k.resize(S);
    h->kmax = 0;
    for (int s = 0; s < S; ++s) {
        h->k[s] = substeps(params[s], h->g.dim);
        h->kmax = h->k[s] > h->kmax ? h->k[s] : h->kmax;
    }
    // sec, upt, then d and e per species, staged in pinned memory: every
    // forward ends in a stream synchronize, so the previous copy out of the
    // staging has landed before it is written again
    float *sec = h->staging, *upt = sec + T * S, *de = upt + T * S;
    for (int i = 0; i < T * S; ++i) {
        sec[i] = (float)params[2 * S + i];
        upt[i] = (float)params[2 * S + T * S + i];
    }
    for (int sp = 0; sp < S; ++sp) {
        de[sp] = (float)(params[sp] / (double)h->k[sp]);
        de[S + sp] = (float)(params[S + sp] / (double)h->k[sp]);
    }
    CU(cudaMemcpyAsync(h->d_sec, h->staging, table_floats(h) * 4, cudaMemcpyHostToDevice, h->stream));
    if (h->seg_kmax != h->kmax) {
        cudaFree(h->seg);
        h->seg = nullptr;
        h->seg_kmax = -1;
        CU(cudaMalloc(&h->seg, (size_t)h->every * (h->kmax + 1) * field_floats(h) * sizeof(float)));
        h->seg_kmax = h->kmax;
    }
    return GLZ_OK;
}

// One step forward of every species, owners of step t, from `in` to `out`
// (n_species * sites each, distinct buffers).
int step_forward(glz_adj *h, int t, const float *in, float *out) {
    const size_t n = h->g.sites;
    ForwardRound a{};
    a.g = h->g;
    a.n_species = h->n_species;
    a.owner = h->owner + (size_t)t * n;
    a.sec = h->d_sec;
    a.upt = h->d_upt;
    a.de = h->d_de;
    const float *cur[glz::kMaxSpecies];
    for (int s = 0; s < h->n_species; ++s) cur[s] = in + (size_t)s * n;
    for (int r = 0; r < h->kmax; ++r) {
        for (int s = 0; s < h->n_species; ++s) {
            Species &p = a.sp[s];
            p.active = r < h->k[s];
            p.last = r == h->k[s] - 1;
            p.in = cur[s];
            p.keep = nullptr;
            p.out = p.last ? out + (size_t)s * n : h->tmp[r & 1] + (size_t)s * n;
            if (p.active) cur[s] = p.out;
        }
        if (int rc = launch_forward(h, a)) return rc;
    }
    return GLZ_OK;
}

// Step `local` of segment `sg` forward, keeping every sub-step state in the
// segment buffers; the output of the segment's last step goes to `last_out`
// (not kept: null).
int keep_step(glz_adj *h, int sg, int local, int len, float *last_out) {
    ForwardRound a{};
    a.g = h->g;
    a.n_species = h->n_species;
    a.sec = h->d_sec;
    a.upt = h->d_upt;
    a.de = h->d_de;
    a.owner = h->owner + (size_t)(sg * h->every + local) * h->g.sites;
    for (int r = 0; r < h->kmax; ++r) {
        for (int s = 0; s < h->n_species; ++s) {
            Species &p = a.sp[s];
            p.active = r < h->k[s];
            p.last = r == h->k[s] - 1;
            if (!p.active) continue;
            p.in = seg_state(h, sg, local, r, s);
            if (p.last) {
                p.keep = seg_state(h, sg, local, h->k[s], s);
                p.out = local + 1 < len ? seg_state(h, sg, local + 1, 0, s)
                                        : (last_out ? last_out + (size_t)s * h->g.sites : nullptr);
            } else {
                p.keep = nullptr;
                p.out = seg_state(h, sg, local, r + 1, s);
            }
        }
        if (int rc = launch_forward(h, a)) return rc;
    }
    return GLZ_OK;
}

// Recompute segment `sg`, keeping every sub-step state; its last step's
// output is not needed.
int recompute(glz_adj *h, int sg, int len) {
    for (int local = 0; local < len; ++local)
        if (int rc = keep_step(h, sg, local, len, nullptr)) return rc;
    return GLZ_OK;
}

void drop_graphs(glz_adj *h) {
    if (h->fwd_exec) cudaGraphExecDestroy(h->fwd_exec);
    if (h->bwd_exec) cudaGraphExecDestroy(h->bwd_exec);
    h->fwd_exec = h->bwd_exec = nullptr;
    h->graph_k.clear();
}

// Record what `body` queues on the handle's stream as a graph, instantiated
// into *exec; the capture ends whatever the body returns.
int capture(glz_adj *h, cudaGraphExec_t *exec, int (*body)(glz_adj *)) {
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body(h);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("adjoint capture: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(GLZ_DRIVER, std::string("adjoint graph: ") + cudaGetErrorString(ei));
    return GLZ_OK;
}

// Every step forward from checkpoint 0: a step's output goes to the next
// checkpoint, to the work buffer the step did not read, or (the last) to
// final_out. The last segment's steps keep their sub-step states as a
// recompute would, so the backward starts without recomputing it.
int forward_sequence(glz_adj *h) {
    const size_t n = field_floats(h);
    const int last = (h->steps - 1) / h->every, t_last = last * h->every;
    const float *cur = h->ckpt;
    for (int t = 0; t < t_last; ++t) {
        float *dst;
        if ((t + 1) % h->every == 0)
            dst = h->ckpt + (size_t)((t + 1) / h->every) * n;
        else
            dst = cur == h->work[0] ? h->work[1] : h->work[0];
        if (int rc = step_forward(h, t, cur, dst)) return rc;
        cur = dst;
    }
    for (int t = t_last; t < h->steps; ++t)
        if (int rc = keep_step(h, last, t - t_last, h->steps - t_last, h->final_out)) return rc;
    return GLZ_OK;
}

// The backward from lam[0] (the loss gradient at the final fields), segment
// by segment from the last: recompute the segment's sub-step states, then
// its rounds backward; the per-block gradient rows summed at the end.
int backward_sequence(glz_adj *h) {
    const int S = h->n_species, T = h->n_types, G = n_grads(h);
    const size_t sites = h->g.sites;
    const int grid = blocks_for(h) < kBlocks ? blocks_for(h) : kBlocks;
    CU(cudaMemsetAsync(h->partial, 0, (size_t)grid * G * 8, h->stream));
    int cur[glz::kMaxSpecies] = {};  // which lam buffer holds each species' adjoint
    BackwardRound a{};
    a.g = h->g;
    a.n_species = S;
    a.n_types = T;
    a.n_grads = G;
    a.sec = h->d_sec;
    a.upt = h->d_upt;
    a.de = h->d_de;
    a.partial = h->partial;
    const size_t smem = ((size_t)kWarps * 2 * T + G) * sizeof(double);
    // owner types held in registers up to 4 or 8 types, else reduced per trip
    auto *backward = !quads(h) ? backward_round
                     : T <= 4  ? backward_quads<4>
                     : T <= 8  ? backward_quads<8>
                               : backward_quads<0>;
    CU(cudaFuncSetAttribute(backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int nseg = (h->steps + h->every - 1) / h->every;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int t0 = sg * h->every, len = (t0 + h->every < h->steps ? t0 + h->every : h->steps) - t0;
        // the forward left the last segment's states in place
        if (sg < nseg - 1)
            if (int rc = recompute(h, sg, len)) return rc;
        for (int local = len - 1; local >= 0; --local) {
            a.owner = h->owner + (size_t)(t0 + local) * sites;
            for (int r = h->kmax - 1; r >= 0; --r) {
                for (int s = 0; s < S; ++s) {
                    Adjoint &p = a.sp[s];
                    p.active = r < h->k[s];
                    p.last = r == h->k[s] - 1;
                    if (!p.active) continue;
                    p.u = seg_state(h, sg, local, r, s);
                    p.exch = seg_state(h, sg, local, h->k[s], s);
                    p.lam = h->lam[cur[s]] + (size_t)s * sites;
                    p.lam_in = h->lam[1 - cur[s]] + (size_t)s * sites;
                    cur[s] = 1 - cur[s];
                }
                CU(launch_after(backward, grid, smem, h->stream, a));
            }
        }
        CU(cudaGetLastError());
    }
    CU(launch_after(reduce_partials, (G + kWarps - 1) / kWarps, 0, h->stream, (const double *)h->partial, grid, G,
                     h->d_grads));
    for (int s = 0; s < S; ++s) h->bwd_cur[s] = cur[s];
    return GLZ_OK;
}

}  // namespace

extern "C" {

int glz_adj_create(int width, int height, int depth, int n_species, int n_types, int steps, int checkpoint_every,
                   glz_adj **out) {
    if (!out) return fail(GLZ_INVALID, "null output handle");
    *out = nullptr;
    if (width <= 0 || height <= 0 || depth <= 0) return fail(GLZ_INVALID, "the lattice has a zero dimension");
    if (n_species < 1 || n_species > glz::kMaxSpecies || n_types < 1 || n_types > 254 || steps < 1 ||
        checkpoint_every < 1)
        return fail(GLZ_INVALID, "species 1..8, types 1..254, steps and checkpoint interval >= 1");
    const long long sites = (long long)width * height * depth;
    if (sites >= (1LL << 31)) return fail(GLZ_INVALID, "the lattice has 2^31 sites or more");
    glz_adj *h = new glz_adj();
    h->g = Grid{width, height, depth, depth > 1 ? 3 : 2, (int)sites, glz::make_divider((uint32_t)width),
                glz::make_divider((uint32_t)height)};
    h->n_species = n_species;
    h->n_types = n_types;
    h->steps = steps;
    h->every = checkpoint_every < steps ? checkpoint_every : steps;
    const size_t n = field_floats(h);
    const int nckpt = (steps + h->every - 1) / h->every;
    auto bail = [&](int rc) {
        glz_adj_destroy(h);
        return rc;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->owner, (size_t)steps * sites) != cudaSuccess ||
        cudaMalloc(&h->ckpt, (size_t)nckpt * n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->tmp[0], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->tmp[1], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->work[0], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->work[1], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->lam[0], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->lam[1], n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->d_sec, table_floats(h) * 4) != cudaSuccess ||
        cudaMallocHost(&h->staging, table_floats(h) * 4) != cudaSuccess ||
        cudaMalloc(&h->final_out, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->partial, (size_t)kBlocks * n_grads(h) * 8) != cudaSuccess ||
        cudaMalloc(&h->d_grads, (size_t)n_grads(h) * 8) != cudaSuccess)
        return bail(fail(GLZ_DRIVER, "adjoint allocation failed"));
    h->d_upt = h->d_sec + (size_t)n_types * n_species;
    h->d_de = h->d_upt + (size_t)n_types * n_species;
    *out = h;
    return GLZ_OK;
}

int glz_adj_set_trajectory(glz_adj *h, const uint8_t *owner_types) {
    if (!h || !owner_types) return fail(GLZ_INVALID, "null handle or trajectory");
    const size_t bytes = (size_t)h->steps * h->g.sites;
    for (size_t i = 0; i < bytes; ++i)
        if (owner_types[i] != kMedium && owner_types[i] >= h->n_types)
            return fail(GLZ_INVALID, "an owner type past the type count (255 is the medium)");
    CU(cudaMemcpyAsync(h->owner, owner_types, bytes, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->have_trajectory = true;
    h->forward_done = false;
    return GLZ_OK;
}

int glz_adj_forward(glz_adj *h, const double *params, const float *fields0, float *fields_final) {
    if (!h || !params || !fields0 || !fields_final) return fail(GLZ_INVALID, "null argument");
    if (!h->have_trajectory) return fail(GLZ_INVALID, "no trajectory set");
    if (fields0 == fields_final) return fail(GLZ_INVALID, "the initial and final fields share a buffer");
    h->forward_done = false;
    if (int rc = set_params(h, params)) return rc;
    // the graphs hold the sub-step structure (and the segment buffers sized
    // for it): new sub-step counts take new graphs
    if (h->graph_k != h->k) drop_graphs(h);
    if (!h->fwd_exec) {
        if (int rc = capture(h, &h->fwd_exec, forward_sequence)) return rc;
        h->graph_k = h->k;
    }
    const size_t n = field_floats(h);
    CU(cudaMemcpyAsync(h->ckpt, fields0, n * 4, cudaMemcpyDeviceToDevice, h->stream));  // checkpoint 0
    CU(cudaGraphLaunch(h->fwd_exec, h->stream));
    CU(cudaMemcpyAsync(fields_final, h->final_out, n * 4, cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->forward_done = true;
    return GLZ_OK;
}

int glz_adj_backward(glz_adj *h, const float *grad_final, double *grad_params, float *grad_fields0) {
    if (!h || !grad_final || !grad_params) return fail(GLZ_INVALID, "null argument");
    if (!h->forward_done) return fail(GLZ_INVALID, "backward before forward");
    const int S = h->n_species, G = n_grads(h);
    const size_t n = field_floats(h), sites = h->g.sites;
    if (!h->bwd_exec)
        if (int rc = capture(h, &h->bwd_exec, backward_sequence)) return rc;
    CU(cudaMemcpyAsync(h->lam[0], grad_final, n * 4, cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaGraphLaunch(h->bwd_exec, h->stream));
    if (grad_fields0)
        for (int s = 0; s < S; ++s)
            CU(cudaMemcpyAsync(grad_fields0 + (size_t)s * sites, h->lam[h->bwd_cur[s]] + (size_t)s * sites, sites * 4,
                               cudaMemcpyDeviceToDevice, h->stream));
    std::vector<double> g(G);
    CU(cudaMemcpyAsync(g.data(), h->d_grads, (size_t)G * 8, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    // d = D / k and e = decay / k, so the D and decay gradients are the
    // per-sub-step ones over k
    for (int s = 0; s < S; ++s) {
        grad_params[s] = g[s] / h->k[s];
        grad_params[S + s] = g[S + s] / h->k[s];
    }
    for (int i = 2 * S; i < G; ++i) grad_params[i] = g[i];
    return GLZ_OK;
}

void *glz_adj_stream(glz_adj *h) { return h ? (void *)h->stream : nullptr; }

void glz_adj_destroy(glz_adj *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graphs(h);
    cudaFree(h->final_out);
    cudaFree(h->owner);
    cudaFree(h->ckpt);
    cudaFree(h->seg);
    cudaFree(h->tmp[0]);
    cudaFree(h->tmp[1]);
    cudaFree(h->work[0]);
    cudaFree(h->work[1]);
    cudaFree(h->lam[0]);
    cudaFree(h->lam[1]);
    cudaFree(h->d_sec);
    cudaFreeHost(h->staging);
    cudaFree(h->partial);
    cudaFree(h->d_grads);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
