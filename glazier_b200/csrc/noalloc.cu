// One Monte Carlo step of the chemical-field solver on caller-owned device
// buffers, allocating nothing.
//
// Some callers cannot call cudaMalloc: a host application that fixes its
// device-memory budget at start-up and forbids allocation afterwards, or a
// coupled solver that hands this library only buffers it owns. For them this
// file keeps the field step's scratch (a status word and the intermediate
// sub-step fields) in one file-scope __device__ array of fixed size. Every GPU
// that loads the library holds that array until the process exits. The
// per-type secretion and uptake rates travel in the kernel's parameters.
//
// The arithmetic is the engine's field step (fields.cu): FTCS diffusion and
// decay per sub-step, exchange folded into each species' last sub-step.

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/glazier_gpu.h"
#include "device.cuh"
#include "engine.h"

namespace {

constexpr int kStatusFloats = 64;                                     // one 256-byte line: the status word
constexpr size_t kScratchFloats = (size_t)GLZ_NOALLOC_FIELD_SCRATCH;   // intermediate fields
constexpr int kTable = glz::kMaxTypes * glz::kMaxSpecies;

// The scratch: a status word (bit 0: a label at or past n_labels, bit 1: a
// cell type at or past n_types), then the intermediate sub-step fields. In
// host code this name is a host-side stand-in, not a device address; the
// kernel is given the address cudaGetSymbolAddress returns for the current
// device.
static __device__ __align__(256) float g_noalloc_scratch[kStatusFloats + kScratchFloats];

// The array's device address per device ordinal, looked up once per device
// by the first call made with that device current. A context that
// cudaDeviceReset replaces gets a new array; this cache does not follow it.
constexpr int kMaxDevices = 64;
std::atomic<float *> g_scratch_ptr[kMaxDevices] = {};


struct NoallocRound {
    int w, h, d, dim, sites, n_species, n_types;
    const float *in[glz::kMaxSpecies];
    float *out[glz::kMaxSpecies];
    float dd[glz::kMaxSpecies], decay[glz::kMaxSpecies];
    int active[glz::kMaxSpecies], last[glz::kMaxSpecies];
    const uint32_t *labels;
    const uint8_t *cell_type;
    uint32_t n_labels;
    unsigned *status;  // the scratch's status word
    float secretion[kTable], uptake[kTable];  // [type][species], n_types * n_species used
};

template <int DIM>
__global__ void __launch_bounds__(256) noalloc_round_kernel(const __grid_constant__ NoallocRound a) {
    const int W = a.w, H = a.h, D = a.d;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)a.sites) return;
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
        float v = __fsub_rn(__fadd_rn(here, __fmul_rn(a.dd[s], __fsub_rn(sum, __fmul_rn(faces, here)))),
                            __fmul_rn(a.decay[s], here));
        if (a.last[s]) {
            if (type < 0) {
                const uint32_t l = a.labels[i];
                // A label past the type table, or a type past the rate tables, is
                // recorded in the status word (the call reports it) and takes no
                // exchange rather than a read out of bounds.
                if (l >= a.n_labels) {
                    atomicOr(a.status, 1u);
                    type = 0x7fffffff;
                } else {
                    type = l == 0 ? 0x7fffffff : a.cell_type[l];
                    if (l != 0 && type >= a.n_types) {
                        atomicOr(a.status, 2u);
                        type = 0x7fffffff;
                    }
                }
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

int fail(int code, const std::string &msg) {
    glz::set_last_error(msg);
    return code;
}

// field.rs:155-160
int substeps(double diffusion, int dimensions) {
    if (diffusion <= 0.0) return 1;
    double k = std::ceil(diffusion / (1.0 / (2.0 * (double)dimensions)));
    return k < 1.0 ? 1 : (int)k;
}

}  // namespace

extern "C" {

int glz_field_step_noalloc(int width, int height, int depth, int n_species, int n_types, const double *diffusion,
                           const double *decay, const double *secretion, const double *uptake,
                           const uint32_t *labels, const uint8_t *cell_type, size_t n_labels,
                           const float *fields_in, float *fields_out, void *stream) {
    if (width <= 0 || height <= 0 || depth <= 0) return fail(GLZ_INVALID, "the lattice has a zero dimension");
    if (n_species < 1 || n_species > glz::kMaxSpecies) return fail(GLZ_INVALID, "n_species must be 1 to 8");
    if (n_types < 1 || n_types > glz::kMaxTypes) return fail(GLZ_INVALID, "n_types must be 1 to 64");
    if (!diffusion || !decay || !secretion || !uptake || !labels || !cell_type || !fields_in || !fields_out)
        return fail(GLZ_INVALID, "a null pointer");
    if (n_labels == 0) return fail(GLZ_INVALID, "the cell type table is empty");
    const long long sites = (long long)width * height * depth;
    if (sites >= (1LL << 31)) return fail(GLZ_INVALID, "the lattice has 2^31 sites or more");
    {
        // The stencil reads a site's neighbours while other threads write the
        // output, so the two buffers may not share a byte.
        const uintptr_t bytes = (uintptr_t)n_species * (uintptr_t)sites * sizeof(float);
        const uintptr_t in0 = reinterpret_cast<uintptr_t>(fields_in), out0 = reinterpret_cast<uintptr_t>(fields_out);
        if (in0 < out0 + bytes && out0 < in0 + bytes)
            return fail(GLZ_INVALID, "fields_in and fields_out overlap; the step needs two distinct buffers");
    }
    const int dim = depth > 1 ? 3 : 2;
    int rounds = 0, k[glz::kMaxSpecies];
    for (int s = 0; s < n_species; ++s) {
        k[s] = substeps(diffusion[s], dim);
        rounds = k[s] > rounds ? k[s] : rounds;
    }
    // Intermediate fields: one buffer per species for two rounds, two from three.
    const size_t buffers = rounds <= 1 ? 0 : (rounds == 2 ? 1 : 2);
    const size_t need = buffers * (size_t)n_species * (size_t)sites;
    if (need > kScratchFloats) {
        char msg[200];
        std::snprintf(msg, sizeof msg,
                      "the step needs %zu scratch floats; this entry point holds at most %zu "
                      "(GLZ_NOALLOC_FIELD_SCRATCH)",
                      need, kScratchFloats);
        return fail(GLZ_INVALID, msg);
    }

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(GLZ_INVALID, "device ordinal past the 64 this entry point tracks");
    float *scratch = g_scratch_ptr[dev].load();
    if (!scratch) {
        // Once per device, with that device current: the array's device
        // address. The host symbol itself is not one. Two threads that race
        // here store the same address.
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        scratch = static_cast<float *>(p);
        g_scratch_ptr[dev].store(scratch);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned *status = reinterpret_cast<unsigned *>(scratch);
    float *fields = scratch + kStatusFloats;
    // The array keeps the last call's contents: the status word starts at zero.
    e = cudaMemsetAsync(status, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("status reset: ") + cudaGetErrorString(e));

    const size_t n = (size_t)sites;
    int cur[glz::kMaxSpecies] = {};  // -1: the caller's input; 0/1: a scratch buffer
    for (int s = 0; s < n_species; ++s) cur[s] = -1;
    for (int r = 0; r < rounds; ++r) {
        NoallocRound a{};
        a.w = width;
        a.h = height;
        a.d = depth;
        a.dim = dim;
        a.sites = (int)sites;
        a.n_species = n_species;
        a.n_types = n_types;
        a.labels = labels;
        a.cell_type = cell_type;
        a.n_labels = (uint32_t)(n_labels > 0xffffffffu ? 0xffffffffu : n_labels);
        a.status = status;
        // the rates as f32, the type the engine's field step uses
        for (int c = 0; c < n_types * n_species; ++c) {
            a.secretion[c] = (float)secretion[c];
            a.uptake[c] = (float)uptake[c];
        }
        for (int s = 0; s < n_species; ++s) {
            a.active[s] = r < k[s];
            a.last[s] = r == k[s] - 1;
            a.dd[s] = (float)(diffusion[s] / (double)k[s]);
            a.decay[s] = (float)(decay[s] / (double)k[s]);
            a.in[s] = cur[s] < 0 ? fields_in + (size_t)s * n : fields + ((size_t)cur[s] * n_species + s) * n;
            const int next = cur[s] < 0 ? 0 : 1 - cur[s];
            a.out[s] = a.last[s] ? fields_out + (size_t)s * n : fields + ((size_t)next * n_species + s) * n;
        }
        const int blocks = (int)((n + 255) / 256);
        if (dim == 2)
            noalloc_round_kernel<2><<<blocks, 256, 0, st>>>(a);
        else
            noalloc_round_kernel<3><<<blocks, 256, 0, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("launch: ") + cudaGetErrorString(e));
        for (int s = 0; s < n_species; ++s)
            if (a.active[s] && !a.last[s]) cur[s] = cur[s] < 0 ? 0 : 1 - cur[s];
    }
    // Wait for the step, then report what the status word recorded.
    unsigned flags = 0;
    e = cudaMemcpyAsync(&flags, status, sizeof flags, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(GLZ_DRIVER, std::string("field step: ") + cudaGetErrorString(e));
    if (flags & 1u) return fail(GLZ_INVALID, "a label is not below the cell type count");
    if (flags & 2u) return fail(GLZ_INVALID, "a cell type is not below the type count");
    return GLZ_OK;
}

}  // extern "C"
