// The band sweep: every colour pass of a large lean plane in one cooperative
// launch, the lattice streamed through shared memory a whole row at a time.
//
// Replaces `cpm_sweep` and its host loop (glazier-cuda/src/lib.rs:436-716,
// 1083-1128) for planes whose copies price contact, volume and surface only,
// with the draws, pricing and commits of the other sweep kernels (sweep.cu),
// so a run is bit for bit the one they and the host replay give.
//
// Layout of the work:
//   - A pass's targets in row y read rows y - 1, y and y + 1 only. The
//     lattice's columns are cut into segments of at most 2048 sites, and the
//     units of work are (segment, target row) pairs: the rows of the pass's
//     colour parity, one segment wide. Each CTA owns a contiguous share of
//     the units, which falls into runs of consecutive target rows of one
//     segment; a run of n target rows needs its 2n + 1 segment rows, which a
//     producer warp streams in order into a ring of row slots by bulk copies
//     (the segment's contiguous stretch, plus 16 bytes of halo at each end
//     from the neighbouring columns, wrapped at the lattice's edges). Short
//     segment rows let the ring hold many of them, so rows land well ahead
//     of the target rows that read them.
//   - The consumer warps share each target row: every lane draws its
//     targets' picks and compares the two labels, a warp queues the targets
//     whose pick carries another label, and prices its queue in full rounds
//     of 32, carrying fewer than 32 queued copies into its next row so the
//     expensive path runs with every lane busy. A row slot goes back to the
//     producer when every consumer warp has finished the target rows that
//     read it (an mbarrier per slot, one arrival per warp).
//   - Passes are separated by a grid barrier (bounded, error flag 4): the
//     per-cell tallies a pass reads are its snapshot, complete only once
//     every CTA has finished the pass before.

#include <cuda_runtime.h>

#include <atomic>

#include "device.cuh"
#include "engine.h"
#include "neighbours.cuh"
#include "pricing.cuh"

namespace glz {

constexpr int kBandPad = 4;         // labels of periodic halo at each end of a ring row (16 bytes)
constexpr int kBandMaxSlots = 16;   // ring rows at most (a power of two)
constexpr int kBandMinSlots = 8;    // five rows in use (a target row's three, the last one's two) and three ahead
constexpr int kBandTypes = 16;      // contact tables up to 16 types live in shared memory
constexpr long long kBandWaitLimit = 1LL << 20;     // mbarrier polls before a wait gives up
constexpr long long kBandBarrierLimit = 1LL << 22;  // grid-barrier polls (each an L2 round trip)
#ifndef GLZ_BAND_WARPS
#define GLZ_BAND_WARPS 16
#endif
#ifndef GLZ_BAND_SEG_MAX
#define GLZ_BAND_SEG_MAX 2048
#endif
constexpr int kBandSegMax = GLZ_BAND_SEG_MAX;  // sites of a column segment at most
#ifndef GLZ_BAND_PER_SM
#define GLZ_BAND_PER_SM 1
#endif
constexpr int kBandWarps = GLZ_BAND_WARPS;  // consumer warps; one more warp produces
constexpr int kBandPerSm = GLZ_BAND_PER_SM;  // CTAs (bands) per SM, each with its share of shared memory
constexpr int kBandThreads = 32 * (kBandWarps + 1);
constexpr int kBandConsumers = 32 * kBandWarps;

struct BandLaunch {
    ResidentLaunch r;
    int slots;  // ring rows, a power of two
    int shift;  // log2(slots)
    int qcap;   // queue entries per consumer warp
    int seg;    // sites of a column segment (a multiple of 4 that divides the width)
};

struct BandHead {
    alignas(8) unsigned long long full[kBandMaxSlots];   // the slot's row has landed
    alignas(8) unsigned long long empty[kBandMaxSlots];  // every consumer warp is done with the slot's row
    unsigned last[kBandMaxSlots];  // sequence number of the latest row put into the slot, plus one
    float contact[kBandTypes * kBandTypes];
    int abort;   // a wait gave up: every warp stops at the pass's end
    int bar_ok;  // the grid barrier's outcome, for the whole block
};

__device__ __forceinline__ bool band_wait(unsigned long long *bar, uint32_t parity) {
    const uint32_t b = smem_addr(bar);
    uint32_t done = 0;
    for (long long spin = 0; spin < kBandWaitLimit && !done; ++spin)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
    return done != 0;
}

// The neighbour offset of pick k, decoded from compile-time constants.
template <int NOFF>
__device__ __forceinline__ void band_offset(int k, int &dx, int &dy) {
    constexpr unsigned px = [] {
        unsigned v = 0;
        for (int i = 0; i < NOFF; ++i) v |= (unsigned)(neighbour_offset<2, NOFF>(i, 0) + 1) << (2 * i);
        return v;
    }();
    constexpr unsigned py = [] {
        unsigned v = 0;
        for (int i = 0; i < NOFF; ++i) v |= (unsigned)(neighbour_offset<2, NOFF>(i, 1) + 1) << (2 * i);
        return v;
    }();
    dx = (int)((px >> (2 * k)) & 3u) - 1;
    dy = (int)((py >> (2 * k)) & 3u) - 1;
}

// A pass's draws and tally view.
struct BandPass {
    int colour;
    uint64_t key_accept;
    const int2 *vs_base;
    const long long *vs_prev;
    unsigned long long *vs_cur;
};

// The per-colour guard: whether cell `old` keeps a site of a colour other
// than the pass's own, which no copy in this pass can take.
__device__ __noinline__ bool band_keeps_other_colour(const SweepLaunch &a, int colour, uint32_t old) {
    int other = 0;
    for (int c = 0; c < 4; ++c)
        if (c != colour) other += a.vol_by_colour[(size_t)old * 4 + c];
    return other != 0;
}

// Price the copy attempt at target (x0 + x, y) whose pick `pick` carries
// another label, and commit it if the Metropolis test takes it:
// direct_target's arithmetic (sweep.cu) operation for operation, the labels
// read from the three ring rows rm, r0, rp (rows y - 1, y, y + 1 of the
// segment starting at column x0, halo included, x counted in the segment).
template <int NOFF, bool UNIFORM>
__device__ __forceinline__ void band_price(const SweepLaunch &a, const BandPass &v, const float *contact,
                                           bool small_types, const uint32_t *rm, const uint32_t *r0,
                                           const uint32_t *rp, int x, int x0, int y, int pick) {
    const auto at = [&](int k) -> uint32_t {
        const int dx = neighbour_offset<2, NOFF>(k, 0), dy = neighbour_offset<2, NOFF>(k, 1);
        return (dy < 0 ? rm : (dy > 0 ? rp : r0))[x + dx];
    };
    const uint32_t target = (uint32_t)(y * a.g.w + x0 + x);
    const uint32_t old = r0[x];
    int pdx, pdy;
    band_offset<NOFF>(pick, pdx, pdy);
    const uint32_t nw = (pdy < 0 ? rm : (pdy > 0 ? rp : r0))[x + pdx];
    int2 base_old = make_int2(0, 0), base_new = make_int2(0, 0);
    long long prev_old = 0, prev_new = 0;
    if (old != 0) {
        base_old = v.vs_base[old];
        prev_old = v.vs_prev[old];
    }
    if (nw != 0) {
        base_new = v.vs_base[nw];
        prev_new = v.vs_prev[nw];
    }
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
                delta = __fsub_rn(delta, small_types ? contact[t_old * a.n_types + tn] : a.t.contact[t_old * a.n_types + tn]);
            else
                ++like_old;
            if (ln != nw)
                delta = __fadd_rn(delta, small_types ? contact[t_new * a.n_types + tn] : a.t.contact[t_new * a.n_types + tn]);
            else
                ++like_new;
        }
    }
    // A like neighbour is a site of another colour, since every neighbour of
    // a target is; only a target with none needs the per-colour count.
    if (old != 0 && like_old == 0 && !band_keeps_other_colour(a, v.colour, old)) return;
    const int ds_old = 2 * like_old - NOFF;
    const int ds_new = NOFF - 2 * like_new;
    int dv, ds;
    unpack_delta(prev_old, dv, ds);
    const int vol_old = base_old.x + dv, surf_old = base_old.y + ds;
    unpack_delta(prev_new, dv, ds);
    const int vol_new = base_new.x + dv, surf_new = base_new.y + ds;
    delta = size_terms<UNIFORM>(a, old, nw, t_old, t_new, vol_old, vol_new, surf_old, surf_new, ds_old, ds_new, delta);
    const float u = to_f32(draw(v.key_accept, target));
    if (!(delta <= 0.0f || u < metropolis_exp(__fmul_rn(-delta, a.beta)))) return;
    a.labels[target] = nw;
    if (old != 0) {
        atomicAdd(&v.vs_cur[old], pack_delta(-1, ds_old));
        atomicSub(&a.vol_by_colour[(size_t)old * 4 + v.colour], 1);
    }
    if (nw != 0) {
        atomicAdd(&v.vs_cur[nw], pack_delta(1, ds_new));
        atomicAdd(&a.vol_by_colour[(size_t)nw * 4 + v.colour], 1);
    }
}

// Grid barrier number k of the launch (k = 0, 1, ...): false if it timed out.
// Every thread of the block calls it. The arrival is a gpu-scope release of
// the block's writes (each thread's fence, then the block barrier, then the
// arriving thread's fence); the waiting thread's acquire load and fence, then
// the block barrier, order what follows after every block's writes.
__device__ __forceinline__ bool band_barrier(unsigned *bar, unsigned k, int *ok_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        if (atomicAdd(&bar[0], 1u) + 1u == gridDim.x * (k + 1u)) {
            __threadfence();
            atomicExch(&bar[1], k + 1u);
        } else {
            long long spin = 0;
            for (;;) {
                unsigned g;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(&bar[1]) : "memory");
                if (g >= k + 1u) break;
                if (++spin > kBandBarrierLimit) {
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        *ok_flag = ok;
    }
    __syncthreads();
    return *(volatile int *)ok_flag != 0;
}

template <int NOFF, bool UNIFORM>
__global__ void __launch_bounds__(kBandThreads, kBandPerSm) band_sweep_kernel(const __grid_constant__ BandLaunch B) {
    const ResidentLaunch &r = B.r;
    const SweepLaunch &a = r.a;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char *base = smem_raw + ((128u - (raw & 127u)) & 127u);
    BandHead &S = *reinterpret_cast<BandHead *>(base);
    const int slots = B.slots, qcap = B.qcap, SW = B.seg;
    const uint32_t mask = (uint32_t)slots - 1u, shift = (uint32_t)B.shift;  // slot q & mask, its use q >> shift
    uint32_t *queues = reinterpret_cast<uint32_t *>(base + ((sizeof(BandHead) + 127) / 128) * 128);
    const int W = a.g.w, H = a.g.h;
    const int RW = SW + 2 * kBandPad;
    uint32_t *ring = queues + (((size_t)kBandWarps * qcap * 4 + 127) / 128) * 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool producer = warp == kBandWarps;

    const int NT = H / 2;                // target rows of a pass in one column segment
    const int NS = W / SW;               // column segments
    const long long units = (long long)NS * NT;
    const long long lo = ((long long)blockIdx.x * units) / gridDim.x;       // this block's units:
    const long long hi = ((long long)(blockIdx.x + 1) * units) / gridDim.x;  // (segment, target row) pairs
    const int HSW = SW / 2;              // targets of a segment row
    const int per_row = (HSW + 32 * kBandWarps - 1) / (32 * kBandWarps);  // a lane's targets a row

    if (tid == 0) {
        for (int s = 0; s < slots; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&S.empty[s])), "r"(kBandWarps));
            S.last[s] = 0;
        }
        S.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const bool small_types = a.n_types <= kBandTypes;
    if (!UNIFORM && small_types)
        for (int k = tid; k < a.n_types * a.n_types; k += blockDim.x) S.contact[k] = a.t.contact[k];
    __syncthreads();

    uint32_t q0 = 0;  // ring sequence number of the next run's first row
    unsigned kbar = 0;
    const unsigned below = (1u << lane) - 1u;
    uint32_t *queue = queues + (size_t)(producer ? 0 : warp) * qcap;
    for (int m = 0; m < r.mcs; ++m) {
        const int32_t step = (int32_t)((uint32_t)r.step0 + (uint32_t)m);
        for (int c = 0; c < 4; ++c) {
            const long long p = r.pass0 + (long long)m * 4 + c;
            const int cx = c & 1, cy = (c >> 1) & 1;
            const BandPass v{c, stream_key(r.seed, step, c, 1), r.vs_base[p % 2], r.vs_delta[(p + 2) % 3],
                             reinterpret_cast<unsigned long long *>(r.vs_delta[p % 3])};
            const uint64_t key_pick = stream_key(r.seed, step, c, 0);
            if (!producer) {
                // The tally rotation for the next pass, which no thread of this one reads.
                int2 *next_base = r.vs_base[(p + 1) % 2];
                long long *clear = r.vs_delta[(p + 1) % 3];
                const size_t stride = (size_t)gridDim.x * kBandConsumers;
                for (size_t l = (size_t)blockIdx.x * kBandConsumers + tid; l < (size_t)a.n_labels; l += stride) {
                    int dv, ds;
                    unpack_delta(v.vs_prev[l], dv, ds);
                    const int2 b = v.vs_base[l];
                    next_base[l] = make_int2(b.x + dv, b.y + ds);
                    clear[l] = 0;
                }
            }
            // The block's units fall into runs, one per column segment they touch:
            // run [t0, t1) of segment `seg` streams rows 2 t0 + cy - 1 ... 2 t1 + cy - 1.
            for (long long u0 = lo; u0 < hi;) {
                const int seg = (int)(u0 / NT);
                const int t0 = (int)(u0 - (long long)seg * NT);
                const long long u1 = hi < (long long)(seg + 1) * NT ? hi : (long long)(seg + 1) * NT;
                const int n = (int)(u1 - u0);  // target rows in this run
                const int rows = 2 * n + 1;
                const int x0 = seg * SW;
                u0 = u1;
                if (producer) {
                    if (lane == 0) {
                        // labels the previous pass wrote (generic proxy) are read by bulk copies (async proxy)
                        asm volatile("fence.proxy.async.global;" ::: "memory");
                        const int xl = x0 == 0 ? W - kBandPad : x0 - kBandPad;  // the left halo's columns
                        const int xr = x0 + SW == W ? 0 : x0 + SW;              // the right halo's
                        for (int j = 0; j < rows; ++j) {
                            if (*(volatile int *)&S.abort) break;
                            const uint32_t q = q0 + (uint32_t)j;
                            const int slot = (int)(q & mask);
                            const uint32_t use = q >> shift;
                            if (use > 0 && !band_wait(&S.empty[slot], (use - 1u) & 1u)) {
                                atomicExch(a.error_flag, 1);
                                S.abort = 1;
                                break;
                            }
                            int yy = 2 * t0 + cy - 1 + j;
                            yy += yy < 0 ? H : (yy >= H ? -H : 0);
                            const uint32_t *src = a.labels + (size_t)yy * W;
                            uint32_t *dst = ring + (size_t)slot * RW;
                            const uint32_t bar = smem_addr(&S.full[slot]);
                            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                                         "r"((uint32_t)(RW * 4))
                                         : "memory");
                            asm volatile(
                                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                                "[%3];" ::"r"(smem_addr(dst + kBandPad)),
                                "l"(src + x0), "r"((uint32_t)(SW * 4)), "r"(bar)
                                : "memory");
                            asm volatile(
                                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                                "[%3];" ::"r"(smem_addr(dst)),
                                "l"(src + xl), "r"((uint32_t)(kBandPad * 4)), "r"(bar)
                                : "memory");
                            asm volatile(
                                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                                "[%3];" ::"r"(smem_addr(dst + kBandPad + SW)),
                                "l"(src + xr), "r"((uint32_t)(kBandPad * 4)), "r"(bar)
                                : "memory");
                            S.last[slot] = q + 1u;
                        }
                    }
                } else if (!*(volatile int *)&S.abort) {
                    const auto row_of = [&](uint32_t q) { return ring + (size_t)(q & mask) * RW + kBandPad; };
                    const auto ready = [&](uint32_t q) { return band_wait(&S.full[q & mask], (q >> shift) & 1u); };
                    // One arrival per warp: the warp's lanes meet first (their reads of
                    // the slot come before lane 0's arrival), so a slot takes as many
                    // arrivals as there are consumer warps, not threads.
                    const auto release = [&](uint32_t q) {
                        __syncwarp();
                        if (lane == 0)
                            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&S.empty[q & mask]))
                                         : "memory");
                    };
                    // entries held over from the previous target row: queue[0, held), its rows and y
                    int held = 0, hy = 0;
                    const uint32_t *hm = nullptr, *h0 = nullptr, *hp = nullptr;
                    bool failed = false;
                    for (int t = 0; t < n; ++t) {
                        const uint32_t q = q0 + 2u * (uint32_t)t + 1u;  // the target row's own ring sequence number
                        const bool ok = (t > 0 || ready(q - 1u)) && ready(q) && ready(q + 1u);
                        if (!__all_sync(0xffffffffu, ok) || *(volatile int *)&S.abort) {
                            if (lane == 0 && !ok) {
                                atomicExch(a.error_flag, 1);
                                S.abort = 1;
                            }
                            failed = true;
                            break;
                        }
                        const uint32_t *rm = row_of(q - 1u), *r0 = row_of(q), *rp = row_of(q + 1u);
                        const int y = 2 * (t0 + t) + cy;
                        // Light pass: the warp's targets whose pick carries another label
                        // join its queue behind the entries held from the previous row.
                        int total = held;
                        for (int part = 0; part < per_row; ++part) {
                            const int i = (part * kBandWarps + warp) * 32 + lane;
                            bool active = false;
                            int pick = 0;
                            if (i < HSW) {
                                const int xs = 2 * i + cx;  // in the segment
                                pick = pick_of<NOFF>(draw(key_pick, (uint32_t)(y * W + x0 + xs)));
                                int dx, dy;
                                band_offset<NOFF>(pick, dx, dy);
                                active = r0[xs] != (dy < 0 ? rm : (dy > 0 ? rp : r0))[xs + dx];
                            }
                            const unsigned bits = __ballot_sync(0xffffffffu, active);
                            if (active) queue[total + __popc(bits & below)] = (uint32_t)i | ((uint32_t)pick << 16);
                            total += __popc(bits);
                        }
                        __syncwarp();
                        // Heavy pass: whole rounds of 32, oldest first; what is left of
                        // the previous row goes in one last short round so its rows can
                        // be let go; fewer than 32 of this row's stay held.
                        int taken = 0;
                        for (;;) {
                            const int left = total - taken;
                            if (left < 32 && taken >= held) break;
                            const int e = taken + lane;
                            if (e < total) {
                                const bool before = e < held;
                                const uint32_t entry = queue[e];
                                band_price<NOFF, UNIFORM>(a, v, S.contact, small_types, before ? hm : rm,
                                                          before ? h0 : r0, before ? hp : rp,
                                                          2 * (int)(entry & 0xffffu) + cx, x0, before ? hy : y,
                                                          (int)(entry >> 16));
                            }
                            taken += left < 32 ? left : 32;
                        }
                        __syncwarp();
                        if (t > 0) {  // the previous target row (sequence q - 2) is done: its rows q - 3, q - 2
                            release(q - 3u);
                            release(q - 2u);
                        }
                        const int keep = total - taken;
                        if (taken > 0 && keep > 0) {
                            const uint32_t e = lane < keep ? queue[taken + lane] : 0u;
                            __syncwarp();
                            if (lane < keep) queue[lane] = e;
                            __syncwarp();
                        }
                        held = keep;
                        hy = y;
                        hm = rm;
                        h0 = r0;
                        hp = rp;
                    }
                    if (!failed) {
                        if (lane < held) {
                            const uint32_t entry = queue[lane];
                            band_price<NOFF, UNIFORM>(a, v, S.contact, small_types, hm, h0, hp,
                                                      2 * (int)(entry & 0xffffu) + cx, x0, hy, (int)(entry >> 16));
                        }
                        const uint32_t ql = q0 + 2u * (uint32_t)n - 1u;  // the run's last target row
                        release(ql - 1u);
                        release(ql);
                        release(ql + 1u);
                    }
                }
                q0 += (uint32_t)rows;
            }
            // this pass's label writes are read by the next pass's bulk copies
            asm volatile("fence.proxy.async.global;" ::: "memory");
            __syncthreads();
            if (*(volatile int *)&S.abort) {
                // let every copy still in flight land before the block leaves
                if (producer && lane == 0)
                    for (int s = 0; s < slots; ++s)
                        if (S.last[s] > 0) band_wait(&S.full[s], ((S.last[s] - 1u) >> shift) & 1u);
                __syncthreads();
                return;
            }
            if (!band_barrier(r.barrier, kbar++, &S.bar_ok)) {
                if (tid == 0) atomicExch(a.error_flag, 4);
                return;
            }
        }
    }
}

// The shared memory a band's CTA may take: the per-block limit, or its share
// of the SM's when several CTAs share one.
static int band_budget(int dev) {
    int optin = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) return 0;
    const int share = per_sm / kBandPerSm - 1024;  // each resident block also holds 1 KB the system reserves
    return share < optin ? share : optin;
}

// The launch shape of the band sweep for a plane of width w: the column
// segment (the widest that divides w, is a multiple of 4 and at most
// kBandSegMax), ring rows (a power of two, kBandMinSlots at least) and queue
// room; false when the plane does not suit it.
static bool band_shape(int w, int h, int smem_budget, int &seg, int &slots, int &shift, int &qcap, size_t &smem) {
    if (w % 4 != 0 || w < 2 * kBandPad || h < 2) return false;
    seg = 0;
    for (int parts = 1; parts <= w / 4; ++parts)
        if (w % parts == 0 && (w / parts) % 4 == 0 && w / parts <= kBandSegMax) {
            seg = w / parts;
            break;
        }
    if (seg < 2 * kBandPad) return false;
    const int per_row = (seg / 2 + 32 * kBandWarps - 1) / (32 * kBandWarps);
    qcap = 32 * per_row + 32;
    const size_t head = (sizeof(BandHead) + 127) / 128 * 128;
    const size_t queue = ((size_t)kBandWarps * qcap * 4 + 127) / 128 * 128;
    const size_t row = (size_t)(seg + 2 * kBandPad) * 4;
    const long long room = (long long)smem_budget - 128 - (long long)head - (long long)queue;
    // the most rows that fit, rounded down to a power of two so a row's slot
    // and phase are a mask and a shift of its sequence number
    const long long fit = room / (long long)row;
    slots = 1;
    shift = 0;
    while (2LL * slots <= fit && 2 * slots <= kBandMaxSlots) {
        slots *= 2;
        ++shift;
    }
    if (slots < kBandMinSlots) return false;
    smem = head + queue + (size_t)slots * row + 128;
    return true;
}

template <int NOFF, bool UNIFORM>
static cudaError_t launch_band(const ResidentLaunch &r, cudaStream_t stream) {
    // the SM count and shared-memory budget, looked up once (handles on other
    // host threads may launch too)
    static std::atomic<int> sms_once{0}, optin_once{0};
    if (!sms_once.load(std::memory_order_acquire)) {
        int dev = 0, n = 0;
        if (cudaError_t e = cudaGetDevice(&dev)) return e;
        if (cudaError_t e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) return e;
        optin_once.store(band_budget(dev), std::memory_order_relaxed);
        sms_once.store(n, std::memory_order_release);
    }
    const int sms = sms_once.load(std::memory_order_acquire), optin = optin_once.load(std::memory_order_relaxed);
    BandLaunch b{};
    b.r = r;
    size_t smem = 0;
    if (!band_shape(r.a.g.w, r.a.g.h, optin, b.seg, b.slots, b.shift, b.qcap, smem)) return cudaErrorNotSupported;
    if (cudaError_t e = cudaFuncSetAttribute(band_sweep_kernel<NOFF, UNIFORM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
        return e;
    int per_sm = 0;
    if (cudaError_t e =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, band_sweep_kernel<NOFF, UNIFORM>, kBandThreads, smem))
        return e;
    if (per_sm < kBandPerSm) return cudaErrorNotSupported;
    void *args[] = {&b};
    return cudaLaunchCooperativeKernel((const void *)band_sweep_kernel<NOFF, UNIFORM>,
                                       dim3((unsigned)(sms * kBandPerSm)), dim3(kBandThreads), args, smem, stream);
}

bool band_sweep_fits(int w, int h) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const int optin = band_budget(dev);
    int seg = 0, slots = 0, shift = 0, qcap = 0;
    size_t smem = 0;
    return band_shape(w, h, optin, seg, slots, shift, qcap, smem);
}

cudaError_t launch_band_sweep(const ResidentLaunch &r, cudaStream_t stream) {
    const Geometry &g = r.a.g;
    if (g.dim != 2 || (g.n_off != 4 && g.n_off != 8)) return cudaErrorNotSupported;
    for (int k = 0; k < g.n_off; ++k)
        for (int axis = 0; axis < 3; ++axis) {
            const int want = g.n_off == 4 ? neighbour_offset<2, 4>(k, axis) : neighbour_offset<2, 8>(k, axis);
            if (g.off[k][axis] != want) return cudaErrorInvalidValue;
        }
    const bool uniform = r.a.uniform_type >= 0 && r.a.uniform_contact_exact;
    if (g.n_off == 4) return uniform ? launch_band<4, true>(r, stream) : launch_band<4, false>(r, stream);
    return uniform ? launch_band<8, true>(r, stream) : launch_band<8, false>(r, stream);
}

}  // namespace glz
