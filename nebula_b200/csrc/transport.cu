// Persistent electron-transport kernel and the kernel-level query kernels.
//
// The transport kernel replaces the reference's event-sorted SIMT driver
// (drivers/gpu/gpu_driver.inl:312-567: init + CUB radix sort + intersect /
// elastic / inelastic launched over the whole slot capacity every
// iteration).  Here each thread keeps one electron in registers and runs
// init -> event passes back to back until the electron terminates or is
// detected, then refills from a device queue with a warp-aggregated atomic.
// Cascades run depth-first, child first: when an event creates a secondary,
// the parent is parked on a small per-thread stack and the secondary is
// simulated at once, so a primary's whole cascade normally stays in one
// thread and never touches global memory.  Only a cascade deeper than the
// stack hands secondaries to the next generation's queue (warp-aggregated
// push).  Detections are tallied per primary tag on the device; detected
// records are optional.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "features.cuh"
#include "kernels.h"
#include "mlp.cuh"
#include "transport.cuh"

namespace cg = cooperative_groups;

namespace nbx {

namespace {

__device__ __forceinline__ void load_electron(const Queue& q, uint32_t i, dev::Electron& e) {
    const float4 a = q.a[i];
    const float4 b = q.b[i];
    const uint4 c = q.c[i];
    e.px = a.x;
    e.py = a.y;
    e.pz = a.z;
    e.E = a.w;
    e.dx = b.x;
    e.dy = b.y;
    e.dz = b.z;
    e.mat = __float_as_int(b.w);
    e.tag = c.x;
    e.uid = uint64_t(c.y) | (uint64_t(c.z) << 32);
    e.last_tri = int(c.w);
    e.step = 0;
}

__device__ __forceinline__ void store_electron(const Queue& q, uint32_t i, const dev::Electron& e) {
    q.a[i] = make_float4(e.px, e.py, e.pz, e.E);
    q.b[i] = make_float4(e.dx, e.dy, e.dz, __int_as_float(e.mat));
    q.c[i] = make_uint4(e.tag, uint32_t(e.uid), uint32_t(e.uid >> 32), uint32_t(e.last_tri));
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Learned mode: statistical weights are powers of two, 2^wexp, so every
// roulette survivor's weight 1 / q is exact and fits in a few bits of the
// parked material word; wexp stays within [kMinWeightExp, kMaxWeightExp].
constexpr int kMaxWeightExp = 12;   // at most 4096 (a chain of roulettes)
constexpr int kMinWeightExp = -4;   // at least 1/16 (a chain of splits)
// An overflowed newborn secondary of the learned mode carries its weight
// exponent in the queue's last-triangle word (a secondary has no last
// triangle): kWeightTag | uint8(wexp); no real triangle index has these bits.
constexpr uint32_t kWeightTag = 0xFFFFFE00u;

// Words per thread of the transport kernel's dynamic shared memory: the leaf
// cache, then the event counters.  Counter slots 0-3 are indexed by the event
// type (dev::kEvNone .. dev::kEvBoundary; slot 0 is never read).
constexpr int kLeafCacheWords = 13;
constexpr int kSlotSteps = 4, kSlotSecondaries = 5, kSlotDetectedSE = 6, kSlotDetectedBSE = 7, kSlotTerminated = 8,
              kSlotPopped = 9;
constexpr int kCounterSlots = 10;
static_assert(dev::kEvNone == 0 && dev::kEvInelastic == 1 && dev::kEvElastic == 2 && dev::kEvBoundary == 3,
              "event types index counter slots 0-3");

struct LearnedSmem {
    mlp::Weights w;
    __nv_bfloat16 xs[8 * 32 * mlp::kIn];   // one 32 x 16 feature tile per warp
};
// The learned-mode kernels' network image and feature tiles (only the
// kernels that call birth_logit hold it).
__shared__ __align__(16) LearnedSmem g_lsm;

// Network logit of this lane's newborn secondary (valid where cand): the
// warp's candidates (ballot m) are packed into the first rows of the warp's
// feature tile and one m-tile (up to 16 candidates) or two go through the
// tensor cores.  Called by the whole warp.  Not inlined, so the network's
// register demand does not raise the transport loop's.
__device__ __noinline__ float birth_logit(unsigned m, bool cand, const dev::SurfaceMap S, float px, float py, float pz,
                                          float dx, float dy, float dz, float E, int mat) {
    const int lane = threadIdx.x & 31;
    const int rank = __popc(m & ((1u << lane) - 1u));
    __nv_bfloat16* xs = g_lsm.xs + (threadIdx.x >> 5) * 32 * mlp::kIn;
    if (cand) {
        float f[6];
        const dev::V3 d = dev::normalised(dev::V3{dx, dy, dz});
        dev::electron_features(S, px, py, pz, d.x, d.y, d.z, logf(E), mat, f);
        __nv_bfloat16* row = xs + rank * mlp::kIn;
#pragma unroll
        for (int k = 0; k < mlp::kIn; ++k) row[k] = __float2bfloat16_rn(k < 6 ? f[k] : 0.0f);
    }
    __syncwarp();
    const float logit =
        __popc(m) <= 16 ? mlp::warp_forward_rows<1>(g_lsm.w, xs) : mlp::warp_forward_rows<2>(g_lsm.w, xs);
    const float mine = __shfl_sync(0xffffffffu, logit, rank);
    __syncwarp();
    return mine;
}

// Per-electron state of the sample mode, parked alongside the electron.
struct Extra {
    int rec;          // sample record slot, -1 none
    uint32_t flags;   // bit 0: sub-cascade produced a detected SE
    uint32_t c0;      // the thread's step count when the record was taken
};

// Parked ancestors of a thread's cascade, in global memory laid out per
// thread (stack_depth entries of three float4: (pos, E), (dir, material),
// (uid, step, last triangle)).  A local-memory array interleaves threads word
// by word, so lanes parked at different depths scatter each of an entry's 13
// words into its own sector; here an entry is 48 contiguous bytes (two
// sectors, three 16-byte accesses).  The tag is not stored: every electron of
// a thread's cascade carries its primary's tag.  With kW (learned mode) the
// material word also carries the weight exponent in its upper 16 bits (the
// material index fits the lower 16).  base == nullptr: use the local array
// instead (callers without a stack buffer).
struct ParkedStack {
    float4* base;
    template <bool kW>
    __device__ __forceinline__ void put(int i, const dev::Electron& e, dev::Electron* local, int wexp) const {
        const int mw = kW ? int((uint32_t(e.mat) & 0xFFFFu) | (uint32_t(wexp) << 16)) : e.mat;
        if (base) {
            float4* p = base + 3 * i;
            p[0] = make_float4(e.px, e.py, e.pz, e.E);
            p[1] = make_float4(e.dx, e.dy, e.dz, __int_as_float(mw));
            p[2] = make_float4(__uint_as_float(uint32_t(e.uid)), __uint_as_float(uint32_t(e.uid >> 32)),
                               __uint_as_float(e.step), __int_as_float(e.last_tri));
        } else {
            local[i] = e;
            local[i].mat = mw;
        }
    }
    template <bool kW>
    __device__ __forceinline__ void get(int i, dev::Electron& e, const dev::Electron* local, int& wexp) const {
        int mw;
        if (base) {
            const float4* p = base + 3 * i;
            const float4 a = p[0], b = p[1], c = p[2];
            e.px = a.x;
            e.py = a.y;
            e.pz = a.z;
            e.E = a.w;
            e.dx = b.x;
            e.dy = b.y;
            e.dz = b.z;
            mw = __float_as_int(b.w);
            e.uid = uint64_t(__float_as_uint(c.x)) | (uint64_t(__float_as_uint(c.y)) << 32);
            e.step = __float_as_uint(c.z);
            e.last_tri = __float_as_int(c.w);
        } else {
            e = local[i];
            mw = e.mat;
        }
        if constexpr (kW) {
            e.mat = int(int16_t(mw & 0xFFFF));
            wexp = mw >> 16;
        } else {
            e.mat = mw;
        }
    }
};

__device__ __forceinline__ uint32_t mix32(uint64_t x) {
    x ^= x >> 33;
    x *= 0xFF51AFD7ED558CCDull;
    x ^= x >> 33;
    return uint32_t(x);
}

// Philox block of a secondary's step 0 that decides its roulette at birth
// (the transport's own draws use blocks 0-2 and 3 + 64 at most).
constexpr uint32_t kBirthBlock = 0x7FFFFFFFu;

// Birth decision of the learned mode for a newborn secondary of weight
// 2^wexp and importance p (the network's escape probability): returns the
// change of its weight exponent -- k > 0 for Russian roulette with survival
// 2^-k (the survivor's weight is 2^(wexp + k)), -1 to split it in two halves,
// 0 to keep it as it is.
//
// Weight window (no cost table): the target weight of importance p is
// rr_threshold / p below rr_threshold (rounded to a power of two, at most
// 2^max_k) and 1 above it; a newborn lighter than its target plays roulette
// up to it, so a lineage is not rouletted twice for the same importance.
// Above split_threshold a newborn of weight >= 1 splits in two.
//
// Cost-aware (cost table set): minimising variance x cost of the tally, a
// particle of weight w whose sub-cascade scores with probability p at mean
// cost c should survive with q = w sqrt(p K / c), K = cost / variance per
// primary of the analogue run; q is rounded to a power of two (roulette
// below 1, at least 2^-max_k; a split in two from sqrt(2) up, for p above
// split_threshold).
__device__ __forceinline__ int birth_decision(const TransportArgs& a, float p, int wexp, float E, int mat) {
    const float pc = fmaxf(p, 1e-30f);
    if (a.cost_bins > 0) {
        const int m = mat < 0 ? 0 : (mat >= a.cost_materials ? a.cost_materials - 1 : mat);
        int b = int(floorf((__logf(E) - a.cost_log_e_min) * a.cost_inv_width));
        b = b < 0 ? 0 : (b >= a.cost_bins ? a.cost_bins - 1 : b);
        const float c = fmaxf(__ldg(a.cost_table + m * a.cost_bins + b), 1.0f);
        const float l2q = float(wexp) + 0.5f * __log2f(pc * a.value_per_cost / c);
        const int k = -int(rintf(l2q));
        if (k >= 1) return k > a.max_roulette_exp ? a.max_roulette_exp : k;
        return (k <= -1 && p > a.split_threshold) ? -1 : 0;
    }
    if (p > a.split_threshold) return wexp >= 0 ? -1 : 0;
    if (!(p < a.rr_threshold)) return 0;
    int kt = int(rintf(__log2f(a.rr_threshold / pc)));
    kt = kt < 0 ? 0 : (kt > a.max_roulette_exp ? a.max_roulette_exp : kt);
    return kt > wexp ? kt - wexp : 0;
}

// The network's importance of a newborn from the importance table: its
// features at birth, each clamped into the table's range, select the cell.
__device__ __forceinline__ float table_importance(const TransportArgs& a, const dev::Electron& se) {
    float f[6];
    const dev::V3 d = dev::approx::normalised(dev::V3{se.dx, se.dy, se.dz});
    dev::electron_features(a.smap, se.px, se.py, se.pz, d.x, d.y, d.z, __logf(se.E), se.mat, f);
    const int m = se.mat < 0 ? 0 : (se.mat >= a.imp_materials ? a.imp_materials - 1 : se.mat);
    const int ie = min(max(int(floorf(f[0] * float(a.imp_ne))), 0), a.imp_ne - 1);
    const int id = min(max(int(floorf(f[1] * float(a.imp_nd))), 0), a.imp_nd - 1);
    const int ic = min(max(int(floorf((f[2] + 1.0f) * 0.5f * float(a.imp_nc))), 0), a.imp_nc - 1);
    return __ldg(a.imp_table + ((size_t(m) * a.imp_ne + ie) * a.imp_nd + id) * a.imp_nc + ic);
}

// MinBlocks: resident blocks per SM the register allocation must allow --
// 256-thread blocks for 2 (128 registers), 3 (80) and 4 (64); 128-thread
// blocks for 7 (72 registers, 28 warps); the host picks the variant.
// Mode: kModePlain (analogue transport), kModeSample (plain transport that
// also records one (features, label, cost) training sample for about one in
// sixteen newborn secondaries), kModeLearned (plain transport of weighted
// electrons: every newborn secondary is scored at birth by the network,
// batched per warp on the tensor cores, and plays Russian roulette or splits
// on that importance; a warp stays in the loop until all its lanes are done,
// so the tensor-core call always has the whole warp), or kModeDeposit (plain
// transport that also appends an energy-deposit record per energy-changing
// scattering event).
template <int MinBlocks, int Mode, bool Penn>
__global__ void __launch_bounds__(MinBlocks == 7 ? 128 : 256, MinBlocks) transport_kernel(const dev::Physics P, const TransportArgs a) {
    // Dynamic shared memory sized by the launch (transport_smem_bytes), per
    // thread and strided by the block size: the leaf cache (13 words), then
    // the thread's event counters (kCounterSlots words), so a 128-thread
    // block does not hold a 256-thread allocation and the rest of the SM's
    // L1 stays with the cascade stacks.  The counters live there rather than
    // in registers, which the octree walk needs: a shared-memory atomic add
    // per event costs one instruction, as a register increment does.
    extern __shared__ float leaf_cache[];
    const dev::LeafCache cache{leaf_cache + threadIdx.x, int(blockDim.x)};
    cache.f(0) = 0.0f;   // location 0: empty
    cache.f(1) = 0.0f;
    uint32_t* const cnt = reinterpret_cast<uint32_t*>(leaf_cache + kLeafCacheWords * blockDim.x) + threadIdx.x;
    const int cs = int(blockDim.x);
#pragma unroll
    for (int k = 0; k < kCounterSlots; ++k) cnt[k * cs] = 0u;
    auto bump = [&](int slot) { atomicAdd(cnt + slot * cs, 1u); };
    constexpr bool kExtra = (Mode == kModeSample);
    constexpr bool kNet = (Mode == kModeLearned);                   // tensor-core inference at birth
    constexpr bool kW = (Mode == kModeLearned || Mode == kModeWeighted);   // weighted electrons
    bool use_net = false, use_rule = false;
    int rule_k = 0;
    if constexpr (kW) {
        // the fixed (distance, energy) rule at birth, when set, replaces the network
        use_rule = a.birth_survival > 0.0f && a.birth_survival < 1.0f;
        rule_k = use_rule ? max(1, min(a.max_roulette_exp, int(rintf(-__log2f(a.birth_survival))))) : 0;
        // the network (or its importance table) is only consulted when its
        // answer can change something
        const bool can_act = a.cost_bins > 0 || a.rr_threshold > 0.0f || a.split_threshold < 1.0f;
        if constexpr (kNet) {
            use_net = !use_rule && a.mlp_params != nullptr && can_act;
            if (use_net) mlp::load_weights(g_lsm.w, a.mlp_params);
            __syncthreads();
        } else {
            use_net = !use_rule && a.imp_table != nullptr && can_act;
        }
    }
    const uint32_t n_in = min(*a.n_in, a.in_capacity);
    dev::Electron e;
    // Child-first depth-first cascade: when an event creates a secondary the
    // parent is parked here and the secondary is simulated at once, so the
    // stack only ever holds the current electron's ancestors.
    dev::Electron stack[kLocalStack];
    const ParkedStack ps{a.stack_mem ? a.stack_mem + (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * 3 * a.stack_depth
                                     : nullptr};
    const int depth = a.stack_mem ? a.stack_depth : kLocalStack;
    Extra ex{-1, 0u, 0u};
    Extra exs[kExtra ? kMaxStack : 1];
    int wexp = 0;   // learned mode: the current electron's weight is 2^wexp
    int sp = 0;
    bool alive = false, drained = false;
    uint32_t probe = 0;   // ranges this thread has found used up (range_cursor)
    uint32_t carry_hit = 0;
    // Per-thread tallies in 32 bits (a thread would need 2^32 steps in one
    // launch to wrap): the frequent ones in the shared-memory slots above,
    // the weighted, sample and deposit modes' own in registers; rare ones
    // (dropped records, queue overflow) go straight to the global counters.
    uint32_t c_inf = 0, c_kill = 0, c_split = 0, c_smp = 0, c_dep = 0, c_dep_drop = 0;
    // Deposit mode: this thread's current chunk [dep_pos, dep_end) of the
    // record buffer, taken kDepositChunk records at a time with one atomic.
    unsigned long long dep_pos = 0, dep_end = 0;
    bool dep_full = false;
    // Hand an electron to the next generation's queue (warp-aggregated push
    // over the lanes that push together).
    auto push_next = [&](const dev::Electron& x, int x_wexp) {
        cg::coalesced_group g = cg::coalesced_threads();
        uint32_t base = 0;
        if (g.thread_rank() == 0) base = atomicAdd(a.out_tail, g.size());
        base = g.shfl(base, 0);
        const uint32_t slot = base + g.thread_rank();
        if (slot < a.out_capacity) {
            store_electron(a.out, slot, x);
            if constexpr (kW) {
                if (x_wexp != 0) a.out.c[slot].w = kWeightTag | (uint32_t(x_wexp) & 0xFFu);
            }
        } else {
            atomicAdd(a.counters + kCntOverflow, 1ull);
        }
    };
    for (;;) {
        if (!alive && !drained) {
            if (sp > 0) {
                ps.get<kW>(--sp, e, stack, wexp);
                if constexpr (kExtra) {
                    ex = exs[sp];
                    ex.flags |= carry_hit;
                    carry_hit = 0;
                }
                alive = true;
            } else {
                uint32_t idx = 0;
                bool got = false;
                if (a.range_cursor) {
                    // this SM's range first, then the following ranges
                    const uint32_t nb = a.n_ranges;
                    uint32_t smid;
                    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
                    while (probe < nb) {
                        uint32_t v = smid % nb + probe;
                        if (v >= nb) v -= nb;
                        const cg::coalesced_group g = cg::coalesced_threads();
                        const cg::coalesced_group part = cg::labeled_partition(g, int(v));
                        uint32_t base = 0;
                        if (part.thread_rank() == 0) base = atomicAdd(a.range_cursor + v, part.size());
                        base = part.shfl(base, 0);
                        const uint32_t lo = uint32_t(uint64_t(n_in) * v / nb);
                        const uint32_t hi = uint32_t(uint64_t(n_in) * (v + 1) / nb);
                        const uint32_t off = base + part.thread_rank();
                        if (off < hi - lo) {
                            idx = lo + off;
                            got = true;
                            break;
                        }
                        ++probe;
                    }
                } else {
                    cg::coalesced_group g = cg::coalesced_threads();
                    uint32_t base = 0;
                    if (g.thread_rank() == 0) base = atomicAdd(a.head, g.size());
                    base = g.shfl(base, 0);
                    idx = base + g.thread_rank();
                    got = idx < n_in;
                }
                if (!got) {
                    drained = true;
                } else {
                    load_electron(a.in, idx, e);
                    if constexpr (kW) {
                        wexp = 0;
                        if ((uint32_t(e.last_tri) & 0xFFFFFF00u) == kWeightTag) {
                            wexp = int(int8_t(uint32_t(e.last_tri) & 0xFFu));
                            e.last_tri = -1;
                        }
                    }
                    if constexpr (kExtra) {
                        ex.rec = -1;
                        ex.flags = 0;
                        carry_hit = 0;
                    }
                    bump(kSlotPopped);
                    alive = true;
                }
            }
        }
        if constexpr (kNet) {
            // the whole warp stays in the loop until all its lanes are done
            // (the tensor-core call at birth needs every lane)
            if (__all_sync(0xffffffffu, !alive)) break;
        } else {
            if (!alive) break;
        }
        if constexpr (Mode == kModeSample) {
            // one in sixteen electrons is recorded at its birth (step 0) in a
            // material: features now; label and sub-cascade cost when it ends
            if (ex.rec < 0 && e.step == 0 && e.mat >= 0 && (mix32(e.uid) & 15u) == 0) {
                const uint32_t slot = atomicAdd(a.sample_count, 1u);
                if (slot < a.sample_capacity) {
                    float f[6];
                    const dev::V3 d = dev::normalised(dev::V3{e.dx, e.dy, e.dz});
                    dev::electron_features(a.smap, e.px, e.py, e.pz, d.x, d.y, d.z, logf(e.E), e.mat, f);
#pragma unroll
                    for (int k = 0; k < 6; ++k) a.sample_feat[size_t(slot) * 6 + k] = f[k];
                    ex.rec = int(slot);
                    ex.c0 = cnt[kSlotSteps * cs];
                    ++c_smp;
                }
            }
        }
        int ev = dev::kEvNone;
        bool has_se = false;
        dev::Electron se;
        int st = dev::kAlive;
        [[maybe_unused]] const float E_before = e.E;
        if (!kNet || alive) {
            st = dev::step<Penn>(P, e, &ev, &se, &has_se, cache);
            bump(kSlotSteps);
        }
        // Learned mode: birth decision for every newborn secondary of the warp
        // (k > 0 roulette at survival 2^-k, -1 split, 0 keep; drop = lost the
        // roulette).  The network scores the warp's candidates together: they
        // are packed into the first rows of the warp's feature tile and one
        // (up to 16 candidates) or two m-tiles go through the tensor cores.
        int bk = 0;
        bool drop = false;
        if constexpr (kW) {
            const bool cand = has_se && !dev::ends_at_init(P, se);
            if (use_rule) {
                // roulette up to the rule's weight 2^rule_k: a newborn that
                // already carries it (its ancestor survived the rule) is kept
                if (cand && wexp < rule_k && se.E < a.birth_max_energy &&
                    dev::surface_distance(a.smap, se.px, se.py, se.pz) >= a.birth_min_distance)
                    bk = rule_k - wexp;
            } else if (use_net) {
                if constexpr (kNet) {
                    const unsigned m = __ballot_sync(0xffffffffu, cand);
                    if (m) {
                        const float logit =
                            birth_logit(m, cand, a.smap, se.px, se.py, se.pz, se.dx, se.dy, se.dz, se.E, se.mat);
                        if ((threadIdx.x & 31) == 0) ++c_inf;
                        if (cand) bk = birth_decision(a, mlp::sigmoid(logit), wexp, se.E, se.mat);
                    }
                } else if (cand) {
                    ++c_inf;
                    bk = birth_decision(a, table_importance(a, se), wexp, se.E, se.mat);
                }
            }
            if (bk > 0) {
                // Russian roulette: survive with probability 2^-bk at weight
                // 2^(wexp + bk); the draw is the secondary's own birth block
                if (wexp + bk > kMaxWeightExp) bk = kMaxWeightExp - wexp;
                if (bk > 0 && !(ldexpf(dev::u01(dev::draw(P.seed, se, kBirthBlock).x), bk) < 1.0f)) drop = true;
            } else if (bk < 0 && wexp <= kMinWeightExp) {
                bk = 0;   // the lineage is already split as far as it may be
            }
            if constexpr (kNet) {
                if (!alive) continue;
            }
        }
        if constexpr (Mode == kModeDeposit) {
            // energydeposit_cpu_driver::simulate_to_end (drivers/cpu/
            // energydeposit_cpu_driver.h:74-96): scattering events only, and
            // only when the energy changed; position after the event.
            if ((ev == dev::kEvElastic || ev == dev::kEvInelastic) && e.E != E_before) {
                if (dep_pos == dep_end && !dep_full) {
                    const unsigned long long base = atomicAdd(a.dep_cursor, (unsigned long long)kDepositChunk);
                    if (base + kDepositChunk <= a.dep_capacity) {
                        dep_pos = base;
                        dep_end = base + kDepositChunk;
                    } else {
                        dep_full = true;
                    }
                }
                if (dep_pos < dep_end) {
                    float* r = a.dep + dep_pos * kDepositWords;
                    r[0] = e.px;
                    r[1] = e.py;
                    r[2] = e.pz;
                    r[3] = E_before;
                    r[4] = E_before - e.E;
                    r[5] = __uint_as_float(e.tag);
                    ++dep_pos;
                    ++c_dep;
                } else {
                    ++c_dep_drop;
                }
            }
        }
        bump(ev);   // slots 1-3 count the event types; slot 0 (no event) is not read
        if (has_se) {
            // an inelastic step never ends its electron: st == kAlive here
            bump(kSlotSecondaries);
            if (drop) {
                ++c_kill;   // the secondary's sub-cascade is not simulated
            } else if (dev::ends_at_init(P, se)) {
                // The secondary's first step would only terminate it (about a
                // quarter of them start below the barrier): tally that step
                // here instead of parking the parent for it.
                bump(kSlotSteps);
                bump(kSlotTerminated);
            } else {
                // the newborn's weight exponent: roulette survivors gain bk,
                // both halves of a split lose one
                const int se_wexp = wexp + (bk < 0 ? -1 : bk);
                if (bk < 0) {
                    // split: the twin takes its own random streams
                    dev::Electron twin = se;
                    twin.uid = dev::secondary_uid(se.uid ^ 0x5DEECE66Dull, 0u);
                    ++c_split;
                    if (sp + 1 < depth) {
                        ps.put<kW>(sp, e, stack, wexp);
                        ps.put<kW>(sp + 1, twin, stack, se_wexp);
                        sp += 2;
                        e = se;
                        wexp = se_wexp;
                        continue;
                    }
                    push_next(twin, se_wexp);
                }
                if (sp < depth) {
                    ps.put<kW>(sp, e, stack, wexp);
                    if constexpr (kExtra) exs[sp] = ex;
                    ++sp;
                    e = se;
                    wexp = se_wexp;
                    if constexpr (kExtra) {
                        ex.rec = -1;
                        ex.flags = 0;
                    }
                    continue;
                }
                // Deep cascade: hand the secondary to the next generation.
                push_next(se, se_wexp);
            }
        }
        if (st == dev::kAlive) {
            if (!dev::ends_at_init(P, e)) continue;
            // The next init pass would only end the electron (energy below
            // the barrier, or it left the domain): tally that step now.
            bump(kSlotSteps);
            st = dev::kTerminated;
        }
        alive = false;
        uint32_t hit = 0;
        if (st == dev::kTerminated) {
            bump(kSlotTerminated);
        } else {
            // detected
            const bool is_se = e.E < 50;
            hit = is_se ? 1u : 0u;
            bump(is_se ? kSlotDetectedSE : kSlotDetectedBSE);
            [[maybe_unused]] const float wt = kW ? ldexpf(1.0f, wexp) : 1.0f;
            if (e.tag < a.n_tags) {
                atomicAdd(is_se ? a.se_count + e.tag : a.bse_count + e.tag, 1u);
                if constexpr (kW) atomicAdd(is_se ? a.se_w + e.tag : a.bse_w + e.tag, wt);
            }
            if (a.hist) {
                int bin = dev::floor_to_int(e.E * a.inv_bin_width);
                bin = bin < 0 ? 0 : (bin >= a.n_bins ? a.n_bins - 1 : bin);
                atomicAdd(a.hist + bin, 1ull);
            }
            if (a.pix_spec && e.tag < a.n_map) {
                // per-pixel exit spectrum; energies past the last bin are not binned
                const uint32_t px = a.pixel_of_tag[e.tag];
                const int bin = dev::floor_to_int(e.E * a.pix_inv_width);
                if (px < a.n_pixels && bin >= 0 && bin < a.pix_bins) atomicAdd(a.pix_spec + size_t(px) * a.pix_bins + bin, wt);
            }
            if (a.rec) {
                const uint32_t slot = atomicAdd(a.rec_count, 1u);
                if (slot < a.rec_capacity) {
                    a.rec[2 * size_t(slot)] = make_float4(e.px, e.py, e.pz, e.dx);
                    a.rec[2 * size_t(slot) + 1] = make_float4(e.dy, e.dz, e.E, __uint_as_float(e.tag));
                } else {
                    atomicAdd(a.counters + kCntRecordsDropped, 1ull);
                }
            }
        }
        if constexpr (Mode == kModeSample) {
            const uint32_t sub = (ex.flags | hit) & 1u;
            if (ex.rec >= 0) {
                a.sample_label[ex.rec] = float(sub);
                if (a.sample_cost) a.sample_cost[ex.rec] = float(cnt[kSlotSteps * cs] - ex.c0);
            }
            carry_hit = sub;
        }
    }
    if constexpr (Mode == kModeDeposit) {
        // mark the unused tail of this thread's last chunk
        for (; dep_pos < dep_end; ++dep_pos) a.dep[dep_pos * kDepositWords + 5] = __uint_as_float(kDepositEmpty);
    }
    // Counters: one atomic per warp per counter.
    unsigned long long v[kNumCounters];
    v[kCntSteps] = cnt[kSlotSteps * cs];
    v[kCntElastic] = cnt[dev::kEvElastic * cs];
    v[kCntInelastic] = cnt[dev::kEvInelastic * cs];
    v[kCntBoundary] = cnt[dev::kEvBoundary * cs];
    v[kCntSecondaries] = cnt[kSlotSecondaries * cs];
    v[kCntDetected] = cnt[kSlotDetectedSE * cs] + cnt[kSlotDetectedBSE * cs];
    v[kCntDetectedSE] = cnt[kSlotDetectedSE * cs];
    v[kCntDetectedBSE] = cnt[kSlotDetectedBSE * cs];
    v[kCntTerminated] = cnt[kSlotTerminated * cs];
    v[kCntRecordsDropped] = 0;
    v[kCntOverflow] = 0;
    v[kCntPopped] = cnt[kSlotPopped * cs];
    v[kCntInferences] = c_inf;
    v[kCntRouletteKilled] = c_kill;
    v[kCntSplit] = c_split;
    v[kCntSamples] = c_smp;
    v[kCntDeposits] = c_dep;
    v[kCntDepositsDropped] = c_dep_drop;
    __syncwarp();
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < kNumCounters; ++i) {
        const unsigned long long s = warp_sum(v[i]);
        if (lane == 0 && s) atomicAdd(a.counters + i, s);
    }
}

// Each thread answers kRaysPerThread consecutive rays, carrying its leaf
// cache from one to the next (a spatially coherent batch exercises the
// cached descent; any batch must give the reference's answers).
constexpr int kRaysPerThread = 8;
__global__ void __launch_bounds__(128) ray_query_kernel(const dev::Geometry g, const float* pos, const float* dir,
                                                        const float* dist, const int32_t* ignore_tri,
                                                        const int32_t* ignore_mat, uint64_t n, float* out_dist,
                                                        int32_t* out_tri) {
    __shared__ float leaf_cache[13 * 128];
    const dev::LeafCache cache{leaf_cache + threadIdx.x, int(blockDim.x)};
    cache.f(0) = 0.0f;
    cache.f(1) = 0.0f;
    const uint64_t first = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) * kRaysPerThread;
    for (uint64_t i = first; i < n && i < first + kRaysPerThread; ++i) {
        int hit;
        const dev::V3 p{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const dev::V3 d{dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
        out_dist[i] = dev::propagate(g, p, d, dist[i], ignore_tri[i], ignore_mat[i], &hit, cache);
        out_tri[i] = hit;
    }
}

__global__ void table_query_kernel(const dev::Material m, int table, const float* x, const float* y, uint64_t n,
                                   float* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        float r;
        switch (table) {
        case 0: r = dev::table1d_get(m.el_imfp, x[i]); break;
        case 1: r = dev::table2d_get(m.el_icdf, x[i], y[i]); break;
        case 2: r = dev::table1d_get(m.in_imfp, x[i]); break;
        case 3: r = dev::table2d_get(m.in_icdf, x[i], y[i]); break;
        default: r = dev::table2d_rounddown(m.ion, x[i], y[i]); break;
        }
        out[i] = r;
    }
}

__global__ void table3_query_kernel(const dev::Material m, int table, const float* x, const float* y, const float* z,
                                    uint64_t n, float* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = table == 0 ? dev::table3d_get(m.q, x[i], y[i], z[i]) : dev::table3d_rounddown(m.ion3, x[i], y[i], z[i]);
}

__global__ void philox_kernel(const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint4 c = make_uint4(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]);
        const uint4 r = dev::philox4x32_10(c, make_uint2(key[2 * i], key[2 * i + 1]));
        out[4 * i] = r.x;
        out[4 * i + 1] = r.y;
        out[4 * i + 2] = r.z;
        out[4 * i + 3] = r.w;
    }
}

// 56-byte nbx_electron record
struct ElectronRecord {
    float pos[3];
    float dir[3];
    float E;
    int32_t mat;
    int32_t last_tri;
    uint32_t tag;
    uint64_t uid;
    uint32_t step;
    uint32_t pad;
};
static_assert(sizeof(ElectronRecord) == 56, "nbx_electron layout");

__device__ __forceinline__ dev::Electron from_record(const ElectronRecord& r) {
    dev::Electron e;
    e.px = r.pos[0];
    e.py = r.pos[1];
    e.pz = r.pos[2];
    e.dx = r.dir[0];
    e.dy = r.dir[1];
    e.dz = r.dir[2];
    e.E = r.E;
    e.mat = r.mat;
    e.last_tri = r.last_tri;
    e.tag = r.tag;
    e.uid = r.uid;
    e.step = r.step;
    return e;
}
__device__ __forceinline__ void to_record(const dev::Electron& e, ElectronRecord& r) {
    r.pos[0] = e.px;
    r.pos[1] = e.py;
    r.pos[2] = e.pz;
    r.dir[0] = e.dx;
    r.dir[1] = e.dy;
    r.dir[2] = e.dz;
    r.E = e.E;
    r.mat = e.mat;
    r.last_tri = e.last_tri;
    r.tag = e.tag;
    r.uid = e.uid;
    r.step = e.step;
    r.pad = 0;
}

__global__ void step_query_kernel(const dev::Physics P, ElectronRecord* el, uint64_t n, int32_t* status,
                                  int32_t* event, ElectronRecord* ses, int32_t* has_se) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        dev::Electron e = from_record(el[i]);
        dev::Electron se{};
        int ev;
        bool hs;
        status[i] = P.penn ? dev::step<true>(P, e, &ev, &se, &hs) : dev::step<false>(P, e, &ev, &se, &hs);
        event[i] = ev;
        has_se[i] = hs ? 1 : 0;
        to_record(e, el[i]);
        if (hs) to_record(se, ses[i]);
    }
}

// se_w / bse_w (learned mode): per-tag weighted detections used instead of
// the counts, so the sums are of per-primary weighted yields and their squares.
// Tags of a scan are usually numbered pixel by pixel, so the lanes of a warp
// mostly share a pixel: they are grouped by pixel and each group adds its
// sums with one set of atomics.
__global__ void pixel_yields_kernel(const uint32_t* se, const uint32_t* bse, const float* se_w, const float* bse_w,
                                    const uint32_t* pixel_of_tag, uint64_t n_tags, uint64_t n_pixels, double* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n_tags;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t p = pixel_of_tag[i];
        if (p >= n_pixels) continue;
        const double s = se_w ? double(se_w[i]) : double(se[i]), b = bse_w ? double(bse_w[i]) : double(bse[i]);
        const cg::coalesced_group grp = cg::labeled_partition(cg::coalesced_threads(), p);
        const double n_sum = cg::reduce(grp, 1.0, cg::plus<double>());
        const double s_sum = cg::reduce(grp, s, cg::plus<double>());
        const double s2_sum = cg::reduce(grp, s * s, cg::plus<double>());
        const double b_sum = cg::reduce(grp, b, cg::plus<double>());
        const double b2_sum = cg::reduce(grp, b * b, cg::plus<double>());
        if (grp.thread_rank() == 0) {
            double* o = out + 5 * size_t(p);
            atomicAdd(o + 0, n_sum);
            if (s_sum != 0) {
                atomicAdd(o + 1, s_sum);
                atomicAdd(o + 2, s2_sum);
            }
            if (b_sum != 0) {
                atomicAdd(o + 3, b_sum);
                atomicAdd(o + 4, b2_sum);
            }
        }
    }
}

// Face records: e1 x e2 computed with the transport's arithmetic (the same
// expression propagate and boundary would evaluate) and both materials packed
// as 16-bit halves.
__global__ void triangle_faces_kernel(const float4* tri, float4* face, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 b = tri[3 * i + 1], c = tri[3 * i + 2];
        const dev::V3 nrm = dev::cross(dev::V3{b.x, b.y, b.z}, dev::V3{c.x, c.y, c.z});
        const uint32_t mi = uint32_t(__float_as_int(tri[3 * i].w)), mo = uint32_t(__float_as_int(b.w));
        face[i] = make_float4(nrm.x, nrm.y, nrm.z, __uint_as_float((mo << 16) | (mi & 0xFFFFu)));
    }
}

__global__ void fill_queue_kernel(Queue q, const float* particles, const uint32_t* tags, uint64_t uid_base, uint64_t n,
                                  uint64_t offset) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const float* p = particles + 7 * i;
        const uint64_t uid = uid_base + i;
        const uint64_t s = offset + i;
        q.a[s] = make_float4(p[0], p[1], p[2], p[6]);
        q.b[s] = make_float4(p[3], p[4], p[5], __int_as_float(dev::kVacuum));
        q.c[s] = make_uint4(tags[i], uint32_t(uid), uint32_t(uid >> 32), 0xFFFFFFFFu);
    }
}

// One word set on the device: a run's queue length goes into its control
// block this way rather than by a host-to-device copy, which could wait
// behind a staged batch's copy on the same copy engine.
__global__ void set_word_kernel(uint32_t* p, uint32_t v) { *p = v; }

// Largest of n tags into *out (zeroed by the caller).
__global__ void max_tag_kernel(const uint32_t* v, uint64_t n, uint32_t* out) {
    uint32_t m = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        m = max(m, v[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

int grid_for(uint64_t n, int block) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t need = (n + block - 1) / block;
    const uint64_t cap = uint64_t(sms) * 16;
    return int(need < cap ? (need > 0 ? need : 1) : cap);
}

}  // namespace

// Dynamic shared memory of transport_kernel: per thread, the leaf cache and
// the event counters.
static size_t transport_smem_bytes(int block) {
    return size_t(kLeafCacheWords + kCounterSlots) * sizeof(float) * size_t(block);
}

// Shared-memory carveout that just fits the blocks the registers allow on an
// SM, so the rest of the unified L1 caches what the transport gathers
// (octree words, triangles, tables) and the register spills.  Left to itself
// the driver may pick a larger carveout.  Applied once per (kernel, block
// size, device); the occupancy is checked afterwards and the default restored
// if the hint would cost resident blocks.
template <typename Kernel>
static void fit_carveout(Kernel kernel, int block) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    const void* key = reinterpret_cast<const void*>(kernel);
    const int tag = block * 64 + dev;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& d : done)
        if (d.first == key && d.second == tag) return;
    done.emplace_back(key, tag);
    const size_t dyn = transport_smem_bytes(block);
    int before = 0, after = 0, smem_sm = 0;
    cudaFuncAttributes fa{};
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&before, kernel, block, dyn) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        before <= 0 || smem_sm <= 0) {
        cudaGetLastError();
        return;
    }
    // per resident block: dynamic + static shared memory + 1 KB the runtime reserves
    const size_t need = size_t(before) * (dyn + fa.sharedSizeBytes + 1024);
    const int pct = int(std::min<size_t>(100, (need * 100 + size_t(smem_sm) - 1) / size_t(smem_sm)));
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&after, kernel, block, dyn) != cudaSuccess || after < before) {
        cudaGetLastError();
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, -1);
        cudaGetLastError();
    }
}

template <int Mode, bool Penn>
static cudaError_t launch_mode(const dev::Physics& P, const TransportArgs& a, int grid, int block, int variant,
                               cudaStream_t s) {
    if (block <= 0 || block > (variant == 7 ? 128 : 256)) return cudaErrorInvalidValue;
    const size_t sm = transport_smem_bytes(block);
    switch (variant) {
    case 2: fit_carveout(transport_kernel<2, Mode, Penn>, block); break;
    case 4: fit_carveout(transport_kernel<4, Mode, Penn>, block); break;
    case 7: fit_carveout(transport_kernel<7, Mode, Penn>, block); break;
    default: fit_carveout(transport_kernel<3, Mode, Penn>, block); break;
    }
    switch (variant) {
    case 2: transport_kernel<2, Mode, Penn><<<grid, block, sm, s>>>(P, a); break;
    case 4: transport_kernel<4, Mode, Penn><<<grid, block, sm, s>>>(P, a); break;
    case 7: transport_kernel<7, Mode, Penn><<<grid, block, sm, s>>>(P, a); break;
    default: transport_kernel<3, Mode, Penn><<<grid, block, sm, s>>>(P, a); break;
    }
    return cudaGetLastError();
}

template <bool Penn>
static cudaError_t launch_model(const dev::Physics& P, const TransportArgs& a, int grid, int block, int variant,
                                cudaStream_t s, int mode) {
    if (mode == kModeSample) return launch_mode<kModeSample, Penn>(P, a, grid, block, variant, s);
    if (mode == kModeLearned) return launch_mode<kModeLearned, Penn>(P, a, grid, block, variant, s);
    if (mode == kModeDeposit) return launch_mode<kModeDeposit, Penn>(P, a, grid, block, variant, s);
    if (mode == kModeWeighted) return launch_mode<kModeWeighted, Penn>(P, a, grid, block, variant, s);
    return launch_mode<kModePlain, Penn>(P, a, grid, block, variant, s);
}

cudaError_t launch_transport(const dev::Physics& P, const TransportArgs& a, int grid, int block, int variant,
                             cudaStream_t s, int mode) {
    return P.penn ? launch_model<true>(P, a, grid, block, variant, s, mode)
                  : launch_model<false>(P, a, grid, block, variant, s, mode);
}

template <int Mode>
static int max_blocks_mode(int block, int variant) {
    int n = 0;
    cudaError_t e;
    const size_t sm = transport_smem_bytes(block);
    switch (variant) {
    // both models share launch bounds and shared memory, hence occupancy
    case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_kernel<2, Mode, false>, block, sm); break;
    case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_kernel<4, Mode, false>, block, sm); break;
    case 7: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_kernel<7, Mode, false>, block, sm); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, transport_kernel<3, Mode, false>, block, sm); break;
    }
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

int transport_max_blocks_per_sm(int block, int variant, int mode) {
    if (mode == kModeSample) return max_blocks_mode<kModeSample>(block, variant);
    if (mode == kModeLearned) return max_blocks_mode<kModeLearned>(block, variant);
    if (mode == kModeDeposit) return max_blocks_mode<kModeDeposit>(block, variant);
    if (mode == kModeWeighted) return max_blocks_mode<kModeWeighted>(block, variant);
    return max_blocks_mode<kModePlain>(block, variant);
}

namespace {
__global__ void build_surface_map_kernel(const float4* tri, const uint32_t* brick_start, const int32_t* brick_tris,
                                         int nbx, int nby, int brick, float4* map, float lox, float loy, float loz,
                                         float cell, int nx, int ny, int nz, float d_max) {
    const uint64_t n = uint64_t(nx) * ny * nz;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const int ix = int(i % nx), iy = int((i / nx) % ny), iz = int(i / (uint64_t(nx) * ny));
        const float px = lox + (ix + 0.5f) * cell, py = loy + (iy + 0.5f) * cell, pz = loz + (iz + 0.5f) * cell;
        const uint64_t b = (uint64_t(iz / brick) * nby + iy / brick) * nbx + ix / brick;
        float best = d_max * d_max;
        int bi = -1;
        for (uint32_t k = __ldg(brick_start + b), end = __ldg(brick_start + b + 1); k < end; ++k) {
            const int ti = __ldg(brick_tris + k);
            const float d2 = dev::dist2_to_triangle(tri, ti, px, py, pz);
            if (d2 < best) {
                best = d2;
                bi = ti;
            }
        }
        float4 rec = make_float4(0.0f, 0.0f, 0.0f, -1.0f);   // no surface within d_max
        if (bi >= 0) {
            // distance to the nearest point q and the unit vector from q to
            // the centre; at a centre on the surface, the triangle's normal
            const float4 a = tri[3 * bi], e1 = tri[3 * bi + 1], e2 = tri[3 * bi + 2];
            float qx, qy, qz;
            dev::closest_point_on_triangle(px, py, pz, a, e1, e2, &qx, &qy, &qz);
            const float gx = px - qx, gy = py - qy, gz = pz - qz;
            const float d = sqrtf(gx * gx + gy * gy + gz * gz);
            if (d > 0.0f) {
                rec = make_float4(gx / d, gy / d, gz / d, d);
            } else {
                const float nxv = e1.y * e2.z - e1.z * e2.y, nyv = e1.z * e2.x - e1.x * e2.z,
                            nzv = e1.x * e2.y - e1.y * e2.x;
                const float inv = rsqrtf(nxv * nxv + nyv * nyv + nzv * nzv + 1e-30f);
                rec = make_float4(nxv * inv, nyv * inv, nzv * inv, 0.0f);
            }
        }
        map[i] = rec;
    }
}

__global__ void features_kernel(const dev::SurfaceMap S, const ElectronRecord* el, uint64_t n, float* out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const ElectronRecord& r = el[i];
        const dev::V3 d = dev::normalised(dev::V3{r.dir[0], r.dir[1], r.dir[2]});
        float f[6];
        dev::electron_features(S, r.pos[0], r.pos[1], r.pos[2], d.x, d.y, d.z, logf(r.E), r.mat, f);
        for (int k = 0; k < 6; ++k) out[6 * i + k] = f[k];
    }
}
}  // namespace

cudaError_t launch_triangle_faces(const float4* tri, float4* face, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    triangle_faces_kernel<<<grid_for(uint64_t(n), 256), 256, 0, s>>>(tri, face, n);
    return cudaGetLastError();
}

cudaError_t launch_build_surface_map(const float4* tri, const uint32_t* brick_start, const int32_t* brick_tris,
                                     int nbx, int nby, int brick, float4* map, float lox, float loy, float loz,
                                     float cell, int nx, int ny, int nz, float d_max, cudaStream_t s) {
    const uint64_t n = uint64_t(nx) * ny * nz;
    if (n == 0) return cudaSuccess;
    build_surface_map_kernel<<<grid_for(n, 128), 128, 0, s>>>(tri, brick_start, brick_tris, nbx, nby, brick, map, lox,
                                                              loy, loz, cell, nx, ny, nz, d_max);
    return cudaGetLastError();
}

cudaError_t launch_features(const dev::SurfaceMap& S, const void* electrons, uint64_t n, float* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    features_kernel<<<grid_for(n, 128), 128, 0, s>>>(S, static_cast<const ElectronRecord*>(electrons), n, out);
    return cudaGetLastError();
}

cudaError_t launch_ray_query(const dev::Geometry& g, const float* pos, const float* dir, const float* dist,
                             const int32_t* ignore_tri, const int32_t* ignore_mat, uint64_t n, float* out_dist,
                             int32_t* out_tri, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint64_t threads = (n + kRaysPerThread - 1) / kRaysPerThread;
    const int blocks = int((threads + 127) / 128);
    ray_query_kernel<<<blocks, 128, 0, s>>>(g, pos, dir, dist, ignore_tri, ignore_mat, n, out_dist, out_tri);
    return cudaGetLastError();
}

cudaError_t launch_table_query(const dev::Material& m, int table, const float* x, const float* y, uint64_t n,
                               float* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    table_query_kernel<<<grid_for(n, 256), 256, 0, s>>>(m, table, x, y, n, out);
    return cudaGetLastError();
}

cudaError_t launch_table3_query(const dev::Material& m, int table, const float* x, const float* y, const float* z,
                                uint64_t n, float* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    table3_query_kernel<<<grid_for(n, 256), 256, 0, s>>>(m, table, x, y, z, n, out);
    return cudaGetLastError();
}

cudaError_t launch_philox(const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    philox_kernel<<<grid_for(n, 256), 256, 0, s>>>(ctr, key, n, out);
    return cudaGetLastError();
}

cudaError_t launch_step_query(const dev::Physics& P, void* electrons, uint64_t n, int32_t* status, int32_t* event,
                              void* secondaries, int32_t* has_se, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    step_query_kernel<<<grid_for(n, 128), 128, 0, s>>>(P, static_cast<ElectronRecord*>(electrons), n, status, event,
                                                        static_cast<ElectronRecord*>(secondaries), has_se);
    return cudaGetLastError();
}

cudaError_t launch_pixel_yields(const uint32_t* se, const uint32_t* bse, const float* se_w, const float* bse_w,
                                const uint32_t* pixel_of_tag, uint64_t n_tags, uint64_t n_pixels, double* out,
                                cudaStream_t s) {
    if (n_tags == 0) return cudaSuccess;
    pixel_yields_kernel<<<grid_for(n_tags, 256), 256, 0, s>>>(se, bse, se_w, bse_w, pixel_of_tag, n_tags, n_pixels,
                                                              out);
    return cudaGetLastError();
}

cudaError_t launch_set_word(uint32_t* p, uint32_t v, cudaStream_t s) {
    set_word_kernel<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError();
}

cudaError_t launch_max_tag(const uint32_t* tags, uint64_t n, uint32_t* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    max_tag_kernel<<<grid_for(n, 256), 256, 0, s>>>(tags, n, out);
    return cudaGetLastError();
}

cudaError_t launch_fill_queue(Queue q, const float* particles, const uint32_t* tags, uint64_t uid_base, uint64_t n,
                              uint64_t offset, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    fill_queue_kernel<<<grid_for(n, 256), 256, 0, s>>>(q, particles, tags, uid_base, n, offset);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free transport for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host application whose own caching
// allocator already owns the device memory, or a pipeline that must not let
// an allocation's implicit device synchronisation stall its streams.  For
// them, nbx_run_noalloc runs the same transport kernel with its scratch
// (primary queue, two overflow queues for deep cascades, per-generation
// cursors, counters) carved from the file-scope array below: at most
// kNoAllocMaxPrimaries primaries per call, about 9.5 MB that every GPU which
// loads this library holds until the process exits.  Host code cannot use the
// array's name as a device address: the caller looks the address up with
// noalloc_scratch_address (cudaGetSymbolAddress, with the device current) and
// passes it in.  The array is shared by all calls and keeps the last call's
// contents; each call clears the cursors and counters it needs.  Calls that
// overlap on the GPU race on the array and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocOverflow = 1u << 16;
constexpr int kNoAllocGenerations = 256;
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kQueueBytes(size_t n) { return align256(n * 16) * 2 + align256(n * 16); }
constexpr size_t kOffPrim = 0;
constexpr size_t kOffOv0 = kOffPrim + kQueueBytes(kNoAllocMaxPrimaries);
constexpr size_t kOffOv1 = kOffOv0 + kQueueBytes(kNoAllocOverflow);
constexpr size_t kOffCtl = kOffOv1 + kQueueBytes(kNoAllocOverflow);
constexpr size_t kOffCnt = kOffCtl + align256(sizeof(uint32_t) * (2 * kNoAllocGenerations + 2));
constexpr size_t kNoAllocScratchBytes = kOffCnt + align256(sizeof(unsigned long long) * kNumCounters);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

Queue carve_queue(unsigned char* base, size_t off, size_t n) {
    Queue q;
    q.a = reinterpret_cast<float4*>(base + off);
    q.b = reinterpret_cast<float4*>(base + off + align256(n * 16));
    q.c = reinterpret_cast<uint4*>(base + off + 2 * align256(n * 16));
    return q;
}
}  // namespace

cudaError_t noalloc_scratch_address(void** out) {
    *out = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(out, g_noalloc_scratch);
    if (e != cudaSuccess) *out = nullptr;
    return e;
}

int run_transport_noalloc(const dev::Physics& P, int grid, int block, int variant, cudaStream_t s, void* scratch,
                          const float* d_particles,
                          const uint32_t* d_tags, uint32_t n, uint64_t uid_base, uint32_t* d_se, uint32_t* d_bse,
                          uint64_t n_tags, uint64_t counts[4], const char** err) {
    *err = "";
    if (n > kNoAllocMaxPrimaries) {
        *err = "nbx_run_noalloc takes at most NBX_NOALLOC_MAX_PRIMARIES primaries per call";
        return -1;
    }
    if (!scratch) {
        *err = "no device address for the transport scratch";
        return -3;
    }
    unsigned char* base = static_cast<unsigned char*>(scratch);
    uint32_t* ctl = reinterpret_cast<uint32_t*>(base + kOffCtl);
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base + kOffCnt);
    const Queue prim = carve_queue(base, kOffPrim, kNoAllocMaxPrimaries);
    const Queue ov[2] = {carve_queue(base, kOffOv0, kNoAllocOverflow), carve_queue(base, kOffOv1, kNoAllocOverflow)};
    auto fail = [&](const char* what) {
        *err = what;
        return -3;
    };
    if (cudaMemsetAsync(ctl, 0, sizeof(uint32_t) * (2 * kNoAllocGenerations + 2), s) != cudaSuccess ||
        cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * kNumCounters, s) != cudaSuccess)
        return fail("clearing the transport scratch failed");
    if (n == 0) {
        if (counts) counts[0] = counts[1] = counts[2] = counts[3] = 0;
        return cudaStreamSynchronize(s) == cudaSuccess ? 0 : fail("stream synchronisation failed");
    }
    const uint32_t n_prim = n;
    if (launch_set_word(ctl + 2 * kNoAllocGenerations, n_prim, s) != cudaSuccess)
        return fail("writing the primary count failed");
    fill_queue_kernel<<<grid_for(n, 256), 256, 0, s>>>(prim, d_particles, d_tags, uid_base, n, 0);
    if (cudaGetLastError() != cudaSuccess) return fail("queue fill launch failed");

    TransportArgs a{};
    a.se_count = d_se;
    a.bse_count = d_bse;
    a.n_tags = n_tags;
    a.counters = cnt;
    a.out_capacity = uint32_t(kNoAllocOverflow);
    int g = 0;
    for (;;) {
        for (int k = 0; k < 8 && g < kNoAllocGenerations; ++k, ++g) {
            a.in = g == 0 ? prim : ov[(g - 1) % 2];
            a.in_capacity = uint32_t(g == 0 ? kNoAllocMaxPrimaries : kNoAllocOverflow);
            a.out = ov[g % 2];
            a.n_in = g == 0 ? ctl + 2 * kNoAllocGenerations : ctl + kNoAllocGenerations + (g - 1);
            a.head = ctl + g;
            a.out_tail = ctl + kNoAllocGenerations + g;
            if (launch_transport(P, a, grid, block, variant, s) != cudaSuccess) return fail("transport launch failed");
        }
        uint32_t last = 0;
        if (cudaMemcpyAsync(&last, ctl + kNoAllocGenerations + (g - 1), 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail("transport failed");
        if (last == 0) break;
        if (g >= kNoAllocGenerations) {
            *err = "secondary generations exceed the allocation-free limit";
            return -8;
        }
    }
    unsigned long long c[kNumCounters];
    if (cudaMemcpyAsync(c, cnt, sizeof(c), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return fail("reading counters failed");
    if (counts) {
        counts[0] = c[kCntElastic];
        counts[1] = c[kCntInelastic];
        counts[2] = c[kCntBoundary];
        counts[3] = c[kCntDetected];
    }
    if (c[kCntOverflow]) {
        *err = "overflow queue of the allocation-free transport is full: electrons lost";
        return -8;
    }
    return 0;
}

}  // namespace nbx
