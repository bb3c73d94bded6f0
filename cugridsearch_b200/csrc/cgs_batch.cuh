// cgs_batch.cuh -- the persistent batch kernel: many image pairs of uneven sizes, each with
// its own grid and cost, in one launch.
//
// Work.  Every pair's grid is cut into tasks of the plan's points-per-task (run_task); the
// tasks of all pairs form one global sequence, pair after pair in the order the host chose
// (cheapest pair first, so pairs finish early and the costliest tasks do not trail), and the
// persistent CTAs take tasks from it through an atomic counter.  Each CTA keeps one producer
// thread (thread 0) kStages chunks ahead of its consumers: when the producer passes the last
// chunk of a task it takes the next task from the counter, records it in a small ring in
// shared memory and starts that task's fixed-image chunk copies, so the bulk copies of a pair
// overlap the tail of the previous task even across pairs.  The ring has kRing entries; the
// producer is at most kStages chunks (hence kStages + 1 tasks) ahead, so an entry is never
// rewritten before the consumers have read it, and every ring write precedes at least one
// CTA barrier before its read.
//
// Completion.  A pair's last task (the one that completes its task count) writes its decoded
// argmin.  Optional per-pair time stamps (globaltimer) record the start of the pair's first
// task and the end of its last.
//
// Faults.  A bounded wait that gives up makes its CTA retire, with the timeout status, the
// task it was running, the tasks queued in its ring and every task still in the counter, so
// every pair still gets a result (with status CGS_ERROR_DEVICE_TIMEOUT where work was lost).
#pragma once
#include "cgs_kernels.cuh"

namespace cgs {

constexpr uint32_t kEndTask = 0xffffffffu;
constexpr int kRing = 4;

struct BatchParams {
    const SearchParams *pairs;   // [n_pairs], device
    const uint32_t *task_begin;  // [n_pairs + 1]: first global task of each pair; [n_pairs] = total
    uint32_t n_pairs, total_tasks;
    unsigned int *next_task;     // task counter, zero at launch
    unsigned long long *t_start; // [n_pairs] first task start (globaltimer ns), all ones at launch; or null
    unsigned long long *t_end;   // [n_pairs] last task end, zero at launch; or null
    int32_t stage_floats;        // stage capacity: the largest chunk of any pair
};

// The pair of global task t: the largest i with task_begin[i] <= t (pairs without tasks have
// equal bounds and are skipped).
__device__ __forceinline__ uint32_t pair_of_task(const BatchParams &b, uint32_t t) {
    uint32_t lo = 0, hi = b.n_pairs;  // task_begin[lo] <= t < task_begin[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(b.task_begin + mid) <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Producer state, held by thread 0 of the CTA.
template <int C>
struct BatchProducer {
    const BatchParams *b;
    const CtaSmem *sm;
    uint2 *ring;        // shared [kRing]: {global task, pair}; task kEndTask ends the CTA's work
    uint32_t fetched;   // tasks taken from the counter (ring slot of the next one)
    uint32_t issued;    // chunk iterations issued
    uint32_t pair, chunk, nchunks;
    bool live;          // the cursor is on a task

    __device__ __forceinline__ void fetch() {
        const uint32_t t = atomicAdd(b->next_task, 1u);
        uint2 e = make_uint2(kEndTask, 0u);
        live = t < b->total_tasks;
        if (live) {
            pair = pair_of_task(*b, t);
            chunk = 0;
            nchunks = (uint32_t)b->pairs[pair].num_chunks;
            e = make_uint2(t, pair);
        }
        ring[fetched % kRing] = e;
        fetched++;
    }
    __device__ __forceinline__ void issue_next() {
        issue_chunk<C>(b->pairs[pair], *sm, issued++, (int)chunk);
        if (++chunk == nchunks) fetch();
    }
    __device__ __forceinline__ void after_chunk(uint32_t) {
        if (live) issue_next();
    }
};

// Register budget: 8 points per warp need more than 128 registers, so those plans allow one
// CTA of up to 8 warps per SM at 255 registers.
__host__ __device__ constexpr int batch_min_blocks(int G, int NW) {
    return ((G >= 8 ? 8 : 16) / NW) < 1 ? 1 : (G >= 8 ? 8 : 16) / NW;
}

// Points per warp of a pair under a plan of G: MI pairs take at most 2 (their histograms, one
// per point and warp, would not fit in shared memory at more), the other costs take the plan's
// G.  A cost's values do not depend on its points per warp.
__host__ __device__ constexpr int batch_pair_points(int cost, int G) {
    return cost == CGS_COST_MI ? (G < 2 ? G : 2) : G;
}

// Costs the batch kernel evaluates (each pair picks one).
__host__ __device__ constexpr bool batch_cost_supported(int cost) {
    return cost == CGS_COST_SAD_AVG || cost == CGS_COST_SQD_REF || cost == CGS_COST_NCC_REF ||
           cost == CGS_COST_ZNCC || cost == CGS_COST_MI;
}

template <int C, int G, int NW, bool BSPLIT>
__global__ void __launch_bounds__(NW * 32, batch_min_blocks(G, NW)) batch_kernel(const __grid_constant__ BatchParams b) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint2 ring[kRing];
    const CtaSmem sm = carve_smem<G, NW>(smem, b.stage_floats);
    BatchProducer<C> prod{&b, &sm, ring, 0u, 0u, 0u, 0u, 0u, false};
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&sm.bars[s], 1);
        fence_mbar_init();
        *sm.abort_flag = 0;
        prod.fetch();
        for (int s = 0; s < kStages && prod.live; s++) prod.issue_next();
    }
    __syncthreads();

    uint32_t it = 0;
    for (uint32_t k = 0;; k++) {
        const uint2 e = ring[k % kRing];
        if (e.x == kEndTask) break;
        const uint32_t pair = e.y;
        const SearchParams &p = b.pairs[pair];
        const uint32_t task = e.x - __ldg(b.task_begin + pair);
        if (threadIdx.x == 0 && b.t_start) atomicMin(b.t_start + pair, (unsigned long long)global_ns());
        bool ok = true;
        switch (p.cost) {
            case CGS_COST_SAD_AVG: ok = run_task<CGS_COST_SAD_AVG, C, G, NW, kTapsTexture, BSPLIT>(p, task, sm, it, prod); break;
            case CGS_COST_SQD_REF: ok = run_task<CGS_COST_SQD_REF, C, G, NW, kTapsTexture, BSPLIT>(p, task, sm, it, prod); break;
            case CGS_COST_NCC_REF: ok = run_task<CGS_COST_NCC_REF, C, G, NW, kTapsTexture, BSPLIT>(p, task, sm, it, prod); break;
            case CGS_COST_ZNCC:  // quads staged: taps from the pre-gathered quads
                ok = p.mov_quad ? run_task<CGS_COST_ZNCC, C, G, NW, kTapsQuad, BSPLIT>(p, task, sm, it, prod)
                                : run_task<CGS_COST_ZNCC, C, G, NW, kTapsTexture, BSPLIT>(p, task, sm, it, prod);
                break;
            default: {  // CGS_COST_MI: the host admits only batch_cost_supported() costs
                constexpr int GM = batch_pair_points(CGS_COST_MI, G);
                ok = run_task<CGS_COST_MI, C, GM, NW, kTapsLoads, BSPLIT>(p, task, sm, it, prod);
                break;
            }
        }
        if (!ok) {
            if (threadIdx.x == 0) {
                // retire the task in hand, the tasks queued behind it, and all tasks not yet taken
                for (uint32_t j = k; j < prod.fetched; j++) {
                    const uint2 q = ring[j % kRing];
                    if (q.x != kEndTask) retire_tasks(b.pairs[q.y], ~0ull, 1u, true);
                }
                if (prod.live) {
                    for (;;) {
                        const uint32_t t = atomicAdd(b.next_task, 1u);
                        if (t >= b.total_tasks) break;
                        retire_tasks(b.pairs[pair_of_task(b, t)], ~0ull, 1u, true);
                    }
                }
            }
            return;
        }
        if (threadIdx.x == 0 && b.t_end) atomicMax(b.t_end + pair, (unsigned long long)global_ns());
    }
}

}  // namespace cgs

// Instantiates batch_kernel<1, G, NW, split> for NW in {4, 8, 16} and both splits.
#define CGS_DEFINE_BATCH_GETTER(NAME, GV)                                                      \
    namespace cgs {                                                                           \
    const void *NAME(int NW, bool bsplit) {                                                   \
        if (NW == 4) return bsplit ? (const void *)batch_kernel<1, GV, 4, true>                \
                                   : (const void *)batch_kernel<1, GV, 4, false>;              \
        if (NW == 8) return bsplit ? (const void *)batch_kernel<1, GV, 8, true>                \
                                   : (const void *)batch_kernel<1, GV, 8, false>;              \
        if (NW == 16) return bsplit ? (const void *)batch_kernel<1, GV, 16, true>              \
                                    : (const void *)batch_kernel<1, GV, 16, false>;            \
        return nullptr;                                                                       \
    }                                                                                         \
    }
