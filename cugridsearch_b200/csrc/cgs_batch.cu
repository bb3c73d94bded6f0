// cgs_batch.cu -- C ABI of the batched search: a handle that stages many image pairs, orders
// their tasks, holds a CUDA graph of one launch sequence -- clear, stage, the persistent batch
// kernel over the per-sample pairs, the multi-pair span kernel over the ZNCC pairs that
// cgs_search runs on its span kernel, and cgs_search's own launches for large MI pairs that it
// runs on the MI span kernel -- replays it, and tunes the persistent kernel's plan by timing
// candidates on a sample of every pair's grid.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cgs_batch.cuh"
#include "cgs_internal.h"

namespace cgs {

const void *batch_kernel_g1(int NW, bool bsplit);
const void *batch_kernel_g2(int NW, bool bsplit);
const void *batch_kernel_g4(int NW, bool bsplit);
const void *batch_kernel_g8(int NW, bool bsplit);

static const void *batch_kernel_for(const cgs_batch_plan &pl) {
    const bool bs = pl.block_split != 0;
    switch (pl.points_per_warp) {
        case 1: return batch_kernel_g1(pl.warps_per_block, bs);
        case 2: return batch_kernel_g2(pl.warps_per_block, bs);
        case 4: return batch_kernel_g4(pl.warps_per_block, bs);
        case 8: return batch_kernel_g8(pl.warps_per_block, bs);
        default: return nullptr;
    }
}

// Scratch words of a pair (the layout the search kernels and prep_body use): argmin key,
// task counter, status, max |moving pixel| (bytes 16-19), the ZNCC shifts (bytes 24-31).
constexpr size_t kHeaderBytes = 32;

// key = all ones, counter = status = 0 for n headers (a tuning run's fresh results).
__global__ void header_reset_kernel(char *headers, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    char *h = headers + (size_t)i * kHeaderBytes;
    *reinterpret_cast<unsigned long long *>(h) = ~0ull;
    *reinterpret_cast<unsigned int *>(h + 8) = 0u;
    *reinterpret_cast<unsigned int *>(h + 12) = 0u;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Span-kernel tasks per SM from which an MI pair (or a ZNCC pair outside the multi-pair span
// kernel's plan) is searched by its own span launches (CGS_BATCH_SPAN_TASKS_PER_SM overrides
// it; 0 routes every span-eligible pair).
constexpr uint32_t kSpanRouteTasksPerSm = 4;
static uint32_t span_route_tasks_per_sm() {
    const char *v = std::getenv("CGS_BATCH_SPAN_TASKS_PER_SM");
    if (!v || !*v) return kSpanRouteTasksPerSm;
    const long t = std::strtol(v, nullptr, 10);
    return t < 0 ? kSpanRouteTasksPerSm : (uint32_t)std::min<long>(t, 1L << 20);
}

// %globaltimer (ns) into *t: the start and end stamps of a pair searched by its own launches.
__global__ void stamp_kernel(unsigned long long *t) {
    unsigned long long v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    *t = v;
}

}  // namespace cgs

using namespace cgs;

// The handle.  Device memory is one block:
//   zeroed per launch:    headers [n x 32 B] | task counter (16 B) | t_end [n] | span task counter (16 B)
//   all ones per launch:  t_start [n]
//   per plan:             params [n] | task_begin [n + 1]
//   fixed:                prep params [n] | span pairs' params, task_begin, stamp slots, staging
//                         arguments | staged planes (one tex_align-aligned block per pair) | span
//                         pairs' row prefix sums | own-launch pairs' scratch
//   tuning:               params [n] | task_begin [n + 1] | task counter | headers [n] | results [n]
// Pairs are kept in execution order (ascending estimated work); order[i] is the caller's index.
// Routes (execution order): 0 the persistent kernel, 1 the multi-pair span kernel, 2 the pair's
// own cgs_search launches.
struct cgs_batch {
    int dev = -1;
    int sms = 0;
    uint32_t n = 0;
    std::vector<uint32_t> order;
    std::vector<SearchParams> params;  // execution order, device pointers filled
    std::vector<int> mi_bins;
    int32_t stage_floats = 0;
    int64_t max_stage_elems = 0;
    char *mem = nullptr;
    size_t zero_off = 0, zero_bytes = 0, ones_off = 0, ones_bytes = 0;
    char *headers = nullptr;
    unsigned int *next_task = nullptr;
    unsigned long long *t_start = nullptr, *t_end = nullptr;
    SearchParams *d_params = nullptr;
    uint32_t *d_task_begin = nullptr;
    PrepParams *d_prep = nullptr;
    SearchParams *d_tparams = nullptr;
    uint32_t *d_ttask_begin = nullptr;
    unsigned int *t_next = nullptr;
    char *t_headers = nullptr;
    cgs_argmin *t_results = nullptr;
    std::vector<cudaTextureObject_t> tex;
    std::vector<uint8_t> route;
    // route 2: searched after the kernels by the same launches as cgs_search, in scratch of their own
    std::vector<cgs_pair> span_pair;
    std::vector<size_t> span_off, span_bytes;
    // route 1: the multi-pair span kernel's launch and staging step
    uint32_t g_n = 0, g_blocks = 0;
    int g_prep_blocks = 0;
    size_t g_smem = 0;
    const void *g_kfn = nullptr;
    SpanBatchParams g_args{};
    SpanPrepArgs *d_gprep = nullptr;
    cgs_batch_plan plan = {2, 16, 0, 0};
    uint32_t total_tasks = 0;
    uint32_t blocks = 0;
    int32_t kernel_nodes = 0;  // kernel launches per replay of the graph
    size_t smem = 0;
    const void *kfn = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t last = nullptr;
};

namespace cgs {

static void release(cgs_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaTextureObject_t t : b->tex)
        if (t) cudaDestroyTextureObject(t);
    if (b->mem) {  // back to the pool (kept there for the next batch), in the batch's stream order
        cudaFreeAsync(b->mem, b->cap);
        cudaStreamSynchronize(b->cap);
    }
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->last) cudaEventDestroy(b->last);
    delete b;
}

static bool plan_valid(const cgs_batch_plan &pl) {
    const bool g = pl.points_per_warp == 1 || pl.points_per_warp == 2 || pl.points_per_warp == 4 ||
                   pl.points_per_warp == 8;
    const bool w = pl.warps_per_block == 4 || pl.warps_per_block == 8 || pl.warps_per_block == 16;
    return g && w && (pl.block_split == 0 || pl.block_split == 1);
}

// Kernel shape of a plan over the batch's pairs: per-pair task counts (of at most `cap`
// points each when cap > 0), shared memory, resident CTAs.  Fails with UNSUPPORTED when the
// plan does not fit an SM.
struct Shape {
    std::vector<uint32_t> tasks;
    uint32_t total = 0;
    size_t smem = 0;
    uint32_t blocks = 0;
    const void *kfn = nullptr;
};

static cgs_status plan_shape(const cgs_batch &b, const cgs_batch_plan &pl, uint32_t cap, Shape *sh) {
    if (!plan_valid(pl)) return fail(CGS_ERROR_INVALID_VALUE, "batch plan: points_per_warp 1/2/4/8, warps_per_block 4/8/16, block_split 0/1");
    const int G = pl.points_per_warp, NW = pl.warps_per_block;
    const bool bs = pl.block_split != 0;
    size_t acc = 0;
    sh->tasks.assign(b.n, 0u);
    uint64_t total = 0;
    for (uint32_t i = 0; i < b.n; i++) {
        if (b.route[i]) continue;                               // searched by span kernels
        const int gi = batch_pair_points(b.params[i].cost, G);  // this pair's points per warp
        const uint32_t ppt = (uint32_t)(bs ? gi : gi * NW);     // points per task
        const uint32_t pts = cap ? std::min(cap, b.params[i].n) : b.params[i].n;
        sh->tasks[i] = (pts + ppt - 1) / ppt;
        total += sh->tasks[i];
        acc = std::max(acc, acc_bytes(b.params[i].cost, gi, NW, bs, b.mi_bins[i]));
    }
    if (total >= kEndTask) return fail(CGS_ERROR_GRID_TOO_LARGE, "batch has too many tasks for this plan");
    sh->total = (uint32_t)total;
    sh->smem = cta_smem_bytes(G, NW, (size_t)b.stage_floats * 4, acc);
    if (sh->smem > 227 * 1024) return fail(CGS_ERROR_UNSUPPORTED, "batch plan exceeds 227 KB of shared memory");
    sh->kfn = batch_kernel_for(pl);
    if (!sh->kfn) return fail(CGS_ERROR_UNSUPPORTED, "no batch kernel for this plan");
    CGS_CUDA(cudaFuncSetAttribute(sh->kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh->smem),
             "cudaFuncSetAttribute");
    CGS_CUDA(cudaFuncSetAttribute(sh->kfn, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxL1),
             "cudaFuncSetAttribute");
    int per_sm = 0;
    CGS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sh->kfn, NW * 32, sh->smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(CGS_ERROR_UNSUPPORTED, "batch plan does not fit on an SM");
    sh->blocks = std::max<uint32_t>(1u, std::min<uint32_t>(sh->total, (uint32_t)(b.sms * per_sm)));
    return CGS_SUCCESS;
}

static std::vector<uint32_t> prefix(const std::vector<uint32_t> &tasks) {
    std::vector<uint32_t> tb(tasks.size() + 1, 0u);
    for (size_t i = 0; i < tasks.size(); i++) tb[i + 1] = tb[i] + tasks[i];
    return tb;
}

static BatchParams batch_args(const cgs_batch &b, bool tuning, uint32_t total) {
    BatchParams a;
    a.pairs = tuning ? b.d_tparams : b.d_params;
    a.task_begin = tuning ? b.d_ttask_begin : b.d_task_begin;
    a.n_pairs = b.n;
    a.total_tasks = total;
    a.next_task = tuning ? b.t_next : b.next_task;
    a.t_start = tuning ? nullptr : b.t_start;
    a.t_end = tuning ? nullptr : b.t_end;
    a.stage_floats = b.stage_floats;
    return a;
}

// Stream work of one batch launch: clear the scratch words, stage every pair, run the kernel.
static cgs_status enqueue_launch(const cgs_batch &b, cudaStream_t s) {
    CGS_CUDA(cudaMemsetAsync(b.mem + b.zero_off, 0, b.zero_bytes, s), "cudaMemsetAsync");
    CGS_CUDA(cudaMemsetAsync(b.mem + b.ones_off, 0xff, b.ones_bytes, s), "cudaMemsetAsync");
    const unsigned px = (unsigned)std::max<int64_t>(1, std::min<int64_t>(64, (b.max_stage_elems + 255) / 256));
    const PrepParams *qs = b.d_prep;
    void *pargs[] = {&qs};
    CGS_CUDA(cudaLaunchKernel(batch_prep_kernel_fn(), dim3(px, b.n), dim3(256), pargs, 0, s), "batch_prep_kernel");
    // the multi-pair span kernel first: its pairs take the least time each, so running them
    // before the per-sample pairs lowers the pairs' completion times (the launch takes as long)
    if (b.g_n > 0) {
        CGS_CUDA(launch_span_prep_batch(b.d_gprep, (int)b.g_n, b.g_prep_blocks, s), "span_prep_batch_kernel");
        SpanBatchParams ga = b.g_args;
        void *gargs[] = {&ga};
        CGS_CUDA(cudaLaunchKernel(b.g_kfn, dim3(b.g_blocks), dim3(16 * 32), gargs, b.g_smem, s), "span_batch_kernel");
    }
    BatchParams a = batch_args(b, false, b.total_tasks);
    void *kargs[] = {&a};
    if (b.total_tasks > 0)
        CGS_CUDA(cudaLaunchKernel(b.kfn, dim3(b.blocks), dim3(b.plan.warps_per_block * 32), kargs, b.smem, s),
                 "batch_kernel");
    for (uint32_t j = 0; j < b.n; j++) {
        if (b.route[j] != 2) continue;
        stamp_kernel<<<1, 1, 0, s>>>(b.t_start + j);
        CGS_CUDA(cudaGetLastError(), "stamp_kernel");
        const cgs_status st = span_route_enqueue(b.span_pair[j], b.mem + b.span_off[j], b.span_bytes[j], s);
        if (st != CGS_SUCCESS) return fail(st, "pair " + std::to_string(b.order[j]) + ": " + cgs_last_error());
        stamp_kernel<<<1, 1, 0, s>>>(b.t_end + j);
        CGS_CUDA(cudaGetLastError(), "stamp_kernel");
    }
    return CGS_SUCCESS;
}

// Applies a plan: task counts and prefix, the device parameter array, and the launch graph.
static cgs_status apply_plan(cgs_batch *b, const cgs_batch_plan &pl) {
    Shape sh;
    cgs_status s;
    if ((s = plan_shape(*b, pl, 0, &sh)) != CGS_SUCCESS) return s;
    std::vector<SearchParams> ps = b->params;
    for (uint32_t i = 0; i < b->n; i++) ps[i].num_tasks = sh.tasks[i];
    const std::vector<uint32_t> tb = prefix(sh.tasks);
    CGS_CUDA(cudaStreamSynchronize(b->cap), "cudaStreamSynchronize");
    CGS_CUDA(cudaMemcpy(b->d_params, ps.data(), sizeof(SearchParams) * b->n, cudaMemcpyHostToDevice), "cudaMemcpy");
    CGS_CUDA(cudaMemcpy(b->d_task_begin, tb.data(), sizeof(uint32_t) * tb.size(), cudaMemcpyHostToDevice),
             "cudaMemcpy");
    b->plan = pl;
    b->total_tasks = sh.total;
    b->blocks = sh.blocks;
    b->smem = sh.smem;
    b->kfn = sh.kfn;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    CGS_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    s = enqueue_launch(*b, b->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (s != CGS_SUCCESS) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    b->graph = g;
    size_t nn = 0;
    CGS_CUDA(cudaGraphGetNodes(b->graph, nullptr, &nn), "cudaGraphGetNodes");
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) CGS_CUDA(cudaGraphGetNodes(b->graph, nodes.data(), &nn), "cudaGraphGetNodes");
    b->kernel_nodes = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        CGS_CUDA(cudaGraphNodeGetType(nd, &t), "cudaGraphNodeGetType");
        if (t == cudaGraphNodeTypeKernel) b->kernel_nodes++;
    }
    CGS_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
    return CGS_SUCCESS;
}

// Estimated work of a pair, for the execution order (pixel evaluations, MI weighted for its
// slower inner loop).
static double pair_work(const SearchParams &p) {
    const double w = p.cost == CGS_COST_MI ? 2.5 : 1.0;
    return w * (double)p.n * (double)p.fix.w * (double)p.fix.h;
}

}  // namespace cgs

extern "C" {

cgs_status cgs_batch_create(const cgs_pair *pairs, int32_t n, const cgs_batch_plan *plan, cgs_batch **out) {
    if (!out) return fail(CGS_ERROR_INVALID_VALUE, "out is null");
    *out = nullptr;
    if (!pairs || n < 1) return fail(CGS_ERROR_INVALID_VALUE, "a batch needs at least one pair");
    cgs_status s;

    // validate every pair and build its kernel parameters (host part), then its staging layout
    struct Pending {
        SearchParams p;
        Staging st;
        int mi_bins;
        int64_t stage_elems;
        bool quads = false;
        int route = 0;
        size_t span_bytes = 0;
        SpanPlan zp;         // route 1: the pair's span plan
        size_t prefix_off = 0;
    };
    SpanPlan gplan;          // the multi-pair span kernel's plan (of its first pair)
    bool have_group = false;
    std::vector<Pending> pend((size_t)n);
    for (int32_t i = 0; i < n; i++) {
        const cgs_pair &q = pairs[i];
        const std::string at = "pair " + std::to_string(i) + ": ";
        int mi_bins = 32;
        if ((s = check_request(&q.moving, &q.fixed, &q.grid, &q.options, &mi_bins)) != CGS_SUCCESS)
            return fail(s, at + cgs_last_error());
        if (!q.result) return fail(CGS_ERROR_INVALID_VALUE, at + "result is null");
        if (!batch_cost_supported(q.options.cost))
            return fail(CGS_ERROR_UNSUPPORTED, at + "the batch kernel evaluates SAD_AVG, SQD_REF, NCC_REF, ZNCC and MI");
        if (q.fixed.channels != 1) return fail(CGS_ERROR_UNSUPPORTED, at + "the batch kernel is single-channel");
        Pending &pd = pend[i];
        int64_t n64 = 0;
        if ((s = fill_params(&q.moving, &q.fixed, &q.grid, q.options, mi_bins, &pd.p, &n64)) != CGS_SUCCESS)
            return fail(s, at + cgs_last_error());
        if (n64 <= 0) return fail(CGS_ERROR_INVALID_VALUE, at + "the grid has no points");
        pd.mi_bins = mi_bins;
    }
    DeviceInfo di;
    if ((s = device_info(&di)) != CGS_SUCCESS) return s;
    const uint64_t route_tasks = (uint64_t)span_route_tasks_per_sm() * (uint64_t)di.sms;
    for (int32_t i = 0; i < n; i++) {
        const cgs_pair &q = pairs[i];
        Pending &pd = pend[i];
        // ZNCC pairs that cgs_search runs on its span kernel share one multi-pair span launch
        // (same kernel plan); other span-eligible pairs are searched by their own launches once
        // their grid fills the GPU by itself (a few tasks per SM), and stay in the persistent
        // kernel below that (a refinement level's local grids, balanced there many at once)
        uint32_t ppt = 0;
        if ((q.options.cost == CGS_COST_ZNCC || q.options.cost == CGS_COST_MI) &&
            span_route_bytes(q, &pd.span_bytes, &ppt)) {
            SpanPlan zp;
            const bool grouped = q.options.cost == CGS_COST_ZNCC && span_plan(q.moving, q.fixed, q.options, &zp) &&
                                 kernel_span_zncc_batch(zp.G, zp.NW, zp.TX, zp.check) != nullptr &&
                                 (!have_group || (zp.G == gplan.G && zp.NW == gplan.NW && zp.TX == gplan.TX &&
                                                  zp.TH == gplan.TH && zp.pitch_mod == gplan.pitch_mod));
            if (grouped) {
                pd.route = 1;
                pd.zp = zp;
                if (!have_group) gplan = zp;
                have_group = true;
            } else if ((uint64_t)pd.p.n >= route_tasks * ppt) {
                pd.route = 2;
            }
        }
        // ZNCC pairs of the persistent kernel on the fast sampling path read pre-gathered tap
        // quads, as single searches do
        const int fl = q.options.flags;
        pd.quads = pd.route == 1 || (pd.route == 0 && q.options.cost == CGS_COST_ZNCC &&
                                     ((fl & CGS_FLAG_QUAD_TAPS) ||
                                      (!exact_samples(CGS_COST_ZNCC, fl) && !(fl & CGS_FLAG_TEXTURE_TAPS))));
        pd.st = staging_layout(q.moving, q.fixed, di.tex_align, di.tex_pitch_align, false, false, pd.quads);
        set_chunks(&pd.p, pd.st, 1, q.fixed.height);
        pd.stage_elems = pd.st.mplane + pd.st.fplane;
    }

    cgs_batch *b = new cgs_batch();
    b->dev = di.dev;
    b->sms = di.sms;
    b->n = (uint32_t)n;
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0u);
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](uint32_t x, uint32_t y) { return pair_work(pend[x].p) < pair_work(pend[y].p); });

    // device layout
    const size_t un = (size_t)n;
    size_t off = 0;
    b->zero_off = off;
    const size_t hdr_off = off;
    off += un * kHeaderBytes;
    const size_t next_off = off;
    off += 16;
    const size_t tend_off = off;
    off += un * 8;
    const size_t gnext_off = off;
    off += 16;
    b->zero_bytes = off - b->zero_off;
    off = align_up(off, 256);
    b->ones_off = off;
    b->ones_bytes = un * 8;
    off += un * 8;
    off = align_up(off, 256);
    const size_t par_off = off;
    off = align_up(off + un * sizeof(SearchParams), 256);
    const size_t tb_off = off;
    off = align_up(off + (un + 1) * 4, 256);
    const size_t prep_off = off;
    off = align_up(off + un * sizeof(PrepParams), 256);
    const size_t tpar_off = off;
    off = align_up(off + un * sizeof(SearchParams), 256);
    const size_t ttb_off = off;
    off = align_up(off + (un + 1) * 4, 256);
    const size_t tnext_off = off;
    off += 256;
    const size_t thdr_off = off;
    off = align_up(off + un * kHeaderBytes, 256);
    const size_t tres_off = off;
    off = align_up(off + un * sizeof(cgs_argmin), 256);
    // the multi-pair span kernel's pairs: one shared-memory carve for all of them (the largest
    // tile count, one window stage size), as span_plan sizes it for one pair
    uint32_t gn = 0;
    int gtiles = 0;
    for (int32_t i = 0; i < n; i++)
        if (pend[i].route == 1) {
            gn++;
            gtiles = std::max(gtiles, pend[i].zp.tiles_x * pend[i].zp.tiles_y);
        }
    int gcap = 0;
    if (gn > 0) {
        const size_t budget = 227 * 1024;
        const size_t fixed = span_kernel_smem(gplan.G, gplan.NW, gplan.TH, gplan.TX, gtiles, 0);
        gcap = fixed + (size_t)kMinSpanCap * 32 > budget ? 0 : (int)((budget - fixed) / 32);
        gcap = std::max(gcap, kMinSpanCap + gplan.TH * 32 * gplan.TX / 4);
        const size_t gsm = span_kernel_smem(gplan.G, gplan.NW, gplan.TH, gplan.TX, gtiles, gcap);
        if (fixed + (size_t)kMinSpanCap * 32 > budget || gsm > budget) {
            for (int32_t i = 0; i < n; i++) pend[i].route = pend[i].route == 1 ? 0 : pend[i].route;
            gn = 0;  // cannot happen for the sizes span_plan admits; the pairs go to the persistent kernel
        }
    }
    const size_t gpar_off = off;
    off = align_up(off + gn * sizeof(SearchParams), 256);
    const size_t gtb_off = off;
    off = align_up(off + (gn + 1) * 4, 256);
    const size_t gslot_off = off;
    off = align_up(off + gn * 4, 256);
    const size_t gprep_off = off;
    off = align_up(off + gn * sizeof(SpanPrepArgs), (size_t)di.tex_align);
    std::vector<size_t> stage_off(un);
    for (uint32_t j = 0; j < b->n; j++) {
        stage_off[j] = off;
        off = align_up(off + pend[b->order[j]].st.bytes, (size_t)di.tex_align);
    }
    for (uint32_t j = 0; j < b->n; j++) {
        Pending &pd = pend[b->order[j]];
        if (pd.route != 1) continue;
        pd.prefix_off = off;
        const cgs_pair &q = pairs[b->order[j]];
        off = align_up(off + (size_t)q.fixed.height * (size_t)(q.fixed.width + 1) * sizeof(double2), 256);
    }
    off = align_up(off, (size_t)di.tex_align);
    b->route.assign(un, 0);
    b->span_pair.resize(un);
    b->span_off.assign(un, 0);
    b->span_bytes.assign(un, 0);
    for (uint32_t j = 0; j < b->n; j++) {
        const Pending &pd = pend[b->order[j]];
        b->route[j] = (uint8_t)pd.route;
        if (pd.route != 2) continue;
        b->span_pair[j] = pairs[b->order[j]];
        b->span_off[j] = off;
        b->span_bytes[j] = pd.span_bytes;
        off = align_up(off + pd.span_bytes, (size_t)di.tex_align);
    }
    const size_t total = off;

    // one block from the library's stream-ordered pool: batches created one after another (a
    // refinement loop) reuse its memory instead of mapping new memory each time
    cudaMemPool_t pool;
    if ((s = get_pool(di.dev, &pool)) != CGS_SUCCESS) {
        release(b);
        return s;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&b->mem), total, pool, b->cap);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->cap);
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "cudaMallocFromPoolAsync (batch)");
    }
    b->headers = b->mem + hdr_off;
    b->next_task = reinterpret_cast<unsigned int *>(b->mem + next_off);
    b->t_end = reinterpret_cast<unsigned long long *>(b->mem + tend_off);
    b->t_start = reinterpret_cast<unsigned long long *>(b->mem + b->ones_off);
    b->d_params = reinterpret_cast<SearchParams *>(b->mem + par_off);
    b->d_task_begin = reinterpret_cast<uint32_t *>(b->mem + tb_off);
    b->d_prep = reinterpret_cast<PrepParams *>(b->mem + prep_off);
    b->d_tparams = reinterpret_cast<SearchParams *>(b->mem + tpar_off);
    b->d_ttask_begin = reinterpret_cast<uint32_t *>(b->mem + ttb_off);
    b->t_next = reinterpret_cast<unsigned int *>(b->mem + tnext_off);
    b->t_headers = b->mem + thdr_off;
    b->t_results = reinterpret_cast<cgs_argmin *>(b->mem + tres_off);

    std::vector<PrepParams> preps(un);
    b->params.resize(un);
    b->mi_bins.resize(un);
    b->tex.assign(un, 0);
    std::vector<SearchParams> gpar;
    std::vector<uint32_t> gtasks, gslot;
    std::vector<SpanPrepArgs> gprep;
    for (uint32_t j = 0; j < b->n; j++) {
        const uint32_t i = b->order[j];
        const cgs_pair &q = pairs[i];
        Pending &pd = pend[i];
        SearchParams &p = pd.p;
        char *sb = b->headers + (size_t)j * kHeaderBytes;
        char *org = b->mem + stage_off[j];
        float *mstage = reinterpret_cast<float *>(org + pd.st.mov_off);
        float *fstage = reinterpret_cast<float *>(org + pd.st.fix_off);
        p.key = reinterpret_cast<unsigned long long *>(sb);
        p.done = reinterpret_cast<unsigned int *>(sb + 8);
        p.status = reinterpret_cast<unsigned int *>(sb + 12);
        p.vmax = reinterpret_cast<float *>(sb + 16);
        p.shifts = reinterpret_cast<const float *>(sb + 24);
        p.mov = Plane{mstage, q.moving.height, q.moving.width, 1, pd.st.mpitch, pd.st.mplane};
        p.fix = Plane{fstage, q.fixed.height, q.fixed.width, 1, pd.st.fpitch, pd.st.fplane};
        p.costs = q.costs;
        p.result = q.result;
        preps[j] = make_prep(&q.moving, &q.fixed, pd.st, sb, mstage, fstage);
        if (pd.quads) {
            p.mov_quad = reinterpret_cast<const float4 *>(org + pd.st.quad_off);
            p.quad_pitch = q.moving.width;
            p.quad_plane = pd.st.qplane;
            preps[j].quad_dst = reinterpret_cast<float4 *>(org + pd.st.quad_off);
            preps[j].qplane = pd.st.qplane;
        }
        // the staged moving plane as a (W + 1) x (H + 1) texture (point sampling, border 0)
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypePitch2D;
        rd.res.pitch2D.devPtr = mstage;
        rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
        rd.res.pitch2D.width = (size_t)q.moving.width + 1;
        rd.res.pitch2D.height = (size_t)q.moving.height + 1;
        rd.res.pitch2D.pitchInBytes = (size_t)pd.st.mpitch * 4;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        e = cudaCreateTextureObject(&b->tex[j], &rd, &td, nullptr);
        if (e != cudaSuccess) {
            release(b);
            return cuda_fail(e, "cudaCreateTextureObject");
        }
        p.mov_tex = b->tex[j];
        if (pd.route == 1) {
            // as cgs_search sets up its span kernel: quads in the span form with the moving
            // shift folded in, the fixed rows' prefix sums, tiles and the (common) window stage
            preps[j].quad_form = 1;
            double2 *prefix = reinterpret_cast<double2 *>(b->mem + pd.prefix_off);
            p.fix_prefix = prefix;
            p.tile_h = pd.zp.TH;
            p.tiles_x = pd.zp.tiles_x;
            p.tiles_y = pd.zp.tiles_y;
            p.win_cap = gcap;
            p.win_pitch_mod = pd.zp.pitch_mod;
            const uint32_t per_task = (uint32_t)(pd.zp.G * pd.zp.NW);
            p.num_tasks = (p.n + per_task - 1) / per_task;
            gpar.push_back(p);
            gtasks.push_back(p.num_tasks);
            gslot.push_back(j);
            SpanPrepArgs ga;
            int blocks = 0;
            span_prep_batch_args(fstage, pd.st.fpitch, q.fixed.width, q.fixed.height, prefix,
                                 reinterpret_cast<float4 *>(org + pd.st.quad_off), pd.st.qplane, p.shifts, &ga,
                                 &blocks);
            gprep.push_back(ga);
            b->g_prep_blocks = std::max(b->g_prep_blocks, blocks);
        }
        b->params[j] = p;
        b->mi_bins[j] = pd.mi_bins;
        if (pd.route == 0) b->stage_floats = std::max<int32_t>(b->stage_floats, p.chunk_rows * pd.st.fpitch);
        b->max_stage_elems = std::max<int64_t>(b->max_stage_elems, pd.stage_elems);
    }
    e = cudaMemcpy(b->d_prep, preps.data(), sizeof(PrepParams) * un, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->last, cudaEventDisableTiming);
    if (e == cudaSuccess && gn > 0) {
        // the multi-pair span kernel: its pairs, task prefix, stamp slots, staging arguments, launch shape
        const std::vector<uint32_t> gtb = prefix(gtasks);
        b->g_n = gn;
        b->d_gprep = reinterpret_cast<SpanPrepArgs *>(b->mem + gprep_off);
        SpanBatchParams &ga = b->g_args;
        ga.pairs = reinterpret_cast<const SearchParams *>(b->mem + gpar_off);
        ga.task_begin = reinterpret_cast<const uint32_t *>(b->mem + gtb_off);
        ga.slot = reinterpret_cast<const uint32_t *>(b->mem + gslot_off);
        ga.n_pairs = gn;
        ga.total_tasks = gtb[gn];
        ga.next_task = reinterpret_cast<unsigned int *>(b->mem + gnext_off);
        ga.t_start = b->t_start;
        ga.t_end = b->t_end;
        ga.tile_h = gplan.TH;
        ga.tiles = gtiles;
        ga.cap = gcap;
        b->g_kfn = kernel_span_zncc_batch(gplan.G, gplan.NW, gplan.TX, gplan.check);
        b->g_smem = span_kernel_smem(gplan.G, gplan.NW, gplan.TH, gplan.TX, gtiles, gcap);
        e = cudaMemcpy(b->mem + gpar_off, gpar.data(), sizeof(SearchParams) * gn, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->mem + gtb_off, gtb.data(), 4 * gtb.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->mem + gslot_off, gslot.data(), 4 * gn, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_gprep, gprep.data(), sizeof(SpanPrepArgs) * gn, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(b->g_kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->g_smem);
        int per_sm = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->g_kfn, 16 * 32, b->g_smem);
        if (e == cudaSuccess && per_sm < 1) e = cudaErrorInvalidConfiguration;
        b->g_blocks = std::max<uint32_t>(1u, std::min<uint32_t>(ga.total_tasks, (uint32_t)(di.sms * per_sm)));
    }
    if (e != cudaSuccess) {
        release(b);
        return cuda_fail(e, "batch setup");
    }
    cgs_batch_plan pl = {4, 16, 0, 0};
    if (plan) {
        pl = *plan;
    } else {
        // default: 4 points per warp (MI pairs take 2), 16 warps, warp-private MI histograms;
        // 2 points per warp, then block-shared histograms, where those do not fit
        Shape sh;
        if (plan_shape(*b, pl, 0, &sh) != CGS_SUCCESS) pl.points_per_warp = 2;
        if (plan_shape(*b, pl, 0, &sh) != CGS_SUCCESS) pl.block_split = 1;
    }
    if ((s = apply_plan(b, pl)) != CGS_SUCCESS) {
        const std::string msg = cgs_last_error();
        release(b);
        return fail(s, msg);
    }
    *out = b;
    return CGS_SUCCESS;
}

cgs_status cgs_batch_launch(cgs_batch *b, cgs_stream_t stream) {
    if (!b || !b->exec) return fail(CGS_ERROR_INVALID_VALUE, "batch is null");
    int dev = -1;
    CGS_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != b->dev) return fail(CGS_ERROR_INVALID_VALUE, "the batch was created on another device");
    CGS_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "cudaGraphLaunch");
    CGS_CUDA(cudaEventRecord(b->last, (cudaStream_t)stream), "cudaEventRecord");
    return CGS_SUCCESS;
}

cgs_status cgs_batch_set_plan(cgs_batch *b, const cgs_batch_plan *plan) {
    if (!b || !plan) return fail(CGS_ERROR_INVALID_VALUE, "batch or plan is null");
    CGS_CUDA(cudaEventSynchronize(b->last), "cudaEventSynchronize");
    return apply_plan(b, *plan);
}

cgs_status cgs_batch_get_plan(const cgs_batch *b, cgs_batch_plan *plan) {
    if (!b || !plan) return fail(CGS_ERROR_INVALID_VALUE, "batch or plan is null");
    *plan = b->plan;
    return CGS_SUCCESS;
}

cgs_status cgs_batch_kernel_launches(const cgs_batch *b, int32_t *n) {
    if (!b || !n) return fail(CGS_ERROR_INVALID_VALUE, "batch or output is null");
    *n = b->kernel_nodes;
    return CGS_SUCCESS;
}

cgs_status cgs_batch_pair_times(cgs_batch *b, uint64_t *start_ns, uint64_t *end_ns) {
    if (!b || !start_ns || !end_ns) return fail(CGS_ERROR_INVALID_VALUE, "batch or output is null");
    CGS_CUDA(cudaEventSynchronize(b->last), "cudaEventSynchronize");
    std::vector<unsigned long long> ts(b->n), te(b->n);
    CGS_CUDA(cudaMemcpy(ts.data(), b->t_start, 8 * b->n, cudaMemcpyDeviceToHost), "cudaMemcpy");
    CGS_CUDA(cudaMemcpy(te.data(), b->t_end, 8 * b->n, cudaMemcpyDeviceToHost), "cudaMemcpy");
    for (uint32_t j = 0; j < b->n; j++) {
        start_ns[b->order[j]] = ts[j];
        end_ns[b->order[j]] = te[j];
    }
    return CGS_SUCCESS;
}

cgs_status cgs_batch_autotune(cgs_batch *b, int32_t sample_points, cgs_tune_entry *entries, int32_t max_entries,
                              int32_t *n_entries, cgs_batch_plan *best) {
    if (!b) return fail(CGS_ERROR_INVALID_VALUE, "batch is null");
    if (n_entries) *n_entries = 0;
    const uint32_t cap = sample_points > 0 ? (uint32_t)sample_points : 4096u;
    cudaStream_t st = b->cap;
    cgs_status s;
    CGS_CUDA(cudaEventSynchronize(b->last), "cudaEventSynchronize");
    // stage the images once (the tuning runs read the staged planes and max |pixel|)
    {
        CGS_CUDA(cudaMemsetAsync(b->mem + b->zero_off, 0, b->zero_bytes, st), "cudaMemsetAsync");
        const unsigned px = (unsigned)std::max<int64_t>(1, std::min<int64_t>(64, (b->max_stage_elems + 255) / 256));
        const PrepParams *qs = b->d_prep;
        void *pargs[] = {&qs};
        CGS_CUDA(cudaLaunchKernel(batch_prep_kernel_fn(), dim3(px, b->n), dim3(256), pargs, 0, st),
                 "batch_prep_kernel");
    }
    // the tuning copy of the parameters: the first `cap` points of every grid, no cost dump,
    // results into tuning scratch
    std::vector<SearchParams> tp = b->params;
    for (uint32_t j = 0; j < b->n; j++) {
        char *sb = b->t_headers + (size_t)j * kHeaderBytes;
        tp[j].n = std::min(cap, tp[j].n);
        tp[j].key = reinterpret_cast<unsigned long long *>(sb);
        tp[j].done = reinterpret_cast<unsigned int *>(sb + 8);
        tp[j].status = reinterpret_cast<unsigned int *>(sb + 12);
        tp[j].costs = nullptr;
        tp[j].result = b->t_results + j;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CGS_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(CGS_ERROR_CUDA, "cudaEventCreate");
    }
    const int Gs[4] = {1, 2, 4, 8}, NWs[3] = {4, 8, 16};
    float best_ms = INFINITY;
    cgs_batch_plan best_plan = b->plan;
    int32_t ne = 0;
    s = CGS_SUCCESS;
    for (int bs = 0; bs < 2 && s == CGS_SUCCESS; bs++)
        for (int gi = 0; gi < 4 && s == CGS_SUCCESS; gi++)
            for (int wi = 0; wi < 3 && s == CGS_SUCCESS; wi++) {
                const cgs_batch_plan pl = {Gs[gi], NWs[wi], bs, 0};
                Shape sh;
                float ms = INFINITY;
                cgs_status cs = plan_shape(*b, pl, cap, &sh);
                if (cs == CGS_SUCCESS) {
                    for (uint32_t j = 0; j < b->n; j++) tp[j].num_tasks = sh.tasks[j];
                    const std::vector<uint32_t> tb = prefix(sh.tasks);
                    cudaError_t e = cudaStreamSynchronize(st);
                    if (e == cudaSuccess)
                        e = cudaMemcpy(b->d_tparams, tp.data(), sizeof(SearchParams) * b->n, cudaMemcpyHostToDevice);
                    if (e == cudaSuccess)
                        e = cudaMemcpy(b->d_ttask_begin, tb.data(), 4 * tb.size(), cudaMemcpyHostToDevice);
                    BatchParams a = batch_args(*b, true, sh.total);
                    void *kargs[] = {&a};
                    char *th = b->t_headers;
                    uint32_t nn = b->n;
                    void *rargs[] = {&th, &nn};
                    for (int rep = 0; rep < 3 && e == cudaSuccess; rep++) {  // one warm-up, two timed
                        e = cudaMemsetAsync(b->t_next, 0, 16, st);
                        if (e == cudaSuccess)
                            e = cudaLaunchKernel((const void *)header_reset_kernel, dim3((nn + 127) / 128), dim3(128),
                                                 rargs, 0, st);
                        if (e == cudaSuccess) e = cudaEventRecord(e0, st);
                        if (e == cudaSuccess)
                            e = cudaLaunchKernel(sh.kfn, dim3(sh.blocks), dim3(pl.warps_per_block * 32), kargs,
                                                 sh.smem, st);
                        if (e == cudaSuccess) e = cudaEventRecord(e1, st);
                        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                        float t = 0.0f;
                        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
                        if (e == cudaSuccess && rep > 0) ms = std::min(ms, t);
                    }
                    if (e != cudaSuccess) s = cuda_fail(e, "autotune run");
                    cs = s;
                }
                if (entries && ne < max_entries) entries[ne] = cgs_tune_entry{pl, ms, (int32_t)cs};
                ne++;
                if (cs == CGS_SUCCESS && ms < best_ms) {
                    best_ms = ms;
                    best_plan = pl;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_entries) *n_entries = std::min(ne, max_entries);
    if (s != CGS_SUCCESS) return s;
    if (!(best_ms < INFINITY)) return fail(CGS_ERROR_UNSUPPORTED, "no batch plan fits this batch");
    if (best) *best = best_plan;
    return apply_plan(b, best_plan);
}

cgs_status cgs_batch_destroy(cgs_batch *b) {
    if (!b) return CGS_SUCCESS;
    cudaEventSynchronize(b->last);
    cudaStreamSynchronize(b->cap);
    release(b);
    return CGS_SUCCESS;
}

cgs_status cgs_search_batched(const cgs_pair *pairs, int32_t n, const cgs_batch_plan *plan, cgs_stream_t stream) {
    cgs_batch *b = nullptr;
    cgs_status s = cgs_batch_create(pairs, n, plan, &b);
    if (s != CGS_SUCCESS) return s;
    s = cgs_batch_launch(b, stream);
    if (s == CGS_SUCCESS) {
        const cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) s = cuda_fail(e, "cudaStreamSynchronize");
    }
    cgs_batch_destroy(b);
    return s;
}

cgs_status cgs_autotune(const cgs_pair *pairs, int32_t n, int32_t sample_points, cgs_batch_plan *best) {
    if (!best) return fail(CGS_ERROR_INVALID_VALUE, "best is null");
    cgs_batch *b = nullptr;
    cgs_status s = cgs_batch_create(pairs, n, nullptr, &b);
    if (s != CGS_SUCCESS) return s;
    s = cgs_batch_autotune(b, sample_points, nullptr, 0, nullptr, best);
    cgs_batch_destroy(b);
    return s;
}

}  // extern "C"
