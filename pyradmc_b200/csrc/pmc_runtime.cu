// pmc_runtime.cu — the engine behind the C-ABI of include/pyradmc_b200.h.
//
// Host orchestration of WarpEngine.run / run_dij (pyradmc/backends/warp/
// engine.py:454-1572), re-planned for one resident B200 engine:
//   * uploads persist across calls; buffers grow on demand and are reused;
//   * a batch is one launch of a CUDA graph whose conditional WHILE node runs
//     [photon kernel -> electron kernel] until the device reports no work left
//     (the Warp engine read every queue count back to the host, engine.py:
//     2766-2831);
//   * the fold, finalize, truncation and CSC compaction (including its prefix
//     sum) run on the device; only the kept CSC entries cross to the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pyradmc_b200.h"
#include "../../include/pyradmc_b200_presolve.h"
#include "pmc_common.cuh"
#include "pmc_reduce.cuh"
#include "pmc_transport.cuh"

using namespace pmc;

namespace {

constexpr long long kDefaultMaxSteps = 10000000LL;  // per particle
constexpr long long kMaxRounds = 1000000LL;         // per batch

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// Launch shape of the primary generator and the two transport kernels.
struct LaunchShape {
    int grid_ph = 0, grid_el = 0, block = 0;
    int grid_gen = 0;                 // primary generator, blocks of 256
    bool smem = false;                // table rows staged in shared memory
    int occ = 0;                      // register-budget variant (0, 3 or 4)
    size_t smem_ph = 0, smem_el = 0;  // dynamic shared memory of each kernel
};

}  // namespace

struct pmc_engine {
    int device = 0;
    cudaStream_t stream = nullptr;        // the stream every call runs on
    cudaStream_t own_stream = nullptr;    // the engine's private stream
    std::string error;
    int sm_count = 0;

    // transport grid
    bool has_grid = false;
    int max_material = 0;
    GridInfo gi{};
    float2* d_vox = nullptr;
    size_t vox_cap = 0;           // bytes allocated behind d_vox (reused while large enough)
    double voxel_volume = 0.0;    // product of the float64 spacings of the grid
    DevBuf stage;                 // raw grid / GS arrays on their way to their packed form

    // scoring geometry
    GridInfo si{};
    int score_mode = 0;           // 0 rectilinear (si), 1 cylindrical (cyl)
    CylInfo cyl{};
    float* d_cyl_z = nullptr;
    float* d_cyl_r2 = nullptr;
    bool custom_scoring = false;
    double* d_mass = nullptr;
    size_t mass_cap = 0;
    long long mass_len = 0;

    // tables
    bool has_tables = false;
    bool has_gs = false;
    Tables tab{};
    std::vector<void*> table_allocs;
    float4* d_gs4 = nullptr;
    size_t gs_cap = 0;

    // transport buffers
    DevBuf q[4];
    unsigned int q_capacity = 0;
    DevBuf edep, s1, s2;          // [columns][col_stride] quanta and float64 sums
    DevBuf dirty, touched;        // sector bitmaps of edep / of the sums (pmc_reduce.cuh)
    bool edep_clean = false;      // every quanta entry is zero (true after a completed run)
    long long col_stride = 0;     // entries per column of the maps in the current call
    Sched* d_sched = nullptr;
    Counters* d_counters = nullptr;
    GenDesc* d_gen = nullptr;
    unsigned long long* d_total_q = nullptr;
    unsigned long long* d_colmax = nullptr;
    long long colmax_len = 0;
    DevBuf tile_counts, tile_offsets, col_counts, out_idx, out_dose, out_sigma, col_nhist;
    unsigned long long* d_nnz = nullptr;
    std::vector<DevBuf> run_pool;  // per-call generator arrays, reused across calls
    size_t run_used = 0;           // pool slots taken by the current call or group

    // graph of the drain loop
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    LaunchShape graph_shape;
    TransportParams graph_params{};

    // the CSC of the last Dij: indptr on the host, entries in out_* on the device
    std::vector<long long> dij_indptr;
    long long csc_nnz = 0;

    pmc_counters counters{};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> batch_ev;  // three per batch of a group, read once per group
    unsigned long long h2d_bytes = 0;  // cumulative over the engine's life
    unsigned long long d2h_bytes = 0;
    pmc_progress_fn progress = nullptr;
    void* progress_user = nullptr;
};

namespace {

int fail(pmc_engine* e, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (e) e->error = buf;
    return code;
}

#define PMC_CUDA(e, call)                                                                  \
    do {                                                                                   \
        cudaError_t _st = (call);                                                          \
        if (_st != cudaSuccess) {                                                          \
            return fail((e), _st == cudaErrorMemoryAllocation ? PMC_ERR_OOM : PMC_ERR_CUDA, \
                        "CUDA error %s at %s:%d: %s", cudaGetErrorName(_st), __FILE__,     \
                        __LINE__, cudaGetErrorString(_st));                                \
        }                                                                                  \
    } while (0)

int ensure(pmc_engine* e, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return PMC_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    PMC_CUDA(e, cudaMalloc(&b.p, std::max<size_t>(bytes, 16)));
    b.bytes = std::max<size_t>(bytes, 16);
    return PMC_OK;
}

// A device array behind a raw pointer, reallocated only when it must grow
// (a re-upload of the same grid, scoring grid or GS window reuses it).
template <typename T>
int ensure_ptr(pmc_engine* e, T*& p, size_t& cap, size_t bytes) {
    if (p && cap >= bytes) return PMC_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    PMC_CUDA(e, cudaMalloc((void**)&p, std::max<size_t>(bytes, 16)));
    cap = std::max<size_t>(bytes, 16);
    return PMC_OK;
}

// voxel (density, material bits) and, when mass is not null, the default
// scoring mass density * volume in float64 (the host arithmetic of the
// scorer: one correctly rounded product).
__global__ void pack_voxels_kernel(const float* density, const uint8_t* material, long long n,
                                   double volume, float2* vox, double* mass) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float d = density[i];
        vox[i] = make_float2(d, __int_as_float((int)material[i]));
        if (mass) mass[i] = __dmul_rn((double)d, volume);
    }
}

__global__ void mass_from_voxels_kernel(const float2* vox, long long n, double volume, double* mass) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        mass[i] = __dmul_rn((double)vox[i].x, volume);
}

// The four bilinear corners of every GS bin in one 16-byte row.
__global__ void pack_gs_kernel(const float* v, int n_eta, int n_t2, int n_u, float4* g4) {
    const long long cells = (long long)(n_eta - 1) * (n_t2 - 1) * n_u;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cells;
         c += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(c % n_u);
        const long long r = c / n_u;
        const int j = (int)(r % (n_t2 - 1)), i = (int)(r / (n_t2 - 1));
        auto at = [&](int a, int b) { return v[((long long)a * n_t2 + b) * n_u + u]; };
        g4[c] = make_float4(at(i, j), at(i + 1, j), at(i, j + 1), at(i + 1, j + 1));
    }
}

int grid_blocks(long long n) {
    const long long b = (n + 255) / 256;
    return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 16);
}

// A generator array for the current group: the next slot of a pool of device
// buffers kept across calls (grown only when too small), filled by a copy
// ordered on the engine's stream — after the kernels of the previous group
// that read the same slot — with no device-wide synchronization.  (A pageable
// source is staged before the call returns, so v may go away afterwards.)
template <typename T>
int upload_vec(pmc_engine* e, const std::vector<T>& v, const T** out) {
    if (e->run_used == e->run_pool.size()) e->run_pool.emplace_back();
    DevBuf& b = e->run_pool[e->run_used++];
    const size_t bytes = v.size() * sizeof(T);
    const int rc = ensure(e, b, bytes);
    if (rc) return rc;
    if (!v.empty()) PMC_CUDA(e, cudaMemcpyAsync(b.p, v.data(), bytes, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)bytes;
    *out = (const T*)b.p;
    return PMC_OK;
}

// At least n timing events for the batches of a group (created once, reused).
int ensure_batch_events(pmc_engine* e, size_t n) {
    while (e->batch_ev.size() < n) {
        cudaEvent_t ev = nullptr;
        PMC_CUDA(e, cudaEventCreate(&ev));
        e->batch_ev.push_back(ev);
    }
    return PMC_OK;
}

// The pool's slots are free for the next group (the buffers stay allocated).
void free_run_allocs(pmc_engine* e) { e->run_used = 0; }

void free_tables(pmc_engine* e) {
    for (void* p : e->table_allocs) cudaFree(p);
    e->table_allocs.clear();
    e->has_tables = false;
}

void destroy_graph(pmc_engine* e) {
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
    e->cond = 0;
}

GridInfo make_grid(int nx, int ny, int nz, const double o[3], const double s[3]) {
    // Bounds computed in float64 and stored as float32, as the Warp GridInfo
    // struct does (engine.py:3336-3345).
    GridInfo g{};
    g.x_lo = (float)o[0];
    g.y_lo = (float)o[1];
    g.z_lo = (float)o[2];
    g.x_hi = (float)(o[0] + nx * s[0]);
    g.y_hi = (float)(o[1] + ny * s[1]);
    g.z_hi = (float)(o[2] + nz * s[2]);
    g.sx = (float)s[0];
    g.sy = (float)s[1];
    g.sz = (float)s[2];
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.n_voxels = (long long)nx * ny * nz;
    return g;
}

constexpr int kDefaultTailSteps = 96;  // steps after a round runs dry before a particle is parked

// Kernel variants: tables in shared memory or not, and the register budget
// (resident blocks of 256 per SM: 0 = each kernel's default, else 3 or 4).
void* photon_fn(bool smem, int occ) {
    if (occ == 4) return smem ? (void*)photon_kernel<true, 4> : (void*)photon_kernel<false, 4>;
    return smem ? (void*)photon_kernel<true, 3> : (void*)photon_kernel<false, 3>;
}
void* electron_fn(bool smem, int occ) {
    if (occ == 3) return smem ? (void*)electron_kernel<true, 3> : (void*)electron_kernel<false, 3>;
    return smem ? (void*)electron_kernel<true, 4> : (void*)electron_kernel<false, 4>;
}

int transport_launch_shape(pmc_engine* e, const pmc_run_params* p, LaunchShape* L) {
    int bs = p->block_size > 0 ? p->block_size : 256;
    if (bs % 32 != 0 || bs > 256) return fail(e, PMC_ERR_INVALID, "block_size must be a multiple of 32 and <= 256");
    const size_t rows = (size_t)e->tab.n_materials * (size_t)e->tab.n_points;
    L->smem_ph = rows * sizeof(float4) + (size_t)e->tab.n_points * sizeof(float);
    L->smem_el = rows * (sizeof(float4) + sizeof(float2));
    // auto: stage when both kernels keep their register-limited residency
    // (one material at 2048 nodes: 40 KB and 48 KB per block)
    L->smem = p->smem_tables > 0 || (p->smem_tables == 0 && L->smem_ph <= 48 * 1024 && L->smem_el <= 48 * 1024);
    if (!L->smem) L->smem_ph = L->smem_el = 0;
    int max_smem = 0;
    PMC_CUDA(e, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, e->device));
    L->occ = (p->blocks_per_sm == 3 || p->blocks_per_sm == 4) ? p->blocks_per_sm : 0;
    if (L->smem && (L->smem_ph + 1024 > (size_t)max_smem || L->smem_el + 1024 > (size_t)max_smem))
        return fail(e, PMC_ERR_INVALID, "tables of %d materials do not fit shared memory; use smem_tables=-1",
                    e->tab.n_materials);
    PMC_CUDA(e, cudaFuncSetAttribute(photon_fn(L->smem, L->occ), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem_ph));
    PMC_CUDA(e, cudaFuncSetAttribute(electron_fn(L->smem, L->occ), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem_el));
    int per_sm_ph = 0, per_sm_el = 0;
    PMC_CUDA(e, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ph, photon_fn(L->smem, L->occ), bs, L->smem_ph));
    PMC_CUDA(e, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_el, electron_fn(L->smem, L->occ), bs, L->smem_el));
    if (p->blocks_per_sm > 0) {
        per_sm_ph = std::min(per_sm_ph, p->blocks_per_sm);
        per_sm_el = std::min(per_sm_el, p->blocks_per_sm);
    }
    per_sm_ph = std::max(per_sm_ph, 1);
    per_sm_el = std::max(per_sm_el, 1);
    int per_sm_gen = 0;
    PMC_CUDA(e, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_gen, generate_kernel, 256, 0));
    L->grid_gen = std::max(1, std::min(per_sm_gen, 4)) * e->sm_count;
    L->grid_ph = per_sm_ph * e->sm_count;
    L->grid_el = per_sm_el * e->sm_count;
    L->block = bs;
    return PMC_OK;
}

// The drain graph: WHILE(remaining) { generate_kernel; photon_kernel; electron_kernel }.
int build_graph(pmc_engine* e, const TransportParams& P, const LaunchShape& L) {
    destroy_graph(e);
    PMC_CUDA(e, cudaGraphCreate(&e->graph, 0));
    PMC_CUDA(e, cudaGraphConditionalHandleCreate(&e->cond, e->graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = e->cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    PMC_CUDA(e, cudaGraphAddNode(&cnode, e->graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];

    e->graph_params = P;
    void* args[] = {&e->graph_params};
    cudaKernelNodeParams kp{};
    kp.func = (void*)generate_kernel;
    kp.gridDim = dim3(L.grid_gen);
    kp.blockDim = dim3(256);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    cudaGraphNode_t n_gen, n_ph, n_el;
    PMC_CUDA(e, cudaGraphAddKernelNode(&n_gen, body, nullptr, 0, &kp));
    kp.func = photon_fn(L.smem, L.occ);
    kp.gridDim = dim3(L.grid_ph);
    kp.blockDim = dim3(L.block);
    kp.sharedMemBytes = (unsigned int)L.smem_ph;
    PMC_CUDA(e, cudaGraphAddKernelNode(&n_ph, body, &n_gen, 1, &kp));
    kp.func = electron_fn(L.smem, L.occ);
    kp.gridDim = dim3(L.grid_el);
    kp.sharedMemBytes = (unsigned int)L.smem_el;
    PMC_CUDA(e, cudaGraphAddKernelNode(&n_el, body, &n_ph, 1, &kp));
    PMC_CUDA(e, cudaGraphInstantiate(&e->graph_exec, e->graph, 0));
    e->graph_shape = L;
    return PMC_OK;
}

__global__ void init_batch_kernel(Sched* S, int batch, unsigned long long block_end,
                                  unsigned long long budget, long long max_rounds,
                                  unsigned long long cond) {
    S->p_in = 0;
    S->e_in = 0;
    for (int i = 0; i < 4; ++i) {
        S->count[i] = 0u;
        S->head[i] = 0u;
    }
    S->cursor = 0ull;
    S->block_end = block_end;
    S->budget = budget;
    S->limit = budget < block_end ? budget : block_end;
    S->blocks_done = 0u;
    S->remaining = 1;
    S->batch = batch;
    S->rounds = 0;
    S->max_rounds = max_rounds;
    S->cond_handle = cond;
}

struct SchedHost {
    Sched s;
};

int read_sched(pmc_engine* e, Sched* out) {
    PMC_CUDA(e, cudaMemcpyAsync(out, e->d_sched, sizeof(Sched), cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof(Sched));
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    return PMC_OK;
}

int check_flags(pmc_engine* e, const Sched& s) {
    if (s.flags & kFlagOverflow)
        return fail(e, PMC_ERR_QUEUE_OVERFLOW,
                    "particle queue overflow (capacity %u). Lower chunk_size or raise queue_factor.",
                    e->q_capacity);
    if (s.flags & kFlagStepCap)
        return fail(e, PMC_ERR_STEP_CAP,
                    "a particle exceeded the per-particle step cap; transport stopped early");
    if (s.flags & kFlagRoundCap)
        return fail(e, PMC_ERR_STEP_CAP, "a batch exceeded the transport round cap");
    return PMC_OK;
}

struct RunPlan {
    LaunchShape shape;
    unsigned long long budget = 0;
    long long max_steps = 0;
    int tail_steps = 0;
};

// max_block: the most primaries one batch block of this call holds; admission
// never needs more than that per round.
int prepare_transport(pmc_engine* e, const pmc_run_params* p, unsigned long long max_block,
                      RunPlan* plan) {
    if (!e->has_grid) return fail(e, PMC_ERR_STATE, "no transport grid uploaded");
    if (!e->has_tables) return fail(e, PMC_ERR_STATE, "no cross-section tables uploaded");
    if (p->msc_gs && !e->has_gs)
        return fail(e, PMC_ERR_STATE, "msc_model='gs' needs the Goudsmit-Saunderson grid");
    if (p->n_batches < 1) return fail(e, PMC_ERR_INVALID, "need at least one batch, got %d", p->n_batches);
    if (e->max_material >= e->tab.n_materials)
        return fail(e, PMC_ERR_INVALID, "material index %d beyond the cross-section source (%d materials)",
                    e->max_material, e->tab.n_materials);
    int rc = transport_launch_shape(e, p, &plan->shape);
    if (rc) return rc;
    const unsigned long long resident =
        (unsigned long long)std::max(plan->shape.grid_ph, plan->shape.grid_el) * plan->shape.block;
    plan->budget = p->chunk_size > 0 ? (unsigned long long)p->chunk_size : 16ull * resident;
    plan->budget = std::max(1ull, std::min(plan->budget, max_block));
    const int qf = p->queue_factor > 0 ? p->queue_factor : 16;
    const unsigned long long cap64 = plan->budget * (unsigned long long)qf;
    if (cap64 > 0x7fffffffull)
        return fail(e, PMC_ERR_INVALID, "chunk_size * queue_factor exceeds the queue index range");
    const unsigned int cap = (unsigned int)cap64;
    if (cap > e->q_capacity) {
        for (int i = 0; i < 4; ++i) {
            rc = ensure(e, e->q[i], (size_t)cap * sizeof(Slot));
            if (rc) return rc;
        }
        e->q_capacity = cap;
    }
    plan->max_steps = p->max_steps > 0 ? p->max_steps : kDefaultMaxSteps;
    plan->tail_steps = p->tail_steps > 0 ? p->tail_steps
                       : p->tail_steps < 0 ? 0x7fffffff : kDefaultTailSteps;
    return PMC_OK;
}

TransportParams make_params(pmc_engine* e, const pmc_run_params* p, const RunPlan& plan) {
    TransportParams P{};
    P.gi = e->gi;
    P.si = e->si;
    P.score_mode = e->score_mode;
    P.cyl = e->cyl;
    P.vox = e->d_vox;
    P.tab = e->tab;
    for (int i = 0; i < 4; ++i) P.q[i] = (Slot*)e->q[i].p;
    P.capacity = e->q_capacity;
    P.sched = e->d_sched;
    P.gen = e->d_gen;
    P.edep = (unsigned long long*)e->edep.p;
    P.dirty = (unsigned int*)e->dirty.p;
    P.col_stride = e->col_stride;
    P.counters = e->d_counters;
    P.seed_lo = (uint32_t)(p->seed & 0xffffffffull);
    P.seed_hi = (uint32_t)(p->seed >> 32);
    P.pcut = (float)p->pcut;
    P.ecut = (float)p->ecut;
    P.step_fraction = (float)p->step_energy_fraction;
    P.deposit_resolution = (float)p->deposit_resolution;
    P.transport_electrons = p->transport_electrons ? 1 : 0;
    P.msc_gs = p->msc_gs ? 1 : 0;
    P.dose_to_water = p->dose_to_water ? 1 : 0;
    P.split_n = p->photon_split_n > 1 ? p->photon_split_n : 1;
    P.max_steps = (int)std::min<long long>(plan.max_steps, 0x7ffffffeLL);
    P.tail_steps = plan.tail_steps;
    return P;
}

// Transport one statistical batch of the current group into e->edep.
int run_batch(pmc_engine* e, const pmc_run_params* p, const RunPlan& plan, TransportParams& P,
              int batch, unsigned long long block) {
    if (block == 0) return PMC_OK;
    const bool graph = p->use_graph != 0;
    if (graph) {
        const LaunchShape& g = e->graph_shape;
        const LaunchShape& L = plan.shape;
        const bool same = e->graph_exec && g.grid_ph == L.grid_ph && g.grid_el == L.grid_el &&
                          g.grid_gen == L.grid_gen &&
                          g.block == L.block && g.smem == L.smem && g.occ == L.occ &&
                          g.smem_ph == L.smem_ph &&
                          g.smem_el == L.smem_el &&
                          std::memcmp(&e->graph_params, &P, sizeof P) == 0;
        if (!same) {
            int rc = build_graph(e, P, L);
            if (rc) return rc;
        }
    }
    init_batch_kernel<<<1, 1, 0, e->stream>>>(e->d_sched, batch, block, plan.budget, kMaxRounds,
                                              graph ? (unsigned long long)e->cond : 0ull);
    PMC_CUDA(e, cudaGetLastError());
    e->counters.kernel_launches += 1;
    if (graph) {
        PMC_CUDA(e, cudaGraphLaunch(e->graph_exec, e->stream));
        e->counters.transport_launches += 1;
        return PMC_OK;
    }
    for (long long round = 0; round < kMaxRounds; ++round) {
        const LaunchShape& L = plan.shape;
        generate_kernel<<<L.grid_gen, 256, 0, e->stream>>>(P);
        void* args[] = {&P};
        PMC_CUDA(e, cudaLaunchKernel(photon_fn(L.smem, L.occ), dim3(L.grid_ph), dim3(L.block), args,
                                     L.smem_ph, e->stream));
        PMC_CUDA(e, cudaLaunchKernel(electron_fn(L.smem, L.occ), dim3(L.grid_el), dim3(L.block),
                                     args, L.smem_el, e->stream));
        PMC_CUDA(e, cudaGetLastError());
        e->counters.transport_launches += 3;
        Sched s;
        int rc = read_sched(e, &s);
        if (rc) return rc;
        if (!s.remaining) break;
    }
    return PMC_OK;
}

long long stride_for(long long n_vox) {
    return (n_vox + kTileVoxels - 1) / kTileVoxels * kTileVoxels;
}

int reduce_blocks(long long n_tiles) {
    return (int)((n_tiles + kReduceThreads / 32 - 1) / (kReduceThreads / 32));
}

int launch_fold(pmc_engine* e, long long n_vox, int group, const double* d_col_nhist) {
    const int tpc = (int)(e->col_stride / kTileVoxels);
    const long long n_tiles = (long long)tpc * group;
    fold_sparse_kernel<<<reduce_blocks(n_tiles), kReduceThreads, 0, e->stream>>>(
        (unsigned long long*)e->edep.p, e->d_mass, d_col_nhist, n_vox, e->col_stride, tpc, n_tiles,
        (double*)e->s1.p, (double*)e->s2.p, (unsigned int*)e->dirty.p,
        (unsigned int*)e->touched.p, e->d_total_q);
    PMC_CUDA(e, cudaGetLastError());
    e->counters.reduce_launches += 1;
    return PMC_OK;
}

int ensure_colmax(pmc_engine* e, int group) {
    if (group > e->colmax_len) {
        if (e->d_colmax) cudaFree(e->d_colmax);
        PMC_CUDA(e, cudaMalloc(&e->d_colmax, sizeof(unsigned long long) * group));
        e->colmax_len = group;
    }
    return PMC_OK;
}

int launch_finalize(pmc_engine* e, long long n_vox, int group, int n_batches) {
    int rc = ensure_colmax(e, group);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemsetAsync(e->d_colmax, 0, sizeof(unsigned long long) * group, e->stream));
    const int tpc = (int)(e->col_stride / kTileVoxels);
    const long long n_tiles = (long long)tpc * group;
    finalize_sparse_kernel<<<reduce_blocks(n_tiles), kReduceThreads, 0, e->stream>>>(
        (double*)e->s1.p, (double*)e->s2.p, n_vox, e->col_stride, tpc, n_tiles, n_batches,
        (const unsigned int*)e->touched.p, e->d_colmax);
    PMC_CUDA(e, cudaGetLastError());
    e->counters.reduce_launches += 1;
    return PMC_OK;
}

// Grow a device buffer to at least `bytes`, keeping its first `keep` bytes.
int grow_keep(pmc_engine* e, DevBuf& b, size_t bytes, size_t keep) {
    if (b.p && b.bytes >= bytes) return PMC_OK;
    const size_t cap = std::max(bytes, b.bytes + b.bytes / 2);
    void* p = nullptr;
    PMC_CUDA(e, cudaMalloc(&p, cap));
    if (keep) PMC_CUDA(e, cudaMemcpyAsync(p, b.p, keep, cudaMemcpyDeviceToDevice, e->stream));
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    if (b.p) cudaFree(b.p);
    b.p = p;
    b.bytes = cap;
    return PMC_OK;
}

// First half of the truncation of the finalized group held in s1 (mean):
// count the kept entries per (column, tile) and scan them on the device.
// Returns the group's entry total and per-column counts on the host.
int truncate_count(pmc_engine* e, long long n_vox, int group, double truncation,
                   unsigned long long* nnz, std::vector<long long>* counts) {
    const int tpc = (int)(e->col_stride / kTileVoxels);
    const long long n_tc = (long long)tpc * group;
    int rc = ensure(e, e->tile_counts, sizeof(unsigned int) * n_tc);
    if (!rc) rc = ensure(e, e->tile_offsets, sizeof(unsigned long long) * n_tc);
    if (!rc) rc = ensure(e, e->col_counts, sizeof(long long) * group);
    if (rc) return rc;
    count_kept_sparse_kernel<<<reduce_blocks(n_tc), kReduceThreads, 0, e->stream>>>(
        (const double*)e->s1.p, n_vox, e->col_stride, tpc, n_tc, truncation, e->d_colmax,
        (const unsigned int*)e->touched.p, (unsigned int*)e->tile_counts.p);
    scan_tiles_kernel<<<1, 1024, 0, e->stream>>>(
        (const unsigned int*)e->tile_counts.p, n_tc, (unsigned long long*)e->tile_offsets.p, group,
        tpc, (long long*)e->col_counts.p, e->d_nnz);
    PMC_CUDA(e, cudaGetLastError());
    e->counters.reduce_launches += 2;
    counts->resize(group);
    PMC_CUDA(e, cudaMemcpyAsync(nnz, e->d_nnz, sizeof *nnz, cudaMemcpyDeviceToHost, e->stream));
    PMC_CUDA(e, cudaMemcpyAsync(counts->data(), e->col_counts.p, sizeof(long long) * group,
                                cudaMemcpyDeviceToHost, e->stream));
    e->d2h_bytes += sizeof *nnz + sizeof(long long) * group;
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    return PMC_OK;
}

// Second half: write the kept entries behind the CSC already accumulated on
// the device (earlier groups), in ascending voxel order per column.
int truncate_compact(pmc_engine* e, long long n_vox, int group, double truncation,
                     unsigned long long nnz, const std::vector<long long>& counts) {
    const int tpc = (int)(e->col_stride / kTileVoxels);
    const long long n_tc = (long long)tpc * group;
    const size_t base = (size_t)e->csc_nnz;
    const size_t total = base + (size_t)nnz;
    int rc = grow_keep(e, e->out_idx, sizeof(long long) * total, sizeof(long long) * base);
    if (!rc) rc = grow_keep(e, e->out_dose, sizeof(double) * total, sizeof(double) * base);
    if (!rc) rc = grow_keep(e, e->out_sigma, sizeof(double) * total, sizeof(double) * base);
    if (rc) return rc;
    if (nnz > 0) {
        compact_sparse_kernel<<<reduce_blocks(n_tc), kReduceThreads, 0, e->stream>>>(
            (const double*)e->s1.p, (const double*)e->s2.p, n_vox, e->col_stride, tpc, n_tc,
            truncation, e->d_colmax, (const unsigned int*)e->touched.p,
            (const unsigned long long*)e->tile_offsets.p, (long long*)e->out_idx.p + base,
            (double*)e->out_dose.p + base, (double*)e->out_sigma.p + base);
        PMC_CUDA(e, cudaGetLastError());
        e->counters.reduce_launches += 1;
    }
    e->csc_nnz = (long long)total;
    for (int c = 0; c < group; ++c) e->dij_indptr.push_back(e->dij_indptr.back() + counts[c]);
    return PMC_OK;
}

// The [group][stride] maps and their bitmaps, sized for `group` columns of
// `n_vox` entries.  A freshly allocated quanta map is not yet zero.
int ensure_maps(pmc_engine* e, int group, long long n_vox) {
    e->col_stride = stride_for(n_vox);
    const long long n = e->col_stride * group;
    if (e->edep.bytes < sizeof(double) * (size_t)n) e->edep_clean = false;
    int rc = ensure(e, e->edep, sizeof(double) * (size_t)n);
    if (!rc) rc = ensure(e, e->s1, sizeof(double) * (size_t)n);
    if (!rc) rc = ensure(e, e->s2, sizeof(double) * (size_t)n);
    if (!rc) rc = ensure(e, e->dirty, sizeof(unsigned int) * (size_t)(n / kWordEntries));
    if (!rc) rc = ensure(e, e->touched, sizeof(unsigned int) * (size_t)(n / kWordEntries));
    return rc;
}

// Start scoring `group` columns: quanta all zero (cleared in bulk only after a
// run that did not complete), both bitmaps empty.  The float64 sums are not
// cleared: a sector's first fold writes it whole.
int begin_maps(pmc_engine* e, int group) {
    if (!e->edep_clean) {
        PMC_CUDA(e, cudaMemsetAsync(e->edep.p, 0, e->edep.bytes, e->stream));
        e->edep_clean = true;
    }
    const size_t words = sizeof(unsigned int) * (size_t)(e->col_stride * group / kWordEntries);
    PMC_CUDA(e, cudaMemsetAsync(e->dirty.p, 0, words, e->stream));
    PMC_CUDA(e, cudaMemsetAsync(e->touched.p, 0, words, e->stream));
    e->edep_clean = false;  // until every batch of the call has been folded
    return PMC_OK;
}

int fill_bitmap(pmc_engine* e, DevBuf& b, int group, unsigned int v) {
    const long long words = e->col_stride * group / kWordEntries;
    fill_u32_kernel<<<std::max(1, (int)std::min<long long>(4 * e->sm_count, (words + 255) / 256)), 256, 0,
                      e->stream>>>((unsigned int*)b.p, words, v);
    PMC_CUDA(e, cudaGetLastError());
    return PMC_OK;
}

int reset_counters(pmc_engine* e) {
    std::memset(&e->counters, 0, sizeof e->counters);
    PMC_CUDA(e, cudaMemsetAsync(e->d_counters, 0, sizeof(Counters), e->stream));
    PMC_CUDA(e, cudaMemsetAsync(e->d_sched, 0, sizeof(Sched), e->stream));
    return PMC_OK;
}

int finish_counters(pmc_engine* e, pmc_books* books) {
    Counters c{};
    Sched s{};
    PMC_CUDA(e, cudaMemcpyAsync(&c, e->d_counters, sizeof c, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof c);
    PMC_CUDA(e, cudaMemcpyAsync(&s, e->d_sched, sizeof s, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof s);
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->counters.rounds = s.total_rounds;
    e->counters.kernel_launches += 3 * s.total_rounds + e->counters.reduce_launches;
    e->counters.photon_flights = (int64_t)c.flights;
    e->counters.photon_interactions = (int64_t)c.interactions;
    e->counters.electron_substeps = (int64_t)c.substeps;
    e->counters.deposits = (int64_t)c.deposits;
    e->counters.queue_pushes = (int64_t)c.pushes;
    e->counters.primaries = (int64_t)c.primaries;
    if (books) {
        books->escaped = c.escaped;
        books->unscored = c.unscored;
        books->emitted = c.emitted;
        books->majorant_violations = c.violations;
        if (c.deposited != 0) books->deposited = c.deposited;  // dose-to-water physical book
    }
    if (c.violations != 0)
        return fail(e, PMC_ERR_MAJORANT,
                    "Woodcock majorant violated in the kernel despite table headroom. The geometry "
                    "contains material or density the majorant declaration did not cover.");
    return PMC_OK;
}

int upload_f32(pmc_engine* e, const std::vector<float>& v, const float** out) {
    return upload_vec(e, v, out);
}

int fill_gen_spectrum(pmc_engine* e, GenDesc& G, int n_bins, const double* edges,
                      const double* cdf) {
    if (n_bins < 1 || !edges || !cdf) return fail(e, PMC_ERR_INVALID, "spectral source without a spectrum");
    std::vector<float> ed(edges, edges + n_bins + 1), cd(cdf, cdf + n_bins);
    G.n_bins = n_bins;
    int rc = upload_f32(e, ed, &G.edges);
    if (!rc) rc = upload_f32(e, cd, &G.cdf);
    return rc;
}

float int_bits(int v) {
    float f;
    std::memcpy(&f, &v, sizeof f);
    return f;
}

// Append one spectrum as a segment of n_bins + 1 entries starting at the same
// index in both arrays; returns that index.
int append_spectrum(std::vector<float>* edges, std::vector<float>* cdf, int n_bins,
                    const double* e_in, const double* c_in) {
    const int first = (int)edges->size();
    for (int k = 0; k <= n_bins; ++k) edges->push_back((float)e_in[k]);
    for (int k = 0; k < n_bins; ++k) cdf->push_back((float)c_in[k]);
    cdf->push_back(1.0f);  // unused: keeps the segments aligned
    return first;
}

BeamletRec lattice_rec(double energy, double z0, double x_lo, double x_ext, double y_lo, double y_ext) {
    BeamletRec r{};
    r.a = make_float4((float)x_lo, (float)x_ext, (float)y_lo, (float)y_ext);
    r.b = make_float4((float)z0, (float)energy, 0.0f, 0.0f);
    r.d = make_float4(0.0f, 0.0f, 0.0f, int_bits(0));
    return r;
}

BeamletRec fan_rec(const double focal[3], const double center[3], const double u[3], const double v[3],
                   double width_u, double width_v, int first, int n_bins) {
    BeamletRec r{};
    r.a = make_float4((float)focal[0], (float)focal[1], (float)focal[2], (float)width_u);
    r.b = make_float4((float)center[0], (float)center[1], (float)center[2], (float)width_v);
    r.c = make_float4((float)u[0], (float)u[1], (float)u[2], int_bits(first));
    r.d = make_float4((float)v[0], (float)v[1], (float)v[2], int_bits(1 | (n_bins << 1)));
    return r;
}

// The per-beamlet records of an in-kernel beamlet source (nothing for the
// upload route), its mixture selection and its spectra.
int beamlet_records(pmc_engine* e, const pmc_beamlet_desc* src, std::vector<BeamletRec>* recs,
                    int* n_comp, std::vector<float>* comp_cdf, std::vector<float>* edges,
                    std::vector<float>* cdf) {
    const int n = src->n_beamlets;
    *n_comp = 1;
    comp_cdf->assign(1, 1.0f);
    switch (src->type) {
        case PMC_BEAMLET_LATTICE:
            if (!src->x_lo || !src->x_extent || !src->y_lo || !src->y_extent)
                return fail(e, PMC_ERR_INVALID, "lattice source without bounds");
            for (int j = 0; j < n; ++j)
                recs->push_back(lattice_rec(src->energy, src->z0, src->x_lo[j], src->x_extent[j],
                                            src->y_lo[j], src->y_extent[j]));
            edges->assign(2, 0.0f);
            cdf->assign(2, 1.0f);
            return PMC_OK;
        case PMC_BEAMLET_SPECTRAL: {
            if (!src->centers) return fail(e, PMC_ERR_INVALID, "spectral beamlets without centres");
            if (src->n_bins < 1 || !src->edges || !src->cdf)
                return fail(e, PMC_ERR_INVALID, "spectral source without a spectrum");
            const int first = append_spectrum(edges, cdf, src->n_bins, src->edges, src->cdf);
            for (int j = 0; j < n; ++j)
                recs->push_back(fan_rec(src->focal, src->centers + 3 * j, src->u_axis, src->v_axis,
                                        src->width_u, src->width_v, first, src->n_bins));
            return PMC_OK;
        }
        case PMC_BEAMLET_RECORDS: {
            const int nc = src->n_components;
            if (nc < 1 || !src->records) return fail(e, PMC_ERR_INVALID, "record source without records");
            if (nc > 1 && !src->component_cdf)
                return fail(e, PMC_ERR_INVALID, "a mixture needs its component cdf");
            std::vector<int> first(std::max(src->n_spectra, 0));
            for (int k = 0, at = 0; k < src->n_spectra; ++k) {
                const int nb = src->spectrum_bins[k];
                if (nb < 1) return fail(e, PMC_ERR_INVALID, "empty spectrum %d", k);
                first[k] = append_spectrum(edges, cdf, nb, src->spectrum_edges + at + k,
                                           src->spectrum_cdf + at);
                at += nb;
            }
            if (edges->empty()) {
                edges->assign(2, 0.0f);
                cdf->assign(2, 1.0f);
            }
            *n_comp = nc;
            comp_cdf->resize(nc);
            for (int c = 0; c < nc; ++c) (*comp_cdf)[c] = nc > 1 ? (float)src->component_cdf[c] : 1.0f;
            for (long long i = 0; i < (long long)n * nc; ++i) {
                const pmc_beamlet_rec& r = src->records[i];
                if (r.type == PMC_BEAMLET_LATTICE) {
                    recs->push_back(lattice_rec(r.energy, r.z0, r.x_lo, r.x_extent, r.y_lo, r.y_extent));
                } else if (r.type == PMC_BEAMLET_SPECTRAL) {
                    if (r.spectrum < 0 || r.spectrum >= src->n_spectra)
                        return fail(e, PMC_ERR_INVALID, "record %lld names spectrum %d of %d", i,
                                    r.spectrum, src->n_spectra);
                    recs->push_back(fan_rec(r.focal, r.center, r.u_axis, r.v_axis, r.width_u, r.width_v,
                                            first[r.spectrum], src->spectrum_bins[r.spectrum]));
                } else {
                    return fail(e, PMC_ERR_INVALID, "record %lld has unknown type %d", i, r.type);
                }
            }
            return PMC_OK;
        }
        case PMC_BEAMLET_UPLOAD:
            if (!src->sample) return fail(e, PMC_ERR_INVALID, "upload source without a sampler");
            return PMC_OK;
        default:
            return fail(e, PMC_ERR_INVALID, "unknown beamlet source type %d", src->type);
    }
}

}  // namespace

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

int pmc_abi_version(void) { return PMC_ABI_VERSION; }

int pmc_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int pmc_create(pmc_engine** out, int device_ordinal) {
    if (!out) return PMC_ERR_INVALID;
    *out = nullptr;
    pmc_engine* e = new pmc_engine();
    e->device = device_ordinal;
    cudaError_t st = cudaSetDevice(device_ordinal);
    if (st == cudaSuccess) st = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
    e->stream = e->own_stream;
    if (st == cudaSuccess) st = cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, device_ordinal);
    if (st == cudaSuccess) st = cudaMalloc(&e->d_sched, sizeof(Sched));
    if (st == cudaSuccess) st = cudaMalloc(&e->d_counters, sizeof(Counters));
    if (st == cudaSuccess) st = cudaMalloc(&e->d_gen, sizeof(GenDesc));
    if (st == cudaSuccess) st = cudaMalloc(&e->d_total_q, sizeof(unsigned long long));
    if (st == cudaSuccess) st = cudaMalloc(&e->d_nnz, sizeof(unsigned long long));
    for (int i = 0; i < 4 && st == cudaSuccess; ++i) st = cudaEventCreate(&e->ev[i]);
    if (st != cudaSuccess) {
        pmc_destroy(e);
        return PMC_ERR_CUDA;
    }
    *out = e;
    return PMC_OK;
}

void pmc_destroy(pmc_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    destroy_graph(e);
    for (DevBuf& b : e->run_pool)
        if (b.p) cudaFree(b.p);
    e->run_pool.clear();
    free_tables(e);
    if (e->d_gs4) cudaFree(e->d_gs4);
    if (e->d_vox) cudaFree(e->d_vox);
    if (e->d_mass) cudaFree(e->d_mass);
    if (e->d_cyl_z) cudaFree(e->d_cyl_z);
    if (e->d_cyl_r2) cudaFree(e->d_cyl_r2);
    for (DevBuf* b : {&e->q[0], &e->q[1], &e->q[2], &e->q[3], &e->edep, &e->s1, &e->s2,
                      &e->tile_counts, &e->tile_offsets, &e->col_counts, &e->out_idx,
                      &e->out_dose, &e->out_sigma, &e->col_nhist, &e->dirty, &e->touched,
                      &e->stage})
        if (b->p) cudaFree(b->p);
    for (void* p : {(void*)e->d_sched, (void*)e->d_counters, (void*)e->d_gen,
                    (void*)e->d_total_q, (void*)e->d_colmax, (void*)e->d_nnz})
        if (p) cudaFree(p);
    for (cudaEvent_t ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : e->batch_ev) cudaEventDestroy(ev);
    if (e->own_stream) cudaStreamDestroy(e->own_stream);
    delete e;
}

const char* pmc_last_error(const pmc_engine* e) { return e ? e->error.c_str() : "no engine"; }

int pmc_upload_grid(pmc_engine* e, int32_t nx, int32_t ny, int32_t nz, const double origin[3],
                    const double spacing[3], const float* density, const uint8_t* material) {
    if (!e) return PMC_ERR_INVALID;
    if (nx < 1 || ny < 1 || nz < 1) return fail(e, PMC_ERR_INVALID, "empty grid shape");
    if (!origin || !spacing || !density || !material) return fail(e, PMC_ERR_INVALID, "null grid array");
    for (int i = 0; i < 3; ++i)
        if (!(spacing[i] > 0.0)) return fail(e, PMC_ERR_INVALID, "non-positive spacing");
    PMC_CUDA(e, cudaSetDevice(e->device));
    const long long n = (long long)nx * ny * nz;
    int max_mat = 0;
    for (long long i = 0; i < n; ++i) {
        if (!(density[i] > 0.0f)) return fail(e, PMC_ERR_INVALID, "non-positive voxel density; vacuum is not supported");
        max_mat = std::max(max_mat, (int)material[i]);
    }
    // the raw arrays cross the bus once; the device packs voxels (and the
    // default scoring masses) from them
    const size_t dens_bytes = sizeof(float) * (size_t)n;
    const size_t mat_off = (dens_bytes + 255) & ~(size_t)255;
    int rc = ensure(e, e->stage, mat_off + (size_t)n);
    if (!rc) rc = ensure_ptr(e, e->d_vox, e->vox_cap, sizeof(float2) * (size_t)n);
    const bool default_mass = !e->custom_scoring;
    if (!rc && default_mass) rc = ensure_ptr(e, e->d_mass, e->mass_cap, sizeof(double) * (size_t)n);
    if (rc) return rc;
    float* d_density = (float*)e->stage.p;
    uint8_t* d_material = (uint8_t*)e->stage.p + mat_off;
    PMC_CUDA(e, cudaMemcpyAsync(d_density, density, dens_bytes, cudaMemcpyHostToDevice, e->stream));
    PMC_CUDA(e, cudaMemcpyAsync(d_material, material, (size_t)n, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)(dens_bytes + (size_t)n);
    const double volume = spacing[0] * spacing[1] * spacing[2];
    e->voxel_volume = volume;
    pack_voxels_kernel<<<grid_blocks(n), 256, 0, e->stream>>>(d_density, d_material, n, volume, e->d_vox,
                                                               default_mass ? e->d_mass : nullptr);
    PMC_CUDA(e, cudaGetLastError());
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->gi = make_grid(nx, ny, nz, origin, spacing);
    e->has_grid = true;
    e->max_material = max_mat;
    if (default_mass) {
        e->score_mode = 0;
        e->si = e->gi;
        e->mass_len = n;
    }
    return PMC_OK;
}

int pmc_set_scoring(pmc_engine* e, const pmc_scoring_desc* s) {
    if (!e) return PMC_ERR_INVALID;
    if (!e->has_grid) return fail(e, PMC_ERR_STATE, "upload the transport grid first");
    PMC_CUDA(e, cudaSetDevice(e->device));
    if (!s) {
        e->custom_scoring = false;
        e->score_mode = 0;
        e->si = e->gi;
        const long long n = e->gi.n_voxels;
        int rc = ensure_ptr(e, e->d_mass, e->mass_cap, sizeof(double) * (size_t)n);
        if (rc) return rc;
        mass_from_voxels_kernel<<<grid_blocks(n), 256, 0, e->stream>>>(e->d_vox, n, e->voxel_volume,
                                                                       e->d_mass);
        PMC_CUDA(e, cudaGetLastError());
        PMC_CUDA(e, cudaStreamSynchronize(e->stream));
        e->mass_len = n;
        return PMC_OK;
    }
    if (!s->voxel_mass) return fail(e, PMC_ERR_INVALID, "invalid scoring grid");
    long long n = 0;
    if (s->mode == 1) {
        const int nd = s->n_depth, ns = s->n_shells;
        if (nd < 1 || ns < 1 || !s->depth_edges || !s->radial_edges)
            return fail(e, PMC_ERR_INVALID, "a cylindrical scoring grid needs depth and radial edges");
        for (int k = 0; k < nd; ++k)
            if (!(s->depth_edges[k + 1] > s->depth_edges[k]))
                return fail(e, PMC_ERR_INVALID, "depth_edges must be strictly increasing");
        for (int k = 0; k < ns; ++k)
            if (!(s->radial_edges[k + 1] > s->radial_edges[k]) || s->radial_edges[k] < 0.0)
                return fail(e, PMC_ERR_INVALID, "radial_edges must be non-negative and strictly increasing");
        n = (long long)nd * ns;
        std::vector<float> ze(nd + 1), re2(ns + 1);
        for (int k = 0; k <= nd; ++k) ze[k] = (float)s->depth_edges[k];
        for (int k = 0; k <= ns; ++k) re2[k] = (float)(s->radial_edges[k] * s->radial_edges[k]);
        for (float** dst : {&e->d_cyl_z, &e->d_cyl_r2})
            if (*dst) cudaFree(*dst), *dst = nullptr;
        PMC_CUDA(e, cudaMalloc(&e->d_cyl_z, sizeof(float) * ze.size()));
        PMC_CUDA(e, cudaMalloc(&e->d_cyl_r2, sizeof(float) * re2.size()));
        PMC_CUDA(e, cudaMemcpy(e->d_cyl_z, ze.data(), sizeof(float) * ze.size(), cudaMemcpyHostToDevice));
        PMC_CUDA(e, cudaMemcpy(e->d_cyl_r2, re2.data(), sizeof(float) * re2.size(), cudaMemcpyHostToDevice));
        e->h2d_bytes += sizeof(float) * (ze.size() + re2.size());
        CylInfo c{};
        c.ax = (float)s->axis[0];
        c.ay = (float)s->axis[1];
        c.z_lo = ze.front();
        c.z_hi = ze.back();
        c.r_in_sq = re2.front();
        c.r_out_sq = re2.back();
        c.n_depth = nd;
        c.n_shells = ns;
        c.z_edges = e->d_cyl_z;
        c.r_edges_sq = e->d_cyl_r2;
        e->cyl = c;
        e->score_mode = 1;
        e->si = GridInfo{};
        e->si.n_voxels = n;
    } else {
        if (s->nx < 1 || s->ny < 1 || s->nz < 1) return fail(e, PMC_ERR_INVALID, "invalid scoring grid");
        n = (long long)s->nx * s->ny * s->nz;
        e->si = make_grid(s->nx, s->ny, s->nz, s->origin, s->spacing);
        e->score_mode = 0;
    }
    int rc_mass = ensure_ptr(e, e->d_mass, e->mass_cap, sizeof(double) * (size_t)n);
    if (rc_mass) return rc_mass;
    PMC_CUDA(e, cudaMemcpy(e->d_mass, s->voxel_mass, sizeof(double) * n, cudaMemcpyHostToDevice));
    e->h2d_bytes += (unsigned long long)(sizeof(double) * n);
    e->mass_len = n;
    e->custom_scoring = true;
    return PMC_OK;
}

int pmc_upload_tables(pmc_engine* e, const pmc_tables_desc* t) {
    if (!e || !t) return PMC_ERR_INVALID;
    const int M = t->n_materials, N = t->n_points;
    if (M < 1 || M > 256) return fail(e, PMC_ERR_INVALID, "the B200 backend addresses 1..256 materials (uint8 voxel map); got %d", M);
    if (N < 2) return fail(e, PMC_ERR_INVALID, "need at least two table nodes");
    const double* req[] = {t->mu_compton, t->mu_photo, t->mu_pair, t->mu_rayleigh, t->majorant,
                           t->stopping_restricted, t->stopping_radiative, t->moller,
                           t->csda_range, t->scattering_power, t->log_eta, t->restricted_range,
                           t->energy_of_restricted_range};
    for (const double* a : req)
        if (!a) return fail(e, PMC_ERR_INVALID, "null table array");
    PMC_CUDA(e, cudaSetDevice(e->device));
    free_tables(e);
    const size_t MN = (size_t)M * N;
    std::vector<float4> ch(MN), ea(MN);
    std::vector<float2> eb(MN);
    std::vector<float> maj(N), ec(MN), er(MN);
    for (size_t i = 0; i < MN; ++i) {
        ch[i] = make_float4((float)t->mu_compton[i], (float)t->mu_photo[i], (float)t->mu_pair[i],
                            (float)t->mu_rayleigh[i]);
        ea[i] = make_float4((float)t->csda_range[i], (float)t->moller[i],
                            (float)t->restricted_range[i], (float)t->stopping_radiative[i]);
        eb[i] = make_float2((float)t->scattering_power[i], (float)t->log_eta[i]);
        ec[i] = (float)t->stopping_restricted[i];
        er[i] = (float)t->energy_of_restricted_range[i];
    }
    for (int i = 0; i < N; ++i) maj[i] = (float)t->majorant[i];
    auto put = [&](const void* src, size_t bytes, const void** dst) -> int {
        void* p = nullptr;
        PMC_CUDA(e, cudaMalloc(&p, std::max<size_t>(bytes, 16)));
        PMC_CUDA(e, cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
    e->h2d_bytes += (unsigned long long)(bytes);
        e->table_allocs.push_back(p);
        *dst = p;
        return PMC_OK;
    };
    Tables T{};
    int rc = put(ch.data(), sizeof(float4) * MN, (const void**)&T.ch);
    if (!rc) rc = put(maj.data(), sizeof(float) * N, (const void**)&T.maj);
    if (!rc) rc = put(ea.data(), sizeof(float4) * MN, (const void**)&T.ea);
    if (!rc) rc = put(eb.data(), sizeof(float2) * MN, (const void**)&T.eb);
    if (!rc) rc = put(ec.data(), sizeof(float) * MN, (const void**)&T.ec);
    if (!rc) rc = put(er.data(), sizeof(float) * MN, (const void**)&T.er);
    if (rc) return rc;
    const int NC = t->n_coherent;
    std::vector<float> cx(std::max(NC, 2), 0.0f), cc((size_t)M * std::max(NC, 2), 0.0f);
    if (NC >= 2 && t->coherent_x && t->coherent_cumulative) {
        for (int i = 0; i < NC; ++i) cx[i] = (float)t->coherent_x[i];
        for (size_t i = 0; i < (size_t)M * NC; ++i) cc[i] = (float)t->coherent_cumulative[i];
        T.n_coherent = NC;
    } else {
        cx[1] = 1.0f;
        T.n_coherent = 2;
    }
    rc = put(cx.data(), sizeof(float) * cx.size(), (const void**)&T.coh_x);
    if (!rc) rc = put(cc.data(), sizeof(float) * cc.size(), (const void**)&T.coh_cum);
    if (rc) return rc;
    T.n_points = N;
    T.n_materials = M;
    T.p_log_min = (float)t->photon_log_e_min;
    T.p_inv_dlog = (float)t->photon_inv_dlog;
    T.e_log_min = (float)t->electron_log_e_min;
    T.e_inv_dlog = (float)t->electron_inv_dlog;
    T.r_log_min = (float)t->range_log_r_min;
    T.r_inv_dlog = (float)t->range_inv_dlog;
    // keep the GS part of an earlier upload
    T.gs4 = e->tab.gs4;
    T.gs_ix0 = e->tab.gs_ix0;
    T.gs_iy0 = e->tab.gs_iy0;
    T.gs_n_eta = e->tab.gs_n_eta;
    T.gs_n_theta2 = e->tab.gs_n_theta2;
    T.gs_n_u = e->tab.gs_n_u;
    T.gs_bins_per_log = e->tab.gs_bins_per_log;
    e->tab = T;
    e->has_tables = true;
    return PMC_OK;
}

int pmc_upload_gs(pmc_engine* e, const float* values, int32_t ix0, int32_t iy0, int32_t n_eta,
                  int32_t n_theta2, int32_t n_u, double bins_per_log) {
    if (!e) return PMC_ERR_INVALID;
    if (!values || n_eta < 2 || n_theta2 < 2 || n_u < 1 || !(bins_per_log > 0.0))
        return fail(e, PMC_ERR_INVALID, "invalid Goudsmit-Saunderson grid");
    PMC_CUDA(e, cudaSetDevice(e->device));
    const size_t cells = (size_t)(n_eta - 1) * (n_theta2 - 1) * n_u;
    const size_t raw = sizeof(float) * (size_t)n_eta * n_theta2 * n_u;
    int rc = ensure(e, e->stage, raw);
    if (!rc) rc = ensure_ptr(e, e->d_gs4, e->gs_cap, sizeof(float4) * cells);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemcpyAsync(e->stage.p, values, raw, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)raw;
    pack_gs_kernel<<<grid_blocks((long long)cells), 256, 0, e->stream>>>((const float*)e->stage.p, n_eta,
                                                                         n_theta2, n_u, e->d_gs4);
    PMC_CUDA(e, cudaGetLastError());
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->tab.gs4 = e->d_gs4;
    e->tab.gs_ix0 = ix0;
    e->tab.gs_iy0 = iy0;
    e->tab.gs_n_eta = n_eta;
    e->tab.gs_n_theta2 = n_theta2;
    e->tab.gs_n_u = n_u;
    e->tab.gs_bins_per_log = (float)bins_per_log;
    e->has_gs = true;
    return PMC_OK;
}

// The beam-limiting stack of a collimated source and its attenuation rows,
// checked and uploaded in float32 (the generator's precision).  The table's
// energies must be log-uniform (np.geomspace, as _StackTransmission builds
// them, geometry/collimation.py:961-969).
static int fill_gen_stack(pmc_engine* e, GenDesc& G, const pmc_head_stack* st, const pmc_head_mu* mu) {
    if (!st) return PMC_OK;
    const int n = st->n_devices;
    if (n < 1 || n > pmc_head::kMaxDevices || !mu || mu->n_rows < n || mu->n_table < 2 || !mu->log_energy ||
        !mu->log_total || !st->kind || !st->z_top || !st->z_bottom)
        return fail(e, PMC_ERR_INVALID, "bad collimation stack or attenuation table");
    const int nt = mu->n_table;
    const double l0 = mu->log_energy[0], l1 = mu->log_energy[nt - 1];
    if (!(l1 > l0)) return fail(e, PMC_ERR_INVALID, "attenuation table energies must ascend");
    const double step = (l1 - l0) / (nt - 1);
    for (int k = 0; k < nt; ++k)
        if (std::fabs(mu->log_energy[k] - (l0 + k * step)) > 1e-6 * std::max(1.0, std::fabs(step)))
            return fail(e, PMC_ERR_INVALID, "attenuation table energies must be log-uniform");
    long long n_edges = 0, n_tips = 0;
    for (int j = 0; j < n; ++j) {
        if (st->kind[j] != 0 && st->kind[j] != 1) return fail(e, PMC_ERR_INVALID, "unknown device kind");
        if (st->kind[j] == 1) {
            const long long np_ = st->mlc_n_pairs[j];
            n_edges = std::max(n_edges, (long long)st->mlc_edges_off[j] + np_ + 1);
            n_tips = std::max(n_tips, (long long)st->mlc_tips_off[j] + np_);
            if (np_ < 1 || st->mlc_edges_off[j] < 0 || st->mlc_tips_off[j] < 0)
                return fail(e, PMC_ERR_INVALID, "bad leaf offsets");
        }
    }
    if (n_edges > st->n_leaf_edges || n_tips > st->n_tips)
        return fail(e, PMC_ERR_INVALID, "leaf offsets beyond the leaf arrays");
    auto f32 = [](const double* a, long long m) {
        std::vector<float> v((size_t)std::max(m, 1ll), 0.0f);
        for (long long i = 0; i < m; ++i) v[(size_t)i] = a ? (float)a[i] : 0.0f;
        return v;
    };
    auto i32 = [](const int32_t* a, long long m) {
        std::vector<int> v((size_t)std::max(m, 1ll), 0);
        for (long long i = 0; i < m; ++i) v[(size_t)i] = a ? a[i] : 0;
        return v;
    };
    pmc_head::Stack& S = G.stack;
    S.n = n;
    for (int k = 0; k < 3; ++k) S.origin[k] = (float)st->origin[k];
    for (int k = 0; k < 9; ++k) S.rot[k] = (float)st->rotation[k];
    int rc = upload_vec(e, i32(st->kind, n), &S.kind);
    if (!rc) rc = upload_f32(e, f32(st->z_top, n), &S.z_top);
    if (!rc) rc = upload_f32(e, f32(st->z_bottom, n), &S.z_bottom);
    if (!rc) rc = upload_vec(e, i32(st->jaw_axis, n), &S.jaw_axis);
    if (!rc) rc = upload_f32(e, f32(st->jaw_edge_neg, n), &S.jaw_neg);
    if (!rc) rc = upload_f32(e, f32(st->jaw_edge_pos, n), &S.jaw_pos);
    if (!rc) rc = upload_vec(e, i32(st->jaw_focused, n), &S.jaw_focused);
    if (!rc) rc = upload_f32(e, f32(st->mlc_tip_radius, n), &S.tip_radius);
    if (!rc) rc = upload_vec(e, i32(st->mlc_focused_sides, n), &S.focused_sides);
    if (!rc) rc = upload_vec(e, i32(st->mlc_n_pairs, n), &S.n_pairs);
    if (!rc) rc = upload_vec(e, i32(st->mlc_edges_off, n), &S.edges_off);
    if (!rc) rc = upload_vec(e, i32(st->mlc_tips_off, n), &S.tips_off);
    if (!rc) rc = upload_f32(e, f32(st->leaf_edges_v, st->n_leaf_edges), &S.leaf_edges);
    if (!rc) rc = upload_f32(e, f32(st->tips_neg, st->n_tips), &S.tips_neg);
    if (!rc) rc = upload_f32(e, f32(st->tips_pos, st->n_tips), &S.tips_pos);
    pmc_head::Mu& M = G.stack_mu;
    M.n_rows = n;
    M.n_table = nt;
    M.log_e0 = (float)l0;
    M.inv_dlog = (float)(1.0 / step);
    if (!rc) rc = upload_f32(e, f32(mu->log_total, (long long)n * nt), &M.log_total);
    M.log_compton = M.log_total;
    if (rc) return rc;
    G.stacked = 1;
    G.book_emitted = 1;  // weighted primaries: the emitted energy is booked one by one
    return PMC_OK;
}

// The transmission mask of a PMC_SRC_SPECTRAL_MASKED source, checked as
// _MaskTransmission.__init__ does (geometry/collimation.py:1013-1029) and
// uploaded in float32, the precision of the Warp twin's mask array.
struct MaskFields {
    const double* mask;
    long long nu, nv;
    const double *center, *u, *v;
    double wu, wv;
};
#define PMC_MASK_FIELDS(d) \
    MaskFields { (d)->mask, (d)->mask_n_u, (d)->mask_n_v, (d)->mask_center, (d)->mask_u_axis, \
                 (d)->mask_v_axis, (d)->mask_width_u, (d)->mask_width_v }

static int fill_gen_mask(pmc_engine* e, GenDesc& G, const MaskFields& f) {
    const MaskFields* src = &f;
    const long long nu = src->nu, nv = src->nv;
    if (!src->mask || nu < 1 || nv < 1 || nu * nv > (1ll << 28))
        return fail(e, PMC_ERR_INVALID, "the mask must be a non-empty 2D array, got shape (%lld, %lld)", nu, nv);
    std::vector<float> m((size_t)(nu * nv));
    for (long long i = 0; i < nu * nv; ++i) {
        const double v = src->mask[i];
        if (!std::isfinite(v) || v < 0.0 || v > 1.0)
            return fail(e, PMC_ERR_INVALID, "mask values must be finite and within 0..1");
        m[(size_t)i] = (float)v;
    }
    if (!(src->wu > 0.0) || !(src->wv > 0.0))
        return fail(e, PMC_ERR_INVALID, "widths must be positive, got %g, %g", src->wu, src->wv);
    const double* u = src->u;
    const double* v = src->v;
    const double nuu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double nvv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (std::fabs(nuu - 1.0) > 1e-9 || std::fabs(nvv - 1.0) > 1e-9)
        return fail(e, PMC_ERR_INVALID, "mask axes must be unit vectors");
    if (std::fabs(u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) > 1e-9)
        return fail(e, PMC_ERR_INVALID, "u_axis and v_axis must be orthogonal");
    G.masked = 1;
    G.mask_n_u = (int)nu;
    G.mask_n_v = (int)nv;
    G.mcx = (float)src->center[0]; G.mcy = (float)src->center[1]; G.mcz = (float)src->center[2];
    G.mux = (float)u[0]; G.muy = (float)u[1]; G.muz = (float)u[2];
    G.mvx = (float)v[0]; G.mvy = (float)v[1]; G.mvz = (float)v[2];
    G.mask_wu = (float)src->wu;
    G.mask_wv = (float)src->wv;
    G.book_emitted = 1;  // weighted primaries: the emitted energy is booked one by one
    return upload_f32(e, m, &G.mask);
}

int pmc_run_forward(pmc_engine* e, const pmc_source_desc* src, const pmc_run_params* p,
                    double* dose, double* dose_sigma, pmc_books* books) {
    if (!e || !src || !p || !dose || !dose_sigma) return PMC_ERR_INVALID;
    PMC_CUDA(e, cudaSetDevice(e->device));
    if (p->n_histories < 1) return fail(e, PMC_ERR_INVALID, "need at least one history, got %lld", (long long)p->n_histories);
    if (p->n_batches < 1 || p->n_histories % p->n_batches != 0)
        return fail(e, PMC_ERR_INVALID, "n_histories=%lld not divisible by n_batches=%d", (long long)p->n_histories, p->n_batches);
    RunPlan plan;
    int rc = prepare_transport(e, p, (unsigned long long)(p->n_histories / p->n_batches), &plan);
    if (rc) return rc;
    const long long n_vox = e->si.n_voxels;
    rc = ensure_maps(e, 1, n_vox);
    if (rc) return rc;
    rc = ensure(e, e->col_nhist, sizeof(double));
    if (rc) return rc;
    free_run_allocs(e);

    const long long per_batch = p->n_histories / p->n_batches;
    GenDesc G{};
    G.forward = 1;
    G.group = 1;
    G.kind = src->kind;
    G.per_batch_fwd = per_batch;
    G.energy = (float)src->energy;
    std::vector<float> z1(1, 0.0f);
    switch (src->type) {
        case PMC_SRC_PENCIL:
            G.type = 0;
            G.px = (float)src->position[0]; G.py = (float)src->position[1]; G.pz = (float)src->position[2];
            G.dx = (float)src->direction[0]; G.dy = (float)src->direction[1]; G.dz = (float)src->direction[2];
            break;
        case PMC_SRC_PARALLEL: {
            G.type = 1;
            G.z0 = (float)src->z0;
            std::vector<float> a(1, (float)src->x_lo), b(1, (float)src->x_extent),
                c(1, (float)src->y_lo), d(1, (float)src->y_extent);
            rc = upload_f32(e, a, &G.x_lo);
            if (!rc) rc = upload_f32(e, b, &G.x_ext);
            if (!rc) rc = upload_f32(e, c, &G.y_lo);
            if (!rc) rc = upload_f32(e, d, &G.y_ext);
            break;
        }
        case PMC_SRC_SPECTRAL:
        case PMC_SRC_SPECTRAL_MASKED: {
            G.type = 2;
            G.kind = PMC_PHOTON;
            G.book_emitted = 1;
            G.fx = (float)src->focal[0]; G.fy = (float)src->focal[1]; G.fz = (float)src->focal[2];
            G.uax = (float)src->u_axis[0]; G.uay = (float)src->u_axis[1]; G.uaz = (float)src->u_axis[2];
            G.vax = (float)src->v_axis[0]; G.vay = (float)src->v_axis[1]; G.vaz = (float)src->v_axis[2];
            G.width_u = (float)src->width_u;
            G.width_v = (float)src->width_v;
            std::vector<float> cx(1, (float)src->center[0]), cy(1, (float)src->center[1]),
                cz(1, (float)src->center[2]);
            rc = upload_f32(e, cx, &G.cx);
            if (!rc) rc = upload_f32(e, cy, &G.cy);
            if (!rc) rc = upload_f32(e, cz, &G.cz);
            if (!rc) rc = fill_gen_spectrum(e, G, src->n_bins, src->edges, src->cdf);
            if (!rc && src->type == PMC_SRC_SPECTRAL_MASKED) rc = fill_gen_mask(e, G, PMC_MASK_FIELDS(src));
            if (!rc && src->type == PMC_SRC_SPECTRAL && src->mask) rc = fill_gen_mask(e, G, PMC_MASK_FIELDS(src));
            break;
        }
        case PMC_SRC_PHASESPACE: {
            G.type = 5;
            G.book_emitted = 1;
            const long long n = src->n_records;
            if (n < 1 || !src->up_kind || !src->up_energy || !src->up_pos || !src->up_dir || !src->up_weight)
                return fail(e, PMC_ERR_INVALID, "phase-space source without records");
            for (long long i = 0; i < n; ++i)
                if (src->up_kind[i] < 0 || src->up_kind[i] > 2)
                    return fail(e, PMC_ERR_INVALID, "bad particle kind in the phase space");
            G.n_records = n;
            std::vector<int> k(src->up_kind, src->up_kind + n);
            std::vector<float> en(src->up_energy, src->up_energy + n), ps(src->up_pos, src->up_pos + 3 * n),
                dr(src->up_dir, src->up_dir + 3 * n), w(src->up_weight, src->up_weight + n);
            rc = upload_vec(e, k, &G.up_kind);
            if (!rc) rc = upload_f32(e, en, &G.up_energy);
            if (!rc) rc = upload_f32(e, ps, &G.up_pos);
            if (!rc) rc = upload_f32(e, dr, &G.up_dir);
            if (!rc) rc = upload_f32(e, w, &G.up_weight);
            break;
        }
        case PMC_SRC_PHASESPACE_DEVICE: {  // records already on this device
            G.type = 5;
            G.book_emitted = 1;
            if (src->n_records < 1 || !src->up_kind || !src->up_energy || !src->up_pos || !src->up_dir ||
                !src->up_weight)
                return fail(e, PMC_ERR_INVALID, "device phase-space source without records");
            G.n_records = src->n_records;
            G.up_kind = src->up_kind;
            G.up_energy = src->up_energy;
            G.up_pos = src->up_pos;
            G.up_dir = src->up_dir;
            G.up_weight = src->up_weight;
            break;
        }
        case PMC_SRC_UPLOAD: {
            G.type = 3;
            G.book_emitted = 1;
            if (!src->up_kind || !src->up_energy || !src->up_pos || !src->up_dir || !src->up_weight)
                return fail(e, PMC_ERR_INVALID, "upload source without records");
            const size_t n = (size_t)p->n_histories;
            std::vector<int> k(src->up_kind, src->up_kind + n);
            std::vector<float> en(src->up_energy, src->up_energy + n), ps(src->up_pos, src->up_pos + 3 * n),
                dr(src->up_dir, src->up_dir + 3 * n), w(src->up_weight, src->up_weight + n);
            for (size_t i = 0; i < n; ++i)
                if (k[i] < 0 || k[i] > 2) return fail(e, PMC_ERR_INVALID, "bad particle kind in upload");
            rc = upload_vec(e, k, &G.up_kind);
            if (!rc) rc = upload_f32(e, en, &G.up_energy);
            if (!rc) rc = upload_f32(e, ps, &G.up_pos);
            if (!rc) rc = upload_f32(e, dr, &G.up_dir);
            if (!rc) rc = upload_f32(e, w, &G.up_weight);
            break;
        }
        default:
            return fail(e, PMC_ERR_INVALID, "unknown source type %d", src->type);
    }
    if (!rc && src->mask && (src->type == PMC_SRC_PENCIL || src->type == PMC_SRC_PARALLEL))
        rc = fill_gen_mask(e, G, PMC_MASK_FIELDS(src));
    if (!rc) rc = fill_gen_stack(e, G, src->stack, src->stack_mu);
    if (rc) return rc;
    if (G.kind != PMC_PHOTON && G.kind != PMC_ELECTRON && G.type != 3 && G.type != 5)
        return fail(e, PMC_ERR_INVALID, "unknown primary kind %d", G.kind);
    PMC_CUDA(e, cudaMemcpyAsync(e->d_gen, &G, sizeof G, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)(sizeof G);
    const double nh = (double)per_batch;
    PMC_CUDA(e, cudaMemcpyAsync(e->col_nhist.p, &nh, sizeof nh, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)(sizeof nh);

    rc = reset_counters(e);
    if (rc) return rc;
    // The whole dense map goes back to the caller: zero sums, every sector
    // marked touched (the fold then adds into them, finalize visits them all).
    rc = begin_maps(e, 1);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemsetAsync(e->s1.p, 0, sizeof(double) * n_vox, e->stream));
    PMC_CUDA(e, cudaMemsetAsync(e->s2.p, 0, sizeof(double) * n_vox, e->stream));
    rc = fill_bitmap(e, e->touched, 1, 0xffffffffu);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemsetAsync(e->d_total_q, 0, sizeof(unsigned long long), e->stream));
    TransportParams P = make_params(e, p, plan);
    float t_tr = 0.0f, t_red = 0.0f;
    for (int b = 0; b < p->n_batches; ++b) {
        PMC_CUDA(e, cudaEventRecord(e->ev[0], e->stream));
        rc = run_batch(e, p, plan, P, b, (unsigned long long)per_batch);
        if (rc) return rc;
        PMC_CUDA(e, cudaEventRecord(e->ev[1], e->stream));
        rc = launch_fold(e, n_vox, 1, (const double*)e->col_nhist.p);
        if (rc) return rc;
        PMC_CUDA(e, cudaEventRecord(e->ev[2], e->stream));
        PMC_CUDA(e, cudaEventSynchronize(e->ev[2]));
        float a = 0, c = 0;
        cudaEventElapsedTime(&a, e->ev[0], e->ev[1]);
        cudaEventElapsedTime(&c, e->ev[1], e->ev[2]);
        t_tr += a;
        t_red += c;
        Sched s;
        rc = read_sched(e, &s);
        if (rc) return rc;
        rc = check_flags(e, s);
        if (rc) return rc;
        if (e->progress) e->progress(e->progress_user, per_batch);
    }
    PMC_CUDA(e, cudaEventRecord(e->ev[0], e->stream));
    rc = launch_finalize(e, n_vox, 1, p->n_batches);
    if (rc) return rc;
    PMC_CUDA(e, cudaEventRecord(e->ev[1], e->stream));
    PMC_CUDA(e, cudaMemcpyAsync(dose, e->s1.p, sizeof(double) * n_vox, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof(double) * n_vox);
    PMC_CUDA(e, cudaMemcpyAsync(dose_sigma, e->s2.p, sizeof(double) * n_vox, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof(double) * n_vox);
    unsigned long long total_q = 0;
    PMC_CUDA(e, cudaMemcpyAsync(&total_q, e->d_total_q, sizeof total_q, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof total_q);
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->edep_clean = true;  // every batch folded: every quanta entry consumed
    float c = 0;
    cudaEventElapsedTime(&c, e->ev[0], e->ev[1]);
    e->counters.transport_ms = t_tr;
    e->counters.reduce_ms = t_red + c;
    if (books) {
        std::memset(books, 0, sizeof *books);
        books->deposited = (int64_t)total_q;
    }
    return finish_counters(e, books);
}

int pmc_run_dij(pmc_engine* e, const pmc_beamlet_desc* src, const int64_t* counts,
                const pmc_run_params* p, int64_t* nnz_out, pmc_books* books) {
    if (!e || !src || !counts || !p || !nnz_out) return PMC_ERR_INVALID;
    PMC_CUDA(e, cudaSetDevice(e->device));
    const int n_beam = src->n_beamlets;
    if (n_beam < 1) return fail(e, PMC_ERR_INVALID, "need at least one beamlet");
    if (p->n_batches < 1) return fail(e, PMC_ERR_INVALID, "need at least one batch");
    for (int j = 0; j < n_beam; ++j) {
        if (counts[j] < 1) return fail(e, PMC_ERR_INVALID, "need at least one history per beamlet, got %lld", (long long)counts[j]);
        if (counts[j] % p->n_batches != 0)
            return fail(e, PMC_ERR_INVALID, "n_histories_per_beamlet=%lld not divisible by n_batches=%d", (long long)counts[j], p->n_batches);
    }
    if (p->truncation < 0.0) return fail(e, PMC_ERR_INVALID, "negative truncation %g", p->truncation);
    unsigned long long all_block = 0;
    for (int j = 0; j < n_beam; ++j) all_block += (unsigned long long)(counts[j] / p->n_batches);
    RunPlan plan;
    int rc = prepare_transport(e, p, all_block, &plan);
    if (rc) return rc;
    const long long n_vox = e->si.n_voxels;
    int group = p->beamlet_group_size > 0 ? p->beamlet_group_size : 0;
    const int all_cols = std::min(n_beam, 4096);
    const size_t all_n = (size_t)stride_for(n_vox) * (size_t)all_cols;
    if (group == 0 && e->edep.bytes >= sizeof(double) * all_n && e->s1.bytes >= sizeof(double) * all_n &&
        e->s2.bytes >= sizeof(double) * all_n && e->dirty.bytes >= sizeof(unsigned int) * (all_n / kWordEntries) &&
        e->touched.bytes >= sizeof(unsigned int) * (all_n / kWordEntries))
        group = all_cols;  // the maps held already cover every column: no memory query
    if (group == 0) {
        // Auto: the largest group whose dense maps (int64 quanta + two float64
        // sums = 24 bytes per entry, plus the two sector bitmaps) fit half of
        // the free memory, counting the maps this engine already holds.  The
        // query can take a millisecond or far more on a busy GPU host, hence
        // the shortcut above.
        size_t free_b = 0, total_b = 0;
        PMC_CUDA(e, cudaMemGetInfo(&free_b, &total_b));
        const double held = (double)(e->edep.bytes + e->s1.bytes + e->s2.bytes + e->dirty.bytes +
                                     e->touched.bytes);
        const double budget = 0.5 * ((double)free_b + held);
        group = (int)std::max(1.0, std::floor(budget / (24.0625 * (double)stride_for(n_vox))));
        group = std::min(group, std::min(n_beam, 4096));
    }
    group = std::min(group, n_beam);
    rc = ensure_maps(e, group, n_vox);
    if (!rc) rc = ensure(e, e->col_nhist, sizeof(double) * group);
    if (rc) return rc;
    // Every in-kernel beamlet source becomes per-beamlet records; the upload
    // route samples each batch on the host through the caller's callback.
    std::vector<BeamletRec> recs;
    std::vector<float> comp_cdf, spec_edges, spec_cdf;
    int n_comp = 1;
    rc = beamlet_records(e, src, &recs, &n_comp, &comp_cdf, &spec_edges, &spec_cdf);
    if (rc) return rc;

    std::vector<long long> offset(n_beam);
    long long acc = 0;
    for (int j = 0; j < n_beam; ++j) {
        offset[j] = src->history_offsets ? src->history_offsets[j] : acc;
        if (offset[j] < 0) return fail(e, PMC_ERR_INVALID, "negative history offset");
        acc += counts[j];
    }
    rc = reset_counters(e);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemsetAsync(e->d_total_q, 0, sizeof(unsigned long long), e->stream));
    e->dij_indptr.assign(1, 0);
    e->csc_nnz = 0;
    float t_tr = 0.0f, t_red = 0.0f;

    for (int g0 = 0; g0 < n_beam; g0 += group) {
        const int gs = std::min(group, n_beam - g0);
        free_run_allocs(e);
        GenDesc G{};
        G.forward = 0;
        G.group = gs;
        G.correlated = p->correlated ? 1 : 0;
        G.kind = PMC_PHOTON;
        std::vector<long long> pb(gs), pre(gs + 1, 0), off(gs);
        std::vector<double> nh(gs);
        for (int k = 0; k < gs; ++k) {
            pb[k] = counts[g0 + k] / p->n_batches;
            pre[k + 1] = pre[k] + pb[k];
            off[k] = offset[g0 + k];
            nh[k] = (double)pb[k];
        }
        rc = upload_vec(e, pb, &G.per_batch);
        if (!rc) rc = upload_vec(e, pre, &G.pb_prefix);
        if (!rc) rc = upload_vec(e, off, &G.hist_offset);
        if (rc) return rc;
        std::vector<float> up_energy, up_pos, up_dir, up_weight;
        if (src->type == PMC_BEAMLET_UPLOAD) {
            G.type = 3;
            G.book_emitted = 1;
            const size_t n = (size_t)pre[gs];
            up_energy.resize(n);
            up_pos.resize(3 * n);
            up_dir.resize(3 * n);
            up_weight.resize(n);
            rc = upload_f32(e, up_energy, &G.up_energy);  // sized once per group, filled per batch
            if (!rc) rc = upload_f32(e, up_pos, &G.up_pos);
            if (!rc) rc = upload_f32(e, up_dir, &G.up_dir);
            if (!rc) rc = upload_f32(e, up_weight, &G.up_weight);
        } else {
            G.type = 4;
            G.book_emitted = 1;
            G.n_comp = n_comp;
            std::vector<BeamletRec> slice(recs.begin() + (size_t)g0 * n_comp,
                                          recs.begin() + (size_t)(g0 + gs) * n_comp);
            rc = upload_vec(e, slice, &G.recs);
            if (!rc) rc = upload_f32(e, comp_cdf, &G.comp_cdf);
            if (!rc) rc = upload_f32(e, spec_edges, &G.edges);
            if (!rc) rc = upload_f32(e, spec_cdf, &G.cdf);
            if (!rc) rc = fill_gen_stack(e, G, src->stack, src->stack_mu);
            if (!rc && src->mask) rc = fill_gen_mask(e, G, PMC_MASK_FIELDS(src));
        }
        if (rc) return rc;
        PMC_CUDA(e, cudaMemcpyAsync(e->d_gen, &G, sizeof G, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)(sizeof G);
        PMC_CUDA(e, cudaMemcpyAsync(e->col_nhist.p, nh.data(), sizeof(double) * gs, cudaMemcpyHostToDevice,
                                    e->stream));
    e->h2d_bytes += (unsigned long long)(sizeof(double) * gs);
        rc = begin_maps(e, gs);
        if (!rc) rc = ensure_batch_events(e, 3 * (size_t)p->n_batches);
        if (rc) return rc;
        TransportParams P = make_params(e, p, plan);
        // every batch is enqueued back to back; its timing events are read
        // once the group's last batch is done (no host round trip per batch)
        for (int b = 0; b < p->n_batches; ++b) {
            cudaEvent_t* bev = e->batch_ev.data() + 3 * b;
            if (G.type == 3) {  // this batch's primaries, sampled on the host
                for (int k = 0; k < gs; ++k) {
                    const long long r0 = (long long)b * pb[k];
                    const long long key = (p->correlated ? 0 : off[k]) + r0;
                    const size_t at = (size_t)pre[k];
                    if (src->sample(src->sample_user, g0 + k, key, pb[k], up_energy.data() + at,
                                    up_pos.data() + 3 * at, up_dir.data() + 3 * at,
                                    up_weight.data() + at) != 0)
                        return fail(e, PMC_ERR_INVALID, "the host sampler failed for beamlet %d", g0 + k);
                }
                const size_t n = (size_t)pre[gs];
                PMC_CUDA(e, cudaMemcpyAsync((void*)G.up_energy, up_energy.data(), 4 * n, cudaMemcpyHostToDevice, e->stream));
                PMC_CUDA(e, cudaMemcpyAsync((void*)G.up_pos, up_pos.data(), 12 * n, cudaMemcpyHostToDevice, e->stream));
                PMC_CUDA(e, cudaMemcpyAsync((void*)G.up_dir, up_dir.data(), 12 * n, cudaMemcpyHostToDevice, e->stream));
                PMC_CUDA(e, cudaMemcpyAsync((void*)G.up_weight, up_weight.data(), 4 * n, cudaMemcpyHostToDevice, e->stream));
                e->h2d_bytes += 32ull * n;
            }
            PMC_CUDA(e, cudaEventRecord(bev[0], e->stream));
            rc = run_batch(e, p, plan, P, b, (unsigned long long)pre[gs]);
            if (rc) return rc;
            PMC_CUDA(e, cudaEventRecord(bev[1], e->stream));
            rc = launch_fold(e, n_vox, gs, (const double*)e->col_nhist.p);
            if (rc) return rc;
            PMC_CUDA(e, cudaEventRecord(bev[2], e->stream));
        }
        PMC_CUDA(e, cudaEventSynchronize(e->batch_ev[3 * (size_t)p->n_batches - 1]));
        for (int b = 0; b < p->n_batches; ++b) {
            const cudaEvent_t* bev = e->batch_ev.data() + 3 * b;
            float a = 0, c = 0;
            cudaEventElapsedTime(&a, bev[0], bev[1]);
            cudaEventElapsedTime(&c, bev[1], bev[2]);
            t_tr += a;
            t_red += c;
        }
        Sched s;
        rc = read_sched(e, &s);
        if (rc) return rc;
        rc = check_flags(e, s);
        if (rc) return rc;
        e->edep_clean = true;  // every batch of the group folded: every quanta entry consumed
        // finalize + count + scan, then (after the entry total is known) compact;
        // device time only, the host read of the total in between excluded.
        unsigned long long g_nnz = 0;
        std::vector<long long> g_counts;
        PMC_CUDA(e, cudaEventRecord(e->ev[0], e->stream));
        rc = launch_finalize(e, n_vox, gs, p->n_batches);
        if (rc) return rc;
        PMC_CUDA(e, cudaEventRecord(e->ev[1], e->stream));
        rc = truncate_count(e, n_vox, gs, p->truncation, &g_nnz, &g_counts);
        if (rc) return rc;
        // room for this group's entries; after the first of several groups,
        // for all of them at its density plus a quarter (a few large grows
        // instead of one per group: each grow is an allocation and a copy)
        unsigned long long want = e->csc_nnz + g_nnz;
        if (g0 == 0 && n_beam > gs) {
            const unsigned long long est = (unsigned long long)((double)g_nnz * (double)n_beam / gs * 1.25);
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && est * 24ull < free_b / 2)
                want = std::max(want, est);  // 24 bytes per entry: index, mean, sigma
        }
        rc = grow_keep(e, e->out_idx, sizeof(long long) * want, sizeof(long long) * e->csc_nnz);
        if (!rc) rc = grow_keep(e, e->out_dose, sizeof(double) * want, sizeof(double) * e->csc_nnz);
        if (!rc) rc = grow_keep(e, e->out_sigma, sizeof(double) * want, sizeof(double) * e->csc_nnz);
        if (rc) return rc;
        PMC_CUDA(e, cudaEventRecord(e->ev[2], e->stream));
        rc = truncate_compact(e, n_vox, gs, p->truncation, g_nnz, g_counts);
        if (rc) return rc;
        PMC_CUDA(e, cudaEventRecord(e->ev[3], e->stream));
        PMC_CUDA(e, cudaEventSynchronize(e->ev[3]));
        float c0 = 0, c1 = 0;
        cudaEventElapsedTime(&c0, e->ev[0], e->ev[1]);  // finalize (count+scan ride in the
        cudaEventElapsedTime(&c1, e->ev[2], e->ev[3]);  // synchronizing read; tiny kernels)
        t_red += c0 + c1;
        if (e->progress) {
            long long done = 0;
            for (int k = 0; k < gs; ++k) done += counts[g0 + k];
            e->progress(e->progress_user, done);
        }
    }
    free_run_allocs(e);
    unsigned long long total_q = 0;
    PMC_CUDA(e, cudaMemcpyAsync(&total_q, e->d_total_q, sizeof total_q, cudaMemcpyDeviceToHost, e->stream));
        e->d2h_bytes += (unsigned long long)(sizeof total_q);
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->counters.transport_ms = t_tr;
    e->counters.reduce_ms = t_red;
    *nnz_out = (int64_t)e->csc_nnz;
    if (books) {
        std::memset(books, 0, sizeof *books);
        books->deposited = (int64_t)total_q;
    }
    return finish_counters(e, books);
}

int pmc_dij_fetch(pmc_engine* e, int64_t* indptr, int64_t* indices, double* dose, double* sigma) {
    if (!e || !indptr) return PMC_ERR_INVALID;
    PMC_CUDA(e, cudaSetDevice(e->device));
    const size_t nnz = (size_t)e->csc_nnz;
    std::memcpy(indptr, e->dij_indptr.data(), sizeof(int64_t) * e->dij_indptr.size());
    if (nnz) {
        if (!indices || !dose || !sigma) return fail(e, PMC_ERR_INVALID, "null CSC buffer");
        PMC_CUDA(e, cudaMemcpyAsync(indices, e->out_idx.p, sizeof(int64_t) * nnz, cudaMemcpyDeviceToHost, e->stream));
        PMC_CUDA(e, cudaMemcpyAsync(dose, e->out_dose.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, e->stream));
        PMC_CUDA(e, cudaMemcpyAsync(sigma, e->out_sigma.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, e->stream));
        PMC_CUDA(e, cudaStreamSynchronize(e->stream));
        e->d2h_bytes += 3 * 8 * nnz;
    }
    return PMC_OK;
}

int pmc_dij_device_view(pmc_engine* e, int64_t* indptr, const int64_t** indices,
                        const double** dose, const double** sigma) {
    if (!e || !indptr || !indices || !dose || !sigma) return PMC_ERR_INVALID;
    std::memcpy(indptr, e->dij_indptr.data(), sizeof(int64_t) * e->dij_indptr.size());
    *indices = (const int64_t*)e->out_idx.p;
    *dose = (const double*)e->out_dose.p;
    *sigma = (const double*)e->out_sigma.p;
    return PMC_OK;
}

int pmc_set_stream(pmc_engine* e, void* stream) {
    if (!e) return PMC_ERR_INVALID;
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    e->stream = stream ? (cudaStream_t)stream : e->own_stream;
    return PMC_OK;
}

int pmc_set_progress(pmc_engine* e, pmc_progress_fn fn, void* user) {
    if (!e) return PMC_ERR_INVALID;
    e->progress = fn;
    e->progress_user = user;
    return PMC_OK;
}

int pmc_get_counters(const pmc_engine* e, pmc_counters* c) {
    if (!e || !c) return PMC_ERR_INVALID;
    *c = e->counters;
    c->h2d_bytes_total = (int64_t)e->h2d_bytes;
    c->d2h_bytes_total = (int64_t)e->d2h_bytes;
    return PMC_OK;
}

int pmc_reduce_dense(pmc_engine* e, const int64_t* quanta, int32_t n_batches, int32_t n_cols,
                     int64_t n_vox, const double* voxel_mass, const double* histories_per_batch,
                     double* mean, double* sigma, int64_t* total_quanta) {
    if (!e || !quanta || !voxel_mass || !histories_per_batch || !mean || !sigma) return PMC_ERR_INVALID;
    if (n_batches < 1 || n_cols < 1 || n_vox < 1) return fail(e, PMC_ERR_INVALID, "empty reduction");
    PMC_CUDA(e, cudaSetDevice(e->device));
    int rc = ensure_maps(e, n_cols, n_vox);
    if (!rc) rc = ensure(e, e->col_nhist, sizeof(double) * n_cols);
    if (rc) return rc;
    // The reduction runs against the given masses, not the engine's scoring grid.
    double* saved_mass = e->d_mass;
    double* mass = nullptr;
    PMC_CUDA(e, cudaMalloc(&mass, sizeof(double) * n_vox));
    PMC_CUDA(e, cudaMemcpy(mass, voxel_mass, sizeof(double) * n_vox, cudaMemcpyHostToDevice));
    e->h2d_bytes += (unsigned long long)(sizeof(double) * n_vox);
    PMC_CUDA(e, cudaMemcpy(e->col_nhist.p, histories_per_batch, sizeof(double) * n_cols, cudaMemcpyHostToDevice));
    e->h2d_bytes += (unsigned long long)(sizeof(double) * n_cols);
    e->d_mass = mass;
    rc = begin_maps(e, n_cols);
    PMC_CUDA(e, cudaMemsetAsync(e->d_total_q, 0, sizeof(unsigned long long), e->stream));
    const size_t row = sizeof(int64_t) * (size_t)n_vox, pitch = sizeof(int64_t) * (size_t)e->col_stride;
    for (int b = 0; b < n_batches && !rc; ++b) {
        // The host map is dense: every sector of it counts as deposited.
        PMC_CUDA(e, cudaMemcpy2DAsync(e->edep.p, pitch, quanta + (size_t)b * n_cols * n_vox, row, row,
                                      (size_t)n_cols, cudaMemcpyHostToDevice, e->stream));
        rc = fill_bitmap(e, e->dirty, n_cols, 0xffffffffu);
        if (!rc) rc = launch_fold(e, n_vox, n_cols, (const double*)e->col_nhist.p);
    }
    if (!rc) rc = launch_finalize(e, n_vox, n_cols, n_batches);
    unsigned long long tq = 0;
    if (!rc) {
        cudaMemcpy2DAsync(mean, row, e->s1.p, pitch, row, (size_t)n_cols, cudaMemcpyDeviceToHost, e->stream);
        cudaMemcpy2DAsync(sigma, row, e->s2.p, pitch, row, (size_t)n_cols, cudaMemcpyDeviceToHost, e->stream);
        cudaMemcpyAsync(&tq, e->d_total_q, sizeof tq, cudaMemcpyDeviceToHost, e->stream);
        if (cudaStreamSynchronize(e->stream) == cudaSuccess) e->edep_clean = true;
    }
    e->d_mass = saved_mass;
    cudaFree(mass);
    if (total_quanta) *total_quanta = (int64_t)tq;
    if (rc) return rc;
    PMC_CUDA(e, cudaGetLastError());
    return PMC_OK;
}

int pmc_truncate_dense(pmc_engine* e, const double* mean, const double* sigma, int32_t n_cols,
                       int64_t n_vox, double truncation, int64_t* counts, int64_t* nnz) {
    if (!e || !mean || !sigma || !nnz) return PMC_ERR_INVALID;
    if (n_cols < 1 || n_vox < 1) return fail(e, PMC_ERR_INVALID, "empty truncation");
    if (truncation < 0.0) return fail(e, PMC_ERR_INVALID, "negative truncation %g", truncation);
    PMC_CUDA(e, cudaSetDevice(e->device));
    int rc = ensure_maps(e, n_cols, n_vox);
    if (rc) return rc;
    const size_t row = sizeof(double) * (size_t)n_vox, pitch = sizeof(double) * (size_t)e->col_stride;
    PMC_CUDA(e, cudaMemcpy2DAsync(e->s1.p, pitch, mean, row, row, (size_t)n_cols, cudaMemcpyHostToDevice, e->stream));
    PMC_CUDA(e, cudaMemcpy2DAsync(e->s2.p, pitch, sigma, row, row, (size_t)n_cols, cudaMemcpyHostToDevice, e->stream));
    e->h2d_bytes += (unsigned long long)(2 * row * n_cols);
    rc = fill_bitmap(e, e->touched, n_cols, 0xffffffffu);  // a dense map: every sector counts
    if (rc) return rc;
    rc = ensure_colmax(e, n_cols);
    if (rc) return rc;
    PMC_CUDA(e, cudaMemsetAsync(e->d_colmax, 0, sizeof(unsigned long long) * n_cols, e->stream));
    {
        const int n_tiles = (int)(e->col_stride / kTileVoxels);
        colmax_kernel<<<dim3(n_tiles, n_cols), kReduceThreads, 0, e->stream>>>(
            (const double*)e->s1.p, n_vox, e->col_stride, e->d_colmax);
        PMC_CUDA(e, cudaGetLastError());
    }
    e->dij_indptr.assign(1, 0);
    e->csc_nnz = 0;
    unsigned long long t_nnz = 0;
    std::vector<long long> t_counts;
    rc = truncate_count(e, n_vox, n_cols, truncation, &t_nnz, &t_counts);
    if (!rc) rc = truncate_compact(e, n_vox, n_cols, truncation, t_nnz, t_counts);
    if (rc) return rc;
    PMC_CUDA(e, cudaStreamSynchronize(e->stream));
    if (counts)
        for (int c = 0; c < n_cols; ++c) counts[c] = e->dij_indptr[c + 1] - e->dij_indptr[c];
    *nnz = (int64_t)e->csc_nnz;
    return PMC_OK;
}

}  // extern "C"

// ============================================================================
// Allocation-free truncation + CSC compaction (pmc_dij_compact_static)
// ============================================================================
// Some callers cannot call cudaMalloc: an application that owns all device
// memory through its own pool or allocator, or a process that forbids
// allocation after start-up so its footprint stays fixed.  For them the
// truncation + compaction scratch (column maxima, per-tile counts and offsets,
// per-column counts, the entry total) lives in this file-scope device array
// instead of engine-owned buffers.  Every GPU that loads the library holds it
// until the process exits.  The call reads the entry total back to the host
// and synchronizes its stream, so it cannot be recorded into a CUDA graph.
namespace {

constexpr int kStaticMaxCols = 4096;
constexpr long long kStaticMaxTiles = 262144;  // columns x ceil(voxels / 4096)

struct StaticScratch {
    unsigned long long col_max[kStaticMaxCols];
    long long col_counts[kStaticMaxCols];
    unsigned long long total;
    unsigned long long pad[31];
    unsigned int tile_counts[kStaticMaxTiles];
    unsigned long long tile_offsets[kStaticMaxTiles];
};

static __device__ __align__(256) StaticScratch g_static_scratch;

constexpr int kStaticMaxDevices = 64;
StaticScratch* g_scratch_ptr[kStaticMaxDevices] = {};
std::mutex g_scratch_mutex;

// Host code cannot use g_static_scratch's address directly (on the host the
// name is only a stand-in for the device symbol), so the device address is
// looked up once per device, with that device current, and kept for the life
// of the process (a cudaDeviceReset of the device would invalidate it).
cudaError_t static_scratch(int device, StaticScratch** out) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (device < 0 || device >= kStaticMaxDevices) return cudaErrorInvalidDevice;
    if (!g_scratch_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t st = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (st != cudaSuccess) return st;
        g_scratch_ptr[device] = (StaticScratch*)ptr;
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" {

int pmc_dij_compact_static(const double* mean, const double* sigma, int32_t n_cols, int64_t n_vox,
                           double truncation, int64_t out_capacity, int64_t* col_counts,
                           int64_t* out_indices, double* out_dose, double* out_sigma,
                           int64_t* nnz, void* stream) {
    if (!mean || !sigma || !col_counts || !nnz || n_cols < 1 || n_vox < 1 || out_capacity < 0)
        return PMC_ERR_INVALID;
    if (!(truncation >= 0.0)) return PMC_ERR_INVALID;
    const long long n_tiles = (n_vox + kTileVoxels - 1) / kTileVoxels;
    if (n_cols > kStaticMaxCols || n_tiles * n_cols > kStaticMaxTiles)
        return PMC_ERR_INVALID;  // beyond the static scratch: at most 4096 columns and
                                 // 262144 tiles of 4096 voxels
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return PMC_ERR_CUDA;
    StaticScratch* scratch = nullptr;
    if (static_scratch(device, &scratch) != cudaSuccess) return PMC_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    // The array keeps the previous call's contents: the maxima must restart at 0.
    if (cudaMemsetAsync(scratch->col_max, 0, sizeof(unsigned long long) * n_cols, st) != cudaSuccess)
        return PMC_ERR_CUDA;
    const dim3 grid((unsigned)n_tiles, (unsigned)n_cols);
    colmax_kernel<<<grid, kReduceThreads, 0, st>>>(mean, n_vox, n_vox, scratch->col_max);
    count_kept_kernel<<<grid, kReduceThreads, 0, st>>>(mean, n_vox, (int)n_tiles, truncation,
                                                        scratch->col_max, scratch->tile_counts);
    scan_tiles_kernel<<<1, 1024, 0, st>>>(scratch->tile_counts, n_tiles * n_cols,
                                          scratch->tile_offsets, n_cols, (int)n_tiles,
                                          scratch->col_counts, &scratch->total);
    if (cudaGetLastError() != cudaSuccess) return PMC_ERR_CUDA;
    unsigned long long total = 0;
    if (cudaMemcpyAsync(&total, &scratch->total, sizeof total, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PMC_ERR_CUDA;
    *nnz = (int64_t)total;
    // Too small: report the size needed; neither out_* nor col_counts is written.
    if ((long long)total > out_capacity) return PMC_ERR_CAPACITY;
    if (total > 0) {
        if (!out_indices || !out_dose || !out_sigma) return PMC_ERR_INVALID;
        compact_kernel<<<grid, kReduceThreads, 0, st>>>(
            mean, sigma, n_vox, (int)n_tiles, truncation, scratch->col_max, scratch->tile_offsets,
            (long long*)out_indices, out_dose, out_sigma);
    }
    if (cudaMemcpyAsync(col_counts, scratch->col_counts, sizeof(long long) * n_cols,
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return PMC_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return PMC_ERR_CUDA;
    return PMC_OK;
}

}  // extern "C"
