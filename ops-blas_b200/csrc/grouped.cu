// aclblasSgetrfGetrsGrouped*: factor and solve many matrices of different orders in one
// persistent launch. No counterpart in the reference (an extension beside the drop-in chain);
// per instance the results are bit-identical to aclblasSgetrfBatched followed by
// aclblasSgetrsBatched (trans N) on the same matrix, because the same LU and solve building
// blocks (lu_core.cuh) run here.
//
// A plan describes the batch: groups of instances that share n, nrhs, lda and ldb. Creating it
// chooses, per group, the lanes per matrix (n <= 32) or the warps per matrix and rows per lane
// (32 < n <= 128) from a tuning table written by autotune_grouped.py (or from the caller),
// orders the work largest first, and uploads the task lists to the device. Each execution is
// then one launch of grouped_lu_kernel on the handle's stream (plus the regular batched kernels
// for groups with n > 128): a grid of one wave of 256-thread CTAs that take tasks from two
// device counters --
//   phase 1, CTA tasks (n > 32): the CTA (8 warps) or each 4-warp / 2-warp team factors one matrix
//     held in registers (reg_getrf_core), stores LU, pivots and info, and solves the
//     right-hand sides from a copy of the factors in shared memory (med_solve_core);
//   phase 2, warp tasks (n <= 32): each warp takes 32/lanes matrices, factors them in
//     registers (small_getrf_core) and solves from the registers (small_solve_core).
// The last CTA to finish resets the counters, so consecutive executions on one stream need no
// host work, and executions of one plan must not overlap in time.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "internal.h"
#include "lu_core.cuh"

namespace opsblas {

constexpr int kGrpThreads = 256;
constexpr int kGrpWarps = kGrpThreads / 32;
constexpr int kGrpMaxN = 128;  // larger orders use the batched kernels

struct GroupDev {
    int n, nrhs, lda, ldb;
    long long piv_off;  // first pivot of the group's first instance
    int first;          // index of the group's first instance in the pointer arrays
    int lanes;          // n <= 32: lanes per matrix (SEG)
    int warps;          // n > 32: warps per matrix (2, 4 or 8)
    int rows;           // n > 32: rows per lane (2, 3 or 4; 32 * rows >= n)
    int team_floats;    // n > 32: shared-memory floats between consecutive teams' staged factors
    int pad;
};

struct GroupTask {
    int group;
    int first;  // first instance within the group
    int count;  // instances in this task
    int pad;
};

// ------------------------------------------------------------------------------ n > 32 --
// One matrix per team of NW warps: registers hold the matrix (reg_getrf_core). With right-hand
// sides, the factors are also staged in the team's shared memory (physical rows, odd column
// stride) so that the team's warps solve their columns from there (med_solve_core) while the
// factors go to global memory.
template <int R, int NW>
__device__ __forceinline__ void grouped_reg(const GroupDev& g, int li, float* const* Aarray, float* const* Barray,
                                            int* piv, int* info, RegTeamSmem& S, float* sa, int warp, int lane,
                                            int bar)
{
    constexpr int CW = RegShape<R, NW>::CW;
    const int n = g.n;
    const long long inst = (long long)g.first + li;
    float* A = Aarray[inst];
    int* pm = piv + g.piv_off + (long long)li * n;
    float a[R][CW];
    int pos[R];
    reg_load<R, NW>(a, A, g.lda, n, warp, lane);
#pragma unroll
    for (int t = 0; t < R; t++) pos[t] = lane + 32 * t;
    for (int i = warp * 32 + lane; i < n; i += NW * 32) pm[i] = 0;
    team_sync<NW * 32>(bar);
    const int inf = reg_getrf_core<R, NW, true>(a, pos, n, S, pm, warp, lane, bar);
    const int ld = n | 1;
    if (g.nrhs > 0) {
#pragma unroll
        for (int s = 0; s < CW; s++) {
            const int j = s * NW + warp;
#pragma unroll
            for (int t = 0; t < R; t++) {
                const int p = lane + 32 * t;
                if (p < n && j < n) sa[p + j * ld] = a[t][s];
            }
        }
        if (warp == 0) {
#pragma unroll
            for (int t = 0; t < R; t++)
                if (lane + 32 * t < n) S.lmap[pos[t]] = lane + 32 * t;
        }
    }
    reg_store<R, NW>(a, pos, A, g.lda, n, warp, lane);
    if (g.nrhs > 0) {
        team_sync<NW * 32>(bar);  // staged factors and row map visible to the team
        float* Bm = Barray[inst];
        for (int c = warp; c < g.nrhs; c += NW) {
            float* bc = Bm + (long long)c * g.ldb;
            float y[kMedRows];
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                const int i = lane + 32 * t;
                y[t] = i < n ? bc[S.lmap[i]] : 0.0f;
            }
            __syncwarp();  // every lane has read its b before any lane writes x
            med_solve_core(sa, S.lmap, n, ld, lane, y);
            __syncwarp();
#pragma unroll
            for (int t = 0; t < kMedRows; t++) {
                const int i = lane + 32 * t;
                if (i < n) bc[i] = y[t];
            }
        }
    }
    if (warp == 0 && lane == 0) info[inst] = inf;
}

template <int NW>
__device__ __forceinline__ void grouped_reg_dispatch(const GroupDev& g, int li, float* const* Aarray,
                                                     float* const* Barray, int* piv, int* info, RegTeamSmem& S,
                                                     float* sa, int warp, int lane, int bar)
{
    if (NW == 2) {
        grouped_reg<2, 2>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
    } else if (NW == 4) {
        if (g.rows == 2)
            grouped_reg<2, 4>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
        else
            grouped_reg<3, 4>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
    } else {
        if (g.rows == 2)
            grouped_reg<2, 8>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
        else if (g.rows == 3)
            grouped_reg<3, 8>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
        else
            grouped_reg<4, 8>(g, li, Aarray, Barray, piv, info, S, sa, warp, lane, bar);
    }
}

// ----------------------------------------------------------------------------- n <= 32 --
template <int N, int SEG>
__device__ __forceinline__ void grouped_small(const GroupDev& g, const GroupTask& task, float* const* Aarray,
                                              float* const* Barray, int* piv, int* info, float* rowbuf, int* owner,
                                              int lane)
{
    constexpr int NC = (N + 3) / 4;
    const int seg = lane / SEG;
    const int r = lane % SEG;
    const int li = task.first + seg;
    const bool mvalid = seg < task.count;
    const bool rvalid = mvalid && r < N;
    const long long inst = (long long)g.first + li;
    const int lda = g.lda;
    float* A = mvalid ? Aarray[inst] : nullptr;
    float4 a4[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) a4[c] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (rvalid) {
        const float* Ar = A + r;
#pragma unroll
        for (int j = 0; j < N; j++) qset<N>(a4, j, Ar[(long long)j * lda]);
    }
    int pos, mypiv, inf;
    small_getrf_core<N, true, SEG>(a4, pos, mypiv, inf, rowbuf, seg, r, mvalid, rvalid);
    if (g.nrhs > 0) {
        float* Bm = mvalid ? Barray[inst] : nullptr;
        for (int c = 0; c < g.nrhs; c++) {
            float* bc = rvalid ? Bm + (long long)c * g.ldb : nullptr;
            float y = rvalid ? bc[r] : 0.0f;
            y = small_solve_core<N, SEG>(a4, pos, rvalid, seg, r, owner + seg * SEG, y);
            if (rvalid) bc[pos] = y;
        }
    }
    if (rvalid) {
        float* Ap = A + pos;
#pragma unroll
        for (int j = 0; j < N; j++) Ap[(long long)j * lda] = qget<N>(a4, j);
        piv[g.piv_off + (long long)li * N + r] = mypiv;
        if (r == 0) info[inst] = inf;
    }
}

template <int N>
__device__ __forceinline__ void grouped_small_dispatch(const GroupDev& g, const GroupTask& task,
                                                       float* const* Aarray, float* const* Barray, int* piv,
                                                       int* info, float* rowbuf, int* owner, int lane)
{
    constexpr int NAT = SmallShape<N>::SEG;
    if (NAT == 32 || g.lanes == NAT)
        grouped_small<N, NAT>(g, task, Aarray, Barray, piv, info, rowbuf, owner, lane);
    else
        grouped_small<N, 32>(g, task, Aarray, Barray, piv, info, rowbuf, owner, lane);
}

__global__ void __launch_bounds__(kGrpThreads, 2)
grouped_lu_kernel(const GroupDev* groups, const GroupTask* __restrict__ cta_tasks, int n_cta,
                  const GroupTask* __restrict__ warp_tasks, int n_warp, int* __restrict__ counters,
                  float* const* Aarray, float* const* Barray, int* piv, int* info)
{
    extern __shared__ __align__(16) float dyn[];  // per team: staged factors for the solve
    __shared__ RegTeamSmem team[4];
    __shared__ int s_task;
    __shared__ __align__(16) float rowbuf[kGrpWarps][2][32];
    __shared__ int owner[kGrpWarps][32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // phase 1: one matrix per CTA (or per 4-warp team), largest first
    for (;;) {
        if (tid == 0) s_task = atomicAdd(&counters[0], 1);
        __syncthreads();
        const int t = s_task;
        __syncthreads();
        if (t >= n_cta) break;
        const GroupTask task = cta_tasks[t];
        const GroupDev& g = groups[task.group];  // fields read when needed: fewer live registers
        if (g.warps == 2) {  // four 2-warp teams, one matrix each
            const int tm = warp >> 1;
            if (tm < task.count)
                grouped_reg_dispatch<2>(g, task.first + tm, Aarray, Barray, piv, info, team[tm],
                                        dyn + (size_t)tm * g.team_floats, warp & 1, lane, 1 + tm);
        } else if (g.warps == 4) {
            const int tm = warp >> 2;
            if (tm < task.count)
                grouped_reg_dispatch<4>(g, task.first + tm, Aarray, Barray, piv, info, team[tm],
                                        dyn + (size_t)tm * g.team_floats, warp & 3, lane,
                                        1 + tm);
        } else {
            grouped_reg_dispatch<8>(g, task.first, Aarray, Barray, piv, info, team[0], dyn, warp, lane, -1);
        }
    }

    // phase 2: warp tasks, each warp on its own
    for (;;) {
        __syncwarp();  // the previous task's shared-memory reads are done before rowbuf is reused
        int t = 0;
        if (lane == 0) t = atomicAdd(&counters[1], 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_warp) break;
        const GroupTask task = warp_tasks[t];
        const GroupDev g = groups[task.group];
        switch (g.n) {
#define OPSBLAS_GROUPED_CASE(NN)                                                                                    \
    case NN:                                                                                                        \
        grouped_small_dispatch<NN>(g, task, Aarray, Barray, piv, info, &rowbuf[warp][0][0], owner[warp], lane);     \
        break;
            OPSBLAS_FOR_N_1_32(OPSBLAS_GROUPED_CASE)
#undef OPSBLAS_GROUPED_CASE
            default:
                break;
        }
    }

    // the last CTA out resets the counters for the next execution
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const int f = atomicAdd(&counters[2], 1);
        if (f == (int)gridDim.x - 1) {
            atomicExch(&counters[0], 0);
            atomicExch(&counters[1], 0);
            atomicExch(&counters[2], 0);
        }
    }
}

// ------------------------------------------------------------------------- host side --
struct TuneRow {
    int lo, hi, lanes, warps, rows;
};

// Built-in choices, used when no tuning table is found: natural lanes; 8 warps, ceil(n/32) rows.
static void default_config(int n, int cfg[3])
{
    if (n <= 32) {
        cfg[0] = n <= 4 ? 4 : (n <= 8 ? 8 : (n <= 16 ? 16 : 32));
        cfg[1] = 0;
        cfg[2] = 0;
    } else {
        cfg[0] = 0;
        reg_default_shape(n, cfg[2], cfg[1]);
    }
}

static std::string tuning_path()
{
    const char* env = std::getenv("OPSBLAS_GROUPED_TUNING");
    if (env && *env) return env;
    Dl_info dli;
    if (dladdr(reinterpret_cast<void*>(&default_config), &dli) && dli.dli_fname) {
        std::string p(dli.dli_fname);
        const size_t s = p.rfind('/');
        return (s == std::string::npos ? std::string(".") : p.substr(0, s)) + "/grouped_tuning.txt";
    }
    return "grouped_tuning.txt";
}

// Table rows "n_lo n_hi lanes warps rows"; '#' starts a comment.
static std::vector<TuneRow> load_tuning()
{
    std::vector<TuneRow> rows;
    FILE* f = std::fopen(tuning_path().c_str(), "r");
    if (!f) return rows;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        TuneRow r;
        if (std::sscanf(line, "%d %d %d %d %d", &r.lo, &r.hi, &r.lanes, &r.warps, &r.rows) == 5) rows.push_back(r);
    }
    std::fclose(f);
    return rows;
}

// Makes cfg valid for n: lanes in {natural, 32} (n <= 32); an instantiated (rows, warps) shape
// with 32 * rows >= n (n > 32).
static void sanitize_config(int n, int cfg[3])
{
    int def[3];
    default_config(n, def);
    if (n <= 32) {
        if (cfg[0] != def[0] && cfg[0] != 32) cfg[0] = def[0];
        cfg[1] = 0;
        cfg[2] = 0;
    } else {
        cfg[0] = 0;
        if (!reg_shape_valid(n, cfg[2], cfg[1])) {
            cfg[1] = def[1];
            cfg[2] = def[2];
        }
    }
}

struct GroupHost {
    int n, nrhs, lda, ldb, size, first;
    long long piv_off;
    int cfg[3];
};

}  // namespace opsblas

struct _aclblas_grouped_plan {
    int device = 0;
    std::vector<opsblas::GroupHost> groups;
    int total = 0;
    void* dmem = nullptr;
    opsblas::GroupDev* d_groups = nullptr;
    opsblas::GroupTask* d_cta = nullptr;
    opsblas::GroupTask* d_warp = nullptr;
    int* d_counters = nullptr;
    int n_cta = 0, n_warp = 0;
    int grid = 0;
    size_t smem = 0;      // dynamic shared memory per CTA
    bool has_persistent = false;
};

using namespace opsblas;

extern "C" aclblasStatus_t aclblasSgetrfGetrsGroupedPlanCreate(aclblasHandle_t handle, int groupCount,
                                                               const int nArray[], const int nrhsArray[],
                                                               const int ldaArray[], const int ldbArray[],
                                                               const int groupSizeArray[], const int* configArray,
                                                               aclblasGroupedPlan_t* plan)
{
    static const char* kApi = "aclblasSgetrfGetrsGroupedPlanCreate";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (plan == nullptr || groupCount < 0) {
        log_error(kApi, "plan must not be nullptr and groupCount must be >= 0");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    *plan = nullptr;
    if (groupCount > 0 && (!nArray || !nrhsArray || !ldaArray || !ldbArray || !groupSizeArray)) {
        log_error(kApi, "group arrays must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    long long total = 0;
    for (int g = 0; g < groupCount; g++) {
        const int n = nArray[g];
        if (n < 0 || nrhsArray[g] < 0 || groupSizeArray[g] < 0 || ldaArray[g] < max1(n) || ldbArray[g] < max1(n)) {
            log_error(kApi, "group %d: n=%d nrhs=%d lda=%d ldb=%d size=%d is invalid", g, n, nrhsArray[g],
                      ldaArray[g], ldbArray[g], groupSizeArray[g]);
            return ACLBLAS_STATUS_INVALID_VALUE;
        }
        total += groupSizeArray[g];
    }
    if (total > 0x7fffffffLL) {
        log_error(kApi, "more than 2^31-1 instances");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }

    auto* p = new _aclblas_grouped_plan();
    p->device = handle->device;
    const std::vector<TuneRow> table = load_tuning();
    long long piv_off = 0;
    int first = 0;
    for (int g = 0; g < groupCount; g++) {
        GroupHost h;
        h.n = nArray[g];
        h.nrhs = nrhsArray[g];
        h.lda = ldaArray[g];
        h.ldb = ldbArray[g];
        h.size = groupSizeArray[g];
        h.first = first;
        h.piv_off = piv_off;
        default_config(h.n, h.cfg);
        for (const TuneRow& r : table)
            if (h.n >= r.lo && h.n <= r.hi) {
                h.cfg[0] = r.lanes;
                h.cfg[1] = r.warps;
                h.cfg[2] = r.rows;
            }
        if (configArray) {
            for (int q = 0; q < 3; q++)
                if (configArray[3 * g + q] > 0) h.cfg[q] = configArray[3 * g + q];
        }
        sanitize_config(h.n, h.cfg);
        first += h.size;
        piv_off += (long long)h.n * h.size;
        p->groups.push_back(h);
    }
    p->total = first;

    // task lists, largest matrices first
    std::vector<int> order(groupCount);
    for (int g = 0; g < groupCount; g++) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p->groups[a].n > p->groups[b].n; });
    std::vector<GroupTask> cta, warp;
    size_t smem = 0;
    std::vector<int> team_stride(std::max(groupCount, 1), 0);
    for (int g : order) {
        const GroupHost& h = p->groups[g];
        if (h.n == 0 || h.size == 0 || h.n > kGrpMaxN) continue;
        if (h.n > 32) {
            const int per = kGrpWarps / h.cfg[1];  // matrices per CTA task (teams)
            for (int i = 0; i < h.size; i += per) cta.push_back({g, i, std::min(per, h.size - i), 0});
            if (h.nrhs > 0) {
                // staged factors, 16-byte rounded; team t's region starts at t * f, the teams of a
                // CTA stage side by side
                const size_t f = ((size_t)(h.n | 1) * h.n + 3) & ~(size_t)3;
                team_stride[g] = (int)f;
                smem = std::max(smem, (size_t)per * f * 4);
            }
        } else {
            const int per = 32 / h.cfg[0];
            for (int i = 0; i < h.size; i += per) warp.push_back({g, i, std::min(per, h.size - i), 0});
        }
    }
    p->n_cta = (int)cta.size();
    p->n_warp = (int)warp.size();
    p->has_persistent = p->n_cta + p->n_warp > 0;
    p->smem = smem;

    std::vector<GroupDev> gd(std::max(groupCount, 1));
    for (int g = 0; g < groupCount; g++) {
        const GroupHost& h = p->groups[g];
        gd[g] = {h.n, h.nrhs, h.lda, h.ldb, h.piv_off, h.first, h.cfg[0], h.cfg[1], h.cfg[2], team_stride[g], 0};
    }
    if (p->has_persistent) {
        const size_t bg = gd.size() * sizeof(GroupDev);
        const size_t bc = std::max<size_t>(cta.size(), 1) * sizeof(GroupTask);
        const size_t bw = std::max<size_t>(warp.size(), 1) * sizeof(GroupTask);
        cudaError_t err = cudaMalloc(&p->dmem, bg + bc + bw + 256);
        if (err != cudaSuccess) {
            log_error(kApi, "cannot allocate %zu bytes for the plan", bg + bc + bw + 256);
            delete p;
            return ACLBLAS_STATUS_ALLOC_FAILED;
        }
        char* d = static_cast<char*>(p->dmem);
        p->d_counters = reinterpret_cast<int*>(d);
        p->d_groups = reinterpret_cast<GroupDev*>(d + 256);
        p->d_cta = reinterpret_cast<GroupTask*>(d + 256 + bg);
        p->d_warp = reinterpret_cast<GroupTask*>(d + 256 + bg + bc);
        err = cudaMemset(p->d_counters, 0, 256);
        if (err == cudaSuccess) err = cudaMemcpy(p->d_groups, gd.data(), bg, cudaMemcpyHostToDevice);
        if (err == cudaSuccess && !cta.empty())
            err = cudaMemcpy(p->d_cta, cta.data(), cta.size() * sizeof(GroupTask), cudaMemcpyHostToDevice);
        if (err == cudaSuccess && !warp.empty())
            err = cudaMemcpy(p->d_warp, warp.data(), warp.size() * sizeof(GroupTask), cudaMemcpyHostToDevice);
        if (err == cudaSuccess)
            err = ensure_smem_limit(grouped_lu_kernel, (int)std::max<size_t>(p->smem, 1));
        int per_sm = 0;
        if (err == cudaSuccess)
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_lu_kernel, kGrpThreads, p->smem);
        if (err != cudaSuccess || per_sm < 1) {
            log_error(kApi, "plan set-up failed: %s", cudaGetErrorString(err));
            cudaFree(p->dmem);
            delete p;
            return err != cudaSuccess ? launch_status(kApi, err) : ACLBLAS_STATUS_NOT_SUPPORTED;
        }
        const long long want = (long long)p->n_cta + (p->n_warp + kGrpWarps - 1) / kGrpWarps;
        p->grid = (int)std::max(1LL, std::min<long long>(want, (long long)per_sm * sm_count()));
    }
    *plan = p;
    return ACLBLAS_STATUS_SUCCESS;
}

extern "C" aclblasStatus_t aclblasSgetrfGetrsGroupedPlanGetConfig(aclblasGroupedPlan_t plan, int* configArray)
{
    if (plan == nullptr || configArray == nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    for (size_t g = 0; g < plan->groups.size(); g++)
        for (int q = 0; q < 3; q++) configArray[3 * g + q] = plan->groups[g].cfg[q];
    return ACLBLAS_STATUS_SUCCESS;
}

extern "C" aclblasStatus_t aclblasSgetrfGetrsGroupedPlanDestroy(aclblasGroupedPlan_t plan)
{
    if (plan == nullptr) return ACLBLAS_STATUS_INVALID_VALUE;
    if (plan->dmem) cudaFree(plan->dmem);
    delete plan;
    return ACLBLAS_STATUS_SUCCESS;
}

extern "C" aclblasStatus_t aclblasSgetrfGetrsGroupedBatched(aclblasHandle_t handle, aclblasGroupedPlan_t plan,
                                                            float* const Aarray[], int* PivotArray, int* infoArray,
                                                            float* const Barray[])
{
    static const char* kApi = "aclblasSgetrfGetrsGroupedBatched";
    if (handle == nullptr) {
        log_error(kApi, "handle is nullptr");
        return ACLBLAS_STATUS_HANDLE_IS_NULLPTR;
    }
    if (plan == nullptr) {
        log_error(kApi, "plan is nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (plan->total == 0) return ACLBLAS_STATUS_SUCCESS;
    bool need_b = false;
    for (const GroupHost& h : plan->groups) need_b |= h.nrhs > 0 && h.n > 0 && h.size > 0;
    if (!Aarray || !PivotArray || !infoArray || (need_b && !Barray)) {
        log_error(kApi, "Aarray, PivotArray, infoArray (and Barray when a group has nrhs > 0) must not be nullptr");
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    if (handle->device != plan->device) {
        log_error(kApi, "the plan was made on device %d, the handle is on device %d", plan->device, handle->device);
        return ACLBLAS_STATUS_INVALID_VALUE;
    }
    cudaStream_t st = handle->stream;
    if (plan->has_persistent) {
        grouped_lu_kernel<<<(unsigned)plan->grid, kGrpThreads, plan->smem, st>>>(
            plan->d_groups, plan->d_cta, plan->n_cta, plan->d_warp, plan->n_warp, plan->d_counters, Aarray, Barray,
            PivotArray, infoArray);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return launch_status(kApi, err);
    }
    // groups beyond the persistent kernel's sizes: the regular batched kernels
    for (const GroupHost& h : plan->groups) {
        if (h.n <= kGrpMaxN || h.size == 0) continue;
        aclblasStatus_t s = aclblasSgetrfBatched(handle, h.n, Aarray + h.first, h.lda, PivotArray + h.piv_off,
                                                 infoArray + h.first, h.size);
        if (s != ACLBLAS_STATUS_SUCCESS) return s;
        if (h.nrhs > 0) {
            cudaError_t err = getrs_launch(st, false, h.n, h.nrhs, Aarray + h.first, h.lda, PivotArray + h.piv_off,
                                           Barray + h.first, h.ldb, h.size);
            if (err != cudaSuccess) return launch_status(kApi, err);
        }
    }
    return ACLBLAS_STATUS_SUCCESS;
}
