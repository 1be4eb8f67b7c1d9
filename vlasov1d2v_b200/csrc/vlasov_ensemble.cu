// Batched heterogeneous ensemble: many independent problems (different grids, orders and
// physics) advanced by one set of launches per RK stage.
//
// Each member is an ordinary vl_ctx with its own state buffers and loop state.  Per RK stage the
// ensemble issues the forward DFT of every member's field solve and the inverse DFT (+ loop
// bookkeeping) as one launch each, then the stage work in one of two forms:
//   fused     one persistent kernel whose CTAs walk a precomputed list of work items (member,
//             x element, tile group), built on the host by longest-processing-time-first
//             assignment of estimated costs; block size, CTAs per SM and items per CTA are the
//             schedule's tunables;
//   by order  one persistent kernel per order present, compiled for that order alone, over its
//             own item list (member-major, least-loaded CTA first); orders marked native instead
//             launch each member through its own context's single-problem stage kernel; all
//             launches of a stage run on concurrent streams forked from the caller's.
// The autotuner in vlasov1d2v_b200/ensemble.py picks among them.
//
// The ensemble kernels run the register-pencil tile body (orders 1..9) with the order-specific
// up / xi tables in constant memory; the member's velocity weights and scalars come from its
// descriptor.  Members whose loop state is inactive (final time reached) are skipped by every
// kernel, so a batch of K steps is correct for members of any final time.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <queue>
#include <string>
#include <type_traits>
#include <vector>

#include "vlasov_ctx.cuh"
#include "vlasov_field.cuh"
#include "vlasov_stage.cuh"

namespace vl {

template <typename T>
struct EnsTables {
    T up[NMAX * NMAX];
    T xi[NMAX * 2];
};

__constant__ EnsTables<double> c_ens64[NMAX + 1];
__constant__ EnsTables<float> c_ens32[NMAX + 1];

template <typename T>
__device__ __forceinline__ const EnsTables<T> &ens_tables(int n);
template <>
__device__ __forceinline__ const EnsTables<double> &ens_tables<double>(int n) { return c_ens64[n]; }
template <>
__device__ __forceinline__ const EnsTables<float> &ens_tables<float>(int n) { return c_ens32[n]; }

struct EnsMember {
    StageArgs a;               // scalars and pointers; in / fn / out / kind set per stage
    const void *f, *sa, *sb;   // the member's state and stage buffers
    int n;
    int G;                     // CTA groups per x element (moment partials per element)
    double qw[NMAX * NMAX];    // w_j w_k / (J_u J_v)
};

struct EnsItem {
    int member, e, g, pad;
};

// RK stage s of the nonlinear SSP-RK3 (main/timestep.py:157-163, :174-182)
__host__ __device__ __forceinline__ void ens_stage_args(StageArgs &a, const EnsMember &m, int s) {
    if (s == 0) {
        a.in = m.f;
        a.fn = nullptr;
        a.out = const_cast<void *>(m.sa);
        a.ghost_out = const_cast<void *>(m.f);
        a.kind = KIND_EULER;
    } else if (s == 1) {
        a.in = m.sa;
        a.fn = m.f;
        a.out = const_cast<void *>(m.sb);
        a.ghost_out = nullptr;
        a.kind = KIND_COMBINE;
        a.c0 = 3.0 / 4.0;
        a.c1 = 1.0 / 4.0;
        a.c2 = 1.0 / 4.0;
    } else {
        a.in = m.sb;
        a.fn = m.f;
        a.out = const_cast<void *>(m.f);
        a.ghost_out = nullptr;
        a.kind = KIND_COMBINE;
        a.c0 = 1.0 / 3.0;
        a.c1 = 2.0 / 3.0;
        a.c2 = 2.0 / 3.0;
    }
}

template <int N>
struct EnsJC {
    // j values per thread so that NT / 32 warps cover the n rows
    template <int NT>
    static constexpr int jc() { return (N + NT / 32 - 1) / (NT / 32); }
};

template <typename T, int NT>
__global__ void __launch_bounds__(NT) ens_stage_kernel(const EnsMember *__restrict__ members,
                                                      const int *__restrict__ cta_items,
                                                      const EnsItem *__restrict__ items, int stage) {
    __shared__ StageArgs sArgs;
    __shared__ int sActive;
    for (int it = cta_items[blockIdx.x]; it < cta_items[blockIdx.x + 1]; ++it) {
        const EnsItem item = items[it];
        const EnsMember &m = members[item.member];
        __syncthreads();   // the previous item is done with the shared arguments and tiles
        if (threadIdx.x == 0) {
            StageArgs a = m.a;
            ens_stage_args(a, m, stage);
            sArgs = a;
            sActive = (a.state == nullptr) || (a.state->active != 0);
        }
        __syncthreads();
        if (!sActive) continue;
        const int n = m.n;
        switch (n) {
#define VL_ENS_CASE(NN)                                                                            \
    case NN:                                                                                       \
        pencil_stage_body<NN, T, EnsJC<NN>::template jc<NT>(), NT, EnsTables<T>>(                 \
            sArgs, ens_tables<T>(NN), m.qw, item.e, item.g, m.G);                                  \
        break;
            VL_ENS_CASE(1)
            VL_ENS_CASE(2)
            VL_ENS_CASE(3)
            VL_ENS_CASE(4)
            VL_ENS_CASE(5)
            VL_ENS_CASE(6)
            VL_ENS_CASE(7)
            VL_ENS_CASE(8)
            VL_ENS_CASE(9)
#undef VL_ENS_CASE
            default: break;
        }
    }
}

// Register cap of the by-order kernels.  The body reads its arguments from shared memory (they
// differ per work item), not from the constant bank as the single-problem kernel does, and needs
// more registers: at a cap of 128 the order-9 FP32 body spills 624 bytes; uncapped (255) it uses
// 254 registers without spills and the 64-member benchmark ensemble steps in 4.09 ms against
// 4.26 ms at a cap of 168 and 4.35 ms at 128.
// order groups of a by-order stage launched on concurrent streams (1) or one after another (0)
#ifndef VL_ENS_CONCURRENT
#define VL_ENS_CONCURRENT 1
#endif

#ifndef VL_ENS_REG_CAP
#define VL_ENS_REG_CAP 255
#endif

// j values per thread of the FP32 by-order kernels (capped at the order): one warp per CTA with
// all j rows for orders up to 8.  64-member FP32 ensemble, ms per step at 8 items per CTA: 3.99
// with the single-problem kernel's 4 (two warps per CTA for orders 5..8), 3.24 with 8, 6.3 with
// 2 and 10.8 with 1; the one-warp CTAs synchronise within a warp and hold more rows in registers.
// FP64 keeps the single-problem kernel's 2.
#ifndef VL_ENS_JC32
#define VL_ENS_JC32 8
#endif

// block shape and resident CTAs per SM requested from the compiler for one order's kernel
template <int N, typename T>
struct EnsOrderGeom {
    static constexpr int JC0 = sizeof(T) == 4 ? (VL_ENS_JC32 < N ? VL_ENS_JC32 : N) : PencilGeom<N, T>::JC;
    static constexpr int JS = (N + JC0 - 1) / JC0;              // warps (j chunks)
    static constexpr int JC = (N + JS - 1) / JS;                // balanced chunk
    static constexpr int THREADS = 32 * JS;
    static constexpr int MIN_BLOCKS = 65536 / (THREADS * VL_ENS_REG_CAP) > 0 ? 65536 / (THREADS * VL_ENS_REG_CAP) : 1;
    static constexpr size_t smem_bytes() { return PencilGeom<N, T>::se_offset(THREADS) + sizeof(double) * N; }
};

// The members of one order only, with the register-pencil tile body: one body instantiation per
// warp (the j chunk a template constant, so the u coefficients are constant-bank operands) and
// the order's own register allocation instead of the largest order's.
template <typename T, int N>
__global__ void __launch_bounds__(EnsOrderGeom<N, T>::THREADS, EnsOrderGeom<N, T>::MIN_BLOCKS)
ens_order_kernel(const EnsMember *__restrict__ members, const int *__restrict__ cta_items,
                 const EnsItem *__restrict__ items, int stage) {
    using GP = EnsOrderGeom<N, T>;
    __shared__ StageArgs sArgs;
    __shared__ int sActive;
    for (int it = cta_items[blockIdx.x]; it < cta_items[blockIdx.x + 1]; ++it) {
        const EnsItem item = items[it];
        const EnsMember &m = members[item.member];
        __syncthreads();   // the previous item is done with the shared arguments and tiles
        if (threadIdx.x == 0) {
            StageArgs a = m.a;
            ens_stage_args(a, m, stage);
            sArgs = a;
            sActive = (a.state == nullptr) || (a.state->active != 0);
        }
        __syncthreads();
        if (!sActive) continue;
        pencil_body_per_warp<N, T, GP::JC, GP::THREADS, EnsTables<T>>(sArgs, ens_tables<T>(N), m.qw, item.e,
                                                                      item.g, m.G, (int)(threadIdx.x >> 5));
    }
}

// field solves of all members: one thread-block cluster of FC CTAs per member (vlasov_field.cuh)
__global__ void __launch_bounds__(FS_THREADS) ens_field_kernel(const FieldArgs *__restrict__ fa) {
    field_cluster_body(fa[blockIdx.x / FC]);
}

}  // namespace vl

struct vl_ens {
    std::vector<vl_ctx *> ctx;
    int precision = VL_FP64;
    int device = 0, sm_count = 148;
    // binding per member
    std::vector<vl::EnsMember> members;
    std::vector<vl::FieldArgs> field[3];   // promote, require-active, record
    std::vector<int> bound;
    // schedule
    int threads = 128, ctas = 0;
    std::vector<int> G;
    // by-order schedule: one stage launch per order present (ctas CTAs from cta_items[base])
    struct Group {
        int n, ctas, base;
        bool native;   // members launched one by one through their context's stage kernel
    };
    bool by_order = false;
    std::vector<Group> groups;
    std::vector<char> native;   // by order: member i launched through its own context
    // the launches of one by-order stage (one per ordinary group, one per member of a native
    // group) run concurrently: launch q on lane q mod LANES (lane 0 the caller's stream, lane k > 0
    // side[k - 1]), the side streams forked from and joined back into the caller's stream by
    // events (graph branches when captured)
    static constexpr int LANES = 8;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> joined;
    cudaEvent_t forked = nullptr;
    vl::EnsMember *d_members = nullptr;
    vl::FieldArgs *d_field[3] = {nullptr, nullptr, nullptr};
    int *d_cta_items = nullptr;
    vl::EnsItem *d_items = nullptr;
    size_t field_smem = 0;   // dynamic shared memory of the field kernel: the largest member's
    bool dirty = true;
};

namespace {

int efail(int code, const std::string &msg) {
    vl_internal_set_error(msg.c_str());
    return code;
}

#define VL_ECUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) return efail(VL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int tiles_of(const vl_ctx *c) {
    const int epw = 32 / c->cfg.n > 0 ? 32 / c->cfg.n : 1;
    return c->cfg.nu * ((c->cfg.nv + epw - 1) / epw);
}

size_t partial_bytes(const vl_ctx *c, int G) {
    const size_t b = sizeof(double) * (size_t)c->cfg.nx * G * c->cfg.n;
    return (b + 255) & ~(size_t)255;
}

template <typename T>
size_t ens_smem(int threads) {
    size_t m = 0;
    for (int n = 1; n <= vl::NMAX; ++n) {
        const int rw = (32 / n) * n;
        const size_t b = ((sizeof(double) * (size_t)n * threads + sizeof(T) * (size_t)(n * n * rw + n * n) + 7) &
                          ~(size_t)7) + sizeof(double) * n;   // + the E values (vl::PencilGeom::se_offset)
        m = std::max(m, b);
    }
    return m;
}

template <typename T, int NT>
int launch_stage(vl_ens *E, int stage, cudaStream_t s) {
    const size_t smem = ens_smem<T>(NT);
    vl::ens_stage_kernel<T, NT><<<E->ctas, NT, smem, s>>>(E->d_members, E->d_cta_items, E->d_items, stage);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return efail(VL_ERR_CUDA, std::string("ens_stage_kernel: ") + cudaGetErrorString(e));
    return VL_OK;
}

// resident CTAs per SM of one order's kernel (sets its dynamic shared-memory limit first)
template <typename T, int N>
int order_blocks(int *blocks) {
    using GP = vl::EnsOrderGeom<N, T>;
    VL_ECUDA(cudaFuncSetAttribute(vl::ens_order_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)GP::smem_bytes()));
    VL_ECUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, vl::ens_order_kernel<T, N>, GP::THREADS,
                                                           GP::smem_bytes()));
    if (*blocks < 1) return efail(VL_ERR_CUDA, "ens_order_kernel: no resident CTA");
    return VL_OK;
}

template <typename T, int N>
int launch_order(vl_ens *E, const vl_ens::Group &g, int stage, cudaStream_t s) {
    using GP = vl::EnsOrderGeom<N, T>;
    vl::ens_order_kernel<T, N><<<g.ctas, GP::THREADS, GP::smem_bytes(), s>>>(E->d_members, E->d_cta_items + g.base,
                                                                              E->d_items, stage);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return efail(VL_ERR_CUDA, std::string("ens_order_kernel: ") + cudaGetErrorString(e));
    return VL_OK;
}

// compile-time order from a runtime one: F is called with std::integral_constant<int, n>
template <typename F>
int with_order(int n, F &&f) {
    switch (n) {
        case 1: return f(std::integral_constant<int, 1>());
        case 2: return f(std::integral_constant<int, 2>());
        case 3: return f(std::integral_constant<int, 3>());
        case 4: return f(std::integral_constant<int, 4>());
        case 5: return f(std::integral_constant<int, 5>());
        case 6: return f(std::integral_constant<int, 6>());
        case 7: return f(std::integral_constant<int, 7>());
        case 8: return f(std::integral_constant<int, 8>());
        case 9: return f(std::integral_constant<int, 9>());
        default: return efail(VL_ERR_UNSUPPORTED, "ensemble members take orders 1..9");
    }
}

// one member's RK stage st through its context's single-problem stage kernel
int native_stage(vl_ens *E, int i, int st, cudaStream_t s) {
    vl_ctx *c = E->ctx[i];
    const vl::EnsMember &m = E->members[i];
    vl::StageArgs a = vl_internal_stage_args(c);
    a.E = m.a.E;
    a.dt = m.a.dt;
    a.state = m.a.state;
    a.err = m.a.err;
    a.partials = m.a.partials;
    a.xhalo = m.a.xhalo;
    vl::ens_stage_args(a, m, st);
    return vl_internal_stage(c, a, s);
}

int stage(vl_ens *E, int st, cudaStream_t s) {
    if (E->by_order) {
        // launches of this stage: ordinary groups, then the members of native groups
        std::vector<std::pair<int, int>> work;   // (group, member or -1)
        for (int k = 0; k < (int)E->groups.size(); ++k) {
            if (!E->groups[k].native) {
                work.push_back({k, -1});
            } else {
                for (int i = 0; i < (int)E->ctx.size(); ++i)
                    if (E->native[i] && E->ctx[i]->cfg.n == E->groups[k].n) work.push_back({k, i});
            }
        }
        const int lanes = VL_ENS_CONCURRENT ? std::min<int>(vl_ens::LANES, (int)work.size()) : 1;
        if (lanes > 1) {
            VL_ECUDA(cudaEventRecord(E->forked, s));
            for (int k = 1; k < lanes; ++k) VL_ECUDA(cudaStreamWaitEvent(E->side[k - 1], E->forked, 0));
        }
        for (int q = 0; q < (int)work.size(); ++q) {
            const vl_ens::Group &g = E->groups[work[q].first];
            cudaStream_t ls = (q % lanes == 0) ? s : E->side[q % lanes - 1];
            int rc;
            if (work[q].second >= 0) {
                rc = native_stage(E, work[q].second, st, ls);
            } else {
                rc = with_order(g.n, [&](auto nc) {
                    constexpr int N = decltype(nc)::value;
                    return E->precision == VL_FP64 ? launch_order<double, N>(E, g, st, ls)
                                                   : launch_order<float, N>(E, g, st, ls);
                });
            }
            if (rc) return rc;
        }
        if (lanes > 1) {
            for (int k = 1; k < lanes; ++k) {
                VL_ECUDA(cudaEventRecord(E->joined[k - 1], E->side[k - 1]));
                VL_ECUDA(cudaStreamWaitEvent(s, E->joined[k - 1], 0));
            }
        }
        return VL_OK;
    }
    if (E->precision == VL_FP64)
        return E->threads == 64 ? launch_stage<double, 64>(E, st, s) : launch_stage<double, 128>(E, st, s);
    return E->threads == 64 ? launch_stage<float, 64>(E, st, s) : launch_stage<float, 128>(E, st, s);
}

int field(vl_ens *E, int kind, cudaStream_t s) {
    const int count = (int)E->ctx.size();
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(vl::FC * count);
    cfg.blockDim = dim3(vl::FS_THREADS);
    cfg.dynamicSmemBytes = E->field_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = vl::FC;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, vl::ens_field_kernel, static_cast<const vl::FieldArgs *>(E->d_field[kind]));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return efail(VL_ERR_CUDA, std::string("ens_field_kernel: ") + cudaGetErrorString(e));
    return VL_OK;
}

template <typename T>
int upload_tables(const std::vector<vl_ctx *> &ctxs) {
    vl::EnsTables<T> tabs[vl::NMAX + 1];
    std::memset(tabs, 0, sizeof(tabs));
    for (const vl_ctx *c : ctxs) {
        const int n = c->cfg.n;
        for (int i = 0; i < n * n; ++i) tabs[n].up[i] = (T)c->up[i];
        for (int i = 0; i < 2 * n; ++i) tabs[n].xi[i] = (T)c->xi[i];
    }
    if (sizeof(T) == 8)
        VL_ECUDA(cudaMemcpyToSymbol(vl::c_ens64, tabs, sizeof(tabs)));
    else
        VL_ECUDA(cudaMemcpyToSymbol(vl::c_ens32, tabs, sizeof(tabs)));
    return VL_OK;
}

struct CostItem {
    double cost;
    vl::EnsItem it;
};

// items in member-major order (members, then x elements, then tile groups), each onto the
// least-loaded of P CTAs: with items of similar cost this deals them round-robin, so CTAs
// working at the same time hold neighbouring x elements of one member and the face planes they
// share are read from L2 (against longest-processing-time order: 64-member FP32 ensemble 2% faster
// at 4 items per CTA, 11% at 1)
void assign_in_order(const std::vector<CostItem> &items, int P, std::vector<int> &offs,
                     std::vector<vl::EnsItem> &flat) {
    std::vector<std::vector<vl::EnsItem>> per(P);
    using Load = std::pair<double, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int p = 0; p < P; ++p) heap.push({0.0, p});
    for (const CostItem &it : items) {
        Load l = heap.top();
        heap.pop();
        per[l.second].push_back(it.it);
        heap.push({l.first + it.cost, l.second});
    }
    for (int p = 0; p < P; ++p) {
        offs.push_back((int)flat.size());
        flat.insert(flat.end(), per[p].begin(), per[p].end());
    }
    offs.push_back((int)flat.size());
}

// longest processing time first onto the least-loaded of P CTAs
void assign_lpt(std::vector<CostItem> &items, int P, std::vector<int> &offs, std::vector<vl::EnsItem> &flat) {
    std::stable_sort(items.begin(), items.end(), [](const CostItem &a, const CostItem &b) { return a.cost > b.cost; });
    assign_in_order(items, P, offs, flat);
}

// rebuild the device descriptors and the item list after a bind or schedule change
int commit(vl_ens *E) {
    const int count = (int)E->ctx.size();
    for (int i = 0; i < count; ++i)
        if (!E->bound[i]) return efail(VL_ERR_INVALID, "ensemble member " + std::to_string(i) + " is not bound");
    // item costs: tiles per item x n^3 (DOFs per tile ~ 32 n^2, contraction length n); items of
    // order n go to list n (by-order schedule) or all to list 0
    std::vector<CostItem> items[vl::NMAX + 1];
    E->field_smem = 0;
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        const int G = E->G[i];
        const double n = c->cfg.n;
        const int tiles = tiles_of(c);
        // by order: members launched through their own contexts have no items
        std::vector<CostItem> &list = items[E->by_order ? (E->native[i] ? 0 : c->cfg.n) : 0];
        for (int e = 0; e < c->cfg.nx; ++e)
            for (int g = 0; g < G; ++g) {
                const int nt = (tiles - g + G - 1) / G;
                list.push_back({nt * n * n * n, {i, e, g, 0}});
            }
        E->members[i].G = G;
        for (int k = 0; k < 3; ++k) E->field[k][i].G = G;
        // a member launched through its own context: the solve after the Euler stage reads the
        // partials of that context's Euler-stage grid
        if (E->by_order && E->native[i]) E->field[1][i].G = c->stage_grid_g1;
        E->field_smem = std::max(E->field_smem, vl::field_solve_smem(c->cfg.n, c->cfg.n_modes));
    }
    std::vector<int> offs;
    std::vector<vl::EnsItem> flat;
    if (E->by_order) {
        for (vl_ens::Group &g : E->groups) {
            if (g.native) continue;
            std::vector<CostItem> &list = items[g.n];
            g.ctas = std::max(1, std::min(g.ctas, (int)list.size()));
            g.base = (int)offs.size();
            assign_in_order(list, g.ctas, offs, flat);
        }
    } else {
        const int P = std::max(1, std::min(E->ctas, (int)items[0].size()));
        E->ctas = P;
        assign_lpt(items[0], P, offs, flat);
    }
    if (offs.empty()) offs.push_back(0);   // every group native: no work list
    cudaFree(E->d_cta_items);
    cudaFree(E->d_items);
    E->d_cta_items = nullptr;
    E->d_items = nullptr;
    VL_ECUDA(cudaMalloc((void **)&E->d_cta_items, sizeof(int) * offs.size()));
    VL_ECUDA(cudaMalloc((void **)&E->d_items, sizeof(vl::EnsItem) * std::max<size_t>(flat.size(), 1)));
    VL_ECUDA(cudaMemcpy(E->d_cta_items, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice));
    VL_ECUDA(cudaMemcpy(E->d_items, flat.data(), sizeof(vl::EnsItem) * flat.size(), cudaMemcpyHostToDevice));
    VL_ECUDA(cudaMemcpy(E->d_members, E->members.data(), sizeof(vl::EnsMember) * count, cudaMemcpyHostToDevice));
    for (int k = 0; k < 3; ++k)
        VL_ECUDA(cudaMemcpy(E->d_field[k], E->field[k].data(), sizeof(vl::FieldArgs) * count,
                            cudaMemcpyHostToDevice));
    E->dirty = false;
    return VL_OK;
}

}  // namespace

extern "C" {

VL_API int vl_ens_create(vl_ctx *const *ctxs, int32_t count, vl_ens **out) {
    if (!ctxs || !out || count < 1) return efail(VL_ERR_INVALID, "need at least one context");
    *out = nullptr;
    vl_ens *E = new vl_ens();
    E->precision = ctxs[0]->cfg.precision;
    for (int i = 0; i < count; ++i) {
        if (!ctxs[i]) {
            delete E;
            return efail(VL_ERR_INVALID, "null context");
        }
        if (ctxs[i]->cfg.precision != E->precision) {
            delete E;
            return efail(VL_ERR_INVALID, "ensemble members must share one precision");
        }
        if (ctxs[i]->cfg.n > 9) {
            delete E;
            return efail(VL_ERR_UNSUPPORTED, "ensemble members take orders 1..9");
        }
        if (ctxs[i]->bg_rb != nullptr) {
            delete E;
            return efail(VL_ERR_UNSUPPORTED, "ensemble members run without the background split");
        }
        E->ctx.push_back(ctxs[i]);
    }
    E->device = ctxs[0]->device;
    E->sm_count = ctxs[0]->sm_count;
    E->members.resize(count);
    for (int k = 0; k < 3; ++k) E->field[k].resize(count);
    E->bound.assign(count, 0);
    E->G.assign(count, 1);
    E->ctas = E->sm_count * 4;
    std::memset(E->members.data(), 0, sizeof(vl::EnsMember) * count);
    int rc = E->precision == VL_FP64 ? upload_tables<double>(E->ctx) : upload_tables<float>(E->ctx);
    if (rc) {
        delete E;
        return rc;
    }
    cudaError_t e = cudaMalloc((void **)&E->d_members, sizeof(vl::EnsMember) * count);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        e = cudaMalloc((void **)&E->d_field[k], sizeof(vl::FieldArgs) * count);
    if (e != cudaSuccess) {
        vl_ens_destroy(E);
        return efail(VL_ERR_CUDA, std::string("cudaMalloc(ensemble): ") + cudaGetErrorString(e));
    }
    for (int t : {64, 128}) {
        const size_t smem = E->precision == VL_FP64 ? ens_smem<double>(t) : ens_smem<float>(t);
        if (E->precision == VL_FP64)
            cudaFuncSetAttribute(t == 64 ? vl::ens_stage_kernel<double, 64> : vl::ens_stage_kernel<double, 128>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        else
            cudaFuncSetAttribute(t == 64 ? vl::ens_stage_kernel<float, 64> : vl::ens_stage_kernel<float, 128>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    cudaFuncSetAttribute(vl::ens_field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)vl::field_solve_smem(vl::NMAX, vl::FIELD_MAX_MODES));
    *out = E;
    return VL_OK;
}

VL_API int vl_ens_destroy(vl_ens *E) {
    if (!E) return VL_OK;
    cudaFree(E->d_members);
    for (int k = 0; k < 3; ++k) cudaFree(E->d_field[k]);
    cudaFree(E->d_cta_items);
    cudaFree(E->d_items);
    for (cudaStream_t st : E->side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : E->joined) cudaEventDestroy(ev);
    if (E->forked) cudaEventDestroy(E->forked);
    delete E;
    return VL_OK;
}

VL_API size_t vl_ens_workspace_bytes(const vl_ens *E, int32_t i) {
    if (!E || i < 0 || i >= (int)E->ctx.size()) return 0;
    const vl_ctx *c = E->ctx[i];
    return partial_bytes(c, tiles_of(c));   // partials for any schedule
}

VL_API int vl_ens_bind(vl_ens *E, int32_t i, void *f, void *sa, void *sb, double *Ef, double *phi,
                       vl_run_state *state, void *workspace) {
    if (!E || i < 0 || i >= (int)E->ctx.size()) return efail(VL_ERR_INVALID, "member index");
    if (!f || !sa || !sb || !Ef || !state || !workspace) return efail(VL_ERR_INVALID, "null argument");
    const vl_ctx *c = E->ctx[i];
    vl::EnsMember &m = E->members[i];
    std::memset(&m, 0, sizeof(m));
    m.f = f;
    m.sa = sa;
    m.sb = sb;
    m.n = c->cfg.n;
    m.G = E->G[i];
    std::memcpy(m.qw, c->qw, sizeof(m.qw));
    vl::StageArgs &a = m.a;
    a.E = Ef;
    a.dt = &state->dt;
    a.state = state;
    a.err = &state->status;
    a.u_nodes = c->d_unodes;
    a.v_nodes = c->d_vnodes;
    a.partials = static_cast<double *>(workspace);
    a.tables = c->d_tables;
    a.nx = c->cfg.nx;
    a.nu = c->cfg.nu;
    a.nv = c->cfg.nv;
    a.xhalo = VL_XHALO_PERIODIC;
    a.accel = c->cfg.accel;
    a.bfield = c->cfg.bfield;
    a.jx = c->cfg.jx;
    a.ju = c->cfg.ju;
    a.jv = c->cfg.jv;
    const int modes[3] = {vl::FIELD_PROMOTE, vl::FIELD_REQUIRE_ACTIVE,
                          vl::FIELD_REQUIRE_ACTIVE | vl::FIELD_RECORD};
    for (int k = 0; k < 3; ++k) {
        vl::FieldArgs &fa = E->field[k][i];
        std::memset(&fa, 0, sizeof(fa));
        fa.partials = static_cast<double *>(workspace);
        fa.G = m.G;
        fa.E = Ef;
        fa.phi = (k == 2) ? phi : nullptr;
        fa.state = state;
        fa.mode = modes[k];
        fa.ell = c->d_ell;
        fa.phase = c->d_phase;
        fa.qnode = c->d_qnode;
        fa.k = c->d_k;
        fa.xw = c->d_xw;
        fa.nx = c->cfg.nx;
        fa.n = c->cfg.n;
        fa.M = c->cfg.n_modes;
        fa.kappa = c->cfg.kappa;
        fa.dx = c->cfg.dx;
        fa.length = c->cfg.length_x;
        fa.accel = c->cfg.accel;
        fa.bfield = c->cfg.bfield;
        fa.umax = c->cfg.umax;
        fa.vmax = c->cfg.vmax;
        fa.du = c->cfg.du;
        fa.dv = c->cfg.dv;
        fa.courant = c->cfg.courant;
    }
    E->bound[i] = 1;
    E->dirty = true;
    return VL_OK;
}

VL_API int vl_ens_schedule(vl_ens *E, int32_t threads, int32_t ctas_per_sm, int32_t items_per_cta) {
    if (!E) return efail(VL_ERR_INVALID, "null ensemble");
    if (threads != 64 && threads != 128) return efail(VL_ERR_INVALID, "threads must be 64 or 128");
    if (ctas_per_sm < 1 || ctas_per_sm > 32 || items_per_cta < 1 || items_per_cta > 64)
        return efail(VL_ERR_INVALID, "ctas_per_sm in 1..32, items_per_cta in 1..64");
    E->by_order = false;
    E->threads = threads;
    E->ctas = E->sm_count * ctas_per_sm;
    // split each member's x slabs into tile groups so that the item count is about
    // ctas x items_per_cta with items of similar cost
    const int count = (int)E->ctx.size();
    double total = 0.0;
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        const double n = c->cfg.n;
        total += (double)c->cfg.nx * tiles_of(c) * n * n * n;
    }
    const double target = total / ((double)E->ctas * items_per_cta);
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        const double n = c->cfg.n;
        const int tiles = tiles_of(c);
        int G = (int)(tiles * n * n * n / target + 0.5);
        E->G[i] = std::max(1, std::min(G, tiles));
    }
    E->dirty = true;
    return VL_OK;
}

VL_API int vl_ens_schedule_by_order(vl_ens *E, int32_t items_per_cta, uint32_t native_orders) {
    if (!E) return efail(VL_ERR_INVALID, "null ensemble");
    if (items_per_cta < 1 || items_per_cta > 64) return efail(VL_ERR_INVALID, "items_per_cta in 1..64");
    const int count = (int)E->ctx.size();
    // members launched through their own contexts: those of the orders in the mask, or with
    // VL_ENS_NATIVE_AUTO those whose context stages its tiles by TMA (fragment kernel, TMA
    // kernel, the generic kernel's TMA form), which beat the ensemble's register-pencil body
    std::vector<char> native(count, 0);
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        if (native_orders == VL_ENS_NATIVE_AUTO)
            native[i] = c->stage_kernel == VL_STAGE_FRAG || c->stage_kernel == VL_STAGE_TMA ||
                        (c->stage_kernel == VL_STAGE_GEN && (c->gen_tma || c->gen_pair));
        else
            native[i] = (native_orders >> c->cfg.n) & 1u;
    }
    double total[vl::NMAX + 1] = {};
    bool any_native[vl::NMAX + 1] = {};
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        const double n = c->cfg.n;
        if (native[i])
            any_native[c->cfg.n] = true;
        else
            total[c->cfg.n] += (double)c->cfg.nx * tiles_of(c) * n * n * n;
    }
    // per order present: a native group (its members one launch each) and / or an ensemble
    // group (as many CTAs of the order's ensemble kernel as it keeps resident)
    std::vector<vl_ens::Group> groups;
    int launches = 0;
    for (int n = vl::NMAX; n >= 1; --n) {
        if (any_native[n]) {
            groups.push_back({n, 0, 0, true});
            for (int i = 0; i < count; ++i) launches += (native[i] && E->ctx[i]->cfg.n == n);
        }
        if (total[n] == 0.0) continue;
        int blocks = 0;
        const int rc = with_order(n, [&](auto nc) {
            constexpr int N = decltype(nc)::value;
            return E->precision == VL_FP64 ? order_blocks<double, N>(&blocks) : order_blocks<float, N>(&blocks);
        });
        if (rc) return rc;
        groups.push_back({n, E->sm_count * blocks, 0, false});
        ++launches;
    }
    // tile groups per member: its context's own for native members (the partials layout of the
    // single-problem kernel), else about items_per_cta items of similar cost per CTA of its order
    for (int i = 0; i < count; ++i) {
        const vl_ctx *c = E->ctx[i];
        if (native[i]) {
            E->G[i] = c->stage_grid_g;
            continue;
        }
        const double n = c->cfg.n;
        int ctas = 1;
        for (const vl_ens::Group &g : groups)
            if (g.n == c->cfg.n && !g.native) ctas = g.ctas;
        const double target = total[c->cfg.n] / ((double)ctas * items_per_cta);
        const int tiles = tiles_of(c);
        const int G = (int)(tiles * n * n * n / target + 0.5);
        E->G[i] = std::max(1, std::min(G, tiles));
    }
    if (!E->forked) VL_ECUDA(cudaEventCreateWithFlags(&E->forked, cudaEventDisableTiming));
    const int lanes = std::min(vl_ens::LANES, std::max(launches, 1));
    while ((int)E->side.size() + 1 < lanes) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        VL_ECUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        E->side.push_back(st);
        VL_ECUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        E->joined.push_back(ev);
    }
    E->groups = groups;
    E->native = native;
    E->by_order = true;
    E->dirty = true;
    return VL_OK;
}

VL_API int vl_ens_commit(vl_ens *E) {
    if (!E) return efail(VL_ERR_INVALID, "null ensemble");
    return commit(E);
}

VL_API int vl_ens_steps(vl_ens *E, int32_t nsteps, void *stream) {
    if (!E) return efail(VL_ERR_INVALID, "null ensemble");
    if (nsteps < 0) return efail(VL_ERR_INVALID, "nsteps < 0");
    if (E->dirty) return efail(VL_ERR_INVALID, "ensemble changed since the last vl_ens_commit");
    int rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int count = (int)E->ctx.size();
    // density partials of every member's f^n for the first field solve
    for (int i = 0; i < count; ++i)
        if ((rc = vl_internal_moment(E->ctx[i], E->members[i].f, E->members[i].a.partials, E->G[i], s)))
            return rc;
    for (int it = 0; it < nsteps; ++it) {
        if ((rc = field(E, 0, s))) return rc;
        if ((rc = stage(E, 0, s))) return rc;
        if ((rc = field(E, 1, s))) return rc;
        if ((rc = stage(E, 1, s))) return rc;
        if ((rc = field(E, 2, s))) return rc;
        if ((rc = stage(E, 2, s))) return rc;
    }
    return VL_OK;
}

}  // extern "C"
