// batch.cu -- many independent operator instances in one persistent launch.
//
// Each instance is a full EvaluatorNonLin (its own grid, DG degree and quadrature rule);
// the instances' coefficient vectors are concatenated. A persistent kernel (grid = resident
// CTAs of the device) pulls work items (instance, first cell, number of tiles) from a
// queue counter in device memory and evaluates them with the tile routine of the generic
// kernel specialised for the instance's degree. Work items are ordered longest first
// (or round-robin, as the autotuner decides), so uneven instances balance over the SMs.
// The residual and VJP launches of a batch can be captured once into a CUDA graph and
// replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "batch.h"
#include "dg_slab_kernel.cuh"
#include "handle.h"

namespace bosss {

struct BatchInst {
    EvalArgs a;
    long long dom_off, cod_off;
    int K, Q;
};

struct WorkItem {
    int inst;
    int ntiles;
    long long c0;
};

// degrees with batched kernels: Q = K+1 (Linear(), order 2K / 2K+1) and 2K+1 (NonLinear(3)).
// Two tile kernels: the generic cell tile (every case) and the register-blocked slab tile
// (cases with at most 5 nodes per direction, where it is the faster one).
#define BOSSS_BATCH_CASES(X) X(1, 2) X(2, 3) X(3, 4) X(4, 5) X(1, 3) X(2, 5) X(3, 7)
#define BOSSS_BATCH_SLAB_CASES(X) X(1, 2) X(2, 3) X(3, 4) X(4, 5) X(1, 3) X(2, 5)

// tile configuration of a case in the generic (SLAB = false) or slab batched kernel
template <class Phys, int K, int Q, int MODE, bool SLAB>
struct BatchTile {
    using G = Cfg<Phys, K, Q, MODE>;
    using S = SlabCfg<Phys, K, Q, MODE>;
    static constexpr int CPB = SLAB ? S::CPB : G::CPB;
    static constexpr size_t SMEM_BYTES = SLAB ? S::SMEM_BYTES : G::SMEM_BYTES;
    static constexpr int NT = SLAB ? S::NT : G::NT;
};

// threads per CTA and resident CTAs per SM the batched kernel is compiled for. One kernel
// holds the tiles of every case, so its register budget is the largest case's: no
// min-blocks bound beyond the register file (a tighter one spills kilobytes per thread)
template <int MODE, bool SLAB>
struct BatchBlock {
    static constexpr int NT = (SLAB && MODE == MODE_VJP) ? 128 : 256;
    static constexpr int MINB = (SLAB && MODE == MODE_VJP) ? 2 : 1;
};

template <class Phys, int MODE, bool SLAB>
constexpr size_t batch_smem() {
    size_t m = 0;
#define BOSSS_SMEM_MAX(K, Q)                                                                                   \
    m = m > BatchTile<Phys, K, Q, MODE, SLAB>::SMEM_BYTES ? m : BatchTile<Phys, K, Q, MODE, SLAB>::SMEM_BYTES;
    if constexpr (SLAB) {
        BOSSS_BATCH_SLAB_CASES(BOSSS_SMEM_MAX)
    } else {
        BOSSS_BATCH_CASES(BOSSS_SMEM_MAX)
    }
#undef BOSSS_SMEM_MAX
    return m;
}

template <class Phys, int K, int Q, int MODE, bool SLAB>
__device__ __forceinline__ void run_item(const EvalArgs& a, const WorkItem& w, double* smem) {
    using BT = BatchTile<Phys, K, Q, MODE, SLAB>;
    static_assert(BT::NT <= BatchBlock<MODE, SLAB>::NT, "tile needs more threads than the batched CTA has");
    for (int t = 0; t < w.ntiles; ++t) {
        const long long c0 = w.c0 + (long long)t * BT::CPB;
        if (c0 >= a.g.J) break;
        if constexpr (SLAB) slab_tile<Phys, K, Q, MODE>(a, a.tab, c0, smem);
        else cell_tile<Phys, K, Q, MODE>(a, c0, smem);
        __syncthreads();
    }
}

template <class Phys, int MODE, bool SLAB>
__global__ void __launch_bounds__(BatchBlock<MODE, SLAB>::NT, BatchBlock<MODE, SLAB>::MINB)
batch_kernel(const BatchInst* __restrict__ inst, const WorkItem* __restrict__ items, int nitems,
             int* __restrict__ counter, const double* U, const double* V, double* out, double alpha, double beta,
             double time) {
    extern __shared__ double smem[];
    __shared__ EvalArgs sa;
    __shared__ WorkItem w;
    __shared__ int K, Q;
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(counter, 1);
            w.inst = -1;
            if (it < nitems) w = items[it];
        }
        __syncthreads();
        if (w.inst < 0) break;
        const BatchInst* b = inst + w.inst;
        for (int i = threadIdx.x; i < (int)(sizeof(EvalArgs) / 8); i += blockDim.x)
            reinterpret_cast<double*>(&sa)[i] = reinterpret_cast<const double*>(&b->a)[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            sa.U = U + b->dom_off;
            sa.V = V ? V + ((MODE == MODE_VJP) ? b->cod_off : b->dom_off) : nullptr;
            sa.out = out + ((MODE == MODE_VJP) ? b->dom_off : b->cod_off);
            sa.alpha = alpha;
            sa.beta = beta;
            sa.time = time;
            K = b->K;
            Q = b->Q;
        }
        __syncthreads();
#define BOSSS_CASE(KK, QQ) \
    if (K == KK && Q == QQ) run_item<Phys, KK, QQ, MODE, SLAB>(sa, w, smem);
        if constexpr (SLAB) {
            BOSSS_BATCH_SLAB_CASES(BOSSS_CASE)
        } else {
            BOSSS_BATCH_CASES(BOSSS_CASE)
        }
#undef BOSSS_CASE
        __syncthreads();
    }
}

template <class Phys, int MODE, bool SLAB>
static bool batch_supported(int K, int Q) {
#define BOSSS_SUP(KK, QQ) \
    if (K == KK && Q == QQ) return BatchTile<Phys, KK, QQ, MODE, SLAB>::SMEM_BYTES <= 227 * 1024;
    if constexpr (SLAB) {
        BOSSS_BATCH_SLAB_CASES(BOSSS_SUP)
    } else {
        BOSSS_BATCH_CASES(BOSSS_SUP)
    }
#undef BOSSS_SUP
    return false;
}

template <class Phys, int MODE, bool SLAB>
static int cpb_of(int K, int Q) {
#define BOSSS_CPB(KK, QQ) \
    if (K == KK && Q == QQ) return BatchTile<Phys, KK, QQ, MODE, SLAB>::CPB;
    if constexpr (SLAB) {
        BOSSS_BATCH_SLAB_CASES(BOSSS_CPB)
    } else {
        BOSSS_BATCH_CASES(BOSSS_CPB)
    }
#undef BOSSS_CPB
    return 1;
}

using BatchLaunch = cudaError_t (*)(const BatchInst*, const WorkItem*, int, int*, const double*, const double*, double*,
                                    double, double, double, int, cudaStream_t);

template <class Phys, int MODE, bool SLAB>
static cudaError_t launch_batch(const BatchInst* inst, const WorkItem* items, int nitems, int* counter, const double* U,
                                const double* V, double* out, double alpha, double beta, double time, int grid,
                                cudaStream_t s) {
    constexpr size_t smem = batch_smem<Phys, MODE, SLAB>();
    static unsigned long long done = 0ull;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(done & (1ull << (dev & 63)))) {
        cudaError_t e =
            cudaFuncSetAttribute(batch_kernel<Phys, MODE, SLAB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(batch_kernel<Phys, MODE, SLAB>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        done |= 1ull << (dev & 63);
    }
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    batch_kernel<Phys, MODE, SLAB><<<grid, BatchBlock<MODE, SLAB>::NT, smem, s>>>(inst, items, nitems, counter, U, V, out,
                                                                                  alpha, beta, time);
    return cudaGetLastError();
}

template <class Phys, int MODE, bool SLAB>
static int resident_grid() {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    constexpr size_t smem = batch_smem<Phys, MODE, SLAB>();
    cudaFuncSetAttribute(batch_kernel<Phys, MODE, SLAB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(batch_kernel<Phys, MODE, SLAB>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel<Phys, MODE, SLAB>, BatchBlock<MODE, SLAB>::NT, smem);
    return std::max(1, per) * std::max(1, nsm);
}

// ---- per-class schedule: one launch per (K, Q) class over the tiles of all its instances, one
// tile per CTA, with the single-grid kernel's launch configuration (threads, resident CTAs per
// SM) and the class's 1D tables in the kernel-parameter bank (they depend on K and Q only)
template <class Phys, int K, int Q, int MODE, bool SLAB>
struct ClassBlock {
    static constexpr int NT = SLAB ? SlabCfg<Phys, K, Q, MODE>::NT : Cfg<Phys, K, Q, MODE>::NT;
    static constexpr int MINB = SLAB ? SlabCfg<Phys, K, Q, MODE>::MINB : 1;
};

template <class Phys, int K, int Q, int MODE, bool SLAB>
__global__ void __launch_bounds__(ClassBlock<Phys, K, Q, MODE, SLAB>::NT, ClassBlock<Phys, K, Q, MODE, SLAB>::MINB)
batch_class_kernel(const __grid_constant__ Tables1D tab, const BatchInst* __restrict__ inst,
                   const WorkItem* __restrict__ items, const double* U, const double* V, double* out, double alpha,
                   double beta, double time) {
    extern __shared__ double smem[];
    __shared__ EvalArgs sa;
    const WorkItem w = items[blockIdx.x];
    const BatchInst* b = inst + w.inst;
    for (int i = threadIdx.x; i < (int)(sizeof(EvalArgs) / 8); i += blockDim.x)
        reinterpret_cast<double*>(&sa)[i] = reinterpret_cast<const double*>(&b->a)[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        sa.U = U + b->dom_off;
        sa.V = V ? V + ((MODE == MODE_VJP) ? b->cod_off : b->dom_off) : nullptr;
        sa.out = out + ((MODE == MODE_VJP) ? b->dom_off : b->cod_off);
        sa.alpha = alpha;
        sa.beta = beta;
        sa.time = time;
    }
    __syncthreads();
    if constexpr (SLAB) slab_tile<Phys, K, Q, MODE>(sa, tab, w.c0, smem);
    else cell_tile<Phys, K, Q, MODE>(sa, w.c0, smem);
}

using ClassLaunch = cudaError_t (*)(const Tables1D&, const BatchInst*, const WorkItem*, int, const double*,
                                    const double*, double*, double, double, double, cudaStream_t);

template <class Phys, int K, int Q, int MODE, bool SLAB>
static cudaError_t launch_class(const Tables1D& tab, const BatchInst* inst, const WorkItem* items, int n,
                                const double* U, const double* V, double* out, double alpha, double beta, double time,
                                cudaStream_t s) {
    constexpr size_t smem = BatchTile<Phys, K, Q, MODE, SLAB>::SMEM_BYTES;
    static unsigned long long done = 0ull;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(done & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(batch_class_kernel<Phys, K, Q, MODE, SLAB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(batch_class_kernel<Phys, K, Q, MODE, SLAB>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        done |= 1ull << (dev & 63);
    }
    if (n <= 0) return cudaSuccess;
    batch_class_kernel<Phys, K, Q, MODE, SLAB><<<n, ClassBlock<Phys, K, Q, MODE, SLAB>::NT, smem, s>>>(
        tab, inst, items, U, V, out, alpha, beta, time);
    return cudaGetLastError();
}

template <class Phys, int MODE, bool SLAB>
static ClassLaunch class_launch_of(int K, int Q) {
#define BOSSS_CL(KK, QQ) \
    if (K == KK && Q == QQ) return &launch_class<Phys, KK, QQ, MODE, SLAB>;
    if constexpr (SLAB) {
        BOSSS_BATCH_SLAB_CASES(BOSSS_CL)
    } else {
        BOSSS_BATCH_CASES(BOSSS_CL)
    }
#undef BOSSS_CL
    return nullptr;
}

}  // namespace bosss

using namespace bosss;


namespace bosss {

// calls f(Phys{}, integral_constant<MODE>, bool_constant<SLAB>) for the batch's physics family
template <class Fn>
static auto batch_dispatch(int phys, int mode, bool slab, Fn&& f) {
    auto by_mode = [&](auto P) {
        auto by_slab = [&](auto M) { return slab ? f(P, M, std::true_type{}) : f(P, M, std::false_type{}); };
        if (mode == MODE_RES) return by_slab(std::integral_constant<int, MODE_RES>{});
        if (mode == MODE_JVP) return by_slab(std::integral_constant<int, MODE_JVP>{});
        return by_slab(std::integral_constant<int, MODE_VJP>{});
    };
    if (phys == PHYS_SIP) return by_mode(PhysScalar<3, true>{});
    return by_mode(PhysScalar<3, false>{});
}

static BatchLaunch batch_launcher(int phys, int D, int mode, bool slab) {
    if (D != 3 || (phys != PHYS_SIP && phys != PHYS_TRANSPORT)) return nullptr;
    return batch_dispatch(phys, mode, slab, [](auto P, auto M, auto S) -> BatchLaunch {
        return &launch_batch<decltype(P), decltype(M)::value, decltype(S)::value>;
    });
}

static bool batch_ok(int phys, int mode, int K, int Q, bool slab) {
    return batch_dispatch(phys, mode, slab, [&](auto P, auto M, auto S) {
        return batch_supported<decltype(P), decltype(M)::value, decltype(S)::value>(K, Q);
    });
}

static int batch_cpb(int phys, int mode, int K, int Q, bool slab) {
    return batch_dispatch(phys, mode, slab, [&](auto P, auto M, auto S) {
        return cpb_of<decltype(P), decltype(M)::value, decltype(S)::value>(K, Q);
    });
}

static int batch_grid(int phys, int mode, bool slab) {
    return batch_dispatch(phys, mode, slab, [](auto P, auto M, auto S) {
        return resident_grid<decltype(P), decltype(M)::value, decltype(S)::value>();
    });
}

// work items of one mode, ordered by the batch's schedule
static int build_items(bosss_batch* b, int mode) {
    struct Tmp {
        WorkItem w;
        double cost;
    };
    std::vector<Tmp> v;
    for (int i = 0; i < b->n; ++i) {
        const bosss_handle* h = b->h[i];
        const int cpb = batch_cpb(b->phys, mode, h->K, h->Q, b->slab[mode]);
        int r = 1;
        auto it = b->tiles.find({h->K, h->Q});
        if (it != b->tiles.end()) r = it->second;
        const long long J = h->base.g.J, step = (long long)cpb * r;
        // cost of a cell ~ (quadrature nodes) x (modes)
        const double cell_cost = (double)h->Q * h->Q * h->Q * (h->K + 1) * (h->K + 2) * (h->K + 3) / 6.0;
        for (long long c0 = 0; c0 < J; c0 += step) {
            Tmp t;
            t.w.inst = i;
            t.w.ntiles = r;
            t.w.c0 = c0;
            t.cost = cell_cost * (double)std::min(step, J - c0);
            v.push_back(t);
        }
    }
    if (b->lpt)
        std::stable_sort(v.begin(), v.end(), [](const Tmp& x, const Tmp& y) { return x.cost > y.cost; });
    std::vector<WorkItem> w(v.size());
    for (size_t k = 0; k < v.size(); ++k) w[k] = v[k].w;
    cudaFree(b->d_items[mode]);
    b->d_items[mode] = nullptr;
    CUDA_TRY(cudaMalloc(&b->d_items[mode], sizeof(WorkItem) * std::max<size_t>(w.size(), 1)));
    CUDA_TRY(cudaMemcpy(b->d_items[mode], w.data(), sizeof(WorkItem) * w.size(), cudaMemcpyHostToDevice));
    b->nitems[mode] = (int)w.size();
    return BOSSS_OK;
}

static ClassLaunch class_launcher(int phys, int mode, int K, int Q, bool slab) {
    return batch_dispatch(phys, mode, slab, [&](auto P, auto M, auto S) {
        return class_launch_of<decltype(P), decltype(M)::value, decltype(S)::value>(K, Q);
    });
}

// tiles of the per-class schedule of one mode: instances grouped by (K, Q), one tile per item
static int build_class_items(bosss_batch* b, int mode, int want) {
    std::vector<WorkItem> w;
    b->runs[mode].clear();
    std::vector<std::pair<int, int>> classes;
    for (auto* h : b->h)
        if (std::find(classes.begin(), classes.end(), std::make_pair(h->K, h->Q)) == classes.end())
            classes.push_back({h->K, h->Q});
    for (auto kq : classes) {
        bosss_batch::ClassRun r;
        r.K = kq.first;
        r.Q = kq.second;
        r.slab = want != 1 && batch_ok(b->phys, mode, r.K, r.Q, true) && (want == 2 || r.Q <= 5);
        r.first = (int)w.size();
        const int cpb = batch_cpb(b->phys, mode, r.K, r.Q, r.slab);
        for (int i = 0; i < b->n; ++i) {
            const bosss_handle* h = b->h[i];
            if (h->K != r.K || h->Q != r.Q) continue;
            for (long long c0 = 0; c0 < h->base.g.J; c0 += cpb) w.push_back(WorkItem{i, 1, c0});
        }
        r.count = (int)w.size() - r.first;
        b->runs[mode].push_back(r);
    }
    cudaFree(b->d_class_items[mode]);
    b->d_class_items[mode] = nullptr;
    CUDA_TRY(cudaMalloc(&b->d_class_items[mode], sizeof(WorkItem) * std::max<size_t>(w.size(), 1)));
    CUDA_TRY(cudaMemcpy(b->d_class_items[mode], w.data(), sizeof(WorkItem) * w.size(), cudaMemcpyHostToDevice));
    return BOSSS_OK;
}

static int batch_run(bosss_batch* b, int mode, double alpha, double beta, const double* U, const double* V, double* out,
                     double time, cudaStream_t s, int counter_slot) {
    if (b->classes) {
        for (const auto& r : b->runs[mode]) {
            ClassLaunch CL = class_launcher(b->phys, mode, r.K, r.Q, r.slab);
            if (!CL) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "no batched class kernel for this degree");
            const bosss_handle* h0 = nullptr;
            for (auto* h : b->h)
                if (h->K == r.K && h->Q == r.Q) {
                    h0 = h;
                    break;
                }
            CUDA_TRY(CL(h0->base.tab, b->d_inst, b->d_class_items[mode] + r.first, r.count, U, V, out, alpha, beta,
                        time, s));
        }
        return BOSSS_OK;
    }
    BatchLaunch L = batch_launcher(b->phys, b->D, mode, b->slab[mode]);
    if (!L) return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "no batched kernel for this physics");
    CUDA_TRY(L(b->d_inst, b->d_items[mode], b->nitems[mode], b->d_counter + counter_slot, U, V, out, alpha, beta, time,
               b->grid[mode], s));
    return BOSSS_OK;
}

static std::string table_key(int phys, int D, int K, int Q) {
    std::ostringstream o;
    o << "phys" << phys << "_D" << D << "_K" << K << "_Q" << Q;
    return o.str();
}

}  // namespace bosss

extern "C" {

int bosss_b200_batch_create(int32_t n, const bosss_op_desc* ops, const bosss_grid_desc* grids,
                            const bosss_options* opt, bosss_batch** out) {
    if (!ops || !grids || !out || n < 1) return fail(BOSSS_ERR_BAD_ARG, "bad batch arguments");
    *out = nullptr;
    bosss_batch* b = new bosss_batch();
    b->n = n;
    b->dom_off.assign(1, 0);
    b->cod_off.assign(1, 0);
    for (int i = 0; i < n; ++i) {
        bosss_handle* h = nullptr;
        int rc = bosss_b200_create(&ops[i], &grids[i], opt, &h);
        if (rc) {
            bosss_b200_batch_destroy(b);
            return rc;
        }
        b->h.push_back(h);
        if (i == 0) {
            b->phys = h->phys;
            b->D = h->D;
            b->device = h->device;
        } else if (h->phys != b->phys || h->D != b->D || h->device != b->device) {
            bosss_b200_batch_destroy(b);
            return fail(BOSSS_ERR_BAD_ARG, "batch instances must share physics family, dimension and device");
        }
        for (int m = 0; m < 3; ++m)
            if (!batch_ok(h->phys, m, h->K, h->Q, false)) {
                bosss_b200_batch_destroy(b);
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT,
                            "no batched kernel for degree " + std::to_string(h->K) + " with " + std::to_string(h->Q) +
                                " Gauss nodes (batched path: 3D scalar transport / advection-diffusion)");
            }
        b->dom_off.push_back(b->dom_off.back() + h->ndom);
        b->cod_off.push_back(b->cod_off.back() + h->ncod);
    }
    if (!batch_launcher(b->phys, b->D, MODE_RES, false)) {
        bosss_b200_batch_destroy(b);
        return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "batched path: 3D scalar transport / advection-diffusion only");
    }
    // tile kernel per mode (the single-grid rule, measured on B200): slab tiles when every
    // instance has at most 5 nodes per direction; kernel selector 1
    // keeps the generic tiles, 2 asks for slab tiles wherever the batch allows them
    const int want = opt ? opt->kernel : 0;
    for (int m = 0; m < 3; ++m) {
        bool ok = want != 1;
        for (auto* h : b->h) {
            ok = ok && batch_ok(b->phys, m, h->K, h->Q, true);
            if (want == 0) ok = ok && h->Q <= 5;
        }
        b->slab[m] = ok;
    }
    auto bail = [&](cudaError_t e) {
        bosss_b200_batch_destroy(b);
        return fail(BOSSS_ERR_CUDA, std::string("batch setup: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    std::vector<BatchInst> hi(n);
    for (int i = 0; i < n; ++i) {
        hi[i].a = b->h[i]->base;
        hi[i].dom_off = b->dom_off[i];
        hi[i].cod_off = b->cod_off[i];
        hi[i].K = b->h[i]->K;
        hi[i].Q = b->h[i]->Q;
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_inst, sizeof(BatchInst) * n);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_inst, hi.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int) * 2);
    if (e != cudaSuccess) return bail(e);
    for (int m = 0; m < 3; ++m) {
        b->grid[m] = batch_grid(b->phys, m, b->slab[m]);
        int rc = build_items(b, m);
        if (!rc) rc = build_class_items(b, m, want);
        if (rc) {
            bosss_b200_batch_destroy(b);
            return rc;
        }
    }
    *out = b;
    return BOSSS_OK;
}

int bosss_b200_batch_destroy(bosss_batch* b) {
    if (!b) return BOSSS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (int m = 0; m < 3; ++m) {
        cudaFree(b->d_items[m]);
        cudaFree(b->d_class_items[m]);
    }
    cudaFree(b->d_inst);
    cudaFree(b->d_counter);
    for (auto* h : b->h) bosss_b200_destroy(h);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return BOSSS_OK;
}

int bosss_b200_batch_get_sizes(const bosss_batch* b, int64_t* domain_offsets, int64_t* codomain_offsets) {
    if (!b) return fail(BOSSS_ERR_BAD_ARG, "null batch");
    for (int i = 0; i <= b->n; ++i) {
        if (domain_offsets) domain_offsets[i] = b->dom_off[i];
        if (codomain_offsets) codomain_offsets[i] = b->cod_off[i];
    }
    return BOSSS_OK;
}

int bosss_b200_batch_evaluate_device(bosss_batch* b, int32_t mode, double alpha, double beta, const double* U_dev,
                                     const double* V_dev, double* out_dev, double time, void* stream) {
    if (!b || !U_dev || !out_dev || mode < 0 || mode > 2) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    if (mode != MODE_RES && !V_dev) return fail(BOSSS_ERR_BAD_ARG, "JVP/VJP need a second vector");
    CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
    return batch_run(b, mode, alpha, beta, U_dev, V_dev, out_dev, time, s, 0);
}

int bosss_b200_batch_evaluate(bosss_batch* b, int32_t mode, double alpha, double beta, const double* U,
                              const double* V, double* out, double time) {
    if (!b || !U || !out || mode < 0 || mode > 2) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    if (mode != MODE_RES && !V) return fail(BOSSS_ERR_BAD_ARG, "JVP/VJP need a second vector");
    CUDA_TRY(cudaSetDevice(b->device));
    const long long nd = b->dom_off.back(), nc = b->cod_off.back();
    const long long nin2 = (mode == MODE_VJP) ? nc : nd, nout = (mode == MODE_VJP) ? nd : nc;
    double *dU = nullptr, *dV = nullptr, *dO = nullptr;
    cudaStream_t s = b->stream;
    auto cleanup = [&]() {
        cudaFree(dU);
        cudaFree(dV);
        cudaFree(dO);
    };
    cudaError_t e = cudaMalloc(&dU, sizeof(double) * nd);
    if (e == cudaSuccess && mode != MODE_RES) e = cudaMalloc(&dV, sizeof(double) * nin2);
    if (e == cudaSuccess) e = cudaMalloc(&dO, sizeof(double) * nout);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dU, U, sizeof(double) * nd, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && dV) e = cudaMemcpyAsync(dV, V, sizeof(double) * nin2, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && mode == MODE_RES && beta != 0.0)
        e = cudaMemcpyAsync(dO, out, sizeof(double) * nout, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        cleanup();
        return fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    int rc = batch_run(b, mode, alpha, beta, dU, dV, dO, time, s, 0);
    if (!rc) {
        e = cudaMemcpyAsync(out, dO, sizeof(double) * nout, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    cleanup();
    return rc;
}

int bosss_b200_batch_capture(bosss_batch* b, const double* U_dev, const double* W_dev, double* R_dev, double* G_dev,
                             double time) {
    if (!b || !U_dev || !W_dev || !R_dev || !G_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(b->device));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = batch_run(b, MODE_RES, 1.0, 0.0, U_dev, nullptr, R_dev, time, b->stream, 0);
    if (!rc) rc = batch_run(b, MODE_VJP, 1.0, 0.0, U_dev, W_dev, G_dev, time, b->stream, 1);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return BOSSS_OK;
}

int bosss_b200_batch_replay(bosss_batch* b, void* stream) {
    if (!b || !b->graph) return fail(BOSSS_ERR_BAD_ARG, "no captured graph");
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaGraphLaunch(b->graph, stream ? (cudaStream_t)stream : b->stream));
    return BOSSS_OK;
}

int bosss_b200_batch_autotune(bosss_batch* b, const double* U_dev, const double* W_dev, double* R_dev, double* G_dev,
                              const char* table_path) {
    if (!b || !U_dev || !W_dev || !R_dev || !G_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(b->device));
    // persisted table: "<key> <tiles>" per line, plus "schedule lpt|fifo"
    std::map<std::string, int> table;
    bool have_sched = false, lpt = true, per_class = false;
    if (table_path && *table_path) {
        std::ifstream f(table_path);
        std::string k;
        int v = 0;
        while (f >> k) {
            if (k == "schedule") {
                std::string sv;
                f >> sv;
                have_sched = true;
                lpt = (sv != "fifo");
                per_class = (sv == "classes");
            } else if (f >> v) {
                table[k] = v;
            }
        }
    }
    b->classes = false;   // tiles per item are timed on the persistent queue
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    auto time_once = [&](float& ms) -> int {
        for (int m : {MODE_RES, MODE_VJP}) {
            int rc = build_items(b, m);
            if (rc) return rc;
        }
        for (int rep = 0; rep < 2; ++rep) {   // warm-up
            int rc = batch_run(b, MODE_RES, 1.0, 0.0, U_dev, nullptr, R_dev, 0.0, b->stream, 0);
            if (!rc) rc = batch_run(b, MODE_VJP, 1.0, 0.0, U_dev, W_dev, G_dev, 0.0, b->stream, 1);
            if (rc) return rc;
        }
        CUDA_TRY(cudaEventRecord(e0, b->stream));
        for (int rep = 0; rep < 3; ++rep) {
            int rc = batch_run(b, MODE_RES, 1.0, 0.0, U_dev, nullptr, R_dev, 0.0, b->stream, 0);
            if (!rc) rc = batch_run(b, MODE_VJP, 1.0, 0.0, U_dev, W_dev, G_dev, 0.0, b->stream, 1);
            if (rc) return rc;
        }
        CUDA_TRY(cudaEventRecord(e1, b->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        return BOSSS_OK;
    };
    // classes present in the batch
    std::vector<std::pair<int, int>> classes;
    for (auto* h : b->h)
        if (std::find(classes.begin(), classes.end(), std::make_pair(h->K, h->Q)) == classes.end())
            classes.push_back({h->K, h->Q});
    int rc = 0;
    for (auto kq : classes) {
        // tiles per item depend on the tile kernels of the timed pair (residual, VJP)
        const std::string key = table_key(b->phys, b->D, kq.first, kq.second) + (b->slab[MODE_RES] ? "_slabR" : "") +
                                (b->slab[MODE_VJP] ? "_slabV" : "");
        if (table.count(key)) {
            b->tiles[kq] = table[key];
            continue;
        }
        int best = 1;
        float best_ms = 1e30f;
        for (int r : {1, 2, 4, 8}) {
            b->tiles[kq] = r;
            float ms = 0.f;
            rc = time_once(ms);
            if (rc) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = r;
            }
        }
        if (rc) break;
        b->tiles[kq] = best;
        table[key] = best;
    }
    if (!rc) {
        if (have_sched) {
            b->lpt = lpt;
            b->classes = per_class;
        } else {
            // persistent queue longest-first, persistent queue in instance order, or one launch
            // per (K, Q) class: the fastest of the three
            float ms_l = 0.f, ms_f = 0.f, ms_c = 0.f;
            b->lpt = true;
            rc = time_once(ms_l);
            if (!rc) {
                b->lpt = false;
                rc = time_once(ms_f);
            }
            if (!rc) {
                b->classes = true;
                rc = time_once(ms_c);
                b->classes = false;
            }
            b->lpt = rc ? true : (ms_l <= ms_f);
            b->classes = !rc && ms_c < std::min(ms_l, ms_f);
        }
        for (int m = 0; m < 3 && !rc; ++m) rc = build_items(b, m);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (table_path && *table_path) {
        std::ofstream f(table_path);
        for (auto& kv : table) f << kv.first << " " << kv.second << "\n";
        f << "schedule " << (b->classes ? "classes" : (b->lpt ? "lpt" : "fifo")) << "\n";
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;   // items changed: the caller re-captures
    }
    return BOSSS_OK;
}

int bosss_b200_batch_tiles(const bosss_batch* b, int32_t K, int32_t Q, int32_t* tiles, int32_t* lpt) {
    if (!b) return fail(BOSSS_ERR_BAD_ARG, "null batch");
    auto it = b->tiles.find({K, Q});
    if (tiles) *tiles = (it == b->tiles.end()) ? 1 : it->second;
    if (lpt) *lpt = b->classes ? 2 : (b->lpt ? 1 : 0);
    return BOSSS_OK;
}

}  // extern "C"

// ======================================================================================
// Batched evaluation that allocates nothing.
//
// Some callers cannot call cudaMalloc: code that must not allocate device memory while it
// runs (a host application whose device memory is owned by another allocator or pool, or
// a time-critical loop where an allocation would synchronise the device). For them,
// bosss_b200_batch_evaluate_noalloc evaluates a batch of single-instance handles with the
// same persistent kernel design, but its scratch -- the work-queue counter, the instance
// table and the per-instance tile prefix sums -- lives in the file-scope device array
// below, of fixed size. The handles come from bosss_b200_create, which allocates no
// device memory; inputs and outputs are the caller's device buffers.
// ======================================================================================
namespace bosss {

constexpr size_t NOALLOC_SCRATCH_BYTES = 1u << 20;   // 1 MiB
constexpr int NOALLOC_MAX_INSTANCES = 512;

// Shared by every call on a device: each call overwrites it, so calls whose kernels
// overlap on the GPU race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

struct NoallocLayout {
    static constexpr size_t counter = 0;                       // int, cleared by every call
    static constexpr size_t inst = 256;                        // BatchInst[n]
    static size_t prefix(int n) { return inst + ((sizeof(BatchInst) * n + 255) / 256) * 256; }   // long long[n+1]
    static size_t bytes(int n) { return prefix(n) + sizeof(long long) * (n + 1); }
};

template <class Phys, int MODE>
__global__ void __launch_bounds__(256) batch_kernel_noalloc(unsigned char* scratch, int n, const double* U,
                                                            const double* V, double* out, double alpha, double beta,
                                                            double time, size_t prefix_off) {
    extern __shared__ double smem[];
    __shared__ EvalArgs sa;
    __shared__ WorkItem w;
    __shared__ int K, Q;
    int* counter = reinterpret_cast<int*>(scratch + NoallocLayout::counter);
    const BatchInst* inst = reinterpret_cast<const BatchInst*>(scratch + NoallocLayout::inst);
    const long long* prefix = reinterpret_cast<const long long*>(scratch + prefix_off);
    const long long total = prefix[n];
    for (;;) {
        if (threadIdx.x == 0) {
            const long long it = atomicAdd(counter, 1);
            w.inst = -1;
            if (it < total) {
                int lo = 0, hi = n;   // prefix[lo] <= it < prefix[hi]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) / 2;
                    if (prefix[mid] <= it) lo = mid;
                    else hi = mid;
                }
                w.inst = lo;
                w.ntiles = 1;
                w.c0 = it - prefix[lo];   // tile index; scaled by the instance's tile size below
            }
        }
        __syncthreads();
        if (w.inst < 0) break;
        const BatchInst* b = inst + w.inst;
        for (int i = threadIdx.x; i < (int)(sizeof(EvalArgs) / 8); i += blockDim.x)
            reinterpret_cast<double*>(&sa)[i] = reinterpret_cast<const double*>(&b->a)[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            sa.U = U + b->dom_off;
            sa.V = V ? V + ((MODE == MODE_VJP) ? b->cod_off : b->dom_off) : nullptr;
            sa.out = out + ((MODE == MODE_VJP) ? b->dom_off : b->cod_off);
            sa.alpha = alpha;
            sa.beta = beta;
            sa.time = time;
            K = b->K;
            Q = b->Q;
        }
        __syncthreads();
#define BOSSS_CASE(KK, QQ)                                                     \
    if (K == KK && Q == QQ) {                                                 \
        WorkItem wt = w;                                                      \
        wt.c0 *= Cfg<Phys, KK, QQ, MODE>::CPB;                                 \
        run_item<Phys, KK, QQ, MODE, false>(sa, wt, smem);                           \
    }
        BOSSS_BATCH_CASES(BOSSS_CASE)
#undef BOSSS_CASE
        __syncthreads();
    }
}

template <class Phys, int MODE>
static cudaError_t launch_noalloc(unsigned char* scratch, int n, const double* U, const double* V, double* out,
                                  double alpha, double beta, double time, size_t prefix_off, cudaStream_t s) {
    constexpr size_t smem = batch_smem<Phys, MODE, false>();
    cudaError_t e = cudaFuncSetAttribute(batch_kernel_noalloc<Phys, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel_noalloc<Phys, MODE>, 256, smem);
    batch_kernel_noalloc<Phys, MODE><<<std::max(1, per) * std::max(1, nsm), 256, smem, s>>>(scratch, n, U, V, out, alpha,
                                                                                          beta, time, prefix_off);
    return cudaGetLastError();
}

// device address of the scratch array, looked up once per device (first call on it)
static unsigned char* noalloc_scratch_ptr(int dev, int& rc) {
    static std::mutex mu;
    static unsigned char* ptrs[64] = {nullptr};
    rc = 0;
    if (dev < 0 || dev >= 64) {
        rc = fail(BOSSS_ERR_BAD_ARG, "device ordinal out of range");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            rc = fail(BOSSS_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
            return nullptr;
        }
        ptrs[dev] = static_cast<unsigned char*>(p);
    }
    return ptrs[dev];
}

}  // namespace bosss

extern "C" int bosss_b200_batch_evaluate_noalloc(int32_t n, bosss_handle* const* instances, int32_t mode, double alpha,
                                                 double beta, const double* U_dev, const double* V_dev, double* out_dev,
                                                 double time, void* stream) {
    if (!instances || !U_dev || !out_dev || mode < 0 || mode > 2) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    if (mode != MODE_RES && !V_dev) return fail(BOSSS_ERR_BAD_ARG, "JVP/VJP need a second vector");
    if (n < 1 || n > NOALLOC_MAX_INSTANCES || NoallocLayout::bytes(n) > NOALLOC_SCRATCH_BYTES)
        return fail(BOSSS_ERR_BAD_ARG, "allocation-free batch: between 1 and " + std::to_string(NOALLOC_MAX_INSTANCES) +
                                           " instances (scratch array of " +
                                           std::to_string(NOALLOC_SCRATCH_BYTES >> 10) + " KiB)");
    const bosss_handle* h0 = instances[0];
    if (!h0) return fail(BOSSS_ERR_BAD_ARG, "null instance handle");
    const int phys = h0->phys, D = h0->D, dev = h0->device;
    if (D != 3 || (phys != PHYS_SIP && phys != PHYS_TRANSPORT))
        return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "allocation-free batch: 3D scalar transport / advection-diffusion");
    // pack the instance table and tile prefix sums in a fixed host staging area
    static std::mutex stage_mu;
    static BatchInst stage_inst[NOALLOC_MAX_INSTANCES];
    static long long stage_prefix[NOALLOC_MAX_INSTANCES + 1];
    std::lock_guard<std::mutex> lock(stage_mu);
    long long doff = 0, coff = 0;
    stage_prefix[0] = 0;
    for (int i = 0; i < n; ++i) {
        const bosss_handle* h = instances[i];
        if (!h || h->phys != phys || h->D != D || h->device != dev)
            return fail(BOSSS_ERR_BAD_ARG, "instances must share physics family, dimension and device");
        // the batched kernel evaluates every cell of an instance: a part of a partitioned grid
        // (ghost planes, global box) would have its ghost cells evaluated too
        bool part = h->base.cbeg != 0 || h->base.cend != h->base.g.J;
        for (int d = 0; d < 3; ++d) part = part || h->base.g.gn[d] != h->base.g.n[d] || h->base.g.goff[d] != 0;
        if (part) return fail(BOSSS_ERR_BAD_ARG, "allocation-free batch: instance " + std::to_string(i) +
                                                     " is a part of a partitioned grid; whole grids only");
        for (int m = 0; m < 3; ++m)
            if (!batch_ok(phys, m, h->K, h->Q, false))
                return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "no batched kernel for degree " + std::to_string(h->K) +
                                                                 " with " + std::to_string(h->Q) + " Gauss nodes");
        stage_inst[i].a = h->base;
        stage_inst[i].dom_off = doff;
        stage_inst[i].cod_off = coff;
        stage_inst[i].K = h->K;
        stage_inst[i].Q = h->Q;
        doff += h->ndom;
        coff += h->ncod;
        const long long cpb = batch_cpb(phys, mode, h->K, h->Q, false);
        stage_prefix[i + 1] = stage_prefix[i] + (h->base.g.J + cpb - 1) / cpb;
    }
    if (stage_prefix[n] > 2000000000LL) return fail(BOSSS_ERR_BAD_ARG, "allocation-free batch: too many cell tiles");
    CUDA_TRY(cudaSetDevice(dev));
    int rc = 0;
    unsigned char* scratch = noalloc_scratch_ptr(dev, rc);
    if (rc) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : h0->stream;
    const size_t poff = NoallocLayout::prefix(n);
    CUDA_TRY(cudaMemsetAsync(scratch + NoallocLayout::counter, 0, sizeof(int), s));
    CUDA_TRY(cudaMemcpyAsync(scratch + NoallocLayout::inst, stage_inst, sizeof(BatchInst) * n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(scratch + poff, stage_prefix, sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, s));
    cudaError_t e;
    if (phys == PHYS_SIP) {
        e = (mode == MODE_RES) ? launch_noalloc<PhysScalar<3, true>, MODE_RES>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s)
          : (mode == MODE_JVP) ? launch_noalloc<PhysScalar<3, true>, MODE_JVP>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s)
                               : launch_noalloc<PhysScalar<3, true>, MODE_VJP>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s);
    } else {
        e = (mode == MODE_RES) ? launch_noalloc<PhysScalar<3, false>, MODE_RES>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s)
          : (mode == MODE_JVP) ? launch_noalloc<PhysScalar<3, false>, MODE_JVP>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s)
                               : launch_noalloc<PhysScalar<3, false>, MODE_VJP>(scratch, n, U_dev, V_dev, out_dev, alpha, beta, time, poff, s);
    }
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, std::string("allocation-free batch launch: ") + cudaGetErrorString(e));
    // no synchronisation: the staging arrays are pageable host memory, and a host-to-device
    // cudaMemcpyAsync from pageable memory returns only after the runtime has copied the source
    // into its own staging buffer, so the next call may overwrite them at once
    return BOSSS_OK;
}
