// Uneven batches: products of different ring sizes and moduli in one graph.
//
// pm_batch_create builds, once, everything a run needs: a plan per product
// (prime basis sized for its N and bits(q), CRT constants and weights),
// packed device buffers for a, b, c and the residue planes, per-product tensor
// maps, and flat work tables:
//   conversion items  (product, prime group, polynomial, column group) ordered
//                     prime group first -- one persistent launch of k1t_convert;
//   row items         (product, prime, first row) per ring size class -- one
//                     launch per class: the persistent k2p_rows for rows of
//                     1024 values or more (items prime/row first, so a CTA
//                     stages a row's twiddles once for every product that
//                     has it), k2_rows_items for shorter rows;
//   CRT items         (product, column group) per width class -- one persistent
//                     launch of k3t_crt per class.
// These launches are captured into a CUDA graph (the classes of a phase on
// parallel branches), so pm_batch_run is a single cudaGraphLaunch.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "../../include/polymul.h"
#include "pm_internal.h"
#include "rows_persistent.cuh"
#include "tensor_kernels.cuh"

namespace pm {

// rows of a class, (product, prime, first row) items; one CTA per item
template <int LOGC, int KP>
__global__ void __launch_bounds__(k2_threads(LOGC), k2_min_blocks(LOGC))
    k2_rows_items(const uint4* __restrict__ items, const BatchProduct* __restrict__ prod, uint32_t* __restrict__ work,
                  const PrimeConst* __restrict__ pcs, const uint2* __restrict__ tw_fwd,
                  const uint2* __restrict__ tw_inv, int logR) {
    constexpr int T = (1 << LOGC) / 8;
    const uint4 it = items[blockIdx.x];
    const BatchProduct& d = prod[it.x];
    const int sub = threadIdx.x / T, tid = threadIdx.x % T;
    const int rows_per_cta = blockDim.x / T;
    k2_row_body<LOGC, KP>(work + d.ws_off, pcs[it.y], tw_fwd, tw_inv, d.n, logR, d.P, int(it.y), int(it.z) + sub,
                          sub, tid, rows_per_cta);
}

// rows of one size class from a table of (product, prime, row) items
struct TableRowWork {
    const uint4* items;
    int nitems;
    const BatchProduct* prod;
    uint32_t* work;
    __device__ int total() const { return nitems; }
    __device__ RowItem item(int k) const {
        const uint4 v = items[k];
        const BatchProduct& d = prod[v.x];
        return RowItem{int(v.y), int(v.z), work + d.ws_off + size_t(v.y) * d.n + (size_t(v.z) << d.logC),
                       size_t(d.P) * d.n};
    }
};

namespace {

int sm_count_dev() {
    int dev = 0, count = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    return count ? count : 148;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cuda_check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
                   "look up cuTensorMapEncodeTiled");
        if (!p || q != cudaDriverEntryPointSuccess) throw Failure(PM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

CUtensorMap encode(CUtensorMapDataType type, const void* base, const cuuint64_t dims[4], const cuuint64_t strides[3],
                   const cuuint32_t box[4], CUtensorMapSwizzle swizzle) {
    CUtensorMap map;
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = encode_tiled()(&map, type, 4, const_cast<void*>(base), dims, strides, box, es,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Failure(PM_ERR_CUDA, "cuTensorMapEncodeTiled failed for a batch product");
    return map;
}

template <int LOGC, int KP>
void launch_rows_class(const uint4* items, int count, int rows_per_item, const BatchProduct* prod, uint32_t* work,
                       const DeviceBasis& B, uint32_t* err, cudaStream_t st) {
    constexpr int C = 1 << LOGC, T = C / 8;
    if constexpr (LOGC >= 10) {
        const size_t smem = k2p_smem_bytes(LOGC);
        cuda_check(cudaFuncSetAttribute(k2p_rows<LOGC, KP, TableRowWork>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(smem)),
                   "batch row shared memory");
        const TableRowWork w{items, count, prod, work};
        const int ctas = std::min(count, sm_count_dev() * k2p_min_blocks(LOGC));
        k2p_rows<LOGC, KP, TableRowWork><<<ctas, k2p_threads(LOGC, KP), smem, st>>>(w, B.d_pc, B.d_tw_fwd,
                                                                                    B.d_tw_inv, 4, err);
    } else {
        const size_t smem = size_t(rows_per_item) * 24 * C;
        if (smem > 48 * 1024)
            cuda_check(cudaFuncSetAttribute(k2_rows_items<LOGC, KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(smem)),
                       "batch row shared memory");
        k2_rows_items<LOGC, KP><<<count, rows_per_item * T, smem, st>>>(items, prod, work, B.d_pc, B.d_tw_fwd,
                                                                        B.d_tw_inv, 4);
    }
}

template <int LOGC>
void launch_rows_radix(int radix_log, const uint4* items, int count, int rows, const BatchProduct* prod,
                       uint32_t* work, const DeviceBasis& B, uint32_t* err, cudaStream_t st) {
    if (radix_log == 2)
        launch_rows_class<LOGC, 2>(items, count, rows, prod, work, B, err, st);
    else if (LOGC >= 10 && radix_log == 4)  // radix-16 passes: the persistent kernel only
        launch_rows_class<LOGC, LOGC >= 10 ? 4 : 3>(items, count, rows, prod, work, B, err, st);
    else
        launch_rows_class<LOGC, 3>(items, count, rows, prod, work, B, err, st);
}

void launch_rows_any(int logC, int radix_log, const uint4* items, int count, int rows, const BatchProduct* prod,
                     uint32_t* work, const DeviceBasis& B, uint32_t* err, cudaStream_t st) {
    switch (logC) {
        case 4: return launch_rows_radix<4>(radix_log, items, count, rows, prod, work, B, err, st);
        case 5: return launch_rows_radix<5>(radix_log, items, count, rows, prod, work, B, err, st);
        case 6: return launch_rows_radix<6>(radix_log, items, count, rows, prod, work, B, err, st);
        case 7: return launch_rows_radix<7>(radix_log, items, count, rows, prod, work, B, err, st);
        case 8: return launch_rows_radix<8>(radix_log, items, count, rows, prod, work, B, err, st);
        case 9: return launch_rows_radix<9>(radix_log, items, count, rows, prod, work, B, err, st);
        case 10: return launch_rows_radix<10>(radix_log, items, count, rows, prod, work, B, err, st);
        case 11: return launch_rows_radix<11>(radix_log, items, count, rows, prod, work, B, err, st);
        case 12: return launch_rows_radix<12>(radix_log, items, count, rows, prod, work, B, err, st);
        default: throw Failure(PM_ERR_UNSUPPORTED, "row size outside the batch kernels");
    }
}

template <int W>
void launch_crt_class(const TableCrtWork& w, int ctas, const DeviceBasis& B, uint32_t* err, cudaStream_t st) {
    const size_t smem = k3t_smem_bytes<4>();
    cuda_check(cudaFuncSetAttribute(k3t_crt<4, W, TableCrtWork>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem)),
               "batch CRT shared memory");
    k3t_crt<4, W, TableCrtWork><<<ctas, tc::kCrtThreads, smem, st>>>(w, B.d_pc, B.d_tw_inv, err);
}

void launch_crt_any(int W, const TableCrtWork& w, int ctas, const DeviceBasis& B, uint32_t* err, cudaStream_t st) {
    switch (W) {
        case 4: return launch_crt_class<4>(w, ctas, B, err, st);
        case 8: return launch_crt_class<8>(w, ctas, B, err, st);
        case 12: return launch_crt_class<12>(w, ctas, B, err, st);
        case 16: return launch_crt_class<16>(w, ctas, B, err, st);
        case 20: return launch_crt_class<20>(w, ctas, B, err, st);
        case 24: return launch_crt_class<24>(w, ctas, B, err, st);
        case 28: return launch_crt_class<28>(w, ctas, B, err, st);
        default: throw Failure(PM_ERR_UNSUPPORTED, "unsupported width");
    }
}

}  // namespace

struct BatchCore {
    int device = 0;
    uint32_t count = 0, coef_limbs = 0;
    std::vector<std::unique_ptr<PlanCore>> plans;
    std::vector<uint64_t> io_off;  // u64 words per product
    size_t io_words = 0;           // u64 words of one of a, b, c
    uint64_t* d_a = nullptr;
    uint64_t* d_b = nullptr;
    uint64_t* d_c = nullptr;
    uint32_t* d_work = nullptr;
    BatchProduct* d_prod = nullptr;
    CUtensorMap* d_maps = nullptr;
    uint4* d_conv_items = nullptr;
    uint4* d_row_items = nullptr;
    uint2* d_crt_items = nullptr;
    uint32_t* d_err = nullptr;
    int conv_items = 0;
    struct RowClass {
        int logC, radix_log, rows, count;
        size_t offset;  // into d_row_items
    };
    struct CrtClass {
        int W, count;
        size_t offset;  // into d_crt_items
    };
    std::vector<RowClass> row_classes;
    std::vector<CrtClass> crt_classes;
    cudaGraphExec_t graph = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    int conv_ctas_per_sm = 3, crt_ctas_per_sm = 2;  // persistent grid sizes (autotuned)

    ~BatchCore() {
        cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        for (auto s : streams) cudaStreamDestroy(s);
        for (auto e : events) cudaEventDestroy(e);
        cudaFree(d_a);
        cudaFree(d_b);
        cudaFree(d_c);
        cudaFree(d_work);
        cudaFree(d_prod);
        cudaFree(d_maps);
        cudaFree(d_conv_items);
        cudaFree(d_row_items);
        cudaFree(d_crt_items);
        cudaFree(d_err);
    }

    // Issue the three phases on streams[0], classes of a phase on forked streams.
    void enqueue(cudaStream_t st0) {
        const DeviceBasis& B = *plans[0]->basis;
        const int sms = sm_count_dev();
        TableConvWork cw{d_conv_items, conv_items, d_prod, d_maps, d_work};
        k1t_convert<4, TableConvWork><<<std::min(conv_items, sms * conv_ctas_per_sm), tc::kConvThreads, k1t_smem_bytes(), st0>>>(
            cw, B.d_pc, B.d_conv_weights, B.d_tw_fwd, d_err);
        cuda_check(cudaGetLastError(), "batch conversion launch");
        auto fork = [&](size_t k) {
            cudaStream_t s = streams[1 + k % (streams.size() - 1)];
            cuda_check(cudaEventRecord(events[0], st0), "batch fork");
            cuda_check(cudaStreamWaitEvent(s, events[0], 0), "batch fork");
            return s;
        };
        auto join = [&](cudaStream_t s, size_t k) {
            cudaEvent_t e = events[1 + k % (events.size() - 1)];
            cuda_check(cudaEventRecord(e, s), "batch join");
            cuda_check(cudaStreamWaitEvent(st0, e, 0), "batch join");
        };
        std::vector<cudaStream_t> used;
        for (size_t k = 0; k < row_classes.size(); ++k) {
            const RowClass& rc = row_classes[k];
            cudaStream_t s = fork(k);
            launch_rows_any(rc.logC, rc.radix_log, d_row_items + rc.offset, rc.count, rc.rows, d_prod, d_work, B, d_err,
                            s);
            used.push_back(s);
        }
        for (size_t k = 0; k < used.size(); ++k) join(used[k], k);
        used.clear();
        for (size_t k = 0; k < crt_classes.size(); ++k) {
            const CrtClass& cc = crt_classes[k];
            cudaStream_t s = fork(k);
            TableCrtWork w{d_crt_items + cc.offset, cc.count, d_prod, d_maps, d_work, reinterpret_cast<uint32_t*>(d_c)};
            launch_crt_any(cc.W, w, std::min(cc.count, sms * crt_ctas_per_sm), B, d_err, s);
            used.push_back(s);
        }
        for (size_t k = 0; k < used.size(); ++k) join(used[k], k);
        cuda_check(cudaGetLastError(), "batch launches");
    }

    void build(uint32_t cnt, const uint32_t* ns, const uint64_t* const* qs, const uint32_t* q_limbs, uint32_t limbs) {
        count = cnt;
        coef_limbs = limbs;
        if (limbs % 2) throw Failure(PM_ERR_UNSUPPORTED, "batches need an even coef_limbs (16-byte coefficient rows)");
        cuda_check(cudaGetDevice(&device), "cudaGetDevice");
        std::vector<BatchProduct> prod(cnt);
        std::vector<size_t> ws_off(cnt);
        size_t io = 0, ws = 0;
        for (uint32_t z = 0; z < cnt; ++z) {
            if (ns[z] < 256) throw Failure(PM_ERR_UNSUPPORTED, "batched products need n >= 256");
            auto p = std::make_unique<PlanCore>();
            p->init_tables_only(ns[z], qs[z], q_limbs[z], limbs, PM_CONVERT_TENSOR);
            if (p->logR != 4) throw Failure(PM_ERR_UNSUPPORTED, "batched products need 16-row views");
            io_off.push_back(io);
            ws_off[z] = ws;
            io += size_t(p->n) * limbs;
            ws += p->workspace_bytes / 4;
            BatchProduct& d = prod[z];
            d.n = int(p->n);
            d.logC = int(p->logC);
            d.P = int(p->P);
            d.W = int(p->W);
            d.sbits = int(p->qbits);
            d.delta = p->delta;
            d.stride = int(p->stride);
            d.mu_q = p->mu_q;
            d.io_off = 2 * io_off[z];
            d.ws_off = ws_off[z];
            d.scale = p->d_scale;
            d.consts = p->d_consts;
            d.ktab = p->d_ktab;
            d.crt_w = p->d_crt_weights;
            d.kfrac = p->d_kfrac;
            plans.push_back(std::move(p));
        }
        io_words = io;
        cuda_check(cudaMalloc(&d_a, io * 8), "batch a");
        cuda_check(cudaMalloc(&d_b, io * 8), "batch b");
        cuda_check(cudaMalloc(&d_c, io * 8), "batch c");
        cuda_check(cudaMalloc(&d_work, ws * 4), "batch workspace");
        cuda_check(cudaMalloc(&d_err, 4), "batch error word");
        cuda_check(cudaMemset(d_err, 0, 4), "batch error word");
        // tensor maps: a, b coefficient bytes and residue planes of each product
        std::vector<CUtensorMap> maps(3 * size_t(cnt));
        for (uint32_t z = 0; z < cnt; ++z) {
            const PlanCore& p = *plans[z];
            const cuuint64_t C = 1ull << p.logC, R = 1ull << p.logR, sb = p.stride * 4ull;
            const cuuint32_t Gc = cuuint32_t(C < 8 ? C : 8);
            const cuuint64_t cdims[4] = {sb, C, R, 1};
            const cuuint64_t cstr[3] = {sb, sb * C, sb * C * R};
            const cuuint32_t cbox[4] = {128, Gc, cuuint32_t(R), 1};
            maps[3 * z] = encode(CU_TENSOR_MAP_DATA_TYPE_UINT8, d_a + io_off[z], cdims, cstr, cbox,
                                 CU_TENSOR_MAP_SWIZZLE_128B);
            maps[3 * z + 1] = encode(CU_TENSOR_MAP_DATA_TYPE_UINT8, d_b + io_off[z], cdims, cstr, cbox,
                                     CU_TENSOR_MAP_SWIZZLE_128B);
            // box lands as [row][64 primes][column]: a constant row stride (primes past P read as zero)
            const cuuint64_t rdims[4] = {C, p.P, R, 1};
            const cuuint64_t rstr[3] = {C * R * 4, C * 4, p.workspace_bytes};
            const cuuint32_t rbox[4] = {Gc, cuuint32_t(tc::kMaxPrimes), cuuint32_t(R), 1};
            maps[3 * z + 2] = encode(CU_TENSOR_MAP_DATA_TYPE_UINT32, d_work + ws_off[z], rdims, rstr, rbox,
                                     CU_TENSOR_MAP_SWIZZLE_NONE);
        }
        // work tables
        std::vector<uint4> conv;
        for (int pg = 0; pg < 4; ++pg)
            for (uint32_t z = 0; z < cnt; ++z) {
                const PlanCore& p = *plans[z];
                if (pg * 16 >= int(p.P)) continue;
                const uint32_t groups = (1u << p.logC) / 8;
                for (uint32_t poly = 0; poly < 2; ++poly)
                    for (uint32_t cg = 0; cg < groups; ++cg) conv.push_back(make_uint4(z, pg, poly, cg));
            }
        conv_items = int(conv.size());
        std::map<int, std::vector<uint4>> rows_by_c;
        std::map<int, int> rows_per_item;
        for (uint32_t z = 0; z < cnt; ++z) {
            const PlanCore& p = *plans[z];
            const int T = (1 << p.logC) / 8, R = 1 << p.logR;
            int rows = T >= 128 ? 1 : 128 / T;
            if (rows > R) rows = R;
            rows_per_item[int(p.logC)] = rows;
            for (uint32_t i = 0; i < p.P; ++i)
                for (int r = 0; r < R; r += rows) rows_by_c[int(p.logC)].push_back(make_uint4(z, i, uint32_t(r), 0));
        }
        std::vector<uint4> row_items;
        for (auto& [logC, items] : rows_by_c) {
            if (logC >= 10)  // the persistent row kernel: consecutive items share a (prime, row) pair
                std::stable_sort(items.begin(), items.end(), [](const uint4& x, const uint4& y) {
                    return x.y != y.y ? x.y < y.y : x.z < y.z;
                });
            // the radix the autotuner picked for plans of this row size; by default radix 16
            // for the persistent kernel's rows (C >= 1024), radix 8 below
            int radix_log = logC >= 10 ? 4 : 3;
            for (auto& p : plans)
                if (int(p->logC) == logC && p->tune.tuned) radix_log = p->tune.row_radix_log;
            row_classes.push_back(RowClass{logC, radix_log, rows_per_item[logC], int(items.size()), row_items.size()});
            row_items.insert(row_items.end(), items.begin(), items.end());
        }
        std::map<int, std::vector<uint2>> crt_by_w;
        for (uint32_t z = 0; z < cnt; ++z) {
            const PlanCore& p = *plans[z];
            for (uint32_t cg = 0; cg < (1u << p.logC) / 8; ++cg) crt_by_w[int(p.W)].push_back(make_uint2(z, cg));
        }
        std::vector<uint2> crt_items;
        for (auto& [W, items] : crt_by_w) {
            crt_classes.push_back(CrtClass{W, int(items.size()), crt_items.size()});
            crt_items.insert(crt_items.end(), items.begin(), items.end());
        }
        auto upload = [](auto** dst, const auto& v, const char* what) {
            using T = std::remove_pointer_t<std::remove_reference_t<decltype(*dst)>>;
            cuda_check(cudaMalloc(dst, v.size() * sizeof(T)), what);
            cuda_check(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
        };
        upload(&d_prod, prod, "batch descriptors");
        upload(&d_maps, maps, "batch tensor maps");
        upload(&d_conv_items, conv, "batch conversion items");
        upload(&d_row_items, row_items, "batch row items");
        upload(&d_crt_items, crt_items, "batch CRT items");
        // streams for capture: the main one and one per concurrent class
        const size_t branches = std::max<size_t>(2, std::max(row_classes.size(), crt_classes.size()) + 1);
        streams.resize(branches);
        events.resize(branches);
        for (auto& s : streams) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch stream");
        for (auto& e : events) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
        capture();
    }

    // (Re)build the graph from the current launch shapes.  One warm run outside
    // capture first sets every kernel's shared-memory attribute.
    void capture() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        cuda_check(cudaFuncSetAttribute(k1t_convert<4, TableConvWork>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(k1t_smem_bytes())),
                   "batch conversion shared memory");
        enqueue(streams[0]);
        cuda_check(cudaStreamSynchronize(streams[0]), "batch warm-up");
        cudaGraph_t g = nullptr;
        cuda_check(cudaStreamBeginCapture(streams[0], cudaStreamCaptureModeThreadLocal), "batch capture");
        try {
            enqueue(streams[0]);
        } catch (...) {
            cudaStreamEndCapture(streams[0], &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cuda_check(cudaStreamEndCapture(streams[0], &g), "batch capture end");
        const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "batch graph instantiate");
    }

    // Device time of one graph run (mean of `reps`).
    double time_us(int reps) {
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "batch timing");
        cuda_check(cudaEventCreate(&e1), "batch timing");
        cuda_check(cudaGraphLaunch(graph, streams[0]), "batch timing");
        cuda_check(cudaEventRecord(e0, streams[0]), "batch timing");
        for (int r = 0; r < reps; ++r) cuda_check(cudaGraphLaunch(graph, streams[0]), "batch timing");
        cuda_check(cudaEventRecord(e1, streams[0]), "batch timing");
        cuda_check(cudaEventSynchronize(e1), "batch timing");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return 1000.0 * ms / reps;
    }

    // Coordinate descent over the launch shapes, whole-graph time as the objective.
    double tune(int reps) {
        double best = time_us(reps);
        auto attempt = [&](auto apply, auto undo) {
            apply();
            capture();
            const double t = time_us(reps);
            if (t < best) {
                best = t;
                return;
            }
            undo();
            capture();
        };
        for (auto& rc : row_classes)
            for (int k : {2, 3, 4}) {
                const int cur = rc.radix_log;
                if (k == cur || (k == 4 && rc.logC < 10)) continue;  // radix 16: persistent kernel rows only
                attempt([&] { rc.radix_log = k; }, [&] { rc.radix_log = cur; });
            }
        for (int k : {2, 3, 4}) {
            const int old = conv_ctas_per_sm;
            if (k == old) continue;
            attempt([&] { conv_ctas_per_sm = k; }, [&] { conv_ctas_per_sm = old; });
        }
        {
            const int old = crt_ctas_per_sm;
            attempt([&] { crt_ctas_per_sm = 1; }, [&] { crt_ctas_per_sm = old; });
        }
        return best;
    }

    void run(cudaStream_t st) {
        cuda_check(cudaGraphLaunch(graph, st), "batch graph launch");
        count_launches(1 + row_classes.size() + crt_classes.size());
    }
};

}  // namespace pm

struct pm_batch {
    pm::BatchCore core;
};

extern "C" int pm_batch_create(pm_batch** out, uint32_t count, const uint32_t* n, const uint64_t* const* q,
                               const uint32_t* q_limbs, uint32_t coef_limbs) {
    if (!out || !n || !q || !q_limbs || count == 0) return pm::fail(PM_ERR_INVALID, "NULL argument or empty batch");
    *out = nullptr;
    try {
        auto b = std::make_unique<pm_batch>();
        b->core.build(count, n, q, q_limbs, coef_limbs);
        *out = b.release();
        return PM_OK;
    } catch (const pm::Failure& f) {
        return pm::fail(f.status, f.what());
    } catch (const std::exception& e) {
        return pm::fail(PM_ERR_INVALID, e.what());
    }
}

extern "C" int pm_batch_buffers(pm_batch* batch, uint64_t** a, uint64_t** b, uint64_t** c, uint64_t* offsets) {
    if (!batch) return pm::fail(PM_ERR_INVALID, "NULL batch");
    const auto& s = batch->core;
    if (a) *a = s.d_a;
    if (b) *b = s.d_b;
    if (c) *c = s.d_c;
    if (offsets)
        for (uint32_t z = 0; z < s.count; ++z) offsets[z] = s.io_off[z];
    return PM_OK;
}

extern "C" int pm_batch_copy_in(pm_batch* batch, const uint64_t* a, const uint64_t* b, pm_stream stream) {
    if (!batch || !a || !b) return pm::fail(PM_ERR_INVALID, "NULL argument");
    auto& s = batch->core;
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(s.d_a, a, s.io_words * 8, cudaMemcpyDefault, st) != cudaSuccess ||
        cudaMemcpyAsync(s.d_b, b, s.io_words * 8, cudaMemcpyDefault, st) != cudaSuccess)
        return pm::fail(PM_ERR_CUDA, "batch copy in");
    return PM_OK;
}

extern "C" int pm_batch_copy_out(pm_batch* batch, uint64_t* c, pm_stream stream) {
    if (!batch || !c) return pm::fail(PM_ERR_INVALID, "NULL argument");
    auto& s = batch->core;
    if (cudaMemcpyAsync(c, s.d_c, s.io_words * 8, cudaMemcpyDefault, reinterpret_cast<cudaStream_t>(stream)) !=
        cudaSuccess)
        return pm::fail(PM_ERR_CUDA, "batch copy out");
    return PM_OK;
}

extern "C" int pm_batch_run(pm_batch* batch, pm_stream stream) {
    if (!batch) return pm::fail(PM_ERR_INVALID, "NULL batch");
    try {
        batch->core.run(reinterpret_cast<cudaStream_t>(stream));
        return PM_OK;
    } catch (const pm::Failure& f) {
        return pm::fail(f.status, f.what());
    }
}

extern "C" int pm_batch_check(pm_batch* batch) {
    if (!batch) return pm::fail(PM_ERR_INVALID, "NULL batch");
    uint32_t err = 0;
    if (cudaMemcpy(&err, batch->core.d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return pm::fail(PM_ERR_CUDA, "read batch error word");
    if (err) {
        cudaMemset(batch->core.d_err, 0, 4);
        return pm::fail(PM_ERR_TIMEOUT, "a tensor-core wait timed out during a batch run");
    }
    return PM_OK;
}

extern "C" int pm_batch_autotune(pm_batch* batch, uint32_t reps, double* us_per_run) {
    if (!batch) return pm::fail(PM_ERR_INVALID, "NULL batch");
    try {
        const double us = batch->core.tune(reps ? int(reps) : 3);
        if (us_per_run) *us_per_run = us;
        return PM_OK;
    } catch (const pm::Failure& f) {
        return pm::fail(f.status, f.what());
    }
}

extern "C" int pm_batch_destroy(pm_batch* batch) {
    delete batch;
    return PM_OK;
}
