// pcc_objects.h -- the opaque objects of include/pcc.h and the error helpers
// shared by the translation units that implement the C ABI.
#pragma once
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "pcc.h"
#include "pcc_internal.h"

namespace pcc {
struct Server;

// Launch tables of one batch march: BatchSolve[], int2 items[], class
// counters and march counters, in device memory with a pinned staging copy.
struct BatchTables {
    void* d = nullptr;
    size_t d_bytes = 0;
    void* h = nullptr;
    size_t h_bytes = 0;
    size_t cnt_off = 0;         // offset of the march counters
    cudaEvent_t ev[2]{};        // bracket of the march launch
    MarchLaunchInfo info{};
};
}  // namespace pcc

struct pcc_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    std::mutex err_mu;  // guards last_error
    std::vector<pcc_solve*> solves;  // live solves; destroyed with the context
    // LU workspace (grown on demand)
    void* lu_work = nullptr;
    size_t lu_work_bytes = 0;
    pcc::BatchTables batch;         // tables of the synchronous batch entry points
    pcc::Server* server = nullptr;  // serving loop (serve.cu), guarded by serve_mu
    std::mutex serve_mu;            // start, stop and the lookups of pcc_submit/poll/wait/stats
};

struct pcc_solve {
    pcc_ctx* ctx = nullptr;
    pcc_solve_desc d{};
    int nn = 0;      // Nnewton
    int ngrid = 0;   // nl + nr + 1
    int stages = 2;
    double a[3][3]{}, b[3]{}, c[3]{};
    double dm2c = 0.0;
    std::vector<double> grid;
    // device buffers
    double* d_grid = nullptr;
    double2* d_tw = nullptr;
    double* d_in0 = nullptr;
    double* d_out0 = nullptr;
    double* d_J = nullptr;
    double* d_yinit = nullptr;    // [2*(nn+1)][N]
    double* d_yfinal = nullptr;   // [2*(nn+1)][N]
    double* d_outc = nullptr;     // [nn+1][nn]
    int* d_status = nullptr;      // [2*(nn+1)] march status
    int* d_fail = nullptr;        // [2*(nn+1)]
    int* d_cstatus = nullptr;     // [nn+1] epilogue status
    int* d_counters_i = nullptr;  // [4] work counters
    unsigned long long* d_counters = nullptr;  // [4] march counters
    double* d_scratch = nullptr;
    int scratch_ctas = 0;
    int* d_item_side = nullptr;   // pcc_sweep
    // Sweep lists (slots 2 column + side, see pcc::sweep_list) of the column
    // pipelines: the build over columns [0, nn] (Jacobian and base shoot),
    // the Jacobian over [0, nn) and the base shoot alone, on the host and in
    // d_sweeps at sweep_off[0..2]; sweep_off[3] holds the list of the last
    // other column range (range_c0, range_c1).
    std::vector<int> sweeps_build, sweeps_jac, sweeps_base, sweeps_range;
    int* d_sweeps = nullptr;      // [8 (nn + 1)]
    int* d_sched = nullptr;       // [kMarchSchedWords] two-ended claiming of the single-solve march
    int sweep_off[4] = {0, 0, 0, 0};
    int range_c0 = -1, range_c1 = -1;
    double* d_xs = nullptr;       // pcc_sweep / test entry points (x_in, x_out)
    int* d_its = nullptr;
    // device-resident Newton iteration (newton.cu)
    pcc::NewtonDev* d_newton = nullptr;
    double* d_in0old = nullptr;
    double* d_rhs = nullptr;
    double* d_dx = nullptr;
    int* d_ipiv = nullptr;
    int* d_info = nullptr;    // [2]: LU info, FP64 fallback flag
    void* d_luw = nullptr;    // mixed-precision LU workspace
    int* d_cancel = nullptr;  // nonzero: remaining sweeps of this solve are skipped
    size_t footprint = 0;     // device bytes held by this solve
    cudaStream_t alloc_stream = nullptr;  // stream-ordered allocation (serving), else cudaMalloc
    std::vector<double2> tw_host;         // twiddle table (source of the asynchronous upload)
    int h_newton = -1;        // host copy of the Newton state code (-1: no iteration begun)
    // last asynchronous build
    int pend_c0 = 0, pend_c1 = 0;
    bool pending = false;
    cudaEvent_t ev[5]{};
    // the captured Jacobian build of pcc_jacobian_device (CUDA graph), for one
    // set of device pointers
    cudaGraphExec_t build_graph = nullptr;
    const void* graph_key[3] = {nullptr, nullptr, nullptr};
    pcc::MarchLaunchInfo last_launch{};
};


namespace pcc {

// Stops the serving loop of ctx, if one runs, and releases its solves.
void server_shutdown(pcc_ctx* ctx);

// Building blocks shared with the serving loop (pcc_abi.cu).
struct BatchItem {
    pcc_solve* s;
    int item;  // 2 column + side
};
// The sweeps (slots 2 column + side) a pipeline over columns [c0, c1) marches,
// right sides first, each side in column order.  With side reuse (the
// default; pcc_solve_desc.shoot_both_sides = 0) a column marches only the
// sides that read its free datum, and the base shoot's sides are added where
// a column takes one of them.
void sweep_list(const pcc_solve* s, int c0, int c1, std::vector<int>& out);
// The host list of columns [0, ncols) for ncols = nn (Jacobian) or nn + 1 (build).
const std::vector<int>& sweeps_from_zero(const pcc_solve* s, int ncols);
// A solve whose buffers come from cudaMallocAsync on alloc_st (nullptr: cudaMalloc)
// and which is not registered with its context.
pcc_status solve_create(pcc_ctx* ctx, const pcc_solve_desc* desc, cudaStream_t alloc_st, bool registered,
                        pcc_solve** out);
void solve_release(pcc_solve* s);
size_t solve_footprint(const pcc_solve_desc& d, int sms);
pcc_status newton_reset(pcc_solve* s, const double* in0_host, cudaStream_t st);
pcc_status newton_prologue(pcc_solve* s, cudaStream_t st);
pcc_status newton_tail(pcc_solve* s, pcc_precision prec, cudaStream_t st, int* lu_steps, int* lu_fallback);
// One persistent launch over an explicit list of sweeps (every solve batch-supported).
pcc_status batch_march_items(pcc_ctx* ctx, BatchTables& tab, const std::vector<BatchItem>& items,
                             cudaStream_t st, int max_ctas);
pcc_status batch_tables_reserve(pcc_ctx* ctx, BatchTables& tab, size_t bytes);
void batch_tables_free(BatchTables& tab);

inline pcc_status fail(pcc_ctx* ctx, pcc_status s, const std::string& msg)
{
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->err_mu);  // the serving thread reports here too
        ctx->last_error = msg;
    }
    return s;
}

// Free data handed in through host pointers must be finite: a NaN or an
// infinity would only surface later as a failed IRK iteration.
inline bool all_finite(const double* v, int n)
{
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

}  // namespace pcc

#define PCC_CUDA(ctx, call)                                                                          \
    do {                                                                                             \
        cudaError_t _e = (call);                                                                     \
        if (_e != cudaSuccess) {                                                                     \
            return pcc::fail((ctx), _e == cudaErrorMemoryAllocation ? PCC_ERR_OOM : PCC_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(_e));                    \
        }                                                                                            \
    } while (0)
