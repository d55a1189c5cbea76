// pcc_abi.cu -- the C ABI of include/pcc.h over the CUDA kernels.
//
// A Jacobian build (NewtonSolver::assembleJacobian, NewtonSolver.cpp:615-702)
// is one stream-ordered pipeline over columns [c0, c1):
//   1. prologue : per (column, side) unpack + Taylor expansion  -> y_init
//   2. march    : ONE persistent launch over all 2*(c1-c0) sweeps -> y_final
//   3. epilogue : per column mismatch, fields, pack               -> out_c
//   4. fd       : J[:, c] = (out_c - out0) / eps (tiled transpose)
// Column index Nnewton denotes the unperturbed base shoot.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "pcc.h"
#include "pcc_internal.h"
#include "pcc_objects.h"

using namespace pcc;

cudaStream_t pcc_ctx_stream(pcc_ctx* ctx) { return ctx->stream; }
int pcc_ctx_device(pcc_ctx* ctx) { return ctx->device; }
void pcc_ctx_set_error(pcc_ctx* ctx, const char* msg) { fail(ctx, PCC_OK, msg); }

namespace {

const char* kStatusNames[] = {"PCC_OK",
                              "PCC_ERR_INVALID_ARG",
                              "PCC_ERR_CUDA",
                              "PCC_ERR_OOM",
                              "PCC_ERR_IRK_NO_CONVERGENCE",
                              "PCC_ERR_DELTA_MISMATCH",
                              "PCC_ERR_NAN",
                              "PCC_ERR_LU_SINGULAR",
                              "PCC_ERR_IR_STALL",
                              "PCC_ERR_UNSUPPORTED",
                              "PCC_ERR_NEWTON_NO_CONVERGENCE",
                              "PCC_ERR_BUSY",
                              "PCC_ERR_TIMEOUT"};

// Gauss-Legendre tableaux exactly as ODEStepper.cpp:27-79 builds them.
int tableau(int scheme, double a[3][3], double b[3], double c[3])
{
    for (int i = 0; i < 3; ++i) {
        b[i] = c[i] = 0.0;
        for (int j = 0; j < 3; ++j) a[i][j] = 0.0;
    }
    if (scheme == 1) {
        a[0][0] = 0.5;
        b[0] = 1.0;
        c[0] = 0.5;
        return 1;
    }
    if (scheme == 3) {
        a[0][0] = 5.0 / 36.0;
        a[0][1] = 2.0 / 9.0 - 1.0 / std::sqrt(15.0);
        a[0][2] = 5.0 / 36.0 - 0.5 / std::sqrt(15.0);
        a[1][0] = 5.0 / 36.0 + std::sqrt(15.0) / 24.0;
        a[1][1] = 2.0 / 9.0;
        a[1][2] = 5.0 / 36.0 - std::sqrt(15.0) / 24.0;
        a[2][0] = 5.0 / 36.0 + 0.5 / std::sqrt(15.0);
        a[2][1] = 2.0 / 9.0 + 1.0 / std::sqrt(15.0);
        a[2][2] = 5.0 / 36.0;
        b[0] = b[2] = 5.0 / 18.0;
        b[1] = 4.0 / 9.0;
        c[0] = 0.5 - std::sqrt(15.0) / 10.0;
        c[1] = 0.5;
        c[2] = 0.5 + std::sqrt(15.0) / 10.0;
        return 3;
    }
    a[0][0] = 0.25;
    a[0][1] = 0.25 - 0.5 / std::sqrt(3.0);
    a[1][0] = 0.25 + 0.5 / std::sqrt(3.0);
    a[1][1] = 0.25;
    b[0] = b[1] = 0.5;
    c[0] = 0.5 - 0.5 / std::sqrt(3.0);
    c[1] = 0.5 + 0.5 / std::sqrt(3.0);
    return 2;
}

// Integrated Lagrange basis on the Gauss nodes c: int_0^theta l_j(tau) dtau
// = sum_k lq[j][k] theta^(k+1), l_j(tau) = prod_{m != j} (tau - c_m)/(c_j - c_m).
// Used by the optional stage predictor of the march.
void lagrange_integrals(int stages, const double c[3], double lq[3][3])
{
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) lq[j][k] = 0.0;
    for (int j = 0; j < stages; ++j) {
        double p[3] = {1.0, 0.0, 0.0};  // coefficients of l_j, ascending powers
        int deg = 0;
        for (int m = 0; m < stages; ++m) {
            if (m == j) continue;
            const double d = c[j] - c[m];
            double q[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k <= deg; ++k) {
                q[k + 1] += p[k] / d;
                q[k] -= p[k] * c[m] / d;
            }
            ++deg;
            for (int k = 0; k < 3; ++k) p[k] = q[k];
        }
        for (int k = 0; k <= deg; ++k) lq[j][k] = p[k] / (k + 1);
    }
}

// exp(+2 pi i k/n), k < n, rounded from long-double trigonometry, followed
// for the march's sizes by its per-pass tables (march_twiddle_count(n)
// entries in all), whose entries are copies of point twiddles: the
// exponent r k/(NS R) of a length-M pass is 2 r k M/(NS R) / n.
int twiddle_count(int n) { return march_supported(n, 1) ? march_twiddle_count(n) : n; }

std::vector<double2> twiddles(int n)
{
    std::vector<double2> tw(twiddle_count(n));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
        const long double a = two_pi * (long double)k / (long double)n;
        tw[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    if ((int)tw.size() > n) {
        const int M = n / 2;
        for (int ns = 8; ns < M; ns *= 8) {
            const int R = pass_radix(M, ns);
            double2* tab = tw.data() + n + pass_table_offset(M, ns);
            for (int r = 1; r < R; ++r)
                for (int k = 0; k < ns; ++k) tab[(r - 1) * ns + k] = tw[2 * (r * k * (M / (ns * R)))];
        }
    }
    if (n == 1024 && (int)tw.size() >= w512_table_offset(n) + kW512Tables) {
        // the warp-exchange length-512 tables (march.cuh): exp(+2 pi i e/512) = tw[2 e mod 1024]
        double2* w = tw.data() + w512_table_offset(n);
        for (int k = 0; k < 8; ++k)
            for (int q = 0; q < 8; ++q) w[k * 8 + q] = tw[16 * ((q * k) % 64)];
        for (int r = 0; r < 8; ++r)
            for (int t = 0; t < 64; ++t) {
                w[64 + r * 64 + t] = tw[2 * (((t & 7) * ((t >> 3) + 8 * r)) % 512)];
                w[64 + 512 + r * 64 + t] = tw[2 * (((t >> 3) * ((t & 7) + 8 * r)) % 512)];
            }
    }
    return tw;
}

// NewtonSolver::generateGrid (NewtonSolver.cpp:477-519): uniform in logit x.
// This runs once per solve on the host, as the reference's driver does.
void make_grid(const pcc_solve_desc& d, std::vector<double>& g)
{
    const int il = 0, im = d.nl, ir = d.nl + d.nr;
    g.assign(ir + 1, 0.0);
    g[il] = d.xl;
    g[im] = d.xm;
    g[ir] = d.xr;
    const double zl = std::log(d.xl) - std::log(1.0 - d.xl);
    const double zm = std::log(d.xm) - std::log(1.0 - d.xm);
    const double zr = std::log(d.xr) - std::log(1.0 - d.xr);
    const double dzl = (zm - zl) / (double)d.nl;
    const double dzr = (zr - zm) / (double)d.nr;
    for (int j = il + 1; j < im; ++j) {
        const double e = zl + (double)(j - il) * dzl;
        g[j] = std::exp(e) / (1.0 + std::exp(e));
    }
    for (int j = im + 1; j < ir; ++j) {
        const double e = zm + (double)(j - im) * dzr;
        g[j] = std::exp(e) / (1.0 + std::exp(e));
    }
}

bool desc_ok(const pcc_solve_desc* d, std::string& why)
{
    if (!d) return why = "null descriptor", false;
    if (!march_supported(d->ntau, d->scheme)) return why = "Ntau must be 128..2048 (power of two), scheme 1..3", false;
    if (d->nl < 1 || d->nr < 1) return why = "NLeft and NRight must be positive", false;
    if (!(d->xl > 0.0 && d->xl < d->xm && d->xm < d->xr && d->xr < 1.0)) return why = "need 0 < XLeft < XMid < XRight < 1", false;
    if (!(d->eps_newton > 0.0)) return why = "EpsNewton must be positive", false;
    if (d->max_irk < 1) return why = "MaxIterIRK must be positive", false;
    if (!std::isfinite(d->dim) || d->dim <= 2.0) return why = "Dim must be finite and > 2", false;
    return true;
}

int boundary_ctas(pcc_solve* s, int items)
{
    int c = s->scratch_ctas;
    return items < c ? items : c;
}

MarchParams march_params(pcc_solve* s)
{
    MarchParams P{};
    P.grid = s->d_grid;
    P.nl = s->d.nl;
    P.nr = s->d.nr;
    P.dim = s->d.dim;
    P.dim_m2_cubed = s->dm2c;
    P.prec = s->d.prec_irk;
    P.max_its = s->d.max_irk;
    P.stages = s->stages;
    for (int i = 0; i < 3; ++i) {
        P.b[i] = s->b[i];
        P.c[i] = s->c[i];
        for (int j = 0; j < 3; ++j) P.a[i][j] = s->a[i][j];
    }
    P.predictor = s->d.irk_predictor ? 1 : 0;
    lagrange_integrals(s->stages, s->c, P.lq);
    P.twN = s->d_tw;
    P.status = s->d_status;
    P.fail_index = s->d_fail;
    P.counters = s->d_counters;
    return P;
}

bool reuses_sides(const pcc_solve* s) { return s->d.shoot_both_sides == 0; }

// The slot whose final state column col takes for side (0 left, 1 right).
int source_slot(int nn, bool reuse, int col, int side)
{
    const bool moves = side ? column_moves_right(col, nn) : column_moves_left(col, nn);
    return 2 * (reuse && !moves ? nn : col) + side;
}
int source_slot(const pcc_solve* s, int col, int side) { return source_slot(s->nn, reuses_sides(s), col, side); }

// The sweep list of columns [c0, c1) of a solve with nn free data (pcc::sweep_list).
void sweep_list_of(int nn, bool reuse, int c0, int c1, std::vector<int>& out)
{
    out.clear();
    bool base_needed[2] = {false, false};
    const bool has_base = c0 <= nn && nn < c1;
    for (int side = 1; side >= 0; --side) {
        for (int c = c0; c < c1; ++c) {
            const int src = source_slot(nn, reuse, c, side);
            if (src == 2 * c + side)
                out.push_back(src);
            else
                base_needed[side] = true;
        }
        if (base_needed[side] && !has_base) out.push_back(2 * nn + side);
    }
}

// The device copy of the sweep list of columns [c0, c1) and its length; a
// range other than the three fixed ones is built and uploaded (stream-ordered
// on st) when it differs from the last one.
pcc_status device_sweeps(pcc_solve* s, int c0, int c1, cudaStream_t st, const int** list, int* count)
{
    const int nn = s->nn;
    const std::vector<int>* v = nullptr;
    int k = 3;
    if (c0 == 0 && c1 == nn + 1) v = &s->sweeps_build, k = 0;
    else if (c0 == 0 && c1 == nn) v = &s->sweeps_jac, k = 1;
    else if (c0 == nn && c1 == nn + 1) v = &s->sweeps_base, k = 2;
    else {
        if (c0 != s->range_c0 || c1 != s->range_c1) {
            sweep_list(s, c0, c1, s->sweeps_range);
            s->range_c0 = s->range_c1 = -1;
            PCC_CUDA(s->ctx, cudaMemcpyAsync(s->d_sweeps + s->sweep_off[3], s->sweeps_range.data(),
                                             s->sweeps_range.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            s->range_c0 = c0;
            s->range_c1 = c1;
        }
        v = &s->sweeps_range;
    }
    *list = s->d_sweeps + s->sweep_off[k];
    *count = (int)v->size();
    return PCC_OK;
}

// The first failure among columns [c0, c1) of the last march and epilogue:
// the first column (in column order) whose left or right final state (left
// first, the order a shoot marches them) comes from a sweep that did not
// converge, else the first column with a Delta mismatch.  st and fi are the
// march's per-slot statuses and failing grid indices, cs the epilogue's
// statuses of the columns from c0.  Returns the status and sets col, side
// (-1 for a Delta mismatch) and the grid index.
pcc_status first_failure(const pcc_solve* s, int c0, int c1, const std::vector<int>& st,
                         const std::vector<int>& fi, const std::vector<int>& cs, int* col, int* side, int* idx)
{
    *col = *side = *idx = -1;
    for (int c = c0; c < c1; ++c)
        for (int sd = 0; sd < 2; ++sd) {
            const int slot = source_slot(s, c, sd);
            if (st[slot] != 0) {
                *col = c;
                *side = sd;
                *idx = fi[slot];
                return PCC_ERR_IRK_NO_CONVERGENCE;
            }
        }
    for (int c = c0; c < c1; ++c)
        if (cs[c - c0] != 0) {
            *col = c;
            return PCC_ERR_DELTA_MISMATCH;
        }
    return PCC_OK;
}

BoundaryParams boundary_params(pcc_solve* s, int c0)
{
    BoundaryParams B{};
    B.ntau = s->d.ntau;
    B.nn = s->nn;
    B.c0 = c0;
    B.dim = s->d.dim;
    B.xl = s->d.xl;
    B.xr = s->d.xr;
    B.eps = s->d.eps_newton;
    B.prec = s->d.prec_irk;
    B.dim_m2_cubed = s->dm2c;
    B.in0 = s->d_in0;
    B.out0 = s->d_out0;
    B.yinit = s->d_yinit;
    B.yfinal = s->d_yfinal;
    B.outc = s->d_outc;
    B.status = s->d_cstatus;
    B.scratch = s->d_scratch;
    B.tw = s->d_tw;
    return B;
}

// Boundary data of the sweeps of columns [c0, c1) from d_in0 -> d_yinit (and
// cleared counters and march statuses: a slot the list leaves out keeps
// status 0).
pcc_status enqueue_prologue(pcc_solve* s, int c0, int c1, cudaStream_t st)
{
    pcc_ctx* ctx = s->ctx;
    const int* list = nullptr;
    int items = 0;
    pcc_status r = device_sweeps(s, c0, c1, st, &list, &items);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_counters_i, 0, 4 * sizeof(int), st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_counters, 0, 4 * sizeof(unsigned long long), st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_status, 0, 2 * (s->nn + 1) * sizeof(int), st));
    BoundaryParams B = boundary_params(s, c0);
    B.n_items = items;
    B.sweeps = list;
    B.work_counter = s->d_counters_i + 0;
    PCC_CUDA(ctx, launch_prologue(B, boundary_ctas(s, items), st));
    return PCC_OK;
}

// The single-solve march over the sweeps of columns [c0, c1) (the list the
// prologue used).
pcc_status enqueue_march(pcc_solve* s, int c0, int c1, MarchParams& P, cudaStream_t st)
{
    const int* list = nullptr;
    int items = 0;
    pcc_status r = device_sweeps(s, c0, c1, st, &list, &items);
    if (r != PCC_OK) return r;
    P.n_items = items;
    P.item_map = list;
    P.mode = 0;
    P.yinit = s->d_yinit;
    P.yfinal = s->d_yfinal;
    P.work_counter = s->d_counters_i + 1;
    // two-ended claiming (march_claim_ends) unless PCC_MARCH_ENDS=0; read per
    // launch, so that a process can compare the two orders
    const char* ends = std::getenv("PCC_MARCH_ENDS");
    if (!(ends && std::string(ends) == "0")) {
        PCC_CUDA(s->ctx, cudaMemsetAsync(s->d_sched, 0, kMarchSchedWords * sizeof(int), st));
        P.sched = s->d_sched;
    }
    PCC_CUDA(s->ctx, launch_march(s->d.ntau, s->stages, P, 0, st, &s->last_launch));
    return PCC_OK;
}

// Mismatch of columns [c0, c1) -> d_outc, then (fd) J's columns [c0, min(c1, nn)).
pcc_status enqueue_epilogue(pcc_solve* s, int c0, int c1, bool fd, double* d_J, cudaStream_t st)
{
    pcc_ctx* ctx = s->ctx;
    const int ncols = c1 - c0;
    BoundaryParams B = boundary_params(s, c0);
    B.n_items = ncols;
    B.abs_slots = 1;
    B.reuse = reuses_sides(s) ? 1 : 0;
    B.work_counter = s->d_counters_i + 2;
    PCC_CUDA(ctx, launch_epilogue(B, boundary_ctas(s, ncols), st));
    if (fd) {
        // the base column (index nn) has no difference
        const int nfd = (c1 > s->nn ? s->nn : c1) - c0;
        if (nfd > 0) PCC_CUDA(ctx, launch_fd(s->d_outc, s->d_out0, d_J, s->nn, c0, nfd, s->d.eps_newton, st));
    }
    return PCC_OK;
}

// Records ev on st; while st is being captured into a CUDA graph the record
// becomes an external event node, so that it still timestamps each replay.
cudaError_t record_event(cudaEvent_t ev, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, st);
}

// Enqueues the build pipeline for columns [c0, c1) reading d_in0 (and d_out0
// for the differences when fd is set).  Events bracket the stages.
pcc_status enqueue_columns(pcc_solve* s, int c0, int c1, bool fd, double* d_J)
{
    pcc_ctx* ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    PCC_CUDA(ctx, record_event(s->ev[0], st));
    pcc_status r = enqueue_prologue(s, c0, c1, st);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, record_event(s->ev[1], st));
    MarchParams P = march_params(s);
    r = enqueue_march(s, c0, c1, P, st);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, record_event(s->ev[2], st));
    r = enqueue_epilogue(s, c0, c1, fd, d_J, st);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, record_event(s->ev[3], st));
    return PCC_OK;
}

// Reads statuses and counters of the last build (synchronises the stream).
pcc_status collect(pcc_solve* s, int c0, int c1, pcc_stats* stats)
{
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int ncols = c1 - c0;
    std::vector<int> st(2 * (s->nn + 1)), fi(2 * (s->nn + 1)), cs(ncols);
    unsigned long long cnt[4] = {0, 0, 0, 0};
    PCC_CUDA(ctx, cudaMemcpy(st.data(), s->d_status, st.size() * sizeof(int), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(fi.data(), s->d_fail, fi.size() * sizeof(int), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(cs.data(), s->d_cstatus, cs.size() * sizeof(int), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(cnt, s->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    int fcol = -1, fside = -1, fidx = -1;
    const pcc_status result = first_failure(s, c0, c1, st, fi, cs, &fcol, &fside, &fidx);
    if (fside < 0) fside = 0;
    if (stats) {
        float ms[3] = {0, 0, 0};
        cudaEventElapsedTime(&ms[0], s->ev[0], s->ev[1]);
        cudaEventElapsedTime(&ms[1], s->ev[1], s->ev[2]);
        cudaEventElapsedTime(&ms[2], s->ev[2], s->ev[3]);
        stats->rhs_evals = (long long)cnt[0];
        stats->irk_iterations = (long long)cnt[1];
        stats->irk_steps = (long long)cnt[2];
        stats->shoots = ncols;
        stats->ms_prologue = ms[0];
        stats->ms_sweep = ms[1];
        stats->ms_epilogue = ms[2];
        stats->ms_total = (double)ms[0] + ms[1] + ms[2];
        stats->fail_column = fcol;
        stats->fail_side = fside;
        stats->fail_grid_index = fidx;
        stats->sweep_ctas = s->last_launch.ctas;
    }
    if (result != PCC_OK) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "%s at column %d side %d grid index %d", kStatusNames[result], fcol, fside, fidx);
        fail(ctx, result, buf);
    }
    return result;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// The autotuner's cache: one line per (device name, Ntau, stages) with the
// chosen schedule and the probe times.  $PCC_AUTOTUNE_CACHE, else
// ~/.cache/pcc_b200/autotune.txt; $PCC_AUTOTUNE=0 disables tuning (paired
// transforms everywhere).
std::string autotune_cache_path()
{
    if (const char* p = std::getenv("PCC_AUTOTUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : ".") + "/.cache/pcc_b200/autotune.txt";
}

std::mutex g_autotune_mu;

// Makes sure the march kernel's transform schedule for (Ntau, stages) is
// chosen on the context's device: from the cache file, else by timing both
// schedules now (march_autotune) and appending the result to the cache.
void ensure_march_tuned(pcc_ctx* ctx, int ntau, int stages, const double2* d_tw, cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(g_autotune_mu);
    if (march_tuning(ctx->device, ntau, stages, nullptr)) return;
    if (const char* off = std::getenv("PCC_AUTOTUNE"))
        if (std::string(off) == "0") return;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return;
    const std::string name = prop.name;
    const std::string path = autotune_cache_path();
    {
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream is(line);
            std::string dev;
            int n = 0, s = 0, pair = 1;
            double mp = 0, ms = 0;
            if (!std::getline(is, dev, '\t')) continue;
            if (!(is >> n >> s >> pair >> mp >> ms)) continue;
            if (dev == name && n == ntau && s == stages) {
                march_set_tuning(ctx->device, ntau, stages, MarchTuning{pair, 0.0, 0.0, 0.0});
                return;
            }
        }
    }
    MarchTuning t{};
    if (march_autotune(ntau, stages, d_tw, st, &t) != cudaSuccess) {
        cudaGetLastError();  // keep the default schedule
        return;
    }
    std::error_code ec;
    std::filesystem::create_directories(std::filesystem::path(path).parent_path(), ec);
    std::ofstream out(path, std::ios::app);
    if (out)
        out << name << '\t' << ntau << ' ' << stages << ' ' << t.pair << ' ' << t.ms_pair << ' ' << t.ms_single << ' '
            << t.ms_wx << '\n';
}

// One persistent launch over the sweeps of columns [0, ncols[i]) of every
// solve in v (ncols nn or nn + 1, their sweep lists), with the context's own
// tables.
pcc_status enqueue_batch_march(pcc_ctx* ctx, const std::vector<pcc_solve*>& v, const std::vector<int>& ncols,
                               cudaStream_t st)
{
    std::vector<BatchItem> items;
    for (size_t i = 0; i < v.size(); ++i)
        for (int slot : sweeps_from_zero(v[i], ncols[i])) items.push_back({v[i], slot});
    return batch_march_items(ctx, ctx->batch, items, st, 0);
}

// Reads the counters and timing of the last batch march (stream synchronised).
void batch_stats(pcc_ctx* ctx, const std::vector<int>& ncols, pcc_stats* stats)
{
    if (!stats) return;
    std::memset(stats, 0, sizeof(*stats));
    unsigned long long cnt[4] = {0, 0, 0, 0};
    cudaMemcpy(cnt, static_cast<char*>(ctx->batch.d) + ctx->batch.cnt_off, 3 * sizeof(unsigned long long),
               cudaMemcpyDeviceToHost);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->batch.ev[0], ctx->batch.ev[1]);
    stats->rhs_evals = (long long)cnt[0];
    stats->irk_iterations = (long long)cnt[1];
    stats->irk_steps = (long long)cnt[2];
    long long shoots = 0;
    for (int c : ncols) shoots += c;
    stats->shoots = shoots;
    stats->ms_sweep = ms;
    stats->ms_total = ms;
    stats->fail_column = -1;
    stats->fail_grid_index = -1;
    stats->sweep_ctas = ctx->batch.info.ctas;
}

// Finds the first failing sweep or column of a solve's last shoots.
void solve_failure(pcc_solve* s, int ncols, int* col, int* side, int* idx)
{
    *col = *side = *idx = -1;
    std::vector<int> st(2 * (s->nn + 1)), fi(2 * (s->nn + 1)), cs(ncols);
    if (cudaMemcpy(st.data(), s->d_status, st.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    cudaMemcpy(fi.data(), s->d_fail, fi.size() * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(cs.data(), s->d_cstatus, cs.size() * sizeof(int), cudaMemcpyDeviceToHost);
    first_failure(s, 0, ncols, st, fi, cs, col, side, idx);
}

// After the march of one Newton iteration (base column nn and columns 0..nn-1):
// mismatches, the device-side check of NewtonSolver.cpp:300-325, J, the
// Newton solve and the damped update, all on stream st.
pcc_status enqueue_newton_tail(pcc_solve* s, pcc_precision prec, cudaStream_t st, int* lu_steps, int* lu_fallback)
{
    pcc_ctx* ctx = s->ctx;
    const int nn = s->nn;
    pcc_status r = enqueue_epilogue(s, 0, nn + 1, false, nullptr, st);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, s->d_outc + (size_t)nn * nn, nn * sizeof(double),
                                  cudaMemcpyDeviceToDevice, st));
    PCC_CUDA(ctx, launch_newton_check(s->d_newton, s->d_out0, nn, s->d_status, s->d_cstatus, s->d.prec_newton,
                                      s->d_rhs, st));
    PCC_CUDA(ctx, launch_fd(s->d_outc, s->d_out0, s->d_J, nn, 0, nn, s->d.eps_newton, st));
    *lu_steps = -1;
    *lu_fallback = 0;
    if (prec == PCC_PREC_MIXED) {
        double resid = -1.0;
        PCC_CUDA(ctx, lu_solve_mixed(s->d_J, s->d_rhs, s->d_dx, nn, s->d_luw, lu_mixed_work_bytes(nn), s->d_ipiv,
                                     s->d_info, 30, 1e-15, lu_steps, &resid, st));
    } else {
        PCC_CUDA(ctx, lu_solve_fp64(s->d_J, s->d_rhs, s->d_dx, nn, nullptr, s->d_ipiv, s->d_info, st));
    }
    PCC_CUDA(ctx, launch_newton_update(s->d_newton, s->d_in0, s->d_in0old, s->d_dx, s->d_info, nn,
                                       s->d.slow_error, s->d.max_newton, st));
    return PCC_OK;
}

void newton_state_from_dev(const NewtonDev& nd, pcc_newton_state* out)
{
    out->iterations = nd.its;
    out->code = nd.state;
    out->err = nd.err;
    out->err_old = nd.err_old;
    out->fail_column = out->fail_side = out->fail_grid_index = -1;
    out->lu_refinement_steps = -1;
    out->lu_fell_back = 0;
}

}  // namespace

void pcc::sweep_list(const pcc_solve* s, int c0, int c1, std::vector<int>& out)
{
    sweep_list_of(s->nn, reuses_sides(s), c0, c1, out);
}

const std::vector<int>& pcc::sweeps_from_zero(const pcc_solve* s, int ncols)
{
    return ncols > s->nn ? s->sweeps_build : s->sweeps_jac;
}

// ------------------------------------------------ shared with the serving loop
namespace pcc {

// Device bytes of one solve's buffers (the allocations of solve_create).
size_t solve_footprint(const pcc_solve_desc& d, int sms)
{
    const size_t n = d.ntau, nn = 3 * n / 4, cols = nn + 1, ngrid = (size_t)d.nl + d.nr + 1;
    const size_t dbl = sizeof(double), in = sizeof(int);
    return ngrid * dbl + twiddle_count(n) * sizeof(double2) + 2 * nn * dbl + nn * nn * dbl + 2 * (2 * cols * n * dbl) +
           cols * nn * dbl + 2 * (2 * cols * in) + cols * in + 4 * in + 4 * sizeof(unsigned long long) +
           (size_t)2 * sms * kBoundaryArrays * n * dbl + 2 * cols * in + 8 * cols * in + kMarchSchedWords * in + 4 * cols * dbl + 2 * cols * in +
           sizeof(NewtonDev) + 3 * nn * dbl + nn * in + 4 * in + lu_mixed_work_bytes((int)nn) + in;
}

pcc_status solve_create(pcc_ctx* ctx, const pcc_solve_desc* desc, cudaStream_t alloc_st, bool registered,
                        pcc_solve** out)
{
    if (!ctx || !out) return PCC_ERR_INVALID_ARG;
    *out = nullptr;
    std::string why;
    if (!desc_ok(desc, why)) return fail(ctx, PCC_ERR_INVALID_ARG, why);
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    auto* s = new pcc_solve;
    s->ctx = ctx;
    s->d = *desc;
    s->alloc_stream = alloc_st;
    s->nn = 3 * desc->ntau / 4;
    s->ngrid = desc->nl + desc->nr + 1;
    s->stages = tableau(desc->scheme, s->a, s->b, s->c);
    s->dm2c = std::pow(desc->dim - 2.0, 3);
    make_grid(*desc, s->grid);
    const int n = desc->ntau, nn = s->nn, cols = nn + 1;
    s->scratch_ctas = 2 * ctx->sms;
    auto cleanup = [&](pcc_status st, const std::string& m) {
        solve_release(s);
        return fail(ctx, st, m);
    };
#define ALLOC(ptr, bytes)                                                                                    \
    do {                                                                                                     \
        cudaError_t _e = alloc_st ? cudaMallocAsync((void**)&(ptr), (bytes), alloc_st)                       \
                                  : cudaMalloc((void**)&(ptr), (bytes));                                     \
        if (_e != cudaSuccess) return cleanup(PCC_ERR_OOM, std::string("cudaMalloc ") + #ptr + ": " + cudaGetErrorString(_e)); \
        s->footprint += (bytes);                                                                             \
    } while (0)
    ALLOC(s->d_grid, s->ngrid * sizeof(double));
    ALLOC(s->d_tw, twiddle_count(n) * sizeof(double2));
    ALLOC(s->d_in0, nn * sizeof(double));
    ALLOC(s->d_out0, nn * sizeof(double));
    ALLOC(s->d_J, (size_t)nn * nn * sizeof(double));
    ALLOC(s->d_yinit, (size_t)2 * cols * n * sizeof(double));
    ALLOC(s->d_yfinal, (size_t)2 * cols * n * sizeof(double));
    ALLOC(s->d_outc, (size_t)cols * nn * sizeof(double));
    ALLOC(s->d_status, 2 * cols * sizeof(int));
    ALLOC(s->d_fail, 2 * cols * sizeof(int));
    ALLOC(s->d_cstatus, cols * sizeof(int));
    ALLOC(s->d_counters_i, 4 * sizeof(int));
    ALLOC(s->d_counters, 4 * sizeof(unsigned long long));
    ALLOC(s->d_scratch, (size_t)s->scratch_ctas * kBoundaryArrays * n * sizeof(double));
    ALLOC(s->d_item_side, 2 * cols * sizeof(int));
    ALLOC(s->d_sweeps, 8 * cols * sizeof(int));
    ALLOC(s->d_sched, kMarchSchedWords * sizeof(int));
    ALLOC(s->d_xs, 4 * cols * sizeof(double));
    ALLOC(s->d_its, 2 * cols * sizeof(int));
    ALLOC(s->d_newton, sizeof(NewtonDev));
    ALLOC(s->d_in0old, nn * sizeof(double));
    ALLOC(s->d_rhs, nn * sizeof(double));
    ALLOC(s->d_dx, nn * sizeof(double));
    ALLOC(s->d_ipiv, nn * sizeof(int));
    ALLOC(s->d_info, 4 * sizeof(int));  // singular index, fell back, tensor-core wait error
    ALLOC(s->d_luw, lu_mixed_work_bytes(nn));
    ALLOC(s->d_cancel, sizeof(int));
#undef ALLOC
    cudaStream_t st = alloc_st ? alloc_st : ctx->stream;
    sweep_list(s, 0, nn + 1, s->sweeps_build);
    sweep_list(s, 0, nn, s->sweeps_jac);
    sweep_list(s, nn, nn + 1, s->sweeps_base);
    s->sweep_off[0] = 0;
    s->sweep_off[1] = 2 * cols;
    s->sweep_off[2] = 4 * cols;
    s->sweep_off[3] = 4 * cols + 2;
    const std::vector<int>* lists[3] = {&s->sweeps_build, &s->sweeps_jac, &s->sweeps_base};
    s->tw_host = twiddles(n);
    cudaError_t e = cudaMemcpyAsync(s->d_tw, s->tw_host.data(), s->tw_host.size() * sizeof(double2),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d_grid, s->grid.data(), s->ngrid * sizeof(double), cudaMemcpyHostToDevice, st);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(s->d_sweeps + s->sweep_off[k], lists[k]->data(), lists[k]->size() * sizeof(int),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_cancel, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_newton, 0, sizeof(NewtonDev), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host tables may go once copied
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreate(&s->ev[i]);
    if (e != cudaSuccess) return cleanup(PCC_ERR_CUDA, cudaGetErrorString(e));
    // serving runs the batch kernel only, and must not synchronise the device
    if (!alloc_st) ensure_march_tuned(ctx, n, s->stages, s->d_tw, st);
    if (registered) ctx->solves.push_back(s);
    *out = s;
    return PCC_OK;
}

void solve_release(pcc_solve* s)
{
    void* ptrs[] = {s->d_grid, s->d_tw, s->d_in0, s->d_out0, s->d_J, s->d_yinit, s->d_yfinal, s->d_outc,
                    s->d_status, s->d_fail, s->d_cstatus, s->d_counters_i, s->d_counters, s->d_scratch,
                    s->d_item_side, s->d_xs, s->d_its, s->d_newton, s->d_in0old, s->d_rhs, s->d_dx,
                    s->d_ipiv, s->d_info, s->d_luw, s->d_cancel, s->d_sweeps, s->d_sched};
    for (void* p : ptrs)
        if (p) {
            if (s->alloc_stream)
                cudaFreeAsync(p, s->alloc_stream);  // stream-ordered: no device-wide synchronisation
            else
                cudaFree(p);
        }
    for (auto& ev : s->ev)
        if (ev) cudaEventDestroy(ev);
    if (s->build_graph) cudaGraphExecDestroy(s->build_graph);
    delete s;
}

pcc_status newton_reset(pcc_solve* s, const double* in0_host, cudaStream_t st)
{
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0_host, s->nn * sizeof(double), cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, launch_newton_reset(s->d_newton, s->d_in0, s->d_in0old, s->nn, st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_cancel, 0, sizeof(int), st));
    s->h_newton = kNewtonRunning;
    return PCC_OK;
}

pcc_status newton_prologue(pcc_solve* s, cudaStream_t st) { return enqueue_prologue(s, 0, s->nn + 1, st); }

pcc_status newton_tail(pcc_solve* s, pcc_precision prec, cudaStream_t st, int* lu_steps, int* lu_fallback)
{
    return enqueue_newton_tail(s, prec, st, lu_steps, lu_fallback);
}

pcc_status batch_tables_reserve(pcc_ctx* ctx, BatchTables& tab, size_t bytes)
{
    if (tab.d_bytes < bytes) {
        if (tab.d) cudaFree(tab.d);
        tab.d = nullptr;
        tab.d_bytes = 0;
        PCC_CUDA(ctx, cudaMalloc(&tab.d, bytes));
        tab.d_bytes = bytes;
    }
    if (tab.h_bytes < bytes) {
        if (tab.h) cudaFreeHost(tab.h);
        tab.h = nullptr;
        tab.h_bytes = 0;
        PCC_CUDA(ctx, cudaMallocHost(&tab.h, bytes));
        tab.h_bytes = bytes;
    }
    for (auto& ev : tab.ev)
        if (!ev) PCC_CUDA(ctx, cudaEventCreate(&ev));
    return PCC_OK;
}

void batch_tables_free(BatchTables& tab)
{
    if (tab.d) cudaFree(tab.d);
    if (tab.h) cudaFreeHost(tab.h);
    for (auto& ev : tab.ev)
        if (ev) cudaEventDestroy(ev);
    tab = BatchTables{};
}

// Item table: Ntau classes in decreasing order; inside a class the longest
// sweeps first (longest-processing-time order), ties in list order.
pcc_status batch_march_items(pcc_ctx* ctx, BatchTables& tab, const std::vector<BatchItem>& items,
                             cudaStream_t st, int max_ctas)
{
    static const int kOrder[kBatchMaxClasses] = {1024, 512, 256, 128};
    if (items.empty()) return PCC_OK;
    std::vector<pcc_solve*> solves;
    std::vector<int> sidx(items.size());
    for (size_t i = 0; i < items.size(); ++i) {
        pcc_solve* s = items[i].s;
        if (!march_batch_supported(s->d.ntau, s->stages))
            return fail(ctx, PCC_ERR_UNSUPPORTED, "batch: Ntau must be 128..1024 with 2 IRK stages");
        auto it = std::find(solves.begin(), solves.end(), s);
        sidx[i] = (int)(it - solves.begin());
        if (it == solves.end()) solves.push_back(s);
    }
    BatchParams B{};
    std::vector<int2> table;
    table.reserve(items.size());
    B.n_classes = 0;
    for (int n : kOrder) {
        std::vector<std::pair<int, size_t>> cls;  // (steps, index into items)
        for (size_t i = 0; i < items.size(); ++i) {
            const pcc_solve* s = items[i].s;
            if (s->d.ntau == n) cls.push_back({(items[i].item & 1) ? s->d.nr : s->d.nl, i});
        }
        if (cls.empty()) continue;
        // longest sweeps first; among equal lengths the right sides first (the
        // single-solve march's order, measured faster at C3)
        std::stable_sort(cls.begin(), cls.end(), [&](const auto& a, const auto& b) {
            if (a.first != b.first) return a.first > b.first;
            return (items[a.second].item & 1) > (items[b.second].item & 1);
        });
        B.cls_ntau[B.n_classes] = n;
        B.cls_begin[B.n_classes] = (int)table.size();
        // two-ended claiming where the class is at most four waves deep: it
        // shortens one build's last wave by about 2 %, while four builds in
        // one launch (ten waves) ran about 1 % slower with it
        const int spc = n == 128 ? MarchShape<128, 2>::SPC : n == 256 ? MarchShape<256, 2>::SPC
                        : n == 512 ? MarchShape<512, 2>::SPC : MarchShape<1024, 2>::SPC;
        const long long slots = (long long)(max_ctas > 0 ? max_ctas : 2 * ctx->sms) * spc;
        B.cls_ends[B.n_classes] = (long long)cls.size() <= 4 * slots ? 1 : 0;
        for (auto& c : cls) table.push_back(make_int2(sidx[c.second], items[c.second].item));
        B.n_classes += 1;
    }
    B.cls_begin[B.n_classes] = (int)table.size();
    const size_t o_items = align_up(solves.size() * sizeof(BatchSolve), 16);
    const size_t o_cls = align_up(o_items + table.size() * sizeof(int2), 16);
    const size_t o_rank = align_up(o_cls + 3 * kBatchMaxClasses * sizeof(int), 16);
    const size_t o_cnt = align_up(o_rank + (size_t)kBatchMaxClasses * kMarchSchedSms * sizeof(int), 16);
    const size_t bytes = o_cnt + 4 * sizeof(unsigned long long);
    pcc_status r = batch_tables_reserve(ctx, tab, bytes);
    if (r != PCC_OK) return r;
    char* h = static_cast<char*>(tab.h);
    char* d = static_cast<char*>(tab.d);
    auto* hs = reinterpret_cast<BatchSolve*>(h);
    for (size_t i = 0; i < solves.size(); ++i) {
        const pcc_solve* s = solves[i];
        BatchSolve& b = hs[i];
        b.grid = s->d_grid;
        b.twN = s->d_tw;
        b.yinit = s->d_yinit;
        b.yfinal = s->d_yfinal;
        b.status = s->d_status;
        b.fail_index = s->d_fail;
        b.cancel = s->d_cancel;
        b.dim = s->d.dim;
        b.dm2c = s->dm2c;
        b.prec = s->d.prec_irk;
        b.nl = s->d.nl;
        b.nr = s->d.nr;
        b.max_its = s->d.max_irk;
        b.ntau = s->d.ntau;
        b.predictor = s->d.irk_predictor ? 1 : 0;
    }
    std::memcpy(h + o_items, table.data(), table.size() * sizeof(int2));
    std::memset(h + o_cls, 0, bytes - o_cls);
    PCC_CUDA(ctx, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
    B.solves = reinterpret_cast<const BatchSolve*>(d);
    B.items = reinterpret_cast<const int2*>(d + o_items);
    B.cls_counter = reinterpret_cast<int*>(d + o_cls);
    const char* ends = std::getenv("PCC_MARCH_ENDS");  // 0: claim in list order, as march_claim_ends
    B.sm_rank = ends && std::string(ends) == "0" ? nullptr : reinterpret_cast<int*>(d + o_rank);
    B.counters = reinterpret_cast<unsigned long long*>(d + o_cnt);
    tab.cnt_off = o_cnt;
    const pcc_solve* s0 = solves[0];
    for (int i = 0; i < 3; ++i) {
        B.b[i] = s0->b[i];
        B.c[i] = s0->c[i];
        for (int j = 0; j < 3; ++j) B.a[i][j] = s0->a[i][j];
    }
    lagrange_integrals(s0->stages, s0->c, B.lq);
    PCC_CUDA(ctx, cudaEventRecord(tab.ev[0], st));
    PCC_CUDA(ctx, launch_march_batch(B, max_ctas, st, &tab.info));
    PCC_CUDA(ctx, cudaEventRecord(tab.ev[1], st));
    return PCC_OK;
}

}  // namespace pcc

extern "C" {

const char* pcc_status_string(pcc_status s)
{
    const int i = (int)s;
    return (i >= 0 && i < (int)(sizeof(kStatusNames) / sizeof(kStatusNames[0]))) ? kStatusNames[i] : "PCC_UNKNOWN";
}

const char* pcc_last_error(pcc_ctx* ctx)
{
    if (!ctx) return "null context";
    static thread_local std::string copy;  // stable for the calling thread until its next call
    std::lock_guard<std::mutex> lk(ctx->err_mu);
    copy = ctx->last_error;
    return copy.c_str();
}

pcc_status pcc_ctx_create(int device, const pcc_ctx_opts* opts, pcc_ctx** out)
{
    if (!out) return PCC_ERR_INVALID_ARG;
    *out = nullptr;
    if (opts && opts->reserved != 0) return PCC_ERR_INVALID_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return PCC_ERR_CUDA;
    auto* ctx = new pcc_ctx;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return PCC_ERR_CUDA;
    }
    *out = ctx;
    return PCC_OK;
}

pcc_status pcc_ctx_destroy(pcc_ctx* ctx)
{
    if (!ctx) return PCC_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    server_shutdown(ctx);
    while (!ctx->solves.empty()) pcc_solve_destroy(ctx->solves.back());
    if (ctx->lu_work) cudaFree(ctx->lu_work);
    batch_tables_free(ctx->batch);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PCC_OK;
}

pcc_status pcc_solve_create(pcc_ctx* ctx, const pcc_solve_desc* desc, pcc_solve** out)
{
    return solve_create(ctx, desc, nullptr, true, out);
}

int pcc_sweep_plan(int ntau, int shoot_both_sides, int c0, int c1, int* slots, int cap)
{
    if (ntau < 4 || ntau % 4 != 0) return -1;
    const int nn = 3 * ntau / 4;
    if (c0 < 0 || c1 > nn + 1 || c0 >= c1 || cap < 0 || (cap > 0 && !slots)) return -1;
    std::vector<int> v;
    sweep_list_of(nn, shoot_both_sides == 0, c0, c1, v);
    for (int i = 0; i < (int)v.size() && i < cap; ++i) slots[i] = v[i];
    return (int)v.size();
}

pcc_status pcc_solve_destroy(pcc_solve* s)
{
    if (!s) return PCC_ERR_INVALID_ARG;
    auto& v = s->ctx->solves;
    v.erase(std::remove(v.begin(), v.end(), s), v.end());
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    solve_release(s);
    return PCC_OK;
}

pcc_status pcc_solve_grid(pcc_solve* s, double* grid_out)
{
    if (!s || !grid_out) return PCC_ERR_INVALID_ARG;
    std::memcpy(grid_out, s->grid.data(), s->grid.size() * sizeof(double));
    return PCC_OK;
}

pcc_status pcc_jacobian_columns(pcc_solve* s, const double* in0, const double* out0, int c0, int c1, double* cols,
                                pcc_stats* stats)
{
    if (!s || !in0 || !cols) return PCC_ERR_INVALID_ARG;
    if (c0 < 0 || c1 > s->nn + 1 || c0 >= c1) return fail(s->ctx, PCC_ERR_INVALID_ARG, "column range");
    const bool base_only = (c0 == s->nn);
    if (!base_only && !out0) return PCC_ERR_INVALID_ARG;
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (out0) PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, out0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    pcc_status r = enqueue_columns(s, c0, c1, false, nullptr);
    if (r != PCC_OK) return r;
    // columns as differences (or the raw packed output for the base column)
    const int ncols = c1 - c0;
    std::vector<double> outc((size_t)ncols * nn), o0(nn);
    PCC_CUDA(ctx, cudaMemcpyAsync(outc.data(), s->d_outc, outc.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    r = collect(s, c0, c1, stats);
    for (int i = 0; i < ncols; ++i) {
        const int col = c0 + i;
        for (int j = 0; j < nn; ++j) {
            const double v = outc[(size_t)i * nn + j];
            cols[(size_t)i * nn + j] = (col == nn) ? v : (v - out0[j]) / s->d.eps_newton;
        }
    }
    return r;
}

pcc_status pcc_shoot(pcc_solve* s, const double* in0, double* out0, pcc_stats* stats)
{
    if (!s || !in0 || !out0) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    return pcc_jacobian_columns(s, in0, nullptr, s->nn, s->nn + 1, out0, stats);
}

pcc_status pcc_shoot_debug(pcc_solve* s, const double* in0, double* out0, int debug_nx, int max_snaps, int* count,
                           int* grid_idx, double* fields, pcc_stats* stats)
{
    if (!s || !in0 || !out0 || !count || debug_nx < 1 || max_snaps < 0) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    pcc_ctx* ctx = s->ctx;
    const int nl = s->d.nl, nr = s->d.nr, n = s->d.ntau, nn = s->nn;
    // snapshot grid indices in the reference's export order
    std::vector<int> idx;
    for (int i = 0; i < nl; ++i)
        if (i % debug_nx == 0 || i == nl - 1) idx.push_back(i);
    for (int i = nl + nr; i > nl; --i)
        if (i % debug_nx == 0 || i == nl + 1 || i == nl + nr) idx.push_back(i);
    *count = (int)idx.size();
    if ((int)idx.size() > max_snaps || !grid_idx || !fields)
        return fail(ctx, PCC_ERR_INVALID_ARG, "pcc_shoot_debug: max_snaps is below the snapshot count (see *count)");
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int k = (int)idx.size();
    std::vector<int> slot(s->ngrid, -1);
    std::vector<double> xs(k);
    for (int j = 0; j < k; ++j) {
        slot[idx[j]] = j;
        xs[j] = s->grid[idx[j]];
    }
    char* buf = nullptr;
    const size_t bytes = s->ngrid * sizeof(int) + 16 + (size_t)k * n * sizeof(double) * 5 + k * sizeof(double);
    PCC_CUDA(ctx, cudaMalloc(&buf, bytes));
    int* d_slot = reinterpret_cast<int*>(buf);
    double* d_snap = reinterpret_cast<double*>(buf + align_up(s->ngrid * sizeof(int), 16));
    double* d_fields = d_snap + (size_t)k * n;
    double* d_xs = d_fields + (size_t)k * 4 * n;
    auto run = [&]() -> pcc_status {
        PCC_CUDA(ctx, cudaMemcpyAsync(d_slot, slot.data(), s->ngrid * sizeof(int), cudaMemcpyHostToDevice, st));
        PCC_CUDA(ctx, cudaMemcpyAsync(d_xs, xs.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
        PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, nn * sizeof(double), cudaMemcpyHostToDevice, st));
        PCC_CUDA(ctx, cudaEventRecord(s->ev[0], st));
        pcc_status r = enqueue_prologue(s, nn, nn + 1, st);
        if (r != PCC_OK) return r;
        PCC_CUDA(ctx, cudaEventRecord(s->ev[1], st));
        MarchParams P = march_params(s);
        P.snap_slot = d_slot;
        P.snap = d_snap;
        r = enqueue_march(s, nn, nn + 1, P, st);
        if (r != PCC_OK) return r;
        PCC_CUDA(ctx, cudaEventRecord(s->ev[2], st));
        r = enqueue_epilogue(s, nn, nn + 1, false, nullptr, st);
        if (r != PCC_OK) return r;
        PCC_CUDA(ctx, cudaEventRecord(s->ev[3], st));
        if (k > 0)
            PCC_CUDA(ctx, launch_debug_fields(n, s->d.dim, s->dm2c, k, d_snap, d_xs, d_fields, s->d_scratch,
                                              s->scratch_ctas, s->d_tw, st));
        PCC_CUDA(ctx, cudaMemcpyAsync(out0, s->d_outc, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        PCC_CUDA(ctx, cudaMemcpyAsync(fields, d_fields, (size_t)k * 4 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
        return collect(s, nn, nn + 1, stats);
    };
    const pcc_status r = run();
    cudaStreamSynchronize(st);
    cudaFree(buf);
    for (int j = 0; j < k; ++j) grid_idx[j] = idx[j];
    return r;
}

pcc_status pcc_jacobian_device(pcc_solve* s, const double* d_in0, const double* d_out0, double* d_J)
{
    if (!s || !d_in0 || !d_out0 || !d_J) return PCC_ERR_INVALID_ARG;
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn;
    cudaStream_t st = ctx->stream;
    auto enqueue = [&]() -> pcc_status {
        if (d_in0 != s->d_in0)
            PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, d_in0, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (d_out0 != s->d_out0)
            PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, d_out0, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return enqueue_columns(s, 0, nn, true, d_J);
    };
    // The build is captured once per set of pointers into a CUDA graph and
    // replayed: one graph launch for the copies, counter resets, boundary
    // kernels, the persistent march and the differencing.
    const void* key[3] = {d_in0, d_out0, d_J};
    if (!s->build_graph || std::memcmp(key, s->graph_key, sizeof(key)) != 0) {
        if (s->build_graph) cudaGraphExecDestroy(s->build_graph);
        s->build_graph = nullptr;
        cudaGraph_t g = nullptr;
        PCC_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const pcc_status r = enqueue();
        const cudaError_t ec = cudaStreamEndCapture(st, &g);
        if (r != PCC_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (ec != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&s->build_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            s->build_graph = nullptr;
            return fail(ctx, PCC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        std::memcpy(s->graph_key, key, sizeof(key));
    }
    PCC_CUDA(ctx, cudaGraphLaunch(s->build_graph, st));
    s->pend_c0 = 0;
    s->pend_c1 = nn;
    s->pending = true;
    return PCC_OK;
}

pcc_status pcc_jacobian_columns_device(pcc_solve* s, const double* d_in0, const double* d_out0, int c0, int c1,
                                       double* d_cols)
{
    if (!s || !d_in0 || !d_out0 || !d_cols) return PCC_ERR_INVALID_ARG;
    if (c0 < 0 || c1 > s->nn || c0 >= c1) return fail(s->ctx, PCC_ERR_INVALID_ARG, "column range");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn;
    if (d_in0 != s->d_in0)
        PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, d_in0, nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if (d_out0 != s->d_out0)
        PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, d_out0, nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    pcc_status r = enqueue_columns(s, c0, c1, false, nullptr);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, launch_fd_cols(s->d_outc, s->d_out0, d_cols, nn, c1 - c0, s->d.eps_newton, ctx->stream));
    s->pend_c0 = c0;
    s->pend_c1 = c1;
    s->pending = true;
    return PCC_OK;
}

pcc_status pcc_solve_sync(pcc_solve* s, pcc_stats* stats)
{
    if (!s) return PCC_ERR_INVALID_ARG;
    if (!s->pending) {
        cudaStreamSynchronize(s->ctx->stream);
        return PCC_OK;
    }
    s->pending = false;
    return collect(s, s->pend_c0, s->pend_c1, stats);
}

pcc_status pcc_jacobian(pcc_solve* s, const double* in0, const double* out0, double* J, pcc_stats* stats)
{
    if (!s || !in0 || !out0 || !J) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn) || !all_finite(out0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, out0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    pcc_status r = enqueue_columns(s, 0, nn, true, s->d_J);
    if (r != PCC_OK) return r;
    PCC_CUDA(ctx, cudaMemcpyAsync(J, s->d_J, (size_t)nn * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return collect(s, 0, nn, stats);
}

pcc_status pcc_boundary_data(pcc_solve* s, const double* in0, double* y_left, double* y_right)
{
    if (!s || !in0 || !y_left || !y_right) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn, n = s->d.ntau;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_counters_i, 0, 4 * sizeof(int), ctx->stream));
    BoundaryParams B{};
    B.ntau = n;
    B.nn = nn;
    B.c0 = nn;  // base column: no perturbation
    B.dim = s->d.dim;
    B.xl = s->d.xl;
    B.xr = s->d.xr;
    B.eps = s->d.eps_newton;
    B.in0 = s->d_in0;
    B.yinit = s->d_yinit;
    B.scratch = s->d_scratch;
    B.tw = s->d_tw;
    B.n_items = 2;
    B.work_counter = s->d_counters_i;
    PCC_CUDA(ctx, launch_prologue(B, 2, ctx->stream));
    PCC_CUDA(ctx, cudaMemcpyAsync(y_left, s->d_yinit, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PCC_CUDA(ctx, cudaMemcpyAsync(y_right, s->d_yinit + n, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PCC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PCC_OK;
}

pcc_status pcc_sweep(pcc_solve* s, int count, const int* sides, const double* y_init, double* y_final,
                     pcc_stats* stats)
{
    if (!s || count < 1 || !sides || !y_init || !y_final) return PCC_ERR_INVALID_ARG;
    if (count > 2 * (s->nn + 1)) return fail(s->ctx, PCC_ERR_INVALID_ARG, "too many sweeps for this solve");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = s->d.ntau;
    cudaStream_t st = ctx->stream;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_yinit, y_init, (size_t)count * n * sizeof(double), cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_item_side, sides, count * sizeof(int), cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_counters_i, 0, 4 * sizeof(int), st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_counters, 0, 4 * sizeof(unsigned long long), st));
    MarchParams P = march_params(s);
    P.n_items = count;
    P.mode = 0;
    P.yinit = s->d_yinit;
    P.yfinal = s->d_yfinal;
    P.item_side = s->d_item_side;
    P.work_counter = s->d_counters_i;
    PCC_CUDA(ctx, cudaEventRecord(s->ev[1], st));
    PCC_CUDA(ctx, launch_march(n, s->stages, P, 0, st, &s->last_launch));
    PCC_CUDA(ctx, cudaEventRecord(s->ev[2], st));
    PCC_CUDA(ctx, cudaMemcpyAsync(y_final, s->d_yfinal, (size_t)count * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    PCC_CUDA(ctx, cudaStreamSynchronize(st));
    std::vector<int> stv(count), fi(count);
    unsigned long long cnt[4];
    PCC_CUDA(ctx, cudaMemcpy(stv.data(), s->d_status, count * sizeof(int), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(fi.data(), s->d_fail, count * sizeof(int), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(cnt, s->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    pcc_status r = PCC_OK;
    int fcol = -1, fidx = -1, fside = 0;
    for (int i = 0; i < count; ++i)
        if (stv[i]) {
            r = PCC_ERR_IRK_NO_CONVERGENCE;
            fcol = i;
            fside = sides[i];
            fidx = fi[i];
            break;
        }
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, s->ev[1], s->ev[2]);
        std::memset(stats, 0, sizeof(*stats));
        stats->rhs_evals = (long long)cnt[0];
        stats->irk_iterations = (long long)cnt[1];
        stats->irk_steps = (long long)cnt[2];
        stats->ms_sweep = ms;
        stats->ms_total = ms;
        stats->fail_column = fcol;
        stats->fail_side = fside;
        stats->fail_grid_index = fidx;
        stats->sweep_ctas = s->last_launch.ctas;
    }
    return r;
}

// ODEStepper-level entry points: a temporary solve-less march launch.
static pcc_status single_states(pcc_ctx* ctx, int ntau, double dim, int scheme, double precision, int max_its,
                                int count, const double* y, const double* x_in, const double* x_out, double* y_out,
                                int* its_out, int mode)
{
    if (!ctx || count < 1 || !y || !x_in || !y_out || !march_supported(ntau, scheme)) return PCC_ERR_INVALID_ARG;
    if (mode == 2 && !x_out) return PCC_ERR_INVALID_ARG;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    double *d_y = nullptr, *d_o = nullptr, *d_x = nullptr;
    double2* d_tw = nullptr;
    int *d_i = nullptr;
    unsigned long long* d_c = nullptr;
    const size_t yb = (size_t)count * ntau * sizeof(double);
    auto release = [&]() {
        cudaFree(d_y);
        cudaFree(d_o);
        cudaFree(d_x);
        cudaFree(d_tw);
        cudaFree(d_i);
        cudaFree(d_c);
    };
    if (cudaMalloc(&d_y, yb) != cudaSuccess || cudaMalloc(&d_o, yb) != cudaSuccess ||
        cudaMalloc(&d_x, 2 * count * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&d_tw, twiddle_count(ntau) * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&d_i, (3 * count + 4) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_c, 4 * sizeof(unsigned long long)) != cudaSuccess) {
        release();
        return fail(ctx, PCC_ERR_OOM, "allocation for the state batch");
    }
    const std::vector<double2> tw = twiddles(ntau);
    std::vector<double> xs(2 * count);
    for (int i = 0; i < count; ++i) {
        xs[i] = x_in[i];
        xs[count + i] = x_out ? x_out[i] : 0.0;
    }
    cudaError_t e = cudaMemcpy(d_y, y, yb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_x, xs.data(), 2 * count * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_i, 0, (3 * count + 4) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_c, 0, 4 * sizeof(unsigned long long));
    MarchParams P{};
    double a[3][3], b[3], c[3];
    const int S = tableau(scheme, a, b, c);
    P.n_items = count;
    P.mode = mode;
    P.yinit = d_y;
    P.yfinal = d_o;
    P.dim = dim;
    P.dim_m2_cubed = std::pow(dim - 2.0, 3);
    P.prec = precision;
    P.max_its = max_its;
    P.stages = S;
    for (int i = 0; i < 3; ++i) {
        P.b[i] = b[i];
        P.c[i] = c[i];
        for (int j = 0; j < 3; ++j) P.a[i][j] = a[i][j];
    }
    P.twN = d_tw;
    P.x_in = d_x;
    P.x_out = d_x + count;
    P.work_counter = d_i + 3 * count;
    P.status = d_i;
    P.fail_index = d_i + count;
    P.its_out = d_i + 2 * count;
    P.counters = d_c;
    if (e == cudaSuccess) e = launch_march(ntau, S, P, 0, st, nullptr);
    if (e == cudaSuccess) e = cudaMemcpyAsync(y_out, d_o, yb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && its_out) e = cudaMemcpyAsync(its_out, d_i + 2 * count, count * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    release();
    if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
    return PCC_OK;
}

pcc_status pcc_rhs_eval(pcc_ctx* ctx, int ntau, double dim, int count, const double* y, const double* x, double* dy)
{
    return single_states(ctx, ntau, dim, 2, 1e-15, 1, count, y, x, nullptr, dy, nullptr, 1);
}

pcc_status pcc_irk_step(pcc_ctx* ctx, int ntau, double dim, int scheme, double precision, int max_its, int count,
                        const double* y_in, const double* x_in, const double* x_out, double* y_out, int* its_out)
{
    if (max_its < 1) return PCC_ERR_INVALID_ARG;
    return single_states(ctx, ntau, dim, scheme, precision, max_its, count, y_in, x_in, x_out, y_out, its_out, 2);
}

pcc_status pcc_lu_solve(pcc_ctx* ctx, int n, const double* A, const double* rhs, double* x, pcc_precision prec,
                        pcc_refine_report* report)
{
    if (!ctx || n < 1 || !A || !rhs || !x) return PCC_ERR_INVALID_ARG;
    if (prec != PCC_PREC_FP64 && prec != PCC_PREC_MIXED) return PCC_ERR_INVALID_ARG;
    if (n > lu_max_order()) return fail(ctx, PCC_ERR_INVALID_ARG, "pcc_lu_solve: n above " + std::to_string(lu_max_order()));
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t nb = (size_t)n * n * sizeof(double);
    const size_t need = nb + 3 * n * sizeof(double) + 2 * n * sizeof(int) + 16 + lu_mixed_work_bytes(n);
    if (ctx->lu_work_bytes < need) {
        if (ctx->lu_work) cudaFree(ctx->lu_work);
        ctx->lu_work = nullptr;
        ctx->lu_work_bytes = 0;
        PCC_CUDA(ctx, cudaMalloc(&ctx->lu_work, need));
        ctx->lu_work_bytes = need;
    }
    char* w = static_cast<char*>(ctx->lu_work);
    double* dA = reinterpret_cast<double*>(w);
    double* db = dA + (size_t)n * n;
    double* dx = db + n;
    double* dtmp = dx + n;
    int* ipiv = reinterpret_cast<int*>(dtmp + n);
    int* info = ipiv + n;
    void* mixed_work = reinterpret_cast<char*>(info + n) + 16;
    cudaEvent_t e0, e1;
    PCC_CUDA(ctx, cudaEventCreate(&e0));
    PCC_CUDA(ctx, cudaEventCreate(&e1));
    PCC_CUDA(ctx, cudaMemcpyAsync(dA, A, nb, cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, cudaMemcpyAsync(db, rhs, n * sizeof(double), cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, cudaEventRecord(e0, st));
    int steps = 0;
    double resid = -1.0;
    if (prec == PCC_PREC_FP64) {
        PCC_CUDA(ctx, lu_solve_fp64(dA, db, dx, n, dtmp, ipiv, info, st));
    } else {
        PCC_CUDA(ctx, lu_solve_mixed(dA, db, dx, n, mixed_work, lu_mixed_work_bytes(n), ipiv, info, 30, 1e-15,
                                     &steps, &resid, st));
    }
    PCC_CUDA(ctx, cudaEventRecord(e1, st));
    int hinfo[2] = {0, 0};
    PCC_CUDA(ctx, cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    PCC_CUDA(ctx, cudaMemcpyAsync(hinfo, info, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PCC_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (report) {
        report->rel_err_vs_fp64 = -1.0;
        report->residual_norm = resid;
        report->refinement_steps = steps;
        report->fell_back_to_fp64 = hinfo[1];
        report->ms = ms;
    }
    if (hinfo[0] != 0) return fail(ctx, PCC_ERR_LU_SINGULAR, "zero pivot in LU");
    return PCC_OK;
}

pcc_status pcc_newton_step(pcc_solve* s, double* in0, double* err_out, pcc_precision prec, pcc_stats* stats,
                           pcc_refine_report* report)
{
    if (!s || !in0) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = s->nn;
    // base shoot and all Jacobian columns in one pipeline (columns 0..nn)
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    pcc_status r = enqueue_columns(s, 0, nn + 1, false, nullptr);
    if (r != PCC_OK) return r;
    // out0 = base column output, then J
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, s->d_outc + (size_t)nn * nn, nn * sizeof(double),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
    PCC_CUDA(ctx, launch_fd(s->d_outc, s->d_out0, s->d_J, nn, 0, nn, s->d.eps_newton, ctx->stream));
    r = collect(s, 0, nn + 1, stats);
    if (r != PCC_OK) return r;
    std::vector<double> out0(nn), J((size_t)nn * nn), rhs(nn), dx(nn);
    PCC_CUDA(ctx, cudaMemcpy(out0.data(), s->d_out0, nn * sizeof(double), cudaMemcpyDeviceToHost));
    PCC_CUDA(ctx, cudaMemcpy(J.data(), s->d_J, J.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double ss = 0.0;
    for (int i = 0; i < nn; ++i) ss += out0[i] * out0[i];
    const double err = std::sqrt(ss / (double)nn);  // computeL2Norm (NewtonSolver.cpp:763-768)
    if (err_out) *err_out = err;
    for (int i = 0; i < nn; ++i) rhs[i] = -out0[i];
    r = pcc_lu_solve(ctx, nn, J.data(), rhs.data(), dx.data(), prec, report);
    if (r != PCC_OK) return r;
    const double fac = std::min(1.0, s->d.slow_error / err);  // NewtonSolver.cpp:350
    for (int i = 0; i < nn; ++i) in0[i] += fac * dx[i];       // :358
    return PCC_OK;
}

static pcc_status pack_common(pcc_ctx* ctx, int ntau, double* up, double* psic, double* fc, double* z, int dir)
{
    if (!ctx || !up || !psic || !fc || !z) return PCC_ERR_INVALID_ARG;
    if (!march_supported(ntau, 2)) return fail(ctx, PCC_ERR_INVALID_ARG, "Ntau must be 128..2048, power of two");
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int nn = 3 * ntau / 4;
    cudaStream_t st = ctx->stream;
    double* d = nullptr;
    const size_t fields = 3 * (size_t)ntau, scr = (size_t)kBoundaryArrays * ntau;
    const size_t total = fields + nn + scr + 2 * (size_t)ntau;
    PCC_CUDA(ctx, cudaMalloc(&d, total * sizeof(double)));
    double *dup = d, *dps = d + ntau, *dfc = d + 2 * ntau, *dz = d + fields, *dscr = dz + nn;
    double2* dtw = reinterpret_cast<double2*>(dscr + scr);
    const std::vector<double2> tw = twiddles(ntau);
    cudaError_t e = cudaMemcpyAsync(dtw, tw.data(), ntau * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && dir == 0) {
        e = cudaMemcpyAsync(dup, up, ntau * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dps, psic, ntau * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dfc, fc, ntau * sizeof(double), cudaMemcpyHostToDevice, st);
    } else if (e == cudaSuccess) {
        e = cudaMemcpyAsync(dz, z, nn * sizeof(double), cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = launch_pack(ntau, dtw, dscr, dup, dps, dfc, dz, dir, st);
    if (e == cudaSuccess && dir == 0) {
        e = cudaMemcpyAsync(z, dz, nn * sizeof(double), cudaMemcpyDeviceToHost, st);
    } else if (e == cudaSuccess) {
        e = cudaMemcpyAsync(up, dup, ntau * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(psic, dps, ntau * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(fc, dfc, ntau * sizeof(double), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
    return PCC_OK;
}

pcc_status pcc_pack_fields(pcc_ctx* ctx, int ntau, const double* up, const double* psic, const double* fc, double* z)
{
    return pack_common(ctx, ntau, const_cast<double*>(up), const_cast<double*>(psic), const_cast<double*>(fc), z, 0);
}

pcc_status pcc_unpack_fields(pcc_ctx* ctx, int ntau, const double* z, double* up, double* psic, double* fc)
{
    return pack_common(ctx, ntau, up, psic, fc, const_cast<double*>(z), 1);
}

pcc_status pcc_expansions(pcc_ctx* ctx, int ntau, double dim, double delta, double x_l, double x_r,
                          const double* fc, const double* psic, const double* up, double* y_left, double* y_right)
{
    if (!ctx || (!y_left && !y_right) || (y_left && (!fc || !psic)) || (y_right && !up)) return PCC_ERR_INVALID_ARG;
    if (!march_supported(ntau, 2)) return fail(ctx, PCC_ERR_INVALID_ARG, "Ntau must be 128..2048, power of two");
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t n = ntau, scr = 2 * (size_t)kBoundaryArrays * n;
    double* d = nullptr;
    PCC_CUDA(ctx, cudaMalloc(&d, (5 * n + scr + 2 * n) * sizeof(double)));
    double *dfc = d, *dps = d + n, *dup = d + 2 * n, *dyl = d + 3 * n, *dyr = d + 4 * n, *dscr = d + 5 * n;
    double2* dtw = reinterpret_cast<double2*>(dscr + scr);
    const std::vector<double2> tw = twiddles(ntau);
    cudaError_t e = cudaMemcpyAsync(dtw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && y_left) e = cudaMemcpyAsync(dfc, fc, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && y_left) e = cudaMemcpyAsync(dps, psic, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && y_right) e = cudaMemcpyAsync(dup, up, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_expansions(ntau, dim, delta, x_l, x_r, dtw, dscr, dfc, dps, dup, y_left ? dyl : nullptr,
                              y_right ? dyr : nullptr, st);
    if (e == cudaSuccess && y_left) e = cudaMemcpyAsync(y_left, dyl, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && y_right) e = cudaMemcpyAsync(y_right, dyr, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
    return PCC_OK;
}

pcc_status pcc_solve_set_grid(pcc_solve* s, const double* grid)
{
    if (!s || !grid) return PCC_ERR_INVALID_ARG;
    for (int i = 1; i < s->ngrid; ++i)
        if (!(grid[i] > grid[i - 1])) return fail(s->ctx, PCC_ERR_INVALID_ARG, "grid must increase strictly");
    PCC_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
    s->grid.assign(grid, grid + s->ngrid);
    PCC_CUDA(s->ctx, cudaMemcpyAsync(s->d_grid, s->grid.data(), s->ngrid * sizeof(double), cudaMemcpyHostToDevice,
                                     s->ctx->stream));
    PCC_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return PCC_OK;
}

pcc_status pcc_dft(pcc_ctx* ctx, int n, int count, int sign, const double* in, double* out)
{
    if (!ctx || !in || !out || count < 1 || n < 2 || n > 4096 || (n & (n - 1)) || (sign != 1 && sign != -1))
        return PCC_ERR_INVALID_ARG;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t bytes = (size_t)count * n * sizeof(double2);
    double2* d = nullptr;
    PCC_CUDA(ctx, cudaMalloc(&d, 2 * bytes + n * sizeof(double2)));
    double2* dtw = d + 2 * (size_t)count * n;
    const std::vector<double2> tw = twiddles(n);
    cudaError_t e = cudaMemcpyAsync(dtw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_dft(n, count, sign, dtw, d, d + (size_t)count * n, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + (size_t)count * n, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
    return PCC_OK;
}

pcc_status pcc_resample_fields(pcc_ctx* ctx, int ntau_in, int ntau_out, int count, const double* in, double* out)
{
    if (!ctx || !in || !out || count < 1) return PCC_ERR_INVALID_ARG;
    auto pow2 = [](int n) { return n >= 4 && (n & (n - 1)) == 0; };
    if (!pow2(ntau_in) || !pow2(ntau_out) || ntau_out < ntau_in || ntau_out > 4096)
        return fail(ctx, PCC_ERR_INVALID_ARG, "resample: powers of two with 4 <= Ntau_in <= Ntau_out <= 4096");
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t m = (size_t)count * ntau_out;
    std::vector<double2> tws;
    std::vector<size_t> tw_off;
    for (int n = ntau_in; n <= ntau_out; n *= 2) {
        tw_off.push_back(tws.size());
        const std::vector<double2> t = twiddles(n);
        tws.insert(tws.end(), t.begin(), t.end());
    }
    char* buf = nullptr;
    const size_t bytes = 2 * m * sizeof(double2) + 2 * m * sizeof(double) + tws.size() * sizeof(double2);
    PCC_CUDA(ctx, cudaMalloc(&buf, bytes));
    double2* w0 = reinterpret_cast<double2*>(buf);
    double2* w1 = w0 + m;
    double* x0 = reinterpret_cast<double*>(w1 + m);
    double* x1 = x0 + m;
    double2* dtw = reinterpret_cast<double2*>(x1 + m);
    cudaError_t e = cudaMemcpyAsync(dtw, tws.data(), tws.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x0, in, (size_t)count * ntau_in * sizeof(double), cudaMemcpyHostToDevice, st);
    double* cur = x0;
    double* nxt = x1;
    for (int n = ntau_in, k = 0; n < ntau_out && e == cudaSuccess; n *= 2, ++k) {
        e = launch_double_fields(n, count, cur, nxt, dtw + tw_off[k], dtw + tw_off[k + 1], w0, w1, st);
        std::swap(cur, nxt);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, cur, m * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
    return PCC_OK;
}

pcc_status pcc_march_tuning(pcc_ctx* ctx, int ntau, int stages, int* pair, double* ms_pair, double* ms_single)
{
    if (!ctx || !pair) return PCC_ERR_INVALID_ARG;
    if (!march_supported(ntau, stages)) return fail(ctx, PCC_ERR_INVALID_ARG, "Ntau 128..2048, 1..3 stages");
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    MarchTuning t{};
    if (!march_tuning(ctx->device, ntau, stages, &t)) {
        double2* d_tw = nullptr;
        const std::vector<double2> tw = twiddles(ntau);
        PCC_CUDA(ctx, cudaMalloc(&d_tw, tw.size() * sizeof(double2)));
        cudaError_t e = cudaMemcpy(d_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) ensure_march_tuned(ctx, ntau, stages, d_tw, ctx->stream);
        cudaFree(d_tw);
        if (e != cudaSuccess) return fail(ctx, PCC_ERR_CUDA, cudaGetErrorString(e));
        if (!march_tuning(ctx->device, ntau, stages, &t)) t = MarchTuning{1, 0.0, 0.0, 0.0};  // tuning disabled
    }
    *pair = t.pair;
    if (ms_pair) *ms_pair = t.ms_pair;
    if (ms_single) *ms_single = t.ms_single;
    return PCC_OK;
}

pcc_status pcc_fp64_peak(pcc_ctx* ctx, double* tflops)
{
    if (!ctx || !tflops) return PCC_ERR_INVALID_ARG;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    PCC_CUDA(ctx, fp64_peak_probe(tflops, ctx->stream));
    return PCC_OK;
}

// ------------------------------------------------ batches and device Newton

pcc_status pcc_jacobian_batch(pcc_ctx* ctx, int count, pcc_solve* const* solves, const double* const* in0,
                              const double* const* out0, double* const* J, pcc_stats* stats)
{
    if (!ctx || count < 1 || !solves || !in0 || !out0 || !J) return PCC_ERR_INVALID_ARG;
    std::vector<pcc_solve*> v(solves, solves + count);
    for (int i = 0; i < count; ++i) {
        if (!v[i] || v[i]->ctx != ctx || !in0[i] || !out0[i] || !J[i]) return PCC_ERR_INVALID_ARG;
        if (!all_finite(in0[i], v[i]->nn) || !all_finite(out0[i], v[i]->nn)) return fail(ctx, PCC_ERR_NAN, "non-finite value in the free data");
        if (!march_batch_supported(v[i]->d.ntau, v[i]->stages))
            return fail(ctx, PCC_ERR_UNSUPPORTED, "batch: Ntau must be 128..1024 with 2 IRK stages");
        for (int j = 0; j < i; ++j)
            if (v[j] == v[i]) return fail(ctx, PCC_ERR_INVALID_ARG, "batch: a solve is listed twice");
    }
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<int> ncols(count);
    for (int i = 0; i < count; ++i) {
        pcc_solve* s = v[i];
        ncols[i] = s->nn;
        PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0[i], s->nn * sizeof(double), cudaMemcpyHostToDevice, st));
        PCC_CUDA(ctx, cudaMemcpyAsync(s->d_out0, out0[i], s->nn * sizeof(double), cudaMemcpyHostToDevice, st));
        pcc_status r = enqueue_prologue(s, 0, s->nn, st);
        if (r != PCC_OK) return r;
    }
    pcc_status r = enqueue_batch_march(ctx, v, ncols, st);
    if (r != PCC_OK) return r;
    for (int i = 0; i < count; ++i) {
        pcc_solve* s = v[i];
        r = enqueue_epilogue(s, 0, s->nn, true, s->d_J, st);
        if (r != PCC_OK) return r;
        PCC_CUDA(ctx, cudaMemcpyAsync(J[i], s->d_J, (size_t)s->nn * s->nn * sizeof(double), cudaMemcpyDeviceToHost,
                                      st));
    }
    PCC_CUDA(ctx, cudaStreamSynchronize(st));
    batch_stats(ctx, ncols, stats);
    for (int i = 0; i < count; ++i) {
        int col, side, idx;
        solve_failure(v[i], ncols[i], &col, &side, &idx);
        if (col >= 0) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "batch solve %d: %s at column %d side %d grid index %d", i,
                          side >= 0 ? "IRK no convergence" : "Delta mismatch", col, side, idx);
            if (stats) {
                stats->fail_column = col;
                stats->fail_side = side < 0 ? 0 : side;
                stats->fail_grid_index = idx;
            }
            return fail(ctx, side >= 0 ? PCC_ERR_IRK_NO_CONVERGENCE : PCC_ERR_DELTA_MISMATCH, buf);
        }
    }
    return PCC_OK;
}

pcc_status pcc_newton_begin(pcc_solve* s, const double* in0)
{
    if (!s || !in0) return PCC_ERR_INVALID_ARG;
    if (!all_finite(in0, s->nn)) return fail(s->ctx, PCC_ERR_NAN, "non-finite value in the free data");
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    PCC_CUDA(ctx, cudaMemcpyAsync(s->d_in0, in0, s->nn * sizeof(double), cudaMemcpyHostToDevice, st));
    PCC_CUDA(ctx, launch_newton_reset(s->d_newton, s->d_in0, s->d_in0old, s->nn, st));
    PCC_CUDA(ctx, cudaMemsetAsync(s->d_cancel, 0, sizeof(int), st));
    PCC_CUDA(ctx, cudaStreamSynchronize(st));
    s->h_newton = kNewtonRunning;
    return PCC_OK;
}

pcc_status pcc_newton_iterate(pcc_ctx* ctx, int count, pcc_solve* const* solves, pcc_precision prec,
                              pcc_newton_state* states, pcc_stats* stats)
{
    if (!ctx || count < 1 || !solves) return PCC_ERR_INVALID_ARG;
    if (prec != PCC_PREC_FP64 && prec != PCC_PREC_MIXED) return PCC_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        if (!solves[i] || solves[i]->ctx != ctx) return PCC_ERR_INVALID_ARG;
        for (int j = 0; j < i; ++j)
            if (solves[j] == solves[i]) return fail(ctx, PCC_ERR_INVALID_ARG, "a solve is listed twice");
    }
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<pcc_solve*> run, batch, single;
    for (int i = 0; i < count; ++i)
        if (solves[i]->h_newton == kNewtonRunning) {
            run.push_back(solves[i]);
            (march_batch_supported(solves[i]->d.ntau, solves[i]->stages) ? batch : single).push_back(solves[i]);
        }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<int> steps(count, -1), fb(count, 0);
    if (!run.empty()) {
        for (pcc_solve* s : run) {
            pcc_status r = enqueue_prologue(s, 0, s->nn + 1, st);
            if (r != PCC_OK) return r;
        }
        if (!batch.empty()) {
            std::vector<int> ncols;
            for (pcc_solve* s : batch) ncols.push_back(s->nn + 1);
            pcc_status r = enqueue_batch_march(ctx, batch, ncols, st);
            if (r != PCC_OK) return r;
        }
        for (pcc_solve* s : single) {
            MarchParams P = march_params(s);
            pcc_status r = enqueue_march(s, 0, s->nn + 1, P, st);
            if (r != PCC_OK) return r;
        }
        for (int i = 0; i < count; ++i) {
            pcc_solve* s = solves[i];
            if (s->h_newton != kNewtonRunning) continue;
            pcc_status r = enqueue_newton_tail(s, prec, st, &steps[i], &fb[i]);
            if (r != PCC_OK) return r;
        }
        PCC_CUDA(ctx, cudaStreamSynchronize(st));
        if (stats && !batch.empty()) {
            std::vector<int> ncols;
            for (pcc_solve* s : batch) ncols.push_back(s->nn + 1);
            batch_stats(ctx, ncols, stats);
        }
        if (stats) {
            for (pcc_solve* s : single) {
                unsigned long long cnt[4];
                PCC_CUDA(ctx, cudaMemcpy(cnt, s->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
                stats->rhs_evals += (long long)cnt[0];
                stats->irk_iterations += (long long)cnt[1];
                stats->irk_steps += (long long)cnt[2];
                stats->shoots += s->nn + 1;
            }
        }
    }
    for (int i = 0; i < count; ++i) {
        pcc_solve* s = solves[i];
        NewtonDev nd{};
        PCC_CUDA(ctx, cudaMemcpy(&nd, s->d_newton, sizeof(nd), cudaMemcpyDeviceToHost));
        s->h_newton = nd.state;
        if (states) {
            newton_state_from_dev(nd, &states[i]);
            states[i].lu_refinement_steps = steps[i];
            int info[2] = {0, 0};
            PCC_CUDA(ctx, cudaMemcpy(info, s->d_info, sizeof(info), cudaMemcpyDeviceToHost));
            states[i].lu_fell_back = prec == PCC_PREC_MIXED ? info[1] : 0;
            if (nd.state == kNewtonIrkFailed || nd.state == kNewtonDeltaMismatch)
                solve_failure(s, s->nn + 1, &states[i].fail_column, &states[i].fail_side,
                              &states[i].fail_grid_index);
        }
    }
    return PCC_OK;
}

pcc_status pcc_newton_result(pcc_solve* s, double* in0_out, pcc_newton_state* state)
{
    if (!s || !in0_out) return PCC_ERR_INVALID_ARG;
    pcc_ctx* ctx = s->ctx;
    PCC_CUDA(ctx, cudaSetDevice(ctx->device));
    PCC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    NewtonDev nd{};
    PCC_CUDA(ctx, cudaMemcpy(&nd, s->d_newton, sizeof(nd), cudaMemcpyDeviceToHost));
    // a solve stopped by the divergence safeguard returns its last improving iterate (NewtonSolver.cpp:317-321)
    const double* src = nd.state == kNewtonStopped ? s->d_in0old : s->d_in0;
    PCC_CUDA(ctx, cudaMemcpy(in0_out, src, s->nn * sizeof(double), cudaMemcpyDeviceToHost));
    if (state) newton_state_from_dev(nd, state);
    return PCC_OK;
}

pcc_status pcc_newton_solve(pcc_ctx* ctx, int count, pcc_solve* const* solves, double* const* in0,
                            pcc_precision prec, pcc_newton_state* states, pcc_stats* stats)
{
    if (!ctx || count < 1 || !solves || !in0) return PCC_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        if (!solves[i] || !in0[i]) return PCC_ERR_INVALID_ARG;
        pcc_status r = pcc_newton_begin(solves[i], in0[i]);
        if (r != PCC_OK) return r;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    std::vector<pcc_newton_state> cur(count);
    for (;;) {
        bool any = false;
        for (int i = 0; i < count; ++i) any = any || solves[i]->h_newton == kNewtonRunning;
        if (!any) break;
        pcc_stats it{};
        pcc_status r = pcc_newton_iterate(ctx, count, solves, prec, cur.data(), &it);
        if (r != PCC_OK) return r;
        if (stats) {
            stats->rhs_evals += it.rhs_evals;
            stats->irk_iterations += it.irk_iterations;
            stats->irk_steps += it.irk_steps;
            stats->shoots += it.shoots;
            stats->ms_sweep += it.ms_sweep;
            stats->ms_total += it.ms_total;
            stats->sweep_ctas = it.sweep_ctas;
        }
        if (states)
            for (int i = 0; i < count; ++i) states[i] = cur[i];
    }
    for (int i = 0; i < count; ++i) {
        pcc_newton_state fin{};
        pcc_status r = pcc_newton_result(solves[i], in0[i], &fin);
        if (r != PCC_OK) return r;
        if (states) {
            fin.fail_column = cur[i].fail_column;
            fin.fail_side = cur[i].fail_side;
            fin.fail_grid_index = cur[i].fail_grid_index;
            fin.lu_refinement_steps = cur[i].lu_refinement_steps;
            fin.lu_fell_back = cur[i].lu_fell_back;
            states[i] = fin;
        }
    }
    return PCC_OK;
}

}  // extern "C"
