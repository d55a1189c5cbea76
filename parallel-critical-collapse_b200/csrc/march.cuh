// march.cuh -- the hot path: persistent FP64 Gauss-Legendre IRK march of the
// shooting sweeps (ShootingSolver::integrateToMatchPoint, ShootingSolver.cpp:
// 53-145; ODEStepper::stepIRK, ODEStepper.cpp:163-292; ODEStepper::
// computeDerivatives, ODEStepper.cpp:92-136; InitialConditionGenerator::
// StateVectorToFields/FieldsToStateVector, InitialConditionGenerator.cpp:
// 766-884; SpectralTransformer::solveInhom, SpectralTransformer.cpp:264-292).
//
// Work unit ("sweep"): one (Jacobian column, side) pair, marched over all grid
// steps of that side by S stage groups of TG = Ntau/16 threads (one group per
// IRK stage).  Persistent sweep slots pull sweeps from an atomic counter.
//
// Half-length spectral formulation.  The reference evaluates each RHS with
// seven complex FFTs of length N = Ntau on the band-limited state Y (N/2
// modes, |m| <= N/4).  U and V are anti-periodic over half an echoing period
// (odd Fourier modes only) and F, IA2 are periodic over half a period (even
// modes only), so with M = N/2 and w = exp(-2 pi i/N):
//   U_j + i V_j = w^j   * IDFT_M(c_odd)_j        (c_odd[k'] = c[2k'+1])
//   F_j         = Im IDFT_M(c_even)_j            (c_even[k'] = c[2k'])
//   dU, dV      = the same with c -> -i m k0 c
//   solveInhom  : four length-M transforms of real half-period data
//   Y'[odd 2k'+1] = DFT_M((dUdx + i dVdx) w^-j)/M, Y'[even 2k'] = DFT_M(i dFdx)/M
// for j < M, which equals the reference's split
//   U = (Re Z_j - Re Z_{j+M})/2, F = (Im Z_j + Im Z_{j+M})/2, ...
// (InitialConditionGenerator.cpp:849-874) exactly in real arithmetic.  The
// quirks of the reference are kept: doubleModes stores the full Y[N/4] at
// index 3N/4 and half of it at N/4 (SpectralTransformer.cpp:238-245), the
// phase fix Re c[2] = -Re c[N-2] (InitialConditionGenerator.cpp:800), and the
// frozen Delta slot Re dY[2] = 0 (ODEStepper.cpp:128).
//
// Data layout per thread t of a stage group: DFT position p_q = t + TG q,
// q = 0..7, serves both as physical point j and as spectral index k'.  The
// state modes a thread owns are exactly those its positions q in {0,1,6,7}
// produce ("slots": sigma = 2*ri + parity, ri -> q in {0,1,6,7}), so every
// state array is slot-indexed [sigma][t] and the IRK update touches only the
// thread's own entries.  Shared memory per sweep: y, the stage values yk, and
// two exchange buffers per stage; the stage RHS f is written into the
// exchange buffer that the next transform writes first, which is idle from
// the end of one RHS evaluation to the start of the next.
#pragma once
#include "pcc_device.cuh"

namespace pcc {

struct MarchParams {
    int n_items;
    int mode;                       // 0 march, 1 single RHS evaluation, 2 single IRK step
    const double* __restrict__ yinit;  // [item][N], interleaved modes
    double* __restrict__ yfinal;       // [item][N]
    const int* __restrict__ item_side; // optional, else side = item & 1
    const int* __restrict__ item_map;  // optional (mode 0): work index -> item (slot 2 column + side)
    int* sched;  // optional (with item_map): kMarchSchedWords zeroed words, see march_claim_ends
    const double* __restrict__ grid;   // nl + nr + 1
    int nl, nr;
    double dim;
    double dim_m2_cubed;  // std::pow(Dim - 2.0, 3) as computed by the host
    double prec;
    int max_its;
    int stages;
    double a[3][3], b[3], c[3];
    int predictor;                     // 1: stage iteration starts from the extrapolated collocation polynomial
    double lq[3][3];                   // int_0^theta l_j = sum_k lq[j][k] theta^(k+1) (Lagrange basis on c)
    const double2* __restrict__ twN;   // exp(+2 pi i k/N), k < N, then the pass tables (march_twiddle_count)
    const double* __restrict__ x_in;   // [item] (modes 1 and 2)
    const double* __restrict__ x_out;  // [item] (mode 2)
    int* work_counter;
    int* status;       // [item]: 0 ok, 1 IRK no convergence
    int* fail_index;   // [item]: grid index the failing step started from
    int* its_out;      // [item] (mode 2), may be null
    unsigned long long* counters;  // [0] RHS evaluations [1] IRK iterations [2] steps
    const int* snap_slot;          // optional, per grid index: snapshot slot of the state there, or -1
    double* snap;                  // [slot][N] states at the start of the steps snap_slot marks
};

// Transform schedules: 0 single transforms, 1 paired (dft_m2), 2 paired with
// the warp-exchange length-512 transforms (Ntau = 1024 only; other sizes
// treat 2 as 1).
template <int N, int S, int PAIR = 1>
struct MarchShape {
    static constexpr int M = N / 2;
    static constexpr int Q = N / 4;
    static constexpr int TG = M / 8;        // threads per stage group
    static constexpr int ST = S * TG;       // working threads per sweep
    // padded sweep width: power of two below a warp, else a multiple of 32
    static constexpr int STP = ST <= 8 ? 8 : ST <= 16 ? 16 : ST <= 32 ? 32 : ((ST + 31) / 32) * 32;
    static constexpr int SPC = STP >= 128 ? 1 : 128 / STP;  // sweeps per CTA
    static constexpr int NT = SPC * STP;                      // threads per CTA
    static constexpr int NW = STP >= 32 ? STP / 32 : 1;       // warps per sweep
    static constexpr int MP = M;                              // exchange length (swizzled)
    static constexpr int EXA = S * 2 * MP;                    // exchange pairs of the first transform
    static constexpr int YS = 8 * TG;                         // slot-indexed y
    static constexpr int YK = S * 8 * TG;                     // slot-indexed stage values
    static constexpr int UV = S * M;                          // U and V per stage (doubles -> M double2)
    static constexpr int MISC = (S + NW + 1) / 2 + 2;          // lam, red, item, zero (in double2)
    // paired transforms (dft_m2) need a second set of exchange pairs; shapes
    // whose shared memory would not fit keep single transforms, and PAIR =
    // false (a variant the autotuner may pick) never pairs
    static constexpr bool DUAL = PAIR != 0 && (size_t)SPC * (2 * EXA + YS + YK + UV + MISC) * 16 <= 200 * 1024;
    static constexpr bool WX = PAIR == 2 && DUAL && M == 512 && S * TG == STP;  // warp-exchange transforms
    static constexpr int EX = DUAL ? 2 * EXA : EXA;           // exchange double2s
    static constexpr int PER_SWEEP = EX + YS + YK + UV + MISC; // double2 per sweep
    static constexpr size_t SMEM = (size_t)SPC * PER_SWEEP * sizeof(double2);
    static constexpr int NP = M == 64 ? 2 : (M <= 512 ? 3 : 4);
    static constexpr int R_LAST = M == 64 ? 8 : M == 128 ? 2 : M == 256 ? 4 : M == 512 ? 8 : 2;
};

// ---------------------------------------------------------------- DFT kernels
template <int SG>
__device__ __forceinline__ void dft2(double2& a0, double2& a1)
{
    const double2 t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <int SG>
__device__ __forceinline__ void dft4(double2& b0, double2& b1, double2& b2, double2& b3)
{
    const double2 t0 = cadd(b0, b2), t1 = csub(b0, b2);
    const double2 t2 = cadd(b1, b3), t3 = cmul_si<SG>(csub(b1, b3));
    b0 = cadd(t0, t2);
    b2 = csub(t0, t2);
    b1 = cadd(t1, t3);
    b3 = csub(t1, t3);
}

// X_k = sum_r a_r exp(SG 2 pi i r k / 8): radix-2 decimation in frequency on
// the array in place, outputs in natural order.
template <int SG>
__device__ __forceinline__ void dft8(double2 (&a)[8])
{
    constexpr double c = 0.70710678118654752440;
    // stage 1: butterflies (r, r+4), twiddle W8^r on the difference
    dft2<SG>(a[0], a[4]);
    dft2<SG>(a[1], a[5]);
    dft2<SG>(a[2], a[6]);
    dft2<SG>(a[3], a[7]);
    a[5] = make_double2(c * (a[5].x - SG * a[5].y), c * (a[5].y + SG * a[5].x));
    a[6] = cmul_si<SG>(a[6]);
    a[7] = make_double2(c * (-a[7].x - SG * a[7].y), c * (-a[7].y + SG * a[7].x));
    // stage 2: butterflies (r, r+2) within each half, twiddle W4 on the difference
    dft2<SG>(a[0], a[2]);
    dft2<SG>(a[1], a[3]);
    a[3] = cmul_si<SG>(a[3]);
    dft2<SG>(a[4], a[6]);
    dft2<SG>(a[5], a[7]);
    a[7] = cmul_si<SG>(a[7]);
    // stage 3
    dft2<SG>(a[0], a[1]);
    dft2<SG>(a[2], a[3]);
    dft2<SG>(a[4], a[5]);
    dft2<SG>(a[6], a[7]);
    // bit-reversed -> natural order: swap (1,4), (3,6)
    double2 t = a[1];
    a[1] = a[4];
    a[4] = t;
    t = a[3];
    a[3] = a[6];
    a[6] = t;
}

// Per-pass twiddle tables.  The twiddle buffer of a march holds the N = 2M
// point twiddles exp(+2 pi i k/N) followed by one table per Stockham pass of
// span NS = 8, 64, 512 (< M) of the length-M transforms: the pass of radix
// R = min(8, M/NS) stores exp(+2 pi i r k/(NS R)) at (r-1) NS + k, r < R,
// k < NS.  The threads of a warp take consecutive k, so a pass's twiddle
// loads are contiguous; read from the point table they would be strided by
// 2 r k entries (up to one cache line per thread).
__host__ __device__ constexpr int pass_radix(int M, int NS) { return M / NS < 8 ? M / NS : 8; }
__host__ __device__ constexpr int pass_table_offset(int M, int NS)
{
    int off = 0;
    for (int s = 8; s < NS; s *= 8) off += (pass_radix(M, s) - 1) * s;
    return off;
}
// Tables of the warp-exchange length-512 transforms (Ntau = 1024, below),
// after the pass tables: T64[k][q] = exp(+2 pi i q k/64) (k, q < 8), then
// TB_ST[r][t] = exp(+2 pi i (t&7)((t>>3) + 8r)/512) and TB_TS[r][t] =
// exp(+2 pi i (t>>3)((t&7) + 8r)/512) for r < 8, t < 64; every entry is a copy
// of a point twiddle.
__host__ __device__ constexpr int w512_table_offset(int N) { return N + pass_table_offset(N / 2, N / 2); }
constexpr int kW512Tables = 64 + 512 + 512;
// double2 entries of the twiddle buffer of a march over Ntau = N
__host__ __device__ constexpr int march_twiddle_count(int N)
{
    return w512_table_offset(N) + (N == 1024 ? kW512Tables : 0);
}

// Twiddles of one Stockham pass (radix R, span NS) for thread t: element r of
// butterfly u = t + TG u' is multiplied by w_M^{SG r k M/(NS R)}, k = j mod NS.
// Fetched separately so that the loads can be issued before the barrier that
// precedes the pass and their latency overlaps the barrier wait.
template <int M, int TG, int R, int NS, int SG>
__device__ __forceinline__ void fetch_twiddles(double2 (&w)[7], int t, const double2* __restrict__ twN, int zoff)
{
    static_assert(R == pass_radix(M, NS), "pass table radix");
    constexpr int B = 8 / R;
    const double2* __restrict__ tab = twN + 2 * M + pass_table_offset(M, NS);
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const int k = (t + TG * u) & (NS - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) {
            double2 x = __ldg(&tab[(r - 1) * NS + k + zoff]);
            if (SG < 0) x.y = -x.y;
            w[u * (R - 1) + (r - 1)] = x;
        }
    }
}

// One Stockham pass of radix R over span NS on the standard layout: thread t
// holds x[t + TG q]; butterfly j = t + TG u takes x[j + r M/R] = v[u + r*8/R].
template <int M, int TG, int R, int NS, int SG, bool LAST>
__device__ __forceinline__ void stockham_pass(double2 (&v)[8], double2* __restrict__ out, int t,
                                              const double2 (&w)[7])
{
    constexpr int B = 8 / R;
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const int j = t + TG * u;
        const int k = j & (NS - 1);
        double2 a[8];
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = v[u + r * B];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) a[r] = cmul(a[r], w[u * (R - 1) + (r - 1)]);
        }
        if (R == 8) {
            dft8<SG>(a);
        } else if (R == 4) {
            dft4<SG>(a[0], a[1], a[2], a[3]);
        } else {
            dft2<SG>(a[0], a[1]);
        }
        if (LAST) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[u + r * B] = a[r];
        } else {
            const int base = (j / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) out[swz8(base + r * NS)] = a[r];
        }
    }
}

template <int TG>
__device__ __forceinline__ void fetch_point_twiddles(double2* pj, int t, const double2* __restrict__ twN, int zoff)
{
#pragma unroll
    for (int q = 0; q < 8; ++q) pj[q] = __ldg(&twN[t + TG * q + zoff]);
}

// the per-point twiddles w_N^j (N = 1024) in layout T of the warp-exchange
// transforms: register q of thread t holds point j = (t >> 3) + 8 (t & 7) + 64 q
__device__ __forceinline__ void fetch_point_twiddles_t(double2* pj, int t, const double2* __restrict__ twN, int zoff)
{
    const int j0 = (t >> 3) + 8 * (t & 7);
#pragma unroll
    for (int q = 0; q < 8; ++q) pj[q] = __ldg(&twN[j0 + 64 * q + zoff]);
}

template <int TG>
__device__ __forceinline__ void load_std(double2 (&v)[8], const double2* __restrict__ in, int t)
{
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = in[swz8(t + TG * q)];
}

// Length-M DFT, X_k = sum_j x_j exp(SG 2 pi i jk/M), unscaled, from and to the
// standard register layout.  bufs[0..1] ping-pong; `cur` selects the first
// buffer written and is advanced so that the next transform never writes a
// buffer that a lagging thread may still be reading.
template <int M, int TG, int SG, class SY>
__device__ __forceinline__ void dft_m(double2 (&v)[8], double2* __restrict__ b0, double2* __restrict__ b1,
                                      int& cur, int t, const double2* __restrict__ twN, const SY& sy,
                                      bool active, const volatile int* zero)
{
    constexpr int NP = M == 64 ? 2 : (M <= 512 ? 3 : 4);
    constexpr int RL = M == 64 ? 8 : M == 128 ? 2 : M == 256 ? 4 : M == 512 ? 8 : 2;
    // A zero read from shared memory, added to every twiddle index of this
    // transform: the backend cannot prove two transforms use the same twiddle
    // addresses, so it does not keep all of them live in registers across the
    // whole RHS evaluation (which costs ~50 registers and spills).
    const int zoff = *zero;
    double2* w0 = cur ? b1 : b0;
    double2* w1 = cur ? b0 : b1;
    double2 tw[7];
    if (active) stockham_pass<M, TG, 8, 1, SG, false>(v, w0, t, tw);  // span 1: no twiddles
    if constexpr (NP == 2) {
        if (active) fetch_twiddles<M, TG, RL, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w0, t);
        if (active) stockham_pass<M, TG, RL, 8, SG, true>(v, w0, t, tw);
        cur ^= 1;
    } else if constexpr (NP == 3) {
        if (active) fetch_twiddles<M, TG, 8, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w0, t);
        if (active) stockham_pass<M, TG, 8, 8, SG, false>(v, w1, t, tw);
        if (active) fetch_twiddles<M, TG, RL, 64, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w1, t);
        if (active) stockham_pass<M, TG, RL, 64, SG, true>(v, w1, t, tw);
    } else {
        if (active) fetch_twiddles<M, TG, 8, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w0, t);
        if (active) stockham_pass<M, TG, 8, 8, SG, false>(v, w1, t, tw);
        if (active) fetch_twiddles<M, TG, 8, 64, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w1, t);
        if (active) stockham_pass<M, TG, 8, 64, SG, false>(v, w0, t, tw);
        if (active) fetch_twiddles<M, TG, RL, 512, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) load_std<TG>(v, w0, t);
        if (active) stockham_pass<M, TG, RL, 512, SG, true>(v, w0, t, tw);
        cur ^= 1;
    }
}

// Two independent length-M DFTs of the same direction in one set of passes:
// the same arithmetic as two dft_m calls, with one twiddle fetch and one
// barrier per pass for both and twice the independent work between barriers.
// v uses the buffer pair (a0, a1), u the pair (c0, c1), both selected by cur.
template <int M, int TG, int SG, class SY>
__device__ __forceinline__ void dft_m2(double2 (&v)[8], double2 (&u)[8], double2* __restrict__ a0,
                                       double2* __restrict__ a1, double2* __restrict__ c0,
                                       double2* __restrict__ c1, int& cur, int t, const double2* __restrict__ twN,
                                       const SY& sy, bool active, const volatile int* zero)
{
    constexpr int NP = M == 64 ? 2 : (M <= 512 ? 3 : 4);
    constexpr int RL = M == 64 ? 8 : M == 128 ? 2 : M == 256 ? 4 : M == 512 ? 8 : 2;
    const int zoff = *zero;
    double2* wa0 = cur ? a1 : a0;
    double2* wa1 = cur ? a0 : a1;
    double2* wc0 = cur ? c1 : c0;
    double2* wc1 = cur ? c0 : c1;
    double2 tw[7];
    if (active) {
        stockham_pass<M, TG, 8, 1, SG, false>(v, wa0, t, tw);
        stockham_pass<M, TG, 8, 1, SG, false>(u, wc0, t, tw);
    }
    if constexpr (NP == 2) {
        if (active) fetch_twiddles<M, TG, RL, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) {
            load_std<TG>(v, wa0, t);
            load_std<TG>(u, wc0, t);
            stockham_pass<M, TG, RL, 8, SG, true>(v, wa0, t, tw);
            stockham_pass<M, TG, RL, 8, SG, true>(u, wc0, t, tw);
        }
        cur ^= 1;
    } else if constexpr (NP == 3) {
        if (active) fetch_twiddles<M, TG, 8, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) {
            load_std<TG>(v, wa0, t);
            load_std<TG>(u, wc0, t);
            stockham_pass<M, TG, 8, 8, SG, false>(v, wa1, t, tw);
            stockham_pass<M, TG, 8, 8, SG, false>(u, wc1, t, tw);
            fetch_twiddles<M, TG, RL, 64, SG>(tw, t, twN, zoff);
        }
        sy.sync();
        if (active) {
            load_std<TG>(v, wa1, t);
            load_std<TG>(u, wc1, t);
            stockham_pass<M, TG, RL, 64, SG, true>(v, wa1, t, tw);
            stockham_pass<M, TG, RL, 64, SG, true>(u, wc1, t, tw);
        }
    } else {
        if (active) fetch_twiddles<M, TG, 8, 8, SG>(tw, t, twN, zoff);
        sy.sync();
        if (active) {
            load_std<TG>(v, wa0, t);
            load_std<TG>(u, wc0, t);
            stockham_pass<M, TG, 8, 8, SG, false>(v, wa1, t, tw);
            stockham_pass<M, TG, 8, 8, SG, false>(u, wc1, t, tw);
            fetch_twiddles<M, TG, 8, 64, SG>(tw, t, twN, zoff);
        }
        sy.sync();
        if (active) {
            load_std<TG>(v, wa1, t);
            load_std<TG>(u, wc1, t);
            stockham_pass<M, TG, 8, 64, SG, false>(v, wa0, t, tw);
            stockham_pass<M, TG, 8, 64, SG, false>(u, wc0, t, tw);
            fetch_twiddles<M, TG, RL, 512, SG>(tw, t, twN, zoff);
        }
        sy.sync();
        if (active) {
            load_std<TG>(v, wa0, t);
            load_std<TG>(u, wc0, t);
            stockham_pass<M, TG, RL, 512, SG, true>(v, wa0, t, tw);
            stockham_pass<M, TG, RL, 512, SG, true>(u, wc0, t, tw);
        }
        cur ^= 1;
    }
}

// ------------------------------------------- warp-exchange length-512 DFT
// A length-512 transform on a stage group of 64 threads (two warps) in which
// one of the two data exchanges stays inside a warp.  Index p = a + 8b + 64c
// (digits < 8), k = ka + 8kb + 64kc:
//   X[k] = sum_a w^{a(ka+8kb)} w8^{a kc} sum_b w64^{b ka} w8^{b kb} sum_c w8^{c ka} x[p]
// with w = exp(SG 2 pi i/512): a radix-8 pass over each digit, registers
// holding the digit being summed.  A thread t has lo = t & 7, hi = t >> 3
// (hi's top bit is the warp), and its register q holds index
//   layout S:  lo + 8 hi + 64 q      layout T:  hi + 8 lo + 64 q.
// An exchange swaps the register digit with one thread digit: with lo (the
// thread keeps hi) it stays inside a warp and needs only __syncwarp; with hi
// it crosses warps and needs the group barrier.  A transform from S sums c,
// then b (= hi: cross-warp exchange), then a (= lo: warp-local) and leaves
// its output in layout T; a transform from T sums c, b (= lo: warp-local),
// a (= hi: cross-warp) and leaves layout S.  The RHS alternates them: the
// state and spectra live in layout S, the physical-space fields in layout T.
//
// Buffers (b0, b1 of the stage).  Every read is "thread t, register q reads
// t + 64 q", so a warp reads only the entries whose bits 3..5 are its own hi
// values; a warp-local exchange writes only such entries too.  An S->T
// transform exchanges through b0 twice (the warp-local exchange rewrites the
// warp's own part of b0 after the warp has read it); a T->S transform makes
// its warp-local exchange in b0 and its cross-warp one in b1; the stage RHS
// then goes to b1 (each thread its own slots).  Between two writes of a
// buffer by different warps there is always a group barrier after the last
// read of the first write, since the two kinds of transform alternate.
// The index swizzle i ^ ((i >> 6) & 7) makes every write and read pattern
// map the 8 lanes of a 16-byte access phase to 8 distinct bank groups.
__device__ __forceinline__ int swz64(int i) { return i ^ ((i >> 6) & 7); }

// exchange write patterns: register r of thread t goes to
//   cross: thread lo + 8 r, register hi      (index lo + 8 r + 64 hi)
//   local: thread r + 8 hi, register lo      (index r + 8 hi + 64 lo)
__device__ __forceinline__ int wx_cross(int t, int r) { return swz64((t & 7) + 8 * r + 64 * (t >> 3)); }
__device__ __forceinline__ int wx_local(int t, int r) { return swz64(r + 8 * (t >> 3) + 64 * (t & 7)); }

template <int SG, bool IN_T>
__device__ __forceinline__ void w512_fetch_a(double2 (&w)[7], int t, const double2* __restrict__ tab, int zoff)
{
    // after the first exchange: register q holds digit b, twiddle w64^{b ka},
    // ka = t >> 3 (from S) or t & 7 (from T)
    const int k = IN_T ? (t & 7) : (t >> 3);
#pragma unroll
    for (int q = 1; q < 8; ++q) {
        double2 x = __ldg(&tab[k * 8 + q + zoff]);
        if (SG < 0) x.y = -x.y;
        w[q - 1] = x;
    }
}

template <int SG, bool IN_T>
__device__ __forceinline__ void w512_fetch_b(double2 (&w)[8], int t, const double2* __restrict__ tab, int zoff)
{
    const double2* __restrict__ tb = tab + 64 + (IN_T ? 512 : 0);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        double2 x = __ldg(&tb[r * 64 + t + zoff]);
        if (SG < 0) x.y = -x.y;
        w[r] = x;
    }
}

__device__ __forceinline__ void w512_store(const double2 (&v)[8], double2* __restrict__ buf, int t, bool cross)
{
#pragma unroll
    for (int r = 0; r < 8; ++r) buf[cross ? wx_cross(t, r) : wx_local(t, r)] = v[r];
}

__device__ __forceinline__ void w512_load(double2 (&v)[8], const double2* __restrict__ buf, int t)
{
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = buf[swz64(t + 64 * q)];
}

// One length-512 transform, layout S -> T (IN_T false) or T -> S (IN_T true),
// X_k = sum_j x_j exp(SG 2 pi i jk/512), unscaled.  tab: the W tables
// (twN + w512_table_offset(1024)).
template <int SG, bool IN_T, class SY>
__device__ __forceinline__ void dft_w512(double2 (&v)[8], double2* __restrict__ b0, double2* __restrict__ b1, int t,
                                         const double2* __restrict__ tab, const SY& gsy, const volatile int* zero)
{
    const int zoff = *zero;
    double2 ta[7], tb[8];
    dft8<SG>(v);
    w512_fetch_a<SG, IN_T>(ta, t, tab, zoff);
    if constexpr (!IN_T) {
        w512_store(v, b0, t, true);
        gsy.sync();
    } else {
        __syncwarp();
        w512_store(v, b0, t, false);
        __syncwarp();
    }
    w512_load(v, b0, t);
#pragma unroll
    for (int q = 1; q < 8; ++q) v[q] = cmul(v[q], ta[q - 1]);
    dft8<SG>(v);
    w512_fetch_b<SG, IN_T>(tb, t, tab, zoff);
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = cmul(v[r], tb[r]);
    if constexpr (!IN_T) {
        __syncwarp();
        w512_store(v, b0, t, false);
        __syncwarp();
        w512_load(v, b0, t);
    } else {
        w512_store(v, b1, t, true);
        gsy.sync();
        w512_load(v, b1, t);
    }
    dft8<SG>(v);
}

// Two independent length-512 transforms of the same direction and layout in
// one set of passes (v through b0/b1, u through c0/c1).
template <int SG, bool IN_T, class SY>
__device__ __forceinline__ void dft_w512_2(double2 (&v)[8], double2 (&u)[8], double2* __restrict__ b0,
                                           double2* __restrict__ b1, double2* __restrict__ c0,
                                           double2* __restrict__ c1, int t, const double2* __restrict__ tab,
                                           const SY& gsy, const volatile int* zero)
{
    const int zoff = *zero;
    double2 tw[8];
    dft8<SG>(v);
    dft8<SG>(u);
    if constexpr (!IN_T) {
        w512_store(v, b0, t, true);
        w512_store(u, c0, t, true);
        gsy.sync();
    } else {
        __syncwarp();
        w512_store(v, b0, t, false);
        w512_store(u, c0, t, false);
        __syncwarp();
    }
    {
        double2 ta[7];
        w512_fetch_a<SG, IN_T>(ta, t, tab, zoff);
        w512_load(v, b0, t);
        w512_load(u, c0, t);
#pragma unroll
        for (int q = 1; q < 8; ++q) {
            v[q] = cmul(v[q], ta[q - 1]);
            u[q] = cmul(u[q], ta[q - 1]);
        }
    }
    dft8<SG>(v);
    dft8<SG>(u);
    w512_fetch_b<SG, IN_T>(tw, t, tab, zoff);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        v[r] = cmul(v[r], tw[r]);
        u[r] = cmul(u[r], tw[r]);
    }
    if constexpr (!IN_T) {
        __syncwarp();
        w512_store(v, b0, t, false);
        w512_store(u, c0, t, false);
        __syncwarp();
        w512_load(v, b0, t);
        w512_load(u, c0, t);
    } else {
        w512_store(v, b1, t, true);
        w512_store(u, c1, t, true);
        gsy.sync();
        w512_load(v, b1, t);
        w512_load(u, c1, t);
    }
    dft8<SG>(v);
    dft8<SG>(u);
}

// --------------------------------------------------------------- slot maps
// Slot sigma = 2*ri + parity; ri -> position q in {0, 1, 6, 7}; parity 0 odd
// modes, 1 even modes.  Returns the state mode index (0..M-1).
template <int N>
__device__ __forceinline__ int slot_mode(int sigma, int t)
{
    constexpr int M = N / 2, Q = N / 4, TG = M / 8;
    const int ri = sigma >> 1;
    const int q = ri < 2 ? ri : ri + 4;
    const int p = t + TG * q;
    if ((sigma & 1) == 0) {
        const int k = 2 * p + 1;
        return k < Q ? k : k - M;
    }
    if (t == 0 && q == 6) return Q;
    const int k = 2 * p;
    return k < Q ? k : k - M;
}

__device__ __forceinline__ int slot_q(int sigma)
{
    const int ri = sigma >> 1;
    return ri < 2 ? ri : ri + 4;
}

// ------------------------------------------------------------------ the RHS
// dY/dx of one stage state at x (ODEStepper::computeDerivatives,
// ODEStepper.cpp:92-136).  yks: this stage's slot-indexed state (shared);
// b0/b1: this stage's exchange buffers; the result is written slot-indexed
// into (cur ? b1 : b0), the buffer the next transform would write first.
// DUAL: the three pairs of independent transforms (U+iV with F, the last IA2
// transform with dU+idV, the odd with the even forward transform) run as
// paired transforms (dft_m2) through the second exchange pair c0/c1.
template <int N, bool DUAL, bool WX, class SY>
__device__ __forceinline__ void rhs_eval(const double2* __restrict__ yks, double* __restrict__ uvs, double x,
                                         double dim, double dm2c, double k0, int t, double2* __restrict__ b0,
                                         double2* __restrict__ b1, double2* __restrict__ c0,
                                         double2* __restrict__ c1, int& cur, double* lam_slot,
                                         const double2* __restrict__ twN, const SY& sy, bool active,
                                         const volatile int* zero)
{
    constexpr int M = N / 2, TG = M / 8;
    constexpr double invM = 1.0 / M;
    static_assert(!WX || (M == 512 && DUAL), "warp-exchange transforms: Ntau 1024, paired");
    // warp-exchange transforms: fixed buffer roles, the stage RHS goes to b1
    if constexpr (WX) cur = 1;
    const double2* __restrict__ wtab = twN + w512_table_offset(N);
    double2 v[8];
    double F[8];
    double* Us = uvs;      // [q][t], this thread's own entries only
    double* Vs = uvs + M;

    double2 u[8];  // the second transform of a pair (DUAL)
    // F from the even modes: doubleModes (with its N/4 quirk) + phase fix
    auto even_input = [&](double2 (&w)[8]) {
#pragma unroll
        for (int q = 0; q < 8; ++q) w[q] = make_double2(0.0, 0.0);
        if (active) {
            w[0] = yks[1 * TG + t];
            if (t == 1) w[0].x = -yks[7 * TG + TG - 1].x;  // Re c[2] = -Re c[N-2] = -Re Y[M-2]
            w[1] = yks[3 * TG + t];
            const double2 yq = yks[5 * TG + t];
            if (t == 0) w[2] = make_double2(0.5 * yq.x, 0.5 * yq.y);  // c[N/4] = Y[N/4]/2
            w[6] = yq;                                                  // c[3N/4] = Y[N/4] (t = 0)
            w[7] = yks[7 * TG + t];
        }
    };

    // --- U + iV from the odd modes (IDFT_M, post-twiddle w^j) ----------------
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = make_double2(0.0, 0.0);
    if (active) {
        v[0] = yks[0 * TG + t];
        v[1] = yks[2 * TG + t];
        v[6] = yks[4 * TG + t];
        v[7] = yks[6 * TG + t];
    }
    // the per-point twiddles w_N^{t + TG q} of the post- and pre-twiddles are
    // fetched after the transforms they follow: prefetched before the last
    // exchange barrier they held 32 registers through the heaviest pass
    // (1.5 % slower per C3 build, measured A/B)
    double2 pj[8];
    if constexpr (WX) {
        even_input(u);
        dft_w512_2<-1, false>(v, u, b0, b1, c0, c1, t, wtab, sy, zero);
        fetch_point_twiddles_t(pj, t, twN, *zero);
    } else if constexpr (DUAL) {
        even_input(u);
        dft_m2<M, TG, -1>(v, u, b0, b1, c0, c1, cur, t, twN, sy, active, zero);
        if (active) fetch_point_twiddles<TG>(pj, t, twN, *zero);
    } else {
        dft_m<M, TG, -1>(v, b0, b1, cur, t, twN, sy, active, zero);
        if (active) fetch_point_twiddles<TG>(pj, t, twN, *zero);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double2 o = cmul(v[q], cconj(pj[q]));
        if (active) {
            Us[q * TG + t] = o.x;
            Vs[q * TG + t] = o.y;
        }
    }

    // --- F ---------------------------------------------------------------------
    if constexpr (DUAL) {
#pragma unroll
        for (int q = 0; q < 8; ++q) F[q] = u[q].y;
    } else {
        even_input(v);
        dft_m<M, TG, -1>(v, b0, b1, cur, t, twN, sy, active, zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) F[q] = v[q].y;
    }

    // --- IA2 constraint coefficients (InitialConditionGenerator.cpp:876-881) --
    const double c8 = dm2c / (8.0 * x);  // (D-2)^3 / (8x), once per evaluation
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double U = Us[q * TG + t], V = Vs[q * TG + t];
        const double co = -(((x + F[q]) * U * U + (x - F[q]) * V * V) * c8 + (dim - 3.0));
        v[q] = make_double2(co, 0.0);
    }

    // --- solveInhom (SpectralTransformer.cpp:264-292) on half-period data ----
    if constexpr (WX)
        dft_w512<1, true>(v, b0, b1, t, wtab, sy, zero);
    else
        dft_m<M, TG, 1>(v, b0, b1, cur, t, twN, sy, active, zero);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = make_double2(v[q].x * invM, v[q].y * invM);
    if (active && t == 0) *lam_slot = v[0].x;  // lambda = f_hat[0] (real: imag is exactly 0)
    // lamIntegrate(f_hat, 0): out_k = f_k / (-i m k0) = i f_k / (m k0); DC and Nyquist -> 0.
    // Only thread 0 holds the DC (q = 0) and Nyquist (p = M/2 = 4 TG: q = 4)
    // entries, so every entry takes the general formula without a branch and
    // thread 0 overwrites those two afterwards.
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = 2 * (t + TG * q);
        const int m = k < M ? k : k - N;
        const double r = 1.0 / (m * k0);
        v[q] = make_double2(-v[q].y * r, v[q].x * r);
    }
    if (t == 0) {
        v[0] = make_double2(0.0, 0.0);
        v[4] = make_double2(0.0, 0.0);
    }
    if constexpr (WX)
        dft_w512<-1, false>(v, b0, b1, t, wtab, sy, zero);
    else
        dft_m<M, TG, -1>(v, b0, b1, cur, t, twN, sy, active, zero);
    double Fr[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double e = exp(v[q].x);
        Fr[q] = 1.0 / e;                         // e^{-F}, kept for X e^{-F}
        v[q] = make_double2(-(dim - 3.0) * e, 0.0);  // h = -g e^F
    }
    // lambda (written by thread 0 after the first IA2 transform, two exchange
    // barriers ago) and the DC and Nyquist factors of the division below,
    // taken by every thread before the transform so that they stay off the
    // critical path
    const double lam = *lam_slot;
    const double ilam = lam != 0.0 ? 1.0 / lam : 0.0;
    // Nyquist: the reference multiplies h by the complex quotient
    // (lambda + 0i) / (lambda^2 + s^2 + 0i), s = k0 N/2 (Smith's method in
    // std::complex division), which is lambda / (lambda^2 + s^2) exactly
    const double qn = lam / (lam * lam - 0.0 * 0.0 + (k0 * N / 2.0) * (k0 * N / 2.0));
    if constexpr (WX)
        dft_w512<1, true>(v, b0, b1, t, wtab, sy, zero);
    else
        dft_m<M, TG, 1>(v, b0, b1, cur, t, twN, sy, active, zero);
    {
        // out_k = h_k / (lambda - i s) = h_k (lambda + i s) / (lambda^2 + s^2), s = m k0,
        // with the DC and Nyquist rules of lamIntegrate for thread 0's q = 0 and
        // q = 4 entries applied after the branch-free general formula
        const double2 h0 = make_double2(v[0].x * invM, v[0].y * invM);
        const double2 h4 = make_double2(v[4].x * invM, v[4].y * invM);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = 2 * (t + TG * q);
            const int m = k < M ? k : k - N;
            const double2 h = make_double2(v[q].x * invM, v[q].y * invM);
            const double sm = m * k0;
            const double den = lam * lam + sm * sm;  // |lambda - i s|^2
            const double r = 1.0 / den;
            v[q] = den < 1e-28 ? make_double2(0.0, 0.0)
                               : make_double2((h.x * lam - h.y * sm) * r, (h.y * lam + h.x * sm) * r);
        }
        if (t == 0) {
            v[0] = make_double2(h0.x * ilam, h0.y * ilam);
            v[4] = cmul(make_double2(qn, 0.0), h4);
        }
    }
    // dU + i dV from -i m k0 c on the odd modes
    auto du_input = [&](double2 (&w)[8]) {
#pragma unroll
        for (int q = 0; q < 8; ++q) w[q] = make_double2(0.0, 0.0);
        if (active) {
#pragma unroll
            for (int ri = 0; ri < 4; ++ri) {
                const int q = ri < 2 ? ri : ri + 4;
                const int k = 2 * (t + TG * q) + 1;
                const int m = k < M ? k : k - N;
                const double s = m * k0;
                const double2 a = yks[(2 * ri) * TG + t];
                w[q] = make_double2(s * a.y, -(s * a.x));
            }
        }
    };
    double IA2[8];
    if constexpr (WX) {
        du_input(u);
        dft_w512_2<-1, false>(v, u, b0, b1, c0, c1, t, wtab, sy, zero);
        fetch_point_twiddles_t(pj, t, twN, *zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) IA2[q] = v[q].x * Fr[q];  // X e^{-F}
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = u[q];
    } else if constexpr (DUAL) {
        du_input(u);
        dft_m2<M, TG, -1>(v, u, b0, b1, c0, c1, cur, t, twN, sy, active, zero);
        if (active) fetch_point_twiddles<TG>(pj, t, twN, *zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) IA2[q] = v[q].x * Fr[q];  // X e^{-F}
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = u[q];
    } else {
        dft_m<M, TG, -1>(v, b0, b1, cur, t, twN, sy, active, zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) IA2[q] = v[q].x * Fr[q];  // X e^{-F}
        du_input(v);
        dft_m<M, TG, -1>(v, b0, b1, cur, t, twN, sy, active, zero);
        if (active) fetch_point_twiddles<TG>(pj, t, twN, *zero);
    }

    // --- pointwise Einstein-scalar RHS (ODEStepper.cpp:109-122) ---------------
    // divisions are taken as reciprocals shared between terms (one for 1/IA2,
    // one for both characteristic denominators): ulp-level rounding changes
    const double xinv = 1.0 / x;
    double fx[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const double2 w = pj[q];
        const double2 dO = cmul(v[q], cconj(w));
        const double dU = dO.x, dV = dO.y;
        const double U = Us[q * TG + t], V = Vs[q * TG + t];
        const double ia = 1.0 / IA2[q];
        const double g = 2.0 * (dim - 3.0) * ia - (dim - 2.0);
        const double fp = 2.0 * x * (F[q] + x), fm = 2.0 * x * (F[q] - x);
        const double rr = 1.0 / (fp * fm);  // one reciprocal for both denominators
        const double ux = (F[q] * ((dim - 2.0) * V - g * U) - 2.0 * x * dU) * (fm * rr);
        const double vx = (F[q] * ((dim - 2.0) * U - g * V) + 2.0 * x * dV) * (fp * rr);
        fx[q] = (dim - 3.0) * F[q] * (1.0 - IA2[q]) * ia * xinv;
        v[q] = cmul(make_double2(ux, vx), w);  // pre-twiddle exp(+2 pi i j/N)
    }

    // --- FieldsToStateVector: odd modes, then the even modes with the
    // halveModes fold of N/4 and 3N/4 and the frozen Delta slot ----------------
    auto write_f = [&](const double2 (&od)[8], const double2 (&ev)[8]) {
        if (active) {
            double2* fslot = cur ? b1 : b0;
            double2 e0 = make_double2(ev[0].x * invM, ev[0].y * invM);
            if (t == 1) e0.x = 0.0;  // dYdx[2] real part (Delta) frozen
            double2 e6 = make_double2(ev[6].x * invM, ev[6].y * invM);
            if (t == 0) e6 = cadd(make_double2(ev[2].x * invM, ev[2].y * invM), e6);  // in[N/4] + in[3N/4]
            fslot[0 * TG + t] = od[0];
            fslot[1 * TG + t] = e0;
            fslot[2 * TG + t] = od[1];
            fslot[3 * TG + t] = make_double2(ev[1].x * invM, ev[1].y * invM);
            fslot[4 * TG + t] = od[6];
            fslot[5 * TG + t] = e6;
            fslot[6 * TG + t] = od[7];
            fslot[7 * TG + t] = make_double2(ev[7].x * invM, ev[7].y * invM);
        }
    };
    if constexpr (WX) {
#pragma unroll
        for (int q = 0; q < 8; ++q) u[q] = make_double2(0.0, fx[q]);
        dft_w512_2<1, true>(v, u, b0, b1, c0, c1, t, wtab, sy, zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = make_double2(v[q].x * invM, v[q].y * invM);
        __syncwarp();  // the last exchange's reads of b1 are done before the RHS goes there
        write_f(v, u);
    } else if constexpr (DUAL) {
#pragma unroll
        for (int q = 0; q < 8; ++q) u[q] = make_double2(0.0, fx[q]);
        dft_m2<M, TG, 1>(v, u, b0, b1, c0, c1, cur, t, twN, sy, active, zero);
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = make_double2(v[q].x * invM, v[q].y * invM);
        write_f(v, u);
    } else {
        dft_m<M, TG, 1>(v, b0, b1, cur, t, twN, sy, active, zero);
        double2 od[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) od[q] = make_double2(v[q].x * invM, v[q].y * invM);
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = make_double2(0.0, fx[q]);
        dft_m<M, TG, 1>(v, b0, b1, cur, t, twN, sy, active, zero);
        write_f(od, v);
    }
}

// ------------------------------------------------------------ sweep reduce
template <int STP, int NW, class SY>
__device__ __forceinline__ double sweep_sum(double x, double* red, int lt, const SY& sy)
{
    constexpr int W = STP < 32 ? STP : 32;
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) x += __shfl_xor_sync(sy.mask, x, o, 32);
    if constexpr (NW == 1) {
        return x;
    } else {
        if ((lt & 31) == 0) red[lt >> 5] = x;
        sy.sync();
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) s += red[w];
        sy.sync();  // red is reused by the next reduction
        return s;
    }
}

// ------------------------------------------------------------ sweep slot
// Shared-memory partition and thread roles of one sweep slot of a CTA.
template <int N, int S, int PAIR = 1>
struct Slot {
    using K = MarchShape<N, S, PAIR>;
    double2* ex;    // [S][2][MP]; the stage RHS lands in one buffer of each pair
    double2* ys;    // [8][TG] slot-indexed y
    double2* ykm;   // this group's stage values [8][TG]
    double* uvm;    // this group's U, V [2][M]
    double* lam;    // [S]
    double* red;    // [NW]
    int* item_slot;
    volatile int* zero;
    double2* b0;
    double2* b1;
    double2* c0;  // the second transform's exchange pair (K::DUAL)
    double2* c1;
    int slot_id, lt, s, t;
    bool active;    // a working lane (constant true where the sweep has no padding lanes)
    SweepSync<(K::STP > 32)> sy;  // the whole sweep: IRK update, reductions, state hand-over
    SweepSync<(K::TG > 32)> gsy;  // this stage group only: the transforms of its RHS evaluation

    __device__ __forceinline__ Slot(double2* smem, int tid)
    {
        constexpr int TG = K::TG, STP = K::STP;
        slot_id = tid / STP;
        lt = tid % STP;
        const int s_raw = lt / TG;
        active = K::ST == K::STP ? true : s_raw < S;
        s = active ? s_raw : S - 1;
        t = lt % TG;
        if constexpr (STP < 32) {
            sy.bar_id = 0;
            sy.nthreads = STP;
            sy.mask = ((1u << STP) - 1u) << ((tid & 31) / STP * STP);
        } else if constexpr (STP == 32) {
            sy.bar_id = 0;
            sy.nthreads = 32;
            sy.mask = 0xffffffffu;
        } else {
            sy.bar_id = 1 + slot_id;
            sy.nthreads = STP;
            sy.mask = 0xffffffffu;
        }
        // A stage's transforms exchange data only inside its own group, so
        // they synchronise the group alone and the groups of a sweep drift
        // apart between the IRK updates.  Groups of 64 or more threads are
        // whole warps (ST is then a multiple of 32: no inactive lanes).
        if constexpr (TG < 32) {
            gsy.bar_id = 0;
            gsy.nthreads = TG;
            gsy.mask = ((1u << TG) - 1u) << ((tid & 31) / TG * TG);
        } else if constexpr (TG == 32) {
            gsy.bar_id = 0;
            gsy.nthreads = 32;
            gsy.mask = 0xffffffffu;
        } else {
            gsy.bar_id = 1 + K::SPC + slot_id * S + s_raw;
            gsy.nthreads = TG;
            gsy.mask = 0xffffffffu;
        }
        double2* base = smem + (size_t)slot_id * K::PER_SWEEP;
        ex = base;
        ys = ex + K::EX;
        double2* yks = ys + K::YS;
        double* uv = reinterpret_cast<double*>(yks + K::YK);
        double* misc = uv + 2 * K::UV;
        lam = misc;
        red = misc + S;
        item_slot = reinterpret_cast<int*>(misc + S + K::NW);
        zero = item_slot + 1;
        b0 = ex + (size_t)s * 2 * K::MP;
        b1 = b0 + K::MP;
        c0 = ex + K::EXA + (size_t)s * 2 * K::MP;
        c1 = c0 + K::MP;
        ykm = yks + (size_t)s * 8 * TG;
        uvm = uv + (size_t)s * 2 * K::M;
    }
};

// state -> slots: y (group 0) and every stage value (its own group)
template <int N, int S, int PAIR>
__device__ __forceinline__ void load_state(const Slot<N, S, PAIR>& sl, const double* __restrict__ yin)
{
    constexpr int TG = MarchShape<N, S, PAIR>::TG;
    if (sl.active) {
#pragma unroll
        for (int sg = 0; sg < 8; ++sg) {
            const int m = slot_mode<N>(sg, sl.t);
            const double2 v = make_double2(yin[2 * m], yin[2 * m + 1]);
            sl.ykm[sg * TG + sl.t] = v;
            if (sl.s == 0) sl.ys[sg * TG + sl.t] = v;
        }
    }
}

// Per-sweep values of the single-solve kernel: kernel parameters.
struct ParamScalars {
    const MarchParams& P;
    __device__ __forceinline__ double dim() const { return P.dim; }
    __device__ __forceinline__ double dm2c() const { return P.dim_m2_cubed; }
    __device__ __forceinline__ double prec() const { return P.prec; }
    __device__ __forceinline__ int max_its() const { return P.max_its; }
    __device__ __forceinline__ int nl() const { return P.nl; }
    __device__ __forceinline__ int nr() const { return P.nr; }
    __device__ __forceinline__ double grid(int i) const { return P.grid[i]; }
    __device__ __forceinline__ const double2* twN() const { return P.twN; }
    __device__ __forceinline__ double a(int i, int j) const { return P.a[i][j]; }
    __device__ __forceinline__ double b(int i) const { return P.b[i]; }
    __device__ __forceinline__ double c(int i) const { return P.c[i]; }
    __device__ __forceinline__ int predictor() const { return P.predictor; }
    __device__ __forceinline__ double lq(int j, int k) const { return P.lq[j][k]; }
    __device__ __forceinline__ int mode() const { return P.mode; }
    __device__ __forceinline__ double x_in(int item) const { return P.x_in[item]; }
    __device__ __forceinline__ double x_out(int item) const { return P.x_out[item]; }
    __device__ __forceinline__ double* yout(int item, int n) const { return P.yfinal + (size_t)item * n; }
    __device__ __forceinline__ int* status(int item) const { return P.status + item; }
    __device__ __forceinline__ int* fail_index(int item) const { return P.fail_index + item; }
    __device__ __forceinline__ int* its_out(int item) const { return P.its_out ? P.its_out + item : nullptr; }
    __device__ __forceinline__ int snap_slot(int gi) const { return P.snap_slot ? P.snap_slot[gi] : -1; }
    __device__ __forceinline__ double* snap_base() const { return P.snap; }
};

// ------------------------------------------------------------ one sweep
// March one (column, side) sweep: ShootingSolver::integrateToMatchPoint's
// loop over the grid (ShootingSolver.cpp:53-145) with ODEStepper::stepIRK's
// fixed-point iteration (ODEStepper.cpp:163-292) at every step.  Mode 2
// takes the single step x_in -> x_out instead (the IRK step test entry).
// The caller has loaded the state (load_state) and synchronised.  Outputs
// are addressed through sc only where they are written, so that no output
// pointer stays live across the march.
template <int N, int S, int PAIR, class SC>
__device__ __forceinline__ void march_item(const SC& sc, const Slot<N, S, PAIR>& sl, double k0, int side, int item,
                                           unsigned long long& n_its, unsigned long long& n_steps)
{
    const int mode = sc.mode();
    using K = MarchShape<N, S, PAIR>;
    constexpr int TG = K::TG, STP = K::STP;
    const int s = sl.s, t = sl.t;
    const bool active = sl.active;
    double2* const ex = sl.ex;
    double2* const ys = sl.ys;
    double2* const ykm = sl.ykm;
    int cur = 0;
    const int nsteps = mode == 2 ? 1 : (side == 0 ? sc.nl() : sc.nr());
    int status = 0, fail_at = -1;
    double dx_prev = 0.0;

    for (int st = 0; st < nsteps; ++st) {
        double xin, xout;
        int gi;
        if (mode == 2) {
            xin = sc.x_in(item);
            xout = sc.x_out(item);
            gi = 0;
        } else if (side == 0) {
            gi = st;
            xin = sc.grid(gi);
            xout = sc.grid(gi + 1);
        } else {
            gi = sc.nl() + sc.nr() - st;
            xin = sc.grid(gi);
            xout = sc.grid(gi - 1);
        }
        const double dx = xout - xin;
        const double xs = xin + dx * sc.c(s);
        if (mode == 0 && st > 0 && sc.predictor()) {
            // Optional start of the stage iteration (the reference restarts
            // at y): the previous step's collocation polynomial at this
            // step's stage abscissae, Y_s = y_{n+1} + h_n sum_j (L_j(theta_s)
            // - b_j) f_j with theta_s = 1 + c_s h_{n+1} / h_n, L_j the
            // integrated Lagrange basis on the nodes and f_j the previous
            // step's last stage derivatives.  ykm holds y_{n+1} here.
            const double th = 1.0 + sc.c(s) * (dx / dx_prev);
            double w[S];
#pragma unroll
            for (int j = 0; j < S; ++j) {
                double L = 0.0, pw = th;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    L = fma(sc.lq(j, k), pw, L);
                    pw *= th;
                }
                w[j] = dx_prev * (L - sc.b(j));
            }
            if (active) {
#pragma unroll
                for (int sg = 0; sg < 8; ++sg) {
                    double2 y = ykm[sg * TG + t];
#pragma unroll
                    for (int j = 0; j < S; ++j) {
                        const double2 f = ex[(size_t)(j * 2 + cur) * K::MP + sg * TG + t];
                        y.x = fma(w[j], f.x, y.x);
                        y.y = fma(w[j], f.y, y.y);
                    }
                    ykm[sg * TG + t] = y;
                }
            }
            sl.sy.sync();  // every group has read the stage derivatives
        }
        dx_prev = dx;
        if (mode == 0) {
            // the state at the start of this step, for the Debug field export
            // (ShootingSolver.cpp:85-97, 128-138)
            const int slot = sc.snap_slot(gi);
            if (slot >= 0 && active && s == 0) {
                double* o = sc.snap_base() + (size_t)slot * N;
#pragma unroll
                for (int sg = 0; sg < 8; ++sg) {
                    const int m = slot_mode<N>(sg, t);
                    const double2 y = ys[sg * TG + t];
                    o[2 * m] = y.x;
                    o[2 * m + 1] = y.y;
                }
            }
        }

        bool converged = false;
        int its_reached = 0;
        const int max_its = sc.max_its();
        for (int its = 0; its < max_its; ++its) {
            ++its_reached;
            rhs_eval<N, K::DUAL, K::WX>(ykm, sl.uvm, xs, sc.dim(), sc.dm2c(), k0, t, sl.b0, sl.b1, sl.c0, sl.c1, cur,
                                 &sl.lam[s], sc.twN(), sl.gsy, active, sl.zero);
            sl.sy.sync();  // every stage RHS is in shared memory
            double part = 0.0;
            if (active) {
#pragma unroll
                for (int sg = 0; sg < 8; ++sg) {
                    double2 nv = ys[sg * TG + t];
#pragma unroll
                    for (int kk = 0; kk < S; ++kk) {
                        const double w = dx * sc.a(s, kk);
                        const double2 f = ex[(size_t)(kk * 2 + cur) * K::MP + sg * TG + t];
                        nv.x = fma(w, f.x, nv.x);
                        nv.y = fma(w, f.y, nv.y);
                    }
                    const double2 old = ykm[sg * TG + t];
                    const double ex_ = old.x - nv.x, ey_ = old.y - nv.y;
                    part = fma(ex_, ex_, part);
                    part = fma(ey_, ey_, part);
                    ykm[sg * TG + t] = nv;
                }
            }
            const double tot = sweep_sum<STP, K::NW>(part, sl.red, sl.lt, sl.sy);
            const double norm2 = sqrt(tot / (double)(N * S));
            const double prec = sc.prec();
            double p10 = prec;
            if (its > max_its / 2) p10 = prec * 10.0 * (2.0 * (double)its / (double)max_its - 0.5);
            if (norm2 < p10) {
                converged = true;
                break;
            }
            if constexpr (K::NW == 1) sl.sy.sync();  // new stage values visible to every lane
        }
        n_its += its_reached;
        n_steps += 1;
        // y += dx sum_i b_i f_i with the RHS of the last evaluation; stages restart at y
        if (active) {
#pragma unroll
            for (int sg = 0; sg < 8; ++sg) {
                double2 y = ys[sg * TG + t];
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    const double w = dx * sc.b(i);
                    const double2 f = ex[(size_t)(i * 2 + cur) * K::MP + sg * TG + t];
                    y.x = fma(w, f.x, y.x);
                    y.y = fma(w, f.y, y.y);
                }
                ykm[sg * TG + t] = y;
            }
        }
        sl.sy.sync();  // every group has read the old y
        if (active && s == 0) {
#pragma unroll
            for (int sg = 0; sg < 8; ++sg) ys[sg * TG + t] = ykm[sg * TG + t];
        }
        if (mode == 2 && active && s == 0 && t == 0) {
            int* its_out = sc.its_out(item);
            if (its_out) *its_out = converged ? its_reached : -its_reached;
        }
        if (!converged) {
            status = 1;
            fail_at = gi;
            break;
        }
    }
    // write the final state
    if (active && s == 0) {
        double* yout = sc.yout(item, N);
#pragma unroll
        for (int sg = 0; sg < 8; ++sg) {
            const int m = slot_mode<N>(sg, t);
            const double2 y = ys[sg * TG + t];
            yout[2 * m] = y.x;
            yout[2 * m + 1] = y.y;
        }
        if (t == 0) {
            *sc.status(item) = status;
            *sc.fail_index(item) = fail_at;
        }
    }
    sl.sy.sync();
}

// ------------------------------------------------------------------ kernel
// The item a sweep slot takes for work index w, or -1 when the work is done.
// With an item map the host has ordered the sweeps.  A march over (column,
// side) items without one (item = 2 column + side, no explicit side map)
// hands out every right-side sweep first, then the left-side ones: the right
// side marches into the stiff x -> 1 end and takes more IRK iterations
// (22,761 against 16,913 per sweep at Ntau 1024, 4000 + 4000 points), so this
// hands out the longest sweeps first.  The sweeps and their results are the
// same in any order.  Measured on that build (1536 sweeps, the same 60.9 M
// RHS evaluations): 1.187 s against 1.246 s in column order.
__device__ __forceinline__ int march_item_of(int w, const MarchParams& P)
{
    if (w >= P.n_items) return -1;
    if (P.item_map) return P.item_map[w];
    if (P.mode != 0 || P.item_side || (P.n_items & 1)) return w;
    const int h = P.n_items >> 1;
    return w < h ? 2 * w + 1 : 2 * (w - h);
}

// Two-ended claiming over a longest-first item map (MarchParams::sched):
// word 0 counts claims, word 1 the items taken from the front, word 2 those
// taken from the back, words 3.. count the sweep slots that started on each
// SM (%smid).  A slot of even rank on its SM takes the longest remaining
// sweep, one of odd rank the shortest, so the two sweeps sharing an SM are
// a long and a short one.  Claims stop after n_items in total, so the front
// and back ranges never overlap and every item runs once; %smid only steers
// the choice (a slot whose SM id is out of range counts as rank 0).
constexpr int kMarchSchedSms = 512;
constexpr int kMarchSchedWords = 3 + kMarchSchedSms;

__device__ __forceinline__ unsigned sm_id()
{
    unsigned id;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(id));
    return id;
}

__device__ __forceinline__ int march_claim_ends(const MarchParams& P, bool front)
{
    if (atomicAdd(P.sched, 1) >= P.n_items) return -1;
    const int w = front ? atomicAdd(P.sched + 1, 1) : P.n_items - 1 - atomicAdd(P.sched + 2, 1);
    return P.item_map[w];
}

template <int N, int S, int MINB, int PAIR>
__global__ void __launch_bounds__(MarchShape<N, S, PAIR>::NT, MINB) march_kernel(MarchParams P)
{
    using K = MarchShape<N, S, PAIR>;
    constexpr int TG = K::TG;
    extern __shared__ double2 smem[];
    const Slot<N, S, PAIR> sl(smem, threadIdx.x);
    if (sl.lt == 0) *sl.zero = 0;
    const ParamScalars sc{P};
    unsigned long long n_its = 0, n_steps = 0;
    bool front = true;
    if (P.sched) {
        if (sl.lt == 0) {
            const unsigned id = sm_id();
            *sl.item_slot = id < (unsigned)kMarchSchedSms ? atomicAdd(P.sched + 3 + id, 1) : 0;
        }
        sl.sy.sync();
        front = (*sl.item_slot & 1) == 0;
        sl.sy.sync();
    }

    for (;;) {
        if (sl.lt == 0)
            *sl.item_slot = P.sched ? march_claim_ends(P, front) : march_item_of(atomicAdd(P.work_counter, 1), P);
        sl.sy.sync();
        const int item = *sl.item_slot;
        sl.sy.sync();
        if (item < 0) break;

        const double* yin = P.yinit + (size_t)item * N;
        const double delta = yin[4];
        const double k0 = 2.0 * kPi / delta;
        load_state<N, S>(sl, yin);
        sl.sy.sync();

        if (P.mode == 1) {
            // single RHS evaluation of the state at x_in[item]
            int cur = 0;
            rhs_eval<N, K::DUAL, K::WX>(sl.ykm, sl.uvm, P.x_in[item], P.dim, P.dim_m2_cubed, k0, sl.t, sl.b0, sl.b1,
                                 sl.c0, sl.c1, cur, &sl.lam[sl.s], P.twN, sl.gsy, sl.active, sl.zero);
            sl.sy.sync();
            if (sl.active && sl.s == 0) {
                const double2* fr = cur ? sl.b1 : sl.b0;
                double* yo = P.yfinal + (size_t)item * N;
#pragma unroll
                for (int sg = 0; sg < 8; ++sg) {
                    const int m = slot_mode<N>(sg, sl.t);
                    const double2 f = fr[sg * TG + sl.t];
                    yo[2 * m] = f.x;
                    yo[2 * m + 1] = f.y;
                }
            }
            sl.sy.sync();
            continue;
        }

        const int side = P.item_side ? P.item_side[item] : (item & 1);
        march_item<N, S>(sc, sl, k0, side, item, n_its, n_steps);
    }
    if (sl.lt == 0 && P.counters) {
        atomicAdd(&P.counters[0], n_its * (unsigned long long)S);
        atomicAdd(&P.counters[1], n_its);
        atomicAdd(&P.counters[2], n_steps);
    }
}

// ------------------------------------------------------------ batch kernel
// Sweeps of several solves (uneven Ntau, grid sizes and dimensions) in one
// persistent launch.  Items are grouped into Ntau classes, largest first; a
// CTA works through the classes in that order, and inside a class every sweep
// slot pulls its own next (solve, item) from the class's longest-first list,
// from the front or the back by the slot's rank on its SM (as
// march_claim_ends), so sweeps of different solves share a CTA.  All classes use the same 128-thread CTA and
// the same stage count (the Gauss-Legendre tableau is a kernel parameter).
struct BatchSolve {
    const double* grid;
    const double2* twN;
    const double* yinit;  // [item][Ntau]
    double* yfinal;
    int* status;          // [item]
    int* fail_index;      // [item]
    const int* cancel;    // optional: nonzero skips the solve's remaining sweeps
    double dim, dm2c, prec;
    int nl, nr, max_its, ntau;
    int predictor;
};

constexpr int kBatchMaxClasses = 4;

struct BatchParams {
    const BatchSolve* solves;
    const int2* items;  // {solve, item = 2 column + side}, class by class
    int n_classes;
    int cls_ntau[kBatchMaxClasses];
    int cls_begin[kBatchMaxClasses + 1];
    int* cls_counter;   // [3 kBatchMaxClasses]: per class the claims and the items taken from the front and the back
    int* sm_rank;       // [kBatchMaxClasses][kMarchSchedSms]: sweep slots started per class and SM
                        // (null: every slot claims from the front, in list order)
    int cls_ends[kBatchMaxClasses];  // 1: class c claims from both ends (a few waves deep), 0: list order
    double a[3][3], b[3], c[3];
    double lq[3][3];               // as MarchParams::lq
    unsigned long long* counters;  // [0] RHS evaluations [1] IRK iterations [2] steps
};

// Per-sweep values of the batch kernel, staged in shared memory by the slot's
// first thread when it takes an item.
struct SweepScalars {
    const double* grid;
    const double2* twN;
    const double* yin;
    double* yout;
    int* status;
    int* fail_index;
    double dim, dm2c, prec;
    int nl, nr, max_its, side;
    int predictor;
    int front;  // claims from the front of the class's list (else from the back)
};

// As march_claim_ends, over class c (n items) of a batch launch.
__device__ __forceinline__ int batch_claim(const BatchParams& B, int c, int n, int front)
{
    int* ctr = B.cls_counter + 3 * c;
    if (atomicAdd(ctr, 1) >= n) return -1;
    return front ? atomicAdd(ctr + 1, 1) : n - 1 - atomicAdd(ctr + 2, 1);
}

struct SmemScalars {
    const SweepScalars* p;
    const BatchParams& B;
    __device__ __forceinline__ double dim() const { return p->dim; }
    __device__ __forceinline__ double dm2c() const { return p->dm2c; }
    __device__ __forceinline__ double prec() const { return p->prec; }
    __device__ __forceinline__ int max_its() const { return p->max_its; }
    __device__ __forceinline__ int nl() const { return p->nl; }
    __device__ __forceinline__ int nr() const { return p->nr; }
    __device__ __forceinline__ double grid(int i) const { return p->grid[i]; }
    __device__ __forceinline__ const double2* twN() const { return p->twN; }
    __device__ __forceinline__ double a(int i, int j) const { return B.a[i][j]; }
    __device__ __forceinline__ double b(int i) const { return B.b[i]; }
    __device__ __forceinline__ double c(int i) const { return B.c[i]; }
    __device__ __forceinline__ int predictor() const { return p->predictor; }
    __device__ __forceinline__ double lq(int j, int k) const { return B.lq[j][k]; }
    __device__ __forceinline__ int mode() const { return 0; }
    __device__ __forceinline__ double x_in(int) const { return 0.0; }
    __device__ __forceinline__ double x_out(int) const { return 0.0; }
    __device__ __forceinline__ double* yout(int, int) const { return p->yout; }
    __device__ __forceinline__ int* status(int) const { return p->status; }
    __device__ __forceinline__ int* fail_index(int) const { return p->fail_index; }
    __device__ __forceinline__ int* its_out(int) const { return nullptr; }
    __device__ __forceinline__ int snap_slot(int) const { return -1; }
    __device__ __forceinline__ double* snap_base() const { return nullptr; }
};

template <int S>
struct BatchShape {
    static constexpr int NT = 128;
    static constexpr size_t max2(size_t x, size_t y) { return x > y ? x : y; }
    static constexpr size_t SWEEPS =
        max2(max2(MarchShape<128, S>::SMEM, MarchShape<256, S>::SMEM), max2(MarchShape<512, S>::SMEM, MarchShape<1024, S>::SMEM));
    static constexpr int MAX_SPC = MarchShape<128, S>::SPC;
    static constexpr size_t SMEM = SWEEPS + MAX_SPC * sizeof(SweepScalars);
};

template <int N, int S>
__device__ __forceinline__ void batch_class(const BatchParams& B, int c, double2* smem, unsigned long long& n_its,
                                            unsigned long long& n_steps)
{
    using K = MarchShape<N, S>;
    static_assert(K::NT == BatchShape<S>::NT, "every class uses the same CTA");
    const Slot<N, S> sl(smem, threadIdx.x);
    if (sl.lt == 0) *sl.zero = 0;
    SweepScalars* sp = reinterpret_cast<SweepScalars*>(reinterpret_cast<char*>(smem) + BatchShape<S>::SWEEPS) +
                       sl.slot_id;
    const SmemScalars sc{sp, B};
    const int n = B.cls_begin[c + 1] - B.cls_begin[c];
    unsigned long long c_its = 0, c_steps = 0;  // this slot's sweeps in this class
    // two-ended claiming over the class's longest-first items, as march_claim_ends
    if (sl.lt == 0) {
        const unsigned id = sm_id();
        const int rank = B.sm_rank && B.cls_ends[c] && id < (unsigned)kMarchSchedSms
                             ? atomicAdd(B.sm_rank + c * kMarchSchedSms + id, 1)
                             : 0;
        sp->front = (rank & 1) == 0;
    }
    for (;;) {
        if (sl.lt == 0) {
            int i;
            for (;;) {
                i = batch_claim(B, c, n, sp->front);
                if (i < 0) break;
                const int2 it = B.items[B.cls_begin[c] + i];
                const BatchSolve& so = B.solves[it.x];
                if (so.cancel && *(const volatile int*)so.cancel) continue;  // the solve no longer needs this sweep
                sp->grid = so.grid;
                sp->twN = so.twN;
                sp->yin = so.yinit + (size_t)it.y * N;
                sp->yout = so.yfinal + (size_t)it.y * N;
                sp->status = so.status + it.y;
                sp->fail_index = so.fail_index + it.y;
                sp->dim = so.dim;
                sp->dm2c = so.dm2c;
                sp->prec = so.prec;
                sp->nl = so.nl;
                sp->nr = so.nr;
                sp->max_its = so.max_its;
                sp->side = it.y & 1;
                sp->predictor = so.predictor;
                break;
            }
            *sl.item_slot = i;
        }
        sl.sy.sync();
        const int item = *sl.item_slot;
        if (item < 0) break;
        const double* yin = sp->yin;
        const double k0 = 2.0 * kPi / yin[4];
        load_state<N, S>(sl, yin);
        sl.sy.sync();
        march_item<N, S>(sc, sl, k0, sp->side, item, c_its, c_steps);
    }
    if (sl.lt == 0) {  // one thread per slot reports the slot's work
        n_its += c_its;
        n_steps += c_steps;
    }
}

template <int S>
__global__ void __launch_bounds__(128, 2) march_batch_kernel(BatchParams B)
{
    extern __shared__ double2 smem[];
    unsigned long long n_its = 0, n_steps = 0;
    for (int c = 0; c < B.n_classes; ++c) {
        switch (B.cls_ntau[c]) {
            case 1024: batch_class<1024, S>(B, c, smem, n_its, n_steps); break;
            case 512: batch_class<512, S>(B, c, smem, n_its, n_steps); break;
            case 256: batch_class<256, S>(B, c, smem, n_its, n_steps); break;
            case 128: batch_class<128, S>(B, c, smem, n_its, n_steps); break;
            default: break;
        }
        __syncthreads();  // the next class partitions shared memory differently
    }
    if (n_steps && B.counters) {
        atomicAdd(&B.counters[0], n_its * (unsigned long long)S);
        atomicAdd(&B.counters[1], n_its);
        atomicAdd(&B.counters[2], n_steps);
    }
}

}  // namespace pcc
