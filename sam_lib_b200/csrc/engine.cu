// GPU numeric phase of SPR for sm_100a: supernodal multifrontal LDL'
// factorisation and the forward/diagonal/back solves.
//
// Semantics follow the reference routines (file:line in src/SPR):
//   SPRF11 multifrontal loop ............ sprfc1.f:286-713
//   SPRF12/13/14 extend-add ............. sprfc1.f:716-982
//   SPRF15/SPRF17 (+LMVY18) pivots ...... sprfc1.f:985-1299, lmvy18.f
//   LMMY18 Schur update ................. lmmy18.f:5-192
//   SPRFS3/5/6 forward + diagonal ....... sprfs1.f:266-1141
//   SPRBS4/6 back substitution .......... sprbs1.f:251-574
// The arithmetic is FP64 throughout; the order of the floating-point updates
// differs from the reference (blocked, FMA), so results agree to rounding.
//
// Execution: one pass per elimination-tree level (leaves first).  Fronts of
// order <= kSmallMaxF are assembled, factored and written back by one CTA in
// shared memory (fused extend-add + LDL' + Schur update).  Larger fronts are
// assembled into dense column-major buffers in HBM and factored with a
// blocked right-looking LDL' (diagonal block, panel TRSM, FP64 DMMA Schur
// update), all fronts of the level batched into each launch.
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>

#include "engine.h"
#include "smhash.h"

namespace sprb {

bool trace_on() {
    static const bool on = [] {
        const char* e = std::getenv("SPR_B200_TRACE");
        return e && e[0] == '1';
    }();
    return on;
}
static std::chrono::steady_clock::time_point g_trace_t0;
void trace_reset() {
    if (trace_on()) g_trace_t0 = std::chrono::steady_clock::now();
}
void trace_point(const char* what) {
    if (!trace_on()) return;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - g_trace_t0).count();
    fprintf(stderr, "[spr_b200 trace] %9.3f ms  %s\n", ms, what);
}


#define CK(x)                                                                    \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess) {                                                 \
            fprintf(stderr, "spr_b200: CUDA error %s at %s:%d\n",                \
                    cudaGetErrorString(e_), __FILE__, __LINE__);                 \
            return -4;                                                           \
        }                                                                        \
    } while (0)

constexpr int kMaxRHS = 16;          // right-hand sides per solve pass

// NVTX range for the host timeline of a profiler (no-op without one).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

// ---------------------------------------------------------------------------
// Device views
// ---------------------------------------------------------------------------
struct Stats {
    int zero_count;
    int first_zero;          // smallest 0-based column with an exact zero diagonal
    int any_fail;            // exact zero diagonal found: nothing is factored (sprfc1.f:488)
    int pivot_fail;          // some pivot failed the TOL(1) test
    unsigned long long numneg;
    double tol2;             // max(a_jj / d_j), sprfc1.f:1284
    double trace;            // sum a_jj, sprfc1.f:483
    double mindpos;          // smallest positive pivot, sprfc1.f:690-697
    int tc_timeout;          // a tensor-core update CTA gave up waiting (see tc_gemm.cuh)
    unsigned long long nsing;    // SPRFC3: pivots replaced by the TOL(1)/TOL(4) rule
    unsigned long long near_piv; // pivots with |d| < near_tol |a_jj| (mixed-mode inertia guard)
    int solve_timeout;       // a triangle task of the solves gave up waiting for a block (k_*_tri)
};

struct PV {
    const int32_t *fst, *S, *F, *child_ptr, *child, *rows, *rel, *cchild, *ct, *buf_ld;
    const int64_t *lnz_off, *rel_off, *rbase, *cptr, *buf_off, *upd_off;
    double* arena;
    double* lnz;
    double* dvec;
    double* adiag;
    int32_t* sn_neg;
    int32_t* sn_fail;
    int32_t* sn_bad;         // front failed, or depends on a failed front
    double* sn_faild;
    double* sn_faila;
    Stats* st;
    const int64_t* linv_off;
    double* linv;            // inverses of the unit-lower diagonal blocks
    const int64_t* xinv_off;
    double* xinv;            // inverses of the kSolveBlock-wide diagonal blocks
    const int64_t* rect_off;
    const int64_t* fwd_off;
    const int64_t* tri_off;  // first block-ready flag of each large front (solves)
    double tol1;
    // SPRFC3 semantics (sprfc3.f:549-572, 1083-1099): a zero diagonal becomes
    // 1 and a pivot at or below TOL(1)|a_jj| is replaced instead of stopping;
    // both are recorded in DCOR(2,NEQ) (dcor[2j], dcor[2j+1])
    int fc3;
    double tol4;
    double* dcor;
    // partial factorisation: 1 for the retained supernodes (null if none)
    const uint8_t* ret;
    // inertia guard of the mixed mode: pivots with |d| < near_tol |a_jj| are
    // counted (their sign may depend on the TF32 rounding); 0 = off
    double near_tol;
    // time limit of every mbarrier wait of the tensor-core update (ns), and a
    // test switch: when set, CTA 0 of each tensor-core launch skips its first
    // operand load, so that its waits run out and the launch reports a timeout
    unsigned long long wait_ns;
    int tc_drop;
    // streamed factorisation: the original diagonal gathered on the host
    // (the pre-pass then reads it instead of LNZ, which is still uploading)
    const double* adiag_in;
    // node mask of a run split across GPUs: supernodes with skip[js] != 0 are
    // left alone (null: none)
    const uint8_t* skip;
};

struct Engine::Dev {
    // plan arrays
    int32_t *fst = nullptr, *S = nullptr, *F = nullptr, *child_ptr = nullptr, *child = nullptr,
            *rows = nullptr, *rel = nullptr, *cchild = nullptr, *ct = nullptr, *buf_ld = nullptr;
    int64_t *lnz_off = nullptr, *rel_off = nullptr, *rbase = nullptr, *cptr = nullptr,
            *buf_off = nullptr, *upd_off = nullptr;
    Job* jobs = nullptr;
    int64_t* linv_off = nullptr;
    double* linv = nullptr;
    int64_t* xinv_off = nullptr;
    double* xinv = nullptr;
    int32_t* task_map = nullptr;
    int64_t* rect_off = nullptr;
    int64_t* fwd_off = nullptr;
    int64_t* tri_off = nullptr;
    double* pbuf = nullptr;                      // back-solve rectangle partial sums
    int32_t* level_nodes = nullptr;              // small nodes of every level, concatenated
    std::vector<int64_t> small_begin;            // per level offset into level_nodes
    int32_t* all_nodes = nullptr;                // all nodes of every level (solves)
    std::vector<int64_t> all_begin, all_count;
    // work
    double* arena = nullptr;
    double* adiag = nullptr;
    int32_t* sn_neg = nullptr;
    int32_t* sn_fail = nullptr;
    int32_t* sn_bad = nullptr;
    uint8_t* ret = nullptr;                      // retained supernodes (partial factorisation)
    double* sn_faild = nullptr;
    double* sn_faila = nullptr;
    Stats* st = nullptr;
    double* vbuf = nullptr;                      // solve front vectors
    double* vbuf2 = nullptr;                     // solved diagonal blocks (same layout)
    int64_t vbuf_rhs = 0;
    double* bbuf = nullptr;                      // contiguous copy of B (ldb = NEQ)
    int64_t bbuf_rhs = 0;
    uint8_t* skip = nullptr;                     // node mask of a split run
    bool skip_on = false;
    int32_t* tri_tasks = nullptr;                // the solves' triangle tasks (node, block)
    int32_t* tri_sync = nullptr;                 // block-ready flags, then one task counter per level
    std::vector<void*> owned;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // page-locked, device-mapped mailbox for the few words the host reads
    // after each call (the factorisation's Stats, a hash, the solve's
    // timeout flag): a kernel writes them over the bus, so the read does not
    // queue on the copy engine behind a streamed factorisation's downloads
    unsigned long long* mbox = nullptr;         // host address
    unsigned long long* mbox_dev = nullptr;     // its device address
    unsigned long long* hbuf = nullptr;          // result of k_sm_hash
    // tensor-core (mixed) updates: operand slabs and the TMA map over them
    float* slab = nullptr;
    alignas(64) CUtensorMap slab_map;
    float* slab_far = nullptr;                   // slabs of the side-stream launches
    alignas(64) CUtensorMap slab_map_far;
    cudaStream_t side = nullptr;                 // side stream: trailing updates beyond the next super-panel
    cudaStream_t ahead = nullptr;                // look-ahead stream: in-super-panel columns after the next panel
    cudaStream_t wbs = nullptr;                  // early writes of final super-panels to LNZ (streamed copies)
    std::vector<cudaEvent_t> evpool;             // fork/join events of one factorisation
};

template <typename T>
static int dev_upload(std::vector<void*>& owned, T** dst, const std::vector<T>& src) {
    size_t n = std::max<size_t>(src.size(), 1);
    CK(cudaMalloc((void**)dst, n * sizeof(T)));
    owned.push_back(*dst);
    if (!src.empty()) CK(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

// ---------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_double(double* addr, double v) {
    unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
    unsigned long long old = *a;
    while (__longlong_as_double((long long)old) < v) {
        unsigned long long assumed = old;
        old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
        if (old == assumed) break;
    }
}

__device__ __forceinline__ int64_t find_job(const Job* jobs, int64_t n, int64_t t) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if (jobs[mid].task0 <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// job of a task: one load from the launch's task map, or a binary search
// over the jobs' first tasks when no map is given
__device__ __forceinline__ const Job& job_of(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t t) {
    return tmap ? jobs[tmap[t]] : jobs[find_job(jobs, njobs, t)];
}

// packed lower, column-major, order F: column j holds rows j..F-1
__device__ __forceinline__ int pk(int i, int j, int F) { return j * F - ((j * (j - 1)) >> 1) + (i - j); }

__host__ __device__ __forceinline__ int64_t lnz_col(int64_t j, int64_t F) { return j * F - (j * (j - 1)) / 2; }

// record a failed pivot (sprfc1.f:1274-1279): first failure per supernode wins
// A failed front poisons its ancestors only: fronts earlier in postorder than
// the first failure are still factored, so NUMNEG matches the reference's count
// of negative pivots met before it stops (sprfc1.f:610-616).
__device__ void record_fail(const PV& P, int js, int col, double d, double ad) {
    P.sn_fail[js] = col;
    P.sn_faild[js] = d;
    P.sn_faila[js] = ad;
    P.sn_bad[js] = 1;
    atomicExch(&P.st->pivot_fail, 1);
}

// A retained supernode of a partial factorisation (MSPAR(57) > 0, SUPSUP > 0):
// assembled but not eliminated (sprfc1.f:587), skipped by the solves
// (sprfs1.f:371, sprbs1.f:347).
__device__ __forceinline__ bool is_retained(const PV& P, int js) { return P.ret != nullptr && P.ret[js] != 0; }

// SPRF37 (sprfc3.f:1083-1099): the pivot d of a column with original
// diagonal ad becomes sign(TOL(1) max(1, |TOL(4) ad|), d) when |d| <= TOL(1)|ad|.
__device__ __forceinline__ double fc3_pivot(const PV& P, double d, double ad) {
    return fabs(d) <= P.tol1 * fabs(ad) ? copysign(fabs(P.tol1 * fmax(1.0, fabs(P.tol4 * ad))), d) : d;
}

// DCOR entries of column col (0-based) for the pivot d0 before and dn after
// the replacement: DCOR(1) = d0 on a replacement, else (or if d0 == 0) dn when
// dn < 0; DCOR(2) = dn on a replacement.  One thread per column.
__device__ __forceinline__ void fc3_record(const PV& P, int col, double d0, double dn) {
    const bool sing = fabs(d0) <= P.tol1 * fabs(P.adiag[col]);
    double* dc = P.dcor + 2 * (int64_t)col;
    double c1 = sing ? d0 : 0.0;
    if (dn < 0.0 && c1 == 0.0) c1 = dn;
    if (sing || dn < 0.0) dc[0] = c1;
    if (sing) {
        dc[1] = dn;
        atomicAdd(&P.st->nsing, 1ull);
    }
}

// a supernode another GPU handles (split runs)
__device__ __forceinline__ bool node_off(const PV& P, int js) { return P.skip != nullptr && P.skip[js] != 0; }

__device__ __forceinline__ bool children_bad(const PV& P, int js) {
    for (int k = P.child_ptr[js]; k < P.child_ptr[js + 1]; ++k)
        if (P.sn_bad[P.child[k]]) return true;
    return false;
}

// ---------------------------------------------------------------------------
// Pre-pass: original diagonal, zero test, trace (sprfc1.f:465-488)
// ---------------------------------------------------------------------------
__global__ void k_prepass(PV P, int64_t nsuper) {
    const int lane = threadIdx.x & 31;
    for (int64_t js = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; js < nsuper;
         js += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int s = P.S[js], f = P.F[js], fst = P.fst[js];
        double* col = P.lnz + P.lnz_off[js];
        if (is_retained(P, js)) {                     // D stays 0 (sprfc1.f:463-467, sprfc3.f:551-554)
            for (int j = lane; j < s; j += 32) {
                P.adiag[fst + j] = 0.0;
                P.dvec[fst + j] = 0.0;
                if (P.fc3) {
                    P.dcor[2 * (int64_t)(fst + j)] = 0.0;
                    P.dcor[2 * (int64_t)(fst + j) + 1] = 0.0;
                }
            }
            continue;
        }
        for (int j = lane; j < s; j += 32) {
            double a = P.adiag_in ? P.adiag_in[fst + j] : col[lnz_col(j, f)];
            if (P.fc3) {                                  // sprfc3.f:561-572
                double* dc = P.dcor + 2 * (int64_t)(fst + j);
                dc[0] = 0.0;
                dc[1] = 0.0;
                if (a == 0.0) {
                    a = 1.0;
                    dc[1] = 1.0;
                    col[lnz_col(j, f)] = 1.0;
                }
                P.adiag[fst + j] = a;
                continue;
            }
            P.adiag[fst + j] = a;
            if (a == 0.0) {
                atomicAdd(&P.st->zero_count, 1);
                atomicMin(&P.st->first_zero, fst + j);
                atomicExch(&P.st->any_fail, 1);
            }
        }
    }
}

// Content hash of a device array (see smhash.h): each thread sums its words'
// mixes, the partial sums meet in one 64-bit atomic add (order-free).
__global__ void k_sm_hash(const double* a, int64_t n, unsigned long long* out) {
    unsigned long long acc = 0ull;
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += sm_mix(__ldcs(reinterpret_cast<const unsigned long long*>(w + i)), (uint64_t)i);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Deterministic single-CTA reductions over a vector: sum, or min over positives.
template <bool kMinPos>
__global__ void k_reduce(const double* v, int64_t n, double* out) {
    __shared__ double red[1024];
    double acc = kMinPos ? 0.0 : 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = v[i];
        if (kMinPos) {
            if (x > 0.0 && (acc == 0.0 || x < acc)) acc = x;
        } else {
            acc += x;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            const double a = red[threadIdx.x], b = red[threadIdx.x + s];
            if (kMinPos) {
                red[threadIdx.x] = (a == 0.0) ? b : ((b == 0.0) ? a : (a < b ? a : b));
            } else {
                red[threadIdx.x] = a + b;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// ---------------------------------------------------------------------------
// Small fronts: fused extend-add + LDL' + Schur update, one CTA per front.
// Shared memory holds the packed lower front F(F+1)/2 plus one column.
// ---------------------------------------------------------------------------
// Pivot rules of the factorisation kernels: SPRF17's |d| <= TOL(1)|a| stops
// (sprfc1.f:1274), SPRF37 replaces the pivot (sprfc3.f:1083), SPRF27's
// d <= TOL(1)|a| stops the Cholesky form (sprfc2.f:1001-1008; the C C'
// factor is formed from L D L' afterwards, see k_chol_convert).
// SPRF47 (sprfc4.f:978-1000) is the Cholesky form of SPRF37: a pivot below
// -TOL(1)|a_jj| stops, one in [-TOL(1)|a_jj|, TOL(1)|a_jj|] is replaced by
// TOL(1) max(1, |TOL(4) a_jj|) and recorded in DCOR(1:2, j).
enum PivotRule { kPivotLDL = 0, kPivotReplace = 1, kPivotChol = 2, kPivotChol4 = 3 };

// A NaN or infinite pivot (a NaN or Inf anywhere in SM reaches some pivot
// through the Schur updates) fails the test as well, so that the call reports
// an error instead of a factor full of NaN.
// 1/c for the pivots: the hardware reciprocal approximation (rcp.approx.ftz.f64)
// refined by two Newton-Raphson steps x <- x + x (1 - c x), each with fused
// multiply-adds; within one ulp of 1/c for normal c (tests compare it with
// the IEEE quotient 1.0 / c over many values).  Zero, subnormal, huge and
// non-finite c take the quotient itself.  It replaces a division on the
// pivot chain of every elimination step.
__device__ __forceinline__ double recip_nr(double c) {
    const double ac = fabs(c);
    if (!(ac >= 2.2250738585072014e-308 && ac <= 8.98846567431158e307)) return 1.0 / c;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(c));
    r = fma(r, fma(-c, r, 1.0), r);
    r = fma(r, fma(-c, r, 1.0), r);
    return r;
}

__global__ void k_recip_check(const double* x, int64_t n, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        out[2 * i] = recip_nr(x[i]);
        out[2 * i + 1] = 1.0 / x[i];
    }
}

__device__ __forceinline__ bool pivot_fails(int rule, double d, double ad, double tol1) {
    if (!isfinite(d)) return true;
    if (rule == kPivotChol4) return d < -tol1 * fabs(ad);
    return rule == kPivotChol ? d <= tol1 * fabs(ad) : fabs(d) <= tol1 * fabs(ad);
}

// SPRF47's replacement of a small pivot (not a failing one): returns the
// pivot to use and records DCOR(1,j) = d, DCOR(2,j) = the replacement.
__device__ __forceinline__ double chol4_pivot(const PV& P, int col, double d, double ad, bool record) {
    if (!(d <= P.tol1 * fabs(ad)) || d < -P.tol1 * fabs(ad)) return d;
    const double dn = P.tol1 * fmax(1.0, fabs(P.tol4 * ad));
    if (record) {
        P.dcor[2 * (int64_t)col] = d;
        P.dcor[2 * (int64_t)col + 1] = dn;
        atomicAdd(&P.st->nsing, 1ull);
    }
    return dn;
}

// SPRF47 on a failing (negative) pivot: DCOR(1,j) = DCOR(2,j) = d.
__device__ __forceinline__ void chol4_fail_record(const PV& P, int col, double d) {
    P.dcor[2 * (int64_t)col] = d;
    P.dcor[2 * (int64_t)col + 1] = d;
}

// Mixed-mode inertia guard: a pivot this close to zero relative to its
// original diagonal may have its sign decided by the TF32 rounding of the
// updates that formed it.
__device__ __forceinline__ bool near_zero_pivot(const PV& P, double d, double ad) {
    return P.near_tol > 0.0 && fabs(d) < P.near_tol * fabs(ad);
}

template <int PR>
__global__ void __launch_bounds__(256) k_small_front(const int32_t* nodes, PV P) {
    extern __shared__ double sh[];
    if (P.st->any_fail) return;
    const int js = nodes[blockIdx.x];
    if (node_off(P, js)) return;
    if (children_bad(P, js)) {
        if (threadIdx.x == 0) P.sn_bad[js] = 1;
        return;
    }
    const int F = P.F[js], S = P.S[js], fst = P.fst[js];
    const int npk = F * (F + 1) / 2;
    double* A = sh;
    double* wcol = sh + npk;
    double* rdk = wcol + F;                   // 1 / d_k of the S pivots
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    // fully-summed columns: the packed trapezoid of LNZ is the front's first SUPSZE entries
    const int supsze = F * S - (S * (S - 1)) / 2;
    const double* lnz = P.lnz + P.lnz_off[js];
    for (int i = tid; i < npk; i += blockDim.x) A[i] = (i < supsze) ? lnz[i] : 0.0;
    __syncthreads();
    // extend-add, children last sibling first (sprfc1.f:534-584)
    for (int k = P.child_ptr[js + 1] - 1; k >= P.child_ptr[js]; --k) {
        const int c = P.child[k];
        const int q = P.F[c] - P.S[c];
        if (q <= 0) continue;
        const int32_t* rel = P.rel + P.rel_off[c];
        const double* U = P.arena + P.upd_off[c];
        const int ld = P.buf_ld[c];
        for (int t = warp; t < q; t += nwarp) {
            const int pj = rel[t];
            const double* Ut = U + (int64_t)t * ld;
            int r = t + lane;
            for (; r + 32 < q; r += 64) {
                const int p0 = pk(rel[r], pj, F), p1 = pk(rel[r + 32], pj, F);
                const double u0 = __ldcg(Ut + r), u1 = __ldcg(Ut + r + 32);
                const double a0 = A[p0], a1 = A[p1];
                A[p0] = a0 + u0;
                A[p1] = a1 + u1;
            }
            if (r < q) A[pk(rel[r], pj, F)] += Ut[r];
        }
        __syncthreads();
    }
    // LDL' of the S fully-summed columns with the trailing (Schur) update;
    // a retained front is only assembled
    int neg = 0;
    double tmax = 0.0;
    bool failed = false;
    const bool ret = is_retained(P, js);
    for (int k = 0; k < (ret ? 0 : S); ++k) {
        double d = A[pk(k, k, F)];
        const double ad = P.adiag[fst + k];
        if (PR == kPivotReplace) {
            const double d0 = d;
            d = fc3_pivot(P, d0, ad);
            if (tid == 0) fc3_record(P, fst + k, d0, d);
        } else if (pivot_fails(PR, d, ad, P.tol1)) {   // sprfc1.f:1274, sprfc2.f:1004, sprfc4.f:980
            if (tid == 0) {
                record_fail(P, js, k, d, ad);
                if (PR == kPivotChol4) chol4_fail_record(P, fst + k, d);
            }
            failed = true;
            break;
        } else if (PR == kPivotChol4) {
            d = chol4_pivot(P, fst + k, d, ad, tid == 0);
        }
        if (d < 0.0) ++neg;
        if (tid == 0 && near_zero_pivot(P, d, ad)) atomicAdd(&P.st->near_piv, 1ull);
        tmax = fmax(tmax, ad / d);
        const double rd = recip_nr(d);
        if (tid == 0) rdk[k] = rd;
        // rows below the S columns stay unscaled until the trailing update
        for (int i = k + 1 + tid; i < F; i += blockDim.x) {
            const double a = A[pk(i, k, F)];
            wcol[i] = a;
            if (i < S) A[pk(i, k, F)] = a * rd;
        }
        __syncthreads();
        if ((PR == kPivotReplace || PR == kPivotChol4) && tid == 0) A[pk(k, k, F)] = d;   // every thread has read the old pivot
        // rank-1 update of the remaining fully-summed columns (all their rows)
        for (int j = k + 1 + warp; j < S; j += nwarp) {
            const double ljk = A[pk(j, k, F)];
            double* cj = A + pk(j, j, F) - j;
            // loads of four rows ahead of their stores (shared-memory latency overlaps)
            int i = j + lane;
            for (; i + 96 < F; i += 128) {
                const double a0 = cj[i], a1 = cj[i + 32], a2 = cj[i + 64], a3 = cj[i + 96];
                const double w0 = wcol[i], w1 = wcol[i + 32], w2 = wcol[i + 64], w3 = wcol[i + 96];
                cj[i] = a0 - w0 * ljk;
                cj[i + 32] = a1 - w1 * ljk;
                cj[i + 64] = a2 - w2 * ljk;
                cj[i + 96] = a3 - w3 * ljk;
            }
            for (; i < F; i += 32) cj[i] -= wcol[i] * ljk;
        }
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) {
            P.sn_neg[js] = neg;
            atomicAdd(&P.st->numneg, (unsigned long long)neg);
        }
        return;
    }
    if (!ret && S > 0 && S < F) {
        // The trailing (F-S)^2 block: each thread keeps 4x4 tiles in registers
        // and applies c -= w_ik (w_jk / d_k) for k = 0 .. S-1 in order, the
        // same operations in the same order as S rank-1 steps, with one
        // shared-memory read-modify-write per entry instead of S.
        const int q = F - S, nt = (q + 3) >> 2;
        const int ntiles = nt * (nt + 1) / 2;
        for (int t = tid; t < ntiles; t += blockDim.x) {
            int bi = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
            while (bi * (bi + 1) / 2 > t) --bi;
            while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
            const int bj = t - bi * (bi + 1) / 2;
            const int i0 = S + 4 * bi, j0 = S + 4 * bj;
            double c[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int i = i0 + a, j = j0 + b;
                    c[a][b] = (i < F && j <= i) ? A[pk(i, j, F)] : 0.0;
                }
            for (int k = 0; k < S; ++k) {
                const double r = rdk[k];
                const int base = pk(0, k, F);            // A[base + i] = entry (i, k), i >= k
                double w[4], l[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) w[a] = (i0 + a < F) ? A[base + i0 + a] : 0.0;
#pragma unroll
                for (int b = 0; b < 4; ++b) l[b] = ((j0 + b < F) ? A[base + j0 + b] : 0.0) * r;
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) c[a][b] -= w[a] * l[b];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int i = i0 + a, j = j0 + b;
                    if (i < F && j <= i) A[pk(i, j, F)] = c[a][b];
                }
        }
        __syncthreads();
        // and now the rows below the S columns to L
        for (int e = tid; e < S * q; e += blockDim.x) {
            const int k = e / q, i = S + e % q;
            A[pk(i, k, F)] *= rdk[k];
        }
        __syncthreads();
    }
    // write back the S columns (LNZ layout == packed layout) and the pivots
    double* lnzw = P.lnz + P.lnz_off[js];
    for (int i = tid; i < supsze; i += blockDim.x) lnzw[i] = A[i];
    if (!ret)
        for (int j = tid; j < S; j += blockDim.x) P.dvec[fst + j] = A[pk(j, j, F)];
    const int q = F - S;
    if (q > 0) {
        double* U = P.arena + P.upd_off[js];
        const int ld = P.buf_ld[js];
        for (int t = warp; t < q; t += nwarp)
            for (int r = t + lane; r < q; r += 32) U[r + (int64_t)t * ld] = A[pk(S + r, S + t, F)];
    }
    if (tid == 0) {
        P.sn_neg[js] = neg;
        atomicAdd(&P.st->numneg, (unsigned long long)neg);
        atomic_max_double(&P.st->tol2, tmax);
    }
}

// ---------------------------------------------------------------------------
// Large fronts
// ---------------------------------------------------------------------------

// A large front whose child failed (or depends on a failure) is skipped.
__global__ void k_poison(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const int js = jobs[j].node;
    if (!node_off(P, js) && children_bad(P, js)) P.sn_bad[js] = 1;
}

// Extend-add into a dense column-major front: one warp per front column.
// The column is built in chunks of kAsmRows rows in shared memory: the chunk
// starts as the LNZ column (fully-summed columns) or zero, receives the
// children's update entries whose parent rows fall into it (each child's rows
// are increasing in the parent, so a per-child cursor, kept in one lane,
// advances chunk by chunk), and is written once.  Each front entry is written
// once and each child entry read once, in the same order of additions as a
// column-at-a-time scatter (deterministic, no atomics).  A column with more
// than 32 contributions (one cursor per lane) scatters into HBM instead.
constexpr int kAsmRows = 256;

__device__ __forceinline__ void asm_scatter_column(const PV& P, double* col, int j, int F, int S, const double* src,
                                                   int64_t e0, int64_t e1, int lane) {
    if (j < S) {
        int i = j + lane;
        for (; i + 96 < F; i += 128) {
            const double a0 = __ldcg(src + i), a1 = __ldcg(src + i + 32), a2 = __ldcg(src + i + 64),
                         a3 = __ldcg(src + i + 96);
            col[i] = a0;
            col[i + 32] = a1;
            col[i + 64] = a2;
            col[i + 96] = a3;
        }
        for (; i < F; i += 32) col[i] = __ldcg(src + i);
    } else {
        for (int i = j + lane; i < F; i += 32) col[i] = 0.0;
    }
    __syncwarp();
    for (int64_t e = e0; e < e1; ++e) {
        const int c = P.cchild[e], t = P.ct[e];
        const int q = P.F[c] - P.S[c];
        const int32_t* rel = P.rel + P.rel_off[c];
        const double* U = P.arena + P.upd_off[c] + (int64_t)t * P.buf_ld[c];
        for (int r = t + lane; r < q; r += 32) col[rel[r]] += U[r];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) k_assemble(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks,
                                                  PV P) {
    __shared__ double chunk[8][kAsmRows];
    if (P.st->any_fail) return;
    const int lane = threadIdx.x & 31;
    const int64_t task = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int j = jb.c0 + (int)(task - jb.task0);
    const int F = P.F[js], S = P.S[js];
    const int ld = P.buf_ld[js];
    double* col = P.arena + P.buf_off[js] + (int64_t)j * ld;
    const double* src = (j < S) ? P.lnz + P.lnz_off[js] + lnz_col(j, F) - j : nullptr;
    const int64_t e0 = P.cptr[P.rbase[js] + j], e1 = P.cptr[P.rbase[js] + j + 1];
    const int ne = (int)(e1 - e0);
    if (ne > 32) {
        asm_scatter_column(P, col, j, F, S, src, e0, e1, lane);
        return;
    }
    // lane k holds contribution k: child, its update column, rows, cursor
    int my_c = 0, my_t = 0, my_q = 0, cur = 0;
    if (lane < ne) {
        my_c = P.cchild[e0 + lane];
        my_t = P.ct[e0 + lane];
        my_q = P.F[my_c] - P.S[my_c];
        cur = my_t;
    }
    double* acc = chunk[threadIdx.x >> 5];
    for (int lo = j; lo < F; lo += kAsmRows) {
        const int n = min(kAsmRows, F - lo), hi = lo + n;
        for (int i = lane; i < n; i += 32) acc[i] = src ? __ldcg(src + lo + i) : 0.0;
        __syncwarp();
        for (int k = 0; k < ne; ++k) {
            const int c = __shfl_sync(0xffffffffu, my_c, k);
            const int t = __shfl_sync(0xffffffffu, my_t, k);
            const int q = __shfl_sync(0xffffffffu, my_q, k);
            int r = __shfl_sync(0xffffffffu, cur, k);
            const int32_t* rel = P.rel + P.rel_off[c];
            const double* U = P.arena + P.upd_off[c] + (int64_t)t * P.buf_ld[c];
            for (;;) {
                // four 32-row steps with their loads first; the rows inside
                // [lo, hi) form a prefix (the parent rows increase)
                int ri[4];
                double u[4];
#pragma unroll
                for (int st = 0; st < 4; ++st) {
                    const int rr = r + 32 * st + lane;
                    ri[st] = rr < q ? __ldg(rel + rr) : 0x7fffffff;
                    u[st] = rr < q ? __ldcg(U + rr) : 0.0;
                }
                bool more = true;
#pragma unroll
                for (int st = 0; st < 4; ++st) {
                    if (!more) break;
                    const bool in = ri[st] < hi;
                    if (in) acc[ri[st] - lo] += u[st];
                    const unsigned m = __ballot_sync(0xffffffffu, in);
                    r += __popc(m);
                    more = (m == 0xffffffffu);
                }
                if (!more) break;
            }
            if (lane == k) cur = r;
            __syncwarp();
        }
        for (int i = lane; i < n; i += 32) col[lo + i] = acc[i];
        __syncwarp();
    }
}

// LDL' of one nb x nb diagonal block, pivot test / inertia / TOL(2) as
// SPRF17 (sprfc1.f:1272-1294).  256 threads on a 16x16 grid, each owning
// rows i = tx + 16a and columns j = ty + 16b of the block; right-looking with
// the unscaled column (a_ij -= a_ik * a_jk / d_k), scaled to L at the end.
// Also forms X = L11^-1 (unit lower) for the panel TRSM and the solves.
template <int PR>
__global__ void __launch_bounds__(256) k_diag(const Job* jobs, PV P) {
    // Register-resident: thread (tx, ty) keeps entries (tx + 16a, ty + 16b) of
    // the block in v[a][b] through the elimination and of X = L^-1 in x[a][b]
    // through the inverse; each step publishes one column of the block (or one
    // row of X) through shared memory, one barrier per step.  Entries outside
    // the lower triangle are carried along as don't-care values (never
    // published nor stored), which keeps the step free of per-entry tests.
    __shared__ double A[kNB][kNB + 1];      // L (lower, d on the diagonal)
    __shared__ double vec[2][kNB];          // the published column / row (double buffered)
    __shared__ double rdv[kNB];
    __shared__ double dd[kNB];
    __shared__ double adv[kNB];
    __shared__ double Tb[kNB * kNB / 4];    // T = L21 X11 of the inverse's doubling passes
    __shared__ int s_fail;
    if (P.st->any_fail) return;
    const Job& jb = jobs[blockIdx.x];
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int ld = P.buf_ld[js], fst = P.fst[js];
    double* front = P.arena + P.buf_off[js];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    constexpr int R = kNB / 16;
    double v[R][R];
#pragma unroll
    for (int b = 0; b < R; ++b)
#pragma unroll
        for (int a = 0; a < R; ++a) {
            const int i = tx + 16 * a, j = ty + 16 * b;
            v[a][b] = (i >= j && i < nb && j < nb) ? __ldcg(front + (int64_t)(k0 + i) + (int64_t)(k0 + j) * ld) : 0.0;
        }
    if (tid < nb) adv[tid] = __ldcg(P.adiag + fst + k0 + tid);
    for (int k = tid; k < 2 * kNB; k += blockDim.x) vec[k / kNB][k % kNB] = 0.0;
    __syncthreads();
    int failed = -1;
    // columns in groups of 16 (kb static inside a group, so the publishing
    // threads read their register v[a][kb] directly)
#pragma unroll
    for (int kb = 0; kb < R; ++kb) {
      if (16 * kb >= nb || failed >= 0) break;
      for (int kk = 0; kk < 16; ++kk) {
        const int k = 16 * kb + kk;
        if (k >= nb) break;
        const int buf = k & 1;
        if (ty == kk) {
#pragma unroll
            for (int a = 0; a < R; ++a) {
                const int i = tx + 16 * a;
                double c = v[a][kb];
                if (PR == kPivotReplace && i == k) {
                    const double c0 = c;
                    c = fc3_pivot(P, c0, adv[k]);
                    fc3_record(P, fst + k0 + k, c0, c);
                }
                if (PR == kPivotChol4 && i == k && !pivot_fails(PR, c, adv[k], P.tol1))
                    c = chol4_pivot(P, fst + k0 + k, c, adv[k], true);
                if (i >= k && i < nb) vec[buf][i] = c;
                if (i == k) {
                    dd[k] = c;
                    rdv[k] = recip_nr(c);
                }
            }
        }
        __syncthreads();
        const double d = vec[buf][k];
        // SPRFC4's rule records replacements while it goes, so it stops at a
        // failing pivot here; the other rules are tested after the loop (the
        // steps after a failure only compute values that are thrown away)
        if (PR == kPivotChol4 && pivot_fails(PR, d, adv[k], P.tol1)) {
            failed = k;
            if (tid == 0) {
                record_fail(P, js, k0 + k, d, adv[k]);
                chol4_fail_record(P, fst + k0 + k, d);
            }
            break;
        }
        const double rd = rdv[k];
        double vj[R];
#pragma unroll
        for (int b = 0; b < R; ++b) vj[b] = vec[buf][ty + 16 * b];
#pragma unroll
        for (int a = 0; a < R; ++a) {
            const double aik = vec[buf][tx + 16 * a] * rd;
#pragma unroll
            for (int b = 0; b < R; ++b)
                if (ty + 16 * b > k) v[a][b] -= aik * vj[b];
        }
      }
    }
    // the first failing pivot (sprfc1.f:1274-1279), for the rules tested here
    if (PR == kPivotLDL || PR == kPivotChol) {
        __syncthreads();
        if (tid < 32) {
            int f = nb;
            for (int k = tid; k < nb; k += 32)
                if (pivot_fails(PR, dd[k], adv[k], P.tol1)) f = min(f, k);
            for (int o = 16; o > 0; o >>= 1) f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
            if (tid == 0) {
                if (f < nb) record_fail(P, js, k0 + f, dd[f], adv[f]);
                s_fail = f;
            }
        }
        __syncthreads();
        failed = s_fail < nb ? s_fail : -1;
    }
    // inertia and TOL(2) of the processed columns (sprfc1.f:1280-1290)
    if (tid < 32) {
        const int kend = failed < 0 ? nb : failed;
        int neg = 0, near = 0;
        double tmax = 0.0;
        for (int k = tid; k < kend; k += 32) {
            if (dd[k] < 0.0) ++neg;
            if (near_zero_pivot(P, dd[k], adv[k])) ++near;
            tmax = fmax(tmax, adv[k] / dd[k]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            neg += __shfl_xor_sync(0xffffffffu, neg, o);
            near += __shfl_xor_sync(0xffffffffu, near, o);
            tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
        }
        if (tid == 0) {
            P.sn_neg[js] += neg;
            atomicAdd(&P.st->numneg, (unsigned long long)neg);
            if (near) atomicAdd(&P.st->near_piv, (unsigned long long)near);
            if (failed < 0) atomic_max_double(&P.st->tol2, tmax);
        }
    }
    if (failed >= 0) return;
    // L below the diagonal (scaled), d on it
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
            const int i = tx + 16 * a, j = ty + 16 * b;
            if (i >= j && i < nb && j < nb)
                A[i][j] = (i > j) ? v[a][b] * rdv[j] : ((PR == kPivotReplace || PR == kPivotChol4) ? dd[j] : v[a][b]);
        }
    __syncthreads();
    // X = L^-1 by recursive doubling: after the pass of order b, each aligned
    // diagonal block of X of order 2b is final, its lower-left quarter being
    // X21 = -X22 (L21 X11) (X11, X22 from the pass before; unit diagonals).
    // X is kept transposed in the free upper triangle of A (X[i][j] at A[j][i]),
    // T = L21 X11 in Tb; 12 barriers instead of one per column.
    // Each thread takes up to kInvQ elements of a pass and runs their sums side
    // by side (independent chains), each in the same order as one at a time.
    constexpr int kInvQ = kNB * kNB / 4 / 256;
    for (int b = 1; b < kNB; b <<= 1) {
        const int bb = b * b, tot = (kNB / (2 * b)) * bb;
        int e_[kInvQ], gi_[kInvQ], gj_[kInvQ], bs_[kInvQ], i_[kInvQ], j_[kInvQ];
        bool on[kInvQ];
        double t[kInvQ];
#pragma unroll
        for (int q = 0; q < kInvQ; ++q) {
            const int e = tid + q * (int)blockDim.x;
            const int kq = e / bb, r = e - kq * bb;
            e_[q] = e;
            i_[q] = r / b;
            j_[q] = r - i_[q] * b;
            bs_[q] = 2 * kq * b;
            gi_[q] = bs_[q] + b + i_[q];
            gj_[q] = bs_[q] + j_[q];
            on[q] = e < tot && gi_[q] < nb;
            t[q] = on[q] ? A[gi_[q]][gj_[q]] : 0.0;                // X11[j][j] = 1
        }
        for (int m = 1; m < b; ++m)
#pragma unroll
            for (int q = 0; q < kInvQ; ++q)                            // L21[i][m] X11[m][j], m > j
                if (on[q] && m > j_[q]) t[q] += A[gi_[q]][bs_[q] + m] * A[gj_[q]][bs_[q] + m];
#pragma unroll
        for (int q = 0; q < kInvQ; ++q)
            if (e_[q] < tot) Tb[e_[q]] = t[q];
        __syncthreads();
        double x[kInvQ];
#pragma unroll
        for (int q = 0; q < kInvQ; ++q) x[q] = e_[q] < tot ? Tb[e_[q]] : 0.0;   // X22[i][i] = 1
        for (int m = 0; m + 1 < b; ++m)
#pragma unroll
            for (int q = 0; q < kInvQ; ++q)                            // X22[i][m] T[m][j], m < i
                if (e_[q] < tot && m < i_[q])
                    x[q] += A[bs_[q] + b + m][gi_[q]] * Tb[(e_[q] / bb) * bb + m * b + j_[q]];
#pragma unroll
        for (int q = 0; q < kInvQ; ++q)
            if (e_[q] < tot) A[bs_[q] + j_[q]][gi_[q]] = -x[q];
        __syncthreads();
    }
    double* lv = P.linv + P.linv_off[js] + (int64_t)(k0 / kNB) * kNB * kNB;
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        const int i = e % kNB, j = e / kNB;
        lv[e] = (i < nb && j < nb) ? (i > j ? A[j][i] : (i == j ? 1.0 : 0.0)) : 0.0;
    }
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
        for (int b = 0; b < R; ++b) {
            const int i = tx + 16 * a, j = ty + 16 * b;
            if (i >= j && i < nb && j < nb) front[(int64_t)(k0 + i) + (int64_t)(k0 + j) * ld] = A[i][j];
        }
    if (tid < nb) P.dvec[fst + k0 + tid] = A[tid][tid];
}

namespace gemm {
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}
}  // namespace gemm

// Panel TRSM as a product with the stored inverse: for a 64-row block of the
// rows below the diagonal block, W = A21 X' (X = L11^-1), L21 = W D^-1.
// 128 threads = 2x2 warps of 32x32 DMMA tiles; the block is read completely
// into shared memory before it is overwritten, so the update is in place.
constexpr int kTrsmLds = kNB + 4;
constexpr size_t kTrsmSmem = sizeof(double) * (2 * (size_t)kNB * kTrsmLds + kNB);

__global__ void __launch_bounds__(128) k_trsm(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P) {
    extern __shared__ double tsh[];
    double(*As)[kTrsmLds] = reinterpret_cast<double(*)[kTrsmLds]>(tsh);              // As[m][i]
    double(*Xs)[kTrsmLds] = reinterpret_cast<double(*)[kTrsmLds]>(tsh + kNB * kTrsmLds);  // Xs[m][c] = X[c][m]
    double* rd = tsh + 2 * kNB * kTrsmLds;
    if (P.st->any_fail) return;
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int F = P.F[js], ld = P.buf_ld[js];
    const int r0 = jb.c0 + (int)(task - jb.task0) * kTRSMRows;
    double* front = P.arena + P.buf_off[js];
    const double* lv = P.linv + P.linv_off[js] + (int64_t)(k0 / kNB) * kNB * kNB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // loads in groups of 8 per thread before their shared-memory stores
    for (int e0 = 0; e0 < kNB * kNB; e0 += 8 * 128) {
        double av[8], xv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * 128 + tid;
            const int i = e % kNB, m = e / kNB;
            av[u] = (m < nb && r0 + i < F) ? __ldcg(front + (int64_t)(r0 + i) + (int64_t)(k0 + m) * ld) : 0.0;
            xv[u] = __ldcg(lv + i + m * kNB);          // X[i][m]: row i (output column), col m
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * 128 + tid;
            As[e / kNB][e % kNB] = av[u];
            Xs[e / kNB][e % kNB] = xv[u];
        }
    }
    for (int c = tid; c < kNB; c += blockDim.x)
        rd[c] = (c < nb) ? 1.0 / front[(int64_t)(k0 + c) * (ld + 1)] : 0.0;
    __syncthreads();
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll 4
    for (int k4 = 0; k4 < kNB; k4 += 4) {
        const int kk = k4 + (lane & 3);
        double av[4], bv[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) av[mi] = As[kk][wm + mi * 8 + (lane >> 2)];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) bv[ni] = Xs[kk][wn + ni * 8 + (lane >> 2)];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) gemm::dmma(acc[mi][ni][0], acc[mi][ni][1], av[mi], bv[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
        const int r = r0 + wm + mi * 8 + (lane >> 2);
        if (r >= F) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = wn + ni * 8 + 2 * (lane & 3) + h;
                if (c < nb) front[(int64_t)r + (int64_t)(k0 + c) * ld] = acc[mi][ni][h] * rd[c];
            }
    }
}

// Inverse of the unit-lower diagonal blocks straight from LNZ (used when the
// factor in SM was not produced by this engine, e.g. a solve-only call).
__global__ void __launch_bounds__(64) k_linv(const Job* jobs, PV P) {
    __shared__ double L[kNB][kNB + 1];      // L strictly lower, X = L^-1 transposed above
    const Job& jb = jobs[blockIdx.x];
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    const int F = P.F[js];
    const double* base = P.lnz + P.lnz_off[js];
    const int tid = threadIdx.x;
    for (int e = tid; e < nb * nb; e += blockDim.x) {
        const int i = e % nb, j = e / nb;
        if (i > j) L[i][j] = base[lnz_col(k0 + j, F) - (k0 + j) + (k0 + i)];
    }
    __syncthreads();
    if (tid < nb) {
        const int j = tid;
        for (int i = j + 1; i < nb; ++i) {
            double acc = -L[i][j];
            for (int m = j + 1; m < i; ++m) acc -= L[i][m] * L[j][m];
            L[j][i] = acc;
        }
    }
    __syncthreads();
    double* lv = P.linv + P.linv_off[js] + (int64_t)(k0 / kNB) * kNB * kNB;
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        const int i = e % kNB, j = e / kNB;
        lv[e] = (i < nb && j < nb) ? (i > j ? L[j][i] : (i == j ? 1.0 : 0.0)) : 0.0;
    }
}

// Schur update C -= L D L' on T x T lower-triangle tiles with FP64 DMMA
// (mma.sync m8n8k4 f64).  A = rows i of L scaled by D (the scaling is applied
// to the A fragments), B = rows j of L, both read from the front buffer.
// Warps of WM x WN; K is staged through shared memory in 16-wide slices with
// a STAGES-deep cp.async pipeline (16-byte copies of row pairs).
namespace gemm {
constexpr int BK = 16;

__device__ __forceinline__ void cp_async16(double* dst, const double* src, int bytes) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    const int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int T, int WM, int WN, int STAGES>
struct Cfg {
    static constexpr int NWM = T / WM, NWN = T / WN, NT = NWM * NWN * 32;
    static constexpr int LDS = T + 4;                       // bank-conflict-free fragment reads
    static constexpr int MI = WM / 8, NI = WN / 8;
    static constexpr size_t smem = sizeof(double) * ((size_t)2 * STAGES * BK * LDS + (size_t)STAGES * BK);
};
}  // namespace gemm

template <int T, int WM, int WN, int STAGES>
__global__ void __launch_bounds__(gemm::Cfg<T, WM, WN, STAGES>::NT)
k_gemm(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P) {
    using namespace gemm;
    using C = Cfg<T, WM, WN, STAGES>;
    extern __shared__ __align__(16) double gsh[];
    double* As = gsh;                                // [STAGES][BK][LDS]
    double* Bs = As + STAGES * BK * C::LDS;
    double* Ds = Bs + STAGES * BK * C::LDS;         // [STAGES][BK]
    if (P.st->any_fail) return;
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int ld = P.buf_ld[js];
    // decode the lower-triangle tile (column tile jt, row tile it >= jt)
    const int64_t u = task - jb.task0;
    const int nct = (jb.c_end - jb.c0 + T - 1) / T;
    const int nr = (jb.r_end - jb.c0 + T - 1) / T;
    int lo = 0, hi = nct - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t pre = (int64_t)mid * nr - ((int64_t)mid * (mid - 1)) / 2;
        if (pre <= u) lo = mid;
        else hi = mid - 1;
    }
    const int jt = lo;
    const int it = jt + (int)(u - ((int64_t)jt * nr - ((int64_t)jt * (jt - 1)) / 2));
    const int i0 = jb.c0 + it * T, j0 = jb.c0 + jt * T;
    const int r_end = jb.r_end, c_end = jb.c_end;
    const double* front = P.arena + P.buf_off[js];
    double* frontw = P.arena + P.buf_off[js];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp % C::NWM) * WM, wn = (warp / C::NWM) * WN;

    double acc[C::MI][C::NI][2];
#pragma unroll
    for (int a = 0; a < C::MI; ++a)
#pragma unroll
        for (int b = 0; b < C::NI; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    const int k_lo = jb.k_lo, k_hi = jb.k_hi;
    const int nk = (k_hi - k_lo + BK - 1) / BK;
    // 16-byte copies need an even first row (the buffer base and ld are
    // 32-byte multiples); tiles of jobs starting on an odd column use 8 bytes
    const bool even = ((i0 | j0) & 1) == 0;
    auto load_stage = [&](int stage, int kt) {
        const int kb = k_lo + kt * BK;
        double* as = As + stage * BK * C::LDS;
        double* bs = Bs + stage * BK * C::LDS;
#pragma unroll
        for (int e = 0; e < (T / 2 * BK + C::NT - 1) / C::NT; ++e) {
            const int idx = tid + e * C::NT;
            if (idx < T / 2 * BK) {
                const int pr = idx % (T / 2), k = idx / (T / 2);
                const int r = 2 * pr, kk = kb + k;
                const bool kv = kk < k_hi;
                const int64_t col = (int64_t)(kv ? kk : k_lo) * ld;
                const int ra = i0 + r, rb = j0 + r;
                const int na = kv ? max(0, min(2, r_end - ra)) : 0;
                const int nbb = kv ? max(0, min(2, r_end - rb)) : 0;
                if (even) {
                    cp_async16(as + k * C::LDS + r, front + col + (na > 0 ? ra : i0), 8 * na);
                    cp_async16(bs + k * C::LDS + r, front + col + (nbb > 0 ? rb : j0), 8 * nbb);
                } else {
                    cp_async8(as + k * C::LDS + r, front + col + (na > 0 ? ra : i0), na > 0);
                    cp_async8(as + k * C::LDS + r + 1, front + col + (na > 1 ? ra + 1 : i0), na > 1);
                    cp_async8(bs + k * C::LDS + r, front + col + (nbb > 0 ? rb : j0), nbb > 0);
                    cp_async8(bs + k * C::LDS + r + 1, front + col + (nbb > 1 ? rb + 1 : j0), nbb > 1);
                }
            }
        }
        if (tid < BK) {
            const int kk = kb + tid;
            cp_async8(Ds + stage * BK + tid, front + (int64_t)(kk < k_hi ? kk : k_lo) * (ld + 1), kk < k_hi);
        }
    };

#pragma unroll
    for (int st = 0; st < STAGES - 1; ++st) {
        if (st < nk) load_stage(st, st);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nxt = kt + STAGES - 1;
        if (nxt < nk) load_stage(nxt % STAGES, nxt);
        cp_async_commit();
        const int cur = kt % STAGES;
        const double* as = As + cur * BK * C::LDS;
        const double* bs = Bs + cur * BK * C::LDS;
        const double* ds = Ds + cur * BK;
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            const int kk = k4 + (lane & 3);
            const double dk = ds[kk];
            double a[C::MI], b[C::NI];
#pragma unroll
            for (int mi = 0; mi < C::MI; ++mi) a[mi] = as[kk * C::LDS + wm + mi * 8 + (lane >> 2)] * dk;
#pragma unroll
            for (int ni = 0; ni < C::NI; ++ni) b[ni] = bs[kk * C::LDS + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
                for (int ni = 0; ni < C::NI; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
    }
    cp_async_wait<0>();
    // epilogue: C -= acc on the lower part, inside [.., r_end) x [.., c_end);
    // in two halves of the warp tile, each with its loads ahead of its
    // stores, so that the loads overlap instead of waiting one latency each
    constexpr int MH = C::MI > 1 ? C::MI / 2 : 1;
#pragma unroll
    for (int m0 = 0; m0 < C::MI; m0 += MH) {
        double cv[MH][C::NI][2];
#pragma unroll
        for (int q = 0; q < MH; ++q) {
            const int r = i0 + wm + (m0 + q) * 8 + (lane >> 2);
#pragma unroll
            for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = j0 + wn + ni * 8 + 2 * (lane & 3) + h;
                    cv[q][ni][h] =
                        (r < r_end && c < c_end && r >= c) ? __ldcg(front + (int64_t)r + (int64_t)c * ld) : 0.0;
                }
        }
#pragma unroll
        for (int q = 0; q < MH; ++q) {
            const int r = i0 + wm + (m0 + q) * 8 + (lane >> 2);
            if (r >= r_end) continue;
#pragma unroll
            for (int ni = 0; ni < C::NI; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = j0 + wn + ni * 8 + 2 * (lane & 3) + h;
                    if (c < c_end && r >= c)
                        frontw[(int64_t)r + (int64_t)c * ld] = cv[q][ni][h] - acc[m0 + q][ni][h];
                }
        }
    }
}

#ifndef SPR_GEMM_BIG_WM
#define SPR_GEMM_BIG_WM 32
#endif
#ifndef SPR_GEMM_BIG_WN
#define SPR_GEMM_BIG_WN 32
#endif
#ifndef SPR_GEMM_STAGES
#define SPR_GEMM_STAGES 3
#endif
using GemmBig = gemm::Cfg<kTileBig, SPR_GEMM_BIG_WM, SPR_GEMM_BIG_WN, SPR_GEMM_STAGES>;
using GemmSmall = gemm::Cfg<kTile, 32, 32, SPR_GEMM_STAGES>;
using GemmTiny = gemm::Cfg<kTileTiny, 16, 16, SPR_GEMM_STAGES>;
#define K_GEMM_BIG k_gemm<kTileBig, SPR_GEMM_BIG_WM, SPR_GEMM_BIG_WN, SPR_GEMM_STAGES>
#define K_GEMM_SMALL k_gemm<kTile, 32, 32, SPR_GEMM_STAGES>
#define K_GEMM_TINY k_gemm<kTileTiny, 16, 16, SPR_GEMM_STAGES>

// Mixed-precision Schur update: C -= L D L' with 3xTF32 split products on
// the tensor cores (mma.sync m16n8k8 tf32, FP32 accumulation inside each
// 64-wide slice of K, FP64 accumulation across slices and in C).  Each FP64
// operand a is rounded to FP32, then split a = hi + lo with hi = tf32(a),
// lo = tf32(a - hi); the product uses hi*hi + hi*lo + lo*hi.
namespace x3 {
__device__ __forceinline__ uint32_t tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split(double v, uint32_t& hi, uint32_t& lo) {
    const float f = (float)v;
    hi = tf32(f);
    lo = tf32(f - __uint_as_float(hi));
}
__device__ __forceinline__ void mma(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
}  // namespace x3

#include "tc_gemm.cuh"

__global__ void __launch_bounds__(128) k_gemm_x3(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P) {
    using namespace gemm;
    constexpr int T = kTile, STAGES = 3, LDS = T + 4;
    extern __shared__ __align__(16) double gsh[];
    double* As = gsh;
    double* Bs = As + STAGES * BK * LDS;
    double* Ds = Bs + STAGES * BK * LDS;
    if (P.st->any_fail) return;
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int ld = P.buf_ld[js];
    const int64_t u = task - jb.task0;
    const int nct = (jb.c_end - jb.c0 + T - 1) / T;
    const int nr = (jb.r_end - jb.c0 + T - 1) / T;
    int lo = 0, hi = nct - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t pre = (int64_t)mid * nr - ((int64_t)mid * (mid - 1)) / 2;
        if (pre <= u) lo = mid;
        else hi = mid - 1;
    }
    const int jt = lo;
    const int it = jt + (int)(u - ((int64_t)jt * nr - ((int64_t)jt * (jt - 1)) / 2));
    const int i0 = jb.c0 + it * T, j0 = jb.c0 + jt * T;
    const int r_end = jb.r_end, c_end = jb.c_end;
    const double* front = P.arena + P.buf_off[js];
    double* frontw = P.arena + P.buf_off[js];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    float acc[2][4][4];
    double acc64[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                acc[a][b][c] = 0.f;
                acc64[a][b][c] = 0.0;
            }
    const int k_lo = jb.k_lo, k_hi = jb.k_hi;
    const int nk = (k_hi - k_lo + BK - 1) / BK;
    const bool even = ((i0 | j0) & 1) == 0;
    auto load_stage = [&](int stage, int kt) {
        const int kb = k_lo + kt * BK;
        double* as = As + stage * BK * LDS;
        double* bs = Bs + stage * BK * LDS;
#pragma unroll
        for (int e = 0; e < (T / 2 * BK + 127) / 128; ++e) {
            const int idx = tid + e * 128;
            if (idx < T / 2 * BK) {
                const int pr = idx % (T / 2), k = idx / (T / 2);
                const int r = 2 * pr, kk = kb + k;
                const bool kv = kk < k_hi;
                const int64_t col = (int64_t)(kv ? kk : k_lo) * ld;
                const int ra = i0 + r, rb = j0 + r;
                const int na = kv ? max(0, min(2, r_end - ra)) : 0;
                const int nbb = kv ? max(0, min(2, r_end - rb)) : 0;
                if (even) {
                    cp_async16(as + k * LDS + r, front + col + (na > 0 ? ra : i0), 8 * na);
                    cp_async16(bs + k * LDS + r, front + col + (nbb > 0 ? rb : j0), 8 * nbb);
                } else {
                    cp_async8(as + k * LDS + r, front + col + (na > 0 ? ra : i0), na > 0);
                    cp_async8(as + k * LDS + r + 1, front + col + (na > 1 ? ra + 1 : i0), na > 1);
                    cp_async8(bs + k * LDS + r, front + col + (nbb > 0 ? rb : j0), nbb > 0);
                    cp_async8(bs + k * LDS + r + 1, front + col + (nbb > 1 ? rb + 1 : j0), nbb > 1);
                }
            }
        }
        if (tid < BK) {
            const int kk = kb + tid;
            cp_async8(Ds + stage * BK + tid, front + (int64_t)(kk < k_hi ? kk : k_lo) * (ld + 1), kk < k_hi);
        }
    };
#pragma unroll
    for (int st = 0; st < STAGES - 1; ++st) {
        if (st < nk) load_stage(st, st);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nxt = kt + STAGES - 1;
        if (nxt < nk) load_stage(nxt % STAGES, nxt);
        cp_async_commit();
        const int cur = kt % STAGES;
        const double* as = As + cur * BK * LDS;
        const double* bs = Bs + cur * BK * LDS;
        const double* ds = Ds + cur * BK;
#pragma unroll
        for (int k8 = 0; k8 < BK; k8 += 8) {
            const double d0 = ds[k8 + t], d1 = ds[k8 + t + 4];
            uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int r0 = wm + mi * 16 + g;
                x3::split(as[(k8 + t) * LDS + r0] * d0, ah[mi][0], al[mi][0]);
                x3::split(as[(k8 + t) * LDS + r0 + 8] * d0, ah[mi][1], al[mi][1]);
                x3::split(as[(k8 + t + 4) * LDS + r0] * d1, ah[mi][2], al[mi][2]);
                x3::split(as[(k8 + t + 4) * LDS + r0 + 8] * d1, ah[mi][3], al[mi][3]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int c = wn + ni * 8 + g;
                x3::split(bs[(k8 + t) * LDS + c], bh[ni][0], bl[ni][0]);
                x3::split(bs[(k8 + t + 4) * LDS + c], bh[ni][1], bl[ni][1]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) {
                    x3::mma(acc[mi][ni], al[mi], bh[ni][0], bh[ni][1]);
                    x3::mma(acc[mi][ni], ah[mi], bl[ni][0], bl[ni][1]);
                    x3::mma(acc[mi][ni], ah[mi], bh[ni][0], bh[ni][1]);
                }
        }
        if ((kt & 3) == 3 || kt == nk - 1) {           // FP64 accumulation across 64-wide K slices
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        acc64[a][b][c] += (double)acc[a][b][c];
                        acc[a][b][c] = 0.f;
                    }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = i0 + wm + mi * 16 + g + 8 * h;
            if (r >= r_end) continue;
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int c = j0 + wn + ni * 8 + 2 * t + q;
                    if (c < c_end && r >= c) frontw[(int64_t)r + (int64_t)c * ld] -= acc64[mi][ni][2 * h + q];
                }
        }
}

// Store the S factored columns of a dense front into LNZ (sprfc1.f:630-637).
__global__ void k_writeback(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P) {
    if (P.st->any_fail) return;
    const int lane = threadIdx.x & 31;
    const int64_t task = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (P.sn_bad[js] || node_off(P, js)) return;
    const int j = jb.c0 + (int)(task - jb.task0);
    const int F = P.F[js], ld = P.buf_ld[js];
    const double* col = P.arena + P.buf_off[js] + (int64_t)j * ld;
    double* dst = P.lnz + P.lnz_off[js] + lnz_col(j, F) - j;
    int i = j + lane;
    for (; i + 96 < F; i += 128) {
        const double a0 = __ldcg(col + i), a1 = __ldcg(col + i + 32), a2 = __ldcg(col + i + 64),
                     a3 = __ldcg(col + i + 96);
        dst[i] = a0;
        dst[i + 32] = a1;
        dst[i + 64] = a2;
        dst[i + 96] = a3;
    }
    for (; i < F; i += 32) dst[i] = col[i];
}

// ---------------------------------------------------------------------------
// Solves (multi-RHS), one CTA per front, level by level.
// Front vectors live in vbuf: front p uses F_p x nrhs doubles at rbase[p]*nrhs
// (column r at offset r*F_p).  After the forward sweep, rows S..F of a front
// vector are its update vector for the parent.
// ---------------------------------------------------------------------------
constexpr int kSolveThreads = 256;
// threads of a one-CTA-per-front launch (factor or solve) of a size class:
// the smallest fronts take 128, so that twice as many fronts are in flight
// per SM (their shared memory allows it)
inline int small_threads(int maxF) { return maxF <= 64 ? 128 : 256; }

// Small fronts (F <= kSmallMaxF): the front vector and one 32-column block of
// L live in shared memory; per block, one warp solves the 32x32 triangle and
// all threads apply the block to the rows below it (3 barriers per block).
constexpr int kSmallBlk = 32;
constexpr size_t kSmallSolveSmem = sizeof(double) * ((size_t)kSmallMaxF * kMaxRHS + (size_t)kSmallMaxF * (kSmallBlk + 1));
// shared memory of one small-front solve CTA: the front vector (F x nrhs) and
// one 32-column block of L (F x 33)
inline size_t small_solve_smem(int maxF, int nrhs) {
    return sizeof(double) * ((size_t)maxF * nrhs + (size_t)maxF * (kSmallBlk + 1));
}

__global__ void __launch_bounds__(kSolveThreads)
k_forward(const int32_t* nodes, PV P, double* vbuf, double* b, int64_t ldb, int nrhs) {
    extern __shared__ double wsm[];           // w[i * nrhs + r], then Ls[(i - j0) * (kSmallBlk + 1) + c]
    const int js = nodes[blockIdx.x];
    if (node_off(P, js)) return;
    const int F = P.F[js], S = P.S[js], fst = P.fst[js];
    double* Ls = wsm + (size_t)F * nrhs;
    double* wg = vbuf + P.rbase[js] * nrhs;   // update rows for the parent (r*F + i)
    const double* Lb = P.lnz + P.lnz_off[js];
    const int tid = threadIdx.x, lane = tid & 31;
    for (int e = tid; e < F * nrhs; e += blockDim.x) {
        const int i = e % F, r = e / F;
        double v = (i < S) ? b[(int64_t)(fst + i) + r * ldb] : 0.0;
        const int64_t e0 = P.cptr[P.rbase[js] + i], e1 = P.cptr[P.rbase[js] + i + 1];
        for (int64_t q = e0; q < e1; ++q) {
            const int c = P.cchild[q], t = P.ct[q];
            v += vbuf[P.rbase[c] * nrhs + (int64_t)r * P.F[c] + P.S[c] + t];
        }
        wsm[i * nrhs + r] = v;
    }
    // a retained front only passes its sums on (own rows to B, the rest to the parent)
    const bool ret = is_retained(P, js);
    for (int j0 = 0; j0 < (ret ? 0 : S); j0 += kSmallBlk) {
        const int nb = min(kSmallBlk, S - j0), m = F - j0;
        for (int e = tid; e < m * nb; e += blockDim.x) {
            const int i = e % m, c = e / m;
            Ls[i * (kSmallBlk + 1) + c] = (i > c) ? Lb[lnz_col(j0 + c, F) - (j0 + c) + (j0 + i)] : 0.0;
        }
        __syncthreads();
        // triangle of the block (SPRFS5 :600-608): a warp per right-hand side,
        // lane i holding y_i; y_c reaches the lanes below it by a shuffle
        for (int r = tid >> 5; r < nrhs; r += (int)(blockDim.x >> 5)) {
            double yi = lane < nb ? wsm[(j0 + lane) * nrhs + r] : 0.0;
            for (int c = 0; c < nb - 1; ++c) {
                const double yc = __shfl_sync(0xffffffffu, yi, c);
                if (lane > c && lane < nb) yi -= yc * Ls[lane * (kSmallBlk + 1) + c];
            }
            if (lane < nb) wsm[(j0 + lane) * nrhs + r] = yi;
        }
        __syncthreads();
        for (int e = tid; e < (m - nb) * nrhs; e += blockDim.x) {   // rectangle (SPRFS6)
            const int i = nb + e % (m - nb), r = e / (m - nb);
            double v = wsm[(j0 + i) * nrhs + r];
            for (int c = 0; c < nb; ++c) v -= Ls[i * (kSmallBlk + 1) + c] * wsm[(j0 + c) * nrhs + r];
            wsm[(j0 + i) * nrhs + r] = v;
        }
        __syncthreads();
    }
    for (int e = tid; e < F * nrhs; e += blockDim.x) {
        const int i = e % F, r = e / F;
        if (i < S) b[(int64_t)(fst + i) + r * ldb] = ret ? wsm[i * nrhs + r] : wsm[i * nrhs + r] / Lb[lnz_col(i, F)];
        else wg[(int64_t)r * F + i] = wsm[i * nrhs + r];
    }
}

__global__ void __launch_bounds__(kSolveThreads)
k_backward(const int32_t* nodes, PV P, double* vbuf, double* b, int64_t ldb, int nrhs) {
    extern __shared__ double wsm[];
    const int js = nodes[blockIdx.x];
    if (node_off(P, js)) return;
    if (is_retained(P, js)) return;
    const int F = P.F[js], S = P.S[js], fst = P.fst[js];
    double* Ls = wsm + (size_t)F * nrhs;
    const double* Lb = P.lnz + P.lnz_off[js];
    const int tid = threadIdx.x, lane = tid & 31;
    (void)vbuf;
    // own rows (forward result) and the ancestors' solved rows; the row list
    // of front js starts at rbase[js] (LINDX concatenates the row lists)
    for (int e = tid; e < F * nrhs; e += blockDim.x) {
        const int i = e % F, r = e / F;
        const int row = (i < S) ? (fst + i) : P.rows[P.rbase[js] + i];
        wsm[i * nrhs + r] = b[(int64_t)row + r * ldb];
    }
    const int nblk = (S + kSmallBlk - 1) / kSmallBlk;
    for (int bi = nblk - 1; bi >= 0; --bi) {
        const int j0 = bi * kSmallBlk, nb = min(kSmallBlk, S - j0), m = F - j0;
        __syncthreads();
        for (int e = tid; e < m * nb; e += blockDim.x) {
            const int i = e % m, c = e / m;
            Ls[i * (kSmallBlk + 1) + c] = (i > c) ? Lb[lnz_col(j0 + c, F) - (j0 + c) + (j0 + i)] : 0.0;
        }
        __syncthreads();
        for (int e = tid; e < nb * nrhs; e += blockDim.x) {         // rows below the block (SPRBS6)
            const int c = e % nb, r = e / nb;
            double v = 0.0;
            for (int i = nb; i < m; ++i) v += Ls[i * (kSmallBlk + 1) + c] * wsm[(j0 + i) * nrhs + r];
            wsm[(j0 + c) * nrhs + r] -= v;
        }
        __syncthreads();
        // triangle of the block, bottom-up: a warp per right-hand side, lane c
        // holding x_c; each finished x_i is shuffled to the lanes above it
        for (int r = tid >> 5; r < nrhs; r += (int)(blockDim.x >> 5)) {
            double xc = lane < nb ? wsm[(j0 + lane) * nrhs + r] : 0.0;
            for (int i = nb - 1; i > 0; --i) {
                const double xi = __shfl_sync(0xffffffffu, xc, i);
                if (lane < i) xc -= Ls[i * (kSmallBlk + 1) + lane] * xi;
            }
            if (lane < nb) wsm[(j0 + lane) * nrhs + r] = xc;
        }
    }
    __syncthreads();
    for (int e = tid; e < S * nrhs; e += blockDim.x) {
        const int i = e % S, rr = e / S;
        b[(int64_t)(fst + i) + rr * ldb] = wsm[i * nrhs + rr];
    }
}

// ---------------------------------------------------------------------------
// Solves of the large fronts: batched like the factorisation, one launch per
// panel step for all large fronts of a level.  L is read from LNZ (packed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ const double* lcol(const PV& P, int js, int F, int j) {
    return P.lnz + P.lnz_off[js] + lnz_col(j, F) - j;      // index with the row
}

// gather of the forward sweep: own rows of B plus the children's update vectors
__global__ void k_fwd_gather(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, double* vbuf,
                             const double* b, int64_t ldb, int nrhs) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int i = (int)(task - jb.task0);
    const int F = P.F[js], S = P.S[js], fst = P.fst[js];
    double* w = vbuf + P.rbase[js] * nrhs;
    const int64_t e0 = P.cptr[P.rbase[js] + i], e1 = P.cptr[P.rbase[js] + i + 1];
    for (int r = 0; r < nrhs; ++r) {
        double v = (i < S) ? b[(int64_t)(fst + i) + r * ldb] : 0.0;
        for (int64_t e = e0; e < e1; ++e) {
            const int c = P.cchild[e], t = P.ct[e];
            v += vbuf[P.rbase[c] * nrhs + (int64_t)r * P.F[c] + P.S[c] + t];
        }
        w[(int64_t)r * F + i] = v;
    }
}

// Solve steps of kSolveBlock (256) columns.  Forward: one CTA per front
// solves the block's unit-lower triangle (4 diagonal blocks of 64, each a
// product with its stored inverse X, then the rows below it inside the
// block), stores the block in ysol; then k_fwd_blk_upd applies it to every
// row below the block (thread per row, SPRFS6).  Backward mirrors it.

// w[m] -= sum_{c < n} L[row0 + c, m] x[c][.] by one warp (column m of L contiguous)
// Reduce-scatter of NR per-lane partial sums over a warp: halving exchanges
// (NR/2 + NR/4 + ... shuffles) then full sums over the remaining lane bits.
// Returns the total of partial index `rhs`; the lanes whose remaining bits
// are zero (lane & (first_rem * 2 - 1)) == 0 hold distinct totals.
template <int NR>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[NR], int lane, int& rhs, int& owner_mask) {
    int base = 0, o = 16;
#pragma unroll
    for (int h = NR / 2; h >= 1; h >>= 1, o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < h; ++j) {
            const double send = up ? v[j] : v[j + h];
            const double keep = up ? v[j + h] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
        if (up) base += h;
    }
    owner_mask = 2 * o - 1;
#pragma unroll
    for (; o >= 1; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    rhs = base;
    return v[0];
}

__device__ __forceinline__ void warp_col_dot_smem(const double* cm_row0, int n, const double (*x)[kSolveBlock],
                                                  double* wm, int64_t F, int nrhs) {
    const int lane = threadIdx.x & 31;
    double acc[kMaxRHS];
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r) acc[r] = 0.0;
    for (int c = lane; c < n; c += 32) {
        const double l = cm_row0[c];
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r)
            if (r < nrhs) acc[r] += l * x[r][c];
    }
    int r, om;
    const double v = warp_reduce_scatter<kMaxRHS>(acc, lane, r, om);
    if ((lane & om) == 0 && r < nrhs) wm[(int64_t)r * F] = __ldcg(wm + (int64_t)r * F) - v;
}

// In-block update of the back sweep: w[m] -= L[k0:k1, m]' x_block for the
// columns m in [0, k0) of the block's front (kBwdCols columns per task).
__device__ void bwd_blk_upd_task(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t task, const PV& P,
                                 double* vbuf, const double* xsol, int nrhs, double* sh) {
    double(*x)[kSolveBlock] = reinterpret_cast<double(*)[kSolveBlock]>(sh);     // RHS-major
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node, k0 = jb.k_lo, k1 = jb.k_hi;
    const int F = P.F[js], nbk = k1 - k0;
    const int64_t vb = P.rbase[js] * nrhs;
    double* w = vbuf + vb;
    const double* base = P.lnz + P.lnz_off[js];
    for (int e = threadIdx.x; e < nbk * nrhs; e += blockDim.x) {
        const int i = e % nbk, r = e / nbk;
        x[r][i] = __ldcg(xsol + vb + (int64_t)r * F + k0 + i);
    }
    __syncthreads();
    const int m = (int)(task - jb.task0) * kBwdCols + (threadIdx.x >> 5);
    if (m >= jb.c_end) return;
    warp_col_dot_smem(base + lnz_col(m, F) - m + k0, nbk, x, w + m, F, nrhs);
}

constexpr size_t kBwdSmem = sizeof(double) * (size_t)kMaxRHS * kSolveBlock;

__global__ void __launch_bounds__(256) k_bwd_blk_upd(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P, double* vbuf,
                                                     const double* xsol, int nrhs) {
    extern __shared__ double bsh[];
    bwd_blk_upd_task(jobs, njobs, tmap, blockIdx.x, P, vbuf, xsol, nrhs, bsh);
}

// Inverse X = L_blk^-1 of one kSolveBlock-wide unit-lower diagonal block of a
// large front, from the stored 64x64 inverses: X_jj = inv(L_jj),
// X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj (64x64 tiles, FP64 CUDA cores).
// Written column-major (ld = nb) into xinv; used by the block solves.
constexpr size_t kInvSmem = sizeof(double) * 3 * (size_t)kNB * (kNB + 1);

__device__ void tile_mm(const double (*A)[kNB + 1], const double (*B)[kNB + 1], double acc[4][4], int tid) {
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
    for (int k = 0; k < kNB; ++k) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = A[r0 + u][k];
            b[u] = B[k][c0 + u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
}

__global__ void __launch_bounds__(256) k_inv_block(const Job* jobs, PV P) {
    extern __shared__ double ish[];
    double(*As)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(ish);
    double(*Bs)[kNB + 1] = As + kNB;
    double(*Ts)[kNB + 1] = Bs + kNB;
    const Job& jb = jobs[blockIdx.x];
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    if ((P.sn_bad && P.sn_bad[js]) || node_off(P, js)) return;
    const int F = P.F[js];
    const double* base = P.lnz + P.lnz_off[js];
    const double* lv0 = P.linv + P.linv_off[js] + (int64_t)(k0 / kNB) * kNB * kNB;
    double* X = P.xinv + P.xinv_off[js] + (int64_t)(k0 / kSolveBlock) * kSolveBlock * kSolveBlock;
    const int tid = threadIdx.x;
    const int q = (nb + kNB - 1) / kNB;
    const int r0 = (tid & 15) * 4, c0 = (tid >> 4) * 4;
    auto xat = [&](int i, int j) -> double& { return X[(int64_t)i + (int64_t)j * nb]; };
    for (int j = 0; j < q; ++j) {
        const int sj = min(kNB, nb - kNB * j);
        // diagonal block and the zero blocks above it
        for (int e = tid; e < kNB * kNB; e += blockDim.x) {
            const int a = e % kNB, b = e / kNB;
            if (a < sj && b < sj) xat(kNB * j + a, kNB * j + b) = lv0[(int64_t)j * kNB * kNB + e];
        }
        for (int i = 0; i < j; ++i)
            for (int e = tid; e < kNB * kNB; e += blockDim.x) {
                const int a = e % kNB, b = e / kNB;
                if (kNB * i + a < nb && b < sj) xat(kNB * i + a, kNB * j + b) = 0.0;
            }
        __syncthreads();
        for (int i = j + 1; i < q; ++i) {
            const int si = min(kNB, nb - kNB * i);
            double acc[4][4] = {};
            for (int k = j; k < i; ++k) {
                const int sk = min(kNB, nb - kNB * k);
                for (int e = tid; e < kNB * kNB; e += blockDim.x) {
                    const int a = e % kNB, b = e / kNB;
                    const int row = k0 + kNB * i + a, col = k0 + kNB * k + b;
                    As[a][b] = (a < si && b < sk) ? base[lnz_col(col, F) - col + row] : 0.0;
                    Bs[a][b] = (a < sk && b < sj) ? xat(kNB * k + a, kNB * j + b) : 0.0;
                }
                __syncthreads();
                tile_mm(As, Bs, acc, tid);
                __syncthreads();
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) Ts[r0 + u][c0 + v] = acc[u][v];
            for (int e = tid; e < kNB * kNB; e += blockDim.x) {
                const int a = e % kNB, b = e / kNB;
                As[a][b] = (a < si && b < si) ? lv0[(int64_t)i * kNB * kNB + e] : 0.0;
            }
            __syncthreads();
            double acc2[4][4] = {};
            tile_mm(As, Ts, acc2, tid);
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    if (r0 + u < si && c0 + v < sj) xat(kNB * i + r0 + u, kNB * j + c0 + v) = -acc2[u][v];
            __syncthreads();
        }
    }
}

// y_block = X w_block: 32 rows per CTA, 8 warps split the columns
constexpr size_t kMvSmem = sizeof(double) * ((size_t)kSolveBlock * kMaxRHS + 8 * 32 * (kMaxRHS + 1));
constexpr size_t kUpdSmem = sizeof(double) * ((size_t)kSolveBlock * kMaxRHS + (size_t)128 * (kMaxRHS + 1));

__device__ void fwd_blk_mv_task(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t task, const PV& P,
                                const double* vbuf, double* ysol, int nrhs, double* msh) {
    double(*wb)[kMaxRHS] = reinterpret_cast<double(*)[kMaxRHS]>(msh);
    double(*part)[32][kMaxRHS + 1] = reinterpret_cast<double(*)[32][kMaxRHS + 1]>(msh + kSolveBlock * kMaxRHS);
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    const int F = P.F[js];
    const int64_t vb = P.rbase[js] * nrhs;
    const double* w = vbuf + vb;
    const double* X = P.xinv + P.xinv_off[js] + (int64_t)(k0 / kSolveBlock) * kSolveBlock * kSolveBlock;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < nb * nrhs; e += blockDim.x) {
        const int i = e % nb, r = e / nb;
        wb[i][r] = __ldcg(w + (int64_t)r * F + k0 + i);
    }
    __syncthreads();
    const int i = (int)(task - jb.task0) * 32 + lane;
    double acc[kMaxRHS];
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r) acc[r] = 0.0;
    if (i < nb) {
        const int m1 = min(32 * warp + 32, i + 1);
        for (int m = 32 * warp; m < m1; ++m) {
            const double x = X[(int64_t)i + (int64_t)m * nb];
#pragma unroll
            for (int r = 0; r < kMaxRHS; ++r)
                if (r < nrhs) acc[r] += x * wb[m][r];
        }
    }
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r)
        if (r < nrhs) part[warp][lane][r] = acc[r];
    __syncthreads();
    if (warp == 0 && i < nb)
        for (int r = 0; r < nrhs; ++r) {
            double v = 0.0;
            for (int g = 0; g < 8; ++g) v += part[g][lane][r];
            ysol[vb + (int64_t)r * F + k0 + i] = v;
        }
}

__global__ void __launch_bounds__(256) k_fwd_blk_mv(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P, const double* vbuf,
                                                    double* ysol, int nrhs) {
    extern __shared__ double msh[];
    fwd_blk_mv_task(jobs, njobs, tmap, blockIdx.x, P, vbuf, ysol, nrhs, msh);
}

// x_block = X' w_block: 32 columns per CTA, 4 per warp, lanes over rows
__device__ void bwd_blk_mv_task(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t task, const PV& P,
                                const double* vbuf, double* xsol, int nrhs, double* sh) {
    double(*wb)[kSolveBlock] = reinterpret_cast<double(*)[kSolveBlock]>(sh);     // RHS-major
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node, k0 = jb.k_lo, nb = jb.k_hi - jb.k_lo;
    const int F = P.F[js];
    const int64_t vb = P.rbase[js] * nrhs;
    const double* w = vbuf + vb;
    const double* X = P.xinv + P.xinv_off[js] + (int64_t)(k0 / kSolveBlock) * kSolveBlock * kSolveBlock;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < nb * nrhs; e += blockDim.x) {
        const int i = e % nb, r = e / nb;
        wb[r][i] = __ldcg(w + (int64_t)r * F + k0 + i);
    }
    __syncthreads();
    for (int cc = 0; cc < 4; ++cc) {
        const int c = (int)(task - jb.task0) * 32 + warp * 4 + cc;
        if (c >= nb) break;
        double acc[kMaxRHS];
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r) acc[r] = 0.0;
        for (int m = c + lane; m < nb; m += 32) {
            const double x = X[(int64_t)m + (int64_t)c * nb];
#pragma unroll
            for (int r = 0; r < kMaxRHS; ++r)
                if (r < nrhs) acc[r] += x * wb[r][m];
        }
        int r, om;
        const double v = warp_reduce_scatter<kMaxRHS>(acc, lane, r, om);
        if ((lane & om) == 0 && r < nrhs) xsol[vb + (int64_t)r * F + k0 + c] = v;
    }
}

__global__ void __launch_bounds__(256) k_bwd_blk_mv(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P, const double* vbuf,
                                                    double* xsol, int nrhs) {
    extern __shared__ double bsh[];
    bwd_blk_mv_task(jobs, njobs, tmap, blockIdx.x, P, vbuf, xsol, nrhs, bsh);
}

// rows below a solve block: w[i] -= L[i, k0:k1] y; 128 rows per CTA, the two
// halves of the 256 columns summed through shared memory
__device__ void fwd_blk_upd2_task(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t task, const PV& P,
                                  double* vbuf, const double* ysol, int nrhs, double* ush) {
    double(*y)[kMaxRHS] = reinterpret_cast<double(*)[kMaxRHS]>(ush);
    double(*part)[kMaxRHS + 1] = reinterpret_cast<double(*)[kMaxRHS + 1]>(ush + kSolveBlock * kMaxRHS);
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node, k0 = jb.k_lo, k1 = jb.k_hi;
    const int F = P.F[js], nbk = k1 - k0;
    const int64_t vb = P.rbase[js] * nrhs;
    double* w = vbuf + vb;
    const double* base = P.lnz + P.lnz_off[js];
    const int tid = threadIdx.x;
    for (int e = tid; e < nbk * nrhs; e += blockDim.x) {
        const int i = e % nbk, r = e / nbk;
        y[i][r] = __ldcg(ysol + vb + (int64_t)r * F + k0 + i);
    }
    __syncthreads();
    const int row = tid & (kSolveRows - 1), half = tid / kSolveRows;
    const int i = jb.c0 + (int)(task - jb.task0) * kSolveRows + row;
    double acc[kMaxRHS];
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r) acc[r] = 0.0;
    const int hc = (nbk + 1) / 2;
    const int r_end = jb.r_end;
    if (i < r_end) {
        const int c0 = half * hc, c1 = min(nbk, c0 + hc);
#pragma unroll 8
        for (int c = c0; c < c1; ++c) {
            const int col = k0 + c;
            const double l = base[lnz_col(col, F) - col + i];
#pragma unroll
            for (int r = 0; r < kMaxRHS; ++r)
                if (r < nrhs) acc[r] += l * y[c][r];
        }
    }
    if (half == 1)
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r)
            if (r < nrhs) part[row][r] = acc[r];
    __syncthreads();
    if (half == 0 && i < r_end)
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r)
            if (r < nrhs) w[(int64_t)r * F + i] = __ldcg(w + (int64_t)r * F + i) - (acc[r] + part[row][r]);
}

__global__ void __launch_bounds__(256) k_fwd_blk_upd2(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P,
                                                      double* vbuf, const double* ysol, int nrhs) {
    extern __shared__ double ush[];
    fwd_blk_upd2_task(jobs, njobs, tmap, blockIdx.x, P, vbuf, ysol, nrhs, ush);
}


// forward sweep, rows [S, F): w[i] -= sum_{c < S} L[i][c] y[c].  Phase 1: one
// CTA per (kRectRows rows, kRectCols columns) tile, a thread per row, writes
// the tile's partial sums; phase 2 (k_fwd_rect_sum) adds the column tiles'
// partials of each row in a fixed order (deterministic).
template <int NR>
__global__ void __launch_bounds__(256) k_fwd_rect_part(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P,
                                                       const double* ysol, double* pbuf, int nrhs) {
    __shared__ double ys[kRectCols][kMaxRHS];
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int F = P.F[js], S = P.S[js];
    const int ncc = jb.k_hi;
    const int64_t u = task - jb.task0;
    const int cc = (int)(u % ncc), rc = (int)(u / ncc);
    const int64_t vb = P.rbase[js] * nrhs;
    const int tid = threadIdx.x;
    const int rbeg = S + rc * kRectRows, nr = min(kRectRows, F - rbeg);
    const int cbeg = cc * kRectCols, ncol = min(kRectCols, S - cbeg);
    for (int e = tid; e < ncol * nrhs; e += blockDim.x) {
        const int c = e % ncol, r = e / ncol;
        ys[c][r] = ysol[vb + (int64_t)r * F + cbeg + c];
    }
    __syncthreads();
    if (tid >= nr) return;
    const int i = rbeg + tid;
    const double* base = P.lnz + P.lnz_off[js];
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
#pragma unroll 16
    for (int c = 0; c < ncol; ++c) {
        const int col = cbeg + c;
        const double l = __ldcs(base + lnz_col(col, F) - col + i);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) acc[r] += l * ys[c][r];
    }
    double* part = pbuf + (P.fwd_off[js] + (int64_t)cc * (F - S) + (i - S)) * kMaxRHS;
#pragma unroll
    for (int r = 0; r < NR; ++r)
        if (r < nrhs) part[r] = acc[r];
}

__global__ void k_fwd_rect_sum(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, double* vbuf,
                               const double* pbuf, int nrhs) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int F = P.F[js], S = P.S[js];
    const int row = S + (int)(task - jb.task0);
    const int ncc = (S + kRectCols - 1) / kRectCols;
    double* w = vbuf + P.rbase[js] * nrhs;
    const double* part = pbuf + (P.fwd_off[js] + (row - S)) * kMaxRHS;
    // column tiles in ascending order for every right-hand side; the loads
    // of several tiles are in flight together
    double v[kMaxRHS];
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r) v[r] = 0.0;
#pragma unroll 4
    for (int k = 0; k < ncc; ++k) {
        const double* pk = part + (int64_t)k * (F - S) * kMaxRHS;
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r)
            if (r < nrhs) v[r] += __ldcg(pk + r);
    }
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r)
        if (r < nrhs) w[(int64_t)r * F + row] -= v[r];
}

// back sweep, update rows [S, F): w[c] -= L[S:F, c]' w[S:F].  Phase 1: one
// CTA per (kRectCols columns, kRectRows rows) stages its rows of the vector in
// shared memory once and writes one partial dot product per column (a warp
// per column at a time, 32 columns per warp); phase 2 (k_bwd_rect_sum) adds
// the partials of each column in a fixed order, so the result is
// deterministic.
template <int NR>
__global__ void __launch_bounds__(256, NR <= 4 ? 3 : 2) k_bwd_rect_part(const Job* jobs, int64_t njobs, const int32_t* tmap, PV P,
                                                       const double* vbuf, double* pbuf, int nrhs) {
    __shared__ double ws[kMaxRHS][kRectRows];
    const int64_t task = blockIdx.x;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int F = P.F[js], S = P.S[js];
    const int ncc = jb.k_hi;
    const int64_t u = task - jb.task0;
    const int cc = (int)(u % ncc), rc = (int)(u / ncc);
    const int64_t vb = P.rbase[js] * nrhs;
    const double* w = vbuf + vb;
    const double* base = P.lnz + P.lnz_off[js];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rbeg = S + rc * kRectRows, nr = min(kRectRows, F - rbeg);
    for (int e = tid; e < nr * nrhs; e += blockDim.x) {
        const int i = e % nr, r = e / nr;
        ws[r][i] = w[(int64_t)r * F + rbeg + i];
    }
    __syncthreads();
    double* part = pbuf + (P.rect_off[js] + (int64_t)rc * S) * kMaxRHS;
    const int cw = kRectCols / 8;
    // CG columns at a time per warp (CG x UR loads in flight per lane)
    constexpr int CG = NR <= 4 ? 4 : 2;
    constexpr int UR = NR <= 4 ? 4 : 2;                // row steps in flight
    for (int a = 0; a < cw; a += CG) {
        const int c0 = cc * kRectCols + warp * cw + a;
        if (c0 >= S) break;
        const double* col[CG];
        bool cv[CG];
#pragma unroll
        for (int q = 0; q < CG; ++q) {
            cv[q] = c0 + q < S;
            const int c = cv[q] ? c0 + q : c0;
            col[q] = base + lnz_col(c, F) - c + rbeg;
        }
        double acc[CG][NR];
#pragma unroll
        for (int q = 0; q < CG; ++q)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[q][r] = 0.0;
#pragma unroll(UR)
        for (int i = lane; i < nr; i += 32) {
            double l[CG];
#pragma unroll
            for (int q = 0; q < CG; ++q) l[q] = __ldcs(col[q] + i);
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) {
                    const double x = ws[r][i];
#pragma unroll
                    for (int q = 0; q < CG; ++q) acc[q][r] += l[q] * x;
                }
        }
#pragma unroll
        for (int q = 0; q < CG; ++q) {
            int r, om;
            const double v = warp_reduce_scatter<NR>(acc[q], lane, r, om);
            if ((lane & om) == 0 && cv[q] && r < nrhs) part[(int64_t)(c0 + q) * kMaxRHS + r] = v;
        }
    }
}

// Each column is summed by a group of kSumLanes lanes: lane g of the group
// adds the row tiles g, g + kSumLanes, ... in ascending order, and the
// group's partial sums are added by a fixed butterfly (deterministic), so
// the few row tiles of a column are loaded together instead of one after
// another.
constexpr int kSumLanes = 8;
__device__ __forceinline__ double group_sum(double v) {
    const unsigned gmask = 0xffu << (threadIdx.x & 31 & ~(kSumLanes - 1));
#pragma unroll
    for (int o = kSumLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(gmask, v, o, kSumLanes);
    return v;
}

__global__ void k_bwd_rect_sum(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, double* vbuf,
                               const double* pbuf, int nrhs) {
    const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t task = gt / kSumLanes;              // the group's lanes share the task
    const int g = (int)(gt % kSumLanes);
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int F = P.F[js], S = P.S[js];
    if (F <= S || is_retained(P, js)) return;
    const int c = (int)(task - jb.task0);
    const int nrc = (F - S + kRectRows - 1) / kRectRows;
    double* w = vbuf + P.rbase[js] * nrhs;
    const double* part = pbuf + (P.rect_off[js] + c) * kMaxRHS;
    double v[kMaxRHS];
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r) v[r] = 0.0;
#pragma unroll 2
    for (int k = g; k < nrc; k += kSumLanes) {
        const double* pk = part + (int64_t)k * S * kMaxRHS;
#pragma unroll
        for (int r = 0; r < kMaxRHS; ++r)
            if (r < nrhs) v[r] += __ldcg(pk + r);
    }
#pragma unroll
    for (int r = 0; r < kMaxRHS; ++r)
        if (r < nrhs) {
            const double t = group_sum(v[r]);
            if (g == 0) w[(int64_t)r * F + c] -= t;
        }
}

// y_j /= d_j and scatter of the own rows (thread per column)
// (a retained front passes its gathered sums through: the rows keep them)
__global__ void k_fwd_finish(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, const double* ysol,
                             const double* gathered, double* b, int64_t ldb, int nrhs) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int j = (int)(task - jb.task0);
    const int F = P.F[js], fst = P.fst[js];
    if (is_retained(P, js)) {
        const double* g = gathered + P.rbase[js] * nrhs;
        for (int r = 0; r < nrhs; ++r) b[(int64_t)(fst + j) + r * ldb] = g[(int64_t)r * F + j];
        return;
    }
    const double* y = ysol + P.rbase[js] * nrhs;
    const double d = lcol(P, js, F, j)[j];
    for (int r = 0; r < nrhs; ++r) b[(int64_t)(fst + j) + r * ldb] = y[(int64_t)r * F + j] / d;
}

// ---------------------------------------------------------------------------
// Triangles of the solves as one dataflow launch per level.  Task (js, rb) is
// the 64-row block rb of front js (rows [64 rb, 64 rb + 64) of [0, S)).
// Forward: y_rb = X_rb (w_rb - sum_{b < rb} L[rb, b] y_b), X_rb = L_rb,rb^-1
// (the stored 64x64 inverse); backward: x_cb = X_cb' (w_cb - sum_{r > cb}
// L[r, cb]' x_r).  Persistent CTAs take tasks in order from a counter (forward
// block-major ascending, backward descending), so a task only waits for
// tasks taken before it, by CTAs that are running: the waits always end.
// Each wait is bounded (PV::wait_ns); one that gives up sets
// Stats::solve_timeout and an abort word every CTA checks, and the host
// turns it into an error.  Per tile, a thread owns one row (forward) or one
// column (backward) and a quarter of the 64 columns (rows).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long tri_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// thread 0 waits (bounded) for flag; returns false when the launch aborts
__device__ __forceinline__ bool tri_wait(const int* flag, int* abort_word, const PV& P) {
    if (ld_acquire(flag)) return true;
    const unsigned long long t0 = tri_now();
    for (int spin = 0;; ++spin) {
        if (ld_acquire(flag)) return true;
        if (ld_acquire(abort_word)) return false;
        if ((spin & 63) == 63 && tri_now() - t0 > P.wait_ns) {
            atomicExch(&P.st->solve_timeout, 1);
            st_release(abort_word, 1);
            return false;
        }
        __nanosleep(64);
    }
}

constexpr int kTriLd = kMaxRHS + 1;

template <int NR>
__global__ void __launch_bounds__(256) k_fwd_tri(const int32_t* tasks, int ntasks, int32_t* flags, int32_t* counter,
                                                 PV P, const double* vbuf, double* ysol, int nrhs) {
    __shared__ double ys[kNB][kTriLd];
    __shared__ double part[4][kNB][kTriLd];
    __shared__ int task_sh, ok_sh;
    int* abort_word = counter + 1;
    const int tid = threadIdx.x, row = tid & (kNB - 1), q = tid >> 6;
    for (;;) {
        if (tid == 0) task_sh = atomicAdd(counter, 1);
        __syncthreads();
        const int t = task_sh;
        if (t >= ntasks) break;
        const int js = tasks[2 * t], rb = tasks[2 * t + 1];
        if (node_off(P, js)) {
            __syncthreads();                                          // all have read task_sh
            continue;
        }
        const int F = P.F[js], S = P.S[js];
        const int r0 = rb * kNB, nrow = min(kNB, S - r0);
        const double* base = P.lnz + P.lnz_off[js];
        const int64_t vb = P.rbase[js] * nrhs;
        int32_t* fl = flags + P.tri_off[js];
        // loads that need no other task: this row's X entries (the product
        // with the block inverse at the end) and the right-hand side
        const double* lv = P.linv + P.linv_off[js] + (int64_t)rb * kNB * kNB;
        constexpr bool kPreX = NR <= 4;                                      // registers allow it
        double xr[kPreX ? 16 : 1];
        if constexpr (kPreX) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int m = 16 * q + k;
                xr[k] = (m <= row) ? __ldg(lv + row + m * kNB) : 0.0;       // X[row][m], unit lower
            }
        }
        double wv[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            wv[r] = (tid < kNB && row < nrow && r < nrhs) ? __ldcg(vbuf + vb + (int64_t)r * F + r0 + row) : 0.0;
        double acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0.0;
        bool ok = true;
        for (int b = 0; b < rb; ++b) {
            // this thread's 16 entries of the tile L[rb, b] first: they do not
            // depend on block b, so their latency overlaps the wait for it
            double lr[16];
            {
                const int c0 = kNB * b + 16 * q;
                int64_t p = lnz_col(c0, F) - c0 + r0 + row;           // L[r0 + row][c0]
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    lr[k] = (row < nrow) ? __ldg(base + p) : 0.0;
                    p += F - (c0 + k) - 1;                            // next column, same row
                }
            }
            if (tid == 0) ok_sh = tri_wait(fl + b, abort_word, P);
            __syncthreads();
            if (!ok_sh) {
                ok = false;
                break;
            }
            for (int e = tid; e < kNB * nrhs; e += blockDim.x) {
                const int i = e & (kNB - 1), r = e >> 6;
                ys[i][r] = __ldcg(ysol + vb + (int64_t)r * F + kNB * b + i);
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 16; ++k)
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) acc[r] += lr[k] * ys[16 * q + k][r];
            __syncthreads();
        }
        if (!ok) break;
        // v = w - sum of the four quarters, then y = X v
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) part[q][row][r] = acc[r];
        __syncthreads();
        if (tid < kNB)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs)
                    ys[row][r] = (row < nrow) ? wv[r] - ((part[0][row][r] + part[1][row][r]) +
                                                         (part[2][row][r] + part[3][row][r]))
                                              : 0.0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            double x;
            if constexpr (kPreX) {
                x = xr[k];
            } else {
                const int m = 16 * q + k;
                x = (m <= row) ? __ldg(lv + row + m * kNB) : 0.0;
            }
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) acc[r] += x * ys[16 * q + k][r];
        }
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) part[q][row][r] = acc[r];
        __syncthreads();
        if (tid < kNB && row < nrow)
            for (int r = 0; r < nrhs; ++r)
                ysol[vb + (int64_t)r * F + r0 + row] =
                    (part[0][row][r] + part[1][row][r]) + (part[2][row][r] + part[3][row][r]);
        __threadfence();
        __syncthreads();
        // (watchdog test switch: the first task of the launch never reports)
        if (tid == 0 && !(P.tc_drop && t == 0)) st_release(fl + rb, 1);
    }
}

template <int NR>
__global__ void __launch_bounds__(256) k_bwd_tri(const int32_t* tasks, int ntasks, int32_t* flags, int32_t* counter,
                                                 PV P, const double* vbuf, double* xsol, int nrhs) {
    __shared__ double xs[kNB][kTriLd];
    __shared__ double part[4][kNB][kTriLd];
    __shared__ int task_sh, ok_sh;
    int* abort_word = counter + 1;
    const int tid = threadIdx.x, col = tid & (kNB - 1), q = tid >> 6;
    for (;;) {
        if (tid == 0) task_sh = atomicAdd(counter, 1);
        __syncthreads();
        if (task_sh >= ntasks) break;
        const int t = ntasks - 1 - task_sh;                          // descending blocks
        const int js = tasks[2 * t], cb = tasks[2 * t + 1];
        if (node_off(P, js)) {
            __syncthreads();
            continue;
        }
        const int F = P.F[js], S = P.S[js];
        const int c0 = cb * kNB, ncol = min(kNB, S - c0);
        const int nblk = (S + kNB - 1) / kNB;
        const double* base = P.lnz + P.lnz_off[js];
        const int64_t vb = P.rbase[js] * nrhs;
        int32_t* fl = flags + P.tri_off[js];
        double acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0.0;
        bool ok = true;
        const int64_t pc = (col < ncol) ? lnz_col(c0 + col, F) - (c0 + col) : 0;   // column c0 + col, row 0
        const double* lv = P.linv + P.linv_off[js] + (int64_t)cb * kNB * kNB;
        constexpr bool kPreX = NR <= 4;
        double xr[kPreX ? 16 : 1];
        if constexpr (kPreX) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int m = 16 * q + k;
                xr[k] = (m >= col) ? __ldg(lv + m + col * kNB) : 0.0;       // X[m][col]
            }
        }
        double wv[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            wv[r] = (tid < kNB && col < ncol && r < nrhs) ? __ldcg(vbuf + vb + (int64_t)r * F + c0 + col) : 0.0;
        // the blocks below finish from the bottom up: take them in that order,
        // so that only the nearest one (cb + 1, the last to finish) is waited for
        for (int rb = nblk - 1; rb > cb; --rb) {
            const int nr = min(kNB, S - rb * kNB);
            double lr[16];                                   // L[64 rb + 16 q + k][c0 + col], ahead of the wait
            {
                const int i0 = kNB * rb + 16 * q;
#pragma unroll
                for (int k = 0; k < 16; ++k) lr[k] = (col < ncol && 16 * q + k < nr) ? __ldg(base + pc + i0 + k) : 0.0;
            }
            if (tid == 0) ok_sh = tri_wait(fl + rb, abort_word, P);
            __syncthreads();
            if (!ok_sh) {
                ok = false;
                break;
            }
            for (int e = tid; e < kNB * nrhs; e += blockDim.x) {
                const int i = e & (kNB - 1), r = e >> 6;
                xs[i][r] = (i < nr) ? __ldcg(xsol + vb + (int64_t)r * F + kNB * rb + i) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 16; ++k)
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) acc[r] += lr[k] * xs[16 * q + k][r];
            __syncthreads();
        }
        if (!ok) break;
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) part[q][col][r] = acc[r];
        __syncthreads();
        if (tid < kNB)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs)
                    xs[col][r] = (col < ncol) ? wv[r] - ((part[0][col][r] + part[1][col][r]) +
                                                         (part[2][col][r] + part[3][col][r]))
                                              : 0.0;
        __syncthreads();
        // x = X' v: x[col] = sum_{m >= col} X[m][col] v[m]
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int m = 16 * q + k;
            double x;
            if constexpr (kPreX) {
                x = xr[k];
            } else {
                x = (m >= col) ? __ldg(lv + m + col * kNB) : 0.0;
            }
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) acc[r] += x * xs[m][r];
        }
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) part[q][col][r] = acc[r];
        __syncthreads();
        if (tid < kNB && col < ncol)
            for (int r = 0; r < nrhs; ++r)
                xsol[vb + (int64_t)r * F + c0 + col] =
                    (part[0][col][r] + part[1][col][r]) + (part[2][col][r] + part[3][col][r]);
        __threadfence();
        __syncthreads();
        if (tid == 0 && !(P.tc_drop && t == ntasks - 1)) st_release(fl + cb, 1);
    }
}

// gather of the back sweep: own rows (forward result) and ancestors' solution
__global__ void k_bwd_gather(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, double* vbuf,
                             const double* b, int64_t ldb, int nrhs) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    const int i = (int)(task - jb.task0);
    const int F = P.F[js], S = P.S[js], fst = P.fst[js];
    double* w = vbuf + P.rbase[js] * nrhs;
    const int row = (i < S) ? (fst + i) : P.rows[P.rbase[js] + i];
    for (int r = 0; r < nrhs; ++r) w[(int64_t)r * F + i] = b[(int64_t)row + r * ldb];
}


__global__ void k_bwd_finish(const Job* jobs, int64_t njobs, const int32_t* tmap, int64_t ntasks, PV P, const double* xsol, double* b,
                             int64_t ldb, int nrhs) {
    const int64_t task = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (task >= ntasks) return;
    const Job& jb = job_of(jobs, njobs, tmap, task);
    const int js = jb.node;
    if (node_off(P, js)) return;
    if (is_retained(P, js)) return;
    const int j = (int)(task - jb.task0);
    const int F = P.F[js], fst = P.fst[js];
    const double* w = xsol + P.rbase[js] * nrhs;
    for (int r = 0; r < nrhs; ++r) b[(int64_t)(fst + j) + r * ldb] = w[(int64_t)r * F + j];
}

// ---------------------------------------------------------------------------
// Cholesky form (SPRFC2, src/SPR/sprfc2.f:1013-1032): column j of C is
// L(:, j) sqrt(d_j) with sqrt(d_j) on the diagonal and in D; back again, d_j =
// c_jj^2 and L(:, j) = C(:, j) / c_jj.  Retained fronts are left as assembled.
// One CTA per supernode, one warp per column of the packed trapezoid.
// ---------------------------------------------------------------------------
template <bool TO_CHOL>
__global__ void k_chol_convert(PV P, int64_t nsuper) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int64_t js = blockIdx.x; js < nsuper; js += gridDim.x) {
        if (is_retained(P, (int)js)) continue;
        const int S = P.S[js], F = P.F[js], fst = P.fst[js];
        double* base = P.lnz + P.lnz_off[js];
        for (int j = warp; j < S; j += nwarp) {
            double* col = base + lnz_col(j, F);          // col[0] is the diagonal
            const double x = col[0];
            const double diag = TO_CHOL ? sqrt(x) : x * x;
            const double sc = TO_CHOL ? diag : 1.0 / x;
            for (int i = 1 + lane; i < F - j; i += 32) col[i] *= sc;
            __syncwarp();
            if (lane == 0) {
                col[0] = diag;
                P.dvec[fst + j] = diag;
            }
        }
    }
}

// b(i, r) times sqrt(d_i) (divide = 0) or divided by it, where d_i > 0:
// C^-1 b = D^1/2 (D^-1 L^-1 b) after the L D L' forward sweep, and
// C^-T y = L^-T (D^-1/2 y) before the back sweep (SPRFS9/SPRBS9,
// sprfs2.f:575-610, sprbs2.f:500-540, with C = L D^1/2).
__global__ void k_scale_sqrt_d(const double* dvec, double* b, int64_t ldb, int64_t n, int64_t nrhs, int divide) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * nrhs;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, r = e / n;
        const double d = dvec[i];
        if (d > 0.0) {
            const double sq = sqrt(d);
            double* x = b + i + r * ldb;
            *x = divide ? *x / sq : *x * sq;
        }
    }
}

// ---------------------------------------------------------------------------
// Residual of the FP64 matrix for iterative refinement (the product SPRPRQ
// forms from the packed pattern, src/SPR/sprprm.f:243-325): the nonzeros of
// the assembled LNZ are compacted once into a full symmetric CSR with rows
// sorted by column, so r = b - K x is a deterministic warp-per-row SpMV.
// ---------------------------------------------------------------------------
__global__ void k_csr_count(PV P, int64_t nsuper, int* rowcnt) {
    const int lane = threadIdx.x & 31;
    for (int64_t js = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; js < nsuper;
         js += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int F = P.F[js], S = P.S[js], fst = P.fst[js];
        const int32_t* rows = P.rows + P.rbase[js];
        const double* col = P.lnz + P.lnz_off[js];
        for (int j = 0; j < S; ++j) {
            const double* cj = col + lnz_col(j, F) - j;
            for (int i = j + lane; i < F; i += 32)
                if (cj[i] != 0.0) {
                    atomicAdd(&rowcnt[rows[i]], 1);
                    if (i != j) atomicAdd(&rowcnt[fst + j], 1);
                }
        }
    }
}

__global__ void k_csr_fill(PV P, int64_t nsuper, int* fillpos, int32_t* ci, double* cv) {
    const int lane = threadIdx.x & 31;
    for (int64_t js = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; js < nsuper;
         js += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int F = P.F[js], S = P.S[js], fst = P.fst[js];
        const int32_t* rows = P.rows + P.rbase[js];
        const double* col = P.lnz + P.lnz_off[js];
        for (int j = 0; j < S; ++j) {
            const double* cj = col + lnz_col(j, F) - j;
            for (int i = j + lane; i < F; i += 32) {
                const double a = cj[i];
                if (a == 0.0) continue;
                const int row = rows[i];
                int p = atomicAdd(&fillpos[row], 1);
                ci[p] = fst + j;
                cv[p] = a;
                if (i != j) {
                    p = atomicAdd(&fillpos[fst + j], 1);
                    ci[p] = row;
                    cv[p] = a;
                }
            }
        }
    }
}

// insertion sort of each row by column (rows are short: ~81 entries for hex8)
__global__ void k_csr_sort(const int64_t* rowptr, int64_t neq, int32_t* ci, double* cv, double* rowabs) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= neq) return;
    const int64_t p0 = rowptr[r], p1 = rowptr[r + 1];
    double sabs = 0.0;
    for (int64_t p = p0 + 1; p < p1; ++p) {
        const int32_t c = ci[p];
        const double v = cv[p];
        int64_t q = p - 1;
        while (q >= p0 && ci[q] > c) {
            ci[q + 1] = ci[q];
            cv[q + 1] = cv[q];
            --q;
        }
        ci[q + 1] = c;
        cv[q + 1] = v;
    }
    for (int64_t p = p0; p < p1; ++p) sabs += fabs(cv[p]);
    rowabs[r] = sabs;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// r = b - K x for up to NR right-hand sides in one pass over each row (a warp
// per row, rows taken grid-stride).  Per right-hand side the products of a
// row are added in the same order as a pass per right-hand side would add
// them (lane-strided, then the xor tree).  norms[3q..3q+2] = max|r|, max|x|,
// max|b|: kept per warp in shared memory and reduced per CTA before one
// atomic each; the maxima compare bit patterns, so a NaN ranks above every
// number, as in the atomic.
constexpr int kResThreads = 256;
__device__ __forceinline__ double max_nonneg(double a, double v) {
    return __double_as_longlong(v) > __double_as_longlong(a) ? v : a;
}
template <int NR>
__global__ void __launch_bounds__(kResThreads) k_residual(const int64_t* rowptr, const int32_t* ci, const double* cv,
                                                          int64_t neq, const double* b, const double* x, double* r,
                                                          int64_t ld, int nrhs, double* norms) {
    constexpr int kW = kResThreads / 32;
    __shared__ double red[kW][3 * NR];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int e = 0; e < 3 * NR; ++e) red[warp][e] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kW;
    for (int64_t row = (int64_t)blockIdx.x * kW + warp; row < neq; row += stride) {
        const int64_t p0 = rowptr[row], p1 = rowptr[row + 1];
        double acc[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) acc[q] = 0.0;
        for (int64_t p = p0 + lane; p < p1; p += 32) {
            const double v = cv[p];
            const int64_t c = ci[p];
#pragma unroll
            for (int q = 0; q < NR; ++q)
                if (q < nrhs) acc[q] += v * x[c + q * ld];
        }
#pragma unroll
        for (int q = 0; q < NR; ++q)
            if (q < nrhs)
                for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < NR; ++q)
                if (q < nrhs) {
                    const double bi = b[row + q * ld], ri = bi - acc[q];
                    r[row + q * ld] = ri;
                    red[warp][3 * q] = max_nonneg(red[warp][3 * q], fabs(ri));
                    red[warp][3 * q + 1] = max_nonneg(red[warp][3 * q + 1], fabs(x[row + q * ld]));
                    red[warp][3 * q + 2] = max_nonneg(red[warp][3 * q + 2], fabs(bi));
                }
    }
    __syncthreads();
    if (threadIdx.x < 3 * nrhs && threadIdx.x < 3 * NR) {
        double m = 0.0;
        for (int w = 0; w < kW; ++w) m = max_nonneg(m, red[w][threadIdx.x]);
        atomic_max_nonneg(&norms[threadIdx.x], m);
    }
}

__global__ void k_axpy(double* x, const double* d, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] += d[i];
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
#define TMAP(l) ((l).map_begin >= 0 ? d_->task_map + (l).map_begin : nullptr)
// Copy plan of the streamed factorisation.  Levels below L1 form group 0; each
// level L >= L1 is group L - L1 + 1 (L1 is the lowest level with at most
// kMaxTopNodes supernodes at or above it, so the copies stay few).  A group's
// LNZ ranges are its supernodes' blocks, adjacent blocks merged; group 0 is
// the gaps between the others.
struct Engine::Transfer {
    static constexpr int64_t kMaxTopNodes = 1024;
    int L1 = 0;
    std::vector<std::vector<std::pair<int64_t, int64_t>>> ranges;   // per group: (LNZ offset, doubles)
    std::vector<cudaEvent_t> up, done;                             // per group
    cudaStream_t ups = nullptr;                                    // uploads (the caller's copy stream: downloads)
    // the last level's super-panels come back as they become final: per panel
    // step, the LNZ ranges of the super-panels ending there and their event
    int32_t early_level = -1;
    std::vector<std::vector<std::pair<int64_t, int64_t>>> spranges;
    std::vector<cudaEvent_t> spev;
    // per group, the download ranges: the upload ranges without the early
    // fronts' LNZ
    std::vector<std::vector<std::pair<int64_t, int64_t>>> dranges;
    // the early fronts and a device copy of their uploaded LNZ: a front whose
    // pivot fails later gets its original columns back, in the device LNZ and
    // on the host, as a factorisation without early writes leaves them
    std::vector<int32_t> early_nodes;
    std::vector<std::pair<int64_t, int64_t>> early_ranges;      // LNZ offset, doubles (backup offsets: running sum)
    double* d_backup = nullptr;
    cudaEvent_t start = nullptr, fin = nullptr;
    cudaEvent_t ts = nullptr, tu = nullptr, tf = nullptr, te = nullptr;   // timing: start, group 0 up, factor end, last download
    cudaEvent_t tf0 = nullptr;                                            // timing: factorisation start
    std::vector<int64_t> diag_pos;                                 // LNZ offset of each equation's diagonal
    double* h_diag = nullptr;                                      // pinned
    double* d_diag = nullptr;
    ~Transfer() {
        if (ups) cudaStreamDestroy(ups);
        for (cudaEvent_t e : spev) cudaEventDestroy(e);
        if (d_backup) cudaFree(d_backup);
        for (cudaEvent_t e : up) cudaEventDestroy(e);
        for (cudaEvent_t e : done) cudaEventDestroy(e);
        if (start) cudaEventDestroy(start);
        if (fin) cudaEventDestroy(fin);
        if (ts) cudaEventDestroy(ts);
        if (tu) cudaEventDestroy(tu);
        if (te) cudaEventDestroy(te);
        if (tf) cudaEventDestroy(tf);
        if (tf0) cudaEventDestroy(tf0);
        if (h_diag) cudaFreeHost(h_diag);
        if (d_diag) cudaFree(d_diag);
    }
    int group(int32_t level) const { return level < L1 ? 0 : level - L1 + 1; }
};

Engine::Engine() : d_(new Dev()) {
    const char* e = getenv("SPR_B200_GRAPHS");
    use_graphs_ = !(e && e[0] == '0');
}

cudaGraphExec_t Engine::find_graph(const GraphKey& k) {
    for (auto& g : graphs_)
        if (g.key == k) return g.exec;
    return nullptr;
}

int64_t Engine::graph_launches(const GraphKey& k) {
    for (auto& g : graphs_)
        if (g.key == k) return g.launches;
    return 0;
}

void Engine::store_graph(const GraphKey& k, cudaGraphExec_t exec, int64_t launches) {
    if (graphs_.size() >= 16) {
        cudaGraphExecDestroy(graphs_.front().exec);
        graphs_.erase(graphs_.begin());
    }
    graphs_.push_back(GraphEntry{k, exec, launches});
}

Engine::~Engine() {
    for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t e : d_->evpool) cudaEventDestroy(e);
    if (d_->side) cudaStreamDestroy(d_->side);
    if (d_->ahead) cudaStreamDestroy(d_->ahead);
    if (d_->wbs) cudaStreamDestroy(d_->wbs);
    if (d_->mbox) cudaFreeHost(d_->mbox);
    if (d_->slab) cudaFree(d_->slab);
    if (d_->slab_far) cudaFree(d_->slab_far);
    if (csr_.rowptr) cudaFree(csr_.rowptr);
    if (csr_.ci) cudaFree(csr_.ci);
    if (csr_.cv) cudaFree(csr_.cv);
    if (csr_.rowabs) cudaFree(csr_.rowabs);
    if (rbuf_) cudaFree(rbuf_);
    if (nbuf_) cudaFree(nbuf_);
    if (guard_copy_) cudaFree(guard_copy_);
    xfer_.reset();
    if (!d_) return;
    for (void* p : d_->owned) cudaFree(p);
    if (d_->arena) cudaFree(d_->arena);
    if (d_->vbuf) cudaFree(d_->vbuf);
    if (d_->vbuf2) cudaFree(d_->vbuf2);
    if (d_->bbuf) cudaFree(d_->bbuf);
    if (d_->ev0) cudaEventDestroy(d_->ev0);
    if (d_->ev1) cudaEventDestroy(d_->ev1);
}

int Engine::open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa) {
    int rc = build_plan(mspar, mtrees, msifa, P_);
    if (rc != 0) return rc;
    Dev& D = *d_;
    auto& o = D.owned;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev));
    {
        // side and look-ahead streams and the fork/join events of one
        // factorisation (two per step that forks a far or look-ahead update)
        size_t nev = 0;
        for (const LevelPlan& lp : P_.levels)
            for (size_t st = 0; st < lp.far.size(); ++st) {
                if (!lp.far[st].empty() || !lp.far_tc[st].empty()) nev += 2;
                if (!lp.ahead[st].empty()) nev += 2;
                if (st < lp.wb_sp.size() && lp.wb_sp[st].ntasks > 0) nev += 1;
            }
        for (const LevelPlan& lp : P_.levels)           // the join after a level's early writes
            for (const Launch& w : lp.wb_sp)
                if (w.ntasks > 0) {
                    nev += 1;
                    break;
                }
        CK(cudaStreamCreateWithFlags(&D.side, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&D.ahead, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&D.wbs, cudaStreamNonBlocking));
        D.evpool.resize(nev);
        for (cudaEvent_t& e : D.evpool) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (dev_upload(o, &D.fst, P_.fst) || dev_upload(o, &D.S, P_.S) || dev_upload(o, &D.F, P_.F) ||
        dev_upload(o, &D.child_ptr, P_.child_ptr) || dev_upload(o, &D.child, P_.child) ||
        dev_upload(o, &D.rows, P_.rows) || dev_upload(o, &D.rel, P_.rel) ||
        dev_upload(o, &D.cchild, P_.cchild) || dev_upload(o, &D.ct, P_.ct) ||
        dev_upload(o, &D.buf_ld, P_.buf_ld) || dev_upload(o, &D.lnz_off, P_.lnz_off) ||
        dev_upload(o, &D.rel_off, P_.rel_off) || dev_upload(o, &D.rbase, P_.rbase) ||
        dev_upload(o, &D.cptr, P_.cptr) || dev_upload(o, &D.buf_off, P_.buf_off) ||
        dev_upload(o, &D.upd_off, P_.upd_off) || dev_upload(o, &D.jobs, P_.jobs) ||
        dev_upload(o, &D.linv_off, P_.linv_off) || dev_upload(o, &D.xinv_off, P_.xinv_off) ||
        dev_upload(o, &D.rect_off, P_.rect_off) || dev_upload(o, &D.fwd_off, P_.fwd_off) ||
        dev_upload(o, &D.task_map, P_.task_map))
        return -4;
    CK(cudaMalloc((void**)&D.pbuf,
                  std::max<int64_t>(std::max(P_.rect_entries, P_.fwd_entries), 1) * kMaxRHS * sizeof(double)));
    o.push_back(D.pbuf);
    CK(cudaMalloc((void**)&D.xinv, std::max<int64_t>(P_.xinv_doubles, 1) * sizeof(double)));
    o.push_back(D.xinv);
    CK(cudaMalloc((void**)&D.linv, std::max<int64_t>(P_.linv_doubles, 1) * sizeof(double)));
    o.push_back(D.linv);
    std::vector<int32_t> small, all;
    D.small_begin.clear();
    D.all_begin.clear();
    D.all_count.clear();
    for (const LevelPlan& lp : P_.levels) {
        D.small_begin.push_back((int64_t)small.size());
        small.insert(small.end(), lp.small_nodes.begin(), lp.small_nodes.end());
        D.all_begin.push_back((int64_t)all.size());
        all.insert(all.end(), lp.small_nodes.begin(), lp.small_nodes.end());
        all.insert(all.end(), lp.large_nodes.begin(), lp.large_nodes.end());
        D.all_count.push_back((int64_t)(lp.small_nodes.size() + lp.large_nodes.size()));
    }
    if (dev_upload(o, &D.level_nodes, small) || dev_upload(o, &D.all_nodes, all)) return -4;
    D.ret = nullptr;
    if (P_.any_retained && dev_upload(o, &D.ret, P_.retained)) return -4;
    CK(cudaMalloc((void**)&D.arena, std::max<int64_t>(P_.arena_doubles, 32) * sizeof(double)));
    CK(cudaMalloc((void**)&D.adiag, P_.neq * sizeof(double)));
    o.push_back(D.adiag);
    CK(cudaMalloc((void**)&D.sn_neg, P_.nsuper * sizeof(int32_t)));
    o.push_back(D.sn_neg);
    CK(cudaMalloc((void**)&D.sn_fail, P_.nsuper * sizeof(int32_t)));
    o.push_back(D.sn_fail);
    CK(cudaMalloc((void**)&D.sn_bad, P_.nsuper * sizeof(int32_t)));
    o.push_back(D.sn_bad);
    CK(cudaMalloc((void**)&D.sn_faild, P_.nsuper * sizeof(double)));
    o.push_back(D.sn_faild);
    CK(cudaMalloc((void**)&D.sn_faila, P_.nsuper * sizeof(double)));
    o.push_back(D.sn_faila);
    CK(cudaMalloc((void**)&D.st, sizeof(Stats)));
    o.push_back(D.st);
    CK(cudaMalloc((void**)&D.hbuf, sizeof(unsigned long long)));
    o.push_back(D.hbuf);
    if (dev_upload(o, &D.tri_tasks, P_.tri_tasks)) return -4;
    if (dev_upload(o, &D.tri_off, P_.tri_off)) return -4;
    CK(cudaMalloc((void**)&D.tri_sync, sizeof(int32_t) * (size_t)(P_.tri_flags + 2 * (int64_t)P_.levels.size() + 2)));
    o.push_back(D.tri_sync);
    {
        const char* v = std::getenv("SPR_B200_SOLVE_BLOCKS");
        tri_solve_ = !(v && v[0] == '1');
    }
    CK(cudaHostAlloc((void**)&D.mbox, 32 * sizeof(unsigned long long), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&D.mbox_dev, D.mbox, 0));
    CK(cudaEventCreate(&D.ev0));
    CK(cudaEventCreate(&D.ev1));
    int smem_max = 0;
    CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t need = ((size_t)kSmallMaxF * (kSmallMaxF + 1) / 2 + 2 * kSmallMaxF) * sizeof(double);
    if ((size_t)smem_max < need) return -4;
    CK(cudaFuncSetAttribute(k_small_front<kPivotLDL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    CK(cudaFuncSetAttribute(k_small_front<kPivotReplace>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    CK(cudaFuncSetAttribute(k_small_front<kPivotChol>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    CK(cudaFuncSetAttribute(k_small_front<kPivotChol4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    CK(cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
    CK(cudaFuncSetAttribute(k_fwd_blk_mv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMvSmem));
    CK(cudaFuncSetAttribute(k_fwd_blk_upd2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem));
    CK(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSolveSmem));
    CK(cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSolveSmem));
    CK(cudaFuncSetAttribute(k_inv_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem));
    CK(cudaFuncSetAttribute(K_GEMM_BIG, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GemmBig::smem));
    CK(cudaFuncSetAttribute(K_GEMM_SMALL, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GemmSmall::smem));
    CK(cudaFuncSetAttribute(K_GEMM_TINY, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GemmTiny::smem));
    CK(cudaFuncSetAttribute(k_gemm_x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GemmSmall::smem));
    CK(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kSmem));
    return 0;
}

// Operand slabs of the tensor-core updates and the 2-D TMA map over them:
// [slab_rows][32] fp32, box 32 x 128 rows, 128-byte swizzle.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int make_slab(int64_t rows_needed, float** slab, CUtensorMap* map) {
    const int64_t rows = std::max<int64_t>(rows_needed, tc::kTM);
    if (rows >= (int64_t(1) << 31)) return -3;                 // TMA row coordinates are 32-bit
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
        return -4;
    CK(cudaMalloc((void**)slab, rows * tc::kBK * sizeof(float)));
    const cuuint64_t dims[2] = {(cuuint64_t)tc::kBK, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)tc::kBK * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)tc::kBK, (cuuint32_t)tc::kTM};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = ((EncodeTiledFn)fn)(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, *slab, dims, strides, box, es,
                                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        cudaFree(*slab);
        *slab = nullptr;
        return -4;
    }
    return 0;
}

int Engine::ensure_slabs() {
    Dev& D = *d_;
    if (D.slab && D.slab_far) return 0;
    if (!D.slab) {
        const int rc = make_slab(P_.slab_rows, &D.slab, &D.slab_map);
        if (rc != 0) return rc;
    }
    if (!D.slab_far) return make_slab(P_.slab_rows_far, &D.slab_far, &D.slab_map_far);
    return 0;
}


static cudaEvent_t record_event(cudaStream_t s) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    return e;
}

static PV make_view(Engine::Dev& D, const Plan& P, double* d_sm, double tol1) {
    PV v;
    v.fst = D.fst;
    v.S = D.S;
    v.F = D.F;
    v.child_ptr = D.child_ptr;
    v.child = D.child;
    v.rows = D.rows;
    v.rel = D.rel;
    v.cchild = D.cchild;
    v.ct = D.ct;
    v.buf_ld = D.buf_ld;
    v.lnz_off = D.lnz_off;
    v.rel_off = D.rel_off;
    v.rbase = D.rbase;
    v.cptr = D.cptr;
    v.buf_off = D.buf_off;
    v.upd_off = D.upd_off;
    v.arena = D.arena;
    v.dvec = d_sm;
    v.lnz = d_sm + P.neq;
    v.adiag = D.adiag;
    v.sn_neg = D.sn_neg;
    v.sn_fail = D.sn_fail;
    v.sn_bad = D.sn_bad;
    v.sn_faild = D.sn_faild;
    v.sn_faila = D.sn_faila;
    v.st = D.st;
    v.linv_off = D.linv_off;
    v.linv = D.linv;
    v.xinv_off = D.xinv_off;
    v.xinv = D.xinv;
    v.rect_off = D.rect_off;
    v.fwd_off = D.fwd_off;
    v.tri_off = D.tri_off;
    v.tol1 = tol1;
    v.fc3 = 0;
    v.tol4 = 0.0;
    v.dcor = nullptr;
    v.ret = D.ret;
    v.near_tol = 0.0;
    v.wait_ns = 2000000000ull;
    v.tc_drop = 0;
    v.adiag_in = nullptr;
    v.skip = D.skip_on ? D.skip : nullptr;
    return v;
}

void Engine::launch_diag(const Launch& pl, cudaStream_t s, const PV& pv) {
    const Job* jobs = d_->jobs + pl.job_begin;
    const int n = (int)pl.job_count;
    if (pv.fc3 == 2) k_diag<kPivotChol4><<<n, 256, 0, s>>>(jobs, pv);
    else if (pv.fc3) k_diag<kPivotReplace><<<n, 256, 0, s>>>(jobs, pv);
    else if (chol_) k_diag<kPivotChol><<<n, 256, 0, s>>>(jobs, pv);
    else k_diag<kPivotLDL><<<n, 256, 0, s>>>(jobs, pv);
}

void Engine::launch_gemm(const Launch& l, cudaStream_t s, const PV& pv, std::vector<cudaEvent_t>& gev) {
    if (l.ntasks <= 0) return;
    if (profile_) gev.push_back(record_event(s));
    const Job* jobs = d_->jobs + l.job_begin;
    if (mixed_ == 2) {
        k_gemm_x3<<<(int)l.ntasks, 128, GemmSmall::smem, s>>>(jobs, l.job_count, TMAP(l), pv);
    } else if (l.tile == kTileBig) {
        K_GEMM_BIG<<<(int)l.ntasks, GemmBig::NT, GemmBig::smem, s>>>(jobs, l.job_count, TMAP(l), pv);
    } else if (small_tile_ == kTileTiny && l.alt >= 0) {
        const Launch& a = P_.alt[l.alt];
        K_GEMM_TINY<<<(int)a.ntasks, GemmTiny::NT, GemmTiny::smem, s>>>(d_->jobs + a.job_begin, a.job_count,
                                                                       TMAP(a), pv);
    } else {
        K_GEMM_SMALL<<<(int)l.ntasks, GemmSmall::NT, GemmSmall::smem, s>>>(jobs, l.job_count, TMAP(l), pv);
    }
    if (profile_) gev.push_back(record_event(s));
    ++timing.launches;
    ++timing.gemm_launches;
}

void Engine::launch_tc(const TcLaunch& t, cudaStream_t s, const PV& pv, std::vector<cudaEvent_t>& gev, bool far) {
    if (t.gemm.ntasks <= 0) return;
    Dev& D = *d_;
    if (profile_) {
        tc_pairs_.push_back(gev.size());
        gev.push_back(record_event(s));
    }
    k_split_tc<<<(int)t.split.ntasks, 256, 0, s>>>(D.jobs + t.split.job_begin, t.split.job_count, TMAP(t.split), pv,
                                                   far ? D.slab_far : D.slab);
    // a side-stream launch leaves a quarter of the SMs to the panel chain
    // (a persistent tensor-core CTA holds most of an SM's shared memory)
    const int cap = (far && !profile_) ? std::max(1, sm_count_ * far_cap_q_ / 4) : sm_count_;
    const int grid = (int)std::min<int64_t>(t.gemm.ntasks, cap);
    k_gemm_tc<<<grid, tc::kThreads, tc::kSmem, s>>>(D.jobs + t.gemm.job_begin, t.gemm.job_count, TMAP(t.gemm),
                                                    t.gemm.ntasks, pv, far ? D.slab_map_far : D.slab_map);
    if (profile_) gev.push_back(record_event(s));
    timing.launches += 2;
    ++timing.gemm_launches;
}

// ---------------------------------------------------------------------------
// Split across GPUs: node mask and the exchange of subtree roots' update
// blocks (factor) and update vectors (forward solve).
// ---------------------------------------------------------------------------
int Engine::set_skip(const uint8_t* host_mask) {
    Dev& D = *d_;
    if (!host_mask) {
        D.skip_on = false;
        split_ = !fout_.empty() || !fin_.empty() || !vout_.empty() || !vin_.empty();
        return 0;
    }
    if (!D.skip) {
        CK(cudaMalloc((void**)&D.skip, std::max<int64_t>(P_.nsuper, 1)));
        D.owned.push_back(D.skip);
    }
    CK(cudaMemcpy(D.skip, host_mask, P_.nsuper, cudaMemcpyHostToDevice));
    D.skip_on = true;
    split_ = true;
    return 0;
}

void Engine::set_exchange(std::vector<Xfer> fo, std::vector<Xfer> fi, std::vector<Xfer> vo, std::vector<Xfer> vi) {
    fout_ = std::move(fo);
    fin_ = std::move(fi);
    vout_ = std::move(vo);
    vin_ = std::move(vi);
    split_ = d_->skip_on || !fout_.empty() || !fin_.empty() || !vout_.empty() || !vin_.empty();
}

// node js's update block <-> buf ((F-S) x (F-S), leading dimension F-S)
void Engine::block_copy(int32_t js, double* buf, bool out, cudaStream_t s) {
    const int64_t q = P_.F[js] - P_.S[js];
    if (q <= 0) return;
    double* blk = d_->arena + P_.upd_off[js];
    const size_t ld = (size_t)P_.buf_ld[js] * sizeof(double), w = (size_t)q * sizeof(double);
    if (out)
        cudaMemcpy2DAsync(buf, w, blk, ld, w, q, cudaMemcpyDeviceToDevice, s);
    else
        cudaMemcpy2DAsync(blk, ld, buf, w, w, q, cudaMemcpyDeviceToDevice, s);
}

// node js's forward update vector (rows [S, F) of its front vector, per RHS) <-> buf ((F-S) x nrhs)
void Engine::vec_copy(int32_t js, double* buf, bool out, int64_t nrhs, cudaStream_t s) {
    const int64_t f = P_.F[js], q = f - P_.S[js];
    if (q <= 0) return;
    double* v = d_->vbuf + P_.rbase[js] * nrhs + P_.S[js];
    const size_t ld = (size_t)f * sizeof(double), w = (size_t)q * sizeof(double);
    if (out)
        cudaMemcpy2DAsync(buf, w, v, ld, w, nrhs, cudaMemcpyDeviceToDevice, s);
    else
        cudaMemcpy2DAsync(v, ld, buf, w, w, nrhs, cudaMemcpyDeviceToDevice, s);
}

namespace {
// The exchange lists as level hooks: "in" entries before their parent's
// level, "out" entries after their node's level.
struct ExchangeHooks : LevelHooks {
    const Plan* P = nullptr;
    const std::vector<Engine::Xfer>* out = nullptr;
    const std::vector<Engine::Xfer>* in = nullptr;
    std::function<void(int32_t, double*, bool, cudaStream_t)> copy;
    void before(size_t L, cudaStream_t s) const override {
        for (const Engine::Xfer& x : *in) {
            const int32_t p = P->parent[x.node];
            if (p >= 0 && (size_t)P->level[p] == L) copy(x.node, x.buf, false, s);
        }
    }
    void after(size_t L, cudaStream_t s) const override {
        for (const Engine::Xfer& x : *out)
            if ((size_t)P->level[x.node] == L) copy(x.node, x.buf, true, s);
    }
};
}  // namespace

// Copies n 8-byte words to the mailbox (one thread per word).
__global__ void k_mailbox(const unsigned long long* src, int n, unsigned long long* dst) {
    const int i = threadIdx.x;
    if (i < n) dst[i] = src[i];
}

void Engine::enqueue_factor(const PV& pv, cudaStream_t s, std::vector<cudaEvent_t>& gev) {
    Dev& D = *d_;
    timing.launches = 0;
    timing.tc_flops = 0.0;
    auto mark = [&](int phase) {
        if (profile_) marks_.emplace_back(phase, record_event(s));
    };
    // side stream for the trailing-update columns beyond the next super-panel,
    // look-ahead stream for the in-super-panel columns after the next panel
    // (profile mode keeps everything on one stream so the events time it)
    cudaStream_t u = (profile_ || !D.side) ? s : D.side;
    cudaStream_t la = (profile_ || !D.ahead) ? s : D.ahead;
    size_t evi = 0;
    cudaEvent_t far_done = nullptr, ahead_done = nullptr;
    auto join_far = [&]() {
        if (far_done) {
            cudaStreamWaitEvent(s, far_done, 0);
            far_done = nullptr;
        }
    };
    auto join_ahead = [&]() {
        if (ahead_done) {
            cudaStreamWaitEvent(s, ahead_done, 0);
            ahead_done = nullptr;
        }
    };
    mark(0);
    k_prepass<<<(int)std::min<int64_t>((P_.nsuper * 32 + 255) / 256, 4736), 256, 0, s>>>(pv, P_.nsuper);
    k_reduce<false><<<1, 1024, 0, s>>>(D.adiag, P_.neq, &D.st->trace);
    timing.launches += 2;
    char lname[48];
    for (size_t L = 0; L < P_.levels.size(); ++L) {
        const LevelPlan& lp = P_.levels[L];
        snprintf(lname, sizeof lname, "factor level %zu", L);
        NvtxRange level_range(lname);
        trace_point(lname);
        if (hooks_) hooks_->before(L, s);
        struct AfterLevel {                      // runs at every exit of this iteration
            const LevelHooks* h;
            size_t L;
            cudaStream_t s;
            ~AfterLevel() {
                if (h) h->after(L, s);
            }
        } after_level{hooks_, L, s};
        if (!lp.small_nodes.empty()) {
            mark(1);
            for (const LevelPlan::SmallClass& c : lp.small_classes) {
                const int F = c.maxF;
                const size_t smem = ((size_t)F * (F + 1) / 2 + 2 * F) * sizeof(double);
                const int thr = small_threads(F);
                const int32_t* nodes = D.level_nodes + D.small_begin[L] + c.begin;
                if (pv.fc3 == 2)
                    k_small_front<kPivotChol4><<<c.count, thr, smem, s>>>(nodes, pv);
                else if (pv.fc3)
                    k_small_front<kPivotReplace><<<c.count, thr, smem, s>>>(nodes, pv);
                else if (chol_)
                    k_small_front<kPivotChol><<<c.count, thr, smem, s>>>(nodes, pv);
                else
                    k_small_front<kPivotLDL><<<c.count, thr, smem, s>>>(nodes, pv);
                ++timing.launches;
            }
        }
        if (lp.large_nodes.empty()) continue;
        const Job* jobs = D.jobs;
        const bool early = hooks_ && hooks_->early_columns(L);
        bool wrote_early = false;
        {
            mark(2);
            const Launch& l = lp.assemble;
            k_poison<<<(int)((l.job_count + 127) / 128), 128, 0, s>>>(jobs + l.job_begin, l.job_count, TMAP(l), pv);
            const int64_t threads = l.ntasks * 32;
            k_assemble<<<(int)((threads + 255) / 256), 256, 0, s>>>(jobs + l.job_begin, l.job_count, TMAP(l), l.ntasks, pv);
            ++timing.launches;
        }
        for (size_t st = 0; st < lp.panel.size(); ++st) {
            const Launch& pl = lp.panel[st];
            mark(3);
            launch_diag(pl, s, pv);
            ++timing.launches;
            if (pl.ntasks > 0) {
                mark(4);
                k_trsm<<<(int)pl.ntasks, 128, kTrsmSmem, s>>>(jobs + pl.job_begin, pl.job_count, TMAP(pl), pv);
                ++timing.launches;
            }
            const bool has_far = !lp.far[st].empty() || !lp.far_tc[st].empty();
            const bool far_tc = mixed_ == 1 && lp.far_flops[st] >= tc_min_flops_;
            if (has_far && u != s) {
                // the super-panel is final: fork the far columns of its trailing update
                cudaEvent_t e = D.evpool[evi++];
                cudaEventRecord(e, s);
                cudaStreamWaitEvent(u, e, 0);
            }
            if (early && st < lp.wb_sp.size() && lp.wb_sp[st].ntasks > 0) {
                // super-panels that end here are final: write them to LNZ beside
                // the rest of the level, for the caller to copy early
                const Launch& w = lp.wb_sp[st];
                cudaEvent_t e = D.evpool[evi++];
                cudaEventRecord(e, s);
                cudaStreamWaitEvent(D.wbs, e, 0);
                k_writeback<<<(int)((w.ntasks * 32 + 255) / 256), 256, 0, D.wbs>>>(jobs + w.job_begin, w.job_count,
                                                                                 TMAP(w), w.ntasks, pv);
                ++timing.launches;
                hooks_->columns_written(L, st, D.wbs);
                wrote_early = true;
            }
            mark(5);
            // a trailing update's next-super-panel columns were also updated by
            // the previous super-panel's far launch: wait for it first
            if ((st + 1) % (kSuperPanel / kNB) == 0) join_far();
            // the previous step's look-ahead update also wrote the columns
            // that this step's chain update is about to update
            join_ahead();
            cudaEvent_t fork_ahead = nullptr;
            if (!lp.ahead[st].empty() && la != s) {
                fork_ahead = D.evpool[evi++];
                cudaEventRecord(fork_ahead, s);
            }
            // the updates inside the panel chain (K = 64: the next panel's
            // columns; K = kSuperPanel: the next super-panel's columns) are on the
            // critical path.  The K = 64 ones are small: the FP64 kernel's
            // 64x64 tiles start sooner than a split + tensor-core pair, so they
            // stay FP64 in both modes; in mixed mode the K = kSuperPanel one takes the
            // tensor cores when large enough.  They are issued first, the
            // look-ahead columns after them.
            if (mixed_ == 1 && !lp.next_tc[st].empty() && lp.next_flops[st] >= tc_min_flops_) {
                for (const TcLaunch& t : lp.next_tc[st]) launch_tc(t, s, pv, gev);
                timing.tc_flops += lp.next_flops[st];
            } else {
                for (const Launch& ul : lp.update[st]) launch_gemm(ul, s, pv, gev);
            }
            if (!lp.ahead[st].empty()) {
                if (fork_ahead) cudaStreamWaitEvent(la, fork_ahead, 0);
                for (const Launch& al : lp.ahead[st]) launch_gemm(al, la, pv, gev);
                if (la != s) {
                    ahead_done = D.evpool[evi++];
                    cudaEventRecord(ahead_done, la);
                }
            }
            if (has_far) {
                if (far_tc) {
                    for (const TcLaunch& t : lp.far_tc[st]) launch_tc(t, u, pv, gev, true);
                    timing.tc_flops += lp.far_flops[st];
                }
                else {
                    for (const Launch& fl : lp.far[st]) launch_gemm(fl, u, pv, gev);
                }
                if (u != s) {
                    far_done = D.evpool[evi++];
                    cudaEventRecord(far_done, u);
                }
            }
        }
        join_ahead();
        join_far();
        mark(6);
        if (mixed_ == 1 && lp.outer_flops >= tc_min_flops_) {
            for (const TcLaunch& t : lp.outer_tc) launch_tc(t, s, pv, gev);
            timing.tc_flops += lp.outer_flops;
        } else
            for (const Launch& ol : lp.outer) launch_gemm(ol, s, pv, gev);
        if (wrote_early) {
            // the level's own write-back rewrites the same values: after the early ones
            cudaEvent_t e = D.evpool[evi++];
            cudaEventRecord(e, D.wbs);
            cudaStreamWaitEvent(s, e, 0);
        }
        {
            mark(7);
            const Launch& l = lp.writeback;
            const int64_t threads = l.ntasks * 32;
            k_writeback<<<(int)((threads + 255) / 256), 256, 0, s>>>(jobs + l.job_begin, l.job_count, TMAP(l), l.ntasks, pv);
            ++timing.launches;
        }
    }
    mark(8);
    if (!tri_solve_ && P_.inv_blocks.job_count > 0) {
        k_inv_block<<<(int)P_.inv_blocks.job_count, 256, kInvSmem, s>>>(D.jobs + P_.inv_blocks.job_begin, pv);
        ++timing.launches;
    }
    k_reduce<true><<<1, 1024, 0, s>>>(pv.dvec, P_.neq, &D.st->mindpos);
    ++timing.launches;
}

int Engine::factor(double* d_sm, double tol1, FactorResult& res, const Singular* fc3) {
    NvtxRange range("spr_b200 factor");
    Dev& D = *d_;
    cudaStream_t s = stream_;
    PV pv = make_view(D, P_, d_sm, tol1);
    if (fc3) {
        if (!fc3->d_dcor) return -2;
        pv.fc3 = chol_ ? 2 : 1;               // SPRF47 (SPRFC4) or SPRF37 (SPRFC3)
        pv.tol4 = fc3->tol4;
        pv.dcor = fc3->d_dcor;
    }
    pv.wait_ns = wait_ns_;
    pv.tc_drop = tc_drop_ ? 1 : 0;
    pv.adiag_in = streamed_diag_;
    linv_valid_ = false;
    last_near_ = 0;
    last_refactor_ = false;
    if (mixed_ == 1) {
        const int rc = ensure_slabs();
        if (rc != 0) return rc;
    }
    // inertia guard: keep the assembled SM, so that the factorisation can be
    // redone in FP64 when a pivot's sign may depend on the TF32 rounding
    const bool guard = mixed_ != 0 && guard_tol_ > 0.0;
    const int64_t nsm = P_.neq + P_.nzerol;
    if (guard) {
        if (guard_cap_ < nsm) {
            if (guard_copy_) cudaFree(guard_copy_);
            guard_copy_ = nullptr;
            guard_cap_ = 0;
            CK(cudaMalloc((void**)&guard_copy_, nsm * sizeof(double)));
            guard_cap_ = nsm;
        }
        CK(cudaMemcpyAsync(guard_copy_, d_sm, nsm * sizeof(double), cudaMemcpyDeviceToDevice, s));
        pv.near_tol = guard_tol_;
    }
    Stats init{};
    init.first_zero = 0x7fffffff;
    CK(cudaMemcpyAsync(D.st, &init, sizeof(Stats), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(D.sn_neg, 0, P_.nsuper * sizeof(int32_t), s));
    CK(cudaMemsetAsync(D.sn_fail, 0xff, P_.nsuper * sizeof(int32_t), s));
    CK(cudaMemsetAsync(D.sn_bad, 0, P_.nsuper * sizeof(int32_t), s));
    timing.gemm_ms = 0.f;
    timing.gemm_launches = 0;
    tc_pairs_.clear();
    CK(cudaEventRecord(D.ev0, s));
    std::vector<cudaEvent_t> gev;
    // the legacy default stream cannot be captured: graphs need a stream of our own;
    // the watchdog test launches kernel by kernel (its settings are not in the key)
    // a streamed factorisation enqueues its copies' waits between the levels;
    // a split run its exchanges
    ExchangeHooks xh;
    const LevelHooks* saved_hooks = hooks_;
    if (split_ && !hooks_) {
        xh.P = &P_;
        xh.out = &fout_;
        xh.in = &fin_;
        xh.copy = [this](int32_t js, double* b, bool o, cudaStream_t st) { block_copy(js, b, o, st); };
        hooks_ = &xh;
    }
    struct RestoreHooks {
        const LevelHooks** h;
        const LevelHooks* v;
        ~RestoreHooks() { *h = v; }
    } restore{&hooks_, saved_hooks};
    const bool graph = use_graphs_ && !profile_ && s != nullptr && !tc_drop_ && wait_ns_ == 2000000000ull && !hooks_;
    if (graph) {
        const GraphKey key{(const void*)d_sm, nullptr, tol1, far_cap_q_,
                           mixed_ | (chol_ ? 16 : 0) | (small_tile_ == kTileTiny ? 32 : 0),
                           (int64_t)std::min(tc_min_flops_, 9.0e18), (const void*)pv.dcor, pv.tol4,
                           pv.near_tol};
        cudaGraphExec_t exec = find_graph(key);
        if (!exec) {
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            enqueue_factor(pv, s, gev);
            cudaGraph_t g = nullptr;
            CK(cudaStreamEndCapture(s, &g));
            CK(cudaGraphInstantiate(&exec, g, 0));
            cudaGraphDestroy(g);
            store_graph(key, exec, timing.launches);
        } else {
            timing.launches = graph_launches(key);
        }
        CK(cudaGraphLaunch(exec, s));
    } else {
        enqueue_factor(pv, s, gev);
    }
    trace_point(graph ? "factor graph launched" : "factor launches enqueued");
    CK(cudaEventRecord(D.ev1, s));
    CK(cudaGetLastError());
    Stats hs;
    static_assert(sizeof(Stats) % 8 == 0 && sizeof(Stats) / 8 <= 32, "Stats fits the mailbox");
    k_mailbox<<<1, 32, 0, s>>>(reinterpret_cast<const unsigned long long*>(D.st), (int)(sizeof(Stats) / 8),
                               D.mbox_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    std::memcpy(&hs, D.mbox, sizeof(Stats));
    trace_point("factor stream synchronised");
    CK(cudaEventElapsedTime(&timing.factor_ms, D.ev0, D.ev1));
    timing.tc_ms = 0.f;
    size_t tp = 0;
    for (size_t k = 0; k + 1 < gev.size(); k += 2) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, gev[k], gev[k + 1]);
        timing.gemm_ms += ms;
        if (tp < tc_pairs_.size() && tc_pairs_[tp] == k) {
            timing.tc_ms += ms;
            ++tp;
        }
    }
    tc_pairs_.clear();
    for (cudaEvent_t e : gev) cudaEventDestroy(e);
    for (int k = 0; k < 9; ++k) timing.phase_ms[k] = 0.f;
    for (size_t k = 0; k < marks_.size(); ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, marks_[k].second, k + 1 < marks_.size() ? marks_[k + 1].second : D.ev1);
        timing.phase_ms[marks_[k].first] += ms;
        cudaEventDestroy(marks_[k].second);
    }
    marks_.clear();
    res = FactorResult();
    last_trace_ = hs.trace;
    if (hs.tc_timeout) {
        fprintf(stderr, "spr_b200: a tensor-core update gave up waiting for its operands\n");
        return -4;
    }
    if (guard && (hs.near_piv > 0 || (hs.pivot_fail && hs.zero_count == 0))) {
        // a pivot within guard_tol_ |a_jj| of zero, or a failed pivot test,
        // after TF32 updates: decide inertia and the pivot test in FP64
        const float first_ms = timing.factor_ms;
        const int64_t near = (int64_t)hs.near_piv;
        CK(cudaMemcpyAsync(d_sm, guard_copy_, nsm * sizeof(double), cudaMemcpyDeviceToDevice, s));
        const int mode = mixed_;
        mixed_ = 0;
        const int rc = factor(d_sm, tol1, res, fc3);
        mixed_ = mode;
        timing.factor_ms += first_ms;
        last_near_ = near;
        last_refactor_ = true;
        return rc;
    }
    last_near_ = (int64_t)hs.near_piv;
    if (hs.zero_count > 0) {                       // sprfc1.f:474-488
        // the reference's pre-pass has already replaced D by the original diagonal
        CK(cudaMemcpy(pv.dvec, D.adiag, P_.neq * sizeof(double), cudaMemcpyDeviceToDevice));
        res.lierr = -35;
        res.numneg = hs.zero_count;
        res.supeqt = (int64_t)hs.first_zero + 1;
        res.tol2 = 0.0;
        res.tol3 = hs.trace;
        return 0;
    }
    if (hs.pivot_fail) {                           // sprfc1.f:610-616
        std::vector<int32_t> fail(P_.nsuper), neg(P_.nsuper);
        CK(cudaMemcpy(fail.data(), D.sn_fail, P_.nsuper * sizeof(int32_t), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(neg.data(), D.sn_neg, P_.nsuper * sizeof(int32_t), cudaMemcpyDeviceToHost));
        int64_t jf = -1;
        for (int64_t js = 0; js < P_.nsuper; ++js)
            if (fail[js] >= 0) {
                jf = js;
                break;
            }
        int64_t nn = 0;
        for (int64_t js = 0; js <= jf; ++js) nn += neg[js];
        double fd = 0.0, fa = 0.0;
        CK(cudaMemcpy(&fd, D.sn_faild + jf, sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&fa, D.sn_faila + jf, sizeof(double), cudaMemcpyDeviceToHost));
        res.lierr = -30;
        res.numneg = nn;
        res.supeqt = (int64_t)P_.fst[jf] + fail[jf] + 1;
        res.tol2 = fd;
        res.tol3 = fa;
        return 0;
    }
    linv_valid_ = true;
    if (fc3 && hs.nsing > 0) {                     // sprfc3.f:796-799, sprfc4.f:719-722
        res.lierr = chol_ ? -33 : -31;
        res.supeqt = (int64_t)hs.nsing;
    }
    res.numneg = hs.numneg;
    res.tol2 = (hs.tol2 != 0.0) ? 1.0 / hs.tol2 : 0.0;          // sprfc1.f:699-703
    res.tol3 = (hs.mindpos != 0.0) ? hs.trace / hs.mindpos : 0.0;  // sprfc1.f:704-708
    if (chol_) {                                                   // sprfc2.f:699-716
        const double m = std::sqrt(hs.mindpos);
        res.tol3 = (m != 0.0) ? hs.trace / (m * m) : 0.0;
    }
    return 0;
}

int Engine::hash(const double* d_a, int64_t n, uint64_t& h) {
    Dev& D = *d_;
    unsigned long long hv = 0ull;
    CK(cudaMemsetAsync(D.hbuf, 0, sizeof(unsigned long long), stream_));
    if (n > 0) {
        const int grid = (int)std::min<int64_t>((n + 255) / 256, 8 * (int64_t)std::max(sm_count_, 1));
        k_sm_hash<<<grid, 256, 0, stream_>>>(d_a, n, D.hbuf);
        CK(cudaGetLastError());
    }
    k_mailbox<<<1, 32, 0, stream_>>>(D.hbuf, 1, D.mbox_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
    hv = D.mbox[0];
    h = (uint64_t)hv;
    return 0;
}

// dst[0 .. n) = src[0 .. n) on the device (the early fronts' backup).
__global__ void k_copy_d(const double* __restrict__ src, double* __restrict__ dst, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

namespace {
// Host-side pacing of the streamed copies.  Hundreds of queued copy
// operations make the next kernel launch wait until they drain, and copies
// in one direction share the copy engine whatever their stream, so neither
// all uploads nor all downloads are queued at once: one thread queues a
// group's uploads once the group two below it is up, another queues a
// group's downloads once its last level has finished on the device.  The
// enqueueing thread waits, before a level's first launch, until that level's
// upload event has been recorded, and marks each group's end event as
// recorded after its last level.
struct CopyScheduler {
    // a download: once ev has completed, copy these LNZ ranges to the host
    struct Item {
        cudaEvent_t ev;
        const std::vector<std::pair<int64_t, int64_t>>* ranges;
        bool last;
    };
    std::mutex mu;
    std::condition_variable cv;
    std::vector<char> up_recorded;
    std::deque<Item> downloads;                 // in the order the enqueueing thread recorded them
    bool abort = false;
    int status = 0;
    void push(const Item& it) {
        {
            std::lock_guard<std::mutex> lk(mu);
            downloads.push_back(it);
        }
        cv.notify_all();
    }
    bool pop(Item& it) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !downloads.empty() || abort; });
        if (downloads.empty()) return false;
        it = downloads.front();
        downloads.pop_front();
        return true;
    }
    void mark(std::vector<char>& v, size_t g) {
        {
            std::lock_guard<std::mutex> lk(mu);
            v[g] = 1;
        }
        cv.notify_all();
    }
    bool wait(std::vector<char>& v, size_t g) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return v[g] != 0 || abort; });
        return v[g] != 0;
    }
    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu);
            abort = true;
        }
        cv.notify_all();
    }
};

struct StreamHooks : LevelHooks {
    const Engine::Transfer* t = nullptr;
    CopyScheduler* cs_sched = nullptr;
    double* d_lnz = nullptr;
    int sm_count = 148;
    size_t nlev = 0;
    void before(size_t L, cudaStream_t s) const override {
        const int g = t->group((int32_t)L);
        if (L == 0 || (g > 0)) {
            if (!cs_sched->wait(cs_sched->up_recorded, (size_t)g)) return;
            cudaStreamWaitEvent(s, t->up[g], 0);
        }
        if ((int32_t)L == t->early_level) {
            // the early fronts' uploaded LNZ, kept in case a pivot of theirs fails
            int64_t b = 0;
            for (const auto& r : t->early_ranges) {
                k_copy_d<<<2 * sm_count, 256, 0, s>>>(d_lnz + r.first, t->d_backup + b, r.second);
                b += r.second;
            }
        }
    }
    void after(size_t L, cudaStream_t s) const override {
        const int g = t->group((int32_t)L);
        const bool last_of_group = (L + 1 == nlev) || t->group((int32_t)(L + 1)) != g;
        if (!last_of_group) return;
        cudaEventRecord(t->done[g], s);
        cs_sched->push({t->done[g], &t->dranges[g], (size_t)g + 1 == t->dranges.size()});
    }
    bool early_columns(size_t L) const override { return (int32_t)L == t->early_level; }
    void columns_written(size_t L, size_t st, cudaStream_t ws) const override {
        cudaEventRecord(t->spev[st], ws);
        cs_sched->push({t->spev[st], &t->spranges[st], false});
    }
};
}  // namespace

int Engine::factor_streamed(double* h_sm, double* d_sm, double tol1, FactorResult& res, cudaStream_t cs) {
    NvtxRange range("spr_b200 factor (streamed copies)");
    const int64_t neq = P_.neq;
    if (!xfer_) {
        std::unique_ptr<Transfer> t(new Transfer());
        const int32_t nlev = (int32_t)P_.levels.size();
        std::vector<int64_t> at_level(nlev + 1, 0);
        for (int64_t js = 0; js < P_.nsuper; ++js) ++at_level[P_.level[js]];
        int64_t above = 0;
        t->L1 = nlev;
        for (int32_t L = nlev - 1; L >= 1; --L) {
            above += at_level[L];
            if (above > Transfer::kMaxTopNodes) break;
            t->L1 = L;
        }
        const int ng = 1 + (nlev - t->L1);
        // the last level's eliminated large fronts: their columns come back
        // super-panel by super-panel, not with the level's group
        std::vector<char> early(P_.nsuper, 0);
        if (nlev > 0) {
            const LevelPlan& lp = P_.levels[nlev - 1];
            t->spranges.assign(lp.wb_sp.size(), {});
            for (size_t st = 0; st < lp.wb_sp.size(); ++st) {
                const Launch& w = lp.wb_sp[st];
                for (int64_t j = 0; j < w.job_count; ++j) {
                    const Job& jb = P_.jobs[w.job_begin + j];
                    const int64_t f = P_.F[jb.node];
                    const int64_t a = P_.lnz_off[jb.node] + lnz_col(jb.c0, f);
                    t->spranges[st].emplace_back(a, lnz_col(jb.c_end, f) - lnz_col(jb.c0, f));
                    early[jb.node] = 1;
                    t->early_level = nlev - 1;
                }
            }
            t->spev.resize(lp.wb_sp.size());
            for (cudaEvent_t& e : t->spev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        t->ranges.assign(ng, {});
        t->dranges.assign(ng, {});
        auto append = [](std::vector<std::pair<int64_t, int64_t>>& rg, int64_t off, int64_t len) {
            if (!rg.empty() && rg.back().first + rg.back().second == off)
                rg.back().second += len;
            else
                rg.emplace_back(off, len);
        };
        int64_t nbackup = 0;
        for (int64_t js = 0; js < P_.nsuper; ++js) {
            const int64_t f = P_.F[js], sw = P_.S[js];
            const int64_t off = P_.lnz_off[js], len = f * sw - sw * (sw - 1) / 2;
            const int g = t->group(P_.level[js]);
            append(t->ranges[g], off, len);
            if (early[js]) {
                t->early_nodes.push_back((int32_t)js);
                t->early_ranges.emplace_back(off, len);
                nbackup += len;
            } else {
                append(t->dranges[g], off, len);
            }
        }
        if (nbackup > 0) CK(cudaMalloc((void**)&t->d_backup, nbackup * sizeof(double)));
        t->up.resize(ng);
        t->done.resize(ng);
        for (int g = 0; g < ng; ++g) {
            CK(cudaEventCreateWithFlags(&t->up[g], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&t->done[g], cudaEventDisableTiming));
        }
        CK(cudaStreamCreateWithFlags(&t->ups, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&t->start, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&t->fin, cudaEventDisableTiming));
        CK(cudaEventCreate(&t->ts));
        CK(cudaEventCreate(&t->tu));
        CK(cudaEventCreate(&t->te));
        CK(cudaEventCreate(&t->tf));
        CK(cudaEventCreate(&t->tf0));
        t->diag_pos.resize(neq);
        for (int64_t js = 0; js < P_.nsuper; ++js)
            for (int64_t j = 0; j < P_.S[js]; ++j) t->diag_pos[P_.fst[js] + j] = P_.lnz_off[js] + lnz_col(j, P_.F[js]);
        CK(cudaMallocHost((void**)&t->h_diag, std::max<int64_t>(neq, 1) * sizeof(double)));
        CK(cudaMalloc((void**)&t->d_diag, std::max<int64_t>(neq, 1) * sizeof(double)));
        xfer_ = std::move(t);
    }
    Transfer& t = *xfer_;
    const size_t ng = t.ranges.size();
    cudaStream_t s = stream_;
    double* h_lnz = h_sm + neq;
    double* d_lnz = d_sm + neq;
    // the pre-pass needs every original diagonal before anything is factored
    // (the zero test of sprfc1.f:465-488): gathered first, so that D and the
    // diagonals are the first uploads in the copy engine's queue
    {
        const int nt = (int)std::min<int64_t>(8, std::max<int64_t>(1, neq / 65536));
        std::vector<std::thread> pool;
        for (int k = 0; k < nt; ++k)
            pool.emplace_back([&, k]() {
                for (int64_t j = neq * k / nt; j < neq * (k + 1) / nt; ++j) t.h_diag[j] = h_lnz[t.diag_pos[j]];
            });
        for (auto& th : pool) th.join();
    }
    CK(cudaEventRecord(t.ts, s));
    // D on the compute stream (the pre-pass writes D of retained supernodes)
    CK(cudaMemcpyAsync(d_sm, h_sm, neq * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(t.d_diag, t.h_diag, neq * sizeof(double), cudaMemcpyHostToDevice, s));
    // the copy streams start after the compute stream's earlier work
    CK(cudaEventRecord(t.start, s));
    CK(cudaStreamWaitEvent(cs, t.start, 0));
    CK(cudaStreamWaitEvent(t.ups, t.start, 0));
    CopyScheduler sched;
    sched.up_recorded.assign(ng, 0);
    std::thread uploader([&]() {
        for (size_t g = 0; g < ng; ++g) {
            if (g >= 2 && cudaEventSynchronize(t.up[g - 2]) != cudaSuccess) sched.status = -4;
            for (const auto& r : t.ranges[g])
                if (cudaMemcpyAsync(d_lnz + r.first, h_lnz + r.first, r.second * sizeof(double),
                                    cudaMemcpyHostToDevice, t.ups) != cudaSuccess)
                    sched.status = -4;
            if (cudaEventRecord(t.up[g], t.ups) != cudaSuccess) sched.status = -4;
            if (g == 0) cudaEventRecord(t.tu, t.ups);
            sched.mark(sched.up_recorded, g);
        }
    });
    std::thread downloader([&]() {
        CopyScheduler::Item it;
        while (sched.pop(it)) {
            if (cudaEventSynchronize(it.ev) != cudaSuccess) sched.status = -4;
            for (const auto& r : *it.ranges)
                if (cudaMemcpyAsync(h_lnz + r.first, d_lnz + r.first, r.second * sizeof(double),
                                    cudaMemcpyDeviceToHost, cs) != cudaSuccess)
                    sched.status = -4;
            if (it.last) return;
        }
    });
    if (trace_on()) {
        size_t nu = 0;
        for (const auto& u : t.ranges) nu += u.size();
        char b[96];
        snprintf(b, sizeof b, "diagonal gathered, copy threads started (%zu ranges each way)", nu);
        trace_point(b);
    }
    StreamHooks hk;
    hk.t = &t;
    hk.cs_sched = &sched;
    hk.d_lnz = d_lnz;
    hk.sm_count = std::max(sm_count_, 1);
    hk.nlev = P_.levels.size();
    hooks_ = &hk;
    streamed_diag_ = t.d_diag;
    cudaEventRecord(t.tf0, s);
    const int rc = factor(d_sm, tol1, res, nullptr);
    hooks_ = nullptr;
    streamed_diag_ = nullptr;
    if (rc != 0) sched.stop();                  // a level that was never enqueued records no end event
    uploader.join();
    downloader.join();
    trace_point("copy threads joined");
    if (rc != 0 || sched.status != 0) {
        cudaStreamSynchronize(t.ups);
        cudaStreamSynchronize(cs);
        return rc != 0 ? rc : -4;
    }
    if (res.lierr != 0 && !t.early_nodes.empty()) {
        // an early front that failed keeps its uploaded columns, on the device
        // and on the host (its early super-panels are undone)
        std::vector<int32_t> bad(t.early_nodes.size(), 0);
        for (size_t i = 0; i < t.early_nodes.size(); ++i)
            CK(cudaMemcpy(&bad[i], d_->sn_bad + t.early_nodes[i], sizeof(int32_t), cudaMemcpyDeviceToHost));
        int64_t b = 0;
        for (size_t i = 0; i < t.early_nodes.size(); ++i) {
            const auto& r = t.early_ranges[i];
            if (bad[i]) k_copy_d<<<2 * std::max(sm_count_, 1), 256, 0, s>>>(t.d_backup + b, d_lnz + r.first, r.second);
            b += r.second;
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(t.fin, s));
        CK(cudaStreamWaitEvent(cs, t.fin, 0));
        for (size_t i = 0; i < t.early_nodes.size(); ++i)
            if (bad[i]) {
                const auto& r = t.early_ranges[i];
                CK(cudaMemcpyAsync(h_lnz + r.first, d_lnz + r.first, r.second * sizeof(double),
                                   cudaMemcpyDeviceToHost, cs));
            }
    }
    // D is final only now (and on a zero diagonal it holds the original diagonal)
    CK(cudaEventRecord(t.fin, s));
    CK(cudaEventRecord(t.tf, s));
    CK(cudaStreamWaitEvent(cs, t.fin, 0));
    CK(cudaMemcpyAsync(h_sm, d_sm, neq * sizeof(double), cudaMemcpyDeviceToHost, cs));
    CK(cudaEventRecord(t.te, cs));
    return 0;
}

int Engine::streamed_times(double* out) {
    out[0] = out[1] = out[2] = 0.0;
    if (!xfer_) return 0;
    float a = 0.f, c = 0.f;
    // from the call's first copy to the factorisation's first launch, and from
    // its end to the end of the last download
    if (cudaEventElapsedTime(&a, xfer_->ts, xfer_->tf0) != cudaSuccess ||
        cudaEventElapsedTime(&c, xfer_->tf, xfer_->te) != cudaSuccess)
        return -4;
    out[0] = a;
    out[1] = timing.factor_ms;
    out[2] = c;
    return 0;
}

int Engine::factor_chol(double* d_sm, double tol1, FactorResult& res, const Singular* fc4) {
    chol_ = true;
    const int rc = factor(d_sm, tol1, res, fc4);
    chol_ = false;
    return rc;
}

int Engine::chol_convert(double* d_sm, bool to_chol) {
    Dev& D = *d_;
    PV pv = make_view(D, P_, d_sm, 0.0);
    const int grid = (int)std::min<int64_t>(P_.nsuper, 8 * (int64_t)std::max(sm_count_, 1));
    if (to_chol)
        k_chol_convert<true><<<grid, 256, 0, stream_>>>(pv, P_.nsuper);
    else
        k_chol_convert<false><<<grid, 256, 0, stream_>>>(pv, P_.nsuper);
    CK(cudaGetLastError());
    linv_valid_ = false;
    return 0;
}

int Engine::scale_sqrt_d(const double* d_sm, double* d_b, int64_t ldb, int64_t nrhs, bool divide) {
    const int64_t n = P_.neq * nrhs;
    if (n <= 0) return 0;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 8 * (int64_t)std::max(sm_count_, 1));
    k_scale_sqrt_d<<<grid, 256, 0, stream_>>>(d_sm, d_b, ldb, P_.neq, nrhs, divide ? 1 : 0);
    CK(cudaGetLastError());
    return 0;
}

int Engine::sn_stats(int32_t* neg, int32_t* fail) {
    Dev& D = *d_;
    CK(cudaMemcpy(neg, D.sn_neg, P_.nsuper * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(fail, D.sn_fail, P_.nsuper * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return 0;
}

void Engine::ensure_vectors(int64_t nrhs) {
    Dev& D = *d_;
    if (D.vbuf_rhs < nrhs) {
        if (D.vbuf) cudaFree(D.vbuf);
        if (D.vbuf2) cudaFree(D.vbuf2);
        D.vbuf = D.vbuf2 = nullptr;
        const size_t bytes = std::max<int64_t>(P_.rbase.back(), 1) * nrhs * sizeof(double);
        if (cudaMalloc((void**)&D.vbuf, bytes) != cudaSuccess || cudaMalloc((void**)&D.vbuf2, bytes) != cudaSuccess)
            return;
        D.vbuf_rhs = nrhs;
    }
}

void Engine::enqueue_solve(const PV& pv, cudaStream_t s, double* d_b, int64_t ldb, int64_t nrhs, int which,
                           int64_t& nl) {
    Dev& D = *d_;
    auto mark = [&](int phase) {
        if (profile_) marks_.emplace_back(9 + phase, record_event(s));
    };
    const int64_t chunk = std::min<int64_t>(nrhs, kMaxRHS);
    for (int64_t r0 = 0; r0 < nrhs; r0 += chunk) {
        const int nr = (int)std::min<int64_t>(chunk, nrhs - r0);
        double* b = d_b + r0 * ldb;
        const Job* jobs = D.jobs;
        auto blocks = [](int64_t threads) { return (int)((threads + 255) / 256); };
        const size_t tri_bytes = sizeof(int32_t) * (size_t)(P_.tri_flags + 2 * (int64_t)P_.levels.size());
        if (which & 1) {
            if (tri_solve_) cudaMemsetAsync(D.tri_sync, 0, tri_bytes, s);
            // split run: the other ranks' subtree roots' update vectors come in
            // before their parent's level, this rank's go out after their level
            ExchangeHooks vx;
            vx.P = &P_;
            vx.out = &vout_;
            vx.in = &vin_;
            vx.copy = [this, nr](int32_t js, double* buf, bool o, cudaStream_t st) { vec_copy(js, buf, o, nr, st); };
            const bool vexch = !vout_.empty() || !vin_.empty();
            for (size_t L = 0; L < P_.levels.size(); ++L) {
                const LevelPlan& lp = P_.levels[L];
                if (vexch) vx.before(L, s);
                struct AfterLevel {
                    const ExchangeHooks* h;
                    size_t L;
                    cudaStream_t s;
                    ~AfterLevel() {
                        if (h) h->after(L, s);
                    }
                } after_level{vexch ? &vx : nullptr, L, s};
                if (!lp.small_nodes.empty()) {
                    mark(0);
                    for (const LevelPlan::SmallClass& c : lp.small_classes) {
                        k_forward<<<c.count, small_threads(c.maxF), small_solve_smem(c.maxF, nr), s>>>(
                            D.level_nodes + D.small_begin[L] + c.begin, pv, D.vbuf, b, ldb, nr);
                        ++nl;
                    }
                }
                if (lp.large_nodes.empty()) continue;
                const Launch& ga = lp.assemble;
                mark(1);
                k_fwd_gather<<<blocks(ga.ntasks), 256, 0, s>>>(jobs + ga.job_begin, ga.job_count, TMAP(ga), ga.ntasks, pv,
                                                               D.vbuf, b, ldb, nr);
                ++nl;
                mark(2);
                if (tri_solve_ && lp.tri_count > 0) {
                    const int nt = (int)lp.tri_count;
                    const int grid = std::min(nt, 4 * std::max(sm_count_, 1));
                    int32_t* ctr = D.tri_sync + P_.tri_flags + 2 * L;
                    if (nr <= 4)
                        k_fwd_tri<4><<<grid, 256, 0, s>>>(D.tri_tasks + 2 * lp.tri_begin, nt, D.tri_sync, ctr, pv,
                                                          D.vbuf, D.vbuf2, nr);
                    else
                        k_fwd_tri<kMaxRHS><<<grid, 256, 0, s>>>(D.tri_tasks + 2 * lp.tri_begin, nt, D.tri_sync, ctr, pv,
                                                                D.vbuf, D.vbuf2, nr);
                    ++nl;
                } else {
                    for (size_t sb = 0; sb < lp.fs_upd.size(); ++sb) {
                        const Launch& ml = lp.blk_mv[sb];
                        k_fwd_blk_mv<<<(int)ml.ntasks, 256, kMvSmem, s>>>(jobs + ml.job_begin, ml.job_count, TMAP(ml), pv,
                                                                     D.vbuf, D.vbuf2, nr);
                        ++nl;
                        const Launch& fl = lp.fs_upd[sb];
                        if (fl.ntasks > 0) {
                            k_fwd_blk_upd2<<<(int)fl.ntasks, 256, kUpdSmem, s>>>(jobs + fl.job_begin, fl.job_count,
                                                                           TMAP(fl), pv, D.vbuf, D.vbuf2, nr);
                            ++nl;
                        }
                    }
                }
                const Launch& rl = lp.rect;
                if (rl.ntasks > 0) {
                    mark(3);
                    if (nr <= 4)
                        k_fwd_rect_part<4><<<(int)rl.ntasks, 256, 0, s>>>(jobs + rl.job_begin, rl.job_count, TMAP(rl),
                                                                          pv, D.vbuf2, D.pbuf, nr);
                    else
                        k_fwd_rect_part<kMaxRHS><<<(int)rl.ntasks, 256, 0, s>>>(jobs + rl.job_begin, rl.job_count,
                                                                                TMAP(rl), pv, D.vbuf2, D.pbuf, nr);
                    const Launch& rr = lp.rect_rows;
                    k_fwd_rect_sum<<<blocks(rr.ntasks), 256, 0, s>>>(jobs + rr.job_begin, rr.job_count, TMAP(rr),
                                                                      rr.ntasks, pv, D.vbuf, D.pbuf, nr);
                    nl += 2;
                }
                const Launch& wb = lp.writeback;
                mark(4);
                k_fwd_finish<<<blocks(wb.ntasks), 256, 0, s>>>(jobs + wb.job_begin, wb.job_count, TMAP(wb), wb.ntasks, pv,
                                                               D.vbuf2, D.vbuf, b, ldb, nr);
                ++nl;
            }
        }
        if (which & 2) {
            if (tri_solve_) cudaMemsetAsync(D.tri_sync, 0, tri_bytes, s);
            for (size_t L = P_.levels.size(); L-- > 0;) {
                const LevelPlan& lp = P_.levels[L];
                if (!lp.small_nodes.empty()) {
                    mark(5);
                    for (const LevelPlan::SmallClass& c : lp.small_classes) {
                        k_backward<<<c.count, small_threads(c.maxF), small_solve_smem(c.maxF, nr), s>>>(
                            D.level_nodes + D.small_begin[L] + c.begin, pv, D.vbuf, b, ldb, nr);
                        ++nl;
                    }
                }
                if (lp.large_nodes.empty()) continue;
                const Launch& ga = lp.assemble;
                mark(6);
                k_bwd_gather<<<blocks(ga.ntasks), 256, 0, s>>>(jobs + ga.job_begin, ga.job_count, TMAP(ga), ga.ntasks, pv,
                                                               D.vbuf, b, ldb, nr);
                ++nl;
                const Launch& wb = lp.writeback;
                const Launch& rl = lp.rect;
                if (rl.ntasks > 0) {
                    mark(7);
                    if (nr <= 4)
                        k_bwd_rect_part<4><<<(int)rl.ntasks, 256, 0, s>>>(jobs + rl.job_begin, rl.job_count, TMAP(rl),
                                                                          pv, D.vbuf, D.pbuf, nr);
                    else
                        k_bwd_rect_part<kMaxRHS><<<(int)rl.ntasks, 256, 0, s>>>(jobs + rl.job_begin, rl.job_count,
                                                                                TMAP(rl), pv, D.vbuf, D.pbuf, nr);
                    ++nl;
                    k_bwd_rect_sum<<<blocks(wb.ntasks * kSumLanes), 256, 0, s>>>(jobs + wb.job_begin, wb.job_count, TMAP(wb), wb.ntasks, pv,
                                                                      D.vbuf, D.pbuf, nr);
                    ++nl;
                }
                mark(8);
                if (tri_solve_ && lp.tri_count > 0) {
                    const int nt = (int)lp.tri_count;
                    const int grid = std::min(nt, 4 * std::max(sm_count_, 1));
                    int32_t* ctr = D.tri_sync + P_.tri_flags + 2 * L;
                    if (nr <= 4)
                        k_bwd_tri<4><<<grid, 256, 0, s>>>(D.tri_tasks + 2 * lp.tri_begin, nt, D.tri_sync, ctr, pv,
                                                          D.vbuf, D.vbuf2, nr);
                    else
                        k_bwd_tri<kMaxRHS><<<grid, 256, 0, s>>>(D.tri_tasks + 2 * lp.tri_begin, nt, D.tri_sync, ctr, pv,
                                                                D.vbuf, D.vbuf2, nr);
                    ++nl;
                } else {
                    for (size_t sb = lp.bs_upd.size(); sb-- > 0;) {
                        const Launch& ml = lp.blk_mv[sb];
                        k_bwd_blk_mv<<<(int)ml.ntasks, 256, kBwdSmem, s>>>(jobs + ml.job_begin, ml.job_count, TMAP(ml), pv,
                                                                     D.vbuf, D.vbuf2, nr);
                        ++nl;
                        const Launch& bl = lp.bs_upd[sb];
                        if (bl.ntasks > 0) {
                            k_bwd_blk_upd<<<(int)bl.ntasks, 256, kBwdSmem, s>>>(jobs + bl.job_begin, bl.job_count,
                                                                         TMAP(bl), pv, D.vbuf, D.vbuf2, nr);
                            ++nl;
                        }
                    }
                }
                mark(10);
                k_bwd_finish<<<blocks(wb.ntasks), 256, 0, s>>>(jobs + wb.job_begin, wb.job_count, TMAP(wb), wb.ntasks, pv,
                                                               D.vbuf2, b, ldb, nr);
                ++nl;
            }
        }
    }
}

int Engine::solve(const double* d_sm, double* d_b, int64_t ldb, int64_t nrhs, int which) {
    NvtxRange range("spr_b200 solve");
    Dev& D = *d_;
    cudaStream_t s = stream_;
    PV pv = make_view(D, P_, const_cast<double*>(d_sm), 0.0);
    pv.wait_ns = wait_ns_;
    pv.tc_drop = tc_drop_ ? 1 : 0;
    const int64_t chunk = std::min<int64_t>(nrhs, kMaxRHS);
    ensure_vectors(chunk);
    if (!D.vbuf || !D.vbuf2) return -4;
    CK(cudaEventRecord(D.ev0, s));
    int64_t nl = 0;
    CK(cudaMemsetAsync(&D.st->solve_timeout, 0, sizeof(int), s));
    if (!linv_valid_) {
        for (const LevelPlan& lp : P_.levels)
            for (const Launch& pl : lp.panel)
                if (pl.job_count > 0) {
                    k_linv<<<(int)pl.job_count, 64, 0, s>>>(D.jobs + pl.job_begin, pv);
                    ++nl;
                }
        if (!tri_solve_ && P_.inv_blocks.job_count > 0) {
            PV pvi = pv;
            pvi.sn_bad = nullptr;
            k_inv_block<<<(int)P_.inv_blocks.job_count, 256, kInvSmem, s>>>(D.jobs + P_.inv_blocks.job_begin, pvi);
            ++nl;
        }
        linv_valid_ = true;
    }
    if (use_graphs_ && !profile_ && s != nullptr && !tc_drop_ && wait_ns_ == 2000000000ull && !split_) {
        const GraphKey key{(const void*)d_sm, (const void*)d_b, (double)ldb, nrhs, which, (int64_t)(uintptr_t)D.vbuf};
        cudaGraphExec_t exec = find_graph(key);
        if (!exec) {
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            enqueue_solve(pv, s, d_b, ldb, nrhs, which, nl);
            cudaGraph_t g = nullptr;
            CK(cudaStreamEndCapture(s, &g));
            CK(cudaGraphInstantiate(&exec, g, 0));
            cudaGraphDestroy(g);
            store_graph(key, exec, nl);
        } else {
            nl += graph_launches(key);
        }
        CK(cudaGraphLaunch(exec, s));
    } else {
        enqueue_solve(pv, s, d_b, ldb, nrhs, which, nl);
    }
    CK(cudaEventRecord(D.ev1, s));
    CK(cudaGetLastError());
    k_mailbox<<<1, 32, 0, s>>>(reinterpret_cast<const unsigned long long*>(D.st), (int)(sizeof(Stats) / 8),
                               D.mbox_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    Stats hs;
    std::memcpy(&hs, D.mbox, sizeof(Stats));
    const int tri_timeout = hs.solve_timeout;
    CK(cudaEventElapsedTime(&timing.solve_ms, D.ev0, D.ev1));
    timing.solve_launches = nl;
    if (tri_timeout) {
        fprintf(stderr, "spr_b200: a triangle task of the solve gave up waiting for a block\n");
        return -4;
    }
    if (profile_) {
        for (int k = 9; k < 20; ++k) timing.phase_ms[k] = 0.f;
        for (size_t k = 0; k < marks_.size(); ++k) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, marks_[k].second, k + 1 < marks_.size() ? marks_[k + 1].second : D.ev1);
            timing.phase_ms[marks_[k].first] += ms;
            cudaEventDestroy(marks_[k].second);
        }
        marks_.clear();
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Blocked LDL' of one dense front with caller-provided scratch (no device
// allocation).  Same kernels and step order as the large-front path of
// Engine::factor for a front with S = F = n.
// ---------------------------------------------------------------------------
size_t dense_scratch_bytes(int64_t n) {
    const int64_t nblk = (n + kNB - 1) / kNB;
    const int64_t njobs = 3 * nblk;
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) / 256 * 256; };
    add(sizeof(Stats));
    add(sizeof(double) * n);                       // original diagonal
    add(sizeof(double) * nblk * kNB * kNB);        // inverses of the diagonal blocks
    add(sizeof(Job) * njobs);
    add(sizeof(int32_t) * 16);                     // node arrays (one node)
    add(sizeof(int64_t) * 8);
    add(sizeof(double) * 4);
    return b;
}

int dense_factor_setup() {
    // k_trsm and the small-tile update use more than the default 48 KB of
    // dynamic shared memory; the opt-in is per function and per device.
    CK(cudaFuncSetAttribute(k_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
    CK(cudaFuncSetAttribute(K_GEMM_SMALL, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GemmSmall::smem));
    return 0;
}

int dense_factor_with_scratch(double* a, int64_t n, int64_t lda, double tol1, double* d, void* scratch,
                              size_t scratch_bytes, cudaStream_t s, double* out) {
    if (n <= 0 || lda < n || (lda % 4) != 0 || ((uintptr_t)a % 32) != 0) return -2;
    if (dense_scratch_bytes(n) > scratch_bytes) return -3;
    const int64_t nblk = (n + kNB - 1) / kNB;
    char* p = static_cast<char*>(scratch);
    auto take = [&](size_t bytes) {
        char* q = p;
        p += (bytes + 255) / 256 * 256;
        return q;
    };
    Stats* st = reinterpret_cast<Stats*>(take(sizeof(Stats)));
    double* adiag = reinterpret_cast<double*>(take(sizeof(double) * n));
    double* linv = reinterpret_cast<double*>(take(sizeof(double) * nblk * kNB * kNB));
    Job* jobs = reinterpret_cast<Job*>(take(sizeof(Job) * 3 * nblk));
    int32_t* i32 = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 16));
    int64_t* i64 = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * 8));
    double* f64 = reinterpret_cast<double*>(take(sizeof(double) * 4));
    // node arrays: fst, S, F, buf_ld, sn_neg, sn_fail, sn_bad (int32); buf_off, linv_off (int64)
    int32_t hi32[16] = {0, (int32_t)n, (int32_t)n, (int32_t)lda, 0, -1, 0};
    int64_t hi64[8] = {0, 0};
    Stats init{};
    init.first_zero = 0x7fffffff;
    // jobs of every step (host side, fixed-size per block, no allocation)
    struct StepJobs {
        int64_t panel_begin, panel_tasks, upd_begin, upd_jobs, upd_tasks;
    };
    constexpr int kMaxBlocks = 1024;
    if (nblk > kMaxBlocks) return -3;
    static thread_local Job hjobs[3 * kMaxBlocks];
    static thread_local StepJobs steps[kMaxBlocks];
    int64_t nj = 0;
    auto tiles = [](int64_t c0, int64_t c_end, int64_t r_end) -> int64_t {
        const int64_t nct = (c_end - c0 + kTile - 1) / kTile, nr = (r_end - c0 + kTile - 1) / kTile;
        return nct * nr - nct * (nct - 1) / 2;
    };
    for (int64_t stp = 0; stp < nblk; ++stp) {
        const int32_t k0 = (int32_t)(stp * kNB);
        const int32_t nb = (int32_t)std::min<int64_t>(kNB, n - k0);
        const int32_t c0 = k0 + nb;
        StepJobs& sj = steps[stp];
        sj.panel_begin = nj;
        sj.panel_tasks = (n - c0 + kTRSMRows - 1) / kTRSMRows;
        hjobs[nj++] = Job{0, c0, c0, (int32_t)n, k0, c0, 0};
        sj.upd_begin = nj;
        sj.upd_jobs = 0;
        sj.upd_tasks = 0;
        const int32_t sp0 = (k0 / kSuperPanel) * kSuperPanel;
        const int32_t sp1 = (int32_t)std::min<int64_t>(sp0 + kSuperPanel, n);
        if (c0 < sp1) {
            hjobs[nj] = Job{0, c0, sp1, (int32_t)n, k0, c0, sj.upd_tasks};
            sj.upd_tasks += tiles(c0, sp1, n);
            ++nj;
            ++sj.upd_jobs;
        }
        if (c0 == sp1 && sp1 < n) {
            hjobs[nj] = Job{0, sp1, (int32_t)n, (int32_t)n, sp0, sp1, sj.upd_tasks};
            sj.upd_tasks += tiles(sp1, n, n);
            ++nj;
            ++sj.upd_jobs;
        }
    }
    CK(cudaMemcpyAsync(jobs, hjobs, sizeof(Job) * nj, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(i32, hi32, sizeof(hi32), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(i64, hi64, sizeof(hi64), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st, &init, sizeof(Stats), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(f64, 0, sizeof(double) * 4, s));
    // the pivot test compares with the diagonal before factorisation (sprfc1.f:1272-1279)
    CK(cudaMemcpy2DAsync(adiag, sizeof(double), a, (lda + 1) * sizeof(double), sizeof(double), n,
                         cudaMemcpyDeviceToDevice, s));
    PV pv{};
    pv.fst = i32 + 0;
    pv.S = i32 + 1;
    pv.F = i32 + 2;
    pv.buf_ld = i32 + 3;
    pv.sn_neg = i32 + 4;
    pv.sn_fail = i32 + 5;
    pv.sn_bad = i32 + 6;
    pv.buf_off = i64 + 0;
    pv.linv_off = i64 + 1;
    pv.arena = a;
    pv.dvec = d;
    pv.lnz = nullptr;
    pv.adiag = adiag;
    pv.linv = linv;
    pv.sn_faild = f64 + 0;
    pv.sn_faila = f64 + 1;
    pv.st = st;
    pv.tol1 = tol1;
    for (int64_t stp = 0; stp < nblk; ++stp) {
        const StepJobs& sj = steps[stp];
        k_diag<kPivotLDL><<<1, 256, 0, s>>>(jobs + sj.panel_begin, pv);
        if (sj.panel_tasks > 0) k_trsm<<<(int)sj.panel_tasks, 128, kTrsmSmem, s>>>(jobs + sj.panel_begin, 1, nullptr, pv);
        if (sj.upd_tasks > 0)
            K_GEMM_SMALL<<<(int)sj.upd_tasks, GemmSmall::NT, GemmSmall::smem, s>>>(jobs + sj.upd_begin, sj.upd_jobs, nullptr,
                                                                                 pv);
    }
    CK(cudaGetLastError());
    Stats hs;
    int32_t hfail = -1;
    double hf[2] = {0.0, 0.0};
    CK(cudaMemcpyAsync(&hs, st, sizeof(Stats), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&hfail, i32 + 5, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hf, f64, sizeof(hf), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // out[0]=NUMNEG out[1]=first failing column (1-based, 0 if none) out[2]=failing pivot out[3]=its a_jj
    // out[4]=max(a_jj/d_j)
    out[0] = (double)hs.numneg;
    out[1] = hs.pivot_fail ? (double)(hfail + 1) : 0.0;
    out[2] = hf[0];
    out[3] = hf[1];
    out[4] = hs.tol2;
    return 0;
}

// ---------------------------------------------------------------------------
// Autotuner of the mixed-mode factorisation: which Schur updates go to the
// tensor cores (launches of at least tc_min_flops; the rest stay on the FP64
// kernel) and how many SMs the side-stream tensor-core launches may take.
// Every candidate factors a copy of the assembled SM twice (the second,
// graph-replayed pass is timed); the fastest is kept.  out[0] = chosen
// tc_min_flops, out[1] = chosen quarters of the SMs, out[2] = its factor ms,
// out[3] = factor ms of the default choice, out[4] = candidates tried.
// ---------------------------------------------------------------------------
int Engine::autotune(const double* d_sm_assembled, double* out) {
    const int64_t n = P_.neq + P_.nzerol;
    double* work = nullptr;
    CK(cudaMalloc((void**)&work, n * sizeof(double)));
    const int mode0 = mixed_;
    const double t0 = tc_min_flops_;
    const int q0 = far_cap_q_;
    mixed_ = 1;
    const double mins[] = {0.0, 1.0e9, 1.0e10, 1.0e11, 1.0e300};
    const int caps[] = {2, 3, 4};
    double best = 1e300, best_min = 0.0, def_ms = 0.0;
    int best_cap = 3, tried = 0, rc = 0;
    for (double m : mins)
        for (int q : caps) {
            if (m >= 1.0e300 && q != 3) continue;              // no tensor-core launches: the cap is moot
            tc_min_flops_ = m;
            far_cap_q_ = q;
            float ms = 0.f;
            for (int rep = 0; rep < 2 && rc == 0; ++rep) {
                if (cudaMemcpyAsync(work, d_sm_assembled, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_) !=
                    cudaSuccess) {
                    rc = -4;
                    break;
                }
                FactorResult r;
                rc = factor(work, 1.0e-12, r);
                ms = timing.factor_ms;
            }
            if (rc != 0) break;
            ++tried;
            if (m == 0.0 && q == 3) def_ms = ms;
            if (ms < best) {
                best = ms;
                best_min = m;
                best_cap = q;
            }
        }
    cudaFree(work);
    mixed_ = mode0;
    if (rc != 0) {
        tc_min_flops_ = t0;
        far_cap_q_ = q0;
        return rc;
    }
    tc_min_flops_ = best_min;
    far_cap_q_ = best_cap;
    out[0] = best_min;
    out[1] = best_cap;
    out[2] = best;
    out[3] = def_ms;
    out[4] = tried;
    return 0;
}

// Tile shape of the small Schur updates (those with fewer than 4 x 64 rows):
// each candidate (64 x 64 tiles, 32 x 32 tiles) factors a copy of the
// assembled SM twice and the faster one is kept.  out[0] = the tile chosen,
// out[1] / out[2] = factor ms with 64 / 32.
int Engine::autotune_tiles(const double* d_sm_assembled, double* out) {
    const int64_t n = P_.neq + P_.nzerol;
    double* work = nullptr;
    CK(cudaMalloc((void**)&work, n * sizeof(double)));
    const int t0 = small_tile_;
    const int cand[2] = {kTile, kTileTiny};
    double ms[2] = {0.0, 0.0};
    int rc = 0;
    for (int c = 0; c < 2 && rc == 0; ++c) {
        small_tile_ = cand[c];
        float best = 1e30f;
        for (int rep = 0; rep < 2 && rc == 0; ++rep) {
            if (cudaMemcpyAsync(work, d_sm_assembled, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_) !=
                cudaSuccess) {
                rc = -4;
                break;
            }
            FactorResult r;
            rc = factor(work, 1.0e-12, r);
            best = std::min(best, timing.factor_ms);
        }
        ms[c] = best;
    }
    cudaFree(work);
    if (rc != 0) {
        small_tile_ = t0;
        return rc;
    }
    small_tile_ = ms[1] < ms[0] ? kTileTiny : kTile;
    out[0] = small_tile_;
    out[1] = ms[0];
    out[2] = ms[1];
    return 0;
}

// ---------------------------------------------------------------------------
// Iterative refinement against the FP64 matrix
// ---------------------------------------------------------------------------
int Engine::build_residual(const double* d_sm_assembled) {
    Dev& D = *d_;
    cudaStream_t s = stream_;
    PV pv = make_view(D, P_, const_cast<double*>(d_sm_assembled), 0.0);
    const int64_t neq = P_.neq;
    int* cnt = nullptr;
    CK(cudaMalloc((void**)&cnt, (neq + 1) * sizeof(int)));
    CK(cudaMemsetAsync(cnt, 0, (neq + 1) * sizeof(int), s));
    const int grid = (int)std::min<int64_t>((P_.nsuper * 32 + 255) / 256, 4736);
    k_csr_count<<<grid, 256, 0, s>>>(pv, P_.nsuper, cnt);
    std::vector<int> hc(neq);
    CK(cudaMemcpyAsync(hc.data(), cnt, neq * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<int64_t> rp(neq + 1, 0);
    for (int64_t i = 0; i < neq; ++i) rp[i + 1] = rp[i] + hc[i];
    const int64_t nnz = rp[neq];
    if (csr_.rowptr) cudaFree(csr_.rowptr);
    if (csr_.ci) cudaFree(csr_.ci);
    if (csr_.cv) cudaFree(csr_.cv);
    if (csr_.rowabs) cudaFree(csr_.rowabs);
    CK(cudaMalloc((void**)&csr_.rowptr, (neq + 1) * sizeof(int64_t)));
    CK(cudaMalloc((void**)&csr_.ci, std::max<int64_t>(nnz, 1) * sizeof(int32_t)));
    CK(cudaMalloc((void**)&csr_.cv, std::max<int64_t>(nnz, 1) * sizeof(double)));
    CK(cudaMalloc((void**)&csr_.rowabs, neq * sizeof(double)));
    CK(cudaMemcpyAsync(csr_.rowptr, rp.data(), (neq + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    std::vector<int> fp(rp.begin(), rp.end() - 1);
    CK(cudaMemcpyAsync(cnt, fp.data(), neq * sizeof(int), cudaMemcpyHostToDevice, s));
    k_csr_fill<<<grid, 256, 0, s>>>(pv, P_.nsuper, cnt, csr_.ci, csr_.cv);
    k_csr_sort<<<(int)((neq + 255) / 256), 256, 0, s>>>(csr_.rowptr, neq, csr_.ci, csr_.cv, csr_.rowabs);
    std::vector<double> ra(neq);
    CK(cudaMemcpyAsync(ra.data(), csr_.rowabs, neq * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    cudaFree(cnt);
    csr_.norm_inf = 0.0;
    for (double v : ra) csr_.norm_inf = std::max(csr_.norm_inf, v);
    csr_.nnz = nnz;
    return 0;
}

int Engine::residual(const double* d_b, const double* d_x, double* d_r, int64_t ld, int64_t nrhs, double* berr) {
    if (!csr_.rowptr) return -2;
    cudaStream_t s = stream_;
    if (nbuf_cap_ < 3 * nrhs) {
        if (nbuf_) cudaFree(nbuf_);
        nbuf_ = nullptr;
        nbuf_cap_ = 0;
        CK(cudaMalloc((void**)&nbuf_, 3 * nrhs * sizeof(double)));
        nbuf_cap_ = 3 * nrhs;
    }
    double* norms = nbuf_;
    CK(cudaMemsetAsync(norms, 0, 3 * nrhs * sizeof(double), s));
    const int64_t neq = P_.neq;
    constexpr int kW = kResThreads / 32;
    const int grid =
        (int)std::max<int64_t>(1, std::min<int64_t>((neq + kW - 1) / kW, 8 * (int64_t)std::max(sm_count_, 1)));
    for (int64_t q0 = 0; q0 < nrhs; q0 += kMaxRHS) {          // kMaxRHS right-hand sides per pass
        const int nq = (int)std::min<int64_t>(kMaxRHS, nrhs - q0);
        const int64_t o = q0 * ld;
        if (nq <= 4)
            k_residual<4><<<grid, kResThreads, 0, s>>>(csr_.rowptr, csr_.ci, csr_.cv, neq, d_b + o, d_x + o, d_r + o,
                                                       ld, nq, norms + 3 * q0);
        else
            k_residual<kMaxRHS><<<grid, kResThreads, 0, s>>>(csr_.rowptr, csr_.ci, csr_.cv, neq, d_b + o, d_x + o,
                                                             d_r + o, ld, nq, norms + 3 * q0);
    }
    CK(cudaGetLastError());
    std::vector<double> h(3 * nrhs);
    CK(cudaMemcpyAsync(h.data(), norms, 3 * nrhs * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double worst = 0.0;
    for (int64_t q = 0; q < nrhs; ++q) {
        const double den = csr_.norm_inf * h[3 * q + 1] + h[3 * q + 2];
        worst = std::max(worst, den > 0.0 ? h[3 * q] / den : 0.0);
    }
    *berr = worst;
    return 0;
}

int Engine::refine(const double* d_sm, const double* d_b, double* d_x, int64_t ld, int64_t nrhs, double tol,
                   int maxit, double* out) {
    Dev& D = *d_;
    cudaStream_t s = stream_;
    const int64_t n = ld * nrhs;
    if (rbuf_cap_ < n) {
        if (rbuf_) cudaFree(rbuf_);
        rbuf_ = nullptr;
        rbuf_cap_ = 0;
        CK(cudaMalloc((void**)&rbuf_, n * sizeof(double)));
        rbuf_cap_ = n;
    }
    (void)D;
    CK(cudaMemcpyAsync(d_x, d_b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (solve(d_sm, d_x, ld, nrhs, 3) != 0) return -4;
    float solve_ms = timing.solve_ms;
    double berr = 0.0;
    int it = 0;
    for (;;) {
        if (residual(d_b, d_x, rbuf_, ld, nrhs, &berr) != 0) return -4;
        if (berr <= tol || it >= maxit) break;
        if (solve(d_sm, rbuf_, ld, nrhs, 3) != 0) return -4;
        solve_ms += timing.solve_ms;
        k_axpy<<<(int)((n + 255) / 256), 256, 0, s>>>(d_x, rbuf_, n);
        ++it;
    }
    CK(cudaStreamSynchronize(s));
    out[0] = it;
    out[1] = berr;
    out[2] = solve_ms;
    return 0;
}

// Self-test of recip_nr: out[2i] = recip_nr(x[i]), out[2i+1] = 1.0 / x[i]
// (host arrays, n values).
int recip_check(const double* h_x, int64_t n, double* h_out) {
    double *dx = nullptr, *dout = nullptr;
    CK(cudaMalloc((void**)&dx, std::max<int64_t>(n, 1) * sizeof(double)));
    CK(cudaMalloc((void**)&dout, std::max<int64_t>(2 * n, 1) * sizeof(double)));
    CK(cudaMemcpy(dx, h_x, n * sizeof(double), cudaMemcpyHostToDevice));
    if (n > 0) k_recip_check<<<(int)((n + 255) / 256), 256>>>(dx, n, dout);
    CK(cudaGetLastError());
    CK(cudaMemcpy(h_out, dout, 2 * n * sizeof(double), cudaMemcpyDeviceToHost));
    cudaFree(dx);
    cudaFree(dout);
    return 0;
}

}  // namespace sprb
