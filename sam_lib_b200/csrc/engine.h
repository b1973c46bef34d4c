// GPU numeric phase of SPR: device state and entry points used by the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "plan.h"

namespace sprb {

// SPR_B200_TRACE=1: wall-clock milestones on stderr (ms since trace_reset),
// for locating host time in the entry points.
bool trace_on();
// Self-test of the pivot reciprocal: out[2i] = it, out[2i+1] = 1.0 / x[i].
int recip_check(const double* h_x, int64_t n, double* h_out);
void trace_reset();
void trace_point(const char* what);


// Outcome of a factorisation, in the reference's terms (SPRF11/SPRFC1,
// src/SPR/sprfc1.f:240-283 and :690-708).
struct FactorResult {
    int64_t lierr = 0;       // 0, -30 (pivot below threshold), -35 (zero diagonal) or,
                             // SPRFC3 semantics, -31 (pivots replaced)
    int64_t numneg = 0;      // MSPAR(26)
    int64_t supeqt = 0;      // MSPAR(27) on error; SPRFC3: the number of replaced pivots
    double tol2 = 0.0;       // TOL(2)
    double tol3 = 0.0;       // TOL(3)
};

struct Timing {              // CUDA-event times of the last calls (ms)
    float factor_ms = 0.f, solve_ms = 0.f;
    float gemm_ms = 0.f;     // Schur-update kernels only (sum over launches)
    float tc_ms = 0.f;       // of those, the split + tensor-core launch pairs
    double tc_flops = 0.0;   // algorithmic flops of the tensor-core launches enqueued by the last factorisation
    int64_t gemm_launches = 0, launches = 0, solve_launches = 0;
    // profile mode: factor time by phase (CUDA events between launch groups):
    // 0 pre-pass, 1 small fronts, 2 extend-add, 3 diagonal blocks, 4 panel
    // TRSM, 5 in-panel/trailing updates, 6 K = S update, 7 write-back, 8 end;
    // solve: 9 small-front forward, 10 forward gather, 11 forward blocks
    // (block products and in-block updates), 12 forward rectangles, 13 forward finish, 14 small-front
    // back, 15 back gather, 16 back rectangles, 17 back blocks (block
    // products and in-block updates), 18 unused, 19 back finish
    float phase_ms[20] = {};
};

// Callbacks around each elimination-tree level of a factorisation's launch
// sequence (streamed factorisation: waits for a level's upload before it,
// downloads of its finished columns after it).
struct LevelHooks {
    virtual ~LevelHooks() = default;
    virtual void before(size_t level, cudaStream_t s) const = 0;
    virtual void after(size_t level, cudaStream_t s) const = 0;
    // A level whose super-panels are written to LNZ as soon as they are final
    // (on a stream of their own); columns_written follows each such write.
    virtual bool early_columns(size_t level) const { return false; }
    virtual void columns_written(size_t level, size_t step, cudaStream_t ws) const {}
};

class Engine {
public:
    Engine();
    ~Engine();
    // Builds the plan and uploads the symbolic structure.  Returns 0 or IERR-style code.
    int open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa);
    const Plan& plan() const { return P_; }
    void set_stream(cudaStream_t s) { stream_ = s; }
    cudaStream_t stream() const { return stream_; }
    // Device-resident factorisation of sm = [D(NEQ) | LNZ(NZEROL)] (device pointer).
    int factor(double* d_sm, double tol1, FactorResult& res) { return factor(d_sm, tol1, res, nullptr); }
    // SPRFC3 semantics (src/SPR/sprfc3.f:372-806): zero diagonals become 1 and
    // pivots at or below TOL(1)|a_jj| are replaced by
    // sign(TOL(1) max(1, |TOL(4) a_jj|), d); the factorisation always completes
    // and records both in d_dcor (device, DCOR(2,NEQ) column-major).
    struct Singular {
        double tol4;
        double* d_dcor;
    };
    int factor(double* d_sm, double tol1, FactorResult& res, const Singular* fc3);
    // SPRFC2 semantics (src/SPR/sprfc2.f:276-725): the pivot test is SPRF27's
    // d <= TOL(1)|a_jj| (a non-positive pivot stops) and TOL(3) is
    // trace / min(sqrt d)^2.  With fc4, SPRFC4 semantics (sprfc4.f:265-725):
    // zero diagonals become 1, a pivot below -TOL(1)|a_jj| stops, one up to
    // TOL(1)|a_jj| is replaced by TOL(1) max(1, |TOL(4) a_jj|), both recorded in
    // DCOR; LIERR -33 with SUPEQT = the number replaced.  The device SM is left in L D L' form; chol_convert
    // turns it into the C C' form (C = L D^1/2, sqrt d in D) and back.
    int factor_chol(double* d_sm, double tol1, FactorResult& res, const Singular* fc4 = nullptr);
    // SPRFC1 semantics with the host copies overlapped: h_sm (pinned host
    // memory, NEQ + NZEROL doubles) is uploaded level by level on the copy
    // stream cs while the lower levels factor, and each level's finished
    // columns go back into h_sm while the higher levels factor.  On return the
    // factorisation is complete on the device (res as factor()); the last
    // downloads may still run on cs: synchronise cs before reading h_sm.
    int factor_streamed(double* h_sm, double* d_sm, double tol1, FactorResult& res, cudaStream_t cs);
    // After the copy stream of the last streamed factorisation has finished:
    // out[0] = ms from its start until the lowest level group was up (the
    // upload not overlapped), out[1] = factorisation ms, out[2] = ms from the
    // end of the factorisation to the end of the last download.
    int streamed_times(double* out);
    int chol_convert(double* d_sm, bool to_chol);
    // b (device, ldb x nrhs, the first NEQ rows) times sqrt(d), or divided by
    // it, for every equation with d > 0 (d = the D part of an L D L' device SM)
    int scale_sqrt_d(const double* d_sm, double* d_b, int64_t ldb, int64_t nrhs, bool divide);
    // Device-resident forward (which=1), back (which=2) or both (3) on b (device, ldb x nrhs).
    int solve(const double* d_sm, double* d_b, int64_t ldb, int64_t nrhs, int which);
    // Iterative refinement (mixed precision): build_residual() compacts the
    // assembled (unfactored) SM into a CSR of the FP64 matrix; refine() runs
    // x = solve(b), then r = b - K x, x += solve(r) until the normwise
    // backward error max|r| / (||K||inf max|x| + max|b|) <= tol.
    // out[0] = correction steps, out[1] = final backward error, out[2] = solve ms.
    int build_residual(const double* d_sm_assembled);
    int residual(const double* d_b, const double* d_x, double* d_r, int64_t ld, int64_t nrhs, double* berr);
    int refine(const double* d_sm, const double* d_b, double* d_x, int64_t ld, int64_t nrhs, double tol, int maxit,
               double* out);
    // Mixed mode autotuner (see engine.cu): times candidate engine choices on a
    // copy of the assembled SM and keeps the fastest.  out: 5 doubles.
    int autotune(const double* d_sm_assembled, double* out);
    // Tile autotuner of the small FP64 Schur updates (64x64 or 32x32 tiles),
    // timed on a copy of the assembled SM; out: tile, ms with 64, ms with 32.
    int autotune_tiles(const double* d_sm_assembled, double* out);
    void set_small_tile(int t) { small_tile_ = (t == kTileTiny) ? kTileTiny : kTile; }
    int small_tile() const { return small_tile_; }
    // Content hash (smhash.h) of n doubles of device memory, on the engine's stream.
    int hash(const double* d_a, int64_t n, uint64_t& h);
    // Per-supernode negative-pivot counts and failing column of the last factor().
    int sn_stats(int32_t* neg, int32_t* fail);
    // The solves use the inverses of the diagonal blocks that factor() stores;
    // after SM was replaced by a factor from elsewhere, call this so the next
    // solve rebuilds them from LNZ.
    void invalidate_factor() { linv_valid_ = false; }
    // Timing of the Schur-update kernels can be switched on (events around each launch).
    void set_profile(bool on) { profile_ = on; }
    // CUDA-graph replay of the factor/solve launch sequences (on by default;
    // SPR_B200_GRAPHS=0 or set_graphs(false) launches kernel by kernel).
    void set_graphs(bool on) { use_graphs_ = on; }
    // Mixed precision: the Schur updates of the large fronts as 3xTF32 split
    // products (FP64 diagonal blocks, TRSM, small fronts and storage).
    // 0 = FP64, 1 = tcgen05 tensor cores (k_gemm_tc), 2 = mma.sync (k_gemm_x3).
    void set_mixed(int mode) { mixed_ = mode; }
    int mixed() const { return mixed_; }
    // Inertia guard of the mixed mode: when a pivot with |d| < tau |a_jj|
    // (or a pivot failure) is met, the factorisation is redone in FP64 from
    // a copy of the assembled SM taken before it, so NUMNEG and the pivot
    // test are decided in FP64.  tau = 0 switches the guard (and the copy) off.
    void set_inertia_guard(double tau) { guard_tol_ = tau; }
    double inertia_guard() const { return guard_tol_; }
    int64_t last_near_pivots() const { return last_near_; }
    double last_trace() const { return last_trace_; }
    bool last_refactored() const { return last_refactor_; }
    // Watchdog of the kernels that wait on device flags (the tensor-core
    // update's mbarriers, the solves' block-ready flags): time limit of each
    // wait (ns), and a test switch that makes some waits run out (one CTA's
    // operand load, one solve task's report is skipped); the factorisation or
    // solve then returns -4 and the engine stays usable.
    void set_watchdog(unsigned long long wait_ns, bool drop) {
        wait_ns_ = wait_ns;
        tc_drop_ = drop;
    }
    // A system split across GPUs (one engine per rank, the same plan on all):
    // supernodes with mask[js] != 0 are left alone by factor() and solve()
    // (another rank factors them); null clears the mask.  The exchange lists
    // of the following factor() move update blocks ((F-S) x (F-S) doubles,
    // column-major, leading dimension F-S), those of the forward sweep of the
    // following solve() update vectors ((F-S) x nrhs): an "out" entry is
    // copied from the node's block/vector into buf right after the node's
    // level, an "in" entry from buf into it right before its parent's level,
    // both on the engine's stream.  The lists stay until replaced.
    struct Xfer {
        int32_t node;
        double* buf;
    };
    int set_skip(const uint8_t* host_mask);
    void set_exchange(std::vector<Xfer> factor_out, std::vector<Xfer> factor_in, std::vector<Xfer> vec_out,
                      std::vector<Xfer> vec_in);
    Timing timing;
    struct Dev;              // device copies of the plan and work buffers
    struct Transfer;         // copy ranges and events of the streamed factorisation

private:
    struct GraphKey {
        const void* a;
        const void* b;
        double x;
        int64_t n;
        int w;
        int64_t v;
        const void* c = nullptr;
        double y = 0.0;
        double z = 0.0;
        bool operator==(const GraphKey& o) const {
            return a == o.a && b == o.b && x == o.x && n == o.n && w == o.w && v == o.v && c == o.c && y == o.y &&
                   z == o.z;
        }
    };
    struct GraphEntry {
        GraphKey key;
        cudaGraphExec_t exec;
        int64_t launches;
    };
    cudaGraphExec_t find_graph(const GraphKey& k);
    int64_t graph_launches(const GraphKey& k);
    void store_graph(const GraphKey& k, cudaGraphExec_t exec, int64_t launches);
    void enqueue_factor(const struct PV& pv, cudaStream_t s, std::vector<cudaEvent_t>& gev);
    void enqueue_solve(const struct PV& pv, cudaStream_t s, double* d_b, int64_t ldb, int64_t nrhs, int which,
                       int64_t& nl);
    std::vector<GraphEntry> graphs_;
    bool use_graphs_ = true;
    bool tri_solve_ = true;                  // solve triangles as one dataflow launch per level
    std::vector<Xfer> fout_, fin_, vout_, vin_;   // exchange lists of a split run
    bool split_ = false;                     // a mask or exchange lists are set (no graphs)
    void block_copy(int32_t js, double* buf, bool out, cudaStream_t s);
    void vec_copy(int32_t js, double* buf, bool out, int64_t nrhs, cudaStream_t s);
    const LevelHooks* hooks_ = nullptr;      // set during a streamed factorisation
    const double* streamed_diag_ = nullptr;  // its host-gathered original diagonal (device)
    std::unique_ptr<Transfer> xfer_;
    int mixed_ = 0;
    double guard_tol_ = 1.0e-3;
    int64_t last_near_ = 0;
    double last_trace_ = 0.0;
    bool last_refactor_ = false;
    double* guard_copy_ = nullptr;           // assembled SM kept for the FP64 redo of the guard
    int64_t guard_cap_ = 0;
    unsigned long long wait_ns_ = 2000000000ull;
    bool tc_drop_ = false;
    bool chol_ = false;                      // factor with SPRF27's pivot rule
    double tc_min_flops_ = 0.0;   // mixed mode: launches below this stay on the FP64 kernel
    int far_cap_q_ = 3;           // side-stream tensor-core launches: quarters of the SMs
    int small_tile_ = kTile;      // tile of the small FP64 Schur updates (kTile or kTileTiny)
    std::vector<std::pair<int, cudaEvent_t>> marks_;
    std::vector<size_t> tc_pairs_;        // profile mode: event pairs of the tensor-core launches
    int sm_count_ = 148;
    int ensure_slabs();
    void launch_tc(const TcLaunch& t, cudaStream_t s, const struct PV& pv, std::vector<cudaEvent_t>& gev,
                   bool far = false);
    struct Csr {
        int64_t* rowptr = nullptr;
        int32_t* ci = nullptr;
        double* cv = nullptr;
        double* rowabs = nullptr;
        int64_t nnz = 0;
        double norm_inf = 0.0;
    } csr_;
    double* rbuf_ = nullptr;
    int64_t rbuf_cap_ = 0;
    double* nbuf_ = nullptr;      // the residual's max norms (3 per right-hand side)
    int64_t nbuf_cap_ = 0;
    void launch_gemm(const Launch& l, cudaStream_t s, const struct PV& pv, std::vector<cudaEvent_t>& gev);
    void launch_diag(const Launch& pl, cudaStream_t s, const struct PV& pv);
    void upload_plan();
    void ensure_vectors(int64_t nrhs);
    Plan P_;
    cudaStream_t stream_ = nullptr;
    bool profile_ = false;
    bool linv_valid_ = false;
    std::unique_ptr<Dev> d_;
};

// Blocked LDL' of one dense front a (n x n, column-major, leading dimension
// lda, lower triangle used) in place, with every scratch buffer carved out
// of the caller's `scratch` (no device allocation).  d receives the pivots.
// Returns 0, -2 for a bad shape/alignment (lda % 4 == 0 and a 32-byte
// aligned are required), -3 when the scratch is too small, -4 on CUDA
// errors.  out[0]=NUMNEG out[1]=first failing column (1-based, 0 if none)
// out[2]=that pivot out[3]=its original a_jj out[4]=max(a_jj/d_j).
size_t dense_scratch_bytes(int64_t n);
// Per-device set-up of dense_factor_with_scratch's kernels (their shared-memory
// opt-in) on the current device; allocates nothing.  0 or -4.
int dense_factor_setup();
int dense_factor_with_scratch(double* a, int64_t n, int64_t lda, double tol1, double* d, void* scratch,
                              size_t scratch_bytes, cudaStream_t s, double* out);

}  // namespace sprb
