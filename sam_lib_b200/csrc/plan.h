// Host-side execution plan for the GPU numeric phase of SPR.
//
// Built once per symbolic structure (MSPAR/MTREES/MSIFA as produced by the
// SPR host pipeline, src/SPR/sprtrs.f + sprsmb.f + sprpmp.f) and cached by the
// C-ABI layer.  It turns SPR's postordered supernode list into
//   * elimination-tree levels (all fronts of a level are independent),
//   * relative-index maps child -> parent (the integer merge of SPRF12,
//     src/SPR/sprfc1.f:716-790, done once instead of per factorisation),
//   * per-parent contribution lists (which child update column lands on which
//     parent column), so extend-add is a deterministic, atomic-free gather,
//   * a device arena layout for fronts / update matrices (first-fit reuse:
//     a child's buffer is released once its parent level is assembled),
//   * the batched task lists of the panel steps of the large fronts.
#pragma once
#include <cstdint>
#include <vector>

namespace sprb {

constexpr int kSmallMaxF = 176;     // fronts up to this order: one CTA, shared memory
constexpr int kNB = 64;             // panel width of the blocked LDL' for large fronts
constexpr int kTRSMRows = 64;       // rows per CTA in the panel (TRSM) kernel
constexpr int kTile = 64;           // Schur-update tile of small updates (rows x cols)
#ifndef SPR_TILE_BIG
#define SPR_TILE_BIG 64
#endif
constexpr int kTileBig = SPR_TILE_BIG;   // Schur-update tile of large updates
constexpr int kTileTiny = 32;            // the autotuner's alternative tile for the small updates
constexpr int kSuperPanel = 512;    // trailing updates are applied per 512 columns (K = 512)
constexpr int kAsmChunk = 256;      // rows per warp pass in the large-front assembly

// A job is one front's share of one batched launch.  Tasks inside a job are
// decoded on the device (binary search over `task0`, then closed-form
// arithmetic), so the plan stays O(fronts x steps) instead of O(tiles).
//   assembly / write-back : one task per column in [c0, c_end)
//   panel (TRSM)          : task 0 = diagonal-block CTA, then row blocks of
//                           kTRSMRows rows starting at c0 (= k_hi)
//   Schur update          : lower-triangle tiles (Launch::tile) of rows
//                           [c0, r_end) x columns [c0, c_end), contraction
//                           over [k_lo, k_hi)
// Blocked right-looking LDL' of the S fully-summed columns with two levels:
// 64-wide panels (diagonal block + TRSM) whose updates stay inside their
// kSuperPanel-wide super-panel, one K = kSuperPanel trailing update per
// super-panel for the remaining fully-summed columns, and one K=S update of
// the (F-S) block.
struct Job {
    int32_t node;
    int32_t c0, c_end, r_end;
    int32_t k_lo, k_hi;
    int64_t task0;                   // first task of this job within its launch
    int64_t slab = 0;                // tensor-core updates: first row of the job's operand slabs
};

struct Launch {                      // a contiguous range of Plan::jobs
    int64_t job_begin = 0, job_count = 0, ntasks = 0;
    int32_t tile = kTile;            // Schur-update launches: tile size of the decode
    int64_t map_begin = -1;          // task -> job map of this launch in Plan::task_map
    int32_t alt = -1;                // a kTile update launch: the same jobs in kTileTiny tiles (Plan::alt)
};

// A tensor-core Schur-update launch: the split of the panel into FP32 hi/lo
// operand slabs, then the 128x128-tile update (one task per lower tile).
constexpr int kTcTile = 128;
constexpr int kTcBK = 32;
struct TcLaunch {
    Launch split;                    // one task per 32 rows x 32 columns of each job's panel
    Launch gemm;                     // one task per lower 128x128 tile of each job's block
};

struct LevelPlan {
    std::vector<int32_t> small_nodes;        // fronts done by the fused one-CTA kernel
    std::vector<int32_t> large_nodes;        // fronts done by the blocked path (assembly, write-back)
    std::vector<int32_t> elim_nodes;         // of those, the ones eliminated (not retained)
    int32_t small_maxF = 0;
    // small fronts in size classes (F <= 64, 96, 128, 176), one launch each so
    // that the smaller fronts get the shared memory (and occupancy) they need:
    // {first index into small_nodes, count, largest F}
    struct SmallClass {
        int32_t begin, count, maxF;
    };
    std::vector<SmallClass> small_classes;
    Launch assemble;                          // large fronts: extend-add into dense fronts
    std::vector<Launch> panel;                // per panel step: diagonal block + TRSM
    std::vector<std::vector<Launch>> update;  // per panel step: Schur updates (one launch per tile size)
    // per panel step inside a super-panel: the update of the columns after the
    // next panel (look-ahead stream, beside the next diagonal block and TRSM)
    std::vector<std::vector<Launch>> ahead;
    // mixed precision: a super-panel's K = kSuperPanel update of the next super-panel's
    // columns (the update[st] jobs of a step that ends a super-panel) as a
    // split + tensor-core pair, and its algorithmic flops
    std::vector<std::vector<TcLaunch>> next_tc;
    std::vector<double> next_flops;
    std::vector<Launch> outer;                // update block, K = S (one launch per tile size)
    Launch writeback;                         // S columns -> LNZ
    // per panel step: the columns of the super-panels that end at that step
    // (their last panel's TRSM is done), for writing LNZ early
    std::vector<Launch> wb_sp;
    std::vector<Launch> fsolve;               // forward step: 1 diagonal CTA + row blocks below
    std::vector<Launch> bsolve;               // back step: 1 diagonal CTA + column groups [0, k0)
    // solves in kSolveBlock-wide steps: per step, the diagonal-block launch uses
    // the job list (one CTA per job), the update launch its tasks
    std::vector<Launch> fs_upd;               // rows [k1, F) below the block, kSolveRows per task
    std::vector<Launch> bs_upd;               // columns [0, k0) before the block, kBwdCols per task
    std::vector<Launch> blk_mv;               // product with the block inverse, 32 rows/columns per task
    Launch rect;                              // rectangle rows [S, F): one task per 256 x 256 tile
    Launch rect_rows;                         // forward solve, rows [S, F): one task per row
    // triangle of the solves as one dataflow launch: tasks (node, 64-row
    // block) of the level's eliminated large fronts, block-major, in
    // Plan::tri_tasks[tri_begin .. tri_begin + tri_count)
    int64_t tri_begin = 0, tri_count = 0;
    // trailing update columns beyond the next super-panel (side stream)
    std::vector<std::vector<Launch>> far;
    std::vector<std::vector<TcLaunch>> far_tc;
    std::vector<double> far_flops;            // algorithmic flops of each step's far launches
    double outer_flops = 0.0;                 // and of the K = S update
    std::vector<TcLaunch> outer_tc;                 // mixed precision: the K = S update
};

constexpr int kBwdCols = 8;                   // columns per CTA in the back-solve update
constexpr int kSolveBlock = 256;              // width of a solve step (4 diagonal blocks of kNB)
constexpr int kSolveRows = 128;               // rows per CTA in the forward update (x 2 column halves)
constexpr int kRectCols = 64;                 // columns per CTA of the solves' rectangle launches
constexpr int kRectRows = 256;                // rows per CTA of the solves' rectangle launches

struct Plan {
    // sizes
    int64_t neq = 0, nsuper = 0, nzerol = 0, nofsub = 0, maxsup = 0, mfront = 0;
    // per supernode (postorder index js = 0..nsuper-1)
    std::vector<int32_t> fst, S, F, parent, level;
    std::vector<int64_t> lnz_off, lindx_off;
    std::vector<int32_t> child_ptr, child;   // children in SIBL order
    std::vector<int32_t> rows;               // LINDX (0-based rows), concatenated like LINDX
    // partial factorisation (MSPAR(57) > 0): the retained supernodes
    // (SUPSUP > 0, src/SPR/sprtrs.f:1142-1204) are assembled but not
    // eliminated (sprfc1.f:587) and skipped by the solves (sprfs1.f:371)
    std::vector<uint8_t> retained;
    bool any_retained = false;
    // update-row -> parent-row maps, one per non-root supernode with F > S
    std::vector<int64_t> rel_off;            // per node, offset into rel
    std::vector<int32_t> rel;
    // contribution CSR: for parent p, column j: entries [cptr[rbase[p]+j], cptr[rbase[p]+j+1])
    std::vector<int64_t> rbase;              // per node, prefix of F
    std::vector<int64_t> cptr;
    std::vector<int32_t> cchild, ct;         // (child, child update column)
    // device arena (units of doubles)
    std::vector<int64_t> buf_off;            // per node: start of its buffer
    std::vector<int32_t> buf_ld;             // leading dimension of the front / update buffer
    std::vector<int64_t> upd_off;            // per node: where its update matrix (F-S)^2 starts
    int64_t arena_doubles = 0;
    // inverses of the unit-lower diagonal blocks of the large fronts: block st
    // of node js is the column-major kNB x kNB matrix at linv_off[js] + st*kNB*kNB
    std::vector<int64_t> linv_off;
    int64_t linv_doubles = 0;
    // inverses of the kSolveBlock-wide unit-lower diagonal blocks (the solves):
    // block b of node js is column-major nb x nb (nb = min(kSolveBlock, S - b*kSolveBlock))
    // at xinv_off[js] + b*kSolveBlock*kSolveBlock
    std::vector<int64_t> xinv_off;
    int64_t xinv_doubles = 0;
    Launch inv_blocks;                        // one task per (large front, solve block)
    // back-solve rectangle partial sums: node js uses rect_off[js] .. + nchunk*S entries
    // (each kMaxRHS doubles) of a scratch of rect_entries entries (max over levels)
    std::vector<int64_t> rect_off;
    int64_t rect_entries = 0;
    std::vector<int64_t> fwd_off;            // forward-sweep rectangle partials, per level
    int64_t fwd_entries = 0;
    // the solves' triangle tasks (pairs node, 64-row block) of every level
    // and, per large front, the first of its blocks' ready flags
    std::vector<int32_t> tri_tasks;
    std::vector<int64_t> tri_off;
    int64_t tri_flags = 0;
    bool any_large = false;
    // levels and tasks
    std::vector<LevelPlan> levels;
    std::vector<Job> jobs;
    // for every launch: the job (relative to Launch::job_begin) of each task,
    // so a CTA finds its job with one load instead of a binary search
    std::vector<int32_t> task_map;
    std::vector<Launch> alt;                 // kTileTiny versions of the small-tile update launches
    // statistics (the reference's own counters are recomputed for reporting)
    double factor_flops = 0.0;               // = RINFO(3) formula, src/SPR/sprtrs.f:1961-1969
    double solve_flops = 0.0;                // = RINFO(4) formula, src/SPR/sprtrs.f:1976-1980
    double gemm_flops = 0.0;                 // algorithmic flops of the Schur-update launches
    double tc_flops = 0.0;                   // of those, the updates the mixed mode runs on tensor cores
    int64_t slab_rows = 0;                   // largest operand-slab need of one tensor-core launch (128-byte rows)
    int64_t slab_rows_far = 0;               // the same for the side-stream launches
    double small_flops = 0.0;                // factor flops done by the fused small-front kernel
};

// Builds the plan from the SPR control arrays.  Returns 0 on success or a
// negative code when the structure is inconsistent (mirrors IERR=-2 checks).
int build_plan(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, Plan& plan);

// Size in doubles of a node's device buffer (update matrix or dense front).
int64_t buffer_doubles(const Plan& P, int64_t js);
// Self-check of the arena layout and the index maps: counts buffers outside
// the arena plus relative-index / contribution-list entries out of range or
// not used exactly once (oob), and overlaps between buffers that are live at
// the same level.
void check_plan(const Plan& P, int64_t& oob, int64_t& overlaps);
// Schur-update coverage: every column c of every large front must receive
// exactly the K ranges that tile [0, 64 floor(c / 64)) for c < S (earlier
// panels; a column's own panel is eliminated by the diagonal block and TRSM)
// and [0, S) for c >= S (nothing for a retained front),
// once, across the update, far and K = S launches.  Counts the columns that
// do not, for the FP64 launch lists (fp64) and the tensor-core lists in the
// mixed mode's use (tc: FP64 panel-chain updates + tensor-core far and K = S).
void check_coverage(const Plan& P, int64_t& fp64, int64_t& tc);
// Happens-before check of the factorisation's two-stream launch schedule
// (panels, panel-chain and far updates, K = S update, write-back): the number
// of ordering violations, 0 for a race-free schedule.  tc: the far and K = S
// updates on the tensor-core path; skip_join: the schedule without its
// side-stream joins (a self-test: must report violations where far launches exist).
int64_t check_schedule(const Plan& P, bool tc, int skip_join);
// Self-check of the solves' plan: every eliminated large front of a level has
// each of its 64-row triangle blocks as one task of that level's dataflow
// launch, after the task of the block above it (the forward sweep takes them
// in list order, the back sweep in reverse), with its own ready flag (the
// fronts' flag ranges disjoint and inside Plan::tri_flags); each front with
// F > S has one rectangle job and one forward-rows job of the right sizes,
// and the partial-sum ranges of a level's fronts (rect_off, fwd_off) are
// disjoint and inside their scratch.  Returns the number of violations.
// plant: 0 checks P as built; 1 swaps the first two blocks of a front in a
// copy, 2 moves one front's forward partials onto another's in a copy (a
// self-test: both must report violations where such fronts exist).
int64_t check_solve_plan(const Plan& P, int plant, int64_t* tasks = nullptr);

}  // namespace sprb
