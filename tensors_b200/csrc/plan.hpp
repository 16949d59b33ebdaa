// Device execution plan of the supernodal factorization and solves.
//
// The symbolic analysis yields the reference's supernodes, whose partition is
// part of the drop-in contract (SN_rp, SN_inner, the value layout).  Many of
// them are thin -- a separator node with a private neighbour in an ancestor
// separator always starts a new fundamental supernode -- and a chain of thin
// supernodes is a chain of large, nearly identical update matrices.  The GPU
// therefore computes on *fronts*: maximal runs of supernodes in which each is
// the last child of the next (so their rows are contiguous) merged while the
// structural zeros this adds stay within relaxation limits (the classical
// relaxed-supernode amalgamation).  A front's column set is that of its top
// supernode; zeros it carries stay exactly zero through every kernel.  The
// reference's per-supernode layout (row-major U0 squares, U1 rectangles at
// SN_tri_ptr / SN_rec_ptr) is produced from the fronts by an export kernel on
// request.
//
//  * the factor arena holds, per front, U0 (n0 x n0, row-major upper), U1
//    (n0 x n1, row-major), rows padded to kLdAlign entries (32-byte aligned
//    rows for vector and bulk copies), and an update-matrix region in which each front's
//    n1 x n1 contribution block V (Multifrontal.hpp:165) lives from its
//    front's level until its parent's level; V regions are reused across
//    levels by a best-fit allocator and zeroed by the level that owns them;
//  * fronts are grouped in levels by height in the front tree (leaves are
//    level 0); a level runs after all lower levels;
//  * within a level, children's update matrices are added into their parents
//    in child-rank passes (pass r adds every parent's r-th child), so no two
//    tasks of a launch write the same entry and the summation order is the
//    reference's (A, then children in order, Multifrontal.hpp:210-224);
//  * each front's pivots are eliminated in panels of kPanel rows: a potrf
//    launch factors the panel's diagonal block in place (one CTA per front),
//    a trsm launch solves the panel's row of the front against it (one CTA
//    per kRestChunk columns), an update launch applies the rank-kPanel
//    trailing update to the remaining rows of U0 and U1 as 64 x 64 GEMM
//    tiles, and in the update launch of a front's last panel its
//    V -= U1^T U1 tiles run with the full depth K = n0.
#pragma once

#include <cstdint>
#include <vector>

#include "symbolic.hpp"

namespace tb
{

constexpr int kPanel     = 64;    // pivot panel width
constexpr int kTile      = 64;    // GEMM output tile (kTile x kTile)
constexpr int kRestChunk = 64;    // rest columns per panel-solve CTA
constexpr int kSolveRest = 64;    // rows per solve-update task
constexpr int kLdAlign   = 4;     // row padding of every front block (entries)
constexpr std::uint64_t kDiagFlag = 1ull << 62;   // marks diagonal entries in the assembly map

// Relaxed amalgamation limits: a merge whose front has at most nrelax[0]
// rows is always taken; otherwise the fraction of structural zeros in the
// merged front must stay below zrelax[k] for the first k with
// rows <= nrelax[k] (zrelax[2] beyond).
struct Relaxation
{
    std::int32_t nrelax[3] = { 8, 32, 64 };
    double       zrelax[3] = { 0.8, 0.2, 0.1 };
};

// C[m0:m0+64, c0:c0+64] -= A[0:K, m0:m0+64]^T * B[0:K, c0:c0+64]; all
// operands row-major in the arena.  upper: only entries with (row <= col)
// in C's coordinates are written (diagonal tiles of symmetric blocks).
struct GemmTask
{
    std::int64_t a, b, c;          // arena offsets of A[0][0], B[0][0], C[0][0]
    std::int32_t lda, ldb, ldc;
    std::int32_t K, M, N;
    std::int32_t m0, c0;
    std::int32_t upper;
    std::int32_t pad;
};

// Panel [r0, r0+nb) of a front.  As a potrf task: factor the diagonal block
// in place.  As a trsm task: solve the panel's rows for rest columns
// [c0, c0 + kRestChunk) against the factored block: rest column j is U0
// column r0+nb+j when j < n0-r0-nb, else U1 column j-(n0-r0-nb).  row0 is
// the front's first global row (failures report the failing global row);
// bit r of single_rows marks panel rows that form a 1 x 1 reference
// supernode, whose pivot is taken as sqrt(|a|) (Multifrontal.hpp:471).
struct PanelTask
{
    std::int64_t u0, u1;
    std::int32_t n0, n1;
    std::int32_t ld0, ld1;         // leading dimensions of U0 / U1
    std::int32_t r0, c0;
    std::int32_t row0;
    std::int32_t panel;            // index of the panel (its potrf task, SolveDiagTask and inverse block)
    std::int64_t single_rows;      // bit r set: panel row r is a 1 x 1 reference supernode
    std::int64_t img;              // FP32 path: the front's first operand-image block (see TcTask)
    std::int32_t img_t0, img_tf;   // its U0 column tiles, and U0 + U1 column tiles per k-chunk segment
};

// The FP32 path's Schur-complement tiles on the 5th-generation tensor cores
// read their operands from an *operand image*: every panel row of a front,
// once its trsm is done, split into TF32 hi and lo parts (x = hi + lo) and
// stored transposed in blocks of kImgRows U columns x kImgK U rows (row-major
// inside the block: the 32 k values of one U column are 128 contiguous bytes,
// one 128-byte-swizzled row of a K-major tensor-core operand).  Block
// (k-chunk kc, part hl, column tile ct) of front f is
//     img + (kc * 2 + hl) * tf + ct,
// where column tiles 0 .. t0-1 are U0 columns and t0 .. tf-1 are U1 columns
// (each 64-aligned), so every operand tile is a few whole blocks: one tensor
// map over the whole image serves every front.
constexpr int kImgRows = 64;
constexpr int kImgK    = 32;
constexpr int kTcM     = 128;     // tensor-core tile rows
constexpr int kTcNMax  = 256;     // widest tensor-core tile

// C[m0 : m0+kTcM, c0 : c0+nt] -= A^T B for K panel rows: A's columns are
// operand-image column tiles ta, ta+1 (the C rows), B's are tb .. tb+nt/64-1,
// over the k-chunks blk, blk + 2 tf, ... (hi; lo at + tf).  Rows >= M and
// columns >= N are not written; upper: only (row <= col) entries.
struct TcTask
{
    std::int64_t c;                // arena offset of C[0][0]
    std::int64_t blk;              // image block of (first k-chunk, hi, column tile 0)
    std::int32_t ldc, M, N;
    std::int32_t m0, c0;
    std::int32_t K;
    std::int32_t ta, tb, tf;
    std::int32_t nt;               // tile width: 64, 128, 192 or 256
    std::int32_t upper;
    std::int32_t pad;
};

// Add rows [row_begin, row_end) of child update W (m1 x m1, upper) into the
// parent front through lut (Multifrontal.hpp:324-436).
struct ExtendTask
{
    std::int64_t w, u0, u1, v;
    std::int64_t lut;              // offset into the lut array
    std::int32_t m1, mid;
    std::int32_t n0p, n1p;         // parent dimensions
    std::int32_t ldw;              // leading dimension of the child's W
    std::int32_t ld0p, ld1p, ldvp; // leading dimensions of the parent's U0 / U1 / V
    std::int32_t row_begin, row_end;
};

// Diagonal block of panel [r0, r0+nb) of a front whose first row is row0.
// Its inverse (kPanel x kPanel, row-major, identity-padded beyond nb) is
// block k of the inverse-diagonal buffer, k = the task's index.
struct SolveDiagTask
{
    std::int64_t u0;
    std::int32_t n0, r0, row0, ld0;
};

// One CTA of a solve step for panel [r0, r0+nb) of a front: rows [c0, c1)
// of the panel's rest (U0 rows below the panel, then the front's U1 columns,
// whose global rows come from SN_inner at offset inner), or c0 = -1, c1 = 0
// for a panel without rest rows.  The task with c0 <= 0 also applies the
// inverse diagonal block to the panel's own rows.  panel = index of the
// panel's SolveDiagTask.
struct SolveRestTask
{
    std::int64_t u0, u1, inner;
    std::int32_t n0, n1, r0, row0, c0, c1;
    std::int32_t ld0, ld1;
    std::int32_t panel, pad;
};

// Zero rows [row_begin, row_end) of the upper triangle of the n x n update
// matrix at arena offset `offset` (leading dimension ld): columns [r, n) of
// row r, `count` entries in all.  The strictly lower triangle is never read.
struct ZeroTask
{
    std::int64_t offset, count;
    std::int32_t n, ld, row_begin, row_end;
};

// Copy rows [r_begin, r_end) of reference supernode sn from its front into
// the reference layout: tri (n0s x n0s upper) and rec (n0s x n1s) blocks.
struct ExportTask
{
    std::int64_t fu0, fu1;         // front U0 / U1 arena offsets
    std::int64_t tri, rec;         // destination offsets (tri region / rec region)
    std::int64_t colmap;           // offset into colmap (== SN_outer[sn])
    std::int32_t fn0, fn1;         // front dimensions
    std::int32_t fld0, fld1;       // front leading dimensions
    std::int32_t roff;             // first row of sn within the front
    std::int32_t n0s, n1s;         // supernode dimensions
    std::int32_t r_begin, r_end;
    std::int32_t pad;
};

// One task of the factorization's task graph, executed by one CTA of the
// persistent factorization kernel: `index` into the task array of `kind`.
// Before it runs, counter wait[i] must have reached target[i] (unused
// waits: -1); when it is done it increments the counters signal[0..1]
// (-1: none).  The task list is in a topological order: every target is
// reached by tasks earlier in the list, which the plan check verifies.
constexpr int kDagWaits = 4;
constexpr int kDagMinSteps = 8;      // levels from the first with this many panel steps run as the task graph
constexpr int kSolveDagMinSteps = 4; // the same for the solves
constexpr int kDeferSteps = 3;       // panel steps over which a front's trailing update is deferred

struct DagTask
{
    std::int32_t kind, index;
    std::int32_t signal[2];
    std::int32_t wait[kDagWaits];
    std::int32_t target[kDagWaits];
};

enum class LaunchKind : std::int32_t { Zero = 0, Extend = 1, Trsm = 2, Gemm = 3, Invert = 4, Solve = 5, Potrf = 6,
                                       SuperInv = 8, SuperDiag = 9, SuperRest = 10, ExtendPull = 11 };

// Extend-add by parent rows (the level launches): one CTA adds, child by
// child in rank order, the rows of every child that map into one block of
// a parent's rows (pivot rows: U0 / U1; update rows: V).  The segments are
// ExtendTasks whose [row_begin, row_end) are those child rows.  Every parent
// entry receives the same additions in the same order as in the passes by
// child rank (the persistent schedule's extend tasks), in one launch per
// level instead of one per child rank.
struct ExtendPullTask
{
    std::int64_t seg_first;        // its segments in Plan::extend_segs
    std::int32_t seg_count;
    std::int32_t space;            // 0: pivot rows (U0 / U1), 1: update rows (V)
    std::int32_t b0, b1;           // its parent rows [b0, b1) in that space
};
constexpr std::int64_t kExtendPullEntries = 4096;    // target child entries per pull task

// The solve of a large front steps through its pivot rows 512 at a time
// (super-panels) instead of 64 at a time: the inverse of each 512 x 512
// diagonal block of U0 (T, FP64, upper triangular, row-major, built from
// the 64-row panel inverses after the factorization by block back
// substitution) turns eight sequential panel steps into one.  A front uses
// super-panels when it has at least kSuperMinRows pivot rows.
constexpr int kSuperPanels  = 8;
constexpr int kSuperRows    = kSuperPanels * kPanel;   // 512
constexpr int kSuperMinRows = 256;

struct SuperPanel
{
    std::int64_t u0, u1, inner;    // the front's U0 / U1 arena offsets and its SN_inner offset
    std::int64_t t;                // offset of the inverse (ldt x ldt doubles, row-major)
    std::int32_t n0, n1, ld0, ld1;
    std::int32_t r0, rows;         // first pivot row of the block (a multiple of 512) and its row count
    std::int32_t row0;             // the front's first global row
    std::int32_t panel[kSuperPanels];   // inverse-block index of each 64-row panel (-1 beyond rows)
    std::int32_t ldt;              // the inverse's edge: rows rounded up to 64
};

// Block (i, j = i + d) of a super-panel's inverse, formed in round d:
// d = 0 copies panel i's inverse; d > 0: T_ij = -T_ii sum_{k=i+1..j} U_ik T_kj.
struct SuperInvTask
{
    std::int32_t sp, i, j, pad;
};

// A super-panel solve task.  Diag: the pair (blk, c0) of 64-row blocks, one
// term of the block's solution x_blk = sum_{i<=blk} T_{i,blk}^T y_i (forward,
// i = c0 <= blk) or sum_{j>=blk} T_{blk,j} (y_j + z_j) (back, j = c0 >= blk).
// Rest: block blk and rest rows [c0, c1) of the front after the super-panel
// (U0 rows, then its U1 columns): forward y_rest -= U_{blk,rest}^T x_blk; back
// z_blk -= U_{blk,rest} x_rest.
struct SuperSolveTask
{
    std::int32_t sp, blk, c0, c1;
};

// One launch: `count` tasks starting at `first` in the array of its kind.
// A panel step's GEMM tiles come as two launches: part 0 updates the next
// panel's rows (the next potrf / trsm wait for it), part 1 the rest of the
// trailing matrix and the update matrices (it may overlap the next panel).
struct Launch
{
    LaunchKind   kind;
    std::int32_t count;
    std::int64_t first;
    std::int32_t level;
    std::int32_t step;
    std::int32_t part = 0;
    // Gemm launches, FP32 path: the first small_count tiles belong to fronts
    // without an operand image (64 x 64 tiles); the updates of the other
    // tiles are the tensor-core tiles [tc_first, tc_first + tc_count)
    std::int64_t tc_first = 0;
    std::int32_t tc_count = 0;
    std::int32_t small_count = 0;
    // ExtendPull launches: the level's extend tasks in pass order are
    // [tc_first, tc_first + tc_count) of Plan::extend (what the persistent
    // schedule runs instead)
};

struct Plan
{
    Relaxation relax;
    std::int32_t defer_steps = kDeferSteps;   // panel steps over which a front's trailing update is deferred (1-4)
    std::int32_t tc_nmax = kTcNMax;           // widest tensor-core tile of the FP32 path (128 or 256)
    std::int32_t threads = 0;                 // host threads of the build and the check (<= 0: every hardware thread)

    // fronts: runs [sn_first, sn_last] of reference supernodes
    std::int32_t front_count = 0;
    std::vector<std::int32_t> front_sn_first, front_sn_last;
    std::vector<std::int32_t> front_row0, front_n0, front_n1;
    std::vector<std::int64_t> front_cols;      // offset of the column set in SN_inner
    std::vector<std::int32_t> front_parent;    // front_count = root
    std::vector<std::int32_t> front_of_sn;

    // arena layout (doubles): [U0 of all fronts][U1 of all fronts][update region];
    // rows are padded to a multiple of kLdAlign entries so every row of every
    // block starts on a 32-byte boundary
    std::int64_t u0_size = 0, u1_size = 0, v_size = 0;
    std::vector<std::int64_t> front_u0, front_u1, front_v;   // arena offsets
    std::vector<std::int32_t> front_ld0, front_ld1;          // U0 / U1 leading dimensions (V uses ld1)

    std::int32_t levels = 0;
    std::vector<std::int32_t> level_of;     // per front

    // extend-add lookup: lut[front_lut[t] + i] = position of column i of front
    // t in its parent (row of U0 when < mid, else position in the parent's
    // column set)
    std::vector<std::int32_t> lut;
    std::vector<std::int64_t> front_lut;

    // assembly map over the upper triangle of the permuted matrix
    std::vector<std::int64_t> asm_src;      // index into the caller's value array
    std::vector<std::int64_t> asm_dst;      // arena offset, | kDiagFlag on the diagonal

    // export to the reference layout: colmap[SN_outer[s] + l] = U0 column
    // (>= 0) or -(U1 column + 1) of column l of supernode s within its front
    std::vector<std::int32_t> colmap;
    std::vector<ExportTask>   exports;
    std::vector<std::int64_t> diag_offset;  // per row: arena offset of U(i,i)

    std::vector<GemmTask>      gemm;
    std::vector<TcTask>        tc;             // the GEMM updates as tensor-core tiles (FP32 path, level launches)
    std::vector<std::int64_t>  front_img;      // per front: first operand-image block
    std::int64_t img_blocks = 0;               // operand-image size in blocks of kImgRows x kImgK floats
    std::vector<PanelTask>     potrf;          // one per (front, panel)
    std::vector<PanelTask>     panel;          // trsm chunks
    std::vector<ExtendTask>    extend;
    std::vector<ZeroTask>      zero;
    std::vector<SolveDiagTask> sdiag;          // one per (front, panel); also the inverse-block list
    std::vector<SolveRestTask> srest;          // solve-step tasks, owner first per panel

    std::vector<Launch> factor_launches;    // in order; the last one inverts the diagonal blocks
    std::vector<DagTask> dag;               // the levels from dag_split_level up as one dependency-ordered task list
    std::int32_t dag_counters = 0;
    std::int32_t dag_min_steps = kDagMinSteps;   // set before build(): 0 puts every level in the task graph
    std::int32_t dag_split_level = 0;       // first level in the task graph
    std::int32_t dag_first_panel = 0;       // first panel (sdiag index) of that level
    std::vector<Launch> pre_dag_launches;   // the levels below, as launches, then their inversions
    double dag_makespan_us = 0.0;           // simulated duration of the scheduled list (schedule.cpp)
    std::vector<Launch> lower_launches;     // forward solve U^T y = b
    std::vector<Launch> upper_launches;     // back solve U x = y

    // Super-panel solve (see SuperPanel): the launch lists with the large
    // fronts' panel steps replaced by super-panel steps (per level: the other
    // fronts' step launches, then per super-panel step a diag and a rest
    // launch); the inverses are formed by the launches of sinv_launches after
    // the factorization.  Empty lists: no front is large enough.
    bool use_super = true;                  // set before build(): false keeps every front on panel steps
    std::vector<SuperPanel> spanels;
    std::vector<SuperInvTask> sinv;
    std::vector<Launch> sinv_launches;
    std::vector<SuperSolveTask> ssolve;
    std::vector<ExtendPullTask> extend_pull;
    std::vector<ExtendTask> extend_segs;
    std::vector<Launch> lower_launches_sp, upper_launches_sp;
    std::int64_t super_inv_size = 0;        // doubles of all inverses

    // Solve task graph: the levels from solve_split_level up run as one
    // persistent launch per sweep, the levels below as the launches above.
    // A graph task is an srest task; its targets are the panels its rest
    // rows belong to (panel ids relative to solve_first_panel).  Forward:
    // a panel's tasks start once the solve_fwd_expected[p] graph tasks that
    // target it have applied their updates; each task signals its targets.
    // Back: a task starts once every target panel has all of its
    // solve_panel_tasks tasks done; each task signals its own panel.
    std::int32_t solve_split_level = 0;
    std::int32_t solve_default_split = 0;         // first level with kSolveDagMinSteps or more panel steps
    std::int32_t solve_first_panel = 0;
    std::int64_t solve_first_task = 0;
    std::vector<std::int32_t> solve_fwd_order;    // srest indices of the graph in forward order
    std::vector<std::int32_t> solve_bwd_order;    // the same in back-sweep order
    std::vector<std::int64_t> solve_target_ptr;   // per graph task (srest index - solve_first_task), + 1
    std::vector<std::int32_t> solve_targets;
    std::vector<std::int32_t> solve_fwd_expected; // per graph panel
    std::vector<std::int32_t> solve_panel_tasks;  // per graph panel

    double gemm_flops = 0.0;                // useful flops of all GEMM tiles (upper part of diagonal tiles)
    double gemm_tile_flops = 0.0;           // the flops the 64 x 64 tiles execute (full tiles, full depth)
    double factor_flops = 0.0;              // reference supernodes: Sum [n0^3/3 + n0^2 n1 + n0 n1^2]
    double front_flops  = 0.0;              // the same sum over fronts (work actually executed)
    double nnz_u = 0.0;                     // reference supernodes: Sum [n0(n0+1)/2 + n0 n1]
    double front_entries = 0.0;             // the same over fronts

    std::int64_t arena_size() const { return u0_size + u1_size + v_size; }

    void build( const Symbolic & sym );
    template<typename RangeOf, typename RangeCount>
    void build_super( const std::vector<std::vector<std::int32_t>> & front_panels, RangeOf range_of, RangeCount ranges,
                      const std::vector<std::vector<std::int32_t>> & by_level );
    // Fills the solve task graph for the levels from `split` up (levels: none).
    void build_solve_graph( const Symbolic & sym, std::int32_t split );
};

} // namespace tb
