// Host-side symbolic analysis for the GPU multifrontal Cholesky.
//
// Replaces the analysis half of the reference's solver call (MKL PARDISO phase 12,
// CalcNonstat3DLine/pardiso.cpp:69-111).  The ordering is a nested dissection:
// coordinate bisection with one-sided vertex separators when unknown positions
// are known (edge midpoints of the tensor-product mesh: the separators are then
// exactly the in-plane edges of one node plane), breadth-first level-set
// bisection otherwise.  The dissection tree is the assembly tree: every leaf
// block and every separator becomes one front whose pivot columns are
// contiguous in the new numbering.
//
// Everything the numeric phase needs on the device is flattened here:
//   * front offsets / sizes, entry map (matrix value -> front slot),
//   * child -> parent relative row maps for extend-add,
//   * per-level, per-panel task lists for the batched dense kernels,
//   * per-front row index lists for the triangular solves.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace tdem {

constexpr int kPanel = 64;       // dense panel width of the factorization and solves
constexpr int kOuter = 512;      // outer panel width: trailing updates of rank up to kOuter
constexpr int kTileSyrk = 64;    // tile edge of the update inside an outer panel
constexpr int kTileBig = 128;    // tile edge of the rank-kOuter trailing update
constexpr int kTrsmRows = 128;   // rows per CTA of the panel triangular solve
constexpr int kSolveRows = 256;  // rows per CTA of the solve updates
constexpr int kSolveChunk = 8;   // 64 x 64 blocks accumulated by one level-solve unit
constexpr int kUnitInts = 16;    // ints per level-solve unit record (64 bytes)
constexpr int kSolveLookahead = 8;  // extra blocks a chain unit takes ahead of its newest one
// Trailing updates on the integer tensor pipe (FP64 by the Ozaki splitting): each
// row of the outer panel is split into kOzSlices signed 7-bit digits after scaling
// by a power of two; only launches whose panels total at most kOzRowsCap rows (the
// slice buffer) and at least kOzMinFlops flops take that path.
constexpr int kOzSlices = 8;
constexpr int kOzK = kOuter;          // digits per row and slice (K of an outer panel, padded)
constexpr int64_t kOzRowsCap = 1 << 19;
constexpr double kOzMinFlops = 2e9;
// most blocks one level-solve unit accumulates (a chain unit, or a short row)
constexpr int kUnitBlocks = (kSolveLookahead + 1 > kSolveChunk + 1) ? kSolveLookahead + 1 : kSolveChunk + 1;

struct FrontInfo {
  int c0 = 0, c1 = 0;      // pivot columns [c0, c1) (permuted numbering)
  int parent = -1;
  int level = 0;           // height in the assembly tree (leaves = 0)
  std::vector<int> rows;   // rows below the pivot block (permuted, sorted)
  std::vector<int> children;
  int m() const { return (c1 - c0) + (int)rows.size(); }
  int k() const { return c1 - c0; }
};

// One batched launch: a list of fronts and the CTA prefix over them.
struct TaskList {
  int64_t off = 0;     // offset (in ints) into Symbolic::tasks of the front list
  int64_t pre = 0;     // offset (in int64) into Symbolic::task_prefix (count+1 entries)
  int count = 0;       // number of fronts
  int64_t ctas = 0;    // total CTAs
};

// One 64-wide inner panel [j0, j1) of the factorization, j1 = min(k, j0 + 64).  The
// outer panel is [J0, J1), J0 = floor(j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter).
struct PanelStep {
  int j0 = 0;          // panel start (fronts with k > j0 take part)
  TaskList potrf;      // one CTA per front
  TaskList trsm;       // ceil((m - j1) / kTrsmRows) CTAs per front
  TaskList syrk;       // update of columns [j1, J1) (rows >= j1) by the inner panel, 64-tiles
  TaskList syrk_wide;  // the same update in 128-row x 64-column tiles (FP64 tensor-pipe kernel)
  // syrk_wide split for the look-ahead: the column tile of the next inner panel
  // [j1, j1 + 64) (syrk_next) and the tiles right of it (syrk_rest)
  TaskList syrk_next, syrk_rest;
  TaskList syrk_big;   // at the end of an outer panel: trailing [J1, m) by [J0, J1), 128-tiles
  // Ozaki path of syrk_big (ozaki true): the panel rows [J1, m) of every front of
  // syrk_big are split into digits, front after front (task_aux of the syrk_big
  // entries: the front's first row in the slice buffer), by oz_slice (64 rows per CTA)
  bool ozaki = false;
  int64_t oz_rows = 0;
  TaskList oz_slice;
  TaskList solve_upd;  // ceil((m - j1) / kSolveRows) CTAs per front (fwd update / bwd partials)
};

struct LevelPlan {
  std::vector<int> fronts;             // fronts at this height
  std::vector<TaskList> extend_slots;  // extend-add launches (one per child slot), 8 columns per CTA
  std::vector<TaskList> extend_vec;    // solve extend-add per child slot, kSolveRows rows per CTA
  TaskList assemble;                   // solve: front-vector init, ceil(m / kSolveRows) CTAs each
  std::vector<PanelStep> panels;
  // Level triangular solves: units (kUnitInts ints each, see Symbolic::solve_units)
  // at solve_units[kUnitInts * off ...], taken by CTAs in list (ticket) order.
  // Units are sorted by the last pivot block they wait for, so every unit a CTA
  // waits for has a smaller ticket.
  int64_t fwd_off = 0, fwd_count = 0;
  int64_t bwd_off = 0, bwd_count = 0;
};

struct Symbolic {
  int n = 0;                  // unknowns
  int64_t nnz_lower = 0;      // entries of the analysed lower triangle (incl. diagonal)
  std::vector<int> perm;      // perm[old] = new
  std::vector<int> iperm;     // iperm[new] = old
  std::vector<FrontInfo> fronts;
  std::vector<LevelPlan> levels;

  // device-bound flat arrays.  A front is stored split: its pivot columns (m x k,
  // leading dimension m) live in the persistent factor L at l_off; its update
  // block (r x r, r = m - k, leading dimension r) lives in the update workspace
  // at u_off from the level it is factored until its parent has assembled it.
  std::vector<int64_t> l_off;        // offset of each front's m x k block in L
  std::vector<int64_t> u_off;        // offset of each front's r x r block in the workspace
  std::vector<int> front_m, front_k, front_c0, front_parent;
  std::vector<int64_t> entry_dst;    // lower-CSR entry q -> offset in L
  std::vector<int64_t> rel_off;      // per front: offset of its rel map (rows -> parent slot)
  std::vector<int> rel;              // concatenated rel maps
  std::vector<int64_t> rows_off;     // per front: offset of its full row list (k + r entries)
  std::vector<int> rows_all;         // concatenated [c0..c1) U rows, permuted numbering
  std::vector<int64_t> wvec_off;     // per front: offset of its m-long solve vector
  std::vector<int> tasks;            // concatenated task front lists
  std::vector<int64_t> task_aux;     // per task entry: launch-specific value (see PanelStep)
  std::vector<int64_t> task_prefix;  // concatenated CTA prefix sums

  std::vector<int> solve_items;      // (front, block) pairs of the diagonal-block inversions
  // level-solve units, kUnitInts ints each: {row/column block, lo, hi, partial
  // slot, row counter, partials to add (final unit), final flag, m, k, first
  // pivot-block flag of the front, l_off, w_off, dinv_off (int64 as lo/hi ints)};
  // w_off is also the front's offset into rows_all
  std::vector<int> solve_units;
  int64_t n_counters = 0;            // row counters over all levels and both directions
  int64_t solve_slots = 0;           // partial-sum slots (64 x nrhs each) of the largest level
  std::vector<int64_t> flag_off;     // per front: index of its first pivot-block flag
  std::vector<int64_t> dinv_off;     // per front: offset of its inverted diagonal blocks
  int64_t n_flags = 0;               // pivot blocks over all fronts
  int64_t dinv_elems = 0;            // sum over pivot blocks of w^2 (w = block width)
  int64_t inv_off = 0, inv_count = 0;  // items of the diagonal-block inversion (all pivot blocks)

  int64_t u_elems = 0;        // peak update-workspace size (elements)
  int64_t u_sum = 0;          // sum of r^2 (workspace without reuse)
  int64_t wvec_elems = 0;     // sum of m
  int64_t nnz_l = 0;          // sum of m*k (stored factor entries incl. diagonal blocks)
  double flops = 0.0;         // factorization flops
  double oz_flops = 0.0;      // flops of the trailing updates on the Ozaki path
  double oz_macs = 0.0;       // 8-bit multiply-adds those updates issue on the tensor pipe
  int64_t oz_rows_max = 0;    // slice-buffer rows the Ozaki path needs
  int max_m = 0, max_k = 0;
  int64_t solve_partials = 0; // scratch entries per RHS column for backward partial sums
};

// FNV-1a hash of the ordering, the fronts' columns and rows, the entry map and the
// level-solve units (equal hashes: identical factorization and solve launches)
uint64_t plan_digest(const Symbolic& sy);

// Analyse the lower triangle (row i holds columns j <= i, diagonal included)
// of a symmetric n x n matrix.  coords (n x 3) are optional unknown positions.
// Returns an empty string on success, an error message otherwise.
// adj_ptr/adj (optional): the same matrix's symmetric adjacency without the diagonal,
// each row ascending (n + 1 row starts); when given it is used instead of being built
// from the lower triangle, and the result is the same.
std::string analyse(int n, const int64_t* rowptr, const int* colind, const double* coords,
                    Symbolic& out, int leaf_size = 128, const int64_t* adj_ptr = nullptr,
                    const int* adj = nullptr);

}  // namespace tdem
