// Device data layout of one 2D evaluation (all arrays live in HBM, owned by
// the context and reused across calls).
//
// Particles are kept in tree (Morton) order as SoA doubles; `perm` maps a
// sorted slot back to the caller's particle index. Cells are level-major and,
// within a level, in Morton order of (ix, iy); every cell covers the
// contiguous particle range [lo, hi) of the sorted arrays. Leaves are listed
// in the same order in `leaf_cells`.
#pragma once

#include "prims.cuh"

namespace vpm {

constexpr int kMaxLevels2D = 31;   // key resolution limit (2 bits per level, 62-bit keys)
constexpr int kList2Cap = 27;      // list 2 of a cell has at most 27 members
constexpr int kList4Cap = 16;      // list 4 (coarser leaves next to the parent) slots
constexpr int kQueueCap = 160;     // BFS queue of TreeCell::intList / extList
constexpr int kListSlot1 = 32;     // fixed slots of list 1 / list 3 per leaf in the one-pass build
constexpr int kListSlot3 = 32;
constexpr int kMaxP = 30;          // largest expansion order

enum CellFlags : uint8_t { CELL_LEAF = 1, CELL_ACTIVE = 2 };

// Geometry record written by the bounding-box kernel (exact IEEE arithmetic,
// treeCell.cpp:1061-1092).
struct Geom2D {
    double minx, maxx, miny, maxy;
    double root;        // rootLength
    double pivx, pivy;  // pivotCoord
    double size_k;      // cell size at the key level
};

// Counts produced on the device by the tree build.
struct TreeInfo2D {
    int level_start[kMaxLevels2D + 3];  // first cell index of each level
    int leaf_start[kMaxLevels2D + 3];   // first leaf index of each level
    int n_cells;
    int n_leaves;
    int depth;           // deepest level holding a cell
    int min_leaf_level;
    int max_leaf_level;
    int l2_irregular;    // 1 when some list-2 decision is not the integer-offset rule (cells so
                         // small that the distance tolerance matters): the per-parent M2L is off
    unsigned long long list1_len, list3_len;     // CSR totals
    unsigned long long p2p_pairs, m2l_pairs, m2p_pairs;
};

struct Tree2D {
    int n;
    int key_levels;       // Lk
    int cap_cells;
    Geom2D* geom;
    TreeInfo2D* info;
    // sorted particles
    uint64_t* key;
    uint32_t* perm;
    double *px, *py, *pq;
    uint8_t* pact;
    uint32_t* actscan;    // n + 1 entries: exclusive prefix of active flags
    // cells
    int32_t *c_lo, *c_hi, *c_src, *c_parent, *c_child0, *c_ix, *c_iy, *c_leafidx;
    uint8_t *c_flags, *c_chmask, *c_level;
    double *c_cx, *c_cy;
    uint64_t* c_code;
    int32_t* leaf_cells;
    // Non-leaf cells in cell order (level-major, Morton within a level; the
    // root first): n_cells - n_leaves entries, or nullptr (not recorded).
    int32_t* nonleaf;
    // Dense lookup grid: dense[reference cell ID] = cell index for levels
    // <= dense_levels (nullptr: none). Entries are never cleared: a lookup
    // accepts an entry only if that cell has the queried level and index.
    int32_t* dense;
    int dense_levels;
    // Grid-barrier counters of the cooperative kernels (M2M levels at 2, L2L
    // levels at 4, particle sort at 6), zeroed with the tickets at the start
    // of every evaluation, each used by one kernel; nullptr: launch level by
    // level.
    unsigned* gbar;
};

// Dense grid levels for n particles: the deepest L <= 13 with 4^(L-4) < n
// (level 13 from n > 262,144: 89.5M entries, 358 MB of the 180 GB HBM, so
// that the cells of every level a tree of that size reaches are found with
// one load).
inline int dense_levels_for(int n) {
    int L = 4;
    while (L < 13 && (1ll << (2 * (L - 3))) < (long long)n) ++L;
    return L;
}
inline long long dense_entries(int levels) { return ((1ll << (2 * (levels + 1))) - 1) / 3; }

// Interaction lists. Lists 2 and 4 are fixed-width per cell; lists 1 and 3 are
// CSR over leaves.
struct Lists2D {
    int32_t* l2_src;     // [cap_cells][27] source cell
    uint8_t* l2_slot;    // [cap_cells][27] offset slot 0..39 of the source
    uint8_t* l2_n;       // [cap_cells]
    int32_t* l4_src;     // [cap_cells][16]
    uint8_t* l4_n;       // [cap_cells]
    uint32_t* l1_cnt;    // [cap_leaves] then CSR offsets (cap_leaves + 1)
    uint32_t* l1_off;
    int32_t* l1_src;     // [cap_l1]
    uint32_t* l3_cnt;
    uint32_t* l3_off;
    int32_t* l3_src;     // [cap_l3]
    // [cap_cells][32] per non-leaf cell P (indexed by P): the list-2 candidates
    // of P's children, child d of P's k-th neighbour (k = 0..7 without P itself,
    // the reference's neighbour order) at entry 4 k + d, or -1 where that cell
    // is missing, inactive or its parent is a leaf or inactive; written by the
    // first child of P. Every list 2 of a child of P is the subset of these
    // entries separated from it (nullptr: not recorded).
    int32_t* l2_blk;
    int32_t* l1_slot;    // [cap_leaves][kListSlot1] one-pass staging of list 1 (nullptr: two passes)
    int32_t* l3_slot;    // [cap_leaves][kListSlot3]
    int cap_leaves;
    long long cap_l1, cap_l3;
};

// Where a near-field kernel reads list 1 from: the CSR, the fixed slots of the
// one-pass build (leaves with more entries than kListSlot1 skipped), or the
// CSR for exactly those leaves.
constexpr int kP2PListCsr = 0, kP2PListSlots = 1, kP2PListSpill = 2;

// Scratch of the tree build.
constexpr int kBBoxBlocks = 296;
constexpr int kFlatTile = 256;   // particles per block of the flat tree build
constexpr int kTicketWords = kMaxLevels2D + 2 + 8;  // level tickets, bbox counter, 3 x 2 barrier words
constexpr int kBarrierWordsAt = kMaxLevels2D + 2;

// Cooperative sort (one launch for bounding box, keys, radix passes, gather
// and active scan): at most kCoopSortGridMax blocks of kCoopSortMaxChunk
// particles; larger inputs take the multi-kernel path.
constexpr int kCoopSortGridMax = 160;
constexpr int kCoopSortMaxChunk = 16384;
constexpr int kCoopSortWords = 1024 * kCoopSortGridMax + 544;

struct TreeScratch2D {
    double* bbox_partial;   // [kBBoxBlocks * 4]
    uint64_t* key_alt;
    uint32_t* val_alt;
    uint32_t* act_u32;
    unsigned* lvl_ticket;   // [kTicketWords]: bbox counter at kMaxLevels2D + 1, then the grid-barrier words
    uint32_t* pinfo;        // [n] per sorted particle: level it starts a group at, big-level + 1, cell levels
    uint32_t* tile_cnt;     // [2][kMaxLevels2D + 1][flat_tiles] cells / leaves per tile and level, then offsets
    uint32_t* level_tot;    // [2][kMaxLevels2D + 1] cells / leaves per level
    int flat_tiles;         // tiles of kFlatTile particles
    uint32_t* coop_words;   // [kCoopSortWords] count tables of the cooperative sort (nullptr: multi-kernel sort)
    SortScratch sort;
    ScanScratch scan;
};

// Tree build: bounding box through level splits. All launches are enqueued on
// `st`; nothing is read back. Returns the number of launches in *launches.
cudaError_t build_tree2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                         TreeScratch2D& s, int max_src, int max_par, double exp_pct, unsigned* err, cudaStream_t st,
                         int* launches);

// The two halves of build_tree2d: bounding box, keys, sort, gather and the
// active-count scan; then the level-by-level cell construction.
// shallow_cap = min(max_src, max_par): lets the cooperative sort try three
// radix passes first (see sort2d_coop); 0 always sorts the full keys.
// q = null sorts without the strengths: t.pq is then left for
// gather_strengths2d, so that the strengths can still be in flight from the
// host while the tree and the lists are built.
// items_per_block: particles per block of the cooperative sort (a solve with
// the GPU to itself spreads over as many SMs as it can fill; solves sharing
// the GPU in a batch take fewer, fuller blocks so that several sorts fit at
// once).
cudaError_t keys_sort2d(const double* x, const double* y, const double* q, const uint8_t* act, Tree2D& t,
                        TreeScratch2D& s, double exp_pct, unsigned* err, cudaStream_t st, int* launches,
                        int shallow_cap = 0, int items_per_block = 1024);
// t.pq[i] = q[t.perm[i]] for i < t.n.
cudaError_t gather_strengths2d(const Tree2D& t, const double* q, unsigned* err, cudaStream_t st, int* launches);
cudaError_t levels2d(Tree2D& t, TreeScratch2D& s, int max_src, int max_par, unsigned* err, cudaStream_t st,
                     int* launches);

// Lists 2 and 4 (fixed width), and lists 1 and 3 (count, scan, fill); the two
// are independent of each other.
cudaError_t build_ext_lists2d(const Tree2D& t, Lists2D& l, double eps, unsigned* err, cudaStream_t st,
                              int* launches);
cudaError_t build_int_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                              cudaStream_t st, int* launches);
// The two halves of build_int_lists2d with fixed slots (l.l1_slot, l.l3_slot):
// counts and the first kListSlot1 / kListSlot3 entries of every leaf; then
// the CSR (scans, compaction, the leaves that outgrew their slots, totals).
bool int_lists_slotted(const Lists2D& l);
cudaError_t build_int_slots2d(const Tree2D& t, Lists2D& l, double eps, unsigned* err, cudaStream_t st, int* launches);
cudaError_t build_int_csr2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                            cudaStream_t st, int* launches);
// Lists 1-4 (count, scan, fill). Requires the tree on `st`.
cudaError_t build_lists2d(const Tree2D& t, Lists2D& l, ScanScratch& scan, double eps, unsigned* err,
                          cudaStream_t st, int* launches);

// Translation coefficients for order P, three (kMaxP+1)^2 tables of doubles
// in device memory owned by the caller (each context keeps its own):
//   m2m[p][k] = C(p-1,k-1) * (p/k)                (fmm2D.cpp:372-374)
//   m2l[p][k] = C(p+k-1,k-1) * (-1)^k / k         (fmm2D.cpp:477-479)
//   l2l[p][k] = C(k,p)                            (fmm2D.cpp:640-641)
// with C from the reference's 32-bit binComb or exact. The upload
// synchronises `st` (the host table is temporary).
constexpr int kCoefTable = (kMaxP + 1) * (kMaxP + 1);
constexpr int kCoefM2M = 0, kCoefM2L = kCoefTable, kCoefL2L = 2 * kCoefTable;
cudaError_t set_coefficients2d(int P, bool exact_binom, double* dst, cudaStream_t st);
cudaError_t set_m2l_operators2d(int P, bool exact_binom, double2* dst, cudaStream_t st);

// FP64 evaluation (plain form): P2M+M2M, M2L, L2L chain + M2P + L2P, P2P.
// ex/ey are written in the caller's particle order.
struct Expansions2D {
    double2* a;          // [cap_cells][P+1] multipole
    double2* b;          // [cap_cells][P+1] local (M2L part only)
    unsigned* up_count;  // [cap_cells] children completed (upward pass)
    double* coef;        // [3 * kCoefTable] translation coefficients
    double2* op;         // [49][P+1][P] list-2 M2L operators, or nullptr (direct formula)
    double* fx;          // [n] far-field Ex in sorted order
    double* fy;
};

cudaError_t fmm2d_upward(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches);
// The same moments in two launches (cells of up to 1024 particles straight
// from their particles, the larger ones by a cooperative M2M level loop from
// the deepest level holding one) when upward_direct_ok; else fmm2d_upward.
// Uses grid-barrier words 2 and 3 of t.gbar (zeroed before every evaluation).
bool upward_direct_ok(int P, bool exact);
// mid (may be null): recorded on st once every cell's moments except those of
// the cells left to the M2M loop are final (at the end when there is no loop).
cudaError_t fmm2d_upward_direct(const Tree2D& t, Expansions2D& e, int P, bool exact, unsigned* err, cudaStream_t st,
                                int* launches, cudaEvent_t mid = nullptr);
cudaError_t fmm2d_m2l(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                      int* launches);  // M2L followed by the L2L levels
// Potential (fmm2D::calcPotential): b_0 of the M2L after fmm2d_m2l_only, then
// after the L2L levels the far-field and list-1 potential into out (caller order).
cudaError_t fmm2d_m2l_b0(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                         int* launches);
cudaError_t fmm2d_potential_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, double* out,
                                 unsigned* err, cudaStream_t st, int* launches);
// Leaves' full local expansions straight from their ancestors' M2L parts
// (replaces the level-by-level L2L when l2l_direct_ok: exact binomials up to
// order P).
bool l2l_direct_ok(int P, bool exact);
cudaError_t fmm2d_l2l_leaves(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches);
// List-2 M2L of the mixed form per parent (m2l_tc.cu, m2l_parent_tc): one
// tensor-core product over all non-leaf cells, orders 1..16; list 4 in FP64.
bool m2l_parent_supported(int P);
// The same per-parent list-2 M2L on the FP32 pipes through the operator's
// diagonal-real-diagonal structure (m2l_parent_f32), orders 1..16; list 4 in
// FP64.
// part 0: every parent, then list 4 (fmm2d_m2l_list4); part 1: the parents
// at levels >= the deepest level holding a cell moved by the M2M loop (their
// children's sources are final once upward_direct2d is done); part 2: the
// other parents. Parts 1 and 2 leave list 4 to the caller, after both.
bool m2l_parent_f32_supported(int P);
cudaError_t fmm2d_m2l_parent_f32(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, bool exact,
                                 unsigned* err, cudaStream_t st, int* launches, int part = 0);
// List 4 (and list 2 of an irregular tree) added to b in FP64.
cudaError_t fmm2d_m2l_list4(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                            int* launches);
cudaError_t set_m2l_parent_operators(int P, const double2* op_dev, float* dst, cudaStream_t st);
cudaError_t fmm2d_m2l_parent(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, float* rows,
                             const float* ops, unsigned* err, cudaStream_t st, int* launches);
bool m2l_tc_supported(int P);
size_t m2l_tc_rows_bytes(int cap_cells);
size_t m2l_tc_ops_bytes();
cudaError_t set_m2l_tc_operators(int P, const double2* op_dev, float* dst, cudaStream_t st);
cudaError_t fmm2d_m2l_tc(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, float* rows, const float* ops,
                         unsigned* err, cudaStream_t st, int* launches);
cudaError_t fmm2d_m2l_only(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err,
                           cudaStream_t st, int* launches);
cudaError_t fmm2d_l2l(const Tree2D& t, Expansions2D& e, int P, unsigned* err, cudaStream_t st, int* launches);
cudaError_t fmm2d_eval(const Tree2D& t, const Lists2D& l, Expansions2D& e, int P, unsigned* err, cudaStream_t st,
                       int* launches);
cudaError_t fmm2d_p2p(const Tree2D& t, const Lists2D& l, const Expansions2D& e, double* ex, double* ey,
                      unsigned* err, cudaStream_t st, int* launches);

}  // namespace vpm
