// spgemm.cuh -- host-side entry points shared by the SpGEMM forms.
#pragma once

#include "spgemm_kernels.cuh"

namespace clb {

int validate_spgemm(const clb_dcsr &A, const clb_dcsr &B);
// Builds B's dense row map when worthwhile and fills the row view.
int prepare_b(clb_controls *ctl, const clb_dcsr &B, Temp<uint64_t> &dense, BRows &b);
// B's rows as word runs for the bitmap insertion: built when b has the dense
// row map, B has at least B_WORDS_MIN_NNZ entries and (hinfo, rows per bin,
// when given) some row is in a bitmap bin; otherwise b is left as it is.
// products (when known, else 0): the product's total; the runs are skipped
// when B's entries are read fewer than B_WORDS_MIN_REUSE times on average.
constexpr uint64_t B_WORDS_MIN_NNZ = 1ull << 16;
constexpr uint64_t B_WORDS_MIN_REUSE = 4;
int prepare_b_words(clb_controls *ctl, const clb_dcsr &B, const uint32_t *hinfo, Temp<uint64_t> &wdense,
                    Temp<uint2> &wpairs, BRows &b, uint64_t products = 0);
// work[i] = products of A row i; *d_total += their sum.
int launch_workload(clb_controls *ctl, const AView &a, const BRows &b, uint32_t *work, uint64_t *d_total);
// Histogram + scatter of the rows into accumulator bins.  The bound of
// distinct columns is cap[i] when cap is non-null, else min(work[i], ncols).
// flags[i] = 1 for rows with products (input of the C row-position scan).
int launch_binning(clb_controls *ctl, const uint32_t *work, const uint32_t *cap, uint64_t n, uint64_t ncols,
                   uint32_t *info, uint32_t *list, uint32_t *flags, const Tuning &t = Tuning());
// Runs every bin's accumulator kernel (symbolic or numeric).  bin_rows
// (host, optional): rows per bin; empty bins are then skipped.
int launch_accumulators(clb_controls *ctl, bool numeric, const BinLists &bl, const AView &a, const BRows &b,
                        const RowOut &o, uint64_t ncols, uint64_t nrows_max, const Tuning &t = Tuning(),
                        const uint32_t *bin_rows = nullptr);
// C.rpt/C.rows from the row flags' exclusive scan (pos) and the row offsets.
int launch_assemble(clb_controls *ctl, const uint32_t *work, const uint32_t *pos, const uint64_t *off,
                    const uint32_t *a_rows, uint64_t n, uint64_t *c_rpt, uint32_t *c_rows, uint64_t nzr, uint64_t nnz);
// Deferred bitmap rows (RowOut::defer; at most nmax of them): bitmaps from
// their slots, columns to ccols + off[i].
int launch_bitmap_expand(clb_controls *ctl, const uint32_t *list, const uint32_t *count, uint64_t nmax,
                         const uint64_t *slot_off, const uint32_t *slots, const uint64_t *off,
                         const uint32_t *row_ncols, uint64_t ncols, uint32_t *ccols);
// The same by step, from the deferred rows' step records (RowOut::defer_steps).
int launch_bitmap_expand_steps(clb_controls *ctl, const uint32_t *list, const uint32_t *count, const uint32_t *steps,
                               const uint64_t *slot_off, const uint32_t *slots, const uint64_t *off,
                               uint32_t *ccols);
// Numeric accumulators without (hash_bins = false) the hash bins.
int launch_accumulators_subset(clb_controls *ctl, const BinLists &bl, const AView &a, const BRows &b,
                               const RowOut &o, uint64_t ncols, uint64_t nmax, bool hash_bins,
                               const Tuning &t = Tuning(), const uint32_t *bin_rows = nullptr,
                               bool bitmap_bins = true);
// Single-pass forms (spgemm_single.cu): capacity slots, one numeric pass,
// exact fallback for rows that outgrew their capacity, compaction.
int spgemm_single_pass(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const AView &a, const BRows &b,
                       const uint32_t *work, uint32_t *cap, bool esc, uint64_t products, clb_dcsr *out,
                       clb_spgemm_stats *st, uint64_t arena_div, const Tuning &t = Tuning());
// Per-row pair context of a stacked batch (the learned form's row features
// are relative to each row's own pair): row_pair[i] = pair of stacked row i,
// pairs[k] = that pair's first row id in the stack, its rows and the density
// feature of its right operand.
struct PairFeat {
    uint32_t row0;
    uint32_t nrows;
    float density;
    uint32_t pad;
};
struct BatchRows {
    const uint32_t *row_pair = nullptr;
    const PairFeat *pairs = nullptr;
};
// log2(B.nrows * B.ncols / nnz(B)) / 16: the density feature of a right operand.
float learned_density_feature(const clb_dcsr &B);
// Learned capacities (mlp.cu): work[i] = products of A row i and cap[i] =
// its slot (predicted for rows over t.bitmap_min products, exact below;
// never above min(work, the row's columns)); batch = per-row pair context
// of a stacked batch, or null.
// defer: the caller keeps the bitmaps of dense enough bitmap rows in their
// slots (RowOut::defer), so those rows get room for their bitmap.
int learned_caps(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const AView &a, const BRows &b,
                 const clb_sizer *sizer, float margin_log2, float slack, const Tuning &t, const BatchRows *batch,
                 uint32_t *work, uint32_t *cap, bool defer = false);
// The learned single pass: learned capacities, one numeric pass with the
// spill arena, exact fallback of the rows that outgrew both, compaction.
int spgemm_learned(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const clb_sizer *sizer,
                   float margin_log2, float slack, const Tuning &t, const BatchRows *batch, clb_dcsr *c,
                   clb_spgemm_stats *st);
// Learned sizing of the host-sync-free form: capacities from the predictor
// and a spill arena of arena_capacity entries for the rows that outgrow them.
struct CaptureLearned {
    const clb_sizer *sizer;
    float margin_log2, slack;
    BatchRows batch;
    uint64_t arena_capacity;
};
// Flags of the host-sync-free form (bits of its device flag word).
constexpr uint32_t CAPTURE_SLOTS_FULL = 1u;    // slot capacity too small: rows left empty
constexpr uint32_t CAPTURE_COLS_FULL = 2u;     // column capacity too small: rows not written
constexpr uint32_t CAPTURE_DEVICE_CHECK = 4u;  // an accumulator's device check failed
constexpr uint32_t CAPTURE_ROW_OVERFLOW = 8u;  // a row outgrew its learned slot and the arena: left empty
// The ESC single pass with every size from the caller and no host read:
// slots (slot_capacity entries) and the stream-ordered temporaries are
// allocated on ctl's stream, C goes to the caller's arrays (rpt: A.nzr + 1,
// rows: A.nzr, cols: cols_capacity), d_result[0..1] = nzr, nnz and
// d_result[2..] = per-pair row and column bounds (first[k] = first stacked
// row of pair k, row_base[k] = its row-id offset, both on the device).
int spgemm_esc_capture(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const Tuning &t,
                       uint64_t slot_capacity, const uint64_t *first, const uint32_t *row_base, uint32_t count,
                       uint64_t *c_rpt, uint32_t *c_rows, uint32_t *c_cols, uint64_t cols_capacity,
                       uint64_t *d_result, uint32_t *d_flags, const CaptureLearned *learned = nullptr);
// cap[i] = min(work[i], ncols): the exact upper bound of a row's count.
int launch_upper_bound_caps(clb_controls *ctl, const uint32_t *work, uint64_t n, uint64_t ncols, uint32_t *cap);
// Public tuning struct -> internal tuning (zero fields: defaults), and its check.
Tuning to_tuning(const clb_spgemm_tuning *t);
int check_tuning(const clb_spgemm_tuning *t);
// keep: the symbolic pass keeps the bitmap rows' bitmaps (128 KB a row at 2^20
// columns) for the numeric pass, which expands them instead of inserting
// their products again; without room for them (or for rows wider than one
// bitmap chunk) the plain form runs.
int spgemm_hash_two_pass(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, clb_dcsr *out,
                         clb_spgemm_stats *stats, const Tuning &t = Tuning(), bool keep = false);

}  // namespace clb
