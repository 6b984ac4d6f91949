// Internal host-side interface between the C ABI (fap_capi.cu) and the
// kernel launchers (fap_device.cu).  Not installed.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fapb {

// One part of a solve batch.  All offsets are in elements.
struct PartDesc {
  int32_t part;      // 1-based part id
  int32_t start;     // first sorted position of the part
  int32_t s;         // vertices in the part
  int32_t b;         // boundary vertices (sorted first)
  int64_t row_base;  // first output row of the part's block
  int64_t f_off;     // offset of the part's padded Floyd matrix in the F arena
  int32_t ldf;       // padded Floyd leading dimension (multiple of kFloydTile)
  int32_t bd_row;    // first row of the part's boundary rows in the resident cache /
                     // boundary index space (prefix sum of the boundary counts)
  int32_t flags;     // kPartLocal
  int32_t bd_col;    // first column of the part's boundary vertices in dB when its
                     // columns are padded per part to 16-byte starts (Bellman-Ford closure)
};

// PartDesc::flags.  kPartLocal: the Floyd matrix is built from the part's
// own edges only (boundary rows included), i.e. the local closure (the
// boundary-graph form of stage 1).
constexpr int32_t kPartLocal = 1;

// Per part id (1..K) for the boundary-graph expansion.
struct BPart {
  int32_t voff;   // first sorted position
  int32_t b;      // boundary count
  int32_t boff;   // first index in the boundary index space
  int32_t ldf;    // Floyd leading dimension
  int64_t f_off;  // the part's local closure in the Floyd arena
};

// Rows-from-cache work: up to kRowsGroup output rows of one part.
constexpr int kRowsGroup = 16;
struct RowGroup {
  int32_t pidx;   // index into the cache's part descriptors
  int32_t first;  // first entry of the group in the row lists
  int32_t count;  // rows in the group (<= kRowsGroup)
  int32_t pad_;
};

// One min-plus work row: BM output rows of one part (index into the batch).
struct MPWork {
  int32_t pidx;
  int32_t m0;
};

// Packed 16-bit min-plus of one batch (int32 distances): per batch part
// (index pidx) and column, the least finite entry of its boundary rows in D
// (off); per column tile of kMinplusBN columns the largest finite entry minus
// its column's off (range); per part the largest finite A = F[b+i][k]
// (maxA).  A tile runs packed when maxA + range < kPackCap, otherwise in
// int32.  Buffers: off [nparts][ldD], range [nparts][ntiles], maxA [nparts].
// Optional pre-packed operands (s16 null: every packed tile converts its
// stages in shared memory): s16 [rows][ldD] uint16 holds the boundary rows
// of D shifted by off and clamped at kPackCap, at [rows][at_ld] uint32 the
// inner-to-boundary distances F[b+i][k] clamped at kPackCap in both halves,
// k-major (column i); part pidx's boundary vertex k is row krow[pidx] + k of
// both (krow < 0: the part has no work).
struct Pack16 {
  int32_t *off;
  int32_t *range;
  int32_t *maxA;
  int32_t ntiles;
  unsigned long long *tiles;  // [2]: tiles run packed, tiles run (cumulative)
  uint16_t *s16;
  uint32_t *at;
  const int32_t *krow;
  int32_t at_ld;
  int32_t max_b;              // largest boundary count of the work's parts
  int64_t prows;              // rows of s16 and at
};

// Packed 16-bit form of the tiled expansion of the boundary graph (int32):
// per part q (index in the launch's part list) and boundary index g, off =
// the least finite dB[g][b'] over q's boundary columns b'; per (q, 128-row
// tile of dB) the largest finite dB[g][b'] - off (range); per part the
// largest finite F_q[b'][v], b' < b_q, v < s_q (maxB).  A tile runs packed
// when range + maxB < kPackCap (rows shifted by off, see tma_minplus_tile16).
struct Expand16 {
  int32_t *off;     // [nparts][nbB]
  int32_t *range;   // [nparts][nrt]
  int32_t *maxB;    // [nparts]
  int32_t nrt;      // 128-row tiles of dB
  unsigned long long *tiles;  // [2]: tiles run packed, tiles run (cumulative)
  // Optional operands packed beforehand (ap null: every packed tile converts
  // its stages in shared memory).  ap [rows][ap_ld] words: the dB rows at
  // part q's boundary columns, shifted by off and clamped at kPackCap, two
  // rows a word (row 2p in the low half), k-major: word p of row bd_row + k.
  // bd [rows][bd_ld] words: F_q[k][v] clamped at kPackCap in both halves,
  // row bd_row + k, column v (kPackCap past the part's s columns).
  uint32_t *ap;
  uint32_t *bd;
  int32_t ap_ld, bd_ld, max_b;
  int64_t rows;
};

// Work queue of the batched Floyd-Warshall in one persistent launch: items
// 0..nitems-1 are listed (kind, batch index, pivot block, tile) so that
// every item's dependencies come earlier in the list, and CTAs claim them in
// list order from a counter; a CTA waits (bounded) for the per-part
// counters its item depends on.  When the batch's min-plus merge follows the
// Floyd directly (stage 1 by SSSP), the boundary-row scatter of each part and
// the min-plus tiles (mp_work x column tiles, after the listed items) are in
// the same launch, each part's starting as soon as its own closure is done.
struct QItem {
  int32_t kind;  // kQFloyd1..3, kQScatter
  int32_t pidx;  // batch index of the part
  int32_t kb;    // pivot block (Floyd) / first boundary row / kQScatterRows (scatter)
  int32_t t;     // tile index within the phase
};
constexpr int32_t kQFloyd1 = 1, kQFloyd2 = 2, kQFloyd3 = 3, kQScatter = 4;
// Symmetric matrices: the row-panel tile (kb, j) and the remainder tile
// (i, j), i <= j, each also storing its transpose; t = i << 16 | j.
constexpr int32_t kQFloyd2S = 5, kQFloyd3S = 6;
constexpr int kQScatterRows = 8;
struct FloydQueue {
  const QItem *items;
  int32_t nitems;
  int32_t mp_work;   // min-plus work items (MPWork) appended after the list (0: none)
  int32_t *cnt;      // per batch part `stride` counters, then the abort flag and the claim counter
  int32_t stride;    // 2 + 2 * max_nb: Floyd-1 rounds done, scatter items done, then per pivot
                     // block the Floyd-2 and the Floyd-3 items done
  int32_t nparts;
  int32_t sym;       // the Floyd items are the symmetric kinds
};

constexpr int kFloydTile = 128;
constexpr int kMinplusBM = 128;
constexpr int kMinplusBN = 128;
constexpr int kLdAlign = 128;  // output leading dimension multiple (= kMinplusBN)

// Launchers.  T is int32_t or float.  All asynchronous on `stream`; each
// returns the cudaError_t of its launch(es) and adds the number of kernel
// launches it issued to *launches.
// Stage 1.  row_offset/col/w/sources are in work space; with perm_out
// (original vertex -> work id) the CTAs compute in `scratch` (sssp_scratch_rows
// rows of n) and write out[v] = dist[perm_out[v]].
template <typename T>
cudaError_t launch_sssp(const int32_t *row_offset, const int32_t *col, const T *w, int n,
                        const int32_t *sources, const int64_t *out_rows, int num_sources, T *out,
                        int64_t ld, int64_t init_cols, const int32_t *perm_out, T *scratch,
                        T delta, int chain, int precheck, int64_t max_rounds, int *status,
                        cudaStream_t stream, int64_t *launches);

// Tiled form of stage 1 (multi-source Bellman-Ford over in-edges, kMsbfS
// sources per tile; see fap_device.cu).  items: the work list, one entry
// per vertex and chunk of up to 32 in-edges (tro/tcol/tw, original ids);
// sources are sorted positions (st2ed maps them to vertices); row s of the
// output is out_rows[s] (original column order, init_cols columns).  With
// sources == nullptr the sources are the work graph's vertices 0..num-1, and
// with out_rows == nullptr source s goes to row s.  ztiles tiles run side
// by side: Dt holds ztiles x n x kMsbfS values, act 2 x ztiles x ceil(n/32)
// words, changed 4 ints on the
// device and host_changed 4 ints on the host (the launcher synchronises the
// stream every 4 iterations to test convergence).
constexpr int kMsbfS = 128;
constexpr int kMsbfRoundLimit = 1;  // = kDevSsspRoundLimit
struct MsbfItem {
  int32_t v;
  int32_t e0;
};
template <typename T>
cudaError_t launch_msbf(const MsbfItem *items, int nitems, const int32_t *tro, const int32_t *tcol, const T *tw,
                        int n, const int32_t *st2ed, const int32_t *sources, const int64_t *out_rows,
                        int num_sources, T *out, int64_t ld, int64_t init_cols, int ztiles, T *Dt, uint32_t *act,
                        int *changed, int *host_changed, int64_t max_rounds, int *status, cudaStream_t stream,
                        int64_t *launches);

// Rows of scratch the relabelled SSSP needs (= CTAs it launches) for
// num_sources sources on this device.
int sssp_scratch_rows(int n, int num_sources);

template <typename T>
cudaError_t launch_gather(const PartDesc *parts, int nparts, int max_ldf, const int32_t *row_offset,
                          const int32_t *col, const T *w, const int32_t *graph_id,
                          const int32_t *st2ed, const int32_t *ed2st, const T *D, int64_t ldD,
                          T *F, cudaStream_t stream, int64_t *launches);

// The Floyd arena F holds the batch's parts as equal padded squares of
// leading dimension ld (a multiple of kFloydTile), part i at i * ld * ld.

// Batched: one CTA per part closes its matrix and writes its boundary rows'
// own-part columns back into D.
template <typename T>
cudaError_t launch_floyd_parts(const PartDesc *parts, int nparts, T *F, int64_t ld, T *D,
                               int64_t ldD, const int32_t *st2ed, int *status, cudaStream_t stream,
                               int64_t *launches);

// Batched, multi-launch: every part's pivot round in three launches
// (3 x max_nb launches in all); no boundary-row decode.
template <typename T>
cudaError_t launch_floyd_parts_multi(const PartDesc *parts, int nparts, int max_nb, T *F, int64_t ld,
                                     int *status, cudaStream_t stream, int64_t *launches);

// Plain: one padded matrix (ld a multiple of kFloydTile, nb tiles per side
// in use), one launch per phase per pivot block.  status may be null.  s:
// the real rows and columns (the rest is padding holding the sentinel,
// whose pivots and tile halves are skipped); -1 = all of the nb tiles.
template <typename T>
cudaError_t launch_floyd_matrix(T *mat, int64_t ld, int nb, int *status, cudaStream_t stream,
                                int64_t *launches, int s = -1);

// Boundary rows of the listed parts: F[i][j] -> D[row_base+i][st2ed[start+j]].
template <typename T>
cudaError_t launch_bdy_scatter(const PartDesc *parts, int nparts, const T *F, T *D, int64_t ldD,
                               const int32_t *st2ed, int max_b, int max_s, cudaStream_t stream,
                               int64_t *launches);

// The batched Floyd-Warshall of every part as one persistent launch over a
// work queue (FloydQueue; nparts = the squares in the arena F, which the
// queue's parts index by f_off); with q.mp_work > 0 also the boundary-row scatter
// into D (as launch_bdy_scatter) and the min-plus tiles (as
// launch_minplus_parts, pk as there).  q.cnt must be zero (nparts * stride
// + 2 ints) when the launch starts.
template <typename T>
cudaError_t launch_floyd_queue(const PartDesc *parts, int nparts, T *F, int64_t ldf, const FloydQueue &q,
                               const MPWork *work, int n, T *D, int64_t ldD, int64_t drows,
                               const int32_t *st2ed, const int32_t *graph_id, const int32_t *ed2st,
                               int *status, cudaStream_t stream, int64_t *launches, const Pack16 *pk);

// Min-plus merge of the inner rows of the batch's parts, with the own-part
// columns taken from the closed Floyd matrices (fused decode).
// (F is the batch's Floyd arena with leading dimension ldf and nparts parts;
// D has drows rows.)
// pk (int32 only, may be null): buffers of the packed 16-bit form; the
// launcher first fills them for the work's parts, then every tile that
// provably fits runs packed (two relaxations per DPX instruction).
template <typename T>
cudaError_t launch_minplus_parts(const PartDesc *parts, int nparts, const MPWork *work, int nwork, int n,
                                 const T *F, int64_t ldf, T *D, int64_t ldD, int64_t drows,
                                 const int32_t *graph_id, const int32_t *ed2st, int *status,
                                 cudaStream_t stream, int64_t *launches, const Pack16 *pk = nullptr);

// Same for parts with at most kThinBoundary boundary vertices (store-bound
// shape): thin_parts[0..nthin) are batch indices of such parts, max_m bounds
// their inner row counts.
constexpr int kThinBoundary = 16;
template <typename T>
cudaError_t launch_minplus_thin(const PartDesc *parts, const int32_t *thin_parts, int nthin, int max_m,
                                int n, const T *F, T *D, int64_t ldD, const int32_t *graph_id,
                                const int32_t *ed2st, cudaStream_t stream, int64_t *launches);

// Predecessor rows of the listed parts' output rows (max_s bounds the
// parts' sizes).  The gather rule: P[row][j] = the in-neighbour u of j
// (in-edge CSR tro/tcol/tw) with the least D[row][u] + w(u, j), the
// smallest u on ties; the row's vertex maps to itself, an unreachable j to
// -1.  It gives the boundary rows, the own-part columns, and every row of
// parts with more than kPredThinB boundary vertices.  Inner rows of the
// other parts take, for columns outside their part, the predecessor on the
// row of the boundary vertex k* that the min-plus merge chose (the first k
// with the least F[i][k] + D[k][j]): P[i][j] = P[k*][j].  F is the batch's
// closed Floyd arena.
constexpr int kPredThinB = 12;
enum PredMode : int {
  kPredAll = 0,           // every row, every column
  kPredBoundaryRows = 1,  // rows < b, every column
  kPredOwnColumns = 2,    // every row, own-part columns, parts with b <= kPredThinB
  kPredThickInner = 3,    // rows >= b, every column, parts with b > kPredThinB
};
template <typename T>
cudaError_t launch_pred(const PartDesc *parts, int nparts, int max_s, const T *D, int32_t *P,
                        int64_t ldD, int n, const int32_t *tro, const int32_t *tcol, const T *tw,
                        const int32_t *st2ed, const T *F, cudaStream_t stream, int64_t *launches);

// Boundary-graph form of stage 1 (exact shortest distances from boundary
// vertices without SSSP).  With every part's local closure in F:
//   launch_bgraph: dB (nbB x nbB, ld ldB) = INF; dB[b1][b2] = F_p[b1][b2] for
//     boundary vertices of one part; cross-part arcs u -> v: dB[u][v] =
//     min(.., w).  Then close dB with launch_floyd_matrix.
//   launch_bdy_expand: for each listed (boundary index g, output row r):
//     D[r][v] = min over boundary b' of v's part q of dB[g][b'] + F_q[b'][v].
template <typename T>
cudaError_t launch_bgraph(const PartDesc *parts, int nparts, int max_b, const T *F, T *dB, int64_t ldB,
                          const int32_t *row_offset, const int32_t *col, const T *w, int n,
                          const int32_t *graph_id, const int32_t *ed2st, const BPart *bpart,
                          cudaStream_t stream, int64_t *launches);
//     Own-part entries also go to FB[g][j] (FB: boundary index x part-local
//     column, ld ldFB).
//   launch_local_fixup: turns every part's local closure in F into its
//     exact closure (inner rows: min over leaving through a boundary vertex;
//     boundary rows: FB), so that the min-plus merge and its decode run as in
//     the SSSP form.
//     With Tc (maxb x ldD values, may be null) the launch first writes the
//     column table Tc[k][v] = F_q[k][j(v)] (k < b_q, the sentinel up to
//     maxb, maxb >= every b_q), so that the expansion reads it with
//     coalesced loads instead of gathering from F.
template <typename T>
cudaError_t launch_bdy_expand(const int64_t *rows, int nrows, const BPart *bpart, const int32_t *graph_id,
                              const int32_t *ed2st, int n, const T *dB, int64_t ldB, int nbB, const T *F,
                              T *D, int64_t ldD, T *FB, int64_t ldFB, T *Tc, int maxb, cudaStream_t stream,
                              int64_t *launches);
// Boundary graph closed by Bellman-Ford (large boundary sets), ztiles tiles
// of kMsbfS sources side by side, alternating a local step (per part whose
// rows changed: min-plus of the tile's rows with the part's local closure
// F_p) and a cross step (the heads of cross-part arcs whose tails changed
// pull over their cross-part in-arcs; CSRs over boundary indices: in-arcs
// itro/itcol/itw, out-arcs otro/otcol); gpart: part id of every boundary
// index; pcol: its dB column; Dt ztiles x nb x kMsbfS; act 3 x ztiles x nb
// ints; pact ztiles x (K + 1) ints; wl 2 x ztiles x nb ints (two work
// lists); wl_count 3 ints; changed 4 ints; host_changed 4 pinned ints
// (convergence is tested on the host every 4 iterations).  Writes rows
// 0..nb-1 of dB at columns pcol[0..nb).
template <typename T>
cudaError_t launch_bgraph_bf(const PartDesc *parts, int nparts, int max_b, const T *F, const int32_t *itro,
                             const int32_t *itcol, const T *itw, const int32_t *otro, const int32_t *otcol,
                             const int32_t *gpart, const int32_t *pcol, int nb, int K, int ztiles, T *dB,
                             int64_t ldB, T *Dt, int *act, int *pact, int *wl, int *wl_count, int *changed,
                             int *host_changed, int64_t max_rounds, int *status, cudaStream_t stream,
                             int64_t *launches);
// Expansion with TMA-fed tiles (dB closed by Bellman-Ford, its columns
// padded per part: part q's boundary columns start at bd_col, a multiple of
// 4): grid (column tiles, boundary-index tiles, parts); A boxes from dB,
// B boxes from the F arena (nparts_f squares of side ldf).  A stage that
// never completes sets kDevTmaTimeout in status.
template <typename T>
cudaError_t launch_bdy_expand_tma(const PartDesc *parts, int nparts, int max_s, int nbB, const int64_t *grow,
                                  const int32_t *st2ed, const T *dB, int64_t ldB, const T *F, int64_t ldf,
                                  int nparts_f, T *D, int64_t ldD, T *FB, int64_t ldFB, int *status,
                                  cudaStream_t stream, int64_t *launches, const Expand16 *xk = nullptr);
// Tiled expansion (any boundary count): grid (boundary-index tiles, column
// tiles, parts); a CTA is a min-plus tile dB[g][b'_q] (x) F_q[b'][j] written
// to D[grow[g]][st2ed[start_q + j]] (and FB[g][j] for g of part q).
template <typename T>
cudaError_t launch_bdy_expand_tiled(const PartDesc *parts, int nparts, int max_s, int nbB, const int64_t *grow,
                                    const int32_t *st2ed, const T *dB, int64_t ldB, const T *F, T *D,
                                    int64_t ldD, T *FB, int64_t ldFB, cudaStream_t stream, int64_t *launches);
template <typename T>
cudaError_t launch_local_fixup(const PartDesc *parts, int nparts, int max_s, T *F, const T *FB, int64_t ldFB,
                               cudaStream_t stream, int64_t *launches);

// Resident cache: copy each listed part's boundary rows Bd[bd_row + i] into
// D[row_base + i] (all ldD columns).
template <typename T>
cudaError_t launch_bdy_copy(const PartDesc *parts, int nparts, int max_b, const T *Bd, T *D,
                            int64_t ldD, cudaStream_t stream, int64_t *launches);

// out[r][0..n) = src[idx[r]][0..n) for r < rows.
template <typename T>
cudaError_t launch_row_gather(const T *src, int64_t ld_src, const int64_t *idx, int64_t rows, int n,
                              T *out, int64_t ld_out, const int64_t *out_rows, cudaStream_t stream,
                              int64_t *launches);

// Distance rows of inner vertices from the resident cache: for entry e of
// group g (part parts[g.pidx], local row loc[e] >= b),
//   out[out_row[e]][j] = F[loc][local(j)]                     j in the part,
//                      = min(INF, min_k F[loc][k] + Bd[bd_row + k][j])   else,
// the same terms as the block min-plus and its decode.
template <typename T>
cudaError_t launch_minplus_rows(const PartDesc *parts, const RowGroup *groups, int ngroups,
                                const int32_t *loc, const int64_t *out_row, int max_b, int n,
                                const T *F, const T *Bd, int64_t ldD, const int32_t *graph_id,
                                const int32_t *ed2st, T *out, int64_t ld_out, cudaStream_t stream,
                                int64_t *launches);

// Generic C = min(INF, A (x) B).
template <typename T>
cudaError_t launch_minplus_generic(int M, int N, int K, const T *A, int64_t lda, const T *B,
                                   int64_t ldb, T *C, int64_t ldc, cudaStream_t stream,
                                   int64_t *launches);

// Fill rows x cols of a row-major matrix with v.
template <typename T>
cudaError_t launch_fill(T *p, int64_t rows, int64_t cols, int64_t ld, T v, cudaStream_t stream,
                        int64_t *launches);

// Per-row checksums of int32 distances (the float overload reads int32
// distances already converted to float, every value an exact integer).
cudaError_t launch_row_checksums(const int32_t *D, int64_t rows, int64_t n, int64_t ld,
                                 uint64_t *out, cudaStream_t stream, int64_t *launches);
cudaError_t launch_row_checksums(const float *D, int64_t rows, int64_t n, int64_t ld,
                                 uint64_t *out, cudaStream_t stream, int64_t *launches);

// int32 -> float copy of a rows x n block into a dense buffer.
cudaError_t launch_i32_to_f32(const int32_t *src, int64_t rows, int64_t n, int64_t ld, float *dst,
                              cudaStream_t stream, int64_t *launches);

// Relaxation-throughput microbenchmark; returns relaxations performed.
template <typename T>
cudaError_t launch_relax_peak(T *sink, int blocks, int iters, cudaStream_t stream,
                              double *relax_count);

}  // namespace fapb
