// Batched and served PCG: many independent systems of uneven size solved by
// one CUDA-graph launch whose body kernels sweep all running systems at once.
//
// The reference solves one system per CG<LAD> call; it has no batched path.
// Each system here follows the reference's recurrence (Jacobi-PCG,
// linear_solver/cg.h:165-246) inside an MPIR-style refinement
// (linear_solver/mpir.cc:52-230): FP64 residual, update and test around an
// FP32 inner solve, or, in FP64 mode, a plain FP64 (P)CG.
//
// Work decomposition: every system is cut into items of consecutive rows (a
// multiple of 32; each pass kernel has its own item size, picked by the
// tuner); one warp handles one item at a time (round-robin over the item
// list across all warps of the grid), so large and small systems share every
// launch and the warps of a block never wait on one another.
//
// Per-system sums are deterministic and deferred: an item stores its partial
// sums, and the next kernel's items each re-add their system's partials in a
// fixed order and take the system's decision themselves (alpha in K2, the
// residual, rz and the inner test in K3).  A system's arithmetic therefore
// does not depend on what else is in the batch or on the order its items ran
// in, and no item waits on a fence or an atomic ticket in K1 or K2.  Systems
// with more than kDirectItems items in a list (millions of rows) hand their
// totals on through a last-arriver ticket instead, since re-adding costs
// count^2 loads.  Scalars that one kernel both reads and updates are
// double-buffered by pass parity.
//
// Matrices are stored twice: CSR as uploaded (host-facing, setup), and a
// sliced ELL copy used by both SpMVs: slices of 32 rows, every row padded to
// the system's longest row `ell`; entry k of row 32s+l sits at
// (s*ell + k)*32 + l, so a warp reads 32 consecutive values per step and the
// loads of one row do not depend on a row pointer.  When every row's columns
// are the row plus a subset of one ascending set of at most kMaxStencil
// offsets (FE matrices on structured grids: the 9- and 27-point Q1
// couplings), the copy holds values only: position k of a row is its entry
// at column row + soff[k], 0 where the row has none, and no column is
// stored (values-only "stencil" layout; the products a row adds are the same
// in the same order, with exact zeros between them).
//
// Each system walks through phases; a phase changes only after every item of
// the system has passed (last-arriver ticket), so all items of a system see
// one phase per launch:
//   RESID   K1: r64 = b - A64 x (FP64), ||r64||, outer test; the inner solve
//               goes on from c = 0 with its residual replaced: r = (T)r64 -> START
//   START   K3: the search direction from the new residual, z = invD r and
//               p = z + beta p with beta = r.z / (r.z before the last step)
//               (the direction is kept: residual replacement, "reliable
//               updates"), or p = z on the first pass, after a breakdown, or
//               when the batch restarts its inner solves as MPIR does; then
//               opens the inner solve (-> INNER) once every item has passed
//   INNER   K1: Ap = A p, p.Ap partials
//           K2: alpha = rz / p.Ap; r -= alpha Ap; r.r, r.z partials
//           K3: inner test on r.r; if it goes on, c += alpha p and
//               p = z + beta p; if it ends, x += (double)(c + alpha p) and
//               -> RESID (mixed) or DONE (FP64 mode)
//   DONE    skipped by every kernel
// One pass of the device loop is K1 K2 K3; the last block of K3 ends the
// pass and clears the graph's WHILE condition when no system is running or
// the pass budget is spent, so the device loop always ends.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "internal.cuh"

namespace b200la {

enum BatchPhase : int { PH_EMPTY = 0, PH_RESID = 1, PH_INNER = 2, PH_CORRECT = 3, PH_DONE = 4, PH_START = 5 };

// Device descriptor of one system slot.
constexpr int kMaxStencil = 27;

template <typename T> struct SysDesc {
  int n;
  int nnz;
  const int *rowptr;  // CSR as uploaded
  const int *col;
  const double *val64;
  int ell;            // sliced ELL width (longest row)
  int col16;          // 1: sliced ELL columns stored as int16 offsets from the row
  int max_off;        // largest |column - row| of the stored entries
  const void *scol;   // sliced ELL columns: int32, or int16 (column - row) when col16
  const T *sval;      // sliced ELL values in the inner type
  const double *sval64;  // sliced ELL values in FP64 (== sval in FP64 mode)
  const double *b;
  double *x;
  T *c, *r, *p, *Ap;
  const T *invd;
  int stencil;        // 1: values-only layout, entry k of a row at column row + soff[k] (scol unused)
  int soff[kMaxStencil];  // ascending column offsets of the stencil layout (ell of them)
};

// Per-system scalars and counters (device).
struct SysState {
  int phase;
  int inner_iter;      // iterations of the current inner solve
  int total_iter;      // inner iterations over all passes
  int outer;           // refinement passes started
  double rz, pAp, alpha, beta;
  double res_in, res_in0;      // inner recurrence residual and its start value
  double res, res0;            // FP64 true residual and the initial one
  unsigned long long t_begin;  // %globaltimer at the system's first residual
  unsigned long long t_done;   // %globaltimer when the system finished
  int state;                   // B200LA_* iterate state at the end
  unsigned bad_row;            // first row without a usable diagonal (Jacobi), else ~0u
  unsigned ticket[4];
  double rzb[2];               // r.z of the current inner iteration, by pass parity
  double rz_keep;              // r.z before the last step of the previous inner solve
  int keep_p;                  // 1: the next START keeps the search direction
  double alphab[2];            // this pass's step (K2 writes, K3 reads), by pass parity
  int okb[2];                  // 0: this pass's step broke down
  int itb[2];                  // inner iterations done, by pass parity
  int totb[2];                 // inner iterations over all passes, by pass parity
  double tot[3];               // ticket path totals: K1 p.Ap; K2 r.r, r.z
};

struct BatchParams {
  int max_outer;
  int inner_maxits;
  double atol, rtol, dtol;  // outer (FP64) test
  double inner_rtol;        // inner test relative to its start residual
  int precond;
  int mixed;                // 1: FP32 inner + FP64 refinement; 0: FP64 CG
  int restart_inner;        // 1: every inner solve restarts from p = z
};

struct BatchGlobals {
  int active;          // systems not DONE (and not EMPTY)
  int passes;          // passes taken by this launch
  int max_passes;      // pass budget of this launch
  unsigned ticket;     // last block of K3
  int ntiles[3];       // items in the K1, K2 and K3 lists
  int tile_rows[3];    // rows per item of each list
  unsigned pass_total; // passes since the batch was created (parity of the buffered scalars)
  unsigned long long t_start;
};

// One warp's work item: rows row0 .. row0 + tile_rows - 1 of one system (the
// last item of a system is shorter).  Items of a system are consecutive in
// the list, so its first item is t - row0 / tile_rows and it has
// ceil(n / tile_rows) items; tile_rows is uniform over the list.  The record
// also carries where the system's partial sums of the previous kernel's list
// sit (K2 items: the system's K1 items; K3 items: its K2 items), so an item
// can load them as soon as it has its record, without first looking the
// system's descriptor or item table up.
struct __align__(16) Tile {
  int sys;
  int row0;    // a multiple of tile_rows (itself a multiple of 32)
  int pfirst;  // the system's first item in the previous kernel's list
  int pcount;  // and how many items it has there
};

// Geometry of item t: rows, first item of the system, items of the system.
struct ItemGeo {
  int rows, first, count;
};
__device__ __forceinline__ ItemGeo item_geo(const Tile &tl, int t, int n, int tile_rows) {
  ItemGeo g;
  g.rows = min(tile_rows, n - tl.row0);
  g.first = t - tl.row0 / tile_rows;
  g.count = (n + tile_rows - 1) / tile_rows;
  return g;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Sum of p[0..n) over the 32 lanes of a warp, in a fixed order: lane l adds
// p[l + 128 j + 32 u] into chain u (u = 0..3), the four chains combine in a
// fixed tree, then the lanes in the shuffle tree.  Every caller gets the same
// bits for the same values, and each lane keeps four loads in flight (a
// single chain waited for one L2 round trip per 32 values: the last item of
// a system of 6,000 items spent ~100 us on it).  Read through L2 only: other
// warps of the same kernel wrote the values.
// The values sit at p[0], p[step], p[2 step], ...
__device__ __forceinline__ double warp_sum_array(const double *p, int n, int step = 1) {
  const int lane = threadIdx.x & 31;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = lane; i < n; i += 128) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int j = i + 32 * u;
      if (j < n) a[u] += __ldcg(p + (int64_t)j * step);
    }
  }
  return warp_sum((a[0] + a[1]) + (a[2] + a[3]));
}

// Deterministic per-system reduction over warp items, in two levels so that
// no counter takes more than kGroup atomic increments per kernel: the warp's
// sums go to part[k][item]; the last item to finish of each group of kGroup
// consecutive items of the system (a ticket per group, gtick[leader], the
// leader being the group's first item) adds the group's partials into
// gpart[k][leader]; the last group to finish (the system's ticket over its
// groups) adds the group sums.  Both levels add in a fixed order, so the
// totals do not depend on the order in which items finished.  (One ticket
// for all of a system's items queued thousands of returning atomics on one
// address: 110 of 358 us of a K1 pass over 3D systems of 0.75 M rows.)
// Returns true in every lane of the warp that completes the system, with
// the totals in v[] of every lane.  Must be called by all 32 lanes.  The
// tickets wrap back to 0 by themselves (atomicInc modulus).
constexpr int kGroup = 64;

template <int NV>
__device__ __forceinline__ bool warp_sum_last(double (&v)[NV], double *part, double *gpart, unsigned *gtick,
                                              int64_t stride, int item, int first, int count, unsigned *ticket) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  const int gi = (item - first) / kGroup;
  const int leader = first + gi * kGroup;
  const int gsize = min(kGroup, count - gi * kGroup);
  const int ngroups = (count + kGroup - 1) / kGroup;
  unsigned t = 0;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) part[k * stride + item] = v[k];
    __threadfence();
    t = atomicInc(gtick + leader, (unsigned)gsize - 1);
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  if (t != (unsigned)gsize - 1) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum_array(part + k * stride + leader, gsize);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) gpart[k * stride + leader] = v[k];
    __threadfence();
    t = atomicInc(ticket, (unsigned)ngroups - 1);
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  if (t != (unsigned)ngroups - 1) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum_array(gpart + k * stride + first, ngroups, kGroup);
  return true;
}

// Ticket only: true in every lane of the warp that handles the system's
// last item to arrive.
__device__ __forceinline__ bool warp_last(int count, unsigned *ticket) {
  unsigned t = 0;
  if ((threadIdx.x & 31) == 0) {
    __threadfence();
    t = atomicInc(ticket, (unsigned)count - 1);
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  if (t != (unsigned)count - 1) return false;
  __threadfence();
  return true;
}

__device__ __forceinline__ int outer_check(double res, double res0, const BatchParams &p) {
  if (res <= p.atol) return B200LA_SUCCESS_ABS;
  if (res < p.rtol * res0) return B200LA_SUCCESS_REL;
  if (!(res <= p.dtol * res0)) return B200LA_FAIL_DIV;
  return B200LA_ITERATE;
}

// A system's phase (and alpha, beta) can change inside a kernel only when its
// last item to arrive writes them, after every other item of that system has
// read them; kernel launches refresh the read-only cache.  So the read-only
// path is safe, and it keeps the items of one large system from all asking
// L2 for the same line.
__device__ __forceinline__ int load_phase(const SysState *s) { return __ldg(&s->phase); }

__device__ __forceinline__ void finish_system(SysState &S, BatchGlobals *g, int state) {
  S.state = state;
  S.phase = PH_DONE;
  S.t_done = globaltimer();
  atomicSub(&g->active, 1);
}

// One row of y = A x per lane from the sliced ELL layout (V = value type of
// the stored values, X = type of x, I = stored column type: int, or short
// holding column - row).  The products are added in the row's stored order
// whatever I is, so both column types give the same bits.
template <typename V, typename X, typename I, int UNROLL>
__device__ __forceinline__ V sell_row_t(const I *__restrict__ scol, const V *__restrict__ sval, int ell,
                                        const X *__restrict__ x, int slice, int lane) {
  const int64_t base = (int64_t)slice * ell * 32 + lane;
  const I *cp = scol + base;
  const V *vp = sval + base;
  const int row = slice * 32 + lane;
  V sum = V(0);
#pragma unroll UNROLL
  for (int k = 0; k < ell; ++k) {
    const int c = sizeof(I) == 2 ? row + (int)ld_stream(cp + k * 32) : (int)ld_stream(cp + k * 32);
    sum = fma(ld_stream(vp + k * 32), (V)ld_keep(x + c), sum);
  }
  return sum;
}

// The same from the values-only layout: column row + soff[k], clamped into
// [0, n) where the row has no entry there (its value is 0).  soff points at
// the system's offsets in global memory (the loop index is not a constant).
template <typename V, typename X, int UNROLL>
__device__ __forceinline__ V stencil_row(const int *__restrict__ soff, const V *__restrict__ sval, int ell, int n,
                                         const X *__restrict__ x, int slice, int lane) {
  const int64_t base = (int64_t)slice * ell * 32 + lane;
  const V *vp = sval + base;
  const int row = slice * 32 + lane;
  V sum = V(0);
#pragma unroll UNROLL
  for (int k = 0; k < ell; ++k) {
    const int c = min(max(row + __ldg(soff + k), 0), n - 1);
    sum = fma(ld_stream(vp + k * 32), (V)ld_keep(x + c), sum);
  }
  return sum;
}

// A row from the system's sliced copy, whatever its column storage.
template <typename V, typename X, int UNROLL = 9, typename T>
__device__ __forceinline__ V sell_row(const SysDesc<T> &d, const SysDesc<T> *dg, const V *__restrict__ sval,
                                      const X *__restrict__ x, int slice, int lane) {
  if (d.stencil) return stencil_row<V, X, UNROLL>(dg->soff, sval, d.ell, d.n, x, slice, lane);
  return d.col16 ? sell_row_t<V, X, short, UNROLL>((const short *)d.scol, sval, d.ell, x, slice, lane)
                 : sell_row_t<V, X, int, UNROLL>((const int *)d.scol, sval, d.ell, x, slice, lane);
}

// Column type tag of the values-only layout (spmv_item's I).
struct StencilCols {};

// Warp-item loop shared by the pass kernels: warp w of the grid (W warps)
// takes items w, w + W, w + 2W, ... and calls body(tile, item, phase).  The
// records run two items ahead and the system phase one item ahead, so an
// item starts with its phase at hand: one dependent round trip fewer per
// item.  (Reading the phase early is safe: it changes only after every item
// of its system has arrived at the system's ticket, and this warp's item has
// not.  Claiming items from an atomic counter instead was measured slower:
// thousands of warps contend on one address; so was giving each warp a
// contiguous run of items: 194 against 158 us for the 1,024-system K1, the
// warps' concurrent reads then spread over the whole batch.)
//
// rev: walk the list from its end.  Consecutive pass kernels walk in
// opposite directions (K1 forward on even passes, K2 the other way, K3 as
// K1), so each kernel starts on the rows its predecessor touched last,
// whose vectors are the likeliest to be still in L2.
template <typename F>
__device__ __forceinline__ void for_each_item(const Tile *__restrict__ tiles, int ntiles, const SysState *st, bool rev,
                                              F &&body) {
  const int nw = gridDim.x * (kBlock / 32);
  int k = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);  // position in the walk
  auto at = [&](int j) { return rev ? ntiles - 1 - j : j; };
  Tile tl = k < ntiles ? tiles[at(k)] : Tile{};
  Tile nx = k + nw < ntiles ? tiles[at(k + nw)] : Tile{};
  int ph = k < ntiles ? load_phase(st + tl.sys) : (int)PH_EMPTY;
  while (k < ntiles) {
    const int kn = k + nw;
    const Tile nn = kn + nw < ntiles ? tiles[at(kn + nw)] : Tile{};
    const int nph = kn < ntiles ? load_phase(st + nx.sys) : (int)PH_EMPTY;
    body(tl, at(k), ph);
    tl = nx;
    nx = nn;
    ph = nph;
    k = kn;
  }
}

// Static variant (timing kernels): warp w takes items w, w + W, ...
template <typename F>
__device__ __forceinline__ void for_each_item_static(const Tile *__restrict__ tiles, int ntiles, F &&body) {
  const int nw = gridDim.x * (kBlock / 32);
  for (int t = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5); t < ntiles; t += nw) body(tiles[t], t);
}


}  // namespace b200la

namespace b200la {

// ---- deferred per-system reductions -----------------------------------------
// K1 and K2 only store each item's partial sums.  The next kernel's items
// re-add their system's partials -- every item the same values in the same
// fixed order (lane-strided, then a shuffle tree), so all get the same bits --
// and each makes the system's decision itself: K2 derives alpha from K1's
// partials (its first item passes alpha on to K3), K3 the residual, rz and
// the inner test from K2's.  Scalars
// that K3 both reads and updates are double-buffered by pass parity: kernels
// of pass P read slot P & 1; the one writer of each system (its first item)
// writes slot (P + 1) & 1.  Phase changes still wait for every item of the
// system (last-arriver ticket), because other items read the phase.

// Lists of the three pass kernels as one kernel argument.
struct PassLists {
  const Tile *tiles[3];
  double *part[3];           // [3][stride] partial sums per item
  double *gpart[3];          // [3][stride] group sums of the two-level ticket path (at group leaders)
  unsigned *gtick[3];        // [stride] group tickets of the two-level ticket path (at group leaders)
  int64_t stride[3];
  const int *sysfirst;       // [capacity][3]: each system's first item in each list
};

// A system with more items than this in a list hands its totals on through a
// last-arriver ticket (warp_sum_last into SysState::tot) instead: re-adding
// every partial in every consumer item costs count^2 loads per kernel, which
// for systems of millions of rows (thousands of items) exceeds the kernel's
// own traffic.  Both paths add the partials in a fixed order.
constexpr int kDirectItems = 1024;

// Sum of partial slot `slot` over a system's items in list k (all lanes; at
// most kDirectItems values: one chain per lane measured faster here than
// warp_sum_array's four).
__device__ __forceinline__ double sum_partials(const PassLists &L, int k, int slot, int first, int count) {
  const int lane = threadIdx.x & 31;
  const double *p = L.part[k] + slot * L.stride[k] + first;
  double a = 0.0;
  for (int i = lane; i < count; i += 32) a += __ldg(p + i);
  return warp_sum(a);
}

// Total of partial slot `slot` of list k for a system: re-added from the
// items' partials, or the ticket path's total.
__device__ __forceinline__ double sys_total(const PassLists &L, const SysState &S, int k, int slot, int first,
                                            int count) {
  if (count <= kDirectItems) return sum_partials(L, k, slot, first, count);
  return __ldcg(&S.tot[k == 0 ? 0 : 1 + slot]);
}

// Stores an item's partial sums v[] (one value per lane) for list k: as the
// item's partials, or through the ticket into S.tot.  All 32 lanes call it.
// The system's first item and item count are looked up here, after the
// item's main loop, so they are not held in registers across it.
template <int NV>
__device__ __forceinline__ void put_partials(const PassLists &L, SysState *st, int k, double (&v)[NV], int item,
                                             int sys, int n, int tile_rows) {
  const int lane = threadIdx.x & 31;
  const int count = (n + tile_rows - 1) / tile_rows;
  if (count <= kDirectItems) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      const double s = warp_sum(v[j]);
      if (lane == 0) L.part[k][j * L.stride[k] + item] = s;
    }
    return;
  }
  const int first = __ldg(L.sysfirst + 3 * sys + k);
  SysState &S = st[sys];
  if (warp_sum_last<NV>(v, L.part[k], L.gpart[k], L.gtick[k], L.stride[k], item, first, count, &S.ticket[k]) &&
      lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) S.tot[k == 0 ? 0 : 1 + j] = v[j];
  }
}

// The step size of the current inner iteration from K1's partials, as K2
// computes it (tl: a K2 item, whose record locates the system's K1 items).
// False on breakdown (p.Ap == 0 or alpha not finite).
__device__ __forceinline__ bool step_alpha(const PassLists &L, const Tile &tl, const SysState &S, double rz,
                                           double *alpha) {
  const double pap = sys_total(L, S, 0, 0, tl.pfirst, tl.pcount);
  const double a = rz / pap;
  *alpha = a;
  return pap != 0.0 && isfinite(a);
}

}  // namespace b200la

namespace b200la {

// ---- RESID items (run by K1): FP64 residual, outer test, inner restart ------
// r64 = b - A64 x with the FP64 sliced-ELL values, ||r64||, then the inner
// solve goes on from c = 0 with r = (T)r64 (K3's START items form the new
// direction from it).  The system's last item applies the outer test: DONE,
// or START.  It also seeds the next pass's slot of the double-buffered
// scalars.
template <typename T, bool PRE>
__device__ __forceinline__ void resid_item(const Tile &tl, int t, const ItemGeo &ig, const SysDesc<T> &d,
                                           const SysDesc<T> *dg, SysState &S, const PassLists &L, BatchGlobals *g,
                                           const BatchParams &prm, int q) {
  Acc<double> rr64;
  Acc<T> rrin, rzin;
  const int lane = threadIdx.x & 31;
  const int nsl = (ig.rows + 31) >> 5;
  const int end = tl.row0 + ig.rows;
  for (int sl = 0; sl < nsl; ++sl) {
    const int slice = (tl.row0 >> 5) + sl;
    const double y = sell_row<double, double, 3>(d, dg, d.sval64, d.x, slice, lane);
    const int row = slice * 32 + lane;
    if (row < end) {
      const double r64 = d.b[row] - y;
      rr64.add(r64 * r64);
      const T r = (T)r64;
      d.r[row] = r;
      d.c[row] = T(0);
      const T z = PRE ? r * d.invd[row] : r;
      rrin.add(r * r);
      rzin.add(r * z);
    }
  }
  double v[3] = {rr64.value(), rrin.value(), rzin.value()};
  if (warp_sum_last<3>(v, L.part[0], L.gpart[0], L.gtick[0], L.stride[0], t, ig.first, ig.count, &S.ticket[3]) &&
      lane == 0) {
    const double res = sqrt(v[0]);
    S.res = res;
    if (S.outer == 0) {
      S.res0 = res;
      S.t_begin = globaltimer();
    }
    int s = outer_check(res, S.res0, prm);
    if (s == B200LA_ITERATE && S.outer >= prm.max_outer) s = B200LA_FAIL_MAXITS;
    // a replaced residual more than twice the recurrence's last one: the
    // inner recurrence drifted from the true residual, so START restarts the
    // direction (p = z) instead of keeping it
    if (S.outer > 0 && sqrt(v[1]) > 2.0 * S.res_in) S.keep_p = 0;
    if (prm.precond && S.bad_row != 0xffffffffu) s = B200LA_FAIL_BREAKDOWN;  // Jacobi needs every diagonal
    if (s != B200LA_ITERATE) {
      finish_system(S, g, s);
    } else {
      S.outer += 1;
      S.inner_iter = 0;
      S.res_in = S.res_in0 = sqrt(v[1]);
      S.rzb[q ^ 1] = PRE ? v[2] : v[1];
      S.itb[q ^ 1] = 0;
      S.totb[q ^ 1] = S.totb[q];
      S.phase = PH_START;
    }
  }
}

// Ap = A p over an item's rows and the item's share of p.Ap, for rows of
// exactly E stored entries (E a compile-time width): software-pipelined, so
// the next slice's values and columns stream in while the current slice's
// gathers of p are in flight.  Same products, same order as sell_row.
//
// STAGE (banded systems): the warp first copies the window of p its rows can
// reach -- rows row0 - max_off .. row0 + rows + max_off, at most kWin values
// -- into its slice of shared memory with coalesced loads, so the gathers of
// every slice read shared memory instead of waiting on L1/L2.
constexpr int kWin = 1280;  // values of p per warp window (FP32: 5 KB)

template <typename T, typename I, int E, bool STAGE>
__device__ __forceinline__ double spmv_item_fixed(int row0, int rows, const SysDesc<T> &d, int lane, T *win) {
  // I = StencilCols: values-only layout, columns row + soff[k] (no column loads)
  constexpr bool SC = std::is_same<I, StencilCols>::value;
  using IC = typename std::conditional<SC, short, I>::type;
  Acc<T> acc;
  const int nsl = (rows + 31) >> 5;
  const int end = row0 + rows;
  const IC *__restrict__ scol = (const IC *)d.scol;
  const T *__restrict__ sval = d.sval;
  const T *__restrict__ p = d.p;
  int slice = row0 >> 5;
  IC cv[E];
  T vv[E];
  {
    const int64_t base = (int64_t)slice * E * 32 + lane;
#pragma unroll
    for (int k = 0; k < E; ++k) {
      if (!SC) cv[k] = ld_stream(scol + base + k * 32);
      vv[k] = ld_stream(sval + base + k * 32);
    }
  }
  int lo = 0;
  if (STAGE) {
    // the window in 16-byte chunks by asynchronous copies (cp.async, L2 only):
    // every lane issues all its chunks before waiting, so the window costs
    // one round trip instead of one per load.  lo is rounded down to a chunk
    // and the end up; a slot's vectors are 256-byte aligned allocations of
    // whole 256-byte units, so the last chunk stays inside p's allocation
    // (the values past n it reads are never gathered: columns are < n).
    lo = max(row0 - d.max_off, 0) & ~3;
    const int hi = (min(end + d.max_off, d.n) + 3) & ~3;
    const unsigned wbase = (unsigned)__cvta_generic_to_shared(win);
    for (int i = lo + 4 * lane; i < hi; i += 128)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(wbase + 4u * (unsigned)(i - lo)),
                   "l"(p + i)
                   : "memory");
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
  }
  for (int sl = 0; sl < nsl; ++sl, ++slice) {
    const int row = slice * 32 + lane;
    T xs[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      // stencil: a column outside [0, n) belongs to an absent entry (value 0)
      const int c = SC ? min(max(row + d.soff[k], 0), d.n - 1)
                       : (sizeof(IC) == 2 ? row + (int)cv[k] : (int)cv[k]);
      xs[k] = STAGE ? win[c - lo] : ld_keep(p + c);
    }
    T vc[E];
#pragma unroll
    for (int k = 0; k < E; ++k) vc[k] = vv[k];
    if (sl + 1 < nsl) {
      const int64_t base = (int64_t)(slice + 1) * E * 32 + lane;
#pragma unroll
      for (int k = 0; k < E; ++k) {
        if (!SC) cv[k] = ld_stream(scol + base + k * 32);
        vv[k] = ld_stream(sval + base + k * 32);
      }
    }
    T y = T(0);
#pragma unroll
    for (int k = 0; k < E; ++k) y = fma(vc[k], xs[k], y);
    if (row < end) {
      d.Ap[row] = y;
      acc.add(y * (STAGE ? win[row - lo] : p[row]));
    }
  }
  if (STAGE) __syncwarp();  // the window is rewritten by the warp's next item
  return acc.value();
}

// Ap = A p over an item's rows and the item's share of p.Ap.
template <typename T, typename I>
__device__ __forceinline__ double spmv_item(int row0, int rows, const SysDesc<T> &d, const SysDesc<T> *dg, int lane,
                                            T *win) {
  constexpr bool SC = std::is_same<I, StencilCols>::value;
  if (sizeof(T) == 4 && d.ell == 9) {
    // (+6: the window's ends are rounded out to 16-byte chunks)
    if (win && rows + 2 * d.max_off + 6 <= kWin) return spmv_item_fixed<T, I, 9, true>(row0, rows, d, lane, win);
    return spmv_item_fixed<T, I, 9, false>(row0, rows, d, lane, nullptr);
  }
  Acc<T> acc;
  const int nsl = (rows + 31) >> 5;
  const int end = row0 + rows;
  using IC = typename std::conditional<SC, short, I>::type;
  const IC *scol = (const IC *)d.scol;
  for (int sl = 0; sl < nsl; ++sl) {
    const int slice = (row0 >> 5) + sl;
    const T y = SC ? stencil_row<T, T, 9>(dg->soff, d.sval, d.ell, d.n, d.p, slice, lane)
                   : sell_row_t<T, T, IC, 9>(scol, d.sval, d.ell, d.p, slice, lane);
    const int row = slice * 32 + lane;
    if (row < end) {
      d.Ap[row] = y;
      acc.add(y * d.p[row]);
    }
  }
  return acc.value();
}

// ---- K1: Ap = A p and the items' p.Ap partials (INNER); RESID systems -------
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock, 4) batch_spmv_kernel(PassLists L, const SysDesc<T> *__restrict__ desc,
                                                               SysState *st, BatchGlobals *g, BatchParams prm) {
  const int lane = threadIdx.x & 31;
  // per-warp window of p for banded FP32 systems (see spmv_item_fixed)
  constexpr int kWinT = sizeof(T) == 4 ? kWin : 1;
  __shared__ __align__(16) T win_all[kBlock / 32][kWinT];
  T *win = sizeof(T) == 4 ? win_all[threadIdx.x >> 5] : nullptr;
  const int tr = g->tile_rows[0];
  const int q = (int)(__ldg(&g->pass_total) & 1u);
  for_each_item(L.tiles[0], g->ntiles[0], st, q != 0, [&](const Tile &tl, int t, int ph) {
    if (ph != PH_INNER && ph != PH_RESID) return;
    SysState &S = st[tl.sys];
    const SysDesc<T> d = desc[tl.sys];
    const ItemGeo ig = item_geo(tl, t, d.n, tr);
    if (ph == PH_RESID) {
      resid_item<T, PRE>(tl, t, ig, d, desc + tl.sys, S, L, g, prm, q);
      return;
    }
    // one column type per item, so each slice loop is a straight stream
    double pap[1] = {d.stencil ? spmv_item<T, StencilCols>(tl.row0, ig.rows, d, desc + tl.sys, lane, win)
                     : d.col16 ? spmv_item<T, short>(tl.row0, ig.rows, d, desc + tl.sys, lane, win)
                               : spmv_item<T, int>(tl.row0, ig.rows, d, desc + tl.sys, lane, win)};
    put_partials<1>(L, st, 0, pap, t, tl.sys, d.n, tr);
  });
}

// ---- K2: r -= alpha Ap and the items' r.r, r.z partials ----------------------
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock, 4) batch_update_kernel(PassLists L, const SysDesc<T> *__restrict__ desc,
                                                                 SysState *st, BatchGlobals *g, BatchParams prm) {
  const int lane = threadIdx.x & 31;
  const int tr = g->tile_rows[1];
  const int q = (int)(__ldg(&g->pass_total) & 1u);
  for_each_item(L.tiles[1], g->ntiles[1], st, q == 0, [&](const Tile &tl, int t, int ph) {
    if (ph != PH_INNER) return;
    SysState &S = st[tl.sys];
    const SysDesc<T> d = desc[tl.sys];
    const ItemGeo ig = item_geo(tl, t, d.n, tr);
    double alpha_d;
    const bool ok = step_alpha(L, tl, S, __ldg(&S.rzb[q]), &alpha_d);
    if (t == ig.first && lane == 0) {  // the step, for K3
      S.alphab[q] = ok ? alpha_d : 0.0;
      S.okb[q] = ok ? 1 : 0;
    }
    // breakdown: no update; K3 folds c into x as it stands
    if (!ok) return;
    const T alpha = (T)alpha_d;
    Acc<T> rr, rz;
    // 16-byte vectors (item starts are multiples of 32 rows and every slot
    // vector is 256-byte aligned), then the ragged tail
    using V = typename Vec16<T>::type;
    constexpr int W = Vec16<T>::n;
    const int nv = ig.rows / W;
    // two vectors per lane per step: their six loads are in flight together
    for (int qv = lane; qv < nv; qv += 64) {
      const bool two = qv + 32 < nv;
      V rv[2], av[2], dv[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (u == 1 && !two) break;
        const int i = tl.row0 + (qv + 32 * u) * W;
        rv[u] = *reinterpret_cast<const V *>(d.r + i);
        av[u] = *reinterpret_cast<const V *>(d.Ap + i);
        if (PRE) dv[u] = *reinterpret_cast<const V *>(d.invd + i);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (u == 1 && !two) break;
        T *rs = reinterpret_cast<T *>(&rv[u]);
        const T *as = reinterpret_cast<const T *>(&av[u]);
        const T *ds = reinterpret_cast<const T *>(&dv[u]);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          rs[k] = fma(-alpha, as[k], rs[k]);
          rr.add(rs[k] * rs[k]);
          if (PRE) rz.add(rs[k] * (rs[k] * ds[k]));
        }
        *reinterpret_cast<V *>(d.r + tl.row0 + (qv + 32 * u) * W) = rv[u];
      }
    }
    const int end = tl.row0 + ig.rows;
    for (int i = tl.row0 + nv * W + lane; i < end; i += 32) {
      const T r = fma(-alpha, d.Ap[i], d.r[i]);
      d.r[i] = r;
      rr.add(r * r);
      if (PRE) rz.add(r * (r * d.invd[i]));
    }
    double sums[2] = {rr.value(), rz.value()};
    put_partials<2>(L, st, 1, sums, t, tl.sys, d.n, tr);
  });
}

// ---- K3: the inner step's decision; c += alpha p, p = z + beta p, or x += c --
template <typename T, bool PRE, bool IN_GRAPH = true>
__global__ void __launch_bounds__(kBlock, 4) batch_direction_kernel(PassLists L, const SysDesc<T> *__restrict__ desc,
                                                                    SysState *st, BatchGlobals *g, BatchParams prm,
                                                                    cudaGraphConditionalHandle loop) {
  const int lane = threadIdx.x & 31;
  const int tr = g->tile_rows[2];
  const int q = (int)(__ldg(&g->pass_total) & 1u);
  for_each_item(L.tiles[2], g->ntiles[2], st, q != 0, [&](const Tile &tl, int t, int ph) {
    if (ph != PH_INNER && ph != PH_START) return;
    SysState &S = st[tl.sys];
    const SysDesc<T> d = desc[tl.sys];
    const ItemGeo ig = item_geo(tl, t, d.n, tr);
    const int end = tl.row0 + ig.rows;
    if (ph == PH_START) {
      // K1 replaced the residual: the new direction p = z + beta p (or z),
      // then the inner solve opens once every item of the system has passed
      const bool keep = __ldg(&S.keep_p) != 0;
      const double beta_d = keep ? __ldg(&S.rzb[q ^ 1]) / __ldg(&S.rz_keep) : 0.0;
      const bool use = keep && isfinite(beta_d);
      const T beta = (T)beta_d;
      for (int i = tl.row0 + lane; i < end; i += 32) {
        const T z = PRE ? d.r[i] * d.invd[i] : d.r[i];
        d.p[i] = use ? fma(beta, d.p[i], z) : z;
      }
      if (warp_last(ig.count, &S.ticket[2]) && lane == 0) S.phase = PH_INNER;
      return;
    }
    // INNER: every item of the system makes the same decision from K1's and
    // K2's partials (IterateControl for the FP64 recurrence, the inner
    // tolerance for mixed precision)
    const double rz_cur = __ldg(&S.rzb[q]);
    const int it = __ldg(&S.itb[q]), tot = __ldg(&S.totb[q]);
    double alpha_d = __ldg(&S.alphab[q]), res = 0.0, rz_new = 0.0;
    const bool ok = __ldg(&S.okb[q]) != 0;
    int state = B200LA_ITERATE;
    bool done = true;
    if (!ok) {
      alpha_d = 0.0;  // breakdown: no step; x takes the correction so far
      state = B200LA_FAIL_BREAKDOWN;
    } else {
      const double rr = sys_total(L, S, 1, 0, tl.pfirst, tl.pcount);
      const double rzs = sys_total(L, S, 1, 1, tl.pfirst, tl.pcount);
      res = sqrt(rr);
      rz_new = PRE ? rzs : rr;
      const int it1 = it + 1;
      const double res_in0 = __ldg(&S.res_in0);
      if (prm.mixed) {
        // inner solve: stop at inner_rtol (strict, as IterateControl), no
        // tighter than half the outer target (the last pass does not
        // over-solve), or at its iteration budget
        const double target = fmax(prm.inner_rtol * res_in0, 0.5 * prm.rtol * __ldg(&S.res0));
        done = res < target || it1 >= prm.inner_maxits || !(res == res);
      } else {
        // FP64 CG: IterateControl::Check on the recurrence residual (cg.h:214-225)
        if (res <= prm.atol) state = B200LA_SUCCESS_ABS;
        else if (res < prm.rtol * res_in0) state = B200LA_SUCCESS_REL;
        else if (res > prm.dtol * res_in0) state = B200LA_FAIL_DIV;
        else if (it1 >= prm.inner_maxits) state = B200LA_FAIL_MAXITS;
        done = state != B200LA_ITERATE;
      }
    }
    const T alpha = (T)alpha_d;
    const int steps = ok ? 1 : 0;
    if (t == ig.first && lane == 0) {
      S.rzb[q ^ 1] = ok ? rz_new : rz_cur;
      S.itb[q ^ 1] = it + steps;
      S.totb[q ^ 1] = tot + steps;
      S.inner_iter = it + steps;
      S.total_iter = tot + steps;
      if (ok) S.res_in = res;
      if (done) {
        // the next inner solve continues this direction (p is left as the
        // direction of this last step) unless it broke down
        S.rz_keep = rz_cur;
        S.keep_p = (ok && isfinite(res) && !prm.restart_inner) ? 1 : 0;
      }
    }
    if (!done) {
      // this step's correction c += alpha p (with p before its update), then
      // the new direction p = z + beta p
      const T beta = (T)(rz_new / rz_cur);
      using V = typename Vec16<T>::type;
      constexpr int W = Vec16<T>::n;
      const int nv = ig.rows / W;
      for (int qv = lane; qv < nv; qv += 32) {
        const int i = tl.row0 + qv * W;
        V pv = *reinterpret_cast<const V *>(d.p + i);
        V cv = *reinterpret_cast<const V *>(d.c + i);
        const V rv = *reinterpret_cast<const V *>(d.r + i);
        V dv;
        if (PRE) dv = *reinterpret_cast<const V *>(d.invd + i);
        T *ps = reinterpret_cast<T *>(&pv);
        T *cs = reinterpret_cast<T *>(&cv);
        const T *rs = reinterpret_cast<const T *>(&rv);
        const T *ds = reinterpret_cast<const T *>(&dv);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          cs[k] = fma(alpha, ps[k], cs[k]);
          ps[k] = fma(beta, ps[k], PRE ? rs[k] * ds[k] : rs[k]);
        }
        *reinterpret_cast<V *>(d.c + i) = cv;
        *reinterpret_cast<V *>(d.p + i) = pv;
      }
      for (int i = tl.row0 + nv * W + lane; i < end; i += 32) {
        const T pi = d.p[i];
        d.c[i] = fma(alpha, pi, d.c[i]);
        d.p[i] = fma(beta, pi, PRE ? d.r[i] * d.invd[i] : d.r[i]);
      }
      return;
    }
    // the inner solve ends: the last step's correction, then x += c
    for (int i = tl.row0 + lane; i < end; i += 32) d.x[i] += (double)fma(alpha, d.p[i], d.c[i]);
    // the phase moves on only after every item of the system did its part
    if (warp_last(ig.count, &S.ticket[2]) && lane == 0) {
      if (prm.mixed) {
        S.phase = PH_RESID;
      } else {
        if (ok) S.res = res;
        finish_system(S, g, state);
      }
    }
  });
  // the last block of the launch ends the pass and decides whether the
  // device loop runs another one
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicInc(&g->ticket, gridDim.x - 1) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const int passes = g->passes + 1;
    g->passes = passes;
    g->pass_total = g->pass_total + 1;
    const int active = *(volatile int *)&g->active;
    if (IN_GRAPH) cudaGraphSetConditional(loop, (active > 0 && passes < g->max_passes) ? 1u : 0u);
  }
}

__global__ void batch_start_kernel(BatchGlobals *g) {
  g->passes = 0;
  g->ticket = 0;
  g->t_start = globaltimer();
}

// Slot set-up after the CSR arrived: sliced-ELL copies (inner type and
// FP64), the inverse diagonal in the inner type, zero work vectors.
template <typename T>
__device__ void slot_setup_rows(const SysDesc<T> &d, unsigned *bad, int64_t first, int64_t stride, bool zero_x) {
  const int64_t padded_rows = (int64_t)(d.n + 31) / 32 * 32;
  for (int64_t i = first; i < padded_rows; i += stride) {
    // padding repeats a column the row reads (an empty row: its own index);
    // padding rows past n (last slice) read column n - 1
    int start = 0, len = 0, pad = d.n - 1;
    if (i < d.n) {
      start = d.rowptr[i];
      len = d.rowptr[i + 1] - start;
      pad = len > 0 ? d.col[start + len - 1] : (int)i;
    }
    const int64_t base = (i >> 5) * (int64_t)d.ell * 32 + (i & 31);
    if (d.stencil) {
      // values-only layout: position k holds the entry at column i + soff[k]
      // (the device check made every row's offsets an ascending subset)
      int j = start;
      for (int k = 0; k < d.ell; ++k) {
        const int64_t pos = base + (int64_t)k * 32;
        double v = 0.0;
        if (j < start + len && d.col[j] == (int)i + d.soff[k]) v = d.val64[j++];
        const_cast<T *>(d.sval)[pos] = (T)v;
        if ((const void *)d.sval64 != (const void *)d.sval) const_cast<double *>(d.sval64)[pos] = v;
      }
      continue;
    }
    for (int k = 0; k < d.ell; ++k) {
      const bool real = k < len;
      const int64_t pos = base + (int64_t)k * 32;
      if (d.col16) const_cast<short *>((const short *)d.scol)[pos] = (short)((real ? d.col[start + k] : pad) - (int)i);
      else const_cast<int *>((const int *)d.scol)[pos] = real ? d.col[start + k] : pad;
      const_cast<T *>(d.sval)[pos] = real ? (T)d.val64[start + k] : T(0);
      if ((const void *)d.sval64 != (const void *)d.sval)
        const_cast<double *>(d.sval64)[pos] = real ? d.val64[start + k] : 0.0;
    }
  }
  for (int64_t i = first; i < d.n; i += stride) {
    int k = -1;
    for (int j = d.rowptr[i]; j < d.rowptr[i + 1]; ++j)
      if (d.col[j] == i) { k = j; break; }
    const T a = k >= 0 ? (T)d.val64[k] : T(0);
    if (a == T(0)) {
      atomicMin(bad, (unsigned)i);
      const_cast<T *>(d.invd)[i] = T(0);
    } else {
      const_cast<T *>(d.invd)[i] = T(1) / a;
    }
    d.c[i] = T(0);
    d.r[i] = T(0);
    d.p[i] = T(0);
    d.Ap[i] = T(0);
    if (zero_x) d.x[i] = 0.0;
  }
}

// One system's sliced-ELL copy, inverse diagonal and zero work vectors.
template <typename T>
__global__ void slot_setup_kernel(SysDesc<T> d, unsigned *bad) {
  slot_setup_rows(d, bad, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x, false);
}

// The systems of one add_many call: job k is system k's descriptor, slot and
// whether x starts at zero.
template <typename T> struct SetupJob {
  SysDesc<T> d;
  int slot;
  int zero_x;
};

// Descriptor and fresh RESID state of every job's slot (thread per job).
template <typename T>
__global__ void slot_init_many_kernel(const SetupJob<T> *__restrict__ jobs, int count, SysDesc<T> *desc,
                                      SysState *st) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int s = jobs[k].slot;
    desc[s] = jobs[k].d;
    SysState z{};
    z.phase = PH_RESID;
    z.bad_row = 0xffffffffu;
    st[s] = z;
  }
}

// slot_setup_kernel for every job: blockIdx.y walks the jobs, blockIdx.x
// and the threads the rows of one system.
template <typename T>
__global__ void slot_setup_many_kernel(const SetupJob<T> *__restrict__ jobs, int count, SysState *st) {
  for (int k = blockIdx.y; k < count; k += gridDim.y) {
    const SetupJob<T> &j = jobs[k];
    slot_setup_rows(j.d, &st[j.slot].bad_row, (int64_t)blockIdx.x * blockDim.x + threadIdx.x,
                    (int64_t)gridDim.x * blockDim.x, j.zero_x != 0);
  }
}

// Plain batched SpMV Ap = A p over every item (timing only).
template <typename T>
__global__ void __launch_bounds__(kBlock, 6) batch_spmv_plain_kernel(const Tile *__restrict__ tiles, int ntiles,
                                                                     int tile_rows,
                                                                     const SysDesc<T> *__restrict__ desc) {
  const int lane = threadIdx.x & 31;
  for_each_item_static(tiles, ntiles, [&](const Tile &tl, int) {
    const SysDesc<T> d = desc[tl.sys];
    const int rows = min(tile_rows, d.n - tl.row0);
    const int nsl = (rows + 31) >> 5;
    for (int sl = 0; sl < nsl; ++sl) {
      const int slice = (tl.row0 >> 5) + sl;
      const T y = sell_row<T, T>(d, desc + tl.sys, d.sval, d.p, slice, lane);
      const int row = slice * 32 + lane;
      if (row < tl.row0 + rows) d.Ap[row] = y;
    }
  });
}

// Saves (save = 1) or restores the carried vectors x, c, r, p of the listed
// slots: one block per slot; slot k's values start at offs[k] in xs and at
// 3*offs[k] in vs.  Lets the tuner time real passes and leave every system
// as it found it.
template <typename T>
__global__ void __launch_bounds__(kBlock) slot_snapshot_kernel(const int *__restrict__ slots,
                                                               const int64_t *__restrict__ offs,
                                                               const SysDesc<T> *__restrict__ desc, double *xs, T *vs,
                                                               int save) {
  const SysDesc<T> d = desc[slots[blockIdx.x]];
  const int64_t o = offs[blockIdx.x];
  T *vc = vs + 3 * o, *vr = vc + d.n, *vp = vr + d.n;
  for (int i = threadIdx.x; i < d.n; i += kBlock) {
    if (save) {
      xs[o + i] = d.x[i];
      vc[i] = d.c[i];
      vr[i] = d.r[i];
      vp[i] = d.p[i];
    } else {
      d.x[i] = xs[o + i];
      d.c[i] = vc[i];
      d.r[i] = vr[i];
      d.p[i] = vp[i];
    }
  }
}

// Checks of an uploaded CSR (those of the host validate_csr): rowptr[0] == 0,
// rowptr[n] == nnz, non-decreasing, 0 <= col < n; also the longest row and
// the largest |col - row|.  The first failing row (and why) is kept with a
// 64-bit atomicMin on (row << 8 | code); columns are read only for rows
// whose bounds lie inside [0, nnz].
enum CsrCheckCode : int { kChkStart = 1, kChkDecrease = 2, kChkBounds = 3, kChkColumn = 4 };
struct CsrCheck {
  unsigned long long err;  // ~0: valid
  int max_row;
  int max_off;
  int stencil;             // 1 while every row checked fits the stencil below
  int slen;                // offsets of the stencil (those of the middle row), 0: none
  int soff[kMaxStencil];
};

__global__ void csr_check_init_kernel(int count, CsrCheck *c) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    CsrCheck z{};
    z.err = ~0ull;
    z.stencil = 1;
    c[k] = z;
  }
}

// The candidate stencil of a system: the column offsets of its middle row,
// if that row's extent lies in [0, nnz], it has 1..kMaxStencil entries and
// its columns ascend strictly; len 0 otherwise.  Every block derives the same
// candidate (the row is checked before it is read).
__device__ int stencil_candidate(int n, int nnz, const int *__restrict__ rowptr, const int *__restrict__ col,
                                 int *off) {
  const int m = n / 2;
  const int a = rowptr[m], b = rowptr[m + 1];
  if (a < 0 || b > nnz || b - a < 1 || b - a > kMaxStencil) return 0;
  for (int j = a; j < b; ++j) {
    off[j - a] = col[j] - m;
    if (j > a && off[j - a] <= off[j - a - 1]) return 0;
  }
  return b - a;
}

__device__ void csr_check_rows(int n, int nnz, const int *__restrict__ rowptr, const int *__restrict__ col,
                               CsrCheck *out, int first, int stride, const int *soff, int slen) {
  int mr = 0, mo = 0;
  bool fits = slen > 0;  // every row's offsets an ascending subset of soff
  unsigned long long err = ~0ull;
  for (int i = first; i < n; i += stride) {
    const int a = rowptr[i], b = rowptr[i + 1];
    unsigned long long e = ~0ull;
    if ((i == 0 && a != 0) || (i == n - 1 && b != nnz)) e = ((unsigned long long)i << 8) | kChkStart;
    else if (b < a) e = ((unsigned long long)i << 8) | kChkDecrease;
    else if (a < 0 || b > nnz) e = ((unsigned long long)i << 8) | kChkBounds;
    if (e != ~0ull) {
      err = min(err, e);
      continue;
    }
    mr = max(mr, b - a);
    int k = 0;
    for (int j = a; j < b; ++j) {
      const int c = col[j];
      if (c < 0 || c >= n) {
        err = min(err, ((unsigned long long)i << 8) | kChkColumn);
        break;
      }
      mo = max(mo, abs(c - i));
      if (fits) {
        while (k < slen && soff[k] < c - i) ++k;
        if (k < slen && soff[k] == c - i) ++k;
        else fits = false;
      }
    }
  }
  if (err != ~0ull) atomicMin(&out->err, err);
  if (mr) atomicMax(&out->max_row, mr);
  if (mo) atomicMax(&out->max_off, mo);
  if (!fits) atomicMin(&out->stencil, 0);
}

// The uploaded CSR arrays of one add_many call, one job per system (n = 0:
// nothing to check, the system was refused on the host).
struct CheckJob {
  const int *rowptr, *col;
  int n, nnz;
};

// csr_check for every job: blockIdx.y walks the jobs, blockIdx.x and the
// threads the rows of one system; out[k] collects job k's verdict.
__global__ void csr_check_many_kernel(const CheckJob *__restrict__ jobs, int count, CsrCheck *out) {
  __shared__ int soff[kMaxStencil];
  __shared__ int slen;
  for (int k = blockIdx.y; k < count; k += gridDim.y) {
    const CheckJob j = jobs[k];
    __syncthreads();  // the previous job's stencil is no longer read
    if (threadIdx.x == 0) {
      slen = j.n > 0 ? stencil_candidate(j.n, j.nnz, j.rowptr, j.col, soff) : 0;
      if (blockIdx.x == 0) {
        out[k].slen = slen;
        for (int q = 0; q < slen; ++q) out[k].soff[q] = soff[q];
      }
    }
    __syncthreads();
    if (j.n > 0)
      csr_check_rows(j.n, j.nnz, j.rowptr, j.col, out + k, blockIdx.x * blockDim.x + threadIdx.x,
                     gridDim.x * blockDim.x, soff, slen);
  }
}

// Restart every listed slot from x = 0: RESID phase, counters cleared.
template <typename T>
__global__ void __launch_bounds__(kBlock) batch_restart_kernel(const int *__restrict__ slots,
                                                               const SysDesc<T> *__restrict__ desc, SysState *st) {
  const int s = slots[blockIdx.x];
  const SysDesc<T> d = desc[s];
  for (int i = threadIdx.x; i < d.n; i += kBlock) d.x[i] = 0.0;
  if (threadIdx.x == 0) {
    SysState &S = st[s];
    const unsigned bad = S.bad_row;
    S = SysState{};
    S.phase = PH_RESID;
    S.bad_row = bad;
  }
}

}  // namespace b200la

using namespace b200la;

namespace {

// Host record of one slot.
struct HostSys {
  bool used = false;
  int n = 0;
  int nnz = 0;
  void *chunk = nullptr;   // CSR as uploaded and the vectors
  void *chunk2 = nullptr;  // the sliced-ELL copy (sized once the rows are known)
  size_t bytes = 0;
  SysDesc<double> d64{};
  SysDesc<float> d32{};
  double *out = nullptr;   // registered host destination of the solution
  bool out_copied = false; // its copy is queued on the transfer stream
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

constexpr int kDefaultRows[3] = {256, 1024, 512};

// One work-item list: host copy, device copy, per-item partial sums.
struct ItemList {
  int rows = 256;           // rows per item (upper bound when adaptive)
  int used = 256;           // rows per item of the current list
  int64_t cap = 0;          // device capacity (items)
  Tile *dev = nullptr;      // [cap]
  double *part = nullptr;   // [3][cap]
  double *gpart = nullptr;  // [3][cap] group sums (two-level ticket path)
  unsigned *gtick = nullptr;  // [cap] group tickets, zero between kernels
  std::vector<Tile> host;
};

}  // namespace

struct b200la_batch_s {
  b200la_ctx ctx;
  b200la_batch_params prm;
  BatchParams kp;
  int capacity;
  std::vector<HostSys> sys;
  // item lists of K1 (SpMV, residual), K2 (update + dots), K3 (direction)
  ItemList lst[3];
  int *sysfirst;      // device [capacity][3]: each system's first item in each list
  std::vector<int> sysfirst_host;
  unsigned pass_total; // passes since creation, as the device last reported it
  bool adaptive;      // shrink items when few rows are running
  int warps[3];       // resident warps of each pass kernel's grid (0 = not yet known)
  // device
  void *desc;         // SysDesc<T>[capacity]
  SysState *st;       // [capacity]
  BatchGlobals *glob;
  CsrCheck *chk;       // device verdicts of the checks, one per system of an add
  CsrCheck *chk_host;  // pinned mirror
  int chk_cap;
  // per-add job lists (check jobs, then setup jobs): pinned host staging and
  // its device copy, chk_cap entries of each
  void *jobs_host;
  void *jobs_dev;
  // host mirrors
  SysState *st_host;  // pinned [capacity]
  BatchGlobals *glob_host;
  int64_t device_bytes;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  // adds run on their own stream, so they overlap a launch in flight on the
  // context stream; the context stream waits for xfer_done before later work
  cudaStream_t xfer;
  cudaEvent_t xfer_done;
  // a removal clears slot states on the context stream, after any launch in
  // flight that may still read them; the next add (on xfer) waits for it
  // before it writes a reused slot's descriptor and fresh state
  cudaEvent_t rm_done;
  bool rm_pending;
  bool xfer_copies;   // solution copies queued on xfer since its last wait
  bool in_flight;     // a b200la_batch_launch not yet completed
};

namespace {

using BatchHandle = b200la_batch;

template <typename T> SysDesc<T> &desc_of(HostSys &h);
template <> SysDesc<double> &desc_of<double>(HostSys &h) { return h.d64; }
template <> SysDesc<float> &desc_of<float>(HostSys &h) { return h.d32; }

// Bytes of a slot's two allocations: the CSR as uploaded plus the vectors,
// and the sliced-ELL copy.  Their sum is the admission test of the request loop.
size_t csr_part_bytes(int64_t n, int64_t nnz, bool mixed) {
  const size_t tb = mixed ? 4 : 8;
  size_t b = align256(sizeof(int) * (n + 1)) + align256(sizeof(int) * nnz) + align256(8 * nnz);
  b += 2 * align256(8 * n);   // b, x
  b += 5 * align256(tb * n);  // c, r, p, Ap, invd
  return b;
}
size_t sell_part_bytes(int64_t n, int64_t ell, bool mixed, bool col16, bool stencil = false) {
  const size_t tb = mixed ? 4 : 8;
  const size_t padded = (size_t)((n + 31) / 32) * 32 * (size_t)ell;
  size_t b = (stencil ? 0 : align256((col16 ? 2 : 4) * padded)) + align256(tb * padded);  // columns and values
  if (mixed) b += align256(8 * padded);                                     // FP64 values (residual)
  return b;
}
size_t slot_bytes(int64_t n, int64_t nnz, int64_t ell, bool mixed, bool col16 = false) {
  return csr_part_bytes(n, nnz, mixed) + sell_part_bytes(n, ell, mixed, col16);
}

// Allocates a slot's CSR part (one chunk: CSR as uploaded, b, x and the
// work vectors) and carves it into a descriptor.
template <typename T>
int alloc_csr_part(BatchHandle B, int slot, int n, int64_t nnz, SysDesc<T> *out) {
  HostSys &h = B->sys[slot];
  cudaStream_t st = B->xfer;
  const bool mixed = B->kp.mixed != 0;
  const size_t bytes = csr_part_bytes(n, nnz, mixed);
  B_CUDA(cudaMallocAsync(&h.chunk, bytes, st));
  h.bytes = bytes;
  char *p = (char *)h.chunk;
  auto take = [&](size_t nb) { char *q = p; p += align256(nb); return (void *)q; };
  SysDesc<T> d{};
  d.n = n;
  d.nnz = (int)nnz;
  d.rowptr = (const int *)take(sizeof(int) * (n + 1));
  d.col = (const int *)take(sizeof(int) * nnz);
  d.val64 = (const double *)take(8 * nnz);
  d.b = (const double *)take(8 * n);
  d.x = (double *)take(8 * n);
  d.c = (T *)take(sizeof(T) * n);
  d.r = (T *)take(sizeof(T) * n);
  d.p = (T *)take(sizeof(T) * n);
  d.Ap = (T *)take(sizeof(T) * n);
  d.invd = (const T *)take(sizeof(T) * n);
  *out = d;
  return B200LA_OK;
}

// Allocates the sliced-ELL part (second chunk) once ell and the column type
// are known.
// stencil (soff of ell ascending offsets, or null): the values-only layout.
template <typename T>
int alloc_sell_part(BatchHandle B, int slot, int ell, bool col16, SysDesc<T> &d, cudaStream_t st,
                    const int *stencil = nullptr) {
  HostSys &h = B->sys[slot];
  const bool mixed = B->kp.mixed != 0;
  const size_t bytes = sell_part_bytes(d.n, ell, mixed, col16, stencil != nullptr);
  B_CUDA(cudaMallocAsync(&h.chunk2, bytes, st));
  h.bytes += bytes;
  char *p = (char *)h.chunk2;
  auto take = [&](size_t nb) { char *q = p; p += align256(nb); return (void *)q; };
  const size_t padded = (size_t)((d.n + 31) / 32) * 32 * (size_t)ell;
  d.ell = ell;
  d.col16 = col16 ? 1 : 0;
  d.stencil = stencil ? 1 : 0;
  for (int k = 0; k < kMaxStencil; ++k) d.soff[k] = stencil && k < ell ? stencil[k] : 0;
  d.scol = stencil ? nullptr : take((col16 ? 2 : 4) * padded);
  d.sval = (const T *)take(sizeof(T) * padded);
  d.sval64 = mixed ? (const double *)take(8 * padded) : (const double *)d.sval;
  return B200LA_OK;
}

void free_slot_memory(BatchHandle B, HostSys &h) {
  cudaStream_t st = B->ctx->stream;
  if (h.chunk) cudaFreeAsync(h.chunk, st);
  if (h.chunk2) cudaFreeAsync(h.chunk2, st);
  h.chunk = h.chunk2 = nullptr;
}

// Uploads the descriptor and a fresh RESID state, then builds the sliced-ELL
// copies, the inverse diagonal and zero work vectors on the device.
template <typename T>
int finish_slot(BatchHandle B, int slot, const SysDesc<T> &d, cudaStream_t st) {
  HostSys &h = B->sys[slot];
  desc_of<T>(h) = d;
  SysState &s0 = B->st_host[slot];
  memset(&s0, 0, sizeof(SysState));
  s0.phase = PH_RESID;
  s0.bad_row = 0xffffffffu;
  B_CUDA(cudaMemcpyAsync(B->st + slot, &s0, sizeof(SysState), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync((SysDesc<T> *)B->desc + slot, &desc_of<T>(h), sizeof(SysDesc<T>), cudaMemcpyHostToDevice,
                         st));
  const int64_t work = (int64_t)d.n + 32;
  const int grid = (int)std::min<int64_t>(std::max<int64_t>((work + kBlock - 1) / kBlock, 1),
                                          (int64_t)B->ctx->num_sms * 8);
  slot_setup_kernel<T><<<grid, kBlock, 0, st>>>(d, &B->st[slot].bad_row);
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

// Uploading a host CSR system into a slot, in two stages: (1) the CSR part
// is allocated and copied, and a device check (those of validate_csr, plus
// the longest row and the largest |column - row|) writes its verdict to
// `chk`; (2) after the caller has read the verdict back, the sliced-ELL part
// is sized and built, or the error is reported.  One small read-back per
// system (or per bulk add) replaces two O(nnz) host passes.
// Allocates a slot's CSR part and queues the copies of its arrays (x stays
// for the setup kernel to zero when no x0 is given).
template <typename T>
int upload_stage(BatchHandle B, int slot, int n, int64_t nnz, const int *rowptr, const int *col, const double *val,
                 const double *b, const double *x0, SysDesc<T> *d) {
  cudaStream_t st = B->xfer;
  B_TRY(alloc_csr_part<T>(B, slot, n, nnz, d));
  B_CUDA(cudaMemcpyAsync((void *)d->rowptr, rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
  if (nnz) {
    B_CUDA(cudaMemcpyAsync((void *)d->col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    B_CUDA(cudaMemcpyAsync((void *)d->val64, val, 8 * nnz, cudaMemcpyHostToDevice, st));
  }
  B_CUDA(cudaMemcpyAsync((void *)d->b, b, 8 * n, cudaMemcpyHostToDevice, st));
  if (x0) B_CUDA(cudaMemcpyAsync(d->x, x0, 8 * n, cudaMemcpyHostToDevice, st));
  return B200LA_OK;
}

template <typename T>
int finish_stage(BatchHandle B, int slot, const CsrCheck &c, SysDesc<T> &d) {
  if (c.err != ~0ull) {
    const int row = (int)(c.err >> 8), code = (int)(c.err & 0xff);
    if (code == kChkStart)
      return fail(B200LA_ERR_MATRIX, "csr: rowptr[0] != 0 or rowptr[nrow] != nnz %d", d.nnz);
    if (code == kChkDecrease) return fail(B200LA_ERR_MATRIX, "csr: rowptr decreases at row %d", row);
    if (code == kChkBounds) return fail(B200LA_ERR_MATRIX, "csr: rowptr out of [0, nnz] at row %d", row);
    return fail(B200LA_ERR_MATRIX, "csr: a column of row %d is out of range [0,%d)", row, d.n);
  }
  const bool col16 = B->prm.index_bits != 32 && c.max_off <= 32767;
  // values-only layout when every row fits the system's stencil (index_bits 0)
  const bool stencil = B->prm.index_bits == 0 && c.stencil && c.slen >= c.max_row && c.slen > 0;
  B_TRY(alloc_sell_part<T>(B, slot, stencil ? c.slen : std::max(c.max_row, 1), col16, d, B->xfer,
                           stencil ? c.soff : nullptr));
  d.max_off = c.max_off;
  return B200LA_OK;
}

// Grows the per-batch check records (device and pinned host) to `count`.
size_t jobs_bytes(int cap) {
  return align256(sizeof(CheckJob) * cap) + sizeof(SetupJob<double>) * (size_t)cap;
}

int ensure_checks(BatchHandle B, int count) {
  if (count <= B->chk_cap) return B200LA_OK;
  cudaStream_t st = B->xfer;
  const int cap = std::max(count, 2 * B->chk_cap);
  // pinned buffers are freed only after the copies queued from them
  B_CUDA(cudaStreamSynchronize(st));
  if (B->chk) cudaFreeAsync(B->chk, st);
  if (B->chk_host) cudaFreeHost(B->chk_host);
  if (B->jobs_dev) cudaFreeAsync(B->jobs_dev, st);
  if (B->jobs_host) cudaFreeHost(B->jobs_host);
  B->chk = nullptr;
  B->chk_host = nullptr;
  B->jobs_dev = B->jobs_host = nullptr;
  B->chk_cap = 0;
  B_CUDA(cudaMallocAsync(&B->chk, sizeof(CsrCheck) * cap, st));
  B_CUDA(cudaMallocHost(&B->chk_host, sizeof(CsrCheck) * cap));
  B_CUDA(cudaMallocAsync(&B->jobs_dev, jobs_bytes(cap), st));
  B_CUDA(cudaMallocHost(&B->jobs_host, jobs_bytes(cap)));
  B->chk_cap = cap;
  return B200LA_OK;
}

// Q1 rows couple nodes at most one cell away: largest |column - row| is
// m + 1 in 2D and m^2 + m + 1 in 3D, with m = cells + 1 nodes per axis.
int64_t q1_max_off(int dim, int cells) {
  const int64_t m = (int64_t)cells + 1;
  return dim == 2 ? m + 1 : m * m + m + 1;
}
bool q1_col16(int dim, int cells) { return q1_max_off(dim, cells) <= 32767; }

int kernel_grid(b200la_ctx c, const void *k, int *grid) {
  int o = 0;
  B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k, kBlock, 0));
  *grid = c->num_sms * std::max(o, 1);
  return B200LA_OK;
}

template <typename T, bool PRE, bool IN_GRAPH>
int pass_grids(BatchHandle B, int g[3]) {
  b200la_ctx c = B->ctx;
  B_TRY(kernel_grid(c, (const void *)batch_spmv_kernel<T, PRE>, &g[0]));
  B_TRY(kernel_grid(c, (const void *)batch_update_kernel<T, PRE>, &g[1]));
  B_TRY(kernel_grid(c, (const void *)batch_direction_kernel<T, PRE, IN_GRAPH>, &g[2]));
  return B200LA_OK;
}

// Resident warps of each pass kernel's grid (the adaptive item rule).
int grid_warps(BatchHandle B) {
  int g[3] = {1, 1, 1};
  const bool pre = B->kp.precond != 0;
  int rc;
  if (B->kp.mixed) rc = pre ? pass_grids<float, true, true>(B, g) : pass_grids<float, false, true>(B, g);
  else rc = pre ? pass_grids<double, true, true>(B, g) : pass_grids<double, false, true>(B, g);
  B_TRY(rc);
  for (int k = 0; k < 3; ++k) B->warps[k] = g[k] * (kBlock / 32);
  return B200LA_OK;
}

// The three lists as the pass kernels' argument.
PassLists pass_lists(BatchHandle B) {
  PassLists L;
  for (int k = 0; k < 3; ++k) {
    L.tiles[k] = B->lst[k].dev;
    L.part[k] = B->lst[k].part;
    L.gpart[k] = B->lst[k].gpart;
    L.gtick[k] = B->lst[k].gtick;
    L.stride[k] = B->lst[k].cap;
  }
  L.sysfirst = B->sysfirst;
  return L;
}

// One pass (K1 K2 K3) on stream st: captured into the graph body, or
// launched from the host loop when graphs are off.
template <typename T, bool PRE, bool IN_GRAPH>
void launch_pass(BatchHandle B, const int g[3], cudaStream_t st, cudaGraphConditionalHandle h) {
  const SysDesc<T> *desc = (const SysDesc<T> *)B->desc;
  const PassLists L = pass_lists(B);
  batch_spmv_kernel<T, PRE><<<g[0], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp);
  batch_update_kernel<T, PRE><<<g[1], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp);
  batch_direction_kernel<T, PRE, IN_GRAPH><<<g[2], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp, h);
}

// Graph: start kernel -> WHILE(pass).
template <typename T, bool PRE>
int build_graph_t(BatchHandle B) {
  if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
  if (B->graph) { cudaGraphDestroy(B->graph); B->graph = nullptr; }
  int grids[3] = {1, 1, 1};
  B_TRY((pass_grids<T, PRE, true>(B, grids)));
  cudaGraph_t g;
  B_CUDA(cudaGraphCreate(&g, 0));
  B->graph = g;
  cudaGraphConditionalHandle h;
  B_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaStream_t cs;
  B_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  B_CUDA(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  batch_start_kernel<<<1, 1, 0, cs>>>(B->glob);
  cudaGraph_t cap;
  cudaError_t e1 = cudaStreamEndCapture(cs, &cap);
  if (e1 != cudaSuccess) {
    cudaStreamDestroy(cs);
    B_CUDA(e1);
  }
  size_t nn = 0;
  B_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  B_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t wnode;
  B_CUDA(cudaGraphAddNode(&wnode, g, nodes.data(), nn, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  B_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_pass<T, PRE, true>(B, grids, cs, h);
  cudaError_t e2 = cudaStreamEndCapture(cs, &cap);
  cudaStreamDestroy(cs);
  B_CUDA(e2);
  B_CUDA(cudaGraphInstantiate(&B->exec, g, 0));
  return B200LA_OK;
}

int build_graph(BatchHandle B) {
  const bool pre = B->kp.precond != 0;
  if (B->kp.mixed) return pre ? build_graph_t<float, true>(B) : build_graph_t<float, false>(B);
  return pre ? build_graph_t<double, true>(B) : build_graph_t<double, false>(B);
}

// Host-loop mode (graphs off, B200LA_GRAPHS=0): the same kernels, with the
// pass budget and the running count checked from the host every 8 passes.
template <typename T, bool PRE>
int host_loop_t(BatchHandle B) {
  cudaStream_t st = B->ctx->stream;
  int grids[3] = {1, 1, 1};
  B_TRY((pass_grids<T, PRE, false>(B, grids)));
  batch_start_kernel<<<1, 1, 0, st>>>(B->glob);
  for (;;) {
    for (int k = 0; k < 8; ++k) launch_pass<T, PRE, false>(B, grids, st, 0);
    B_CUDA(cudaGetLastError());
    B_CUDA(cudaMemcpyAsync(B->glob_host, B->glob, sizeof(BatchGlobals), cudaMemcpyDeviceToHost, st));
    B_CUDA(cudaStreamSynchronize(st));
    if (B->glob_host->active <= 0 || B->glob_host->passes >= B->glob_host->max_passes) break;
  }
  return B200LA_OK;
}

int host_loop(BatchHandle B) {
  const bool pre = B->kp.precond != 0;
  if (B->kp.mixed) return pre ? host_loop_t<float, true>(B) : host_loop_t<float, false>(B);
  return pre ? host_loop_t<double, true>(B) : host_loop_t<double, false>(B);
}

// Grows list k's item and partial arrays to hold nt items (the graph bakes
// their addresses in, so it is rebuilt after a reallocation).
int ensure_items(BatchHandle B, int k, int64_t nt) {
  ItemList &L = B->lst[k];
  if (nt <= L.cap) return B200LA_OK;
  cudaStream_t st = B->ctx->stream;
  const int64_t cap = std::max<int64_t>(nt, 2 * L.cap);
  if (L.dev) cudaFreeAsync(L.dev, st);
  if (L.part) cudaFreeAsync(L.part, st);
  if (L.gpart) cudaFreeAsync(L.gpart, st);
  if (L.gtick) cudaFreeAsync(L.gtick, st);
  L.dev = nullptr;
  L.part = L.gpart = nullptr;
  L.gtick = nullptr;
  L.cap = 0;
  B_CUDA(cudaMallocAsync(&L.dev, sizeof(Tile) * cap, st));
  B_CUDA(cudaMallocAsync(&L.part, sizeof(double) * 3 * cap, st));
  B_CUDA(cudaMallocAsync(&L.gpart, sizeof(double) * 3 * cap, st));
  B_CUDA(cudaMallocAsync(&L.gtick, sizeof(unsigned) * cap, st));
  B_CUDA(cudaMemsetAsync(L.gtick, 0, sizeof(unsigned) * cap, st));
  L.cap = cap;
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  return B200LA_OK;
}

// Both item lists over the given slots (all used slots, or only those still
// running); writes the slot count and the SpMV's algorithmic bytes.
int upload_tiles(BatchHandle B, bool running_only, int *count, int64_t *alg_bytes) {
  for (ItemList &L : B->lst) L.host.clear();
  int act = 0;
  int64_t bytes = 0;
  const int64_t vb = B->kp.mixed ? 4 : 8;
  std::vector<int> run;
  for (int s = 0; s < B->capacity; ++s) {
    const HostSys &h = B->sys[s];
    if (!h.used) continue;
    const int ph = B->st_host[s].phase;
    if (running_only && (ph == PH_DONE || ph == PH_EMPTY)) continue;
    ++act;
    run.push_back(s);
    bytes += (int64_t)h.nnz * (vb + 4) + (int64_t)(h.n + 1) * 4 + 2 * (int64_t)h.n * vb;
  }
  if (B->adaptive && !B->warps[0]) B_TRY(grid_warps(B));
  for (int k = 0; k < 3; ++k) {
    ItemList &L = B->lst[k];
    // adaptive: halve the item (down to one 32-row slice) while the list
    // would give the kernel's warps fewer than one item each, so a lightly
    // loaded pass is not bound by one warp's long serial chain
    int rows = L.rows;
    if (B->adaptive)
      while (rows > 32) {
        int64_t items = 0;
        for (int s : run) items += (B->sys[s].n + rows - 1) / rows;
        if (items >= (int64_t)B->warps[k]) break;
        rows = std::max(32, (rows / 2) & ~31);
      }
    L.used = rows;
    for (int s : run) {
      const int n = B->sys[s].n;
      const int first = (int)L.host.size();
      B->sysfirst_host[3 * s + k] = first;
      // the system's items in the previous kernel's list (K1: its own)
      const int pk = k == 0 ? 0 : k - 1;
      const int pfirst = k == 0 ? first : B->sysfirst_host[3 * s + pk];
      const int prows = k == 0 ? rows : B->lst[pk].used;
      const int pcount = (n + prows - 1) / prows;
      for (int row0 = 0; row0 < n; row0 += rows) L.host.push_back(Tile{s, row0, pfirst, pcount});
    }
  }
  cudaStream_t st = B->ctx->stream;
  for (int k = 0; k < 3; ++k) {
    ItemList &L = B->lst[k];
    const int64_t nt = (int64_t)L.host.size();
    B_TRY(ensure_items(B, k, nt));
    if (nt) B_CUDA(cudaMemcpyAsync(L.dev, L.host.data(), sizeof(Tile) * nt, cudaMemcpyHostToDevice, st));
  }
  B_CUDA(cudaMemcpyAsync(B->sysfirst, B->sysfirst_host.data(), sizeof(int) * 3 * B->capacity,
                         cudaMemcpyHostToDevice, st));
  // the staging vectors must outlive the copies
  B_CUDA(cudaStreamSynchronize(st));
  *count = act;
  if (alg_bytes) *alg_bytes = bytes;
  return B200LA_OK;
}

// Host globals of a launch over the current lists.
void set_globals(BatchHandle B, int active, int max_passes) {
  BatchGlobals &g = *B->glob_host;
  memset(&g, 0, sizeof(g));
  g.active = active;
  g.max_passes = max_passes;
  g.pass_total = B->pass_total;
  for (int k = 0; k < 3; ++k) {
    g.ntiles[k] = (int)B->lst[k].host.size();
    g.tile_rows[k] = B->lst[k].used;
  }
}

int find_free_slot(BatchHandle B) {
  for (int s = 0; s < B->capacity; ++s)
    if (!B->sys[s].used) return s;
  return -1;
}

template <typename T>
int time_plain(BatchHandle B, int reps, float *ms) {
  cudaStream_t st = B->ctx->stream;
  const ItemList &L = B->lst[0];
  const int nt = (int)L.host.size();
  int grid = 1;
  B_TRY(kernel_grid(B->ctx, (const void *)batch_spmv_plain_kernel<T>, &grid));
  const SysDesc<T> *desc = (const SysDesc<T> *)B->desc;
  batch_spmv_plain_kernel<T><<<grid, kBlock, 0, st>>>(L.dev, nt, L.used, desc);
  cudaEvent_t e0, e1;
  B_CUDA(cudaEventCreate(&e0));
  B_CUDA(cudaEventCreate(&e1));
  B_CUDA(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r) batch_spmv_plain_kernel<T><<<grid, kBlock, 0, st>>>(L.dev, nt, L.used, desc);
  B_CUDA(cudaEventRecord(e1, st));
  B_CUDA(cudaEventSynchronize(e1));
  B_CUDA(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B_CUDA(cudaGetLastError());
  *ms /= reps;
  return B200LA_OK;
}

// Pass timing (instrumentation and the tuner): over the current item list,
// one untimed pass, then `reps` passes timed kernel by kernel with CUDA
// events on the context stream; ms[k] is the mean time of K1/K2/K3.  The
// passes advance the systems like a run does.
template <typename T, bool PRE>
int time_passes_t(BatchHandle B, int reps, double ms[3]) {
  cudaStream_t st = B->ctx->stream;
  // `active` is only read by the end-of-pass test, which host mode ignores
  set_globals(B, B->capacity, 1 << 30);
  B_CUDA(cudaMemcpyAsync(B->glob, B->glob_host, sizeof(BatchGlobals), cudaMemcpyHostToDevice, st));
  int grids[3] = {1, 1, 1};
  B_TRY((pass_grids<T, PRE, false>(B, grids)));
  const SysDesc<T> *desc = (const SysDesc<T> *)B->desc;
  const PassLists L = pass_lists(B);
  batch_start_kernel<<<1, 1, 0, st>>>(B->glob);
  launch_pass<T, PRE, false>(B, grids, st, 0);
  // every timed pass is queued before the wait (behind the untimed pass
  // above), so the kernels run back to back and no host launch gap falls
  // between an event pair
  std::vector<cudaEvent_t> ev((size_t)reps * 4);
  for (auto &e : ev) B_CUDA(cudaEventCreate(&e));
  double acc[3] = {0.0, 0.0, 0.0};
  int rc = B200LA_OK;
  for (int r = 0; r < reps; ++r) {
    cudaEvent_t *e = &ev[(size_t)r * 4];
    cudaEventRecord(e[0], st);
    batch_spmv_kernel<T, PRE><<<grids[0], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp);
    cudaEventRecord(e[1], st);
    batch_update_kernel<T, PRE><<<grids[1], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp);
    cudaEventRecord(e[2], st);
    batch_direction_kernel<T, PRE, false><<<grids[2], kBlock, 0, st>>>(L, desc, B->st, B->glob, B->kp, 0);
    cudaEventRecord(e[3], st);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    rc = fail(B200LA_ERR_CUDA, "batch pass timing: %s", cudaGetErrorString(cudaGetLastError()));
  } else {
    for (int r = 0; r < reps; ++r)
      for (int k = 0; k < 3; ++k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[(size_t)r * 4 + k], ev[(size_t)r * 4 + k + 1]);
        acc[k] += t;
      }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  B_TRY(rc);
  B_CUDA(cudaGetLastError());
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / reps;
  return B200LA_OK;
}

// Device copy of every used slot's carried state (SysState array and the
// x, c, r, p vectors), for the tuner.
struct Snapshot {
  SysState *st = nullptr;
  void *buf = nullptr;  // [slots int][offs int64][x double][c r p T]
  int nslots = 0;
};

template <typename T>
int snapshot_copy_t(BatchHandle B, const Snapshot &sn, int save) {
  const int *slots = (const int *)sn.buf;
  const int64_t *offs = (const int64_t *)((char *)sn.buf + align256(sizeof(int) * sn.nslots));
  double *xs = (double *)((char *)offs + align256(sizeof(int64_t) * sn.nslots));
  int64_t n = 0;
  for (const HostSys &h : B->sys)
    if (h.used) n += h.n;
  T *vs = (T *)((char *)xs + align256(sizeof(double) * n));
  slot_snapshot_kernel<T><<<sn.nslots, kBlock, 0, B->ctx->stream>>>(slots, offs, (const SysDesc<T> *)B->desc, xs,
                                                                      vs, save);
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

void snapshot_free(BatchHandle B, Snapshot *sn) {
  cudaStream_t st = B->ctx->stream;
  if (sn->st) cudaFreeAsync(sn->st, st);
  if (sn->buf) cudaFreeAsync(sn->buf, st);
  cudaStreamSynchronize(st);
  *sn = Snapshot();
}

int snapshot_save(BatchHandle B, Snapshot *sn) {
  cudaStream_t st = B->ctx->stream;
  std::vector<int> slots;
  std::vector<int64_t> offs;
  int64_t n = 0;
  for (int s = 0; s < B->capacity; ++s)
    if (B->sys[s].used) {
      slots.push_back(s);
      offs.push_back(n);
      n += B->sys[s].n;
    }
  sn->nslots = (int)slots.size();
  if (!sn->nslots) return B200LA_OK;
  const size_t tb = B->kp.mixed ? 4 : 8;
  const size_t bytes = align256(sizeof(int) * slots.size()) + align256(sizeof(int64_t) * slots.size()) +
                       align256(sizeof(double) * n) + 3 * tb * (size_t)n;
  if (cudaMallocAsync(&sn->st, sizeof(SysState) * B->capacity, st) != cudaSuccess ||
      cudaMallocAsync(&sn->buf, bytes, st) != cudaSuccess) {
    snapshot_free(B, sn);
    return fail(B200LA_ERR_NOMEM, "batch_tune: no room for the state snapshot (%zu bytes)", bytes);
  }
  const int64_t *doffs = (const int64_t *)((char *)sn->buf + align256(sizeof(int) * slots.size()));
  B_CUDA(cudaMemcpyAsync(sn->buf, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync((void *)doffs, offs.data(), sizeof(int64_t) * offs.size(), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync(sn->st, B->st, sizeof(SysState) * B->capacity, cudaMemcpyDeviceToDevice, st));
  B_TRY(B->kp.mixed ? snapshot_copy_t<float>(B, *sn, 1) : snapshot_copy_t<double>(B, *sn, 1));
  // the host vectors must outlive the copies
  B_CUDA(cudaStreamSynchronize(st));
  return B200LA_OK;
}

int snapshot_restore(BatchHandle B, const Snapshot &sn) {
  if (!sn.nslots) return B200LA_OK;
  cudaStream_t st = B->ctx->stream;
  B_CUDA(cudaMemcpyAsync(B->st, sn.st, sizeof(SysState) * B->capacity, cudaMemcpyDeviceToDevice, st));
  B_TRY(B->kp.mixed ? snapshot_copy_t<float>(B, sn, 0) : snapshot_copy_t<double>(B, sn, 0));
  B_CUDA(cudaStreamSynchronize(st));
  return B200LA_OK;
}

// Removals clear slot states on the context stream (after a launch in flight
// that may still read them); adds run on the transfer stream.  A removal
// records rm_done, and the next add makes the transfer stream wait for it, so
// a reused slot's descriptor and fresh state are written after the removed
// system's state was cleared and after every kernel that could read it.
int note_removal(BatchHandle B) {
  B_CUDA(cudaEventRecord(B->rm_done, B->ctx->stream));
  B->rm_pending = true;
  return B200LA_OK;
}

int order_after_removals(BatchHandle B) {
  if (!B->rm_pending) return B200LA_OK;
  B_CUDA(cudaStreamWaitEvent(B->xfer, B->rm_done, 0));
  B->rm_pending = false;
  return B200LA_OK;
}

// Adds `count` host CSR systems: every system's copies and device check are
// queued first, the verdicts are read back with one wait, then each valid
// system gets its sliced-ELL part.  status[k] is each system's outcome; the
// return value is the first failure's (its message stays in last_error).
template <typename T>
int add_many_t(BatchHandle B, int count, const int *n, const int64_t *nnz, const int *const *rowptr,
               const int *const *col, const double *const *val, const double *const *rhs,
               const double *const *x0, int *slots, int *status) {
  // all of an add runs on the transfer stream: it overlaps a launch in flight
  cudaStream_t st = B->xfer;
  B_TRY(order_after_removals(B));
  B_TRY(ensure_checks(B, count));
  csr_check_init_kernel<<<std::max(1, std::min((count + kBlock - 1) / kBlock, 64)), kBlock, 0, st>>>(count, B->chk);
  B_CUDA(cudaGetLastError());
  std::vector<int> sl(count, -1);
  std::vector<SysDesc<T>> d(count);
  int first = B200LA_OK;
  std::string first_msg;
  auto note = [&](int k, int rc) {
    status[k] = rc;
    if (first == B200LA_OK && rc != B200LA_OK) {
      first = rc;
      first_msg = b200la_last_error();
    }
  };
  for (int k = 0; k < count; ++k) {
    slots[k] = -1;
    status[k] = B200LA_OK;
    int rc = B200LA_OK;
    if (n[k] <= 0) rc = fail(B200LA_ERR_INVALID, "batch_add: empty system");
    else if (nnz[k] < 0 || nnz[k] >= (int64_t)INT32_MAX)
      rc = fail(B200LA_ERR_MATRIX, "csr: nnz %lld exceeds int32 indexing", (long long)nnz[k]);
    else if (!rowptr[k]) rc = fail(B200LA_ERR_MATRIX, "csr: rowptr is NULL");
    else if (nnz[k] && (!col[k] || !val[k])) rc = fail(B200LA_ERR_MATRIX, "csr: col or val is NULL");
    else if (!rhs[k]) rc = fail(B200LA_ERR_INVALID, "batch_add: rhs is NULL");
    if (rc != B200LA_OK) {
      note(k, rc);
      continue;
    }
    const int slot = find_free_slot(B);
    if (slot < 0) {
      note(k, fail(B200LA_ERR_NOMEM, "batch_add: all %d slots are in use", B->capacity));
      continue;
    }
    HostSys &h = B->sys[slot];
    h = HostSys();
    h.n = n[k];
    h.nnz = (int)nnz[k];
    h.used = true;  // reserved while its copies and check are in flight
    rc = upload_stage<T>(B, slot, n[k], nnz[k], rowptr[k], col[k], val[k], rhs[k], x0 ? x0[k] : nullptr, &d[k]);
    if (rc != B200LA_OK) {
      free_slot_memory(B, h);
      h = HostSys();
      note(k, rc);
      continue;
    }
    sl[k] = slot;
  }
  // one check kernel over every uploaded system (the previous add's copies
  // out of the staging buffer finished at its wait below)
  CheckJob *cj = (CheckJob *)B->jobs_host;
  int max_n = 1;
  for (int k = 0; k < count; ++k) {
    cj[k] = sl[k] < 0 ? CheckJob{nullptr, nullptr, 0, 0} : CheckJob{d[k].rowptr, d[k].col, d[k].n, d[k].nnz};
    if (sl[k] >= 0) max_n = std::max(max_n, d[k].n);
  }
  B_CUDA(cudaMemcpyAsync(B->jobs_dev, cj, sizeof(CheckJob) * count, cudaMemcpyHostToDevice, st));
  {
    const dim3 grid((unsigned)std::min((max_n + kBlock - 1) / kBlock, 64), (unsigned)std::min(count, 65535));
    csr_check_many_kernel<<<grid, kBlock, 0, st>>>((const CheckJob *)B->jobs_dev, count, B->chk);
    B_CUDA(cudaGetLastError());
  }
  B_CUDA(cudaMemcpyAsync(B->chk_host, B->chk, sizeof(CsrCheck) * count, cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  SetupJob<T> *sj = (SetupJob<T> *)((char *)B->jobs_host + align256(sizeof(CheckJob) * B->chk_cap));
  int nsetup = 0;
  max_n = 1;
  for (int k = 0; k < count; ++k) {
    if (sl[k] < 0) continue;
    HostSys &h = B->sys[sl[k]];
    const int rc = finish_stage<T>(B, sl[k], B->chk_host[k], d[k]);
    if (rc != B200LA_OK) {
      free_slot_memory(B, h);
      h = HostSys();
      note(k, rc);
      continue;
    }
    desc_of<T>(h) = d[k];
    SysState &s0 = B->st_host[sl[k]];
    memset(&s0, 0, sizeof(SysState));
    s0.phase = PH_RESID;
    s0.bad_row = 0xffffffffu;
    sj[nsetup++] = SetupJob<T>{d[k], sl[k], (x0 && x0[k]) ? 0 : 1};
    max_n = std::max(max_n, d[k].n);
    B->device_bytes += (int64_t)h.bytes;
    slots[k] = sl[k];
  }
  if (nsetup) {
    // descriptors, fresh states, sliced-ELL copies, inverse diagonals and
    // zero vectors of every added system in two launches
    void *sj_dev = (char *)B->jobs_dev + align256(sizeof(CheckJob) * B->chk_cap);
    B_CUDA(cudaMemcpyAsync(sj_dev, sj, sizeof(SetupJob<T>) * nsetup, cudaMemcpyHostToDevice, st));
    slot_init_many_kernel<T><<<(nsetup + kBlock - 1) / kBlock, kBlock, 0, st>>>(
        (const SetupJob<T> *)sj_dev, nsetup, (SysDesc<T> *)B->desc, B->st);
    const dim3 grid((unsigned)std::min((max_n + 32 + kBlock - 1) / kBlock, 256), (unsigned)std::min(nsetup, 65535));
    slot_setup_many_kernel<T><<<grid, kBlock, 0, st>>>((const SetupJob<T> *)sj_dev, nsetup, B->st);
    B_CUDA(cudaGetLastError());
  }
  // later work on the context stream (runs, results, removals) follows the add
  B_CUDA(cudaEventRecord(B->xfer_done, st));
  B_CUDA(cudaStreamWaitEvent(B->ctx->stream, B->xfer_done, 0));
  if (first != B200LA_OK) set_error(first_msg);
  return first;
}

int wait_early_copies(b200la_batch B);

}  // namespace

extern "C" {

int b200la_batch_slot_bytes(int64_t n, int64_t nnz, int max_row, int mixed, int64_t *bytes) {
  B_CHECK(bytes && n >= 0 && nnz >= 0 && max_row >= 0, B200LA_ERR_INVALID, "batch_slot_bytes: bad argument");
  *bytes = (int64_t)slot_bytes(n, nnz, std::max(max_row, 1), mixed != 0);
  return B200LA_OK;
}

int b200la_batch_destroy(b200la_batch B) {
  if (!B) return B200LA_OK;
  cudaStream_t st = B->ctx->stream;
  if (B->xfer) cudaStreamSynchronize(B->xfer);
  cudaStreamSynchronize(st);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  for (HostSys &h : B->sys) free_slot_memory(B, h);
  void *bufs[] = {B->desc, B->st, B->glob, B->chk, B->sysfirst};
  for (void *p : bufs)
    if (p) cudaFreeAsync(p, st);
  for (ItemList &L : B->lst) {
    if (L.dev) cudaFreeAsync(L.dev, st);
    if (L.part) cudaFreeAsync(L.part, st);
    if (L.gpart) cudaFreeAsync(L.gpart, st);
    if (L.gtick) cudaFreeAsync(L.gtick, st);
  }
  if (B->jobs_dev) cudaFreeAsync(B->jobs_dev, st);
  if (B->st_host) cudaFreeHost(B->st_host);
  if (B->chk_host) cudaFreeHost(B->chk_host);
  if (B->jobs_host) cudaFreeHost(B->jobs_host);
  if (B->glob_host) cudaFreeHost(B->glob_host);
  cudaStreamSynchronize(st);
  if (B->xfer_done) cudaEventDestroy(B->xfer_done);
  if (B->rm_done) cudaEventDestroy(B->rm_done);
  if (B->xfer) cudaStreamDestroy(B->xfer);
  {
    // return the pool's free blocks to the driver (the context keeps freed
    // blocks while batches add and remove systems)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, B->ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  }
  delete B;
  return B200LA_OK;
}

int b200la_batch_create(b200la_ctx ctx, const b200la_batch_params *p, b200la_batch *out) {
  B_CHECK(ctx && p && out, B200LA_ERR_INVALID, "batch_create: null argument");
  B_CHECK(p->capacity > 0 && p->capacity <= (1 << 20), B200LA_ERR_INVALID, "batch_create: capacity %d", p->capacity);
  B_CHECK(p->max_outer >= 1 && p->max_outer <= 1000, B200LA_ERR_INVALID, "batch_create: max_outer %d", p->max_outer);
  B_CHECK(p->inner_maxits >= 1 && p->inner_maxits <= 10000000, B200LA_ERR_INVALID, "batch_create: inner_maxits");
  B_CHECK(p->atol >= 0 && p->rtol >= 0 && p->dtol > 0, B200LA_ERR_INVALID, "batch_create: tolerances");
  B_CHECK(!p->mixed || (p->inner_rtol > 0 && p->inner_rtol < 1), B200LA_ERR_INVALID, "batch_create: inner_rtol");
  B_CHECK(p->index_bits == 0 || p->index_bits == 16 || p->index_bits == 32, B200LA_ERR_INVALID,
          "batch_create: index_bits %d (0, 16 or 32)", p->index_bits);
  B_CHECK(p->tile_rows == 0 || (p->tile_rows >= 32 && p->tile_rows <= 65536 && p->tile_rows % 32 == 0),
          B200LA_ERR_INVALID, "batch_create: tile_rows %d (32..65536, multiple of 32)", p->tile_rows);
  b200la_batch B = new b200la_batch_s();
  B->ctx = ctx;
  B->prm = *p;
  B->kp = BatchParams{p->max_outer, p->inner_maxits, p->atol, p->rtol, p->dtol, p->inner_rtol, p->precond ? 1 : 0,
                      p->mixed ? 1 : 0, p->restart_inner ? 1 : 0};
  // K1 sweeps 256-row items (8 slices per warp keep its gather chains
  // short); K2 streams 1024-row items, K3 512; the tuner may change them
  for (int k = 0; k < 3; ++k) B->lst[k].rows = p->tile_rows ? p->tile_rows : kDefaultRows[k];
  B->adaptive = p->adaptive != 0;
  B->capacity = p->capacity;
  B->sys.resize(p->capacity);
  B->sysfirst_host.assign(3 * (size_t)p->capacity, 0);
  cudaStream_t st = ctx->stream;
  const size_t dsz = p->mixed ? sizeof(SysDesc<float>) : sizeof(SysDesc<double>);
  bool ok = cudaStreamCreateWithFlags(&B->xfer, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&B->xfer_done, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&B->rm_done, cudaEventDisableTiming) == cudaSuccess &&
            cudaMallocAsync(&B->desc, dsz * p->capacity, st) == cudaSuccess &&
            cudaMallocAsync(&B->st, sizeof(SysState) * p->capacity, st) == cudaSuccess &&
            cudaMallocAsync(&B->glob, sizeof(BatchGlobals), st) == cudaSuccess &&
            cudaMallocAsync(&B->sysfirst, sizeof(int) * 3 * p->capacity, st) == cudaSuccess &&
            ensure_checks(B, 64) == B200LA_OK &&
            cudaMallocHost(&B->st_host, sizeof(SysState) * p->capacity) == cudaSuccess &&
            cudaMallocHost(&B->glob_host, sizeof(BatchGlobals)) == cudaSuccess;
  if (ok) {
    memset(B->st_host, 0, sizeof(SysState) * p->capacity);
    memset(B->glob_host, 0, sizeof(BatchGlobals));
    ok = cudaMemsetAsync(B->st, 0, sizeof(SysState) * p->capacity, st) == cudaSuccess &&
         cudaMemsetAsync(B->glob, 0, sizeof(BatchGlobals), st) == cudaSuccess &&
         cudaStreamSynchronize(B->xfer) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
  }
  if (!ok) {
    b200la_batch_destroy(B);
    return fail(B200LA_ERR_NOMEM, "batch_create: allocation failed");
  }
  *out = B;
  return B200LA_OK;
}

int b200la_batch_add(b200la_batch B, int n, int64_t nnz, const int *rowptr, const int *col, const double *val,
                     const double *b, const double *x0, int *slot_out) {
  B_CHECK(B && slot_out && b, B200LA_ERR_INVALID, "batch_add: null argument");
  int status = B200LA_OK;
  const double *x0s[1] = {x0};
  return B->kp.mixed ? add_many_t<float>(B, 1, &n, &nnz, &rowptr, &col, &val, &b, x0s, slot_out, &status)
                     : add_many_t<double>(B, 1, &n, &nnz, &rowptr, &col, &val, &b, x0s, slot_out, &status);
}

int b200la_batch_add_many(b200la_batch B, int count, const int *n, const int64_t *nnz, const int *const *rowptr,
                          const int *const *col, const double *const *val, const double *const *rhs,
                          const double *const *x0, int *slots, int *status) {
  B_CHECK(B && count >= 0 && (count == 0 || (n && nnz && rowptr && col && val && rhs && slots && status)),
          B200LA_ERR_INVALID, "batch_add_many: null argument");
  if (count == 0) return B200LA_OK;
  return B->kp.mixed ? add_many_t<float>(B, count, n, nnz, rowptr, col, val, rhs, x0, slots, status)
                     : add_many_t<double>(B, count, n, nnz, rowptr, col, val, rhs, x0, slots, status);
}

int b200la_batch_add_q1(b200la_batch B, int dim, int cells, uint64_t seed, double sigma, int *slot_out) {
  B_CHECK(B && slot_out, B200LA_ERR_INVALID, "batch_add_q1: null argument");
  B_CHECK((dim == 2 || dim == 3) && cells >= 1 && sigma >= 0.0, B200LA_ERR_INVALID, "batch_add_q1: dim %d cells %d",
          dim, cells);
  const int64_t n64 = q1_rows(dim, cells), nnz = q1_nnz(dim, cells);
  B_CHECK(nnz < (int64_t)INT32_MAX, B200LA_ERR_UNSUPPORTED, "batch_add_q1: nnz exceeds int32 indexing");
  const int n = (int)n64;
  const int slot = find_free_slot(B);
  B_CHECK(slot >= 0, B200LA_ERR_NOMEM, "batch_add_q1: all %d slots are in use", B->capacity);
  B_TRY(order_after_removals(B));
  HostSys &h = B->sys[slot];
  h = HostSys();
  h.n = n;
  h.nnz = (int)nnz;
  cudaStream_t st = B->xfer;  // like every add: overlaps a launch in flight
  const int ell = cells >= 2 ? (dim == 2 ? 9 : 27) : (dim == 2 ? 4 : 8);
  auto go = [&](auto tag) -> int {
    using T = decltype(tag);
    SysDesc<T> d{};
    B_TRY(alloc_csr_part<T>(B, slot, n, nnz, &d));
    // Q1 couplings: the node offsets dz*m^2 + dy*m + dx, ascending (m = cells + 1
    // nodes per axis, m >= 3 so they are distinct); every row, Dirichlet rows
    // included, stores an ascending subset of them
    int stencil[kMaxStencil];
    const bool use_stencil = B->prm.index_bits == 0 && cells >= 2;
    if (use_stencil) {
      const int64_t m = (int64_t)cells + 1;
      int k = 0;
      for (int dz = (dim == 3 ? -1 : 0); dz <= (dim == 3 ? 1 : 0); ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) stencil[k++] = (int)(dz * m * m + dy * m + dx);
    }
    B_TRY(alloc_sell_part<T>(B, slot, ell, B->prm.index_bits != 32 && q1_col16(dim, cells), d, st,
                             use_stencil ? stencil : nullptr));
    d.max_off = (int)std::min<int64_t>(q1_max_off(dim, cells), INT32_MAX);
    B_TRY(q1_assemble(st, B->ctx->num_sms, dim, cells, seed, sigma, (int *)d.rowptr, (int *)d.col,
                      (double *)d.val64, (double *)d.b));
    B_CUDA(cudaMemsetAsync(d.x, 0, 8 * (size_t)n, st));
    return finish_slot<T>(B, slot, d, st);
  };
  const int rc = B->kp.mixed ? go(float()) : go(double());
  if (cudaEventRecord(B->xfer_done, st) != cudaSuccess ||
      cudaStreamWaitEvent(B->ctx->stream, B->xfer_done, 0) != cudaSuccess) {
    free_slot_memory(B, h);
    h = HostSys();
    return fail(B200LA_ERR_CUDA, "batch_add_q1: stream ordering failed");
  }
  if (rc != B200LA_OK) {
    free_slot_memory(B, h);
    h = HostSys();
    return rc;
  }
  h.used = true;
  B->device_bytes += (int64_t)h.bytes;
  *slot_out = slot;
  return B200LA_OK;
}

int b200la_batch_get_system(b200la_batch B, int slot, int *rowptr, int *col, double *val, double *rhs) {
  B_CHECK(B && slot >= 0 && slot < B->capacity && B->sys[slot].used, B200LA_ERR_INVALID, "batch_get_system: slot");
  const HostSys &h = B->sys[slot];
  cudaStream_t st = B->ctx->stream;
  const int *rp = B->kp.mixed ? h.d32.rowptr : h.d64.rowptr;
  const int *cl = B->kp.mixed ? h.d32.col : h.d64.col;
  const double *vv = B->kp.mixed ? h.d32.val64 : h.d64.val64;
  const double *bb = B->kp.mixed ? h.d32.b : h.d64.b;
  if (rowptr) B_CUDA(cudaMemcpyAsync(rowptr, rp, sizeof(int) * (h.n + 1), cudaMemcpyDeviceToHost, st));
  if (col) B_CUDA(cudaMemcpyAsync(col, cl, sizeof(int) * (size_t)h.nnz, cudaMemcpyDeviceToHost, st));
  if (val) B_CUDA(cudaMemcpyAsync(val, vv, 8 * (size_t)h.nnz, cudaMemcpyDeviceToHost, st));
  if (rhs) B_CUDA(cudaMemcpyAsync(rhs, bb, 8 * (size_t)h.n, cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  return B200LA_OK;
}

int b200la_batch_slot_size(b200la_batch B, int slot, int *n, int64_t *nnz) {
  B_CHECK(B && slot >= 0 && slot < B->capacity && B->sys[slot].used, B200LA_ERR_INVALID, "batch_slot_size: slot");
  if (n) *n = B->sys[slot].n;
  if (nnz) *nnz = B->sys[slot].nnz;
  return B200LA_OK;
}

int b200la_batch_remove(b200la_batch B, int slot) {
  B_CHECK(B && slot >= 0 && slot < B->capacity && B->sys[slot].used, B200LA_ERR_INVALID, "batch_remove: slot %d",
          slot);
  B_TRY(wait_early_copies(B));  // a queued solution copy may still read the slot
  HostSys &h = B->sys[slot];
  cudaStream_t st = B->ctx->stream;
  // stream-ordered: the slot's memory is released after the work queued
  // before it, and its device state is cleared; no host wait
  free_slot_memory(B, h);
  B->device_bytes -= (int64_t)h.bytes;
  h = HostSys();
  memset(&B->st_host[slot], 0, sizeof(SysState));
  B_CUDA(cudaMemsetAsync(B->st + slot, 0, sizeof(SysState), st));
  return note_removal(B);
}

int b200la_batch_remove_many(b200la_batch B, int count, const int *slots) {
  B_CHECK(B && count >= 0 && (count == 0 || slots), B200LA_ERR_INVALID, "batch_remove_many: bad argument");
  std::vector<char> seen(B->capacity, 0);
  for (int k = 0; k < count; ++k) {
    const int s = slots[k];
    B_CHECK(s >= 0 && s < B->capacity && B->sys[s].used && !seen[s], B200LA_ERR_INVALID,
            "batch_remove_many: slot %d (out of range, free or listed twice)", s);
    seen[s] = 1;
  }
  if (count == 0) return B200LA_OK;
  B_TRY(wait_early_copies(B));  // a queued solution copy may still read a slot
  cudaStream_t st = B->ctx->stream;
  for (int k = 0; k < count; ++k) {
    HostSys &h = B->sys[slots[k]];
    free_slot_memory(B, h);
    B->device_bytes -= (int64_t)h.bytes;
    h = HostSys();
    memset(&B->st_host[slots[k]], 0, sizeof(SysState));
  }
  // device states cleared in runs of consecutive slots, one memset per run
  for (int s = 0; s < B->capacity;) {
    if (!seen[s]) { ++s; continue; }
    int e = s;
    while (e < B->capacity && seen[e]) ++e;
    B_CUDA(cudaMemsetAsync(B->st + s, 0, sizeof(SysState) * (size_t)(e - s), st));
    s = e;
  }
  return note_removal(B);
}

}  // extern "C"

namespace {
// Queues, on the transfer stream, the solution copy of every registered
// system that the last state read-back shows finished.  A finished system's
// x is no longer written (the item lists hold running systems only), so the
// copy may overlap the passes that follow.
int issue_early_copies(b200la_batch B) {
  const bool mixed = B->kp.mixed != 0;
  for (int s = 0; s < B->capacity; ++s) {
    HostSys &h = B->sys[s];
    if (!h.used || !h.out || h.out_copied || B->st_host[s].phase != PH_DONE) continue;
    const double *xd = mixed ? h.d32.x : h.d64.x;
    B_CUDA(cudaMemcpyAsync(h.out, xd, 8 * (size_t)h.n, cudaMemcpyDeviceToHost, B->xfer));
    h.out_copied = true;
    B->xfer_copies = true;
  }
  return B200LA_OK;
}

// Waits for the queued solution copies (before x is reset or freed, and
// before results are handed out).
int wait_early_copies(b200la_batch B) {
  if (!B->xfer_copies) return B200LA_OK;
  B_CUDA(cudaStreamSynchronize(B->xfer));
  B->xfer_copies = false;
  return B200LA_OK;
}

// Completes a b200la_batch_launch: the states and globals come back after the
// launch (and after any add queued since, which the context stream waits for).
int complete_inflight(b200la_batch B) {
  if (!B->in_flight) return B200LA_OK;
  cudaStream_t st = B->ctx->stream;
  B->in_flight = false;
  B_CUDA(cudaMemcpyAsync(B->st_host, B->st, sizeof(SysState) * B->capacity, cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaMemcpyAsync(B->glob_host, B->glob, sizeof(BatchGlobals), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  B->pass_total = B->glob_host->pass_total;
  return issue_early_copies(B);
}
}  // namespace

extern "C" {

int b200la_batch_launch(b200la_batch B, int max_passes) {
  B_CHECK(B && max_passes >= 1, B200LA_ERR_INVALID, "batch_launch: bad argument");
  B_TRY(complete_inflight(B));
  cudaStream_t st = B->ctx->stream;
  int active = 0;
  B_TRY(upload_tiles(B, true, &active, nullptr));
  BatchGlobals &g = *B->glob_host;
  if (active == 0) return B200LA_OK;
  if (!B->ctx->use_graphs) {  // the host loop waits on the device anyway
    int a = 0;
    return b200la_batch_run(B, max_passes, &a);
  }
  if (!B->exec) B_TRY(build_graph(B));
  set_globals(B, active, max_passes);
  B_CUDA(cudaMemcpyAsync(B->glob, &g, sizeof(BatchGlobals), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaGraphLaunch(B->exec, st));
  B->in_flight = true;
  return B200LA_OK;
}

int b200la_batch_run(b200la_batch B, int max_passes, int *active_out) {
  B_CHECK(B && max_passes >= 1, B200LA_ERR_INVALID, "batch_run: bad argument");
  B_TRY(complete_inflight(B));
  cudaStream_t st = B->ctx->stream;
  int active = 0;
  B_TRY(upload_tiles(B, true, &active, nullptr));
  BatchGlobals &g = *B->glob_host;
  if (active == 0) {
    g.passes = 0;
    if (active_out) *active_out = 0;
    return B200LA_OK;
  }
  if (B->ctx->use_graphs && !B->exec) B_TRY(build_graph(B));
  set_globals(B, active, max_passes);
  B_CUDA(cudaMemcpyAsync(B->glob, &g, sizeof(BatchGlobals), cudaMemcpyHostToDevice, st));
  if (B->ctx->use_graphs) B_CUDA(cudaGraphLaunch(B->exec, st));
  else B_TRY(host_loop(B));
  B_CUDA(cudaMemcpyAsync(B->st_host, B->st, sizeof(SysState) * B->capacity, cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaMemcpyAsync(B->glob_host, B->glob, sizeof(BatchGlobals), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  B->pass_total = B->glob_host->pass_total;
  if (active_out) *active_out = B->glob_host->active;
  return issue_early_copies(B);
}

int b200la_batch_solve(b200la_batch B, int chunk_passes, int *total_passes) {
  B_CHECK(B && chunk_passes >= 1, B200LA_ERR_INVALID, "batch_solve: bad argument");
  int active = 1, total = 0;
  // each run ends after chunk_passes passes; the next run's tile list holds
  // only the systems still running, so finished systems stop costing passes
  while (active > 0) {
    B_TRY(b200la_batch_run(B, chunk_passes, &active));
    total += B->glob_host->passes;
  }
  B->glob_host->passes = total;
  if (total_passes) *total_passes = total;
  return B200LA_OK;
}

int b200la_batch_last_run(b200la_batch B, int *passes, double *reserved) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_last_run: null batch");
  if (passes) *passes = B->glob_host->passes;
  if (reserved) *reserved = 0.0;
  return B200LA_OK;
}

namespace {
// Host copy of a slot's result from the last run's state read-back; the
// solution copy, if asked for, is queued on the context stream.
int fill_result(b200la_batch B, int slot, double *x_host, b200la_sys_result *r) {
  B_CHECK(B && r && slot >= 0 && slot < B->capacity && B->sys[slot].used, B200LA_ERR_INVALID,
          "batch_result: slot %d", slot);
  HostSys &h = B->sys[slot];
  const SysState &s = B->st_host[slot];
  memset(r, 0, sizeof(*r));
  r->phase_done = s.phase == PH_DONE;
  r->state = s.phase == PH_DONE ? s.state : B200LA_ITERATE;
  r->iters = s.total_iter;
  r->outer = s.outer;
  r->res = s.res;
  r->res_init = s.res0;
  r->res_rel = s.res0 > 0 ? s.res / s.res0 : 0.0;
  r->device_us = (s.phase == PH_DONE && s.t_done >= s.t_begin) ? (double)(s.t_done - s.t_begin) / 1e3 : 0.0;
  if (B->kp.precond && s.bad_row != 0xffffffffu) r->state = B200LA_FAIL_BREAKDOWN;
  if (r->state == B200LA_SUCCESS_ABS || r->state == B200LA_SUCCESS_REL) r->solver_state = B200LA_SOLVER_SUCCESS;
  else if (r->state == B200LA_FAIL_DIV || r->state == B200LA_FAIL_MAXITS || r->state == B200LA_ITERATE)
    r->solver_state = B200LA_SOLVER_EXCEEDED;
  else r->solver_state = B200LA_SOLVER_ERROR;
  // a registered destination that already has its copy queued needs none;
  // a read with a destination ends the registration (a status-only read not)
  if (x_host) {
    if (!(x_host == h.out && h.out_copied)) {
      const double *xd = B->kp.mixed ? h.d32.x : h.d64.x;
      B_CUDA(cudaMemcpyAsync(x_host, xd, 8 * (size_t)h.n, cudaMemcpyDeviceToHost, B->ctx->stream));
    }
    h.out = nullptr;
    h.out_copied = false;
  }
  return B200LA_OK;
}
}  // namespace

int b200la_batch_result(b200la_batch B, int slot, double *x_host, b200la_sys_result *r) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_result: null batch");
  B_TRY(complete_inflight(B));
  B_TRY(fill_result(B, slot, x_host, r));
  if (x_host) B_CUDA(cudaStreamSynchronize(B->ctx->stream));
  return wait_early_copies(B);
}

int b200la_batch_results(b200la_batch B, int count, const int *slots, double *const *x_host,
                         b200la_sys_result *results) {
  B_CHECK(B && count >= 0 && (count == 0 || (slots && results)), B200LA_ERR_INVALID, "batch_results: bad argument");
  B_TRY(complete_inflight(B));
  bool any = false;
  for (int k = 0; k < count; ++k) {
    double *x = x_host ? x_host[k] : nullptr;
    B_TRY(fill_result(B, slots[k], x, &results[k]));
    any = any || x;
  }
  if (any) B_CUDA(cudaStreamSynchronize(B->ctx->stream));
  return wait_early_copies(B);
}

int b200la_batch_set_outputs(b200la_batch B, int count, const int *slots, double *const *x) {
  B_CHECK(B && count >= 0 && (count == 0 || (slots && x)), B200LA_ERR_INVALID, "batch_set_outputs: bad argument");
  for (int k = 0; k < count; ++k)
    B_CHECK(slots[k] >= 0 && slots[k] < B->capacity && B->sys[slots[k]].used, B200LA_ERR_INVALID,
            "batch_set_outputs: slot %d", slots[k]);
  for (int k = 0; k < count; ++k) {
    HostSys &h = B->sys[slots[k]];
    if (h.out_copied && h.out != x[k]) B_TRY(wait_early_copies(B));  // the old destination's copy
    h.out = x[k];
    h.out_copied = false;
  }
  return B200LA_OK;
}

int b200la_batch_info(b200la_batch B, int *used_slots, int64_t *device_bytes) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_info: null batch");
  int u = 0;
  for (const HostSys &h : B->sys) u += h.used ? 1 : 0;
  if (used_slots) *used_slots = u;
  if (device_bytes) *device_bytes = B->device_bytes;
  return B200LA_OK;
}

int b200la_batch_restart(b200la_batch B) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_restart: null batch");
  B_TRY(complete_inflight(B));
  // queued solution copies read x, which the restart zeroes; registrations end
  B_TRY(wait_early_copies(B));
  for (HostSys &h : B->sys) {
    h.out = nullptr;
    h.out_copied = false;
  }
  std::vector<int> slots;
  for (int s = 0; s < B->capacity; ++s)
    if (B->sys[s].used) slots.push_back(s);
  if (slots.empty()) return B200LA_OK;
  cudaStream_t st = B->ctx->stream;
  int *d_slots = nullptr;
  B_CUDA(cudaMallocAsync(&d_slots, sizeof(int) * slots.size(), st));
  B_CUDA(cudaMemcpyAsync(d_slots, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, st));
  if (B->kp.mixed)
    batch_restart_kernel<float><<<(int)slots.size(), kBlock, 0, st>>>(d_slots, (const SysDesc<float> *)B->desc, B->st);
  else
    batch_restart_kernel<double><<<(int)slots.size(), kBlock, 0, st>>>(d_slots, (const SysDesc<double> *)B->desc,
                                                                        B->st);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaFreeAsync(d_slots, st));
  B_CUDA(cudaStreamSynchronize(st));
  for (int s : slots) {
    const unsigned bad = B->st_host[s].bad_row;
    memset(&B->st_host[s], 0, sizeof(SysState));
    B->st_host[s].phase = PH_RESID;
    B->st_host[s].bad_row = bad;
  }
  return B200LA_OK;
}

int b200la_batch_set_items(b200la_batch B, int rows_spmv, int rows_update, int rows_direction, int adaptive) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_set_items: null batch");
  const int r[3] = {rows_spmv, rows_update, rows_direction};
  for (int k = 0; k < 3; ++k)
    B_CHECK(r[k] >= 32 && r[k] <= 65536 && r[k] % 32 == 0, B200LA_ERR_INVALID,
            "batch_set_items: %d rows (32..65536, multiple of 32)", r[k]);
  for (int k = 0; k < 3; ++k) B->lst[k].rows = r[k];
  B->adaptive = adaptive != 0;
  return B200LA_OK;
}

int b200la_batch_get_items(b200la_batch B, int *rows) {
  B_CHECK(B && rows, B200LA_ERR_INVALID, "batch_get_items: null argument");
  for (int k = 0; k < 3; ++k) rows[k] = B->lst[k].rows;
  return B200LA_OK;
}

int b200la_batch_tune(b200la_batch B, int *rows, double *usec) {
  B_CHECK(B, B200LA_ERR_INVALID, "batch_tune: null batch");
  B_TRY(complete_inflight(B));
  B_TRY(wait_early_copies(B));  // the passes below rewrite x
  // Both SpMVs use the sliced-ELL layout (one row per lane, 32-row slices,
  // coalesced steps).  The free parameters are the item sizes: rows per
  // warp work item of K1 (SpMV), K2 (update and dots) and K3 (direction).
  // Small items give more independent warps, short serial chains and
  // balance when few large systems run; large items amortise the per-item
  // record, state and reduction.  Unless the batch was created with a fixed
  // tile_rows, each candidate set is timed on real passes over the running
  // systems (each kernel's time depends only on its own item size, so every
  // kernel picks its own best), and every system's carried state (x, c, r,
  // p and its scalars) is restored after each trial.  Each kernel keeps the
  // smallest item within 3% of its best time: mid-solve passes, where
  // finished systems and residual passes mix in, favour short items.
  // K1 is held to 128..256 rows and keeps 128 unless 256 is more than 8%
  // faster: fresh passes (what a trial times) favour larger K1 items by up
  // to ~2.5%, but whole solves, where residual items (FP64, about twice the
  // work) and finished systems mix in, ran 204 ms at 128 rows against 220 ms
  // at 256 (1,024-system batch).
  static const int cand[4][3] = {{128, 256, 256}, {256, 512, 512}, {256, 1024, 1024}, {256, 2048, 2048}};
  int active = 0;
  B_TRY(upload_tiles(B, true, &active, nullptr));
  double best_ms = 0.0;
  if (active) {
    const bool pre = B->kp.precond != 0;
    auto trial = [&](double *k) -> int {
      if (B->kp.mixed) return pre ? time_passes_t<float, true>(B, 3, k) : time_passes_t<float, false>(B, 3, k);
      return pre ? time_passes_t<double, true>(B, 3, k) : time_passes_t<double, false>(B, 3, k);
    };
    Snapshot snap;
    B_TRY(snapshot_save(B, &snap));
    int rc = B200LA_OK;
    if (B->prm.tile_rows == 0) {
      double t[4][3];
      for (int c = 0; c < 4 && rc == B200LA_OK; ++c) {
        for (int k = 0; k < 3; ++k) B->lst[k].rows = cand[c][k];
        rc = upload_tiles(B, true, &active, nullptr);
        if (rc == B200LA_OK) rc = trial(t[c]);
        if (rc == B200LA_OK) rc = snapshot_restore(B, snap);
      }
      if (rc == B200LA_OK) {
        for (int k = 0; k < 3; ++k) {
          int best = 0;
          for (int c = 1; c < 4; ++c)
            if (t[c][k] < t[best][k]) best = c;
          const double slack = k == 0 ? 1.08 : 1.03;
          for (int c = 0; c < best; ++c)
            if (t[c][k] <= slack * t[best][k]) {
              best = c;
              break;
            }
          B->lst[k].rows = cand[best][k];
          best_ms += t[best][k];
        }
        rc = upload_tiles(B, true, &active, nullptr);
      }
    } else {
      double k[3] = {0, 0, 0};
      rc = trial(k);
      if (rc == B200LA_OK) rc = snapshot_restore(B, snap);
      best_ms = k[0] + k[1] + k[2];
    }
    snapshot_free(B, &snap);
    B_TRY(rc);
  }
  if (rows)
    for (int k = 0; k < 3; ++k) rows[k] = B->lst[k].rows;
  if (usec) *usec = 1000.0 * best_ms;
  return B200LA_OK;
}

int b200la_batch_profile_pass(b200la_batch B, int reps, double *ms, int64_t *algorithmic_bytes) {
  B_CHECK(B && ms && reps >= 1 && reps <= 16, B200LA_ERR_INVALID, "batch_profile_pass: bad argument (reps 1..16)");
  B_TRY(b200la_batch_restart(B));
  int count = 0;
  B_TRY(upload_tiles(B, false, &count, nullptr));
  for (int k = 0; k < 3; ++k) ms[k] = 0.0;
  int64_t n = 0, nnz = 0;
  for (const HostSys &h : B->sys)
    if (h.used) {
      n += h.n;
      nnz += h.nnz;
    }
  const int64_t tb = B->kp.mixed ? 4 : 8;
  const int64_t vecs_k2 = B->kp.precond ? 4 : 3, vecs_k3 = B->kp.precond ? 6 : 5;
  if (algorithmic_bytes) {
    algorithmic_bytes[0] = nnz * (tb + 4) + (n + count) * 4 + 2 * n * tb;
    algorithmic_bytes[1] = vecs_k2 * n * tb;
    algorithmic_bytes[2] = vecs_k3 * n * tb;
  }
  if (count) {
    const bool pre = B->kp.precond != 0;
    int rc;
    if (B->kp.mixed) rc = pre ? time_passes_t<float, true>(B, reps, ms) : time_passes_t<float, false>(B, reps, ms);
    else rc = pre ? time_passes_t<double, true>(B, reps, ms) : time_passes_t<double, false>(B, reps, ms);
    B_TRY(rc);
  }
  return b200la_batch_restart(B);
}

int b200la_batch_profile(b200la_batch B, int reps, double *ms_spmv, int64_t *algorithmic_bytes) {
  B_CHECK(B && ms_spmv && reps >= 1, B200LA_ERR_INVALID, "batch_profile: bad argument");
  B_TRY(complete_inflight(B));
  B_TRY(wait_early_copies(B));  // the passes below rewrite x
  int count = 0;
  int64_t bytes = 0;
  B_TRY(upload_tiles(B, false, &count, &bytes));
  float ms = 0.f;
  if (count) B_TRY(B->kp.mixed ? time_plain<float>(B, reps, &ms) : time_plain<double>(B, reps, &ms));
  *ms_spmv = ms;
  if (algorithmic_bytes) *algorithmic_bytes = bytes;
  return B200LA_OK;
}

}  // extern "C"
