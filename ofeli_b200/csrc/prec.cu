// prec.cu -- OFELI's Prec<real_t> on the device: DIAG, D-ILU (= OFELI's ILU)
// and SSOR (symmetric Gauss-Seidel), with the triangular sweeps of
// SpMatrix::DILUSolve / SSORSolve (include/linear_algebra/SpMatrix_impl.h
// :882-942) and the pivot recurrence of DILUFactorize (:837-870).
//
// Sweep scheduling.  Rows keep OFELI's natural order, so the preconditioner
// is the reference's own.  Rows are cut into strands: maximal runs of
// consecutive rows where each row depends on the row just before it (on a
// structured mesh one strand is one grid line of unknowns).  A warp takes
// the next strand from a ticket counter and walks it in 32-row segments.
// Readiness travels with the data: every result buffer is pre-filled with a
// NaN payload that arithmetic never produces, a producer publishes a row by
// storing its value (one relaxed 8-byte store, no fence), and a consumer of
// a row in an earlier strand spins on that value with a bounded wait.
// Tickets are taken in row order by running warps, so every row a warp waits
// for belongs to a warp that is already running: the sweep always drains.
// Within a segment the dependence on the previous row is a first-order
// affine recurrence z_r = C_r + M_r z_{r-1}, resolved with a 5-step warp
// scan; segments with other intra-segment couplings fall back to an exact
// wave over the warp.  The D-ILU factorisation uses the same machinery in
// its exact form, with the reference's operation order (no FMA
// contraction), so its pivots are bit-identical to the reference's.
//
// Per application: 12*nnz + 4*n (matrix, once per sweep over its half) +
// ~40*n bytes of vectors.  Time is set by the dependency chain (one
// segment step per grid line on a structured 2-D mesh, plus one per segment
// of a line), not by bandwidth; the solve sweeps hand the values of a strand
// to the next one through shared memory where both belong to one block.
#include <algorithm>

#include "internal.cuh"

namespace ofg {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kPre = 8;  // dependency entries per row fetched together
constexpr int kMinStrand = 32;
constexpr int kMaxStrand = 1 << 16;
constexpr long long kSpinFast = 2048;
constexpr long long kSpinSlow = 1 << 22;  // x ~0.5 us sleep: a few seconds at most

enum { FWD_DILU = 0, FWD_SSOR = 1, BWD_DILU = 2, BWD_SSOR = 3, FACTOR = 4 };

struct SweepArgs {
   int64_t n;
   const int32_t* rp;
   const int32_t* col;
   const double* val;
   const int32_t* dpos;
   const int32_t* tpos;    // FACTOR: CSR index of the transposed entry, -1 if absent
   const double* piv;      // DILU: inverse pivots; SSOR: diagonal
   const double* in;       // FWD: b; BWD: t
   double* out;            // results, sentinel-filled on entry
   double* reset;          // entries of this buffer get the sentinel (row by row), may be null
   const double* dot_with; // optional: accumulates (dot_with, out)
   double* strand_dot;     // per-strand partial sums
   double* dot_out;        // the sum, written by the last warp
   const int32_t* sstart;  // strand starts in logical row order, nstrands+1
   int64_t nstrands;
   int* ticket;            // [0] next strand, [1] finished strands
   int* status;
   const int* skip;        // optional: the whole launch is a no-op while *skip != 0
   int* worked;            // profiling flag
};

__device__ __forceinline__ bool is_sentinel(double v)
{
   return (unsigned long long)__double_as_longlong(v) == kSentinelBits;
}

__device__ __forceinline__ double sentinel_value()
{
   return __longlong_as_double((long long)kSentinelBits);
}

__device__ __noinline__ double wait_value_slow(const double* p, int* status)
{
   double v;
   for (long long it = 0; it < kSpinFast; ++it) {
      v = ld_relaxed(p);
      if (!is_sentinel(v)) return v;
   }
   for (long long it = 0; it < kSpinSlow; ++it) {
      __nanosleep(500);
      v = ld_relaxed(p);
      if (!is_sentinel(v)) return v;
   }
   atomicOr(status, 1);
   return 0.0;
}

// Value of an earlier row, waiting (bounded) until its producer stored it.
__device__ __forceinline__ double wait_value(const double* p, int* status)
{
   const double v = ld_relaxed(p);
   return is_sentinel(v) ? wait_value_slow(p, status) : v;
}

// One thread waits, as a sweep does, for a value that nothing produces.
__global__ void wait_selftest(const double* p, int* status, double* out)
{
   if (blockIdx.x == 0 && threadIdx.x == 0) *out = wait_value(p, status);
}

template <int MODE>
__device__ __forceinline__ double finish_row(double s, double bi, double pv)
{
   if (MODE == FWD_DILU) return pv * (bi - s);
   if (MODE == FWD_SSOR) return (bi - s) / pv;
   if (MODE == BWD_DILU) return bi - pv * s;
   return bi - s / pv;  // BWD_SSOR
}

template <int MODE>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) sweep_kernel(SweepArgs g)
{
   constexpr bool FWD = (MODE == FWD_DILU || MODE == FWD_SSOR || MODE == FACTOR);
   __shared__ double seg[kWarpsPerBlock][32];
   const int lane = threadIdx.x & 31;
   const int w = threadIdx.x >> 5;
   const unsigned FULL = 0xffffffffu;
   const int64_t n = g.n;
   if (g.skip && *g.skip) return;
   prof_mark(g.worked);

   for (;;) {
      int s = 0;
      if (lane == 0) s = atomicAdd(&g.ticket[0], 1);
      s = __shfl_sync(FULL, s, 0);
      if (s >= g.nstrands) break;
      const int64_t beg = g.sstart[s], end = g.sstart[s + 1];
      double carry = 0.0;
      bool have_carry = false;
      double dotp = 0.0;

      for (int64_t s0 = beg; s0 < end; s0 += 32) {
         const int64_t rho = s0 + lane;
         const bool valid = rho < end;
         const int64_t row = FWD ? rho : n - 1 - rho;
         int32_t kb = 0, ke = 0, dk = 0;
         if (valid) {
            dk = g.dpos[row];
            if (FWD) { kb = g.rp[row]; ke = dk; }
            else { kb = dk + 1; ke = g.rp[row + 1]; }
         }
         // external part of the row sum (rows of earlier segments), in
         // column order; intra-segment couplings are recorded
         double sext = 0.0, m1 = 0.0;
         bool other_intra = false;
         // FACTOR: the coupling to the row before, when it is the row's
         // last lower entry (then the sum subtracts it last)
         bool has_prev = false;
         double a_prev = 0.0, t_prev = 0.0;
         if (MODE == FACTOR) sext = valid ? g.val[dk] : 0.0;
         // the first kPre entries: all loads (matrix and earlier results)
         // are issued before any is consumed, so their latencies overlap
         int32_t pc[kPre];
         double pa[kPre], pz[kPre];
#pragma unroll
         for (int q = 0; q < kPre; ++q) {
            const int32_t k = kb + q;
            pc[q] = -1;
            if (k < ke) {
               pc[q] = g.col[k];
               pa[q] = g.val[k];
            }
         }
#pragma unroll
         for (int q = 0; q < kPre; ++q) {
            pz[q] = 0.0;
            if (pc[q] >= 0) {
               const int64_t lj = FWD ? pc[q] : n - 1 - pc[q];
               if (lj < s0 && !(lj == s0 - 1 && have_carry)) pz[q] = ld_relaxed(g.out + pc[q]);
            }
         }
#pragma unroll
         for (int q = 0; q < kPre; ++q) {
            if (pc[q] < 0) continue;
            const int64_t j = pc[q];
            const int64_t lj = FWD ? j : n - 1 - j;
            const double a = pa[q];
            double v = 0.0;
            if (lj < s0) {
               v = (lj == s0 - 1 && have_carry) ? carry
                                                : (is_sentinel(pz[q]) ? wait_value_slow(g.out + j, g.status) : pz[q]);
            }
            if (MODE == FACTOR) {
               const int32_t tp = g.tpos[kb + q];
               if (tp < 0) continue;
               if (lj >= s0) {
                  if (lj == rho - 1 && kb + q == ke - 1) {
                     has_prev = true;
                     a_prev = a;
                     t_prev = g.val[tp];
                  }
                  else other_intra = true;
                  continue;
               }
               sext = __dsub_rn(sext, __dmul_rn(__dmul_rn(a, v), g.val[tp]));
            }
            else {
               if (lj >= s0) {
                  if (lj == rho - 1) m1 = a;
                  else other_intra = true;
                  continue;
               }
               sext += a * v;
            }
         }
         for (int32_t k = kb + kPre; k < ke; ++k) {
            const int64_t j = g.col[k];
            const int64_t lj = FWD ? j : n - 1 - j;
            const double a = g.val[k];
            if (MODE == FACTOR) {
               const int32_t tp = g.tpos[k];
               if (tp < 0) continue;
               if (lj >= s0) {
                  if (lj == rho - 1 && k == ke - 1) {
                     has_prev = true;
                     a_prev = a;
                     t_prev = g.val[tp];
                  }
                  else other_intra = true;
                  continue;
               }
               const double v = (lj == s0 - 1 && have_carry) ? carry : wait_value(g.out + j, g.status);
               sext = __dsub_rn(sext, __dmul_rn(__dmul_rn(a, v), g.val[tp]));
            }
            else {
               if (lj >= s0) {
                  if (lj == rho - 1) m1 = a;
                  else other_intra = true;
                  continue;
               }
               const double v = (lj == s0 - 1 && have_carry) ? carry : wait_value(g.out + j, g.status);
               sext += a * v;
            }
         }
         double bi = 0.0, pv = 0.0;
         if (valid && MODE != FACTOR) {
            bi = g.in[row];
            pv = g.piv[row];
         }
         double z;
         const bool chain = (MODE == FACTOR) && !__any_sync(FULL, other_intra);
         const bool exact = !chain && ((MODE == FACTOR) || __any_sync(FULL, other_intra));
         if (chain) {
            // pivots in lane order: a lane coupled only to the row before
            // takes that row's pivot by a shuffle and subtracts its term
            // last, in OFELI's order; the others need nothing from the
            // segment
            z = 0.0;
            if (valid && !has_prev) z = __ddiv_rn(1.0, sext);
            for (int i = 1; i < 32; ++i) {
               const double v = __shfl_sync(FULL, z, i - 1);
               if (lane == i && valid && has_prev)
                  z = __ddiv_rn(1.0, __dsub_rn(sext, __dmul_rn(__dmul_rn(a_prev, v), t_prev)));
            }
         }
         else if (!exact) {
            // z = C + M * z_prev with z_prev the previous lane's result
            double C, M;
            if (MODE == FWD_DILU) { C = pv * (bi - sext); M = -pv * m1; }
            else if (MODE == FWD_SSOR) { C = (bi - sext) / pv; M = -m1 / pv; }
            else if (MODE == BWD_DILU) { C = bi - pv * sext; M = -pv * m1; }
            else { C = bi - sext / pv; M = -m1 / pv; }
            if (!valid) { C = 0.0; M = 0.0; }
            if (lane == 0) M = 0.0;  // lane 0 has no intra-segment predecessor
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
               const double Cp = __shfl_up_sync(FULL, C, o);
               const double Mp = __shfl_up_sync(FULL, M, o);
               if (lane >= o) {
                  C = C + M * Cp;
                  M = M * Mp;
               }
            }
            z = C;
         }
         else {
            // exact wave: a lane computes once all its intra-segment
            // predecessors are in shared memory
            seg[w][lane] = sentinel_value();
            __syncwarp();
            bool done = !valid;
            z = 0.0;
            for (int round = 0; round < 32; ++round) {
               if (!done) {
                  bool ready = true;
                  double acc = sext;
                  for (int32_t k = kb; k < ke && ready; ++k) {
                     const int64_t j = g.col[k];
                     const int64_t lj = FWD ? j : n - 1 - j;
                     if (lj < s0) continue;
                     if (MODE == FACTOR && g.tpos[k] < 0) continue;
                     const double v = seg[w][lj - s0];
                     if (is_sentinel(v)) { ready = false; break; }
                     if (MODE == FACTOR)
                        acc = __dsub_rn(acc, __dmul_rn(__dmul_rn(g.val[k], v), g.val[g.tpos[k]]));
                     else
                        acc += g.val[k] * v;
                  }
                  if (ready) {
                     if (MODE == FACTOR) z = __ddiv_rn(1.0, acc);
                     else z = finish_row<MODE>(acc, bi, pv);
                     done = true;
                  }
               }
               __syncwarp();
               if (done && valid) seg[w][lane] = z;
               __syncwarp();
               if (__all_sync(FULL, done)) break;
            }
            if (!__all_sync(FULL, done)) {
               if (lane == 0) atomicOr(g.status, 2);
            }
         }
         if (valid) {
            st_relaxed(g.out + row, z);
            if (g.reset) g.reset[row] = sentinel_value();
            if (g.dot_with) dotp += g.dot_with[row] * z;
         }
         const int64_t last = min((int64_t)31, end - 1 - s0);
         carry = __shfl_sync(FULL, z, (int)last);
         have_carry = true;
      }
      if (g.dot_with) {
         // last-finisher reduction over strands, in strand order
         dotp = warp_sum(dotp);
         int last = 0;
         if (lane == 0) {
            g.strand_dot[s] = dotp;
            __threadfence();
            last = atomicAdd(&g.ticket[1], 1) == (int)g.nstrands - 1;
         }
         last = __shfl_sync(FULL, last, 0);
         if (last) {
            __threadfence();
            double acc = 0.0;
            for (int64_t t = lane; t < g.nstrands; t += 32) acc += ld_relaxed(g.strand_dot + t);
            acc = warp_sum(acc);
            if (lane == 0) *g.dot_out = acc;
         }
      }
   }
}

__global__ void fill_sentinel_kernel(double* p, int64_t n)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   const double s = __longlong_as_double((long long)kSentinelBits);
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = s;
}

__global__ void diag_setup(int64_t n, const int32_t* dpos, const double* val, double* piv,
                           int invert, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const int32_t d = dpos[i];
      const double a = d >= 0 ? val[d] : 0.0;
      if (a == 0.0) atomicMin(bad, (int)i);
      piv[i] = invert ? 1.0 / a : a;
   }
}

__global__ void diag_apply(int64_t n, const double* piv, const double* r, double* z,
                           const int* skip)
{
   if (skip && *skip) return;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      z[i] = r[i] * piv[i];
}

// Transposed positions for the strictly lower entries: tpos[k] = index of
// (col[k], row) in the upper part of row col[k], -1 when absent.
__global__ void transpose_positions(int64_t n, const int32_t* rp, const int32_t* col,
                                    const int32_t* dpos, int32_t* tpos)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
      for (int32_t k = rp[l]; k < rp[l + 1]; ++k) {
         const int32_t i = col[k];
         int32_t pos = -1;
         if (i < l) {
            int32_t lo = dpos[i] + 1, hi = rp[i + 1] - 1;
            while (lo <= hi) {
               const int32_t mid = (lo + hi) >> 1;
               const int32_t c = col[mid];
               if (c == (int32_t)l) { pos = mid; break; }
               if (c < (int32_t)l) lo = mid + 1;
               else hi = mid - 1;
            }
         }
         tpos[k] = pos;
      }
   }
}

// ------------------------------------------------------- solve sweeps ----
// The forward / backward sweeps of DILUSolve and SSORSolve over the slot
// layout.  Per segment a lane holds one row: its dependency slots (column,
// value) arrive as coalesced lines, the next segment's slots, b and pivot
// are fetched while the current segment waits for its earlier-row values.
// A lane holds 4 or 8 slots in registers (the plan's widest segment); rows
// wider than 8 take a slow loop.

struct SolveArgs {
   int64_t n;
   const int32_t* tseg;
   const int32_t* seg_off;
   const int32_t* sl_col;
   const double* sl_val;
   const double* piv;
   const double* in;
   double* out;
   double* reset;
   const double* dot_with;
   double* strand_dot;
   double* dot_out;
   const int32_t* sstart;
   int64_t nstrands;
   int* ticket;
   int* status;
   const int* skip;
   int* worked;
   const int32_t* seg_keep;
};

// Band hand-off.  A block takes a band of kBandWarps consecutive strands,
// one warp each.  Besides storing its results to global memory (for the
// strands of other blocks), a warp keeps the latest kRing of them in a
// shared-memory ring and publishes how far it got (done_end: the logical
// row one past its last finished segment) with a CTA-scope release; the
// next warp of the band waits once per segment, with an acquire, until the
// rows of the previous strand that the segment needs are published, and
// reads them from the ring instead of waiting for them to travel through
// L2.  A segment reads the ring when the lowest previous-strand row its
// register slots need is within kRing / 2 of the highest such row needed
// by it or an earlier segment of its strand (a property of the plan);
// otherwise it reads them from global memory.  Every warp also publishes
// keep_from: the lowest previous-strand row that it, or a later segment of
// its strand, still reads from the ring (the plan's seg_keep); before
// writing a segment into its ring, a warp waits (bounded) until its
// consumer's keep_from is past the rows those slots held.  That wait always
// ends: while the consumer waits for a row r, every ring row it will still
// read is above r - kRing / 2, below what the producer overwrites before
// publishing r.  The arithmetic is the same on either path, so the results
// are bit for bit equal.
//
// The time of a sweep is about (strands) x (the part of a segment step
// between the previous strand's publish and this strand's), so that part
// is kept short: everything that does not depend on the previous strand
// (the other slots' values, the coupling to the row before, the
// multiplicative half of the affine scan, the consumer check) is done
// before the wait, the ring is read without a branch, and the ring and
// the release go out before the global copy.  The register slots are sized
// to the plan's widest segment (NS = 4 or 8), indices are 32-bit, and the
// previous strand is waited for once per segment.
constexpr int kBandWarps = 16;
constexpr int kRing = 256;
constexpr long long kSpinSmemFast = 1 << 14;
constexpr long long kSpinSmemSlow = 1 << 22;  // x ~0.5 us sleep: a few seconds at most
// A segment step waits for the slot data of the next segment (loaded one
// segment ahead into registers); the slot data of the segment kPrefetch
// ahead is pulled into L2 first (one bulk prefetch per array, issued by
// lane 0: a strand's segments are contiguous in the slot layout), and its
// right-hand side, pivots and dot_with entries likewise, one row per lane.
constexpr int kPrefetch = 4;

__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes)
{
   asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void* p)
{
   asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ int ld_acquire_cta(const int* p)
{
   int v;
   asm volatile("ld.acquire.cta.shared.s32 %0, [%1];"
                : "=r"(v)
                : "r"((unsigned)__cvta_generic_to_shared(p))
                : "memory");
   return v;
}

__device__ __forceinline__ int ld_relaxed_cta(const int* p)
{
   int v;
   asm volatile("ld.relaxed.cta.shared.s32 %0, [%1];"
                : "=r"(v)
                : "r"((unsigned)__cvta_generic_to_shared(p))
                : "memory");
   return v;
}

__device__ __forceinline__ void st_relaxed_cta(int* p, int v)
{
   asm volatile("st.relaxed.cta.shared.s32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)),
                "r"(v)
                : "memory");
}

// waits (bounded) until *done_end > need; returns the value seen, or -1
// when the wait ran out (status set)
__device__ __noinline__ int wait_published(const int* done_end, int need, int* status)
{
   int de = ld_acquire_cta(done_end);
   for (long long it = 0; de <= need; ++it) {
      if (it >= kSpinSmemFast + kSpinSmemSlow) {
         atomicOr(status, 1);
         return -1;
      }
      if (it >= kSpinSmemFast) __nanosleep(500);
      de = ld_acquire_cta(done_end);
   }
   return de;
}

// waits until the previous warp of the band has published past row `need`:
// relaxed polls, then one fence (an acquire of what was seen); returns the
// value seen, or -1 when the wait ran out (status set)
__device__ __forceinline__ int wait_previous(const int* prev_done, int need, int* status)
{
   int de = ld_relaxed_cta(prev_done);
   for (int q = 0; q < 32 && de <= need; ++q) de = ld_relaxed_cta(prev_done);
   if (de <= need) de = wait_published(prev_done, need, status);
   asm volatile("fence.acq_rel.cta;" ::: "memory");
   return de;
}

// Polls (bounded) the earlier rows of the slots in `pend` until none holds
// the sentinel: every round issues the loads of all pending slots before it
// tests any, so that slots published together cost one round trip.  On
// time-out the status is set and the missing values read as 0.
template <int NS>
__device__ __forceinline__ void poll_slots(const double* out, const int32_t (&c)[NS], unsigned pend,
                                        double (&v)[NS], int* status)
{
   for (long long it = 0; pend; ++it) {
      if (it >= kSpinFast + kSpinSlow) {
         atomicOr(status, 1);
#pragma unroll
         for (int k = 0; k < NS; ++k)
            if ((pend >> k) & 1) v[k] = 0.0;
         return;
      }
      if (it >= kSpinFast) __nanosleep(500);
#pragma unroll
      for (int k = 0; k < NS; ++k)
         if ((pend >> k) & 1) v[k] = ld_relaxed(out + c[k]);
#pragma unroll
      for (int k = 0; k < NS; ++k)
         if (((pend >> k) & 1) && !is_sentinel(v[k])) pend &= ~(1u << k);
   }
}

// The additive half of a segment's affine scan: row rho's result is
// C(rho) + M(rho) z(rho - 1), C from the slot sum; Mr[r] is the product of M
// over the 2^r rows ending at this lane (the multiplicative half)
template <int MODE>
__device__ __forceinline__ double affine_scan(double sext, double bi, double pv, bool valid,
                                              const double (&Mr)[5], int lane)
{
   const unsigned FULL = 0xffffffffu;
   double C;
   if (MODE == FWD_DILU) C = pv * (bi - sext);
   else if (MODE == FWD_SSOR) C = (bi - sext) / pv;
   else if (MODE == BWD_DILU) C = bi - pv * sext;
   else C = bi - sext / pv;
   if (!valid) C = 0.0;
#pragma unroll
   for (int r = 0; r < 5; ++r) {
      const double Cp = __shfl_up_sync(FULL, C, 1 << r);
      if (lane >= (1 << r)) C = C + Mr[r] * Cp;
   }
   return C;
}

template <int NS>
struct SegRegs {
   int32_t off, w, keep;
   int32_t c[NS];
   double a[NS];
   double b, pv, dw;  // dw: the row's entry of dot_with (0 without)
};

template <bool FWD, int NS>
__device__ __forceinline__ void load_segment(const SolveArgs& g, int64_t s, int32_t s0, int32_t end,
                                             int lane, SegRegs<NS>& R)
{
   R.off = g.seg_off[s];
   R.w = (g.seg_off[s + 1] - R.off) >> 5;
   R.keep = g.seg_keep[s];
#pragma unroll
   for (int k = 0; k < NS; ++k) {
      R.c[k] = -1;
      R.a[k] = 0.0;
      if (k < R.w) {
         R.c[k] = g.sl_col[R.off + k * 32 + lane];
         R.a[k] = g.sl_val[R.off + k * 32 + lane];
      }
   }
   const int32_t rho = s0 + lane;
   R.b = 0.0;
   R.pv = 1.0;
   R.dw = 0.0;
   if (rho < end) {
      const int32_t row = FWD ? rho : (int32_t)g.n - 1 - rho;
      R.b = g.in[row];
      R.pv = g.piv[row];
      if (g.dot_with) R.dw = g.dot_with[row];
   }
}

template <int MODE, int NS>
__global__ void __launch_bounds__(kBandWarps * 32, 1) solve_sweep(SolveArgs g)
{
   constexpr bool FWD = (MODE == FWD_DILU || MODE == FWD_SSOR);
   __shared__ double segv[kBandWarps][32];
   __shared__ double ring[kBandWarps][kRing];
   __shared__ int done_end[kBandWarps];
   __shared__ int keep_from[kBandWarps];
   __shared__ int band_sh;
   const int lane = threadIdx.x & 31;
   const int w = threadIdx.x >> 5;
   const unsigned FULL = 0xffffffffu;
   const int32_t n = (int32_t)g.n;
   if (g.skip && *g.skip) return;
   prof_mark(g.worked);
   const int nbands = (int)((g.nstrands + kBandWarps - 1) / kBandWarps);

   for (;;) {
      // every warp finished the previous band: the rings are free
      __syncthreads();
      if (threadIdx.x == 0) band_sh = atomicAdd(&g.ticket[0], 1);
      __syncthreads();
      const int band = band_sh;
      if (band >= nbands) break;
      const int64_t t = (int64_t)band * kBandWarps + w;
      const bool active = t < g.nstrands;
      const int32_t beg = active ? g.sstart[t] : 0, end = active ? g.sstart[t + 1] : 0;
      // the previous strand is this block's warp w - 1 (rows pbeg .. beg-1)
      const int32_t pbeg = (active && w > 0) ? g.sstart[t - 1] : beg;
      if (lane == 0) {
         done_end[w] = beg;
         keep_from[w] = active ? g.seg_keep[g.tseg[t]] : INT32_MAX;
      }
      __syncthreads();
      if (!active) continue;
      // the next strand of the band, which reads this warp's ring
      const bool has_consumer = w + 1 < kBandWarps && t + 1 < g.nstrands;
      int run_need = -1;  // highest previous-strand row needed so far
      const int* prev_done = &done_end[w > 0 ? w - 1 : 0];
      const double* prev_ring = ring[w > 0 ? w - 1 : 0];
      const int64_t sfirst = g.tseg[t], slast = g.tseg[t + 1];
      double carry = 0.0;
      bool have_carry = false;
      double dotp = 0.0;
      SegRegs<NS> cur, nxt;
      load_segment<FWD, NS>(g, sfirst, beg, end, lane, cur);
      for (int64_t s = sfirst; s < slast; ++s) {
         const int32_t s0 = beg + 32 * (int32_t)(s - sfirst);
         if (s + kPrefetch < slast) {
            const int32_t rp = s0 + 32 * kPrefetch + lane;
            if (lane == 0) {
               const int32_t o0 = g.seg_off[s + kPrefetch], o1 = g.seg_off[s + kPrefetch + 1];
               if (o1 > o0) {
                  prefetch_l2_bulk(g.sl_col + o0, (uint32_t)(o1 - o0) * 4u);
                  prefetch_l2_bulk(g.sl_val + o0, (uint32_t)(o1 - o0) * 8u);
               }
            }
            if (rp < end) {
               const int32_t row = FWD ? rp : n - 1 - rp;
               prefetch_l2(g.in + row);
               prefetch_l2(g.piv + row);
               if (g.dot_with) prefetch_l2(g.dot_with + row);
            }
         }
         if (s + 1 < slast) load_segment<FWD, NS>(g, s + 1, s0 + 32, end, lane, nxt);
         const int32_t rho = s0 + lane;
         const bool valid = rho < end;
         // Before the wait: the values of the slots that do not come from
         // the previous strand (the carry, this strand's earlier segments,
         // other blocks' strands), the coupling to the row before (m1) and
         // the multiplicative half of the segment scan.  Once the previous
         // strand's rows are published, only their reads, the slot sum, the
         // additive half of the scan and the publish remain on the chain
         // that runs from strand to strand.
         int32_t lj[NS];
         double pre[NS];
         bool from_prev[NS];
         int need = -1, low = INT32_MAX;
         double m1 = 0.0;
         bool other_intra = false;
         unsigned gpend = 0;  // slots loaded from global memory
#pragma unroll
         for (int k = 0; k < NS; ++k) {
            const int32_t c = cur.c[k];
            lj[k] = c < 0 ? -1 : (FWD ? c : n - 1 - c);
            pre[k] = 0.0;
            from_prev[k] = false;
            if (c < 0) continue;
            if (lj[k] >= s0) {
               if (lj[k] == rho - 1) m1 = cur.a[k];
               else other_intra = true;
            }
            else if (lj[k] == s0 - 1 && have_carry) pre[k] = carry;
            else if (lj[k] >= beg || lj[k] < pbeg) {
               // this strand's earlier segments or another block's strand:
               // loaded from global memory, all such slots together
               pre[k] = ld_relaxed(g.out + c);
               gpend |= 1u << k;
            }
            else {
               from_prev[k] = true;
               need = max(need, lj[k]);
               low = min(low, lj[k]);
            }
         }
         for (int k = NS; k < cur.w; ++k) {  // rows wider than the register slots
            const int32_t c = g.sl_col[cur.off + k * 32 + lane];
            if (c < 0) continue;
            const int32_t l = FWD ? c : n - 1 - c;
            if (l >= s0) {
               if (l == rho - 1) m1 = g.sl_val[cur.off + k * 32 + lane];
               else other_intra = true;
            }
         }
         const bool affine = !__any_sync(FULL, other_intra);
         const double bi = cur.b, pv = cur.pv;
         double Mr[5];  // M of the scan at the start of each round
         if (affine) {
            double M;
            if (MODE == FWD_DILU || MODE == BWD_DILU) M = -pv * m1;
            else M = -m1 / pv;
            if (!valid || lane == 0) M = 0.0;
#pragma unroll
            for (int r = 0; r < 5; ++r) {
               Mr[r] = M;
               const double Mp = __shfl_up_sync(FULL, M, 1 << r);
               if (lane >= (1 << r)) M = M * Mp;
            }
         }
         // global slots whose value was not there yet (the first strand of a
         // band waiting for the previous block's last strand): polled together
#pragma unroll
         for (int k = 0; k < NS; ++k)
            if (!is_sentinel(pre[k])) gpend &= ~(1u << k);
         if (gpend) poll_slots<NS>(g.out, cur.c, gpend, pre, g.status);
         // the consumer no longer reads the ring slots this segment overwrites
         if (has_consumer && ld_acquire_cta(&keep_from[w + 1]) <= s0 + 31 - kRing)
            wait_published(&keep_from[w + 1], s0 + 31 - kRing, g.status);
         need = __reduce_max_sync(FULL, need);
         low = __reduce_min_sync(FULL, low);
         run_need = max(run_need, need);
         // ring reads are safe when the rows lie within half the ring of the
         // highest row needed so far (the plan's back-pressure covers them)
         const bool ring_ok = need >= 0 && run_need - low < kRing / 2;
         double zr;
         if (affine && cur.w <= NS && (need < 0 || ring_ok)) {
            // the common step: chosen before the wait, so that nothing after
            // it branches.  Every slot reads the ring (the empty ones a
            // harmless slot) and selects.
            if (need >= 0) wait_previous(prev_done, need, g.status);
            double rv[NS];
#pragma unroll
            for (int k = 0; k < NS; ++k) rv[k] = prev_ring[lj[k] & (kRing - 1)];
            double sext = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) {
               if (cur.c[k] < 0 || lj[k] >= s0) continue;
               sext += cur.a[k] * (from_prev[k] ? rv[k] : pre[k]);
            }
            zr = affine_scan<MODE>(sext, bi, pv, valid, Mr, lane);
         }
         else {
            bool from_ring = false;
            if (need >= 0) from_ring = wait_previous(prev_done, need, g.status) > need && ring_ok;
            double sext = 0.0;
            if (from_ring) {
               double rv[NS];
#pragma unroll
               for (int k = 0; k < NS; ++k) rv[k] = prev_ring[lj[k] & (kRing - 1)];
#pragma unroll
               for (int k = 0; k < NS; ++k) {
                  if (cur.c[k] < 0 || lj[k] >= s0) continue;
                  sext += cur.a[k] * (from_prev[k] ? rv[k] : pre[k]);
               }
            }
            else {
#pragma unroll
               for (int k = 0; k < NS; ++k) {
                  if (cur.c[k] < 0 || lj[k] >= s0) continue;
                  const double v = from_prev[k] ? wait_value(g.out + cur.c[k], g.status) : pre[k];
                  sext += cur.a[k] * v;
               }
            }
            for (int k = NS; k < cur.w; ++k) {
               const int32_t c = g.sl_col[cur.off + k * 32 + lane];
               if (c < 0) continue;
               const int32_t l = FWD ? c : n - 1 - c;
               if (l >= s0) continue;
               const double a = g.sl_val[cur.off + k * 32 + lane];
               const double v = (l == s0 - 1 && have_carry) ? carry : wait_value(g.out + c, g.status);
               sext += a * v;
            }
            if (affine) zr = affine_scan<MODE>(sext, bi, pv, valid, Mr, lane);
            else {
               // exact wave over the intra-segment couplings
               segv[w][lane] = sentinel_value();
               __syncwarp();
               bool done = !valid;
               zr = 0.0;
               for (int round = 0; round < 32; ++round) {
                  if (!done) {
                     bool ready = true;
                     double acc = sext;
                     // (re-read from the slot arrays: indexing the register
                     // copies with a run-time k would move them to local memory)
                     for (int k = 0; k < cur.w && ready; ++k) {
                        const int32_t c = g.sl_col[cur.off + k * 32 + lane];
                        if (c < 0) continue;
                        const int32_t l = FWD ? c : n - 1 - c;
                        if (l < s0) continue;
                        const double v = segv[w][l - s0];
                        if (is_sentinel(v)) { ready = false; break; }
                        acc += g.sl_val[cur.off + k * 32 + lane] * v;
                     }
                     if (ready) {
                        zr = finish_row<MODE>(acc, bi, pv);
                        done = true;
                     }
                  }
                  __syncwarp();
                  if (done && valid) segv[w][lane] = zr;
                  __syncwarp();
                  if (__all_sync(FULL, done)) break;
               }
               if (!__all_sync(FULL, done) && lane == 0) atomicOr(g.status, 2);
            }
         }
         // publish the segment: the ring and the release for the next warp
         // of the band first, the global copy (for other blocks' strands,
         // whose readers spin on its sentinel) after.  One fence, then
         // relaxed stores (every lane the same value): a release of both,
         // with no branch on the lane.
         if (valid) ring[w][rho & (kRing - 1)] = zr;
         __syncwarp();
         __threadfence_block();
         st_relaxed_cta(&keep_from[w], s + 1 < slast ? nxt.keep : INT32_MAX);
         st_relaxed_cta(&done_end[w], min(end, s0 + 32));
         if (valid) {
            const int32_t row = FWD ? rho : n - 1 - rho;
            st_relaxed(g.out + row, zr);
            if (g.reset) g.reset[row] = sentinel_value();
            // dot_with's entry came with the segment's slot data
            dotp += cur.dw * zr;
         }
         const int last = min(31, end - 1 - s0);
         carry = __shfl_sync(FULL, zr, last);
         have_carry = true;
         if (s + 1 < slast) cur = nxt;
      }
      if (g.dot_with) {
         dotp = warp_sum(dotp);
         int lastw = 0;
         if (lane == 0) {
            g.strand_dot[t] = dotp;
            __threadfence();
            lastw = atomicAdd(&g.ticket[1], 1) == (int)g.nstrands - 1;
         }
         lastw = __shfl_sync(FULL, lastw, 0);
         if (lastw) {
            __threadfence();
            double acc = 0.0;
            for (int64_t q = lane; q < g.nstrands; q += 32) acc += ld_relaxed(g.strand_dot + q);
            acc = warp_sum(acc);
            if (lane == 0) *g.dot_out = acc;
         }
      }
   }
}

__global__ void slot_values(int64_t total, const int32_t* src, const double* val, double* out)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      const int32_t s = src[i];
      out[i] = s >= 0 ? val[s] : 0.0;
   }
}

// chain[rho] = 1 when logical row rho depends on logical row rho-1
__global__ void chain_flags(int64_t n, const int32_t* rp, const int32_t* col, const int32_t* dpos,
                            int fwd, int8_t* chain)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t rho = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rho < n; rho += stride) {
      int8_t c = 0;
      if (rho > 0) {
         if (fwd) {
            const int64_t r = rho;
            for (int32_t k = rp[r]; k < dpos[r]; ++k)
               if (col[k] == r - 1) c = 1;
         }
         else {
            const int64_t r = n - 1 - rho;
            for (int32_t k = dpos[r] + 1; k < rp[r + 1]; ++k)
               if (col[k] == r + 1) c = 1;
         }
      }
      chain[rho] = c;
   }
}


}  // namespace

void fill_sentinel(double* p, int64_t n)
{
   if (n <= 0) return;
   fill_sentinel_kernel<<<grid_for(n, 256), 256, 0, stream()>>>(p, n);
   count_launch();
   OFG_LAUNCH_CHECK();
}

namespace {

// Strands start where a row does not depend on its predecessor; runs shorter
// than kMinStrand are merged forward, runs longer than kMaxStrand are split.
void build_plan(ofg_matrix* A, bool fwd, SweepPlan& plan)
{
   const int64_t n = A->n;
   DBuf<int8_t> chain(n > 0 ? n : 1);
   if (n) {
      chain_flags<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p, A->dpos.p,
                                                          fwd ? 1 : 0, chain.p);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   std::vector<int8_t> c = chain.to_host(n);
   std::vector<int32_t> starts;
   int64_t cur = 0;
   for (int64_t r = 1; r <= n; ++r) {
      const bool brk = (r == n) || !c[r];
      if ((brk && r - cur >= kMinStrand) || r - cur >= kMaxStrand || r == n) {
         if (r > cur) starts.push_back((int32_t)cur);
         cur = r;
      }
   }
   starts.push_back((int32_t)n);
   plan.nstrands = (int64_t)starts.size() - 1;
   plan.start.alloc(starts.size());
   plan.start.upload(starts.data(), starts.size());
   plan.strand_dot.alloc(plan.nstrands > 0 ? plan.nstrands : 1);
   plan.ticket.alloc(4);

   // slot layout: one 32-row segment per warp step, dependency entries
   // column-major in CSR column order
   std::vector<int32_t> rp = A->row_ptr.to_host(n + 1);
   std::vector<int32_t> col = A->col.to_host(A->nnz);
   std::vector<int32_t> dp = A->dpos.to_host(n);
   auto dep_range = [&](int64_t rho, int32_t& kb, int32_t& ke) {
      const int64_t r = fwd ? rho : n - 1 - rho;
      if (fwd) { kb = rp[r]; ke = dp[r]; }
      else { kb = dp[r] + 1; ke = rp[r + 1]; }
   };
   std::vector<int32_t> tseg(plan.nstrands + 1, 0), seg_off(1, 0);
   for (int64_t t = 0; t < plan.nstrands; ++t) {
      const int64_t b = starts[t], e = starts[t + 1];
      for (int64_t s0 = b; s0 < e; s0 += 32) {
         int32_t wmax = 0;
         for (int64_t rho = s0; rho < std::min(e, s0 + 32); ++rho) {
            int32_t kb, ke;
            dep_range(rho, kb, ke);
            wmax = std::max(wmax, ke - kb);
         }
         seg_off.push_back(seg_off.back() + 32 * wmax);
      }
      tseg[t + 1] = (int32_t)(seg_off.size() - 1);
   }
   const int64_t nslot = seg_off.back();
   plan.wmax = 0;
   for (size_t q = 0; q + 1 < seg_off.size(); ++q)
      plan.wmax = std::max(plan.wmax, (seg_off[q + 1] - seg_off[q]) / 32);
   OFG_REQUIRE(nslot < (int64_t(1) << 31), OFG_ERR_PATTERN, "sweep layout exceeds 2^31 slots");
   std::vector<int32_t> slc(nslot > 0 ? nslot : 1, -1), sls(nslot > 0 ? nslot : 1, -1);
   for (int64_t t = 0, s = 0; t < plan.nstrands; ++t) {
      const int64_t b = starts[t], e = starts[t + 1];
      for (int64_t s0 = b; s0 < e; s0 += 32, ++s) {
         for (int64_t rho = s0; rho < std::min(e, s0 + 32); ++rho) {
            int32_t kb, ke;
            dep_range(rho, kb, ke);
            for (int32_t k = kb; k < ke; ++k) {
               const int64_t slot = seg_off[s] + (int64_t)(k - kb) * 32 + (rho - s0);
               slc[slot] = col[k];
               sls[slot] = k;
            }
         }
      }
   }
   plan.nseg = (int64_t)seg_off.size() - 1;
   // ring reads of the solve sweeps: a segment of strand t (not the first
   // of its band) reads the previous strand's rows from the ring when the
   // lowest of the rows its register slots need is within half the ring of
   // the highest row needed by it or an earlier segment of the strand; keep
   // is the suffix minimum of the lowest such row over the strand's segments
   {
      const int ns = plan.wmax <= 4 ? 4 : 8;  // register slots of the launch
      std::vector<int32_t> keep(plan.nseg > 0 ? plan.nseg : 1, INT32_MAX);
      for (int64_t t = 0, s = 0; t < plan.nstrands; ++t) {
         const int64_t b = starts[t], e = starts[t + 1];
         const int64_t s_first = s;
         int64_t run_need = -1;
         for (int64_t s0 = b; s0 < e; s0 += 32, ++s) {
            if (t % kBandWarps == 0) continue;
            const int64_t pb = starts[t - 1];
            int64_t need = -1, low = INT64_MAX;
            for (int64_t rho = s0; rho < std::min(e, s0 + 32); ++rho) {
               int32_t kb, ke;
               dep_range(rho, kb, ke);
               for (int32_t k = kb; k < ke && k - kb < ns; ++k) {
                  const int64_t l = fwd ? col[k] : n - 1 - col[k];
                  if (l >= pb && l < b) {
                     need = std::max(need, l);
                     low = std::min(low, l);
                  }
               }
            }
            run_need = std::max(run_need, need);
            if (need >= 0 && run_need - low < kRing / 2) keep[s] = (int32_t)low;
         }
         for (int64_t q = s - 2; q >= s_first; --q) keep[q] = std::min(keep[q], keep[q + 1]);
      }
      plan.seg_keep.alloc(keep.size());
      plan.seg_keep.upload(keep.data(), keep.size());
   }
   plan.tseg.alloc(tseg.size());
   plan.tseg.upload(tseg.data(), tseg.size());
   plan.seg_off.alloc(seg_off.size());
   plan.seg_off.upload(seg_off.data(), seg_off.size());
   plan.sl_col.alloc(slc.size());
   plan.sl_col.upload(slc.data(), slc.size());
   plan.sl_src.alloc(sls.size());
   plan.sl_src.upload(sls.data(), sls.size());
   plan.sl_val.alloc(sls.size());
   OFG_CUDA(cudaStreamSynchronize(stream()));
}

void fill_slot_values(ofg_matrix* A, SweepPlan& plan)
{
   const int64_t total = plan.sl_val.n;
   slot_values<<<grid_for(total, 256), 256, 0, stream()>>>(total, plan.sl_src.p, A->val.p,
                                                           plan.sl_val.p);
   count_launch();
   OFG_LAUNCH_CHECK();
}

SolveArgs solve_args(ofg_prec* P, const SweepPlan& plan)
{
   SolveArgs g{};
   g.n = P->A->n;
   g.tseg = plan.tseg.p;
   g.seg_off = plan.seg_off.p;
   g.seg_keep = plan.seg_keep.p;
   g.sl_col = plan.sl_col.p;
   g.sl_val = plan.sl_val.p;
   g.piv = P->pivot.p;
   g.sstart = plan.start.p;
   g.nstrands = plan.nstrands;
   g.ticket = plan.ticket.p;
   g.strand_dot = plan.strand_dot.p;
   g.status = P->status.p;
   return g;
}

template <int MODE>
void launch_solve(ofg_prec* P, SweepPlan& plan, SolveArgs g)
{
   if (!plan.nstrands) return;
   OFG_CUDA(cudaMemsetAsync(plan.ticket.p, 0, 4 * sizeof(int), stream()));
   int blocks = (int)std::min<int64_t>((plan.nstrands + kBandWarps - 1) / kBandWarps,
                                       (int64_t)P->solve_grid);
   if (blocks < 1) blocks = 1;
   g.worked = prof_begin();
   // register slots sized to the plan's widest segment
   if (plan.wmax <= 4) solve_sweep<MODE, 4><<<blocks, kBandWarps * 32, 0, stream()>>>(g);
   else solve_sweep<MODE, 8><<<blocks, kBandWarps * 32, 0, stream()>>>(g);
   // algorithmic bytes: one triangle of the off-diagonal entries (FP64 value
   // + int32 column), the pivots, the input, the output and the reset
   const ofg_matrix* A = P->A;
   prof_end(PROF_SWEEP, 6.0 * (double)(A->nnz - A->n) + 32.0 * (double)A->n);
   count_launch();
   OFG_LAUNCH_CHECK();
}

SweepArgs base_args(ofg_prec* P, const SweepPlan& plan)
{
   ofg_matrix* A = P->A;
   SweepArgs g{};
   g.n = A->n;
   g.rp = A->row_ptr.p;
   g.col = A->col.p;
   g.val = A->val.p;
   g.dpos = A->dpos.p;
   g.tpos = P->tpos.p;
   g.piv = P->pivot.p;
   g.sstart = plan.start.p;
   g.nstrands = plan.nstrands;
   g.ticket = plan.ticket.p;
   g.strand_dot = plan.strand_dot.p;
   g.status = P->status.p;
   return g;
}

template <int MODE>
void launch_sweep(ofg_prec* P, SweepPlan& plan, SweepArgs g)
{
   if (!plan.nstrands) return;
   OFG_CUDA(cudaMemsetAsync(plan.ticket.p, 0, 4 * sizeof(int), stream()));
   int blocks = (int)std::min<int64_t>((plan.nstrands + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                       (int64_t)P->grid);
   if (blocks < 1) blocks = 1;
   g.worked = prof_begin();
   sweep_kernel<MODE><<<blocks, kWarpsPerBlock * 32, 0, stream()>>>(g);
   prof_end(PROF_SWEEP, 0.0);
   count_launch();
   OFG_LAUNCH_CHECK();
}

}  // namespace

void check_status(ofg_prec* P)
{
   if (P->type != OFG_DILU && P->type != OFG_ILU && P->type != OFG_SSOR) return;
   int h = 0;
   P->status.download(&h, 1);
   if (h) {
      P->status.zero();
      throw Error(OFG_ERR_TIMEOUT, "triangular sweep wait ran out (status " + std::to_string(h) + ")");
   }
}

void prec_setup(ofg_prec* P)
{
   ofg_matrix* A = P->A;
   const int64_t n = A->n;
   ensure_dpos(A);
   OFG_REQUIRE(A->dpos_complete || P->type == OFG_IDENT, OFG_ERR_PIVOT,
               "a row has no diagonal entry");
   P->version = A->version;
   if (P->type == OFG_IDENT) return;
   if (P->type == OFG_LEARNED) {
      learned_setup(P);
      return;
   }
   P->pivot.reserve(n > 0 ? n : 1);
   DBuf<int> bad(1);
   int big = INT32_MAX;
   bad.upload(&big, 1);
   const int invert = (P->type == OFG_SSOR) ? 0 : 1;
   if (n) {
      diag_setup<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->dpos.p, A->val.p, P->pivot.p, invert,
                                                         bad.p);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   int h = 0;
   bad.download(&h, 1);
   if (h != INT32_MAX)
      throw Error(OFG_ERR_PIVOT, "zero pivot detected in row " + std::to_string(h + 1));
   if (P->type == OFG_DIAG) return;

   if (!P->fwd.start.p) {
      int per_sm = 0;
      OFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<FWD_DILU>,
                                                             kWarpsPerBlock * 32, 0));
      P->grid = std::max(1, per_sm) * num_sms();
      OFG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, solve_sweep<FWD_DILU, 8>,
                                                             kBandWarps * 32, 0));
      P->solve_grid = std::max(1, per_sm) * num_sms();
      build_plan(A, true, P->fwd);
      build_plan(A, false, P->bwd);
      P->status.alloc(1);
      P->t.alloc(n > 0 ? n : 1);
      P->dot.alloc(1);
   }
   P->status.zero();
   fill_sentinel(P->t.p, n);
   fill_slot_values(A, P->fwd);
   fill_slot_values(A, P->bwd);
   if (P->type == OFG_DILU || P->type == OFG_ILU) {
      if (!P->tpos.p) {
         P->tpos.alloc(A->nnz > 0 ? A->nnz : 1);
         if (n) {
            transpose_positions<<<grid_for(n, 256), 256, 0, stream()>>>(n, A->row_ptr.p, A->col.p,
                                                                        A->dpos.p, P->tpos.p);
            count_launch();
            OFG_LAUNCH_CHECK();
         }
      }
      // pivots = 1/(a_ll - sum a_li pinv_i a_il), rows in natural order
      fill_sentinel(P->pivot.p, n);
      SweepArgs g = base_args(P, P->fwd);
      g.out = P->pivot.p;
      launch_sweep<FACTOR>(P, P->fwd, g);
      check_status(P);
   }
}

void prec_apply_device(ofg_prec* P, const double* r, double* z, double* rz, const int* skip)
{
   const int64_t n = P->A->n;
   if (!n) return;
   switch (P->type) {
      case OFG_IDENT:
         if (z != r) {
            OFG_REQUIRE(!skip, OFG_ERR_ARG, "IDENT copy cannot be skipped on the device");
            OFG_CUDA(cudaMemcpyAsync(z, r, n * sizeof(double), cudaMemcpyDeviceToDevice, stream()));
         }
         return;
      case OFG_DIAG:
         diag_apply<<<grid_for(n, 256), 256, 0, stream()>>>(n, P->pivot.p, r, z, skip);
         count_launch();
         OFG_LAUNCH_CHECK();
         return;
      case OFG_LEARNED: learned_apply(P, r, z, rz, skip); return;
      default: break;
   }
   const bool dilu = (P->type != OFG_SSOR);
   // forward: t = L-solve(r); clears z for the backward sweep
   SolveArgs f = solve_args(P, P->fwd);
   f.in = r;
   f.out = P->t.p;
   f.reset = z;
   f.skip = skip;
   if (dilu) launch_solve<FWD_DILU>(P, P->fwd, f);
   else launch_solve<FWD_SSOR>(P, P->fwd, f);
   // backward: z = U-solve(t); clears t for the next application
   SolveArgs b = solve_args(P, P->bwd);
   b.in = P->t.p;
   b.out = z;
   b.reset = P->t.p;
   b.skip = skip;
   if (rz && r != z) {
      b.dot_with = r;
      b.dot_out = rz;
   }
   if (dilu) launch_solve<BWD_DILU>(P, P->bwd, b);
   else launch_solve<BWD_SSOR>(P, P->bwd, b);
}

}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_prec_create(ofg_matrix* A, int type, ofg_prec** out)
{
   return guarded("ofg_prec_create", [&] {
      OFG_REQUIRE(A && out, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(type >= OFG_IDENT && type <= OFG_SSOR, OFG_ERR_ARG, "unknown preconditioner");
      auto P = new ofg_prec();
      P->A = A;
      P->type = type;
      try {
         prec_setup(P);
      }
      catch (...) {
         delete P;
         throw;
      }
      *out = P;
   });
}

int ofg_prec_destroy(ofg_prec* P)
{
   return guarded("ofg_prec_destroy", [&] {
      delete P;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_prec_update(ofg_prec* P)
{
   return guarded("ofg_prec_update", [&] {
      OFG_REQUIRE(P, OFG_ERR_ARG, "null preconditioner");
      prec_setup(P);
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_prec_freeze(ofg_prec* P, int on)
{
   return guarded("ofg_prec_freeze", [&] {
      OFG_REQUIRE(P, OFG_ERR_ARG, "null preconditioner");
      P->frozen = on != 0;
   });
}

int ofg_prec_apply(ofg_prec* P, const double* b, double* x)
{
   return guarded("ofg_prec_apply", [&] {
      OFG_REQUIRE(P && b && x, OFG_ERR_ARG, "null argument");
      if (prec_stale(P)) prec_setup(P);
      const int64_t n = P->A->n;
      In<double> db(b, n);
      InOut<double> dx(x, n, false);
      prec_apply_device(P, db.d, dx.d);
      dx.finish();
      check_status(P);
   });
}

int ofg_selftest_wait(void)
{
   return guarded("ofg_selftest_wait", [&] {
      DBuf<double> cell(2);
      DBuf<int> status(1);
      status.zero();
      fill_sentinel(cell.p, 1);
      wait_selftest<<<1, 32, 0, stream()>>>(cell.p, status.p, cell.p + 1);
      count_launch();
      OFG_LAUNCH_CHECK();
      int h = 0;
      status.download(&h, 1);
      if (h) throw Error(OFG_ERR_TIMEOUT, "the bounded wait ran out, as intended");
      throw Error(OFG_ERR_ARG, "the wait ended without its value");
   });
}

int ofg_prec_get_pivot(const ofg_prec* P, double* pivot)
{
   return guarded("ofg_prec_get_pivot", [&] {
      OFG_REQUIRE(P && pivot, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(P->type != OFG_IDENT, OFG_ERR_ARG, "IDENT has no pivots");
      OFG_CUDA(cudaMemcpyAsync(pivot, P->pivot.p, P->A->n * sizeof(double), cudaMemcpyDefault,
                               stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

}  // extern "C"
