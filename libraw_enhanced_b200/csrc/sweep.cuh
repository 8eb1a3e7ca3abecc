// sweep.cuh -- in-order (Gauss-Seidel) sweeps over an image on the GPU.
//
// Several demosaic passes of the reference rewrite a plane in place while
// reading neighbours that the same row-major loop has already rewritten
// (DCB's nyquist, pp, refinement clamp and last color_full loop; AAHD's
// hot-pixel pass and direction refinement).  Their result is defined by that
// order.  k_gs_sweep reproduces it exactly:
//   * a warp owns a band of 32 rows (lane = row) and walks the columns with
//     a skew of SKEW columns per row (per PAIR rows), so every neighbour that
//     precedes a site in row-major order is already updated and every one
//     that follows is not;
//   * the band's rows, its halo rows and the read-only inputs are staged
//     through a shared-memory ring of kRing columns; the next group's columns
//     are copied with cp.async while the current group runs;
//   * bands are chained through per-band progress counters in global memory
//     (release by the band above after its stores, acquire by the band below
//     before it stages the upper halo); band numbers are handed out in CTA
//     start order by an atomic ticket, so a band only waits for one that is
//     already running;
//   * every wait is bounded: on time-out the kernel raises an error flag and
//     stops waiting, and the host reports the failure.
// An op supplies NS state planes + inputs (NP planes per warp), HALO, SKEW,
// PAIR, NCH (independent channels run as separate warps), LAG (how many
// columns behind its walk position a cell may still write), RING (ring
// columns, a power of two) and a cell(t, r, c, g) that updates the site
// (r, c) through the ring accessor t.
#pragma once

#include <climits>
#include <string>

#include "common.cuh"
#include "lre_internal.h"

namespace lre {
namespace {

constexpr int kRing = 128;  // default shared-memory ring width in columns (power of two)

struct Geo {
  int W, H;
  uint32_t filters;
  float maxv;
  const float* aux;  // optional device scalars an op reads (nullptr when unused)
  __device__ __forceinline__ unsigned fc(int r, int c) const { return fcol3((unsigned)r, (unsigned)c, filters); }
  __device__ __forceinline__ size_t at(int r, int c) const { return (size_t)r * W + c; }
};

// 2D launch helper: (32 x 8) threads, grid-strided in y.  Along x a block
// covers 64 columns and each thread takes two of them of the same parity in
// two half-passes (lane l: columns 2l, then 2l + 1), so the 32 lanes of a
// warp see one Bayer colour at a time and do not diverge on it.  Launch with
// (W + 63) / 64 blocks in x.
#define GS_FOR_PIXELS(g)                                                                        \
  for (int r = blockIdx.y * blockDim.y + threadIdx.y; r < (g).H; r += gridDim.y * blockDim.y)   \
    for (int gs_half = 0; gs_half < 2; gs_half++)                                                \
      for (int c = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + gs_half; c < (g).W;             \
           c += 2 * gridDim.x * blockDim.x)

struct SweepArgs {
  float* plane[4];  // state planes first, then read-only inputs
  Geo g;
  int r_lo, r_hi, c_lo, c_hi;  // updated rectangle (inclusive)
  int* ticket;
  int* err;
  int* progress;  // per band: columns < progress[b] of band b are final in HBM
  const int* skip_if_zero;  // optional: every band returns at once when *skip_if_zero == 0
  long long wait_cycles;    // bound of one wait for the band above (SM clock cycles)
  int hold_ticket;          // fault injection: this band never publishes (-1: none)
};

// The sweep's shared-memory ring, addressed through the __shared__ symbol
// itself so every access compiles to a shared-memory instruction.
extern __shared__ float sweep_smem[];

template <int NP, int HALO, int PAD, int RING>
struct Ring {
  static constexpr int ROWS = 32 + 2 * HALO;
  static constexpr int PITCH = RING + PAD;
  static constexpr int PLANE = ROWS * PITCH;
  static constexpr size_t BYTES = (size_t)NP * PLANE * sizeof(float);
  int rbase;
  __device__ __forceinline__ float& operator()(int p, int r, int c) const {
    return sweep_smem[p * PLANE + (r - rbase) * PITCH + (c & (RING - 1))];
  }
};

// Row padding so the 32 lanes of a step hit 32 different banks: lane l
// reads row l + k at column t - SKEW * (l / PAIR), so with PAIR = 1 a pitch
// of SKEW + 1 (mod 32) gives bank l + const; with PAIR = 2 and an odd SKEW a
// pitch of 16 (mod 32) gives bank (32 - SKEW) * (l / 2) + 16 * (l & 1) +
// const, 32 distinct banks.
template <class Op>
using RingOf = Ring<Op::NP, Op::HALO, (Op::PAIR == 2 ? 16 : Op::SKEW + 1), Op::RING>;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr long long kWaitCycles = 4000000000LL;  // default wait bound: ~2 s at 1.9 GHz

__device__ __forceinline__ void cp_async4(float* s, const float* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Steps per group.  Each group first makes the columns it needs resident
// (copies issued one group earlier), then issues the copies for the next
// group, then runs its GS steps while those copies are in flight.
constexpr int kGroup = 16;

// Groups staged ahead of the one being computed.
constexpr int kAhead = 1;
// Warps per CTA: one runs the steps, three move data.
constexpr int kSweepWarps = 4;

// One CTA per band (and channel), four warps:
//   * warp 0 runs the GS-step groups, touching only shared memory;
//   * warp 1 handles the band boundaries: in iteration g (while warp 0 runs
//     group g) it flushes the columns that became final with group g - 1,
//     publishes them at once (a release after the stores), then waits for
//     the band above as far as group g + kAhead needs and loads those
//     upper-halo rows into the ring;
//   * warps 2 and 3 copy group g + kAhead's band-local rows and inputs with
//     cp.async and wait for them.
// The warps meet at a named barrier once per group, so global-memory latency
// overlaps the steps.  Ring capacity: a group reads columns down to
// t0 - SPAN - HALO - LAG while the copies reach t0 + (kAhead + 1) * GS + HALO.
template <class Op>
__global__ void __launch_bounds__(kSweepWarps * 32) k_gs_sweep(SweepArgs a) {
  using R = RingOf<Op>;
  constexpr int HALO = Op::HALO, NS = Op::NS, NP = Op::NP, NCH = Op::NCH, GS = kGroup;
  constexpr int SPAN = Op::SKEW * (31 / Op::PAIR);  // column lag of lane 31 behind lane 0
  static_assert((kAhead + 1) * GS + SPAN + 2 * HALO + Op::LAG <= Op::RING, "sweep ring too small for this op");
  if (a.skip_if_zero && *a.skip_if_zero == 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, lc = lane & 15, lr = lane >> 4;
  __shared__ int s_ticket;
  if (threadIdx.x == 0) s_ticket = atomicAdd(a.ticket, 1);
  __syncthreads();
  // Tickets go out in CTA start order; ticket k is band k / NCH, channel
  // k % NCH, and waits only for ticket k - NCH (same channel, band above).
  const int ticket = s_ticket;
  const int band = ticket / NCH, ch = ticket % NCH;
  const int r0 = a.r_lo + band * 32;
  const int W = a.g.W, H = a.g.H;
  const R t{r0 - HALO};
  const int t_end = a.c_hi + SPAN;
  const int ngroups = (t_end - a.c_lo) / GS + 1;
  auto group_barrier = []() { asm volatile("bar.sync 1, %0;" ::"n"(kSweepWarps * 32) : "memory"); };

  if (warp == 0) {
    const int r = r0 + lane;
    const bool row_on = r <= a.r_hi;
    __syncthreads();  // prologue staged
    for (int g = 0; g < ngroups; g++) {
      const int t0 = a.c_lo + g * GS;
#pragma unroll 4
      for (int s = 0; s < GS; s++) {
        const int c = t0 + s - Op::SKEW * (lane / Op::PAIR);
        if (row_on && c >= a.c_lo && c <= a.c_hi) Op::cell(t, r, c, a.g);
        __syncwarp();
      }
      group_barrier();
    }
    return;
  }

  // ---- data movement
  // Per-CTA plane pointers (with NCH = 2 the argument holds
  // {state ch0, state ch1, input ch0, input ch1}).
  const float* src[NP];
  float* dst[NS];
#pragma unroll
  for (int p = 0; p < NP; p++) {
    if (NCH == 1) src[p] = a.plane[p];
    else src[p] = p < NS ? (ch ? a.plane[1] : a.plane[0]) : (ch ? a.plane[3] : a.plane[2]);
  }
#pragma unroll
  for (int p = 0; p < NS; p++) dst[p] = NCH == 1 ? a.plane[p] : (ch ? a.plane[1] : a.plane[0]);
  const int st_r0 = max(r0 - HALO, 0), st_r1 = min(r0 + 31 + HALO, H - 1);
  const int out_r1 = min(r0 + 31, a.r_hi);
  const int c_stop = a.c_hi + HALO + 1;  // staging never reaches past this column
  // Rows above r0 belong to the band above: its state planes are read by
  // warp 1 only after that band has published the columns, with L2-coherent
  // loads.  Everything else is band-local or read-only and goes through
  // warps 2 and 3.
  auto upper = [&](int p, int rr) { return band > 0 && p < NS && rr < r0; };
  int staged = a.c_lo - HALO;

  if (warp >= 2) {
    const int sub = warp - 2;  // rows st_r0 + 2 * sub + lr, step 4
    auto stage_local = [&](int hi) {
      hi = min(hi, c_stop);
      if (hi <= staged) return;
#pragma unroll
      for (int p = 0; p < NP; p++)
        for (int c = staged + lc; c < hi; c += 16)
          for (int rr = st_r0 + 2 * sub + lr; rr <= st_r1; rr += 4)
            if (!upper(p, rr)) cp_async4(&t(p, rr, c), src[p] + (size_t)rr * W + c);
      staged = hi;
    };
    stage_local(a.c_lo + kAhead * GS + HALO);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    for (int g = 0; g < ngroups; g++) {
      const int t0 = a.c_lo + g * GS;
      stage_local(t0 + (kAhead + 1) * GS + HALO);
      cp_async_commit();
      asm volatile("cp.async.wait_group %0;" ::"n"(kAhead - 1) : "memory");  // group g + 1 resident
      group_barrier();
    }
    cp_async_wait_all();
    return;
  }

  // ---- warp 1: band boundaries
  int flushed = a.c_lo, published = a.c_lo;
  bool waiting = band > 0;
  int above = 0;
  // Progress of the band above as last observed by lane 0 (acquire loads;
  // the shuffle after the wait orders every lane's later loads).
  auto wait_above = [&](int need) {
    if (!waiting) return;
    int ok = 1;
    if (lane == 0 && above < need) {
      const long long start = clock64();
      while ((above = ld_acquire(a.progress + ticket - NCH)) < need) {
        __nanosleep(32);
        if (clock64() - start > a.wait_cycles) {
          atomicExch(a.err, 1);
          ok = 0;
          break;
        }
      }
    }
    if (!__shfl_sync(0xffffffffu, ok, 0)) waiting = false;
  };
  // Upper-halo rows of the band above, read once it has published them.
  auto stage_upper = [&](int hi) {
    hi = min(hi, c_stop);
    if (hi <= staged) return;
    if (band > 0) {
      wait_above(min(hi, a.c_hi + 1));
#pragma unroll
      for (int p = 0; p < NS; p++)
        for (int c = staged + lc; c < hi; c += 16)
          for (int rr = st_r0 + lr; rr < r0; rr += 2) t(p, rr, c) = __ldcg(src[p] + (size_t)rr * W + c);
    }
    staged = hi;
  };
  auto flush = [&](int hi) {
    if (hi <= flushed) return;
#pragma unroll
    for (int p = 0; p < NS; p++)
      for (int c = flushed + lc; c < hi; c += 16)
        for (int rr = r0 + lr; rr <= out_r1; rr += 2) __stcg(dst[p] + (size_t)rr * W + c, t(p, rr, c));
    flushed = hi;
  };
  // Release by lane 0 after a warp barrier, so it covers every lane's stores.
  auto publish = [&](int upto) {
    if (upto <= published) return;
    __syncwarp();
    if (lane == 0 && ticket != a.hold_ticket) st_release(a.progress + ticket, upto > a.c_hi ? INT_MAX : upto);
    published = upto;
  };

  stage_upper(a.c_lo + kAhead * GS + HALO);
  __syncwarp();
  __syncthreads();
  for (int g = 0; g < ngroups; g++) {
    const int t0 = a.c_lo + g * GS;
    flush(min(t0 - SPAN - Op::LAG, a.c_hi + 1));
    publish(flushed);
    stage_upper(t0 + (kAhead + 1) * GS + HALO);
    __syncwarp();
    group_barrier();
  }
  flush(a.c_hi + 1);
  publish(flushed);
}

template <class Op>
lre_status sweep(Context* c, const SweepArgs& base, int* sync, int nb_max, const char* what) {
  if (base.r_hi < base.r_lo || base.c_hi < base.c_lo) return LRE_OK;
  using R = RingOf<Op>;
  const int nb = (base.r_hi - base.r_lo + 32) / 32 * Op::NCH;
  if (nb > nb_max) return fail(c, LRE_ERR_CUDA, std::string(what) + ": band table too small");
  SweepArgs a = base;
  a.ticket = sync;
  a.progress = sync + 64;
  a.wait_cycles = c->sweep_wait_cycles > 0 ? c->sweep_wait_cycles : kWaitCycles;
  // a held band (host-side fault injection, one sweep only) never reports
  // its progress, so the band below it waits until its bound runs out
  a.hold_ticket = c->sweep_hold_band >= 0 ? c->sweep_hold_band * Op::NCH : -1;
  c->sweep_hold_band = -1;
  LRE_CUDA_TRY(c, cudaMemsetAsync(sync, 0, sizeof(int), c->stream));
  LRE_CUDA_TRY(c, cudaMemsetAsync(a.progress, 0, (size_t)nb * sizeof(int), c->stream));
  LRE_CUDA_TRY(c, cudaFuncSetAttribute(k_gs_sweep<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R::BYTES));
  k_gs_sweep<Op><<<nb, kSweepWarps * 32, R::BYTES, c->stream>>>(a);
  count_launch(c);
  return check_launch(c, what);
}

bool bayer_2x2(uint32_t filters) {
  // DCB's loops address non-green sites by column parity; that is the
  // reference's intent only for 2x2 Bayer layouts with green on a
  // checkerboard and R/B on the other two sites.
  for (unsigned r = 0; r < 8; r++) {
    const unsigned a = fcol3(r, 0, filters), b = fcol3(r, 1, filters);
    if ((a == 1) == (b == 1)) return false;
    if (fcol3(r, 2, filters) != a || fcol3((r + 2) & 7, 0, filters) != a || fcol3((r + 2) & 7, 1, filters) != b)
      return false;
  }
  const unsigned n0 = fcol3(0, 0, filters) == 1 ? fcol3(0, 1, filters) : fcol3(0, 0, filters);
  const unsigned n1 = fcol3(1, 0, filters) == 1 ? fcol3(1, 1, filters) : fcol3(1, 0, filters);
  if (fcol3(0, 0, filters) == 1 && fcol3(1, 0, filters) == 1) return false;
  return n0 + n1 == 2 && n0 != n1;
}

constexpr int kSyncInts = 64;  // ticket, error flag, then per-band progress


}  // namespace
}  // namespace lre
