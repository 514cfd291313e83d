// egpu_batch.cu -- batched mixed-precision solver: many independent systems, one
// persistent launch per chunk of inner iterations, FP64 refinement between chunks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "egpu_batch.cuh"
#include "egpu_solve.h"

namespace egpu {

// ------------------------------------------------------------------------------------
// device helpers

__device__ __forceinline__ float bprec(float v, float d, int precond) {
  return (precond == EGPU_PREC_DIAGONAL && fabsf(d) > (float)EGPU_AEPS) ? v / d : v;
}

// block-wide: compact systems whose status is in the mask, prefix their slice counts
__device__ void batch_compact(const BatchArgs &a, BatchShared &sh, unsigned mask) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int base = 0, tot = 0;
    for (int c = 0; c < a.nsys; c += 32) {
      const int s = c + lane;
      const bool on = s < a.nsys && ((mask >> sh.status[s]) & 1u);
      const int ns = on ? a.sys[s].nslices : 0;
      const unsigned bal = __ballot_sync(0xffffffffu, on);
      const int pos = base + __popc(bal & ((1u << lane) - 1u));
      // inclusive scan of ns over the lanes that are on
      int v = ns;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += t;
      }
      if (on) {
        sh.act[pos] = s;
        sh.pre[pos] = tot + v - ns;
      }
      tot += __shfl_sync(0xffffffffu, v, 31);
      base += __popc(bal);
    }
    if (lane == 0) {
      sh.nact = base;
      sh.pre[base] = tot;
      sh.total = tot;
    }
  }
  __syncthreads();
}

// iterate this block's share of the active slices: f(act_index, sys, slice)
template <typename F>
__device__ __forceinline__ void batch_slices(const BatchShared &sh, F &&f) {
  const int total = sh.total, nb = gridDim.x;
  const int lo = (int)((long long)total * blockIdx.x / nb), hi = (int)((long long)total * (blockIdx.x + 1) / nb);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int a = 0;
  for (int q = lo + warp; q < hi; q += nw) {
    // act index containing slice rank q (pre is ascending; warps move forward)
    int l = 0, r = sh.nact - 1;
    while (l < r) {
      const int m = (l + r + 1) >> 1;
      if (sh.pre[m] <= q)
        l = m;
      else
        r = m - 1;
    }
    a = l;
    f(a, sh.act[a], q - sh.pre[a]);
  }
}

// For the SpMV phases, lane 0 of a warp prefetches into L2 the values and column offsets of
// the slices the warp takes next (one bulk request each; slices start at multiples of 32
// entries, so both requests are 16-byte aligned and sized) while the current ones are
// summed; the next slices' positions are loaded a round earlier still, so the requests never
// wait for them.  Slices of systems that do not run are not prefetched.
struct SliceMeta {
  const void *vals, *cols;
  unsigned vbytes, cbytes;
};

__device__ __forceinline__ int batch_locate(const BatchShared &sh, int q) {
  int l = 0, r = sh.nact - 1;
  while (l < r) {
    const int m = (l + r + 1) >> 1;
    if (sh.pre[m] <= q)
      l = m;
    else
      r = m - 1;
  }
  return l;
}

__device__ __forceinline__ SliceMeta batch_slice_meta(const BatchArgs &ba, const BatchShared &sh, int q, int hi,
                                                      unsigned run) {
  SliceMeta m{nullptr, nullptr, 0u, 0u};
  if (q >= hi) return m;
  const int a = batch_locate(sh, q);
  const int s = sh.act[a];
  if (!((run >> sh.status[s]) & 1u)) return m;
  const SysDesc &d = ba.sys[s];
  const int sl = q - sh.pre[a];
  if (sl < 0 || sl >= d.nslices) return m;
  const int p = __ldg(d.sell_ptr + sl), w = __ldg(d.sell_w + sl);
  if (w <= 0) return m;
  m.vals = d.svals + p;
  m.vbytes = (unsigned)(32 * w * (int)sizeof(float));
  if (d.scols16) {
    m.cols = d.scols16 + p;
    m.cbytes = (unsigned)(32 * w * (int)sizeof(int16_t));
  } else {
    m.cols = d.scols + p;
    m.cbytes = (unsigned)(32 * w * (int)sizeof(int));
  }
  return m;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// flush this block's per-system partials (slots v0/v1 of red) to the global accumulators
__device__ __forceinline__ void batch_flush(const BatchArgs &a, BatchShared &sh, int slot0, int slot1, int slot2 = -1,
                                            int slot3 = -1) {
  __syncthreads();
  const int slot[4] = {slot0, slot1, slot2, slot3};
  for (int t = threadIdx.x; t < sh.nact; t += blockDim.x) {
    const int s = sh.act[t];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double x = sh.red[4 * t + v];
      if (x != 0.0 && slot[v] >= 0) atomicAdd(&a.acc[slot[v] * BATCH_MAX_SYS + s], x);
      sh.red[4 * t + v] = 0.0;
    }
  }
  __syncthreads();
}

// CG accumulator slot v (0 gamma, 1 delta, 2 (r, r), 3 (z, s)) of set `set` (iteration parity)
__device__ __forceinline__ int cg_slot(int set, int v) {
  return set ? BA_CG1 + v : (v == 0 ? BA_RHO : v == 1 ? BA_PQ : v == 2 ? BA_RR : BA_SS);
}

// designated block of system s clears accumulator slots
__device__ __forceinline__ void batch_clear(const BatchArgs &a, int slot) {
  for (int s = threadIdx.x; s < a.nsys; s += blockDim.x)
    if (s % gridDim.x == (int)blockIdx.x) a.acc[slot * BATCH_MAX_SYS + s] = 0.0;
}

// SELL SpMV of one slice: lane's row sum of A x
__device__ __forceinline__ float slice_spmv(const SysDesc &d, int slice, int lane, const float *x) {
  const int r = (slice << 5) + lane;
  const int w = __ldg(d.sell_w + slice);
  const int base = __ldg(d.sell_ptr + slice) + lane;
  float s = 0.f;
#pragma unroll 8
  for (int k = 0; k < w; ++k) {
    const int e = base + (k << 5);
    const float v = __ldcs(d.svals + e);
    const int c = d.scols16 ? r + (int)__ldcs(d.scols16 + e) : __ldcs(d.scols + e);
    s = fmaf(v, __ldca(x + c), s);
  }
  return s;
}

// Two slices of (possibly) different systems summed in one interleaved loop: a tet row has
// about 15 entries, so one slice alone gives each lane a short chain of dependent gathers and
// leaves the warp waiting on memory; two slices double the loads in flight.  d0 / d1 null:
// that slice does not run.  Each row sums in entry order.
__device__ __forceinline__ void slice_spmv2(const SysDesc *d0, int sl0, const float *x0, const SysDesc *d1, int sl1,
                                            const float *x1, int lane, float &y0, float &y1) {
  int w0 = 0, w1 = 0, b0 = 0, b1 = 0;
  if (d0) {
    w0 = __ldg(d0->sell_w + sl0);
    b0 = __ldg(d0->sell_ptr + sl0) + lane;
  }
  if (d1) {
    w1 = __ldg(d1->sell_w + sl1);
    b1 = __ldg(d1->sell_ptr + sl1) + lane;
  }
  const int r0 = (sl0 << 5) + lane, r1 = (sl1 << 5) + lane;
  const int wm = max(w0, w1);
  float s0 = 0.f, s1 = 0.f;
#pragma unroll 4
  for (int k = 0; k < wm; ++k) {
    if (k < w0) {
      const int e = b0 + (k << 5);
      const float v = __ldcs(d0->svals + e);
      const int c = d0->scols16 ? r0 + (int)__ldcs(d0->scols16 + e) : __ldcs(d0->scols + e);
      s0 = fmaf(v, __ldca(x0 + c), s0);
    }
    if (k < w1) {
      const int e = b1 + (k << 5);
      const float v = __ldcs(d1->svals + e);
      const int c = d1->scols16 ? r1 + (int)__ldcs(d1->scols16 + e) : __ldcs(d1->scols + e);
      s1 = fmaf(v, __ldca(x1 + c), s1);
    }
  }
  y0 = s0;
  y1 = s1;
}

// SpMV phase over this block's share of the active slices, one slice per warp at a time;
// lane 0 prefetches the next one into L2.  run: bit mask of the statuses whose systems take
// part; src(s): the vector system s multiplies; epi(act_index, s, slice, y): once per
// running slice, y the lane's row sum.  Slices of other systems are skipped (warp-uniform).
template <typename SRC, typename EPI>
__device__ __forceinline__ void batch_spmv1(const BatchArgs &ba, const BatchShared &sh, unsigned run, SRC &&src,
                                            EPI &&epi) {
  const int total = sh.total, nb = gridDim.x;
  const int lo = (int)((long long)total * blockIdx.x / nb), hi = (int)((long long)total * (blockIdx.x + 1) / nb);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  SliceMeta next = batch_slice_meta(ba, sh, lo + warp + nw, hi, run);
  for (int q = lo + warp; q < hi; q += nw) {
    const int a = batch_locate(sh, q);
    if (lane == 0 && next.vbytes) {
      prefetch_l2_bulk(next.vals, next.vbytes);
      prefetch_l2_bulk(next.cols, next.cbytes);
    }
    next = batch_slice_meta(ba, sh, q + 2 * nw, hi, run);
    const int s = sh.act[a];
    if (!((run >> sh.status[s]) & 1u)) continue;
    const int slice = q - sh.pre[a];
    epi(a, s, slice, slice_spmv(ba.sys[s], slice, lane, src(s)));
  }
}

// The same phase with two slices per warp at a time (slice_spmv2).
template <typename SRC, typename EPI>
__device__ __forceinline__ void batch_spmv2(const BatchArgs &ba, const BatchShared &sh, unsigned run, SRC &&src,
                                            EPI &&epi) {
  const int total = sh.total, nb = gridDim.x;
  const int lo = (int)((long long)total * blockIdx.x / nb), hi = (int)((long long)total * (blockIdx.x + 1) / nb);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  const int g = ba.spw == 2 ? 2 : 1, step = g * nw;  // slices a warp takes at once, and its stride
  SliceMeta n0 = batch_slice_meta(ba, sh, lo + warp + step, hi, run),
            n1 = batch_slice_meta(ba, sh, g == 2 ? lo + warp + step + nw : hi, hi, run);
  for (int q0 = lo + warp; q0 < hi; q0 += step) {
    const int q1 = g == 2 ? q0 + nw : hi;
    if (lane == 0) {
      if (n0.vbytes) {
        prefetch_l2_bulk(n0.vals, n0.vbytes);
        prefetch_l2_bulk(n0.cols, n0.cbytes);
      }
      if (n1.vbytes) {
        prefetch_l2_bulk(n1.vals, n1.vbytes);
        prefetch_l2_bulk(n1.cols, n1.cbytes);
      }
    }
    n0 = batch_slice_meta(ba, sh, q0 + 2 * step, hi, run);
    n1 = batch_slice_meta(ba, sh, g == 2 ? q1 + 2 * step : hi, hi, run);
    const int a0 = batch_locate(sh, q0), s0 = sh.act[a0], sl0 = q0 - sh.pre[a0];
    int a1 = -1, s1 = 0, sl1 = 0;
    if (q1 < hi) {
      a1 = batch_locate(sh, q1);
      s1 = sh.act[a1];
      sl1 = q1 - sh.pre[a1];
    }
    const bool run0 = (run >> sh.status[s0]) & 1u, run1 = a1 >= 0 && ((run >> sh.status[s1]) & 1u);
    if (!run0 && !run1) continue;
    float y0, y1;
    slice_spmv2(run0 ? &ba.sys[s0] : nullptr, sl0, run0 ? src(s0) : nullptr, run1 ? &ba.sys[s1] : nullptr, sl1,
                run1 ? src(s1) : nullptr, lane, y0, y1);
    if (run0) epi(a0, s0, sl0, y0);
    if (run1) epi(a1, s1, sl1, y1);
  }
}

// SPW (1 or 2, chosen by the autotuner) slices per warp; each form is its own instantiation of
// the inner kernel, so neither pays the other's registers
template <int SPW, typename SRC, typename EPI>
__device__ __forceinline__ void batch_spmv(const BatchArgs &ba, const BatchShared &sh, unsigned run, SRC &&src,
                                           EPI &&epi) {
  if (SPW == 2)
    batch_spmv2(ba, sh, run, src, epi);
  else
    batch_spmv1(ba, sh, run, src, epi);
}

// Sync-free ILU0 solves over the systems in RUN state, slots interleaved across systems:
// slot q -> system act[q % nact], position q / nact of its level order.  A row's
// dependencies sit at smaller positions of the same system, hence at smaller slots, and
// every participant takes its slots in increasing order: deadlock free.  The next slot's
// packed entries are fetched while the current one waits.
__device__ __forceinline__ bool batch_slot(const BatchArgs &a, const BatchShared &sh, long long q, int &ai, int &pos) {
  ai = (int)(q % sh.nact);
  pos = (int)(q / sh.nact);
  const int s = sh.act[ai];
  return sh.status[s] == ST_RUN && pos < a.sys[s].n;
}

template <bool LOWER, typename RHS, typename OUT>
__device__ __forceinline__ void batch_tri(const BatchArgs &a, const BatchShared &sh, int yoff, int zoff, RHS &&rhs,
                                          OUT &&out) {
  const int local = threadIdx.x >> 5;
  if (local >= a.tri_warps_per_block || sh.nact == 0) return;
  const int lane = threadIdx.x & 31;
  const int P = a.tri_warps_per_block * gridDim.x;
  int maxn = 0;
  for (int t = 0; t < sh.nact; ++t)
    if (sh.status[sh.act[t]] == ST_RUN) maxn = max(maxn, a.sys[sh.act[t]].n);
  const long long nslot = (long long)maxn * sh.nact;
  auto fetch = [&](long long q, int ai, int pos, TriRow<float> &t, float &dinv) {
    const SysDesc &d = a.sys[sh.act[ai]];
    const int *order = LOWER ? d.lower_order : d.upper_order;
    const int *ptr = LOWER ? d.lo_ptr : d.up_ptr;
    const int *cols = LOWER ? d.lo_cols : d.up_cols;
    const float *vals = LOWER ? d.lo_vals : d.up_vals;
    tri_fetch(t, pos, order, ptr, cols, vals, lane, d.n, a.err);
    dinv = LOWER ? 0.f : __ldg(d.up_dinv + pos);
    (void)q;
  };
  // first valid slot of this participant, and its successor
  long long q = local * gridDim.x + blockIdx.x;
  int ai = 0, pos = 0;
  while (q < nslot && !batch_slot(a, sh, q, ai, pos)) q += P;
  if (q >= nslot) return;
  TriRow<float> nxt;
  float dnext;
  fetch(q, ai, pos, nxt, dnext);
  while (q < nslot) {
    const TriRow<float> cur = nxt;
    const float dinv = dnext;
    const int cai = ai;
    long long qn = q + P;
    while (qn < nslot && !batch_slot(a, sh, qn, ai, pos)) qn += P;
    if (qn < nslot) fetch(qn, ai, pos, nxt, dnext);
    const int s = sh.act[cai];
    const SysDesc &d = a.sys[s];
    const int *cols = LOWER ? d.lo_cols : d.up_cols;
    const float *vals = LOWER ? d.lo_vals : d.up_vals;
    float *y = d.w + yoff * d.ldw, *z = d.w + zoff * d.ldw;
    if (cur.row >= 0) {
      float r = 0.f;
      if (LOWER && lane == 0) r = rhs(cai, s, d, cur.row);
      const float acc = tri_dot(cur, LOWER ? y : z, cols, vals, lane, a.err);
      if (lane == 0) {
        if (LOWER) {
          Sentinel<float>::publish(y + cur.row, r - acc);
        } else {
          const float yi = Sentinel<float>::wait(y + cur.row, a.err);
          const float zi = dinv * (yi - acc);
          Sentinel<float>::publish(z + cur.row, zi);
          out(cai, s, d, cur.row, zi);
        }
      }
    }
    q = qn;
  }
}

// The same with G rows per warp (TS = 32 / G lanes each), the G consecutive slots of a slot
// group.  Consecutive slots belong to different systems when at least G systems are active,
// and every dependency of a row lies at least nact slots back, so all dependencies of a
// group lie in earlier groups: a warp can wait for its G rows together (one collective poll)
// without ever waiting on itself.  With many systems each warp would otherwise take its
// slots one after another, each a full publish/observe round trip; G rows in flight per
// warp divide that chain by G.
template <bool LOWER, int G, typename RHS, typename OUT>
__device__ __forceinline__ void batch_tri_group(const BatchArgs &a, const BatchShared &sh, int yoff, int zoff,
                                                RHS &&rhs, OUT &&out) {
  constexpr int TS = 32 / G;
  constexpr int E = G >= 8 ? 4 : 2;  // entries per lane held in registers
  const int local = threadIdx.x >> 5;
  if (local >= a.tri_warps_per_block || sh.nact < G) return;
  const int lane = threadIdx.x & 31, sub = lane / TS, sl = lane % TS;
  const int P = a.tri_warps_per_block * gridDim.x;
  int maxn = 0;
  for (int t = 0; t < sh.nact; ++t)
    if (sh.status[sh.act[t]] == ST_RUN) maxn = max(maxn, a.sys[sh.act[t]].n);
  const long long nslot = (long long)maxn * sh.nact;
  const long long ngrp = (nslot + G - 1) / G;
  for (long long g = (long long)local * gridDim.x + blockIdx.x; g < ngrp; g += P) {
    const long long q = g * G + sub;
    int ai = 0, pos = 0;
    bool valid = q < nslot && batch_slot(a, sh, q, ai, pos);
    if (!__any_sync(0xffffffffu, valid)) continue;
    const int s = valid ? sh.act[ai] : 0;
    const SysDesc &d = a.sys[s];
    int row = -1, beg = 0, end = 0;
    int c[E];
    float v[E], dinv = 0.f;
#pragma unroll
    for (int u = 0; u < E; ++u) {
      c[u] = -1;
      v[u] = 0.f;
    }
    if (valid) {
      const int *order = LOWER ? d.lower_order : d.upper_order;
      const int *ptr = LOWER ? d.lo_ptr : d.up_ptr;
      const int *cols = LOWER ? d.lo_cols : d.up_cols;
      const float *vals = LOWER ? d.lo_vals : d.up_vals;
      row = __ldg(order + pos);
      beg = __ldg(ptr + pos);
      end = __ldg(ptr + pos + 1);
      if (row < 0 || row >= d.n || end < beg) {
        if (sl == 0) atomicExch(a.err, (int)EGPU_ERR_ARG);
        valid = false;
        row = -1;
      } else {
#pragma unroll
        for (int u = 0; u < E; ++u) {
          const int e = beg + sl + TS * u;
          if (e < end) {
            c[u] = __ldg(cols + e);
            v[u] = __ldg(vals + e);
            if (c[u] < 0 || c[u] >= d.n) {
              atomicExch(a.err, (int)EGPU_ERR_ARG);
              c[u] = -1;
            }
          }
        }
        if (!LOWER) dinv = __ldg(d.up_dinv + pos);
      }
    }
    float *y = valid ? d.w + yoff * d.ldw : nullptr, *z = valid ? d.w + zoff * d.ldw : nullptr;
    const float *x = LOWER ? y : z;
    float r = 0.f;
    if (LOWER && valid && sl == 0) r = rhs(ai, s, d, row);
    float xv[E];
#pragma unroll
    for (int u = 0; u < E; ++u) xv[u] = c[u] >= 0 ? Sentinel<float>::peek(x + c[u]) : 0.f;
    warp_wait_all<float, E>(xv, c, x, a.err);
    float acc = 0.f;
#pragma unroll
    for (int u = 0; u < E; ++u)
      if (c[u] >= 0) acc += v[u] * xv[u];
    if (valid) {  // rows longer than E TS entries
      const int *cols = LOWER ? d.lo_cols : d.up_cols;
      const float *vals = LOWER ? d.lo_vals : d.up_vals;
      for (int e = beg + E * TS + sl; e < end; e += TS) {
        const int cc = __ldg(cols + e);
        if (cc < 0 || cc >= d.n) {
          atomicExch(a.err, (int)EGPU_ERR_ARG);
          continue;
        }
        acc += __ldg(vals + e) * Sentinel<float>::wait(x + cc, a.err);
      }
    }
#pragma unroll
    for (int off = TS / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (valid && sl == 0) {
      if (LOWER) {
        Sentinel<float>::publish(y + row, r - acc);
      } else {
        const float yi = Sentinel<float>::wait(y + row, a.err);
        const float zi = dinv * (yi - acc);
        Sentinel<float>::publish(z + row, zi);
        out(ai, s, d, row, zi);
      }
    }
  }
}

// G rows per warp when the batch allows it (a.tri_group) and enough systems are active
template <bool LOWER, typename RHS, typename OUT>
__device__ __forceinline__ void batch_tri_any(const BatchArgs &a, const BatchShared &sh, int yoff, int zoff, RHS &&rhs,
                                              OUT &&out) {
  if (a.tri_group >= 8 && sh.nact >= 8)
    batch_tri_group<LOWER, 8>(a, sh, yoff, zoff, rhs, out);
  else if (a.tri_group >= 4 && sh.nact >= 4)
    batch_tri_group<LOWER, 4>(a, sh, yoff, zoff, rhs, out);
  else if (a.tri_group >= 2 && sh.nact >= 2)
    batch_tri_group<LOWER, 2>(a, sh, yoff, zoff, rhs, out);
  else
    batch_tri<LOWER>(a, sh, yoff, zoff, rhs, out);
}

// ------------------------------------------------------------------------------------
// the kernel

// One Jacobi sweep over the running systems' ILU0 factors (see sweep_phase in
// egpu_krylov.cuh): a warp per slice, lane = row, the entries with col < row (LOWER) or
// col > row (UPPER) of the slice's k range.  zin(s): the vector system s multiplies;
// epi(s, row, sum) for rows < n.
template <bool UPPER, typename ZIN, typename EPI>
__device__ __forceinline__ void batch_sweep(const BatchArgs &ba, const BatchShared &sh, ZIN &&zin, EPI &&epi) {
  const int total = sh.total, nb = gridDim.x;
  const int lo = (int)((long long)total * blockIdx.x / nb), hi = (int)((long long)total * (blockIdx.x + 1) / nb);
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  for (int q = lo + warp; q < hi; q += nw) {
    const int a = batch_locate(sh, q);
    const int s = sh.act[a];
    if (sh.status[s] != ST_RUN) continue;
    const SysDesc &d = ba.sys[s];
    const int slice = q - sh.pre[a];
    const int r = (slice << 5) + lane;
    const int w = __ldg(d.sell_w + slice);
    const int2 rg = __ldg(d.swr + slice);
    const int k0 = UPPER ? rg.y : 0, k1 = UPPER ? w : rg.x;
    const int base = __ldg(d.sell_ptr + slice) + lane;
    const float *z = zin(s);
    float sum = 0.f;
#pragma unroll 4
    for (int k = k0; k < k1; ++k) {
      const int e = base + (k << 5);
      const int c = d.scols16 ? r + (int)__ldcs(d.scols16 + e) : __ldcs(d.scols + e);
      const float v = __ldcs(d.isvals + e);
      const bool take = UPPER ? c > r : c < r;
      sum = fmaf(take ? v : 0.f, __ldca(z + c), sum);
    }
    if (r < d.n) epi(s, r, sum);
  }
}

// work vector `tgt` = M^-1 (work vector `src`) of every running system by ba.sweeps sweeps
// per triangle (src complete; ends without a closing grid barrier).  Scratch: work vectors
// 8, 9 (y) and 12.  Returns false when a grid barrier failed.
__device__ __forceinline__ bool batch_sweep_apply(const BatchArgs &a, const BatchShared &sh, int src, int tgt,
                                                  unsigned int &epoch) {
  const int m = a.sweeps;
  const int z0s = (m % 2 == 0) ? tgt : 12;
  int yin = src;
  for (int j = 1; j <= m; ++j) {
    const int yout = (j & 1) ? 8 : 9;
    const bool last = j == m;
    batch_sweep<false>(a, sh, [&](int s) -> const float * { return a.sys[s].w + yin * a.sys[s].ldw; },
                       [&](int s, int r, float sum) {
      const SysDesc &d = a.sys[s];
      const float y = d.w[src * d.ldw + r] - sum;
      d.w[yout * d.ldw + r] = y;
      if (last) d.w[z0s * d.ldw + r] = d.idinv[r] * y;
    });
    if (!grid_barrier(a.bar, a.err, epoch)) return false;
    yin = yout;
  }
  int zin = z0s;
  for (int j = 1; j <= m; ++j) {
    const int zout = ((m - j) % 2 == 0) ? tgt : 12;
    batch_sweep<true>(a, sh, [&](int s) -> const float * { return a.sys[s].w + zin * a.sys[s].ldw; },
                      [&](int s, int r, float sum) {
      const SysDesc &d = a.sys[s];
      d.w[zout * d.ldw + r] = d.idinv[r] * (d.w[yin * d.ldw + r] - sum);
    });
    if (j < m && !grid_barrier(a.bar, a.err, epoch)) return false;
    zin = zout;
  }
  return true;
}

template <int SPW>
__global__ void __launch_bounds__(EGPU_BLOCK, 2) k_batch_inner(BatchArgs a, int parity0) {
  __shared__ BatchShared sh;
  __shared__ double rho_s[BATCH_MAX_SYS];
  unsigned int epoch = 0;
  const int lane = threadIdx.x & 31;
  const bool bicg = a.method == EGPU_BICGSTAB;
  const bool ilu = a.precond == EGPU_PREC_ILU0;
  const float SENT = Sentinel<float>::value();
  for (int t = threadIdx.x; t < 4 * BATCH_MAX_SYS; t += blockDim.x) sh.red[t] = 0.0;
  int it = 0;
  for (; it < a.kmax; ++it) {
    const int rd = (parity0 + it) & 1, wr = rd ^ 1;
    if (threadIdx.x == 0) sh.any_done = 0;
    __syncthreads();
    // ---------------- top: decisions for every system (identical in every block)
    for (int s = threadIdx.x; s < a.nsys; s += blockDim.x) {
      SysState st = a.state[rd * BATCH_MAX_SYS + s];
      const int status0 = st.status;
      const double *acc = a.acc;
      float beta = 0.f;
      float alpha_f = 0.f;
      if (st.status == ST_INIT) {
        st.status = ST_INIT + 10;  // init work this iteration
        st.k = 0;
      } else if (!bicg) {
        // single-reduction CG: the sums of the previous iteration's phase A (set rd ^ 1)
        if (st.status == ST_INIT + 10 || st.status == ST_RUN) {
          const double g = acc[cg_slot(rd ^ 1, 0) * BATCH_MAX_SYS + s];
          const double dl = acc[cg_slot(rd ^ 1, 1) * BATCH_MAX_SYS + s];
          const double rq = a.sys[s].unit_diag ? g : acc[cg_slot(rd ^ 1, 2) * BATCH_MAX_SYS + s];
          double b = 0.0, eta = dl;
          bool go = false;
          if (st.status == ST_INIT + 10) {
            st.r0norm = sqrt(rq);
            st.k = 1;
            st.residual = 1.0;
            if (!(st.r0norm > 0.0)) {
              st.status = ST_DONE;
              st.info = EGPU_HUTI_CONVERGENCE;
              st.iters = 0;
              st.residual = 0.0;
            } else {
              // resumed: p = z + b P and s = w + b S with the carried P, S; eta formed exactly
              if (st.resume) {
                b = g / st.carry_rho;
                eta = dl + 2.0 * b * acc[cg_slot(rd ^ 1, 3) * BATCH_MAX_SYS + s] + b * b * st.eta;
              }
              st.status = ST_RUN;
              go = true;
            }
          } else {
            st.residual = sqrt(rq) / st.r0norm;
            if (st.residual <= a.tol) {
              st.status = ST_DONE;
              st.info = EGPU_HUTI_CONVERGENCE;
              st.iters = st.k;
            } else if (st.k + 1 > a.maxit) {
              st.status = ST_DONE;
              st.info = EGPU_HUTI_MAXITER;
              st.iters = st.k;
            } else {
              b = g / st.rho;
              eta = dl - b * g / st.alpha;
              st.k += 1;
              go = true;
            }
          }
          if (go && (g == 0.0 || !(eta != 0.0))) {
            st.status = ST_DONE;
            st.info = EGPU_HUTI_CG_RHO;
            st.iters = st.k;
            go = false;
          }
          if (go) {
            st.oldrho = st.rho;
            st.rho = g;
            st.alpha = g / eta;
            st.eta = eta;
            beta = (float)b;
            alpha_f = (float)st.alpha;
          }
        }
      } else if (st.status == ST_INIT + 10) {
        st.rho = acc[BA_RHO * BATCH_MAX_SYS + s];
        st.r0norm = sqrt(acc[BA_RR * BATCH_MAX_SYS + s]);
        st.k = 1;
        if (st.resume) {  // alpha, omega carried; rho_{k-1} given in the new scale
          st.oldrho = st.carry_rho;
        } else {
          st.alpha = 0.0;
          st.omega = 1.0;
          st.oldrho = 1.0;
        }
        st.residual = 1.0;
        if (!(st.r0norm > 0.0)) {
          st.status = ST_DONE;
          st.info = EGPU_HUTI_CONVERGENCE;
          st.iters = 0;
          st.residual = 0.0;
        } else {
          st.status = ST_RUN;
        }
      } else if (st.status == ST_RUN) {
        const double rho_new = acc[BA_RHO * BATCH_MAX_SYS + s];
        const double rr = acc[BA_RR * BATCH_MAX_SYS + s];
        st.residual = sqrt(rr) / st.r0norm;
        if (bicg && sqrt(acc[BA_SS * BATCH_MAX_SYS + s]) < EGPU_HUTI_EPSILON) {
          st.status = ST_DONE;
          st.info = EGPU_HUTI_BICGSTAB_SNORM;
          st.iters = st.k;
        } else if (st.residual <= a.tol) {
          st.status = ST_DONE;
          st.info = EGPU_HUTI_CONVERGENCE;
          st.iters = st.k;
        } else if (bicg && st.omega == 0.0) {
          st.status = ST_DONE;
          st.info = EGPU_HUTI_BICGSTAB_OMEGA;
          st.iters = st.k;
        } else if (st.k + 1 > a.maxit) {
          st.status = ST_DONE;
          st.info = EGPU_HUTI_MAXITER;
          st.iters = st.k;
        } else if (rho_new == 0.0) {
          st.status = ST_DONE;
          st.info = bicg ? EGPU_HUTI_BICGSTAB_RHO : EGPU_HUTI_CG_RHO;
          st.iters = st.k;
        } else {
          st.oldrho = st.rho;
          st.rho = rho_new;
          st.k += 1;
        }
      }
      if (st.status == ST_DONE && status0 != ST_DONE) sh.any_done = 1;
      if (bicg && st.status == ST_RUN) beta = (float)((st.rho * st.alpha) / (st.oldrho * st.omega));
      sh.status[s] = st.status;
      sh.fresh[s] = st.resume ? 0 : 1;
      sh.kk[s] = st.k;
      sh.sb[s] = beta;
      sh.sa[s] = bicg ? (float)st.omega : alpha_f;
      rho_s[s] = st.rho;
      if (s % gridDim.x == (int)blockIdx.x) a.state[wr * BATCH_MAX_SYS + s] = st;
    }
    __syncthreads();
    batch_compact(a, sh, (1u << ST_RUN) | (1u << (ST_INIT + 10)));
    if (sh.nact == 0) {
      ++it;
      break;
    }
    if (!bicg) {
      // ============ CG, single reduction ============
      // (A. T. Chronopoulos and C. W. Gear, "s-step iterative methods for symmetric linear
      // systems", J. Comput. Appl. Math. 25 (1989), the s = 1 case.)  The inner solve is a
      // correction equation that the FP64 refinement checks, so it is not bound to HUTI's
      // operation order.  With S = A P and W = A Z kept as vectors, both inner products of an
      // iteration come out of the pass that computes its one SpMV, and the scalars follow as
      //   beta = gamma / gamma_old,  eta = delta - beta gamma / alpha_old,  alpha = gamma / eta
      // (gamma = (R, Z), delta = (W, Z)): two phases and two grid barriers per iteration
      // instead of three.  A resumed segment forms its first eta exactly from the carried P, S:
      // eta = delta + 2 b (Z, S) + b^2 eta_old, b = gamma / carry_rho (A symmetric).
      // layout R Z P W S; this iteration sums into set rd
      // B: P = Z + beta P; S = W + beta S; X += alpha P; R -= alpha S; Z = M^-1 R
      //    (init: R = B, X = 0, Z = M^-1 R);  clear set rd
      for (int v = 0; v < 4; ++v) batch_clear(a, cg_slot(rd, v));
      batch_slices(sh, [&](int, int s, int slice) {
        const SysDesc &d = a.sys[s];
        const int r = (slice << 5) + lane;
        if (r >= d.n) return;
        float *R = d.w, *Z = d.unit_diag ? d.w : d.w + d.ldw, *P = d.w + 2 * d.ldw, *W = d.w + 3 * d.ldw,
              *S = d.w + 4 * d.ldw;
        const float *dv = d.w + 13 * d.ldw;
        float rv;
        if (sh.status[s] == ST_RUN) {
          const float be = sh.sb[s], al = sh.sa[s];
          const bool fresh1 = sh.kk[s] == 1 && sh.fresh[s];
          const float z = Z[r], w = W[r];
          const float p = fresh1 ? z : z + be * P[r];
          const float sv = fresh1 ? w : w + be * S[r];
          P[r] = p;
          S[r] = sv;
          d.x[r] = d.x[r] + al * p;
          rv = (d.unit_diag ? z : R[r]) - al * sv;
        } else {
          rv = d.b[r];
          d.x[r] = 0.f;
        }
        R[r] = rv;
        if (!d.unit_diag) Z[r] = bprec(rv, dv[r], a.precond);
      });
      if (!grid_barrier(a.bar, a.err, epoch)) return;
      // A: W = A Z; gamma = (R, Z), delta = (W, Z), (R, R), and (Z, S) for a resumed start
      batch_spmv<SPW>(a, sh, (1u << ST_RUN) | (1u << (ST_INIT + 10)),
                      [&](int s) -> const float * { const SysDesc &d = a.sys[s]; return d.unit_diag ? d.w : d.w + d.ldw; },
                      [&](int ai, int s, int slice, float w) {
        const SysDesc &d = a.sys[s];
        const int r = (slice << 5) + lane;
        const bool resume0 = sh.status[s] != ST_RUN && !sh.fresh[s];
        double g = 0.0, dl = 0.0, rq = 0.0, ep = 0.0;
        if (r < d.n) {
          const float *Z = d.unit_diag ? d.w : d.w + d.ldw;
          d.w[3 * d.ldw + r] = w;
          const float z = Z[r];
          const float rv = d.unit_diag ? z : d.w[r];
          g = (double)rv * (double)z;
          dl = (double)w * (double)z;
          if (!d.unit_diag) rq = (double)rv * (double)rv;
          if (resume0) ep = (double)z * (double)d.w[4 * d.ldw + r];
        }
        g = warp_sum(g);
        dl = warp_sum(dl);
        if (!d.unit_diag) rq = warp_sum(rq);
        if (resume0) ep = warp_sum(ep);
        if (lane == 0) {
          batch_acc_add(sh, ai, 0, g);
          batch_acc_add(sh, ai, 1, dl);
          if (!d.unit_diag) batch_acc_add(sh, ai, 2, rq);
          if (resume0) batch_acc_add(sh, ai, 3, ep);
        }
      });
      batch_flush(a, sh, cg_slot(rd, 0), cg_slot(rd, 1), cg_slot(rd, 2), cg_slot(rd, 3));
      if (!grid_barrier(a.bar, a.err, epoch)) return;
    } else {
      // ============ BiCGStab ============  layout R RT P V T S T1 T2 Y1 Y2
      // 1: P = R + beta (P - omega V); T1 = M^-1 P;  clear TS, TT
      batch_clear(a, BA_TS);
      batch_clear(a, BA_TT);
      if (ilu && a.sweeps > 0) {
        batch_slices(sh, [&](int, int s, int slice) {
          if (sh.status[s] != ST_RUN) return;
          const SysDesc &d = a.sys[s];
          const int r = (slice << 5) + lane;
          if (r >= d.n) return;
          float *R = d.w, *P = d.w + 2 * d.ldw, *V = d.w + 3 * d.ldw;
          P[r] = R[r] + sh.sb[s] * (P[r] - sh.sa[s] * V[r]);
        });
        if (!grid_barrier(a.bar, a.err, epoch)) return;
        if (!batch_sweep_apply(a, sh, 2, 6, epoch)) return;
      } else if (ilu) {
        batch_tri_any<true>(a, sh, 8, 6, [&](int, int s, const SysDesc &d, int i) {
          float *R = d.w, *P = d.w + 2 * d.ldw, *V = d.w + 3 * d.ldw;
          const float p = R[i] + sh.sb[s] * (P[i] - sh.sa[s] * V[i]);
          P[i] = p;
          return p;
        }, [&](int, int, const SysDesc &, int, float) {});
        batch_tri_any<false>(a, sh, 8, 6, [&](int, int, const SysDesc &, int) { return 0.f; },
                         [&](int, int, const SysDesc &, int, float) {});
      } else {
        batch_slices(sh, [&](int, int s, int slice) {
          if (sh.status[s] != ST_RUN) return;
          const SysDesc &d = a.sys[s];
          const int r = (slice << 5) + lane;
          if (r >= d.n) return;
          float *R = d.w, *P = d.w + 2 * d.ldw, *V = d.w + 3 * d.ldw, *T1 = d.w + 6 * d.ldw;
          const float p = R[r] + sh.sb[s] * (P[r] - sh.sa[s] * V[r]);
          P[r] = p;
          T1[r] = bprec(p, d.w[13 * d.ldw + r], a.precond);
        });
      }
      if (!grid_barrier(a.bar, a.err, epoch)) return;
      // 2: V = A T1; RV;  clear RHO, RR, SS
      batch_clear(a, BA_RHO);
      batch_clear(a, BA_RR);
      batch_clear(a, BA_SS);
      batch_spmv<SPW>(a, sh, 1u << ST_RUN, [&](int s) -> const float * { return a.sys[s].w + 6 * a.sys[s].ldw; },
                  [&](int ai, int s, int slice, float v) {
        const SysDesc &d = a.sys[s];
        const int r = (slice << 5) + lane;
        const float *RT = d.w + d.ldw;
        float *V = d.w + 3 * d.ldw;
        double rv = 0.0;
        if (r < d.n) {
          V[r] = v;
          rv = (double)RT[r] * (double)v;
        }
        rv = warp_sum(rv);
        if (lane == 0) batch_acc_add(sh, ai, 0, rv);
      });
      batch_flush(a, sh, BA_PQ, -1);
      if (!grid_barrier(a.bar, a.err, epoch)) return;
      // 3: alpha = rho / RV; S = R - alpha V; SS; T2 = M^-1 S
      for (int t = threadIdx.x; t < sh.nact; t += blockDim.x) {
        const int s = sh.act[t];
        if (sh.status[s] != ST_RUN) continue;
        const double al = rho_s[s] / a.acc[BA_PQ * BATCH_MAX_SYS + s];
        rho_s[s] = al;  // rho is not needed again in this iteration: keep alpha here
        if (s % gridDim.x == (int)blockIdx.x) a.state[wr * BATCH_MAX_SYS + s].alpha = al;
      }
      __syncthreads();
      if (ilu && a.sweeps > 0) {
        batch_slices(sh, [&](int ai, int s, int slice) {
          if (sh.status[s] != ST_RUN) return;
          const SysDesc &d = a.sys[s];
          const int r = (slice << 5) + lane;
          double ss = 0.0;
          if (r < d.n) {
            float *R = d.w, *V = d.w + 3 * d.ldw, *S = d.w + 5 * d.ldw;
            const float sv = R[r] - (float)rho_s[s] * V[r];
            S[r] = sv;
            ss = (double)sv * (double)sv;
          }
          ss = warp_sum(ss);
          if (lane == 0) batch_acc_add(sh, ai, 0, ss);
        });
        batch_flush(a, sh, BA_SS, -1);
        if (!grid_barrier(a.bar, a.err, epoch)) return;
        if (!batch_sweep_apply(a, sh, 5, 7, epoch)) return;
      } else if (ilu) {
        batch_tri_any<true>(a, sh, 9, 7, [&](int ai, int s, const SysDesc &d, int i) {
          float *R = d.w, *V = d.w + 3 * d.ldw, *S = d.w + 5 * d.ldw;
          const float sv = R[i] - (float)rho_s[s] * V[i];
          S[i] = sv;
          atomicAdd(&sh.red[4 * ai], (double)sv * (double)sv);
          return sv;
        }, [&](int, int, const SysDesc &, int, float) {});
        batch_tri_any<false>(a, sh, 9, 7, [&](int, int, const SysDesc &, int) { return 0.f; },
                         [&](int, int, const SysDesc &, int, float) {});
      } else {
        batch_slices(sh, [&](int ai, int s, int slice) {
          if (sh.status[s] != ST_RUN) return;
          const SysDesc &d = a.sys[s];
          const int r = (slice << 5) + lane;
          double ss = 0.0;
          if (r < d.n) {
            float *R = d.w, *V = d.w + 3 * d.ldw, *S = d.w + 5 * d.ldw, *T2 = d.w + 7 * d.ldw;
            const float sv = R[r] - (float)rho_s[s] * V[r];
            S[r] = sv;
            ss = (double)sv * (double)sv;
            T2[r] = bprec(sv, d.w[13 * d.ldw + r], a.precond);
          }
          ss = warp_sum(ss);
          if (lane == 0) batch_acc_add(sh, ai, 0, ss);
        });
      }
      batch_flush(a, sh, BA_SS, -1);
      if (!grid_barrier(a.bar, a.err, epoch)) return;
      // 4: T = A T2; TS, TT;  clear PQ
      batch_clear(a, BA_PQ);
      batch_spmv<SPW>(a, sh, 1u << ST_RUN, [&](int s) -> const float * { return a.sys[s].w + 7 * a.sys[s].ldw; },
                  [&](int ai, int s, int slice, float t) {
        const SysDesc &d = a.sys[s];
        const int r = (slice << 5) + lane;
        const float *S = d.w + 5 * d.ldw;
        float *T = d.w + 4 * d.ldw;
        double ts = 0.0, tt = 0.0;
        if (r < d.n) {
          T[r] = t;
          ts = (double)t * (double)S[r];
          tt = (double)t * (double)t;
        }
        ts = warp_sum(ts);
        tt = warp_sum(tt);
        if (lane == 0) {
          batch_acc_add(sh, ai, 0, ts);
          batch_acc_add(sh, ai, 1, tt);
        }
      });
      batch_flush(a, sh, BA_TS, BA_TT);
      if (!grid_barrier(a.bar, a.err, epoch)) return;
      // 5: omega = TS/TT; X += alpha T1 + omega T2; R = S - omega T; RHO, RR  (init: R = RT = B ...)
      for (int t = threadIdx.x; t < sh.nact; t += blockDim.x) {
        const int s = sh.act[t];
        if (sh.status[s] != ST_RUN) continue;
        const double ss = a.acc[BA_SS * BATCH_MAX_SYS + s];
        const double om = sqrt(ss) < EGPU_HUTI_EPSILON ? 0.0 : a.acc[BA_TS * BATCH_MAX_SYS + s] / a.acc[BA_TT * BATCH_MAX_SYS + s];
        sh.sa[s] = (float)om;
        sh.sb[s] = sqrt(ss) < EGPU_HUTI_EPSILON ? 1.f : 0.f;  // snorm exit: only x += alpha T1
        if (s % gridDim.x == (int)blockIdx.x) a.state[wr * BATCH_MAX_SYS + s].omega = om;
      }
      __syncthreads();
      batch_slices(sh, [&](int ai, int s, int slice) {
        const SysDesc &d = a.sys[s];
        const int r = (slice << 5) + lane;
        double rt_r = 0.0, rr = 0.0;
        if (r < d.n) {
          float *R = d.w, *RT = d.w + d.ldw, *P = d.w + 2 * d.ldw, *V = d.w + 3 * d.ldw, *T = d.w + 4 * d.ldw,
                *S = d.w + 5 * d.ldw, *T1 = d.w + 6 * d.ldw, *T2 = d.w + 7 * d.ldw, *Y1 = d.w + 8 * d.ldw,
                *Y2 = d.w + 9 * d.ldw;
          if (sh.status[s] == ST_RUN) {
            const float al = (float)rho_s[s], om = sh.sa[s];
            if (sh.sb[s] != 0.f) {
              d.x[r] = d.x[r] + al * T1[r];
            } else {
              d.x[r] = d.x[r] + al * T1[r] + om * T2[r];
              const float rv = S[r] - om * T[r];
              R[r] = rv;
              rt_r = (double)RT[r] * (double)rv;
              rr = (double)rv * (double)rv;
            }
          } else {  // init: R = B, X = 0; fresh: RT = B, P = V = 0 (resumed: kept)
            const float b = d.b[r];
            R[r] = b;
            d.x[r] = 0.f;
            if (sh.fresh[s]) {
              RT[r] = b;
              P[r] = 0.f;
              V[r] = 0.f;
            }
            rt_r = (double)RT[r] * (double)b;
            rr = (double)b * (double)b;
          }
          if (ilu && a.sweeps == 0) {
            T1[r] = SENT;
            T2[r] = SENT;
            Y1[r] = SENT;
            Y2[r] = SENT;
          }
        }
        rt_r = warp_sum(rt_r);
        rr = warp_sum(rr);
        if (lane == 0) {
          batch_acc_add(sh, ai, 0, rt_r);
          batch_acc_add(sh, ai, 1, rr);
        }
      });
      batch_flush(a, sh, BA_RHO, BA_RR);
      if (!grid_barrier(a.bar, a.err, epoch)) return;
    }
    // latency mode: hand a finished system back to the host at once (its refinement and
    // retirement happen between launches); the iteration just run completes for the others
    if (a.exit_on_done && sh.any_done) {
      ++it;
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.it_done = it;
}

// ------------------------------------------------------------------------------------
// FP64 refinement kernels over a list of systems (one warp per slice)

struct RefDesc {
  int n, nslices;
  const int *sell_ptr, *sell_w, *scols;
  const double *svals;   // scaled FP64, SELL order
  const double *bs;      // scaled rhs
  double *xs;            // scaled solution
  double *r;             // FP64 residual
  float *r32, *d32;      // inner rhs / solution
  const double *D;       // DiagScaling * ||Db||
  double *x_out;         // back-scaled solution (device)
};

// r = bs - A xs, ||r||^2 per system (atomics into norms[s])
__global__ void k_batch_residual(int nsel, const int *sel, const RefDesc *rd, const int *slice_pre, double *norms) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int total = slice_pre[nsel];
  for (int q = gw; q < total; q += nw) {
    int l = 0, h = nsel - 1;
    while (l < h) {
      const int m = (l + h + 1) >> 1;
      if (slice_pre[m] <= q)
        l = m;
      else
        h = m - 1;
    }
    const int s = sel[l];
    const RefDesc &d = rd[s];
    const int slice = q - slice_pre[l];
    const int r = (slice << 5) + lane;
    const int w = d.sell_w[slice];
    const int base = d.sell_ptr[slice] + lane;
    double acc = 0.0;
    for (int k = 0; k < w; ++k) {
      const int e = base + (k << 5);
      acc = __dadd_rn(acc, __dmul_rn(d.svals[e], d.xs[d.scols[e]]));
    }
    double rr = 0.0;
    if (r < d.n) {
      const double ri = d.bs[r] - acc;
      d.r[r] = ri;
      rr = ri * ri;
    }
    rr = warp_sum(rr);
    if (lane == 0) atomicAdd(norms + s, rr);
  }
}

// r32 = r / ||r|| for systems starting an inner solve
__global__ void k_batch_cast(int nsel, const int *sel, const RefDesc *rd, const int *slice_pre, const double *norms) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int total = slice_pre[nsel];
  for (int q = gw; q < total; q += nw) {
    int l = 0, h = nsel - 1;
    while (l < h) {
      const int m = (l + h + 1) >> 1;
      if (slice_pre[m] <= q)
        l = m;
      else
        h = m - 1;
    }
    const int s = sel[l];
    const RefDesc &d = rd[s];
    const int r = ((q - slice_pre[l]) << 5) + lane;
    if (r < d.n) d.r32[r] = (float)(d.r[r] / sqrt(norms[s]));
  }
}

// xs += ||r|| d  (systems whose inner solve finished)
__global__ void k_batch_update(int nsel, const int *sel, const RefDesc *rd, const int *slice_pre, const double *rnorm) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int total = slice_pre[nsel];
  for (int q = gw; q < total; q += nw) {
    int l = 0, h = nsel - 1;
    while (l < h) {
      const int m = (l + h + 1) >> 1;
      if (slice_pre[m] <= q)
        l = m;
      else
        h = m - 1;
    }
    const int s = sel[l];
    const RefDesc &d = rd[s];
    const int r = ((q - slice_pre[l]) << 5) + lane;
    if (r < d.n) d.xs[r] += rnorm[s] * (double)d.d32[r];
  }
}

// x_out = xs * D (BackScaleLinearSystem) for finished systems
__global__ void k_batch_backscale(int nsel, const int *sel, const RefDesc *rd, const int *slice_pre) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int total = slice_pre[nsel];
  for (int q = gw; q < total; q += nw) {
    int l = 0, h = nsel - 1;
    while (l < h) {
      const int m = (l + h + 1) >> 1;
      if (slice_pre[m] <= q)
        l = m;
      else
        h = m - 1;
    }
    const int s = sel[l];
    const RefDesc &d = rd[s];
    const int r = ((q - slice_pre[l]) << 5) + lane;
    if (r < d.n) d.x_out[r] = d.xs[r] * d.D[r];
  }
}

// ------------------------------------------------------------------------------------
// Team solver (CG with M = I or Jacobi, egpu_batch_solve).  The systems are independent, so
// none needs to wait for another: each system's whole mixed-precision solve (FP64 residual,
// FP32 inner CG segments with reliable updating, FP64 update; the same sequence as
// egpu_batch_step's) runs on a team of CTAs of one cooperative launch.  A small system's team
// is one CTA, synchronised by block barriers only; a large one's is several CTAs that split
// its SELL slices and meet at a barrier of their own (one counter per system).  CTAs take
// (system, member) tasks from a queue ordered largest team first, so every team is formed
// from CTAs that are free at once and the small systems fill in behind.  Dot products: block
// sums, one partial per member, summed in member order by every member (same value in all).

constexpr int TEAM_MAX = 16;
constexpr int TEAM_BLOCK = EGPU_KBLOCK;  // threads of a team CTA
constexpr int TEAM_PER_SM = 65536 / (TEAM_BLOCK * 64);  // CTAs per SM at 64 registers a thread
enum { TS_BB = 0, TS_RHO0, TS_PQ, TS_RHO, TS_RR, TS_RES, TS_NSLOT };

struct TeamSys {
  int n, nslices, team;
  int zr;                  // Z is R: no preconditioner, or Jacobi on a diagonal that is 1.0f everywhere
  const int *sell_ptr, *sell_w;
  const int16_t *scols16;  // col - row (FP32 SpMV), or null: scols
  const int *scols;        // absolute columns
  const float *svals32, *dvals32;
  float *w32;              // R Z P Q D(inner solution), stride ldw
  long long ldw;
  const double *svals64;   // scaled FP64 values, SELL order
  const double *bs;        // scaled right-hand side
  double *xs, *r64;        // scaled solution, FP64 residual
  double bnorm_s;          // ||bs|| (1 when the right-hand side was normalised)
  unsigned int *bar;       // the team's barrier counter
  double *part;            // TS_NSLOT x team partial sums
};

struct TeamOut {
  int info, iters, refinements, pad;
  double residual;
};

struct TeamTask {
  int sys, rank;
};

struct TeamArgs {
  int ntasks;
  const TeamTask *tasks;
  unsigned int *next;      // queue position
  const TeamSys *sys;
  TeamOut *out;
  double tol, inner_tol;
  int inner_maxit, max_iter, max_ref, resume_ok;
  int *err;
};

// barrier of one team (T CTAs; a block barrier when T = 1), bounded like grid_barrier.  The
// error word is read once, by thread 0, and broadcast, so the whole block takes the same way out.
__device__ __forceinline__ bool team_sync(unsigned int *cnt, int team, unsigned int &epoch, int *err) {
  __shared__ int ok_s;
  __syncthreads();
  if (team > 1) {
    epoch += 1;
    if (threadIdx.x == 0) {
      const unsigned int target = epoch * (unsigned int)team;
      red_release_add_u32(cnt, 1u);
      if (ld_acquire_u32(cnt) < target) {
        const unsigned long long t0 = egpu_globaltimer(), lim = egpu_wait_limit(err);
        unsigned int spins = 0;
        while (ld_acquire_u32(cnt) < target) {
          if ((++spins & 63u) == 0) {
            if (*(volatile int *)err) break;
            if (egpu_globaltimer() - t0 > lim) {
              atomicCAS(err, 0, (int)EGPU_ERR_TIMEOUT);
              break;
            }
          }
        }
      }
      __threadfence();
    }
  }
  if (threadIdx.x == 0) ok_s = *(volatile int *)err == 0;
  __syncthreads();
  return ok_s != 0;
}

// NV team-wide sums: the block's sums of v, one partial per member in slots [slot, slot + NV),
// then every member adds the team's partials in member order
template <int NV>
__device__ __forceinline__ bool team_sum(const TeamSys &S, int rank, int slot, double (&v)[NV], double *sm,
                                         unsigned int &epoch, int *err) {
  block_sum<NV>(v, sm);
  if (S.team == 1) return team_sync(S.bar, 1, epoch, err);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) S.part[(slot + k) * S.team + rank] = v[k];
  if (!team_sync(S.bar, S.team, epoch, err)) return false;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int q = 0; q < S.team; ++q) t += __ldcg(S.part + (slot + k) * S.team + q);
    v[k] = t;
  }
  return true;
}

// f(i, VW<W>) over this member's rows [r0, r1): 16-byte groups (r0 is a multiple of 32 and the
// work vectors are 256-byte aligned with a stride of a multiple of 64), then a scalar tail;
// unrolled so each thread keeps several groups' loads in flight
template <typename F>
__device__ __forceinline__ void team_vec(int r0, int r1, F &&f) {
  const int q0 = r0 >> 2, q1 = r1 >> 2;
#pragma unroll 4
  for (int q = q0 + (int)threadIdx.x; q < q1; q += blockDim.x) f(q << 2, VW<4>{});
  for (int i = (q1 << 2) + (int)threadIdx.x; i < r1; i += blockDim.x) f(i, VW<1>{});
}

// one member's whole solve of system S; false on a recorded error
__device__ bool team_solve(const TeamArgs &a, const TeamSys &S, int rank, TeamOut &o, double *sm) {
  const int n = S.n, T = S.team;
  const int per = (S.nslices + T - 1) / T;
  const int sb = min(S.nslices, rank * per), se = min(S.nslices, sb + per);
  const int r0 = sb << 5, r1 = min(n, se << 5);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  float *R = S.w32, *Z = S.zr ? S.w32 : S.w32 + S.ldw, *P = S.w32 + 2 * S.ldw, *Q = S.w32 + 3 * S.ldw,
        *Dd = S.w32 + 4 * S.ldw;
  unsigned int epoch = 0;
  int refinements = 0, inner_total = 0, info = 0, last_info = 0;
  double residual = 0.0, rnorm = 1.0, rnorm_prev = 1.0, carry_rho = 0.0;
  while (true) {
    // cancellation: the host-mapped abort word, read once per refinement (the barrier of the
    // residual's sum below then takes every member out)
    if (threadIdx.x == 0) egpu_poll_abort(a.err);
    // ---- FP64 residual r = bs - A xs on this member's rows (as k_batch_residual)
    double acc[2] = {0.0, 0.0};
    for (int s = sb + warp; s < se; s += nwarp) {
      const int r = (s << 5) + lane;
      const int w = S.sell_w[s];
      const int base = S.sell_ptr[s] + lane;
      double t = 0.0;
      for (int k = 0; k < w; ++k) {
        const int e = base + (k << 5);
        t = __dadd_rn(t, __dmul_rn(S.svals64[e], S.xs[S.scols[e]]));
      }
      if (r < n) {
        const double ri = S.bs[r] - t;
        S.r64[r] = ri;
        acc[0] += ri * ri;
      }
    }
    double rr1[1] = {acc[0]};
    if (!team_sum<1>(S, rank, TS_RES, rr1, sm, epoch, a.err)) return false;
    residual = sqrt(rr1[0]) / S.bnorm_s;
    if (residual < a.tol) {
      info = EGPU_HUTI_CONVERGENCE;
      break;
    }
    if (refinements >= a.max_ref || inner_total >= a.max_iter) {
      info = EGPU_HUTI_MAXITER;
      break;
    }
    rnorm_prev = rnorm;
    rnorm = sqrt(rr1[0]);
    // ---- inner FP32 CG on A d = r / ||r||, d0 = 0 (huti_cg_D.F90:158-240, recursive residual);
    // reliable updating: a segment after a converged one keeps P and continues with
    // rho_{k-1} scaled to the new residual (rho is quadratic in the scale, P linear)
    const bool resume = a.resume_ok && refinements > 0 && last_info == EGPU_HUTI_CONVERGENCE;
    double oldrho = resume ? carry_rho * (rnorm_prev / rnorm) : 1.0;
    acc[0] = acc[1] = 0.0;
    team_vec(r0, r1, [&](int i, auto vw) {
      constexpr int W = decltype(vw)::value;
      float r[W], z[W], d[W];
#pragma unroll
      for (int t = 0; t < W; ++t) r[t] = (float)(S.r64[i + t] / rnorm);
      if (!S.zr) vld<W>(S.dvals32, i, d);
#pragma unroll
      for (int t = 0; t < W; ++t) {
        z[t] = S.zr ? r[t] : diag_prec(r[t], d[t]);
        acc[0] += (double)r[t] * (double)r[t];
        acc[1] += (double)r[t] * (double)z[t];
      }
      vst<W>(R, i, r);
      vfill<W>(Dd, i, 0.f);
      if (!S.zr) vst<W>(Z, i, z);
    });
    if (!team_sum<2>(S, rank, TS_BB, acc, sm, epoch, a.err)) return false;
    const double rhsnorm = sqrt(acc[0]);
    double rho = acc[1], rr_prev = 0.0;
    int k = 1, iters = 0, iinfo = 0;
    while (true) {
      if (k > 1) {
        const double res_in = sqrt(rr_prev) / rhsnorm;
        if (res_in <= a.inner_tol) { iinfo = EGPU_HUTI_CONVERGENCE; iters = k - 1; break; }
        if (k > a.inner_maxit) { iinfo = EGPU_HUTI_MAXITER; iters = k - 1; break; }
      }
      // P = Z (first direction) or Z + beta P
      const float beta = (float)(rho / oldrho);
      const bool first = k == 1 && !resume;
      team_vec(r0, r1, [&](int i, auto vw) {
        constexpr int W = decltype(vw)::value;
        float z[W], p[W];
        vld<W>(Z, i, z);
        if (!first) vld<W>(P, i, p);
#pragma unroll
        for (int t = 0; t < W; ++t) p[t] = first ? z[t] : z[t] + beta * p[t];
        vst<W>(P, i, p);
      });
      if (!team_sync(S.bar, T, epoch, a.err)) return false;
      // Q = A P on this member's slices, (P, Q)
      double pq[1] = {0.0};
      for (int s = sb + warp; s < se; s += nwarp) {
        const int r = (s << 5) + lane;
        const int w = S.sell_w[s];
        const int base = S.sell_ptr[s] + lane;
        const int s2 = s + nwarp;
        if (lane == 0 && s2 < se) {
          const int w2 = S.sell_w[s2], p2 = S.sell_ptr[s2];
          prefetch_l2_bulk(S.svals32 + p2, (unsigned)(128 * w2));
          if (S.scols16) prefetch_l2_bulk(S.scols16 + p2, (unsigned)(64 * w2));
        }
        float t = 0.f;
        if (S.scols16) {
#pragma unroll 16
          for (int kk = 0; kk < w; ++kk) {
            const int e = base + (kk << 5);
            t = fmaf(__ldcs(S.svals32 + e), __ldca(P + r + (int)__ldcs(S.scols16 + e)), t);
          }
        } else {
#pragma unroll 8
          for (int kk = 0; kk < w; ++kk) {
            const int e = base + (kk << 5);
            t = fmaf(__ldcs(S.svals32 + e), __ldca(P + __ldcs(S.scols + e)), t);
          }
        }
        if (r < n) {
          Q[r] = t;
          pq[0] += (double)P[r] * (double)t;
        }
      }
      if (!team_sum<1>(S, rank, TS_PQ, pq, sm, epoch, a.err)) return false;
      if (rho == 0.0) { iinfo = EGPU_HUTI_CG_RHO; iters = k; break; }
      const double alpha_d = rho / pq[0];
      const float alpha = (float)alpha_d;
      // D += alpha P, R -= alpha Q, Z = M^-1 R, (R, Z), (R, R)
      acc[0] = acc[1] = 0.0;
      team_vec(r0, r1, [&](int i, auto vw) {
        constexpr int W = decltype(vw)::value;
        float d[W], p[W], r[W], q[W], g[W], z[W];
        vld<W>(Dd, i, d);
        vld<W>(P, i, p);
        vld<W>(R, i, r);
        vld<W>(Q, i, q);
        if (!S.zr) vld<W>(S.dvals32, i, g);
#pragma unroll
        for (int t = 0; t < W; ++t) {
          d[t] = d[t] + alpha * p[t];
          r[t] = r[t] - alpha * q[t];
          z[t] = S.zr ? r[t] : diag_prec(r[t], g[t]);
          acc[0] += (double)r[t] * (double)z[t];
          acc[1] += (double)r[t] * (double)r[t];
        }
        vst<W>(Dd, i, d);
        vst<W>(R, i, r);
        if (!S.zr) vst<W>(Z, i, z);
      });
      if (!team_sum<2>(S, rank, TS_RHO, acc, sm, epoch, a.err)) return false;
      rr_prev = acc[1];
      oldrho = rho;
      rho = acc[0];
      ++k;
    }
    inner_total += max(1, iters);
    last_info = iinfo;
    carry_rho = oldrho;  // P was built with it
    // xs += ||r|| d on this member's rows; the next residual gathers them
    team_vec(r0, r1, [&](int i, auto vw) {
      constexpr int W = decltype(vw)::value;
#pragma unroll
      for (int t = 0; t < W; ++t) S.xs[i + t] += rnorm * (double)Dd[i + t];
    });
    ++refinements;
    if (!team_sync(S.bar, T, epoch, a.err)) return false;
  }
  o.info = info;
  o.iters = inner_total;
  o.refinements = refinements;
  o.residual = residual;
  return true;
}

__global__ void __launch_bounds__(TEAM_BLOCK, TEAM_PER_SM) k_batch_team(TeamArgs a) {
  __shared__ double sm[32 * 2];
  __shared__ int task;
  __shared__ TeamSys S;  // the system's descriptor, read by every thread (never aliased by the vectors)
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) {
      egpu_poll_abort(a.err);
      task = *(volatile int *)a.err ? a.ntasks : (int)atomicAdd(a.next, 1u);
    }
    __syncthreads();
    const int t = task;
    if (t >= a.ntasks) return;
    const TeamTask tk = a.tasks[t];
    if (threadIdx.x == 0) S = a.sys[tk.sys];
    __syncthreads();
    TeamOut o{};
    if (!team_solve(a, S, tk.rank, o, sm)) return;
    if (tk.rank == 0 && threadIdx.x == 0) a.out[tk.sys] = o;
  }
}

}  // namespace egpu

// =====================================================================================
// host side

using namespace egpu;

struct BatchSys {
  egpu_mat *A = nullptr;
  bool owned = false;
  int phase = 0;          // 0 free, 1 needs residual, 2 in inner solve, 3 finished
  int refinements = 0, inner_iters = 0, info = 0;
  double residual = 0.0, bnorm_s = 1.0, rnorm = 0.0;  // rnorm: ||r|| that started the inner solve
  DevBuf<double> xout;    // back-scaled solution
  double t_admit = 0.0;
  bool reported = false;  // listed as finished by egpu_batch_step
  double rnorm_prev = 1.0;  // ||r|| that started the previous inner segment
  int last_info = 0;        // how the previous inner segment ended
};

struct egpu_batch {
  egpu_ctx *ctx = nullptr;
  std::vector<BatchSys *> sys;       // slot -> system (nullptr = free slot)
  DevBuf<SysDesc> d_desc;
  DevBuf<RefDesc> d_ref;
  DevBuf<SysState> d_state;
  DevBuf<double> d_acc, d_norms;
  DevBuf<int> d_sel, d_pre, d_it;
  std::vector<SysDesc> h_desc;
  std::vector<RefDesc> h_ref;
  int parity = 0;
  bool desc_dirty = true;
  egpu_params prm{};
  int chunk = 64;
  int tri_mult = 2;       // sync-free participants: tri_mult x widest level x running systems
  int bps = 2;            // blocks of the persistent inner kernel per SM (1 or 2)
  int spw = 1;            // SELL slices a warp sums at once in the SpMV phases (1 or 2: 32 or 64 rows)
  int sweeps = 0;         // BiCGStab + ILU0: Jacobi sweeps per triangle in the inner solves (0: exact)
  bool resume_ok = true;  // reliable updating between segments (EGPU_MIXED_RESTART=1: off)
  bool exit_on_done = false;  // latency mode (egpu_batch_set_latency_mode)
  long long launches = 0;
  // the last inner launch: device milliseconds, inner iterations run, nonzeros of its systems
  float last_ms = 0.f;
  int last_iters = 0;
  long long last_nnz = 0;
  // team solver (egpu_batch_solve with CG): descriptors, task queue, results, team barriers,
  // partial sums
  DevBuf<TeamSys> d_team;
  DevBuf<TeamTask> d_tasks;
  DevBuf<TeamOut> d_tout;
  DevBuf<unsigned int> d_tbar;
  DevBuf<double> d_part;
};

static int slot_of(egpu_batch *B) {
  for (size_t i = 0; i < B->sys.size(); ++i)
    if (!B->sys[i]) return (int)i;
  if ((int)B->sys.size() >= BATCH_MAX_SYS) return -1;
  B->sys.push_back(nullptr);
  return (int)B->sys.size() - 1;
}

extern "C" int egpu_batch_create(egpu_ctx *ctx, const egpu_params *prm, egpu_batch **out) {
  if (!ctx || !out || !prm) return EGPU_ERR_ARG;
  if (prm->method != EGPU_CG && prm->method != EGPU_BICGSTAB) return EGPU_ERR_ARG;
  if (prm->method == EGPU_CG && prm->precond == EGPU_PREC_ILU0) return EGPU_ERR_ARG;
  if (prm->precond < EGPU_PREC_NONE || prm->precond > EGPU_PREC_ILU0 || prm->max_iter < 1) return EGPU_ERR_ARG;
  auto *B = new egpu_batch;
  B->ctx = ctx;
  cudaSetDevice(ctx->device);
  if (B->d_desc.alloc(BATCH_MAX_SYS) || B->d_ref.alloc(BATCH_MAX_SYS) || B->d_state.alloc(2 * BATCH_MAX_SYS) ||
      B->d_acc.alloc(BA_NSLOT * BATCH_MAX_SYS) || B->d_norms.alloc(2 * BATCH_MAX_SYS) ||
      B->d_sel.alloc(BATCH_MAX_SYS) || B->d_pre.alloc(BATCH_MAX_SYS + 1) || B->d_it.alloc(4)) {
    delete B;
    return EGPU_ERR_ALLOC;
  }
  cudaMemset(B->d_state.p, 0, 2 * BATCH_MAX_SYS * sizeof(SysState));
  cudaMemset(B->d_acc.p, 0, BA_NSLOT * BATCH_MAX_SYS * sizeof(double));
  B->prm = *prm;
  B->prm.precision = EGPU_MIXED;
  if (const char *e = std::getenv("EGPU_MIXED_RESTART")) B->resume_ok = e[0] != '1';
  B->sweeps = prm->method == EGPU_BICGSTAB ? prm->ilu_sweeps : 0;
  if (const char *e = std::getenv("EGPU_ILU_SWEEPS")) B->sweeps = prm->method == EGPU_BICGSTAB ? std::atoi(e) : 0;
  B->sweeps = std::max(0, std::min(B->sweeps, 16));
  if (B->prm.inner_max_iter < 1) B->prm.inner_max_iter = 2000;
  if (B->prm.max_refinements < 1) B->prm.max_refinements = 100;
  *out = B;
  return EGPU_OK;
}

extern "C" void egpu_batch_free(egpu_batch *B) {
  if (!B) return;
  cudaSetDevice(B->ctx->device);
  cudaStreamSynchronize(B->ctx->stream);
  for (auto *s : B->sys)
    if (s) {
      if (s->owned) egpu_matrix_free(s->A);
      delete s;
    }
  delete B;
}

// prepare one admitted system: scaling, preconditioner, FP32 copies (all on the device)
static int batch_prepare(egpu_batch *B, int slot, const double *b_dev) {
  BatchSys *S = B->sys[slot];
  egpu_mat *A = S->A;
  egpu_ctx *ctx = B->ctx;
  const int n = A->n;
  int rc = reset_sync(ctx);
  if (rc) return rc;
  rc = scale_matrix(A, B->prm.scale_system != 0);
  if (rc) return rc;
  const long long ldw = A->ldw;
  double *W = A->work.p;
  double *bs = W + 10 * ldw, *xs = W + 12 * ldw;
  EGPU_CUDA_TRY(ctx, S->xout.alloc(n));
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(S->xout.p, 0, n * sizeof(double), ctx->stream));
  rc = rhs_scale(A, b_dev ? b_dev : A->rhs.p, S->xout.p, bs, xs, B->prm.scale_system != 0, &S->bnorm_s);
  if (rc) return rc;
  if (B->prm.precond == EGPU_PREC_ILU0) {
    rc = ilu_factor(A, B->prm.ilu_order);
    if (rc) return rc;
  }
  const bool sweeps = B->sweeps > 0 && B->prm.precond == EGPU_PREC_ILU0 && A->ilu_order == 0 && A->ilu_nnz == A->nnz;
  rc = prepare_fp32_public(A, B->prm.precond == EGPU_PREC_ILU0, sweeps);
  if (rc) return rc;
  int unit = 0;
  if (B->prm.method == EGPU_CG && B->prm.precond == EGPU_PREC_DIAGONAL) {
    rc = unit_diagonal_fp32(A, &unit);
    if (rc) return rc;
  }
  S->phase = S->bnorm_s < 0 ? 3 : 1;  // negative: zero right-hand side, x = 0
  if (S->bnorm_s < 0) {
    S->info = EGPU_HUTI_CONVERGENCE;
    S->residual = 0.0;
  }
  const long long ldw32 = A->ldw;
  SysDesc d{};
  d.n = n;
  d.unit_diag = unit;
  d.nslices = A->nslices;
  d.sell_ptr = A->sell_ptr.p;
  d.sell_w = A->sell_w.p;
  d.scols16 = A->sell_c16.p;
  d.scols = A->sell_cols.p;
  d.svals = A->sell_vals32.p;
  d.dvals = A->work32.p + 13 * ldw32;
  d.ilu = A->ilu32.p;
  d.rows = A->rows.p;
  d.cols = A->cols.p;
  d.diag = A->diag.p;
  d.lower_order = A->tri.lower_order.p;
  d.upper_order = A->tri.upper_order.p;
  d.lo_ptr = A->tri.lo_ptr.p;
  d.lo_cols = A->tri.lo_cols.p;
  d.up_ptr = A->tri.up_ptr.p;
  d.up_cols = A->tri.up_cols.p;
  d.lo_vals = A->lo_vals32.p;
  d.up_vals = A->up_vals32.p;
  d.up_dinv = A->up_dinv32.p;
  d.isvals = sweeps ? A->ilu_sell32.p : nullptr;
  d.idinv = sweeps ? A->ilu_dinv32.p : nullptr;
  d.swr = A->sell_swr.p;
  d.w = A->work32.p;
  d.ldw = ldw32;
  d.b = A->work32.p + 10 * ldw32;
  d.x = A->work32.p + 11 * ldw32;
  RefDesc r{};
  r.n = n;
  r.nslices = A->nslices;
  r.sell_ptr = A->sell_ptr.p;
  r.sell_w = A->sell_w.p;
  r.scols = A->sell_cols.p;
  r.svals = A->sell_vals.p;
  r.bs = bs;
  r.xs = xs;
  r.r = W;
  r.r32 = A->work32.p + 10 * ldw32;
  r.d32 = A->work32.p + 11 * ldw32;
  r.D = A->dscale.p;
  r.x_out = S->xout.p;
  if ((int)B->h_desc.size() <= slot) {
    B->h_desc.resize(slot + 1);
    B->h_ref.resize(slot + 1);
  }
  B->h_desc[slot] = d;
  B->h_ref[slot] = r;
  B->desc_dirty = true;
  return EGPU_OK;
}

static int batch_add_common(egpu_batch *B, egpu_mat *A, bool owned, const double *b_dev) {
  if (A->ctx != B->ctx) return EGPU_ERR_ARG;
  const int slot = slot_of(B);
  if (slot < 0) return EGPU_ERR_BUDGET;
  auto *S = new BatchSys;
  S->A = A;
  S->owned = owned;
  B->sys[slot] = S;
  int rc = batch_prepare(B, slot, b_dev);
  if (rc) {
    if (owned) egpu_matrix_free(A);
    delete S;
    B->sys[slot] = nullptr;
    return rc;
  }
  return slot;
}

extern "C" int egpu_batch_add(egpu_batch *B, int n, const int *rows, const int *cols, const int *diag,
                              const double *values, const double *rhs) {
  if (!B || !values || !rhs) return EGPU_ERR_ARG;
  egpu_mat *A = nullptr;
  int rc = egpu_matrix_bind(B->ctx, n, rows, cols, diag, values, &A);
  if (rc) return rc;
  EGPU_CUDA_TRY(B->ctx, cudaMemcpyAsync(A->rhs.p, rhs, n * sizeof(double), cudaMemcpyHostToDevice, B->ctx->stream));
  return batch_add_common(B, A, true, nullptr);
}

extern "C" int egpu_batch_add_matrix(egpu_batch *B, egpu_mat *A, const double *b_dev) {
  if (!B || !A || !A->has_values) return EGPU_ERR_ARG;
  return batch_add_common(B, A, false, b_dev);
}

// slice prefix for a selection of slots, uploaded for the refinement kernels
static int upload_selection(egpu_batch *B, const std::vector<int> &sel, int *total) {
  std::vector<int> pre(sel.size() + 1, 0);
  for (size_t i = 0; i < sel.size(); ++i) pre[i + 1] = pre[i] + B->h_ref[sel[i]].nslices;
  *total = pre.back();
  EGPU_CUDA_TRY(B->ctx, cudaMemcpyAsync(B->d_sel.p, sel.data(), sel.size() * sizeof(int), cudaMemcpyHostToDevice,
                                        B->ctx->stream));
  EGPU_CUDA_TRY(B->ctx, cudaMemcpyAsync(B->d_pre.p, pre.data(), pre.size() * sizeof(int), cudaMemcpyHostToDevice,
                                        B->ctx->stream));
  // the host vectors must outlive the async copies
  EGPU_CUDA_TRY(B->ctx, cudaStreamSynchronize(B->ctx->stream));
  return EGPU_OK;
}

// the per-system descriptor tables, uploaded when systems were admitted or removed
static int upload_desc(egpu_batch *B) {
  const int ns = (int)B->sys.size();
  if (!B->desc_dirty || ns == 0) return EGPU_OK;
  std::vector<SysDesc> d(ns);
  std::vector<RefDesc> r(ns);
  for (int i = 0; i < ns; ++i)
    if (B->sys[i] && i < (int)B->h_desc.size()) {
      d[i] = B->h_desc[i];
      r[i] = B->h_ref[i];
    }
  EGPU_CUDA_TRY(B->ctx, cudaMemcpy(B->d_desc.p, d.data(), ns * sizeof(SysDesc), cudaMemcpyHostToDevice));
  EGPU_CUDA_TRY(B->ctx, cudaMemcpy(B->d_ref.p, r.data(), ns * sizeof(RefDesc), cudaMemcpyHostToDevice));
  B->desc_dirty = false;
  return EGPU_OK;
}

// One server step: FP64 residuals + decisions for systems that need them, then one chunk
// of the batched inner solver.  finished[] receives slots completed in this step.
extern "C" int egpu_batch_step(egpu_batch *B, int *finished, int *nfinished) {
  if (!B) return EGPU_ERR_ARG;
  egpu_ctx *ctx = B->ctx;
  cudaSetDevice(ctx->device);
  const int ns = (int)B->sys.size();
  int nf = 0;
  int rc0 = upload_desc(B);
  if (rc0) return rc0;
  // systems that finished while nobody collected the list (egpu_batch_tune) are listed now
  if (finished)
    for (int i = 0; i < ns; ++i)
      if (B->sys[i] && B->sys[i]->phase == 3 && !B->sys[i]->reported) {
        finished[nf++] = i;
        B->sys[i]->reported = true;
      }
  // ---- refinement: residual for systems in phase 1
  std::vector<int> sel;
  for (int i = 0; i < ns; ++i)
    if (B->sys[i] && B->sys[i]->phase == 1) sel.push_back(i);
  std::vector<SysState> st(2 * BATCH_MAX_SYS);
  if (!sel.empty()) {
    int total = 0;
    int rc = upload_selection(B, sel, &total);
    if (rc) return rc;
    EGPU_CUDA_TRY(ctx, cudaMemsetAsync(B->d_norms.p, 0, ns * sizeof(double), ctx->stream));
    const int grid = std::max(1, std::min((total + 7) / 8, ctx->num_sms * 8));
    k_batch_residual<<<grid, 256, 0, ctx->stream>>>((int)sel.size(), B->d_sel.p, B->d_ref.p, B->d_pre.p, B->d_norms.p);
    std::vector<double> nr(ns);
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(nr.data(), B->d_norms.p, ns * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->launches++;
    B->launches++;
    std::vector<int> start, done;
    for (int i : sel) {
      BatchSys *S = B->sys[i];
      S->residual = std::sqrt(nr[i]) / S->bnorm_s;
      if (S->residual < B->prm.tol) {
        S->info = EGPU_HUTI_CONVERGENCE;
        done.push_back(i);
      } else if (S->refinements >= B->prm.max_refinements || S->inner_iters >= B->prm.max_iter) {
        S->info = EGPU_HUTI_MAXITER;
        done.push_back(i);
      } else {
        S->rnorm_prev = S->rnorm;
        S->rnorm = std::sqrt(nr[i]);
        start.push_back(i);
      }
    }
    if (!start.empty()) {
      rc = upload_selection(B, start, &total);
      if (rc) return rc;
      const int grid2 = std::max(1, std::min((total + 7) / 8, ctx->num_sms * 8));
      k_batch_cast<<<grid2, 256, 0, ctx->stream>>>((int)start.size(), B->d_sel.p, B->d_ref.p, B->d_pre.p, B->d_norms.p);
      ctx->launches++;
      B->launches++;
      // state: INIT in the parity the next chunk reads
      EGPU_CUDA_TRY(ctx, cudaMemcpy(st.data(), B->d_state.p, 2 * BATCH_MAX_SYS * sizeof(SysState), cudaMemcpyDeviceToHost));
      for (int i : start) {
        SysState &s = st[B->parity * BATCH_MAX_SYS + i];
        BatchSys *S = B->sys[i];
        // reliable updating: continue the last segment if it converged normally
        const bool resume = B->resume_ok && S->refinements > 0 && s.status == ST_IDLE && S->last_info == EGPU_HUTI_CONVERGENCE;
        if (resume) {
          const double c = S->rnorm_prev / S->rnorm;  // old scale / new scale
          s.carry_rho = B->prm.method == EGPU_CG ? s.rho * c : s.rho;
          s.resume = 1;
        } else {
          std::memset(&s, 0, sizeof(s));
        }
        s.status = ST_INIT;
        S->phase = 2;
        S->refinements++;
      }
      EGPU_CUDA_TRY(ctx, cudaMemcpy(B->d_state.p, st.data(), 2 * BATCH_MAX_SYS * sizeof(SysState), cudaMemcpyHostToDevice));
    }
    if (!done.empty()) {
      rc = upload_selection(B, done, &total);
      if (rc) return rc;
      const int grid3 = std::max(1, std::min((total + 7) / 8, ctx->num_sms * 8));
      k_batch_backscale<<<grid3, 256, 0, ctx->stream>>>((int)done.size(), B->d_sel.p, B->d_ref.p, B->d_pre.p);
      ctx->launches++;
      B->launches++;
      for (int i : done) {
        B->sys[i]->phase = 3;
        if (finished) {
          finished[nf] = i;
          B->sys[i]->reported = true;
        }
        nf++;
      }
    }
  }
  // ---- one chunk of inner iterations for systems in phase 2
  bool any_inner = false;
  for (int i = 0; i < ns; ++i)
    if (B->sys[i] && B->sys[i]->phase == 2) any_inner = true;
  if (any_inner) {
    EGPU_CUDA_TRY(ctx, cudaMemsetAsync(ctx->sync.p, 0, 2 * sizeof(unsigned int), ctx->stream));
    BatchArgs a{};
    a.nsys = ns;
    a.sys = B->d_desc.p;
    a.state = B->d_state.p;
    a.acc = B->d_acc.p;
    a.method = B->prm.method;
    a.precond = B->prm.precond;
    a.kmax = B->chunk;
    a.spw = B->spw;
    a.sweeps = B->sweeps;
    a.exit_on_done = B->exit_on_done ? 1 : 0;
    a.tol = inner_tol_of(&B->prm);
    a.maxit = B->prm.inner_max_iter;
    int maxw = 1;
    for (int i = 0; i < ns; ++i)
      if (B->sys[i] && B->sys[i]->phase == 2) maxw = std::max(maxw, B->sys[i]->A->tri.max_width);
    const void *kern = a.spw == 2 ? (const void *)k_batch_inner<2> : (const void *)k_batch_inner<1>;
    int bps = 0;
    EGPU_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, EGPU_BLOCK, 0));
    bps = std::max(1, std::min(bps, B->bps));
    const int grid = ctx->num_sms * bps;
    int nrun = 0;
    long long nnz_run = 0;
    for (int i = 0; i < ns; ++i)
      if (B->sys[i] && B->sys[i]->phase == 2) {
        nrun++;
        nnz_run += B->sys[i]->A->nnz;
      }
    a.tri_warps_per_block = std::max((nrun + grid - 1) / grid,
                                     std::min(EGPU_BLOCK / 32, (B->tri_mult * maxw * nrun + grid - 1) / grid));
    a.tri_warps_per_block = std::max(1, std::min(EGPU_BLOCK / 32, a.tri_warps_per_block));
    // rows per warp in the sync-free solves: up to 4 (8 lanes, 16 entries in registers; fewer
    // when fewer systems run) or 2 (16 lanes, 32 entries) when the longest strictly-lower /
    // upper row part fits, else 1.  EGPU_BATCH_TRI_GROUP overrides (1, 2, 4 or 8; 8 rows of 4
    // lanes measured slower than 4 on eight 96^3 systems)
    {
      int maxpart = 0;
      for (int i = 0; i < ns; ++i)
        if (B->sys[i] && B->sys[i]->phase == 2)
          maxpart = std::max(maxpart, std::max(B->sys[i]->A->tri.max_lower, B->sys[i]->A->tri.max_upper));
      a.tri_group = maxpart <= 16 ? 4 : maxpart <= 32 ? 2 : 1;
      if (const char *e = std::getenv("EGPU_BATCH_TRI_GROUP")) {
        const int g = std::atoi(e);
        if (g == 1 || g == 2 || g == 4 || g == 8) a.tri_group = g;
      }
    }
    a.bar = ctx->sync.p;
    a.err = (int *)(ctx->sync.p + 1);
    a.it_done = B->d_it.p;
    int parity0 = B->parity;
    void *args[] = {&a, &parity0};
    EGPU_CUDA_TRY(ctx, cudaEventRecord(ctx->ek0, ctx->stream));
    EGPU_CUDA_TRY(ctx, cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(EGPU_BLOCK), args, 0, ctx->stream));
    EGPU_CUDA_TRY(ctx, cudaEventRecord(ctx->ek1, ctx->stream));
    ctx->launches++;
    B->launches++;
    int hit[2] = {0, 0};
    unsigned int herr[2] = {0, 0};
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(hit, B->d_it.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(herr, ctx->sync.p, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (herr[1]) {
      egpu_set_error(ctx, egpu_device_status_text((int)herr[1]) + " in the batched solver");
      return (int)herr[1];
    }
    B->parity = (B->parity + hit[0]) & 1;
    cudaEventElapsedTime(&B->last_ms, ctx->ek0, ctx->ek1);
    B->last_iters = hit[0];
    B->last_nnz = nnz_run;
    EGPU_CUDA_TRY(ctx, cudaMemcpy(st.data(), B->d_state.p, 2 * BATCH_MAX_SYS * sizeof(SysState), cudaMemcpyDeviceToHost));
    std::vector<int> upd;
    for (int i = 0; i < ns; ++i) {
      BatchSys *S = B->sys[i];
      if (!S || S->phase != 2) continue;
      const SysState &s = st[B->parity * BATCH_MAX_SYS + i];
      if (s.status == ST_DONE) {
        S->inner_iters += std::max(1, s.iters);
        S->last_info = s.info;
        upd.push_back(i);
      }
    }
    if (!upd.empty()) {
      // x += ||r|| d, then the system needs a new residual
      std::vector<double> rn(ns, 0.0);
      for (int i : upd) rn[i] = B->sys[i]->rnorm;
      EGPU_CUDA_TRY(ctx, cudaMemcpy(B->d_norms.p + BATCH_MAX_SYS, rn.data(), ns * sizeof(double), cudaMemcpyHostToDevice));
      int total = 0;
      int rc = upload_selection(B, upd, &total);
      if (rc) return rc;
      const int grid4 = std::max(1, std::min((total + 7) / 8, ctx->num_sms * 8));
      // norms of the residuals that started these inner solves are still in d_norms
      k_batch_update<<<grid4, 256, 0, ctx->stream>>>((int)upd.size(), B->d_sel.p, B->d_ref.p, B->d_pre.p,
                                                    B->d_norms.p + BATCH_MAX_SYS);
      ctx->launches++;
      B->launches++;
      for (int i : upd) {
        B->sys[i]->phase = 1;
        st[B->parity * BATCH_MAX_SYS + i].status = ST_IDLE;
      }
      EGPU_CUDA_TRY(ctx, cudaMemcpy(B->d_state.p, st.data(), 2 * BATCH_MAX_SYS * sizeof(SysState), cudaMemcpyHostToDevice));
    }
  }
  if (nfinished) *nfinished = nf;
  return EGPU_OK;
}

extern "C" int egpu_batch_set_config(egpu_batch *B, const egpu_batch_config *cfg) {
  if (!B || !cfg || cfg->chunk_iters < 1 || cfg->blocks_per_sm < 1 || cfg->blocks_per_sm > 2 || cfg->tri_mult < 1 ||
      cfg->slices_per_warp < 0 || cfg->slices_per_warp > 2)
    return EGPU_ERR_ARG;
  B->chunk = cfg->chunk_iters;
  B->bps = cfg->blocks_per_sm;
  B->tri_mult = cfg->tri_mult;
  if (cfg->slices_per_warp) B->spw = cfg->slices_per_warp;
  return EGPU_OK;
}

// Latency mode: a launch returns after the iteration in which any system finished its inner
// segment, so its FP64 refinement (or retirement) follows at once instead of at the end of
// the chunk: lower latency for short requests, more launches.
extern "C" int egpu_batch_set_latency_mode(egpu_batch *B, int on) {
  if (!B) return EGPU_ERR_ARG;
  B->exit_on_done = on != 0;
  return EGPU_OK;
}

extern "C" int egpu_batch_set_chunk(egpu_batch *B, int chunk_iters) {
  if (!B || chunk_iters < 1) return EGPU_ERR_ARG;
  B->chunk = chunk_iters;
  return EGPU_OK;
}

extern "C" int egpu_batch_last_launch(egpu_batch *B, double *ms) {
  if (!B || !ms) return EGPU_ERR_ARG;
  *ms = B->last_ms;
  return EGPU_OK;
}

extern "C" int egpu_batch_result(egpu_batch *B, int sys, egpu_result *res) {
  if (!B || sys < 0 || sys >= (int)B->sys.size() || !B->sys[sys] || !res) return EGPU_ERR_ARG;
  const BatchSys *S = B->sys[sys];
  egpu_result r{};
  r.info = S->phase == 3 ? S->info : 0;
  r.iters = S->inner_iters;
  r.refinements = S->refinements;
  r.residual = S->residual;
  *res = r;
  return S->phase == 3 ? EGPU_OK : EGPU_ERR_STATE;
}

extern "C" int egpu_batch_solution(egpu_batch *B, int sys, double *x) {
  if (!B || sys < 0 || sys >= (int)B->sys.size() || !B->sys[sys] || !x) return EGPU_ERR_ARG;
  BatchSys *S = B->sys[sys];
  if (S->phase != 3) return EGPU_ERR_STATE;
  EGPU_CUDA_TRY(B->ctx, cudaMemcpyAsync(x, S->xout.p, S->A->n * sizeof(double), cudaMemcpyDeviceToHost,
                                        B->ctx->stream));
  EGPU_CUDA_TRY(B->ctx, cudaStreamSynchronize(B->ctx->stream));
  return EGPU_OK;
}

extern "C" int egpu_batch_remove(egpu_batch *B, int sys) {
  if (!B || sys < 0 || sys >= (int)B->sys.size() || !B->sys[sys]) return EGPU_ERR_ARG;
  BatchSys *S = B->sys[sys];
  if (S->phase == 2) return EGPU_ERR_STATE;  // inner solve in flight: finish first
  cudaStreamSynchronize(B->ctx->stream);
  if (S->owned) egpu_matrix_free(S->A);
  delete S;
  B->sys[sys] = nullptr;
  B->desc_dirty = true;
  return EGPU_OK;
}

extern "C" int egpu_batch_pending(egpu_batch *B) {
  if (!B) return EGPU_ERR_ARG;
  int k = 0;
  for (auto *s : B->sys)
    if (s && (s->phase == 1 || s->phase == 2)) ++k;
  return k;
}

// egpu_batch_solve on the team solver (k_batch_team): CG with M = I or Jacobi, when every
// resident system still waits for its first residual (none is inside an inner solve).  Returns
// 1 when it solved them, 0 when the batch does not qualify (EGPU_BATCH_TEAMS=0 turns it off),
// < 0 on an error.
static int batch_solve_teams(egpu_batch *B) {
  if (B->prm.method != EGPU_CG || B->prm.precond == EGPU_PREC_ILU0) return 0;
  if (const char *e = std::getenv("EGPU_BATCH_TEAMS"))
    if (e[0] == '0') return 0;
  egpu_ctx *ctx = B->ctx;
  const int ns = (int)B->sys.size();
  std::vector<int> sel;
  for (int i = 0; i < ns; ++i)
    if (B->sys[i]) {
      if (B->sys[i]->phase == 2) return 0;
      if (B->sys[i]->phase == 1) sel.push_back(i);
    }
  if (sel.empty()) return 0;
  int rc = upload_desc(B);
  if (rc) return rc;
  int bps = 0;
  EGPU_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_team, TEAM_BLOCK, 0));
  if (bps < 1) return 0;
  bps = std::min(bps, TEAM_PER_SM);
  const int G = ctx->num_sms * bps;
  // team sizes from a work estimate (nonzeros x n^(1/3): CG's iteration count grows with the
  // mesh's linear size), at least 64 slices a member; the largest teams take the queue first
  const size_t m = sel.size();
  std::vector<double> wk(m);
  double tot = 0.0;
  for (size_t j = 0; j < m; ++j) {
    const egpu_mat *A = B->sys[sel[j]]->A;
    wk[j] = (double)A->nnz * std::cbrt((double)A->n);
    tot += wk[j];
  }
  const double fair = tot / G;
  std::vector<int> team(m), ord(m);
  for (size_t j = 0; j < m; ++j) {
    const int cap = std::max(1, std::min(TEAM_MAX, B->sys[sel[j]]->A->nslices / 64));
    team[j] = std::max(1, std::min(cap, (int)std::ceil(wk[j] / fair)));
    ord[j] = (int)j;
  }
  std::sort(ord.begin(), ord.end(), [&](int x, int y) { return team[x] != team[y] ? team[x] > team[y] : wk[x] > wk[y]; });
  std::vector<TeamSys> ts(ns);
  std::vector<TeamTask> tasks;
  EGPU_CUDA_TRY(ctx, B->d_team.alloc(BATCH_MAX_SYS));
  EGPU_CUDA_TRY(ctx, B->d_tout.alloc(BATCH_MAX_SYS));
  EGPU_CUDA_TRY(ctx, B->d_tbar.alloc(BATCH_MAX_SYS));
  EGPU_CUDA_TRY(ctx, B->d_part.alloc((size_t)BATCH_MAX_SYS * TS_NSLOT * TEAM_MAX));
  for (size_t j = 0; j < m; ++j) {
    const int i = sel[j];
    const SysDesc &d = B->h_desc[i];
    const RefDesc &r = B->h_ref[i];
    TeamSys t{};
    t.n = d.n;
    t.nslices = d.nslices;
    t.team = team[j];
    t.zr = (B->prm.precond == EGPU_PREC_NONE || d.unit_diag) ? 1 : 0;
    t.sell_ptr = d.sell_ptr;
    t.sell_w = d.sell_w;
    t.scols16 = d.scols16;
    t.scols = r.scols;
    t.svals32 = d.svals;
    t.dvals32 = d.dvals;
    t.w32 = d.w;
    t.ldw = d.ldw;
    t.svals64 = r.svals;
    t.bs = r.bs;
    t.xs = r.xs;
    t.r64 = r.r;
    t.bnorm_s = B->sys[i]->bnorm_s;
    t.bar = B->d_tbar.p + i;
    t.part = B->d_part.p + (size_t)i * TS_NSLOT * TEAM_MAX;
    ts[i] = t;
  }
  for (int j : ord)
    for (int q = 0; q < team[j]; ++q) tasks.push_back(TeamTask{sel[j], q});
  EGPU_CUDA_TRY(ctx, B->d_tasks.alloc(std::max<size_t>(tasks.size(), 1)));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_team.p, ts.data(), ns * sizeof(TeamSys), cudaMemcpyHostToDevice, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_tasks.p, tasks.data(), tasks.size() * sizeof(TeamTask),
                                     cudaMemcpyHostToDevice, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(B->d_tbar.p, 0, BATCH_MAX_SYS * sizeof(unsigned int), ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(B->d_tout.p, 0, BATCH_MAX_SYS * sizeof(TeamOut), ctx->stream));
  // queue position (sync word 0) and error word
  EGPU_CUDA_TRY(ctx, cudaMemsetAsync(ctx->sync.p, 0, 2 * sizeof(unsigned int), ctx->stream));
  TeamArgs a{};
  a.ntasks = (int)tasks.size();
  a.tasks = B->d_tasks.p;
  a.next = ctx->sync.p;
  a.sys = B->d_team.p;
  a.out = B->d_tout.p;
  a.tol = B->prm.tol;
  a.inner_tol = inner_tol_of(&B->prm);
  a.inner_maxit = B->prm.inner_max_iter;
  a.max_iter = B->prm.max_iter;
  a.max_ref = B->prm.max_refinements;
  a.resume_ok = B->resume_ok ? 1 : 0;
  a.err = (int *)(ctx->sync.p + 1);
  void *args[] = {&a};
  EGPU_CUDA_TRY(ctx, cudaEventRecord(ctx->ek0, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaLaunchCooperativeKernel((const void *)k_batch_team, dim3(G), dim3(TEAM_BLOCK), args, 0,
                                                 ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaEventRecord(ctx->ek1, ctx->stream));
  ctx->launches++;
  B->launches++;
  std::vector<TeamOut> out(ns);
  unsigned int herr[2] = {0, 0};
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(out.data(), B->d_tout.p, ns * sizeof(TeamOut), cudaMemcpyDeviceToHost, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaMemcpyAsync(herr, ctx->sync.p, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
  EGPU_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr[1]) {
    egpu_set_error(ctx, egpu_device_status_text((int)herr[1]) + " in the batched team solver");
    return (int)herr[1];
  }
  cudaEventElapsedTime(&B->last_ms, ctx->ek0, ctx->ek1);
  B->last_nnz = 0;
  B->last_iters = 0;
  for (int i : sel) {
    BatchSys *S = B->sys[i];
    S->info = out[i].info;
    S->inner_iters = out[i].iters;
    S->refinements = out[i].refinements;
    S->residual = out[i].residual;
    S->phase = 3;
    B->last_nnz += S->A->nnz;
    B->last_iters = std::max(B->last_iters, out[i].iters);
  }
  int total = 0;
  rc = upload_selection(B, sel, &total);
  if (rc) return rc;
  const int grid3 = std::max(1, std::min((total + 7) / 8, ctx->num_sms * 8));
  k_batch_backscale<<<grid3, 256, 0, ctx->stream>>>((int)sel.size(), B->d_sel.p, B->d_ref.p, B->d_pre.p);
  ctx->launches++;
  B->launches++;
  EGPU_CUDA_TRY(ctx, cudaGetLastError());
  return 1;
}

// Runs every resident system to completion; per_system (optional) receives one result per
// slot (slots that are free get info 0).
extern "C" int egpu_batch_solve(egpu_batch *B, egpu_result *per_system) {
  if (!B) return EGPU_ERR_ARG;
  cudaSetDevice(B->ctx->device);
  EGPU_CUDA_TRY(B->ctx, cudaEventRecord(B->ctx->ev0, B->ctx->stream));
  {
    const int rt = batch_solve_teams(B);
    if (rt < 0) return rt;
  }
  int guard = 0;
  while (egpu_batch_pending(B) > 0) {
    int rc = egpu_batch_step(B, nullptr, nullptr);
    if (rc) return rc;
    if (++guard > 1000000) return EGPU_ERR_STATE;
  }
  EGPU_CUDA_TRY(B->ctx, cudaEventRecord(B->ctx->ev2, B->ctx->stream));
  EGPU_CUDA_TRY(B->ctx, cudaEventSynchronize(B->ctx->ev2));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, B->ctx->ev0, B->ctx->ev2);
  if (per_system)
    for (size_t i = 0; i < B->sys.size(); ++i) {
      egpu_result r{};
      if (B->sys[i]) egpu_batch_result(B, (int)i, &r);
      r.seconds = ms * 1e-3;
      per_system[i] = r;
    }
  return EGPU_OK;
}

// Autotuner.  Runs real steps of the resident systems (their progress is kept) with each
// candidate configuration in turn: chunk length (inner iterations per launch), blocks of
// the persistent kernel per SM, and, with ILU0, the sync-free participant multiplier; then
// rows per warp in the SpMV phases (one or two SELL slices of 32 rows) by alternating steps.  The
// rate of a step is inner iterations x nonzeros of the systems in the launch per device
// second of the launch; the fastest configuration is kept.  Candidates are tried once each,
// in a fixed order, while systems remain in inner solves; systems that finish meanwhile are
// listed by the next egpu_batch_step.
extern "C" int egpu_batch_tune(egpu_batch *B, egpu_batch_config *cfg) {
  if (!B) return EGPU_ERR_ARG;
  struct Cand {
    int chunk, bps, tri_mult, spw;
  };
  std::vector<Cand> cands;
  const bool ilu = B->prm.precond == EGPU_PREC_ILU0;
  for (int bps : {2, 1})
    for (int chunk : {16, 32, 64})
      for (int tm : {1, 2, 4}) {
        if (!ilu && tm != 2) continue;
        cands.push_back({chunk, bps, tm, B->spw});
      }
  Cand best{B->chunk, B->bps, B->tri_mult, B->spw};
  double best_rate = 0.0;
  int tried = 0;
  // a first step brings every system into its inner solve
  int rc = egpu_batch_step(B, nullptr, nullptr);
  if (rc) return rc;
  for (const Cand &c : cands) {
    if (egpu_batch_pending(B) == 0) break;
    B->chunk = c.chunk;
    B->bps = c.bps;
    B->tri_mult = c.tri_mult;
    B->spw = c.spw;
    B->last_iters = 0;
    B->last_ms = 0.f;
    rc = egpu_batch_step(B, nullptr, nullptr);
    if (rc) return rc;
    if (B->last_iters <= 0 || B->last_ms <= 0.f) continue;
    const double rate = (double)B->last_iters * (double)B->last_nnz / (B->last_ms * 1e-3);
    ++tried;
    if (rate > best_rate) {
      best_rate = rate;
      best = c;
    }
  }
  B->chunk = best.chunk;
  B->bps = best.bps;
  B->tri_mult = best.tri_mult;
  B->spw = best.spw;
  // Rows per warp in the SpMV phases, with the rest fixed: steps alternate one and two slices
  // per warp (A B A B ...), so the batch shrinking as systems converge biases neither, and the
  // higher mean rate is kept.
  {
    double sum[2] = {0.0, 0.0};
    int cnt[2] = {0, 0};
    for (int t = 0; t < 6 && egpu_batch_pending(B) > 0; ++t) {
      const int k = t & 1;
      B->spw = k + 1;
      B->last_iters = 0;
      B->last_ms = 0.f;
      rc = egpu_batch_step(B, nullptr, nullptr);
      if (rc) return rc;
      if (B->last_iters <= 0 || B->last_ms <= 0.f) continue;
      sum[k] += (double)B->last_iters * (double)B->last_nnz / (B->last_ms * 1e-3);
      cnt[k]++;
      ++tried;
    }
    if (cnt[0] && cnt[1]) best.spw = sum[1] / cnt[1] > sum[0] / cnt[0] ? 2 : 1;
    B->spw = best.spw;
  }
  if (cfg) {
    cfg->chunk_iters = best.chunk;
    cfg->blocks_per_sm = best.bps;
    cfg->tri_mult = best.tri_mult;
    cfg->slices_per_warp = best.spw;
    cfg->candidates = tried;
    cfg->rate = best_rate;
  }
  return EGPU_OK;
}
