// egpu_tri_plan.h -- host-only planning of the level-synchronous single-block ILU0 solves.
//
// Given the two slot orders of the sync-free schedule (rows sorted by dependency level)
// and the strictly lower / upper entries packed per slot, build for each triangle:
//   lev[L]  = {first slot, rows w, entries per row m, ELL offset}   (offset a multiple of 8)
//   ridx    = ring slot of every ELL entry's column (padding: the zero slot rs)
//   src     = packed entry each ELL entry is filled from (-1 for padding)
//   map     = lower: upper-order slot of the row; upper: the row
// plus the ring size rs and, per value size, the deepest prefetch distance pd whose
// staging windows (sb entries, sr rows) fit the shared-memory budget.
//
// No CUDA dependency: the plan is also checked by CPU-only tools.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <vector>

#ifdef __CUDACC__
#define EGPU_HD __host__ __device__
#else
#define EGPU_HD
#endif

namespace egpu {

// Shared-memory footprint of the level-synchronous solve: the level table (nl levels of
// 16 bytes), staged ELL values and ring indices (sb entries), the ring (rs slots + a zero
// slot), staged per-row data (sr rows: right-hand side, inverted diagonal, auxiliary
// value, map).
EGPU_HD constexpr size_t cta_align16(size_t b) { return (b + 15) & ~(size_t)15; }
EGPU_HD constexpr size_t cta_smem_bytes(int sb, int rs, int sr, int vsize, int nl) {
  return (size_t)nl * 16 + cta_align16((size_t)sb * vsize) + cta_align16((size_t)sb * 2) +
         cta_align16((size_t)(rs + 1) * vsize) + 3 * cta_align16((size_t)sr * vsize) + cta_align16((size_t)sr * 4);
}

namespace plan {

constexpr int PD_MAX = 8;  // prefetch distance limit (cp.async.wait_group immediates 0..7)

struct Lev {
  int x, y, z, w;
};

struct TriPlan {
  int nlev = 0;
  std::vector<int> start;       // nlev + 1 slot offsets
  std::vector<Lev> lev;
  std::vector<long long> off;   // nlev + 1 ELL offsets
  long long nent = 0;           // ELL entries (>= 8)
  std::vector<uint16_t> ridx;
  std::vector<int> src, map;    // map has n + 8 entries (padding zero)
};

struct Plan {
  bool ok = false;              // representable (ring fits 16-bit slots)
  int rs = 0;
  TriPlan lo, up;
  std::vector<int> pos_lo, pos_up;
  bool fits[2] = {false, false};  // [0] FP64, [1] FP32
  int pd[2] = {0, 0}, sb[2] = {0, 0}, sr[2] = {0, 0};
  size_t smem[2] = {0, 0};
};

// level boundaries of a slot order (rows sorted by level)
inline void slot_levels(const std::vector<int> &order, const std::vector<int> &level, TriPlan &T) {
  const int n = (int)order.size();
  T.start.assign(1, 0);
  for (int s = 1; s <= n; ++s)
    if (s == n || level[order[s]] != level[order[s - 1]]) T.start.push_back(s);
  if (n == 0) T.start.push_back(0);
  T.nlev = (int)T.start.size() - 1;
}

// ring slots one triangle needs: slot d must survive until the level of every row that
// reads it has finished (rs >= end(level(reader)) - d), and one level's rows are distinct
inline long long ring_need(const TriPlan &T, const std::vector<int> &ptr, const std::vector<int> &pcols,
                           const std::vector<int> &pos) {
  long long rs = 1;
  for (int L = 0; L < T.nlev; ++L) {
    const int beg = T.start[L], end = T.start[L + 1];
    rs = std::max<long long>(rs, end - beg);
    for (int s = beg; s < end; ++s)
      for (int e = ptr[s]; e < ptr[s + 1]; ++e) rs = std::max<long long>(rs, (long long)end - pos[pcols[e]]);
  }
  return rs;
}

inline void ell_layout(TriPlan &T, const std::vector<int> &ptr) {
  T.off.assign(T.nlev + 1, 0);
  T.lev.resize(T.nlev);
  for (int L = 0; L < T.nlev; ++L) {
    const int beg = T.start[L], w = T.start[L + 1] - beg;
    int m = 0;
    for (int s = beg; s < beg + w; ++s) m = std::max(m, ptr[s + 1] - ptr[s]);
    const long long sz = ((long long)w * m + 7) / 8 * 8;
    T.off[L + 1] = T.off[L] + sz;
    T.lev[L] = Lev{beg, w, m, (int)std::min<long long>(T.off[L], 0x7fffffff)};
  }
  T.nent = std::max<long long>(8, T.off[T.nlev]);
}

// staging windows for prefetch distance pd: entries / rows of pd + 1 consecutive levels
inline void windows(const TriPlan &T, int pd, long long &sb, long long &sr) {
  for (int L = 0; L < T.nlev; ++L) {
    const int e = std::min(T.nlev, L + pd + 1);
    sb = std::max(sb, T.off[e] - T.off[L]);
    sr = std::max<long long>(sr, T.start[e] - T.start[L]);
  }
}

// ELL arrays of one triangle; false if a dependency is not an earlier slot still in the ring
inline bool fill_arrays(TriPlan &T, int n, int rs, const std::vector<int> &ptr, const std::vector<int> &pcols,
                        const std::vector<int> &pos, const std::vector<int> &order, const std::vector<int> *pos_up) {
  T.ridx.assign(T.nent, (uint16_t)rs);
  T.src.assign(T.nent, -1);
  T.map.assign((size_t)n + 8, 0);
  for (int L = 0; L < T.nlev; ++L) {
    const Lev lv = T.lev[L];
    for (int t = 0; t < lv.y; ++t) {
      const int s = lv.x + t;
      for (int k = 0, e = ptr[s]; e < ptr[s + 1]; ++k, ++e) {
        const long long q = (long long)lv.w + (long long)k * lv.y + t;
        const int d = pos[pcols[e]];
        if (d >= lv.x || (long long)T.start[L + 1] - d > rs) return false;
        T.ridx[q] = (uint16_t)(d % rs);
        T.src[q] = e;
      }
      T.map[s] = pos_up ? (*pos_up)[order[s]] : order[s];
    }
  }
  return true;
}

// lo / up: slot orders; lp, lc / upp, uc: packed strictly-lower / strictly-upper entries
// (column ids) per slot.  with_arrays: also build ridx / src / map.
inline void make_plan(int n, const std::vector<int> &rows, const std::vector<int> &cols, const std::vector<int> &diag,
                      const std::vector<int> &lo, const std::vector<int> &up, const std::vector<int> &lp,
                      const std::vector<int> &lc, const std::vector<int> &upp, const std::vector<int> &uc,
                      size_t smem_max, Plan &P) {
  P = Plan();
  if (n <= 0) return;
  std::vector<int> llev(n, 0), ulev(n, 0);
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int j = rows[i]; j < diag[i]; ++j) l = std::max(l, llev[cols[j]] + 1);
    llev[i] = l;
  }
  for (int i = n - 1; i >= 0; --i) {
    int l = 0;
    for (int j = diag[i] + 1; j < rows[i + 1]; ++j) l = std::max(l, ulev[cols[j]] + 1);
    ulev[i] = l;
  }
  P.pos_lo.assign((size_t)n + 8, 0);
  P.pos_up.assign((size_t)n + 8, 0);
  for (int s = 0; s < n; ++s) {
    P.pos_lo[lo[s]] = s;
    P.pos_up[up[s]] = s;
  }
  slot_levels(lo, llev, P.lo);
  slot_levels(up, ulev, P.up);
  const long long rs = std::max(ring_need(P.lo, lp, lc, P.pos_lo), ring_need(P.up, upp, uc, P.pos_up));
  if (rs > 65535) return;
  ell_layout(P.lo, lp);
  ell_layout(P.up, upp);
  if (P.lo.off[P.lo.nlev] > 0x7ffffff0LL || P.up.off[P.up.nlev] > 0x7ffffff0LL) return;
  P.rs = (int)rs;
  P.ok = true;
  for (int v = 0; v < 2; ++v) {
    const int vsize = v == 0 ? 8 : 4;
    for (int pd = PD_MAX; pd >= 1; --pd) {
      long long sb = 8, sr = 1;
      windows(P.lo, pd, sb, sr);
      windows(P.up, pd, sb, sr);
      sb = (sb + 7) / 8 * 8;
      if (sb > (1 << 24) || sr > (1 << 24)) continue;
      const size_t bytes = cta_smem_bytes((int)sb, (int)rs, (int)sr, vsize, std::max(P.lo.nlev, P.up.nlev));
      if (bytes <= smem_max) {
        P.fits[v] = true;
        P.pd[v] = pd;
        P.sb[v] = (int)sb;
        P.sr[v] = (int)sr;
        P.smem[v] = bytes;
        break;
      }
    }
  }
}

inline bool plan_arrays(Plan &P, int n, const std::vector<int> &lo, const std::vector<int> &up,
                        const std::vector<int> &lp, const std::vector<int> &lc, const std::vector<int> &upp,
                        const std::vector<int> &uc) {
  return fill_arrays(P.lo, n, P.rs, lp, lc, P.pos_lo, lo, &P.pos_up) &&
         fill_arrays(P.up, n, P.rs, upp, uc, P.pos_up, up, nullptr);
}

}  // namespace plan
}  // namespace egpu
