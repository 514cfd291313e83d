// CPU model of the level-synchronous single-block ILU0 solve (cta_tri_solve in
// elmerfem_b200/csrc/egpu_krylov.cuh) driven by the product's own planning code
// (egpu_tri_plan.h).  It replays the kernel's staging and ring-buffer index arithmetic
// step by step, with every shared-memory cell tagged by the level (or slot) that wrote
// it, and checks:
//   - a staged copy never overwrites a cell of a level that is still live,
//   - every value a row reads was staged for its own level / produced by the slot the
//     entry depends on, and padding entries read the zero slot,
//   - no ring slot is written and read within one level,
//   - every copy stays inside its global array,
// and returns the model's y / z next to a plain sequential CRS_LUSolve
// (fem/src/CRSMatrix.src:3346-3363) with the same operation order, for a bit-exact
// comparison.  Test infrastructure: built and called by tests/test_tri_plan.py.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "egpu_tri_plan.h"

using egpu::plan::Lev;
using egpu::plan::Plan;
using egpu::plan::TriPlan;

namespace {

// the sync-free schedule's slot orders and packed parts, as ensure_tri_schedule builds them
void orders(int n, const std::vector<int> &rows, const std::vector<int> &cols, const std::vector<int> &diag,
            std::vector<int> &lower, std::vector<int> &upper) {
  std::vector<int> lev(n, 0);
  int nlow = 0;
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int j = rows[i]; j < diag[i]; ++j) l = std::max(l, lev[cols[j]] + 1);
    lev[i] = l;
    nlow = std::max(nlow, l + 1);
  }
  std::vector<int> cnt(nlow + 1, 0);
  for (int i = 0; i < n; ++i) cnt[lev[i] + 1]++;
  for (int l = 0; l < nlow; ++l) cnt[l + 1] += cnt[l];
  lower.assign(n, 0);
  for (int i = 0; i < n; ++i) lower[cnt[lev[i]]++] = i;
  int nup = 0;
  for (int i = n - 1; i >= 0; --i) {
    int l = 0;
    for (int j = diag[i] + 1; j < rows[i + 1]; ++j) l = std::max(l, lev[cols[j]] + 1);
    lev[i] = l;
    nup = std::max(nup, l + 1);
  }
  cnt.assign(nup + 1, 0);
  for (int i = 0; i < n; ++i) cnt[lev[i] + 1]++;
  for (int l = 0; l < nup; ++l) cnt[l + 1] += cnt[l];
  upper.assign(n, 0);
  for (int i = n - 1; i >= 0; --i) upper[cnt[lev[i]]++] = i;
}

template <typename VT>
struct Model {
  const Plan &P;
  int v, SB, SR, RS, PD;
  std::vector<VT> sv, ring, rr, rd;
  std::vector<uint16_t> si;
  std::vector<int> rm;
  std::vector<long long> sv_tag, si_tag, row_tag, ring_tag;
  int err = 0;

  Model(const Plan &p, int vv) : P(p), v(vv) {
    SB = P.sb[v];
    SR = P.sr[v];
    RS = P.rs;
    PD = P.pd[v];
    sv.assign(SB, 0);
    si.assign(SB, 0);
    sv_tag.assign(SB, -1);
    si_tag.assign(SB, -1);
    rr.assign(SR, 0);
    rd.assign(SR, 0);
    rm.assign(SR, 0);
    row_tag.assign(SR, -1);
    ring.assign(RS + 1, 0);
    ring_tag.assign(RS + 1, -1);
  }

  void fail(int code) {
    if (!err) err = code;
  }

  // the kernel's cta_issue for level L (live levels: [live0, L))
  void issue(const TriPlan &T, const std::vector<VT> &vals, int L, int live0, const std::vector<VT> &rowv,
             const std::vector<VT> &dinv, bool upper) {
    const Lev lv = T.lev[L];
    constexpr int PV = 16 / sizeof(VT);
    const int ne = (lv.y * lv.z + 7) & ~7;
    const int sb = lv.w % SB;
    if ((long long)lv.w + ne > T.nent) fail(10);
    if (sb % 8) fail(11);
    for (int c = 0; c < ne / PV; ++c) {
      int d = sb + c * PV;
      if (d >= SB) d -= SB;
      if (d < 0 || d + PV > SB) { fail(12); return; }
      for (int k = 0; k < PV; ++k) {
        if (sv_tag[d + k] >= live0 && sv_tag[d + k] < L) fail(13);
        sv[d + k] = vals[lv.w + c * PV + k];
        sv_tag[d + k] = L;
      }
    }
    for (int c = 0; c < ne / 8; ++c) {
      int d = sb + c * 8;
      if (d >= SB) d -= SB;
      if (d < 0 || d + 8 > SB) { fail(14); return; }
      for (int k = 0; k < 8; ++k) {
        if (si_tag[d + k] >= live0 && si_tag[d + k] < L) fail(15);
        si[d + k] = T.ridx[lv.w + c * 8 + k];
        si_tag[d + k] = L;
      }
    }
    const int rb = lv.x % SR;
    for (int t = 0; t < lv.y; ++t) {
      int d = rb + t;
      if (d >= SR) d -= SR;
      if (d < 0 || d >= SR) { fail(16); return; }
      if (row_tag[d] >= live0 && row_tag[d] < L) fail(17);
      if (lv.x + t >= (int)rowv.size()) fail(18);
      rr[d] = rowv[lv.x + t];
      rm[d] = T.map[lv.x + t];
      if (upper) rd[d] = dinv[lv.x + t];
      row_tag[d] = L;
    }
  }

  // the kernel's cta_level; deps: expected slot of each ELL entry (-1: padding)
  void level(const TriPlan &T, int L, const std::vector<long long> &deps, std::vector<VT> &outv, bool upper) {
    const Lev lv = T.lev[L];
    const int sb = lv.w % SB, rb = lv.x % SR, qb = lv.x % RS;
    std::vector<char> wr(RS + 1, 0), rd_set(RS + 1, 0);
    std::vector<std::pair<int, VT>> writes;
    for (int t = 0; t < lv.y; ++t) {
      int r = rb + t;
      if (r >= SR) r -= SR;
      if (row_tag[r] != L) fail(20);
      VT s = rr[r];
      int e = sb + t;
      if (e >= SB) e -= SB;
      for (int k = 0; k < lv.z; ++k) {
        if (sv_tag[e] != L || si_tag[e] != L) fail(21);
        const int idx = si[e];
        if (idx > RS) { fail(22); break; }
        const long long want = deps[(long long)lv.w + (long long)k * lv.y + t];
        if (want < 0) {
          if (idx != RS) fail(23);
        } else if (ring_tag[idx] != want) {
          fail(24);
        }
        rd_set[idx] = 1;
        if (sizeof(VT) == 8) {
          volatile double prod = (double)sv[e] * (double)ring[idx];
          s = (VT)((double)s - prod);
        } else {
          s = std::fma(-(float)sv[e], (float)ring[idx], (float)s);
        }
        e += lv.y;
        if (e >= SB) e -= SB;
      }
      if (upper) {
        volatile VT z = rd[r] * s;
        s = z;
      }
      int q = qb + t;
      if (q >= RS) q -= RS;
      if (q < 0 || q >= RS) fail(25);
      wr[q] = 1;
      writes.push_back({q, s});
      ring_tag[q] = lv.x + t;
      ring[q] = s;
      const int dst = rm[r];
      if (dst < 0 || dst >= (int)outv.size()) { fail(26); continue; }
      outv[dst] = s;
    }
    for (int q = 0; q <= RS; ++q)
      if (wr[q] && rd_set[q]) fail(27);
  }

  // the kernel's running window positions (CtaPos) must equal the modular ones used here
  struct Pos {
    int sb = 0, rb = 0, qb = 0;
  };
  void advance(Pos &p, const Lev &lv) {
    p.sb += (lv.y * lv.z + 7) & ~7;
    if (p.sb >= SB) p.sb -= SB;
    p.rb += lv.y;
    if (p.rb >= SR) p.rb -= SR;
    p.qb += lv.y;
    if (p.qb >= RS) p.qb -= RS;
  }
  void check_pos(const Pos &p, const Lev &lv) {
    if (p.sb != lv.w % SB || p.rb != lv.x % SR || p.qb != lv.x % RS) fail(30);
    if (p.sb < 0 || p.sb >= SB || p.rb < 0 || p.rb >= SR || p.qb < 0 || p.qb >= RS) fail(31);
  }

  void solve(const TriPlan &T, const std::vector<VT> &vals, const std::vector<long long> &deps,
             const std::vector<VT> &rowv, const std::vector<VT> &dinv, std::vector<VT> &outv, bool upper) {
    ring[RS] = 0;
    ring_tag[RS] = -2;
    const int nlev = T.nlev;
    Pos pi, pp;
    for (int p = 0; p < PD && p < nlev; ++p) {
      check_pos(pi, T.lev[p]);
      issue(T, vals, p, 0, rowv, dinv, upper);
      advance(pi, T.lev[p]);
    }
    for (int L = 0; L < nlev; ++L) {
      if (L + PD < nlev) {
        check_pos(pi, T.lev[L + PD]);
        issue(T, vals, L + PD, L, rowv, dinv, upper);
        advance(pi, T.lev[L + PD]);
      }
      check_pos(pp, T.lev[L]);
      level(T, L, deps, outv, upper);
      advance(pp, T.lev[L]);
    }
  }
};

// expected dependency slot of every ELL entry
std::vector<long long> ell_deps(const TriPlan &T, const std::vector<int> &pcols, const std::vector<int> &pos) {
  std::vector<long long> d(T.nent, -1);
  for (long long q = 0; q < T.nent; ++q)
    if (T.src[q] >= 0) d[q] = pos[pcols[T.src[q]]];
  return d;
}

template <typename VT>
int run(int n, const std::vector<int> &rows, const std::vector<int> &cols, const std::vector<int> &diag,
        const double *vals, const double *b, double *z_model, double *z_ref, size_t smem_max, int v, int *info) {
  std::vector<int> lo, up;
  orders(n, rows, cols, diag, lo, up);
  std::vector<int> lp(n + 1, 0), upp(n + 1, 0);
  for (int q = 0; q < n; ++q) {
    lp[q + 1] = lp[q] + (diag[lo[q]] - rows[lo[q]]);
    upp[q + 1] = upp[q] + (rows[up[q] + 1] - diag[up[q]] - 1);
  }
  std::vector<int> lc(std::max(1, lp[n])), ls(std::max(1, lp[n])), uc(std::max(1, upp[n])), us(std::max(1, upp[n]));
  for (int q = 0; q < n; ++q) {
    const int i = lo[q];
    for (int j = rows[i], k = lp[q]; j < diag[i]; ++j, ++k) {
      lc[k] = cols[j];
      ls[k] = j;
    }
    const int u = up[q];
    for (int j = diag[u] + 1, k = upp[q]; j < rows[u + 1]; ++j, ++k) {
      uc[k] = cols[j];
      us[k] = j;
    }
  }
  Plan P;
  egpu::plan::make_plan(n, rows, cols, diag, lo, up, lp, lc, upp, uc, smem_max, P);
  info[0] = P.ok;
  info[1] = P.fits[v];
  info[2] = P.rs;
  info[3] = P.pd[v];
  info[4] = P.sb[v];
  info[5] = P.sr[v];
  info[6] = (int)P.smem[v];
  info[7] = P.lo.nlev;
  info[8] = P.up.nlev;
  if (!P.ok || !P.fits[v]) return 0;
  if (!egpu::plan::plan_arrays(P, n, lo, up, lp, lc, upp, uc)) return 1;
  // factor values: ELL values from the packed entries, as k_cta_fill does
  auto ell = [&](const TriPlan &T, const std::vector<int> &src_crs) {
    std::vector<VT> e(T.nent, 0);
    for (long long q = 0; q < T.nent; ++q)
      if (T.src[q] >= 0) e[q] = (VT)vals[src_crs[T.src[q]]];
    return e;
  };
  const std::vector<VT> elo = ell(P.lo, ls), eup = ell(P.up, us);
  std::vector<VT> rhs_lo(n), dinv(n), yup(n + 8, 0), z(n, 0);
  for (int s = 0; s < n; ++s) {
    rhs_lo[s] = (VT)b[lo[s]];
    dinv[s] = (VT)vals[diag[up[s]]];
  }
  Model<VT> M(P, v);
  M.solve(P.lo, elo, ell_deps(P.lo, lc, P.pos_lo), rhs_lo, dinv, yup, false);
  if (M.err) return 100 + M.err;
  std::vector<VT> yslot(yup.begin(), yup.begin() + n);
  M.solve(P.up, eup, ell_deps(P.up, uc, P.pos_up), yslot, dinv, z, true);
  if (M.err) return 200 + M.err;
  for (int i = 0; i < n; ++i) z_model[i] = (double)z[i];
  // sequential CRS_LUSolve with the same operation order
  std::vector<VT> x(n);
  for (int i = 0; i < n; ++i) {
    VT s = (VT)b[i];
    for (int j = rows[i]; j < diag[i]; ++j) {
      if (sizeof(VT) == 8) {
        volatile double prod = (double)vals[j] * (double)x[cols[j]];
        s = (VT)((double)s - prod);
      } else {
        s = std::fma(-(float)vals[j], (float)x[cols[j]], (float)s);
      }
    }
    x[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    VT s = x[i];
    for (int j = diag[i] + 1; j < rows[i + 1]; ++j) {
      if (sizeof(VT) == 8) {
        volatile double prod = (double)vals[j] * (double)x[cols[j]];
        s = (VT)((double)s - prod);
      } else {
        s = std::fma(-(float)vals[j], (float)x[cols[j]], (float)s);
      }
    }
    volatile VT zz = (VT)vals[diag[i]] * s;
    x[i] = zz;
  }
  for (int i = 0; i < n; ++i) z_ref[i] = (double)x[i];
  return 0;
}

}  // namespace

// rows (n+1), cols, diag: 0-based CRS; vals: strictly lower L, strictly upper U and the
// inverted U diagonal at the diagonal positions.  v = 0 FP64, 1 FP32.  Returns 0 when every
// check passed (info[1] == 0: the plan does not fit and nothing was modelled).
extern "C" int cta_model_check(int n, const int *rows, const int *cols, const int *diag, const double *vals,
                               const double *b, double *z_model, double *z_ref, long long smem_max, int v,
                               int *info) {
  std::vector<int> r(rows, rows + n + 1), c(cols, cols + rows[n]), d(diag, diag + n);
  if (v == 0) return run<double>(n, r, c, d, vals, b, z_model, z_ref, (size_t)smem_max, 0, info);
  return run<float>(n, r, c, d, vals, b, z_model, z_ref, (size_t)smem_max, 1, info);
}
