// egpu_internal.cuh -- shared device helpers and host-side object layouts.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/elmergpu.h"
#include "egpu_devmem.h"
#include "egpu_tri_plan.h"

// ------------------------------------------------------------------------------------
// constants

// AEPS = 10*EPSILON(1.0_dp), fem/src/Types.src:64
#define EGPU_AEPS (10.0 * 2.220446049250313e-16)
#define EGPU_TINY_DP 2.2250738585072014e-308
#define EGPU_HUTI_EPSILON 1.17549435E-38

// Default upper bound on any device-side spin (grid barrier, sync-free dependency wait):
// after this many nanoseconds the waiting thread records EGPU_ERR_TIMEOUT and the kernel
// unwinds.  A context can set its own bound (egpu_set_wait_limit).
#define EGPU_WAIT_NS 2000000000ull

// The context's device control block is its sync buffer of EGPU_SYNC_WORDS 32-bit words:
// word 0 the grid-barrier counter, word 1 the error word every kernel reports to, words
// 2..63 per-solve scratch (cleared before each solve), and from EGPU_CTL_WORD on the words
// that persist across solves: the wait bound in ns (u64, 0 = EGPU_WAIT_NS) and the device
// address of the host-mapped abort word (u64, 0 = none).  Kernels receive a pointer to the
// error word and find the control words at a fixed distance from it.
#define EGPU_SYNC_WORDS 128
#define EGPU_CTL_WORD 64
#define EGPU_SELFTEST_WORD 96

// Bit patterns that mark "not yet produced" in the sync-free triangular solves and the
// ILU factorisation.  They are NaNs with a payload that arithmetic never produces
// (hardware NaNs are the canonical 0x7FF8... / 0x7FC0... patterns).
#define EGPU_SENTINEL64 0x7FF4DEAD5EED0001ull
#define EGPU_SENTINEL32 0x7FA5EED1u

#define EGPU_BLOCK 512
// the persistent Krylov kernels: one 1024-thread block per SM (32 warps, the register file
// at 64 registers a thread), so block 0 has up to 227 KB of shared memory for the
// level-synchronous triangular solves and the grid barrier has one arrival per SM
#define EGPU_KBLOCK 1024

// ------------------------------------------------------------------------------------
// error plumbing

#define EGPU_CUDA_TRY(ctx, expr)                                                   \
  do {                                                                             \
    cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      egpu_set_error((ctx), std::string(#expr) + ": " + cudaGetErrorString(e_));   \
      return EGPU_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

struct egpu_ctx;
void egpu_set_error(const egpu_ctx *ctx, const std::string &msg);

// text for a status a kernel recorded in the context's error word
inline std::string egpu_device_status_text(int err) {
  switch (err) {
    case EGPU_ERR_TIMEOUT: return "device-side wait expired (EGPU_ERR_TIMEOUT)";
    case EGPU_ERR_ABORT: return "cancelled through the abort word (EGPU_ERR_ABORT)";
    case EGPU_ERR_ARG: return "invalid data found on the device (EGPU_ERR_ARG)";
    default: return "device-side error " + std::to_string(err);
  }
}

// ------------------------------------------------------------------------------------
// device memory owner

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  bool owned = true;  // false: a view of another object's buffer (matrix clones)
  size_t cap = 0;     // bytes of the owned block (at least n elements)
  int dev = 0;        // device of the owned block
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p && owned) egpu::dev_free(p, cap, dev);
    p = nullptr;
    n = 0;
    cap = 0;
    owned = true;
  }
  void view(const DevBuf &o) {
    release();
    p = o.p;
    n = o.n;
    owned = false;
  }
  // a buffer of count elements owned by this object: reused when it already is one, never
  // written through a view (a view is detached first)
  cudaError_t alloc(size_t count) {
    if (count == n && p && owned) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    void *q = nullptr;
    cudaError_t e = egpu::dev_alloc(&q, count * sizeof(T), &cap, &dev);
    if (e == cudaSuccess) {
      p = (T *)q;
      n = count;
    }
    return e;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------------------------------
// host objects

struct egpu_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ek0 = nullptr, ek1 = nullptr;
  mutable std::string last_error;
  long long launches = 0;
  // scratch reused by solves on this context
  DevBuf<unsigned int> sync;    // [0] barrier counter, [1] error flag, [2..] misc
  DevBuf<double> partials;      // per-block partial sums
  unsigned int *sync_host_err = nullptr;
  // host-mapped abort word (egpu_abort): written by any host thread, polled by the kernels
  volatile int *abort_word = nullptr;
};

// One triangle of the level-synchronous solve that a single block runs (CtaTri in
// egpu_krylov.cuh).  Level L owns slots [lev.x, lev.x + lev.y) and an ELL block of
// lev.z entries per row stored column-major at [lev.w, lev.w + round8(lev.y * lev.z)):
// entry k of the level's row t sits at lev.w + k * lev.y + t.  ridx is the ring-buffer
// slot of the entry's column (the column's solve slot modulo the ring size; padding
// entries point at the ring's zero slot), src the packed factor entry it is filled
// from (-1 for padding).  map: lower, the upper-order slot of the row; upper, the row.
struct CtaTriHost {
  int nlev = 0;
  long long nent = 0;
  DevBuf<int4> lev;
  DevBuf<uint16_t> ridx;
  DevBuf<int> src;
  DevBuf<int> map;
};

struct TriSchedule {
  // rows in the order the sync-free solve processes them (ascending dependency level)
  DevBuf<int> lower_order, upper_order;
  // the strictly lower / upper entries of those rows packed in slot order: slot s owns
  // [lo_ptr[s], lo_ptr[s+1]); *_src is the CRS position each packed entry comes from
  DevBuf<int> lo_ptr, lo_cols, lo_src, up_ptr, up_cols, up_src, up_dsrc;
  int lower_levels = 0, upper_levels = 0;
  int max_lower = 0, max_upper = 0;  // longest strictly-lower / strictly-upper row part
  int max_width = 0;                 // most rows in one level (lower or upper)
  // rows per sync-free slot group: bs > 1 when the matrix is made of dense diagonal blocks
  // of bs consecutive rows (node DOFs) and the node-block solve was chosen; the orders then
  // hold whole blocks (slots s*bs .. s*bs+bs-1: lower ascending, upper descending rows) and
  // the levels count blocks
  int bs = 1;
  // level-synchronous single-block schedule; cta_ok[v] for FP64 (v = 0) / FP32 (v = 1)
  CtaTriHost cta_lo, cta_up;
  DevBuf<int> pos_lo, pos_up;        // solve slot of every row in the lower / upper order
  int cta_rs = 0;                    // ring slots
  bool cta_ok[2] = {false, false};
  int cta_pd[2] = {0, 0}, cta_sb[2] = {0, 0}, cta_sr[2] = {0, 0};
  size_t cta_smem[2] = {0, 0};
};

struct AssemblyData {
  int nnodes = 0, nelem = 0, nen = 0, code = 0, dofs = 1, cdim = 3;
  DevBuf<double> xyz;        // nnodes*3
  DevBuf<int> elem_nodes;    // nelem*nen, 0-based node ids, element order
  DevBuf<int> perm;          // nnodes, 0-based row block or -1
  DevBuf<int> color_elems;   // elements grouped by colour
  std::vector<int> color_ptr;
  DevBuf<int> slots;         // per element (nen*dofs)^2 CRS positions (0-based), element order
  bool bound = false;
};

struct egpu_mat {
  egpu_ctx *ctx = nullptr;
  int n = 0;
  long long nnz = 0;
  DevBuf<int> rows, cols, diag;  // 0-based
  DevBuf<double> values;         // as bound / assembled (unscaled)
  DevBuf<double> rhs;            // assembled right-hand side
  bool has_values = false, has_rhs = false;
  // the library's measured choice of path for mixed requests: per path (0 FP64 drop-in,
  // 1 mixed with exact triangular solves, 2 mixed with ILU0 by Jacobi sweeps) the device
  // seconds of its latest timed solve and the number timed; the matrix's first solve (which
  // carries the one-time set-up) is not timed.  They outlive value updates (a time or
  // nonlinear loop re-assembles the same operator).
  double t_path[3] = {0.0, 0.0, 0.0};
  int n_path[3] = {0, 0, 0};
  int n_solved = 0;
  int max_row = 0;               // longest row
  int max_bandwidth = 0;         // max |col - row|
  bool sorted_rows = true;       // columns strictly ascending in every row (CRS_SortMatrix); ILU needs it
  // solve state
  DevBuf<double> scaled;         // D A D
  DevBuf<double> dscale;         // DiagScaling (times the rhs norm during a solve)
  DevBuf<double> ilu;            // ILU0 values on the scaled matrix, inverted U diagonal
  DevBuf<float> ilu32;           // FP32 factor copy for the mixed-precision inner solver
  DevBuf<double> lo_vals, up_vals, up_dinv;        // ILU0 factors packed in solve order
  DevBuf<float> lo_vals32, up_vals32, up_dinv32;
  DevBuf<double> cta_lo_vals, cta_up_vals;        // the factors in the level-synchronous ELL layout
  DevBuf<float> cta_lo_vals32, cta_up_vals32;
  DevBuf<int16_t> cols16;        // column offsets (col - row) when |col-row| < 32768
  DevBuf<int> ilu_done;          // factorisation completion flags
  // SELL-32 copy of the pattern (slice s = rows 32s..32s+31, entry (k, lane) at
  // sell_ptr[s] + 32k + lane; rows padded to the slice width with zero values)
  int nslices = 0;
  long long sell_nnz = 0;
  long long ldw = 0;             // stride of the work vectors (>= n + 32, multiple of 64)
  DevBuf<int> sell_ptr, sell_w, sell_cols;
  DevBuf<int16_t> sell_c16;      // col - row, when every |col - row| < 32768
  // the same offsets compacted: slice s starts at sell_cptr[s] (per entry) or, for a slice
  // whose rows share one offset list, at -sell_cptr[s] - 1 (w entries)
  DevBuf<int> sell_cptr;
  DevBuf<int16_t> sell_csc;
  DevBuf<double> sell_vals;      // scaled values (FP64)
  DevBuf<float> sell_vals32;     // scaled values (FP32)
  // per slice: the k range of the strictly-lower entries ([0, x)) and of the strictly-upper
  // ones ([y, w)); ILU0 factors in the SELL layout (FP32) and the inverted U diagonal in row
  // order, for the Jacobi-sweep application of the preconditioner
  DevBuf<int2> sell_swr;
  DevBuf<float> ilu_sell32, ilu_dinv32;
  // ILU structure: the matrix's own pattern for ILU0, the ILU(n) fill structure otherwise
  // (0-based); the triangular-solve schedules in tri are built on it
  int ilu_order = -1;            // order the structure was built for (-1: not yet, ILU_ORDER_T: ILUT)
  double ilut_tol = 0.0;         // drop tolerance of the current ILUT factor
  long long ilu_nnz = 0;
  int ilu_max_row = 0;
  DevBuf<int> ilu_rows, ilu_cols, ilu_diag;
  DevBuf<int> ilu_scatter;       // ILU(n): position of every matrix entry in the structure
  DevBuf<double> ilu_in;         // ILU(n): the scaled matrix scattered into the structure
  TriSchedule tri;
  bool tri_built = false;
  int solve_count = 0;
  bool ilu_valid = false;
  DevBuf<double> work;           // Krylov work vectors
  DevBuf<double> ext_work;       // GCR directions / BiCGStab(l) vectors
  DevBuf<float> work32;
  DevBuf<double> bx;             // scratch b/x for host-pointer entry points
  AssemblyData asmb;
  // clones share this matrix's pattern: it is deleted when its last clone goes
  egpu_mat *parent = nullptr;
  int clones = 0;
  bool free_pending = false;
};

// ------------------------------------------------------------------------------------
// device helpers

__device__ __forceinline__ unsigned long long egpu_globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_acquire_s32(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_s32(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void red_release_add_u32(unsigned int *p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const void *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const void *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(void *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(void *p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// the context's wait bound (ns), read next to its error word
__device__ __forceinline__ unsigned long long egpu_wait_limit(const int *err) {
  const unsigned long long v =
      *(const volatile unsigned long long *)((const unsigned int *)err + (EGPU_CTL_WORD - 1));
  return v ? v : EGPU_WAIT_NS;
}

// Reads the context's host-mapped abort word (one load over the host link) and, when the host
// has raised it, records EGPU_ERR_ABORT unless another error is already recorded; every
// block then leaves at its next grid barrier or bounded wait.
__device__ __forceinline__ void egpu_poll_abort(int *err) {
  const unsigned long long a =
      *(const volatile unsigned long long *)((const unsigned int *)err + (EGPU_CTL_WORD + 1));
  if (a && *(const volatile int *)a) atomicCAS(err, 0, (int)EGPU_ERR_ABORT);
}

// value type traits for the sync-free solves
template <typename T>
struct Sentinel;
template <>
struct Sentinel<double> {
  __device__ __forceinline__ static double value() { return __longlong_as_double((long long)EGPU_SENTINEL64); }
  __device__ __forceinline__ static bool is(double v) {
    return (unsigned long long)__double_as_longlong(v) == EGPU_SENTINEL64;
  }
  // bounded wait until p holds a produced value; returns it (or the sentinel on timeout)
  __device__ __forceinline__ static double wait(const double *p, int *err) {
    unsigned long long v = ld_relaxed_u64(p);
    if (v != EGPU_SENTINEL64) return __longlong_as_double((long long)v);
    const unsigned long long t0 = egpu_globaltimer(), lim = egpu_wait_limit(err);
    for (unsigned int spin = 1;; ++spin) {
      v = ld_relaxed_u64(p);
      if (v != EGPU_SENTINEL64) break;
      if ((spin & 31u) == 0) {
        if (egpu_globaltimer() - t0 > lim) {
          atomicExch(err, (int)EGPU_ERR_TIMEOUT);
          break;
        }
        if (*(volatile int *)err) break;
      }
    }
    return __longlong_as_double((long long)v);
  }
  // one relaxed load, no wait (the sentinel if not produced yet)
  __device__ __forceinline__ static double peek(const double *p) {
    return __longlong_as_double((long long)ld_relaxed_u64(p));
  }
  __device__ __forceinline__ static void publish(double *p, double v) {
    st_relaxed_u64(p, (unsigned long long)__double_as_longlong(v));
  }
};
template <>
struct Sentinel<float> {
  __device__ __forceinline__ static float value() { return __uint_as_float(EGPU_SENTINEL32); }
  __device__ __forceinline__ static bool is(float v) { return __float_as_uint(v) == EGPU_SENTINEL32; }
  __device__ __forceinline__ static float wait(const float *p, int *err) {
    unsigned int v = ld_relaxed_u32(p);
    if (v != EGPU_SENTINEL32) return __uint_as_float(v);
    const unsigned long long t0 = egpu_globaltimer(), lim = egpu_wait_limit(err);
    for (unsigned int spin = 1;; ++spin) {
      v = ld_relaxed_u32(p);
      if (v != EGPU_SENTINEL32) break;
      if ((spin & 31u) == 0) {
        if (egpu_globaltimer() - t0 > lim) {
          atomicExch(err, (int)EGPU_ERR_TIMEOUT);
          break;
        }
        if (*(volatile int *)err) break;
      }
    }
    return __uint_as_float(v);
  }
  __device__ __forceinline__ static float peek(const float *p) { return __uint_as_float(ld_relaxed_u32(p)); }
  __device__ __forceinline__ static void publish(float *p, float v) { st_relaxed_u32(p, __float_as_uint(v)); }
};

// Grid-wide barrier for a cooperative (co-resident) launch.  count is a monotonically
// increasing arrival counter reset to 0 before the launch; epoch is the per-block count
// of barriers passed.  The wait is bounded by the context's wait limit; on expiry the error
// flag is set.  Block 0 reads the host's abort word every EGPU_ABORT_POLL-th barrier, before
// it arrives (the read crosses the host link, so every other block waits for it: rare enough
// to cost nothing measurable), and block 1 reads it during long waits.  Reads of host memory
// are kept this rare on purpose: hundreds of warps polling it while they wait (the sync-free
// solves, the ILU factorisation) doubled the set-up time of a large solve.  Returns false
// when the kernel must unwind (error flag set by anyone).
#define EGPU_ABORT_POLL 256u
__device__ __forceinline__ bool grid_barrier(unsigned int *count, int *err, unsigned int &epoch) {
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) {
    if (blockIdx.x == 0 && (epoch % EGPU_ABORT_POLL) == 0) egpu_poll_abort(err);
    const unsigned int target = epoch * gridDim.x;
    red_release_add_u32(count, 1u);
    if (ld_acquire_u32(count) < target) {
      const unsigned long long t0 = egpu_globaltimer(), lim = egpu_wait_limit(err);
      unsigned int spins = 0;
      while (ld_acquire_u32(count) < target) {
        if ((++spins & 63u) == 0) {
          // one block polls during long waits (block 0 may be the one still working)
          if ((spins & 1023u) == 0 && blockIdx.x == (gridDim.x > 1 ? 1u : 0u)) egpu_poll_abort(err);
          if (*(volatile int *)err) break;
          if (egpu_globaltimer() - t0 > lim) {
            atomicExch(err, (int)EGPU_ERR_TIMEOUT);
            break;
          }
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int *)err == 0;
}

// Asynchronous global -> shared copies (cp.async, completion tracked per thread in
// commit groups).  16-byte copies bypass L1 (.cg); 4/8-byte copies go through it (.ca).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
template <int B>
__device__ __forceinline__ void cp_async_small(void *smem, const void *gmem) {
  static_assert(B == 4 || B == 8, "4- or 8-byte copy");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// bulk prefetch of a contiguous global range into L2 (no completion to wait for); the
// address must be 16-byte aligned and the size a multiple of 16 bytes
__device__ __forceinline__ void prefetch_l2_bulk(const void *gmem, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gmem), "r"(bytes) : "memory");
}
// wait until at most n (0..7) of this thread's most recent groups are still pending
__device__ __forceinline__ void cp_async_wait(int n) {
  switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
    case 6: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
    case 7: asm volatile("cp.async.wait_group 7;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;  // conservative
  }
}

// Deterministic block sum of NV values per thread (fixed shuffle tree, fixed warp order).
// Result valid in every thread.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /* >= 32*NV */) {
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    v[k] = __shfl_sync(0xffffffffu, t, 0);
  }
  __syncthreads();
}

// Sum of partials[0..nb) read from L2 in a fixed order (same result in every block).
__device__ __forceinline__ double reduce_partials(const double *partials, int nb, double *smem) {
  double t = 0.0;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    for (int i = lane; i < nb; i += 32) t += __ldcg(partials + i);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (lane == 0) smem[0] = t;
  }
  __syncthreads();
  t = smem[0];
  __syncthreads();
  return t;
}
