// fues.cu -- FUES upper envelope of DC-EGM candidate rows (kernel c, part 2).
//
// Restates the Fast Upper-Envelope Scan (Dobrescu & Shanker 2022) with the
// reference's rules (src/_lcm/egm/upper_envelope/fues.py:151-1189):
//   1. sort each row by (grid asc, value desc, policy desc), NaN grid last,
//      ties by input position (a stable lexsort);
//   2. reduce every run of equal grid values to its maximisers, keeping one
//      copy per exogenous savings source;
//   3. scan the sorted row keeping the last two envelope points (k, j); drop a
//      candidate below j on the same segment, one with falling savings and a
//      secant below the previous gradient, or one below the continuation of
//      j's segment; insert segment crossings twice (left / right policy);
//      "same segment" means |d(R - c)/dR| <= jump_thresh.
//
// GPU mapping: one CTA per row.  The CTA sorts an index array in shared
// memory (bitonic), gathers the sorted row into the workspace, reduces the
// coincident groups in parallel, and then warp 0 runs the scan: the scan
// state is held redundantly by all 32 lanes, and each exhaustive look-ahead
// for the next same-segment candidate inspects 32 candidates per step with
// a warp ballot.  Lane 0 writes the emissions.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/lcmx.h"

namespace {

constexpr int kBlock = 256;
constexpr int kMaxSort = 8192;  // largest row the shared-memory sort handles

__device__ __forceinline__ bool isnan_(double x) { return x != x; }

__device__ __forceinline__ double slope(double xa, double ya, double xb, double yb) {
  const double dx = xb - xa;
  return dx == 0.0 ? 0.0 : (yb - ya) / dx;
}

// different segments iff the implied savings (R - c) jump
__device__ __forceinline__ bool policy_jump(double ga, double pa, double gb, double pb, double thr,
                                            bool use_sav, double sa, double sb) {
  const double ia = ga - pa, ib = gb - pb;
  if (ga == gb) return use_sav ? (sa != sb) : (ia != ib);
  return fabs(slope(ga, ia, gb, ib)) > thr;
}

__device__ __forceinline__ void intersect(double xa, double ya, double sa, double xb, double yb, double sb,
                                          double& x, double& y) {
  const double den = sa - sb;
  if (den == 0.0) {
    x = __longlong_as_double(0x7ff8000000000000LL);
    y = ya;
    return;
  }
  x = (yb - ya + sa * xa - sb * xb) / den;
  y = ya + sa * (x - xa);
}

struct Key {
  double g, v, p;
  int i;
};

__device__ __forceinline__ Key load_key(const double* g, const double* v, const double* p, int i, int n) {
  Key k;
  k.i = i;
  if (i >= n) {
    k.g = __longlong_as_double(0x7ff0000000000000LL);  // padding sorts last
    k.v = -k.g;
    k.p = -k.g;
    k.i = 0x7fffffff;
    return k;
  }
  const double gi = g[i], vi = v[i], pi = p[i];
  k.g = isnan_(gi) ? __longlong_as_double(0x7ff0000000000000LL) : gi;
  k.v = isnan_(vi) ? -__longlong_as_double(0x7ff0000000000000LL) : vi;
  k.p = isnan_(pi) ? -__longlong_as_double(0x7ff0000000000000LL) : pi;
  return k;
}

// a before b ?
__device__ __forceinline__ bool key_less(const Key& a, const Key& b) {
  if (a.g != b.g) return a.g < b.g;
  if (a.v != b.v) return a.v > b.v;
  if (a.p != b.p) return a.p > b.p;
  return a.i < b.i;
}

// first same-segment candidate from idx in direction dir among the `window`
// positions idx + dir, ..., idx + dir * window (warp-cooperative)
__device__ __forceinline__ bool find_same_segment(const double* g, const double* p, const double* v, int n,
                                                  double ag, double ap, int idx, int dir, double thr, int window,
                                                  double& fg, double& fp, double& fv) {
  const int lane = threadIdx.x & 31;
  for (int base = idx + dir;; base += 32 * dir) {
    if (dir > 0 ? base >= n : base < 0) break;
    if ((base - idx) * dir > window) break;
    const int k = base + dir * lane;
    bool ok = false;
    double gk = 0.0, pk = 0.0, vk = 0.0;
    if (k >= 0 && k < n && (k - idx) * dir <= window) {
      gk = g[k];
      pk = p[k];
      vk = v[k];
      ok = !isnan_(gk) && !isnan_(vk) && !policy_jump(ag, ap, gk, pk, thr, false, 0.0, 0.0);
    }
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (m) {
      const int src = __ffs(m) - 1;  // nearest candidate
      fg = __shfl_sync(0xffffffffu, gk, src);
      fp = __shfl_sync(0xffffffffu, pk, src);
      fv = __shfl_sync(0xffffffffu, vk, src);
      return true;
    }
  }
  fg = fp = fv = __longlong_as_double(0x7ff8000000000000LL);
  return false;
}

__global__ void __launch_bounds__(kBlock) fues_kernel(const double* __restrict__ grid, const double* __restrict__ policy,
                                                      const double* __restrict__ value,
                                                      const double* __restrict__ savings, int n_rows, int n_in,
                                                      double thr, int window, double* __restrict__ grid_out,
                                                      double* __restrict__ policy_out, double* __restrict__ value_out,
                                                      int n_out, int* __restrict__ n_kept, double* __restrict__ work) {
  __shared__ int sidx[kMaxSort];
  int np2 = 1;
  while (np2 < n_in) np2 <<= 1;
  const bool use_sav = savings != nullptr;
  for (int row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const double* G = grid + (int64_t)row * n_in;
    const double* P = policy + (int64_t)row * n_in;
    const double* V = value + (int64_t)row * n_in;
    const double* S = use_sav ? savings + (int64_t)row * n_in : nullptr;
    double* g = work + (int64_t)row * 4 * n_in;
    double* p = g + n_in;
    double* v = p + n_in;
    double* s = v + n_in;
    // ---- 1. bitonic sort of indices by the lexsort key
    __syncthreads();
    for (int t = threadIdx.x; t < np2; t += kBlock) sidx[t] = t;
    __syncthreads();
    for (int size = 2; size <= np2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = threadIdx.x; t < np2; t += kBlock) {
          const int partner = t ^ stride;
          if (partner > t) {
            const bool ascending = (t & size) == 0;
            const Key a = load_key(G, V, P, sidx[t], n_in);
            const Key b = load_key(G, V, P, sidx[partner], n_in);
            const bool swap = ascending ? key_less(b, a) : key_less(a, b);
            if (swap) {
              const int tmp = sidx[t];
              sidx[t] = sidx[partner];
              sidx[partner] = tmp;
            }
          }
        }
        __syncthreads();
      }
    }
    for (int t = threadIdx.x; t < n_in; t += kBlock) {
      const int i = sidx[t];
      g[t] = G[i];
      p[t] = P[i];
      v[t] = V[i];
      s[t] = use_sav ? S[i] : G[i] - P[i];
    }
    __syncthreads();
    // ---- 2. coincident groups: keep the maximisers, one per savings source
    for (int t = threadIdx.x; t < n_in; t += kBlock) {
      const double gt = g[t];
      bool keep = !isnan_(gt);
      if (keep) {
        int lo = t, hi = t;
        while (lo > 0 && g[lo - 1] == gt) --lo;
        while (hi + 1 < n_in && g[hi + 1] == gt) ++hi;
        if (hi > lo) {
          double vmax = -__longlong_as_double(0x7ff0000000000000LL);
          for (int k = lo; k <= hi; ++k) {
            const double vk = v[k];
            if (!isnan_(vk) && vk > vmax) vmax = vk;
          }
          keep = v[t] == vmax;
          if (keep) {
            for (int k = lo; k < t; ++k)
              if (v[k] == vmax && s[k] == s[t]) keep = false;
          }
        }
      }
      sidx[t] = keep ? 1 : 0;  // reuse shared memory as the keep mask
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n_in; t += kBlock) {
      if (!sidx[t]) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        g[t] = p[t] = v[t] = s[t] = nan;
      }
    }
    __syncthreads();
    // ---- 3. the scan (warp 0; all lanes hold the state, lane 0 writes)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      double* GO = grid_out + (int64_t)row * n_out;
      double* PO = policy_out + (int64_t)row * n_out;
      double* VO = value_out + (int64_t)row * n_out;
      const double nan = __longlong_as_double(0x7ff8000000000000LL);
      for (int t = lane; t < n_out; t += 32) GO[t] = PO[t] = VO[t] = nan;
      __syncwarp();
      int cnt = 0;
      auto emit = [&](double eg, double ep, double ev) {
        if (lane == 0 && cnt < n_out) {
          GO[cnt] = eg;
          PO[cnt] = ep;
          VO[cnt] = ev;
        }
        ++cnt;
      };
      double gk = g[0], pk = p[0], vk = v[0];
      double gj = g[0], pj = p[0], vj = v[0], sj = s[0];
      const double near = 16.0 * 2.220446049250313e-16;
      for (int idx = 1; idx < n_in; ++idx) {
        const double gi = g[idx], pi = p[idx], vi = v[idx], si = s[idx];
        const bool valid = !isnan_(gi) && !isnan_(vi);
        const bool sw = valid && policy_jump(gj, pj, gi, pi, thr, true, sj, si);
        const bool node_crossing = valid && sw && gi == gj && vi == vj;
        const double secant = slope(gj, vj, gi, vi);
        const double grad_before = slope(gk, vk, gj, vj);
        double jg, jp, jv;
        const bool jf = find_same_segment(g, p, v, n_in, gj, pj, idx, 1, thr, window, jg, jp, jv);
        bool below_j = false;
        if (sw && jf) below_j = (gi == jg) ? (vi < jv) : (secant < slope(gi, vi, jg, jv));
        const bool sav_dec = si < sj;
        bool dropped = !valid || ((vi < vj) && !sw) || (sav_dec && secant < grad_before) || below_j;
        dropped = dropped && !node_crossing;
        if (dropped) continue;
        double fg, fp, fv, bg, bp, bv;
        const bool ff = find_same_segment(g, p, v, n_in, gi, pi, idx, 1, thr, window, fg, fp, fv);
        const bool bf = find_same_segment(g, p, v, n_in, gi, pi, idx, -1, thr, window, bg, bp, bv);
        const bool found = ff || bf;
        const double pg = ff ? fg : bg, pp = ff ? fp : bp, pv = ff ? fv : bv;
        const double i_slope = slope(gi, vi, pg, pv);
        const double i_pslope = slope(gi, pi, pg, pp);
        const bool j_dom = sw && found && (secant > i_slope) && !node_crossing;
        const double pslope_kj = slope(gk, pk, gj, pj);
        double k6g, k6v;
        intersect(gj, vj, grad_before, gi, vi, i_slope, k6g, k6v);
        const double k6pl = pj + pslope_kj * (k6g - gj);
        const double k6pr = pi + i_pslope * (k6g - gi);
        const bool kink6 = j_dom && (k6g > gk) && (k6g < gj) && (k6g < gi);
        const double j_slope = jf ? slope(gj, vj, jg, jv) : grad_before;
        const double j_pslope = jf ? slope(gj, pj, jg, jp) : pslope_kj;
        double k5g, k5v;
        intersect(gj, vj, j_slope, gi, vi, i_slope, k5g, k5v);
        const double k5pl = pj + j_pslope * (k5g - gj);
        const double k5pr = pi + i_pslope * (k5g - gi);
        const bool crossing = !j_dom && !node_crossing && sw && found;
        const double tol = near * fmax(fmax(fabs(gj), fabs(gi)), 1.0);
        const bool on_j = crossing && fabs(k5g - gj) <= tol;
        const bool on_i = crossing && !on_j && fabs(k5g - gi) <= tol;
        const bool kink5 = crossing && !on_j && !on_i && (k5g > gj) && (k5g < gi);
        const bool plain = !j_dom && !kink5 && !on_j && !on_i;
        if (kink6) {
          emit(k6g, k6pl, k6v);
          emit(k6g, k6pr, k6v);
        } else if (plain || kink5 || on_j || on_i) {
          emit(gj, pj, vj);
          if (kink5) {
            emit(k5g, k5pl, k5v);
            emit(k5g, k5pr, k5v);
          } else if (on_j) {
            emit(gj, k5pr, k5v);
          } else if (on_i) {
            emit(gi, k5pl, k5v);
          }
        }
        const bool keeps_k = j_dom && !kink6;
        if (!keeps_k) {
          if (kink5) {
            gk = k5g; pk = k5pr; vk = k5v;
          } else if (kink6) {
            gk = k6g; pk = k6pr; vk = k6v;
          } else {
            gk = gj;
            pk = on_j ? k5pr : pj;
            vk = on_j ? k5v : vj;
          }
        }
        gj = gi; pj = pi; vj = vi; sj = si;
      }
      if (!isnan_(gj) && !isnan_(vj)) emit(gj, pj, vj);
      if (lane == 0) n_kept[row] = cnt;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Shared-memory form (rows of up to kSmemMaxN candidates).
//
// Same three stages and the same decisions as fues_kernel, with the sorted
// row staged in shared memory and the scan's per-step work cut to what a
// step uses:
//   * a step without a policy jump between j and i never reads the
//     look-ahead, the intersections or i's own neighbours -- it is dropped
//     or emits j and shifts (k, j) <- (j, i);
//   * when j is the previous candidate (the common case), the policy-jump
//     test and the secant of (j, i) are precomputed for every position in
//     parallel before the scan; grad_before is the previous secant while k is
//     the candidate before j, unmodified;
//   * the look-ahead searches (warp ballot over shared memory) run only on
//     steps with a policy jump.
// Every value the scan uses is computed with the same operations and
// operands as in fues_kernel, so the rows are identical.
constexpr int kSmemMaxN = 4096;
constexpr int kFuesItemWords = 13;

__host__ __device__ constexpr size_t fues_smem_bytes(int n) {
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  return (size_t)5 * n * sizeof(double) + (size_t)np2 * (sizeof(unsigned long long) + sizeof(int));
}

// Monotone 64-bit image of a grid value for the sort: NaN ranks with +inf and
// -0 with +0, as the (double) comparison of the lexsort key treats them.
__device__ __forceinline__ unsigned long long grid_key(double g) {
  if (isnan_(g)) g = __longlong_as_double(0x7ff0000000000000LL);
  if (g == 0.0) g = 0.0;
  const unsigned long long b = (unsigned long long)__double_as_longlong(g);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

struct FuesRowIO {
  const double* G;
  const double* P;
  const double* V;
  const double* S;
  double* GO;
  double* PO;
  double* VO;
  int* nk;
  int n_in;
  int n_out;
  double thr;
  int window;  // look-ahead positions inspected in each direction
};

struct FuesContig {
  const double* grid;
  const double* policy;
  const double* value;
  const double* savings;
  double* go;
  double* po;
  double* vo;
  int* nk;
  int n_rows, n_in, n_out;
  double thr;
  int window;
  __device__ __forceinline__ int count() const { return n_rows; }
  __device__ __forceinline__ FuesRowIO row(int r) const {
    FuesRowIO io;
    io.G = grid + (int64_t)r * n_in;
    io.P = policy + (int64_t)r * n_in;
    io.V = value + (int64_t)r * n_in;
    io.S = savings ? savings + (int64_t)r * n_in : nullptr;
    io.GO = go + (int64_t)r * n_out;
    io.PO = po + (int64_t)r * n_out;
    io.VO = vo + (int64_t)r * n_out;
    io.nk = nk + r;
    io.n_in = n_in;
    io.n_out = n_out;
    io.thr = thr;
    io.window = window;
    return io;
  }
};

// item words: 0 grid, 1 policy, 2 value, 3 savings (0: none), 4 grid_out,
// 5 policy_out, 6 value_out, 7 n_kept (int32), 8 n_rows, 9 n_in, 10 n_out,
// 11 jump_thresh (double bits), 12 look-ahead window (<= 0: exhaustive);
// one tile per row
struct FuesItems {
  const int64_t* items;
  const int* prefix;
  int n_items, n_tiles;
  __device__ __forceinline__ int count() const { return n_tiles; }
  __device__ __forceinline__ FuesRowIO row(int tile) const {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= tile) lo = mid; else hi = mid - 1;
    }
    const int64_t* it = items + (int64_t)lo * kFuesItemWords;
    const int r = tile - prefix[lo];
    FuesRowIO io;
    io.n_in = (int)it[9];
    io.n_out = (int)it[10];
    io.thr = __longlong_as_double(it[11]);
    io.window = it[12] > 0 ? (int)it[12] : io.n_in;
    io.G = reinterpret_cast<const double*>(it[0]) + (int64_t)r * io.n_in;
    io.P = reinterpret_cast<const double*>(it[1]) + (int64_t)r * io.n_in;
    io.V = reinterpret_cast<const double*>(it[2]) + (int64_t)r * io.n_in;
    io.S = it[3] ? reinterpret_cast<const double*>(it[3]) + (int64_t)r * io.n_in : nullptr;
    io.GO = reinterpret_cast<double*>(it[4]) + (int64_t)r * io.n_out;
    io.PO = reinterpret_cast<double*>(it[5]) + (int64_t)r * io.n_out;
    io.VO = reinterpret_cast<double*>(it[6]) + (int64_t)r * io.n_out;
    io.nk = reinterpret_cast<int*>(it[7]) + r;
    return io;
  }
};

// x[t] <- x[sidx[t]] for t < n, through the shared-memory buffer `tmp`
__device__ __forceinline__ void permute_sorted(double* x, double* tmp, const int* sidx, int n) {
  for (int t = threadIdx.x; t < n; t += kBlock) tmp[t] = x[sidx[t]];
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += kBlock) x[t] = tmp[t];
  __syncthreads();
}

template <class Rows>
__global__ void __launch_bounds__(kBlock) fues_smem_kernel(Rows rows) {
  extern __shared__ __align__(16) unsigned char fues_smem[];
  const int total = rows.count();
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  for (int row = blockIdx.x; row < total; row += gridDim.x) {
    const FuesRowIO io = rows.row(row);
    const int n = io.n_in;
    const int n_out = io.n_out;
    const double thr = io.thr;
    const double* G = io.G;
    const double* P = io.P;
    const double* V = io.V;
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    double* g = reinterpret_cast<double*>(fues_smem);
    double* p = g + n;
    double* v = p + n;
    double* s = v + n;
    double* sec = s + n;
    unsigned long long* skey = reinterpret_cast<unsigned long long*>(sec + n);
    int* sidx = reinterpret_cast<int*>(skey + np2);
    __syncthreads();  // the previous row is done with shared memory
    // ---- 1. stage the row in shared memory (input order), sort indices by
    // the lexsort key read from there, then put each array in sorted order
    // through registers
    for (int t = threadIdx.x; t < n; t += kBlock) {
      const double gt = G[t], pt = P[t];
      g[t] = gt;
      p[t] = pt;
      v[t] = V[t];
      s[t] = io.S ? io.S[t] : gt - pt;
    }
    __syncthreads();
    // (grid key, index) pairs: a compare-exchange reads positions t and
    // t ^ stride; only equal grid keys consult value, policy and index
    for (int t = threadIdx.x; t < np2; t += kBlock) {
      sidx[t] = t;
      skey[t] = t < n ? grid_key(g[t]) : ~0ULL;  // padding sorts last
    }
    __syncthreads();
    const int half = np2 >> 1;
    for (int size = 2; size <= np2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const int ls = __ffs(stride) - 1;  // stride = 2^ls
#pragma unroll 4
        for (int j = threadIdx.x; j < half; j += kBlock) {
          // the j-th compare-exchange pair (t, t + stride) of this stage:
          // the positions whose bit ls is clear, in order
          const int t = ((j >> ls) << (ls + 1)) | (j & (stride - 1));
          const int partner = t + stride;
          {
            const bool ascending = (t & size) == 0;
            const unsigned long long ka = skey[t], kb = skey[partner];
            const int ia = sidx[t], ib = sidx[partner];
            bool a_first;  // does (ka, ia) come before (kb, ib)?
            if (ka != kb) {
              a_first = ka < kb;
            } else {
              a_first = !key_less(load_key(g, v, p, ib, n), load_key(g, v, p, ia, n));
            }
            if (ascending != a_first) {
              skey[t] = kb;
              skey[partner] = ka;
              sidx[t] = ib;
              sidx[partner] = ia;
            }
          }
        }
        __syncthreads();
      }
    }
    permute_sorted(g, sec, sidx, n);  // `sec` is free until the scan tables
    permute_sorted(p, sec, sidx, n);
    permute_sorted(v, sec, sidx, n);
    permute_sorted(s, sec, sidx, n);
    // ---- 2. coincident groups: keep the maximisers, one per savings source
    for (int t = threadIdx.x; t < n; t += kBlock) {
      const double gt = g[t];
      bool keep = !isnan_(gt);
      if (keep) {
        int lo = t, hi = t;
        while (lo > 0 && g[lo - 1] == gt) --lo;
        while (hi + 1 < n && g[hi + 1] == gt) ++hi;
        if (hi > lo) {
          double vmax = -__longlong_as_double(0x7ff0000000000000LL);
          for (int k = lo; k <= hi; ++k) {
            const double vk = v[k];
            if (!isnan_(vk) && vk > vmax) vmax = vk;
          }
          keep = v[t] == vmax;
          if (keep) {
            for (int k = lo; k < t; ++k)
              if (v[k] == vmax && s[k] == s[t]) keep = false;
          }
        }
      }
      sidx[t] = keep ? 1 : 0;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += kBlock) {
      if (!sidx[t]) g[t] = p[t] = v[t] = s[t] = nan;
    }
    for (int t = threadIdx.x; t < n_out; t += kBlock) io.GO[t] = io.PO[t] = io.VO[t] = nan;
    __syncthreads();
    // ---- 3a. per position t: policy jump and secant of (t - 1, t)
    for (int t = threadIdx.x + 1; t < n; t += kBlock) {
      sidx[t] = policy_jump(g[t - 1], p[t - 1], g[t], p[t], thr, true, s[t - 1], s[t]) ? 1 : 0;
      sec[t] = slope(g[t - 1], v[t - 1], g[t], v[t]);
    }
    __syncthreads();
    // ---- 3b. the scan (warp 0; all lanes hold the state, lane 0 writes)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      double* GO = io.GO;
      double* PO = io.PO;
      double* VO = io.VO;
      int cnt = 0;
      auto emit = [&](double eg, double ep, double ev) {
        if (lane == 0 && cnt < n_out) {
          GO[cnt] = eg;
          PO[cnt] = ep;
          VO[cnt] = ev;
        }
        ++cnt;
      };
      double gk = g[0], pk = p[0], vk = v[0];
      double gj = g[0], pj = p[0], vj = v[0], sj = s[0];
      int jidx = 0, kidx = 0;  // candidates j and k are (kidx < 0: k is a kink point)
      const double near = 16.0 * 2.220446049250313e-16;
      for (int idx = 1; idx < n; ++idx) {
        // Runs of plain steps, 32 at a time.  While j and k are the two
        // candidates before idx, step t keeps candidate t and only emits j
        // when t is valid, shows no policy jump from t - 1, and is neither
        // below t - 1 nor a savings decrease with a secant under the previous
        // one -- all of it from the per-position tables.  Such a step leaves
        // j = t - 1 + 1 and k = t - 1, so the next step's test is again a
        // table lookup: the lanes test idx .. idx + 31 at once and the warp
        // commits the leading run of passing steps (each emits its j).
        if (kidx >= 0 && jidx == idx - 1 && kidx == jidx - 1) {
          const int t = idx + lane;
          bool ok = false;
          if (t < n) {
            const double gt = g[t], vt = v[t];
            ok = !isnan_(gt) && !isnan_(vt) && sidx[t] == 0 && !(vt < v[t - 1]) &&
                 !(s[t] < s[t - 1] && sec[t] < sec[t - 1]);
          }
          const unsigned fail = ~__ballot_sync(0xffffffffu, ok);
          const int m = fail ? __ffs(fail) - 1 : 32;
          if (m > 0) {
            if (lane < m && cnt + lane < n_out) {
              GO[cnt + lane] = g[idx - 1 + lane];
              PO[cnt + lane] = p[idx - 1 + lane];
              VO[cnt + lane] = v[idx - 1 + lane];
            }
            cnt += m;
            const int nj = idx + m - 1;
            gk = g[nj - 1]; pk = p[nj - 1]; vk = v[nj - 1];
            kidx = nj - 1;
            gj = g[nj]; pj = p[nj]; vj = v[nj]; sj = s[nj];
            jidx = nj;
            idx = nj;  // the loop's increment moves to the first untested step
            continue;
          }
        }
        const double gi = g[idx], vi = v[idx];
        if (isnan_(gi) || isnan_(vi)) continue;
        const double pi = p[idx], si = s[idx];
        const bool prev = jidx == idx - 1;
        const bool sw = prev ? (sidx[idx] != 0) : policy_jump(gj, pj, gi, pi, thr, true, sj, si);
        const bool node_crossing = sw && gi == gj && vi == vj;
        bool have_sec = false, have_gb = false;
        double secant = 0.0, grad_before = 0.0;
        auto get_secant = [&]() {
          if (!have_sec) {
            secant = prev ? sec[idx] : slope(gj, vj, gi, vi);
            have_sec = true;
          }
          return secant;
        };
        auto get_gb = [&]() {
          if (!have_gb) {
            grad_before = (kidx >= 0 && kidx == jidx - 1) ? sec[jidx] : slope(gk, vk, gj, vj);
            have_gb = true;
          }
          return grad_before;
        };
        bool drop = (vi < vj) && !sw;
        if (!drop && si < sj) drop = get_secant() < get_gb();
        double jg = nan, jp = nan, jv = nan;
        bool jf = false;
        if (sw) {
          jf = find_same_segment(g, p, v, n, gj, pj, idx, 1, thr, io.window, jg, jp, jv);
          if (!drop && jf) drop = (gi == jg) ? (vi < jv) : (get_secant() < slope(gi, vi, jg, jv));
        }
        if (drop && !node_crossing) continue;
        if (!sw) {
          emit(gj, pj, vj);
          gk = gj;
          pk = pj;
          vk = vj;
          kidx = jidx;
          gj = gi;
          pj = pi;
          vj = vi;
          sj = si;
          jidx = idx;
          continue;
        }
        const double sc = get_secant();
        const double gb = get_gb();
        double fg, fp, fv, bg, bp, bv;
        const bool ff = find_same_segment(g, p, v, n, gi, pi, idx, 1, thr, io.window, fg, fp, fv);
        const bool bf = find_same_segment(g, p, v, n, gi, pi, idx, -1, thr, io.window, bg, bp, bv);
        const bool found = ff || bf;
        const double pg = ff ? fg : bg, pp = ff ? fp : bp, pv = ff ? fv : bv;
        const double i_slope = slope(gi, vi, pg, pv);
        const double i_pslope = slope(gi, pi, pg, pp);
        const bool j_dom = found && (sc > i_slope) && !node_crossing;
        const double pslope_kj = slope(gk, pk, gj, pj);
        double k6g, k6v;
        intersect(gj, vj, gb, gi, vi, i_slope, k6g, k6v);
        const double k6pl = pj + pslope_kj * (k6g - gj);
        const double k6pr = pi + i_pslope * (k6g - gi);
        const bool kink6 = j_dom && (k6g > gk) && (k6g < gj) && (k6g < gi);
        const double j_slope = jf ? slope(gj, vj, jg, jv) : gb;
        const double j_pslope = jf ? slope(gj, pj, jg, jp) : pslope_kj;
        double k5g, k5v;
        intersect(gj, vj, j_slope, gi, vi, i_slope, k5g, k5v);
        const double k5pl = pj + j_pslope * (k5g - gj);
        const double k5pr = pi + i_pslope * (k5g - gi);
        const bool crossing = !j_dom && !node_crossing && found;
        const double tol = near * fmax(fmax(fabs(gj), fabs(gi)), 1.0);
        const bool on_j = crossing && fabs(k5g - gj) <= tol;
        const bool on_i = crossing && !on_j && fabs(k5g - gi) <= tol;
        const bool kink5 = crossing && !on_j && !on_i && (k5g > gj) && (k5g < gi);
        const bool plain = !j_dom && !kink5 && !on_j && !on_i;
        if (kink6) {
          emit(k6g, k6pl, k6v);
          emit(k6g, k6pr, k6v);
        } else if (plain || kink5 || on_j || on_i) {
          emit(gj, pj, vj);
          if (kink5) {
            emit(k5g, k5pl, k5v);
            emit(k5g, k5pr, k5v);
          } else if (on_j) {
            emit(gj, k5pr, k5v);
          } else if (on_i) {
            emit(gi, k5pl, k5v);
          }
        }
        const bool keeps_k = j_dom && !kink6;
        if (!keeps_k) {
          if (kink5) {
            gk = k5g; pk = k5pr; vk = k5v; kidx = -1;
          } else if (kink6) {
            gk = k6g; pk = k6pr; vk = k6v; kidx = -1;
          } else {
            gk = gj;
            pk = on_j ? k5pr : pj;
            vk = on_j ? k5v : vj;
            kidx = on_j ? -1 : jidx;
          }
        }
        gj = gi; pj = pi; vj = vi; sj = si;
        jidx = idx;
      }
      if (!isnan_(gj) && !isnan_(vj)) emit(gj, pj, vj);
      if (lane == 0) *io.nk = cnt;
    }
  }
}

// the dynamic shared-memory limit of both instantiations, set once per device
std::mutex g_attr_mu;
bool g_attr_done[64] = {};

int fues_smem_attr(std::string& err) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) {
    err = "fues: device ordinal >= 64";
    return LCMX_ERR_ARGS;
  }
  std::lock_guard<std::mutex> g(g_attr_mu);
  if (g_attr_done[dev]) return LCMX_OK;
  const int bytes = (int)fues_smem_bytes(kSmemMaxN);
  cudaError_t e = cudaFuncSetAttribute(fues_smem_kernel<FuesContig>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fues_smem_kernel<FuesItems>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) {
    err = std::string("fues: shared-memory attribute: ") + cudaGetErrorString(e);
    return LCMX_ERR_CUDA;
  }
  g_attr_done[dev] = true;
  return LCMX_OK;
}

int fues_grid(int rows) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return rows < sms * 16 ? rows : sms * 16;
}

}  // namespace

extern "C" size_t lcmx_fues_workspace_bytes(int n_rows, int n_in) {
  if (n_rows <= 0 || n_in <= 0) return 0;
  return (size_t)n_rows * 4 * (size_t)n_in * sizeof(double);
}

static int launch_fues(const double* grid, const double* policy, const double* value, const double* savings,
                       int n_rows, int n_in, double jump_thresh, int window, double* grid_out,
                       double* policy_out, double* value_out, int n_out, int* n_kept, double* work,
                       cudaStream_t stream, std::string& err) {
  if (window <= 0) window = n_in;  // exhaustive look-ahead
  if (n_in <= kSmemMaxN) {
    int rc = fues_smem_attr(err);
    if (rc) return rc;
    FuesContig rows{grid, policy, value, savings, grid_out, policy_out, value_out, n_kept,
                    n_rows, n_in, n_out, jump_thresh, window};
    fues_smem_kernel<FuesContig><<<fues_grid(n_rows), kBlock, fues_smem_bytes(n_in), stream>>>(rows);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string("fues launch: ") + cudaGetErrorString(e);
      return LCMX_ERR_LAUNCH;
    }
    return LCMX_OK;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid_n = n_rows < sms * 4 ? n_rows : sms * 4;
  fues_kernel<<<grid_n, kBlock, 0, stream>>>(grid, policy, value, savings, n_rows, n_in, jump_thresh, window,
                                             grid_out, policy_out, value_out, n_out, n_kept, work);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("fues launch: ") + cudaGetErrorString(e);
    return LCMX_ERR_LAUNCH;
  }
  return LCMX_OK;
}

int lcmx_set_error_from(lcmx_ctx* ctx, int code, const std::string& msg);

extern "C" int lcmx_fues_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                              const double* savings, int n_rows, int n_in, double jump_thresh,
                              int n_points_to_scan, double* grid_out, double* policy_out, double* value_out,
                              int n_out, int* n_kept, void* workspace, size_t workspace_bytes, void* stream) {
  if (!ctx || !grid || !policy || !value || !grid_out || !policy_out || !value_out || !n_kept || n_rows < 0 ||
      n_in < 1 || n_out < 1 || !(jump_thresh > 0.0))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan: bad arguments");
  if (n_in > kMaxSort)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan: rows longer than 8192 candidates");
  if (n_rows == 0) return LCMX_OK;
  if (!workspace || workspace_bytes < lcmx_fues_workspace_bytes(n_rows, n_in))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan: workspace too small");
  std::string err;
  int rc = launch_fues(grid, policy, value, savings, n_rows, n_in, jump_thresh, n_points_to_scan, grid_out,
                       policy_out, value_out, n_out, n_kept, static_cast<double*>(workspace), (cudaStream_t)stream,
                       err);
  if (rc) return lcmx_set_error_from(ctx, rc, err);
  return LCMX_OK;
}

// ---------------------------------------------------------------------------
// Variant that allocates nothing.
//
// Some callers cannot call cudaMalloc on this path: code running inside
// another runtime's execution -- for example an XLA FFI custom-call handler,
// which is how the reference runs its native kernels -- must not allocate
// there (cudaMalloc synchronises the device and bypasses the runtime's
// allocator).  For them lcmx_fues_scan_static takes its workspace from the
// file-scope device array below instead of a caller pointer.
//
// * Size: kStaticScratchBytes (8 MiB) per device, held by every GPU that
//   loads this library until the process exits.  A call needs
//   lcmx_fues_workspace_bytes(n_rows, n_in) <= 8 MiB, i.e. at most
//   262144 / n_in rows (129 rows of 2020 candidates); larger calls are
//   rejected with LCMX_ERR_ARGS.
// * Set-up: the first call on a device, with that device current, looks up
//   the array's device address with cudaGetSymbolAddress (in host code the
//   symbol is only a host-side stand-in, not a device address) and caches it
//   for that device.  Make that first call before any stream capture.  Each
//   call makes the context's device current for the lookup and the launch and
//   then restores the caller's current device.
// * Which rows touch the array: rows of up to 4096 candidates are staged in
//   shared memory and leave it unused; rows of 4097..8192 candidates go
//   through the global-workspace kernel, whose per-row sorted copy lives in
//   the array.
// * Sharing: every call uses the same array, which keeps the last call's
//   contents.  Nothing in it has to start at zero (each row's sorted copy is
//   written in full before it is read), but calls that overlap on the GPU
//   race on it: serialise them (one stream, or events).
namespace {
constexpr size_t kStaticScratchBytes = size_t(8) << 20;
__device__ __align__(256) double g_fues_static_scratch[kStaticScratchBytes / sizeof(double)];
std::mutex g_static_mu;
double* g_static_ptr[64] = {};
}  // namespace

int lcmx_ctx_device_of(const lcmx_ctx* ctx);

extern "C" int lcmx_fues_scan_static(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                                     const double* savings, int n_rows, int n_in, double jump_thresh,
                                     double* grid_out, double* policy_out, double* value_out, int n_out,
                                     int* n_kept, void* stream) {
  if (!ctx || !grid || !policy || !value || !grid_out || !policy_out || !value_out || !n_kept || n_rows < 0 ||
      n_in < 1 || n_out < 1 || !(jump_thresh > 0.0))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan_static: bad arguments");
  if (n_in > kMaxSort)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan_static: rows longer than 8192 candidates");
  const size_t need = lcmx_fues_workspace_bytes(n_rows, n_in);
  if (need > kStaticScratchBytes)
    return lcmx_set_error_from(
        ctx, LCMX_ERR_ARGS,
        "lcmx_fues_scan_static: " + std::to_string(n_rows) + " rows of " + std::to_string(n_in) +
            " candidates need " + std::to_string(need) + " bytes of scratch, more than the 8 MiB static array (at most " +
            std::to_string(kStaticScratchBytes / (4 * sizeof(double) * (size_t)n_in)) + " rows of this length)");
  if (n_rows == 0) return LCMX_OK;
  const int dev = lcmx_ctx_device_of(ctx);
  if (dev < 0 || dev >= 64) return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_scan_static: device ordinal >= 64");
  // The context's device is made current for the symbol lookup and the
  // launch; the caller's current device is put back before every return.
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return lcmx_set_error_from(ctx, LCMX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (prev != dev) {
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return lcmx_set_error_from(ctx, LCMX_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  }
  int rc = LCMX_OK;
  std::string err;
  double* work = nullptr;
  {
    std::lock_guard<std::mutex> g(g_static_mu);
    if (!g_static_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_fues_static_scratch);
      if (e != cudaSuccess || !p) {
        rc = LCMX_ERR_CUDA;
        err = std::string("cudaGetSymbolAddress(static FUES scratch): ") + cudaGetErrorString(e);
      } else {
        g_static_ptr[dev] = static_cast<double*>(p);
      }
    }
    work = g_static_ptr[dev];
  }
  if (rc == LCMX_OK)
    rc = launch_fues(grid, policy, value, savings, n_rows, n_in, jump_thresh, 0, grid_out, policy_out, value_out,
                     n_out, n_kept, work, (cudaStream_t)stream, err);
  if (prev != dev) cudaSetDevice(prev);
  if (rc) return lcmx_set_error_from(ctx, rc, err);
  return LCMX_OK;
}

// ---------------------------------------------------------------------------
// Item form: the rows of several candidate blocks (one per solve instance)
// in one launch; see FuesItems for the item words.
extern "C" int lcmx_fues_step(lcmx_ctx* ctx, const void* items, const int* tile_prefix, int n_items, int n_rows,
                              int max_n_in, void* stream) {
  if (!ctx || n_items < 0 || n_rows < 0 || (n_items > 0 && (!items || !tile_prefix)))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_fues_step: bad arguments");
  if (max_n_in < 1 || max_n_in > kSmemMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_fues_step: rows must hold 1.." + std::to_string(kSmemMaxN) + " candidates");
  if (n_items == 0 || n_rows == 0) return LCMX_OK;
  std::string err;
  int rc = fues_smem_attr(err);
  if (rc) return lcmx_set_error_from(ctx, rc, err);
  FuesItems rows{static_cast<const int64_t*>(items), tile_prefix, n_items, n_rows};
  fues_smem_kernel<FuesItems><<<fues_grid(n_rows), kBlock, fues_smem_bytes(max_n_in), (cudaStream_t)stream>>>(rows);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lcmx_set_error_from(ctx, LCMX_ERR_LAUNCH, std::string("lcmx_fues_step: ") + cudaGetErrorString(e));
  return LCMX_OK;
}
