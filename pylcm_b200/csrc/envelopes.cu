// envelopes.cu -- the LTM, RFC and MSS upper envelopes of DC-EGM candidate
// rows (kernel c, part 2, the alternatives to FUES; MSS is described at
// mss_kernel).
//
// LTM restates the local-upper-bound brute method the reference implements in
// src/_lcm/egm/upper_envelope/ltm.py:35-190: the queries are the live candidate
// grid points in ascending order (ties in input order); the segments join
// consecutive candidates in INPUT order; at each query the envelope is the
// largest linear interpolant over the segments that bracket it (a NaN
// interpolant wins, as a NaN-propagating maximum has it; the policy is that of
// the first segment reaching the maximum); queries without a bracketing
// segment, or with value -inf, are dropped.
//
// RFC restates the rooftop cut of src/_lcm/egm/upper_envelope/rfc.py:40-220:
// the candidates are sorted ascending (NaN last, ties in input order); a dead
// candidate (NaN grid point or value) enters with value -inf, grid point +inf
// and slope 0; candidate l is deleted when a j within `search_radius` sorted
// positions has l strictly below j's tangent line past a noise floor,
// v_l - v_j < mu_j (R_l - R_j) - 16 eps max(|v_l - v_j|, |mu_j (R_l - R_j)|),
// across a policy jump |dc/dR| > jump_thresh.
//
// All publish the survivors in sorted order, NaN-padded to n_out, with their
// count (n_kept > n_out: overflow, the row holds a truncated prefix).
//
// GPU mapping: one CTA per row, the row staged in shared memory and sorted by
// a bitonic sort of (monotone 64-bit grid image, input index) pairs.  The
// CTA then walks the sorted positions in rounds of one position per thread:
// each thread decides its position (LTM: a scan over every segment, all
// threads reading the same segment at once -- a shared-memory broadcast; RFC:
// 2 x search_radius neighbour tests), and a block-wide prefix sum of the
// survivors places them in the output.  Arithmetic that the reference rounds
// step by step is written with explicitly rounded operations (no contraction
// into fused multiply-adds), so the rows equal a step-by-step double
// evaluation.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/lcmx.h"

namespace {

constexpr int kEnvBlock = 256;
constexpr int kEnvMaxN = 4096;
constexpr int kEnvItemWords = 13;
constexpr int kLtm = 1;
constexpr int kRfc = 2;

__device__ __forceinline__ bool env_isnan(double x) { return x != x; }

struct EnvRow {
  const double* G;
  const double* P;
  const double* V;
  const double* M;  // marginal utility (RFC); unused by LTM
  double* GO;
  double* PO;
  double* VO;
  int* nk;
  int n_in;
  int n_out;
  double thr;
  int radius;
};

struct EnvContig {
  const double *grid, *policy, *value, *mu;
  double *go, *po, *vo;
  int* nk;
  int n_rows, n_in, n_out;
  double thr;
  int radius;
  __device__ __forceinline__ int count() const { return n_rows; }
  __device__ __forceinline__ EnvRow row(int r) const {
    EnvRow io;
    io.G = grid + (int64_t)r * n_in;
    io.P = policy + (int64_t)r * n_in;
    io.V = value + (int64_t)r * n_in;
    io.M = mu ? mu + (int64_t)r * n_in : nullptr;
    io.GO = go + (int64_t)r * n_out;
    io.PO = po + (int64_t)r * n_out;
    io.VO = vo + (int64_t)r * n_out;
    io.nk = nk + r;
    io.n_in = n_in;
    io.n_out = n_out;
    io.thr = thr;
    io.radius = radius;
    return io;
  }
};

// item words: 0 grid, 1 policy, 2 value, 3 marginal utility (RFC; 0: none),
// 4 grid_out, 5 policy_out, 6 value_out, 7 n_kept (int32), 8 n_rows, 9 n_in,
// 10 n_out, 11 jump_thresh (double bits), 12 search radius; one tile per row
struct EnvItems {
  const int64_t* items;
  const int* prefix;
  int n_items, n_tiles;
  __device__ __forceinline__ int count() const { return n_tiles; }
  __device__ __forceinline__ EnvRow row(int tile) const {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= tile) lo = mid; else hi = mid - 1;
    }
    const int64_t* it = items + (int64_t)lo * kEnvItemWords;
    const int r = tile - prefix[lo];
    EnvRow io;
    io.n_in = (int)it[9];
    io.n_out = (int)it[10];
    io.thr = __longlong_as_double(it[11]);
    io.radius = (int)it[12];
    io.G = reinterpret_cast<const double*>(it[0]) + (int64_t)r * io.n_in;
    io.P = reinterpret_cast<const double*>(it[1]) + (int64_t)r * io.n_in;
    io.V = reinterpret_cast<const double*>(it[2]) + (int64_t)r * io.n_in;
    io.M = it[3] ? reinterpret_cast<const double*>(it[3]) + (int64_t)r * io.n_in : nullptr;
    io.GO = reinterpret_cast<double*>(it[4]) + (int64_t)r * io.n_out;
    io.PO = reinterpret_cast<double*>(it[5]) + (int64_t)r * io.n_out;
    io.VO = reinterpret_cast<double*>(it[6]) + (int64_t)r * io.n_out;
    io.nk = reinterpret_cast<int*>(it[7]) + r;
    return io;
  }
};

__host__ __device__ constexpr int env_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

// shared memory of a row of n candidates: g, p, v, mu (n doubles each), then
// the sort's keys (np2 x 8 B, reused as a gather buffer) and indices (np2 x 4 B)
__host__ __device__ constexpr size_t env_smem_bytes(int n) {
  return (size_t)4 * n * sizeof(double) + (size_t)env_pow2(n) * (sizeof(unsigned long long) + sizeof(int));
}

// Monotone 64-bit image of a double for an ascending sort; -0 ranks with +0;
// NaN ranks just above +inf.
__device__ __forceinline__ unsigned long long env_key(double x) {
  if (env_isnan(x)) return 0xFFF0000000000001ULL;
  if (x == 0.0) x = 0.0;
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

// inclusive prefix sum of one int per thread over the CTA; `tot` gets the total
__device__ __forceinline__ int env_block_scan(int x, int* warp_sums, int& tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  int before = 0;
  tot = 0;
  for (int w = 0; w < kEnvBlock / 32; ++w) {
    const int s = warp_sums[w];
    if (w < warp) before += s;
    tot += s;
  }
  __syncthreads();  // warp_sums may be rewritten by the next call
  return x + before;
}

// bitonic sort of (key, index) pairs ascending, np2 a power of two; the
// caller synchronises before (the keys are written) and it synchronises after
__device__ __forceinline__ void env_sort(unsigned long long* key, int* idx, int np2) {
  for (int size = 2; size <= np2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < np2; t += kEnvBlock) {
        const int u = t ^ stride;
        if (u > t) {
          const unsigned long long ka = key[t], kb = key[u];
          const int ia = idx[t], ib = idx[u];
          const bool a_gt = ka > kb || (ka == kb && ia > ib);
          const bool up = (t & size) == 0;
          if (a_gt == up) {
            key[t] = kb;
            key[u] = ka;
            idx[t] = ib;
            idx[u] = ia;
          }
        }
      }
      __syncthreads();
    }
  }
}

template <class Rows, int KIND>
__global__ void __launch_bounds__(kEnvBlock) envelope_kernel(Rows rows) {
  extern __shared__ __align__(16) unsigned char env_smem[];
  __shared__ int warp_sums[kEnvBlock / 32];
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  const int total = rows.count();
  for (int row = blockIdx.x; row < total; row += gridDim.x) {
    const EnvRow io = rows.row(row);
    const int n = io.n_in;
    const int np2 = env_pow2(n);
    double* g = reinterpret_cast<double*>(env_smem);
    double* p = g + n;
    double* v = p + n;
    double* m = v + n;
    unsigned long long* key = reinterpret_cast<unsigned long long*>(m + n);
    int* idx = reinterpret_cast<int*>(key + np2);
    __syncthreads();  // the previous row is done with shared memory
    for (int t = threadIdx.x; t < n; t += kEnvBlock) {
      g[t] = io.G[t];
      p[t] = io.P[t];
      v[t] = io.V[t];
      m[t] = (KIND == kRfc && io.M) ? io.M[t] : 0.0;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < np2; t += kEnvBlock) {
      idx[t] = t;
      if (t >= n) {
        key[t] = ~0ULL;  // padding sorts last
      } else if (KIND == kLtm) {
        key[t] = (env_isnan(g[t]) || env_isnan(v[t])) ? env_key(inf) : env_key(g[t]);
      } else {
        key[t] = env_key(g[t]);
      }
    }
    __syncthreads();
    env_sort(key, idx, np2);
    if (KIND == kRfc) {
      // rows in sorted order, through the key buffer (no longer needed)
      double* tmp = reinterpret_cast<double*>(key);
      double* arrs[4] = {g, p, v, m};
      for (int a = 0; a < 4; ++a) {
        for (int t = threadIdx.x; t < n; t += kEnvBlock) tmp[t] = arrs[a][idx[t]];
        __syncthreads();
        for (int t = threadIdx.x; t < n; t += kEnvBlock) arrs[a][t] = tmp[t];
        __syncthreads();
      }
    }
    // decide the sorted positions round by round; survivors go out in order
    int base = 0;
    for (int r0 = 0; r0 < n; r0 += kEnvBlock) {
      const int t = r0 + (int)threadIdx.x;
      bool keep = false;
      double og = nan, op = nan, ov = nan;
      if (t < n) {
        if (KIND == kLtm) {
          const int i = idx[t];
          const double q = g[i];
          if (!(env_isnan(q) || env_isnan(v[i]))) {
            bool found = false;
            double bv = -inf, bp = nan;
            double gl = g[0];
            for (int k = 0; k + 1 < n; ++k) {
              const double gr = g[k + 1];
              const bool br = (gl <= gr) ? (gl <= q && q <= gr) : (gr <= q && q <= gl);
              if (br) {
                const double vl = v[k], vr = v[k + 1];
                if (!(env_isnan(vl) || env_isnan(vr))) {
                  const double w = __dsub_rn(gr, gl);
                  const double rel = (w == 0.0) ? 0.0 : __ddiv_rn(__dsub_rn(q, gl), w);
                  const double vi = __dadd_rn(vl, __dmul_rn(rel, __dsub_rn(vr, vl)));
                  const double pl = p[k], pr = p[k + 1];
                  const double pi = __dadd_rn(pl, __dmul_rn(rel, __dsub_rn(pr, pl)));
                  if (!found) {
                    bv = vi;
                    bp = pi;
                    found = true;
                  } else if (!env_isnan(bv) && (env_isnan(vi) || vi > bv)) {
                    bv = vi;
                    bp = pi;
                  }
                }
              }
              gl = gr;
            }
            if (found && !(bv == -inf)) {
              keep = true;
              og = q;
              op = bp;
              ov = bv;
            }
          }
        } else {
          const double gl_ = g[t], vl_ = v[t];
          const bool dead_l = env_isnan(gl_) || env_isnan(vl_);
          if (!dead_l) {
            const double thr = io.thr;
            const double eps16 = 16.0 * 2.220446049250313e-16;
            bool deleted = false;
            const int j0 = max(0, t - io.radius), j1 = min(n - 1, t + io.radius);
            for (int j = j0; j <= j1 && !deleted; ++j) {
              if (j == t) continue;
              const bool dead_j = env_isnan(g[j]) || env_isnan(v[j]);
              const double gj = dead_j ? inf : g[j];
              const double vj = dead_j ? -inf : v[j];
              const double mj = dead_j ? 0.0 : m[j];
              const double dg = __dsub_rn(gl_, gj);
              const double gap = __dsub_rn(vl_, vj);
              const double tan = __dmul_rn(mj, dg);
              const double ag = fabs(gap), at = fabs(tan);
              const double mx = (env_isnan(ag) || env_isnan(at)) ? nan : (ag > at ? ag : at);
              const double floor_ = __dmul_rn(eps16, mx);
              const bool below = gap < __dsub_rn(tan, floor_);
              const double slope = (dg == 0.0) ? 0.0 : __ddiv_rn(__dsub_rn(p[t], p[j]), dg);
              if (below && fabs(slope) > thr) deleted = true;
            }
            if (!deleted) {
              keep = true;
              og = gl_;
              op = p[t];
              ov = vl_;
            }
          }
        }
      }
      int tot = 0;
      const int incl = env_block_scan(keep ? 1 : 0, warp_sums, tot);
      if (keep) {
        const int pos = base + incl - 1;
        if (pos < io.n_out) {
          io.GO[pos] = og;
          io.PO[pos] = op;
          io.VO[pos] = ov;
        }
      }
      base += tot;
    }
    for (int t = base + (int)threadIdx.x; t < io.n_out; t += kEnvBlock) {
      io.GO[t] = nan;
      io.PO[t] = nan;
      io.VO[t] = nan;
    }
    if (threadIdx.x == 0) *io.nk = base;
  }
}

// ---------------------------------------------------------------------------
// MSS (HARK's EGM upper envelope), src/_lcm/egm/upper_envelope/mss.py:72-629:
// the links join consecutive candidates in input order; a link across a grid
// decrease, or a value decrease past 16 eps max(|v_k|, |v_k+1|), starts a new
// branch and is not live (HARK's monotone split).  At each live abscissa
// (ascending) the envelope is the largest finite interpolant over the live
// bracketing links; the winner is the first link within 16 eps max(1, |max|)
// of it.  Where the winning branch changes between two consecutive live
// queries, the crossing of the two winning links' value lines is inserted
// twice (left, then right policy) when it falls strictly between them and the
// envelope there matches it (finite, within 1e-7 + 1e-5 |value|).
constexpr int kMss = 3;

// extra shared memory of MSS: the winning branch per query (n ints)
__host__ __device__ constexpr size_t mss_smem_bytes(int n) { return env_smem_bytes(n) + (size_t)4 * n; }

// value at q of the live link k: vi (rounded step by step), and whether it brackets q
__device__ __forceinline__ bool mss_link_at(const double* g, const double* v, const int* lseg, int k, double q,
                                            double& vi, double& rel) {
  if (lseg[k] < 0) return false;
  const double gl = g[k], gr = g[k + 1];
  const bool br = (gl <= gr) ? (gl <= q && q <= gr) : (gr <= q && q <= gl);
  if (!br) return false;
  const double w = __dsub_rn(gr, gl);
  rel = (w == 0.0) ? 0.0 : __ddiv_rn(__dsub_rn(q, gl), w);
  vi = __dadd_rn(v[k], __dmul_rn(rel, __dsub_rn(v[k + 1], v[k])));
  return true;
}

// envelope value at q (-inf: no finite bracketing interpolant); `link` the
// winner (first link within the tie band), -1 when no live link brackets q
__device__ double mss_eval(const double* g, const double* v, const int* lseg, int n, double q, int& link) {
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  double env = -inf;
  bool any = false;
  for (int k = 0; k + 1 < n; ++k) {
    double vi, rel;
    if (mss_link_at(g, v, lseg, k, q, vi, rel)) {
      any = true;
      if (isfinite(vi) && vi > env) env = vi;
    }
  }
  link = -1;
  if (!any) return env;
  const double floor_ = __dmul_rn(16.0 * 2.220446049250313e-16, fmax(1.0, fabs(env)));
  const double lo = __dsub_rn(env, floor_);
  for (int k = 0; k + 1 < n; ++k) {
    double vi, rel;
    if (mss_link_at(g, v, lseg, k, q, vi, rel)) {
      const double mv = isfinite(vi) ? vi : -inf;
      if (mv >= lo) {
        link = k;
        break;
      }
    }
  }
  return env;
}

__device__ __forceinline__ double mss_slope(double xa, double ya, double xb, double yb) {
  const double dx = __dsub_rn(xb, xa);
  return dx == 0.0 ? 0.0 : __ddiv_rn(__dsub_rn(yb, ya), dx);
}

template <class Rows>
__global__ void __launch_bounds__(kEnvBlock) mss_kernel(Rows rows) {
  extern __shared__ __align__(16) unsigned char env_smem[];
  __shared__ int warp_sums[kEnvBlock / 32];
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  const double eps16 = 16.0 * 2.220446049250313e-16;
  const int total = rows.count();
  for (int row = blockIdx.x; row < total; row += gridDim.x) {
    const EnvRow io = rows.row(row);
    const int n = io.n_in;
    const int np2 = env_pow2(n);
    double* g = reinterpret_cast<double*>(env_smem);
    double* p = g + n;
    double* v = p + n;
    int* lseg = reinterpret_cast<int*>(v + n);  // branch id of each live link, -1: not live
    int* wl = lseg + n;                         // winning link per sorted query, -1: dropped
    unsigned long long* key = reinterpret_cast<unsigned long long*>(v + 2 * n);
    double* ev = reinterpret_cast<double*>(key);  // envelope value per sorted query (after the sort)
    int* idx = reinterpret_cast<int*>(key + np2);
    int* ws = idx + np2;                          // winning branch per sorted query
    __syncthreads();  // the previous row is done with shared memory
    for (int t = threadIdx.x; t < n; t += kEnvBlock) {
      g[t] = io.G[t];
      p[t] = io.P[t];
      v[t] = io.V[t];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < np2; t += kEnvBlock) {
      idx[t] = t;
      key[t] = t >= n ? ~0ULL : ((env_isnan(g[t]) || env_isnan(v[t])) ? env_key(inf) : env_key(g[t]));
    }
    __syncthreads();
    env_sort(key, idx, np2);
    // links: branch ids (a running count of decreases) and liveness
    int base = 0;
    for (int k0 = 0; k0 < n - 1; k0 += kEnvBlock) {
      const int k = k0 + (int)threadIdx.x;
      bool dec = false, live = false;
      if (k < n - 1) {
        const double vl = v[k], vr = v[k + 1];
        const double al = fabs(vl), ar = fabs(vr);
        const double mx = (env_isnan(al) || env_isnan(ar)) ? nan : (al > ar ? al : ar);
        dec = (g[k + 1] < g[k]) || (vr < __dsub_rn(vl, __dmul_rn(eps16, mx)));
        const bool dead = env_isnan(g[k]) || env_isnan(vl) || env_isnan(g[k + 1]) || env_isnan(vr);
        live = !dead && !dec;
      }
      int tot = 0;
      const int incl = env_block_scan(dec ? 1 : 0, warp_sums, tot);
      if (k < n - 1) lseg[k] = live ? base + incl : -1;
      base += tot;
    }
    __syncthreads();
    // the envelope at every sorted query
    for (int t = threadIdx.x; t < n; t += kEnvBlock) {
      const int i = idx[t];
      int link = -1;
      double e = -inf;
      if (!(env_isnan(g[i]) || env_isnan(v[i]))) e = mss_eval(g, v, lseg, n, g[i], link);
      const bool node = link >= 0 && !(e == -inf);
      ev[t] = e;
      wl[t] = node ? link : -1;
      ws[t] = node ? lseg[link] : -1;
    }
    __syncthreads();
    // emission: per query the crossing (twice) before it, then its node
    int out = 0;
    for (int r0 = 0; r0 < n; r0 += kEnvBlock) {
      const int t = r0 + (int)threadIdx.x;
      bool node = false, cross = false;
      double q = nan, x = nan, y = nan, pa = nan, pb = nan, pol = nan;
      if (t < n && wl[t] >= 0) {
        node = true;
        const int b = wl[t];
        q = g[idx[t]];
        {
          const double w = __dsub_rn(g[b + 1], g[b]);
          const double rel = (w == 0.0) ? 0.0 : __ddiv_rn(__dsub_rn(q, g[b]), w);
          pol = __dadd_rn(p[b], __dmul_rn(rel, __dsub_rn(p[b + 1], p[b])));
        }
        int pr = t - 1;
        while (pr >= 0 && wl[pr] < 0) --pr;
        if (pr >= 0 && ws[pr] != ws[t]) {
          const int a = wl[pr];
          const double qp = g[idx[pr]];
          const double sa = mss_slope(g[a], v[a], g[a + 1], v[a + 1]);
          const double sb = mss_slope(g[b], v[b], g[b + 1], v[b + 1]);
          const double den = __dsub_rn(sa, sb);
          if (den != 0.0) {
            x = __ddiv_rn(__dsub_rn(__dadd_rn(__dsub_rn(v[b], v[a]), __dmul_rn(sa, g[a])), __dmul_rn(sb, g[b])), den);
            y = __dadd_rn(v[a], __dmul_rn(sa, __dsub_rn(x, g[a])));
            const double psa = mss_slope(g[a], p[a], g[a + 1], p[a + 1]);
            const double psb = mss_slope(g[b], p[b], g[b + 1], p[b + 1]);
            pa = __dadd_rn(p[a], __dmul_rn(psa, __dsub_rn(x, g[a])));
            pb = __dadd_rn(p[b], __dmul_rn(psb, __dsub_rn(x, g[b])));
            if (x > qp && x < q) {
              int lk;
              const double ce = mss_eval(g, v, lseg, n, x, lk);
              cross = isfinite(ce) && isfinite(y) &&
                      fabs(__dsub_rn(ce, y)) <= __dadd_rn(1e-7, __dmul_rn(1e-5, fabs(y)));
            }
          }
        }
      }
      const int nrow = (cross ? 2 : 0) + (node ? 1 : 0);
      int tot = 0;
      const int incl = env_block_scan(nrow, warp_sums, tot);
      int pos = out + incl - nrow;
      if (cross) {
        if (pos < io.n_out) { io.GO[pos] = x; io.PO[pos] = pa; io.VO[pos] = y; }
        ++pos;
        if (pos < io.n_out) { io.GO[pos] = x; io.PO[pos] = pb; io.VO[pos] = y; }
        ++pos;
      }
      if (node && pos < io.n_out) {
        io.GO[pos] = q;
        io.PO[pos] = pol;
        io.VO[pos] = ev[t];
      }
      out += tot;
    }
    for (int t = out + (int)threadIdx.x; t < io.n_out; t += kEnvBlock) {
      io.GO[t] = nan;
      io.PO[t] = nan;
      io.VO[t] = nan;
    }
    if (threadIdx.x == 0) *io.nk = out;
  }
}

template <class Rows>
int mss_launch(const Rows& rows, int n_tiles, int max_n, cudaStream_t stream, std::string& err) {
  cudaError_t e = cudaFuncSetAttribute(mss_kernel<Rows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)mss_smem_bytes(kEnvMaxN));
  if (e != cudaSuccess) {
    err = std::string("MSS kernel attribute: ") + cudaGetErrorString(e);
    return LCMX_ERR_LAUNCH;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = n_tiles < sms * 8 ? n_tiles : sms * 8;
  mss_kernel<Rows><<<grid, kEnvBlock, mss_smem_bytes(max_n), stream>>>(rows);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("MSS launch: ") + cudaGetErrorString(e);
    return LCMX_ERR_LAUNCH;
  }
  return LCMX_OK;
}

template <class Rows, int KIND>
int env_attr(std::string& err) {
  const cudaError_t e = cudaFuncSetAttribute(envelope_kernel<Rows, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)env_smem_bytes(kEnvMaxN));
  if (e != cudaSuccess) {
    err = std::string("envelope kernel attribute: ") + cudaGetErrorString(e);
    return LCMX_ERR_LAUNCH;
  }
  return LCMX_OK;
}

int env_grid(int rows) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return rows < sms * 8 ? rows : sms * 8;
}

template <class Rows, int KIND>
int env_launch(const Rows& rows, int n_tiles, int max_n, cudaStream_t stream, std::string& err) {
  int rc = env_attr<Rows, KIND>(err);
  if (rc) return rc;
  envelope_kernel<Rows, KIND><<<env_grid(n_tiles), kEnvBlock, env_smem_bytes(max_n), stream>>>(rows);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("envelope launch: ") + cudaGetErrorString(e);
    return LCMX_ERR_LAUNCH;
  }
  return LCMX_OK;
}

}  // namespace

int lcmx_set_error_from(lcmx_ctx* ctx, int code, const std::string& msg);

extern "C" int lcmx_ltm_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                             int n_rows, int n_in, double* grid_out, double* policy_out, double* value_out,
                             int n_out, int* n_kept, void* stream) {
  if (!ctx || !grid || !policy || !value || !grid_out || !policy_out || !value_out || !n_kept || n_rows < 0 ||
      n_in < 1 || n_out < 1)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_ltm_scan: bad arguments");
  if (n_in > kEnvMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_ltm_scan: rows longer than " + std::to_string(kEnvMaxN) + " candidates");
  if (n_rows == 0) return LCMX_OK;
  EnvContig rows{grid, policy, value, nullptr, grid_out, policy_out, value_out, n_kept, n_rows, n_in, n_out, 0.0, 0};
  std::string err;
  const int rc = env_launch<EnvContig, kLtm>(rows, n_rows, n_in, (cudaStream_t)stream, err);
  return rc ? lcmx_set_error_from(ctx, rc, err) : LCMX_OK;
}

extern "C" int lcmx_rfc_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                             const double* marginal_utility, int n_rows, int n_in, int search_radius,
                             double jump_thresh, double* grid_out, double* policy_out, double* value_out,
                             int n_out, int* n_kept, void* stream) {
  if (!ctx || !grid || !policy || !value || !marginal_utility || !grid_out || !policy_out || !value_out ||
      !n_kept || n_rows < 0 || n_in < 1 || n_out < 1 || search_radius < 1 || !(jump_thresh > 0.0))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_rfc_scan: bad arguments");
  if (n_in > kEnvMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_rfc_scan: rows longer than " + std::to_string(kEnvMaxN) + " candidates");
  if (n_rows == 0) return LCMX_OK;
  EnvContig rows{grid, policy, value, marginal_utility, grid_out, policy_out, value_out, n_kept,
                 n_rows, n_in, n_out, jump_thresh, search_radius};
  std::string err;
  const int rc = env_launch<EnvContig, kRfc>(rows, n_rows, n_in, (cudaStream_t)stream, err);
  return rc ? lcmx_set_error_from(ctx, rc, err) : LCMX_OK;
}

extern "C" int lcmx_mss_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                             int n_rows, int n_in, double* grid_out, double* policy_out, double* value_out,
                             int n_out, int* n_kept, void* stream) {
  if (!ctx || !grid || !policy || !value || !grid_out || !policy_out || !value_out || !n_kept || n_rows < 0 ||
      n_in < 1 || n_out < 1)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_mss_scan: bad arguments");
  if (n_in > kEnvMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_mss_scan: rows longer than " + std::to_string(kEnvMaxN) + " candidates");
  if (n_rows == 0) return LCMX_OK;
  EnvContig rows{grid, policy, value, nullptr, grid_out, policy_out, value_out, n_kept, n_rows, n_in, n_out, 0.0, 0};
  std::string err;
  const int rc = mss_launch<EnvContig>(rows, n_rows, n_in, (cudaStream_t)stream, err);
  return rc ? lcmx_set_error_from(ctx, rc, err) : LCMX_OK;
}

extern "C" int lcmx_envelope_step(lcmx_ctx* ctx, int kind, const void* items, const int* tile_prefix, int n_items,
                                  int n_rows, int max_n_in, void* stream) {
  if (!ctx || (kind != kLtm && kind != kRfc && kind != kMss) || n_items < 0 || n_rows < 0 ||
      (n_items > 0 && (!items || !tile_prefix)))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_envelope_step: bad arguments");
  if (max_n_in < 1 || max_n_in > kEnvMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_envelope_step: rows must hold 1.." + std::to_string(kEnvMaxN) + " candidates");
  if (n_items == 0 || n_rows == 0) return LCMX_OK;
  EnvItems rows{static_cast<const int64_t*>(items), tile_prefix, n_items, n_rows};
  std::string err;
  const int rc = kind == kLtm   ? env_launch<EnvItems, kLtm>(rows, n_rows, max_n_in, (cudaStream_t)stream, err)
                 : kind == kRfc ? env_launch<EnvItems, kRfc>(rows, n_rows, max_n_in, (cudaStream_t)stream, err)
                                : mss_launch<EnvItems>(rows, n_rows, max_n_in, (cudaStream_t)stream, err);
  return rc ? lcmx_set_error_from(ctx, rc, err) : LCMX_OK;
}
