// lcm_device.cuh -- hand-written device helpers shared by every generated
// module (Bellman step, expectation contraction, simulation, DC-EGM).
//
// This header is prepended to the CUDA C that the Python code generator emits
// for one model regime and the whole translation unit is compiled by NVRTC for
// sm_100a.  It must stay free of host code and of any #include (NVRTC builds
// it without the CUDA toolkit headers).
//
// Semantics follow the reference solve path:
//   * zero-safe weighted term: w * v, with w == 0 annihilating +-inf / nan
//     (src/_lcm/zero_safe.py:161-251);
//   * linear interpolation with extrapolation, lower index clipped to
//     [0, n-2] (src/_lcm/regime_building/ndimage.py:29-109);
//   * grid coordinates for lin / log / irregular grids
//     (src/_lcm/grids/coordinates.py:30-167);
//   * argmax = first flat action index attaining the maximum over feasible
//     actions, max initialised at -inf (max_Q_over_a.py:160, argmax.py:6-69).

#pragma once

typedef long long i64;
typedef unsigned long long u64;
typedef unsigned int u32;

#define LCM_INF (__longlong_as_double(0x7ff0000000000000LL))
#define LCM_NAN (__longlong_as_double(0x7ff8000000000000LL))

template <typename T> struct lcm_lim;
template <> struct lcm_lim<double> {
  static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000LL); }
  static __device__ __forceinline__ double nan() { return __longlong_as_double(0x7ff8000000000000LL); }
};
template <> struct lcm_lim<float> {
  static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
  static __device__ __forceinline__ float nan() { return __int_as_float(0x7fc00000); }
};

__device__ __forceinline__ bool lcm_isfinite(double x) {
  return (__double_as_longlong(x) & 0x7ff0000000000000LL) != 0x7ff0000000000000LL;
}
__device__ __forceinline__ bool lcm_isfinite(float x) {
  return (__float_as_int(x) & 0x7f800000) != 0x7f800000;
}
__device__ __forceinline__ bool lcm_isnan(double x) { return x != x; }
__device__ __forceinline__ bool lcm_isnan(float x) { return x != x; }

// item-record word accessors (records are arrays of 64-bit words)
__device__ __forceinline__ double lcm_wd(const i64* it, int k) { return __longlong_as_double(it[k]); }
__device__ __forceinline__ int lcm_wi(const i64* it, int k) { return (int)it[k]; }
template <typename P> __device__ __forceinline__ P* lcm_wp(const i64* it, int k) {
  return reinterpret_cast<P*>(it[k]);
}

// w * v, exactly 0 where w == 0 whatever v is (zero_safe_weighted_term).
template <typename T> __device__ __forceinline__ T lcm_zs(T w, T v) {
  return (w == T(0) && !lcm_isfinite(v)) ? T(0) : w * v;
}

// Lower bracket of a fractional coordinate, clip(floor(c), 0, n-2), as an
// int and as a float.  The coordinate is clamped to [0, n-2] first (fmin/fmax
// send NaN to 0); floor of a value in [0, 2^23) is then a round-down add of
// 2^23, whose low mantissa bits are the integer -- no conversion instruction.
// Valid for grids of fewer than 2^23 points.
__device__ __forceinline__ int lcm_lower(float c, int n, float& lof) {
  float cc = fminf(fmaxf(c, 0.0f), (float)(n - 2));
  float m = __fadd_rd(cc, 8388608.0f);
  lof = m - 8388608.0f;
  return __float_as_int(m) - 0x4B000000;
}
__device__ __forceinline__ int lcm_lower(double c, int n, double& lof) {
  double cc = fmin(fmax(c, 0.0), (double)(n - 2));
  double m = __dadd_rd(cc, 4503599627370496.0);
  lof = m - 4503599627370496.0;
  return (int)(__double_as_longlong(m) - 0x4330000000000000LL);
}

// Coordinate of x on a linearly spaced grid: (x - start) / step, computed as
// a multiply by the host-supplied reciprocal of the step.
template <typename T> __device__ __forceinline__ T lcm_coord_lin(T x, T start, T inv_step) {
  return (x - start) * inv_step;
}

// Coordinate on a log-spaced grid (coordinates.py:73-114): rank in log space,
// then the linear position between the two bracketing grid points.
template <typename T>
__device__ __forceinline__ T lcm_coord_log(T x, T log_start, T log_step) {
  T lv = log(x);
  T c = (lv - log_start) / log_step;
  T lo = floor(c);
  T lower = exp(log_start + log_step * lo);
  T upper = exp(log_start + log_step * (lo + T(1)));
  return lo + (x - lower) / (upper - lower);
}

// Coordinate on an irregular ascending grid (coordinates.py:117-167):
// searchsorted(side="right") clipped to [1, n-1], then linear position.
template <typename T>
__device__ __forceinline__ T lcm_coord_irreg(T x, const double* __restrict__ pts, int n) {
  if (n == 1) return T(0);
  int lo = 0, hi = n;  // first index with pts[i] > x
  double xd = (double)x;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (pts[mid] > xd) hi = mid; else lo = mid + 1;
  }
  int up = lo < 1 ? 1 : (lo > n - 1 ? n - 1 : lo);
  int low = up - 1;
  T pl = (T)pts[low], pu = (T)pts[up];
  return (T)low + (x - pl) / (pu - pl);
}

// Coordinate on a piecewise grid of k segments (piecewise.py:107-118,
// 178-188): the segment is the count of breakpoints (effective starts of
// segments 1..k-1) at or below x; inside it the linear or logarithmic
// coordinate, plus the segment's offset.  tab = [breakpoints (k-1) | start
// (k) | scale (k) | offset (k)], start/scale as lcm_coord_lin's or
// lcm_coord_log's arguments.
template <typename T>
__device__ __forceinline__ T lcm_coord_piece(T x, const double* __restrict__ tab, int k, int is_log) {
  int seg = 0;
  for (int i = 0; i < k - 1; ++i) seg += ((double)x >= tab[i]) ? 1 : 0;
  const double* st = tab + (k - 1);
  const T local = is_log ? lcm_coord_log<T>(x, (T)st[seg], (T)st[k + seg])
                         : lcm_coord_lin<T>(x, (T)st[seg], (T)st[k + seg]);
  return (T)st[2 * k + seg] + local;
}

// 1-D linear read with extrapolation; `row` is contiguous.
template <typename T, typename S>
__device__ __forceinline__ T lcm_interp1(const S* __restrict__ row, int n, T c) {
  T lof;
  int lo = lcm_lower(c, n, lof);
  T wu = c - lof;
  T wl = T(1) - wu;
  T v0 = (T)__ldg(row + lo);
  T v1 = (T)__ldg(row + lo + 1);
  // a finite result implies finite corners; otherwise redo it zero-safely
  T r = wl * v0 + wu * v1;
  if (lcm_isfinite(r)) return r;
  return lcm_zs(wl, v0) + lcm_zs(wu, v1);
}

// 1-D linear read of a float row in shared memory (the collapsed rows of the
// single-precision search), with lcm_interp1's extrapolation and zero-safe
// fallback.
template <typename T>
__device__ __forceinline__ T lcm_interp1s(const float* row, int n, T c) {
  T lof;
  int lo = lcm_lower(c, n, lof);
  T wu = c - lof;
  T wl = T(1) - wu;
  T v0 = (T)row[lo];
  T v1 = (T)row[lo + 1];
  T r = wl * v0 + wu * v1;
  if (lcm_isfinite(r)) return r;
  return lcm_zs(wl, v0) + lcm_zs(wu, v1);
}

// 2-D bilinear read; `blk` is an (n0 x n1) row-major block.  Corner order and
// left-to-right summation follow map_coordinates (ndimage.py:71-97).
template <typename T, typename S>
__device__ __forceinline__ T lcm_interp2(const S* __restrict__ blk, int n0, int n1, T c0, T c1) {
  T f0, f1;
  int l0 = lcm_lower(c0, n0, f0), l1 = lcm_lower(c1, n1, f1);
  T u0 = c0 - f0, u1 = c1 - f1;
  T d0 = T(1) - u0, d1 = T(1) - u1;
  const S* r0 = blk + (i64)l0 * n1;
  const S* r1 = r0 + n1;
  const T a = (T)__ldg(r0 + l1), b = (T)__ldg(r0 + l1 + 1), c = (T)__ldg(r1 + l1), d = (T)__ldg(r1 + l1 + 1);
  T r = d0 * d1 * a + d0 * u1 * b + u0 * d1 * c + u0 * u1 * d;
  if (lcm_isfinite(r)) return r;
  T acc = lcm_zs(d0 * d1, a);
  acc = acc + lcm_zs(d0 * u1, b);
  acc = acc + lcm_zs(u0 * d1, c);
  acc = acc + lcm_zs(u0 * u1, d);
  return acc;
}

// Block statistics of a float expectation row, for the exact skipping of
// action groups in the single-precision search: over 16 consecutive columns
// (16 consecutive threads of a warp), the maximum -- NaN when any value is NaN
// -- and the largest |value| among the finite values.  Lanes without a column
// pass -inf.  Every lane of the warp must call it.
__device__ __forceinline__ float lcm_nanmax(float a, float b) {
  return (a != a) ? a : ((b != b || b > a) ? b : a);
}
__device__ __forceinline__ float2 lcm_block16_stats(float x) {
  float mx = x, ab = lcm_isfinite(x) ? fabsf(x) : 0.0f;
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    const float omx = __shfl_xor_sync(0xffffffffu, mx, o);
    const float oab = __shfl_xor_sync(0xffffffffu, ab, o);
    mx = lcm_nanmax(mx, omx);
    ab = fmaxf(ab, oab);
  }
  return make_float2(mx, ab);
}

// Running (max, first argmax, nan) over feasible actions.
template <typename T> struct LcmBest {
  T v;
  int idx;   // -1: no feasible action seen yet
  int nan;   // 0, or 1 + the smallest index of a feasible action whose Q is NaN
  __device__ __forceinline__ void init() { v = -lcm_lim<T>::inf(); idx = -1; nan = 0; }
  __device__ __forceinline__ void push(T q, int a) {
    if (q != q) { if (!nan) nan = a + 1; return; }
    if (idx < 0 || q > v) { v = q; idx = a; }
  }
  // merge with another partial result over a disjoint action set; ties go to
  // the smaller flat index, so the result equals the sequential first argmax.
  __device__ __forceinline__ void merge(T ov, int oidx, int onan) {
    nan = (nan == 0) ? onan : ((onan == 0 || nan < onan) ? nan : onan);
    if (oidx < 0) return;
    if (idx < 0 || ov > v || (ov == v && oidx < idx)) { v = ov; idx = oidx; }
  }
};

// Running top-2 (value, index) over feasible actions.  The single-precision
// search keeps two candidates so that a near-tie which float rounding may
// misorder is re-ranked in double precision afterwards.
template <typename T> struct LcmBest2 {
  T v, v2;
  int idx, idx2;
  int nan;
  __device__ __forceinline__ void init() {
    v = v2 = -lcm_lim<T>::inf(); idx = idx2 = -1; nan = 0;
  }
  __device__ __forceinline__ static bool better(T a, int ia, T b, int ib) {
    // does (a, ia) rank above (b, ib)?  ties -> smaller index
    if (ia < 0) return false;
    if (ib < 0) return true;
    return a > b || (a == b && ia < ib);
  }
  __device__ __forceinline__ void add(T q, int a) {
    if (better(q, a, v, idx)) { v2 = v; idx2 = idx; v = q; idx = a; }
    else if (a != idx && better(q, a, v2, idx2)) { v2 = q; idx2 = a; }
  }
  // sequential scan within one lane: indices arrive in increasing order, so a
  // tie never displaces an earlier candidate
  __device__ __forceinline__ void push(T q, int a) {
    if (q != q) { nan = 1; return; }
    if (q > v2 || idx2 < 0) {
      if (q > v || idx < 0) { v2 = v; idx2 = idx; v = q; idx = a; }
      else { v2 = q; idx2 = a; }
    }
  }
  __device__ __forceinline__ void merge(T ov, int oi, T ov2, int oi2, int onan) {
    nan |= onan;
    if (oi >= 0) add(ov, oi);
    if (oi2 >= 0) add(ov2, oi2);
  }
};

template <int LANES, typename T>
__device__ __forceinline__ void lcm_group_reduce2(LcmBest2<T>& b) {
#pragma unroll
  for (int off = LANES >> 1; off > 0; off >>= 1) {
    T ov = __shfl_xor_sync(0xffffffffu, b.v, off);
    int oi = __shfl_xor_sync(0xffffffffu, b.idx, off);
    T ov2 = __shfl_xor_sync(0xffffffffu, b.v2, off);
    int oi2 = __shfl_xor_sync(0xffffffffu, b.idx2, off);
    int on = __shfl_xor_sync(0xffffffffu, b.nan, off);
    b.merge(ov, oi, ov2, oi2, on);
  }
}

// Combine LANES consecutive lanes (a power of two <= 32) holding partial
// results for the same state, with warp shuffles.
template <int LANES, typename T>
__device__ __forceinline__ void lcm_group_reduce(LcmBest<T>& b) {
#pragma unroll
  for (int off = LANES >> 1; off > 0; off >>= 1) {
    T ov = __shfl_xor_sync(0xffffffffu, b.v, off);
    int oi = __shfl_xor_sync(0xffffffffu, b.idx, off);
    int on = __shfl_xor_sync(0xffffffffu, b.nan, off);
    b.merge(ov, oi, on);
  }
}

// Tile -> item lookup: prefix[i] is the first tile of item i, prefix[n] = total.
__device__ __forceinline__ int lcm_find_item(const int* __restrict__ prefix, int n_items, int tile) {
  int lo = 0, hi = n_items - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Tile statistics of float expectation rows over two continuous axes, for the
// exact skipping of action groups in the single-precision search.  Each row k
// is an (n1 x n2) row-major block; per tile of 16 (axis 1) x 2 (axis 2) nodes
// it records (maximum -- NaN when any value is NaN --, largest finite |value|)
// at bst[(k * nb1 + b1) * nb2 + b2], nb1 = ceil(n1 / 16), nb2 = ceil(n2 / 2).
// Item words: 0 the float table, 1 the statistics, 2 K (rows), 3 n1, 4 n2.
// One CTA (a multiple of 32 threads) per (item, row, 16-node band of axis 1):
// tile_prefix counts K * nb1 tiles per item.  The threads walk axis 2 (unit
// stride, coalesced) and pair up by a shuffle.
__device__ __forceinline__ void lcm_tile_stats2(const i64* __restrict__ items, const int* __restrict__ tile_prefix,
                                                int n_items, int n_tiles) {
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int item = lcm_find_item(tile_prefix, n_items, tile);
    const i64* it = items + (i64)item * 5;
    const float* __restrict__ ev = lcm_wp<const float>(it, 0);
    float2* bst = lcm_wp<float2>(it, 1);
    const int n1 = lcm_wi(it, 3), n2 = lcm_wi(it, 4);
    const int nb1 = (n1 + 15) >> 4, nb2 = (n2 + 1) >> 1;
    const int r = tile - tile_prefix[item];  // k * nb1 + b1
    const int k = r / nb1, b1 = r - k * nb1;
    const float* rowk = ev + (i64)k * n1 * n2;
    const int i1a = b1 * 16, i1b = min(n1, i1a + 16);
    for (int c0 = 0; c0 < n2; c0 += blockDim.x) {  // uniform over the CTA
      const int i2 = c0 + (int)threadIdx.x;
      float mx = -lcm_lim<float>::inf(), ab = 0.0f;
      if (i2 < n2) {
        for (int i1 = i1a; i1 < i1b; ++i1) {
          const float v = __ldg(rowk + (i64)i1 * n2 + i2);
          mx = lcm_nanmax(mx, v);
          if (lcm_isfinite(v)) ab = fmaxf(ab, fabsf(v));
        }
      }
      const float omx = __shfl_xor_sync(0xffffffffu, mx, 1);
      const float oab = __shfl_xor_sync(0xffffffffu, ab, 1);
      mx = lcm_nanmax(mx, omx);
      ab = fmaxf(ab, oab);
      if (i2 < n2 && (i2 & 1) == 0) bst[(i64)r * nb2 + (i2 >> 1)] = make_float2(mx, ab);
    }
  }
}

// Logsum over discrete choices with max shift (logsum.py:32-64).
template <typename T, int ND>
__device__ __forceinline__ T lcm_logsum(const T* vals, T scale) {
  T vmax = -lcm_lim<T>::inf();
#pragma unroll
  for (int d = 0; d < ND; ++d) vmax = vals[d] > vmax ? vals[d] : vmax;
  T fin = (vmax == -lcm_lim<T>::inf()) ? T(0) : vmax;
  T m = -lcm_lim<T>::inf();
  T sh[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) { sh[d] = (vals[d] - fin) / scale; m = sh[d] > m ? sh[d] : m; }
  if (!lcm_isfinite(m)) m = T(0);
  T s = T(0);
#pragma unroll
  for (int d = 0; d < ND; ++d) s += exp(sh[d] - m);
  return fin + scale * (log(s) + m);
}

// ---------------------------------------------------------------------------
// Counter-based RNG: Philox-4x32 with 10 rounds (Salmon, Moraes, Dror & Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011).  A draw is a pure
// function of (counter, key): the simulation uses counter = (subject, period,
// stream, 0) and key = the 64-bit seed, so results do not depend on launch
// shape or on which thread draws.
struct LcmU4 { u32 x, y, z, w; };

__device__ __forceinline__ LcmU4 lcm_philox4x32(u32 c0, u32 c1, u32 c2, u32 c3, u32 k0, u32 k1) {
  const u32 M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const u32 W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += W0; k1 += W1; }
    const u32 hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
    const u32 hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
    const u32 n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  LcmU4 o; o.x = c0; o.y = c1; o.z = c2; o.w = c3;
  return o;
}

// uniform double in (0, 1) from 53 random bits
__device__ __forceinline__ double lcm_u53(u32 a, u32 b) {
  const u64 m = ((u64)(a >> 5) << 26) | (u64)(b >> 6);
  return ((double)m + 0.5) * 1.1102230246251565404e-16;  // 2^-53
}

struct LcmRng {
  u32 k0, k1, subject, period;
  __device__ __forceinline__ LcmU4 raw(u32 stream) const { return lcm_philox4x32(subject, period, stream, 0u, k0, k1); }
  __device__ __forceinline__ double uniform(u32 stream) const { LcmU4 r = raw(stream); return lcm_u53(r.x, r.y); }
  // standard normal by Box-Muller on two uniforms of the same counter
  __device__ __forceinline__ double normal(u32 stream) const {
    LcmU4 r = raw(stream);
    const double u1 = lcm_u53(r.x, r.y), u2 = lcm_u53(r.z, r.w);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
  // standard Gumbel: -log(-log(u))
  __device__ __forceinline__ double gumbel(u32 stream) const { return -log(-log(uniform(stream))); }
};

// JAX's default stream (the reference's jax.random in 64-bit mode):
// Threefry-2x32 with 20 rounds (Salmon, Moraes, Dror and Shaw 2011) of the
// counter pair (x0, x1) under the key (k0, k1).
__device__ __forceinline__ u32 lcm_rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }
__device__ __forceinline__ void lcm_threefry2x32(u32 k0, u32 k1, u32& x0, u32& x1) {
  const u32 ks[3] = {k0, k1, k0 ^ k1 ^ 0x1BD11BDAu};
  const int rot[2][4] = {{13, 15, 26, 6}, {17, 29, 16, 24}};
  x0 += ks[0];
  x1 += ks[1];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      x0 += x1;
      x1 = lcm_rotl32(x1, rot[i & 1][j]);
      x1 ^= x0;
    }
    x0 += ks[(i + 1) % 3];
    x1 += ks[(i + 2) % 3] + (u32)(i + 1);
  }
}

// Draws of one subject from JAX's stream.  `keys` holds, per stream slot q,
// the key the reference splits into one key per subject (subject s gets the
// hash of the counters (0, s + 1)); a draw of shape () uses the 64 bits of
// the subject key's counters (0, 0), element d of a vector draw those of
// (0, d); uniform: those bits' high 52 as a mantissa in [1, 2) minus one.
struct LcmJaxRng {
  const u32* keys;
  u32 subject;
  __device__ __forceinline__ void subject_key(int q, u32& a, u32& b) const {
    a = 0u;
    b = subject + 1u;
    lcm_threefry2x32(keys[2 * q], keys[2 * q + 1], a, b);
  }
  static __device__ __forceinline__ double u01(u32 k0, u32 k1, u32 c) {
    u32 a = 0u, b = c;
    lcm_threefry2x32(k0, k1, a, b);
    const u64 bits = ((u64)a << 32) | (u64)b;
    return __longlong_as_double((long long)((bits >> 12) | 0x3FF0000000000000ULL)) - 1.0;
  }
  // jax.random.uniform(key, minval=lo, maxval=hi)
  static __device__ __forceinline__ double scaled(double f, double lo, double hi) {
    const double x = f * (hi - lo) + lo;
    return x > lo ? x : lo;
  }
  __device__ __forceinline__ double uniform(int q, double lo = 0.0, double hi = 1.0) const {
    u32 a, b;
    subject_key(q, a, b);
    return scaled(u01(a, b, 0u), lo, hi);
  }
  // sqrt(2) erfinv(u), u uniform on (nextafter(-1, 0), 1)
  static __device__ __forceinline__ double normal_of(u32 a, u32 b) {
    const double lo = -0.99999999999999989;  // nextafter(-1, 0)
    return 1.4142135623730951 * erfinv(scaled(u01(a, b, 0u), lo, 1.0));
  }
  __device__ __forceinline__ double normal(int q) const {
    u32 a, b;
    subject_key(q, a, b);
    return normal_of(a, b);
  }
  // element d of jax.random.gumbel(key, (n,)): -log(-log(u)), u on [tiny, 1)
  __device__ __forceinline__ double gumbel(int q, int d) const {
    u32 a, b;
    subject_key(q, a, b);
    const double u = scaled(u01(a, b, (u32)d), 2.2250738585072014e-308, 1.0);
    return -log(-log(u));
  }
  // normal-mixture innovation: key1, key2 = split(key); component 1 when
  // uniform(key1) < p1; the normal from key2
  __device__ __forceinline__ bool mixture(int q, double p1, double& z) const {
    u32 a, b;
    subject_key(q, a, b);
    u32 a1 = 0u, b1 = 0u, a2 = 0u, b2 = 1u;
    lcm_threefry2x32(a, b, a1, b1);
    lcm_threefry2x32(a, b, a2, b2);
    z = normal_of(a2, b2);
    return u01(a1, b1, 0u) < p1;
  }
};

// jax.random.choice(key, n, p=p): the first index whose cumulative weight
// reaches total * (1 - u)
template <int N>
__device__ __forceinline__ int lcm_jax_choice(const double* p, double u) {
  double cum[N];
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) { acc += p[i]; cum[i] = acc; }
  const double r = acc * (1.0 - u);
  int k = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) k += cum[i] < r ? 1 : 0;
  return k < N - 1 ? k : N - 1;
}

// categorical draw: first index whose cumulative weight exceeds u * total
template <int N>
__device__ __forceinline__ int lcm_categorical(const double* p, double u) {
  double tot = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) tot += p[i];
  const double thr = u * tot;
  double acc = 0.0;
  int pick = N - 1;
  for (int i = 0; i < N; ++i) { acc += p[i]; if (thr < acc) { pick = i; break; } }
  return pick;
}

// ---------------------------------------------------------------------------
// Reads of a NaN-padded, weakly ascending refined row (DC-EGM carry rows),
// with the reference's rules (src/_lcm/egm/interp.py:63-131): linear
// extrapolation below the first node, clamp at or above the last, a
// duplicated abscissa read right-continuously, a -inf endpoint forcing -inf
// in the bracket's interior.  The value read is a cubic Hermite with node
// slopes dp, limited by Fritsch & Carlson (1980); it falls back to linear
// where a slope or endpoint is not finite.  The slope row itself is read
// linearly.  L is the number of valid (non-NaN) leading entries.
// Index of the last node at or below xq (-1 below the first node): a binary
// search for the first node above xq.
__device__ __forceinline__ int lcm_row_bracket(const double* __restrict__ xp, int L, double xq) {
  int lo = 0, hi = L;
  while (lo < hi) { const int mid = (lo + hi) >> 1; if (xp[mid] > xq) hi = mid; else lo = mid + 1; }
  return lo - 1;
}

// The read on one bracket [x0, x1] (node values f0, f1, node slopes d0, d1
// when has_dp) of a row whose bracket index is idx (-1: below the first node;
// the bracket is then the first one) and idx <= L - 2.
__device__ __forceinline__ void lcm_bracket_read(double x0, double x1, double f0, double f1, double d0, double d1,
                                                 bool has_dp, int idx, double xq, double& val, double& slope_val) {
  const double h = x1 - x0;
  const double t = h > 0.0 ? (xq - x0) / h : 0.0;
  double v = h > 0.0 ? f0 + t * (f1 - f0) : f1;
  double s = LCM_NAN;
  if (has_dp) {
    s = h > 0.0 ? d0 + t * (d1 - d0) : d1;
    if (lcm_isfinite(f0) && lcm_isfinite(f1) && lcm_isfinite(d0) && lcm_isfinite(d1) && h > 0.0 && idx >= 0) {
      const double delta = (f1 - f0) / h;
      double e0 = 0.0, e1 = 0.0;
      if (delta != 0.0) {
        double a = d0 / delta, bb = d1 / delta;
        a = a > 0.0 ? a : 0.0;
        bb = bb > 0.0 ? bb : 0.0;
        const double r2 = a * a + bb * bb;
        const double tau = r2 > 9.0 ? 3.0 / sqrt(r2) : 1.0;
        e0 = tau * a * delta;
        e1 = tau * bb * delta;
      }
      const double t2 = t * t, t3 = t2 * t;
      v = (2 * t3 - 3 * t2 + 1) * f0 + (t3 - 2 * t2 + t) * h * e0 + (-2 * t3 + 3 * t2) * f1 + (t3 - t2) * h * e1;
    }
  }
  const bool neg0 = f0 == -LCM_INF, neg1 = f1 == -LCM_INF;
  if (idx >= 0 && (neg0 || neg1) && !((xq == x0) && lcm_isfinite(f0)) && !((xq == x1) && lcm_isfinite(f1))) v = -LCM_INF;
  val = v;
  slope_val = s;
}

// lcm_row_bracket for the 32 converged lanes of a warp reading the same
// sorted row (same xp and L on every lane; `xq` per lane): the brackets of
// the warp's smallest and largest query bound every lane's bracket, so when
// at most 32 nodes lie between them each lane counts the nodes at or below
// its query among those (held one per lane, searched through shuffles)
// instead of searching the row in memory.  The result equals
// lcm_row_bracket's on every lane (a NaN query gets L - 1, as there); with a
// wider window every lane falls back to its own search.
// lcm_row_bracket of two warp-uniform queries qa, qb (same xp and L on every
// lane of a converged warp) by a 32-ary search: each round every lane tests
// one node of the current interval and a ballot keeps the sub-interval that
// holds the first node above the query -- ceil(log32(L)) + 1 dependent rounds
// instead of log2(L).  Invariant: the first node above q lies in [lo, hi],
// where hi == L or xp[hi] > q; a probe at or past hi is "above" without a
// load, so no lane reads past the row.
__device__ __forceinline__ void lcm_row_bracket_coop2(const double* __restrict__ xp, int L, double qa, double qb,
                                                      int& ia, int& ib) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int alo = 0, ahi = L, blo = 0, bhi = L;
  while (alo < ahi || blo < bhi) {
    const int sa = (ahi - alo + 31) >> 5, sb = (bhi - blo + 31) >> 5;
    const int ma = alo + (lane + 1) * sa - 1, mb = blo + (lane + 1) * sb - 1;
    const bool up_a = alo < ahi && (ma >= ahi || xp[ma] > qa);
    const bool up_b = blo < bhi && (mb >= bhi || xp[mb] > qb);
    const unsigned ba = __ballot_sync(full, up_a), bb = __ballot_sync(full, up_b);
    if (alo < ahi) {
      if (ba == 0u) {
        alo = ahi;
      } else {
        const int f = __ffs(ba) - 1, mf = alo + (f + 1) * sa - 1;
        alo += f * sa;
        ahi = mf < ahi ? mf : ahi;
      }
    }
    if (blo < bhi) {
      if (bb == 0u) {
        blo = bhi;
      } else {
        const int f = __ffs(bb) - 1, mf = blo + (f + 1) * sb - 1;
        blo += f * sb;
        bhi = mf < bhi ? mf : bhi;
      }
    }
  }
  ia = alo - 1;
  ib = blo - 1;
}

__device__ __forceinline__ int lcm_row_bracket_warp(const double* __restrict__ xp, int L, double xq) {
  const unsigned full = 0xffffffffu;
  double qmin = xq, qmax = xq;  // fmin / fmax skip NaN queries
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    qmin = fmin(qmin, __shfl_xor_sync(full, qmin, o));
    qmax = fmax(qmax, __shfl_xor_sync(full, qmax, o));
  }
  if (qmin != qmin) return L - 1;  // every query is NaN
  int i_lo, i_hi;
  lcm_row_bracket_coop2(xp, L, qmin, qmax, i_lo, i_hi);
  const int W = i_hi - i_lo;  // nodes in (i_lo, i_hi]
  if (W > 32) {
    // every lane's first node above its query lies in [i_lo + 1, i_hi + 1]
    if (xq != xq) return L - 1;
    int lo = i_lo + 1, hi = i_hi + 1;
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (xp[mid] > xq) hi = mid; else lo = mid + 1; }
    return lo - 1;
  }
  const int lane = threadIdx.x & 31;
  const double node = lane < W ? xp[i_lo + 1 + lane] : LCM_INF;
  int lo = 0, hi = W;
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const int mid = (lo + hi) >> 1;
    const double x = __shfl_sync(full, node, mid & 31);
    if (lo < hi) {
      if (x > xq) hi = mid; else lo = mid + 1;
    }
  }
  return xq != xq ? L - 1 : i_lo + lo;
}

__device__ __forceinline__ void lcm_row_read(const double* __restrict__ xp, const double* __restrict__ fp,
                                             const double* __restrict__ dp, int L, double xq,
                                             double& val, double& slope_val, bool warp_uniform = false) {
  if (L <= 0) { val = slope_val = LCM_NAN; return; }
  if (L == 1) { val = fp[0]; slope_val = dp ? dp[0] : LCM_NAN; return; }
  const int idx = warp_uniform ? lcm_row_bracket_warp(xp, L, xq) : lcm_row_bracket(xp, L, xq);
  if (idx >= L - 1) { val = fp[L - 1]; slope_val = dp ? dp[L - 1] : LCM_NAN; return; }
  const int b = idx < 0 ? 0 : idx;
  lcm_bracket_read(xp[b], xp[b + 1], fp[b], fp[b + 1], dp ? dp[b] : 0.0, dp ? dp[b + 1] : 0.0, dp != nullptr, idx, xq,
                   val, slope_val);
}

// lcm_row_read of K rows at the same per-lane query, for the 32 converged
// lanes of a warp that read the same K rows (row k: xp[k], fp[k], dp[k], L[k]
// equal on every lane).  The rows' searches run interleaved -- one 32-ary
// ballot search with 2K heads (each row's bracket of the warp's smallest and
// largest query), then each row's window search -- so their dependent loads
// overlap.  Every result equals lcm_row_read's.
template <int K>
__device__ __forceinline__ void lcm_row_read_warpk(const double* const* xp, const double* const* fp,
                                                   const double* const* dp, const int* L, double xq, double* val,
                                                   double* slope_val) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  double qmin = xq, qmax = xq;  // fmin / fmax skip NaN queries
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    qmin = fmin(qmin, __shfl_xor_sync(full, qmin, o));
    qmax = fmax(qmax, __shfl_xor_sync(full, qmax, o));
  }
  const bool all_nan = qmin != qmin;
  // heads 2k, 2k + 1: row k at qmin, qmax (rows of fewer than 2 nodes, or
  // every query NaN: no search)
  int lo[2 * K], hi[2 * K];
#pragma unroll
  for (int h = 0; h < 2 * K; ++h) {
    lo[h] = 0;
    hi[h] = (L[h >> 1] >= 2 && !all_nan) ? L[h >> 1] : 0;
  }
  bool active = true;
  while (active) {
    bool up[2 * K];
    int s[2 * K];
#pragma unroll
    for (int h = 0; h < 2 * K; ++h) {
      s[h] = (hi[h] - lo[h] + 31) >> 5;
      const int m = lo[h] + (lane + 1) * s[h] - 1;
      const double q = (h & 1) ? qmax : qmin;
      up[h] = lo[h] < hi[h] && (m >= hi[h] || xp[h >> 1][m] > q);
    }
    active = false;
#pragma unroll
    for (int h = 0; h < 2 * K; ++h) {
      const unsigned b = __ballot_sync(full, up[h]);
      if (lo[h] < hi[h]) {
        if (b == 0u) {
          lo[h] = hi[h];
        } else {
          const int f = __ffs(b) - 1, mf = lo[h] + (f + 1) * s[h] - 1;
          lo[h] += f * s[h];
          hi[h] = mf < hi[h] ? mf : hi[h];
        }
      }
      active = active || lo[h] < hi[h];
    }
  }
  // each row's window (i_lo, i_hi]: one node per lane, then a shuffle search
  double node[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i_lo = lo[2 * k] - 1, W = lo[2 * k + 1] - lo[2 * k];
    node[k] = (L[k] >= 2 && !all_nan && W <= 32 && lane < W) ? xp[k][i_lo + 1 + lane] : LCM_INF;
  }
  int idx[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i_lo = lo[2 * k] - 1, W = lo[2 * k + 1] - lo[2 * k];
    int a = 0, z = W;
#pragma unroll
    for (int st = 0; st < 6; ++st) {
      const int mid = (a + z) >> 1;
      const double x = __shfl_sync(full, node[k], mid & 31);
      if (a < z && W <= 32) {
        if (x > xq) z = mid; else a = mid + 1;
      }
    }
    if (W > 32 && xq == xq) {
      // every lane's first node above its query lies in [i_lo + 1, i_hi + 1]
      a = i_lo + 1;
      z = lo[2 * k + 1];
      while (a < z) { const int mid = (a + z) >> 1; if (xp[k][mid] > xq) z = mid; else a = mid + 1; }
      idx[k] = a - 1;
    } else {
      idx[k] = (xq != xq || all_nan) ? L[k] - 1 : i_lo + a;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int Lk = L[k];
    if (Lk <= 0) { val[k] = slope_val[k] = LCM_NAN; continue; }
    if (Lk == 1) { val[k] = fp[k][0]; slope_val[k] = dp[k] ? dp[k][0] : LCM_NAN; continue; }
    const int ix = idx[k];
    if (ix >= Lk - 1) { val[k] = fp[k][Lk - 1]; slope_val[k] = dp[k] ? dp[k][Lk - 1] : LCM_NAN; continue; }
    const int b = ix < 0 ? 0 : ix;
    const double* d = dp[k];
    lcm_bracket_read(xp[k][b], xp[k][b + 1], fp[k][b], fp[k][b + 1], d ? d[b] : 0.0, d ? d[b + 1] : 0.0, d != nullptr,
                     ix, xq, val[k], slope_val[k]);
  }
}
