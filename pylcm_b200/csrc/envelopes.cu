// envelopes.cu -- the LTM and RFC upper envelopes of DC-EGM candidate rows
// (kernel c, part 2, the alternatives to FUES).
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
// Both publish the survivors in sorted order, NaN-padded to n_out, with their
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
    // bitonic sort of (key, index) ascending
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

extern "C" int lcmx_envelope_step(lcmx_ctx* ctx, int kind, const void* items, const int* tile_prefix, int n_items,
                                  int n_rows, int max_n_in, void* stream) {
  if (!ctx || (kind != kLtm && kind != kRfc) || n_items < 0 || n_rows < 0 ||
      (n_items > 0 && (!items || !tile_prefix)))
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS, "lcmx_envelope_step: bad arguments");
  if (max_n_in < 1 || max_n_in > kEnvMaxN)
    return lcmx_set_error_from(ctx, LCMX_ERR_ARGS,
                               "lcmx_envelope_step: rows must hold 1.." + std::to_string(kEnvMaxN) + " candidates");
  if (n_items == 0 || n_rows == 0) return LCMX_OK;
  EnvItems rows{static_cast<const int64_t*>(items), tile_prefix, n_items, n_rows};
  std::string err;
  const int rc = kind == kLtm ? env_launch<EnvItems, kLtm>(rows, n_rows, max_n_in, (cudaStream_t)stream, err)
                              : env_launch<EnvItems, kRfc>(rows, n_rows, max_n_in, (cudaStream_t)stream, err);
  return rc ? lcmx_set_error_from(ctx, rc, err) : LCMX_OK;
}
