/*
 * lcmx.h -- C ABI of the B200 backward-induction solver (liblcmx.so).
 *
 * The reference (OpenSourceEconomics/pylcm) has no foreign-function boundary
 * on its solve path: the per-period step is a JAX program dispatched from the
 * Python loop in src/_lcm/solution/backward_induction.py:155-275.  The entry
 * points below replace, one for one, the calls that loop makes:
 *
 *   lcmx_module_compile  <- AOT compile of the per-period cores,
 *                           backward_induction.py:577-720 (jax.jit(...).lower
 *                           .compile); here NVRTC for sm_100a, cached by key.
 *   lcmx_bellman_step    <- _GridSearchPeriodKernel.__call__,
 *                           src/_lcm/solution/grid_search.py:192-212 (the
 *                           max_Q_over_a program, max_Q_over_a.py:30-191).
 *   lcmx_expectation     <- the continuation expectation inside Q_and_F,
 *                           src/_lcm/regime_building/Q_and_F.py:466-681 and
 *                           _expectation_over_stochastic_nodes :1145-1209
 *                           (also the tcgen05 form of the single-precision
 *                           search table, 3xTF32 with FP32 accumulation).
 *   lcmx_simulate        <- the per-period simulation step,
 *                           src/_lcm/simulation/simulate.py:465-668.
 *   lcmx_egm_step        <- the DC-EGM per-period core,
 *                           src/_lcm/egm/step_core.py:156-312.
 *   lcmx_fues_scan       <- the FUES upper envelope of DC-EGM candidates,
 *                           src/_lcm/egm/upper_envelope/fues.py:151-338.
 *   lcmx_count_nonfinite <- the per-period NaN/Inf diagnostics,
 *                           backward_induction.py:205-236.
 *   lcmx_copy_rows_d2h   <- the device->host read of a period's value
 *                           arrays (the `np.asarray` of the returned V).
 *
 * Conventions: every pointer argument that names array data is a DEVICE
 * pointer; sizes are element counts; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Every function returns an int status (LCMX_OK = 0)
 * and never frees caller memory; the message of the last failure on a
 * context is returned by lcmx_last_error.
 */
#ifndef LCMX_H
#define LCMX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LCMX_OK = 0,
  LCMX_ERR_ARGS = 1,      /* invalid argument (null pointer, bad size)     */
  LCMX_ERR_COMPILE = 2,   /* NVRTC rejected the generated source           */
  LCMX_ERR_MODULE = 3,    /* module load failed or kernel symbol missing   */
  LCMX_ERR_LAUNCH = 4,    /* kernel launch failed                          */
  LCMX_ERR_CUDA = 5,      /* other CUDA runtime / driver failure           */
  LCMX_ERR_NOMEM = 6,     /* device memory exhausted                       */
  LCMX_ERR_TIMEOUT = 7    /* a bounded device-side wait gave up            */
};

typedef struct lcmx_ctx lcmx_ctx;
typedef struct lcmx_module lcmx_module;

/* One launch of a generated kernel over a list of work items.
 * `items` holds n_items records of 64-bit words whose layout is fixed by the
 * code generator for that kernel; `tile_prefix[i]` is the first tile of item
 * i and tile_prefix[n_items] the total tile count.  grid == 0 selects
 * (SM count x resident CTAs per SM). */
typedef struct {
  const void* items;
  const int* tile_prefix;
  int n_items;
  int n_tiles;
  int grid;
  int block;
  int smem_bytes;
} lcmx_launch_args;

/* One entry of lcmx_launch_list: a generated kernel of `module` over its
 * item records; `seed` is passed only when `with_seed` is non-zero (the
 * simulation kernels' launch seed). */
typedef struct {
  lcmx_module* module;
  const char* kernel;
  lcmx_launch_args args;
  unsigned long long seed;
  int with_seed;
} lcmx_launch_rec;

/* Create / destroy a context bound to CUDA device `device` (primary context). */
int lcmx_ctx_create(int device, lcmx_ctx** out);
int lcmx_ctx_destroy(lcmx_ctx* ctx);
/* Message of the last failure on ctx (never NULL; "" after success). */
const char* lcmx_last_error(const lcmx_ctx* ctx);
/* Device facts used for grid sizing and HBM admission. */
int lcmx_device_info(lcmx_ctx* ctx, int* sm_count, size_t* free_bytes, size_t* total_bytes);

/* Compile CUDA C for sm_100a with NVRTC and load it.  `key` names the source
 * in the in-process and on-disk cubin caches; `options` is a '\n'-separated
 * list of extra NVRTC options (may be NULL). */
int lcmx_module_compile(lcmx_ctx* ctx, const char* cuda_src, const char* key,
                        const char* options, lcmx_module** out);
int lcmx_module_destroy(lcmx_module* mod);
/* Resident CTAs per SM of `kernel` at the given block size / dynamic smem. */
int lcmx_occupancy(lcmx_module* mod, const char* kernel, int block, int smem_bytes,
                   int* blocks_per_sm);

/* Read the int status word `name` (a __device__ global) of a module: 0 when
 * every bounded device-side wait of its kernels completed; the tensor-core
 * expectation sets its word "lcm_status" to 1 when a wait gave up.  A module
 * without the word reports 0.  Synchronous (waits for the device); `reset`
 * clears a non-zero word.  No counterpart in the reference: its XLA programs
 * have no bounded waits to report. */
int lcmx_module_status(lcmx_module* mod, const char* name, int* value, int reset);

/* Kernel (a): fused Q_and_F + max/argmax over actions for a batch of
 * (solve instance, regime, period) items; writes V (double) and the flat
 * argmax action index (int32) per state. */
int lcmx_bellman_step(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args,
                      void* stream);
/* Kernel (b): EV[k, col] = sum_j W[k, j] V'[j, col] / sum_j W[k, j] for a batch
 * of (instance, source regime, target regime) items. */
int lcmx_expectation(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args,
                     void* stream);
/* Kernel (d): one simulated period for a batch of (instance, regime) items,
 * each with its own subjects (Philox-4x32-10 counter RNG; the key of an item
 * is `seed` XOR the item's seed word, the counter is (subject, period,
 * stream id)). */
int lcmx_simulate(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args,
                  unsigned long long seed, void* stream);
/* Kernel (c), part 1: DC-EGM Euler inversion and candidate generation. */
int lcmx_egm_step(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args,
                  void* stream);
/* `n` item launches (any of the four above) issued in order on `stream`: the
 * per-period launch sequence of a solve or simulation plan in one call, in
 * place of the reference's per-(period, regime) dispatch of compiled XLA
 * programs (src/_lcm/solution/backward_induction.py:174-183).  Stops at the
 * first failing launch and returns its status. */
int lcmx_launch_list(const lcmx_launch_rec* recs, int n, void* stream);

/* Kernel (c), part 2: FUES upper envelope of `n_rows` candidate rows of
 * length n_in (row-major; any order within a row, NaN entries are absent
 * candidates).  `savings` (may be NULL) is each candidate's exogenous savings
 * source.  `n_points_to_scan` bounds the same-segment look-ahead to that many
 * positions on either side, as FUESEnvelope(n_points_to_scan=...) does
 * (fues.py:114-128, 1016-1079); <= 0 scans exhaustively (the default).
 * Outputs are (n_rows x n_out) NaN-padded refined rows in ascending
 * grid order; n_kept[row] > n_out signals overflow (the row holds a valid
 * prefix).  `workspace` must hold lcmx_fues_workspace_bytes(n_rows, n_in)
 * bytes of device memory (rows of up to 4096 candidates are staged in shared
 * memory and leave it unused).  Rows of up to 8192 candidates. */
size_t lcmx_fues_workspace_bytes(int n_rows, int n_in);
int lcmx_fues_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                   const double* savings, int n_rows, int n_in, double jump_thresh,
                   int n_points_to_scan, double* grid_out, double* policy_out, double* value_out,
                   int n_out, int* n_kept, void* workspace, size_t workspace_bytes, void* stream);

/* Kernel (c), part 2, item form: the FUES envelope of the rows of n_items
 * candidate blocks (one per solve instance) in one launch, each row staged in
 * shared memory; same rows as lcmx_fues_scan (fues.py:151-338, one
 * refine_envelope per row).  `items` holds n_items records of 13 64-bit
 * words: grid, policy, value, savings (0: none), grid_out, policy_out,
 * value_out, n_kept (int32) device pointers, then n_rows, n_in, n_out,
 * jump_thresh (double bits) and the look-ahead window (<= 0: exhaustive);
 * tile_prefix[i] is the first row of item i and
 * n_rows the total.  max_n_in (the longest row, at most 4096 candidates)
 * sizes the shared memory.  Needs no workspace. */
int lcmx_fues_step(lcmx_ctx* ctx, const void* items, const int* tile_prefix, int n_items, int n_rows,
                   int max_n_in, void* stream);

/* Kernel (c), part 2, the LTM envelope (LTMEnvelope): the local-upper-bound
 * brute method of src/_lcm/egm/upper_envelope/ltm.py:35-190 (refine_envelope),
 * on `n_rows` contiguous candidate rows of length n_in.  Segments join
 * consecutive candidates in input order; at each live candidate abscissa
 * (ascending) the envelope is the largest interpolant over the bracketing
 * segments.  Outputs as lcmx_fues_scan's.  Rows of up to 4096 candidates. */
int lcmx_ltm_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value, int n_rows,
                  int n_in, double* grid_out, double* policy_out, double* value_out, int n_out, int* n_kept,
                  void* stream);

/* Kernel (c), part 2, the RFC envelope (RFCEnvelope): the rooftop cut of
 * src/_lcm/egm/upper_envelope/rfc.py:40-220 (refine_envelope) with the
 * candidates' marginal utility (the value rows' supgradient) as tangent
 * slopes, `search_radius` neighbours on each side and the policy-jump
 * threshold `jump_thresh`.  Outputs as lcmx_fues_scan's (a subset of the
 * sorted candidates).  Rows of up to 4096 candidates. */
int lcmx_rfc_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                  const double* marginal_utility, int n_rows, int n_in, int search_radius, double jump_thresh,
                  double* grid_out, double* policy_out, double* value_out, int n_out, int* n_kept, void* stream);

/* Kernel (c), part 2, the MSS envelope (MSSEnvelope): HARK's EGM upper
 * envelope as src/_lcm/egm/upper_envelope/mss.py:72-629 (refine_envelope)
 * states it -- LTM's evaluation over the monotone links (a grid or value
 * decrease starts a new branch), plus the exact crossing of the two winning
 * links, inserted twice (left, right policy), where the winning branch
 * changes.  Outputs as lcmx_fues_scan's.  Rows of up to 4096 candidates. */
int lcmx_mss_scan(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value, int n_rows,
                  int n_in, double* grid_out, double* policy_out, double* value_out, int n_out, int* n_kept,
                  void* stream);

/* Item form of the LTM (kind 1), RFC (kind 2) and MSS (kind 3) envelopes, one launch over
 * the rows of n_items candidate blocks; item records of 13 64-bit words:
 * grid, policy, value, marginal utility (RFC; 0 for LTM), grid_out,
 * policy_out, value_out, n_kept (int32) device pointers, then n_rows, n_in,
 * n_out, jump_thresh (double bits) and the search radius; tile_prefix[i] is
 * the first row of item i.  max_n_in (at most 4096) sizes the shared memory. */
int lcmx_envelope_step(lcmx_ctx* ctx, int kind, const void* items, const int* tile_prefix, int n_items,
                       int n_rows, int max_n_in, void* stream);

/* lcmx_fues_scan without a caller workspace: for callers that cannot call
 * cudaMalloc on this path (code running inside another runtime's execution,
 * such as an XLA FFI custom-call handler).  No counterpart in the reference.
 * Scratch is an 8 MiB file-scope device array per device, so
 * lcmx_fues_workspace_bytes(n_rows, n_in) must not exceed 8 MiB (larger calls
 * return LCMX_ERR_ARGS).  Rows of up to 4096 candidates are staged in shared
 * memory and leave the array unused; longer rows (up to 8192) keep their
 * sorted copy in it.  The first call on a device resolves the array's
 * address (make it before any stream capture); all calls share the array, so
 * calls that overlap on the GPU race.  The call makes the context's device
 * current while it runs and restores the caller's current device before it
 * returns.  The look-ahead is exhaustive.  Allocates nothing. */
int lcmx_fues_scan_static(lcmx_ctx* ctx, const double* grid, const double* policy, const double* value,
                          const double* savings, int n_rows, int n_in, double jump_thresh,
                          double* grid_out, double* policy_out, double* value_out, int n_out, int* n_kept,
                          void* stream);

/* Count non-finite (and separately NaN) entries of a double array; the two
 * counters are accumulated into counts_dev[0] (nan) and counts_dev[1]
 * (+-inf), which the caller zeroes. */
int lcmx_count_nonfinite(lcmx_ctx* ctx, const double* x, long long n,
                         unsigned long long* counts_dev, void* stream);

/* Asynchronous strided device->host copy of `rows` rows of `row_bytes` bytes:
 * row r goes from src + r * src_pitch (device) to dst + r * dst_pitch (host;
 * page-locked for the copy to overlap kernels).  Used to read one period's
 * slice of every instance's value array while later periods compute.  The
 * one exception to the device-pointer convention: `dst` is a HOST pointer. */
int lcmx_copy_rows_d2h(lcmx_ctx* ctx, void* dst, size_t dst_pitch, const void* src, size_t src_pitch,
                       size_t row_bytes, size_t rows, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LCMX_H */
