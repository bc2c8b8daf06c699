// lcm_tc.cuh -- the single-precision shock expectation on the 5th-generation
// tensor cores (tcgen05), for the single-precision search form of kernel (a).
//
// Computes, for one (source regime, target regime) pair and every instance,
//
//     EV32[k, col] = sum_j W[k, j] V'[j, col] / sum_j W[k, j]
//
// (the continuation expectation of src/_lcm/regime_building/Q_and_F.py:
// 466-681 with the node sum of _expectation_over_stochastic_nodes :1145-1209
// contracted first), as a GEMM D = A B with
//     A[m, j] = V'[j, col0 + m]   (m < 128: a tile of 128 columns),
//     B[j, n] = W[n, j]           (n < NP: the weight rows, zero padded),
// accumulated in FP32 in tensor memory.  The operands are split into two
// TF32 parts (x = hi + lo, hi = tf32(x), lo = tf32(x - hi)) and the product
// is hi*hi + hi*lo + lo*hi ("3xTF32"), which keeps the FP32 table within a
// few units of float rounding of the FP64 contraction; the double-precision
// table and the final FP64 re-evaluation of the search's candidates are not
// affected.  Columns whose V' values are not all finite (infeasible target
// states at -inf) are recomputed in FP64 with the zero-safe rule
// (src/_lcm/zero_safe.py:161-251): a zero weight ignores any value.
//
// Mapping (one CTA of 128 threads = 4 warps per SM slot; a grid-stride loop
// over 128-column tiles of every item):
//   * thread t loads column col0 + t of V' (coalesced over t for each j),
//     splits it and writes it to shared memory in the canonical K-major,
//     no-swizzle layout of the MMA (8-row x 16-byte core matrices);
//   * one elected thread issues 3 x JP/8 tcgen05.mma.cta_group::1.kind::tf32
//     (M = 128, N = NP, K = 8 each) and commits them to an mbarrier;
//   * warp w reads its 32 TMEM lanes (rows 32w .. 32w+31 of D) with
//     tcgen05.ld.32x32b and thread t writes EV32[k, col0 + t] for every k
//     (coalesced over t).
// Every wait is bounded: a wait that gives up sets the module's lcm_status
// word, skips the tile's results and the CTA still frees its tensor memory.

#pragma once

__device__ int lcm_status;  // 0: ok; 1: a tensor-core wait gave up

#define LCM_TC_M 128
#define LCM_TC_THREADS 128

__device__ __forceinline__ u32 lcm_smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

// round-to-nearest TF32 bit pattern of a float (low 13 mantissa bits zero)
__device__ __forceinline__ u32 lcm_tf32(float x) {
  u32 r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo in two TF32 parts (of the float nearest to x)
__device__ __forceinline__ void lcm_tf32_split(double x, u32& hi, u32& lo) {
  const float f = (float)x;
  hi = lcm_tf32(f);
  lo = lcm_tf32(f - __uint_as_float(hi));
}

// Shared-memory matrix descriptor of a K-major operand without swizzle:
// start address, leading-dimension byte offset (between the two 16-byte
// core-matrix columns of one K = 8 step), stride-dimension byte offset
// (between 8-row groups), descriptor version 1 (sm_100), base offset 0.
__device__ __forceinline__ u64 lcm_umma_desc(u32 saddr, u32 lbo, u32 sbo) {
  u64 d = (u64)((saddr & 0x3FFFFu) >> 4);
  d |= (u64)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (u64)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (u64)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, A and B TF32,
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr u32 lcm_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((u32)(N >> 3) << 17) | ((u32)(M >> 4) << 24);
}

__device__ __forceinline__ void lcm_mma_tf32(u32 tmem_d, u64 adesc, u64 bdesc, u32 idesc, u32 accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void lcm_mma_commit(u32 bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void lcm_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void lcm_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void lcm_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void lcm_mbar_init(u32 bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the mbarrier phase with parity `parity`; false if it did not
// complete within about `max_cycles` clock cycles.
__device__ __forceinline__ bool lcm_mbar_wait(u32 bar, u32 parity, long long max_cycles) {
  const long long t0 = clock64();
  for (;;) {
    u32 done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}

__device__ __forceinline__ void lcm_tmem_alloc(u32 slot_addr, u32 ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_addr), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void lcm_tmem_free(u32 taddr, u32 ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void lcm_tmem_ld16(u32 taddr, float* v) {
  u32 r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Sizes of one (K, J) expectation: reduction padded to the MMA step of 8
// TF32 values, N padded to a multiple of 16, TMEM columns a power of two.
template <int K, int J> struct LcmTcShape {
  static constexpr int JP = (J + 7) / 8 * 8;
  static constexpr int NP = (K + 15) / 16 * 16;
  static constexpr int NCOL = NP <= 32 ? 32 : (NP <= 64 ? 64 : (NP <= 128 ? 128 : 256));
  static constexpr int KC = JP / 4;              // 16-byte chunks along the reduction
  static constexpr u32 A_BYTES = LCM_TC_M * JP * 4;
  static constexpr u32 B_BYTES = NP * JP * 4;
  // dynamic shared memory: A hi/lo, B hi/lo, 128 bytes of alignment slack
  static constexpr u32 SMEM = 2 * A_BYTES + 2 * B_BYTES + 128;
};

// Byte offset of element (row r, reduction index j) of a K-major operand with
// `rows` rows (a multiple of 8) in the layout the descriptors below describe:
// 16-byte chunk c = j / 4 outermost, then 8-row group g = r / 8, then the
// core matrix (8 rows x 16 bytes, row-major).
__device__ __forceinline__ u32 lcm_kmajor_off(int r, int j, int rows) {
  return (u32)(((j >> 2) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (j & 3) * 4);
}

// The expectation of one kernel launch.  `wfill(it, W)` writes the item's
// FP64 weights W[k * J + j]; V' rows are `Vt + j * cblk + col` (targets whose
// discrete axes are all stochastic).  Item words: 0 V' (double*), 2 EV32
// (float*), 6 cblk, 7 n_cols, `bst_word` the block statistics of EV32 (per
// row k and 16 columns, see lcm_block16_stats; 0: none).
template <int K, int J, typename WFill>
__device__ __forceinline__ void lcm_tc_expect(const i64* __restrict__ items, const int* __restrict__ tile_prefix,
                                              int n_items, int n_tiles, int e_words, int bst_word,
                                              const WFill& wfill) {
  using S = LcmTcShape<K, J>;
  constexpr int JP = S::JP, NP = S::NP, KC = S::KC;
  extern __shared__ unsigned char lcm_dsmem[];
  __shared__ double Wd[K * J];
  __shared__ float Wscale[K];
  __shared__ __align__(8) u64 mbar;
  __shared__ u32 tmem_slot;
  __shared__ int cur_item;

  unsigned char* base = (unsigned char*)(((unsigned long long)lcm_dsmem + 127) & ~127ull);
  unsigned char* a_hi = base;
  unsigned char* a_lo = a_hi + S::A_BYTES;
  unsigned char* b_hi = a_lo + S::A_BYTES;
  unsigned char* b_lo = b_hi + S::B_BYTES;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const u32 bar = lcm_smem_u32(&mbar);

  if (warp == 0) lcm_tmem_alloc(lcm_smem_u32(&tmem_slot), (u32)S::NCOL);
  if (tid == 0) {
    lcm_mbar_init(bar, 1);
    cur_item = -1;
  }
  lcm_tc_fence_before();
  __syncthreads();
  lcm_tc_fence_after();
  const u32 tmem = tmem_slot;
  const u32 idesc = lcm_idesc_tf32(LCM_TC_M, NP);
  u32 phase = 0;
  bool failed = false;

  for (int tile = blockIdx.x; tile < n_tiles && !failed; tile += gridDim.x) {
    const int item = lcm_find_item(tile_prefix, n_items, tile);
    const i64* it = items + (i64)item * e_words;
    // ---- weights of this item: FP64 table, row scales, B = W^T split in two
    if (item != cur_item) {
      __syncthreads();  // every thread is past the previous tile's reads of B / W
      wfill(it, Wd);
      __syncthreads();
      for (int k = tid; k < K; k += LCM_TC_THREADS) {
        double sw = 0.0;
        for (int j = 0; j < J; ++j) sw += Wd[k * J + j];
        Wscale[k] = (float)(1.0 / (sw > 0.0 ? sw : 1.0));
      }
      for (int e = tid; e < NP * JP; e += LCM_TC_THREADS) {
        const int n = e / JP, j = e % JP;
        u32 hi = 0u, lo = 0u;
        if (n < K && j < J) lcm_tf32_split(Wd[n * J + j], hi, lo);
        const u32 off = lcm_kmajor_off(n, j, NP);
        *reinterpret_cast<u32*>(b_hi + off) = hi;
        *reinterpret_cast<u32*>(b_lo + off) = lo;
      }
      if (tid == 0) cur_item = item;
    }
    const double* __restrict__ Vt = lcm_wp<const double>(it, 0);
    float* __restrict__ EV32 = lcm_wp<float>(it, 2);
    const i64 cblk = lcm_wi(it, 6);
    const int n_cols = lcm_wi(it, 7);
    const int col = (tile - tile_prefix[item]) * LCM_TC_M + tid;
    const bool live = col < n_cols;
    // ---- A: this thread's column, split, four reduction values per store
    bool nonfinite = false;
#pragma unroll
    for (int c = 0; c < KC; ++c) {
      u32 h[4], l[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = c * 4 + q;
        double v = 0.0;
        if (live && j < J) v = Vt[(i64)j * cblk + col];
        if (!lcm_isfinite(v)) {
          nonfinite = true;
          v = 0.0;
        }
        lcm_tf32_split(v, h[q], l[q]);
      }
      const u32 off = lcm_kmajor_off(tid, c * 4, LCM_TC_M);
      *reinterpret_cast<uint4*>(a_hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(a_lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    lcm_fence_async_smem();  // generic-proxy writes -> visible to the tensor core
    __syncthreads();
    // ---- D = Ahi Bhi + Ahi Blo + Alo Bhi, issued by one thread
    if (tid == 0) {
      lcm_tc_fence_after();
      const u32 ah = lcm_smem_u32(a_hi), al = lcm_smem_u32(a_lo);
      const u32 bh = lcm_smem_u32(b_hi), bl = lcm_smem_u32(b_lo);
      constexpr u32 A_LBO = (LCM_TC_M / 8) * 128, B_LBO = (NP / 8) * 128;
#pragma unroll
      for (int term = 0; term < 3; ++term) {
        const u32 a0 = term == 2 ? al : ah;
        const u32 b0 = term == 1 ? bl : bh;
#pragma unroll
        for (int s = 0; s < JP / 8; ++s) {
          const u64 ad = lcm_umma_desc(a0 + (u32)s * 2 * A_LBO, A_LBO, 128);
          const u64 bd = lcm_umma_desc(b0 + (u32)s * 2 * B_LBO, B_LBO, 128);
          lcm_mma_tf32(tmem, ad, bd, idesc, (term > 0 || s > 0) ? 1u : 0u);
        }
      }
      lcm_mma_commit(bar);
    }
    __syncwarp();
    const u32 wait_phase = phase;
    phase ^= 1u;
    // the outcome is made uniform over the CTA: the TMEM loads below are
    // warp-collective and must not diverge
    const bool ok = __syncthreads_and(lcm_mbar_wait(bar, wait_phase, 2000000000ll));
    lcm_tc_fence_after();
    if (!ok) {
      // give the MMAs in flight one more bounded wait before the tensor
      // memory they write is freed
      lcm_mbar_wait(bar, wait_phase, 2000000000ll);
      if (tid == 0) atomicExch(&lcm_status, 1);
      failed = true;
    } else {
      // ---- epilogue: row tid of D (TMEM lane tid) holds EV of column col
      float2* BST = bst_word >= 0 ? lcm_wp<float2>(it, bst_word) : nullptr;
      const int nb16 = (n_cols + 15) >> 4;
      const u32 lane_base = tmem + ((u32)(warp * 32) << 16);
#pragma unroll
      for (int n0 = 0; n0 < NP; n0 += 16) {
        float d[16];
        lcm_tmem_ld16(lane_base + (u32)n0, d);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int k = n0 + q;
          if (k >= K) continue;
          float e = d[q] * Wscale[k];
          if (live && nonfinite) {  // FP64, zero-safe, node by node
            double num = 0.0, sw = 0.0;
            for (int j = 0; j < J; ++j) {
              const double w = Wd[k * J + j];
              sw += w;
              num += lcm_zs(w, Vt[(i64)j * cblk + col]);
            }
            e = (float)(num / (sw > 0.0 ? sw : 1.0));
          }
          if (live) EV32[(i64)k * n_cols + col] = e;
          if (BST) {  // uniform over the CTA (one item per tile)
            const float2 st = lcm_block16_stats(live ? e : -lcm_lim<float>::inf());
            if (live && (tid & 15) == 0) BST[(i64)k * nb16 + (col >> 4)] = st;
          }
        }
      }
    }
    lcm_tc_fence_before();
    __syncthreads();  // TMEM reads and A reads done before the next tile's MMA
  }
  __syncthreads();
  lcm_tc_fence_after();
  if (warp == 0) lcm_tmem_free(tmem, (u32)S::NCOL);
}
