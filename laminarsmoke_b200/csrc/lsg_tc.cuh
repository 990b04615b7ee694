// Tensor-core (tcgen05, sm_100a) inverse of the Newton iteration matrix
// G = I - hr0 J for one cell per thread block, for the mixed-precision form of
// mechanisms with 32 to 128 ODE components.
//
// The reference factorises G with a partial-pivot LU in FP64
// (math/native-ode-solvers/KernelDense.hpp:195-245) and solves with the
// factors.  Here G is inverted by blocked Gauss-Jordan elimination with
// partial pivoting, in FP32 with the products of the blocked updates on the
// tensor cores as split TF32 (3xTF32: a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi,
// FP32 accumulation), and every Newton solve is one product G^-1 r.  The
// Newton iteration of MethodGear::FindCorrection recomputes its residual in
// FP64 at every iterate, so the FP32 inverse only preconditions an FP64
// fixed-point iteration: the iterates converge to the FP64 correction.
//
// Layout and schedule (128 threads = one warpgroup, thread i owns row i):
//   TMEM   [G | I] padded to 128 x 256 FP32: lane = row, column = column of
//          the augmented matrix (256 of the SM's 512 columns per block).
//   panel  32 columns at a time.  The warp owning the panel's rows reads all
//          128 rows x 32 columns (tcgen05.ld), the block eliminates the 32
//          pivots on CUDA cores (pivot: largest magnitude among the rows not
//          yet pivoted, lowest row on ties; implicit row order, no swaps),
//          and accumulates, per row, the coefficients w_i that express its
//          update as a combination of the panel's pivot rows:
//              R_new = R + W R[P]          (W: 128 x 32, R[P]: 32 x N)
//          for every column not yet eliminated and the right half.  That is
//          one tcgen05.mma per 8 columns of K (M = 128, N <= 128, K = 32)
//          with W and R[P] staged in shared memory in the canonical K-major
//          layout (no swizzle; core matrices of 8 rows x 16 bytes).
//   result after the last panel the right half holds P G^-1 (row p_c is row
//          c of G^-1); it is copied to shared memory as RT[j][c] = G^-1[c][j]
//          (column-major), where a solve reads it with unit-stride loads.
#pragma once
#include <cstdint>

namespace lsg {
namespace tc {

constexpr int kRows = 128;            // padded order of G
constexpr int kCols = 256;            // TMEM columns of [G | I]
constexpr int kPanel = 32;
constexpr int kOperandFloats = kRows * kPanel;   // one 128 x 32 operand (16 KB)
constexpr unsigned kWaitLimit = 1u << 24;        // bounded mbarrier wait

// Shared-memory pieces of the inverse (all carved by the caller).
struct Smem {
  float* op;              // 4 operands of kOperandFloats: A_hi, A_lo, B_hi, B_lo (64 KB, 1024-byte aligned);
                          // after the inverse: RT [kRows][kRows] (the same 64 KB)
  float* red;             // [2][4] warp maxima (double-buffered)
  int* redi;              // [2][4] their rows
  float* prow;            // [2][2 * kPanel] the pivot row's panel values and coefficients
  int* pivot_of_row;      // [kRows] panel column (0..127) a row was pivot for, or -1
  unsigned long long* mbar;   // MMA completion barrier (8-byte aligned)
  uint32_t* tmem_slot;    // TMEM base address written by tcgen05.alloc
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// ---- TMEM ----------------------------------------------------------------
// Executed by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive columns of this thread's lane.  taddr: lane base in bits 16+, column in the low bits.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---- MMA -----------------------------------------------------------------
// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; lbo = byte distance of the two core matrices along K of
// one instruction, sbo = byte distance of consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo & 0x3FFFFu) >> 4) << 16;
  d |= (uint64_t)((sbo & 0x3FFFFu) >> 4) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of sm_100
  return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major, M = 128, N.
__device__ __forceinline__ uint32_t idesc_tf32(int N) {
  uint32_t d = 0;
  d |= 1u << 4;                    // D format F32
  d |= 2u << 7;                    // A format TF32
  d |= 2u << 10;                   // B format TF32
  d |= (uint32_t)(N >> 3) << 17;   // N / 8
  d |= (uint32_t)(128 >> 4) << 24; // M / 16
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned long long* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase `parity` of mbar to complete; false after kWaitLimit tries.
__device__ __forceinline__ bool mbar_wait(unsigned long long* mbar, uint32_t parity) {
  const uint32_t a = smem_addr(mbar);
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Byte offset of element (row, k) of a 128 x 32 (rows x K) FP32 operand in the
// canonical K-major layout: 8-row groups 1024 bytes apart, 4-element K groups
// 128 bytes apart, rows of a core matrix 16 bytes apart.
__device__ __forceinline__ uint32_t op_offset(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// ---------------------------------------------------------------------------
// G^-1 for G = I - hr0 J (J: FP64, column-major n x n in global memory,
// element (i, j) at J[j * n + i]; 32 <= n <= 128).  All 128 threads call it.
// tmem: this block's 256-column TMEM allocation.  phase: the MMA barrier's
// parity, carried across calls.  On return (true) S.op holds RT[j * 128 + c] =
// G^-1[c][j] for c, j < n.  false: an MMA did not complete within the wait
// limit.
// ---------------------------------------------------------------------------
__device__ __noinline__ bool gj_inverse(const double* __restrict__ J, int n, double hr0, const Smem& S,
                                        uint32_t tmem, uint32_t* phase) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  // ---- [G | I] into TMEM, row tid ----
#pragma unroll 1
  for (int q = 0; q < kCols / 32; ++q) {
    float v[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const int col = q * 32 + k;
      float g;
      if (col < kRows) {
        if (tid < n && col < n) {
          double x = -hr0 * J[(long)col * n + tid];
          if (col == tid) x += 1.;
          g = (float)x;
        } else {
          g = col == tid ? 1.f : 0.f;
        }
      } else {
        g = (col - kRows) == tid ? 1.f : 0.f;
      }
      v[k] = g;
    }
    tmem_st32(tmem + lane_base + (uint32_t)(q * 32), v);
  }
  tmem_wait_st();
  if (tid < kRows) S.pivot_of_row[tid] = -1;
  bool pivoted = false;
  int my_col = -1;   // the panel column this row became the pivot of
  float* const A_hi = S.op;
  float* const A_lo = S.op + kOperandFloats;
  float* const B_hi = S.op + 2 * kOperandFloats;
  float* const B_lo = S.op + 3 * kOperandFloats;
  bool ok = true;
  const int npanels = (n + kPanel - 1) / kPanel;
  for (int pn = 0; pn < npanels; ++pn) {
    const int k0 = pn * kPanel;
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    float v[32], u[32];
    tmem_ld32(tmem + lane_base + (uint32_t)k0, v);
#pragma unroll
    for (int k = 0; k < 32; ++k) u[k] = 0.f;
    int mine = -1;   // 0..31: this row is the pivot of panel column `mine`
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      const int buf = c & 1;
      // pivot: largest |G(i, k0 + c)| over the rows not yet pivoted, lowest row on ties
      float best = pivoted ? -1.f : fabsf(v[c]);
      if (best != best) best = 0.f;   // a NaN never outranks a number, but its row stays a candidate
      int brow = tid;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
        if (ob > best || (ob == best && orow < brow)) { best = ob; brow = orow; }
      }
      if (lane == 0) { S.red[buf * 4 + warp] = best; S.redi[buf * 4 + warp] = brow; }
      __syncthreads();
      float pb = S.red[buf * 4];
      int prow_i = S.redi[buf * 4];
#pragma unroll
      for (int w = 1; w < 4; ++w) {
        const float ob = S.red[buf * 4 + w];
        const int orow = S.redi[buf * 4 + w];
        if (ob > pb || (ob == pb && orow < prow_i)) { pb = ob; prow_i = orow; }
      }
      float* pr = S.prow + buf * 2 * kPanel;
      if (tid == prow_i) {
        const float a = v[c];
        const float inv = a != 0.f ? 1.f / a : 0.f;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k > c) v[k] *= inv;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k < c) u[k] *= inv;
        u[c] = inv - 1.f;
        v[c] = 1.f;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (k > c) pr[k] = v[k];
          if (k <= c) pr[kPanel + k] = u[k] + (k == c ? 1.f : 0.f);
        }
        pivoted = true;
        mine = c;
      }
      __syncthreads();
      if (tid != prow_i) {
        const float m = v[c];
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (k > c) v[k] = fmaf(-m, pr[k], v[k]);
          if (k <= c) u[k] = fmaf(-m, pr[kPanel + k], u[k]);
        }
        v[c] = 0.f;
      }
    }
    if (mine >= 0) {
      my_col = k0 + mine;
      S.pivot_of_row[tid] = my_col;
    }
    // ---- A = W (row tid: its coefficients u), split into TF32 hi and lo ----
    {
      char* ah = (char*)A_hi;
      char* al = (char*)A_lo;
#pragma unroll
      for (int kg = 0; kg < 8; ++kg) {
        float4 hi, lo;
        float* h4 = &hi.x;
        float* l4 = &lo.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float x = u[kg * 4 + e];
          const float xh = __uint_as_float(to_tf32(x));
          h4[e] = xh;
          l4[e] = __uint_as_float(to_tf32(x - xh));
        }
        *(float4*)(ah + op_offset(tid, kg * 4)) = hi;
        *(float4*)(al + op_offset(tid, kg * 4)) = lo;
      }
    }
    // ---- R[P] and the MMAs, for the columns not yet eliminated (two groups of <= 128) ----
    const int g0[2] = {k0 + kPanel, kRows};
    const int gN[2] = {kRows - (k0 + kPanel), kCols - kRows};
#pragma unroll 1
    for (int g = 0; g < 2; ++g) {
      const int N = gN[g];
      if (N <= 0) continue;
      // B[col][c] = R[p_c][g0 + col]: the pivot rows write their values
#pragma unroll 1
      for (int q = 0; q < N / 32; ++q) {
        float r[32];
        tmem_ld32(tmem + lane_base + (uint32_t)(g0[g] + q * 32), r);
        if (mine >= 0) {
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const float x = r[k];
            const float xh = __uint_as_float(to_tf32(x));
            const uint32_t off = op_offset(q * 32 + k, mine);
            *(float*)((char*)B_hi + off) = xh;
            *(float*)((char*)B_lo + off) = __uint_as_float(to_tf32(x - xh));
          }
        }
      }
      fence_async_smem();
      fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        fence_after_sync();
        const uint32_t idesc = idesc_tf32(N);
        const uint32_t d = tmem + (uint32_t)g0[g];
        const uint32_t ah = smem_addr(A_hi), al = smem_addr(A_lo), bh = smem_addr(B_hi), bl = smem_addr(B_lo);
#pragma unroll
        for (int s = 0; s < kPanel / 8; ++s) {   // K = 8 per instruction: two 4-element core matrices
          const uint32_t ko = (uint32_t)s * 256;
          mma_tf32(d, smem_desc(ah + ko, 128, 1024), smem_desc(bh + ko, 128, 1024), idesc, 1);
          mma_tf32(d, smem_desc(ah + ko, 128, 1024), smem_desc(bl + ko, 128, 1024), idesc, 1);
          mma_tf32(d, smem_desc(al + ko, 128, 1024), smem_desc(bh + ko, 128, 1024), idesc, 1);
        }
        mma_commit(S.mbar);
      }
      const bool done = mbar_wait(S.mbar, *phase);
      *phase ^= 1u;
      if (__syncthreads_or(!done)) ok = false;   // the same decision in every thread
      fence_after_sync();
      if (!ok) break;
    }
    if (!ok) break;
  }
  // ---- right half -> RT[j][c] = G^-1[c][j] (row p_c of the right half is row c of G^-1) ----
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (ok) {
#pragma unroll 1
    for (int q = 0; q < kRows / 32; ++q) {
      float r[32];
      tmem_ld32(tmem + lane_base + (uint32_t)(kRows + q * 32), r);
      if (my_col >= 0 && my_col < n) {
#pragma unroll
        for (int k = 0; k < 32; ++k) S.op[(q * 32 + k) * kRows + my_col] = r[k];
      }
    }
  }
  __syncthreads();
  return ok;
}

// ---------------------------------------------------------------------------
// Multi-tile inverse for 128 < n <= 512 components (MT = 2 or 4 row tiles of
// 128, MT x 128 threads, thread i owns row i).  The matrix no longer fits on
// the SM, so it is inverted in place in global memory (L2), FP32, column-major
// with leading dimension Np = 128 MT: R[c * Np + i].
//
// In-place Gauss-Jordan with implicit row pivoting: when panel column c is
// eliminated with pivot row p_c, its storage slot takes over the augmented
// column of p_c, which before the panel is the unit vector e_{p_c} and after
// it e_{p_c} + W[:, k] (k: c's place in the panel).  Every other slot
// (columns still to eliminate, and the slots already taken over) gets the
// panel's rank-32 update R + W R[P].  After the last panel, slot s holds
// column p_s of E G^-1 (E: the pivot permutation, row p_a of E G^-1 is row a
// of G^-1), so
//     G^-1[a][b] = R[c(b) * Np + p_a]      (c(b): the column row b was pivot of)
// and a solve is x_a = y_{p_a} with y = R r~, r~_s = r_{p_s}.
//
// Schedule per panel: the 32 panel columns are read into registers and
// eliminated on the CUDA cores as in gj_inverse (pivot search over all rows
// through shared memory); the coefficients W (Np x 32) go to shared memory as
// split-TF32 A operands, one per row tile.  Then the columns are updated in
// chunks of 128: each thread stores its row of the chunk into its warpgroup's
// 128 TMEM columns (warpgroup g = row tile g), the pivot rows write R[P] for
// the chunk as the B operand, one thread issues the MT x 4 x 3 MMAs
// (M = 128, N = 128, K = 8 each), and the rows are read back and stored, the
// panel's own slots replaced by e_{p_c} + W[:, k].  TMEM: MT x 128 columns.
// ---------------------------------------------------------------------------
struct SmemL {
  float* A;       // MT x {hi, lo} operands of 128 x 32 (16 KB each), 1024-byte aligned
  float* B;       // {hi, lo} operands of 128 (N) x 32 (K)
  float* red;     // [2][16] warp maxima
  int* redi;      // [2][16]
  float* prow;    // [2][2 * kPanel]
  int* piv;       // [Np] pivot row of column c (persistent: the solves use it)
  int* colof;     // [Np] column row i was pivot of, -1 none (persistent)
  unsigned long long* mbar;
};

template <int MT>
__device__ __noinline__ bool gj_inverse_large(const double* __restrict__ J, int jld, int n, double hr0,
                                              float* __restrict__ R, const SmemL& S, uint32_t tmem,
                                              uint32_t* phase) {
  constexpr int BT = MT * 128, NP = BT, NW = BT / 32;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wg = tid >> 7, r128 = tid & 127;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t col_base = (uint32_t)(wg * 128);
  // G = I - hr0 J, padded with the identity, row tid of every column
#pragma unroll 4
  for (int c = 0; c < NP; ++c) {
    float g;
    if (tid < n && c < n) {
      double x = -hr0 * J[(long)c * jld + tid];
      if (c == tid) x += 1.;
      g = (float)x;
    } else {
      g = c == tid ? 1.f : 0.f;
    }
    R[(long)c * NP + tid] = g;
  }
  S.colof[tid] = -1;
  S.piv[tid] = tid;
  bool pivoted = false;
  bool ok = true;
  const int npanels = (n + kPanel - 1) / kPanel;
  const int nchunks = (n + 127) / 128;
#pragma unroll 1
  for (int pn = 0; pn < npanels; ++pn) {
    const int k0 = pn * kPanel;
    __syncthreads();   // the previous panel's stores of R are visible to the block
    float v[32], u[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = R[(long)(k0 + k) * NP + tid];
#pragma unroll
    for (int k = 0; k < 32; ++k) u[k] = 0.f;
    int mine = -1;
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      const int buf = c & 1;
      float best = pivoted ? -1.f : fabsf(v[c]);
      if (best != best) best = 0.f;
      int brow = tid;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
        if (ob > best || (ob == best && orow < brow)) { best = ob; brow = orow; }
      }
      if (lane == 0) { S.red[buf * 16 + warp] = best; S.redi[buf * 16 + warp] = brow; }
      __syncthreads();
      float pb = S.red[buf * 16];
      int prow_i = S.redi[buf * 16];
#pragma unroll
      for (int w = 1; w < NW; ++w) {
        const float ob = S.red[buf * 16 + w];
        const int orow = S.redi[buf * 16 + w];
        if (ob > pb || (ob == pb && orow < prow_i)) { pb = ob; prow_i = orow; }
      }
      float* pr = S.prow + buf * 2 * kPanel;
      if (tid == prow_i) {
        const float a = v[c];
        const float inv = a != 0.f ? 1.f / a : 0.f;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k > c) v[k] *= inv;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k < c) u[k] *= inv;
        u[c] = inv - 1.f;
        v[c] = 1.f;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (k > c) pr[k] = v[k];
          if (k <= c) pr[kPanel + k] = u[k] + (k == c ? 1.f : 0.f);
        }
        pivoted = true;
        mine = c;
      }
      __syncthreads();
      if (tid != prow_i) {
        const float m = v[c];
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          if (k > c) v[k] = fmaf(-m, pr[k], v[k]);
          if (k <= c) u[k] = fmaf(-m, pr[kPanel + k], u[k]);
        }
        v[c] = 0.f;
      }
    }
    if (mine >= 0) {
      S.colof[tid] = k0 + mine;
      S.piv[k0 + mine] = tid;
    }
    // A operand of row tile wg: this row's coefficients, split into TF32 hi and lo
    {
      char* ah = (char*)(S.A + (size_t)(2 * wg) * kOperandFloats);
      char* al = (char*)(S.A + (size_t)(2 * wg + 1) * kOperandFloats);
#pragma unroll
      for (int kg = 0; kg < 8; ++kg) {
        float4 hi, lo;
        float* h4 = &hi.x;
        float* l4 = &lo.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float x = u[kg * 4 + e];
          const float xh = __uint_as_float(to_tf32(x));
          h4[e] = xh;
          l4[e] = __uint_as_float(to_tf32(x - xh));
        }
        *(float4*)(ah + op_offset(r128, kg * 4)) = hi;
        *(float4*)(al + op_offset(r128, kg * 4)) = lo;
      }
    }
    float* const B_hi = S.B;
    float* const B_lo = S.B + kOperandFloats;
#pragma unroll 1
    for (int ch = 0; ch < nchunks; ++ch) {
      const int c0 = ch * 128;
      // the chunk of this row into TMEM; the pivot rows also write it as the B operand
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {
        float r[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) r[k] = R[(long)(c0 + q * 32 + k) * NP + tid];
        if (mine >= 0) {
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const float x = r[k];
            const float xh = __uint_as_float(to_tf32(x));
            const uint32_t off = op_offset(q * 32 + k, mine);
            *(float*)((char*)B_hi + off) = xh;
            *(float*)((char*)B_lo + off) = __uint_as_float(to_tf32(x - xh));
          }
        }
        tmem_st32(tmem + lane_base + col_base + (uint32_t)(q * 32), r);
      }
      tmem_wait_st();
      fence_async_smem();
      fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        fence_after_sync();
        const uint32_t idesc = idesc_tf32(128);
        const uint32_t bh = smem_addr(B_hi), bl = smem_addr(B_lo);
#pragma unroll 1
        for (int g = 0; g < MT; ++g) {
          const uint32_t d = tmem + (uint32_t)(g * 128);
          const uint32_t ah = smem_addr(S.A + (size_t)(2 * g) * kOperandFloats);
          const uint32_t al = smem_addr(S.A + (size_t)(2 * g + 1) * kOperandFloats);
#pragma unroll
          for (int s = 0; s < kPanel / 8; ++s) {
            const uint32_t ko = (uint32_t)s * 256;
            mma_tf32(d, smem_desc(ah + ko, 128, 1024), smem_desc(bh + ko, 128, 1024), idesc, 1);
            mma_tf32(d, smem_desc(ah + ko, 128, 1024), smem_desc(bl + ko, 128, 1024), idesc, 1);
            mma_tf32(d, smem_desc(al + ko, 128, 1024), smem_desc(bh + ko, 128, 1024), idesc, 1);
          }
        }
        mma_commit(S.mbar);
      }
      const bool done = mbar_wait(S.mbar, *phase);
      *phase ^= 1u;
      if (__syncthreads_or(!done)) ok = false;
      fence_after_sync();
      if (!ok) break;
      // back to R; the panel's slots take over the augmented columns of their pivot rows
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {
        float r[32];
        tmem_ld32(tmem + lane_base + col_base + (uint32_t)(q * 32), r);
        const bool panel = c0 + q * 32 == k0;   // these 32 columns are the panel's (k0 is a multiple of 32)
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const int col = c0 + q * 32 + k;
          const float x = panel ? u[k] + (S.piv[col] == tid ? 1.f : 0.f) : r[k];
          R[(long)col * NP + tid] = x;
        }
      }
      fence_before_sync();
      __syncthreads();   // every warp has read its TMEM columns before the next chunk overwrites them
      fence_after_sync();
    }
    if (!ok) break;
  }
  __syncthreads();
  return ok;
}

}  // namespace tc
}  // namespace lsg
