// Blackwell tensor-core primitives (tcgen05 + TMEM) for split-precision
// (3xTF32) products of small matrices.
//
// Operand tiles live in shared memory in the K-major, non-swizzled
// ("interleaved") canonical layout of the tcgen05 matrix descriptors: core
// matrices of 8 rows x 16 bytes (4 TF32 values), the K-chunks of a row group
// stored one after another.  For a tile with K = 32 (8 chunks) element
// (row r, k) is at float offset
//     (r / 8) * 256 + (k / 4) * 32 + (r % 8) * 4 + (k % 4)
// so a row group spans 1024 bytes (SBO) and neighbouring K-chunks are 128
// bytes apart (LBO).  One MMA consumes K = 8 (two chunks): the descriptor of
// k-step s starts 256 * s bytes into the tile.  Both operands use it: the MMA
// forms D = A * B^T with A (M x K) and B (N x K) stored row by row.  A thread
// writing one row stores 8 float4 and a quarter warp covers 128 contiguous
// bytes, so row writes are free of bank conflicts; a warp whose lanes hold
// columns transposes them in registers first (warp_transpose32).

// A product X * Y with FP32 operands is formed as
//     X_hi Y_hi + X_hi Y_lo + X_lo Y_hi,   X_hi = X truncated to TF32, X_lo = X - X_hi
// with FP32 accumulation in tensor memory (see split()).
#pragma once
#include <cstdint>

namespace pb {
namespace tc {

constexpr int TILE_K = 32;               // K extent of every operand tile
constexpr int RG_FLOATS = 256;           // floats per 8-row group of an A tile (8 chunks x 32)
// instruction descriptors: D = F32, A = B = TF32, both K-major, M = 128, N = 32, 64 or 128
constexpr uint32_t idesc_tf32(uint32_t m, uint32_t n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}
constexpr uint32_t IDESC_M128_N32 = idesc_tf32(128, 32);
constexpr uint32_t IDESC_M128_N64 = idesc_tf32(128, 64);
constexpr uint32_t IDESC_M128_N128 = idesc_tf32(128, 128);
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 24;  // bounded waits on MMA completion

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor (no swizzle, sm_100 version 1)
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}
__device__ __forceinline__ uint64_t desc_k(uint32_t addr) { return desc(addr, 128, 1024); }

// hi = x truncated to TF32 (its top 19 bits, one logic operation), lo = x -
// hi (exact in FP32); the tensor core reads only the TF32 bits of lo, so lo
// needs no conversion.  Each operand then carries about 2^-20 relative error,
// the size of the dropped lo * lo term.  (Rounding both halves with
// cvt.rna.tf32 is 2^-22 but costs two conversions per element: the doubling
// kernels are bound by this CUDA-core work, not by the tensor pipe.)
__device__ __forceinline__ void split(float x, float& hi, float& lo) {
  hi = __uint_as_float(__float_as_uint(x) & 0xffffe000u);
  lo = x - hi;
}

// As split(), with hi rounded to the nearest TF32 value (half an ulp of the
// 10-bit mantissa added to the bit pattern before the low 13 bits are
// cleared: ties away from zero, one more integer operation).  lo = x - hi is
// then of either sign, |lo| <= 2^-11 |x|, so the tensor core's truncation of
// lo errs without bias.  Used by the adding, whose errors accumulate over a
// long chain of combines (about half the TB error of the truncating split
// there, measured), while in the doubling the extra operation cost more
// (2.4 % of the split layer stage) than it gained.
__device__ __forceinline__ void split_rn(float x, float& hi, float& lo) {
  hi = __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
  lo = x - hi;
}

// D[tmem] (+)= A * B^T over K = 8 from the given descriptors (one thread)
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                    uint32_t idesc = IDESC_M128_N32) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// 3xTF32 product of a 128 x 32 A tile pair and an N x 32 B tile pair into
// D = A * B^T (128 lanes x N columns, FP32; N = 32 or 64 by `idesc`).  Issued
// by one thread; completion is signalled on `mbar` through tcgen05.commit.
__device__ __forceinline__ void mma3(uint32_t d_tmem, const float* a_hi, const float* a_lo, const float* b_hi,
                                     const float* b_lo, uint64_t* mbar, uint32_t idesc = IDESC_M128_N32) {
  const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
  uint32_t acc = 0;
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) {
    mma(d_tmem, desc_k(al + 256 * s), desc_k(bh + 256 * s), acc, idesc);
    acc = 1;
  }
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) mma(d_tmem, desc_k(ah + 256 * s), desc_k(bl + 256 * s), 1, idesc);
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) mma(d_tmem, desc_k(ah + 256 * s), desc_k(bh + 256 * s), 1, idesc);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(mbar))
               : "memory");
}

// D[tmem] (+)= A * B^T over K = 8 with A read from tensor memory (lanes =
// rows of A, one TF32 value per column) and B from shared memory (one thread)
__device__ __forceinline__ void mma_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t accumulate,
                                       uint32_t idesc) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate));
}

// 3xTF32 product with the A pair in tensor memory (columns a_hi..a_hi+31 and
// a_lo..a_lo+31 of lanes 0..127) and the B pair in shared memory:
// D = A * B^T, small terms first.  One thread; completion on `mbar`.
__device__ __forceinline__ void mma3_ta(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, const float* b_hi,
                                        const float* b_lo, uint64_t* mbar, uint32_t idesc) {
  const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) mma_ta(d_tmem, a_lo + 8 * s, desc_k(bh + 256 * s), s > 0, idesc);
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) mma_ta(d_tmem, a_hi + 8 * s, desc_k(bl + 256 * s), 1, idesc);
#pragma unroll
  for (int s = 0; s < TILE_K / 8; s++) mma_ta(d_tmem, a_hi + 8 * s, desc_k(bh + 256 * s), 1, idesc);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for phase `parity` of `mbar` to complete; false after `limit` polls
// (a limit of 0 gives up without polling).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit = MBAR_SPIN_LIMIT) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// generic-proxy shared-memory writes -> visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Allocate / free tensor-memory columns (whole warp).  The base address is
// written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :
               : "r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's lane (warp w reads lanes
// 32w..32w+31; taddr carries the lane base in bits 16..31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// As tmem_ld32 without the wait: the 32 registers are valid only after
// tmem_wait_ld(v) on the same array, which names them as its operands so that
// no use of them is scheduled before it.  Both are whole-warp instructions.
__device__ __forceinline__ void tmem_ld32_issue(uint32_t taddr, float (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
        "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]),
        "=f"(v[16]), "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]),
        "=f"(v[24]), "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(float (&v)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                 "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                 "+f"(v[15]), "+f"(v[16]), "+f"(v[17]), "+f"(v[18]), "+f"(v[19]), "+f"(v[20]), "+f"(v[21]),
                 "+f"(v[22]), "+f"(v[23]), "+f"(v[24]), "+f"(v[25]), "+f"(v[26]), "+f"(v[27]), "+f"(v[28]),
                 "+f"(v[29]), "+f"(v[30]), "+f"(v[31])
               :
               : "memory");
}

// Store 32 FP32 values into 32 consecutive columns of this thread's lane
// (warp w writes lanes 32w..32w+31), and wait for the stores to complete.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
      :
      : "r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
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
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// tmem_st32 without its wait, and the wait for two such stores: it names
// both source arrays as operands, so they stay live and unchanged until the
// stores have completed.
__device__ __forceinline__ void tmem_st32_issue(uint32_t taddr, const float (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
      :
      : "r"(taddr), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]),
        "f"(v[8]), "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]),
        "f"(v[16]), "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]),
        "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st2(float (&v)[32], float (&w)[32]) {
  asm volatile("tcgen05.wait::st.sync.aligned;"
               : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7]),
                 "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]), "+f"(v[12]), "+f"(v[13]), "+f"(v[14]),
                 "+f"(v[15]), "+f"(v[16]), "+f"(v[17]), "+f"(v[18]), "+f"(v[19]), "+f"(v[20]), "+f"(v[21]),
                 "+f"(v[22]), "+f"(v[23]), "+f"(v[24]), "+f"(v[25]), "+f"(v[26]), "+f"(v[27]), "+f"(v[28]),
                 "+f"(v[29]), "+f"(v[30]), "+f"(v[31]), "+f"(w[0]), "+f"(w[1]), "+f"(w[2]), "+f"(w[3]),
                 "+f"(w[4]), "+f"(w[5]), "+f"(w[6]), "+f"(w[7]), "+f"(w[8]), "+f"(w[9]), "+f"(w[10]),
                 "+f"(w[11]), "+f"(w[12]), "+f"(w[13]), "+f"(w[14]), "+f"(w[15]), "+f"(w[16]), "+f"(w[17]),
                 "+f"(w[18]), "+f"(w[19]), "+f"(w[20]), "+f"(w[21]), "+f"(w[22]), "+f"(w[23]), "+f"(w[24]),
                 "+f"(w[25]), "+f"(w[26]), "+f"(w[27]), "+f"(w[28]), "+f"(w[29]), "+f"(w[30]), "+f"(w[31])
               :
               : "memory");
}

// Write one 32-value row of a tile pair (hi, lo) from FP32 values.
__device__ __forceinline__ void put_row(float* hi, float* lo, int r, const float (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 8; c++) {
    float4 h, l;
    split(v[4 * c + 0], h.x, l.x);
    split(v[4 * c + 1], h.y, l.y);
    split(v[4 * c + 2], h.z, l.z);
    split(v[4 * c + 3], h.w, l.w);
    const int o = (r >> 3) * RG_FLOATS + c * 32 + (r & 7) * 4;
    *reinterpret_cast<float4*>(hi + o) = h;
    *reinterpret_cast<float4*>(lo + o) = l;
  }
}

// In-register transpose across a warp: lane L holding v[i] = M[i][L] ends
// holding v[i] = M[L][i].  Five butterfly stages exchange the bit b of the
// lane index with the bit b of the register index (16 shuffles each).
__device__ __forceinline__ void warp_transpose32(float (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int b = 16; b >= 1; b >>= 1) {
    const bool upper = (lane & b) != 0;
#pragma unroll
    for (int i = 0; i < 32; i++) {
      if ((i & b) == 0) {
        const int j = i | b;
        const float send = upper ? v[i] : v[j];
        const float recv = __shfl_xor_sync(0xffffffffu, send, b);
        if (upper) v[i] = recv;
        else v[j] = recv;
      }
    }
  }
}

// Whole warp: lane L holds column L of a 32 x 32 matrix X; write X row by
// row into a tile pair (row n = X[n][:]).  `v` is transposed in place.
__device__ __forceinline__ void put_rows_from_cols(float* hi, float* lo, float (&v)[32]) {
  warp_transpose32(v);
  put_row(hi, lo, threadIdx.x & 31, v);
}

}  // namespace tc
}  // namespace pb
