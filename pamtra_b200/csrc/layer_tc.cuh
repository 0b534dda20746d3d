// Split-precision layer stage of the batched form (NUMMU = 16, n = 32): the
// scatcnv / CHECK_NORM4 / INITIALIZE4 / INITIAL_SOURCE4 part is the FP64 code
// of k_layer; the DOUBLING_INTEGRATION4 loop (src/radintg4.f90:174-309,
// SYMMETRIC) runs its matrix products as 3xTF32 tcgen05 MMAs with FP32
// accumulation in tensor memory.
//
// FP32 cannot hold a thin layer's transmission T = I - T~ (|T~| ~ 1e-6) to
// useful relative accuracy, so the loop carries the deviations
//     T~ = I - T,   G~ = G - I,   G = (I - R R)^-1
// and adds identity parts exactly in the epilogues:
//     P  = R R                     V  = R - R T~          (= R T)
//     G~ = P + P^2 + ...   repeated squaring from G~ = 0, X = P:
//                          G~' = G~ + X + X G~,  X' = X X
//     Y  = V + G~ V                Z~ = T~ - G~ + G~ T~   (G T = I - Z~)
//     R' = R + Y - T~ Y            T~' = T~ + Z~ - T~ Z~
// Sources follow the FP64 kernel (R v, G u = u + G~ u, T w = w - T~ w) as
// FP32 matrix-vector products on the CUDA cores, overlapped with the MMAs.
//
// Pairing.  One CTA (4 warps) carries two (layer, frequency) items through
// their doublings in lockstep, and every MMA serves both: with D = A B^T,
//     A = [Y1a^T; Y1b^T; Y2a^T; Y2b^T]   (128 rows: columns of the right factors)
//     B = [X1; X2]                        (64 rows: rows of each item's left factor)
// lane 64i + 32p + m of D, columns 32i..32i+31, is column m of X_i Y_ip.  The
// off-diagonal blocks (X1 Y2a, ...) are computed and ignored, so each item's
// results depend on its own operands only: the pairing does not change any
// value.  Warp 2i + p owns the lanes of product p of item i, so every warp
// does the same kind of work (no idle warps, no divergent roles inside a warp).
// An item that has finished its doublings (or its series steps) while its
// partner goes on keeps its state and skips its epilogues.  M = 128, N = 64,
// K = 32: no row of the MMA is padding.
#pragma once
#include "rt.cuh"
#include "tc.cuh"

namespace pb {

// FP32 masters: 32 x 32, column-major with the 4-float chunks of column c
// XOR-swizzled by c mod 8, so a quarter warp reading one chunk of eight
// neighbouring columns (column loads) and a warp reading one row-slice of a
// column (row loads, mat-vecs) both hit 32 distinct banks without padding.
__device__ __forceinline__ int midx(int r, int c) { return c * 32 + ((((r >> 2) ^ (c & 7)) << 2) | (r & 3)); }

// The eight in-column offsets of row r (one per value of c mod 8): element
// (r, c) sits at c * 32 + off[c & 7].  A thread reading a whole row computes
// them once instead of swizzling every address.
struct RowOff {
  int o[8];
  __device__ __forceinline__ explicit RowOff(int r) {
#pragma unroll
    for (int j = 0; j < 8; j++) o[j] = (((r >> 2) ^ j) << 2) | (r & 3);
  }
};

// FP32 layer record of one (present layer, frequency) item (in its w.lay slot),
// read by the split-precision adding (k_adding_tc): R, T, S+, S-
constexpr int LAY32_R = 0, LAY32_T = 1024, LAY32_SP = 2048, LAY32_SM = 2080, LAY32_FLOATS = 2112;

// storage index s of a swizzled master -> (row, column)
__device__ __forceinline__ void midx_inv(int s, int& r, int& c) {
  c = s >> 5;
  const int p = s & 31;
  r = ((((p >> 2) ^ (c & 7))) << 2) | (p & 3);
}

// Write the FP32 layer record from FP64 R, T (column-major, leading dimension
// LD) and the sources lin (S+ then S-), with T threads.
template <int LD, int T>
__device__ __forceinline__ void lay32_store(const Work& w, int item, const double* R, const double* Tm_,
                                            const double* lin) {
  float* rec = reinterpret_cast<float*>(w.lay + (size_t)item * w.lay_stride);
  for (int s = threadIdx.x; s < 1024; s += T) {
    int r, c;
    midx_inv(s, r, c);
    rec[LAY32_R + s] = (float)R[c * LD + r];
    rec[LAY32_T + s] = (float)Tm_[c * LD + r];
  }
  for (int e = threadIdx.x; e < 64; e += T) rec[LAY32_SP + e] = (float)lin[e];
}

// FP32 state of one item of the pair.
struct TcItemState {
  float rm[1024], tm[1024], gm[1024];    // R, T~, G~
  float vm[1024];                        // V = R T, then Y = G R T
  float xa[1024];                        // series power X, then Z~
  float src[4][32];                      // S+ linear, S+ constant, S- linear, S- constant
  float vv[4][32], uv[4][32], wv[4][32]; // right-hand vectors of the three groups
  float nrm;
  int pad_[3];
};

struct TcTiles {
  float b_hi[64 * 32], b_lo[64 * 32];  // B tile pair (64 rows: 32 per item); the A pair lives in TMEM
};

// FP64 set-up scratch of one item (layer_setup): thin-layer R and T,
// Legendre coefficients, azimuth table, quadrature and sources.
struct TcSetupSmem {
  static constexpr int n = 32, MAT = RTCfg<16>::MAT;
  double r[MAT], t[MAT];
  double coef[3 * MAXNLEG];
  double az[2 * KMAX];
  double lin[2 * n], cst[2 * n];
  double mu[16], wq[16], nrm[16];
  int item, stat;
  __device__ __forceinline__ double* mat(int i) { return i == 0 ? r : i == 1 ? t : i == 4 ? az : coef; }
};

union __align__(128) TcScratch {
  TcTiles tl;
  TcSetupSmem setup;  // the FP64 set-up of one item at a time
};

struct TcPairSmem {
  TcItemState st[2];
  TcScratch u;
};
static_assert(sizeof(TcItemState) % 16 == 0, "tile alignment");

constexpr float NEUMANN_TOL = 1.0e-8f;  // truncation of G~ relative to its size
constexpr float NEUMANN_MAX_NORM = 0.75f;

template <int N>
constexpr size_t layer_tc_smem() {
  return sizeof(TcPairSmem);
}

// thread-owned column helpers of the masters
__device__ __forceinline__ void ld_col(const float* m, int col, float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4) {
    const float4 q = *reinterpret_cast<const float4*>(m + midx(r, col));
    v[r] = q.x; v[r + 1] = q.y; v[r + 2] = q.z; v[r + 3] = q.w;
  }
}
__device__ __forceinline__ void st_col(float* m, int col, const float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4)
    *reinterpret_cast<float4*>(m + midx(r, col)) = make_float4(v[r], v[r + 1], v[r + 2], v[r + 3]);
}

// Operands of one group for the calling thread, split into TF32 hi / lo
// pairs: its A row (column `lane` of master `asrc`) into its own TMEM lane
// at columns ta_hi / ta_lo, and K-chunks 4h..4h+3 of B row `brow` (row
// `lane` of master `bsrc`, read down its columns: conflict-free) into shared
// memory.  The two warps of an item cover the B row's two halves.
__device__ __forceinline__ void build_operands(TcTiles& TL, const float* asrc, const float* bsrc, uint32_t ta_hi,
                                               uint32_t ta_lo, int brow, int h, int lane, const RowOff& ro) {
  // the A stores run while the B half is built; their wait comes last
  float c[32], lo[32];
  ld_col(asrc, lane, c);
#pragma unroll
  for (int r = 0; r < 32; r++) tc::split(c[r], c[r], lo[r]);
  tc::tmem_st32_issue(ta_hi, c);
  tc::tmem_st32_issue(ta_lo, lo);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k0 = 16 * h + 4 * q;
    float4 bh, bl;
    const float* bc = bsrc + k0 * 32;  // k0 = 16 h + 4 q: (k0 + j) mod 8 = (4 q + j) mod 8
    tc::split(bc[0 * 32 + ro.o[(4 * q + 0) & 7]], bh.x, bl.x);
    tc::split(bc[1 * 32 + ro.o[(4 * q + 1) & 7]], bh.y, bl.y);
    tc::split(bc[2 * 32 + ro.o[(4 * q + 2) & 7]], bh.z, bl.z);
    tc::split(bc[3 * 32 + ro.o[(4 * q + 3) & 7]], bh.w, bl.w);
    const int o = (brow >> 3) * tc::RG_FLOATS + (k0 >> 2) * 32 + (brow & 7) * 4;
    *reinterpret_cast<float4*>(TL.b_hi + o) = bh;
    *reinterpret_cast<float4*>(TL.b_lo + o) = bl;
  }
  tc::tmem_wait_st2(c, lo);
}

// (M x0)[r] and (M x1)[r] for a master M (k-ascending FMA chains)
__device__ __forceinline__ void matvec2(const float* __restrict__ M, const float* __restrict__ x0,
                                        const float* __restrict__ x1, const RowOff& ro, float& y0, float& y1) {
  float a0 = 0.f, a1 = 0.f;
#pragma unroll
  for (int k = 0; k < 32; k += 4) {
    const float4 p = *reinterpret_cast<const float4*>(x0 + k);
    const float4 q = *reinterpret_cast<const float4*>(x1 + k);
    const float m0 = M[k * 32 + ro.o[k & 7]], m1 = M[(k + 1) * 32 + ro.o[(k + 1) & 7]];
    const float m2 = M[(k + 2) * 32 + ro.o[(k + 2) & 7]], m3 = M[(k + 3) * 32 + ro.o[(k + 3) & 7]];
    a0 = fmaf(m0, p.x, a0); a1 = fmaf(m0, q.x, a1);
    a0 = fmaf(m1, p.y, a0); a1 = fmaf(m1, q.y, a1);
    a0 = fmaf(m2, p.z, a0); a1 = fmaf(m2, q.z, a1);
    a0 = fmaf(m3, p.w, a0); a1 = fmaf(m3, q.w, a1);
  }
  y0 = a0;
  y1 = a1;
}

// (M x0..x3)[r] for a master M, one row load for four vectors (k-ascending
// FMA chains, each bit-identical to matvec2's)
__device__ __forceinline__ void matvec4(const float* __restrict__ M, const float (*__restrict__ x)[32],
                                        const RowOff& ro, float (&y)[4]) {
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
  for (int k = 0; k < 32; k += 4) {
    const float4 p = *reinterpret_cast<const float4*>(x[0] + k);
    const float4 q = *reinterpret_cast<const float4*>(x[1] + k);
    const float4 r = *reinterpret_cast<const float4*>(x[2] + k);
    const float4 v = *reinterpret_cast<const float4*>(x[3] + k);
    const float m0 = M[k * 32 + ro.o[k & 7]], m1 = M[(k + 1) * 32 + ro.o[(k + 1) & 7]];
    const float m2 = M[(k + 2) * 32 + ro.o[(k + 2) & 7]], m3 = M[(k + 3) * 32 + ro.o[(k + 3) & 7]];
    a0 = fmaf(m0, p.x, a0); a1 = fmaf(m0, q.x, a1); a2 = fmaf(m0, r.x, a2); a3 = fmaf(m0, v.x, a3);
    a0 = fmaf(m1, p.y, a0); a1 = fmaf(m1, q.y, a1); a2 = fmaf(m1, r.y, a2); a3 = fmaf(m1, v.y, a3);
    a0 = fmaf(m2, p.z, a0); a1 = fmaf(m2, q.z, a1); a2 = fmaf(m2, r.z, a2); a3 = fmaf(m2, v.z, a3);
    a0 = fmaf(m3, p.w, a0); a1 = fmaf(m3, q.w, a1); a2 = fmaf(m3, r.w, a2); a3 = fmaf(m3, v.w, a3);
  }
  y[0] = a0; y[1] = a1; y[2] = a2; y[3] = a3;
}

// Series plan for ||X|| = nrm (any sub-multiplicative norm), by the relative
// remainder it leaves: s >= 1 repeated squaring in s + 1 MMAs (remainder
// nrm^(2^(s+1) - 1)), 0: G~ = X (nrm), SERIES_H1: G~ = X + X X in one MMA
// (nrm^2), -1: the FP64 fallback.
constexpr int SERIES_H1 = -3;
__device__ __forceinline__ int series_steps(float nrm) {
  if (!(nrm < NEUMANN_MAX_NORM)) return -1;
  if (nrm > NEUMANN_TOL && nrm * nrm <= NEUMANN_TOL) return SERIES_H1;
  float pw = nrm;  // nrm^(2^(s+1) - 1)
  float pk = nrm;  // nrm^(2^s)
  int s = 0;
  while (pw > NEUMANN_TOL && s < 6) {
    pk = pk * pk;
    pw = pw * pk;
    s++;
  }
  return s;
}

// An item a CTA takes after one of its waits on the tensor core gave up: its
// (column, frequency) gets PAMTRA_B200_ST_TIMEOUT and no layer is computed.
template <int N>
__device__ __forceinline__ void mark_timed_out(const Batch& b, const Work& w, int item) {
  const int Fm = b.max_nfreq, Lm = b.max_nlyrs;
  const int p = item / Fm, fi = item % Fm;
  const int c = w.plist[p] / Lm;
  if (fi < b.col_nfreq(c) && b.col_nummu(c) == N) {
    w.lay_nd[item] = 0;
    atomicOr(&w.status[(size_t)c * Fm + fi], PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT);
  }
}

template <int N>
__global__ void __launch_bounds__(128, 3) k_layer_tc(Batch b, Work w, pamtra_b200_settings st,
                                                     double* __restrict__ ssp_scat) {
  static_assert(N == 16, "the split-precision layer kernel is built for NUMMU = 16");
  constexpr int n = 32, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT;
  enum { G1 = 0, SER = 1, G2 = 2, G3 = 3 };
  extern __shared__ __align__(1024) double smem_raw[];
  TcPairSmem& Q = *reinterpret_cast<TcPairSmem*>(smem_raw);
  TcSetupSmem& S = Q.u.setup;
  TcTiles& TL = Q.u.tl;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_base, s_dead;
  __shared__ int s_valid[2], s_nd[2], s_status[2], s_c[2], s_fi[2];
  __shared__ float s_linfac[2];
  __shared__ float s_mv[2][32];  // item 0, slot 0: its mat-vec results, computed by warp 1
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int mi = warp >> 1, slot = warp & 1;  // my item of the pair, my product
  TcItemState& my = Q.st[mi];
  const int Fm = b.max_nfreq;
  const int P = min(w.counters[0], w.pmax);
  const int nitems = P * Fm;
  scat_weights_mark_ready<N>(w);
  if (warp == 0) tc::tmem_alloc(&tslot, 128);  // D: columns 0..63, A hi: 64..95, A lo: 96..127
  if (t == 0) {
    tc::mbar_init(&mbar, 1);
    s_dead = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t lanes = (uint32_t)(warp * 32) << 16;  // A row = D lane of this thread
  const uint32_t dmine = tslot + lanes + 32u * mi;       // my lanes, my item's columns of D
  const int brow = 32 * mi + lane;                       // B row of my item for my lane
  const RowOff rowoff(lane);                             // my row of the masters
  uint32_t parity = 0;

  for (;;) {
    __syncthreads();
    if (t == 0) s_base = atomicAdd(&w.counters[3], 2);
    __syncthreads();
    const int base = s_base;
    if (base >= nitems) break;
    if (s_dead) {  // after a timed-out wait: report the remaining items, compute nothing
      if (t < 2 && base + t < nitems) mark_timed_out<N>(b, w, base + t);
      continue;
    }
    // ---- FP64 set-up of both items (one at a time through the shared scratch)
    for (int i = 0; i < 2; i++) {
      const int item = base + i;
      if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
      __syncthreads();
      LayerItem it;
      const bool valid = item < nitems && layer_setup<N>(b, w, st, ssp_scat, S, item, it);
      if (valid && it.nd == 0) {
        if (w.lay32) lay32_store<LD, 128>(w, item, S.r, S.t, S.lin);
        else layer_store<N>(w, item, S.r, S.t, S.lin);
      } else if (valid) {
        TcItemState& D = Q.st[i];
        for (int e = t; e < n * n; e += 128) {
          const int cc = e >> 5, r = e & 31;
          D.rm[midx(r, cc)] = (float)S.r[cc * LD + r];
          D.tm[midx(r, cc)] = (float)((r == cc ? 1.0 : 0.0) - S.t[cc * LD + r]);
        }
        if (t < n) {
          D.src[0][t] = (float)S.lin[t];
          D.src[1][t] = (float)S.cst[t];
          D.src[2][t] = (float)S.lin[n + t];
          D.src[3][t] = (float)S.cst[n + t];
        }
      }
      if (t == 0) {
        s_valid[i] = valid;
        s_nd[i] = valid ? it.nd : 0;
        s_status[i] = valid ? it.status : 0;
        s_linfac[i] = valid ? (float)it.linfac : 0.f;
        s_c[i] = valid ? it.c : 0;
        s_fi[i] = valid ? it.fi : 0;
      }
      __syncthreads();  // the scratch is reused by the next set-up / the tiles
    }
    const int ndmax = max(s_nd[0], s_nd[1]);
    const int my_nd = s_nd[mi];
    float linfac = s_linfac[mi];
    bool ok = true;
    if (ndmax > 0) {
      if (my_nd > 0) {  // v = [S- + f C-, C-, S+, C+]
        if (slot == 0) {
          my.vv[2][lane] = my.src[0][lane];
          my.vv[3][lane] = my.src[1][lane];
        } else {
          my.vv[0][lane] = my.src[2][lane] + linfac * my.src[3][lane];
          my.vv[1][lane] = my.src[3][lane];
        }
      }
      // One MMA group per pass: operands, MMA (with the source mat-vec on the
      // CUDA cores meanwhile), epilogue into the masters, barrier, next phase.
      //   G1  [R; T~] x R   -> slot 0: P = R R  -> X;       slot 1: R T~ -> V = R - R T~
      //   SER [X; G~] x X   -> slot 0: X X      -> X next;  slot 1: X G~ -> G~ += X + X G~
      //   G2  [T~; V] x G~  -> slot 0: G~ T~    -> Z~;      slot 1: G~ V -> Y = V + G~ V
      //   G3  [Z~; Y] x T~  -> slot 0: T~ Z~    -> T~';     slot 1: T~ Y -> R'
      int phase = G1, d = 0, k = 0, mys = 0, myg = 0, gmax = 0;  // series plan, MMAs: mine / the pair's
      for (;;) {
        const bool act = d < my_nd;
        const bool on = (phase == SER) ? (k < myg) : act;
        if (on) {
          const float* asrc;
          const float* bsrc;
          if (phase == G1) { asrc = slot ? my.tm : my.rm; bsrc = my.rm; }
          else if (phase == SER) { asrc = slot ? my.gm : my.xa; bsrc = my.xa; }
          else if (phase == G2) { asrc = slot ? my.vm : my.tm; bsrc = my.gm; }
          else { asrc = slot ? my.vm : my.xa; bsrc = my.tm; }
          build_operands(TL, asrc, bsrc, tslot + lanes + 64u, tslot + lanes + 96u, brow, slot, lane, rowoff);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) tc::mma3_ta(tslot, tslot + 64u, tslot + 96u, TL.b_hi, TL.b_lo, &mbar, tc::IDESC_M128_N64);
        float m0 = 0.f, m1 = 0.f;
        float xk[32];  // slot 1 of a series step: its column of X, taken before slot 0 replaces X
        if (on && phase == SER && slot == 1) ld_col(my.xa, lane, xk);
        if (on && phase != SER && warp != 0) {
          // warp 0 spends this time issuing the MMAs: warp 1 takes the
          // mat-vecs of both slots of item 0 (one matrix), warps 2 and 3
          // those of their slot of item 1
          const float* mv = (phase == G1) ? my.rm : (phase == G2) ? my.gm : my.tm;
          const float(*x)[32] = (phase == G1) ? my.vv : (phase == G2) ? my.uv : my.wv;
          if (warp == 1) {
            float y[4];
            matvec4(mv, x, rowoff, y);
            s_mv[0][lane] = y[0];
            s_mv[1][lane] = y[1];
            m0 = y[2];
            m1 = y[3];
          } else {
            matvec2(mv, x[2 * slot], x[2 * slot + 1], rowoff, m0, m1);
          }
        }
        {
          const bool mine = tc::mbar_wait(&mbar, parity, w.spin_limit);
          parity ^= 1;
          ok = __syncthreads_and(mine) != 0;  // one verdict for the whole CTA
          tc::fence_after_sync();
        }
        if (!ok) break;
        if (on) {
          float dv[32], a[32];
          // D is read while the masters' columns are loaded; every use of dv
          // follows a tmem_wait_ld(dv)
          tc::tmem_ld32_issue(dmine, dv);
          if (warp == 0 && phase != SER) {
            m0 = s_mv[0][lane];
            m1 = s_mv[1][lane];
          }
          if (phase == G1) {
            if (slot == 0) {  // X = P, its column-sum norm;  u0 = S+ + R v0, u1 = C+ + R v1
              my.uv[0][lane] = my.src[0][lane] + m0;
              my.uv[1][lane] = my.src[1][lane] + m1;
              tc::tmem_wait_ld(dv);
              st_col(my.xa, lane, dv);
              float sn = 0.f;
#pragma unroll
              for (int r = 0; r < 32; r++) sn += fabsf(dv[r]);
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) sn = fmaxf(sn, __shfl_xor_sync(0xffffffffu, sn, o));
              if (lane == 0) my.nrm = sn;
              // G~ = X when the series needs no step, else 0 to start it (the
              // Gauss-Jordan fallback writes its own)
              const int s0 = series_steps(sn);
              if (s0 != -1) {
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = (s0 == 0) ? dv[r] : 0.f;
                st_col(my.gm, lane, a);
              }
            } else {  // V = R - R T~;  u2 = v0 + R v2, u3 = C- + R v3
              my.uv[2][lane] = my.vv[0][lane] + m0;
              my.uv[3][lane] = my.src[3][lane] + m1;
              ld_col(my.rm, lane, a);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = a[r] - dv[r];
              st_col(my.vm, lane, a);
            }
          } else if (phase == SER) {
            if (mys == SERIES_H1) {
              if (slot == 0) {  // G~ = X + X X
                ld_col(my.xa, lane, a);
                tc::tmem_wait_ld(dv);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] + dv[r];
                st_col(my.gm, lane, a);
              }
            } else if (slot == 0) {
              if (k < mys) {  // X = X X (slot 1 took its column of X before)
                tc::tmem_wait_ld(dv);
                st_col(my.xa, lane, dv);
              }
            } else {  // G~ += X + X G~
              float g[32];
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = xk[r];
              ld_col(my.gm, lane, g);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) g[r] = g[r] + (a[r] + dv[r]);
              st_col(my.gm, lane, g);
            }
          } else if (phase == G2) {
            // w = u + G~ u
            my.wv[2 * slot][lane] = my.uv[2 * slot][lane] + m0;
            my.wv[2 * slot + 1][lane] = my.uv[2 * slot + 1][lane] + m1;
            if (slot == 0) {  // Z~ = (T~ - G~) + G~ T~
              float g[32];
              ld_col(my.tm, lane, a);
              ld_col(my.gm, lane, g);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = (a[r] - g[r]) + dv[r];
              st_col(my.xa, lane, a);
            } else {  // Y = V + G~ V
              ld_col(my.vm, lane, a);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = a[r] + dv[r];
              st_col(my.vm, lane, a);
            }
          } else {
            // T w = w - T~ w for my two vectors
            const float a0 = my.wv[2 * slot][lane] - m0, a1 = my.wv[2 * slot + 1][lane] - m1;
            float z[32];
            if (slot == 0) {  // T~' = T~ + (Z~ - T~ Z~);  S+' = (S+ + a0) + f C+,  C+' = C+ + a1
              ld_col(my.tm, lane, a);
              ld_col(my.xa, lane, z);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = a[r] + (z[r] - dv[r]);
              st_col(my.tm, lane, a);
              const float sp = (my.src[0][lane] + a0) + linfac * my.src[1][lane];
              const float cp = my.src[1][lane] + a1;
              my.src[0][lane] = sp;
              my.src[1][lane] = cp;
              my.vv[2][lane] = sp;
              my.vv[3][lane] = cp;
            } else {  // R' = R + (Y - T~ Y);  S-' = S- + a2,  C-' = C- + a3
              ld_col(my.rm, lane, a);
              ld_col(my.vm, lane, z);
              tc::tmem_wait_ld(dv);
#pragma unroll
              for (int r = 0; r < 32; r++) a[r] = a[r] + (z[r] - dv[r]);
              st_col(my.rm, lane, a);
              const float sm = my.src[2][lane] + a0;
              const float cm = my.src[3][lane] + a1;
              my.src[2][lane] = sm;
              my.src[3][lane] = cm;
              my.vv[0][lane] = sm + (2.0f * linfac) * cm;
              my.vv[1][lane] = cm;
            }
          }
          tc::tmem_wait_ld(dv);  // the paths that did not read D
        }
        __syncthreads();  // masters complete before the next operands are built
        // ---- next phase
        if (phase == G1) {
          const int stp0 = (d < s_nd[0]) ? series_steps(Q.st[0].nrm) : -2;
          const int stp1 = (d < s_nd[1]) ? series_steps(Q.st[1].nrm) : -2;
          for (int i = 0; i < 2; i++) {
            if ((i == 0 ? stp0 : stp1) != -1) continue;
            // ||P|| too large for the series: FP64 Gauss-Jordan on I - X (the tiles are free here)
            double* M = reinterpret_cast<double*>(&TL);
            InvScratch<32>& IS = *reinterpret_cast<InvScratch<32>*>(M + Team<32>::MAT);
            TcItemState& D = Q.st[i];
            for (int e = t; e < n * n; e += 128) {
              const int cc = e >> 5, r = e & 31;
              M[cc * Team<32>::LD + r] = (r == cc ? 1.0 : 0.0) - (double)D.xa[midx(r, cc)];
            }
            __syncthreads();
            if (ginv<32>(M, IS) && t == 0) s_status[i] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
            for (int e = t; e < n * n; e += 128) {
              const int cc = e >> 5, r = e & 31;
              D.gm[midx(r, cc)] = (float)(M[cc * Team<32>::LD + r] - (r == cc ? 1.0 : 0.0));
            }
            __syncthreads();
          }
          mys = mi ? stp1 : stp0;
          myg = (mys >= 1) ? mys + 1 : (mys == SERIES_H1 ? 1 : 0);
          gmax = max((stp0 >= 1) ? stp0 + 1 : (stp0 == SERIES_H1 ? 1 : 0),
                     (stp1 >= 1) ? stp1 + 1 : (stp1 == SERIES_H1 ? 1 : 0));
          k = 0;
          phase = (gmax > 0) ? SER : G2;
        } else if (phase == SER) {
          if (++k >= gmax) phase = G2;
        } else if (phase == G2) {
          phase = G3;
        } else {
          linfac = 2.0f * linfac;
          if (++d >= ndmax) break;
          phase = G1;
        }
      }
      if (!ok && t == 0) {
        s_dead = 1;
        s_status[0] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
        s_status[1] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
      }
      __syncthreads();
      // ---- layer R, T = I - T~, S+/S- in FP64 (FP32 records for the split adding)
      for (int i = 0; i < 2; i++) {
        if (s_nd[i] == 0) continue;
        const TcItemState& D = Q.st[i];
        if (w.lay32) {
          float* rec = reinterpret_cast<float*>(w.lay + (size_t)(base + i) * w.lay_stride);
          for (int s = t; s < n * n; s += 128) {
            int r, cc;
            midx_inv(s, r, cc);
            rec[LAY32_R + s] = D.rm[s];
            rec[LAY32_T + s] = (r == cc ? 1.0f : 0.0f) - D.tm[s];  // T = I - T~
          }
          if (t < n) {
            rec[LAY32_SP + t] = D.src[0][t];
            rec[LAY32_SM + t] = D.src[2][t];
          }
          continue;
        }
        double* out = w.lay + (size_t)(base + i) * w.lay_stride;
        for (int e = t; e < n * n; e += 128) {
          const int cc = e >> 5, r = e & 31;
          out[cc * LD + r] = (double)D.rm[midx(r, cc)];
          out[MAT + cc * LD + r] = (r == cc ? 1.0 : 0.0) - (double)D.tm[midx(r, cc)];
        }
        if (t < n) {
          out[2 * MAT + t] = (double)D.src[0][t];
          out[2 * MAT + n + t] = (double)D.src[2][t];
        }
      }
    }
    if (t < 2 && s_valid[t]) {
      w.lay_nd[base + t] = s_nd[t];
      if (s_status[t]) atomicOr(&w.status[(size_t)s_c[t] * Fm + s_fi[t]], s_status[t]);
    }
  }
  // a timed-out CTA lets its last MMA finish before the memory is released
  // (with the default limit, whatever limit the run's waits had)
  if (s_dead) tc::mbar_wait(&mbar, parity ^ 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tslot, 128);
}

}  // namespace pb
