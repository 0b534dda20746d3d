// Split-precision layer stage for NUMMU = 32 (n = 64): the design of
// k_layer_tc<16> (layer_tc.cuh) with one item per CTA.  The products are
// 64 x 64, so two of them already fill the MMA: with D = A B^T,
//     A = [Ya^T; Yb^T]   (128 rows: the columns of the two right factors)
//     B = X              (64 rows: the left factor; K = 64)
// lane 64p + m of D is column m of X Yp.  Eight warps: warps w and w + 4
// share the TMEM lanes 32 (w mod 4) .. 32 (w mod 4) + 31, so a thread owns
// lane 32 (w mod 4) + lane (product p, column m) for the whole doubling and
// half w / 4 of it: rows 32 h .. 32 h + 31 of its product column (D columns
// 32 h ..), K = 32 h .. of its A row, a quarter of a B row and one mat-vec
// entry.  The deviation forms, phases, series plans, source recurrences and
// bounded waits are those of k_layer_tc<16>.
#pragma once
#include "layer_tc.cuh"

namespace pb {

// FP32 64 x 64 masters, column-major, 4-float chunks of column c XOR-swizzled
// by c mod 16 (conflict-free column loads of eight neighbouring columns and
// row-slice loads across a warp, without padding).
__device__ __forceinline__ int midx64(int r, int c) {
  return c * 64 + ((((r >> 2) ^ (c & 15)) << 2) | (r & 3));
}

struct Tc64Item {
  float rm[4096], tm[4096], gm[4096];      // R, T~, G~
  float vm[4096];                          // V = R T, then Y = G R T
  float xa[4096];                          // series power X, then Z~
  float src[4][64];                        // S+ linear, S+ constant, S- linear, S- constant
  float vv[4][64], uv[4][64], wv[4][64];   // right-hand vectors of the three groups
  int pad_[32];
};

struct Tc64Tiles {
  float b_hi[64 * 64], b_lo[64 * 64];  // B tile pair, K-major, K = 64 (row groups 2048 bytes apart)
};

// FP64 set-up scratch of the item (layer_setup with 256 threads).
struct Tc64Setup {
  static constexpr int n = 64, MAT = RTCfg<32>::MAT;
  double r[MAT], t[MAT];
  double coef[3 * MAXNLEG];
  double az[2 * KMAX];
  double lin[2 * n], cst[2 * n];
  double mu[32], wq[32], nrm[32];
  int item, stat;
  __device__ __forceinline__ double* mat(int i) { return i == 0 ? r : i == 1 ? t : i == 4 ? az : coef; }
};

union __align__(128) Tc64Scratch {
  Tc64Tiles tl;
  Tc64Setup setup;
  double gj[RTCfg<32>::MAT + sizeof(InvScratch<64>) / 8 + 1];  // FP64 fallback inverse
};

struct Tc64Smem {
  Tc64Item it;
  Tc64Scratch u;
};
static_assert(sizeof(Tc64Item) % 128 == 0, "tile alignment");

constexpr size_t layer_tc64_smem() { return sizeof(Tc64Smem); }

// 32 rows (half h) of column `col` of a 64 x 64 master
__device__ __forceinline__ void ld_col64(const float* m, int col, int h, float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4) {
    const float4 q = *reinterpret_cast<const float4*>(m + midx64(32 * h + r, col));
    v[r] = q.x; v[r + 1] = q.y; v[r + 2] = q.z; v[r + 3] = q.w;
  }
}
__device__ __forceinline__ void st_col64(float* m, int col, int h, const float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4)
    *reinterpret_cast<float4*>(m + midx64(32 * h + r, col)) = make_float4(v[r], v[r + 1], v[r + 2], v[r + 3]);
}

// (M x0)[r] and (M x1)[r] for a 64 x 64 master (k-ascending FMA chains)
__device__ __forceinline__ void matvec2_64(const float* __restrict__ M, const float* __restrict__ x0,
                                           const float* __restrict__ x1, int r, float& y0, float& y1) {
  float a0 = 0.f, a1 = 0.f;
#pragma unroll 4
  for (int k = 0; k < 64; k += 4) {
    const float4 p = *reinterpret_cast<const float4*>(x0 + k);
    const float4 q = *reinterpret_cast<const float4*>(x1 + k);
    const float m0 = M[midx64(r, k)], m1 = M[midx64(r, k + 1)], m2 = M[midx64(r, k + 2)], m3 = M[midx64(r, k + 3)];
    a0 = fmaf(m0, p.x, a0); a1 = fmaf(m0, q.x, a1);
    a0 = fmaf(m1, p.y, a0); a1 = fmaf(m1, q.y, a1);
    a0 = fmaf(m2, p.z, a0); a1 = fmaf(m2, q.z, a1);
    a0 = fmaf(m3, p.w, a0); a1 = fmaf(m3, q.w, a1);
  }
  y0 = a0;
  y1 = a1;
}

// (M x)[r] for a 64 x 64 master (the k-ascending FMA chain of matvec2_64)
__device__ __forceinline__ float matvec1_64(const float* __restrict__ M, const float* __restrict__ x, int r) {
  float a = 0.f;
#pragma unroll 4
  for (int k = 0; k < 64; k += 4) {
    const float4 p = *reinterpret_cast<const float4*>(x + k);
    a = fmaf(M[midx64(r, k)], p.x, a);
    a = fmaf(M[midx64(r, k + 1)], p.y, a);
    a = fmaf(M[midx64(r, k + 2)], p.z, a);
    a = fmaf(M[midx64(r, k + 3)], p.w, a);
  }
  return a;
}

// Operands of one group for thread t: half hh (K = 32 hh .. 32 hh + 31) of
// its A row (column `col` of `asrc`) split into TF32 hi / lo in its TMEM lane,
// and K = kq .. kq + 15 of B row `brow` (row brow of `bsrc`) in shared memory;
// the A stores run while the B part is built.
__device__ __forceinline__ void build_operands64(Tc64Tiles& TL, const float* asrc, const float* bsrc, uint32_t ta_hi,
                                                 uint32_t ta_lo, int col, int hh, int brow, int kq) {
  float c[32], lo[32];
  ld_col64(asrc, col, hh, c);
#pragma unroll
  for (int r = 0; r < 32; r++) tc::split(c[r], c[r], lo[r]);
  tc::tmem_st32_issue(ta_hi + 32u * hh, c);
  tc::tmem_st32_issue(ta_lo + 32u * hh, lo);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k0 = kq + 4 * q;
    float4 bh, bl;
    tc::split(bsrc[midx64(brow, k0 + 0)], bh.x, bl.x);
    tc::split(bsrc[midx64(brow, k0 + 1)], bh.y, bl.y);
    tc::split(bsrc[midx64(brow, k0 + 2)], bh.z, bl.z);
    tc::split(bsrc[midx64(brow, k0 + 3)], bh.w, bl.w);
    const int o = (brow >> 3) * 512 + (k0 >> 2) * 32 + (brow & 7) * 4;
    *reinterpret_cast<float4*>(TL.b_hi + o) = bh;
    *reinterpret_cast<float4*>(TL.b_lo + o) = bl;
  }
  tc::tmem_wait_st2(c, lo);
}

// 3xTF32 M = 128, N = 64, K = 64 product: A pair in TMEM, B pair in shared
// memory with 2048-byte row groups.  One thread; completion on `mbar`.
__device__ __forceinline__ void mma3_k64(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, const float* b_hi,
                                         const float* b_lo, uint64_t* mbar) {
  const uint32_t bh = tc::smem_u32(b_hi), bl = tc::smem_u32(b_lo);
#pragma unroll
  for (int s = 0; s < 8; s++)
    tc::mma_ta(d_tmem, a_lo + 8 * s, tc::desc(bh + 256 * s, 128, 2048), s > 0, tc::IDESC_M128_N64);
#pragma unroll
  for (int s = 0; s < 8; s++) tc::mma_ta(d_tmem, a_hi + 8 * s, tc::desc(bl + 256 * s, 128, 2048), 1, tc::IDESC_M128_N64);
#pragma unroll
  for (int s = 0; s < 8; s++) tc::mma_ta(d_tmem, a_hi + 8 * s, tc::desc(bh + 256 * s, 128, 2048), 1, tc::IDESC_M128_N64);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(tc::smem_u32(mbar))
               : "memory");
}

__global__ void __launch_bounds__(256, 1) k_layer_tc64(Batch b, Work w, pamtra_b200_settings st,
                                                      double* __restrict__ ssp_scat) {
  constexpr int N = 32, n = 64, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT;
  enum { G1 = 0, SER = 1, G2 = 2, G3 = 3 };
  extern __shared__ __align__(1024) double smem_raw[];
  Tc64Smem& Q = *reinterpret_cast<Tc64Smem*>(smem_raw);
  Tc64Setup& S = Q.u.setup;
  Tc64Tiles& TL = Q.u.tl;
  Tc64Item& my = Q.it;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_item, s_dead, s_status;
  __shared__ float s_mv[4][64];  // mat-vec results: vector, entry
  __shared__ float s_ns[2][64];  // column abs-sums of P over the two halves of the rows
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int q4 = warp & 3, hh = warp >> 2;      // my TMEM lane quarter; my half of the column (rows, A's K)
  const int arow = 32 * q4 + lane;              // my A row = my D lane
  const int slot = arow >> 6, col = arow & 63;  // my product and my column of it
  const int Fm = b.max_nfreq;
  const int P = min(w.counters[0], w.pmax);
  const int nitems = P * Fm;
  scat_weights_mark_ready<N>(w);
  if (warp == 0) tc::tmem_alloc(&tslot, 256);  // D: columns 0..63, A hi: 64..127, A lo: 128..191
  if (t == 0) {
    tc::mbar_init(&mbar, 1);
    s_dead = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t lanes = (uint32_t)(q4 * 32) << 16;
  const uint32_t dmine = tslot + lanes;
  const uint32_t ahi = tslot + lanes + 64u, alo = tslot + lanes + 128u;
  uint32_t parity = 0;

  for (;;) {
    __syncthreads();
    if (t == 0) s_item = atomicAdd(&w.counters[4], 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    if (s_dead) {  // after a timed-out wait: report the remaining items, compute nothing
      if (t == 0) mark_timed_out<N>(b, w, item);
      continue;
    }
    if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
    __syncthreads();
    LayerItem it;
    if (!layer_setup<N, Tc64Setup, 256>(b, w, st, ssp_scat, S, item, it)) continue;
    const int nd = it.nd;
    if (t == 0) s_status = it.status;
    if (nd == 0) {
      layer_store<N, 256>(w, item, S.r, S.t, S.lin);
    } else {
      for (int e = t; e < n * n; e += 256) {
        const int cc = e >> 6, r = e & 63;
        my.rm[midx64(r, cc)] = (float)S.r[cc * LD + r];
        my.tm[midx64(r, cc)] = (float)((r == cc ? 1.0 : 0.0) - S.t[cc * LD + r]);
      }
      if (t < n) {
        my.src[0][t] = (float)S.lin[t];
        my.src[1][t] = (float)S.cst[t];
        my.src[2][t] = (float)S.lin[n + t];
        my.src[3][t] = (float)S.cst[n + t];
      }
    }
    __syncthreads();  // the set-up scratch becomes the B tiles
    float linfac = (float)it.linfac;
    bool ok = true;
    if (nd > 0) {
      // v = [S- + f C-, C-, S+, C+] (thread t: entry col of the vectors of its slot)
      if (hh == 0 && slot == 0) {
        my.vv[2][col] = my.src[0][col];
        my.vv[3][col] = my.src[1][col];
      } else if (hh == 0) {
        my.vv[0][col] = my.src[2][col] + linfac * my.src[3][col];
        my.vv[1][col] = my.src[3][col];
      }
      //   G1  [R; T~] x R   -> slot 0: P = R R  -> X;       slot 1: R T~ -> V = R - R T~
      //   SER [X; G~] x X   -> slot 0: X X      -> X next;  slot 1: X G~ -> G~ += X + X G~
      //   G2  [T~; V] x G~  -> slot 0: G~ T~    -> Z~;      slot 1: G~ V -> Y = V + G~ V
      //   G3  [Z~; Y] x T~  -> slot 0: T~ Z~    -> T~';     slot 1: T~ Y -> R'
      int phase = G1, d = 0, k = 0, mys = 0, myg = 0;
      for (;;) {
        const bool on = (phase != SER) || (k < myg);
        if (on) {
          const float* asrc;
          const float* bsrc;
          if (phase == G1) { asrc = slot ? my.tm : my.rm; bsrc = my.rm; }
          else if (phase == SER) { asrc = slot ? my.gm : my.xa; bsrc = my.xa; }
          else if (phase == G2) { asrc = slot ? my.vm : my.tm; bsrc = my.gm; }
          else { asrc = slot ? my.vm : my.xa; bsrc = my.tm; }
          build_operands64(TL, asrc, bsrc, ahi, alo, col, hh, col, 32 * slot + 16 * hh);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) mma3_k64(tslot, tslot + 64u, tslot + 128u, TL.b_hi, TL.b_lo, &mbar);
        float m0 = 0.f, m1 = 0.f;
        float xk[32];  // slot 1 of a series step: its half column of X, taken before slot 0 replaces X
        if (phase == SER && slot == 1) ld_col64(my.xa, col, hh, xk);
        if (phase != SER) {
          const float* mv = (phase == G1) ? my.rm : (phase == G2) ? my.gm : my.tm;
          const float(*x)[64] = (phase == G1) ? my.vv : (phase == G2) ? my.uv : my.wv;
          // one vector entry per thread (vector 2 slot + hh, row col); warp 0
          // issues the MMAs meanwhile, so warp 4 (the same rows) takes both
          // vectors of slot 0 for rows 0..31
          if (warp == 4) {
            float y0, y1;
            matvec2_64(mv, x[0], x[1], col, y0, y1);
            s_mv[0][col] = y0;
            s_mv[1][col] = y1;
          } else if (warp != 0) {
            s_mv[2 * slot + hh][col] = matvec1_64(mv, x[2 * slot + hh], col);
          }
        }
        {
          const bool mine = tc::mbar_wait(&mbar, parity, w.spin_limit);
          parity ^= 1;
          ok = __syncthreads_and(mine) != 0;
          tc::fence_after_sync();
        }
        if (!ok) break;
        if (phase != SER) {
          m0 = s_mv[2 * slot][col];
          m1 = s_mv[2 * slot + 1][col];
        }
        if (on) {
          float nsum = 0.f;
          {
            const int h = hh;  // my half of the column
            float dv[32], a[32];
            tc::tmem_ld32(dmine + 32u * h, dv);
            if (phase == G1) {
              if (slot == 0) {  // X = P, column-sum norm
                st_col64(my.xa, col, h, dv);
#pragma unroll
                for (int r = 0; r < 32; r++) nsum += fabsf(dv[r]);
              } else {  // V = R - R T~
                ld_col64(my.rm, col, h, a);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] - dv[r];
                st_col64(my.vm, col, h, a);
              }
            } else if (phase == SER) {
              if (mys == SERIES_H1) {
                if (slot == 0) {  // G~ = X + X X
                  ld_col64(my.xa, col, h, a);
#pragma unroll
                  for (int r = 0; r < 32; r++) a[r] = a[r] + dv[r];
                  st_col64(my.gm, col, h, a);
                }
              } else if (slot == 0) {
                if (k < mys) st_col64(my.xa, col, h, dv);  // X = X X
              } else {  // G~ += X + X G~
                ld_col64(my.gm, col, h, a);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] + (xk[r] + dv[r]);
                st_col64(my.gm, col, h, a);
              }
            } else if (phase == G2) {
              float g[32];
              if (slot == 0) {  // Z~ = (T~ - G~) + G~ T~
                ld_col64(my.tm, col, h, a);
                ld_col64(my.gm, col, h, g);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = (a[r] - g[r]) + dv[r];
                st_col64(my.xa, col, h, a);
              } else {  // Y = V + G~ V
                ld_col64(my.vm, col, h, a);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] + dv[r];
                st_col64(my.vm, col, h, a);
              }
            } else {
              float z[32];
              if (slot == 0) {  // T~' = T~ + (Z~ - T~ Z~)
                ld_col64(my.tm, col, h, a);
                ld_col64(my.xa, col, h, z);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] + (z[r] - dv[r]);
                st_col64(my.tm, col, h, a);
              } else {  // R' = R + (Y - T~ Y)
                ld_col64(my.rm, col, h, a);
                ld_col64(my.vm, col, h, z);
#pragma unroll
                for (int r = 0; r < 32; r++) a[r] = a[r] + (z[r] - dv[r]);
                st_col64(my.rm, col, h, a);
              }
            }
          }
          if (phase == G1 && slot == 0) s_ns[hh][col] = nsum;  // my half of the column's abs-sum
          // the vector parts (entry `col` of the slot's two vectors), by the
          // threads of the first halves
          if (hh == 0 && phase == G1) {
            if (slot == 0) {  // u0 = S+ + R v0, u1 = C+ + R v1
              my.uv[0][col] = my.src[0][col] + m0;
              my.uv[1][col] = my.src[1][col] + m1;
            } else {  // u2 = v0 + R v2, u3 = C- + R v3
              my.uv[2][col] = my.vv[0][col] + m0;
              my.uv[3][col] = my.src[3][col] + m1;
            }
          } else if (hh == 0 && phase == G2) {  // w = u + G~ u
            my.wv[2 * slot][col] = my.uv[2 * slot][col] + m0;
            my.wv[2 * slot + 1][col] = my.uv[2 * slot + 1][col] + m1;
          } else if (hh == 0 && phase == G3) {  // T w = w - T~ w
            const float a0 = my.wv[2 * slot][col] - m0, a1 = my.wv[2 * slot + 1][col] - m1;
            if (slot == 0) {  // S+' = (S+ + a0) + f C+,  C+' = C+ + a1
              const float sp = (my.src[0][col] + a0) + linfac * my.src[1][col];
              const float cp = my.src[1][col] + a1;
              my.src[0][col] = sp;
              my.src[1][col] = cp;
              my.vv[2][col] = sp;
              my.vv[3][col] = cp;
            } else {  // S-' = S- + a2,  C-' = C- + a3
              const float sm = my.src[2][col] + a0;
              const float cm = my.src[3][col] + a1;
              my.src[2][col] = sm;
              my.src[3][col] = cm;
              my.vv[0][col] = sm + (2.0f * linfac) * cm;
              my.vv[1][col] = cm;
            }
          }
        }
        __syncthreads();  // masters complete before the next operands are built
        // ---- next phase
        if (phase == G1) {
          // column-sum norm of P (every warp forms the same value)
          float nrm = fmaxf(s_ns[0][lane] + s_ns[1][lane], s_ns[0][lane + 32] + s_ns[1][lane + 32]);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) nrm = fmaxf(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
          mys = series_steps(nrm);
          if (mys == -1) {
            // ||P|| too large for the series: FP64 Gauss-Jordan on I - X (the tiles are free here)
            double* M = Q.u.gj;
            InvScratch<64>& IS = *reinterpret_cast<InvScratch<64>*>(M + MAT);
            for (int e = t; e < n * n; e += 256) {
              const int cc = e >> 6, r = e & 63;
              M[cc * LD + r] = (r == cc ? 1.0 : 0.0) - (double)my.xa[midx64(r, cc)];
            }
            __syncthreads();
            if (ginv<64, 256>(M, IS) && t == 0) s_status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
            for (int e = t; e < n * n; e += 256) {
              const int cc = e >> 6, r = e & 63;
              my.gm[midx64(r, cc)] = (float)(M[cc * LD + r] - (r == cc ? 1.0 : 0.0));
            }
          } else if (slot == 1) {  // G~ = X (no series), or G~ = 0 to start one (my half)
            float g[32];
            if (mys == 0) ld_col64(my.xa, col, hh, g);
#pragma unroll
            for (int r = 0; r < 32; r++) g[r] = (mys == 0) ? g[r] : 0.f;
            st_col64(my.gm, col, hh, g);
          }
          myg = (mys >= 1) ? mys + 1 : (mys == SERIES_H1 ? 1 : 0);
          __syncthreads();
          k = 0;
          phase = (myg > 0) ? SER : G2;
        } else if (phase == SER) {
          if (++k >= myg) phase = G2;
        } else if (phase == G2) {
          phase = G3;
        } else {
          linfac = 2.0f * linfac;
          if (++d >= nd) break;
          phase = G1;
        }
      }
      if (!ok && t == 0) {
        s_dead = 1;
        s_status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
      }
      __syncthreads();
      // ---- layer R, T = I - T~, S+/S- in FP64
      double* out = w.lay + (size_t)item * w.lay_stride;
      for (int e = t; e < n * n; e += 256) {
        const int cc = e >> 6, r = e & 63;
        out[cc * LD + r] = (double)my.rm[midx64(r, cc)];
        out[MAT + cc * LD + r] = (r == cc ? 1.0 : 0.0) - (double)my.tm[midx64(r, cc)];
      }
      if (t < n) {
        out[2 * MAT + t] = (double)my.src[0][t];
        out[2 * MAT + n + t] = (double)my.src[2][t];
      }
    }
    __syncthreads();
    if (t == 0) {
      w.lay_nd[item] = nd;
      if (s_status) atomicOr(&w.status[(size_t)it.c * Fm + it.fi], s_status);
    }
  }
  // a timed-out CTA lets its last MMA finish before the memory is released
  // (with the default limit, whatever limit the run's waits had)
  if (s_dead) tc::mbar_wait(&mbar, parity ^ 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tslot, 256);
}

}  // namespace pb
