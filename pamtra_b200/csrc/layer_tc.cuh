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
//     P  = R R                     V  = R - R T~
//     G~ = P + P^2 + ... (repeated squaring from G~ = 0, X = P:
//                         G~' = G~ + X + X G~, X' = X X)
//     Y  = V + G~ V                Z~ = T~ - G~ + G~ T~
//     R' = R + Y - T~ Y            T~' = T~ + Z~ - T~ Z~
// Sources follow the FP64 kernel (R v, G u = u + G~ u, T w = w - T~ w).
//
// Products are arranged so that each MMA computes two n x n products that
// share their left factor X:  D = [A1^T; A2^T; v^T] * X^T.  Row m of the A
// tile is column m of a right factor, row n of the B tile is row n of X, and
// TMEM lane m of D is column m of X A1 (lanes 32+m: X A2; lanes 64..67: X v
// for the four source vectors).  Threads hold columns, so A rows are written
// directly and B tiles after an in-register warp transpose.  M = 128 (rows
// 68..127 of the A tile are never used), N = 32, K = 32.
//
// Thread roles (128 threads): warp 0 owns lanes 0..31 (first product), warp 1
// lanes 32..63 (second product), lanes 0..3 of warp 2 the source vectors,
// thread 96 issues the MMAs.  One (layer, frequency) item per CTA at a time;
// 3 CTAs per SM (the launch asks for that many) overlap their MMA chains.
#pragma once
#include "rt.cuh"
#include "tc.cuh"

namespace pb {

constexpr int MS = 36;  // column stride of the FP32 masters: quarter-warp float4 accesses are conflict-free

struct TcSmem {
  float a_hi[9 * 256], a_lo[9 * 256];  // A tile pair, rows 0..71 (the MMA also reads rows 72..127)
  float br_hi[1024], br_lo[1024];      // B tile of the left factor R
  float bt_hi[1024], bt_lo[1024];      // B tile of T~
  float bx_hi[1024], bx_lo[1024];      // B tile of X, then of G~
  float rm[32 * 36], tm[32 * 36], gm[32 * 36], xm[32 * 36];  // FP32 masters, column c at [c * MS]
  float lp[32], cp[32], lmn[32], cmn[32];        // S+ linear, S+ constant, S- linear, S- constant
  float vv[4][32], uv[4][32];
  float nrm, pad_[3];
};
static_assert(sizeof(TcSmem) % 16 == 0, "tile alignment");

constexpr float NEUMANN_TOL = 1.0e-8f;  // truncation of G~ relative to its size
constexpr float NEUMANN_MAX_NORM = 0.75f;

template <int N>
constexpr size_t layer_tc_smem() {
  return (sizeof(LayerSmem<N>) > sizeof(TcSmem) ? sizeof(LayerSmem<N>) : sizeof(TcSmem));
}

// thread-owned column helpers (column-major masters, column stride S)
template <int S = MS>
__device__ __forceinline__ void ld_col(const float* m, int col, float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4) {
    const float4 q = *reinterpret_cast<const float4*>(m + col * S + r);
    v[r] = q.x; v[r + 1] = q.y; v[r + 2] = q.z; v[r + 3] = q.w;
  }
}
template <int S = MS>
__device__ __forceinline__ void st_col(float* m, int col, const float (&v)[32]) {
#pragma unroll
  for (int r = 0; r < 32; r += 4) *reinterpret_cast<float4*>(m + col * S + r) = make_float4(v[r], v[r + 1], v[r + 2], v[r + 3]);
}

// Whole warp, lane L holding column L of a 32 x 32 matrix (v[i] = M[i][L]):
// returns in lane L the sum of row L, sum_m M[L][m] (reduce-scatter in five
// butterfly stages, 31 shuffles; v is consumed).
__device__ __forceinline__ float row_sum_scatter(float (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool upper = (lane & h) != 0;
#pragma unroll
    for (int k = 0; k < h; k++) {
      const float lo = v[k], hi = v[k + h];
      const float send = upper ? lo : hi;
      const float keep = upper ? hi : lo;
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
  return v[0];
}

template <int N>
__global__ void __launch_bounds__(128, 3) k_layer_tc(Batch b, Work w, pamtra_b200_settings st,
                                                     double* __restrict__ ssp_scat) {
  static_assert(N == 16, "the split-precision layer kernel is built for NUMMU = 16");
  constexpr int n = 32, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT;
  extern __shared__ __align__(1024) double smem_raw[];
  LayerSmem<N>& S = *reinterpret_cast<LayerSmem<N>*>(smem_raw);
  TcSmem& Q = *reinterpret_cast<TcSmem*>(smem_raw);  // aliases S after the FP64 setup
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_item, s_dead;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int Fm = b.max_nfreq;
  const int P = min(w.counters[0], w.pmax);
  const int nitems = P * Fm;
  scat_weights_mark_ready<N>(w);
  if (warp == 0) tc::tmem_alloc(&tslot, 64);
  if (t == 0) {
    tc::mbar_init(&mbar, 1);
    s_dead = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm0 = tslot;       // D region 1 (columns 0..31)
  const uint32_t tm1 = tslot + 32;  // D region 2 (columns 32..63)
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t parity = 0;

  // one 3xTF32 group: operands are in place; MMA into `dt`, wait, fence
  auto group = [&](uint32_t dt, const float* bhi, const float* blo) -> bool {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (t == 96) tc::mma3(dt, Q.a_hi, Q.a_lo, bhi, blo, &mbar);
    const bool mine = tc::mbar_wait(&mbar, parity);
    parity ^= 1;
    const bool ok = __syncthreads_and(mine) != 0;  // one verdict for the whole CTA
    tc::fence_after_sync();
    return ok;
  };

  for (;;) {
    __syncthreads();
    if (t == 0) s_item = atomicAdd(&w.counters[3], 1);
    if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
    __syncthreads();
    const int item = s_item;
    if (item >= nitems || s_dead) break;
    LayerItem it;
    if (!layer_setup<N>(b, w, st, ssp_scat, S, item, it)) continue;
    __syncthreads();
    const int nd = it.nd;
    int status = it.status;
    if (nd == 0) {
      layer_store<N>(w, item, S.m[0], S.m[1], S.lin);
    } else {
      // ---- FP64 thin layer -> FP32 masters and tiles (read all, then write: Q aliases S)
      float col[32];
      float linfac = (float)it.linfac;
      if (warp == 0) {
#pragma unroll
        for (int r = 0; r < 32; r++) col[r] = (float)S.m[0][lane * LD + r];
      } else if (warp == 1) {
#pragma unroll
        for (int r = 0; r < 32; r++) col[r] = (float)((r == lane ? 1.0 : 0.0) - S.m[1][lane * LD + r]);
      } else if (warp == 2 && lane < 4) {
        const double* src = (lane == 0) ? S.lin : (lane == 1) ? S.cst : (lane == 2) ? S.lin + n : S.cst + n;
#pragma unroll
        for (int r = 0; r < 32; r++) col[r] = (float)src[r];
      }
      __syncthreads();
      if (warp == 0) {
        st_col(Q.rm, lane, col);
        tc::put_row(Q.a_hi, Q.a_lo, lane, col);
        tc::put_rows_from_cols(Q.br_hi, Q.br_lo, col);
      } else if (warp == 1) {
        st_col(Q.tm, lane, col);
        tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, col);
        tc::put_rows_from_cols(Q.bt_hi, Q.bt_lo, col);
      } else if (warp == 2 && lane < 4) {
        float* dst = (lane == 0) ? Q.lp : (lane == 1) ? Q.cp : (lane == 2) ? Q.lmn : Q.cmn;
#pragma unroll
        for (int r = 0; r < 32; r++) dst[r] = col[r];
      }
      __syncwarp();
      if (warp == 2 && lane < 4) {  // v = [S- + f C-, C-, S+, C+]
        float v[32];
#pragma unroll
        for (int r = 0; r < 32; r++)
          v[r] = (lane == 0) ? Q.lmn[r] + linfac * Q.cmn[r] : (lane == 1) ? Q.cmn[r] : (lane == 2) ? Q.lp[r] : Q.cp[r];
        st_col<32>(&Q.vv[0][0], lane, v);
        tc::put_row(Q.a_hi, Q.a_lo, 64 + lane, v);
      }
      bool ok = true;
      for (int itd = 0; itd < nd && ok; itd++) {
        // ---- group 1: [R; T~; v] x R  ->  P = R R, R T~, R v
        ok = group(tm0, Q.br_hi, Q.br_lo);
        if (!ok) break;
        float d[32];
        if (warp == 0 || warp == 2) tc::tmem_ld32(tm0 + lane_base, d);
        if (warp == 0) {
          // X = P, G~ = X; row-sum norm of P (the lanes hold its columns)
          float a[32];
#pragma unroll
          for (int r = 0; r < 32; r++) a[r] = fabsf(d[r]);
          float rs = row_sum_scatter(a);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) rs = fmaxf(rs, __shfl_xor_sync(0xffffffffu, rs, o));
          if (lane == 0) Q.nrm = rs;
          st_col(Q.xm, lane, d);
          st_col(Q.gm, lane, d);
          tc::put_rows_from_cols(Q.bx_hi, Q.bx_lo, d);
        } else if (warp == 2 && lane < 4) {
          // u = [S+ + Rv0, C+ + Rv1, v0 + Rv2, C- + Rv3]
          float u[32];
#pragma unroll
          for (int r = 0; r < 32; r++) {
            const float base = (lane == 0) ? Q.lp[r] : (lane == 1) ? Q.cp[r] : (lane == 2) ? Q.vv[0][r] : Q.cmn[r];
            u[r] = base + d[r];
          }
          st_col<32>(&Q.uv[0][0], lane, u);
        }
        __syncthreads();
        const float nrm = Q.nrm;
        int steps = 0;  // 0: G~ = X; s > 0: s + 1 factors of the product, one MMA each
        if (nrm < NEUMANN_MAX_NORM) {
          float pw = nrm;  // nrm^(2^(steps+1) - 1)
          float pk = nrm;  // nrm^(2^steps)
          while (pw > NEUMANN_TOL && steps < 6) {
            pk = pk * pk;
            pw = pw * pk;
            steps++;
          }
        } else {
          steps = -1;
        }
        if (steps > 0) {
          // steps + 1 factors (I + X)(I + X^2)...: start from G~ = 0 with A = [X; 0]
          if (warp == 0) {
            ld_col(Q.xm, lane, d);
            tc::put_row(Q.a_hi, Q.a_lo, lane, d);
          } else if (warp == 1) {
            float z[32];
#pragma unroll
            for (int r = 0; r < 32; r++) z[r] = 0.f;
            st_col(Q.gm, lane, z);
            tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, z);
          }
          for (int k = 0; k <= steps && ok; k++) {
            const bool last = (k == steps);
            ok = group(tm1, Q.bx_hi, Q.bx_lo);  // [X; G~] x X -> X X, X G~
            if (!ok) break;
            float e[32];
            if (warp < 2) tc::tmem_ld32(tm1 + lane_base, e);
            if (warp == 1) {
              float x[32], g[32];
              ld_col(Q.xm, lane, x);
              ld_col(Q.gm, lane, g);
#pragma unroll
              for (int r = 0; r < 32; r++) g[r] = g[r] + (x[r] + e[r]);
              st_col(Q.gm, lane, g);
              if (!last) tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, g);
              else tc::put_rows_from_cols(Q.bx_hi, Q.bx_lo, g);
            }
            __syncthreads();  // X_k read before it is replaced
            if (warp == 0 && !last) {
              st_col(Q.xm, lane, e);
              tc::put_row(Q.a_hi, Q.a_lo, lane, e);
              tc::put_rows_from_cols(Q.bx_hi, Q.bx_lo, e);
            }
          }
          if (!ok) break;
        } else if (steps < 0) {
          // ||R R|| too large for the series: FP64 Gauss-Jordan on I - X
          double* M = reinterpret_cast<double*>(Q.a_hi);  // the A tiles are free here
          InvScratch<32>& IS = *reinterpret_cast<InvScratch<32>*>(M + Team<32>::MAT);
          for (int e2 = t; e2 < 1024; e2 += 128) {
            const int cc = e2 >> 5, r = e2 & 31;
            M[cc * Team<32>::LD + r] = (r == cc ? 1.0 : 0.0) - (double)Q.xm[cc * MS + r];
          }
          __syncthreads();
          if (ginv<32>(M, IS)) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
          if (warp == 1) {
            float g[32];
#pragma unroll
            for (int r = 0; r < 32; r++) g[r] = (float)(M[lane * Team<32>::LD + r] - (r == lane ? 1.0 : 0.0));
            st_col(Q.gm, lane, g);
            tc::put_rows_from_cols(Q.bx_hi, Q.bx_lo, g);
          }
          __syncthreads();  // M (in the A tiles) is read before group 2 operands go there
        }
        // ---- group 2: [V; T~; u] x G~  ->  G~V, G~T~, G~u
        if (warp == 1) {
          float rt[32], r0[32];
          tc::tmem_ld32(tm0 + lane_base, rt);  // R T~ (region 1 kept its group-1 result)
          ld_col(Q.rm, lane, r0);
#pragma unroll
          for (int r = 0; r < 32; r++) r0[r] = r0[r] - rt[r];  // V = R - R T~
          st_col(Q.xm, lane, r0);
          tc::put_row(Q.a_hi, Q.a_lo, lane, r0);
          ld_col(Q.tm, lane, rt);
          tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, rt);
        } else if (warp == 2) {
          float u[32];
          if (lane < 4) {
            ld_col<32>(&Q.uv[0][0], lane, u);
            tc::put_row(Q.a_hi, Q.a_lo, 64 + lane, u);
          }
        }
        ok = group(tm0, Q.bx_hi, Q.bx_lo);
        if (!ok) break;
        float keep[32];  // Y (warp 0), Z~ (warp 1), w (warp 2 lanes 0..3)
        if (warp < 3) tc::tmem_ld32(tm0 + lane_base, d);
        if (warp == 0) {
          float v[32];
          ld_col(Q.xm, lane, v);
#pragma unroll
          for (int r = 0; r < 32; r++) keep[r] = v[r] + d[r];  // Y = V + G~V
          tc::put_row(Q.a_hi, Q.a_lo, lane, keep);
        } else if (warp == 1) {
          float tt[32], g[32];
          ld_col(Q.tm, lane, tt);
          ld_col(Q.gm, lane, g);
#pragma unroll
          for (int r = 0; r < 32; r++) keep[r] = (tt[r] - g[r]) + d[r];  // Z~ = T~ - G~ + G~T~
          tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, keep);
        } else if (warp == 2 && lane < 4) {
          float u[32];
          ld_col<32>(&Q.uv[0][0], lane, u);
#pragma unroll
          for (int r = 0; r < 32; r++) keep[r] = u[r] + d[r];  // w = G u
          tc::put_row(Q.a_hi, Q.a_lo, 64 + lane, keep);
        }
        // ---- group 3: [Y; Z~; w] x T~  ->  T~Y, T~Z~, T~w
        ok = group(tm1, Q.bt_hi, Q.bt_lo);
        if (!ok) break;
        if (warp < 3) tc::tmem_ld32(tm1 + lane_base, d);
        if (warp == 0) {
          float r0[32];
          ld_col(Q.rm, lane, r0);
#pragma unroll
          for (int r = 0; r < 32; r++) r0[r] = r0[r] + (keep[r] - d[r]);  // R' = R + Y - T~Y
          st_col(Q.rm, lane, r0);
          tc::put_row(Q.a_hi, Q.a_lo, lane, r0);
          tc::put_rows_from_cols(Q.br_hi, Q.br_lo, r0);
        } else if (warp == 1) {
          float tt[32];
          ld_col(Q.tm, lane, tt);
#pragma unroll
          for (int r = 0; r < 32; r++) tt[r] = tt[r] + (keep[r] - d[r]);  // T~' = T~ + Z~ - T~Z~
          st_col(Q.tm, lane, tt);
          tc::put_row(Q.a_hi, Q.a_lo, 32 + lane, tt);
          tc::put_rows_from_cols(Q.bt_hi, Q.bt_lo, tt);
        } else if (warp == 2 && lane < 4) {
          // a = T w;  S+ = (S+ + a0) + f C+,  C+ += a1,  S- += a2,  C- += a3
          float nv[32];
#pragma unroll
          for (int r = 0; r < 32; r++) {
            const float a = keep[r] - d[r];
            nv[r] = (lane == 0) ? (Q.lp[r] + a) + linfac * Q.cp[r]
                  : (lane == 1) ? Q.cp[r] + a : (lane == 2) ? Q.lmn[r] + a : Q.cmn[r] + a;
          }
          __syncwarp(0xFu);
          float* dst = (lane == 0) ? Q.lp : (lane == 1) ? Q.cp : (lane == 2) ? Q.lmn : Q.cmn;
#pragma unroll
          for (int r = 0; r < 32; r++) dst[r] = nv[r];
          __syncwarp(0xFu);
          const float f2 = 2.0f * linfac;
#pragma unroll
          for (int r = 0; r < 32; r++)
            nv[r] = (lane == 0) ? Q.lmn[r] + f2 * Q.cmn[r] : (lane == 1) ? Q.cmn[r] : (lane == 2) ? Q.lp[r] : Q.cp[r];
          st_col<32>(&Q.vv[0][0], lane, nv);
          tc::put_row(Q.a_hi, Q.a_lo, 64 + lane, nv);
        }
        linfac = 2.0f * linfac;
      }
      if (!ok) {
        status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
        if (t == 0) s_dead = 1;
      }
      __syncthreads();
      // ---- layer R, T = I - T~, S+/S- in FP64
      double* out = w.lay + (size_t)item * w.lay_stride;
      for (int e2 = t; e2 < n * n; e2 += 128) {
        const int cc = e2 >> 5, r = e2 & 31;
        out[cc * LD + r] = (double)Q.rm[cc * MS + r];
        out[MAT + cc * LD + r] = (r == cc ? 1.0 : 0.0) - (double)Q.tm[cc * MS + r];
      }
      if (t < 32) {
        out[2 * MAT + t] = (double)Q.lp[t];
        out[2 * MAT + n + t] = (double)Q.lmn[t];
      }
    }
    if (t == 0) {
      w.lay_nd[item] = nd;
      if (status) atomicOr(&w.status[(size_t)it.c * Fm + it.fi], status);
    }
  }
  // a timed-out CTA lets its last MMA finish before the memory is released
  if (s_dead) tc::mbar_wait(&mbar, parity ^ 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tslot, 64);
}

}  // namespace pb
