// Split-precision adding of the batched form (NUMMU = 16, n = 32): the
// COMBINE_LAYERS4 products (src/radintg4.f90:447-513, one-inverse form) run
// as 3xTF32 tcgen05 MMAs with FP32 accumulation; the (I - R1+ R2)^-1 solve of
// every combine stays FP64 (Neumann series on the FP64 tensor path or
// Gauss-Jordan), and so do the source vectors, the surface coupling and the
// internal radiances (k_adding_finish, the FP64 code of k_adding).
//
// Per (column, frequency) unit the stack (R+, R-, T+, T-) is held in FP32
// masters in shared memory.  With G = (I - R1+ R2)^-1 a combine is five MMA
// passes, each two products with one left factor, and the FP64 inverse
// between the first two:
//   P1  Rp x [R2, T2]   -> Gin = Rp R2 (inverted in FP64 -> G),  Z = Rp T2
//   P2  G  x [Z, Tp]    -> Y = G Z,                 W = G Tp
//   P3  T2 x [Y, W]     -> R+' = R2 + T2 Y,         T+' = T2 W
//   P4  Tm x [R2, T2]   -> V = T1- R2,              Q = T1- T2
//   P5  V  x [W, Y]     -> R-' = R- + V W,          T-' = Q + V Y
// (T1-' = T1- (T2 + R2 Y) = Q + V Y).  The source chains run as FP32
// matrix-vector products on the CUDA cores while the MMAs run:
// w = S1+ + Rp S2-, G w, S+' = S2+ + T2 G w;  m = S2- + R2 S1+,
// Gm m = m + R2 G (Rp m), S-' = S1- + T1- Gm m.
// Carrying T~ = I - T and G~ = G - I instead (as the doubling does) was
// measured no more accurate here: it helps transparent stacks and hurts
// opaque ones, whose T~ is near I.
//
// Pairing as in k_layer_tc: one CTA (4 warps) carries two units in lockstep;
// warp 2i + p owns product p of unit i (its D lanes hold the columns of the
// product); M = 128, N = 64 (B = the two units' left factors), K = 32.
// Off-diagonal blocks are computed and ignored, so a unit's results do not
// depend on its partner.  Consecutive units are the frequencies of one
// column, whose scattering layers coincide, so the pair rarely waits on
// itself.
//
// The layer records come from k_layer_tc in FP32 (R and T in the masters'
// swizzled layout) and are copied into shared memory with cp.async while the
// combine's last pass runs, into the buffers of W and Y (free once that pass
// has its operands); the buffer roles rotate every combine.
#pragma once
#include "layer_tc.cuh"

namespace pb {

// FP32 stack record of one (column, frequency) unit, handed to
// k_adding_finish: R+, R-, T+, T- (masters), S+, S-, the clear-stack
// transmission t1, then the header (sstate, status as int).
constexpr int STK_RP = 0, STK_RM = 1024, STK_TP = 2048, STK_TM = 3072, STK_SP = 4096, STK_SM = 4128, STK_T1 = 4160,
              STK_HDR = 4192, STK_FLOATS = 4224;

struct AddTcItem {
  float m[8][1024];                  // masters; roles rotate every combine
  float s2p[32], s2m[32];            // the next layer's sources as fetched (cp.async target)
  float d2p[32], d2m[32];            // the current layer's sources
  float sp[32], sm[32], t1[32];      // stack sources; clear-stack transmission
  float t2[32], c2p[32], c2m[32];    // a clear layer
  float nsp[32], nsm[32], wv[32], wv2[32], u1[32], u2[32], mw[32], u1b[32];
};

struct AddTcTiles {
  float b_hi[64 * 32], b_lo[64 * 32];  // B tile pair (64 rows: 32 per unit)
};
struct AddTcInv {
  double P[Team<32>::MAT], G[Team<32>::MAT];
  InvScratch<32> inv;
};
union __align__(128) AddTcScratch {
  AddTcTiles tl;
  AddTcInv fp[2];  // FP64 inverses of the two units (at once)
};

struct AddTcSmem {
  AddTcItem it[2];
  AddTcScratch u;
  double mu[16], wq[16];
};
static_assert(sizeof(AddTcItem) % 16 == 0, "alignment of the masters");

constexpr size_t add_tc_smem() { return sizeof(AddTcSmem); }

// barrier of the two warps of unit i (named barriers 1 and 2, 64 threads)
__device__ __forceinline__ void unit_sync(int i) {
  if (i == 0) asm volatile("bar.sync 1, 64;" ::: "memory");
  else asm volatile("bar.sync 2, 64;" ::: "memory");
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// row `lane` of the master M times x (k ascending)
__device__ __forceinline__ float mv32(const float* __restrict__ M, const float* __restrict__ x, const RowOff& ro) {
  float a = 0.f;
#pragma unroll
  for (int k = 0; k < 32; k += 4) {
    const float4 p = *reinterpret_cast<const float4*>(x + k);
    a = fmaf(M[k * 32 + ro.o[k & 7]], p.x, a);
    a = fmaf(M[(k + 1) * 32 + ro.o[(k + 1) & 7]], p.y, a);
    a = fmaf(M[(k + 2) * 32 + ro.o[(k + 2) & 7]], p.z, a);
    a = fmaf(M[(k + 3) * 32 + ro.o[(k + 3) & 7]], p.w, a);
  }
  return a;
}

// Operands of one pass for this thread: its A row (column `lane` of master
// asrc, hi / lo into TMEM) and K-half h of B row `brow` (row `lane` of its
// unit's left factor bsrc); the A stores run while B is built
__device__ __forceinline__ void build_ab(AddTcTiles& TL, const float* asrc, const float* bsrc, uint32_t ta_hi,
                                         uint32_t ta_lo, int brow, int h, int lane, const RowOff& ro) {
  float c[32], lo[32];
  ld_col(asrc, lane, c);
#pragma unroll
  for (int r = 0; r < 32; r++) tc::split_rn(c[r], c[r], lo[r]);
  tc::tmem_st32_issue(ta_hi, c);
  tc::tmem_st32_issue(ta_lo, lo);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k0 = 16 * h + 4 * q;
    float4 bh, bl;
    const float* bc = bsrc + k0 * 32;
    tc::split_rn(bc[0 * 32 + ro.o[(4 * q + 0) & 7]], bh.x, bl.x);
    tc::split_rn(bc[1 * 32 + ro.o[(4 * q + 1) & 7]], bh.y, bl.y);
    tc::split_rn(bc[2 * 32 + ro.o[(4 * q + 2) & 7]], bh.z, bl.z);
    tc::split_rn(bc[3 * 32 + ro.o[(4 * q + 3) & 7]], bh.w, bl.w);
    const int o = (brow >> 3) * tc::RG_FLOATS + (k0 >> 2) * 32 + (brow & 7) * 4;
    *reinterpret_cast<float4*>(TL.b_hi + o) = bh;
    *reinterpret_cast<float4*>(TL.b_lo + o) = bl;
  }
  tc::tmem_wait_st2(c, lo);
}

// Issue the copy of layer record `item` into masters r2 / t2 and the staged
// sources (the 64 threads of the unit).
__device__ __forceinline__ void lay32_fetch(const Work& w, int item, AddTcItem& U, int r2, int t2, int u) {
  const float* rec = reinterpret_cast<const float*>(w.lay + (size_t)item * w.lay_stride);
  for (int q = u; q < 256; q += 64) {
    cp_async16(&U.m[r2][4 * q], rec + LAY32_R + 4 * q);
    cp_async16(&U.m[t2][4 * q], rec + LAY32_T + 4 * q);
  }
  if (u < 8) cp_async16(&U.s2p[4 * u], rec + LAY32_SP + 4 * u);
  else if (u < 16) cp_async16(&U.s2m[4 * (u - 8)], rec + LAY32_SM + 4 * (u - 8));
}

// next scattering layer at or below top-down index k0 of column c (-1: none)
__device__ __forceinline__ int next_scat(const Batch& b, const Work& w, int c, int L, int k0, int& pidx) {
  const int Lm = b.max_nlyrs;
  for (int k = k0; k < L; k++) {
    const int p = w.pres_idx[(size_t)c * Lm + (L - 1 - k)];
    if (p >= 0) { pidx = p; return k; }
  }
  pidx = -1;
  return -1;
}

// One unit's n = 32 FP64 product by its two warps (wl = 0, 1 owns rows
// 16 wl .. 16 wl + 15): C = A B (MM_SET), D + A B (MM_ACC) or I + A B
// (MM_IPLUS), with the fragments and k order of mm(), so the results are
// bit-identical to it.  With INPLACE the unit synchronises between reading
// the operands and writing C.
template <int MODE, bool INPLACE>
__device__ __forceinline__ void mm_unit(const double* A, const double* B, double* C, const double* D, int wl, int mi) {
  constexpr int LD = Team<32>::LD;
  const int lane = threadIdx.x & 31;
  const int row0 = 16 * wl, g = lane >> 2, q = lane & 3;
  double c[2][4][2];
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 4; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = ct * 8 + 2 * q + i;
        c[rt][ct][i] = (MODE == MM_ACC) ? D[col * LD + row] : ((MODE == MM_IPLUS) ? (row == col ? 1.0 : 0.0) : 0.0);
      }
#pragma unroll 2
  for (int kk = 0; kk < 32; kk += 4) {
    const double a0 = A[(kk + q) * LD + row0 + g];
    const double a1 = A[(kk + q) * LD + row0 + 8 + g];
    double bb[4];
#pragma unroll
    for (int ct = 0; ct < 4; ct++) bb[ct] = B[(ct * 8 + g) * LD + kk + q];
#pragma unroll
    for (int ct = 0; ct < 4; ct++) {
      dmma(c[0][ct], a0, bb[ct]);
      dmma(c[1][ct], a1, bb[ct]);
    }
  }
  if (INPLACE) unit_sync(mi);
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 4; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = ct * 8 + 2 * q + i;
        C[col * LD + row] = c[rt][ct][i];
      }
}

// (I - P)^-1 of one unit by its two warps, the Neumann series of
// inv_iminus() (same plan from the infinity norm, Horner or repeated
// squaring, same products): returns the buffer holding the inverse (P or
// G), or nullptr when the norm asks for Gauss-Jordan (P left untouched).
__device__ __forceinline__ double* inv_unit(double* P, double* G, int wl, int mi) {
  constexpr int LD = Team<32>::LD;
  const int lane = threadIdx.x & 31, u = threadIdx.x & 63;
  double r = 0.0;
#pragma unroll 8
  for (int j = 0; j < 32; j++) r += fabs(P[j * LD + lane]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  const double nrm = r;
  int m = 1;
  double pw = nrm;
  while (pw > 5.0e-17 && m < 8) {
    pw = pw * pw;
    m++;
  }
  int kh = 0;
  double ph = nrm * nrm;
  while (ph > 5.0e-17 && kh < 2 * (m - 1)) {
    ph = ph * nrm;
    kh++;
  }
  if (m >= 8) return nullptr;
  for (int e = u; e < 1024; e += 64) {
    const int col = e >> 5, row = e & 31;
    G[col * LD + row] = ((row == col) ? 1.0 : 0.0) + P[col * LD + row];
  }
  unit_sync(mi);
  if (ph <= 5.0e-17 && kh < 2 * (m - 1)) {
    for (int k = 0; k < kh; k++) {
      mm_unit<MM_IPLUS, true>(P, G, G, nullptr, wl, mi);  // G = I + X G
      unit_sync(mi);
    }
    return G;
  }
  for (int k = 1; k < m; k++) {
    mm_unit<MM_SET, true>(P, P, P, nullptr, wl, mi);  // P = P^2
    unit_sync(mi);
    mm_unit<MM_ACC, true>(G, P, G, G, wl, mi);  // G = G + G P
    unit_sync(mi);
  }
  return G;
}

// column `lane`: dst = x0 + dv, dv issued by tmem_ld32_issue (waited for
// here, after the column of x0 is loaded)
__device__ __forceinline__ void epi_add(const float* x0, float (&dv)[32], float* dst, int lane) {
  float a[32];
  ld_col(x0, lane, a);
  tc::tmem_wait_ld(dv);
#pragma unroll
  for (int r = 0; r < 32; r++) a[r] = a[r] + dv[r];
  st_col(dst, lane, a);
}

template <int N>
__global__ void __launch_bounds__(128, 2) k_adding_tc(Batch b, Work w, pamtra_b200_settings st) {
  static_assert(N == 16, "the split-precision adding kernel is built for NUMMU = 16");
  constexpr int n = 32;
  enum { P1 = 0, P2, P3, P4, P5 };
  enum { RP = 0, RM = 1, TM = 3 };  // fixed roles; T+, R2, T2, G and Z rotate
  extern __shared__ __align__(1024) double smem_raw[];
  AddTcSmem& Q = *reinterpret_cast<AddTcSmem*>(smem_raw);
  AddTcTiles& TL = Q.u.tl;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_base, s_dead, s_gg[2], s_gj[2];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int mi = warp >> 1, slot = warp & 1, u = t & 63;
  AddTcItem& U = Q.it[mi];
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  const int nunits = b.ncol * Fm;
  if (warp == 0) tc::tmem_alloc(&tslot, 128);  // D: columns 0..63, A hi: 64..95, A lo: 96..127
  if (t == 0) {
    tc::mbar_init(&mbar, 1);
    s_dead = 0;
  }
  if (t < N) { Q.mu[t] = w.lob_mu[lob_off(N) + t]; Q.wq[t] = w.lob_w[lob_off(N) + t]; }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t lanes = (uint32_t)(warp * 32) << 16;
  const uint32_t ta_hi = tslot + lanes + 64u, ta_lo = tslot + lanes + 96u;
  const uint32_t dmine = tslot + lanes + 32u * mi;
  const int brow = 32 * mi + lane;
  const RowOff ro(lane);
  uint32_t parity = 0;

  for (;;) {
    __syncthreads();
    if (t == 0) s_base = atomicAdd(&w.counters[6], 2);
    __syncthreads();
    const int base = s_base;
    if (base >= nunits) break;
    // ---- my unit
    const int unit = base + mi;
    int c = 0, fi = 0, L = 0, status = 0;
    bool valid = false;
    if (unit < nunits) {
      c = unit / Fm;
      fi = unit % Fm;
      valid = fi < b.col_nfreq(c) && b.col_nummu(c) == N;
    }
    double wl = 0.0;
    if (valid) {
      L = b.nlyrs[c];
      wl = C_LIGHT / (b.freq(c, fi) * 1.e3);
      status = w.col_status[c];
    }
    float* stk = w.add_stk + (size_t)unit * STK_FLOATS;
    if (s_dead) {  // after a timed-out wait: report the unit, compute nothing
      if (valid && u == 0) {
        reinterpret_cast<int*>(stk + STK_HDR)[0] = 0;
        reinterpret_cast<int*>(stk + STK_HDR)[1] = status | PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
      }
      continue;
    }
    const double* hl = w.hgt_lev + (size_t)c * (Lm + 1);
    const double* tl = w.temp_lev + (size_t)c * (Lm + 1);
    int tp = 2, r2 = 4, t2 = 5, gg = 6, zz = 7;  // rotating roles: T+ (then W), R2 (then V), T2 (then Q),
                                                 // G (Gin first, then T+'), Z (then Y)
    int sstate = 0;   // 0 empty, 1 clear (t1, sp, sm), 2 general
    int k = 0;        // next top-down layer
    int pf_k = -1;    // layer whose record is in (or on its way to) r2 / t2
    bool ok = true;
    for (;;) {
      // ---- advance my unit to its next combine (clear layers, the first scattering layer)
      bool comb = false;
      while (valid && k < L) {
        const int z = L - 1 - k;
        const int pidx = w.pres_idx[(size_t)c * Lm + z];
        if (pidx < 0) {
          // NONSCATTER_LAYER4 (src/radintg4.f90:79-117)
          if (u < n) {
            const int jj = u >> 1, i = u & 1;
            const double zdiff = fabs(hl[z + 1] - hl[z]);
            const double gas = fmax(w.kgas[((size_t)c * Fm + fi) * Lm + z], 0.0);
            const double dtau = zdiff * gas;
            const double p0 = planck(tl[z + 1], wl), p1 = planck(tl[z], wl);
            U.t2[u] = (float)exp(-dtau / Q.mu[jj]);
            double a = 0.0, bq = 0.0;
            if (dtau > 0.0 && i == 0) {
              const double path = dtau / Q.mu[jj];
              const double slope = (p1 - p0) / path;
              a = p1 - slope - (p1 - slope * (1.0 + path)) * exp(-path);
              bq = p0 + slope - (p0 + slope * (1.0 + path)) * exp(-path);
            }
            U.c2p[u] = (float)a;
            U.c2m[u] = (float)bq;
          }
          unit_sync(mi);
          if (sstate == 0) {
            if (u < n) { U.t1[u] = U.t2[u]; U.sp[u] = U.c2p[u]; U.sm[u] = U.c2m[u]; }
            sstate = 1;
          } else if (sstate == 1) {
            if (u < n) {
              const float sp = U.c2p[u] + U.t2[u] * U.sp[u];
              const float sm = U.sm[u] + U.t1[u] * U.c2m[u];
              U.t1[u] = U.t2[u] * U.t1[u];
              U.sp[u] = sp;
              U.sm[u] = sm;
            }
          } else {
            // general stack + clear layer: R+ = t2 R+ t2, T+ = t2 T+, T- = T- t2
            if (u < n) U.nsp[u] = U.c2p[u] + U.t2[u] * (U.sp[u] + mv32(U.m[RP], U.c2m, ro));
            else U.nsm[lane] = U.sm[lane] + mv32(U.m[TM], U.c2m, ro);
            unit_sync(mi);
            for (int s = u; s < 1024; s += 64) {
              int r, cc;
              midx_inv(s, r, cc);
              const float t2i = U.t2[r], t2j = U.t2[cc];
              U.m[RP][s] = t2i * (U.m[RP][s] * t2j);
              U.m[tp][s] = t2i * U.m[tp][s];
              U.m[TM][s] = U.m[TM][s] * t2j;
            }
            if (u < n) { U.sp[u] = U.nsp[u]; U.sm[u] = U.nsm[u]; }
          }
          unit_sync(mi);
          k++;
          continue;
        }
        // scattering layer: its record into r2 / t2
        if (pf_k != k) lay32_fetch(w, pidx * Fm + fi, U, r2, t2, u);
        cp_async_wait_all();
        unit_sync(mi);
        if (u < n) { U.d2p[u] = U.s2p[u]; U.d2m[u] = U.s2m[u]; }
        unit_sync(mi);
        pf_k = -1;
        if (sstate == 2) {
          comb = true;
          break;
        }
        if (sstate == 0) {
          for (int s = u; s < 1024; s += 64) {
            const float rr = U.m[r2][s], tt = U.m[t2][s];
            U.m[RP][s] = rr; U.m[RM][s] = rr; U.m[tp][s] = tt; U.m[TM][s] = tt;
          }
          if (u < n) { U.sp[u] = U.d2p[u]; U.sm[u] = U.d2m[u]; }
        } else {
          // clear stack (t1, sp, sm) + scattering layer
          if (u < n) U.nsp[u] = U.d2p[u] + mv32(U.m[t2], U.sp, ro);
          else U.nsm[lane] = U.sm[lane] + U.t1[lane] * (U.d2m[lane] + mv32(U.m[r2], U.sp, ro));
          for (int s = u; s < 1024; s += 64) {
            int r, cc;
            midx_inv(s, r, cc);
            const float t1i = U.t1[r], t1j = U.t1[cc];
            const float rr = U.m[r2][s], tt = U.m[t2][s];
            U.m[RP][s] = rr;
            U.m[RM][s] = t1i * (rr * t1j);
            U.m[tp][s] = tt * t1j;  // T+ = T2 t1
            U.m[TM][s] = t1i * tt;  // T- = t1 T2
          }
          unit_sync(mi);
          if (u < n) { U.sp[u] = U.nsp[u]; U.sm[u] = U.nsm[u]; }
        }
        sstate = 2;
        unit_sync(mi);
        k++;
      }
      const int pending = __syncthreads_or(comb && u == 0);
      if (!pending) break;
      // ---- one combine of both units (a unit without one idles through the passes)
      if (u == 0) s_gg[mi] = gg;  // published by the barriers of P1
      for (int ph = P1; ph <= P5; ph++) {
        if (comb) {
          int asrc, bsrc;
          if (ph == P1) { bsrc = RP; asrc = slot ? t2 : r2; }
          else if (ph == P2) { bsrc = gg; asrc = slot ? tp : zz; }
          else if (ph == P3) { bsrc = t2; asrc = slot ? tp : zz; }
          else if (ph == P4) { bsrc = TM; asrc = slot ? t2 : r2; }
          else { bsrc = r2; asrc = slot ? zz : tp; }
          build_ab(TL, U.m[asrc], U.m[bsrc], ta_hi, ta_lo, brow, slot, lane, ro);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) tc::mma3_ta(tslot, tslot + 64u, tslot + 96u, TL.b_hi, TL.b_lo, &mbar, tc::IDESC_M128_N64);
        if (comb) {
          // source chains on the CUDA cores while the MMA runs: the S+ chain
          // on slot 0, the S- chain on slot 1, except that warp 0 issues the
          // MMAs meanwhile, so warp 1 runs both chains of unit 0
          const bool cp = (mi == 0) ? (warp == 1) : (slot == 0), cm = (slot == 1);
          if (ph == P1) {
            if (cp) U.wv[lane] = U.sp[lane] + mv32(U.m[RP], U.d2m, ro);
            if (cm) U.mw[lane] = U.d2m[lane] + mv32(U.m[r2], U.sp, ro);
          } else if (ph == P2) {
            if (cp) U.wv2[lane] = mv32(U.m[gg], U.wv, ro);
            if (cm) U.u1[lane] = mv32(U.m[RP], U.mw, ro);
          } else if (ph == P3) {
            if (cp) U.nsp[lane] = U.d2p[lane] + mv32(U.m[t2], U.wv2, ro);
            if (cm) U.u2[lane] = mv32(U.m[gg], U.u1, ro);
          } else if (ph == P4) {
            if (cp) U.u1b[lane] = U.mw[lane] + mv32(U.m[r2], U.u2, ro);
          } else {
            if (cp) U.nsm[lane] = U.sm[lane] + mv32(U.m[TM], U.u1b, ro);
            // W and Y (this pass's A operands) are free now: the next
            // scattering layer goes into their buffers
            int pidx;
            const int kn = next_scat(b, w, c, L, k + 1, pidx);
            if (kn >= 0) lay32_fetch(w, pidx * Fm + fi, U, zz, tp, u);
            pf_k = kn;
          }
        }
        {
          const bool mine = tc::mbar_wait(&mbar, parity, w.spin_limit);
          parity ^= 1;
          ok = __syncthreads_and(mine) != 0;
          tc::fence_after_sync();
        }
        if (!ok) break;
        if (comb) {
          float dv[32];
          tc::tmem_ld32_issue(dmine, dv);
          if (ph == P1) {
            tc::tmem_wait_ld(dv);
            st_col(U.m[slot ? zz : gg], lane, dv);  // Gin = Rp R2;  Z = Rp T2
          } else if (ph == P2) {
            tc::tmem_wait_ld(dv);
            st_col(U.m[slot ? tp : zz], lane, dv);  // Y = G Z over Z;  W = G Tp over T+
          } else if (ph == P3) {
            if (slot == 0) {
              epi_add(U.m[r2], dv, U.m[RP], lane);  // R+' = R2 + T2 Y
            } else {
              tc::tmem_wait_ld(dv);
              st_col(U.m[gg], lane, dv);  // T+' = T2 W over G
            }
          } else if (ph == P4) {
            tc::tmem_wait_ld(dv);
            st_col(U.m[slot ? t2 : r2], lane, dv);  // V = Tm R2 over R2;  Q = Tm T2 over T2
          } else {
            if (slot == 0) epi_add(U.m[RM], dv, U.m[RM], lane);  // R-' = R- + V W
            else epi_add(U.m[t2], dv, U.m[TM], lane);            // T-' = Q + V Y
          }
        }
        __syncthreads();
        if (ph == P1) {
          // FP64 G = (I - Gin)^-1: each unit's two warps invert its own, both
          // units at once (the operand tiles are free until the next pass)
          int gj = 0;
          if (comb) {
            AddTcInv& F = Q.u.fp[mi];
            float* gm = U.m[gg];
            for (int s = u; s < 1024; s += 64) {
              int r, cc;
              midx_inv(s, r, cc);
              F.P[cc * Team<32>::LD + r] = (double)gm[s];
            }
            unit_sync(mi);
            const double* Gi = inv_unit(F.P, F.G, slot, mi);
            if (Gi) {
              for (int s = u; s < 1024; s += 64) {
                int r, cc;
                midx_inv(s, r, cc);
                gm[s] = (float)Gi[cc * Team<32>::LD + r];
              }
            } else {
              gj = 1;
            }
          }
          if (u == 0) s_gj[mi] = gj;
          __syncthreads();
          // ||Gin|| >= 0.74: Gauss-Jordan with partial pivoting, one unit at a
          // time with the whole CTA (the fallback of inv_iminus)
          for (int i = 0; i < 2; i++) {
            if (!s_gj[i]) continue;
            AddTcInv& F = Q.u.fp[i];
            for (int e = t; e < 1024; e += 128) {
              const int col = e >> 5, row = e & 31;
              F.P[col * Team<32>::LD + row] = ((row == col) ? 1.0 : 0.0) - F.P[col * Team<32>::LD + row];
            }
            __syncthreads();
            const int sg = ginv<32>(F.P, F.inv);
            if (sg && mi == i) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
            float* gm = Q.it[i].m[s_gg[i]];
            for (int s = t; s < 1024; s += 128) {
              int r, cc;
              midx_inv(s, r, cc);
              gm[s] = (float)F.P[cc * Team<32>::LD + r];
            }
            __syncthreads();
          }
        }
      }
      if (!ok) break;
      if (comb) {
        // T+' is in G's buffer, the next layer in W's and Y's; V and Q are dead
        const int o_tp = tp, o_r2 = r2, o_t2 = t2, o_gg = gg, o_zz = zz;
        tp = o_gg;
        r2 = o_zz;
        t2 = o_tp;
        gg = o_r2;
        zz = o_t2;
        if (u < n) { U.sp[u] = U.nsp[u]; U.sm[u] = U.nsm[u]; }
        k++;
      }
      __syncthreads();
    }
    if (!ok) {
      if (t == 0) s_dead = 1;
      status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT;
      sstate = 0;
      cp_async_wait_all();
    }
    // ---- the stack of my unit for k_adding_finish
    if (valid) {
      if (sstate == 2) {
        for (int s = u; s < 1024; s += 64) {
          stk[STK_RP + s] = U.m[RP][s];
          stk[STK_RM + s] = U.m[RM][s];
          stk[STK_TP + s] = U.m[tp][s];
          stk[STK_TM + s] = U.m[TM][s];
        }
      }
      if (u < n) {
        stk[STK_SP + u] = U.sp[u];
        stk[STK_SM + u] = U.sm[u];
        stk[STK_T1 + u] = U.t1[u];
      }
      if (u == 0) {
        reinterpret_cast<int*>(stk + STK_HDR)[0] = sstate;
        reinterpret_cast<int*>(stk + STK_HDR)[1] = status;
      }
    }
  }
  if (s_dead) tc::mbar_wait(&mbar, parity ^ 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tslot, 128);
}

// Surface, internal radiances and TB of the units k_adding_tc carried, in
// FP64 from their FP32 stacks (the code of k_adding after its layer loop).
template <int N>
__global__ void __launch_bounds__(RTCfg<N>::T) k_adding_finish(Batch b, Work w, pamtra_b200_settings st,
                                                               pamtra_b200_outputs out) {
  constexpr int n = RTCfg<N>::n, LD = RTCfg<N>::LD, T = RTCfg<N>::T;
  extern __shared__ double smem_raw[];
  AddSmem<N>& S = *reinterpret_cast<AddSmem<N>*>(smem_raw);
  const int t = threadIdx.x;
  const int Fm = b.max_nfreq;
  const int nunits = b.ncol * Fm;
  if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    const int c = unit / Fm, fi = unit % Fm;
    if (fi >= b.col_nfreq(c) || b.col_nummu(c) != N) continue;
    const float* stk = w.add_stk + (size_t)unit * STK_FLOATS;
    const int sstate = reinterpret_cast<const int*>(stk + STK_HDR)[0];
    const int status = reinterpret_cast<const int*>(stk + STK_HDR)[1];
    double *Rp = S.m[0], *Rm = S.m[1], *Tp = S.m[2], *Tm = S.m[3];
    if (sstate == 2) {
      for (int s = t; s < 1024; s += T) {
        int r, cc;
        midx_inv(s, r, cc);
        Rp[cc * LD + r] = stk[STK_RP + s];
        Rm[cc * LD + r] = stk[STK_RM + s];
        Tp[cc * LD + r] = stk[STK_TP + s];
        Tm[cc * LD + r] = stk[STK_TM + s];
      }
    }
    if (t < n) {
      S.sp[t] = stk[STK_SP + t];
      S.sm[t] = stk[STK_SM + t];
      S.t1[t] = stk[STK_T1 + t];
    }
    team_sync();
    const double wl = C_LIGHT / (b.freq(c, fi) * 1.e3);
    adding_finish<N>(b, w, st, out, S, c, fi, b.nlyrs[c], wl, sstate, status, Rp, Rm, Tp, Tm, S.m[4], S.m[5],
                     S.m[6], S.m[7], S.m[8]);
    team_sync();
  }
}

}  // namespace pb
