/*
 * kernels_mixed.cu -- the mixed-precision form (OCO_FORM_MIXED) on sm_100a.
 *
 *   k_solve_mixed     persistent kernel, one thread per (column, wavelength); warp tasks are
 *                     (column, 32 wavelengths) with the column's records streamed into shared
 *                     memory by bulk copies (TMA, mbarrier, bounded waits), or 32 consecutive
 *                     items with direct loads when nw is small.  Forward sweep: log2-space
 *                     opacity, scaled rows and the difference-form Thomas elimination in FP32
 *                     (the source function's exponent as integer + FP32 fraction),
 *                     writing kappa and a scratch record per z (|gamma| or q, 1/kappa, u
 *                     mantissa and exponent); reverse sweep: extended-range FP32
 *                     back-substitution, the differences D_j, and the flux from a 6-value
 *                     window of differences, with FP64 outputs.
 * Output stores carry the streaming cache hint (st.global.cs): they are never read back here,
 * and L2 keeps more of the scratch for the reverse sweep (ragged batch -0.3%).
 * See mixed_core.h for the arithmetic and its relation to the reference.
 */
#include <cuda_runtime.h>

#include "mixed_core.h"
#include "oco_internal.h"

namespace oco {
using namespace oco::mx;

constexpr int MZC = 20;            /* z records per staged chunk (20 x 256 B) */
constexpr int MWARPS = 4;          /* warps per 128-thread block */
constexpr long long kMSpinLimit = 1ll << 26;
#ifndef OCO_MIXED_PREFETCH
#define OCO_MIXED_PREFETCH 4 /* reverse-sweep steps whose scratch loads are issued together */
#endif
#ifndef OCO_MIXED_L2_AHEAD
#define OCO_MIXED_L2_AHEAD 8 /* reverse-sweep steps between the L2 prefetch and the load of a scratch level */
#endif

/* Shared-memory record accessor. */
struct MRec {
  const float *p;
  __device__ __forceinline__ float operator[](int f) const { return p[f]; }
};
struct MGRec {
  const float *p;
  __device__ __forceinline__ float operator[](int f) const { return __ldg(p + f); }
};

__device__ __forceinline__ uint32_t msmem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mtry_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

/* Per-warp double-buffered stream of one column's records (see StagedPillars in
 * kernels_fp64.cu for the protocol). */
struct MStaged {
  float *buf;
  uint32_t bar0;
  const float *src;
  int nz, nchunks, cur;
  uint32_t waits, inflight;
  bool failed;
  __device__ __forceinline__ void issue(int c) {
    const int rows = min(MZC, nz - c * MZC);
    const uint32_t bytes = (uint32_t)(rows * MZN * sizeof(float));
    const uint32_t bar = bar0 + 8u * (c & 1);
    const uint32_t dst = msmem(buf + (c & 1) * (MZC * MZN));
    const size_t g = __cvta_generic_to_global(src + (int64_t)c * MZC * MZN);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(g), "r"(bytes), "r"(bar)
                 : "memory");
  }
  __device__ __forceinline__ bool wait(int b) {
    if (!((inflight >> b) & 1u)) return true;
    const uint32_t bar = bar0 + 8u * b;
    const uint32_t parity = (waits >> b) & 1u;
    long long spins = 0;
    while (!mtry_wait(bar, parity))
      if (++spins > kMSpinLimit) return false;
    waits ^= 1u << b;
    inflight &= ~(1u << b);
    return true;
  }
  __device__ __forceinline__ void begin(const float *column) {
    src = column;
    cur = -1;
    nchunks = (nz + MZC - 1) / MZC;
    __syncwarp();
    if ((threadIdx.x & 31) == 0) issue(0);
    inflight |= 1u;
  }
  __device__ __forceinline__ MRec at(int z) {
    const int c = z / MZC;
    if (c != cur) {
      __syncwarp();
      if (!failed && c + 1 < nchunks) {
        if ((threadIdx.x & 31) == 0) issue(c + 1);
        inflight |= 1u << ((c + 1) & 1);
      }
      if (!failed && !wait(c & 1)) failed = true;
      cur = c;
    }
    return MRec{buf + (c & 1) * (MZC * MZN) + (z - c * MZC) * MZN};
  }
};

struct MDirect {
  const float *base;
  __device__ __forceinline__ MGRec at(int z) { return MGRec{base + (int64_t)z * MZN}; }
};

__device__ __forceinline__ void load_lam32(Lam32 &L, const float *__restrict__ t, int iw, int nw) {
  lam32_from(L, [&](int f) { return __ldg(t + (int64_t)f * nw + iw); });
}

/* Everything one (column, wavelength) item needs besides its records. */
struct MItem {
  const float *lam; /* wavelength table [MLN][nw] of the item's grid */
  int nz, nw, iw;
  float dzf;        /* dz */
  float ldz2i, ldz2f; /* log2(dz^2) = integer + fraction */
  float dz2f;       /* dz^2 */
  double dz1;       /* 1/dz */
  double *U;        /* U of z = 0 (ghost zone 0), stride uz, or NULL; written only when active */
  double *K, *V;    /* kappa and V of z = 0 or NULL, strides kz, vz */
  int64_t uz, kz, vz;
  double *vtop, *vbot; /* emergent-flux destinations or NULL */
};

/* Item of the block kernels: column cl of the chunk, wavelength iw. */
__device__ __forceinline__ MItem block_item(const MixedArgs &a, int64_t cl, int iw) {
  MItem it;
  it.lam = a.lam;
  it.nz = a.nz;
  it.nw = a.nw;
  it.iw = iw;
  it.dzf = (float)a.dz;
  it.ldz2i = a.ldz2i;
  it.ldz2f = a.ldz2f;
  it.dz2f = (float)(a.dz * a.dz);
  it.dz1 = 1.0 / a.dz;
  const int64_t idx = (a.layout == 0) ? (int64_t)iw * a.ld_col + a.c_off + cl : (a.c_off + cl) * a.nw + iw;
  it.U = a.U ? a.U + idx * a.U_is : nullptr;
  it.K = a.K ? a.K + idx * a.K_is : nullptr;
  it.V = a.V ? a.V + idx * a.V_is : nullptr;
  it.uz = a.U_zs;
  it.kz = a.K_zs;
  it.vz = a.V_zs;
  const int64_t pidx = (int64_t)iw * a.ld_col + a.c_off + cl;
  it.vtop = a.Vtop ? a.Vtop + pidx : nullptr;
  it.vbot = a.Vbot ? a.Vbot + pidx : nullptr;
  return it;
}

/* The warp's Thomas scratch, one sequential stream per warp.  A record per level is
 * {v, 1/kappa, u mantissa, u exponent} (see the forward sweep); two formats:
 *   MScratch16  one float4 per lane, 512 bytes per level;
 *   MScratch12  12 bytes per lane, 384 per level: the 32 lanes' {v, 1/kappa} pairs (float2),
 *               then their u mantissas, with u's exponent packed into the spare bits of 1/kappa
 *               and of the mantissa (pack_o1_u, mixed_core.h: u's mantissa lies in [1, 2)).  A
 *               record whose u does not fit (exponent outside [-512, 511], or a mantissa that
 *               is not normal) makes put() return false and the item is flagged for the FP64
 *               re-solve (on the AGN and Athena-style grids the exponent stays in [-420, 90]).
 * Both store the same values, so the results are the same bits.  The 12-byte records move a
 * quarter less scratch for ~4% more instructions: the ragged batches (longest columns first, up
 * to 2048 levels) use them (c4 batch 25.0 -> 23.7 ms), the block solves keep float4 records
 * (12-byte records measured 0.7% slower on the 512-level AGN grid, 2% on the 1024-level
 * precision grid). */
struct MScratch16 {
  static constexpr int LEVEL = 32 * 16;
  char *w; /* the warp's level 0 */
  int lane;
  __device__ __forceinline__ float4 *p(int j) const { return (float4 *)(w + (int64_t)j * LEVEL) + lane; }
  __device__ __forceinline__ const char *level(int j) const { return w + (int64_t)j * LEVEL; }
  __device__ __forceinline__ bool put(int j, const float4 &r) const {
    *p(j) = r;
    return true;
  }
  __device__ __forceinline__ float4 get(int j) const { return *p(j); }
  __device__ __forceinline__ float o1(int j) const { return p(j)->y; }
};
struct MScratch12 {
  static constexpr int LEVEL = 32 * 12;
  char *w; /* the warp's level 0 */
  int lane;
  __device__ __forceinline__ float2 *p2(int j) const { return (float2 *)(w + (int64_t)j * LEVEL) + lane; }
  __device__ __forceinline__ float *p1(int j) const { return (float *)(w + (int64_t)j * LEVEL + 256) + lane; }
  __device__ __forceinline__ const char *level(int j) const { return w + (int64_t)j * LEVEL; }
  __device__ __forceinline__ bool put(int j, const float4 &r) const {
    int w1, w2;
    const bool fits = pack_o1_u(r.y, r.z, __float_as_int(r.w), w1, w2);
    *p2(j) = make_float2(r.x, __int_as_float(w1));
    *p1(j) = __int_as_float(w2);
    return fits;
  }
  __device__ __forceinline__ float4 get(int j) const {
    const float2 a = *p2(j);
    float o1, m;
    int e;
    unpack_o1_u(__float_as_int(a.y), __float_as_int(*p1(j)), o1, m, e);
    return make_float4(a.x, o1, m, __int_as_float(e));
  }
  __device__ __forceinline__ float o1(int j) const { return __int_as_float(__float_as_int(p2(j)->y) & 0x7fffffff); }
};
/* One (column, wavelength) item, its scratch records in sc.  An inactive lane runs the forward
 * sweep (to keep a staged warp in step) and writes nothing. */
/* Returns whether the item's emergent flux is ill-conditioned for this arithmetic: with
 * D_k = u_k - q_k U_{k+1} (all three terms >= 0) and the boundary flux proportional to
 * 37 D_a - 8 D_b + D_c (the 6th-order stencil with mirrored ghost differences; a, b, c the
 * three differences next to the boundary), its condition number with respect to relative
 * errors of u, q and U is
 *   (37 C_a + 8 C_b + C_c) / |37 D_a - 8 D_b + D_c|,   C_k = u_k + q_k U_{k+1};
 * FP32 leaves relative errors of a few 1e-6 in u, q and U, so above `cond` the item is
 * flagged for the FP64 re-solve (kernels_repair.cu).  Columns with nz < 4 are not tested (their flux is the
 * reference's stencil on U).  An item whose scratch records do not fit MScratch is flagged too. */
template <class PA, class SC>
__device__ __forceinline__ bool msolve_item(const MItem &it, bool active, PA &pa, const SC &sc, float cond) {
  const int nz = it.nz;
  Lam32 L;
  load_lam32(L, it.lam, it.iw, it.nw);
  double *Ub = active ? it.U : nullptr;
  double *Kb = active ? it.K : nullptr;
  double *Vb = active ? it.V : nullptr;
  const float dzf = it.dzf, dz2f = it.dz2f, ldz2i = it.ldz2i, ldz2f = it.ldz2f;

  Opac32 cur = opacity(pa.at(0), L);
  Opac32 nxt = opacity(pa.at(1), L);
  float kc = kappa_lin(cur), kn = kappa_lin(nxt);
  Row32 r = row_boundary(kc, cur, dzf, dz2f, ldz2i, ldz2f, false);
  float h = r.e, cprev = r.c;
  float an = 2.0f * rcp(kn + kc); /* a' of row 1; then c' of the row below */
  XF u = xexp2(r.ldi, r.ldf);
  u = xnorm(u.m * (r.w * rcp(r.c + h)), u.e);
  float o1 = rcp(kc);
  if (Kb) __stcs(&Kb[0], (double)kc);
  /* scratch record of z = j: {v_j, 1/kappa_j, u_j mantissa, u_j exponent (int bits)} where v_j holds the
   * smaller of q_j = h_j/(c_j+h_j) and |gamma_{j+1}| = c_j/(c_j+h_j) (they sum to 1; a negative
   * v_j stores -|gamma_{j+1}|), written once row j+1 is known */
  float4 pend = make_float4(0.0f, o1, u.m, __int_as_float(u.e));
  bool fits = true;
  for (int j = 1; j < nz; j++) {
    cur = nxt;
    kc = kn;
    if (j < nz - 1) {
      nxt = opacity(pa.at(j + 1), L);
      kn = kappa_lin(nxt);
      r = row_center(an, kc, kn, cur, dz2f, ldz2i, ldz2f);
      an = r.c;
    } else {
      r = row_boundary(kc, cur, dzf, dz2f, ldz2i, ldz2f, true);
    }
    const float rr = rcp(cprev + h);
    const float qv = h * rr, gv = cprev * rr;
    pend.x = (qv < gv) ? qv : -gv;
    fits &= sc.put(j - 1, pend);
    h = r.e + (r.a * rr) * h; /* a'/(c'+h) is O(1); a' h alone can overflow */
    const float rb = rcp(r.c + h);
    u = xaxpy(xexp2(r.ldi, r.ldf), r.w * rb, u, r.a * rb);
    o1 = rcp(kc);
    if (Kb) __stcs(&Kb[(int64_t)j * it.kz], (double)kc);
    pend = make_float4(0.0f, o1, u.m, __int_as_float(u.e));
    cprev = r.c;
  }
  fits &= sc.put(nz - 1, pend);
  if (!active) return false;
  bool flag = !fits;

  /* reverse sweep */
  const int n = nz;
  const double dz1 = it.dz1;
  const int64_t uz = it.uz;
  XF Un = u; /* U_{n-1} */
  if (Ub) __stcs(&Ub[(int64_t)(3 + n - 1) * uz], xtod(Un));
  double vtop = 0.0, vbot = 0.0;
  if (nz >= 4) {
    /* window of differences d0..d5 = D_k..D_{k+5}; V_{k+3} from it */
    double d0, d1, d2, d3, d4, d5;
    double Uk[3];
    /* D_{n-2}, D_{n-3}, D_{n-4} first (top ghosts mirror them) */
    double Dt[3];
    const float nx4_top_o1 = sc.o1(n - 1); /* 1/kappa_{n-1} */
    float o1t[3];
    double Ct[3]; /* C_k = u_k + q_k U_{k+1} of the top differences */
#pragma unroll
    for (int t = 0; t < 3; t++) {
      const int k = n - 2 - t;
      const float4 w = sc.get(k);
      o1t[t] = w.y;
      const float g1 = (w.x >= 0.0f) ? 1.0f - w.x : -w.x;
      const float qk = (w.x >= 0.0f) ? w.x : 1.0f + w.x;
      XF uj;
      uj.m = w.z;
      uj.e = __float_as_int(w.w);
      const double Uk1 = t == 0 ? xtod(Un) : Uk[t - 1];
      Ct[t] = xtod(uj) + (double)qk * Uk1;
      XF Dj;
      xaxpy2(uj, Un, g1, -qk, Un, Dj);
      Uk[t] = xtod(Un);
      if (Ub) __stcs(&Ub[(int64_t)(3 + k) * uz], Uk[t]);
      Dt[t] = xtod(Dj);
    }
    flag = !(37.0 * Ct[0] + 8.0 * Ct[1] + Ct[2] <= (double)cond * fabs(37.0 * Dt[0] - 8.0 * Dt[1] + Dt[2]));
    const float o1_nm2 = o1t[0], o1_nm3 = o1t[1], o1_nm4 = o1t[2];
    /* top ghosts f(n2+i) = 2 f(n2) - f(n2-i) */
    const double fn = xtod(u);
    if (Ub) {
      __stcs(&Ub[(int64_t)(n + 3) * uz], 2.0 * fn - Uk[0]);
      __stcs(&Ub[(int64_t)(n + 4) * uz], 2.0 * fn - Uk[1]);
      __stcs(&Ub[(int64_t)(n + 5) * uz], 2.0 * fn - Uk[2]);
    }
    /* window for V_{n-1}: D_{n-4} .. D_{n+1} = Dt[2], Dt[1], Dt[0], D_{n-1}=Dt[0], D_n=Dt[1], D_{n+1}=Dt[2] */
    d0 = Dt[2]; d1 = Dt[1]; d2 = Dt[0]; d3 = Dt[0]; d4 = Dt[1]; d5 = Dt[2];
    auto emit = [&](int j, float o1j) -> double {
      const double s1 = d2 + d3;
      const double s2 = (s1 + d1) + d4;
      const double s3 = (s2 + d0) + d5;
      const double df = -((1.0 / 60.0) * (((45.0 * s1) - 9.0 * s2) + s3));
      const double v = ((-(double)o1j) * df) * dz1;
      if (Vb) __stcs(&Vb[(int64_t)j * it.vz], v);
      return v;
    };
    vtop = emit(n - 1, nx4_top_o1);
    double U0 = Uk[2], U1 = Uk[1], U2 = Uk[0], U3 = fn; /* the four lowest U seen so far */
    /* o1 ring: r1, r2, r3 = 1/kappa of k+1, k+2, k+3 before step k */
    float r1 = o1_nm4, r2 = o1_nm3, r3 = o1_nm2;
    auto step = [&](int k, const float4 &w) {
      const float g1 = (w.x >= 0.0f) ? 1.0f - w.x : -w.x; /* |gamma_{k+1}| */
      const float qk = (w.x >= 0.0f) ? w.x : 1.0f + w.x;  /* q_k */
      XF uj;
      uj.m = w.z;
      uj.e = __float_as_int(w.w);
      XF Dj;
      xaxpy2(uj, Un, g1, -qk, Un, Dj);
      const double Uv = xtod(Un);
      if (Ub) __stcs(&Ub[(int64_t)(3 + k) * uz], Uv);
      U3 = U2; U2 = U1; U1 = U0; U0 = Uv;
      d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = xtod(Dj);
      emit(k + 3, r3);
      r3 = r2; r2 = r1; r1 = w.y;
    };
    int k = n - 5;
    constexpr int PF = OCO_MIXED_PREFETCH;
    for (; k >= PF - 1; k -= PF) { /* scratch loads of PF steps hoisted off the serial chain */
      float4 w[PF];
      /* the PF scratch levels OCO_MIXED_L2_AHEAD steps ahead into L2, one bulk request from lane
       * 0 (the warp's levels are contiguous; they were written a whole forward sweep ago and
       * have usually left L2) */
      if (k - PF + 1 - OCO_MIXED_L2_AHEAD >= 0 && (threadIdx.x & 31) == 0) /* PF levels, one bulk request */
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(
                         sc.level(k - PF + 1 - OCO_MIXED_L2_AHEAD))),
                     "r"((uint32_t)(PF * SC::LEVEL))
                     : "memory");
#pragma unroll
      for (int q = 0; q < PF; q++) w[q] = sc.get(k - q);
#pragma unroll
      for (int q = 0; q < PF; q++) step(k - q, w[q]);
    }
    for (; k >= 0; k--) step(k, sc.get(k));
    { /* condition number of the bottom flux from D_0, D_1, D_2 (d0, d1, d2) and U_1..U_3 */
      double Cb = 0.0;
#pragma unroll
      for (int t = 0; t < 3; t++) {
        const float4 w = sc.get(t);
        const float qk = (w.x >= 0.0f) ? w.x : 1.0f + w.x;
        XF uj;
        uj.m = w.z;
        uj.e = __float_as_int(w.w);
        const double Ck = xtod(uj) + (double)qk * (t == 0 ? U1 : (t == 1 ? U2 : U3));
        Cb += (t == 0 ? 37.0 : (t == 1 ? 8.0 : 1.0)) * Ck;
      }
      flag = flag || !(Cb <= (double)cond * fabs(37.0 * d0 - 8.0 * d1 + d2));
    }
    /* bottom ghosts f(n1-i) = 2 f(n1) - f(n1+i); ghost differences mirror D_0, D_1, D_2 */
    if (Ub) {
      __stcs(&Ub[(int64_t)2 * uz], 2.0 * U0 - U1);
      __stcs(&Ub[(int64_t)1 * uz], 2.0 * U0 - U2);
      __stcs(&Ub[0], 2.0 * U0 - U3);
    }
    const double D0 = d0, D1 = d1, D2 = d2;
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D0; /* D_{-1} = D_0 */
    emit(2, r3);
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D1; /* D_{-2} = D_1 */
    emit(1, r2);
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D2; /* D_{-3} = D_2 */
    vbot = emit(0, r1);
  } else { /* nz = 2 or 3: U stencil on the ghosted array (the reference's update order) */
    double f[9];
    const int n1 = 3, n2 = nz + 2;
    f[n1 + nz - 1] = xtod(Un);
    for (int j = nz - 2; j >= 0; j--) {
      const float4 w = sc.get(j);
      const float g1 = (w.x >= 0.0f) ? 1.0f - w.x : -w.x;
      XF uj;
      uj.m = w.z;
      uj.e = __float_as_int(w.w);
      XF Dj;
      xaxpy2(uj, Un, g1, 0.0f, Un, Dj);
      f[n1 + j] = xtod(Un);
    }
    for (int i = 1; i <= 3; i++) {
      f[n1 - i] = 2.0 * f[n1] - f[n1 + i];
      f[n2 + i] = 2.0 * f[n2] - f[n2 - i];
    }
    if (Ub)
      for (int m = 0; m < nz + 6; m++) __stcs(&Ub[(int64_t)m * uz], f[m]);
    for (int j = 0; j < nz; j++) {
      const int c = n1 + j;
      const double df = (1.0 / 60.0) * (((45.0 * (f[c + 1] - f[c - 1])) - 9.0 * (f[c + 2] - f[c - 2])) + (f[c + 3] - f[c - 3]));
      const double v = ((-(double)sc.o1(j)) * df) * dz1;
      if (Vb) __stcs(&Vb[(int64_t)j * it.vz], v);
      if (j == 0) vbot = v;
      if (j == nz - 1) vtop = v;
    }
  }
  if (it.vtop) __stcs(it.vtop, vtop);
  if (it.vbot) __stcs(it.vbot, vbot);
  return flag;
}

/* The re-solve's lists (RepairArgs): each flagged item's id goes to ilist (its index there is
 * the item's slot, also stored beside its bit), and each word of flag bits (a column's 32
 * wavelengths) that receives a bit goes to wlist once.  mark_tile serves the tilings whose warp
 * task is one (column, 32-wavelength tile): the tile is one word and no other warp writes it, so
 * lane 0 stores the warp's ballot.  mark_items serves the tilings whose 32 items may span
 * columns: each flagged lane sets its bit, and the lane that finds its word empty lists it. */
__device__ __forceinline__ void list_items(bool flag, unsigned m, unsigned long long id, int64_t word, int iw,
                                           unsigned long long *ilist, unsigned long long *icount, int *slot) {
  const int lane = threadIdx.x & 31, first = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == first) base = atomicAdd(icount, (unsigned long long)__popc(m));
  base = __shfl_sync(0xffffffffu, base, first);
  if (flag) {
    const unsigned long long pos = base + __popc(m & ((1u << lane) - 1u));
    ilist[pos] = id;
    slot[word * 32 + (iw & 31)] = (int)pos;
  }
}

__device__ __forceinline__ void mark_tile(bool flag, int64_t word, int iw, unsigned long long id, unsigned *bits,
                                          int *slot, unsigned long long *wlist, unsigned long long *wcount,
                                          unsigned long long *ilist, unsigned long long *icount) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if (!m) return;
  if ((threadIdx.x & 31) == 0) {
    bits[word] = m;
    wlist[atomicAdd(wcount, 1ull)] = (unsigned long long)word;
  }
  list_items(flag, m, id, word, iw, ilist, icount, slot);
}

__device__ __forceinline__ void mark_items(bool flag, int64_t word, int iw, unsigned long long id, unsigned *bits,
                                           int *slot, unsigned long long *wlist, unsigned long long *wcount,
                                           unsigned long long *ilist, unsigned long long *icount) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if (!m) return;
  if (flag && atomicOr(bits + word, 1u << (iw & 31)) == 0u) wlist[atomicAdd(wcount, 1ull)] = (unsigned long long)word;
  list_items(flag, m, id, word, iw, ilist, icount, slot);
}

template <class SC>
__global__ void __launch_bounds__(128, 5) k_solve_mixed_staged(const MixedArgs a) {
  __shared__ __align__(128) float s_rec[MWARPS][2 * MZC * MZN];
  __shared__ __align__(8) unsigned long long s_bar[MWARPS][2];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ntiles = (a.nw + 31) / 32;
  const unsigned long long ntasks = (unsigned long long)a.ncol * ntiles;
  const SC sc{(char *)(a.s4 + slot * 32 * (int64_t)a.nz), lane}; /* the warp's scratch, contiguous */
  MStaged pa;
  pa.buf = s_rec[wib];
  pa.bar0 = msmem(&s_bar[wib][0]);
  pa.nz = a.nz;
  pa.waits = 0;
  pa.inflight = 0;
  pa.failed = false;
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(a.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int64_t cl = (int64_t)(task / ntiles);
    const int tile = (int)(task - (unsigned long long)cl * ntiles);
    const int iw_raw = tile * 32 + lane;
    const bool active = iw_raw < a.nw;
    const int iw = active ? iw_raw : a.nw - 1;
    pa.begin(a.rec + cl * (int64_t)a.nz * MZN);
    const bool flag = msolve_item(block_item(a, cl, iw), active, pa, sc, a.repair_cond) ||
                      (active && __ldg(a.colflag + cl) != 0u);
    if (__any_sync(0xffffffffu, pa.failed)) {
      if (lane == 0) atomicOr(&a.status[2], 1ull);
      pa.wait(0);
      pa.wait(1);
      return;
    }
    mark_tile(flag, cl * ntiles + iw / 32, iw, (unsigned long long)(cl * a.nw + iw), a.rbits, a.rslot, a.rlist,
              a.rcount, a.ilist, a.icount);
  }
}

template <class SC>
__global__ void __launch_bounds__(128, 5) k_solve_mixed(const MixedArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nitems = a.ncol * a.nw;
  const unsigned long long ntasks = (unsigned long long)((nitems + 31) / 32);
  const SC sc{(char *)(a.s4 + slot * 32 * (int64_t)a.nz), lane}; /* the warp's scratch, contiguous */
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(a.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int64_t item = (int64_t)task * 32 + lane;
    bool flag = false;
    int64_t word = 0;
    int iw = 0;
    if (item < nitems) {
      const int64_t cl = item / a.nw;
      iw = (int)(item - cl * a.nw);
      MDirect pa{a.rec + cl * (int64_t)a.nz * MZN};
      flag = msolve_item(block_item(a, cl, iw), true, pa, sc, a.repair_cond) || __ldg(a.colflag + cl) != 0u;
      word = cl * ((a.nw + 31) / 32) + iw / 32;
    }
    mark_items(flag, word, iw, (unsigned long long)item, a.rbits, a.rslot, a.rlist, a.rcount, a.ilist, a.icount);
  }
}

static bool mixed_uses_staging(int nw) { return (nw >= 64) || (nw % 32) == 0; }

static const void *solve_mixed_fn(int nw) {
  return mixed_uses_staging(nw) ? (const void *)k_solve_mixed_staged<MScratch16> : (const void *)k_solve_mixed<MScratch16>;
}

int solve_mixed_max_blocks_per_sm(int threads, int nw) {
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, solve_mixed_fn(nw), threads, 0);
  return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_solve_mixed(const MixedArgs &a, int blocks, int threads, cudaStream_t s) {
  void *args[] = {(void *)&a};
  return cudaLaunchKernel(solve_mixed_fn(a.nw), dim3(blocks), dim3(threads), args, 0, s);
}

/* ---- ragged batches ---------------------------------------------------------------------- */

/* Item of a batch: wavelength iw of column c. */
__device__ __forceinline__ MItem batch_item(const MixedBatchArgs &b, const MBatchCol &c, int iw) {
  MItem it;
  it.lam = b.lam + c.lam_off;
  it.nz = c.nz;
  it.nw = c.nw;
  it.iw = iw;
  it.dzf = c.dzf;
  it.ldz2i = c.ldz2i;
  it.ldz2f = c.ldz2f;
  it.dz2f = (float)c.dz2; /* as block_item's (float)(dz * dz) */
  it.dz1 = c.dz1;
  if (b.layout == 0) { /* per column [lambda][z] (z fastest) */
    it.U = b.U ? b.U + c.u_off + (int64_t)iw * (c.nz + 6) : nullptr;
    it.K = b.K ? b.K + c.kv_off + (int64_t)iw * c.nz : nullptr;
    it.V = b.V ? b.V + c.kv_off + (int64_t)iw * c.nz : nullptr;
    it.uz = it.kz = it.vz = 1;
  } else { /* per column [z][lambda] */
    it.U = b.U ? b.U + c.u_off + iw : nullptr;
    it.K = b.K ? b.K + c.kv_off + iw : nullptr;
    it.V = b.V ? b.V + c.kv_off + iw : nullptr;
    it.uz = it.kz = it.vz = c.nw;
  }
  it.vtop = b.Vtop ? b.Vtop + c.flux_off + iw : nullptr;
  it.vbot = b.Vbot ? b.Vbot + c.flux_off + iw : nullptr;
  return it;
}

/* Warp-column tiling: tasks (column, 32-wavelength tile) from the device queue, longest
 * columns first; the column's records stream through the warp's shared-memory buffers. */
template <class SC>
__global__ void __launch_bounds__(128, 5) k_batch_mixed_staged(const MixedBatchArgs b) {
  __shared__ __align__(128) float s_rec[MWARPS][2 * MZC * MZN];
  __shared__ __align__(8) unsigned long long s_bar[MWARPS][2];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const SC sc{(char *)(b.s4 + slot * 32 * (int64_t)b.max_nz), lane}; /* the warp's scratch, contiguous */
  MStaged pa;
  pa.buf = s_rec[wib];
  pa.bar0 = msmem(&s_bar[wib][0]);
  pa.waits = 0;
  pa.inflight = 0;
  pa.failed = false;
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(b.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= (unsigned long long)b.ntasks) break;
    const uint2 t = b.tasks[task];
    const MBatchCol c = b.cols[t.x];
    const int iw_raw = (int)t.y * 32 + lane;
    const bool active = iw_raw < c.nw;
    const int iw = active ? iw_raw : c.nw - 1;
    pa.nz = c.nz;
    pa.begin(b.rec + c.rec_off * MZN);
    const bool flag = msolve_item(batch_item(b, c, iw), active, pa, sc, b.repair_cond) ||
                      (active && __ldg(b.colflag + t.x) != 0u);
    if (__any_sync(0xffffffffu, pa.failed)) {
      if (lane == 0) atomicOr(&b.status[2], 1ull);
      pa.wait(0);
      pa.wait(1);
      return;
    }
    mark_tile(flag, (int64_t)t.x * b.rwstride + iw / 32, iw, ((unsigned long long)t.x << 32) | (unsigned)iw, b.rbits,
              b.rslot, b.rlist, b.rcount, b.ilist, b.icount);
  }
}

/* Packed tiling: the (column, wavelength) items of the columns sorted by nz (longest first)
 * form one list; a warp takes 32 consecutive items, so partial wavelength tiles of one column
 * are filled with the next column's items (similar nz, as the list is sorted). */
template <class SC>
__global__ void __launch_bounds__(128, 5) k_batch_mixed_packed(const MixedBatchArgs b) {
  const int lane = threadIdx.x & 31;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const SC sc{(char *)(b.s4 + slot * 32 * (int64_t)b.max_nz), lane}; /* the warp's scratch, contiguous */
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(b.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= (unsigned long long)b.ntasks) break;
    const int64_t item = (int64_t)task * 32 + lane;
    bool flag = false;
    int32_t col = 0; /* a lane past the end solves column 0's first item without storing */
    int iw = 0;
    if (item < b.nitems) {
      int64_t lo = 0, hi = b.ncol; /* item_pre[lo] <= item < item_pre[hi] */
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(b.item_pre + mid) <= item)
          lo = mid;
        else
          hi = mid;
      }
      col = __ldg(b.order + lo);
      iw = (int)(item - __ldg(b.item_pre + lo));
      const MBatchCol c = b.cols[col];
      MDirect pa{b.rec + c.rec_off * MZN};
      flag = msolve_item(batch_item(b, c, iw), true, pa, sc, b.repair_cond) || __ldg(b.colflag + col) != 0u;
    }
    mark_items(flag, (int64_t)col * b.rwstride + iw / 32, iw, ((unsigned long long)(unsigned)col << 32) | (unsigned)iw,
               b.rbits, b.rslot, b.rlist, b.rcount, b.ilist, b.icount);
  }
}

static const void *batch_mixed_fn(int tiling) {
  return tiling == BATCH_TILING_PACKED ? (const void *)k_batch_mixed_packed<MScratch12>
                                       : (const void *)k_batch_mixed_staged<MScratch12>;
}

int batch_mixed_max_blocks_per_sm(int tiling, int threads) {
  int n = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_mixed_fn(tiling), threads, 0);
  if (e != cudaSuccess || n < 1) n = 1;
  return n;
}

cudaError_t launch_batch_mixed(const MixedBatchArgs &a, int tiling, int blocks, int threads, cudaStream_t s) {
  void *args[] = {(void *)&a};
  return cudaLaunchKernel(batch_mixed_fn(tiling), dim3(blocks), dim3(threads), args, 0, s);
}

}  // namespace oco
