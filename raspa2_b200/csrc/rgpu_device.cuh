/* Device building blocks of the B200 GCMC energy path.
 *
 * Shared by the per-call entry points (capi.cu) and the persistent batched
 * engine (engine.cu). Three precisions are instantiated from one template:
 *   MIXED = 0 : FP64 everywhere (the plain path; parity 1e-9 relative);
 *   MIXED = 1 : FP32 pair terms and exp(ik.r) phases on 32-bit fixed-point
 *               coordinates, FP32 per-warp pair sums, FP64 dS(k) and per-move
 *               sums, FP64 structure factors, totals and acceptance;
 *   MIXED = 2 : as 1, but the real-space charge-charge term of every pair, its
 *               distance and the cut-off test in FP64, with FP64 warp sums
 *               (the framework and adsorbate charges stay FP32), and the
 *               exp(ik.r) phases (of the same exact fixed-point angles) and
 *               their products in FP64; the batched engine only.
 */
#ifndef RGPU_DEVICE_CUH
#define RGPU_DEVICE_CUH

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "erfc_fit.h"
#include "rgpu_types.h"

#define RGPU_FULL 0xffffffffu

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11). One uniform double in [0,1) per
 * (seed, system, step, slot): the block counter is (step lo, step hi,
 * slot/2, system), each half of the 128-bit output gives 53 bits. Every
 * thread can draw any slot, so no random state is shared or carried. */
__host__ __device__ inline void rgpu_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                            uint32_t k0, uint32_t k1, uint32_t out[4])
{
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ inline double rgpu_uniform(uint64_t seed, uint32_t sys, uint64_t step, uint32_t slot)
{
  uint32_t o[4];
  rgpu_philox((uint32_t)step, (uint32_t)(step >> 32), slot >> 1, sys, (uint32_t)seed,
              (uint32_t)(seed >> 32), o);
  uint32_t hi = (slot & 1) ? o[2] : o[0];
  uint32_t lo = (slot & 1) ? o[3] : o[1];
  uint64_t x = ((uint64_t)hi << 21) ^ (uint64_t)(lo >> 11);
  return (double)x * (1.0 / 9007199254740992.0);
}

/* both uniforms of one Philox block: slots 2*blk and 2*blk+1 */
__device__ inline void rgpu_uniform_pair(uint64_t seed, uint32_t sys, uint64_t step, uint32_t blk, double *u)
{
  uint32_t o[4];
  rgpu_philox((uint32_t)step, (uint32_t)(step >> 32), blk, sys, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  u[0] = (double)(((uint64_t)o[0] << 21) ^ (uint64_t)(o[1] >> 11)) * (1.0 / 9007199254740992.0);
  u[1] = (double)(((uint64_t)o[2] << 21) ^ (uint64_t)(o[3] >> 11)) * (1.0 / 9007199254740992.0);
}

/* random-draw slots of one MC step (the oracle uses the same numbering) */
enum {
  SLOT_MOVE = 0, SLOT_MOLECULE = 1, SLOT_VNEW = 2, SLOT_AXIS = 3, SLOT_ACCEPT = 4,
  SLOT_FIRST_SELECT = 15, SLOT_FIRST = 16, SLOT_ORIENT_SELECT = 5, SLOT_ORIENT = 64,
  SLOT_ORIENT_OLD = 128  /* retrace orientations of a reinsertion: 128 + 4 * trial */
};

/* ------------------------------------------------------------------------ */
/* geometry */

/* NINT of src/utils.h:60 */
__device__ __forceinline__ double rgpu_nint(double x) { return (double)(int)(x >= 0.0 ? x + 0.5 : x - 0.5); }

/* fixed-point form of a fractional coordinate f: f mod 1 in units of 2^-32 */
__host__ __device__ inline int rgpu_fix_frac(double f)
{
  f -= floor(f);
  long long v = (long long)llrint(f * 4294967296.0);
  return (int)(uint32_t)(v & 0xffffffffLL);
}

__host__ __device__ inline int rgpu_to_fix(double x, double inv_l)
{
  return rgpu_fix_frac(x * inv_l);
}

/* fractional coordinate r (0..2) of the Cartesian point (x, y, z): x_r / L_r
 * in an orthorhombic box, row r of H^-1 times the point in a triclinic one */
__host__ __device__ inline double rgpu_frac(const RgpuSys &S, int r, double x, double y, double z)
{
  if (!S.triclinic) return (r == 0 ? x : (r == 1 ? y : z)) * S.inv_box[r];
  return S.hinv[3 * r] * x + S.hinv[3 * r + 1] * y + S.hinv[3 * r + 2] * z;
}

/* fixed-point fractional coordinates of a Cartesian point */
__host__ __device__ inline void rgpu_fix3(const RgpuSys &S, double x, double y, double z, int &xi, int &yi, int &zi)
{
  if (!S.triclinic) {
    xi = rgpu_to_fix(x, S.inv_box[0]);
    yi = rgpu_to_fix(y, S.inv_box[1]);
    zi = rgpu_to_fix(z, S.inv_box[2]);
    return;
  }
  xi = rgpu_fix_frac(rgpu_frac(S, 0, x, y, z));
  yi = rgpu_fix_frac(rgpu_frac(S, 1, x, y, z));
  zi = rgpu_fix_frac(rgpu_frac(S, 2, x, y, z));
}

/* the point of fractional coordinates (u0, u1, u2) in the box
 * (ConvertFromABCtoXYZ, src/potentials.c:5548) */
__host__ __device__ inline void rgpu_box_point(const RgpuSys &S, double u0, double u1, double u2, double *p)
{
  if (!S.triclinic) {
    p[0] = S.box[0] * u0;
    p[1] = S.box[1] * u1;
    p[2] = S.box[2] * u2;
    return;
  }
  for (int r = 0; r < 3; r++) p[r] = S.hm[3 * r] * u0 + S.hm[3 * r + 1] * u1 + S.hm[3 * r + 2] * u2;
}

/* triclinic minimum image of a Cartesian difference (src/potentials.h:246-262) */
__device__ __forceinline__ void rgpu_min_image_tri(const RgpuSys &S, double &dx, double &dy, double &dz)
{
  double t[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const double f = S.hinv[3 * r] * dx + S.hinv[3 * r + 1] * dy + S.hinv[3 * r + 2] * dz;
    t[r] = f - rgpu_nint(f);
  }
  dx = S.hm[0] * t[0] + S.hm[1] * t[1] + S.hm[2] * t[2];
  dy = S.hm[3] * t[0] + S.hm[4] * t[1] + S.hm[5] * t[2];
  dz = S.hm[6] * t[0] + S.hm[7] * t[1] + S.hm[8] * t[2];
}

/* Cartesian difference from fixed-point fractional differences (FP32) */
__device__ __forceinline__ void rgpu_fix_to_cart_tri(const RgpuSys &S, int ix, int iy, int iz, float &dx, float &dy,
                                                     float &dz)
{
  const float fx = __int2float_rn(ix), fy = __int2float_rn(iy), fz = __int2float_rn(iz);
  dx = fmaf(S.hmf[0], fx, fmaf(S.hmf[1], fy, S.hmf[2] * fz));
  dy = fmaf(S.hmf[4], fy, S.hmf[5] * fz);
  dz = S.hmf[8] * fz;
}

/* A bead position under evaluation. `atom` is the index of the bead in the
 * adsorbate molecule (selects pseudo-atom type and charge). */
struct BeadPos {
  double x, y, z;
  int xi, yi, zi;
  int atom;
  int excl;       /* adsorbate molecule left out of the sums (-1: none) */
  int pad;
};

__device__ __forceinline__ void bead_set(BeadPos &b, const RgpuSys &S, double x, double y, double z, int atom,
                                         int excl)
{
  b.x = x; b.y = y; b.z = z;
  rgpu_fix3(S, x, y, z, b.xi, b.yi, b.zi);
  b.atom = atom;
  b.excl = excl;
}

/* adsorbate atom record: position + tag = molecule*16 + atom index */
struct AdsRec64 { double x, y, z; long long tag; };

/* ------------------------------------------------------------------------ */
/* pair terms */

/* FP32 real-space Ewald kernel erfc(alpha r)/r * K qa qb with the fitted
 * erfc of erfc_fit.h; rinv = 1/r */
__device__ __forceinline__ float rgpu_erfc_f(float x)
{
  float t = __fdividef(1.0f, fmaf(RGPU_ERFC_P, x, 1.0f));
  float p = RGPU_ERFC_C8;
  p = fmaf(p, t, RGPU_ERFC_C7);
  p = fmaf(p, t, RGPU_ERFC_C6);
  p = fmaf(p, t, RGPU_ERFC_C5);
  p = fmaf(p, t, RGPU_ERFC_C4);
  p = fmaf(p, t, RGPU_ERFC_C3);
  p = fmaf(p, t, RGPU_ERFC_C2);
  p = fmaf(p, t, RGPU_ERFC_C1);
  p = fmaf(p, t, RGPU_ERFC_C0);
  /* exp(-x^2) = 2^(-x^2 log2 e) */
  float e = exp2f(-x * x * 1.4426950408889634f);
  return p * e;
}

/* ------------------------------------------------------------------------ */
/* reductions */
__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(RGPU_FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(RGPU_FULL, v, o);
  return v;
}
__device__ __forceinline__ int warp_or(int v)
{
  return __any_sync(RGPU_FULL, v) ? 1 : 0;
}

/* block-wide sum of two doubles; `red` holds >= 2*32 doubles; every thread
 * returns the totals. Contains __syncthreads: call from all threads. */
__device__ inline void block_sum2(double &a, double &b, double *red)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) { red[2 * w] = a; red[2 * w + 1] = b; }
  __syncthreads();
  if (w == 0) {
    a = lane < nw ? red[2 * lane] : 0.0;
    b = lane < nw ? red[2 * lane + 1] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { red[64] = a; red[65] = b; }
  }
  __syncthreads();
  a = red[64];
  b = red[65];
  __syncthreads();
}

/* ------------------------------------------------------------------------ */
/* Batched bead energies.
 *
 * For P bead positions, sums over framework atoms and over the adsorbate atoms
 * not in the bead's own excluded molecule (BeadPos::excl):
 *   res[p] = {host VDW, host real-space charge, adsorbate VDW, adsorbate real}
 * (CalculateFrameworkVDWEnergyAtPosition src/framework_energy.c:60,
 *  CalculateFrameworkChargeEnergyAtPosition :176,
 *  CalculateInterVDWEnergyAdsorbateAtPosition src/inter_energy.c:321,
 *  CalculateInterChargeEnergyAdsorbateAtPosition :393). For p < pair_check,
 * ovf[p] = 1 when any single pair energy reaches EnergyOverlapCriteria (the
 * early-out of the *EnergyDifference routines, e.g.
 * src/framework_energy.c:4988-4990).
 *
 * A call covers a slice of the framework ([fw_lo, fw_hi): tiles on the mixed
 * path, atoms on the FP64 path) and a slice of the adsorbate atoms, so that
 * the CTAs of a cluster can share one system. Work is split into
 * (position, slice chunk) units spread over the warps; a unit's lane sums are
 * warp-reduced and the per-position sums formed in FP64.
 *
 * Mixed path: the framework is stored as compact tiles of RGPU_TILE = 16
 * atoms with a bounding box each. Lanes first test 32 tile boxes against the
 * cut-off sphere at once (a lower bound of the minimum-image distance), then
 * visit the surviving tiles two at a time (half a warp each); pairs inside
 * the cut-off are appended to a
 * per-warp queue and evaluated 32 at a time, so the LJ + erfc arithmetic runs
 * with all lanes busy instead of under a divergent branch.
 */
struct EvalScratch {
  double *uv;     /* [max units] */
  double *uc;
  int *uo;
  int *next;      /* unit counter of the dynamic schedule; 0 when an evaluation starts */
  unsigned long long *cnt;   /* optional {pairs visited, in cut-off, charged in cut-off} */
  float *qr2;     /* per-warp queue of in-cut-off pairs (mixed path): [nwarps][64], or
                   * [nwarps][64] doubles for MIXED = 2 */
  float *qq;
  int *qt;
};

struct EvalPlan {
  int cf, ca;     /* framework / adsorbate chunks per position */
  int nunits;
};

/* nfw: framework items of the slice (tiles or atoms), nads: adsorbate atoms of
 * the slice, minitems: smallest worthwhile chunk of framework items */
__device__ __forceinline__ EvalPlan eval_plan(int P, int nfw, int nads, int nwarps, int max_units, int minitems)
{
  EvalPlan pl;
  int target = nwarps;
  int cf = target / P;                /* at most one framework unit per warp */
  int maxcf = (nfw + minitems - 1) / minitems;
  if (cf > maxcf) cf = maxcf;
  if (cf < 1) cf = 1;
  int ca = 0;
  if (nads > 0) {
    ca = (nads + 255) / 256;
    if (ca > cf) ca = cf;
    if (ca < 1) ca = 1;
  }
  if (nfw == 0) cf = 0;
  while (P * (cf + ca) > max_units && cf > 1) cf--;
  while (P * (cf + ca) > max_units && ca > 1) ca--;
  pl.cf = cf;
  pl.ca = ca;
  pl.nunits = P * (cf + ca);
  return pl;
}

/* The LJ + real-space term of one queued pair; lane `lane` takes entry
 * `lane` of the warp queue. */
__device__ __forceinline__ void pair_mixed_queued(const RgpuLJf *P, float r2, float qj, bool charged, float qa,
                                                  float alpha, bool check, float thr, float &av, float &ac, int &ov,
                                                  int &nch, int type)
{
  const RgpuLJf L = P[type];
  float ri = rsqrtf(r2);
  ri = ri * fmaf(-0.5f * r2, ri * ri, 1.5f);      /* one Newton step */
  const float ir2 = ri * ri;
  float s6 = L.sig2 * ir2;
  s6 = s6 * s6 * s6;
  const float u = fmaf(L.eps4 * s6, s6 - 1.0f, -L.shift);
  av += u;
  if (check && u >= thr) ov = 1;
  if (charged && qj != 0.0f) {
    nch++;
    const float r = r2 * ri;
    const float uc = qa * qj * rgpu_erfc_f(alpha * r) * ri;
    ac += uc;
    if (check && uc >= thr) ov = 1;
  }
}

/* Per-warp queue of pairs inside the cut-off (squared distance, partner
 * charge, LJ table index). Lanes append their pair when `in`; whenever 32 or
 * more pairs are queued, all lanes evaluate 32 of them at once, so the pair
 * arithmetic runs with every lane busy instead of under a divergent branch. */
struct PairQueue {
  float *r2, *q;
  int *t;
  int n;
  const RgpuLJf *P;
  bool charged, check;
  float qa, alpha, thr;
};

__device__ __forceinline__ void queue_add(PairQueue &Q, bool in, float r2, float q, int t, float &av, float &ac,
                                          int &ov, int &nin, int &nch)
{
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(RGPU_FULL, in);
  if (in) {
    const int p = Q.n + __popc(bal & ((1u << lane) - 1u));
    Q.r2[p] = r2;
    Q.q[p] = q;
    Q.t[p] = t;
  }
  Q.n += __popc(bal);
  if (Q.n >= 32) {
    __syncwarp();
    const float e_r2 = Q.r2[lane], e_q = Q.q[lane];
    const int e_t = Q.t[lane];
    float t_r2 = 0.0f, t_q = 0.0f;
    int t_t = 0;
    if (lane < Q.n - 32) { t_r2 = Q.r2[32 + lane]; t_q = Q.q[32 + lane]; t_t = Q.t[32 + lane]; }
    __syncwarp();
    if (lane < Q.n - 32) { Q.r2[lane] = t_r2; Q.q[lane] = t_q; Q.t[lane] = t_t; }
    nin++;
    pair_mixed_queued(Q.P, e_r2, e_q, Q.charged, Q.qa, Q.alpha, Q.check, Q.thr, av, ac, ov, nch, e_t);
    Q.n -= 32;
    __syncwarp();
  }
}

/* evaluates what is left in the queue */
__device__ __forceinline__ void queue_drain(PairQueue &Q, float &av, float &ac, int &ov, int &nin, int &nch)
{
  const int lane = threadIdx.x & 31;
  __syncwarp();
  if (lane < Q.n) {
    nin++;
    pair_mixed_queued(Q.P, Q.r2[lane], Q.q[lane], Q.charged, Q.qa, Q.alpha, Q.check, Q.thr, av, ac, ov, nch,
                      Q.t[lane]);
  }
  Q.n = 0;
  __syncwarp();
}

/* The same queue for MIXED = 2: the squared distance is queued in FP64; the
 * LJ term is formed in FP32 from it as above, the real-space charge-charge
 * term in FP64 (erfc of the CUDA math library) and summed per lane in FP64. */
struct PairQueueQ {
  double *r2;
  float *q;
  int *t;
  int n;
  const RgpuLJf *P;
  bool charged, check;
  double qa, alpha;
  float thr;
};

__device__ __forceinline__ void pair_qq_queued(const PairQueueQ &Q, double r2d, float qj, int type, float &av,
                                               double &ac, int &ov, int &nch)
{
  const RgpuLJf L = Q.P[type];
  const float r2 = (float)r2d;
  float ri = rsqrtf(r2);
  ri = ri * fmaf(-0.5f * r2, ri * ri, 1.5f);
  float s6 = L.sig2 * (ri * ri);
  s6 = s6 * s6 * s6;
  const float u = fmaf(L.eps4 * s6, s6 - 1.0f, -L.shift);
  av += u;
  if (Q.check && u >= Q.thr) ov = 1;
  if (Q.charged && qj != 0.0f) {
    nch++;
    const double r = sqrt(r2d);
    const double uc = Q.qa * (double)qj * (erfc(Q.alpha * r) / r);
    ac += uc;
    if (Q.check && uc >= (double)Q.thr) ov = 1;
  }
}

__device__ __forceinline__ void queue_add(PairQueueQ &Q, bool in, double r2, float q, int t, float &av, double &ac,
                                          int &ov, int &nin, int &nch)
{
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(RGPU_FULL, in);
  if (in) {
    const int p = Q.n + __popc(bal & ((1u << lane) - 1u));
    Q.r2[p] = r2;
    Q.q[p] = q;
    Q.t[p] = t;
  }
  Q.n += __popc(bal);
  if (Q.n >= 32) {
    __syncwarp();
    const double e_r2 = Q.r2[lane];
    const float e_q = Q.q[lane];
    const int e_t = Q.t[lane];
    double t_r2 = 0.0;
    float t_q = 0.0f;
    int t_t = 0;
    if (lane < Q.n - 32) { t_r2 = Q.r2[32 + lane]; t_q = Q.q[32 + lane]; t_t = Q.t[32 + lane]; }
    __syncwarp();
    if (lane < Q.n - 32) { Q.r2[lane] = t_r2; Q.q[lane] = t_q; Q.t[lane] = t_t; }
    nin++;
    pair_qq_queued(Q, e_r2, e_q, e_t, av, ac, ov, nch);
    Q.n -= 32;
    __syncwarp();
  }
}

__device__ __forceinline__ void queue_drain(PairQueueQ &Q, float &av, double &ac, int &ov, int &nin, int &nch)
{
  const int lane = threadIdx.x & 31;
  __syncwarp();
  if (lane < Q.n) {
    nin++;
    pair_qq_queued(Q, Q.r2[lane], Q.q[lane], Q.t[lane], av, ac, ov, nch);
  }
  Q.n = 0;
  __syncwarp();
}

/* FP64 Cartesian difference of two fixed-point positions (MIXED = 2) */
template <bool TRI>
__device__ __forceinline__ double rgpu_fix_r2_d(const RgpuSys &S, int ix, int iy, int iz)
{
  const double k = 2.3283064365386963e-10;     /* 2^-32 */
  const double fx = (double)ix * k, fy = (double)iy * k, fz = (double)iz * k;
  if (!TRI) {
    const double dx = fx * S.box[0], dy = fy * S.box[1], dz = fz * S.box[2];
    return dx * dx + dy * dy + dz * dz;
  }
  const double dx = S.hm[0] * fx + S.hm[1] * fy + S.hm[2] * fz;
  const double dy = S.hm[4] * fy + S.hm[5] * fz;
  const double dz = S.hm[8] * fz;
  return dx * dx + dy * dy + dz * dz;
}

static_assert(RGPU_TILE == 16, "unit_tiles_mixed visits two tiles per warp pass, one per half warp");

/* framework tiles [t0, t1) for bead b, FP32 path (warp-wide); TRI: the
 * box is triclinic (S.triclinic) */
template <bool TRI>
__device__ __forceinline__ void unit_tiles_mixed(const RgpuSys &S, const int4 *fw, const TileRec *tiles, int t0, int t1,
                                                 const BeadPos &b, bool check, float &av, float &ac, int &ov,
                                                 int &nin, int &nch, int &nvis, float *qr2, float *qq, int *qt)
{
  const int lane = threadIdx.x & 31;
  const float sx = S.fix_scale[0], sy = S.fix_scale[1], sz = S.fix_scale[2];
  const float rc2 = S.rc2f;
  PairQueue Q;
  Q.r2 = qr2; Q.q = qq; Q.t = qt; Q.n = 0;
  Q.P = S.ljf_bf[b.atom];
  Q.qa = S.mol_qf[b.atom] * S.coulombf;
  Q.charged = S.fw_charged && Q.qa != 0.0f;
  Q.check = check;
  Q.alpha = S.alphaf;
  Q.thr = (float)S.overlap;
  const bool tri = TRI;
  for (int tb = t0; tb < t1; tb += 32) {
    const int t = tb + lane;
    bool vis = false;
    int tn = 0;                  /* atoms of this lane's tile */
    if (t < t1) {
      const TileRec tr = tiles[t];
      tn = tr.c.w;
      if (!tri) {
        float dx = fmaxf(fabsf(__int2float_rn(tr.c.x - b.xi) * sx) - tr.h.x, 0.0f);
        float dy = fmaxf(fabsf(__int2float_rn(tr.c.y - b.yi) * sy) - tr.h.y, 0.0f);
        float dz = fmaxf(fabsf(__int2float_rn(tr.c.z - b.zi) * sz) - tr.h.z, 0.0f);
        vis = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < rc2;
      } else {
        /* triclinic tile: h = fractional half extents, h.w = Cartesian
         * radius. Every atom's wrapped fractional offset along axis r is at
         * least |t_r| - h_r, so it lies at least that many perpendicular
         * widths away; when no atom can wrap differently from the centre
         * (|t_r| + h_r < 1/2 on every axis), it also lies at least the
         * centre's distance minus the radius away. */
        const int ix = tr.c.x - b.xi, iy = tr.c.y - b.yi, iz = tr.c.z - b.zi;
        const float tx = fabsf(__int2float_rn(ix) * 2.3283064365386963e-10f);
        const float ty = fabsf(__int2float_rn(iy) * 2.3283064365386963e-10f);
        const float tz = fabsf(__int2float_rn(iz) * 2.3283064365386963e-10f);
        const float m = fmaxf(fmaxf((tx - tr.h.x) * S.wperp[0], (ty - tr.h.y) * S.wperp[1]),
                              (tz - tr.h.z) * S.wperp[2]);
        vis = !(m > 0.0f && m * m >= rc2);
        if (vis && tx + tr.h.x < 0.5f && ty + tr.h.y < 0.5f && tz + tr.h.z < 0.5f) {
          float dx, dy, dz;
          rgpu_fix_to_cart_tri(S, ix, iy, iz, dx, dy, dz);
          const float e = fmaxf(sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz))) - tr.h.w, 0.0f);
          vis = e * e < rc2;
        }
      }
    }
    unsigned m = __ballot_sync(RGPU_FULL, vis);
    /* two visible tiles per pass of the warp: lanes 0-15 take the atoms of
     * the first, lanes 16-31 those of the second */
    const int half = lane >> 4, hl = lane & 15;
    while (m) {
      const int i1 = __ffs(m) - 1;
      m &= m - 1;
      const int i2 = m ? __ffs(m) - 1 : -1;
      m &= m - 1;
      const int n1 = __shfl_sync(RGPU_FULL, tn, i1);
      const int n2s = __shfl_sync(RGPU_FULL, tn, i2 >= 0 ? i2 : 0);
      const int n2 = i2 >= 0 ? n2s : 0;
      nvis += n1 + n2;
      const int mine = half ? i2 : i1, nmine = half ? n2 : n1;
      int4 f = make_int4(0, 0, 0, 0);
      if (hl < nmine) f = fw[(tb + mine) * RGPU_TILE + hl];
      float dx, dy, dz;
      if (!tri) {
        dx = __int2float_rn(f.x - b.xi) * sx;
        dy = __int2float_rn(f.y - b.yi) * sy;
        dz = __int2float_rn(f.z - b.zi) * sz;
      } else {
        rgpu_fix_to_cart_tri(S, f.x - b.xi, f.y - b.yi, f.z - b.zi, dx, dy, dz);
      }
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      queue_add(Q, hl < nmine && r2 < rc2, r2, __int_as_float(f.w), f.z & 3, av, ac, ov, nin, nch);
    }
  }
  queue_drain(Q, av, ac, ov, nin, nch);
}

/* unit_tiles_mixed for MIXED = 2: the same tile culling in FP32, then each
 * visited pair's distance and cut-off test in FP64 (queued as FP64), its LJ
 * term in FP32 and its real-space charge-charge term in FP64; qr2 holds 64
 * doubles */
template <bool TRI>
__device__ __forceinline__ void unit_tiles_cc64(const RgpuSys &S, const int4 *fw, const TileRec *tiles, int t0, int t1,
                                                const BeadPos &b, bool check, float &av,
                                                double &ac, int &ov, int &nin, int &nch, int &nvis, float *qr2,
                                                float *qq, int *qt)
{
  const int lane = threadIdx.x & 31;
  const float sx = S.fix_scale[0], sy = S.fix_scale[1], sz = S.fix_scale[2];
  const float rc2 = S.rc2f;
  PairQueueQ Q;
  Q.r2 = reinterpret_cast<double *>(qr2); Q.q = qq; Q.t = qt; Q.n = 0;
  Q.P = S.ljf_bf[b.atom];
  Q.qa = S.mol_q[b.atom] * S.coulomb;
  Q.alpha = S.alpha;
  Q.charged = S.fw_charged && Q.qa != 0.0;
  Q.check = check;
  Q.thr = (float)S.overlap;
  const bool tri = TRI;
  for (int tb = t0; tb < t1; tb += 32) {
    const int t = tb + lane;
    bool vis = false;
    int tn = 0;                  /* atoms of this lane's tile */
    if (t < t1) {
      const TileRec tr = tiles[t];
      tn = tr.c.w;
      if (!tri) {
        float dx = fmaxf(fabsf(__int2float_rn(tr.c.x - b.xi) * sx) - tr.h.x, 0.0f);
        float dy = fmaxf(fabsf(__int2float_rn(tr.c.y - b.yi) * sy) - tr.h.y, 0.0f);
        float dz = fmaxf(fabsf(__int2float_rn(tr.c.z - b.zi) * sz) - tr.h.z, 0.0f);
        vis = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < rc2;
      } else {
        /* triclinic tile: h = fractional half extents, h.w = Cartesian
         * radius. Every atom's wrapped fractional offset along axis r is at
         * least |t_r| - h_r, so it lies at least that many perpendicular
         * widths away; when no atom can wrap differently from the centre
         * (|t_r| + h_r < 1/2 on every axis), it also lies at least the
         * centre's distance minus the radius away. */
        const int ix = tr.c.x - b.xi, iy = tr.c.y - b.yi, iz = tr.c.z - b.zi;
        const float tx = fabsf(__int2float_rn(ix) * 2.3283064365386963e-10f);
        const float ty = fabsf(__int2float_rn(iy) * 2.3283064365386963e-10f);
        const float tz = fabsf(__int2float_rn(iz) * 2.3283064365386963e-10f);
        const float m = fmaxf(fmaxf((tx - tr.h.x) * S.wperp[0], (ty - tr.h.y) * S.wperp[1]),
                              (tz - tr.h.z) * S.wperp[2]);
        vis = !(m > 0.0f && m * m >= rc2);
        if (vis && tx + tr.h.x < 0.5f && ty + tr.h.y < 0.5f && tz + tr.h.z < 0.5f) {
          float dx, dy, dz;
          rgpu_fix_to_cart_tri(S, ix, iy, iz, dx, dy, dz);
          const float e = fmaxf(sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz))) - tr.h.w, 0.0f);
          vis = e * e < rc2;
        }
      }
    }
    unsigned m = __ballot_sync(RGPU_FULL, vis);
    /* two visible tiles per pass of the warp: lanes 0-15 take the atoms of
     * the first, lanes 16-31 those of the second */
    const int half = lane >> 4, hl = lane & 15;
    while (m) {
      const int i1 = __ffs(m) - 1;
      m &= m - 1;
      const int i2 = m ? __ffs(m) - 1 : -1;
      m &= m - 1;
      const int n1 = __shfl_sync(RGPU_FULL, tn, i1);
      const int n2s = __shfl_sync(RGPU_FULL, tn, i2 >= 0 ? i2 : 0);
      const int n2 = i2 >= 0 ? n2s : 0;
      nvis += n1 + n2;
      const int mine = half ? i2 : i1, nmine = half ? n2 : n1;
      int4 f = make_int4(0, 0, 0, 0);
      if (hl < nmine) f = fw[(tb + mine) * RGPU_TILE + hl];
      const double r2 = rgpu_fix_r2_d<TRI>(S, f.x - b.xi, f.y - b.yi, f.z - b.zi);
      queue_add(Q, hl < nmine && r2 < S.rc2, r2, __int_as_float(f.w), f.z & 3, av, ac, ov, nin, nch);
    }
  }
  queue_drain(Q, av, ac, ov, nin, nch);
}

/* framework atoms [lo, hi) of the type-sorted FP64 layout; TRI: the box is
 * triclinic (S.triclinic) */
template <bool TRI>
__device__ __forceinline__ void unit_fw_fp64(const RgpuSys &S, const double4 *fw, const BeadPos &b, int lo,
                                             int hi, bool check, double &av, double &ac, int &ov, int &nin, int &nch,
                                             int &nvis)
{
  const int lane = threadIdx.x & 31;
  const double Lx = S.box[0], Ly = S.box[1], Lz = S.box[2];
  const double ix = S.inv_box[0], iy = S.inv_box[1], iz = S.inv_box[2];
  const double rc2 = S.rc2, thr = S.overlap;
  const double qa = S.mol_q[b.atom] * S.coulomb;
  const bool charged = S.fw_charged && qa != 0.0;
  const double alpha = S.alpha;
  nvis += hi - lo;
  for (int s = 0; s < S.nseg; s++) {
    int a0 = max(lo, S.seg_start[s]), a1 = min(hi, S.seg_start[s + 1]);
    if (a0 >= a1) continue;
    const RgpuLJ P = S.lj_bf[b.atom][s];
    for (int j = a0 + lane; j < a1; j += 32) {
      double4 f = fw[j];
      double dx = b.x - f.x, dy = b.y - f.y, dz = b.z - f.z;
      if (!TRI) {
        dx -= Lx * rgpu_nint(dx * ix);
        dy -= Ly * rgpu_nint(dy * iy);
        dz -= Lz * rgpu_nint(dz * iz);
      } else {
        rgpu_min_image_tri(S, dx, dy, dz);
      }
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < rc2) {
        nin++;
        double s6 = P.sig2 / r2;
        s6 = s6 * s6 * s6;
        double u = P.eps4 * (s6 * (s6 - 1.0)) - P.shift;
        av += u;
        if (check && u >= thr) ov = 1;
        if (charged) {
          nch++;
          double r = sqrt(r2);
          double uc = qa * f.w * (erfc(alpha * r) / r);
          ac += uc;
          if (check && uc >= thr) ov = 1;
        }
      }
    }
  }
}

template <bool TRI>
__device__ __forceinline__ void unit_ads_mixed(const RgpuSys &S, const int4 *ads, const BeadPos &b, int lo,
                                               int hi, int exclude, bool check, float &av, float &ac, int &ov,
                                               int &nin, int &nch, int &nvis, float *qr2, float *qq, int *qt)
{
  const int lane = threadIdx.x & 31;
  const float sx = S.fix_scale[0], sy = S.fix_scale[1], sz = S.fix_scale[2];
  const float rc2 = S.rc2f;
  PairQueue Q;
  Q.r2 = qr2; Q.q = qq; Q.t = qt; Q.n = 0;
  Q.P = S.ljf_bb[b.atom];
  Q.qa = S.mol_qf[b.atom] * S.coulombf;
  Q.charged = S.mol_charged && Q.qa != 0.0f;
  Q.check = check;
  Q.alpha = S.alphaf;
  Q.thr = (float)S.overlap;
  nvis += hi - lo;
  for (int jb = lo; jb < hi; jb += 32) {
    const int j = jb + lane;
    bool in = false;
    float r2 = 0.0f, q = 0.0f;
    int at = 0;
    if (j < hi) {
      const int4 f = ads[j];
      if ((f.w >> 4) != exclude) {
        at = f.w & 15;
        float dx, dy, dz;
        if (!TRI) {
          dx = __int2float_rn(f.x - b.xi) * sx;
          dy = __int2float_rn(f.y - b.yi) * sy;
          dz = __int2float_rn(f.z - b.zi) * sz;
        } else {
          rgpu_fix_to_cart_tri(S, f.x - b.xi, f.y - b.yi, f.z - b.zi, dx, dy, dz);
        }
        r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        in = r2 < rc2;
        q = S.mol_qf[at];
      }
    }
    queue_add(Q, in, r2, q, at, av, ac, ov, nin, nch);
  }
  queue_drain(Q, av, ac, ov, nin, nch);
}

/* unit_ads_mixed for MIXED = 2 (see unit_tiles_cc64) */
template <bool TRI>
__device__ __forceinline__ void unit_ads_cc64(const RgpuSys &S, const int4 *ads, const BeadPos &b, int lo, int hi,
                                              int exclude, bool check, float &av, double &ac, int &ov, int &nin,
                                              int &nch, int &nvis, float *qr2, float *qq, int *qt)
{
  const int lane = threadIdx.x & 31;
  PairQueueQ Q;
  Q.r2 = reinterpret_cast<double *>(qr2); Q.q = qq; Q.t = qt; Q.n = 0;
  Q.P = S.ljf_bb[b.atom];
  Q.qa = S.mol_q[b.atom] * S.coulomb;
  Q.alpha = S.alpha;
  Q.charged = S.mol_charged && Q.qa != 0.0;
  Q.check = check;
  Q.thr = (float)S.overlap;
  nvis += hi - lo;
  for (int jb = lo; jb < hi; jb += 32) {
    const int j = jb + lane;
    bool in = false;
    double r2 = 0.0;
    float q = 0.0f;
    int at = 0;
    if (j < hi) {
      const int4 f = ads[j];
      if ((f.w >> 4) != exclude) {
        at = f.w & 15;
        r2 = rgpu_fix_r2_d<TRI>(S, f.x - b.xi, f.y - b.yi, f.z - b.zi);
        in = r2 < S.rc2;
        q = S.mol_qf[at];
      }
    }
    queue_add(Q, in, r2, q, at, av, ac, ov, nin, nch);
  }
  queue_drain(Q, av, ac, ov, nin, nch);
}

template <bool TRI>
__device__ __forceinline__ void unit_ads_fp64(const RgpuSys &S, const AdsRec64 *ads, const BeadPos &b, int lo,
                                              int hi, int exclude, bool check, double &av, double &ac, int &ov,
                                              int &nin, int &nch, int &nvis)
{
  const int lane = threadIdx.x & 31;
  const double Lx = S.box[0], Ly = S.box[1], Lz = S.box[2];
  const double ix = S.inv_box[0], iy = S.inv_box[1], iz = S.inv_box[2];
  const double rc2 = S.rc2, thr = S.overlap;
  const double qa = S.mol_q[b.atom] * S.coulomb;
  const bool charged = S.mol_charged && qa != 0.0;
  const double alpha = S.alpha;
  nvis += hi - lo;
  for (int j = lo + lane; j < hi; j += 32) {
    AdsRec64 f = ads[j];
    int tag = (int)f.tag;
    if ((tag >> 4) == exclude) continue;
    int at = tag & 15;
    double dx = b.x - f.x, dy = b.y - f.y, dz = b.z - f.z;
    if (!TRI) {
      dx -= Lx * rgpu_nint(dx * ix);
      dy -= Ly * rgpu_nint(dy * iy);
      dz -= Lz * rgpu_nint(dz * iz);
    } else {
      rgpu_min_image_tri(S, dx, dy, dz);
    }
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < rc2) {
      nin++;
      const RgpuLJ P = S.lj_bb[b.atom][at];
      double s6 = P.sig2 / r2;
      s6 = s6 * s6 * s6;
      double u = P.eps4 * (s6 * (s6 - 1.0)) - P.shift;
      av += u;
      if (check && u >= thr) ov = 1;
      double qb = S.mol_q[at];
      if (charged && qb != 0.0) {
        nch++;
        double r = sqrt(r2);
        double uc = qa * qb * (erfc(alpha * r) / r);
        ac += uc;
        if (check && uc >= thr) ov = 1;
      }
    }
  }
}

/* Framework and adsorbate slices of one evaluation */
struct EvalSlice {
  const void *fw;          /* int4 atoms (mixed, tiled) or double4 atoms (FP64, type-sorted) */
  const TileRec *tiles;    /* mixed only */
  int fw_lo, fw_hi;        /* tiles (mixed) or atoms (FP64) */
  const void *ads;         /* int4 or AdsRec64 records */
  int ads_lo, ads_hi;
};

/* The (position, chunk) units of P positions over the slice: the unit of
 * position p and chunk c writes its FP64 sums and overlap flag to
 * sc.uv/uc/uo[p * (cf + ca) + c]. Warps take units dynamically from
 * *sc.next (framework chunks of every position first, then adsorbate
 * chunks), fetching the next index while they work on the current one, so
 * the warps of the block finish together. The stored sums do not depend on
 * which warp evaluated a unit. No block barrier; *sc.next is left past the
 * last unit (the caller resets it after its barrier). Returns the plan. */
template <int MIXED>
__device__ __forceinline__ EvalPlan eval_units(const RgpuSys &S, const EvalSlice &sl, const BeadPos *pos, int P, int pair_check,
                               EvalScratch sc, int max_units)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nfw = sl.fw_hi - sl.fw_lo, nads = sl.ads_hi - sl.ads_lo;
  const EvalPlan pl = eval_plan(P, nfw, nads, nw, max_units, MIXED ? 2 : 64);
  const int per = pl.cf + pl.ca;
  const int nfu = P * pl.cf;     /* framework units */
  /* work counts of this lane, summed over its units (statistics only) */
  int nin = 0, nch = 0, nvis = 0;
  int v = 0;
  if (lane == 0) v = atomicAdd(sc.next, 1);
  v = __shfl_sync(RGPU_FULL, v, 0);
  while (v < pl.nunits) {
    int vn = 0;
    if (lane == 0) vn = atomicAdd(sc.next, 1);
    int p, c;
    if (v < nfu) {
      c = v / P;
      p = v - c * P;
    } else {
      const int v2 = v - nfu;
      const int ca = v2 / P;
      p = v2 - ca * P;
      c = pl.cf + ca;
    }
    const int u = p * per + c;
    const BeadPos b = pos[p];
    const bool check = p < pair_check;
    int ov = 0;
    double e_v, e_q;
    int lo, hi;
    /* chunk bounds; item counts stay far below 2^31 / RGPU_MAX_UNITS */
    if (c < pl.cf) {
      lo = sl.fw_lo + (int)((unsigned)(nfw * c) / (unsigned)pl.cf);
      hi = sl.fw_lo + (int)((unsigned)(nfw * (c + 1)) / (unsigned)pl.cf);
    } else {
      const int cc = c - pl.cf;
      lo = sl.ads_lo + (int)((unsigned)(nads * cc) / (unsigned)pl.ca);
      hi = sl.ads_lo + (int)((unsigned)(nads * (cc + 1)) / (unsigned)pl.ca);
    }
    if constexpr (MIXED == 2) {
      float av = 0.0f;
      double ac = 0.0;
      float *qr2 = sc.qr2 + 128 * w;   /* 64 FP64 squared distances per warp */
      if (c < pl.cf) {
        if (S.triclinic)
          unit_tiles_cc64<true>(S, (const int4 *)sl.fw, sl.tiles, lo, hi, b, check, av, ac, ov, nin, nch, nvis,
                                qr2, sc.qq + 64 * w, sc.qt + 64 * w);
        else
          unit_tiles_cc64<false>(S, (const int4 *)sl.fw, sl.tiles, lo, hi, b, check, av, ac, ov, nin, nch, nvis,
                                 qr2, sc.qq + 64 * w, sc.qt + 64 * w);
      } else if (S.triclinic) {
        unit_ads_cc64<true>(S, (const int4 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis,
                            qr2, sc.qq + 64 * w, sc.qt + 64 * w);
      } else {
        unit_ads_cc64<false>(S, (const int4 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis,
                             qr2, sc.qq + 64 * w, sc.qt + 64 * w);
      }
      e_v = warp_sum((double)av);
      e_q = warp_sum(ac);
    } else if (MIXED) {
      float av = 0.0f, ac = 0.0f;
      if (c < pl.cf) {
        if (S.triclinic)
          unit_tiles_mixed<true>(S, (const int4 *)sl.fw, sl.tiles, lo, hi, b, check, av, ac, ov, nin, nch, nvis,
                                 sc.qr2 + 64 * w, sc.qq + 64 * w, sc.qt + 64 * w);
        else
          unit_tiles_mixed<false>(S, (const int4 *)sl.fw, sl.tiles, lo, hi, b, check, av, ac, ov, nin, nch, nvis,
                                  sc.qr2 + 64 * w, sc.qq + 64 * w, sc.qt + 64 * w);
      } else if (S.triclinic) {
        unit_ads_mixed<true>(S, (const int4 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis,
                             sc.qr2 + 64 * w, sc.qq + 64 * w, sc.qt + 64 * w);
      } else {
        unit_ads_mixed<false>(S, (const int4 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis,
                              sc.qr2 + 64 * w, sc.qq + 64 * w, sc.qt + 64 * w);
      }
      e_v = (double)warp_sum(av);
      e_q = (double)warp_sum(ac);
    } else {
      double av = 0.0, ac = 0.0;
      if (c < pl.cf) {
        if (S.triclinic)
          unit_fw_fp64<true>(S, (const double4 *)sl.fw, b, lo, hi, check, av, ac, ov, nin, nch, nvis);
        else
          unit_fw_fp64<false>(S, (const double4 *)sl.fw, b, lo, hi, check, av, ac, ov, nin, nch, nvis);
      } else if (S.triclinic) {
        unit_ads_fp64<true>(S, (const AdsRec64 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis);
      } else {
        unit_ads_fp64<false>(S, (const AdsRec64 *)sl.ads, b, lo, hi, b.excl, check, av, ac, ov, nin, nch, nvis);
      }
      e_v = warp_sum(av);
      e_q = warp_sum(ac);
    }
    ov = warp_or(ov);
    if (lane == 0) {
      sc.uv[u] = e_v;
      sc.uc[u] = e_q;
      sc.uo[u] = ov;
    }
    v = __shfl_sync(RGPU_FULL, vn, 0);
  }
  if (sc.cnt) {
    nin = __reduce_add_sync(RGPU_FULL, (unsigned)nin);
    nch = __reduce_add_sync(RGPU_FULL, (unsigned)nch);
    if (lane == 0) {
      atomicAdd(&sc.cnt[0], (unsigned long long)nvis);
      atomicAdd(&sc.cnt[1], (unsigned long long)nin);
      atomicAdd(&sc.cnt[2], (unsigned long long)nch);
    }
  }
  return pl;
}

/* Evaluates P bead positions over the slice; all threads of the block must
 * call it. Writes this slice's partial results to res/ovf. */
template <int MIXED>
__device__ void eval_positions(const RgpuSys &S, const EvalSlice &sl, const BeadPos *pos, int P, int pair_check,
                               double (*res)[4], int *ovf, EvalScratch sc, int max_units)
{
  const EvalPlan pl = eval_units<MIXED>(S, sl, pos, P, pair_check, sc, max_units);
  const int per = pl.cf + pl.ca;
  __syncthreads();
  if (threadIdx.x == 0) *sc.next = 0;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    double hv = 0.0, hc = 0.0, av = 0.0, ac = 0.0;
    int ov = 0;
    for (int c = 0; c < per; c++) {
      int u = p * per + c;
      if (c < pl.cf) { hv += sc.uv[u]; hc += sc.uc[u]; }
      else { av += sc.uv[u]; ac += sc.uc[u]; }
      ov |= sc.uo[u];
    }
    res[p][0] = hv; res[p][1] = hc; res[p][2] = av; res[p][3] = ac;
    ovf[p] = ov;
  }
  __syncthreads();
}

/* ------------------------------------------------------------------------ */
/* Ewald Fourier difference (CalculateEwaldFourierAdsorbate,
 * src/ewald.c:6859-7567, charge sites only).
 *
 * Sites carry a signed charge (+q for new, -q for old positions). On the
 * FP64 path (and MIXED = 2) exp(i 2 pi k s) is tabulated per site and axis
 * for k in [-kmax, kmax] and multiplied out per wave vector. On the mixed
 * path (MIXED = 1) each wave vector's angle n.s is reduced exactly in 32-bit
 * integer arithmetic on the fixed-point coordinates and its phase formed
 * directly (ewald_dS), so each phase has FP32 accuracy at every k; MIXED = 2
 * tabulates the per-axis phases of the same exact angles in FP64. */
struct EwSite { BeadPos b; double q; };

template <int MIXED>
struct PhaseT { typedef float2 T; };
template <>
struct PhaseT<0> { typedef double2 T; };
template <>
struct PhaseT<2> { typedef double2 T; };

/* table layout: tab[(site*3 + axis)*KW + (k + kmax)], KW = 2*kmaxall+1;
 * the mixed path (MIXED = 1) keeps no table */
template <int MIXED>
__device__ __forceinline__ void ewald_phases(const RgpuSys &S, const EwSite *sites, int ns, typename PhaseT<MIXED>::T *tab, int kw)
{
  if (MIXED == 1) return;
  const int km = (kw - 1) / 2;
  const int n = ns * 3 * kw;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int kk = i % kw - km;
    int sa = i / kw;
    int axis = sa % 3, s = sa / 3;
    const BeadPos &b = sites[s].b;
    if (MIXED == 2) {
      /* the exact fixed-point angle, its phase in FP64 */
      int xi = axis == 0 ? b.xi : (axis == 1 ? b.yi : b.zi);
      int ang = (int)((unsigned)kk * (unsigned)xi);
      double sn, cs;
      sincospi(2.0 * ((double)ang * 2.3283064365386963e-10), &sn, &cs);
      ((double2 *)tab)[i] = make_double2(cs, sn);
    } else {
      double f;
      if (!S.triclinic) {
        double x = axis == 0 ? b.x : (axis == 1 ? b.y : b.z);
        f = x * S.inv_box[axis];
      } else {
        f = rgpu_frac(S, axis, b.x, b.y, b.z);
      }
      double sn, cs;
      sincospi(2.0 * (double)kk * f, &sn, &cs);
      ((double2 *)tab)[i] = make_double2(cs, sn);
    }
  }
}

/* delta S(k) for wave vector k from the tables */
template <int MIXED>
__device__ __forceinline__ double2 ewald_dS(const typename PhaseT<MIXED>::T *tab, int kw, const EwSite *sites,
                                            int ns, char4 kv)
{
  const int km = (kw - 1) / 2;
  if (MIXED == 1) {
    /* exp(ik.r) of each site in FP32 from its exact angle n.s (the wave
     * vector's integer indices times the fixed-point fractional
     * coordinates, in turns modulo 1): sincospif of the angle's leading 24
     * bits, rotated to first order by its last 8 (at most 3.7e-7 rad);
     * q exp(ik.r) summed in FP64. No phase table. */
    double re = 0.0, im = 0.0;
    for (int s = 0; s < ns; s++) {
      const BeadPos &b = sites[s].b;
      const int ang = (int)((unsigned)kv.x * (unsigned)b.xi + (unsigned)kv.y * (unsigned)b.yi +
                            (unsigned)kv.z * (unsigned)b.zi);
      float sn, cs;
      sincospif(__int2float_rn(ang & ~0xff) * 4.656612873077393e-10f, &sn, &cs);   /* 2^-31: x in [-1, 1) */
      const float d = __int2float_rn(ang & 0xff) * 1.4629180792671596e-09f;       /* 2 pi 2^-32 */
      const float er = fmaf(-sn, d, cs), ei = fmaf(cs, d, sn);
      re = fma(sites[s].q, (double)er, re);
      im = fma(sites[s].q, (double)ei, im);
    }
    return make_double2(re, im);
  } else {
    double re = 0.0, im = 0.0;
    const double2 *t = (const double2 *)tab;
    for (int s = 0; s < ns; s++) {
      double2 a = t[(s * 3 + 0) * kw + kv.x + km];
      double2 b = t[(s * 3 + 1) * kw + kv.y + km];
      double2 c = t[(s * 3 + 2) * kw + kv.z + km];
      double xr = a.x * b.x - a.y * b.y, xi = a.x * b.y + a.y * b.x;
      double er = xr * c.x - xi * c.y, ei = xr * c.y + xi * c.x;
      re += sites[s].q * er;
      im += sites[s].q * ei;
    }
    return make_double2(re, im);
  }
}

/* Sum over wave vectors [k0, k1) of the energy change; every thread returns
 * {e_ads, e_host}:
 * e_ads = sum kf (|S+dS|^2 - |S|^2), e_host = sum kf Re(S_fw^* dS). */
template <int MIXED>
__device__ void ewald_energy_sum(const RgpuSys &S, const typename PhaseT<MIXED>::T *tab, int kw,
                                 const EwSite *sites, int ns, int k0, int k1, double &e_ads, double &e_host,
                                 double *red)
{
  double ea = 0.0, eh = 0.0;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    double2 d = ewald_dS<MIXED>(tab, kw, sites, ns, S.kvec[k]);
    double2 so = S.sk_ads[k];
    double2 sf = S.sk_fw[k];
    double kf = S.kfactor[k];
    ea += kf * (2.0 * (so.x * d.x + so.y * d.y) + d.x * d.x + d.y * d.y);
    eh += kf * (sf.x * d.x + sf.y * d.y);
  }
  block_sum2(ea, eh, red);
  e_ads = ea;
  e_host = eh;
}

/* As ewald_energy_sum, without block reduction: warp w leaves its partial
 * {e_ads, e_host} in red[2w], red[2w+1]. No block barrier. */
template <int MIXED>
__device__ __forceinline__ void ewald_energy_warps(const RgpuSys &S, const typename PhaseT<MIXED>::T *tab, int kw,
                                   const EwSite *sites, int ns, int k0, int k1, double *red)
{
  double ea = 0.0, eh = 0.0;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    double2 d = ewald_dS<MIXED>(tab, kw, sites, ns, S.kvec[k]);
    double2 so = S.sk_ads[k];
    double2 sf = S.sk_fw[k];
    double kf = S.kfactor[k];
    ea += kf * (2.0 * (so.x * d.x + so.y * d.y) + d.x * d.x + d.y * d.y);
    eh += kf * (sf.x * d.x + sf.y * d.y);
  }
  ea = warp_sum(ea);
  eh = warp_sum(eh);
  if ((threadIdx.x & 31) == 0) {
    red[2 * (threadIdx.x >> 5)] = ea;
    red[2 * (threadIdx.x >> 5) + 1] = eh;
  }
}

/* S_ads(k) += dS(k) (AcceptEwaldAdsorbateMove, src/ewald.c:11732). The same
 * ewald_dS call as in the energy sum, so the stored sums are those the
 * accepted energy was computed with. */
template <int MIXED>
__device__ __forceinline__ void ewald_apply(const RgpuSys &S, const typename PhaseT<MIXED>::T *tab, int kw, const EwSite *sites,
                            int ns, int k0, int k1)
{
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    double2 d = ewald_dS<MIXED>(tab, kw, sites, ns, S.kvec[k]);
    double2 so = S.sk_ads[k];
    S.sk_ads[k] = make_double2(so.x + d.x, so.y + d.y);
  }
}

/* complete dU_ads / dU_host of src/ewald.c:7539-7565 for a change of
 * (nnew - nold) molecules, given the k-sums and the exclusion energies */
__device__ inline void ewald_finish(const RgpuSys &S, double e_ads, double e_host, double excl_new,
                                    double excl_old, int dn, double net_ads, double &d_ads, double &d_host)
{
  double dq = dn * S.mol_charge;
  d_ads = e_ads - (excl_new - excl_old) - dn * S.self_mol;
  d_ads += S.uion * (net_ads + dq) * (net_ads + dq) - S.uion * net_ads * net_ads;
  d_host = 2.0 * e_host + 2.0 * S.uion * S.net_fw * dq;
}

#endif
