/* Kernels of the B200 GCMC energy path.
 *
 *  - rgpu_engine_kernel: the persistent batched MC engine. One thread-block
 *    cluster owns one simulation box for the whole launch. The framework and
 *    the wave vectors are split between the CTAs of the cluster (each stages
 *    its share, with its share of S(k), in shared memory); every CTA keeps a
 *    full copy of the adsorbate records, draws the same counter-based random
 *    numbers and takes the same decisions. Each energy evaluation leaves
 *    this CTA's per-position sums in shared memory; after one cluster barrier
 *    the lanes that need a total read the sums of every CTA through
 *    distributed shared memory in rank order, so all CTAs see bitwise
 *    identical totals. Each cluster advances its box by `nsteps` MC moves
 *    (translation, rotation, CBMC insertion, CBMC deletion: src/mc_moves.c:1529,
 *    :2636, :6941, :7150) without returning to the host; FP64 and mixed runs
 *    see identical random streams.
 *  - per-call kernels behind the reference-named C entry points: batched
 *    bead energies, Ewald Fourier difference and accept, structure factors.
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <type_traits>
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "rgpu_chain.h"
#include "rgpu_device.cuh"
#include "rgpu_engine.h"
#include "rgpu_grid.cuh"

namespace cg = cooperative_groups;

#define RGPU_MAX_UNITS 512
#define RGPU_MAX_WARPS 32
#define RGPU_RND 192          /* random slots drawn per MC step */
#define RGPU_CTL_BYTES 6144   /* shared-memory slot of the control block */

/* ------------------------------------------------------------------------ */
/* shared-memory plan of the engine (offsets in bytes from the dynamic base).
 * fw_items: framework records of this CTA's share (atoms; tiles*RGPU_TILE on the
 * mixed path), tiles: tile records of the share (mixed only), k_items: wave
 * vectors of the share staged with their S(k) (0: read from global memory). */
struct EngineLayout {
  size_t sys, fw, tiles, ads, pos, uv, uc, uo, part, q, sites, tab, red, kvec, kf, skfw, skads, ctl, ang, total;
};

/* this CTA's sums for one position of an evaluation: host VDW, host real,
 * adsorbate VDW, adsorbate real, overlap flag. 16-byte aligned (48 bytes) so
 * that v[0..1] and v[2..3] are read as double2. */
struct __align__(16) PosSum {
  double v[4];
  int ov, pad;
};
static_assert(sizeof(PosSum) % 16 == 0, "PosSum must keep 16-byte alignment in arrays");

__host__ __device__ inline size_t rgpu_align(size_t x) { return (x + 255) & ~(size_t)255; }

/* bend and dihedral trigonometry of every trial of a chain growth stage
 * (flexible-chain builds only): {cos theta, sin theta, cos phi, sin phi,
 * torsion Rosenbluth factor} for beads 2.. natom-1 and each trial */
#define RGPU_ANG_STRIDE 5
#define RGPU_ANG_TABLE (RGPU_ANG_STRIDE * (RGPU_MAX_ATOMS - 2) * RGPU_MAX_TRIALS)
#define RGPU_ANG_DOUBLES (RGPU_ANG_TABLE + RGPU_MAX_ATOMS)   /* + the bend angle of each bead (chain_scheme 0) */

__host__ __device__ inline EngineLayout engine_layout(int mixed, int fw_items, int tiles, int max_ads_atoms, int kw,
                                                      int k_items, int nwarps, int flex)
{
  EngineLayout L;
  size_t o = 0;
  L.sys = o; o = rgpu_align(o + sizeof(RgpuSys));
  L.fw = o; o = rgpu_align(o + (size_t)fw_items * (mixed ? sizeof(int4) : sizeof(double4)));
  L.tiles = o; o = rgpu_align(o + (size_t)tiles * sizeof(TileRec));
  L.ads = o; o = rgpu_align(o + (size_t)max_ads_atoms * (mixed ? sizeof(int4) : sizeof(AdsRec64)));
  L.pos = o; o = rgpu_align(o + RGPU_MAX_POS * sizeof(BeadPos));
  L.uv = o; o = rgpu_align(o + RGPU_MAX_UNITS * sizeof(double));
  L.uc = o; o = rgpu_align(o + RGPU_MAX_UNITS * sizeof(double));
  L.uo = o; o = rgpu_align(o + RGPU_MAX_UNITS * sizeof(int));
  L.part = o; o = rgpu_align(o + 2 * RGPU_MAX_POS * sizeof(PosSum));   /* double-buffered */
  /* per-warp pair queues: r2 (FP32, or FP64 for mixed = 2), charge, type */
  L.q = o; o = rgpu_align(o + (mixed ? (size_t)nwarps * 64 * (mixed == 2 ? 16 : 12) : 0));
  L.sites = o; o = rgpu_align(o + 2 * RGPU_MAX_ATOMS * sizeof(EwSite));
  /* per-site phase tables (none on the mixed path) */
  L.tab = o; o = rgpu_align(o + (mixed == 1 ? 0 : (size_t)2 * RGPU_MAX_ATOMS * 3 * kw * sizeof(double2)));
  L.red = o; o = rgpu_align(o + 2 * 2 * RGPU_MAX_WARPS * sizeof(double));
  L.kvec = o; o = rgpu_align(o + (size_t)k_items * sizeof(char4));
  L.kf = o; o = rgpu_align(o + (size_t)k_items * sizeof(double));
  L.skfw = o; o = rgpu_align(o + (size_t)k_items * sizeof(double2));
  L.skads = o; o = rgpu_align(o + (size_t)k_items * sizeof(double2));
  L.ctl = o; o = rgpu_align(o + RGPU_CTL_BYTES);
  L.ang = o; o = rgpu_align(o + (flex ? 2 * RGPU_ANG_DOUBLES * sizeof(double) : 0));   /* growth, retrace */
  L.total = o;
  return L;
}

size_t rgpu_engine_smem_bytes(int mixed, int fw_items, int tiles, int max_ads_atoms, int kw, int k_items,
                              int threads, int flex)
{
  return engine_layout(mixed, fw_items, tiles, max_ads_atoms, kw, k_items, threads / 32, flex).total;
}

/* broadcast/control block in shared memory */
struct Ctl {
  double rnd[2][RGPU_RND];    /* uniforms by slot, double-buffered by step parity */
  double energy[RGPU_NE];     /* running energies (written back by rank 0) */
  long long cnt[RGPU_NCNT];   /* move counters [0, RGPU_CNT_PAIRS) and reinsertion counters (rank 0's written back) */
  BeadPos first;              /* chosen first bead */
  double u[4];                /* energies of the chosen configuration */
  double uo[4];               /* energies of the retraced old configuration (reinsertion) */
  double rosen;
  double rosen_old;
  /* flexible chains: chosen bead positions of the configuration being grown
   * or retraced (cp) and of a reinsertion's new one (cpn), intramolecular
   * energies of the configurations */
  double cp[RGPU_MAX_ATOMS][3];
  double cpn[RGPU_MAX_ATOMS][3];
  double ub[RGPU_MAX_TRIALS];  /* bonded energies of the current bead's trials */
  /* a retrace's beads: trial weight sum, the old bead's host VDW, adsorbate
   * VDW, intramolecular LJ and bonded energy, any valid trial */
  double rb[RGPU_MAX_ATOMS][6];
  double co[RGPU_MAX_ATOMS][3];  /* the old beads of a reinsertion's retrace */
  double uintra, uintra_old;
  double dl[4];
  int nmol;
  int fail;
  int accept;
  int sel;
  int nads;                   /* adsorbate atoms = nmol * natom */
  int status;                 /* RGPU_ERR_* bits */
  /* work done: pairs visited, in cut-off, charged in cut-off, k x site, k */
  unsigned long long work[5];
  long long cyc[2];           /* clock cycles in evaluations and Ewald sums */
  double sums[RGPU_NSUM];     /* ensemble sums of this launch */
  int next;                   /* unit counter of eval_units */
  double ewt[2][2];           /* this CTA's Ewald sums {e_ads, e_host}, by buffer */
  double gv[RGPU_MAX_POS];    /* grid host VDW of the positions of the current evaluation */
  double gq[RGPU_MAX_POS];    /* grid host real-space charge energy of the positions */
};
static_assert(sizeof(Ctl) <= RGPU_CTL_BYTES, "control block exceeds its shared-memory slot");

template <int MIXED, bool FLEX>
struct Eng {
  RgpuSys *S;
  EvalSlice sl;
  void *ads;                 /* int4[] or AdsRec64[] (full copy) */
  BeadPos *pos;
  double *uv, *uc;           /* [RGPU_MAX_UNITS] unit partials */
  int *uo;
  PosSum *part;              /* [2][RGPU_MAX_POS] position sums of this CTA */
  EvalScratch sc;
  EwSite *sites;
  typename PhaseT<MIXED>::T *tab;
  int kw;
  int k0, k1;                /* this CTA's wave vectors */
  double *red;               /* [2][2*RGPU_MAX_WARPS] */
  double *ang;               /* [2][RGPU_ANG_DOUBLES] chain trial trigonometry of a growth and of a retrace
                              * stage (flexible-chain builds) */
  Ctl *ctl;
  const double *rnd;         /* this step's uniforms */
  uint64_t step;             /* index of the current MC step */
  int rank, csize;
  int xb;                    /* exchange buffer (same sequence in every thread and CTA) */
};

/* Position of atom a of molecule m. FP64 records carry the position; on the
 * mixed path the FP64 positions stay in global memory (ads_xyz), which every
 * CTA of the cluster writes with the same values on each accepted move. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void atom_xyz(const Eng<MIXED, FLEX> &E, int m, int a, double *p)
{
  const int idx = m * E.S->natom + a;
  if (MIXED) {
    const double *x = E.S->ads_xyz + 3 * idx;
    p[0] = x[0]; p[1] = x[1]; p[2] = x[2];
  } else {
    const AdsRec64 &r = ((const AdsRec64 *)E.ads)[idx];
    p[0] = r.x; p[1] = r.y; p[2] = r.z;
  }
}

template <int MIXED, bool FLEX>
__device__ __forceinline__ void atom_store(const Eng<MIXED, FLEX> &E, int m, int a, const double *p)
{
  const RgpuSys &S = *E.S;
  const int idx = m * S.natom + a;
  if (MIXED) {
    double *x = E.S->ads_xyz + 3 * idx;
    x[0] = p[0]; x[1] = p[1]; x[2] = p[2];
    int xi, yi, zi;
    rgpu_fix3(S, p[0], p[1], p[2], xi, yi, zi);
    ((int4 *)E.ads)[idx] = make_int4(xi, yi, zi, m * 16 + a);
  } else {
    AdsRec64 r;
    r.x = p[0]; r.y = p[1]; r.z = p[2]; r.tag = m * 16 + a;
    ((AdsRec64 *)E.ads)[idx] = r;
  }
}

/* RotationAround{X,Y,Z}Axis, src/utils.c:876-936 */
__device__ __forceinline__ void rotate_axis(double *c, int axis, double th)
{
  double cs, sn;
  sincos(th, &sn, &cs);
  double x = c[0], y = c[1], z = c[2];
  if (axis == 0) { c[1] = cs * y + sn * z; c[2] = -sn * y + cs * z; }
  else if (axis == 1) { c[0] = cs * x - sn * z; c[2] = sn * x + cs * z; }
  else { c[0] = cs * x + sn * y; c[1] = -sn * x + cs * y; }
}

/* RandomArrayRotationMatrix (Shoemake), src/utils.c:835-874 */
__device__ __forceinline__ void random_rotation(double x0, double y1, double y2, double R[3][3])
{
  y1 *= 2.0 * M_PI;
  y2 *= 2.0 * M_PI;
  double r1 = sqrt(1.0 - x0), r2 = sqrt(x0);
  double s1, c1, s2, c2;
  sincos(y1, &s1, &c1);
  sincos(y2, &s2, &c2);
  double u0 = c2 * r2, u1 = s1 * r1, u2 = c1 * r1, u3 = s2 * r2;
  double ci = 2.0 * u0 * u0 - 1.0, ce = 2.0 * u0;
  R[0][0] = ci + 2.0 * u1 * u1;
  R[1][1] = ci + 2.0 * u2 * u2;
  R[2][2] = ci + 2.0 * u3 * u3;
  R[1][2] = 2.0 * u2 * u3 - ce * u1;
  R[2][0] = 2.0 * u3 * u1 - ce * u2;
  R[0][1] = 2.0 * u1 * u2 - ce * u3;
  R[2][1] = 2.0 * u3 * u2 + ce * u1;
  R[0][2] = 2.0 * u1 * u3 + ce * u2;
  R[1][0] = 2.0 * u2 * u1 + ce * u3;
}

/* share [lo, hi) of n items for rank r of c (1 <= c <= 8; n far below
 * 2^28, so n * c fits in 32 bits) */
__device__ __forceinline__ void share(int n, int r, int c, int &lo, int &hi)
{
  lo = n * r / c;
  hi = n * (r + 1) / c;
}

/* Pair evaluation of P positions on this CTA's share, then one cluster
 * barrier; the totals are read with gather(). All threads call. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void engine_eval(Eng<MIXED, FLEX> &E, int P, int pair_check, int ew_ns = 0)
{
  Ctl &C = *E.ctl;
  const long long t0 = clock64();
  if (ew_ns) {
    /* the Ewald sum of sites E.sites[0..ew_ns) rides along (a displacement,
     * whose sites are known up front): phase tables now, each warp's share
     * of the wave vectors right after its pair units, so it fills the
     * units' tail; the CTA total goes to C.ewt[E.xb] as engine_ewald does */
    ewald_phases<MIXED>(*E.S, E.sites, ew_ns, E.tab, E.kw);
    if (threadIdx.x == 0) {
      C.work[3] += (unsigned long long)(E.k1 - E.k0) * ew_ns;
      C.work[4] += (unsigned long long)(E.k1 - E.k0);
    }
    __syncthreads();
  }
  if (FLEX && E.S->use_grid && E.rank == 0) {
    /* host VDW from the bead types' energy grids (one CTA of the cluster):
     * 8 lanes per position, 4 positions per warp, before the pair units */
    const int lane = threadIdx.x & 31;
    for (int base = (threadIdx.x >> 5) * 4; base < P; base += (blockDim.x >> 5) * 4) {
      const int p = base + (lane >> 3);
      const bool live = p < P;
      const double x[3] = {live ? E.pos[p].x : 0.0, live ? E.pos[p].y : 0.0, live ? E.pos[p].z : 0.0};
      const double g = rgpu_grid_value8(E.S->grid[live ? E.pos[p].atom : 0], E.S->grid_geom, x, lane & 7, live);
      if (live && (lane & 7) == 0) C.gv[p] = g;
      if (E.S->use_coul_grid) {
        /* real-space charge energy: the bead charge times the unit-charge
         * Coulomb grid (InterpolateCoulombGrid, src/grids.c:1200) */
        const double q = live ? E.S->mol_q[E.pos[p].atom] : 0.0;
        const double gq = rgpu_grid_value8(E.S->coul_grid, E.S->coul_geom, x, lane & 7, live && q != 0.0, false);
        if (live && (lane & 7) == 0) C.gq[p] = q * gq;
      }
    }
  }
  const EvalPlan pl = eval_units<MIXED>(*E.S, E.sl, E.pos, P, pair_check, E.sc, RGPU_MAX_UNITS);
  const int per = pl.cf + pl.ca;
  double *ewred = E.red + E.xb * 2 * RGPU_MAX_WARPS;
  if (ew_ns) ewald_energy_warps<MIXED>(*E.S, E.tab, E.kw, E.sites, ew_ns, E.k0, E.k1, ewred);
  __syncthreads();
  if (threadIdx.x == 0) C.next = 0;      /* unit counter of the next evaluation */
  if (ew_ns && threadIdx.x < 32) {
    /* this CTA's Ewald total (warp 0, fixed reduction order) */
    const int nw = blockDim.x >> 5;
    double a = 0.0, h = 0.0;
    if (threadIdx.x < nw) {
      a = ewred[2 * threadIdx.x];
      h = ewred[2 * threadIdx.x + 1];
    }
    a = warp_sum(a);
    h = warp_sum(h);
    if (threadIdx.x == 0) {
      C.ewt[E.xb][0] = a;
      C.ewt[E.xb][1] = h;
    }
  }
  /* this CTA's sum per position, units in order */
  PosSum *ps = E.part + E.xb * RGPU_MAX_POS;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    double hv = 0.0, hc = 0.0, av = 0.0, ac = 0.0;
    int ov = 0;
    for (int c = 0; c < per; c++) {
      const int u = p * per + c;
      if (c < pl.cf) { hv += E.uv[u]; hc += E.uc[u]; }
      else { av += E.uv[u]; ac += E.uc[u]; }
      ov |= E.uo[u];
    }
    if (FLEX && E.S->use_grid && E.rank == 0) {
      const double g = C.gv[p];
      hv += g;
      ov |= g >= E.S->overlap;
      if (E.S->use_coul_grid) hc += C.gq[p];
    }
    ps[p].v[0] = hv; ps[p].v[1] = hc; ps[p].v[2] = av; ps[p].v[3] = ac;
    ps[p].ov = ov;
  }
  cg::this_cluster().sync();
  if (threadIdx.x == 0) C.cyc[0] += clock64() - t0;
}

/* Totals of position p of the last evaluation (buffer b): the CTAs' sums
 * added in rank order. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void gather(const Eng<MIXED, FLEX> &E, int b, int p, double *r, int &ov)
{
  cg::cluster_group cl = cg::this_cluster();
  const PosSum *own = E.part + b * RGPU_MAX_POS + p;
  r[0] = r[1] = r[2] = r[3] = 0.0;
  ov = 0;
  for (int q = 0; q < E.csize; q++) {
    const PosSum *ps = E.csize > 1 ? cl.map_shared_rank(own, q) : own;
    const double2 a = *(const double2 *)&ps->v[0], c = *(const double2 *)&ps->v[2];
    r[0] += a.x; r[1] += a.y; r[2] += c.x; r[3] += c.y;
    ov |= ps->ov;
  }
}

/* Ewald sum over this CTA's wave vectors for the sites in E.sites[0..ns),
 * warp partials left in E.red[b]; one cluster barrier. All threads call. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void engine_ewald(Eng<MIXED, FLEX> &E, int ns)
{
  Ctl &C = *E.ctl;
  const long long t0 = clock64();
  ewald_phases<MIXED>(*E.S, E.sites, ns, E.tab, E.kw);
  if (threadIdx.x == 0) {
    C.work[3] += (unsigned long long)(E.k1 - E.k0) * ns;
    C.work[4] += (unsigned long long)(E.k1 - E.k0);
  }
  __syncthreads();
  double *red = E.red + E.xb * 2 * RGPU_MAX_WARPS;
  ewald_energy_warps<MIXED>(*E.S, E.tab, E.kw, E.sites, ns, E.k0, E.k1, red);
  __syncthreads();
  /* this CTA's total (warp 0, fixed reduction order) */
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    double a = 0.0, h = 0.0;
    if (threadIdx.x < nw) {
      a = red[2 * threadIdx.x];
      h = red[2 * threadIdx.x + 1];
    }
    a = warp_sum(a);
    h = warp_sum(h);
    if (threadIdx.x == 0) {
      C.ewt[E.xb][0] = a;
      C.ewt[E.xb][1] = h;
    }
  }
  cg::this_cluster().sync();
  if (threadIdx.x == 0) C.cyc[1] += clock64() - t0;
}

/* cluster total of the last Ewald sum (buffer b) */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void gather_ewald(const Eng<MIXED, FLEX> &E, int b, double &ea, double &eh)
{
  cg::cluster_group cl = cg::this_cluster();
  ea = eh = 0.0;
  const double *own = &E.ctl->ewt[b][0];
  for (int q = 0; q < E.csize; q++) {
    const double *t = E.csize > 1 ? cl.map_shared_rank(own, q) : own;
    ea += t[0];
    eh += t[1];
  }
}

/* Warp 0: Rosenbluth bookkeeping of n trials (lane t = trial t, nb beads each
 * at positions t*nb + j of buffer b). First bead (nb = 1, first = true):
 * overlap when any energy reaches the criterion (src/cbmc.c:699-701);
 * orientations: when a bead's host VDW energy does (src/cbmc.c:1210-1215).
 * LJ biasing (src/cbmc.c:734-735, :1432-1436). Selection as
 * SelectTrialPosition (src/cbmc.c:563-599). Lane 0 leaves the weight sum
 * (w_sum = sum exp(bf)), the selected trial and its energies in Ctl. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void cbmc_trials(const Eng<MIXED, FLEX> &E, int b, int n, int nb, bool first, bool select, double usel,
                            double &w_sum, int &sel, double *usum, int &any, int off = 0, double *w_sel = nullptr)
{
  const int lane = threadIdx.x & 31;
  const RgpuSys &S = *E.S;
  double e[4] = {0.0, 0.0, 0.0, 0.0};
  int ov = 0;
  double bf = 0.0;
  if (lane < n) {
    for (int j = 0; j < nb; j++) {
      double r[4];
      int o;
      gather(E, b, off + lane * nb + j, r, o);
      if (first) ov |= (r[0] >= S.overlap || r[1] >= S.overlap || r[2] >= S.overlap || r[3] >= S.overlap);
      else ov |= (r[0] >= S.overlap);
      for (int k = 0; k < 4; k++) e[k] += r[k];
    }
    bf = -S.beta * (e[0] + e[2]);
  }
  const bool valid = lane < n && !ov;
  const double w = valid ? exp(bf) : 0.0;
  double largest = valid ? bf : -DBL_MAX;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) largest = fmax(largest, __shfl_xor_sync(RGPU_FULL, largest, o));
  const double ws = valid ? exp(bf - largest) : 0.0;
  const unsigned okmask = __ballot_sync(RGPU_FULL, valid);
  any = okmask != 0u;
  /* the sums run in trial order, as the reference's loops do */
  double wsum = 0.0, shsum = 0.0;
  for (int t = 0; t < n; t++) {
    wsum += __shfl_sync(RGPU_FULL, w, t);
    shsum += __shfl_sync(RGPU_FULL, ws, t);
  }
  int s = 0;
  if (select && any) {
    const double target = usel * shsum;
    double cum = __shfl_sync(RGPU_FULL, ws, 0);
    while (cum < target && s < n - 1) {
      s++;
      cum += __shfl_sync(RGPU_FULL, ws, s);
    }
  }
  w_sum = wsum;
  sel = s;
  for (int k = 0; k < 4; k++) usum[k] = __shfl_sync(RGPU_FULL, e[k], s);
  const double ws_sel = __shfl_sync(RGPU_FULL, w, s);
  if (w_sel) *w_sel = ws_sel;
}

/* ------------------------------------------------------------------------ */
/* translation (mv=0) and rotation (mv=1):
 * TranslationMoveAdsorbate src/mc_moves.c:1529-1762, RotationMoveAdsorbate :2636 */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void step_displace(Eng<MIXED, FLEX> &E, int mv)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const double *R = E.rnd;
  const int na = S.natom, nmol = C.nmol;
  int m = (int)(R[SLOT_MOLECULE] * nmol);
  if (m >= nmol) m = nmol - 1;
  const double vnew = 2.0 * R[SLOT_VNEW] - 1.0;
  int axis = (int)(3.0 * R[SLOT_AXIS]);
  if (axis > 2) axis = 2;
  if (threadIdx.x < na) {
    const int a = threadIdx.x;
    double o[3], n[3];
    atom_xyz(E, m, a, o);
    if (mv == 0) {
      n[0] = o[0]; n[1] = o[1]; n[2] = o[2];
      n[axis] += vnew * S.max_translation;
    } else {
      double sb[3];
      atom_xyz(E, m, S.start_bead, sb);
      double c[3] = {o[0] - sb[0], o[1] - sb[1], o[2] - sb[2]};
      rotate_axis(c, axis, vnew * S.max_rotation);
      n[0] = c[0] + sb[0]; n[1] = c[1] + sb[1]; n[2] = c[2] + sb[2];
    }
    bead_set(E.pos[a], S, n[0], n[1], n[2], a, m);
    bead_set(E.pos[na + a], S, o[0], o[1], o[2], a, m);
    E.sites[a].b = E.pos[a];
    E.sites[a].q = S.mol_q[a];
    E.sites[na + a].b = E.pos[na + a];
    E.sites[na + a].q = -S.mol_q[a];
  }
  __syncthreads();
  const bool ew = S.ewald && S.mol_charged;
  engine_eval(E, 2 * na, na, ew ? 2 * na : 0);
  const int be = E.xb;
  E.xb ^= 1;
  if (threadIdx.x < 32) {
    /* lane a: totals of new position a and old position a (a < na <= 8) */
    const int a = threadIdx.x;
    double rn[4] = {0.0, 0.0, 0.0, 0.0}, ro[4] = {0.0, 0.0, 0.0, 0.0};
    int o1 = 0, o2 = 0;
    if (a < na) {
      gather(E, be, a, rn, o1);
      gather(E, be, na + a, ro, o2);
    }
    const int ov = __any_sync(RGPU_FULL, o1);
    double dl[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = 0; j < na; j++)
      for (int k = 0; k < 4; k++)
        dl[k] += __shfl_sync(RGPU_FULL, rn[k], j) - __shfl_sync(RGPU_FULL, ro[k], j);
    if (a == 0) {
      C.fail = ov;
      for (int k = 0; k < 4; k++) C.dl[k] = dl[k];
      if (ov) C.cnt[RGPU_CNT_OVERLAP]++;
    }
  }
  __syncthreads();
  if (C.fail) return;
  if (threadIdx.x == 0) {
    double d_ads = 0.0, d_host = 0.0;
    if (ew) {
      double ea, eh;
      gather_ewald(E, be, ea, eh);
      /* the exclusion energy of a rigid molecule is the same before and
       * after the displacement (the reference's difference of the two is
       * zero up to rounding) */
      ewald_finish(S, ea, eh, S.excl_mol, S.excl_mol, 0, 0.0, d_ads, d_host);
    }
    double du = C.dl[0] + C.dl[1] + C.dl[2] + C.dl[3] + d_ads + d_host;
    double pacc = exp(-S.beta * du);
    if (!isfinite(du)) C.status |= RGPU_ERR_NONFINITE;
    C.accept = R[SLOT_ACCEPT] < pacc;
    if (C.accept) {
      C.cnt[RGPU_CNT_ACCEPT + mv]++;
      C.energy[RGPU_E_HOST_VDW] += C.dl[0];
      C.energy[RGPU_E_HOST_REAL] += C.dl[1];
      C.energy[RGPU_E_ADS_VDW] += C.dl[2];
      C.energy[RGPU_E_ADS_REAL] += C.dl[3];
      C.energy[RGPU_E_HOST_FOURIER] += d_host;
      C.energy[RGPU_E_ADS_FOURIER] += d_ads;
    }
  }
  __syncthreads();
  if (C.accept) {
    if (threadIdx.x < na) {
      double p[3] = {E.pos[threadIdx.x].x, E.pos[threadIdx.x].y, E.pos[threadIdx.x].z};
      atom_store(E, m, threadIdx.x, p);
    }
    if (ew) ewald_apply<MIXED>(S, E.tab, E.kw, E.sites, 2 * na, E.k0, E.k1);
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* CBMC insertion / deletion of a rigid molecule grown from the starting bead
 * (widom: a test insertion that only samples its Rosenbluth weight,
 * WidomAdsorbateMove src/mc_moves.c:7844-8030):
 * GrowMolecule src/cbmc.c:3056-3181 and RetraceMolecule :2928-3054 with
 * HandleFirstBead :623-795, Rosen/RosenOld :2762-2926, the rigid-group branch
 * of GenerateTrialOrientationsSimpleSphere :1480-1578 and
 * ComputeExternalEnergies :1154-1478, LJ biasing; acceptance of
 * SwapAddAdsorbateMove src/mc_moves.c:7016 and SwapRemoveAdsorbateMove :7228. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void step_swap(Eng<MIXED, FLEX> &E, bool insert, bool widom = false)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  if (widom && threadIdx.x == 0) C.sums[RGPU_SUM_WIDOM_N] += 1.0;   /* overlap samples count with weight 0 */
  const int na = S.natom, sb = S.start_bead, nmol = C.nmol;
  const int nf = S.ntrial_first, nt = S.ntrial;
  int m = nmol;
  if (!insert) {
    m = (int)(E.rnd[SLOT_MOLECULE] * nmol);
    if (m >= nmol) m = nmol - 1;
  }
  const int exclude = insert ? -1 : m;
  const int nb = na - 1;   /* beads grown per orientation trial */
  const bool ew = S.ewald && S.mol_charged;
  /* a deletion retraces the old molecule: its first bead and orientation
   * are trial 0 of each stage, known up front, so both stages' trials and
   * the Ewald sum of the removed molecule go into one evaluation (first-bead
   * trials at positions 0..nf, orientation t's beads at nf + t*nb + j) */
  const bool one = !insert && nf + (na > 1 ? nt * nb : 0) <= RGPU_MAX_POS;
  /* first-bead trials */
  if (threadIdx.x < nf) {
    const int i = threadIdx.x;
    double p[3];
    if (!insert && i == 0) {
      atom_xyz(E, m, sb, p);
    } else {
      rgpu_box_point(S, E.rnd[SLOT_FIRST + 3 * i + 2], E.rnd[SLOT_FIRST + 3 * i + 1], E.rnd[SLOT_FIRST + 3 * i + 0],
                     p);
    }
    bead_set(E.pos[i], S, p[0], p[1], p[2], sb, exclude);
  }
  if (one) {
    /* the retrace orientations about the old first bead (trial 0: the old
     * one) and the removed molecule's Ewald sites (nf, nt <= 16, na <= 8;
     * blocks have at least 64 threads) */
    if (na > 1 && threadIdx.x >= 32 && threadIdx.x < 32 + nt) {
      const int t = threadIdx.x - 32;
      double o[3];
      atom_xyz(E, m, sb, o);
      double R[3][3];
      if (t > 0)
        random_rotation(E.rnd[SLOT_ORIENT + 4 * t + 0], E.rnd[SLOT_ORIENT + 4 * t + 1],
                        E.rnd[SLOT_ORIENT + 4 * t + 2], R);
      int j = 0;
      for (int a = 0; a < na; a++) {
        if (a == sb) continue;
        double p[3];
        if (t == 0) {
          atom_xyz(E, m, a, p);
        } else {
          const double c[3] = {S.mol_ref[a][0] - S.mol_ref[sb][0], S.mol_ref[a][1] - S.mol_ref[sb][1],
                               S.mol_ref[a][2] - S.mol_ref[sb][2]};
          p[0] = o[0] + c[0] * R[0][0] + c[1] * R[0][1] + c[2] * R[0][2];
          p[1] = o[1] + c[0] * R[1][0] + c[1] * R[1][1] + c[2] * R[1][2];
          p[2] = o[2] + c[0] * R[2][0] + c[1] * R[2][1] + c[2] * R[2][2];
        }
        bead_set(E.pos[nf + t * nb + j], S, p[0], p[1], p[2], a, exclude);
        j++;
      }
    }
    if (threadIdx.x >= 48 && threadIdx.x < 48 + na) {
      const int a = threadIdx.x - 48;
      double p[3];
      atom_xyz(E, m, a, p);
      bead_set(E.sites[a].b, S, p[0], p[1], p[2], a, exclude);
      E.sites[a].q = -S.mol_q[a];
    }
  }
  __syncthreads();
  engine_eval(E, one ? nf + (na > 1 ? nt * nb : 0) : nf, 0, one && ew ? na : 0);
  int b1 = E.xb;
  E.xb ^= 1;
  if (threadIdx.x < 32) {
    double wsum, u[4];
    int sel, any;
    cbmc_trials(E, b1, nf, 1, true, insert, E.rnd[SLOT_FIRST_SELECT], wsum, sel, u, any);
    if (threadIdx.x == 0) {
      C.rosen = wsum / (double)nf;
      C.fail = !any || (insert && C.rosen < 1e-150);
      C.sel = sel;
      for (int k = 0; k < 4; k++) C.u[k] = u[k];
      C.first = E.pos[sel];
      if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
    }
    if (one && na > 1 && any) {
      /* the retrace orientations (trial 0 is the old one, not selected) */
      cbmc_trials(E, b1, nt, nb, false, false, E.rnd[SLOT_ORIENT_SELECT], wsum, sel, u, any, nf);
      if (threadIdx.x == 0) {
        if (!any) C.fail = 1;
        else {
          C.rosen *= wsum / (double)nt;
          for (int k = 0; k < 4; k++) C.u[k] += u[k];
        }
        C.sel = sel;
        if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
      }
    }
  }
  __syncthreads();
  if (C.fail) return;
  if (na > 1 && !one) {
    const BeadPos first = C.first;
    if (threadIdx.x < nt) {
      const int t = threadIdx.x;
      if (!insert && t == 0) {
        int j = 0;
        for (int a = 0; a < na; a++) {
          if (a == sb) continue;
          double p[3];
          atom_xyz(E, m, a, p);
          bead_set(E.pos[t * nb + j], S, p[0], p[1], p[2], a, exclude);
          j++;
        }
      } else {
        double R[3][3];
        random_rotation(E.rnd[SLOT_ORIENT + 4 * t + 0], E.rnd[SLOT_ORIENT + 4 * t + 1],
                        E.rnd[SLOT_ORIENT + 4 * t + 2], R);
        int j = 0;
        for (int a = 0; a < na; a++) {
          if (a == sb) continue;
          double c[3] = {S.mol_ref[a][0] - S.mol_ref[sb][0], S.mol_ref[a][1] - S.mol_ref[sb][1],
                         S.mol_ref[a][2] - S.mol_ref[sb][2]};
          double p[3];
          p[0] = first.x + c[0] * R[0][0] + c[1] * R[0][1] + c[2] * R[0][2];
          p[1] = first.y + c[0] * R[1][0] + c[1] * R[1][1] + c[2] * R[1][2];
          p[2] = first.z + c[0] * R[2][0] + c[1] * R[2][1] + c[2] * R[2][2];
          bead_set(E.pos[t * nb + j], S, p[0], p[1], p[2], a, exclude);
          j++;
        }
      }
    }
    __syncthreads();
    engine_eval(E, nt * nb, 0);
    const int b2 = E.xb;
    E.xb ^= 1;
    if (threadIdx.x < 32) {
      double wsum, u[4];
      int sel, any;
      cbmc_trials(E, b2, nt, nb, false, insert, E.rnd[SLOT_ORIENT_SELECT], wsum, sel, u, any);
      if (threadIdx.x == 0) {
        if (!any) C.fail = 1;
        else {
          C.rosen *= wsum / (double)nt;
          if (insert && C.rosen < 1e-150) C.fail = 1;
          for (int k = 0; k < 4; k++) C.u[k] += u[k];
        }
        C.sel = sel;
        if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
      }
    }
    __syncthreads();
    if (C.fail) return;
  }
  int bw = b1;
  if (!one) {
    /* sites of the chosen configuration: first bead + beads of trial C.sel */
    if (threadIdx.x < na) {
      const int a = threadIdx.x;
      BeadPos bp;
      if (a == sb) bp = C.first;
      else {
        int j = a < sb ? a : a - 1;
        bp = E.pos[C.sel * nb + j];
      }
      E.sites[a].b = bp;
      E.sites[a].q = insert ? S.mol_q[a] : -S.mol_q[a];
    }
    __syncthreads();
    if (ew) {
      engine_ewald(E, na);
      bw = E.xb;
      E.xb ^= 1;
    }
  }
  if (threadIdx.x == 0) {
    /* LJ-biasing correction, src/cbmc.c:3171-3178 / :3044-3051 */
    double rosen = C.rosen * exp(-S.beta * (C.u[1] + C.u[3]));
    double d_ads = 0.0, d_host = 0.0;
    if (ew) {
      double ea, eh;
      gather_ewald(E, bw, ea, eh);
      const double ex = S.excl_mol;      /* rigid molecule */
      double net = nmol * S.mol_charge;
      if (insert) ewald_finish(S, ea, eh, ex, 0.0, 1, net, d_ads, d_host);
      else ewald_finish(S, ea, eh, 0.0, ex, -1, net, d_ads, d_host);
    }
    double pacc;
    if (insert) pacc = rosen * exp(-S.beta * (d_ads + d_host)) * S.fugacity_beta_v / (1.0 + nmol);
    else pacc = (double)nmol / (rosen * exp(S.beta * (d_ads + d_host)) * S.fugacity_beta_v);
    if (!(pacc == pacc)) C.status |= RGPU_ERR_NONFINITE;
    C.accept = !widom && E.rnd[SLOT_ACCEPT] < pacc;
    if (widom) C.sums[RGPU_SUM_WIDOM_W] += rosen * exp(-S.beta * (d_ads + d_host));
    const int mv = insert ? 2 : 3;
    if (C.accept) {
      C.cnt[RGPU_CNT_ACCEPT + mv]++;
      double sgn = insert ? 1.0 : -1.0;
      C.energy[RGPU_E_HOST_VDW] += sgn * C.u[0];
      C.energy[RGPU_E_HOST_REAL] += sgn * C.u[1];
      C.energy[RGPU_E_ADS_VDW] += sgn * C.u[2];
      C.energy[RGPU_E_ADS_REAL] += sgn * C.u[3];
      C.energy[RGPU_E_HOST_FOURIER] += d_host;
      C.energy[RGPU_E_ADS_FOURIER] += d_ads;
    }
  }
  __syncthreads();
  if (C.accept) {
    if (insert) {
      if (threadIdx.x < na) {
        double p[3] = {E.sites[threadIdx.x].b.x, E.sites[threadIdx.x].b.y, E.sites[threadIdx.x].b.z};
        atom_store(E, nmol, threadIdx.x, p);
      }
    } else {
      /* RemoveAdsorbateMolecule (src/molecule.c:3193): the last molecule
       * takes the freed slot */
      const int last = nmol - 1;
      if (threadIdx.x < na && m != last) {
        double p[3];
        atom_xyz(E, last, threadIdx.x, p);
        atom_store(E, m, threadIdx.x, p);
      }
    }
    if (ew) ewald_apply<MIXED>(S, E.tab, E.kw, E.sites, na, E.k0, E.k1);
    if (threadIdx.x == 0) {
      C.nmol = insert ? nmol + 1 : nmol - 1;
      C.nads = C.nmol * na;
    }
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* CBMC reinsertion of molecule m, ReinsertionAdsorbateMove src/mc_moves.c:4415-4600:
 * a new configuration is grown with m excluded (GrowMolecule, CBMC_INSERTION)
 * and the old one retraced (RetraceMolecule, CBMC_RETRACE_REINSERTION): the
 * old first bead alone, its weight completed with the new growth's other
 * first-bead trials (src/cbmc.c:750-762), and the old orientation among
 * nt - 1 fresh ones. Accepted with probability
 * exp(-beta dU_Fourier) W(new) / W(old).
 * Evaluation 1 holds the nf new first-bead trials, the old first bead and
 * the retrace orientations (all known up front); evaluation 2 the new
 * orientations around the chosen first bead. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void step_reinsert(Eng<MIXED, FLEX> &E)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int na = S.natom, sb = S.start_bead, nmol = C.nmol;
  const int nf = S.ntrial_first, nt = S.ntrial, nb = na - 1;
  int m = (int)(E.rnd[SLOT_MOLECULE] * nmol);
  if (m >= nmol) m = nmol - 1;
  const int old_first = nf;              /* position of the old first bead */
  const int old_orient = nf + 1;         /* first position of the retrace orientations */
  if (threadIdx.x < nf) {
    const int i = threadIdx.x;
    double p[3];
    rgpu_box_point(S, E.rnd[SLOT_FIRST + 3 * i + 2], E.rnd[SLOT_FIRST + 3 * i + 1], E.rnd[SLOT_FIRST + 3 * i + 0], p);
    bead_set(E.pos[i], S, p[0], p[1], p[2], sb, m);
  } else if (threadIdx.x == nf) {
    double p[3];
    atom_xyz(E, m, sb, p);
    bead_set(E.pos[old_first], S, p[0], p[1], p[2], sb, m);
  }
  if (na > 1 && threadIdx.x >= 32 && threadIdx.x < 32 + nt) {
    const int t = threadIdx.x - 32;
    double o[3];
    atom_xyz(E, m, sb, o);
    double R[3][3];
    if (t > 0)
      random_rotation(E.rnd[SLOT_ORIENT_OLD + 4 * t + 0], E.rnd[SLOT_ORIENT_OLD + 4 * t + 1],
                      E.rnd[SLOT_ORIENT_OLD + 4 * t + 2], R);
    int j = 0;
    for (int a = 0; a < na; a++) {
      if (a == sb) continue;
      double p[3];
      if (t == 0) {
        atom_xyz(E, m, a, p);
      } else {
        const double c[3] = {S.mol_ref[a][0] - S.mol_ref[sb][0], S.mol_ref[a][1] - S.mol_ref[sb][1],
                             S.mol_ref[a][2] - S.mol_ref[sb][2]};
        for (int d = 0; d < 3; d++) p[d] = o[d] + c[0] * R[d][0] + c[1] * R[d][1] + c[2] * R[d][2];
      }
      bead_set(E.pos[old_orient + t * nb + j], S, p[0], p[1], p[2], a, m);
      j++;
    }
  }
  __syncthreads();
  engine_eval(E, nf + 1 + (na > 1 ? nt * nb : 0), 0);
  const int b1 = E.xb;
  E.xb ^= 1;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double wsum, u[4], wsel;
    int sel, any;
    cbmc_trials(E, b1, nf, 1, true, true, E.rnd[SLOT_FIRST_SELECT], wsum, sel, u, any, 0, &wsel);
    /* the old first bead */
    double r[4];
    int o;
    gather(E, b1, old_first, r, o);
    const bool ovo = r[0] >= S.overlap || r[1] >= S.overlap || r[2] >= S.overlap || r[3] >= S.overlap;
    const double w_old1 = ovo ? 0.0 : exp(-S.beta * (r[0] + r[2]));
    /* the retrace orientations (trial 0 = the old one) */
    double wo = 0.0, uo[4] = {r[0], r[1], r[2], r[3]};
    int anyo = 1;
    if (na > 1) {
      double uot[4];
      int selo;
      cbmc_trials(E, b1, nt, nb, false, false, 0.0, wo, selo, uot, anyo, old_orient);
      for (int k = 0; k < 4; k++) uo[k] += uot[k];
    }
    if (lane == 0) {
      C.rosen = wsum / (double)nf;
      double rosen_old = (w_old1 + (wsum - wsel)) / (double)nf;
      if (na > 1) rosen_old *= wo / (double)nt;
      C.fail = !any || C.rosen < 1e-150 || ovo || !anyo;
      C.rosen_old = rosen_old;
      C.sel = sel;
      for (int k = 0; k < 4; k++) {
        C.u[k] = u[k];
        C.uo[k] = uo[k];
      }
      C.first = E.pos[sel];
      if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
    }
  }
  __syncthreads();
  if (C.fail) return;
  if (na > 1) {
    const BeadPos first = C.first;
    if (threadIdx.x < nt) {
      const int t = threadIdx.x;
      double R[3][3];
      random_rotation(E.rnd[SLOT_ORIENT + 4 * t + 0], E.rnd[SLOT_ORIENT + 4 * t + 1],
                      E.rnd[SLOT_ORIENT + 4 * t + 2], R);
      int j = 0;
      for (int a = 0; a < na; a++) {
        if (a == sb) continue;
        const double c[3] = {S.mol_ref[a][0] - S.mol_ref[sb][0], S.mol_ref[a][1] - S.mol_ref[sb][1],
                             S.mol_ref[a][2] - S.mol_ref[sb][2]};
        double p[3];
        p[0] = first.x + c[0] * R[0][0] + c[1] * R[0][1] + c[2] * R[0][2];
        p[1] = first.y + c[0] * R[1][0] + c[1] * R[1][1] + c[2] * R[1][2];
        p[2] = first.z + c[0] * R[2][0] + c[1] * R[2][1] + c[2] * R[2][2];
        bead_set(E.pos[t * nb + j], S, p[0], p[1], p[2], a, m);
        j++;
      }
    }
    __syncthreads();
    engine_eval(E, nt * nb, 0);
    const int b2 = E.xb;
    E.xb ^= 1;
    if (threadIdx.x < 32) {
      double wsum, u[4];
      int sel, any;
      cbmc_trials(E, b2, nt, nb, false, true, E.rnd[SLOT_ORIENT_SELECT], wsum, sel, u, any);
      if (threadIdx.x == 0) {
        if (!any) C.fail = 1;
        else {
          C.rosen *= wsum / (double)nt;
          if (C.rosen < 1e-150) C.fail = 1;
          for (int k = 0; k < 4; k++) C.u[k] += u[k];
        }
        C.sel = sel;
        if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
      }
    }
    __syncthreads();
    if (C.fail) return;
  }
  /* Ewald sites: the new configuration (+q) and the old one (-q) */
  if (threadIdx.x < na) {
    const int a = threadIdx.x;
    BeadPos bp;
    if (a == sb) bp = C.first;
    else bp = E.pos[C.sel * nb + (a < sb ? a : a - 1)];
    E.sites[a].b = bp;
    E.sites[a].q = S.mol_q[a];
    double p[3];
    atom_xyz(E, m, a, p);
    bead_set(E.sites[na + a].b, S, p[0], p[1], p[2], a, m);
    E.sites[na + a].q = -S.mol_q[a];
  }
  __syncthreads();
  const bool ew = S.ewald && S.mol_charged;
  int bw = 0;
  if (ew) {
    engine_ewald(E, 2 * na);
    bw = E.xb;
    E.xb ^= 1;
  }
  if (threadIdx.x == 0) {
    /* LJ-biasing corrections of both Rosenbluth weights, src/cbmc.c:3171-3178, :3044-3051 */
    const double rosen_new = C.rosen * exp(-S.beta * (C.u[1] + C.u[3]));
    const double rosen_old = C.rosen_old * exp(-S.beta * (C.uo[1] + C.uo[3]));
    double d_ads = 0.0, d_host = 0.0;
    if (ew) {
      double ea, eh;
      gather_ewald(E, bw, ea, eh);
      ewald_finish(S, ea, eh, S.excl_mol, S.excl_mol, 0, 0.0, d_ads, d_host);
    }
    const double pacc = exp(-S.beta * (d_ads + d_host)) * rosen_new / rosen_old;
    if (!(pacc == pacc)) C.status |= RGPU_ERR_NONFINITE;
    C.accept = E.rnd[SLOT_ACCEPT] < pacc;
    if (C.accept) {
      C.cnt[RGPU_CNT_REINS_ACCEPT]++;
      C.energy[RGPU_E_HOST_VDW] += C.u[0] - C.uo[0];
      C.energy[RGPU_E_HOST_REAL] += C.u[1] - C.uo[1];
      C.energy[RGPU_E_ADS_VDW] += C.u[2] - C.uo[2];
      C.energy[RGPU_E_ADS_REAL] += C.u[3] - C.uo[3];
      C.energy[RGPU_E_HOST_FOURIER] += d_host;
      C.energy[RGPU_E_ADS_FOURIER] += d_ads;
    }
  }
  __syncthreads();
  if (C.accept) {
    if (threadIdx.x < na) {
      double p[3] = {E.sites[threadIdx.x].b.x, E.sites[threadIdx.x].b.y, E.sites[threadIdx.x].b.z};
      atom_store(E, m, threadIdx.x, p);
    }
    if (ew) ewald_apply<MIXED>(S, E.tab, E.kw, E.sites, 2 * na, E.k0, E.k1);
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* The bend angle and dihedral of trial t of bead i >= 2, as chain_trial
 * draws them, by a group of 8 lanes (lane8 = lane % 8; every lane of the
 * warp calls): lane8 l forms proposals l, l + 8, ... of the bend angle and
 * of the dihedral, and the lowest accepted proposal of each wins, so the
 * result is chain_trial's (its proposals are tried in order and the first
 * accepted one is taken). The draws need no bead position, so a whole
 * growth stage's angles are drawn at once, before its first bead. A group
 * with live = false only takes part in the warp's votes. */
__device__ __forceinline__ void chain_angles_group(const RgpuSys &S, int i, int stage, int t, bool live,
                                                   uint64_t step, int lane, double &theta, double &phi)
{
  auto U = [&](int d) { return rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, t, d)); };
  const int k = 3 * RGPU_CHAIN_TRIES, l8 = lane & 7;
  const unsigned gmask = 0xffu << (lane & ~7);
  theta = S.bend_theta0;
  phi = M_PI;
  bool th_done = !live, ph_done = !live || i < 3;
  if (live && i == 2) phi = 2.0 * M_PI * U(k) - M_PI;
  for (int base = 0; base < RGPU_CHAIN_TRIES; base += 8) {
    if (!__any_sync(RGPU_FULL, !(th_done && ph_done))) break;
    const int a = base + l8;
    double th = 0.0, f = 0.0;
    bool okt = false, okp = false;
    if (!th_done) {
      const double u1 = U(3 * a), u2 = U(3 * a + 1), u3 = U(3 * a + 2);
      th = S.bend_theta0 + S.bend_sigma * sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
      okt = th > 0.0 && th < M_PI && u3 < sin(th);
    }
    if (!ph_done) {
      f = 2.0 * M_PI * U(k + 2 * a) - M_PI;
      okp = U(k + 2 * a + 1) < exp(-S.beta * (chain_torsion_energy(S, cos(f)) - S.torsion_min));
    }
    const unsigned bt = __ballot_sync(RGPU_FULL, okt) & gmask, bp = __ballot_sync(RGPU_FULL, okp) & gmask;
    const double ts = __shfl_sync(RGPU_FULL, th, bt ? __ffs(bt) - 1 : lane);
    const double fs = __shfl_sync(RGPU_FULL, f, bp ? __ffs(bp) - 1 : lane);
    if (!th_done && bt) {
      theta = ts;
      th_done = true;
    }
    if (!ph_done && bp) {
      phi = fs;
      ph_done = true;
    }
  }
}

/* CBMC growth (retrace = false) or retrace (retrace = true) of a flexible
 * chain, bead by bead from atom 0 (GrowMolecule / RetraceMolecule,
 * src/cbmc.c:2928-3181, for a linear chain): the first bead from nf trials
 * (random in the box; for a retrace trial 0 is the old bead), every other
 * bead from nt trials drawn by chain_trial (bonded Boltzmann factor built
 * in). The weight of a trial is exp(-beta (host VDW + adsorbate VDW + LJ
 * with the chain's beads four or more bonds back)); a trial overlaps when
 * one of them reaches the criterion. Leaves in Ctl the Rosenbluth weight
 * (product over beads of sum w / trials), the chosen beads (cp), their
 * host and adsorbate VDW (u[0], u[2]) and the intramolecular energy
 * (uintra: bonded + LJ), or fail. Molecule m is the one retraced; `exclude`
 * leaves a molecule out of the adsorbate sums. All threads call. */
/* The bend angle shared by the trials of bead i >= 2 in the reference's
 * scheme (chain_scheme 0): a growth draws it from sin(theta) exp(-beta
 * U_bend) (proposals in the slots of trial RGPU_REF_THETA_TRIAL from
 * RGPU_REF_THETA_SLOT on, tried in order: the lanes try 32 at once and the
 * lowest accepted wins), the distribution the reference's internal
 * Metropolis chain (src/cbmc.c:1822-2106) samples; a retrace (old !=
 * nullptr) keeps the old bead's angle. Every lane of the warp calls and
 * gets the angle. */
__device__ __noinline__ double chain_ref_theta(const RgpuSys &S, int i, int stage, uint64_t step, int lane,
                                                  const double (*old)[3])
{
  if (old) return chain_angle(old[i - 2], old[i - 1], old[i]);
  for (int base = 0; base < RGPU_CHAIN_TRIES; base += 32) {
    const int k = RGPU_REF_THETA_SLOT + 3 * (base + lane);
    auto U = [&](int d) { return rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, RGPU_REF_THETA_TRIAL, d)); };
    const double u1 = U(k), u2 = U(k + 1), u3 = U(k + 2);
    const double th = S.bend_theta0 + S.bend_sigma * sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
    const unsigned ok = __ballot_sync(RGPU_FULL, th > 0.0 && th < M_PI && u3 < sin(th));
    if (ok) return __shfl_sync(RGPU_FULL, th, __ffs(ok) - 1);
  }
  return S.bend_theta0;
}

/* The reference's bonded trials (chain_scheme 0; GenerateTrialOrientationsMCScheme,
 * src/cbmc.c:1580-2480, for a linear chain) of trial t of bead i >= 2 with
 * the bead's bend angle theta, by one warp (every lane calls), into
 * a[0..4] (lane 0 writes):
 * - the dihedral: ntors uniform candidates (slot k of the trial), one chosen
 *   by its torsion Boltzmann factor with SelectTrialPosition's rule
 *   (src/cbmc.c:563-599, 2403-2408; one uniform in slot
 *   RGPU_REF_TORS_SEL_SLOT). Candidates 2p and 2p+1 come from one Philox
 *   block and belong to lane p % 32 of row p / 32; the cumulative sum runs
 *   row by row as warp scans. A retrace's trial 0 keeps the old dihedral as
 *   its candidate 0 and chooses it. Without a torsion (bead 2) the dihedral
 *   is uniform (src/cbmc.c:2410);
 * - the torsion Rosenbluth factor: the mean of exp(-beta U_torsion) over
 *   candidates 0 .. ntrial-1, the reference's ComputeNormalizedRosenbluthWeight
 *   (src/cbmc.c:542-552 sums up to the global NumberOfTrialPositions; called
 *   at :2401); 1 for bead 2. */
template <bool F32>
__device__ __noinline__ void chain_ref_trial(const RgpuSys &S, int i, int stage, int t, uint64_t step, int lane,
                                                const double (*old)[3], double theta, double *a)
{
  /* F32 (the mixed engine): the candidates' Boltzmann factors in FP32, the
   * chosen dihedral itself from its FP64 uniform as in FP64 */
  typedef typename std::conditional<F32, float, double>::type T;
  const bool keep_old = old && t == 0;
  double phi = 0.0, wt = 1.0;
  if (i == 2) {
    if (!keep_old) phi = 2.0 * M_PI * rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, t, 0)) - M_PI;
  } else {
    const int n = S.ntors, nt = S.ntrial, rows = (n + 63) >> 6;
    const T beta = (T)S.beta;
    const T p0 = (T)S.torsion[0], p1 = (T)S.torsion[1], p2 = (T)S.torsion[2], p3 = (T)S.torsion[3];
    T bf[RGPU_TORS_ROWS][2];
    T big = (T)-1e30, wsum = 0;
#pragma unroll
    for (int j = 0; j < RGPU_TORS_ROWS; j++) {
      const int k0 = 2 * (lane + 32 * j);
      bf[j][0] = bf[j][1] = (T)-1e30;
      if (j < rows && k0 < n) {
        double u[2];
        float uf[2];
        if (F32) {
          /* the leading 24 bits of the two FP64 uniforms of the block
           * (rgpu_uniform_pair: o[0] and o[2] head their 53 bits) */
          uint32_t o[4];
          rgpu_philox((uint32_t)step, (uint32_t)(step >> 32), chain_slot(stage, i, t, k0) >> 1, S.sys_id,
                      (uint32_t)S.seed, (uint32_t)(S.seed >> 32), o);
          uf[0] = (float)(o[0] >> 8) * 5.9604644775390625e-8f;   /* 2^-24 */
          uf[1] = (float)(o[2] >> 8) * 5.9604644775390625e-8f;
        } else {
          rgpu_uniform_pair(S.seed, S.sys_id, step, chain_slot(stage, i, t, k0) >> 1, u);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int k = k0 + h;
          if (k < n) {
            T c;
            if (keep_old && k == 0) c = (T)chain_cos_dihedral(old[i - 3], old[i - 2], old[i - 1], old[i]);
            else if (F32) c = (T)-cospif(2.0f * uf[h]);
            else c = (T)cos(2.0 * M_PI * u[h] - M_PI);
            if (F32) {
              /* chain_torsion_energy in FP32 */
              const T c2 = (T)2 * c * c - (T)1, c3 = c * ((T)4 * c * c - (T)3);
              bf[j][h] = -beta * (p0 + p1 * ((T)1 + c) + p2 * ((T)1 - c2) + p3 * ((T)1 + c3));
            } else {
              bf[j][h] = -beta * (T)chain_torsion_energy(S, (double)c);
            }
            big = big > bf[j][h] ? big : bf[j][h];
            if (k < nt) wsum += F32 ? (T)__expf((float)bf[j][h]) : (T)exp((double)bf[j][h]);
          }
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      const T ob = __shfl_xor_sync(RGPU_FULL, big, o);
      big = big > ob ? big : ob;
      wsum += __shfl_xor_sync(RGPU_FULL, wsum, o);
    }
    wt = (double)wsum / (double)nt;
    if (!keep_old) {
      /* the shifted factors, once: summed here, scanned below */
      T tot = 0;
#pragma unroll
      for (int j = 0; j < RGPU_TORS_ROWS; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const bool v = j < rows && 2 * (lane + 32 * j) + h < n;
          bf[j][h] = v ? (F32 ? (T)__expf((float)(bf[j][h] - big)) : (T)exp((double)(bf[j][h] - big))) : (T)0;
          tot += bf[j][h];
        }
      for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(RGPU_FULL, tot, o);
      const T target =
          (T)rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, t, RGPU_REF_TORS_SEL_SLOT)) * tot;
      /* the first candidate whose cumulative sum reaches the target, row
       * by row; none (rounding only): the last, where the serial search
       * stops */
      int kc = n - 1;
      T before = 0;
      bool done = false;
#pragma unroll
      for (int j = 0; j < RGPU_TORS_ROWS; j++) {
        if (!done && j < rows) {
          const int k0 = 2 * (lane + 32 * j);
          const T e0 = bf[j][0], e1 = bf[j][1];
          const T part = e0 + e1;
          T incl = part;
          for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(RGPU_FULL, incl, o);
            if (lane >= o) incl += y;
          }
          const T c0 = before + (incl - part) + e0;
          const int mine = (k0 < n && c0 >= target) ? k0 : ((k0 + 1 < n && c0 + e1 >= target) ? k0 + 1 : -1);
          const unsigned hit = __ballot_sync(RGPU_FULL, mine >= 0);
          if (hit) {
            kc = __shfl_sync(RGPU_FULL, mine, __ffs(hit) - 1);
            done = true;
          }
          before += __shfl_sync(RGPU_FULL, incl, 31);
        }
      }
      if (lane == 0) {
        const double uk = rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, t, kc));
        if (F32) {
          /* phi = 2 pi u - pi: cos phi = -cospi(2u), sin phi = -sinpi(2u) */
          double sn, cs;
          sincospi(2.0 * uk, &sn, &cs);
          a[2] = -cs;
          a[3] = -sn;
          a[0] = cos(theta);
          a[1] = sin(theta);
          a[4] = wt;
          return;
        }
        phi = 2.0 * M_PI * uk - M_PI;
      }
    }
  }
  if (lane == 0) {
    a[0] = cos(theta);
    a[1] = sin(theta);
    a[2] = cos(phi);
    a[3] = sin(phi);
    a[4] = wt;
  }
}

/* The bend angles and dihedrals of beads 2.. of every trial of a growth
 * stage into `tab`, with each trial's torsion Rosenbluth factor. The
 * reference's scheme (S.chain_scheme 0): one warp per (bead, trial); a
 * retrace passes the old configuration `old` (published by a barrier
 * before the call). Independent draws (S.chain_scheme 1): 8 lanes per
 * (bead, trial), four per warp, and factor 1. The (bead, trial) tasks are
 * shared out over the warps of all CTAs of the cluster; after a cluster
 * barrier each CTA copies the other CTAs' rows from their shared memory.
 * All threads of the cluster call; the caller's next barrier publishes the
 * table. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void chain_angles_table(Eng<MIXED, FLEX> &E, int stage, double *tab,
                                                   const double (*old)[3])
{
  const RgpuSys &S = *E.S;
  const int na = S.natom, nt = S.ntrial;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int ntask = na > 2 ? (na - 2) * nt : 0;
  const int gw = E.rank * nw + (threadIdx.x >> 5), ngw = nw * E.csize;   /* warp of the cluster */
  const int per = S.chain_scheme == 0 ? 1 : 4;                           /* tasks a warp takes at once */
  if (S.chain_scheme == 0) {
    /* each bead's bend angle once (one warp per bead, in every CTA), then
     * one warp per (bead, trial); the angles sit after the table */
    double *theta = tab + RGPU_ANG_TABLE;
    for (int i = 2 + (threadIdx.x >> 5); i < na; i += nw) {
      const double th = chain_ref_theta(S, i, stage, E.step, lane, old);
      if (lane == 0) theta[i] = th;
    }
    __syncthreads();
    for (int task = gw; task < ntask; task += ngw) {
      const int i = 2 + task / nt, t = task % nt;
      chain_ref_trial<(MIXED != 0)>(S, i, stage, t, E.step, lane, old, theta[i],
                             tab + RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS + t));
    }
  } else {
    for (int t0 = gw * 4; t0 < ntask; t0 += ngw * 4) {
      const int task = t0 + (lane >> 3);
      const bool live = task < ntask;
      const int i = live ? 2 + task / nt : 2, t = live ? task % nt : 0;
      double th, ph;
      chain_angles_group(S, i, stage, t, live, E.step, lane, th, ph);
      if (live && (lane & 7) == 0) {
        double *a = tab + RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS + t);
        a[0] = cos(th);
        a[1] = sin(th);
        a[2] = cos(ph);
        a[3] = sin(ph);
        a[4] = 1.0;
      }
    }
  }
  if (E.csize > 1) {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    for (int task = threadIdx.x; task < ntask; task += blockDim.x) {
      const int owner = ((task / per) % ngw) / nw;
      if (owner == E.rank) continue;
      const int off = RGPU_ANG_STRIDE * ((task / nt) * RGPU_MAX_TRIALS + task % nt);
      const double *src = cl.map_shared_rank(tab, owner) + off;
      for (int d = 0; d < RGPU_ANG_STRIDE; d++) tab[off + d] = src[d];
    }
    /* no CTA writes this table again before the next cluster barrier (the
     * evaluation that follows ends with one), so the peers' reads are done
     * by then */
  }
}

/* Retrace of a flexible chain's configuration (RetraceMolecule,
 * src/cbmc.c:3056-3181, for a linear chain). The beads a retrace "chooses"
 * are the old ones, known before anything is evaluated, so the trial sets of
 * several beads are placed together and evaluated at once: beads are taken
 * in growth order in groups whose trials fit one evaluation (RGPU_MAX_POS
 * positions; for 6 beads of 16 trials and 8 first-bead trials, two
 * evaluations instead of six). Each bead's weights are summed by one warp in
 * trial order, and the Rosenbluth weight and the energies are combined bead
 * by bead in growth order, stopping at the first bead without a valid
 * trial, as the bead-by-bead retrace does. The trials draw the same random
 * numbers as that retrace (counter-based, by stage, bead and trial). All
 * threads call. */
/* Beads of a retrace taken in one evaluation: from bead i0 on, as many as
 * fit `room` positions (at least one; room >= RGPU_MAX_TRIALS). */
__device__ __forceinline__ int retrace_group_end(int i0, int na, int nf, int nt, int room, int &P)
{
  int i1 = i0;
  P = 0;
  while (i1 < na && P + (i1 == 0 ? nf : nt) <= room) {
    P += i1 == 0 ? nf : nt;
    i1++;
  }
  return i1;
}

/* Places the trials of retrace beads [i0, i0 + ...) at positions off ..
 * off + P, position j of the group being bead i, trial t in growth order;
 * trial 0 of each bead is the old bead old[i]. Threads t0, t0 + step, ...
 * of the block place. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void retrace_place(Eng<MIXED, FLEX> &E, int stage, int i0, int P, int off,
                                              const double (*old)[3], const double *ang, int exclude, int t0,
                                              int step)
{
  const RgpuSys &S = *E.S;
  const int nf = S.ntrial_first, nt = S.ntrial;
  for (int j = t0; j < P; j += step) {
    int i = i0, t = j;
    while (t >= (i == 0 ? nf : nt)) {
      t -= i == 0 ? nf : nt;
      i++;
    }
    double p[3];
    if (t == 0) {
      p[0] = old[i][0];
      p[1] = old[i][1];
      p[2] = old[i][2];
    } else if (i == 0) {
      rgpu_box_point(S, rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 0)),
                     rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 1)),
                     rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 2)), p);
    } else if (i == 1) {
      const uint64_t stp = E.step;
      chain_trial(S, old, i, [&](int d) { return rgpu_uniform(S.seed, S.sys_id, stp, chain_slot(stage, i, t, d)); },
                  p);
    } else {
      const double *a = ang + RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS + t);
      chain_place_trig(i >= 3 ? old[i - 3] : nullptr, old[i - 2], old[i - 1], S.bond, a[0], a[1], a[2], a[3], p);
    }
    bead_set(E.pos[off + j], S, p[0], p[1], p[2], i, exclude);
  }
}

/* Bookkeeping of retrace beads [i0, i1) evaluated at positions off.. of
 * buffer b: warp w0 + g takes bead i0 + g (warps w0, w0 + 1, ... of the
 * block), sums its weights in trial order and leaves in C.rb[i] the sum,
 * the old bead's host and adsorbate VDW, intramolecular LJ and bonded
 * energy, and whether any trial was valid. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void retrace_book(const Eng<MIXED, FLEX> &E, int b, int i0, int i1, int off,
                                             const double (*old)[3], const double *ang, int w0)
{
  const RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int nf = S.ntrial_first, nt = S.ntrial;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (warp < w0) return;
  for (int g = warp - w0; g < i1 - i0; g += nw - w0) {
    const int i = i0 + g, k = i == 0 ? nf : nt;
    const int o0 = off + (i0 == 0 ? (i == 0 ? 0 : nf + (i - 1) * nt) : g * nt);
    double r[4] = {0.0, 0.0, 0.0, 0.0}, lj = 0.0, bf = 0.0;
    int o = 0, ov = 0;
    if (lane < k) {
      gather(E, b, o0 + lane, r, o);
      const double p[3] = {E.pos[o0 + lane].x, E.pos[o0 + lane].y, E.pos[o0 + lane].z};
      lj = chain_intra_lj(S, old, i, p);
      ov = r[0] >= S.overlap || r[1] >= S.overlap || r[2] >= S.overlap || r[3] >= S.overlap || lj >= S.overlap;
      bf = -S.beta * (r[0] + r[2] + lj);
    }
    const bool valid = lane < k && !ov;
    const double w = valid ? exp(bf) : 0.0;
    const bool any = __ballot_sync(RGPU_FULL, valid) != 0u;
    double wsum = 0.0;
    for (int t = 0; t < k; t++) wsum += __shfl_sync(RGPU_FULL, w, t);
    if (lane == 0) {
      double *rb = C.rb[i];
      /* with the old trial's torsion Rosenbluth factor (1 for independent draws) */
      rb[0] = i >= 2 ? wsum * ang[RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS) + 4] : wsum;
      rb[1] = r[0];
      rb[2] = r[2];
      rb[3] = lj;
      rb[4] = i >= 2 ? chain_bonded_energy(S, old, i, old[i]) : 0.0;
      rb[5] = any ? 1.0 : 0.0;
    }
  }
}

/* Thread 0: the retrace beads [i0, i1) into the Rosenbluth weight and the
 * energies, in growth order, stopping at the first bead without a valid
 * trial. */
__device__ __forceinline__ void retrace_combine(Ctl &C, int i0, int i1, int nf, int nt)
{
  for (int i = i0; i < i1 && !C.fail; i++) {
    const double *rb = C.rb[i];
    C.rosen *= rb[0] / (double)(i == 0 ? nf : nt);
    C.u[0] += rb[1];
    C.u[2] += rb[2];
    C.uintra += rb[3];
    if (i >= 2) C.uintra += rb[4];
    if (rb[5] == 0.0) {
      C.fail = 1;
      C.cnt[RGPU_CNT_OVERLAP]++;
    }
  }
}

/* Retrace of a flexible chain's configuration (RetraceMolecule,
 * src/cbmc.c:3056-3181, for a linear chain). The beads a retrace "chooses"
 * are the old ones, known before anything is evaluated, so the trial sets of
 * several beads are placed together and evaluated at once: beads are taken
 * in growth order in groups whose trials fit one evaluation (RGPU_MAX_POS
 * positions; for 6 beads of 16 trials and 8 first-bead trials, two
 * evaluations instead of six). Each bead's weights are summed by one warp in
 * trial order, and the Rosenbluth weight and the energies are combined bead
 * by bead in growth order, stopping at the first bead without a valid
 * trial, as the bead-by-bead retrace does. The trials draw the same random
 * numbers as that retrace (counter-based, by stage, bead and trial). All
 * threads call. */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void retrace_chain(Eng<MIXED, FLEX> &E, int stage, int m, int exclude)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int na = S.natom, nf = S.ntrial_first, nt = S.ntrial;
  if (threadIdx.x == 0) {
    C.rosen = 1.0;
    C.u[0] = C.u[1] = C.u[2] = C.u[3] = 0.0;
    C.uintra = 0.0;
    C.fail = 0;
  }
  if (threadIdx.x < na) atom_xyz(E, m, threadIdx.x, C.cp[threadIdx.x]);
  if (S.chain_scheme == 0) __syncthreads();   /* the old configuration, read by the table */
  chain_angles_table(E, stage, E.ang, (const double(*)[3])C.cp);
  __syncthreads();
  for (int i0 = 0; i0 < na;) {
    int P;
    const int i1 = retrace_group_end(i0, na, nf, nt, RGPU_MAX_POS, P);
    retrace_place(E, stage, i0, P, 0, C.cp, E.ang, exclude, threadIdx.x, blockDim.x);
    __syncthreads();
    engine_eval(E, P, 0);
    const int b = E.xb;
    E.xb ^= 1;
    retrace_book(E, b, i0, i1, 0, C.cp, E.ang, 0);
    __syncthreads();
    if (threadIdx.x == 0) retrace_combine(C, i0, i1, nf, nt);
    __syncthreads();
    if (C.fail) return;
    i0 = i1;
  }
}

template <int MIXED, bool FLEX>
__device__ __forceinline__ void grow_chain(Eng<MIXED, FLEX> &E, bool retrace, int stage, int m, int exclude,
                                           bool ride = false)
{
  if (retrace) {
    retrace_chain(E, stage, m, exclude);
    return;
  }
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int na = S.natom, nf = S.ntrial_first, nt = S.ntrial;
  if (threadIdx.x == 0) {
    C.rosen = 1.0;
    C.u[0] = C.u[1] = C.u[2] = C.u[3] = 0.0;
    C.uintra = 0.0;
    C.fail = 0;
  }
  /* the bend angles and dihedrals of beads 2.. of every trial, ahead of the
   * first bead (the first barrier below publishes them) */
  chain_angles_table(E, stage, E.ang, nullptr);
  /* ride: a reinsertion's retrace (stage 1) of molecule m rides along with
   * the first beads' evaluations, one group of retrace beads each, in the
   * positions after the growth's trials; its beads' sums are left in C.rb */
  double *ang_r = E.ang + RGPU_ANG_DOUBLES;
  if (ride) {
    if (threadIdx.x < na) atom_xyz(E, m, threadIdx.x, C.co[threadIdx.x]);
    if (S.chain_scheme == 0) __syncthreads();   /* the old configuration, read by the table */
    chain_angles_table(E, 1, ang_r, (const double(*)[3])C.co);
  }
  int r0 = ride ? 0 : na;   /* next retrace bead */
  for (int i = 0; i < na; i++) {
    const int k = i == 0 ? nf : nt;
    int r1 = r0, rP = 0;
    if (r0 < na) {
      r1 = retrace_group_end(r0, na, nf, nt, RGPU_MAX_POS - k, rP);
      if (i == 0) __syncthreads();   /* C.co and the retrace angles */
      if (threadIdx.x >= 32) retrace_place(E, 1, r0, rP, k, C.co, ang_r, m, threadIdx.x - 32, blockDim.x - 32);
    }
    if (threadIdx.x < k) {
      const int t = threadIdx.x;
      double p[3];
      if (retrace && t == 0) {
        atom_xyz(E, m, i, p);
      } else if (i == 0) {
        rgpu_box_point(S, rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 0)),
                       rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 1)),
                       rgpu_uniform(S.seed, S.sys_id, E.step, chain_slot(stage, 0, t, 2)), p);
      } else if (i == 1) {
        const uint64_t step = E.step;
        chain_trial(S, C.cp, i,
                    [&](int d) { return rgpu_uniform(S.seed, S.sys_id, step, chain_slot(stage, i, t, d)); }, p);
      } else {
        const double *a = E.ang + RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS + t);
        chain_place_trig(i >= 3 ? C.cp[i - 3] : nullptr, C.cp[i - 2], C.cp[i - 1], S.bond, a[0], a[1], a[2], a[3], p);
      }
      bead_set(E.pos[t], S, p[0], p[1], p[2], i, exclude);
    }
    __syncthreads();
    engine_eval(E, k + rP, 0);
    const int b = E.xb;
    E.xb ^= 1;
    if (r1 > r0) {
      /* warps 1..: the retrace group's bookkeeping (warp 1 then goes on to
       * this bead's bonded energies) */
      retrace_book(E, b, r0, r1, k, C.co, ang_r, 1);
      r0 = r1;
    }
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      double r[4] = {0.0, 0.0, 0.0, 0.0}, lj = 0.0, bf = 0.0;
      int o = 0, ov = 0;
      if (lane < k) {
        gather(E, b, lane, r, o);
        const double p[3] = {E.pos[lane].x, E.pos[lane].y, E.pos[lane].z};
        lj = chain_intra_lj(S, C.cp, i, p);
        ov = r[0] >= S.overlap || r[1] >= S.overlap || r[2] >= S.overlap || r[3] >= S.overlap || lj >= S.overlap;
        bf = -S.beta * (r[0] + r[2] + lj);
      }
      const bool valid = lane < k && !ov;
      const double w = valid ? exp(bf) : 0.0;
      const bool any = __ballot_sync(RGPU_FULL, valid) != 0u;
      double wsum = 0.0;
      for (int t = 0; t < k; t++) wsum += __shfl_sync(RGPU_FULL, w, t);
      int sel = 0;
      if (!retrace && any) {
        /* SelectTrialPosition (src/cbmc.c:563-599) on the weights themselves */
        const double target = rgpu_uniform(S.seed, S.sys_id, E.step, RGPU_SLOT_CHAIN_SEL + stage * 8 + i) * wsum;
        double cum = __shfl_sync(RGPU_FULL, w, 0);
        while (cum < target && sel < k - 1) {
          sel++;
          cum += __shfl_sync(RGPU_FULL, w, sel);
        }
      }
      const double hv = __shfl_sync(RGPU_FULL, r[0], sel), av = __shfl_sync(RGPU_FULL, r[2], sel);
      const double ljs = __shfl_sync(RGPU_FULL, lj, sel);
      if (lane == 0) {
        /* with the chosen trial's torsion Rosenbluth factor (src/cbmc.c:2793;
         * 1 for independent draws) */
        C.rosen *= wsum / (double)k * (i >= 2 ? E.ang[RGPU_ANG_STRIDE * ((i - 2) * RGPU_MAX_TRIALS + sel) + 4] : 1.0);
        if (!any || (!retrace && C.rosen < 1e-150)) C.fail = 1;
        C.u[0] += hv;
        C.u[2] += av;
        C.uintra += ljs;
        C.sel = sel;
        C.cp[i][0] = E.pos[sel].x;
        C.cp[i][1] = E.pos[sel].y;
        C.cp[i][2] = E.pos[sel].z;
        if (C.fail) C.cnt[RGPU_CNT_OVERLAP]++;
      }
    } else if (i >= 2 && threadIdx.x < 32 + k) {
      /* meanwhile warp 1: the trials' bonded energies (beads i-1.. of C.cp
       * are fixed; warp 0 writes only C.cp[i]) */
      const int t = threadIdx.x - 32;
      const double p[3] = {E.pos[t].x, E.pos[t].y, E.pos[t].z};
      C.ub[t] = chain_bonded_energy(S, C.cp, i, p);
    }
    __syncthreads();
    /* the chosen trial's bonded energy; C.ub and C.sel stay untouched until
     * the next bead's selection, several barriers on */
    if (threadIdx.x == 0 && i >= 2) C.uintra += C.ub[C.sel];
    if (C.fail) return;
  }
}

/* CBMC insertion, deletion and Widom test insertion of a flexible chain
 * (SwapAddAdsorbateMove src/mc_moves.c:7016, SwapRemoveAdsorbateMove :7228,
 * WidomAdsorbateMove :7844; uncharged chains, no Fourier part). */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void step_swap_chain(Eng<MIXED, FLEX> &E, bool insert, bool widom)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int na = S.natom, nmol = C.nmol;
  if (widom && threadIdx.x == 0) C.sums[RGPU_SUM_WIDOM_N] += 1.0;
  int m = nmol;
  if (!insert) {
    m = (int)(E.rnd[SLOT_MOLECULE] * nmol);
    if (m >= nmol) m = nmol - 1;
  }
  grow_chain(E, !insert, insert ? 0 : 1, m, insert ? -1 : m);
  if (C.fail) return;
  if (threadIdx.x == 0) {
    double pacc;
    if (insert) pacc = C.rosen * S.fugacity_beta_v / (1.0 + nmol);
    else pacc = (double)nmol / (C.rosen * S.fugacity_beta_v);
    if (!(pacc == pacc)) C.status |= RGPU_ERR_NONFINITE;
    C.accept = !widom && E.rnd[SLOT_ACCEPT] < pacc;
    if (widom) C.sums[RGPU_SUM_WIDOM_W] += C.rosen;
    if (C.accept) {
      C.cnt[RGPU_CNT_ACCEPT + (insert ? 2 : 3)]++;
      const double sgn = insert ? 1.0 : -1.0;
      C.energy[RGPU_E_HOST_VDW] += sgn * C.u[0];
      C.energy[RGPU_E_ADS_VDW] += sgn * C.u[2];
      C.energy[RGPU_E_INTRA] += sgn * C.uintra;
    }
  }
  __syncthreads();
  if (C.accept) {
    if (insert) {
      if (threadIdx.x < na) atom_store(E, nmol, threadIdx.x, C.cp[threadIdx.x]);
    } else {
      const int last = nmol - 1;
      if (threadIdx.x < na && m != last) {
        double p[3];
        atom_xyz(E, last, threadIdx.x, p);
        atom_store(E, m, threadIdx.x, p);
      }
    }
    if (threadIdx.x == 0) {
      C.nmol = insert ? nmol + 1 : nmol - 1;
      C.nads = C.nmol * na;
    }
    __syncthreads();
  }
}

/* CBMC reinsertion of a flexible chain (ReinsertionAdsorbateMove,
 * src/mc_moves.c:4415): a new configuration grown with molecule m left out,
 * the old one retraced; accepted with W(new) / W(old). */
template <int MIXED, bool FLEX>
__device__ __forceinline__ void step_reinsert_chain(Eng<MIXED, FLEX> &E)
{
  RgpuSys &S = *E.S;
  Ctl &C = *E.ctl;
  const int na = S.natom, nmol = C.nmol;
  int m = (int)(E.rnd[SLOT_MOLECULE] * nmol);
  if (m >= nmol) m = nmol - 1;
  /* the retrace of the old configuration rides along with the growth's
   * first evaluations (it does not depend on the new chain); its beads are
   * combined after a successful growth, as a retrace run after it would */
  grow_chain(E, false, 0, m, m, true);
  if (C.fail) return;
  if (threadIdx.x == 0) {
    C.rosen_old = C.rosen;     /* the new configuration's weight */
    C.dl[0] = C.u[0];
    C.dl[2] = C.u[2];
    C.uintra_old = C.uintra;
    for (int a = 0; a < na; a++)
      for (int d = 0; d < 3; d++) C.cpn[a][d] = C.cp[a][d];
    C.rosen = 1.0;
    C.u[0] = C.u[1] = C.u[2] = C.u[3] = 0.0;
    C.uintra = 0.0;
    retrace_combine(C, 0, na, S.ntrial_first, S.ntrial);
  }
  __syncthreads();
  if (C.fail) return;
  if (threadIdx.x == 0) {
    const double w_new = C.rosen_old, w_old = C.rosen;
    const double pacc = w_new / w_old;
    if (!(pacc == pacc)) C.status |= RGPU_ERR_NONFINITE;
    C.accept = E.rnd[SLOT_ACCEPT] < pacc;
    if (C.accept) {
      C.cnt[RGPU_CNT_REINS_ACCEPT]++;
      C.energy[RGPU_E_HOST_VDW] += C.dl[0] - C.u[0];
      C.energy[RGPU_E_ADS_VDW] += C.dl[2] - C.u[2];
      C.energy[RGPU_E_INTRA] += C.uintra_old - C.uintra;
    }
  }
  __syncthreads();
  if (C.accept) {
    if (threadIdx.x < na) atom_store(E, m, threadIdx.x, C.cpn[threadIdx.x]);
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* Loads a descriptor copy into shared memory. */
__device__ inline void load_sys(RgpuSys *dst, const RgpuSys *src)
{
  const uint32_t *s = (const uint32_t *)src;
  uint32_t *d = (uint32_t *)dst;
  for (int i = threadIdx.x; i < (int)(sizeof(RgpuSys) / 4); i += blockDim.x) d[i] = s[i];
  __syncthreads();
}

/* WIDE: compiled for CTAs of up to 1024 threads (64 registers per thread);
 * otherwise up to 512 threads with 128 registers. The engine picks WIDE for
 * CTAs above 512 threads and when several CTAs must share an SM. FLEX:
 * compiled with flexible-chain moves and energy grids; batches of rigid
 * molecules without grids run the build without them, whose register
 * allocation the chain and grid code does not touch. */
template <int MIXED, bool WIDE, bool FLEX>
__global__ void __launch_bounds__(WIDE ? 1024 : 512) rgpu_engine_kernel(RgpuSys *systems, int nsys, long long nsteps,
                                                                       int kw, int max_ads_atoms, int fw_items,
                                                                       int tile_items, int k_items)
{
  extern __shared__ __align__(256) unsigned char smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int csize = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int sysi = blockIdx.x / csize;
  const int nwarps = blockDim.x >> 5;
  const EngineLayout L = engine_layout(MIXED, fw_items, tile_items, max_ads_atoms, kw, k_items, nwarps, FLEX);
  if (sysi < nsys) {
    Eng<MIXED, FLEX> E;
    E.rank = rank;
    E.csize = csize;
    E.xb = 0;
    E.S = (RgpuSys *)(smem + L.sys);
    E.ads = smem + L.ads;
    E.pos = (BeadPos *)(smem + L.pos);
    E.uv = (double *)(smem + L.uv);
    E.uc = (double *)(smem + L.uc);
    E.uo = (int *)(smem + L.uo);
    E.part = (PosSum *)(smem + L.part);
    E.sc.uv = E.uv;
    E.sc.uc = E.uc;
    E.sc.uo = E.uo;
    E.sc.qr2 = (float *)(smem + L.q);
    E.sc.qq = E.sc.qr2 + nwarps * (MIXED == 2 ? 128 : 64);
    E.sc.qt = (int *)(E.sc.qq + nwarps * 64);
    E.sites = (EwSite *)(smem + L.sites);
    E.tab = (typename PhaseT<MIXED>::T *)(smem + L.tab);
    E.kw = kw;
    E.red = (double *)(smem + L.red);
    E.ang = (double *)(smem + L.ang);
    E.ctl = (Ctl *)(smem + L.ctl);
    Ctl &C = *E.ctl;
    E.sc.cnt = C.work;
    E.sc.next = &C.next;
    load_sys(E.S, &systems[sysi]);
    RgpuSys &S = *E.S;
    /* a system at its step limit (a finished job left in its slot) takes
     * no step in this launch: its CTAs leave before staging anything and
     * write nothing back. All CTAs of the cluster read the same limits, so
     * the whole cluster leaves and none waits at the cluster barrier below. */
    if (S.step[0] >= S.step[1]) return;
    double2 *sk_global = S.sk_ads;
    if (threadIdx.x < 5) C.work[threadIdx.x] = 0ULL;
    if (threadIdx.x < RGPU_NCNT) C.cnt[threadIdx.x] = 0;
    if (threadIdx.x < RGPU_NE) C.energy[threadIdx.x] = S.energy[threadIdx.x];
    if (threadIdx.x == 0) {
      C.cyc[0] = C.cyc[1] = 0;
      C.status = 0;
      C.next = 0;
      for (int k = 0; k < RGPU_NSUM; k++) C.sums[k] = 0.0;
      C.nmol = *S.nmol;
      C.nads = C.nmol * S.natom;
    }
    /* this CTA's framework share, staged in shared memory when it fits */
    if (MIXED) {
      int t0, t1;
      share(S.ntile, rank, csize, t0, t1);
      E.sl.fw_lo = t0;
      E.sl.fw_hi = t1;
      if (S.smem_fw) {
        int4 *dfw = (int4 *)(smem + L.fw);
        TileRec *dt = (TileRec *)(smem + L.tiles);
        for (int i = threadIdx.x; i < (t1 - t0) * RGPU_TILE; i += blockDim.x) dfw[i] = S.fw32[t0 * RGPU_TILE + i];
        for (int i = threadIdx.x; i < t1 - t0; i += blockDim.x) dt[i] = S.tiles[t0 + i];
        E.sl.fw = dfw - (size_t)t0 * RGPU_TILE;
        E.sl.tiles = dt - t0;
      } else {
        E.sl.fw = S.fw32;
        E.sl.tiles = S.tiles;
      }
    } else {
      int a0, a1;
      share(S.nfw, rank, csize, a0, a1);
      E.sl.fw_lo = a0;
      E.sl.fw_hi = a1;
      E.sl.tiles = nullptr;
      if (S.smem_fw) {
        double4 *d = (double4 *)(smem + L.fw);
        for (int i = threadIdx.x; i < a1 - a0; i += blockDim.x) d[i] = S.fw64[a0 + i];
        E.sl.fw = d - a0;
      } else {
        E.sl.fw = S.fw64;
      }
    }
    E.sl.ads = E.ads;
    if (FLEX && S.use_grid) E.sl.fw_hi = E.sl.fw_lo;   /* host VDW from the grids: no framework pairs */
    /* this CTA's wave vectors with their prefactors and S(k) */
    if (S.ewald) share(S.nk, rank, csize, E.k0, E.k1);
    else { E.k0 = 0; E.k1 = 0; }
    const bool k_smem = k_items >= E.k1 - E.k0;
    __syncthreads();
    if (k_smem && E.k1 > E.k0) {
      char4 *kv = (char4 *)(smem + L.kvec);
      double *kf = (double *)(smem + L.kf);
      double2 *sf = (double2 *)(smem + L.skfw);
      double2 *sa = (double2 *)(smem + L.skads);
      for (int i = threadIdx.x; i < E.k1 - E.k0; i += blockDim.x) {
        kv[i] = S.kvec[E.k0 + i];
        kf[i] = S.kfactor[E.k0 + i];
        sf[i] = S.sk_fw[E.k0 + i];
        sa[i] = S.sk_ads[E.k0 + i];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        S.kvec = kv - E.k0;
        S.kfactor = kf - E.k0;
        S.sk_fw = sf - E.k0;
        S.sk_ads = sa - E.k0;
      }
    }
    /* adsorbate records to shared memory (full copy in every CTA) */
    for (int i = threadIdx.x; i < C.nads; i += blockDim.x) {
      const int mm = i / S.natom, a = i - mm * S.natom;
      const double *x = S.ads_xyz + 3 * i;
      if (MIXED) {
        int xi, yi, zi;
        rgpu_fix3(S, x[0], x[1], x[2], xi, yi, zi);
        ((int4 *)E.ads)[i] = make_int4(xi, yi, zi, mm * 16 + a);
      } else
        atom_store(E, mm, a, x);
    }
    __syncthreads();
    const uint64_t step0 = S.step[0], step_end = S.step[1], avg0 = S.step[2];
    const long long t_start = clock64();
    long long it = 0;
    for (; it < nsteps && step0 + (uint64_t)it < step_end; it++) {
      const uint64_t step = step0 + (uint64_t)it;
      /* this step's random numbers, one Philox block per thread */
      double *rb = C.rnd[it & 1];
      for (int i = threadIdx.x; i < RGPU_RND / 2; i += blockDim.x) rgpu_uniform_pair(S.seed, S.sys_id, step, i, &rb[2 * i]);
      __syncthreads();
      E.rnd = rb;
      E.step = step;
      const double u0 = rb[SLOT_MOVE];
      int mv = 0;
      while (mv < 5 && u0 >= S.cum[mv]) mv++;
      const int nmol = C.nmol;
      share(C.nads, rank, csize, E.sl.ads_lo, E.sl.ads_hi);
      if (mv <= 1) {
        if (!(nmol == 0 || (mv == 1 && S.natom == 1))) {
          if (threadIdx.x == 0) { C.cnt[RGPU_CNT_MOVES]++; C.cnt[RGPU_CNT_ATTEMPT + mv]++; }
          step_displace(E, mv);
        }
      } else if (mv == 2) {
        if (threadIdx.x == 0) { C.cnt[RGPU_CNT_MOVES]++; C.cnt[RGPU_CNT_ATTEMPT + 2]++; }
        if (nmol >= S.maxmol) {
          if (threadIdx.x == 0) C.status |= RGPU_ERR_MAXMOL;
        } else if (FLEX && S.flexible) {
          step_swap_chain(E, true, false);
        } else {
          step_swap(E, true);
        }
      } else if (mv == 3) {
        if (threadIdx.x == 0) { C.cnt[RGPU_CNT_MOVES]++; C.cnt[RGPU_CNT_ATTEMPT + 3]++; }
        if (nmol != 0) {
          if (FLEX && S.flexible) step_swap_chain(E, false, false);
          else step_swap(E, false);
        }
      } else if (mv == 4) {
        /* the reference returns before counting when there is no molecule */
        if (nmol != 0) {
          if (threadIdx.x == 0) { C.cnt[RGPU_CNT_MOVES]++; C.cnt[RGPU_CNT_REINS_ATTEMPT]++; }
          if (FLEX && S.flexible) step_reinsert_chain(E);
          else step_reinsert(E);
        }
      } else {
        if (threadIdx.x == 0) C.cnt[RGPU_CNT_MOVES]++;
        if (FLEX && S.flexible) step_swap_chain(E, true, true);
        else step_swap(E, true, true);
      }
      /* ensemble sums after the step (thread 0 owns the running values) */
      if (threadIdx.x == 0 && step >= avg0) {
        const double n = (double)C.nmol;
        const double u = C.energy[0] + C.energy[1] + C.energy[2] + C.energy[3] + C.energy[4] + C.energy[5] +
                         C.energy[RGPU_E_INTRA];
        C.sums[RGPU_SUM_SAMPLES] += 1.0;
        C.sums[RGPU_SUM_N] += n;
        C.sums[RGPU_SUM_N2] += n * n;
        C.sums[RGPU_SUM_U] += u;
        C.sums[RGPU_SUM_UN] += u * n;
        C.sums[RGPU_SUM_U2] += u * u;
      }
    }
    __syncthreads();
    /* write back: positions, molecule count, energies, counters (rank 0);
     * this CTA's share of S(k) and its work counters (every CTA) */
    if (k_smem)
      for (int k = E.k0 + threadIdx.x; k < E.k1; k += blockDim.x) sk_global[k] = S.sk_ads[k];
    if (rank == 0) {
      /* FP64 positions (the mixed path keeps them in global memory already) */
      for (int i = threadIdx.x; !MIXED && i < C.nads; i += blockDim.x) {
        const int mm = i / S.natom, a = i - mm * S.natom;
        double p[3];
        atom_xyz(E, mm, a, p);
        S.ads_xyz[3 * i] = p[0];
        S.ads_xyz[3 * i + 1] = p[1];
        S.ads_xyz[3 * i + 2] = p[2];
      }
      if (threadIdx.x < RGPU_NE) S.energy[threadIdx.x] = C.energy[threadIdx.x];
      if (threadIdx.x == 0) {
        *S.nmol = C.nmol;
        S.step[0] = step0 + (uint64_t)it;
        for (int k = 0; k < RGPU_NSUM; k++) S.sums[k] += C.sums[k];
        for (int c = 0; c < RGPU_CNT_PAIRS; c++) S.counters[c] += C.cnt[c];
        S.counters[RGPU_CNT_REINS_ATTEMPT] += C.cnt[RGPU_CNT_REINS_ATTEMPT];
        S.counters[RGPU_CNT_REINS_ACCEPT] += C.cnt[RGPU_CNT_REINS_ACCEPT];
        *S.status |= C.status;
        S.counters[RGPU_CNT_CYCLES] += clock64() - t_start;
        S.counters[RGPU_CNT_CYC_EVAL] += C.cyc[0];
        S.counters[RGPU_CNT_CYC_EWALD] += C.cyc[1];
      }
    }
    if (threadIdx.x == 0)
      for (int c = 0; c < 5; c++) atomicAdd((unsigned long long *)&S.counters[RGPU_CNT_PAIRS + c], C.work[c]);
  }
  /* no CTA may leave while a peer can still read its shared memory */
  cl.sync();
}

/* the kernel build for (mixed, wide, flex) */
using EngineKernel = void (*)(RgpuSys *, int, long long, int, int, int, int, int);
static EngineKernel engine_kernel(int mixed, bool wide, bool flex)
{
  if (mixed == 2) return wide ? rgpu_engine_kernel<2, true, false> : rgpu_engine_kernel<2, false, false>;
  if (mixed && wide) return flex ? rgpu_engine_kernel<1, true, true> : rgpu_engine_kernel<1, true, false>;
  if (mixed) return flex ? rgpu_engine_kernel<1, false, true> : rgpu_engine_kernel<1, false, false>;
  return flex ? rgpu_engine_kernel<0, false, true> : rgpu_engine_kernel<0, false, false>;
}

cudaError_t rgpu_engine_prepare(int mixed, bool wide, bool flex, size_t smem)
{
  return cudaFuncSetAttribute(engine_kernel(mixed, wide, flex), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t rgpu_engine_launch(int mixed, RgpuSys *d_systems, int nsys, long long nsteps, int kw,
                               int max_ads_atoms, int fw_items, int tile_items, int k_items, int cluster,
                               int threads, bool wide, bool flex, cudaStream_t st)
{
  size_t smem = rgpu_engine_smem_bytes(mixed, fw_items, tile_items, max_ads_atoms, kw, k_items, threads, flex);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nsys * cluster), 1, 1);
  cfg.blockDim = dim3((unsigned)threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  /* the dynamic shared-memory limit is raised by rgpu_engine_prepare, outside
   * any stream capture */
  return cudaLaunchKernelEx(&cfg, engine_kernel(mixed, wide, flex), d_systems, nsys, nsteps, kw, max_ads_atoms,
                            fw_items, tile_items, k_items);
}

struct CallSmem {
  double res[RGPU_MAX_POS][4];
  int ovf[RGPU_MAX_POS];
  double uv[RGPU_MAX_UNITS], uc[RGPU_MAX_UNITS];
  int uo[RGPU_MAX_UNITS];
  BeadPos pos[RGPU_MAX_POS];
  float qr2[8 * 64], qq[8 * 64];
  int qt[8 * 64];
  double red[72];
  int next;
};


/* Energies of P bead positions (P <= RGPU_MAX_POS), given as FP64 xyz with
 * the molecule-atom index of each bead. out[p*4 + k], ov[p].
 *
 * fw_grid (the GRID framework model, with the system's grids set): the
 * framework VDW energy of a bead is its atom's energy-grid value and the
 * framework real-space charge energy its charge times the Coulomb-grid value
 * (zero without a Coulomb grid: an uncharged molecule), with no framework
 * pairs, as CalculateFrameworkVDWEnergyAtPosition and
 * CalculateFrameworkChargeEnergyAtPosition do when the model is GRID
 * (src/framework_energy.c:73-77, :195-198) and the move differences
 * (:4893-4894, :5437-5438). A grid value sets no overlap flag: the
 * reference's grid branches set none. */
template <int MIXED>
__global__ void __launch_bounds__(256) k_point_energies(const RgpuSys *sysp, const void *ads, int nads,
                                                        const double *xyz, const int *atom, const int *excl, int P,
                                                        int pair_check, int fw_grid, double *out, int *ov)
{
  __shared__ RgpuSys S;
  __shared__ CallSmem sm;
  load_sys(&S, sysp);
  for (int p = threadIdx.x; p < P; p += blockDim.x) bead_set(sm.pos[p], S, xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2], atom[p], excl[p]);
  if (threadIdx.x == 0) sm.next = 0;
  __syncthreads();
  EvalScratch sc = {sm.uv, sm.uc, sm.uo, &sm.next, nullptr, sm.qr2, sm.qq, sm.qt};
  EvalSlice sl;
  sl.fw = MIXED ? (const void *)S.fw32 : (const void *)S.fw64;
  sl.tiles = S.tiles;
  sl.fw_lo = 0;
  sl.fw_hi = (fw_grid && S.use_grid) ? 0 : (MIXED ? S.ntile : S.nfw);
  sl.ads = ads;
  sl.ads_lo = 0;
  sl.ads_hi = nads;
  eval_positions<MIXED>(S, sl, sm.pos, P, pair_check, sm.res, sm.ovf, sc, RGPU_MAX_UNITS);
  if (fw_grid && S.use_grid) {
    /* 8 lanes per lookup, 4 positions per warp pass (every lane takes part) */
    const int lane = threadIdx.x & 31;
    for (int base = (threadIdx.x >> 5) * 4; base < P; base += (blockDim.x >> 5) * 4) {
      const int p = base + (lane >> 3);
      const bool live = p < P;
      const int a = live ? atom[p] : 0;
      const double x[3] = {live ? xyz[3 * p] : 0.0, live ? xyz[3 * p + 1] : 0.0, live ? xyz[3 * p + 2] : 0.0};
      const double g = rgpu_grid_value8(S.grid[a], S.grid_geom, x, lane & 7, live);
      double gq = 0.0;
      if (S.use_coul_grid) {
        const double q = S.mol_q[a];
        gq = q * rgpu_grid_value8(S.coul_grid, S.coul_geom, x, lane & 7, live && q != 0.0, false);
      }
      if (live && (lane & 7) == 0) {
        sm.res[p][0] = g;
        sm.res[p][1] = gq;
      }
    }
    __syncthreads();
  }
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    for (int k = 0; k < 4; k++) out[4 * p + k] = sm.res[p][k];
    if (ov) ov[p] = sm.ovf[p];
  }
}

cudaError_t rgpu_point_energies_launch(int mixed, const RgpuSys *d_sys, const void *d_ads, int nads,
                                       const double *d_xyz, const int *d_atom, const int *d_excl, int P,
                                       int pair_check, int fw_grid, double *d_out, int *d_ov, cudaStream_t st)
{
  if (P > RGPU_MAX_POS) return cudaErrorInvalidValue;
  if (mixed)
    k_point_energies<true><<<1, 256, 0, st>>>(d_sys, d_ads, nads, d_xyz, d_atom, d_excl, P, pair_check, fw_grid,
                                              d_out, d_ov);
  else
    k_point_energies<false><<<1, 256, 0, st>>>(d_sys, d_ads, nads, d_xyz, d_atom, d_excl, P, pair_check, fw_grid,
                                               d_out, d_ov);
  return cudaGetLastError();
}

/* Ewald Fourier difference of ns signed sites (FP64 xyz + charges), writing
 * dS(k) of the candidate into d_ds (for a later accept) and {e_ads, e_host}. */
template <int MIXED>
__global__ void __launch_bounds__(256) k_ewald_delta(const RgpuSys *sysp, const double *xyz, const double *q, int ns,
                                                     double2 *d_ds, double *out, int kw)
{
  __shared__ RgpuSys S;
  __shared__ EwSite sites[2 * RGPU_MAX_ATOMS];
  /* phase tables of the FP64 path; the mixed path forms its phases directly */
  __shared__ typename PhaseT<MIXED>::T tab[MIXED == 1 ? 1 : 2 * RGPU_MAX_ATOMS * 3 * 41];
  __shared__ double red[72];
  load_sys(&S, sysp);
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    bead_set(sites[s].b, S, xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2], 0, -1);
    sites[s].q = q[s];
  }
  __syncthreads();
  ewald_phases<MIXED>(S, sites, ns, tab, kw);
  __syncthreads();
  double ea = 0.0, eh = 0.0;
  for (int k = threadIdx.x; k < S.nk; k += blockDim.x) {
    double2 d = ewald_dS<MIXED>(tab, kw, sites, ns, S.kvec[k]);
    double2 so = S.sk_ads[k];
    double2 sf = S.sk_fw[k];
    double kf = S.kfactor[k];
    ea += kf * (2.0 * (so.x * d.x + so.y * d.y) + d.x * d.x + d.y * d.y);
    eh += kf * (sf.x * d.x + sf.y * d.y);
    if (d_ds) d_ds[k] = d;
  }
  block_sum2(ea, eh, red);
  if (threadIdx.x == 0) { out[0] = ea; out[1] = eh; }
}

__global__ void k_ewald_accept(const RgpuSys *sysp, const double2 *d_ds)
{
  const RgpuSys *S = sysp;
  int nk = S->nk;
  double2 *sk = S->sk_ads;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    double2 a = sk[k], d = d_ds[k];
    sk[k] = make_double2(a.x + d.x, a.y + d.y);
  }
}

cudaError_t rgpu_ewald_delta_launch(int mixed, const RgpuSys *d_sys, const double *d_xyz, const double *d_q, int ns,
                                    double2 *d_ds, double *d_out, int kw, cudaStream_t st)
{
  if (ns > 2 * RGPU_MAX_ATOMS || kw > 41) return cudaErrorInvalidValue;
  if (mixed) k_ewald_delta<true><<<1, 256, 0, st>>>(d_sys, d_xyz, d_q, ns, d_ds, d_out, kw);
  else k_ewald_delta<false><<<1, 256, 0, st>>>(d_sys, d_xyz, d_q, ns, d_ds, d_out, kw);
  return cudaGetLastError();
}

cudaError_t rgpu_ewald_accept_launch(const RgpuSys *d_sys, const double2 *d_ds, int nk, cudaStream_t st)
{
  int blocks = (nk + 255) / 256;
  if (blocks < 1) blocks = 1;
  k_ewald_accept<<<blocks, 256, 0, st>>>(d_sys, d_ds);
  return cudaGetLastError();
}

/* S(k) = sum_i q_i exp(i k.r_i) over n sites (FP64), one thread per k */
__global__ void k_structure_factor(const RgpuSys *sysp, const double *xyz, const double *q, int n, double2 *sk)
{
  const RgpuSys *S = sysp;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S->nk) return;
  char4 kv = S->kvec[k];
  double re = 0.0, im = 0.0;
  for (int i = 0; i < n; i++) {
    const double *x = xyz + 3 * i;
    double a;
    if (!S->triclinic)
      a = 2.0 * (kv.x * x[0] * S->inv_box[0] + kv.y * x[1] * S->inv_box[1] + kv.z * x[2] * S->inv_box[2]);
    else
      a = 2.0 * (kv.x * rgpu_frac(*S, 0, x[0], x[1], x[2]) + kv.y * rgpu_frac(*S, 1, x[0], x[1], x[2]) +
                 kv.z * rgpu_frac(*S, 2, x[0], x[1], x[2]));
    double sn, cs;
    sincospi(a, &sn, &cs);
    re += q[i] * cs;
    im += q[i] * sn;
  }
  sk[k] = make_double2(re, im);
}

cudaError_t rgpu_structure_factor_launch(const RgpuSys *d_sys, const double *d_xyz, const double *d_q, int n,
                                         int nk, double2 *d_sk, cudaStream_t st)
{
  int blocks = (nk + 127) / 128;
  if (blocks < 1) blocks = 1;
  k_structure_factor<<<blocks, 128, 0, st>>>(d_sys, d_xyz, d_q, n, d_sk);
  return cudaGetLastError();
}

/* Batched state transfer of an engine's systems through one staging buffer:
 * system i's region starts at off[i] (8-byte aligned) and holds its state
 * block (RgpuState; for an upload only its nmol field is read), then
 * nmol * natom positions (FP64 xyz). One block per system. */
__global__ void k_gather_states(const RgpuSys *systems, const unsigned long long *off, unsigned char *buf)
{
  const RgpuSys &S = systems[blockIdx.x];
  unsigned char *dst = buf + off[blockIdx.x];
  const RgpuState *st = (const RgpuState *)S.energy;   /* energy is the first field of the block */
  const unsigned long long *src8 = (const unsigned long long *)st;
  unsigned long long *dst8 = (unsigned long long *)dst;
  for (int i = threadIdx.x; i < (int)(sizeof(RgpuState) / 8); i += blockDim.x) dst8[i] = src8[i];
  const int n = st->nmol * S.natom * 3;
  double *xd = (double *)(dst + sizeof(RgpuState));
  for (int i = threadIdx.x; i < n; i += blockDim.x) xd[i] = S.ads_xyz[i];
}

__global__ void k_scatter_positions(const RgpuSys *systems, const unsigned long long *off, const unsigned char *buf)
{
  const RgpuSys &S = systems[blockIdx.x];
  const unsigned char *src = buf + off[blockIdx.x];
  const int nmol = ((const RgpuState *)src)->nmol;
  const double *xs = (const double *)(src + sizeof(RgpuState));
  for (int i = threadIdx.x; i < nmol * S.natom * 3; i += blockDim.x) S.ads_xyz[i] = xs[i];
  if (threadIdx.x == 0) *S.nmol = nmol;
}

/* S_ads(k) of every system of an engine from its positions (the batched
 * upload): block (x, y) = wave vectors x*128.. of system y; the same sum, in
 * the same order, as k_structure_factor with the molecule's charges. */
__global__ void k_upload_sk(const RgpuSys *systems)
{
  const RgpuSys &S = systems[blockIdx.y];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= S.nk) return;
  const int n = *S.nmol * S.natom;
  const char4 kv = S.kvec[k];
  double re = 0.0, im = 0.0;
  for (int i = 0; i < n; i++) {
    const double *x = S.ads_xyz + 3 * i;
    const double q = S.mol_q[i % S.natom];
    double a;
    if (!S.triclinic)
      a = 2.0 * (kv.x * x[0] * S.inv_box[0] + kv.y * x[1] * S.inv_box[1] + kv.z * x[2] * S.inv_box[2]);
    else
      a = 2.0 * (kv.x * rgpu_frac(S, 0, x[0], x[1], x[2]) + kv.y * rgpu_frac(S, 1, x[0], x[1], x[2]) +
                 kv.z * rgpu_frac(S, 2, x[0], x[1], x[2]));
    double sn, cs;
    sincospi(a, &sn, &cs);
    re += q * cs;
    im += q * sn;
  }
  S.sk_ads[k] = make_double2(re, im);
}

cudaError_t rgpu_upload_sk_launch(const RgpuSys *d_systems, int n, int max_nk, cudaStream_t st)
{
  if (n <= 0 || max_nk <= 0) return cudaSuccess;
  k_upload_sk<<<dim3((unsigned)((max_nk + 127) / 128), (unsigned)n), 128, 0, st>>>(d_systems);
  return cudaGetLastError();
}

cudaError_t rgpu_gather_states_launch(const RgpuSys *d_systems, int n, const unsigned long long *d_off,
                                      unsigned char *d_buf, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_gather_states<<<n, 256, 0, st>>>(d_systems, d_off, d_buf);
  return cudaGetLastError();
}

cudaError_t rgpu_scatter_positions_launch(const RgpuSys *d_systems, int n, const unsigned long long *d_off,
                                          const unsigned char *d_buf, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_scatter_positions<<<n, 256, 0, st>>>(d_systems, d_off, d_buf);
  return cudaGetLastError();
}

/* adsorbate records (fixed-point and FP64) from the authoritative positions */
__global__ void k_build_records(const RgpuSys *sysp, int nads, int4 *rec32, AdsRec64 *rec64)
{
  const RgpuSys *S = sysp;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nads) return;
  const int m = i / S->natom, a = i - m * S->natom;
  const double x = S->ads_xyz[3 * i], y = S->ads_xyz[3 * i + 1], z = S->ads_xyz[3 * i + 2];
  int xi, yi, zi;
  rgpu_fix3(*S, x, y, z, xi, yi, zi);
  rec32[i] = make_int4(xi, yi, zi, m * 16 + a);
  AdsRec64 r;
  r.x = x; r.y = y; r.z = z; r.tag = m * 16 + a;
  rec64[i] = r;
}

cudaError_t rgpu_records_launch(const RgpuSys *d_sys, int nads, int4 *d_rec32, void *d_rec64, cudaStream_t st)
{
  if (nads <= 0) return cudaSuccess;
  k_build_records<<<(nads + 127) / 128, 128, 0, st>>>(d_sys, nads, d_rec32, (AdsRec64 *)d_rec64);
  return cudaGetLastError();
}
