/* C ABI of libraspa_gpu (include/raspa_gpu.h).
 *
 * Host side of the drop-in boundary: builds the device image of a system
 * (framework sorted by pseudo-atom type, force-field tables resolved for the
 * adsorbate, k-vectors and Ewald prefactors), keeps the adsorbate state on the
 * device, and forwards each reference-named operation to the kernels. No
 * function exits the process; errors are returned as codes.
 */
#include <cuda_runtime.h>
#include <errno.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <string>
#include <mutex>
#include <vector>

#include "../../include/raspa_gpu.h"
#include "rgpu_engine.h"
#include "rgpu_chain.h"
#include "rgpu_device.cuh"
#include "rgpu_types.h"

static thread_local char g_err[512];

static int fail(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(RGPU_E_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char *rgpu_error_string(int code)
{
  if (code == RGPU_SUCCESS) return "success";
  return g_err[0] ? g_err : "unknown error";
}

extern "C" int rgpu_device_count(void)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

struct rgpu_system {
  rgpu_system_desc d;         /* pointer members are not kept */
  RgpuSys h;                  /* host image of the descriptor */
  RgpuSys *d_sys;
  cudaStream_t st;
  int kw;
  /* device buffers */
  double4 *fw64;
  int4 *fw32;
  TileRec *tiles_d;
  char4 *kvec;
  double *kfactor;
  double2 *sk_fw, *sk_ads, *ds;
  double *ads_xyz;
  RgpuState *state;           /* one block; the pointers below point into it */
  int *nmol;
  double *energy;
  unsigned long long *step;
  long long *counters;
  double *sums;
  int *status;
  int4 *rec32;
  void *rec64;
  /* per-call scratch */
  double *io_xyz, *io_out, *io_q;
  int *io_atom, *io_excl, *io_ov;
  /* host mirrors */
  RgpuState h_state;          /* initial state at creation; last state read */
  std::vector<double> h_xyz;  /* [nmol*natom*3] */
  int h_nmol;
  int records_stale;          /* device records must be rebuilt from ads_xyz */
  double net_ads, pending_dq;
  int grid_type_seg;
  int fw_model;               /* RGPU_FRAMEWORK_FULL or _GRID: the per-call energies' framework terms */
  double *d_uc;               /* triclinic box: unit-cell matrices of the VDW and Coulomb grids, 2 x 18 doubles */
  uint64_t fingerprint;       /* of the model a checkpoint must match (checkpoint_fingerprint) */
  std::vector<int> fw_seg_type; /* framework pseudo-atom type of each segment */
  std::vector<double> lj_eps, lj_sig2, lj_shift;
  int ntypes;
};

struct rgpu_engine {
  std::vector<rgpu_system *> sys;
  RgpuSys *d_systems;
  int mixed, threads, kw, max_ads, cluster, fw_items, tile_items, k_items;
  bool wide;                  /* 64-register build of the mixed kernel */
  bool flex;                  /* build with flexible-chain moves and energy grids */
  size_t smem;
  cudaStream_t st;
  /* CUDA graph of one launch, replayed by rgpu_engine_run when enabled */
  int use_graph;
  cudaGraphExec_t gexec;
  long long g_nsteps;
  /* staging of the batched state transfer (allocated at first use):
   * system i's region at off[i], sized for its maxmol */
  std::vector<unsigned long long> off;
  size_t stage_bytes;
  unsigned long long *d_off;
  unsigned char *d_stage;
  unsigned char *h_stage;     /* pinned */
  /* device slot j of d_systems (and of d_off) holds system order[j]. Slots
   * [0, n - nsplit) run in one launch at `cluster`; the last nsplit slots in
   * a second launch at cluster_b on st_b, side by side with the first
   * (rgpu_engine_set_split). */
  std::vector<int> order;
  /* rgpu_engine_replace_system: pinned copies of the slot descriptors and
   * the event of each slot's last copy */
  RgpuSys *h_slots;
  std::vector<cudaEvent_t> slot_ev;
  int smem_max;
  int nsplit, cluster_b, fw_items_b, tile_items_b, k_items_b;
  size_t smem_b;
  cudaStream_t st_b;
  cudaEvent_t ev_fork, ev_join;
};

/* Launch parameters of the systems in device slots [lo, hi) at a cluster
 * size: each CTA's share of the framework (tiles) and of the wave vectors,
 * staged in shared memory as far as it fits, in order of preference:
 * framework share and wave vectors, framework only, wave vectors only,
 * neither. Returns false when not even the adsorbates fit. */
struct EngineGroup {
  int fw_items, tile_items, k_items;
  size_t smem;
};

static bool plan_group(const rgpu_engine *e, int lo, int hi, int cluster, EngineGroup &g)
{
  int maxfw = 0, maxtile = 0, maxk = 0;
  bool all_grids = true;
  for (int j = lo; j < hi; j++) {
    const rgpu_system *s = e->sys[e->order[j]];
    all_grids = all_grids && s->h.use_grid;
    maxfw = std::max(maxfw, (s->d.nfw + cluster - 1) / cluster);
    maxtile = std::max(maxtile, (s->h.ntile + cluster - 1) / cluster);
    if (s->h.ewald) maxk = std::max(maxk, (s->h.nk + cluster - 1) / cluster);
  }
  int fw = e->mixed ? maxtile * RGPU_TILE : maxfw, tiles = e->mixed ? maxtile : 0;
  if (all_grids) {
    /* no framework pairs are evaluated: nothing of the framework to stage */
    fw = 0;
    tiles = 0;
  }
  const int fw_try[4] = {fw, fw, 0, 0}, tile_try[4] = {tiles, tiles, 0, 0}, k_try[4] = {maxk, 0, maxk, 0};
  for (int t = 0; t < 4; t++) {
    const size_t b = rgpu_engine_smem_bytes(e->mixed, fw_try[t], tile_try[t], e->max_ads, e->kw, k_try[t],
                                            e->threads, e->flex);
    if (b <= (size_t)e->smem_max) {
      g.fw_items = fw_try[t];
      g.tile_items = tile_try[t];
      g.k_items = k_try[t];
      g.smem = b;
      return true;
    }
  }
  return false;
}

static void sys_free(rgpu_system *s)
{
  if (!s) return;
  void *ptrs[] = {s->d_uc, s->d_sys, s->fw64, s->fw32, s->tiles_d, s->kvec, s->kfactor, s->sk_fw, s->sk_ads, s->ds, s->ads_xyz,
                  s->state, s->rec32, s->rec64, s->io_xyz,
                  s->io_out, s->io_q, s->io_atom, s->io_excl, s->io_ov};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

extern "C" int rgpu_system_destroy(rgpu_system *sys)
{
  sys_free(sys);
  return RGPU_SUCCESS;
}

/* a triclinic description: any element of cell_matrix set */
static bool desc_triclinic(const rgpu_system_desc *d)
{
  for (int i = 0; i < 9; i++)
    if (d->cell_matrix[i] != 0.0) return true;
  return false;
}

/* inverse of the upper-triangular box matrix m (row-major) */
static void inverse_upper(const double *m, double *v)
{
  const double ax = m[0], bx = m[1], cx = m[2], by = m[4], cy = m[5], cz = m[8];
  for (int i = 0; i < 9; i++) v[i] = 0.0;
  v[0] = 1.0 / ax;
  v[1] = -bx / (ax * by);
  v[2] = (bx * cy - by * cx) / (ax * by * cz);
  v[4] = 1.0 / by;
  v[5] = -cy / (by * cz);
  v[8] = 1.0 / cz;
}

/* perpendicular widths of the box: volume over the area of each pair of cell vectors */
static void perpendicular_widths(const double *m, double *w)
{
  const double a[3] = {m[0], m[3], m[6]}, b[3] = {m[1], m[4], m[7]}, c[3] = {m[2], m[5], m[8]};
  auto cross_norm = [](const double *u, const double *v) {
    const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    return sqrt(x * x + y * y + z * z);
  };
  const double vol = m[0] * m[4] * m[8];
  w[0] = vol / cross_norm(b, c);
  w[1] = vol / cross_norm(c, a);
  w[2] = vol / cross_norm(a, b);
}

/* k-vector list of src/ewald.c:224-259 and the prefactor of :584-591
 * (triclinic: k = 2 pi H^-T n, :560-575) */
static void kvectors(const rgpu_system_desc *d, std::vector<char4> &kv, std::vector<double> &kf)
{
  const int kx = d->kmax[0], ky = d->kmax[1], kz = d->kmax[2];
  const int km = std::max(kx, std::max(ky, kz));
  const double rc = (1.05 * km) * (1.05 * km);
  const bool tri = desc_triclinic(d);
  double hinv[9];
  if (tri) inverse_upper(d->cell_matrix, hinv);
  const double vol = tri ? d->cell_matrix[0] * d->cell_matrix[4] * d->cell_matrix[8] : d->box[0] * d->box[1] * d->box[2];
  for (int i = 0; i <= kx; i++)
    for (int j = -ky; j <= ky; j++)
      for (int k = -kz; k <= kz; k++) {
        int s = i * i + j * j + k * k;
        if (s == 0 || !(s < rc)) continue;
        kv.push_back(make_char4((signed char)i, (signed char)j, (signed char)k, 0));
        double rx, ry, rz;
        if (!tri) {
          rx = 2.0 * M_PI * i / d->box[0], ry = 2.0 * M_PI * j / d->box[1], rz = 2.0 * M_PI * k / d->box[2];
        } else {
          rx = 2.0 * M_PI * (i * hinv[0] + j * hinv[3] + k * hinv[6]);
          ry = 2.0 * M_PI * (i * hinv[1] + j * hinv[4] + k * hinv[7]);
          rz = 2.0 * M_PI * (i * hinv[2] + j * hinv[5] + k * hinv[8]);
        }
        double k2 = rx * rx + ry * ry + rz * rz;
        double pre = (i == 0 ? 2.0 : 4.0) * M_PI / vol;
        kf.push_back(d->coulomb * pre * exp((-0.25 / (d->alpha * d->alpha)) * k2) / k2);
      }
}

static int upload_records(rgpu_system *s)
{
  const int nads = s->h_nmol * s->d.natom;
  CK(rgpu_records_launch(s->d_sys, nads, s->rec32, s->rec64, s->st));
  s->records_stale = 0;
  return RGPU_SUCCESS;
}

/* pulls positions and molecule count back after the engine moved them */
static int refresh_from_device(rgpu_system *s)
{
  if (!s->records_stale) return RGPU_SUCCESS;
  int n = 0;
  CK(cudaMemcpyAsync(&n, s->nmol, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  s->h_nmol = n;
  s->h_xyz.assign((size_t)n * s->d.natom * 3, 0.0);
  if (n)
    CK(cudaMemcpyAsync(s->h_xyz.data(), s->ads_xyz, sizeof(double) * s->h_xyz.size(), cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  s->net_ads = n * s->h.mol_charge;
  return upload_records(s);
}

/* FNV-1a over the parts of a descriptor that a saved state depends on: the
 * box, the framework, the force field, the molecule and the Ewald set-up.
 * Temperature, pressure, move mix and random stream may differ between the
 * system that saved a checkpoint and the one restoring it. */
static uint64_t fnv1a(uint64_t h, const void *p, size_t n)
{
  const unsigned char *b = (const unsigned char *)p;
  for (size_t i = 0; i < n; i++) {
    h ^= b[i];
    h *= 1099511628211ULL;
  }
  return h;
}

static uint64_t checkpoint_fingerprint(const rgpu_system_desc *d)
{
  uint64_t h = 1469598103934665603ULL;
  h = fnv1a(h, d->box, sizeof d->box);
  h = fnv1a(h, &d->cutoff, sizeof d->cutoff);
  h = fnv1a(h, &d->nfw, sizeof d->nfw);
  h = fnv1a(h, d->fw_xyz, sizeof(double) * 3 * d->nfw);
  h = fnv1a(h, d->fw_type, sizeof(int) * d->nfw);
  h = fnv1a(h, d->fw_q, sizeof(double) * d->nfw);
  h = fnv1a(h, &d->ntypes, sizeof d->ntypes);
  h = fnv1a(h, d->eps, sizeof(double) * d->ntypes * d->ntypes);
  h = fnv1a(h, d->sig2, sizeof(double) * d->ntypes * d->ntypes);
  h = fnv1a(h, d->shift, sizeof(double) * d->ntypes * d->ntypes);
  h = fnv1a(h, &d->natom, sizeof d->natom);
  h = fnv1a(h, d->mol_type, sizeof(int) * d->natom);
  h = fnv1a(h, d->mol_q, sizeof(double) * d->natom);
  h = fnv1a(h, d->mol_ref, sizeof(double) * 3 * d->natom);
  h = fnv1a(h, &d->ewald, sizeof d->ewald);
  if (d->ewald) {
    h = fnv1a(h, &d->alpha, sizeof d->alpha);
    h = fnv1a(h, d->kmax, sizeof d->kmax);
  }
  if (desc_triclinic(d)) h = fnv1a(h, d->cell_matrix, sizeof d->cell_matrix);
  h = fnv1a(h, &d->flexible, sizeof d->flexible);
  if (d->flexible) {
    h = fnv1a(h, &d->bond, sizeof d->bond);
    h = fnv1a(h, &d->bend_k, sizeof d->bend_k);
    h = fnv1a(h, &d->bend_theta0, sizeof d->bend_theta0);
    h = fnv1a(h, d->torsion, sizeof d->torsion);
  }
  return h;
}

extern "C" int rgpu_system_create(rgpu_system **out, const rgpu_system_desc *d)
{
  if (!out || !d) return fail(RGPU_E_INVALID, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RGPU_E_NODEVICE, "no CUDA device");
  if (d->natom < 1 || d->natom > RGPU_MAX_ATOMS) return fail(RGPU_E_INVALID, "natom %d outside [1,%d]", d->natom, RGPU_MAX_ATOMS);
  if (d->nfw < 1 || !d->fw_xyz || !d->fw_type || !d->fw_q) return fail(RGPU_E_INVALID, "framework missing");
  if (d->nfw > (1 << 24)) return fail(RGPU_E_INVALID, "nfw %d above 2^24", d->nfw);
  if (d->ntypes < 1 || !d->eps || !d->sig2 || !d->shift) return fail(RGPU_E_INVALID, "LJ table missing");
  if (!d->mol_type || !d->mol_q || !d->mol_ref) return fail(RGPU_E_INVALID, "molecule missing");
  if (d->start_bead < 0 || d->start_bead >= d->natom) return fail(RGPU_E_INVALID, "start_bead");
  if (d->flexible) {
    if (d->start_bead != 0) return fail(RGPU_E_INVALID, "a flexible chain is grown from atom 0 (start_bead 0)");
    if (!(d->bond > 0.0)) return fail(RGPU_E_INVALID, "flexible chain: bond length must be positive");
    if (d->natom > 1 && !(d->bend_k > 0.0)) return fail(RGPU_E_INVALID, "flexible chain: bend_k must be positive");
    for (int a = 0; a < d->natom; a++)
      if (d->mol_q[a] != 0.0) return fail(RGPU_E_INVALID, "flexible chains must be uncharged");
    if (d->chain_scheme != 0 && d->chain_scheme != 1) return fail(RGPU_E_INVALID, "chain_scheme must be 0 or 1");
    if (d->ntors < 0 || d->ntors > RGPU_MAX_TORS)
      return fail(RGPU_E_INVALID, "ntors must be in [0,%d] (0: 100)", RGPU_MAX_TORS);
  }
  if (d->maxmol < 1 || (long long)d->maxmol * d->natom > (1 << 20)) return fail(RGPU_E_INVALID, "maxmol");
  if (d->ntrial_first < 1 || d->ntrial_first > RGPU_MAX_TRIALS || d->ntrial < 1 || d->ntrial > RGPU_MAX_TRIALS)
    return fail(RGPU_E_INVALID, "trial counts must be in [1,%d]", RGPU_MAX_TRIALS);
  if (!d->flexible && d->ntrial * (d->natom - 1) > RGPU_MAX_POS)
    return fail(RGPU_E_INVALID, "ntrial*(natom-1) > %d", RGPU_MAX_POS);
  if (desc_triclinic(d)) {
    const double *m = d->cell_matrix;
    if (m[3] != 0.0 || m[6] != 0.0 || m[7] != 0.0 || !(m[0] > 0.0) || !(m[4] > 0.0) || !(m[8] > 0.0))
      return fail(RGPU_E_INVALID, "cell_matrix must be upper triangular with a positive diagonal");
    double w[3];
    perpendicular_widths(m, w);
    for (int c = 0; c < 3; c++)
      if (!(w[c] >= 2.0 * d->cutoff)) return fail(RGPU_E_INVALID, "perpendicular width %g < 2*cutoff", w[c]);
  } else {
    for (int c = 0; c < 3; c++)
      if (!(d->box[c] >= 2.0 * d->cutoff)) return fail(RGPU_E_INVALID, "box length %g < 2*cutoff", d->box[c]);
  }
  if (d->ewald && (d->kmax[0] < 1 || d->kmax[1] < 1 || d->kmax[2] < 1 ||
                   std::max(d->kmax[0], std::max(d->kmax[1], d->kmax[2])) > 20))
    return fail(RGPU_E_INVALID, "kmax must be in [1,20]");
  for (int i = 0; i < d->nfw; i++)
    if (d->fw_type[i] < 0 || d->fw_type[i] >= d->ntypes) return fail(RGPU_E_INVALID, "framework type %d", d->fw_type[i]);
  for (int a = 0; a < d->natom; a++)
    if (d->mol_type[a] < 0 || d->mol_type[a] >= d->ntypes) return fail(RGPU_E_INVALID, "molecule type");

  rgpu_system *s = new rgpu_system();
  s->fingerprint = checkpoint_fingerprint(d);
  memset(&s->h, 0, sizeof(RgpuSys));
  memset(&s->h_state, 0, sizeof(RgpuState));
  s->h_state.step[1] = ~0ULL;   /* no step limit */
  s->d = *d;
  s->h_nmol = 0;
  s->records_stale = 0;
  s->net_ads = 0.0;
  s->pending_dq = 0.0;
  s->ntypes = d->ntypes;
  s->lj_eps.assign(d->eps, d->eps + d->ntypes * d->ntypes);
  s->lj_sig2.assign(d->sig2, d->sig2 + d->ntypes * d->ntypes);
  s->lj_shift.assign(d->shift, d->shift + d->ntypes * d->ntypes);
  RgpuSys &h = s->h;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    sys_free(s);
    return fail(RGPU_E_CUDA, "stream");
  }
  /* framework sorted by type into segments */
  std::vector<int> order(d->nfw);
  for (int i = 0; i < d->nfw; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d->fw_type[a] < d->fw_type[b]; });
  std::vector<double4> fw64(d->nfw);
  std::vector<int4> fw32(d->nfw);
  int nseg = 0;
  double netq = 0.0;
  int charged = 0;
  for (int idx = 0; idx < d->nfw; idx++) {
    const int i = order[idx];
    if (idx == 0 || d->fw_type[i] != d->fw_type[order[idx - 1]]) {
      if (nseg == RGPU_MAX_FWTYPES) {
        sys_free(s);
        return fail(RGPU_E_INVALID, "more than %d framework types", RGPU_MAX_FWTYPES);
      }
      h.seg_start[nseg] = idx;
      s->fw_seg_type.push_back(d->fw_type[i]);
      nseg++;
    }
    const double x = d->fw_xyz[3 * i], y = d->fw_xyz[3 * i + 1], z = d->fw_xyz[3 * i + 2], q = d->fw_q[i];
    fw64[idx] = make_double4(x, y, z, q);
    float qf = (float)q;
    int qb;
    memcpy(&qb, &qf, 4);
    fw32[idx] = make_int4(0, 0, 0, qb);
    netq += q;
    if (q != 0.0) charged = 1;
  }
  h.seg_start[nseg] = d->nfw;
  h.nseg = nseg;
  h.nfw = d->nfw;
  h.fw_charged = charged && d->ewald;
  for (int c = 0; c < 3; c++) {
    h.box[c] = d->box[c];
    h.inv_box[c] = 1.0 / d->box[c];
    h.fix_scale[c] = (float)(d->box[c] / 4294967296.0);
    h.kmax[c] = d->ewald ? d->kmax[c] : 0;
  }
  const bool tri = desc_triclinic(d);
  double wperp[3] = {d->box[0], d->box[1], d->box[2]};
  if (tri) {
    h.triclinic = 1;
    for (int i = 0; i < 9; i++) {
      h.hm[i] = d->cell_matrix[i];
      h.hmf[i] = (float)(d->cell_matrix[i] / 4294967296.0);
    }
    inverse_upper(h.hm, h.hinv);
    perpendicular_widths(h.hm, wperp);
    for (int c = 0; c < 3; c++) h.wperp[c] = (float)(wperp[c] * (1.0 - 1e-6));
  }
  /* Mixed-precision layout: fixed-point coordinates (see rgpu_types.h), the
   * framework cut into tiles of RGPU_TILE spatially close atoms with a bounding box
   * each, by recursive bisection: the atoms of a group are split at the
   * median of their longest extent (in the unwrapped cell [0, L)) into two
   * groups holding whole tiles, until a group is one tile. Compact tiles
   * make the box test reject most of the atoms outside the cut-off sphere.
   * The two low bits of the z coordinate carry the atom's segment
   * (pseudo-atom type), an offset of at most 3 * L / 2^32 (< 1e-8 A). */
  std::vector<TileRec> tiles;
  {
    std::vector<int> seg_of(d->nfw);
    std::vector<double> fr((size_t)d->nfw * 3);
    for (int idx = 0; idx < d->nfw; idx++) {
      int sgi = 0;
      while (sgi + 1 < nseg && idx >= h.seg_start[sgi + 1]) sgi++;
      seg_of[idx] = sgi;
      const double p[3] = {fw64[idx].x, fw64[idx].y, fw64[idx].z};
      for (int c = 0; c < 3; c++) {
        if (!tri) {
          double f = p[c] * h.inv_box[c];
          fr[3 * (size_t)idx + c] = (f - floor(f)) * d->box[c];
        } else {
          /* fractional coordinate in lengths of the perpendicular width */
          double f = rgpu_frac(h, c, p[0], p[1], p[2]);
          fr[3 * (size_t)idx + c] = (f - floor(f)) * wperp[c];
        }
      }
    }
    std::vector<int> sp(d->nfw);
    for (int i = 0; i < d->nfw; i++) sp[i] = i;
    /* iterative bisection over ranges [b, e) of sp */
    std::vector<std::pair<int, int>> todo{{0, d->nfw}};
    while (!todo.empty()) {
      const int b = todo.back().first, e = todo.back().second;
      todo.pop_back();
      const int n = e - b;
      if (n <= RGPU_TILE) continue;
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int i = b; i < e; i++)
        for (int c = 0; c < 3; c++) {
          lo[c] = std::min(lo[c], fr[3 * (size_t)sp[i] + c]);
          hi[c] = std::max(hi[c], fr[3 * (size_t)sp[i] + c]);
        }
      int ax = 0;
      for (int c = 1; c < 3; c++)
        if (hi[c] - lo[c] > hi[ax] - lo[ax]) ax = c;
      const int nt = (n + RGPU_TILE - 1) / RGPU_TILE;
      const int m = b + RGPU_TILE * (nt / 2);      /* the left group holds whole tiles */
      std::nth_element(sp.begin() + b, sp.begin() + m, sp.begin() + e, [&](int x, int y) {
        const double fx = fr[3 * (size_t)x + ax], fy = fr[3 * (size_t)y + ax];
        return fx < fy || (fx == fy && x < y);
      });
      todo.push_back({b, m});
      todo.push_back({m, e});
    }
    const int ntile = (d->nfw + RGPU_TILE - 1) / RGPU_TILE;
    /* Tiles are stored in bit-reversed order of their place in the
     * bisection, so that every contiguous range of 1/2^k of them (one CTA's
     * share of a cluster, one warp's chunk) samples the whole framework
     * evenly and carries about the same work for any bead position. */
    std::vector<int> order;
    {
      int bits = 0;
      while ((1 << bits) < ntile) bits++;
      for (int i = 0; i < (1 << bits); i++) {
        int r = 0;
        for (int k = 0; k < bits; k++) r |= ((i >> k) & 1) << (bits - 1 - k);
        if (r < ntile) order.push_back(r);
      }
    }
    fw32.assign((size_t)ntile * RGPU_TILE, make_int4(0, 0, 0, 0));
    tiles.resize(ntile);
    for (int o = 0; o < ntile && tri; o++) {
      /* triclinic tile: fractional extents about the first atom (each
       * offset wrapped to the nearest integer), the centre in fixed point,
       * h = fractional half extents, h.w = the Cartesian radius about the
       * centre */
      const int t = order[o];
      const int n = std::min(RGPU_TILE, d->nfw - RGPU_TILE * t);
      const double4 r0 = fw64[sp[RGPU_TILE * t]];
      double f0[3], lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      for (int c = 0; c < 3; c++) f0[c] = rgpu_frac(h, c, r0.x, r0.y, r0.z);
      double off[RGPU_TILE][3];
      for (int j = 0; j < n; j++) {
        const int idx = sp[RGPU_TILE * t + j];
        int v[3];
        rgpu_fix3(h, fw64[idx].x, fw64[idx].y, fw64[idx].z, v[0], v[1], v[2]);
        for (int c = 0; c < 3; c++) {
          double dd = rgpu_frac(h, c, fw64[idx].x, fw64[idx].y, fw64[idx].z) - f0[c];
          dd -= floor(dd + 0.5);
          off[j][c] = dd;
          lo[c] = std::min(lo[c], dd);
          hi[c] = std::max(hi[c], dd);
        }
        v[2] = (v[2] & ~3) | seg_of[idx];
        float qf = (float)fw64[idx].w;
        int qb;
        memcpy(&qb, &qf, 4);
        fw32[(size_t)RGPU_TILE * o + j] = make_int4(v[0], v[1], v[2], qb);
      }
      double cen[3], half[3], rad = 0.0;
      for (int c = 0; c < 3; c++) {
        cen[c] = 0.5 * (lo[c] + hi[c]);
        half[c] = 0.5 * (hi[c] - lo[c]);
      }
      for (int j = 0; j < n; j++) {
        const double u[3] = {off[j][0] - cen[0], off[j][1] - cen[1], off[j][2] - cen[2]};
        double r2 = 0.0;
        for (int r = 0; r < 3; r++) {
          const double x = h.hm[3 * r] * u[0] + h.hm[3 * r + 1] * u[1] + h.hm[3 * r + 2] * u[2];
          r2 += x * x;
        }
        rad = std::max(rad, sqrt(r2));
      }
      float hh[3];
      int cv[3];
      for (int c = 0; c < 3; c++) {
        /* margins for the fixed-point and FP32 rounding */
        hh[c] = half[c] >= 0.25 ? 0.5f : (float)(half[c] * (1.0 + 1e-6) + 1e-8);
        cv[c] = rgpu_fix_frac(f0[c] + cen[c]);
      }
      TileRec tr;
      tr.c = make_int4(cv[0], cv[1], cv[2], n);
      tr.h = make_float4(hh[0], hh[1], hh[2], (float)(rad * (1.0 + 1e-5) + 1e-3));
      tiles[o] = tr;
    }
    for (int o = 0; o < ntile && !tri; o++) {
      const int t = order[o];
      const int n = std::min(RGPU_TILE, d->nfw - RGPU_TILE * t);
      const double4 r0 = fw64[sp[RGPU_TILE * t]];
      double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      for (int j = 0; j < n; j++) {
        const int idx = sp[RGPU_TILE * t + j];
        const double p[3] = {fw64[idx].x, fw64[idx].y, fw64[idx].z};
        const double p0[3] = {r0.x, r0.y, r0.z};
        int v[3];
        for (int c = 0; c < 3; c++) {
          double f = p[c] * h.inv_box[c];
          f -= floor(f);
          long long q = llrint(f * 4294967296.0);
          v[c] = (int)(unsigned)(q & 0xffffffffLL);
          /* offset from the tile's first atom, minimum image */
          double dd = p[c] - p0[c];
          dd -= d->box[c] * floor(dd * h.inv_box[c] + 0.5);
          lo[c] = std::min(lo[c], dd);
          hi[c] = std::max(hi[c], dd);
        }
        v[2] = (v[2] & ~3) | seg_of[idx];
        float qf = (float)fw64[idx].w;
        int qb;
        memcpy(&qb, &qf, 4);
        fw32[(size_t)RGPU_TILE * o + j] = make_int4(v[0], v[1], v[2], qb);
      }
      TileRec tr;
      double cen[3];
      const double p0[3] = {r0.x, r0.y, r0.z};
      float hh[3];
      for (int c = 0; c < 3; c++) {
        cen[c] = p0[c] + 0.5 * (lo[c] + hi[c]);
        double half = 0.5 * (hi[c] - lo[c]);
        /* margin for the fixed-point rounding of centre and atoms */
        hh[c] = (float)(half * (1.0 + 1e-6) + 1e-5);
        if (half >= 0.25 * d->box[c]) hh[c] = (float)(0.5 * d->box[c]);   /* no culling along this axis */
      }
      int cv[3];
      for (int c = 0; c < 3; c++) {
        double f = cen[c] * h.inv_box[c];
        f -= floor(f);
        long long q = llrint(f * 4294967296.0);
        cv[c] = (int)(unsigned)(q & 0xffffffffLL);
      }
      tr.c = make_int4(cv[0], cv[1], cv[2], n);
      tr.h = make_float4(hh[0], hh[1], hh[2], 0.0f);
      tiles[o] = tr;
    }
    h.ntile = ntile;
  }
  h.rc2 = d->cutoff * d->cutoff;
  h.rc2f = (float)h.rc2;
  h.overlap = d->overlap;
  h.beta = d->beta;
  h.coulomb = d->coulomb;
  h.alpha = d->ewald ? d->alpha : 0.0;
  h.coulombf = (float)d->coulomb;
  h.alphaf = (float)h.alpha;
  h.natom = d->natom;
  h.start_bead = d->start_bead;
  h.maxmol = d->maxmol;
  int molq = 0;
  double mq = 0.0, self = 0.0;
  for (int a = 0; a < d->natom; a++) {
    h.mol_q[a] = d->ewald ? d->mol_q[a] : 0.0;
    h.mol_qf[a] = (float)h.mol_q[a];
    if (h.mol_q[a] != 0.0) molq = 1;
    mq += h.mol_q[a];
    self += d->coulomb * h.mol_q[a] * h.mol_q[a] * h.alpha / sqrt(M_PI);
    for (int c = 0; c < 3; c++) h.mol_ref[a][c] = d->mol_ref[3 * a + c];
    const int ta = d->mol_type[a];
    for (int sg = 0; sg < nseg; sg++) {
      const int tb = s->fw_seg_type[sg], ij = ta * d->ntypes + tb;
      h.lj_bf[a][sg].eps4 = 4.0 * d->eps[ij];
      h.lj_bf[a][sg].sig2 = d->sig2[ij];
      h.lj_bf[a][sg].shift = d->shift[ij];
      h.ljf_bf[a][sg].eps4 = (float)(4.0 * d->eps[ij]);
      h.ljf_bf[a][sg].sig2 = (float)d->sig2[ij];
      h.ljf_bf[a][sg].shift = (float)d->shift[ij];
    }
    for (int b = 0; b < d->natom; b++) {
      const int ij = ta * d->ntypes + d->mol_type[b];
      h.lj_bb[a][b].eps4 = 4.0 * d->eps[ij];
      h.lj_bb[a][b].sig2 = d->sig2[ij];
      h.lj_bb[a][b].shift = d->shift[ij];
      h.ljf_bb[a][b].eps4 = (float)(4.0 * d->eps[ij]);
      h.ljf_bb[a][b].sig2 = (float)d->sig2[ij];
      h.ljf_bb[a][b].shift = (float)d->shift[ij];
    }
  }
  h.mol_charged = molq;
  h.mol_charge = mq;
  h.self_mol = self;
  h.flexible = d->flexible;
  if (d->flexible) {
    h.bond = d->bond;
    h.bend_k = d->bend_k;
    h.bend_theta0 = d->bend_theta0;
    h.bend_sigma = d->bend_k > 0.0 ? 1.0 / sqrt(d->beta * d->bend_k) : 0.0;
    for (int c = 0; c < 4; c++) h.torsion[c] = d->torsion[c];
    /* minimum of the torsion energy (scale of the rejection in chain_trial),
     * on a fine grid less a margin so that exp(-beta (U - min)) <= 1 */
    double tmin = 1e300, tmax = -1e300;
    for (int g = 0; g <= 20000; g++) {
      const double e = chain_torsion_energy(h, cos(-M_PI + 2.0 * M_PI * g / 20000.0));
      tmin = std::min(tmin, e);
      tmax = std::max(tmax, e);
    }
    h.torsion_min = tmin - 1e-6 * (tmax - tmin) - 1e-12;
    h.chain_scheme = d->chain_scheme;
    /* NumberOfTrialPositionsTorsion defaults to 100 (src/input.c:349) */
    h.ntors = d->ntors > 0 ? d->ntors : 100;
  }
  /* the exclusion sum K qa qb erf(alpha r)/r over the molecule's charged
   * pairs (src/ewald.c:7312-7330) is a constant of a rigid molecule */
  h.excl_mol = 0.0;
  if (d->ewald)
    for (int a = 0; a < d->natom - 1; a++)
      for (int b = a + 1; b < d->natom; b++) {
        if (d->mol_q[a] == 0.0 || d->mol_q[b] == 0.0) continue;
        const double *ra = d->mol_ref + 3 * a, *rb = d->mol_ref + 3 * b;
        const double r = sqrt((ra[0] - rb[0]) * (ra[0] - rb[0]) + (ra[1] - rb[1]) * (ra[1] - rb[1]) +
                              (ra[2] - rb[2]) * (ra[2] - rb[2]));
        h.excl_mol += d->coulomb * d->mol_q[a] * d->mol_q[b] * erf(d->alpha * r) / r;
      }
  h.ewald = d->ewald;
  for (int c = 0; c < 6; c++) h.cum[c] = d->move_cum[c];
  h.max_translation = d->max_translation;
  h.max_rotation = d->max_rotation;
  h.fugacity_beta_v = d->fugacity_beta_v;
  h.ntrial_first = d->ntrial_first;
  h.ntrial = d->ntrial;
  h.seed = d->seed;
  h.sys_id = d->stream_id;
  h.net_fw = netq;

  std::vector<char4> kv;
  std::vector<double> kf;
  if (d->ewald) kvectors(d, kv, kf);
  h.nk = (int)kv.size();
  s->kw = 2 * std::max(h.kmax[0], std::max(h.kmax[1], h.kmax[2])) + 1;
  double uion = 0.0;
  for (double f : kf) uion += f;
  /* EwaldEnergyIon, src/ewald.c:615-724 */
  h.uion = d->ewald ? -(uion - d->coulomb * h.alpha / sqrt(M_PI)) : 0.0;

  const size_t nads = (size_t)d->maxmol * d->natom;
  const int nk1 = std::max(h.nk, 1);
#define ALLOC(p, n) \
  if (cudaMalloc((void **)&(p), (n)) != cudaSuccess) { sys_free(s); return fail(RGPU_E_CUDA, "cudaMalloc " #p); }
  ALLOC(s->d_sys, sizeof(RgpuSys));
  if (tri) ALLOC(s->d_uc, sizeof(double) * 36);
  ALLOC(s->fw64, sizeof(double4) * d->nfw);
  ALLOC(s->fw32, sizeof(int4) * RGPU_TILE * (size_t)h.ntile);
  ALLOC(s->tiles_d, sizeof(TileRec) * (size_t)h.ntile);
  ALLOC(s->kvec, sizeof(char4) * nk1);
  ALLOC(s->kfactor, sizeof(double) * nk1);
  ALLOC(s->sk_fw, sizeof(double2) * nk1);
  ALLOC(s->sk_ads, sizeof(double2) * nk1);
  ALLOC(s->ds, sizeof(double2) * nk1);
  ALLOC(s->ads_xyz, sizeof(double) * 3 * nads);
  ALLOC(s->state, sizeof(RgpuState));
  s->nmol = &s->state->nmol;
  s->energy = s->state->energy;
  s->step = s->state->step;
  s->counters = s->state->counters;
  s->sums = s->state->sums;
  s->status = &s->state->status;
  ALLOC(s->rec32, sizeof(int4) * nads);
  ALLOC(s->rec64, 32 * nads);
  const size_t io_n = std::max((size_t)RGPU_MAX_POS, std::max((size_t)d->nfw, nads));
  ALLOC(s->io_xyz, sizeof(double) * 3 * io_n);
  ALLOC(s->io_q, sizeof(double) * io_n);
  ALLOC(s->io_out, sizeof(double) * 4 * RGPU_MAX_POS);
  ALLOC(s->io_atom, sizeof(int) * RGPU_MAX_POS);
  ALLOC(s->io_excl, sizeof(int) * RGPU_MAX_POS);
  ALLOC(s->io_ov, sizeof(int) * RGPU_MAX_POS);
#undef ALLOC
  h.fw64 = s->fw64;
  h.fw32 = s->fw32;
  h.tiles = s->tiles_d;
  h.kvec = s->kvec;
  h.kfactor = s->kfactor;
  h.sk_fw = s->sk_fw;
  h.sk_ads = s->sk_ads;
  h.ads_xyz = s->ads_xyz;
  h.nmol = s->nmol;
  h.energy = s->energy;
  h.step = s->step;
  h.counters = s->counters;
  h.sums = s->sums;
  h.status = s->status;
  cudaStream_t st = s->st;
  int rc = RGPU_SUCCESS;
  do {
    if (cudaMemcpyAsync(s->fw64, fw64.data(), sizeof(double4) * d->nfw, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(s->fw32, fw32.data(), sizeof(int4) * RGPU_TILE * (size_t)h.ntile, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(s->tiles_d, tiles.data(), sizeof(TileRec) * (size_t)h.ntile, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(s->state, &s->h_state, sizeof(RgpuState), cudaMemcpyHostToDevice, st) ||
        cudaMemsetAsync(s->sk_ads, 0, sizeof(double2) * nk1, st) ||
        cudaMemsetAsync(s->sk_fw, 0, sizeof(double2) * nk1, st) ||
        cudaMemcpyAsync(s->d_sys, &h, sizeof(RgpuSys), cudaMemcpyHostToDevice, st)) {
      rc = fail(RGPU_E_CUDA, "upload");
      break;
    }
    if (h.nk) {
      if (cudaMemcpyAsync(s->kvec, kv.data(), sizeof(char4) * h.nk, cudaMemcpyHostToDevice, st) ||
          cudaMemcpyAsync(s->kfactor, kf.data(), sizeof(double) * h.nk, cudaMemcpyHostToDevice, st)) {
        rc = fail(RGPU_E_CUDA, "upload k");
        break;
      }
      /* S_fw(k) (PrecomputeFixedEwaldContributions, src/ewald.c:744) from the
       * framework in its original order */
      std::vector<double> q(d->fw_q, d->fw_q + d->nfw);
      if (cudaMemcpyAsync(s->io_xyz, d->fw_xyz, sizeof(double) * 3 * d->nfw, cudaMemcpyHostToDevice, st) ||
          cudaMemcpyAsync(s->io_q, q.data(), sizeof(double) * d->nfw, cudaMemcpyHostToDevice, st) ||
          rgpu_structure_factor_launch(s->d_sys, s->io_xyz, s->io_q, d->nfw, h.nk, s->sk_fw, st)) {
        rc = fail(RGPU_E_CUDA, "S_fw");
        break;
      }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(RGPU_E_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
  } while (0);
  if (rc) {
    sys_free(s);
    return rc;
  }
  *out = s;
  return RGPU_SUCCESS;
}

static int recompute_sk_ads(rgpu_system *s)
{
  const int nads = s->h_nmol * s->d.natom;
  if (!s->h.nk) return RGPU_SUCCESS;
  if (nads == 0) {
    CK(cudaMemsetAsync(s->sk_ads, 0, sizeof(double2) * s->h.nk, s->st));
    return RGPU_SUCCESS;
  }
  std::vector<double> q(nads);
  for (int i = 0; i < nads; i++) q[i] = s->h.mol_q[i % s->d.natom];
  CK(cudaMemcpyAsync(s->io_xyz, s->h_xyz.data(), sizeof(double) * 3 * nads, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->io_q, q.data(), sizeof(double) * nads, cudaMemcpyHostToDevice, s->st));
  CK(rgpu_structure_factor_launch(s->d_sys, s->io_xyz, s->io_q, nads, s->h.nk, s->sk_ads, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_set_adsorbates(rgpu_system *s, int nmol, const double *xyz)
{
  if (!s || nmol < 0 || (nmol > 0 && !xyz)) return fail(RGPU_E_INVALID, "bad argument");
  if (nmol > s->d.maxmol) return fail(RGPU_E_CAPACITY, "nmol %d > maxmol %d", nmol, s->d.maxmol);
  const size_t n = (size_t)nmol * s->d.natom * 3;
  s->h_xyz.assign(xyz, xyz + n);
  s->h_nmol = nmol;
  if (n) CK(cudaMemcpyAsync(s->ads_xyz, s->h_xyz.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->nmol, &s->h_nmol, sizeof(int), cudaMemcpyHostToDevice, s->st));
  s->net_ads = nmol * s->h.mol_charge;
  s->pending_dq = 0.0;
  int rc = upload_records(s);
  if (rc) return rc;
  rc = recompute_sk_ads(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_get_adsorbates(rgpu_system *s, int *nmol, double *xyz, int capacity)
{
  if (!s || !nmol) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  *nmol = s->h_nmol;
  if (xyz) {
    if (capacity < s->h_nmol) return fail(RGPU_E_CAPACITY, "capacity %d < nmol %d", capacity, s->h_nmol);
    memcpy(xyz, s->h_xyz.data(), sizeof(double) * s->h_xyz.size());
  }
  return RGPU_SUCCESS;
}

static int write_molecule(rgpu_system *s, int m, const double *xyz)
{
  const int na = s->d.natom;
  memcpy(&s->h_xyz[(size_t)m * na * 3], xyz, sizeof(double) * 3 * na);
  CK(cudaMemcpyAsync(s->ads_xyz + (size_t)m * na * 3, &s->h_xyz[(size_t)m * na * 3], sizeof(double) * 3 * na,
                     cudaMemcpyHostToDevice, s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_update_molecule(rgpu_system *s, int m, const double *xyz)
{
  if (!s || !xyz) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  if (m < 0 || m >= s->h_nmol) return fail(RGPU_E_INVALID, "molecule %d", m);
  rc = write_molecule(s, m, xyz);
  if (rc) return rc;
  return upload_records(s);
}

extern "C" int rgpu_insert_molecule(rgpu_system *s, const double *xyz)
{
  if (!s || !xyz) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  if (s->h_nmol >= s->d.maxmol) return fail(RGPU_E_CAPACITY, "maxmol %d reached", s->d.maxmol);
  s->h_xyz.resize((size_t)(s->h_nmol + 1) * s->d.natom * 3);
  rc = write_molecule(s, s->h_nmol, xyz);
  if (rc) return rc;
  s->h_nmol++;
  CK(cudaMemcpyAsync(s->nmol, &s->h_nmol, sizeof(int), cudaMemcpyHostToDevice, s->st));
  rc = upload_records(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_remove_molecule(rgpu_system *s, int m)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  if (m < 0 || m >= s->h_nmol) return fail(RGPU_E_INVALID, "molecule %d", m);
  const int na = s->d.natom, last = s->h_nmol - 1;
  if (m != last) {
    std::vector<double> tmp(&s->h_xyz[(size_t)last * na * 3], &s->h_xyz[(size_t)last * na * 3] + 3 * na);
    rc = write_molecule(s, m, tmp.data());
    if (rc) return rc;
  }
  s->h_nmol--;
  s->h_xyz.resize((size_t)s->h_nmol * na * 3);
  CK(cudaMemcpyAsync(s->nmol, &s->h_nmol, sizeof(int), cudaMemcpyHostToDevice, s->st));
  rc = upload_records(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

/* ---------------------------------------------------------------------- */
static int bead_batch(rgpu_system *s, int precision, int n, const double *xyz, const int *atom, const int *excl,
                      int pair_check, double *out, int *ov)
{
  CK(cudaMemcpyAsync(s->io_xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->io_atom, atom, sizeof(int) * n, cudaMemcpyHostToDevice, s->st));
  CK(cudaMemcpyAsync(s->io_excl, excl, sizeof(int) * n, cudaMemcpyHostToDevice, s->st));
  const int mixed = precision == RGPU_MIXED;
  const void *ads = mixed ? (const void *)s->rec32 : (const void *)s->rec64;
  CK(rgpu_point_energies_launch(mixed, s->d_sys, ads, s->h_nmol * s->d.natom, s->io_xyz, s->io_atom, s->io_excl, n,
                                pair_check, s->fw_model == RGPU_FRAMEWORK_GRID, s->io_out, s->io_ov, s->st));
  CK(cudaMemcpyAsync(out, s->io_out, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s->st));
  if (ov) CK(cudaMemcpyAsync(ov, s->io_ov, sizeof(int) * n, cudaMemcpyDeviceToHost, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_bead_energies(rgpu_system *s, int precision, int n, const double *xyz, const int *atom,
                                  const int *exclude, double *out)
{
  if (!s || n < 0 || (n && (!xyz || !atom || !exclude || !out))) return fail(RGPU_E_INVALID, "bad argument");
  if (precision != RGPU_FP64 && precision != RGPU_MIXED) return fail(RGPU_E_INVALID, "precision");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  for (int i = 0; i < n; i++)
    if (atom[i] < 0 || atom[i] >= s->d.natom) return fail(RGPU_E_INVALID, "atom index %d", atom[i]);
  for (int base = 0; base < n; base += RGPU_MAX_POS) {
    int b = std::min(RGPU_MAX_POS, n - base);
    rc = bead_batch(s, precision, b, xyz + 3 * base, atom + base, exclude + base, 0, out + 4 * base, nullptr);
    if (rc) return rc;
  }
  return RGPU_SUCCESS;
}

extern "C" int rgpu_move_energy_difference(rgpu_system *s, int precision, int m, const double *new_xyz, double *out,
                                           int *overlap)
{
  if (!s || !new_xyz || !out) return fail(RGPU_E_INVALID, "bad argument");
  if (precision != RGPU_FP64 && precision != RGPU_MIXED) return fail(RGPU_E_INVALID, "precision");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  if (m < 0 || m >= s->h_nmol) return fail(RGPU_E_INVALID, "molecule %d", m);
  const int na = s->d.natom;
  double xyz[2 * RGPU_MAX_ATOMS * 3], res[2 * RGPU_MAX_ATOMS * 4];
  int atom[2 * RGPU_MAX_ATOMS], excl[2 * RGPU_MAX_ATOMS], ov[2 * RGPU_MAX_ATOMS];
  for (int a = 0; a < na; a++) {
    for (int c = 0; c < 3; c++) {
      xyz[3 * a + c] = new_xyz[3 * a + c];
      xyz[3 * (na + a) + c] = s->h_xyz[((size_t)m * na + a) * 3 + c];
    }
    atom[a] = atom[na + a] = a;
    excl[a] = excl[na + a] = m;
  }
  rc = bead_batch(s, precision, 2 * na, xyz, atom, excl, na, res, ov);
  if (rc) return rc;
  int o = 0;
  for (int k = 0; k < 4; k++) out[k] = 0.0;
  for (int a = 0; a < na; a++) {
    o |= ov[a];
    for (int k = 0; k < 4; k++) out[k] += res[4 * a + k] - res[4 * (na + a) + k];
  }
  if (overlap) *overlap = o;
  return RGPU_SUCCESS;
}

static double exclusion_energy(const rgpu_system *s, const double *xyz)
{
  const RgpuSys &h = s->h;
  double e = 0.0;
  for (int a = 0; a < h.natom - 1; a++)
    for (int b = a + 1; b < h.natom; b++) {
      if (h.mol_q[a] == 0.0 || h.mol_q[b] == 0.0) continue;
      double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1], dz = xyz[3 * a + 2] - xyz[3 * b + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      e += h.coulomb * h.mol_q[a] * h.mol_q[b] * erf(h.alpha * r) / r;
    }
  return e;
}

extern "C" int rgpu_ewald_fourier_difference(rgpu_system *s, int precision, int old_mol, const double *new_xyz,
                                             double *out)
{
  if (!s || !out) return fail(RGPU_E_INVALID, "bad argument");
  if (precision != RGPU_FP64 && precision != RGPU_MIXED) return fail(RGPU_E_INVALID, "precision");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  out[0] = out[1] = out[2] = 0.0;
  s->pending_dq = 0.0;
  if (!s->h.ewald || !s->h.nk) return RGPU_SUCCESS;
  if (old_mol >= s->h_nmol) return fail(RGPU_E_INVALID, "molecule %d", old_mol);
  const int na = s->d.natom;
  double xyz[2 * RGPU_MAX_ATOMS * 3], q[2 * RGPU_MAX_ATOMS];
  int ns = 0;
  double ex_old = 0.0, ex_new = 0.0;
  int dn = 0;
  if (old_mol >= 0) {
    const double *o = &s->h_xyz[(size_t)old_mol * na * 3];
    for (int a = 0; a < na; a++) {
      if (s->h.mol_q[a] == 0.0) continue;
      for (int c = 0; c < 3; c++) xyz[3 * ns + c] = o[3 * a + c];
      q[ns++] = -s->h.mol_q[a];
    }
    ex_old = exclusion_energy(s, o);
    dn--;
  }
  if (new_xyz) {
    for (int a = 0; a < na; a++) {
      if (s->h.mol_q[a] == 0.0) continue;
      for (int c = 0; c < 3; c++) xyz[3 * ns + c] = new_xyz[3 * a + c];
      q[ns++] = s->h.mol_q[a];
    }
    ex_new = exclusion_energy(s, new_xyz);
    dn++;
  }
  double e[2] = {0.0, 0.0};
  if (ns) {
    CK(cudaMemcpyAsync(s->io_xyz, xyz, sizeof(double) * 3 * ns, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->io_q, q, sizeof(double) * ns, cudaMemcpyHostToDevice, s->st));
    CK(rgpu_ewald_delta_launch(precision == RGPU_MIXED, s->d_sys, s->io_xyz, s->io_q, ns, s->ds, s->io_out, s->kw,
                               s->st));
    CK(cudaMemcpyAsync(e, s->io_out, sizeof(double) * 2, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
  } else {
    CK(cudaMemsetAsync(s->ds, 0, sizeof(double2) * s->h.nk, s->st));
  }
  const RgpuSys &h = s->h;
  const double dq = dn * h.mol_charge;
  double d_ads = e[0] - (ex_new - ex_old) - dn * h.self_mol;
  d_ads += h.uion * (s->net_ads + dq) * (s->net_ads + dq) - h.uion * s->net_ads * s->net_ads;
  double d_host = 2.0 * e[1] + 2.0 * h.uion * h.net_fw * dq;
  out[0] = d_ads;
  out[1] = d_host;
  out[2] = dq;
  s->pending_dq = dq;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_ewald_accept(rgpu_system *s)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  if (!s->h.ewald || !s->h.nk) return RGPU_SUCCESS;
  CK(rgpu_ewald_accept_launch(s->d_sys, s->ds, s->h.nk, s->st));
  CK(cudaStreamSynchronize(s->st));
  s->net_ads += s->pending_dq;
  s->pending_dq = 0.0;
  return RGPU_SUCCESS;
}

static bool grid_covers_cell(const int npts[3], const double size[3], const double shift[3], const double cell[3]);

/* The geometry of a grid of system s: npts, size, shift and the unit-cell
 * lengths `cell`; in a triclinic box also the unit-cell matrix (the box
 * matrix's columns scaled to the cell lengths) and its inverse. False when
 * the grid does not span the unit cell (its enclosing box in a triclinic
 * one, src/grids.c:336-360). */
static bool grid_geom_set(rgpu_system *s, int which, RgpuGridGeom &g, const int npts[3], const double size[3],
                          const double shift[3], const double cell[3])
{
  memset(&g, 0, sizeof g);
  for (int c = 0; c < 3; c++) {
    g.npts[c] = npts[c];
    g.size[c] = size[c];
    g.shift[c] = shift[c];
    g.cell[c] = cell[c];
  }
  if (!s->h.triclinic) return grid_covers_cell(npts, size, shift, cell);
  g.tri = 1;
  double uc[18];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) uc[3 * r + c] = s->h.hm[3 * r + c] * (cell[c] / s->d.box[c]);
  inverse_upper(uc, uc + 9);
  for (int r = 0; r < 3; r++) {
    if (npts[r] < 1 || !(size[r] > 0.0) || !(cell[r] > 0.0)) return false;
    double lo = 0.0, hi = 0.0;
    for (int c = 0; c < 3; c++) {
      lo += std::min(0.0, uc[3 * r + c]);
      hi += std::max(0.0, uc[3 * r + c]);
    }
    const double tol = 1e-9 * (hi - lo);
    if (shift[r] > lo + tol || shift[r] + size[r] < hi - tol) return false;
  }
  double *d = s->d_uc + 18 * which;
  if (cudaMemcpyAsync(d, uc, sizeof uc, cudaMemcpyHostToDevice, s->st) != cudaSuccess ||
      cudaStreamSynchronize(s->st) != cudaSuccess)
    return false;
  g.uc = d;
  return true;
}

extern "C" int rgpu_system_set_coulomb_grid(rgpu_system *s, const float *d_grid, const int npts[3],
                                            const double size[3], const double shift[3], const double cell[3])
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  RgpuSys &h = s->h;
  if (!d_grid) {
    if (h.use_grid && h.mol_charged)
      return fail(RGPU_E_INVALID, "the VDW grids of a charged molecule stay on: switch them off first");
    h.use_coul_grid = 0;
    h.coul_grid = nullptr;
  } else {
    if (!npts || !size || !shift || !cell) return fail(RGPU_E_INVALID, "bad argument");
    if (!h.ewald) return fail(RGPU_E_INVALID, "a Coulomb grid needs Ewald summation");
    if ((uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "grids must be 16-byte aligned");
    RgpuGridGeom g;
    if (!grid_geom_set(s, 1, g, npts, size, shift, cell)) return fail(RGPU_E_INVALID, "grid does not cover the cell");
    h.coul_geom = g;
    h.coul_grid = d_grid;
    h.use_coul_grid = 1;
  }
  CK(cudaMemcpyAsync(s->d_sys, &h, sizeof(RgpuSys), cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_set_grids(rgpu_system *s, const float *const *d_grids, const int npts[3],
                                     const double size[3], const double shift[3], const double cell[3])
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  RgpuSys &h = s->h;
  if (!d_grids) {
    h.use_grid = 0;
    s->fw_model = RGPU_FRAMEWORK_FULL;
    for (int a = 0; a < RGPU_MAX_ATOMS; a++) h.grid[a] = nullptr;
  } else {
    if (!npts || !size || !shift || !cell) return fail(RGPU_E_INVALID, "bad argument");
    if (h.mol_charged && !h.use_coul_grid)
      return fail(RGPU_E_INVALID, "a charged molecule needs a Coulomb grid (rgpu_system_set_coulomb_grid) first");
    RgpuGridGeom g;
    if (!grid_geom_set(s, 0, g, npts, size, shift, cell)) return fail(RGPU_E_INVALID, "grid does not cover the cell");
    for (int a = 0; a < h.natom; a++) {
      if (!d_grids[a]) return fail(RGPU_E_INVALID, "no grid for molecule atom %d", a);
      if ((uintptr_t)d_grids[a] % 16) return fail(RGPU_E_INVALID, "grids must be 16-byte aligned");
      h.grid[a] = d_grids[a];
    }
    h.grid_geom = g;
    h.use_grid = 1;
  }
  CK(cudaMemcpyAsync(s->d_sys, &h, sizeof(RgpuSys), cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_set_framework_model(rgpu_system *s, int model)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  if (model != RGPU_FRAMEWORK_FULL && model != RGPU_FRAMEWORK_GRID)
    return fail(RGPU_E_INVALID, "framework model %d", model);
  if (model == RGPU_FRAMEWORK_GRID && !s->h.use_grid)
    return fail(RGPU_E_INVALID, "the GRID framework model needs the system's grids (rgpu_system_set_grids)");
  s->fw_model = model;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_intra_energy(rgpu_system *s, double *out)
{
  if (!s || !out) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  const int na = s->d.natom;
  double e = 0.0;
  if (s->h.flexible)
    for (int m = 0; m < s->h_nmol; m++)
      e += chain_intra_energy(s->h, (const double(*)[3]) & s->h_xyz[(size_t)m * na * 3], na);
  *out = e;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_total_energy(rgpu_system *s, double *out)
{
  if (!s || !out) return fail(RGPU_E_INVALID, "bad argument");
  int rc = refresh_from_device(s);
  if (rc) return rc;
  const int na = s->d.natom, nads = s->h_nmol * na;
  double hv = 0, hc = 0, av = 0, ac = 0;
  std::vector<int> atom(RGPU_MAX_POS), excl(RGPU_MAX_POS);
  std::vector<double> res(4 * RGPU_MAX_POS);
  for (int base = 0; base < nads; base += RGPU_MAX_POS) {
    int b = std::min(RGPU_MAX_POS, nads - base);
    for (int i = 0; i < b; i++) {
      atom[i] = (base + i) % na;
      excl[i] = (base + i) / na;
    }
    rc = bead_batch(s, RGPU_FP64, b, &s->h_xyz[(size_t)base * 3], atom.data(), excl.data(), 0, res.data(), nullptr);
    if (rc) return rc;
    for (int i = 0; i < b; i++) {
      hv += res[4 * i];
      hc += res[4 * i + 1];
      av += res[4 * i + 2];
      ac += res[4 * i + 3];
    }
  }
  double hf = 0.0, af = 0.0;
  const RgpuSys &h = s->h;
  if (h.ewald && h.nk) {
    rc = recompute_sk_ads(s);
    if (rc) return rc;
    std::vector<double2> sa(h.nk), sf(h.nk);
    std::vector<double> kf(h.nk);
    CK(cudaMemcpyAsync(sa.data(), s->sk_ads, sizeof(double2) * h.nk, cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(sf.data(), s->sk_fw, sizeof(double2) * h.nk, cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(kf.data(), s->kfactor, sizeof(double) * h.nk, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int k = 0; k < h.nk; k++) {
      af += kf[k] * (sa[k].x * sa[k].x + sa[k].y * sa[k].y);
      hf += kf[k] * (sf[k].x * sa[k].x + sf[k].y * sa[k].y);
    }
    double ex = 0.0;
    for (int m = 0; m < s->h_nmol; m++) ex += exclusion_energy(s, &s->h_xyz[(size_t)m * na * 3]);
    const double net = s->h_nmol * h.mol_charge;
    af -= ex + s->h_nmol * h.self_mol;
    af += h.uion * net * net;
    hf = 2.0 * hf + 2.0 * h.uion * h.net_fw * net;
    s->net_ads = net;
  }
  out[0] = hv;
  out[1] = 0.5 * av;
  out[2] = hc;
  out[3] = 0.5 * ac;
  out[4] = hf;
  out[5] = af;
  return RGPU_SUCCESS;
}

/* ---------------------------------------------------------------------- */
extern "C" int rgpu_grid_build(rgpu_system *s, int type, const int npts[3], const double size[3], const double shift[3],
                               float *d_grid)
{
  if (!s || !npts || !size || !shift || !d_grid) return fail(RGPU_E_INVALID, "bad argument");
  if ((uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "d_grid must be 16-byte aligned");
  if (type < 0 || type >= s->ntypes) return fail(RGPU_E_INVALID, "type %d", type);
  for (int c = 0; c < 3; c++)
    if (npts[c] < 1) return fail(RGPU_E_INVALID, "npts");
  RgpuLJ lj[RGPU_MAX_FWTYPES];
  memset(lj, 0, sizeof lj);
  for (int sg = 0; sg < s->h.nseg; sg++) {
    const int ij = type * s->ntypes + s->fw_seg_type[sg];
    lj[sg].eps4 = 4.0 * s->lj_eps[ij];
    lj[sg].sig2 = s->lj_sig2[ij];
    lj[sg].shift = s->lj_shift[ij];
  }
  CK(rgpu_grid_build_launch_lj(s->d_sys, lj, npts, size, shift, d_grid, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_build_coulomb(rgpu_system *s, const int npts[3], const double size[3],
                                       const double shift[3], float *d_grid)
{
  if (!s || !npts || !size || !shift || !d_grid) return fail(RGPU_E_INVALID, "bad argument");
  if ((uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "d_grid must be 16-byte aligned");
  if (!s->h.ewald) return fail(RGPU_E_INVALID, "a Coulomb grid needs Ewald summation");
  for (int c = 0; c < 3; c++)
    if (npts[c] < 1) return fail(RGPU_E_INVALID, "npts");
  CK(rgpu_grid_build_launch_coulomb(s->d_sys, npts, size, shift, d_grid, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

/* the lookup wraps points into [0, cell) per axis; the grid must span that
 * range (the grid spans the unit-cell box, src/grids.c:337-359) */
static bool grid_covers_cell(const int npts[3], const double size[3], const double shift[3], const double cell[3])
{
  for (int c = 0; c < 3; c++) {
    if (npts[c] < 1 || !(size[c] > 0.0) || !(cell[c] > 0.0)) return false;
    if (shift[c] > 1e-9 * cell[c] || shift[c] + size[c] < cell[c] * (1.0 - 1e-9)) return false;
  }
  return true;
}

/* ---------------------------------------------------------------------- */
/* grid files (src/grids.c:692-977) */

static const size_t GRID_HDR_BYTES = 8 + 12 + 4 * 24 + 12;   /* the Coulomb file adds 8 */

static long long grid_points(const int npts[3])
{
  return (long long)(npts[0] + 1) * (npts[1] + 1) * (npts[2] + 1);
}

static void hdr_pack(const rgpu_grid_file_header *h, int coulomb, unsigned char *b)
{
  size_t o = 0;
  auto put = [&](const void *p, size_t n) { memcpy(b + o, p, n); o += n; };
  put(&h->spacing, 8);
  put(h->npts, 12);
  put(h->size, 24);
  put(h->shift, 24);
  put(h->delta, 24);
  put(h->unit_cell, 24);
  put(h->unit_cells, 12);
  if (coulomb) put(&h->ewald_precision, 8);
}

static void hdr_unpack(const unsigned char *b, int coulomb, rgpu_grid_file_header *h)
{
  size_t o = 0;
  auto get = [&](void *p, size_t n) { memcpy(p, b + o, n); o += n; };
  memset(h, 0, sizeof *h);
  get(&h->spacing, 8);
  get(h->npts, 12);
  get(h->size, 24);
  get(h->shift, 24);
  get(h->delta, 24);
  get(h->unit_cell, 24);
  get(h->unit_cells, 12);
  if (coulomb) get(&h->ewald_precision, 8);
}

/* opens `path`, reads and checks its header; on success the file is left
 * positioned at the first plane */
static int grid_file_open(const char *path, int coulomb, rgpu_grid_file_header *h, FILE **out)
{
  if (!path || !h) return fail(RGPU_E_INVALID, "bad argument");
  FILE *f = fopen(path, "rb");
  if (!f) return fail(RGPU_E_IO, "cannot open grid file %s", path);
  const size_t hb = GRID_HDR_BYTES + (coulomb ? 8 : 0);
  unsigned char b[GRID_HDR_BYTES + 8];
  if (fread(b, 1, hb, f) != hb) {
    fclose(f);
    return fail(RGPU_E_IO, "%s: short header", path);
  }
  hdr_unpack(b, coulomb, h);
  for (int c = 0; c < 3; c++)
    if (h->npts[c] < 1 || h->npts[c] > (1 << 16)) {
      fclose(f);
      return fail(RGPU_E_IO, "%s: not a grid file (grid points %d)", path, h->npts[c]);
    }
  struct stat st;
  const long long want = (long long)hb + 32LL * grid_points(h->npts);
  if (fstat(fileno(f), &st) || (long long)st.st_size != want) {
    fclose(f);
    return fail(RGPU_E_IO, "%s: %lld bytes, the header announces %lld", path, (long long)st.st_size, want);
  }
  *out = f;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_read_file_header(const char *path, int coulomb, rgpu_grid_file_header *hdr)
{
  FILE *f = nullptr;
  int rc = grid_file_open(path, coulomb, hdr, &f);
  if (rc) return rc;
  fclose(f);
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_read_file(const char *path, int coulomb, rgpu_grid_file_header *hdr, float *d_grid,
                                   size_t capacity)
{
  if (!d_grid || (uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "d_grid must be a 16-byte aligned device pointer");
  FILE *f = nullptr;
  int rc = grid_file_open(path, coulomb, hdr, &f);
  if (rc) return rc;
  const long long npt = grid_points(hdr->npts);
  if ((unsigned long long)capacity < 8ULL * npt) {
    fclose(f);
    return fail(RGPU_E_INVALID, "d_grid holds %zu floats, the grid %lld", capacity, 8LL * npt);
  }
  const size_t bytes = sizeof(float) * 8 * (size_t)npt;
  std::vector<float> host((size_t)8 * npt);
  const size_t got = fread(host.data(), 1, bytes, f);
  fclose(f);
  if (got != bytes) return fail(RGPU_E_IO, "%s: short read", path);
  float *planes = nullptr;
  CK(cudaMalloc((void **)&planes, bytes));
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (!e) e = cudaMemcpyAsync(planes, host.data(), bytes, cudaMemcpyHostToDevice, st);
  if (!e) e = rgpu_grid_planes_to_points_launch(planes, npt, d_grid, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (st) cudaStreamDestroy(st);
  cudaFree(planes);
  if (e) return fail(RGPU_E_CUDA, "grid file upload: %s", cudaGetErrorString(e));
  return RGPU_SUCCESS;
}

/* mkdir -p of the directory part of path (mode 0700) */
static int make_parents(const char *path)
{
  std::string p(path);
  for (size_t i = 1; i < p.size(); i++) {
    if (p[i] != '/') continue;
    const std::string d = p.substr(0, i);
    if (mkdir(d.c_str(), S_IRWXU) && errno != EEXIST) return -1;
  }
  return 0;
}

extern "C" int rgpu_grid_write_file(const char *path, int coulomb, const rgpu_grid_file_header *hdr,
                                    const float *d_grid)
{
  if (!path || !hdr || !d_grid || (uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "bad argument");
  for (int c = 0; c < 3; c++)
    if (hdr->npts[c] < 1) return fail(RGPU_E_INVALID, "grid points %d", hdr->npts[c]);
  const long long npt = grid_points(hdr->npts);
  const size_t bytes = sizeof(float) * 8 * (size_t)npt;
  std::vector<float> host((size_t)8 * npt);
  float *planes = nullptr;
  CK(cudaMalloc((void **)&planes, bytes));
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (!e) e = rgpu_grid_points_to_planes_launch(d_grid, npt, planes, st);
  if (!e) e = cudaMemcpyAsync(host.data(), planes, bytes, cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (st) cudaStreamDestroy(st);
  cudaFree(planes);
  if (e) return fail(RGPU_E_CUDA, "grid file download: %s", cudaGetErrorString(e));
  if (make_parents(path)) return fail(RGPU_E_IO, "cannot create the directories of %s", path);
  FILE *f = fopen(path, "wb");
  if (!f) return fail(RGPU_E_IO, "cannot create grid file %s", path);
  unsigned char b[GRID_HDR_BYTES + 8];
  hdr_pack(hdr, coulomb, b);
  const size_t hb = GRID_HDR_BYTES + (coulomb ? 8 : 0);
  const bool ok = fwrite(b, 1, hb, f) == hb && fwrite(host.data(), 1, bytes, f) == bytes;
  if (fclose(f) || !ok) return fail(RGPU_E_IO, "%s: write failed", path);
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_file_path(char *buf, size_t n, const char *raspa_dir, const char *forcefield,
                                   const char *framework, double spacing, const char *pseudo_atom, int shifted,
                                   const int unit_cells[3])
{
  if (!buf || !raspa_dir || !forcefield || !framework || (!pseudo_atom && !unit_cells))
    return fail(RGPU_E_INVALID, "bad argument");
  int w;
  if (pseudo_atom)
    w = snprintf(buf, n, "%s/share/raspa/grids/%s/%s/%lf/%s_%s_%s.grid", raspa_dir, forcefield, framework, spacing,
                 framework, pseudo_atom, shifted ? "shifted" : "truncated");
  else
    w = snprintf(buf, n, "%s/share/raspa/grids/%s/%s/%lf/%dx%dx%d/%s_Electrostatics_Ewald.grid", raspa_dir,
                 forcefield, framework, spacing, unit_cells[0], unit_cells[1], unit_cells[2], framework);
  if (w < 0 || (size_t)w >= n) return fail(RGPU_E_INVALID, "path buffer of %zu bytes is too small", n);
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_interpolate(const float *d_grid, const int npts[3], const double size[3],
                                     const double shift[3], const double cell[3], int n, const double *xyz,
                                     double *out)
{
  if (!d_grid || !npts || !size || !shift || !cell || n < 0 || (n && (!xyz || !out)))
    return fail(RGPU_E_INVALID, "bad argument");
  if ((uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "d_grid must be 16-byte aligned");
  if (!grid_covers_cell(npts, size, shift, cell)) return fail(RGPU_E_INVALID, "grid does not cover the cell");
  if (n == 0) return RGPU_SUCCESS;
  double *dx = nullptr, *dout = nullptr;
  CK(cudaMalloc((void **)&dx, sizeof(double) * 3 * n));
  if (cudaMalloc((void **)&dout, sizeof(double) * n) != cudaSuccess) {
    cudaFree(dx);
    return fail(RGPU_E_CUDA, "cudaMalloc");
  }
  int rc = RGPU_SUCCESS;
  if (cudaMemcpy(dx, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice) ||
      rgpu_grid_interp_launch(d_grid, npts, size, shift, cell, n, dx, dout, 0) ||
      cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost))
    rc = fail(RGPU_E_CUDA, "grid interpolation: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFree(dx);
  cudaFree(dout);
  return rc;
}

/* ---------------------------------------------------------------------- */
/* Grid lookup without device allocation. The positions and results of one
 * call live in a file-scope device array (one per device, 256 KB); the
 * first call on a device looks up its address with cudaGetSymbolAddress
 * and keeps it (an address of the device's current context: it does not
 * survive cudaDeviceReset). Calls that overlap on one device share the array
 * and race. */
struct NoAllocInterp {
  double xyz[RGPU_NOALLOC_MAX_POINTS * 3];
  double out[RGPU_NOALLOC_MAX_POINTS];
};
static __device__ __align__(256) NoAllocInterp g_noalloc_interp;

#define RGPU_NOALLOC_MAX_DEVICES 64
static std::mutex g_noalloc_mu;
static NoAllocInterp *g_noalloc_ptr[RGPU_NOALLOC_MAX_DEVICES];

static int noalloc_scratch(NoAllocInterp **out)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= RGPU_NOALLOC_MAX_DEVICES) return fail(RGPU_E_INVALID, "device %d", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_interp);
    if (e != cudaSuccess) return fail(RGPU_E_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (NoAllocInterp *)p;
  }
  *out = g_noalloc_ptr[dev];
  return RGPU_SUCCESS;
}

extern "C" int rgpu_grid_interpolate_noalloc(const float *d_grid, const int npts[3], const double size[3],
                                             const double shift[3], const double cell[3], int n,
                                             const double *xyz, double *out)
{
  if (!d_grid || !npts || !size || !shift || !cell || n < 0 || (n && (!xyz || !out)))
    return fail(RGPU_E_INVALID, "bad argument");
  if (n > RGPU_NOALLOC_MAX_POINTS)
    return fail(RGPU_E_INVALID, "n = %d points exceeds RGPU_NOALLOC_MAX_POINTS (%d)", n, RGPU_NOALLOC_MAX_POINTS);
  if ((uintptr_t)d_grid % 16) return fail(RGPU_E_INVALID, "d_grid must be 16-byte aligned");
  if (!grid_covers_cell(npts, size, shift, cell)) return fail(RGPU_E_INVALID, "grid does not cover the cell");
  NoAllocInterp *scr = nullptr;
  int rc = noalloc_scratch(&scr);
  if (rc != RGPU_SUCCESS) return rc;
  if (n == 0) return RGPU_SUCCESS;
  /* results start at zero, so a point the kernel did not write could never
   * return a previous call's value */
  CK(cudaMemsetAsync(scr->out, 0, sizeof(double) * n, 0));
  CK(cudaMemcpyAsync(scr->xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, 0));
  CK(rgpu_grid_interp_launch(d_grid, npts, size, shift, cell, n, scr->xyz, scr->out, 0));
  CK(cudaMemcpyAsync(out, scr->out, sizeof(double) * n, cudaMemcpyDeviceToHost, 0));
  CK(cudaStreamSynchronize(0));
  return RGPU_SUCCESS;
}

/* The device slots: d_systems[j] = system order[j], its framework staged in
 * shared memory when its launch group stages it; d_off (once the staging
 * buffer exists) in the same slot order. */
/* whether system s, in the first launch (second = false) or the second,
 * has its framework share staged in shared memory: the engine stages when
 * its plan holds a framework share and the system's share fits it */
static bool slot_smem_fw(const rgpu_engine *e, const rgpu_system *s, bool second)
{
  const int c = second ? e->cluster_b : e->cluster;
  const int fw_items = second ? e->fw_items_b : e->fw_items, tile_items = second ? e->tile_items_b : e->tile_items;
  const int share_tiles = (s->h.ntile + c - 1) / c, share_fw = (s->d.nfw + c - 1) / c;
  return fw_items > 0 && (e->mixed ? share_tiles * RGPU_TILE <= fw_items && share_tiles <= tile_items
                                   : share_fw <= fw_items);
}

static cudaError_t upload_slots(rgpu_engine *e)
{
  const int n = (int)e->sys.size();
  std::vector<RgpuSys> hs(n);
  for (int j = 0; j < n; j++) {
    hs[j] = e->sys[e->order[j]]->h;
    hs[j].smem_fw = slot_smem_fw(e, e->sys[e->order[j]], j >= n - e->nsplit);
  }
  cudaError_t err = cudaMemcpy(e->d_systems, hs.data(), sizeof(RgpuSys) * n, cudaMemcpyHostToDevice);
  if (err != cudaSuccess || !e->d_off) return err;
  std::vector<unsigned long long> off(n);
  for (int j = 0; j < n; j++) off[j] = e->off[e->order[j]];
  return cudaMemcpy(e->d_off, off.data(), sizeof(unsigned long long) * n, cudaMemcpyHostToDevice);
}

/* ---------------------------------------------------------------------- */
/* Cluster size of an engine launch: the CTAs of one system. More CTAs per
 * system when there are few systems (up to 8, the portable cluster size),
 * one when the systems alone fill the GPU. */
static int auto_cluster(int nsys)
{
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int c = 1;
  while (c < 8 && (long long)nsys * c * 2 <= sms) c *= 2;
  return c;
}

extern "C" int rgpu_engine_create(rgpu_engine **out, rgpu_system *const *systems, int n, int precision, int threads,
                                  int cluster)
{
  return rgpu_engine_create_ex(out, systems, n, precision, threads, cluster, 1);
}

extern "C" int rgpu_engine_create_ex(rgpu_engine **out, rgpu_system *const *systems, int n, int precision,
                                     int threads, int cluster, int ctas_per_sm)
{
  if (!out || !systems || n < 1) return fail(RGPU_E_INVALID, "bad argument");
  if (ctas_per_sm < 1 || ctas_per_sm > 4) return fail(RGPU_E_INVALID, "ctas_per_sm %d outside [1,4]", ctas_per_sm);
  if (precision != RGPU_FP64 && precision != RGPU_MIXED && precision != RGPU_MIXED_CC64)
    return fail(RGPU_E_INVALID, "precision");
  /* the mixed kernels are compiled for up to 1024 threads (64 registers), the
   * FP64 one for up to 512 */
  const int max_threads = precision != RGPU_FP64 ? 1024 : 512;
  if (threads < 64 || threads > max_threads || threads % 32)
    return fail(RGPU_E_INVALID, "threads %d outside [64,%d] or not a multiple of 32", threads, max_threads);
  if (cluster < 0 || cluster > 8) return fail(RGPU_E_INVALID, "cluster %d", cluster);
  /* registers: 128 per thread (the narrow build) unless the CTAs of an SM
   * need more than 65536 together; then the mixed kernel's 64-register build */
  const bool wide = threads > 512 || (long long)threads * 128 * ctas_per_sm > 65536;
  if (wide && precision == RGPU_FP64)
    return fail(RGPU_E_INVALID, "FP64 engine: %d CTAs of %d threads do not fit one SM", ctas_per_sm, threads);
  if ((long long)threads * 64 * ctas_per_sm > 65536)
    return fail(RGPU_E_INVALID, "%d CTAs of %d threads do not fit one SM", ctas_per_sm, threads);
  *out = nullptr;
  rgpu_engine *e = new rgpu_engine();
  e->mixed = precision;     /* 0 FP64, 1 mixed, 2 mixed with FP64 charge-charge terms */
  e->threads = threads;
  e->wide = wide;
  e->flex = false;
  e->cluster = cluster ? cluster : auto_cluster(n);
  e->kw = 1;
  e->max_ads = 0;
  for (int i = 0; i < n; i++) {
    rgpu_system *s = systems[i];
    if (!s) { delete e; return fail(RGPU_E_INVALID, "null system"); }
    e->sys.push_back(s);
    e->order.push_back(i);
    if (s->h.use_grid && s->h.mol_charged && !s->h.use_coul_grid) {
      delete e;
      return fail(RGPU_E_INVALID, "system with VDW grids and a charged molecule but no Coulomb grid");
    }
    e->flex = e->flex || s->h.use_grid || s->h.flexible;
    if (e->flex && precision == RGPU_MIXED_CC64) {
      delete e;
      return fail(RGPU_E_INVALID, "RGPU_MIXED_CC64 covers rigid molecules without energy grids");
    }
    e->kw = std::max(e->kw, s->kw);
    e->max_ads = std::max(e->max_ads, s->d.maxmol * s->d.natom);
  }
  int dev = 0, smem_max = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (ctas_per_sm > 1) {
    /* room for ctas_per_sm CTAs per SM, each with its 1 KB of reserved
     * shared memory */
    int per_sm = 0;
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    smem_max = std::min(smem_max, per_sm / ctas_per_sm - 1024);
  }
  e->smem_max = smem_max;
  EngineGroup g;
  if (!plan_group(e, 0, n, e->cluster, g)) {
    delete e;
    return fail(RGPU_E_INVALID, "adsorbate capacity does not fit in shared memory");
  }
  e->fw_items = g.fw_items;
  e->tile_items = g.tile_items;
  e->k_items = g.k_items;
  e->smem = g.smem;
  e->nsplit = 0;
  e->cluster_b = 0;
  e->fw_items_b = e->tile_items_b = e->k_items_b = 0;
  e->smem_b = 0;
  e->st_b = nullptr;
  e->ev_fork = e->ev_join = nullptr;
  e->use_graph = 0;
  e->gexec = nullptr;
  e->g_nsteps = -1;
  e->stage_bytes = 0;
  e->d_off = nullptr;
  e->d_stage = nullptr;
  e->h_stage = nullptr;
  e->h_slots = nullptr;
  if (cudaMalloc((void **)&e->d_systems, sizeof(RgpuSys) * n) != cudaSuccess) {
    delete e;
    return fail(RGPU_E_CUDA, "cudaMalloc engine");
  }
  /* the engine's own stream: a system may be replaced and destroyed while
   * the engine lives (rgpu_engine_replace_system) */
  if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(e->d_systems);
    delete e;
    return fail(RGPU_E_CUDA, "cudaStreamCreate engine");
  }
  if (upload_slots(e) != cudaSuccess) {
    cudaStreamDestroy(e->st);
    cudaFree(e->d_systems);
    delete e;
    return fail(RGPU_E_CUDA, "upload engine");
  }
  *out = e;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_destroy(rgpu_engine *e)
{
  if (!e) return RGPU_SUCCESS;
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  if (e->d_off) cudaFree(e->d_off);
  if (e->d_stage) cudaFree(e->d_stage);
  if (e->h_stage) cudaFreeHost(e->h_stage);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  if (e->st_b) cudaStreamDestroy(e->st_b);
  for (cudaEvent_t ev : e->slot_ev)
    if (ev) cudaEventDestroy(ev);
  if (e->h_slots) cudaFreeHost(e->h_slots);
  cudaFree(e->d_systems);
  if (e->st) {
    cudaStreamSynchronize(e->st);
    cudaStreamDestroy(e->st);
  }
  delete e;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_set_split(rgpu_engine *e, const int *second, int nsecond, int cluster_b)
{
  if (!e || nsecond < 0 || (nsecond > 0 && !second)) return fail(RGPU_E_INVALID, "bad argument");
  const int n = (int)e->sys.size();
  if (nsecond >= n) return fail(RGPU_E_INVALID, "the first launch needs at least one system");
  if (nsecond > 0 && (cluster_b < 1 || cluster_b > 8))
    return fail(RGPU_E_INVALID, "cluster %d", cluster_b);
  std::vector<char> in_b(n, 0);
  for (int k = 0; k < nsecond; k++) {
    if (second[k] < 0 || second[k] >= n || in_b[second[k]])
      return fail(RGPU_E_INVALID, "system index %d out of range or repeated", second[k]);
    in_b[second[k]] = 1;
  }
  std::vector<int> order;
  for (int i = 0; i < n; i++)
    if (!in_b[i]) order.push_back(i);
  for (int k = 0; k < nsecond; k++) order.push_back(second[k]);
  const std::vector<int> old_order = e->order;
  e->order = order;
  EngineGroup ga, gb = {0, 0, 0, 0};
  if (!plan_group(e, 0, n - nsecond, e->cluster, ga) || (nsecond > 0 && !plan_group(e, n - nsecond, n, cluster_b, gb))) {
    e->order = old_order;
    return fail(RGPU_E_INVALID, "adsorbate capacity does not fit in shared memory");
  }
  if (nsecond > 0 && !e->st_b) {
    if (cudaStreamCreateWithFlags(&e->st_b, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming) != cudaSuccess) {
      e->order = old_order;
      return fail(RGPU_E_CUDA, "split streams");
    }
  }
  /* launches and staging kernels in flight (on any stream) read the old slots */
  CK(cudaDeviceSynchronize());
  e->fw_items = ga.fw_items;
  e->tile_items = ga.tile_items;
  e->k_items = ga.k_items;
  e->smem = ga.smem;
  e->nsplit = nsecond;
  e->cluster_b = nsecond > 0 ? cluster_b : 0;
  e->fw_items_b = gb.fw_items;
  e->tile_items_b = gb.tile_items;
  e->k_items_b = gb.k_items;
  e->smem_b = gb.smem;
  if (e->gexec) {
    cudaGraphExecDestroy(e->gexec);
    e->gexec = nullptr;
  }
  CK(upload_slots(e));
  return RGPU_SUCCESS;
}

/* The engine launch(es) of nsteps steps on stream st: the first group of
 * slots there, the second (if any) on st_b, forked from st and joined back,
 * so that both run side by side and st waits for both (also under stream
 * capture, where the fork and join become graph edges). */
static cudaError_t engine_launch_all(rgpu_engine *e, long long nsteps, cudaStream_t st)
{
  const int n = (int)e->sys.size(), na = n - e->nsplit;
  cudaError_t err;
  if (e->nsplit > 0) {
    if ((err = cudaEventRecord(e->ev_fork, st)) != cudaSuccess) return err;
    if ((err = cudaStreamWaitEvent(e->st_b, e->ev_fork, 0)) != cudaSuccess) return err;
  }
  err = rgpu_engine_launch(e->mixed, e->d_systems, na, nsteps, e->kw, e->max_ads, e->fw_items, e->tile_items,
                           e->k_items, e->cluster, e->threads, e->wide, e->flex, st);
  if (e->nsplit > 0) {
    cudaError_t eb = rgpu_engine_launch(e->mixed, e->d_systems + na, e->nsplit, nsteps, e->kw, e->max_ads,
                                        e->fw_items_b, e->tile_items_b, e->k_items_b, e->cluster_b, e->threads,
                                        e->wide, e->flex, e->st_b);
    if (err == cudaSuccess) err = eb;
    cudaError_t ej = cudaEventRecord(e->ev_join, e->st_b);
    if (ej == cudaSuccess) ej = cudaStreamWaitEvent(st, e->ev_join, 0);
    if (err == cudaSuccess) err = ej;
  }
  return err;
}

extern "C" int rgpu_engine_run(rgpu_engine *e, long long nsteps, void *stream)
{
  if (!e || nsteps < 0) return fail(RGPU_E_INVALID, "bad argument");
  cudaStream_t st = stream ? (cudaStream_t)stream : e->st;
  /* a system given grids after the engine was built needs the engine's
   * flexible-chain/grid build */
  for (rgpu_system *s : e->sys)
    if ((s->h.use_grid || s->h.flexible) && !e->flex)
      return fail(RGPU_E_INVALID, "a system needs the flexible-chain/grid build of the engine");
  /* every system's own stream work (uploads) must be visible to the launch */
  for (rgpu_system *s : e->sys) CK(cudaStreamSynchronize(s->st));
  CK(rgpu_engine_prepare(e->mixed, e->wide, e->flex, std::max(e->smem, e->smem_b)));
  if (!e->use_graph) {
    CK(engine_launch_all(e, nsteps, st));
  } else {
    if (!e->gexec || e->g_nsteps != nsteps) {
      if (e->gexec) {
        CK(cudaGraphExecDestroy(e->gexec));
        e->gexec = nullptr;
      }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = engine_launch_all(e, nsteps, st);
      cudaError_t ce = cudaStreamEndCapture(st, &g);
      if (le != cudaSuccess || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(RGPU_E_CUDA, "engine capture: %s", cudaGetErrorString(le != cudaSuccess ? le : ce));
      }
      cudaError_t ie = cudaGraphInstantiate(&e->gexec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) return fail(RGPU_E_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
      e->g_nsteps = nsteps;
    }
    CK(cudaGraphLaunch(e->gexec, st));
  }
  for (rgpu_system *s : e->sys) s->records_stale = 1;
  return RGPU_SUCCESS;
}

/* Replaces system i of an engine (creation order) by `s`, ordered on
 * `stream` after the work already queued there: the device slot's
 * descriptor is rewritten with one asynchronous copy from a pinned host
 * copy, with no allocation and no device synchronisation, and a captured
 * graph of the engine stays valid. The new system must fit the engine's
 * launch layout: the molecule capacity, the Ewald phase tables and the
 * kernel build; its framework share is staged in shared memory when it
 * fits the engine's staging, else read from global memory (L2). */
extern "C" int rgpu_engine_replace_system(rgpu_engine *e, int i, rgpu_system *s, void *stream)
{
  if (!e || !s || i < 0 || i >= (int)e->sys.size()) return fail(RGPU_E_INVALID, "bad argument");
  if (s->h.use_grid && s->h.mol_charged && !s->h.use_coul_grid)
    return fail(RGPU_E_INVALID, "system with VDW grids and a charged molecule but no Coulomb grid");
  if ((s->h.use_grid || s->h.flexible) && !e->flex)
    return fail(RGPU_E_INVALID, "the system needs the flexible-chain/grid build of the engine");
  if (s->kw > e->kw) return fail(RGPU_E_INVALID, "the system's wave vectors exceed the engine's phase tables");
  if (s->d.maxmol * s->d.natom > e->max_ads) return fail(RGPU_E_INVALID, "molecule capacity exceeds the engine's");
  if (e->d_stage) return fail(RGPU_E_INVALID, "engine with a batched-transfer staging buffer");
  const int n = (int)e->sys.size();
  int j = 0;
  while (e->order[j] != i) j++;
  const bool second = j >= n - e->nsplit;
  if (!e->h_slots) {
    if (cudaMallocHost((void **)&e->h_slots, sizeof(RgpuSys) * n) != cudaSuccess)
      return fail(RGPU_E_CUDA, "cudaMallocHost");
    e->slot_ev.assign(n, nullptr);
  }
  /* the pinned copy of this slot may still be in flight from an earlier
   * replacement */
  if (e->slot_ev[j]) CK(cudaEventSynchronize(e->slot_ev[j]));
  else CK(cudaEventCreateWithFlags(&e->slot_ev[j], cudaEventDisableTiming));
  RgpuSys h = s->h;
  h.smem_fw = slot_smem_fw(e, s, second);
  e->h_slots[j] = h;
  cudaStream_t st = stream ? (cudaStream_t)stream : e->st;
  CK(cudaMemcpyAsync(e->d_systems + j, e->h_slots + j, sizeof(RgpuSys), cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(e->slot_ev[j], st));
  e->sys[i] = s;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_use_graph(rgpu_engine *e, int on)
{
  if (!e) return fail(RGPU_E_INVALID, "bad argument");
  e->use_graph = on != 0;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_cluster(rgpu_engine *e)
{
  return e ? e->cluster : 0;
}

/* ---- batched state transfer ---------------------------------------------- */
static int engine_staging(rgpu_engine *e)
{
  if (e->d_stage) return RGPU_SUCCESS;
  const int n = (int)e->sys.size();
  e->off.resize(n);
  size_t o = 0;
  for (int i = 0; i < n; i++) {
    e->off[i] = o;
    const rgpu_system *s = e->sys[i];
    o += sizeof(RgpuState) + sizeof(double) * 3 * (size_t)s->d.maxmol * s->d.natom;
    o = (o + 255) & ~(size_t)255;
  }
  e->stage_bytes = o;
  if (cudaMalloc((void **)&e->d_off, sizeof(unsigned long long) * n) != cudaSuccess ||
      cudaMalloc((void **)&e->d_stage, o) != cudaSuccess || cudaMallocHost((void **)&e->h_stage, o) != cudaSuccess) {
    if (e->d_off) cudaFree(e->d_off);
    if (e->d_stage) cudaFree(e->d_stage);
    e->d_off = nullptr;
    e->d_stage = nullptr;
    e->h_stage = nullptr;
    return fail(RGPU_E_CUDA, "engine staging allocation");
  }
  CK(upload_slots(e));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_staging_bytes(rgpu_engine *e, size_t *bytes)
{
  if (!e || !bytes) return fail(RGPU_E_INVALID, "bad argument");
  int rc = engine_staging(e);
  if (rc) return rc;
  *bytes = e->stage_bytes;
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_get_state(rgpu_engine *e, double *energy8, long long *counters20, int *nmol, int *status,
                                     unsigned long long *step, double *const *xyz)
{
  if (!e) return fail(RGPU_E_INVALID, "bad argument");
  int rc = engine_staging(e);
  if (rc) return rc;
  const int n = (int)e->sys.size();
  CK(cudaDeviceSynchronize());
  CK(rgpu_gather_states_launch(e->d_systems, n, e->d_off, e->d_stage, e->st));
  CK(cudaMemcpyAsync(e->h_stage, e->d_stage, e->stage_bytes, cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  for (int i = 0; i < n; i++) {
    rgpu_system *s = e->sys[i];
    const unsigned char *r = e->h_stage + e->off[i];
    memcpy(&s->h_state, r, sizeof(RgpuState));
    const RgpuState &st = s->h_state;
    if (energy8) memcpy(energy8 + (size_t)RGPU_NE * i, st.energy, sizeof(double) * RGPU_NE);
    if (counters20) memcpy(counters20 + (size_t)RGPU_NCNT * i, st.counters, sizeof(long long) * RGPU_NCNT);
    if (nmol) nmol[i] = st.nmol;
    if (status) status[i] = st.status;
    if (step) step[i] = st.step[0];
    if (xyz && xyz[i]) memcpy(xyz[i], r + sizeof(RgpuState), sizeof(double) * 3 * (size_t)st.nmol * s->d.natom);
  }
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_set_adsorbates(rgpu_engine *e, const int *nmol, const double *const *xyz)
{
  if (!e || !nmol || !xyz) return fail(RGPU_E_INVALID, "bad argument");
  const int n = (int)e->sys.size();
  for (int i = 0; i < n; i++) {
    if (nmol[i] < 0 || (nmol[i] > 0 && !xyz[i])) return fail(RGPU_E_INVALID, "system %d: bad configuration", i);
    if (nmol[i] > e->sys[i]->d.maxmol)
      return fail(RGPU_E_CAPACITY, "system %d: nmol %d > maxmol %d", i, nmol[i], e->sys[i]->d.maxmol);
  }
  int rc = engine_staging(e);
  if (rc) return rc;
  CK(cudaDeviceSynchronize());
  for (int i = 0; i < n; i++) {
    rgpu_system *s = e->sys[i];
    unsigned char *r = e->h_stage + e->off[i];
    ((RgpuState *)r)->nmol = nmol[i];
    const size_t nx = (size_t)nmol[i] * s->d.natom * 3;
    if (nx) memcpy(r + sizeof(RgpuState), xyz[i], sizeof(double) * nx);
    s->h_xyz.assign(xyz[i], xyz[i] + nx);
    s->h_nmol = nmol[i];
    s->net_ads = nmol[i] * s->h.mol_charge;
    s->pending_dq = 0.0;
  }
  CK(cudaMemcpyAsync(e->d_stage, e->h_stage, e->stage_bytes, cudaMemcpyHostToDevice, e->st));
  CK(rgpu_scatter_positions_launch(e->d_systems, n, e->d_off, e->d_stage, e->st));
  int max_nk = 0;
  for (int i = 0; i < n; i++) {
    rgpu_system *s = e->sys[i];
    CK(rgpu_records_launch(s->d_sys, nmol[i] * s->d.natom, s->rec32, s->rec64, e->st));
    s->records_stale = 0;
    max_nk = std::max(max_nk, s->h.nk);
  }
  CK(rgpu_upload_sk_launch(e->d_systems, n, max_nk, e->st));
  CK(cudaStreamSynchronize(e->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_engine_sync(rgpu_engine *e)
{
  if (!e) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaStreamSynchronize(e->st));
  CK(cudaDeviceSynchronize());
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_state(rgpu_system *s, double *energy8, long long *counters20, int *nmol, int *status,
                                 unsigned long long *step)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(&s->h_state, s->state, sizeof(RgpuState), cudaMemcpyDeviceToHost));
  if (energy8) memcpy(energy8, s->h_state.energy, sizeof(double) * RGPU_NE);
  if (counters20) memcpy(counters20, s->h_state.counters, sizeof(long long) * RGPU_NCNT);
  if (nmol) *nmol = s->h_state.nmol;
  if (status) *status = s->h_state.status;
  if (step) *step = s->h_state.step[0];
  return RGPU_SUCCESS;
}

/* ---- checkpoints ---------------------------------------------------------- */
namespace {
struct CheckpointHeader {
  char magic[8];              /* "RGPUCKP1" */
  uint64_t fingerprint;
  int32_t natom, nk, nmol, pad;
  double net_ads, pending_dq;
};
const char CKPT_MAGIC[8] = {'R', 'G', 'P', 'U', 'C', 'K', 'P', '1'};
}

static size_t checkpoint_bytes(const rgpu_system *s, int nmol)
{
  return sizeof(CheckpointHeader) + sizeof(RgpuState) + sizeof(double) * 3 * (size_t)nmol * s->d.natom +
         sizeof(double2) * (size_t)s->h.nk;
}

extern "C" int rgpu_system_checkpoint_size(rgpu_system *s, size_t *bytes)
{
  if (!s || !bytes) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaDeviceSynchronize());
  int n = 0;
  CK(cudaMemcpy(&n, s->nmol, sizeof(int), cudaMemcpyDeviceToHost));
  *bytes = checkpoint_bytes(s, n);
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_checkpoint(rgpu_system *s, void *buf, size_t bytes)
{
  if (!s || !buf) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaDeviceSynchronize());
  RgpuState st;
  CK(cudaMemcpy(&st, s->state, sizeof(RgpuState), cudaMemcpyDeviceToHost));
  const size_t need = checkpoint_bytes(s, st.nmol);
  if (bytes < need) return fail(RGPU_E_CAPACITY, "checkpoint needs %zu bytes, %zu given", need, bytes);
  int rc = refresh_from_device(s);
  if (rc) return rc;
  char *p = (char *)buf;
  CheckpointHeader hd;
  memset(&hd, 0, sizeof hd);
  memcpy(hd.magic, CKPT_MAGIC, 8);
  hd.fingerprint = s->fingerprint;
  hd.natom = s->d.natom;
  hd.nk = s->h.nk;
  hd.nmol = st.nmol;
  hd.net_ads = s->net_ads;
  hd.pending_dq = s->pending_dq;
  memcpy(p, &hd, sizeof hd);
  p += sizeof hd;
  memcpy(p, &st, sizeof st);
  p += sizeof st;
  const size_t nx = (size_t)st.nmol * s->d.natom * 3;
  if (nx) CK(cudaMemcpy(p, s->ads_xyz, sizeof(double) * nx, cudaMemcpyDeviceToHost));
  p += sizeof(double) * nx;
  if (s->h.nk) CK(cudaMemcpy(p, s->sk_ads, sizeof(double2) * s->h.nk, cudaMemcpyDeviceToHost));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_restore(rgpu_system *s, const void *buf, size_t bytes)
{
  if (!s || !buf || bytes < sizeof(CheckpointHeader) + sizeof(RgpuState)) return fail(RGPU_E_INVALID, "bad argument");
  const char *p = (const char *)buf;
  CheckpointHeader hd;
  memcpy(&hd, p, sizeof hd);
  p += sizeof hd;
  if (memcmp(hd.magic, CKPT_MAGIC, 8)) return fail(RGPU_E_INVALID, "not a checkpoint");
  if (hd.fingerprint != s->fingerprint || hd.natom != s->d.natom || hd.nk != s->h.nk)
    return fail(RGPU_E_INVALID, "checkpoint of another framework, molecule or force field");
  if (hd.nmol < 0 || hd.nmol > s->d.maxmol) return fail(RGPU_E_CAPACITY, "checkpoint holds %d molecules, maxmol %d",
                                                        hd.nmol, s->d.maxmol);
  if (bytes != checkpoint_bytes(s, hd.nmol)) return fail(RGPU_E_INVALID, "checkpoint size %zu", bytes);
  RgpuState st;
  memcpy(&st, p, sizeof st);
  p += sizeof st;
  if (st.nmol != hd.nmol) return fail(RGPU_E_INVALID, "checkpoint inconsistent");
  CK(cudaDeviceSynchronize());
  const size_t nx = (size_t)hd.nmol * s->d.natom * 3;
  s->h_xyz.assign((const double *)p, (const double *)p + nx);
  p += sizeof(double) * nx;
  s->h_nmol = hd.nmol;
  s->net_ads = hd.net_ads;
  s->pending_dq = hd.pending_dq;
  s->h_state = st;
  if (nx) CK(cudaMemcpy(s->ads_xyz, s->h_xyz.data(), sizeof(double) * nx, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->state, &st, sizeof st, cudaMemcpyHostToDevice));
  if (s->h.nk) CK(cudaMemcpy(s->sk_ads, p, sizeof(double2) * s->h.nk, cudaMemcpyHostToDevice));
  int rc = upload_records(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_set_limits(rgpu_system *s, unsigned long long end_step, unsigned long long avg_start)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  unsigned long long v[2] = {end_step ? end_step : ~0ULL, avg_start};
  /* ordered on the system's own stream, which every engine launch waits
   * for; no device-wide synchronisation, so a request loop can set up new
   * systems while a launch of other systems runs */
  CK(cudaMemcpyAsync(s->step + 1, v, sizeof v, cudaMemcpyHostToDevice, s->st));
  CK(cudaStreamSynchronize(s->st));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_averages(rgpu_system *s, double *sums8)
{
  if (!s || !sums8) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(sums8, s->sums, sizeof(double) * RGPU_NSUM, cudaMemcpyDeviceToHost));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_reset_averages(rgpu_system *s)
{
  if (!s) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaDeviceSynchronize());
  CK(cudaMemset(s->sums, 0, sizeof(double) * RGPU_NSUM));
  return RGPU_SUCCESS;
}

extern "C" int rgpu_system_set_energy(rgpu_system *s, const double *energy8)
{
  if (!s || !energy8) return fail(RGPU_E_INVALID, "bad argument");
  CK(cudaMemcpy(s->energy, energy8, sizeof(double) * RGPU_NE, cudaMemcpyHostToDevice));
  return RGPU_SUCCESS;
}
