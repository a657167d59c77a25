/* CPU restatement of the reference's GCMC energy hot path (FP64).
 *
 * TEST INFRASTRUCTURE: the oracle the GPU kernels are checked against; see
 * oracle.h. Pinned against the reference itself through tests/golden/.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SQR(x) ((x) * (x))

/* NINT of src/utils.h:60 */
static inline double nint(double x) { return (double)(int)(x >= 0.0 ? x + 0.5 : x - 0.5); }

/* ApplyBoundaryCondition, src/potentials.h:232-268: the rectangular branch
 * (:241-245), or the triclinic one (:246-262: to fractional coordinates,
 * each wrapped to its nearest integer, back to Cartesian) */
static inline void min_image(const or_sys *s, double *d)
{
  if (!s->triclinic) {
    for (int c = 0; c < 3; c++) d[c] -= s->box[c] * nint(d[c] * (1.0 / s->box[c]));
    return;
  }
  double t[3];
  for (int r = 0; r < 3; r++) {
    const double f = s->hinv[3 * r] * d[0] + s->hinv[3 * r + 1] * d[1] + s->hinv[3 * r + 2] * d[2];
    t[r] = f - nint(f);
  }
  for (int r = 0; r < 3; r++) d[r] = s->hm[3 * r] * t[0] + s->hm[3 * r + 1] * t[1] + s->hm[3 * r + 2] * t[2];
}

/* the point of fractional coordinates u in the box (ConvertFromABCtoXYZ,
 * src/potentials.c:5548) */
static inline void box_point(const or_sys *s, const double *u, double *p)
{
  if (!s->triclinic) {
    for (int c = 0; c < 3; c++) p[c] = s->box[c] * u[c];
    return;
  }
  for (int r = 0; r < 3; r++) p[r] = s->hm[3 * r] * u[0] + s->hm[3 * r + 1] * u[1] + s->hm[3 * r + 2] * u[2];
}

static inline double dist2(const or_sys *s, const double *a, const double *b, double *d)
{
  d[0] = a[0] - b[0];
  d[1] = a[1] - b[1];
  d[2] = a[2] - b[2];
  min_image(s, d);
  return SQR(d[0]) + SQR(d[1]) + SQR(d[2]);
}

/* PotentialValue, LENNARD_JONES case: src/potentials.c:5867-5877 */
double or_lj(const or_sys *s, int ta, int tb, double r2)
{
  int ij = ta * s->ntypes + tb;
  double r3 = s->sig2[ij] / r2;
  r3 = r3 * r3 * r3;
  return 4.0 * s->eps[ij] * (r3 * (r3 - 1.0)) - s->shift[ij];
}

/* PotentialValueCoulombic, EWALD case: src/potentials.c:12471-12472 */
double or_real_ewald(const or_sys *s, double qa, double qb, double r)
{
  return s->coulomb * qa * qb * (erfc(s->alpha * r) / r);
}

/* the framework VDW energy of a type-`type` bead at p from its energy grid;
 * returns 0 (and leaves *e) when that type has none */
static int grid_vdw(const or_sys *s, int type, const double *p, double *e)
{
  if (!s->grid || !s->grid[type]) return 0;
  *e = or_grid_interpolate_cell(s->grid[type], s->grid_npts, s->grid_size, s->grid_shift, s->grid_cell,
                                s->grid_tri ? s->grid_ucm : NULL, s->grid_ucinv, p);
  return 1;
}

/* the framework real-space charge energy of charge q at p from the Coulomb
 * grid (InterpolateCoulombGrid, src/grids.c:1200-1295); 0 when none */
static int grid_coul(const or_sys *s, double q, const double *p, double *e)
{
  if (!s->coul_grid || !s->ewald) return 0;
  *e = q == 0.0 ? 0.0 : q * or_grid_interpolate_cell(s->coul_grid, s->coul_npts, s->coul_size, s->coul_shift,
                                                     s->coul_cell, s->grid_tri ? s->grid_ucm : NULL,
                                                     s->grid_ucinv, p);
  return 1;
}

/* ---------------------------------------------------------------------- */
void or_point_energy(const or_sys *s, int type, double q, const double *p, int exclude,
                     double *out)
{
  double d[3];
  double uv = 0.0, uc = 0.0, av = 0.0, ac = 0.0;
  /* framework VDW: src/framework_energy.c:151-170 (grid: :60-75); charge: :258-279 (grid: :195-198) */
  const int gv = grid_vdw(s, type, p, &uv);
  const int gc = grid_coul(s, q, p, &uc);
  for (int i = 0; i < s->nfw; i++) {
    double r2 = dist2(s, p, s->fw_xyz + 3 * i, d);
    if (!gv && r2 < s->rc2_vdw) uv += or_lj(s, type, s->fw_type[i], r2);
    if (!gc && s->ewald && q != 0.0 && r2 < s->rc2_cc) uc += or_real_ewald(s, q, s->fw_q[i], sqrt(r2));
  }
  /* other adsorbates: src/inter_energy.c:365-388, :455-480 */
  for (int m = 0; m < s->nmol; m++) {
    if (m == exclude) continue;
    for (int a = 0; a < s->natom; a++) {
      const double *pb = s->ads_xyz + 3 * (m * s->natom + a);
      double r2 = dist2(s, p, pb, d);
      if (r2 < s->rc2_vdw) av += or_lj(s, type, s->mol_type[a], r2);
      if (s->ewald && q != 0.0 && r2 < s->rc2_cc) ac += or_real_ewald(s, q, s->mol_q[a], sqrt(r2));
    }
  }
  out[0] = uv; out[1] = uc; out[2] = av; out[3] = ac;
}

/* Sums of |pair term| of or_point_energy: the scale against which the
 * rounding error of a sum of cancelling pair terms is measured. */
void or_point_energy_abs(const or_sys *s, int type, double q, const double *p, int exclude,
                         double *out)
{
  double d[3];
  double uv = 0.0, uc = 0.0, av = 0.0, ac = 0.0;
  for (int i = 0; i < s->nfw; i++) {
    double r2 = dist2(s, p, s->fw_xyz + 3 * i, d);
    if (r2 < s->rc2_vdw) uv += fabs(or_lj(s, type, s->fw_type[i], r2));
    if (s->ewald && q != 0.0 && r2 < s->rc2_cc) uc += fabs(or_real_ewald(s, q, s->fw_q[i], sqrt(r2)));
  }
  for (int m = 0; m < s->nmol; m++) {
    if (m == exclude) continue;
    for (int a = 0; a < s->natom; a++) {
      const double *pb = s->ads_xyz + 3 * (m * s->natom + a);
      double r2 = dist2(s, p, pb, d);
      if (r2 < s->rc2_vdw) av += fabs(or_lj(s, type, s->mol_type[a], r2));
      if (s->ewald && q != 0.0 && r2 < s->rc2_cc) ac += fabs(or_real_ewald(s, q, s->mol_q[a], sqrt(r2)));
    }
  }
  out[0] = uv; out[1] = uc; out[2] = av; out[3] = ac;
}

/* The four difference routines in the order of src/mc_moves.c:1601-1624:
 * CalculateInterVDWEnergyDifferenceAdsorbate (src/inter_energy.c:3071),
 * CalculateInterChargeChargeEnergyDifferenceAdsorbate (:3652),
 * CalculateFrameworkAdsorbateVDWEnergyDifference (src/framework_energy.c:4870),
 * CalculateFrameworkAdsorbateChargeChargeEnergyDifference (:5412).
 * A new-position pair energy >= EnergyOverlapCriteria is an overlap. */
int or_move_delta(const or_sys *s, int m, const double *new_xyz, double *out)
{
  double d[3];
  const double *old_xyz = s->ads_xyz + 3 * m * s->natom;
  double dav = 0.0, dac = 0.0, dhv = 0.0, dhc = 0.0;
  out[0] = out[1] = out[2] = out[3] = 0.0;
  /* adsorbate-adsorbate VDW */
  for (int a = 0; a < s->natom; a++) {
    int ta = s->mol_type[a];
    for (int j = 0; j < s->nmol; j++) {
      if (j == m) continue;
      for (int b = 0; b < s->natom; b++) {
        const double *pb = s->ads_xyz + 3 * (j * s->natom + b);
        double r2 = dist2(s, new_xyz + 3 * a, pb, d);
        if (r2 < s->rc2_vdw) {
          double e = or_lj(s, ta, s->mol_type[b], r2);
          if (e >= s->overlap) return 1;
          dav += e;
        }
        r2 = dist2(s, old_xyz + 3 * a, pb, d);
        if (r2 < s->rc2_vdw) dav -= or_lj(s, ta, s->mol_type[b], r2);
      }
    }
  }
  /* adsorbate-adsorbate charge-charge */
  if (s->ewald) {
    for (int a = 0; a < s->natom; a++) {
      double qa = s->mol_q[a];
      if (qa == 0.0) continue;
      for (int j = 0; j < s->nmol; j++) {
        if (j == m) continue;
        for (int b = 0; b < s->natom; b++) {
          double qb = s->mol_q[b];
          const double *pb = s->ads_xyz + 3 * (j * s->natom + b);
          double r2 = dist2(s, new_xyz + 3 * a, pb, d);
          if (r2 < s->rc2_cc) {
            double e = or_real_ewald(s, qa, qb, sqrt(r2));
            if (e >= s->overlap) return 1;
            dac += e;
          }
          r2 = dist2(s, old_xyz + 3 * a, pb, d);
          if (r2 < s->rc2_cc) dac -= or_real_ewald(s, qa, qb, sqrt(r2));
        }
      }
    }
  }
  /* framework VDW */
  for (int a = 0; a < s->natom; a++) {
    int ta = s->mol_type[a];
    double e;
    if (grid_vdw(s, ta, new_xyz + 3 * a, &e)) {
      if (e >= s->overlap) return 1;
      dhv += e;
      continue;
    }
    for (int i = 0; i < s->nfw; i++) {
      double r2 = dist2(s, new_xyz + 3 * a, s->fw_xyz + 3 * i, d);
      if (r2 < s->rc2_vdw) {
        double e = or_lj(s, ta, s->fw_type[i], r2);
        if (e >= s->overlap) return 1;
        dhv += e;
      }
    }
  }
  for (int a = 0; a < s->natom; a++) {
    int ta = s->mol_type[a];
    double e;
    if (grid_vdw(s, ta, old_xyz + 3 * a, &e)) {
      dhv -= e;
      continue;
    }
    for (int i = 0; i < s->nfw; i++) {
      double r2 = dist2(s, old_xyz + 3 * a, s->fw_xyz + 3 * i, d);
      if (r2 < s->rc2_vdw) dhv -= or_lj(s, ta, s->fw_type[i], r2);
    }
  }
  /* framework charge-charge (grid: src/framework_energy.c:5437-5438, :5506) */
  if (s->ewald && s->coul_grid) {
    for (int a = 0; a < s->natom; a++) {
      double en = 0.0, eo = 0.0;
      grid_coul(s, s->mol_q[a], new_xyz + 3 * a, &en);
      grid_coul(s, s->mol_q[a], old_xyz + 3 * a, &eo);
      dhc += en - eo;
    }
  } else if (s->ewald) {
    for (int a = 0; a < s->natom; a++) {
      double qa = s->mol_q[a];
      if (qa == 0.0) continue;
      for (int i = 0; i < s->nfw; i++) {
        double r2 = dist2(s, new_xyz + 3 * a, s->fw_xyz + 3 * i, d);
        if (r2 < s->rc2_cc) {
          double e = or_real_ewald(s, qa, s->fw_q[i], sqrt(r2));
          if (e >= s->overlap) return 1;
          dhc += e;
        }
      }
    }
    for (int a = 0; a < s->natom; a++) {
      double qa = s->mol_q[a];
      if (qa == 0.0) continue;
      for (int i = 0; i < s->nfw; i++) {
        double r2 = dist2(s, old_xyz + 3 * a, s->fw_xyz + 3 * i, d);
        if (r2 < s->rc2_cc) dhc -= or_real_ewald(s, qa, s->fw_q[i], sqrt(r2));
      }
    }
  }
  out[0] = dhv; out[1] = dav; out[2] = dhc; out[3] = dac;
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Ewald Fourier part */

static double recip_factor(const or_sys *s, const int *k)
{
  /* SetupKVectors, src/ewald.c:560-595: k = 2 pi n / L (orthorhombic), or
   * k = 2 pi H^-T n (triclinic, the inverse box's columns, :562-575) */
  double kx, ky, kz, vol;
  if (!s->triclinic) {
    kx = 2.0 * M_PI * k[0] / s->box[0];
    ky = 2.0 * M_PI * k[1] / s->box[1];
    kz = 2.0 * M_PI * k[2] / s->box[2];
    vol = s->box[0] * s->box[1] * s->box[2];
  } else {
    const double *v = s->hinv;
    kx = 2.0 * M_PI * (k[0] * v[0] + k[1] * v[3] + k[2] * v[6]);
    ky = 2.0 * M_PI * (k[0] * v[1] + k[1] * v[4] + k[2] * v[7]);
    kz = 2.0 * M_PI * (k[0] * v[2] + k[1] * v[5] + k[2] * v[8]);
    vol = s->hm[0] * s->hm[4] * s->hm[8];
  }
  double k2 = kx * kx + ky * ky + kz * kz;
  double pre = (k[0] == 0 ? 2.0 : 4.0) * M_PI / vol;
  return s->coulomb * pre * exp((-0.25 / SQR(s->alpha)) * k2) / k2;
}

/* exp(i k.r) per site for all wave vectors: phase per axis from the
 * fractional coordinate times 2 pi (src/ewald.c:6941-7100) */
static void site_phase(const or_sys *s, const double *p, const int *k, double *re, double *im)
{
  double a;
  if (!s->triclinic) {
    a = 2.0 * M_PI * (k[0] * p[0] / s->box[0] + k[1] * p[1] / s->box[1] + k[2] * p[2] / s->box[2]);
  } else {
    double f[3];
    for (int r = 0; r < 3; r++) f[r] = s->hinv[3 * r] * p[0] + s->hinv[3 * r + 1] * p[1] + s->hinv[3 * r + 2] * p[2];
    a = 2.0 * M_PI * (k[0] * f[0] + k[1] * f[1] + k[2] * f[2]);
  }
  *re = cos(a);
  *im = sin(a);
}

void or_structure_factor(const or_sys *s, int n, const double *q, const double *xyz,
                         double *sk)
{
  for (int kk = 0; kk < s->nk; kk++) {
    const int *k = s->kidx + 3 * kk;
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < n; i++) {
      double re, im;
      site_phase(s, xyz + 3 * i, k, &re, &im);
      sr += q[i] * re;
      si += q[i] * im;
    }
    sk[2 * kk] = sr;
    sk[2 * kk + 1] = si;
  }
}

void or_ewald_setup(or_sys *s)
{
  if (!s->ewald) return;
  for (int kk = 0; kk < s->nk; kk++) s->kfactor[kk] = recip_factor(s, s->kidx + 3 * kk);
  or_structure_factor(s, s->nfw, s->fw_q, s->fw_xyz, s->sk_fw);
  /* EwaldEnergyIon, src/ewald.c:615-724: a unit charge at the origin */
  double e = 0.0;
  for (int kk = 0; kk < s->nk; kk++) e += s->kfactor[kk];
  s->uion = -(e - s->coulomb * s->alpha / sqrt(M_PI));
  double net = 0.0;
  for (int i = 0; i < s->nfw; i++) net += s->fw_q[i];
  s->net_fw = net;
}

/* scale of the Fourier difference: sum over k of the absolute values of the
 * per-k terms of or_ewald_delta (out = {ads scale, host scale}) */
void or_ewald_delta_abs(const or_sys *s, int nold, const double *xold, int nnew,
                        const double *xnew, double *out)
{
  double sa = 0.0, sh = 0.0;
  for (int kk = 0; kk < s->nk; kk++) {
    const int *k = s->kidx + 3 * kk;
    double dr = 0.0, di = 0.0, dm = 0.0;
    for (int o = 0; o < nold + nnew; o++) {
      const double *x = o < nold ? xold + 3 * o * s->natom : xnew + 3 * (o - nold) * s->natom;
      for (int a = 0; a < s->natom; a++) {
        if (s->mol_q[a] == 0.0) continue;
        double re, im;
        site_phase(s, x + 3 * a, k, &re, &im);
        double q = o < nold ? -s->mol_q[a] : s->mol_q[a];
        dr += q * re;
        di += q * im;
        dm += fabs(s->mol_q[a]);
      }
    }
    double f = s->kfactor[kk];
    double so = sqrt(SQR(s->sk_ads[2 * kk]) + SQR(s->sk_ads[2 * kk + 1]));
    double sf = sqrt(SQR(s->sk_fw[2 * kk]) + SQR(s->sk_fw[2 * kk + 1]));
    sa += f * (2.0 * so * dm + dm * dm);
    sh += 2.0 * f * sf * dm;
    (void)dr; (void)di;
  }
  out[0] = sa;
  out[1] = sh;
}

void or_recompute_sk_ads(or_sys *s)
{
  if (!s->ewald) return;
  int n = s->nmol * s->natom;
  double *q = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double net = 0.0;
  for (int m = 0; m < s->nmol; m++)
    for (int a = 0; a < s->natom; a++) {
      q[m * s->natom + a] = s->mol_q[a];
      net += s->mol_q[a];
    }
  or_structure_factor(s, n, q, s->ads_xyz, s->sk_ads);
  s->net_ads = net;
  free(q);
}

/* intramolecular exclusion erf(alpha r)/r over all charged pairs of one
 * molecule (src/ewald.c:7312-7330, exclusion list src/molecule.c:2838-2851) */
static double exclusion_energy(const or_sys *s, const double *xyz)
{
  double e = 0.0;
  for (int a = 0; a < s->natom - 1; a++)
    for (int b = a + 1; b < s->natom; b++) {
      if (s->mol_q[a] == 0.0 || s->mol_q[b] == 0.0) continue;
      double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1],
             dz = xyz[3 * a + 2] - xyz[3 * b + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      e += s->coulomb * s->mol_q[a] * s->mol_q[b] * erf(s->alpha * r) / r;
    }
  return e;
}

static double self_energy(const or_sys *s)
{
  double e = 0.0;
  for (int a = 0; a < s->natom; a++)
    if (s->mol_q[a] != 0.0) e += s->coulomb * SQR(s->mol_q[a]) * s->alpha / sqrt(M_PI);
  return e;
}

static double mol_charge(const or_sys *s)
{
  double q = 0.0;
  for (int a = 0; a < s->natom; a++) q += s->mol_q[a];
  return q;
}

/* CalculateEwaldFourierAdsorbate, src/ewald.c:6859-7567 (charges only) */
void or_ewald_delta(const or_sys *s, int nold, const double *xold, int nnew,
                    const double *xnew, double *out, double *sk_new)
{
  double e_ads = 0.0, e_host = 0.0;
  for (int kk = 0; kk < s->nk; kk++) {
    const int *k = s->kidx + 3 * kk;
    double dr = 0.0, di = 0.0;
    for (int o = 0; o < nold; o++)
      for (int a = 0; a < s->natom; a++) {
        if (s->mol_q[a] == 0.0) continue;
        double re, im;
        site_phase(s, xold + 3 * (o * s->natom + a), k, &re, &im);
        dr -= s->mol_q[a] * re;
        di -= s->mol_q[a] * im;
      }
    for (int o = 0; o < nnew; o++)
      for (int a = 0; a < s->natom; a++) {
        if (s->mol_q[a] == 0.0) continue;
        double re, im;
        site_phase(s, xnew + 3 * (o * s->natom + a), k, &re, &im);
        dr += s->mol_q[a] * re;
        di += s->mol_q[a] * im;
      }
    double sr = s->sk_ads[2 * kk], si = s->sk_ads[2 * kk + 1];
    double nr = sr + dr, ni = si + di;
    double f = s->kfactor[kk];
    e_host += f * (s->sk_fw[2 * kk] * (nr - sr) + s->sk_fw[2 * kk + 1] * (ni - si));
    e_ads += f * (SQR(nr) - SQR(sr) + SQR(ni) - SQR(si));
    if (sk_new) { sk_new[2 * kk] = nr; sk_new[2 * kk + 1] = ni; }
  }
  double excl_new = 0.0, excl_old = 0.0;
  for (int o = 0; o < nnew; o++) excl_new += exclusion_energy(s, xnew + 3 * o * s->natom);
  for (int o = 0; o < nold; o++) excl_old += exclusion_energy(s, xold + 3 * o * s->natom);
  double self = self_energy(s);
  double dq = (nnew - nold) * mol_charge(s);
  double dads = e_ads - (excl_new - excl_old) - (nnew - nold) * self;
  dads += s->uion * SQR(s->net_ads + dq) - s->uion * SQR(s->net_ads);
  double dhost = 2.0 * e_host;
  dhost += 2.0 * s->uion * s->net_fw * (s->net_ads + dq) - 2.0 * s->uion * s->net_fw * s->net_ads;
  out[0] = dads;
  out[1] = dhost;
  out[2] = dq;
}

void or_total_energy(const or_sys *s, double *out)
{
  double hv = 0.0, av = 0.0, hc = 0.0, ac = 0.0, hf = 0.0, af = 0.0;
  double d[3];
  for (int m = 0; m < s->nmol; m++)
    for (int a = 0; a < s->natom; a++) {
      const double *p = s->ads_xyz + 3 * (m * s->natom + a);
      int ta = s->mol_type[a];
      double qa = s->mol_q[a];
      double g, gq;
      const int gv = grid_vdw(s, ta, p, &g);
      if (gv) hv += g;
      const int gc = grid_coul(s, qa, p, &gq);
      if (gc) hc += gq;
      for (int i = 0; i < s->nfw; i++) {
        double r2 = dist2(s, p, s->fw_xyz + 3 * i, d);
        if (!gv && r2 < s->rc2_vdw) hv += or_lj(s, ta, s->fw_type[i], r2);
        if (!gc && s->ewald && qa != 0.0 && r2 < s->rc2_cc) hc += or_real_ewald(s, qa, s->fw_q[i], sqrt(r2));
      }
      for (int j = m + 1; j < s->nmol; j++)
        for (int b = 0; b < s->natom; b++) {
          double r2 = dist2(s, p, s->ads_xyz + 3 * (j * s->natom + b), d);
          if (r2 < s->rc2_vdw) av += or_lj(s, ta, s->mol_type[b], r2);
          if (s->ewald && qa != 0.0 && s->mol_q[b] != 0.0 && r2 < s->rc2_cc)
            ac += or_real_ewald(s, qa, s->mol_q[b], sqrt(r2));
        }
    }
  if (s->ewald) {
    for (int kk = 0; kk < s->nk; kk++) {
      double f = s->kfactor[kk];
      af += f * (SQR(s->sk_ads[2 * kk]) + SQR(s->sk_ads[2 * kk + 1]));
      hf += f * (s->sk_fw[2 * kk] * s->sk_ads[2 * kk] + s->sk_fw[2 * kk + 1] * s->sk_ads[2 * kk + 1]);
    }
    double excl = 0.0;
    for (int m = 0; m < s->nmol; m++) excl += exclusion_energy(s, s->ads_xyz + 3 * m * s->natom);
    af -= excl + s->nmol * self_energy(s);
    af += s->uion * SQR(s->net_ads);
    hf = 2.0 * hf + 2.0 * s->uion * s->net_fw * s->net_ads;
  }
  out[0] = hv; out[1] = av; out[2] = hc; out[3] = ac; out[4] = hf; out[5] = af;
}

/* ---------------------------------------------------------------------- */
/* MT19937-64 (Matsumoto & Nishimura 2004), as seeded and scaled by the
 * reference: src/utils.c:324-378 */
#define MT_NN 312
#define MT_MM 156
#define MT_MATRIX_A 0xB5026F5AA96619E9ULL
#define MT_UM 0xFFFFFFFF80000000ULL
#define MT_LM 0x7FFFFFFFULL

void or_mt_seed(or_mt64 *g, uint64_t seed)
{
  g->mt[0] = seed;
  for (g->mti = 1; g->mti < MT_NN; g->mti++)
    g->mt[g->mti] = 6364136223846793005ULL * (g->mt[g->mti - 1] ^ (g->mt[g->mti - 1] >> 62)) +
                    (uint64_t)g->mti;
}

static uint64_t mt_next(or_mt64 *g)
{
  static const uint64_t mag01[2] = {0ULL, MT_MATRIX_A};
  uint64_t x;
  if (g->mti >= MT_NN) {
    int i;
    for (i = 0; i < MT_NN - MT_MM; i++) {
      x = (g->mt[i] & MT_UM) | (g->mt[i + 1] & MT_LM);
      g->mt[i] = g->mt[i + MT_MM] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    }
    for (; i < MT_NN - 1; i++) {
      x = (g->mt[i] & MT_UM) | (g->mt[i + 1] & MT_LM);
      g->mt[i] = g->mt[i + (MT_MM - MT_NN)] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    }
    x = (g->mt[MT_NN - 1] & MT_UM) | (g->mt[0] & MT_LM);
    g->mt[MT_NN - 1] = g->mt[MT_MM - 1] ^ (x >> 1) ^ mag01[(int)(x & 1ULL)];
    g->mti = 0;
  }
  x = g->mt[g->mti++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= (x >> 43);
  return x;
}

double or_mt_uniform(or_mt64 *g) { return (double)(mt_next(g) >> 11) * (1.0 / 9007199254740991.0); }

double or_rng_mt(void *ctx, int slot)
{
  (void)slot;
  return or_mt_uniform((or_mt64 *)ctx);
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
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

/* One uniform in [0,1) per (seed, system, step, slot): 53 bits from one half
 * of a Philox block; the block counter is (step lo, step hi, slot/2, system). */
double or_philox_uniform(uint64_t seed, uint32_t system, uint64_t step, uint32_t slot)
{
  uint32_t ctr[4] = {(uint32_t)step, (uint32_t)(step >> 32), slot >> 1, system};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  or_philox4x32(ctr, key, o);
  uint32_t hi = (slot & 1) ? o[2] : o[0];
  uint32_t lo = (slot & 1) ? o[3] : o[1];
  uint64_t x = ((uint64_t)hi << 21) ^ (uint64_t)(lo >> 11);
  return (double)x * (1.0 / 9007199254740992.0);
}

typedef struct { uint64_t seed; uint32_t system; uint64_t step; } philox_ctx;
static double rng_philox(void *ctx, int slot)
{
  philox_ctx *c = (philox_ctx *)ctx;
  return or_philox_uniform(c->seed, c->system, c->step, (uint32_t)slot);
}

/* ---------------------------------------------------------------------- */
/* CBMC. Slot numbers name each random draw so that a counter-based stream
 * can serve the same code; the sequential MT stream ignores them and is
 * consumed in the reference's order. */
enum {
  SLOT_MOVE = 0, SLOT_MOLECULE = 1, SLOT_VNEW = 2, SLOT_AXIS = 3, SLOT_ACCEPT = 4,
  SLOT_FIRST_SELECT = 15, SLOT_FIRST = 16,       /* 16 + 3*i + {z,y,x} */
  SLOT_ORIENT_SELECT = 5, SLOT_ORIENT = 64,      /* 64 + 4*i + {X0,Y1,Y2} */
  SLOT_ORIENT_OLD = 128,                          /* retrace of a reinsertion: 128 + 4*i */
  SLOT_SPHERE = 192                               /* discarded sphere vectors */
};
#define MAX_TRIALS 16
#define MAX_ATOMS 8

/* SelectTrialPosition, src/cbmc.c:563-599 */
static int select_trial(const double *bf, const int *ov, int n, double u)
{
  double largest = -DBL_MAX, sum = 0.0, w[MAX_TRIALS];
  for (int i = 0; i < n; i++)
    if (!ov[i] && bf[i] > largest) largest = bf[i];
  for (int i = 0; i < n; i++) {
    w[i] = ov[i] ? 0.0 : exp(bf[i] - largest);
    sum += w[i];
  }
  int sel = 0;
  double cum = w[0], ws = u * sum;
  while (cum < ws) cum += w[++sel];
  return sel;
}

/* RandomNumberOnUnitSphere (src/utils.c:688); for rigid groups the vector is
 * not used but the reference draws it, so the sequential stream must too */
static void discard_sphere(or_rng_fn rng, void *ctx, int trial)
{
  double r1, r2, sq;
  int a = 0;
  do {
    r1 = 2.0 * rng(ctx, SLOT_SPHERE + 2 * (trial * 4 + (a & 3))) - 1.0;
    r2 = 2.0 * rng(ctx, SLOT_SPHERE + 2 * (trial * 4 + (a & 3)) + 1) - 1.0;
    sq = r1 * r1 + r2 * r2;
    a++;
  } while (sq >= 1.0 && a < 64);
}

/* RandomArrayRotationMatrix (Shoemake), src/utils.c:835-874 */
static void random_rotation(double x0, double y1, double y2, double R[3][3])
{
  y1 *= 2.0 * M_PI;
  y2 *= 2.0 * M_PI;
  double r1 = sqrt(1.0 - x0), r2 = sqrt(x0);
  double u0 = cos(y2) * r2, u1 = sin(y1) * r1, u2 = cos(y1) * r1, u3 = sin(y2) * r2;
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

/* energies of one trial configuration of the beads in `beads` (all but the
 * first bead), ComputeExternalEnergies src/cbmc.c:1179-1476: a host VDW
 * energy >= EnergyOverlapCriteria for any bead marks the trial overlapping */
static int trial_energies(const or_sys *s, const double *xyz, int exclude, double *e)
{
  e[0] = e[1] = e[2] = e[3] = 0.0;
  for (int a = 0; a < s->natom; a++) {
    if (a == s->start_bead) continue;
    double pe[4];
    or_point_energy(s, s->mol_type[a], s->mol_q[a], xyz + 3 * a, exclude, pe);
    if (pe[0] >= s->overlap) return 1;
    e[0] += pe[0]; e[1] += pe[1]; e[2] += pe[2]; e[3] += pe[3];
  }
  return 0;
}

/* shared body of GrowMolecule (src/cbmc.c:3056-3181) and RetraceMolecule
 * (:2928-3054) for one rigid group grown from the starting bead.
 * reins: the growth and the retrace of a reinsertion (src/mc_moves.c:4415):
 * molecule m stays excluded while the new configuration is grown; the
 * growth leaves r = w_1(n) - exp(-beta u_1(selected)) in *stored_r, and the
 * retrace evaluates the old first bead alone with w_1(o) = exp(-beta u_1(o))
 * + r (CBMC_RETRACE_REINSERTION, src/cbmc.c:640-641, :750-762). */
static void cbmc_common(const or_sys *s, int retrace, int reins, int m, int nf, int nt, or_rng_fn rng,
                        void *ctx, double *out, double *new_xyz, double *stored_r)
{
  const int sb = s->start_bead, type0 = s->mol_type[sb];
  const double q0 = s->mol_q[sb];
  const int exclude = (retrace || reins) ? m : s->nmol;
  const int nfirst = (retrace && reins) ? 1 : nf;   /* positions evaluated for the first bead */
  const double *old = retrace ? s->ads_xyz + 3 * m * s->natom : NULL;
  double bf[MAX_TRIALS], e1[MAX_TRIALS][4], pos1[MAX_TRIALS][3];
  int ov[MAX_TRIALS];
  int any = 0;
  out[0] = 1.0;
  for (int k = 1; k < 6; k++) out[k] = 0.0;
  /* HandleFirstBead, src/cbmc.c:623-795 */
  for (int i = 0; i < nfirst; i++) {
    if (retrace && i == 0) {
      pos1[0][0] = old[3 * sb]; pos1[0][1] = old[3 * sb + 1]; pos1[0][2] = old[3 * sb + 2];
    } else {
      double u[3];
      u[2] = rng(ctx, SLOT_FIRST + 3 * i + 0);
      u[1] = rng(ctx, SLOT_FIRST + 3 * i + 1);
      u[0] = rng(ctx, SLOT_FIRST + 3 * i + 2);
      box_point(s, u, pos1[i]);      /* src/cbmc.c:655-662 */
    }
    or_point_energy(s, type0, q0, pos1[i], exclude, e1[i]);
    if (e1[i][0] >= s->overlap || e1[i][1] >= s->overlap || e1[i][2] >= s->overlap ||
        e1[i][3] >= s->overlap) {
      ov[i] = 1;
    } else {
      ov[i] = 0;
      any = 1;
      bf[i] = -s->beta * (e1[i][0] + e1[i][2]);      /* LJ_BIASING */
    }
  }
  if (!any) return;
  double w1 = 0.0;
  for (int i = 0; i < nfirst; i++)
    if (!ov[i]) w1 += exp(bf[i]);
  int sel = 0;
  if (!retrace) sel = select_trial(bf, ov, nf, rng(ctx, SLOT_FIRST_SELECT));
  if (reins && !retrace) *stored_r = w1 - exp(bf[sel]);
  if (reins && retrace) w1 += *stored_r;
  double rosen = w1 / (double)nf;
  if (!retrace && rosen < 1e-150) return;   /* MinimumRosenbluthFactor */
  double u[4] = {e1[sel][0], e1[sel][1], e1[sel][2], e1[sel][3]};
  double grown[MAX_ATOMS * 3];
  grown[3 * sb] = pos1[sel][0]; grown[3 * sb + 1] = pos1[sel][1]; grown[3 * sb + 2] = pos1[sel][2];

  if (s->natom > 1) {
    /* Rosen / RosenOld (src/cbmc.c:2762-2926) with the rigid-group branch of
     * GenerateTrialOrientationsSimpleSphere (:1480-1578) */
    double bft[MAX_TRIALS], et[MAX_TRIALS][4], tx[MAX_TRIALS][MAX_ATOMS * 3];
    int ovt[MAX_TRIALS];
    int anyt = 0;
    for (int iu = 0; iu < nt; iu++) {
      if (retrace && iu == 0) {
        for (int a = 0; a < 3 * s->natom; a++) tx[0][a] = old[a];
      } else {
        discard_sphere(rng, ctx, iu);
        const int ob = (retrace && reins) ? SLOT_ORIENT_OLD : SLOT_ORIENT;
        double x0 = rng(ctx, ob + 4 * iu + 0);
        double y1 = rng(ctx, ob + 4 * iu + 1);
        double y2 = rng(ctx, ob + 4 * iu + 2);
        double R[3][3];
        random_rotation(x0, y1, y2, R);
        for (int a = 0; a < s->natom; a++) {
          double c[3];
          for (int d = 0; d < 3; d++) c[d] = s->mol_ref[3 * a + d] - s->mol_ref[3 * sb + d];
          for (int d = 0; d < 3; d++)
            tx[iu][3 * a + d] = grown[3 * sb + d] + c[0] * R[d][0] + c[1] * R[d][1] + c[2] * R[d][2];
        }
      }
      ovt[iu] = trial_energies(s, tx[iu], exclude, et[iu]);
      if (!ovt[iu]) {
        anyt = 1;
        bft[iu] = -s->beta * (et[iu][0] + et[iu][2]);  /* LJ_BIASING */
      } else {
        bft[iu] = 0.0;
      }
    }
    if (!anyt) return;
    double w = 0.0;
    for (int iu = 0; iu < nt; iu++)
      if (!ovt[iu]) w += exp(bft[iu]);
    w /= (double)nt;
    int iw = 0;
    if (!retrace) iw = select_trial(bft, ovt, nt, rng(ctx, SLOT_ORIENT_SELECT));
    rosen *= w;
    if (!retrace && rosen < 1e-150) return;
    for (int k = 0; k < 4; k++) u[k] += et[iw][k];
    for (int a = 0; a < s->natom; a++)
      if (a != sb)
        for (int d = 0; d < 3; d++) grown[3 * a + d] = tx[iw][3 * a + d];
  }
  /* LJ-biasing correction, src/cbmc.c:3171-3178 (and :3044-3051) */
  rosen *= exp(-s->beta * (u[1] + u[3]));
  out[0] = 0.0;
  out[1] = rosen;
  out[2] = u[0]; out[3] = u[2]; out[4] = u[1]; out[5] = u[3];
  if (new_xyz && !retrace)
    for (int a = 0; a < 3 * s->natom; a++) new_xyz[a] = grown[a];
}

void or_cbmc_grow(const or_sys *s, int nf, int nt, or_rng_fn rng, void *ctx, double *out,
                  double *new_xyz)
{
  cbmc_common(s, 0, 0, s->nmol, nf, nt, rng, ctx, out, new_xyz, NULL);
}

void or_cbmc_retrace(const or_sys *s, int m, int nf, int nt, or_rng_fn rng, void *ctx,
                     double *out)
{
  cbmc_common(s, 1, 0, m, nf, nt, rng, ctx, out, NULL, NULL);
}

/* ---------------------------------------------------------------------- */
/* Flexible linear chains. CBMC growth bead by bead from atom 0
 * (GrowMolecule / RetraceMolecule, src/cbmc.c:2928-3181, for a linear
 * chain): bead i >= 1 at the fixed bond length from bead i-1; the bonded
 * part of the trials as the reference draws it (chain_scheme 0, see
 * ref_scheme_angles) or, with chain_scheme 1, each trial's bend angle drawn
 * from sin(theta) exp(-beta U_bend) (Gaussian proposal accepted with
 * probability sin(theta)) and its dihedral from exp(-beta U_torsion)
 * (uniform proposal accepted with exp(-beta (U - min U))). The draws are
 * keyed (stage, bead, trial, draw) in the counter-based stream; the GPU
 * engine uses the same keys. Bend HARMONIC_BEND and torsion TRAPPE_DIHEDRAL
 * as src/internal_energy.c:205, :2324. */
#define CHAIN_SLOT_SEL (1u << 15)
#define CHAIN_SLOT (1u << 16)
#define CHAIN_TRIES 64
/* chain_scheme 0: the shared bend angle's draws sit in the slots of trial
 * REF_THETA_TRIAL from REF_THETA_SLOT on; the torsion choice of trial t in
 * slot REF_TORS_SEL_SLOT; candidate dihedral k of trial t in slot k */
#define MAX_TORS 248
#define REF_TORS_SEL_SLOT 255
#define REF_THETA_TRIAL 15
#define REF_THETA_SLOT 256

static uint32_t chain_slot(int stage, int bead, int trial, int k)
{
  return CHAIN_SLOT + ((((uint32_t)stage * 8u + (uint32_t)bead) * 16u + (uint32_t)trial) << 9) + (uint32_t)k;
}

static double bend_energy(const or_sys *s, double th)
{
  double d = th - s->bend_theta0;
  return 0.5 * s->bend_k * d * d;
}

static double torsion_energy(const or_sys *s, double c)
{
  double c2 = 2.0 * c * c - 1.0, c3 = c * (4.0 * c * c - 3.0);
  return s->torsion[0] + s->torsion[1] * (1.0 + c) + s->torsion[2] * (1.0 - c2) + s->torsion[3] * (1.0 + c3);
}

static double angle3(const double *a, const double *b, const double *c)
{
  double u[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]}, v[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  double cs = (u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) /
              sqrt((u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
  if (cs > 1.0) cs = 1.0;
  if (cs < -1.0) cs = -1.0;
  return acos(cs);
}

static void cross3(const double *a, const double *b, double *o)
{
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static double cos_dihedral(const double *a, const double *b, const double *c, const double *d)
{
  double b1[3], b2[3], b3[3], n1[3], n2[3];
  for (int k = 0; k < 3; k++) { b1[k] = b[k] - a[k]; b2[k] = c[k] - b[k]; b3[k] = d[k] - c[k]; }
  cross3(b1, b2, n1);
  cross3(b2, b3, n2);
  double cs = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) /
              sqrt((n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]) * (n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]));
  if (cs > 1.0) cs = 1.0;
  if (cs < -1.0) cs = -1.0;
  return cs;
}

/* bead at distance L from c with angle theta (b-c-new) and dihedral phi
 * (a-b-c-new); without a, phi is the azimuth about b-c from the coordinate
 * axis least aligned with it */
static void place(const double *a, const double *b, const double *c, double L, double theta, double phi,
                  double *out)
{
  double bc[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  double nb = sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
  for (int k = 0; k < 3; k++) bc[k] /= nb;
  double ref[3] = {0.0, 0.0, 0.0};
  if (a) {
    for (int k = 0; k < 3; k++) ref[k] = b[k] - a[k];
  } else {
    double ax = fabs(bc[0]), ay = fabs(bc[1]), az = fabs(bc[2]);
    if (ax <= ay && ax <= az) ref[0] = 1.0;
    else if (ay <= az) ref[1] = 1.0;
    else ref[2] = 1.0;
  }
  double n[3], m[3];
  cross3(ref, bc, n);
  double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (int k = 0; k < 3; k++) n[k] /= nn;
  cross3(n, bc, m);
  double dx = -L * cos(theta), dy = L * sin(theta) * cos(phi), dz = L * sin(theta) * sin(phi);
  for (int k = 0; k < 3; k++) out[k] = c[k] + dx * bc[k] + dy * m[k] + dz * n[k];
}

static double bonded_energy(const or_sys *s, const double (*x)[3], int i, const double *p)
{
  double e = 0.0;
  if (i >= 2) e += bend_energy(s, angle3(x[i - 2], x[i - 1], p));
  if (i >= 3) e += torsion_energy(s, cos_dihedral(x[i - 3], x[i - 2], x[i - 1], p));
  return e;
}

static double intra_lj(const or_sys *s, const double (*x)[3], int i, const double *p)
{
  double e = 0.0;
  for (int j = 0; j + 4 <= i; j++) {
    double d[3] = {p[0] - x[j][0], p[1] - x[j][1], p[2] - x[j][2]};
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 < s->rc2_vdw) e += or_lj(s, s->mol_type[i], s->mol_type[j], r2);
  }
  return e;
}

double or_intra_energy(const or_sys *s)
{
  double e = 0.0;
  if (!s->flexible) return 0.0;
  for (int m = 0; m < s->nmol; m++) {
    const double(*x)[3] = (const double(*)[3])(s->ads_xyz + 3 * m * s->natom);
    for (int i = 1; i < s->natom; i++) e += bonded_energy(s, x, i, x[i]) + intra_lj(s, x, i, x[i]);
  }
  return e;
}

static double chain_u(const philox_ctx *c, int stage, int i, int t, int k)
{
  return or_philox_uniform(c->seed, c->system, c->step, chain_slot(stage, i, t, k));
}

/* trial position of bead i >= 1 after beads x[0..i-1]; returns its bonded energy */
static double chain_trial(const or_sys *s, const double (*x)[3], int i, const philox_ctx *c, int stage, int t,
                          double *p)
{
  int k = 0;
  if (i == 1) {
    double z = 2.0 * chain_u(c, stage, i, t, 0) - 1.0;
    double psi = 2.0 * M_PI * chain_u(c, stage, i, t, 1);
    double r = sqrt(fmax(0.0, 1.0 - z * z));
    p[0] = x[0][0] + s->bond * r * cos(psi);
    p[1] = x[0][1] + s->bond * r * sin(psi);
    p[2] = x[0][2] + s->bond * z;
    return 0.0;
  }
  double theta = s->bend_theta0;
  for (int a = 0; a < CHAIN_TRIES; a++, k += 3) {
    double u1 = chain_u(c, stage, i, t, k), u2 = chain_u(c, stage, i, t, k + 1), u3 = chain_u(c, stage, i, t, k + 2);
    double th = s->bend_theta0 + s->bend_sigma * sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
    if (th > 0.0 && th < M_PI && u3 < sin(th)) {
      theta = th;
      break;
    }
  }
  k = 3 * CHAIN_TRIES;
  double phi;
  if (i == 2) {
    phi = 2.0 * M_PI * chain_u(c, stage, i, t, k) - M_PI;
  } else {
    phi = M_PI;
    for (int a = 0; a < CHAIN_TRIES; a++, k += 2) {
      double f = 2.0 * M_PI * chain_u(c, stage, i, t, k) - M_PI;
      if (chain_u(c, stage, i, t, k + 1) < exp(-s->beta * (torsion_energy(s, cos(f)) - s->torsion_min))) {
        phi = f;
        break;
      }
    }
  }
  place(i >= 3 ? x[i - 3] : NULL, x[i - 2], x[i - 1], s->bond, theta, phi, p);
  return bonded_energy(s, x, i, p);
}

/* The reference's bonded trials (chain_scheme 0), GenerateTrialOrientationsMCScheme
 * src/cbmc.c:1580-2480 for a linear chain, bead i >= 2 grown from bead i-1:
 * - one bend angle for all trials of the step (the internal Metropolis
 *   chain of src/cbmc.c:1822-2106 samples sin(theta) exp(-beta U_bend);
 *   here the same distribution is drawn directly); a retrace keeps the old
 *   bead's angle (src/cbmc.c:1661, the chain runs only when growing);
 * - per trial, `ntors` rotations about the bond (i-2)-(i-1) by uniform
 *   angles (src/cbmc.c:2361-2399), i.e. uniform dihedrals, one of them
 *   chosen by its torsion Boltzmann factor (SelectTrialPosition,
 *   src/cbmc.c:2403-2410); a retrace's trial 0 keeps the old dihedral as
 *   its first candidate (src/cbmc.c:2376-2377). Without a torsion (i = 2)
 *   the choice is uniform (src/cbmc.c:2410);
 * - the trial's torsion Rosenbluth factor (src/cbmc.c:2401). The reference
 *   computes it with ComputeNormalizedRosenbluthWeight, whose loop runs over
 *   the global NumberOfTrialPositions, not over its argument (src/cbmc.c:548):
 *   it is the mean over the first `nt` candidates only, nt = the CBMC trials
 *   per bead. This is kept, because it sets the reference's GCMC loadings.
 * Fills theta_sh, and per trial t the dihedral phi[t] (unused for the old
 * trial 0 of a retrace) and the torsion factor wt[t]. */
static void ref_scheme_angles(const or_sys *s, const double (*x)[3], int i, int retrace, const double *old, int nt,
                              const philox_ctx *c, int stage, double *theta_sh, double *phi, double *wt)
{
  if (retrace) {
    *theta_sh = angle3(x[i - 2], x[i - 1], old);
  } else {
    double th = s->bend_theta0;
    for (int a = 0; a < CHAIN_TRIES; a++) {
      int k = REF_THETA_SLOT + 3 * a;
      double u1 = chain_u(c, stage, i, REF_THETA_TRIAL, k), u2 = chain_u(c, stage, i, REF_THETA_TRIAL, k + 1);
      double u3 = chain_u(c, stage, i, REF_THETA_TRIAL, k + 2);
      double t = s->bend_theta0 + s->bend_sigma * sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
      if (t > 0.0 && t < M_PI && u3 < sin(t)) {
        th = t;
        break;
      }
    }
    *theta_sh = th;
  }
  for (int t = 0; t < nt; t++) {
    wt[t] = 1.0;
    if (i == 2) {
      phi[t] = 2.0 * M_PI * chain_u(c, stage, i, t, 0) - M_PI;
      continue;
    }
    double bf[MAX_TORS], f[MAX_TORS];
    for (int k = 0; k < s->ntors; k++) {
      double cs;
      if (retrace && t == 0 && k == 0) {
        cs = cos_dihedral(x[i - 3], x[i - 2], x[i - 1], old);
        f[k] = 0.0;
      } else {
        f[k] = 2.0 * M_PI * chain_u(c, stage, i, t, k) - M_PI;
        cs = cos(f[k]);
      }
      bf[k] = -s->beta * torsion_energy(s, cs);
    }
    double sum = 0.0;
    for (int k = 0; k < nt && k < s->ntors; k++) sum += exp(bf[k]);
    wt[t] = sum / (double)nt;
    int sel = 0;
    if (!(retrace && t == 0)) {
      double largest = -DBL_MAX, tot = 0.0;
      for (int k = 0; k < s->ntors; k++)
        if (bf[k] > largest) largest = bf[k];
      for (int k = 0; k < s->ntors; k++) tot += exp(bf[k] - largest);
      double ws = chain_u(c, stage, i, t, REF_TORS_SEL_SLOT) * tot, cum = exp(bf[0] - largest);
      while (cum < ws && sel < s->ntors - 1) cum += exp(bf[++sel] - largest);
    }
    phi[t] = f[sel];
  }
}

/* CBMC growth (retrace = 0) or retrace of a chain; exclude = molecule left
 * out of the adsorbate sums, m = molecule retraced. out = {fail, W, host VDW,
 * adsorbate VDW, intramolecular}; x receives the chosen beads. */
static void chain_grow(const or_sys *s, int retrace, int stage, int m, int exclude, int nf, int nt,
                       const philox_ctx *c, double *out, double (*x)[3])
{
  const int na = s->natom;
  double rosen = 1.0, hv = 0.0, av = 0.0, intra = 0.0;
  out[0] = 1.0;
  for (int i = 0; i < na; i++) {
    const int k = i == 0 ? nf : nt;
    double w[MAX_TRIALS], pe[MAX_TRIALS][4], lj[MAX_TRIALS], ub[MAX_TRIALS], pos[MAX_TRIALS][3];
    double wt[MAX_TRIALS], phi[MAX_TRIALS], theta_sh = 0.0;
    const int ref = s->chain_scheme == 0 && i >= 2;
    if (ref)
      ref_scheme_angles(s, (const double(*)[3])x, i, retrace, s->ads_xyz + 3 * (m * na + i), k, c, stage, &theta_sh,
                        phi, wt);
    int any = 0;
    for (int t = 0; t < k; t++) {
      ub[t] = 0.0;
      if (!ref) wt[t] = 1.0;
      if (retrace && t == 0) {
        for (int d = 0; d < 3; d++) pos[0][d] = s->ads_xyz[3 * (m * na + i) + d];
        ub[0] = bonded_energy(s, (const double(*)[3])x, i, pos[0]);
      } else if (i == 0) {
        double u[3];
        for (int d = 0; d < 3; d++) u[d] = chain_u(c, stage, 0, t, d);
        box_point(s, u, pos[t]);
      } else if (ref) {
        place(i >= 3 ? x[i - 3] : NULL, x[i - 2], x[i - 1], s->bond, theta_sh, phi[t], pos[t]);
        ub[t] = bonded_energy(s, (const double(*)[3])x, i, pos[t]);
      } else {
        ub[t] = chain_trial(s, (const double(*)[3])x, i, c, stage, t, pos[t]);
      }
      or_point_energy(s, s->mol_type[i], s->mol_q[i], pos[t], exclude, pe[t]);
      lj[t] = intra_lj(s, (const double(*)[3])x, i, pos[t]);
      int ov = pe[t][0] >= s->overlap || pe[t][1] >= s->overlap || pe[t][2] >= s->overlap ||
               pe[t][3] >= s->overlap || lj[t] >= s->overlap;
      w[t] = ov ? 0.0 : exp(-s->beta * (pe[t][0] + pe[t][2] + lj[t]));
      if (!ov) any = 1;
    }
    double wsum = 0.0;
    for (int t = 0; t < k; t++) wsum += w[t];
    int sel = 0;
    if (!retrace && any) {
      double target = or_philox_uniform(c->seed, c->system, c->step, CHAIN_SLOT_SEL + stage * 8 + i) * wsum;
      double cum = w[0];
      while (cum < target && sel < k - 1) cum += w[++sel];
    }
    rosen *= wsum / (double)k * wt[sel];
    if (!any || (!retrace && rosen < 1e-150)) return;
    hv += pe[sel][0];
    av += pe[sel][2];
    intra += lj[sel] + ub[sel];
    for (int d = 0; d < 3; d++) x[i][d] = pos[sel][d];
  }
  out[0] = 0.0;
  out[1] = rosen;
  out[2] = hv;
  out[3] = av;
  out[4] = intra;
}

/* ---------------------------------------------------------------------- */
/* Energy grids */

/* CalculateDerivativesAtPositionVDW (src/framework_hessian.c:63-109) with the
 * LJ branch of PotentialThirdDerivative (src/potentials.c:10959-10990).
 * out = {U, dU/dx, dU/dy, dU/dz, d2U/dxdy, d2U/dxdz, d2U/dydz, d3U/dxdydz} */
void or_grid_derivatives(const or_sys *s, int type, const double *p, double *o)
{
  double d[3];
  for (int k = 0; k < 8; k++) o[k] = 0.0;
  for (int i = 0; i < s->nfw; i++) {
    double r2 = dist2(s, p, s->fw_xyz + 3 * i, d);
    if (r2 >= s->rc2_vdw) continue;
    int ij = type * s->ntypes + s->fw_type[i];
    double e = s->eps[ij];
    double r3 = s->sig2[ij] / r2;
    r3 = r3 * r3 * r3;
    double U = 4.0 * e * (r3 * (r3 - 1.0)) - s->shift[ij];
    double DF = 24.0 * e * (r3 * (1.0 - 2.0 * r3)) / r2;
    double DDF = 96.0 * e * (r3 * (7.0 * r3 - 2.0)) / SQR(r2);
    double DDDF = 384.0 * e * (r3 * (5.0 - 28.0 * r3)) / SQR(SQR(r2));
    o[0] += U;
    o[1] += d[0] * DF;
    o[2] += d[1] * DF;
    o[3] += d[2] * DF;
    o[4] += DDF * d[0] * d[1];
    o[5] += DDF * d[0] * d[2];
    o[6] += DDF * d[1] * d[2];
    o[7] += DDDF * d[0] * d[1] * d[2];
  }
}

/* MakeGrid, src/grids.c:512-585: point (i,j,k) at i*size/n + shift, values
 * capped above EnergyOverlapCriteria and stored in "unit cube" scaling.
 * Layout: grid[m][i][j][k] for m=0..7 (the file plane order of
 * src/grids.c:734-738). */
void or_grid_build(const or_sys *s, int type, const int npts[3], const double size[3],
                   const double shift[3], float *grid)
{
  const int nx = npts[0] + 1, ny = npts[1] + 1, nz = npts[2] + 1;
  const size_t plane = (size_t)nx * ny * nz;
  double delta[3];
  for (int c = 0; c < 3; c++) delta[c] = size[c] / (double)npts[c];
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        double p[3] = {i * size[0] / npts[0] + shift[0], j * size[1] / npts[1] + shift[1],
                       k * size[2] / npts[2] + shift[2]};
        double o[8];
        or_grid_derivatives(s, type, p, o);
        if (o[0] > s->overlap) {
          o[0] = 2.0 * s->overlap;
          for (int c = 1; c <= 3; c++) {
            if (o[c] > s->overlap) o[c] = s->overlap;
            if (o[c] < -s->overlap) o[c] = -s->overlap;
          }
          o[4] = o[5] = o[6] = o[7] = 0.0;
        }
        size_t idx = ((size_t)i * ny + j) * nz + k;
        grid[0 * plane + idx] = (float)o[0];
        grid[1 * plane + idx] = (float)o[1] * delta[0];
        grid[2 * plane + idx] = (float)o[2] * delta[1];
        grid[3 * plane + idx] = (float)o[3] * delta[2];
        grid[4 * plane + idx] = (float)o[4] * (delta[0] * delta[1]);
        grid[5 * plane + idx] = (float)o[5] * (delta[0] * delta[2]);
        grid[6 * plane + idx] = (float)o[6] * (delta[1] * delta[2]);
        grid[7 * plane + idx] = (float)o[7] * (delta[0] * delta[1] * delta[2]);
      }
}

/* Cubic Hermite basis on [0,1]: value p0,p1 and slope d0,d1 */
static inline void hermite(double t, double *h)
{
  double t2 = t * t, t3 = t2 * t;
  h[0] = 1.0 - 3.0 * t2 + 2.0 * t3;   /* p0 */
  h[1] = 3.0 * t2 - 2.0 * t3;         /* p1 */
  h[2] = t - 2.0 * t2 + t3;           /* d0 */
  h[3] = -t2 + t3;                    /* d1 */
}

/* The real-space Ewald term f(r) = K q erfc(alpha r) / r of a unit probe
 * charge and its radial derivative factors: d f/dx_i = x_i DF,
 * d2 f/dx_i dx_j = x_i x_j DDF (+ DF for i = j), d3 f/dx dy dz = x y z DDDF
 * (src/framework_hessian.c:142-160). */
void or_grid_derivatives_real(const or_sys *s, const double *p, double *o)
{
  double d[3];
  double rmin = 1e300;
  for (int k = 0; k < 8; k++) o[k] = 0.0;
  const double a2 = s->alpha * s->alpha, c = 2.0 * s->alpha / sqrt(M_PI);
  for (int i = 0; i < s->nfw; i++) {
    double r2 = dist2(s, p, s->fw_xyz + 3 * i, d);
    if (r2 >= s->rc2_cc) continue;
    double r = sqrt(r2);
    if (r < rmin) rmin = r;
    double kq = s->coulomb * s->fw_q[i];
    double e = erfc(s->alpha * r), g = c * r * exp(-a2 * r2), x = a2 * r2;
    double F = kq * e / r;
    double DF = -kq * (g + e) / (r * r2);
    double DDF = kq * (g * (3.0 + 2.0 * x) + 3.0 * e) / (r2 * r2 * r);
    double DDDF = -kq * (g * (15.0 + 10.0 * x + 4.0 * x * x) + 15.0 * e) / (r2 * r2 * r2 * r);
    o[0] += F;
    o[1] += d[0] * DF;
    o[2] += d[1] * DF;
    o[3] += d[2] * DF;
    o[4] += DDF * d[0] * d[1];
    o[5] += DDF * d[0] * d[2];
    o[6] += DDF * d[1] * d[2];
    o[7] += DDDF * d[0] * d[1] * d[2];
  }
  o[8] = rmin;
}

/* src/grids.c:586-690: as or_grid_build, capped where the value exceeds the
 * overlap criterion or a framework atom is within 1 A (:656-668) */
void or_grid_build_coulomb(const or_sys *s, const int npts[3], const double size[3], const double shift[3],
                           float *grid)
{
  const int nx = npts[0] + 1, ny = npts[1] + 1, nz = npts[2] + 1;
  const size_t plane = (size_t)nx * ny * nz;
  double delta[3];
  for (int c = 0; c < 3; c++) delta[c] = size[c] / (double)npts[c];
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        double p[3] = {i * size[0] / npts[0] + shift[0], j * size[1] / npts[1] + shift[1],
                       k * size[2] / npts[2] + shift[2]};
        double o[9];
        or_grid_derivatives_real(s, p, o);
        if (o[0] > s->overlap || o[8] < 1.0) {
          o[0] = 2.0 * s->overlap;
          for (int c = 1; c <= 3; c++) {
            if (o[c] > s->overlap) o[c] = s->overlap;
            if (o[c] < -s->overlap) o[c] = -s->overlap;
          }
          o[4] = o[5] = o[6] = o[7] = 0.0;
        }
        size_t idx = ((size_t)i * ny + j) * nz + k;
        grid[0 * plane + idx] = (float)o[0];
        grid[1 * plane + idx] = (float)o[1] * delta[0];
        grid[2 * plane + idx] = (float)o[2] * delta[1];
        grid[3 * plane + idx] = (float)o[3] * delta[2];
        grid[4 * plane + idx] = (float)o[4] * (delta[0] * delta[1]);
        grid[5 * plane + idx] = (float)o[5] * (delta[0] * delta[2]);
        grid[6 * plane + idx] = (float)o[6] * (delta[1] * delta[2]);
        grid[7 * plane + idx] = (float)o[7] * (delta[0] * delta[1] * delta[2]);
      }
}

/* InterpolateVDWGrid (src/grids.c:979-1077). The reference solves for the 64
 * tricubic coefficients with the Lekien-Marsden matrix and evaluates the
 * polynomial; the same interpolant is the tensor product of 1D cubic Hermite
 * bases over the 8 stored derivatives (f, f_x, f_y, f_z, f_xy, f_xz, f_yz,
 * f_xyz at the 8 corners), which is what is evaluated here. */
double or_grid_interpolate(const float *grid, const int npts[3], const double size[3],
                           const double shift[3], const double cell[3], const double *pin)
{
  return or_grid_interpolate_cell(grid, npts, size, shift, cell, NULL, NULL, pin);
}

double or_grid_interpolate_cell(const float *grid, const int npts[3], const double size[3], const double shift[3],
                                const double cell[3], const double *ucm, const double *ucinv, const double *pin)
{
  double p[3];
  if (!ucm) {
    /* the RECTANGULAR branch, src/grids.c:995-1002 */
    for (int c = 0; c < 3; c++) {
      p[c] = pin[c] - cell[c] * nint(pin[c] / cell[c]);
      if (p[c] < 0.0) p[c] += cell[c];
    }
  } else {
    /* the TRICLINIC branch, src/grids.c:1004-1021 */
    double f[3];
    for (int r = 0; r < 3; r++) {
      f[r] = ucinv[3 * r] * pin[0] + ucinv[3 * r + 1] * pin[1] + ucinv[3 * r + 2] * pin[2];
      f[r] -= nint(f[r]);
      if (f[r] < 0.0) f[r] += 1.0;
    }
    for (int r = 0; r < 3; r++) p[r] = ucm[3 * r] * f[0] + ucm[3 * r + 1] * f[1] + ucm[3 * r + 2] * f[2];
  }
  const int nx = npts[0] + 1, ny = npts[1] + 1, nz = npts[2] + 1;
  const size_t plane = (size_t)nx * ny * nz;
  double sc[3], r[3];
  int i0[3];
  for (int c = 0; c < 3; c++) {
    sc[c] = ((p[c] - shift[c]) / size[c]) * (double)npts[c];
    /* a point on the upper face (p == cell) uses the last cell at r = 1 */
    i0[c] = (int)sc[c];
    if (i0[c] > npts[c] - 1) i0[c] = npts[c] - 1;
    if (i0[c] < 0) i0[c] = 0;
    r[c] = sc[c] - i0[c];
  }
  /* cap, src/grids.c:1058-1060 */
  for (int dx = 0; dx < 2; dx++)
    for (int dy = 0; dy < 2; dy++)
      for (int dz = 0; dz < 2; dz++) {
        size_t idx = ((size_t)(i0[0] + dx) * ny + (i0[1] + dy)) * nz + (i0[2] + dz);
        if (grid[idx] > 1e10f) return 1e8;
      }
  double hx[4], hy[4], hz[4];
  hermite(r[0], hx);
  hermite(r[1], hy);
  hermite(r[2], hz);
  /* derivative plane for (x order, y order, z order) in {0,1}^3 */
  static const int plane_of[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
  double v = 0.0;
  for (int dx = 0; dx < 2; dx++)
    for (int dy = 0; dy < 2; dy++)
      for (int dz = 0; dz < 2; dz++) {
        size_t idx = ((size_t)(i0[0] + dx) * ny + (i0[1] + dy)) * nz + (i0[2] + dz);
        for (int ox = 0; ox < 2; ox++)
          for (int oy = 0; oy < 2; oy++)
            for (int oz = 0; oz < 2; oz++) {
              double f = grid[plane_of[ox][oy][oz] * plane + idx];
              v += f * hx[2 * ox + dx] * hy[2 * oy + dy] * hz[2 * oz + dz];
            }
      }
  return v;
}

/* ---------------------------------------------------------------------- */
/* GCMC engine on the counter-based stream. Move semantics follow
 * src/mc_moves.c: TranslationMoveAdsorbate (:1529-1762),
 * RotationMoveAdsorbate (:2636), SwapAddAdsorbateMove (:6941-7140),
 * SwapRemoveAdsorbateMove (:7150-7350). */

static void rotate_axis(double *c, int axis, double th)
{
  /* RotationAround{X,Y,Z}Axis, src/utils.c:876-936 */
  double cs = cos(th), sn = sin(th);
  double x = c[0], y = c[1], z = c[2];
  if (axis == 0) { c[1] = cs * y + sn * z; c[2] = -sn * y + cs * z; }
  else if (axis == 1) { c[0] = cs * x - sn * z; c[2] = sn * x + cs * z; }
  else { c[0] = cs * x + sn * y; c[1] = -sn * x + cs * y; }
}

void or_mc_run(or_sys *s, const or_mc_params *p, or_mc_state *st, uint64_t step0,
               long long nsteps)
{
  const int na = s->natom;
  double *nk = s->ewald ? (double *)malloc(sizeof(double) * 2 * s->nk) : NULL;
  for (long long it = 0; it < nsteps; it++) {
    philox_ctx ctx = {p->seed, p->system, step0 + (uint64_t)it};
    double u0 = rng_philox(&ctx, SLOT_MOVE);
    int mv = 0;
    while (mv < 5 && u0 >= p->cum[mv]) mv++;
    if (mv == 0 || mv == 1) {
      if (s->nmol == 0 || (mv == 1 && na == 1)) continue;
      st->moves++;
      st->attempts[mv]++;
      int m = (int)(rng_philox(&ctx, SLOT_MOLECULE) * s->nmol);
      if (m >= s->nmol) m = s->nmol - 1;
      double vnew = 2.0 * rng_philox(&ctx, SLOT_VNEW) - 1.0;
      int axis = (int)(3.0 * rng_philox(&ctx, SLOT_AXIS));
      if (axis > 2) axis = 2;
      double nx[MAX_ATOMS * 3];
      const double *ox = s->ads_xyz + 3 * m * na;
      if (mv == 0) {
        for (int a = 0; a < 3 * na; a++) nx[a] = ox[a];
        for (int a = 0; a < na; a++) nx[3 * a + axis] += vnew * p->max_translation;
      } else {
        int sb = s->start_bead;
        for (int a = 0; a < na; a++) {
          double c[3] = {ox[3 * a] - ox[3 * sb], ox[3 * a + 1] - ox[3 * sb + 1],
                         ox[3 * a + 2] - ox[3 * sb + 2]};
          rotate_axis(c, axis, vnew * p->max_rotation);
          for (int d = 0; d < 3; d++) nx[3 * a + d] = c[d] + ox[3 * sb + d];
        }
      }
      double dl[4], de[3] = {0.0, 0.0, 0.0};
      if (or_move_delta(s, m, nx, dl)) continue;
      if (s->ewald) or_ewald_delta(s, 1, ox, 1, nx, de, nk);
      double du = dl[0] + dl[1] + dl[2] + dl[3] + de[0] + de[1];
      if (rng_philox(&ctx, SLOT_ACCEPT) < exp(-s->beta * du)) {
        st->accepted[mv]++;
        for (int a = 0; a < 3 * na; a++) s->ads_xyz[3 * m * na + a] = nx[a];
        if (s->ewald) memcpy(s->sk_ads, nk, sizeof(double) * 2 * s->nk);
        st->u[0] += dl[0]; st->u[1] += dl[1]; st->u[2] += dl[2]; st->u[3] += dl[3];
        st->u[4] += de[1]; st->u[5] += de[0];
      }
    } else if (s->flexible && mv >= 2) {
      /* flexible chains: CBMC insertion, deletion, reinsertion, Widom */
      if (mv == 4 && s->nmol == 0) continue;
      st->moves++;
      st->attempts[mv]++;
      if (mv == 5) st->widom_n += 1.0;
      if (mv == 2 && s->nmol >= s->maxmol) continue;
      if (mv == 3 && s->nmol == 0) continue;
      int m = s->nmol;
      if (mv == 3 || mv == 4) {
        m = (int)(rng_philox(&ctx, SLOT_MOLECULE) * s->nmol);
        if (m >= s->nmol) m = s->nmol - 1;
      }
      double o[5], x[MAX_ATOMS][3];
      if (mv == 2 || mv == 5) {
        chain_grow(s, 0, 0, s->nmol, s->nmol, p->ntrial_first, p->ntrial, &ctx, o, x);
        if (o[0] != 0.0) continue;
        if (mv == 5) {
          st->widom_sum += o[1];
          continue;
        }
        if (rng_philox(&ctx, SLOT_ACCEPT) < o[1] * p->fugacity_beta_v / (1.0 + s->nmol)) {
          st->accepted[2]++;
          for (int a = 0; a < na; a++)
            for (int d = 0; d < 3; d++) s->ads_xyz[3 * (s->nmol * na + a) + d] = x[a][d];
          s->nmol++;
          st->u[0] += o[2]; st->u[1] += o[3]; st->u_intra += o[4];
        }
      } else if (mv == 3) {
        chain_grow(s, 1, 1, m, m, p->ntrial_first, p->ntrial, &ctx, o, x);
        if (o[0] != 0.0) continue;
        if (rng_philox(&ctx, SLOT_ACCEPT) < (double)s->nmol / (o[1] * p->fugacity_beta_v)) {
          st->accepted[3]++;
          int last = s->nmol - 1;
          for (int a = 0; a < 3 * na; a++) s->ads_xyz[3 * m * na + a] = s->ads_xyz[3 * last * na + a];
          s->nmol--;
          st->u[0] -= o[2]; st->u[1] -= o[3]; st->u_intra -= o[4];
        }
      } else {
        double on[5], xn[MAX_ATOMS][3];
        chain_grow(s, 0, 0, m, m, p->ntrial_first, p->ntrial, &ctx, on, xn);
        if (on[0] != 0.0) continue;
        chain_grow(s, 1, 1, m, m, p->ntrial_first, p->ntrial, &ctx, o, x);
        if (o[0] != 0.0) continue;
        if (rng_philox(&ctx, SLOT_ACCEPT) < on[1] / o[1]) {
          st->accepted[4]++;
          for (int a = 0; a < na; a++)
            for (int d = 0; d < 3; d++) s->ads_xyz[3 * (m * na + a) + d] = xn[a][d];
          st->u[0] += on[2] - o[2]; st->u[1] += on[3] - o[3]; st->u_intra += on[4] - o[4];
        }
      }
    } else if (mv == 2) {
      st->moves++;
      st->attempts[2]++;
      if (s->nmol >= s->maxmol) continue;
      double o[6], nx[MAX_ATOMS * 3];
      or_cbmc_grow(s, p->ntrial_first, p->ntrial, rng_philox, &ctx, o, nx);
      if (o[0] != 0.0) continue;
      double w = o[1], de[3] = {0.0, 0.0, 0.0};
      if (s->ewald) {
        or_ewald_delta(s, 0, NULL, 1, nx, de, nk);
        w *= exp(-s->beta * (de[0] + de[1]));
      }
      if (rng_philox(&ctx, SLOT_ACCEPT) < w * p->fugacity_beta_v / (1.0 + s->nmol)) {
        st->accepted[2]++;
        for (int a = 0; a < 3 * na; a++) s->ads_xyz[3 * s->nmol * na + a] = nx[a];
        s->nmol++;
        if (s->ewald) {
          memcpy(s->sk_ads, nk, sizeof(double) * 2 * s->nk);
          s->net_ads += de[2];
        }
        st->u[0] += o[2]; st->u[1] += o[3]; st->u[2] += o[4]; st->u[3] += o[5];
        st->u[4] += de[1]; st->u[5] += de[0];
      }
    } else if (mv == 4) {
      /* ReinsertionAdsorbateMove, src/mc_moves.c:4415-4600 */
      if (s->nmol == 0) continue;
      st->moves++;
      st->attempts[4]++;
      int m = (int)(rng_philox(&ctx, SLOT_MOLECULE) * s->nmol);
      if (m >= s->nmol) m = s->nmol - 1;
      double on[6], oo[6], nx[MAX_ATOMS * 3], r = 0.0, de[3] = {0.0, 0.0, 0.0};
      cbmc_common(s, 0, 1, m, p->ntrial_first, p->ntrial, rng_philox, &ctx, on, nx, &r);
      if (on[0] != 0.0) continue;
      cbmc_common(s, 1, 1, m, p->ntrial_first, p->ntrial, rng_philox, &ctx, oo, NULL, &r);
      if (oo[0] != 0.0) continue;
      const double *ox = s->ads_xyz + 3 * m * na;
      double pre = 1.0;
      if (s->ewald) {
        or_ewald_delta(s, 1, ox, 1, nx, de, nk);
        pre = exp(-s->beta * (de[0] + de[1]));
      }
      if (rng_philox(&ctx, SLOT_ACCEPT) < pre * on[1] / oo[1]) {
        st->accepted[4]++;
        for (int a = 0; a < 3 * na; a++) s->ads_xyz[3 * m * na + a] = nx[a];
        if (s->ewald) memcpy(s->sk_ads, nk, sizeof(double) * 2 * s->nk);
        for (int k = 0; k < 4; k++) st->u[k] += on[2 + k] - oo[2 + k];
        st->u[4] += de[1]; st->u[5] += de[0];
      }
    } else if (mv == 5) {
      /* WidomAdsorbateMove, src/mc_moves.c:7844-8030: Rosenbluth weight of a
       * test insertion, no change of state */
      st->moves++;
      st->attempts[5]++;
      st->widom_n += 1.0;
      double o[6], nx[MAX_ATOMS * 3], de[3] = {0.0, 0.0, 0.0};
      or_cbmc_grow(s, p->ntrial_first, p->ntrial, rng_philox, &ctx, o, nx);
      if (o[0] != 0.0) continue;
      double w = o[1];
      if (s->ewald) {
        or_ewald_delta(s, 0, NULL, 1, nx, de, nk);
        w *= exp(-s->beta * (de[0] + de[1]));
      }
      st->widom_sum += w;
    } else {
      st->moves++;
      st->attempts[3]++;
      if (s->nmol == 0) continue;
      int m = (int)(rng_philox(&ctx, SLOT_MOLECULE) * s->nmol);
      if (m >= s->nmol) m = s->nmol - 1;
      double o[6], de[3] = {0.0, 0.0, 0.0};
      or_cbmc_retrace(s, m, p->ntrial_first, p->ntrial, rng_philox, &ctx, o);
      if (o[0] != 0.0) continue;
      double w = o[1];
      const double *ox = s->ads_xyz + 3 * m * na;
      if (s->ewald) {
        or_ewald_delta(s, 1, ox, 0, NULL, de, nk);
        w *= exp(s->beta * (de[0] + de[1]));
      }
      if (rng_philox(&ctx, SLOT_ACCEPT) < (double)s->nmol / (w * p->fugacity_beta_v)) {
        st->accepted[3]++;
        int last = s->nmol - 1;
        for (int a = 0; a < 3 * na; a++) s->ads_xyz[3 * m * na + a] = s->ads_xyz[3 * last * na + a];
        s->nmol--;
        if (s->ewald) {
          memcpy(s->sk_ads, nk, sizeof(double) * 2 * s->nk);
          s->net_ads += de[2];
        }
        st->u[0] -= o[2]; st->u[1] -= o[3]; st->u[2] -= o[4]; st->u[3] -= o[5];
        st->u[4] += de[1]; st->u[5] += de[0];
      }
    }
  }
  free(nk);
}
