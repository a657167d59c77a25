/* Flexible linear chains (united-atom alkanes and the like): the
 * intramolecular energy terms, the placement of a bead from bond length,
 * bend angle and dihedral, and the draw of a CBMC trial direction.
 *
 * CBMC growth of a chain (the configurational-bias scheme of GrowMolecule,
 * src/cbmc.c:3056-3181): bead i >= 1 is placed at the fixed bond length from
 * bead i-1. The bonded part of its trials follows
 * GenerateTrialOrientationsMCScheme (src/cbmc.c:1580-2480) in the engine's
 * chain_ref_trial (chain_scheme 0: a shared bend angle, torsion candidates
 * and the torsion Rosenbluth factor). chain_trial below is the other
 * scheme (chain_scheme 1): each trial's bend angle theta drawn from
 * p(theta) ~ sin(theta) exp(-beta U_bend(theta)) and its dihedral phi from
 * p(phi) ~ exp(-beta U_torsion(phi)), so the trials carry the bonded
 * Boltzmann factor and the Rosenbluth weights hold only the external energy
 * and the intramolecular LJ. The draws are our own (a Gaussian proposal for
 * theta accepted with probability sin(theta); a uniform proposal for phi
 * accepted with exp(-beta (U_torsion - min U_torsion))), each keyed by
 * (stage, bead, trial, draw) in the system's counter-based stream, so the
 * oracle reproduces every trial.
 *
 * Shared by host and device code; positions are FP64 Cartesian, the chain
 * unwrapped (no periodic image between bonded beads).
 */
#ifndef RGPU_CHAIN_H
#define RGPU_CHAIN_H

#include <math.h>
#include <stdint.h>

#include "rgpu_types.h"

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

#define RGPU_SLOT_CHAIN_SEL (1u << 15)   /* + stage * 8 + bead: selection among the trials */
#define RGPU_SLOT_CHAIN (1u << 16)       /* + draws of one trial, see chain_slot */
#define RGPU_CHAIN_TRIES 64              /* proposals per angle before the fallback */
/* the reference's bonded trials (chain_scheme 0): candidate dihedral k of
 * trial t in slot k of the trial (k < RGPU_MAX_TORS), its choice in slot
 * RGPU_REF_TORS_SEL_SLOT, and the draws of the bend angle shared by a
 * growth step in the slots of trial RGPU_REF_THETA_TRIAL from
 * RGPU_REF_THETA_SLOT on (3 per proposal, RGPU_CHAIN_TRIES proposals) */
#define RGPU_REF_TORS_SEL_SLOT 255
#define RGPU_REF_THETA_TRIAL 15
#define RGPU_REF_THETA_SLOT 256
#define RGPU_TORS_ROWS ((RGPU_MAX_TORS + 63) / 64)   /* rows of candidate pairs per warp */

/* slot of draw k (< 512) of trial t of bead i in growth stage `stage`
 * (0: growth of a new configuration, 1: retrace of an old one) */
__host__ __device__ inline uint32_t chain_slot(int stage, int bead, int trial, int k)
{
  return RGPU_SLOT_CHAIN + (((((uint32_t)stage * 8u + (uint32_t)bead) * 16u + (uint32_t)trial)) << 9) + (uint32_t)k;
}

__host__ __device__ inline double chain_bend_energy(const RgpuSys &S, double theta)
{
  const double d = theta - S.bend_theta0;
  return 0.5 * S.bend_k * d * d;
}

/* TRAPPE_DIHEDRAL, src/internal_energy.c:2324: p0 + p1 (1 + cos phi)
 * + p2 (1 - cos 2phi) + p3 (1 + cos 3phi) */
__host__ __device__ inline double chain_torsion_energy(const RgpuSys &S, double c)
{
  const double c2 = 2.0 * c * c - 1.0, c3 = c * (4.0 * c * c - 3.0);
  return S.torsion[0] + S.torsion[1] * (1.0 + c) + S.torsion[2] * (1.0 - c2) + S.torsion[3] * (1.0 + c3);
}

/* angle a-b-c at b */
__host__ __device__ inline double chain_angle(const double *a, const double *b, const double *c)
{
  const double u[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  const double v[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  double cs = (u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) /
              sqrt((u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
  cs = fmin(1.0, fmax(-1.0, cs));
  return acos(cs);
}

/* cosine of the dihedral a-b-c-d (IUPAC: trans = pi) */
__host__ __device__ inline double chain_cos_dihedral(const double *a, const double *b, const double *c,
                                                     const double *d)
{
  const double b1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double b2[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  const double b3[3] = {d[0] - c[0], d[1] - c[1], d[2] - c[2]};
  const double n1[3] = {b1[1] * b2[2] - b1[2] * b2[1], b1[2] * b2[0] - b1[0] * b2[2], b1[0] * b2[1] - b1[1] * b2[0]};
  const double n2[3] = {b2[1] * b3[2] - b2[2] * b3[1], b2[2] * b3[0] - b2[0] * b3[2], b2[0] * b3[1] - b2[1] * b3[0]};
  double cs = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) /
              sqrt((n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]) * (n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]));
  return fmin(1.0, fmax(-1.0, cs));
}

/* Places a bead at distance L from c, with angle theta at c (b-c-new) and
 * dihedral phi (a-b-c-new). Without a (the third bead of the chain) phi is
 * the azimuth about b-c from a fixed perpendicular reference. */
__host__ __device__ inline void chain_place_trig(const double *a, const double *b, const double *c, double L,
                                                 double ct, double st, double cp, double sp, double *out);

__host__ __device__ inline void chain_place(const double *a, const double *b, const double *c, double L, double theta,
                                            double phi, double *out)
{
  chain_place_trig(a, b, c, L, cos(theta), sin(theta), cos(phi), sin(phi), out);
}

/* chain_place with cos/sin of theta (ct, st) and of phi (cp, sp) given */
__host__ __device__ inline void chain_place_trig(const double *a, const double *b, const double *c, double L,
                                                 double ct, double st, double cp, double sp, double *out)
{
  double bc[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
  double nb = sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
  bc[0] /= nb; bc[1] /= nb; bc[2] /= nb;
  double ref[3];
  if (a) {
    ref[0] = b[0] - a[0]; ref[1] = b[1] - a[1]; ref[2] = b[2] - a[2];
  } else {
    /* the coordinate axis least aligned with b-c */
    const double ax = fabs(bc[0]), ay = fabs(bc[1]), az = fabs(bc[2]);
    ref[0] = (ax <= ay && ax <= az) ? 1.0 : 0.0;
    ref[1] = (ref[0] == 0.0 && ay <= az) ? 1.0 : 0.0;
    ref[2] = (ref[0] == 0.0 && ref[1] == 0.0) ? 1.0 : 0.0;
  }
  /* n = ref x bc, m = n x bc */
  double n[3] = {ref[1] * bc[2] - ref[2] * bc[1], ref[2] * bc[0] - ref[0] * bc[2], ref[0] * bc[1] - ref[1] * bc[0]};
  const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= nn; n[1] /= nn; n[2] /= nn;
  const double m[3] = {n[1] * bc[2] - n[2] * bc[1], n[2] * bc[0] - n[0] * bc[2], n[0] * bc[1] - n[1] * bc[0]};
  const double dx = -L * ct, dy = L * st * cp, dz = L * st * sp;
  for (int k = 0; k < 3; k++) out[k] = c[k] + dx * bc[k] + dy * m[k] + dz * n[k];
}

/* bonded energy (bend + torsion) that bead i adds to beads 0..i-1 */
__host__ __device__ inline double chain_bonded_energy(const RgpuSys &S, const double (*x)[3], int i, const double *p)
{
  double e = 0.0;
  if (i >= 2) e += chain_bend_energy(S, chain_angle(x[i - 2], x[i - 1], p));
  if (i >= 3) e += chain_torsion_energy(S, chain_cos_dihedral(x[i - 3], x[i - 2], x[i - 1], p));
  return e;
}

/* LJ of bead i at p with the beads j <= i - 4 of the chain (lj_bb table) */
__host__ __device__ inline double chain_intra_lj(const RgpuSys &S, const double (*x)[3], int i, const double *p)
{
  double e = 0.0;
  for (int j = 0; j + 4 <= i; j++) {
    const double dx = p[0] - x[j][0], dy = p[1] - x[j][1], dz = p[2] - x[j][2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= S.rc2) continue;
    const RgpuLJ &L = S.lj_bb[i][j];
    double s6 = L.sig2 / r2;
    s6 = s6 * s6 * s6;
    e += L.eps4 * (s6 * (s6 - 1.0)) - L.shift;
  }
  return e;
}

/* whole intramolecular energy of one chain (bonded + intramolecular LJ) */
__host__ __device__ inline double chain_intra_energy(const RgpuSys &S, const double (*x)[3], int n)
{
  double e = 0.0;
  for (int i = 1; i < n; i++) e += chain_bonded_energy(S, x, i, x[i]) + chain_intra_lj(S, x, i, x[i]);
  return e;
}

/* Trial position of bead i >= 1 after beads x[0..i-1]; uniform(slot)
 * supplies the draws. Returns the trial's bonded energy. */
template <typename Uniform>
__host__ __device__ inline double chain_trial(const RgpuSys &S, const double (*x)[3], int i, Uniform uniform,
                                              double *p)
{
  int k = 0;
  if (i == 1) {
    const double z = 2.0 * uniform(k) - 1.0;
    const double psi = 2.0 * M_PI * uniform(k + 1);
    const double r = sqrt(fmax(0.0, 1.0 - z * z));
    p[0] = x[0][0] + S.bond * r * cos(psi);
    p[1] = x[0][1] + S.bond * r * sin(psi);
    p[2] = x[0][2] + S.bond * z;
    return 0.0;
  }
  double theta = S.bend_theta0;
  for (int a = 0; a < RGPU_CHAIN_TRIES; a++, k += 3) {
    const double u1 = uniform(k), u2 = uniform(k + 1), u3 = uniform(k + 2);
    const double th = S.bend_theta0 + S.bend_sigma * sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
    if (th > 0.0 && th < M_PI && u3 < sin(th)) {
      theta = th;
      break;
    }
  }
  k = 3 * RGPU_CHAIN_TRIES;
  double phi;
  if (i == 2) {
    phi = 2.0 * M_PI * uniform(k) - M_PI;
  } else {
    phi = M_PI;
    for (int a = 0; a < RGPU_CHAIN_TRIES; a++, k += 2) {
      const double f = 2.0 * M_PI * uniform(k) - M_PI;
      if (uniform(k + 1) < exp(-S.beta * (chain_torsion_energy(S, cos(f)) - S.torsion_min))) {
        phi = f;
        break;
      }
    }
  }
  chain_place(i >= 3 ? x[i - 3] : nullptr, x[i - 2], x[i - 1], S.bond, theta, phi, p);
  return chain_bonded_energy(S, x, i, p);
}

#endif
