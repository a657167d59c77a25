/* Tricubic lookup in an energy grid (InterpolateVDWGrid, src/grids.c:979-1077).
 *
 * The grid is the layout written by k_grid_build: (nx+1)(ny+1)(nz+1) points,
 * point-major, 8 floats per point (value, three first, three mixed second
 * and the third mixed derivative, scaled to the grid cell). The interpolant
 * is the Hermite tensor product of those values at the 8 corners of the
 * cell holding the point, the same polynomial as the reference's 64 x 64
 * coefficient product. Points are wrapped into the unit cell the grid spans
 * (rgpu_grid_wrap).
 */
#ifndef RGPU_GRID_CUH
#define RGPU_GRID_CUH

#include "rgpu_types.h"

/* the point wrapped into the unit cell the grid spans: per axis in a
 * rectangular cell (src/grids.c:995-1002), through the fractional
 * coordinates in a triclinic one (:1004-1021) */
__device__ __forceinline__ void rgpu_grid_wrap(const RgpuGridGeom &ip, const double *xyz, double *pw)
{
  if (!ip.tri) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double p = xyz[c];
      p -= ip.cell[c] * rgpu_nint(p / ip.cell[c]);
      if (p < 0.0) p += ip.cell[c];
      pw[c] = p;
    }
    return;
  }
  const double *m = ip.uc, *v = ip.uc + 9;
  double f[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    f[r] = __ldg(v + 3 * r) * xyz[0] + __ldg(v + 3 * r + 1) * xyz[1] + __ldg(v + 3 * r + 2) * xyz[2];
    f[r] -= rgpu_nint(f[r]);
    if (f[r] < 0.0) f[r] += 1.0;
  }
#pragma unroll
  for (int r = 0; r < 3; r++) pw[r] = __ldg(m + 3 * r) * f[0] + __ldg(m + 3 * r + 1) * f[1] + __ldg(m + 3 * r + 2) * f[2];
}

/* Cubic Hermite basis on [0,1]: {p0, p1, slope0, slope1} */
__device__ __forceinline__ void rgpu_hermite(double t, double *h)
{
  const double t2 = t * t, t3 = t2 * t;
  h[0] = 1.0 - 3.0 * t2 + 2.0 * t3;
  h[1] = 3.0 * t2 - 2.0 * t3;
  h[2] = t - 2.0 * t2 + t3;
  h[3] = -t2 + t3;
}

/* energy at p (FP64); a corner value above 1e10 (an atom core) gives 1e8,
 * as the reference's cap (src/grids.c:1058-1060) */
__device__ __forceinline__ double rgpu_grid_value(const float *grid, const RgpuGridGeom &ip, const double *xyz)
{
  const int ny = ip.npts[1] + 1, nz = ip.npts[2] + 1;
  double r[3];
  int i0[3];
  double pw[3];
  rgpu_grid_wrap(ip, xyz, pw);
  for (int c = 0; c < 3; c++) {
    const double p = pw[c];
    const double s = ((p - ip.shift[c]) / ip.size[c]) * (double)ip.npts[c];
    /* a point on the upper cell face (p == cell after wrapping) uses the last
     * grid cell at r = 1, so the 2x2x2 corner block stays inside the grid */
    i0[c] = min(max((int)s, 0), ip.npts[c] - 1);
    r[c] = s - i0[c];
  }
  float v[8][8];
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
    const float4 *src = (const float4 *)(grid + (((size_t)(i0[0] + dx) * ny + (i0[1] + dy)) * nz + (i0[2] + dz)) * 8);
    float4 a = __ldg(src), b = __ldg(src + 1);
    v[c][0] = a.x; v[c][1] = a.y; v[c][2] = a.z; v[c][3] = a.w;
    v[c][4] = b.x; v[c][5] = b.y; v[c][6] = b.z; v[c][7] = b.w;
  }
  for (int c = 0; c < 8; c++)
    if (v[c][0] > 1e10f) return 1e8;
  double hx[4], hy[4], hz[4];
  rgpu_hermite(r[0], hx);
  rgpu_hermite(r[1], hy);
  rgpu_hermite(r[2], hz);
  /* stored value index for derivative order (ox, oy, oz) */
  const int idx[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
  double val = 0.0;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
#pragma unroll
    for (int ox = 0; ox < 2; ox++)
#pragma unroll
      for (int oy = 0; oy < 2; oy++)
#pragma unroll
        for (int oz = 0; oz < 2; oz++)
          val += (double)v[c][idx[ox][oy][oz]] * hx[2 * ox + dx] * hy[2 * oy + dy] * hz[2 * oz + dz];
  }
  return val;
}

/* The same lookup by a group of 8 lanes (lane8 = lane % 8; every lane of
 * the warp calls, converged): lane c reads corner c's 8 values and forms its
 * share of the Hermite sum, and three xor-shuffles add the shares, so a
 * lookup costs one memory round trip instead of eight. Every lane of the
 * group returns the value (the same polynomial as rgpu_grid_value, summed in
 * another order). A group with live = false only takes part in the
 * shuffles. cap: the VDW lookup's 1e8 for a corner above 1e10; the Coulomb
 * lookup (InterpolateCoulombGrid, src/grids.c:1200-1295) has none. */
__device__ __forceinline__ double rgpu_grid_value8(const float *grid, const RgpuGridGeom &ip, const double *xyz,
                                                   int lane8, bool live, bool cap = true)
{
  double val = 0.0;
  int big = 0;
  if (live) {
    const int ny = ip.npts[1] + 1, nz = ip.npts[2] + 1;
    double r[3];
    int i0[3];
    double pw[3];
    rgpu_grid_wrap(ip, xyz, pw);
    for (int c = 0; c < 3; c++) {
      const double p = pw[c];
      const double s = ((p - ip.shift[c]) / ip.size[c]) * (double)ip.npts[c];
      i0[c] = min(max((int)s, 0), ip.npts[c] - 1);
      r[c] = s - i0[c];
    }
    const int dx = lane8 & 1, dy = (lane8 >> 1) & 1, dz = lane8 >> 2;
    const float4 *src = (const float4 *)(grid + (((size_t)(i0[0] + dx) * ny + (i0[1] + dy)) * nz + (i0[2] + dz)) * 8);
    const float4 a = __ldg(src), b = __ldg(src + 1);
    const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    big = v[0] > 1e10f;
    double hx[4], hy[4], hz[4];
    rgpu_hermite(r[0], hx);
    rgpu_hermite(r[1], hy);
    rgpu_hermite(r[2], hz);
    const int idx[2][2][2] = {{{0, 3}, {2, 6}}, {{1, 5}, {4, 7}}};
#pragma unroll
    for (int ox = 0; ox < 2; ox++)
#pragma unroll
      for (int oy = 0; oy < 2; oy++)
#pragma unroll
        for (int oz = 0; oz < 2; oz++)
          val += (double)v[idx[ox][oy][oz]] * hx[2 * ox + dx] * hy[2 * oy + dy] * hz[2 * oz + dz];
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    val += __shfl_xor_sync(0xffffffffu, val, o);
    big |= __shfl_xor_sync(0xffffffffu, big, o);
  }
  return (cap && big) ? 1e8 : val;
}

#endif
