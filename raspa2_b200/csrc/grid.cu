/* Energy-grid construction and tricubic lookup.
 *
 * Build: MakeGrid (src/grids.c:431-690) with the per-point derivatives of
 * CalculateDerivativesAtPositionVDW (src/framework_hessian.c:63-109) and the
 * LJ branch of PotentialThirdDerivative (src/potentials.c:10959-10990),
 * computed in FP64 and stored as FP32 like the reference. One thread per grid
 * point; a block covers a 4x8x8 tile and stages, chunk by chunk, only the
 * framework atoms within cutoff + tile radius of the tile centre in shared
 * memory, so each thread visits ~1/7 of the framework at 0.1 A spacing.
 *
 * Device layout is point-major: grid[((i*(ny+1) + j)*(nz+1) + k)*8 + m], so
 * the 8 values of a corner are one 32-byte sector and a lookup gathers eight
 * sectors (the reference's file is plane-major; the Python side converts).
 *
 * Lookup: InterpolateVDWGrid (src/grids.c:979-1077). The reference forms the
 * 64 tricubic coefficients with the Lekien-Marsden matrix and evaluates the
 * polynomial; the same interpolant is evaluated here as the tensor product of
 * 1D cubic Hermite bases over the stored value and derivatives (FP64 math on
 * the FP32 data, as in the reference).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>

#include "rgpu_device.cuh"
#include "rgpu_engine.h"
#include "rgpu_grid.cuh"

#define GRID_TX 4
#define GRID_TY 8
#define GRID_TZ 8
#define GRID_THREADS (GRID_TX * GRID_TY * GRID_TZ)

struct GridParams {
  int npts[3];
  double size[3], shift[3], delta[3];
  RgpuLJ lj[RGPU_MAX_FWTYPES];
};

/* COUL = false: the LJ grid of one probe pseudo-atom (gp.lj by framework
 * segment). COUL = true: the real-space Ewald (Coulomb) grid of a unit probe
 * charge, CalculateDerivativesAtPositionReal (src/framework_hessian.c:111-180)
 * with the framework charges, capped where the value exceeds the overlap
 * criterion or a framework atom is closer than 1 A (src/grids.c:656-668). */
template <bool COUL>
__global__ void __launch_bounds__(GRID_THREADS) k_grid_build(const RgpuSys *sysp, GridParams gp, float *grid)
{
  __shared__ double4 fwc[GRID_THREADS];
  __shared__ int segc[GRID_THREADS];
  __shared__ int wcount[GRID_THREADS / 32];
  __shared__ int nsel;
  const RgpuSys &S = *sysp;
  const int nx = gp.npts[0] + 1, ny = gp.npts[1] + 1, nz = gp.npts[2] + 1;
  const int tilesz = (nz + GRID_TZ - 1) / GRID_TZ, tilesy = (ny + GRID_TY - 1) / GRID_TY;
  int b = blockIdx.x;
  const int tk = b % tilesz; b /= tilesz;
  const int tj = b % tilesy; b /= tilesy;
  const int ti = b;
  const int lk = threadIdx.x % GRID_TZ, lj = (threadIdx.x / GRID_TZ) % GRID_TY, li = threadIdx.x / (GRID_TZ * GRID_TY);
  const int i = ti * GRID_TX + li, j = tj * GRID_TY + lj, k = tk * GRID_TZ + lk;
  const bool valid = i < nx && j < ny && k < nz;
  const double px = i * gp.size[0] / gp.npts[0] + gp.shift[0];
  const double py = j * gp.size[1] / gp.npts[1] + gp.shift[1];
  const double pz = k * gp.size[2] / gp.npts[2] + gp.shift[2];
  /* tile centre and radius for culling */
  const double cx = (ti * GRID_TX + 0.5 * (GRID_TX - 1)) * gp.size[0] / gp.npts[0] + gp.shift[0];
  const double cy = (tj * GRID_TY + 0.5 * (GRID_TY - 1)) * gp.size[1] / gp.npts[1] + gp.shift[1];
  const double cz = (tk * GRID_TZ + 0.5 * (GRID_TZ - 1)) * gp.size[2] / gp.npts[2] + gp.shift[2];
  const double hx = 0.5 * (GRID_TX - 1) * gp.delta[0], hy = 0.5 * (GRID_TY - 1) * gp.delta[1],
               hz = 0.5 * (GRID_TZ - 1) * gp.delta[2];
  const double rcut = sqrt(S.rc2) + sqrt(hx * hx + hy * hy + hz * hz) + 1e-6;
  const double rcut2 = rcut * rcut;
  const double Lx = S.box[0], Ly = S.box[1], Lz = S.box[2];
  const double ix = S.inv_box[0], iy = S.inv_box[1], iz = S.inv_box[2];
  double o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double rmin2 = 1e300;
  const double a2 = S.alpha * S.alpha, two_a_sqrtpi = 2.0 * S.alpha / sqrt(M_PI);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < S.nfw; base += GRID_THREADS) {
    const int a = base + threadIdx.x;
    int keep = 0;
    double4 f = make_double4(0, 0, 0, 0);
    int seg = 0;
    if (a < S.nfw) {
      f = S.fw64[a];
      if (S.triclinic) {
        /* a triclinic box: every atom is staged (its minimum image may
         * differ across the tile's points near half a cell vector) */
        keep = 1;
      } else {
        double dx = cx - f.x, dy = cy - f.y, dz = cz - f.z;
        dx -= Lx * rgpu_nint(dx * ix);
        dy -= Ly * rgpu_nint(dy * iy);
        dz -= Lz * rgpu_nint(dz * iz);
        keep = dx * dx + dy * dy + dz * dz < rcut2;
      }
      while (seg + 1 < S.nseg && a >= S.seg_start[seg + 1]) seg++;
    }
    unsigned m = __ballot_sync(RGPU_FULL, keep);
    if (lane == 0) wcount[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int q = 0; q < GRID_THREADS / 32; q++) { int c = wcount[q]; wcount[q] = s; s += c; }
      nsel = s;
    }
    __syncthreads();
    if (keep) {
      int pos = wcount[w] + __popc(m & ((1u << lane) - 1u));
      fwc[pos] = f;
      segc[pos] = seg;
    }
    __syncthreads();
    if (valid) {
      for (int q = 0; q < nsel; q++) {
        const double4 g = fwc[q];
        double dx = px - g.x, dy = py - g.y, dz = pz - g.z;
        if (S.triclinic) {
          rgpu_min_image_tri(S, dx, dy, dz);
        } else {
          dx -= Lx * rgpu_nint(dx * ix);
          dy -= Ly * rgpu_nint(dy * iy);
          dz -= Lz * rgpu_nint(dz * iz);
        }
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < S.rc2) {
          double U, DF, DDF, DDDF;
          if (COUL) {
            /* f(r) = K q erfc(a r) / r; DF = f'/r, DDF = (f'' - f'/r)/r^2,
             * DDDF = the r-part of the mixed third derivative */
            rmin2 = fmin(rmin2, r2);
            const double r = sqrt(r2), kq = S.coulomb * g.w;
            const double e = erfc(S.alpha * r), gr = two_a_sqrtpi * r * exp(-a2 * r2);
            const double ar2 = a2 * r2;
            U = kq * e / r;
            DF = -kq * (gr + e) / (r * r2);
            DDF = kq * (gr * (3.0 + 2.0 * ar2) + 3.0 * e) / (r2 * r2 * r);
            DDDF = -kq * (gr * (15.0 + 10.0 * ar2 + 4.0 * ar2 * ar2) + 15.0 * e) / (r2 * r2 * r2 * r);
          } else {
            const RgpuLJ P = gp.lj[segc[q]];
            const double eps = 0.25 * P.eps4;
            double r3 = P.sig2 / r2;
            r3 = r3 * r3 * r3;
            U = 4.0 * eps * (r3 * (r3 - 1.0)) - P.shift;
            DF = 24.0 * eps * (r3 * (1.0 - 2.0 * r3)) / r2;
            DDF = 96.0 * eps * (r3 * (7.0 * r3 - 2.0)) / (r2 * r2);
            DDDF = 384.0 * eps * (r3 * (5.0 - 28.0 * r3)) / (r2 * r2 * r2 * r2);
          }
          o[0] += U;
          o[1] += dx * DF;
          o[2] += dy * DF;
          o[3] += dz * DF;
          o[4] += DDF * dx * dy;
          o[5] += DDF * dx * dz;
          o[6] += DDF * dy * dz;
          o[7] += DDDF * dx * dy * dz;
        }
      }
    }
    __syncthreads();
  }
  if (!valid) return;
  /* cap, src/grids.c:546-563 (Coulomb: also within 1 A of an atom, :656-668) */
  if (o[0] > S.overlap || (COUL && rmin2 < 1.0)) {
    o[0] = 2.0 * S.overlap;
    for (int c = 1; c <= 3; c++) {
      if (o[c] > S.overlap) o[c] = S.overlap;
      if (o[c] < -S.overlap) o[c] = -S.overlap;
    }
    o[4] = o[5] = o[6] = o[7] = 0.0;
  }
  const double dx = gp.delta[0], dy = gp.delta[1], dz = gp.delta[2];
  float4 v0 = make_float4((float)o[0], (float)o[1] * (float)dx, (float)o[2] * (float)dy, (float)o[3] * (float)dz);
  float4 v1 = make_float4((float)o[4] * (float)(dx * dy), (float)o[5] * (float)(dx * dz),
                          (float)o[6] * (float)(dy * dz), (float)o[7] * (float)(dx * dy * dz));
  float4 *dst = (float4 *)(grid + (((size_t)i * ny + j) * nz + k) * 8);
  dst[0] = v0;
  dst[1] = v1;
}

/* lj[s]: LJ parameters of the probe pseudo-atom with framework segment s */
cudaError_t rgpu_grid_build_launch_lj(const RgpuSys *d_sys, const RgpuLJ *lj, const int npts[3], const double size[3],
                                      const double shift[3], float *d_grid, cudaStream_t st)
{
  GridParams gp;
  for (int c = 0; c < 3; c++) {
    gp.npts[c] = npts[c];
    gp.size[c] = size[c];
    gp.shift[c] = shift[c];
    gp.delta[c] = size[c] / (double)npts[c];
  }
  for (int s = 0; s < RGPU_MAX_FWTYPES; s++) gp.lj[s] = lj[s];
  const int nx = npts[0] + 1, ny = npts[1] + 1, nz = npts[2] + 1;
  const long long blocks = (long long)((nx + GRID_TX - 1) / GRID_TX) * ((ny + GRID_TY - 1) / GRID_TY) *
                           ((nz + GRID_TZ - 1) / GRID_TZ);
  if (blocks > 2147483647LL) return cudaErrorInvalidValue;
  k_grid_build<false><<<(unsigned)blocks, GRID_THREADS, 0, st>>>(d_sys, gp, d_grid);
  return cudaGetLastError();
}

/* the Coulomb grid of a unit probe charge */
cudaError_t rgpu_grid_build_launch_coulomb(const RgpuSys *d_sys, const int npts[3], const double size[3],
                                           const double shift[3], float *d_grid, cudaStream_t st)
{
  GridParams gp = {};
  for (int c = 0; c < 3; c++) {
    gp.npts[c] = npts[c];
    gp.size[c] = size[c];
    gp.shift[c] = shift[c];
    gp.delta[c] = size[c] / (double)npts[c];
  }
  const int nx = npts[0] + 1, ny = npts[1] + 1, nz = npts[2] + 1;
  const long long blocks = (long long)((nx + GRID_TX - 1) / GRID_TX) * ((ny + GRID_TY - 1) / GRID_TY) *
                           ((nz + GRID_TZ - 1) / GRID_TZ);
  if (blocks > 2147483647LL) return cudaErrorInvalidValue;
  k_grid_build<true><<<(unsigned)blocks, GRID_THREADS, 0, st>>>(d_sys, gp, d_grid);
  return cudaGetLastError();
}

__global__ void k_grid_interp(const float *grid, RgpuGridGeom ip, int n, const double *xyz, double *out)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const double p[3] = {xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]};
  out[q] = rgpu_grid_value(grid, ip, p);
}

cudaError_t rgpu_grid_interp_launch(const float *d_grid, const int npts[3], const double size[3],
                                    const double shift[3], const double cell[3], int n, const double *d_xyz,
                                    double *d_out, cudaStream_t st)
{
  RgpuGridGeom ip;
  memset(&ip, 0, sizeof ip);   /* a rectangular cell (tri = 0) */
  for (int c = 0; c < 3; c++) {
    ip.npts[c] = npts[c];
    ip.size[c] = size[c];
    ip.shift[c] = shift[c];
    ip.cell[c] = cell[c];
  }
  if (n <= 0) return cudaSuccess;
  k_grid_interp<<<(n + 255) / 256, 256, 0, st>>>(d_grid, ip, n, d_xyz, d_out);
  return cudaGetLastError();
}

/* Grid files store the 8 values as planes ([m][i][j][k], src/grids.c:734-738);
 * the device layout is point-major (8 floats per point). One thread per
 * point: the plane reads (or writes) of neighbouring threads are contiguous,
 * and the point's 8 floats move as two 16-byte words. */
__global__ void k_grid_planes_to_points(const float *__restrict__ planes, long long npt, float *__restrict__ points)
{
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npt; p += (long long)gridDim.x * blockDim.x) {
    float v[8];
#pragma unroll
    for (int m = 0; m < 8; m++) v[m] = planes[m * npt + p];
    float4 *dst = (float4 *)(points + 8 * p);
    dst[0] = make_float4(v[0], v[1], v[2], v[3]);
    dst[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
}

__global__ void k_grid_points_to_planes(const float *__restrict__ points, long long npt, float *__restrict__ planes)
{
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npt; p += (long long)gridDim.x * blockDim.x) {
    const float4 *src = (const float4 *)(points + 8 * p);
    const float4 a = src[0], b = src[1];
    const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int m = 0; m < 8; m++) planes[m * npt + p] = v[m];
  }
}

static unsigned transpose_blocks(long long npt)
{
  /* at most 8 CTAs of 256 per SM-count multiple: 148 SMs x 8 */
  const long long want = (npt + 255) / 256;
  return (unsigned)std::min<long long>(want, 148LL * 8);
}

cudaError_t rgpu_grid_planes_to_points_launch(const float *d_planes, long long npt, float *d_points, cudaStream_t st)
{
  if (npt <= 0) return cudaSuccess;
  k_grid_planes_to_points<<<transpose_blocks(npt), 256, 0, st>>>(d_planes, npt, d_points);
  return cudaGetLastError();
}

cudaError_t rgpu_grid_points_to_planes_launch(const float *d_points, long long npt, float *d_planes, cudaStream_t st)
{
  if (npt <= 0) return cudaSuccess;
  k_grid_points_to_planes<<<transpose_blocks(npt), 256, 0, st>>>(d_points, npt, d_planes);
  return cudaGetLastError();
}
