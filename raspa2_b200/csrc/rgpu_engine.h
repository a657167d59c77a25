/* Internal launch interface between capi.cu and the kernel files. */
#ifndef RGPU_ENGINE_H
#define RGPU_ENGINE_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "rgpu_types.h"

/* fw_items / tile_items: framework records / tiles one CTA stages (0: the
 * framework is read from global memory); k_items: wave vectors one CTA
 * stages with their S(k) (0: read from global memory) */
size_t rgpu_engine_smem_bytes(int mixed, int fw_items, int tile_items, int max_ads_atoms, int kw, int k_items,
                              int threads, int flex);
/* raises the kernel's dynamic shared-memory limit to `smem` (call before a
 * launch or a capture of one); flex selects the build with flexible-chain
 * moves and energy grids */
cudaError_t rgpu_engine_prepare(int mixed, bool wide, bool flex, size_t smem);
cudaError_t rgpu_engine_launch(int mixed, RgpuSys *d_systems, int nsys, long long nsteps, int kw,
                               int max_ads_atoms, int fw_items, int tile_items, int k_items, int cluster,
                               int threads, bool wide, bool flex, cudaStream_t st);
cudaError_t rgpu_point_energies_launch(int mixed, const RgpuSys *d_sys, const void *d_ads, int nads,
                                       const double *d_xyz, const int *d_atom, const int *d_excl, int P,
                                       int pair_check, int fw_grid, double *d_out, int *d_ov, cudaStream_t st);
cudaError_t rgpu_ewald_delta_launch(int mixed, const RgpuSys *d_sys, const double *d_xyz, const double *d_q, int ns,
                                    double2 *d_ds, double *d_out, int kw, cudaStream_t st);
cudaError_t rgpu_ewald_accept_launch(const RgpuSys *d_sys, const double2 *d_ds, int nk, cudaStream_t st);
cudaError_t rgpu_structure_factor_launch(const RgpuSys *d_sys, const double *d_xyz, const double *d_q, int n,
                                         int nk, double2 *d_sk, cudaStream_t st);
cudaError_t rgpu_records_launch(const RgpuSys *d_sys, int nads, int4 *d_rec32, void *d_rec64, cudaStream_t st);

/* grids (grid.cu) */
cudaError_t rgpu_grid_build_launch_lj(const RgpuSys *d_sys, const RgpuLJ *lj, const int npts[3],
                                      const double size[3], const double shift[3], float *d_grid, cudaStream_t st);
/* batched state transfer of an engine's systems (see k_gather_states) */
cudaError_t rgpu_gather_states_launch(const RgpuSys *d_systems, int n, const unsigned long long *d_off,
                                      unsigned char *d_buf, cudaStream_t st);
cudaError_t rgpu_upload_sk_launch(const RgpuSys *d_systems, int n, int max_nk, cudaStream_t st);
cudaError_t rgpu_scatter_positions_launch(const RgpuSys *d_systems, int n, const unsigned long long *d_off,
                                          const unsigned char *d_buf, cudaStream_t st);
cudaError_t rgpu_grid_build_launch_coulomb(const RgpuSys *d_sys, const int npts[3], const double size[3],
                                           const double shift[3], float *d_grid, cudaStream_t st);
cudaError_t rgpu_grid_interp_launch(const float *d_grid, const int npts[3], const double size[3],
                                    const double shift[3], const double cell[3], int n, const double *d_xyz,
                                    double *d_out, cudaStream_t st);
/* plane-major (grid file) <-> point-major (device) layout of npt grid points */
cudaError_t rgpu_grid_planes_to_points_launch(const float *d_planes, long long npt, float *d_points, cudaStream_t st);
cudaError_t rgpu_grid_points_to_planes_launch(const float *d_points, long long npt, float *d_planes, cudaStream_t st);

#endif
