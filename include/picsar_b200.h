/*
 * picsar_b200.h -- C ABI of libpicsar_b200.so, the B200 (sm_100a) kernels
 * behind PICSAR's per-step particle loop.
 *
 * Conventions
 *  - Every entry point returns int: 0 on success, otherwise a PXRB_E* code.
 *  - Array arguments are DEVICE pointers unless stated otherwise; bounds
 *    arrays of the Yee routines (int64_t[3]) are HOST pointers.
 *  - Grids follow PICSAR's Fortran layout: float64, column-major (x fastest),
 *    lower bound -guard and upper bound n+guard per axis; the pointer
 *    addresses element (-gx,-gy,-gz).
 *  - Fortran INTEGER(idp) -> int64_t, REAL(num) -> double,
 *    LOGICAL(lp) -> int64_t (0 = .FALSE.).
 *  - Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 *    stream); no entry point synchronises the device.
 *  - Module variables the Fortran routines read implicitly (`dt`,
 *    `particle_pusher`, `clight`) are explicit trailing arguments.
 *  - Gather and deposition ACCUMULATE into their outputs, as the reference
 *    does; the caller zeroes them.
 *
 * Reference citations are paths inside the PICSAR source tree.
 */
#ifndef PICSAR_B200_H
#define PICSAR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PXRB_OK 0
#define PXRB_EINVAL 1        /* null pointer, negative or inconsistent size */
#define PXRB_EUNSUPPORTED 2  /* shape order or option not implemented */
#define PXRB_ELAUNCH 3       /* CUDA launch or runtime error */
#define PXRB_ESCRATCH 4      /* caller's scratch buffer too small */
#define PXRB_ERANGE 5        /* grid too small for its guard cells */
#define PXRB_ETOOLARGE 6     /* job above the fixed limit of a no-allocation entry */

/* ------------------------------------------------------------------------
 * Plain FP64 path (PICSAR arrays, one thread per particle, FP64 atomics)
 * ---------------------------------------------------------------------- */

/* Replaces field_gathering_plus_particle_pusher_{1_1_1,2_2_2,3_3_3}
 * (src/particle_pushers/particle_pusher_manager_3d.F90:1287, :1522, :1820):
 * energy-conserving gather (+=) into ex..bz, then Boris + pxr_set_gamma
 * (particle_pusher = 0) or Vay (1), then pxr_pushxyz, all with `dt`.
 * Only l_lower_order_in_v = .TRUE. exists in the reference fused kernels.
 * `order` selects 1, 2 or 3; the three _n_n_n symbols below fix it. */
int pxrb_field_gathering_plus_particle_pusher(
    int64_t order, int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
    double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx, double* by,
    double* bz, double xmin, double ymin, double zmin, double dx, double dy, double dz,
    double dtt, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard, int64_t nyguard,
    int64_t nzguard, const double* exg, const double* eyg, const double* ezg,
    const double* bxg, const double* byg, const double* bzg, double q, double m,
    int64_t lvect, int64_t l_lower_order_in_v, double dt, int64_t particle_pusher,
    double clight, void* stream);
#define PXRB_FGP_DECL(O)                                                                  \
  int pxrb_field_gathering_plus_particle_pusher_##O##_##O##_##O(                          \
      int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,           \
      double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx,        \
      double* by, double* bz, double xmin, double ymin, double zmin, double dx, double dy, \
      double dz, double dtt, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,         \
      int64_t nyguard, int64_t nzguard, const double* exg, const double* eyg,             \
      const double* ezg, const double* bxg, const double* byg, const double* bzg,         \
      double q, double m, int64_t lvect, int64_t l_lower_order_in_v, double dt,           \
      int64_t particle_pusher, double clight, void* stream);
/* particle_pusher_manager_3d.F90:1287 */
PXRB_FGP_DECL(1)
/* particle_pusher_manager_3d.F90:1522 */
PXRB_FGP_DECL(2)
/* particle_pusher_manager_3d.F90:1820 */
PXRB_FGP_DECL(3)
#undef PXRB_FGP_DECL

/* Replaces geteb3d_energy_conserving
 * (src/field_gathering/field_gathering_manager_3d.F90:295-323): separate
 * gather (+=), both l_lower_order_in_v branches, l_nodal as the nodal-grid
 * module flag.  nox = noy = noz in 1..3; ll4symtry must be 0. */
int pxrb_geteb3d_energy_conserving(
    int64_t np, const double* xp, const double* yp, const double* zp, double* ex, double* ey,
    double* ez, double* bx, double* by, double* bz, double xmin, double ymin, double zmin,
    double dx, double dy, double dz, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,
    int64_t nyguard, int64_t nzguard, int64_t nox, int64_t noy, int64_t noz,
    const double* exg, const double* eyg, const double* ezg, const double* bxg,
    const double* byg, const double* bzg, int64_t ll4symtry, int64_t l_lower_order_in_v,
    int64_t lvect, int64_t field_gathe_algo, int64_t l_nodal, void* stream);

/* Replaces pxr_boris_push_u_3d (src/particle_pushers/boris_pusher/boris_3d.F90:51). */
int pxrb_boris_push_u_3d(int64_t np, double* uxp, double* uyp, double* uzp, double* gaminv,
                         const double* ex, const double* ey, const double* ez,
                         const double* bx, const double* by, const double* bz, double q,
                         double m, double dt, double clight, void* stream);

/* Replaces pxr_ebcancelpush3d (src/particle_pushers/vay_pusher/vay_3d.F90:56),
 * which = 0 (full push), 1 (first half), 2 (second half). */
int pxrb_ebcancelpush3d(int64_t np, double* uxp, double* uyp, double* uzp, double* gi,
                        const double* ex, const double* ey, const double* ez,
                        const double* bx, const double* by, const double* bz, double q,
                        double m, double dt, int64_t which, double clight, void* stream);

/* Replaces pxr_set_gamma (boris_3d.F90:1059). */
int pxrb_set_gamma(int64_t np, const double* uxp, const double* uyp, const double* uzp,
                   double* gaminv, double clight, void* stream);

/* Replaces pxr_pushxyz (boris_3d.F90:849). */
int pxrb_pushxyz(int64_t np, double* xp, double* yp, double* zp, const double* uxp,
                 const double* uyp, const double* uzp, const double* gaminv, double dt,
                 void* stream);

/* Replaces depose_jxjyjz (current_depo_algo = 0: specialised Esirkepov
 * depose_jxjyjz_esirkepov_{1,2,3}) and depose_jxjyjz_esirkepov
 * (current_depo_algo = 1: pxr_depose_jxjyjz_esirkepov_n with its
 * xold + dt*v reconstruction) (src/particle_deposition/current_deposition/
 * current_deposition_manager_3d.F90:47, :75; esirkepov/esirkepov_3d.F90:82,
 * :1734, :3263, :3480).  Accumulates; nox = noy = noz in 1..3.
 * err_flag (device int) is set to 1 if a particle moved more than one cell
 * per axis in one step (impossible under the CFL limit). */
int pxrb_depose_jxjyjz(double* jx, double* jy, double* jz, int64_t np, const double* xp,
                       const double* yp, const double* zp, const double* uxp,
                       const double* uyp, const double* uzp, const double* gaminv,
                       const double* w, double q, double xmin, double ymin, double zmin,
                       double dt, double dx, double dy, double dz, int64_t nx, int64_t ny,
                       int64_t nz, int64_t nxguard, int64_t nyguard, int64_t nzguard,
                       int64_t nox, int64_t noy, int64_t noz, int64_t current_depo_algo,
                       int* err_flag, void* stream);

/* Replaces depose_rho_scalar_{1,2,3}_{1,2,3}_{1,2,3}
 * (src/particle_deposition/charge_deposition/charge_deposition_3d.F90:77,
 * :174, :324).  Accumulates node-centred rho. */
int pxrb_depose_rho(int64_t order, double* rho, int64_t np, const double* xp,
                    const double* yp, const double* zp, const double* w, double q,
                    double xmin, double ymin, double zmin, double dx, double dy, double dz,
                    int64_t nx, int64_t ny, int64_t nz, int64_t nxguard, int64_t nyguard,
                    int64_t nzguard, void* stream);

/* Replaces pxrpush_em3d_evec (src/field_solvers/Maxwell/yee_solver/yee.F90:637).
 * x/y/z lo/hi: loop ranges of Ex/Ey/Ez; <a>lo/<a>hi: array bounds (HOST). */
int pxrb_push_em3d_evec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        double* ex, const int64_t* exlo, const int64_t* exhi, double* ey,
                        const int64_t* eylo, const int64_t* eyhi, double* ez,
                        const int64_t* ezlo, const int64_t* ezhi, const double* bx,
                        const int64_t* bxlo, const int64_t* bxhi, const double* by,
                        const int64_t* bylo, const int64_t* byhi, const double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, const double* jx,
                        const int64_t* jxlo, const int64_t* jxhi, const double* jy,
                        const int64_t* jylo, const int64_t* jyhi, const double* jz,
                        const int64_t* jzlo, const int64_t* jzhi, double mudt, double dtsdx,
                        double dtsdy, double dtsdz, void* stream);

/* Replaces pxrpush_em3d_bvec (yee.F90:1258). */
int pxrb_push_em3d_bvec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        const double* ex, const int64_t* exlo, const int64_t* exhi,
                        const double* ey, const int64_t* eylo, const int64_t* eyhi,
                        const double* ez, const int64_t* ezlo, const int64_t* ezhi,
                        double* bx, const int64_t* bxlo, const int64_t* bxhi, double* by,
                        const int64_t* bylo, const int64_t* byhi, double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, double dtsdx, double dtsdy,
                        double dtsdz, void* stream);

/* Replaces pxrpush_em3d_evec_norder (yee.F90:46-123): E += arbitrary-order
 * curl B - mudt J on nodes [-nxs, nx+nxs] x ... of nine arrays of shape
 * (-guard:n+guard) per axis; dtsdx[norderx/2] ... are HOST arrays of the
 * difference weights times c^2 dt / d (norder even, 2..32); l_nodalgrid != 0
 * selects the nodal stencil.  Stencils are clipped where the arrays end,
 * as in the reference. */
int pxrb_push_em3d_evec_norder(double* ex, double* ey, double* ez, const double* bx,
                               const double* by, const double* bz, const double* jx,
                               const double* jy, const double* jz, double mudt,
                               const double* dtsdx, const double* dtsdy, const double* dtsdz,
                               int64_t nx, int64_t ny, int64_t nz, int64_t norderx,
                               int64_t nordery, int64_t norderz, int64_t nxguard,
                               int64_t nyguard, int64_t nzguard, int64_t nxs, int64_t nys,
                               int64_t nzs, int64_t l_nodalgrid, void* stream);

/* Replaces pxrpush_em3d_bvec_norder (yee.F90:752-821): B -= arbitrary-order
 * curl E, same conventions (weights times dt / d, halved by the caller for a
 * half step as push_bfield does). */
int pxrb_push_em3d_bvec_norder(const double* ex, const double* ey, const double* ez,
                               double* bx, double* by, double* bz, const double* dtsdx,
                               const double* dtsdy, const double* dtsdz, int64_t nx, int64_t ny,
                               int64_t nz, int64_t norderx, int64_t nordery, int64_t norderz,
                               int64_t nxguard, int64_t nyguard, int64_t nzguard, int64_t nxs,
                               int64_t nys, int64_t nzs, int64_t l_nodalgrid, void* stream);

/* Replaces FD_weights (src/submain.F90:927-984): the norder/2 weights of
 * the first derivative on the staggered (l_nodal = 0) or nodal grid, the
 * reference's form of Fornberg's recursion.  Host function; coeffs: HOST
 * double[norder/2]. */
int pxrb_fd_weights(double* coeffs, int64_t norder, int64_t l_nodal);

/* ------------------------------------------------------------------------
 * 2D (x-z) path, plain FP64: grids are 2-D Fortran arrays (-guard:n+guard)
 * in x and z (PICSAR's x-z arrays, ny = 0 with no y guards).
 * ---------------------------------------------------------------------- */

/* Replaces geteb2dxz_energy_conserving (src/field_gathering/
 * field_gathering_manager_2d.F90:61-89 -> the scalar
 * pxr_gete2dxz / pxr_getb2dxz_energy_conserving_scalar_{1_1,2_2,3_3},
 * field_gathering_o{1,2,3}_2d.F90): accumulates into ex..bz; both
 * l_lower_order_in_v branches and the nodal grid; nox = noz in 1..3; the y
 * arguments are accepted and unused, as in the reference. */
int pxrb_geteb2dxz_energy_conserving(
    int64_t np, const double* xp, const double* yp, const double* zp, double* ex, double* ey,
    double* ez, double* bx, double* by, double* bz, double xmin, double ymin, double zmin,
    double dx, double dy, double dz, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,
    int64_t nyguard, int64_t nzguard, int64_t nox, int64_t noy, int64_t noz,
    const double* exg, const double* eyg, const double* ezg, const double* bxg,
    const double* byg, const double* bzg, int64_t l4symtry, int64_t l_lower_order_in_v,
    int64_t lvect, int64_t field_gathe_algo, int64_t l_nodal, void* stream);

/* Replaces depose_jxjyjz_2d (src/particle_deposition/current_deposition/
 * current_deposition_manager_2d.F90:42 -> pxr_depose_jxjyjz_esirkepov2d_
 * {1_1,2_2,3_3}, esirkepov/esirkepov_2d.F90:452-1082): 2-D Esirkepov with
 * the out-of-plane Jy, accumulating; nox = noz in 1..3. */
int pxrb_depose_jxjyjz_2d(double* jx, double* jy, double* jz, int64_t np, const double* xp,
                          const double* yp, const double* zp, const double* uxp,
                          const double* uyp, const double* uzp, const double* gaminv,
                          const double* w, double q, double xmin, double zmin, double dt,
                          double dx, double dz, int64_t nx, int64_t nz, int64_t nxguard,
                          int64_t nzguard, int64_t nox, int64_t noz, int64_t lvect,
                          void* stream);

/* Replace pxrpush_em2d_evec / pxrpush_em2d_bvec (yee.F90:216-310, :912-994);
 * bounds: HOST int64[2] (x, z); dtsdy is accepted and unused. */
int pxrb_push_em2d_evec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        double* ex, const int64_t* exlo, const int64_t* exhi, double* ey,
                        const int64_t* eylo, const int64_t* eyhi, double* ez,
                        const int64_t* ezlo, const int64_t* ezhi, const double* bx,
                        const int64_t* bxlo, const int64_t* bxhi, const double* by,
                        const int64_t* bylo, const int64_t* byhi, const double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, const double* jx,
                        const int64_t* jxlo, const int64_t* jxhi, const double* jy,
                        const int64_t* jylo, const int64_t* jyhi, const double* jz,
                        const int64_t* jzlo, const int64_t* jzhi, double mudt, double dtsdx,
                        double dtsdy, double dtsdz, void* stream);
int pxrb_push_em2d_bvec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        const double* ex, const int64_t* exlo, const int64_t* exhi,
                        const double* ey, const int64_t* eylo, const int64_t* eyhi,
                        const double* ez, const int64_t* ezlo, const int64_t* ezhi,
                        double* bx, const int64_t* bxlo, const int64_t* bxhi, double* by,
                        const int64_t* bylo, const int64_t* byhi, double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, double dtsdx, double dtsdy,
                        double dtsdz, void* stream);

/* Replaces pxr_pushxz (src/particle_pushers/boris_pusher/boris_2d.F90:42). */
int pxrb_pushxz(int64_t np, double* xp, double* zp, const double* uxp, const double* uzp,
                const double* gaminv, double dt, void* stream);

/* Replaces field_bc -> exchange_mpi_3d_grid_array_with_guards for a single
 * periodic domain (src/boundary_conditions/field_boundaries.F90:81-269), for
 * one to three grids of the same shape (f2/f3 may be NULL).  Needs n > g per
 * axis, except an axis with n = 0 and g = 0 (the y axis of x-z grids), which
 * is skipped. */
int pxrb_field_bc_periodic(double* f1, double* f2, double* f3, int64_t nx, int64_t ny,
                           int64_t nz, int64_t nxg, int64_t nyg, int64_t nzg, void* stream);

/* Replaces summation_bcs (field_boundaries.F90:403-503) for a single periodic
 * domain: fold the guards into the interior, then field_bc. */
int pxrb_summation_bcs_periodic(double* f1, double* f2, double* f3, int64_t nx, int64_t ny,
                                int64_t nz, int64_t nxg, int64_t nyg, int64_t nzg,
                                void* stream);

/* Replaces the periodic branch (pbound = 0) of the particle boundary
 * conditions (src/boundary_conditions/particle_boundaries.F90:1109-1300). */
int pxrb_particle_bcs_periodic(int64_t np, double* xp, double* yp, double* zp, double xmin,
                               double ymin, double zmin, double xmax, double ymax,
                               double zmax, void* stream);

/* Replaces the per-side pbound cases of particle_bcs for one domain
 * (src/boundary_conditions/particle_boundaries.F90:1098-1300): pbound (HOST
 * int64[6]: x-, x+, y-, y+, z-, z+) 0 periodic, 1 absorbing (particle
 * removed), 2 reflecting (moved one cell in, u negated), 3 reinjecting
 * (mirrored, u = 0, clamped into the tile region tile_lo..tile_hi (HOST
 * double[3] each) less half a cell).  Removed particles are compacted out,
 * keeping the survivors' order; every array among xp..uzp, gaminv, w and pid
 * (the last three optional) is compacted.  np_out: DEVICE int64, the number
 * left.  scratch: DEVICE bytes >= pxrb_particle_bcs_scratch(np). */
int64_t pxrb_particle_bcs_scratch(int64_t np);
int pxrb_particle_bcs(int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
                      double* uzp, double* gaminv, double* w, double* pid, double xmin_part,
                      double ymin_part, double zmin_part, double xmax_part, double ymax_part,
                      double zmax_part, double dx, double dy, double dz, const int64_t* pbound,
                      const double* tile_lo, const double* tile_hi, void* scratch,
                      int64_t scratch_bytes, int64_t* np_out, void* stream);

/* Replaces pxr_particle_bin_sorting (src/housekeeping/sorting.F90:247-361):
 * particles reordered by bin number iz*nx3*ny3 + iy*nx3 + ix, with
 * (ix, iy, iz) = floor((x - xmin2) / dxf, ...) and nx3 = ceil((xmax2 - xmin2)
 * / dxf) ..., keeping the input order inside a bin (the reference's counting
 * sort is stable).  Positions outside [min2, max2) go to the nearest end bin
 * (the reference checks this only in DEBUG builds).  xp..gam are permuted in
 * place, and w (the pid weight column, the only pid column the reference
 * carries along, sorting.F90:264) when not NULL.  scratch: DEVICE bytes,
 * scratch_bytes >= pxrb_particle_bin_sorting_scratch(np); np < 2^31. */
int64_t pxrb_particle_bin_sorting_scratch(int64_t np);
int pxrb_particle_bin_sorting(int64_t np, double* xp, double* yp, double* zp, double* ux,
                              double* uy, double* uz, double* gam, double* w, double xmin2,
                              double ymin2, double zmin2, double xmax2, double ymax2,
                              double zmax2, double dxf, double dyf, double dzf, void* scratch,
                              int64_t scratch_bytes, void* stream);


/* Spectral (PSATD) field push of one periodic domain in Fourier space:
 * replaces push_psaotd_ebfielfs_3d (src/field_solvers/Maxwell/GPSTD_solver/
 * fourier_psaotd.F90:1538-1643) with the coefficient blocks of
 * compute_cc_mat_merged_fields (init_kspace_3D.F90:1316-1495).  The field
 * spectra are DEVICE complex FP64 (interleaved re, im) arrays of
 * nkx*nky*nkz modes, x fastest: the r2c transforms of the FFT region of
 * ex..bz (updated in place), jx..jz, rho and rho_old.  kxf, kxb (nkx), kyf,
 * kyb (nky), kzf, kzb (nkz): DEVICE complex k-vectors (forward, backward
 * staggering, compute_k_1d); kxc2, kyc2, kzc2: DEVICE |k_centred|^2 per axis;
 * at1, at2, at3: DEVICE per-mode operators c dt sinc(c|k|dt), cos(c|k|dt),
 * (1 - cos)/|k|^2 (init_kspace, with its k = 0 values); norm: 1 / (number
 * of real FFT points), applied to every coefficient as the reference does. */
int pxrb_psatd_push(int64_t nkx, int64_t nky, int64_t nkz, double* ex, double* ey, double* ez,
                    double* bx, double* by, double* bz, const double* jx, const double* jy,
                    const double* jz, const double* rho, const double* rhoold,
                    const double* kxf, const double* kxb, const double* kyf, const double* kyb,
                    const double* kzf, const double* kzb, const double* kxc2,
                    const double* kyc2, const double* kzc2, const double* at1,
                    const double* at2, const double* at3, double clight, double eps0,
                    double mu0, double dt, double norm, void* stream);

/* ------------------------------------------------------------------------
 * Tiled engine (B200-native layout): FP32 mixed precision or FP64.
 *
 * One pxrb_tiled_job describes one periodic simulation.  Fields E, B are
 * stored with `g` periodic guard cells per side in arrays of extent
 * (pitch_x, ny+2g, nz+2g), x fastest, element (i,j,k) at
 * (i+g) + pitch_x*((j+g) + (ny+2g)*(k+g)); the current J is FP64 without
 * guards (nx*ny*nz, periodic indexing).  Particles are SoA sorted by cell
 * tile: a packed cell index (x | y<<11 | z<<22; nx, ny <= 2048, nz <= 1024)
 * plus an in-cell offset in [0,1) per axis, momenta u = gamma*beta and the
 * weight, all in the engine precision.  `prec` selects float (0) or double
 * (1) for fields, offsets, momenta and weights.  `tile_off[t]..tile_off[t+1]`
 * is the particle range of tile t (tiles x fastest).
 * ---------------------------------------------------------------------- */
typedef struct pxrb_tiled_job {
  int32_t nx, ny, nz;        /* cells per axis (periodic) */
  int32_t tx, ty, tz;        /* tile size in cells */
  int32_t ntx, nty, ntz;     /* tiles per axis = ceil(n / t) */
  int32_t g;                 /* guard cells of the E/B arrays (>= 3) */
  int32_t pitch_x;           /* allocated x extent of the E/B arrays (>= nx+2g) */
  int32_t order;             /* shape order 1..3 */
  int32_t pusher;            /* 0 Boris (+ set_gamma), 1 Vay */
  int32_t drift;             /* window margin (cells) around each tile */
  int32_t prec;              /* 0 float, 1 double */
  int32_t pitch_y;           /* allocated y extent of the E/B arrays */
  int64_t np;                /* particles */
  double dx, dy, dz, dt, q, m, clight, mu0, eps0, xmin, ymin, zmin;
  void *ex, *ey, *ez, *bx, *by, *bz;        /* guarded, engine precision */
  double *jx, *jy, *jz;                     /* nx*ny*nz */
  uint32_t* cell;                           /* packed cell index */
  void *ox, *oy, *oz, *ux, *uy, *uz, *w;    /* engine precision */
  uint32_t* cell_b;                         /* sort output buffers */
  void *ox_b, *oy_b, *oz_b, *ux_b, *uy_b, *uz_b, *w_b;
  int32_t *pid, *pid_b;                     /* optional particle ids (NULL: none),
                                               permuted by the sort only */
  int32_t* tile_off;                        /* ntiles + 1 */
  int32_t* tile_cnt;                        /* ntiles + 1 (sort scratch) */
  double* ke_tile;                          /* ntiles: kinetic energy per tile */
  int32_t* counters;                        /* [0] particles on the slow path,
                                               [1] error flag, [2] particles the FP32
                                               kernel deferred to its second pass
                                               (bank classes taken); int32[4] */
  int32_t* cell_cnt;                        /* sort scratch: ntiles * tile^3 */
  int32_t* rank_b;                          /* sort scratch: np */
  int32_t* perm;                            /* sort scratch: np */
  float* tile_stats;                        /* NULL, or 4 per tile: the bounds of the
                                               fixed-point current scale for the
                                               next step (max |u|^2, max |w|, max
                                               particles per window cell, valid);
                                               written by each particle step,
                                               invalidated by the sort */
  int32_t select_lanes;                     /* FP32 engine: 1 = each warp takes lanes of
                                               distinct bank classes and defers the
                                               others to a second, class-bucketed pass;
                                               0 = one pass (faster when many particles
                                               change cell per step) */
  int32_t cell_order;                       /* 1 = the sort leaves each tile's particles
                                               in cell order (the layout of the
                                               cell-grouped kernel, acc 4) and the
                                               bank re-layout leaves them in place;
                                               0 = bank order */
} pxrb_tiled_job;

/* Tile shapes: cubic tiles of edge tx = ty = tz = `tile` in {4, 8} with window
 * margin `drift` in {0, 1, 2} (8) or {0, 1} (4); the E/B arrays are allocated
 * with extents (pitch_x >= ntx*tile + 2g, pitch_y >= nty*tile + 2g,
 * ntz*tile + 2g) so that every tile window fits.  g >= drift + 2.
 * `acc` selects the shared-memory accumulator of a tile's current:
 * 0 FP32 atomics, 1 int32 fixed point, 2 64-bit fixed point held in two
 * native int32 words (default of the FP32 engine), 3 FP64 (FP64 engine),
 * 4 int32 fixed point with the cell-grouped kernel (FP32, shape orders 1 and
 * 3, tile edge 8 with margin 1, at most pxrb_tiled_max_threads(4) threads per
 * CTA): each step sorts a tile's particles by cell in shared memory and gives
 * each thread a pair of particles of one cell, which share every E/B window
 * load and sum their contributions to a J node before one atomic (tiles of
 * fewer than 2^21 particles: a larger tile sets the error flag and is left
 * unprocessed); jobs run with it set
 * `cell_order` so that the sort keeps cell order inside each tile.  The
 * fixed-point scales are bounded per tile from the tile's particle weights,
 * momenta, cell occupancy and fields, so no overflow is possible. */
/* Fused per-step particle kernel of the tiled engine: energy-conserving
 * gather (l_lower_order_in_v), Boris or Vay push, position push, periodic
 * wrap, and Esirkepov deposition from the exact old position into J (+=).
 * Restates, fused, field_gathering_plus_particle_pusher_{n}_{n}_{n}
 * (particle_pusher_manager_3d.F90:1287-2193), particle_bcs (periodic,
 * particle_boundaries.F90:1109-1300) and depose_jxjyjz_esirkepov_{n}_{n}_{n}
 * (esirkepov_3d.F90:82, :1734, :3263).  Persistent CTAs pull (job, tile)
 * items; the tile's E/B window and J accumulator live in shared memory;
 * particles that left the window since the last sort take a global-memory
 * path.  jobs_dev: DEVICE descriptors (all of this `order` and `prec`);
 * work: DEVICE int32 pairs (job, tile), nwork of them (nwork_dev, if not
 * NULL, a DEVICE count <= nwork read at run time); ctr: DEVICE int32 reset by
 * the call; threads: CTA size, multiple of 32, <= pxrb_tiled_max_threads(acc)
 * (256; 512 for the FP64 engine, which runs one CTA per SM); smem: dynamic shared
 * memory bytes, >= pxrb_tiled_smem_bytes() of the largest tile window. */
int pxrb_tiled_particle_step(const pxrb_tiled_job* jobs_dev, int32_t order, int32_t prec,
                             int32_t tile, int32_t drift, int32_t acc, const int32_t* work,
                             int32_t nwork,
                             const int32_t* nwork_dev, int32_t* ctr, int32_t threads,
                             int32_t ctas, int64_t smem, void* stream);

/* Arithmetic-throughput probe (no counterpart in the reference; it measures
 * the compute ceiling the particle kernels are compared with): `blocks` x
 * `threads` threads each run 8 independent chains a <- a*b + c for `iters`
 * rounds, kind 0 in FP32, 1 in packed f32x2 (two FP32 FMAs per instruction),
 * 2 in FP64, and write the sum of their chains to sink (DEVICE float[blocks *
 * threads]).  With b = 1 every chain ends at its start value + iters * c.
 * pxrb_fma_probe_flops gives the launch's floating-point operations (an FMA
 * counts two), or -1 for bad arguments (host function). */
int pxrb_fma_probe(int32_t kind, int32_t blocks, int32_t threads, int32_t iters, float b,
                   float c, float* sink, void* stream);
int64_t pxrb_fma_probe_flops(int32_t kind, int32_t blocks, int32_t threads, int32_t iters);

/* Largest CTA size (threads) pxrb_tiled_particle_step takes with accumulator
 * mode `acc` (host function, no GPU work). */
int32_t pxrb_tiled_max_threads(int32_t acc);

/* sizeof(pxrb_tiled_job), for bindings that mirror the struct. */
int64_t pxrb_tiled_job_size(void);

/* Dynamic shared memory the particle kernel needs for a tile shape, order,
 * window margin and precision (host function, no GPU work). */
int64_t pxrb_tiled_smem_bytes(int32_t order, int32_t prec, int32_t acc, int32_t tx,
                              int32_t ty, int32_t tz, int32_t drift);

/* Yee steps on the engine layout, every job in one launch (yee.F90:1258-1347
 * and :637-740; periodic guard images written by the same kernel).
 * push_b: B -= frac*dt*curl E.  push_e: E += c^2 dt curl B - c^2 mu0 dt J,
 * then J = 0 when zero_j != 0.  cell_off_dev: DEVICE int64[njobs+1], start of
 * each job in a flat cell index whose job segments are padded to multiples of
 * 1024 (PXRB_YEE_CELLS_PER_BLOCK); total_cells = cell_off[njobs] (host value),
 * a multiple of 1024. */
#define PXRB_YEE_CELLS_PER_BLOCK 1024
int pxrb_tiled_push_b(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, double frac,
                      void* stream);
int pxrb_tiled_push_e(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, int32_t zero_j,
                      void* stream);

/* Bank-order re-layout of every tile of njobs jobs, between sorts: each
 * tile's particles are put back into the sort's (level, bank class) order
 * for the cells they occupy now (particles keep their tile).  A step's cost
 * grows as particles change cells after a sort; this restores it for about
 * a third of a sort's memory traffic.  The particles are gathered into the
 * *_b buffers, which then trade places with the particle arrays in the
 * DEVICE descriptors: read the current pointers back from there before
 * using the arrays on the host side.  jobs_dev: DEVICE descriptors of
 * precision `prec` (cubic tiles of edge 4 or 8); max_tiles: at least every
 * job's tile count; max_np: the largest particle count (sizes the grid).
 * rank_b is scratch. */
int pxrb_tiled_relayout(pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                        int32_t max_tiles, int64_t max_np, void* stream);

/* Counting sort of one job's particles by cell tile: the B200 form of
 * pxr_particle_sorting (src/housekeeping/sorting.F90:67-361) with the tile of
 * the particle's cell as key.  Inside a tile the particles are laid out in
 * bank order: numbered within their bank class (the shared-memory bank of
 * their cell in the tile window, whose pitch gives every class the same
 * number of cells), then ordered by (number, class), so 32 consecutive
 * particles fall in distinct banks: a warp of the particle kernel then
 * gathers and deposits without bank conflicts until particles change cells.
 * Rebuilds tile_off.  The sorted particles land in the *_b buffers, which then
 * trade places with the particle arrays in the DEVICE descriptor (as in
 * pxrb_tiled_relayout): read the particle pointers back from there before
 * using the arrays on the host side.  cell_cnt / rank_b / perm are scratch.
 * job_host: host copy (sizes and scratch pointers); job_dev: the device copy
 * the kernels read and update. */
int pxrb_tiled_sort(const pxrb_tiled_job* job_host, pxrb_tiled_job* job_dev, void* stream);

/* The same sort for a batch of jobs in seven launches (an ensemble, the
 * reference's per-species pxr_particle_sorting over many simulations).
 * jobs_dev: DEVICE array of njobs descriptors, all of precision `prec`, each
 * with cubic tiles of edge 4 or 8 and cell_cnt / rank_b / perm set; max_tiles: at
 * least the tile count of every job; max_np: the largest particle count
 * (sizes the grid only).  The counters are cleared on the device, so the
 * call needs no host copy of the descriptors; the particle arrays trade
 * places with the *_b buffers in the descriptors, as in the single sort. */
int pxrb_tiled_sort_batch(pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                          int32_t max_tiles, int64_t max_np, void* stream);

/* Conversions between PICSAR's particle arrays (absolute FP64 positions,
 * u, weight; DEVICE) and the engine SoA of one job (unsorted after a load:
 * call pxrb_tiled_sort), and between PICSAR's guarded FP64 Fortran grids
 * (nguard guards) and the engine: which 0..5 = ex..bz, 6..8 = jx..jz.
 * job_host must hold the current particle pointers (after sorts, read the
 * device descriptor back first). */
int pxrb_tiled_load_particles(const pxrb_tiled_job* job_host, const double* x,
                              const double* y, const double* z, const double* ux,
                              const double* uy, const double* uz, const double* w,
                              void* stream);
int pxrb_tiled_store_particles(const pxrb_tiled_job* job_host, double* x, double* y,
                               double* z, double* ux, double* uy, double* uz,
                               double* gaminv, double* w, void* stream);
/* The same conversion to PICSAR's arrays in the order the particles were
 * added: particle i of the engine goes to row pid[i] of every output (the
 * tracked ids must be a permutation of 0..np-1; rows outside [0, np) are
 * skipped).  The particle pointers and ids are read from the DEVICE
 * descriptor job_dev, so no read-back is needed after sorts; np and prec
 * (0 FP32, 1 FP64) are the job's.  Nothing is written when the descriptor
 * tracks no ids.  One pass, in place of a conversion plus one scatter per
 * column. */
int pxrb_tiled_store_particles_by_id(const pxrb_tiled_job* job_dev, int64_t np, int32_t prec,
                                     double* x, double* y, double* z, double* ux, double* uy,
                                     double* uz, double* gaminv, double* w, void* stream);
int pxrb_tiled_field_import(const pxrb_tiled_job* job_host, int32_t which, const double* src,
                            int64_t nguard_src, void* stream);
int pxrb_tiled_field_export(const pxrb_tiled_job* job_host, int32_t which, double* dst,
                            int64_t nguard_dst, void* stream);

/* FP64 diagnostics of one job (diags.F90:847-1358): out[0] kinetic energy
 * sum (gamma-1) w m c^2 (from ke_tile, written by the particle kernel),
 * out[1..3] E energies (sum 0.5 F^2 dV * eps0), out[4..6] B energies
 * (/ mu0), out[7] || div E * eps0 - rho ||_2 and out[8] || rho ||_2 over the
 * periodic domain, with rho (DEVICE FP64 nx*ny*nz) zeroed and deposited here;
 * rho = NULL computes the energies only (out[7], out[8] = 0).
 * scratch: DEVICE double[scratch_len], scratch_len >= pxrb_tiled_diag_scratch();
 * out: DEVICE double[9]. */
int64_t pxrb_tiled_diag_scratch(const pxrb_tiled_job* job_host);
int pxrb_tiled_diagnostics(const pxrb_tiled_job* job_host, double* rho, double* scratch,
                           int64_t scratch_len, double* out, void* stream);

/* Same diagnostics for callers that cannot allocate device memory (no
 * counterpart in the reference): the rho grid and the partial sums live in a
 * static device array owned by the library, so only the job and out (DEVICE
 * double[9]) are passed; gauss = 0 computes the energies only (any job size).
 * With gauss != 0, jobs of more than 1,048,576 cells are rejected with
 * PXRB_ETOOLARGE.  Every GPU that loads the library keeps the ~8.1 MiB array
 * until exit; calls share it, so calls that overlap on the GPU race.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress)
 * and caches it for the process: make that call before any stream capture,
 * and make no call after cudaDeviceReset (the cached address is then stale). */
int pxrb_tiled_diagnostics_noalloc(const pxrb_tiled_job* job_host, int32_t gauss, double* out,
                                   void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PICSAR_B200_H */
