// Arbitrary-order Yee FDTD on PICSAR's guarded FP64 arrays (plain path):
// pxrpush_em3d_evec_norder / pxrpush_em3d_bvec_norder
// (src/field_solvers/Maxwell/yee_solver/yee.F90:46-123, :752-821) and the
// finite-difference weights FD_weights (src/submain.F90:927-984).
//
// One thread per node of [-nxs, nx+nxs] x [-nys, ny+nys] x [-nzs, nz+nzs];
// each thread updates the three components at its node.  The E kernel reads
// only B and J and the B kernel only E, so nodes are independent.  Per
// component the terms are added in the reference's order: -mudt*J first,
// then the stencil pairs i = 1, 2, ... of the first transverse axis, then
// those of the second.  The stencil is clipped where the array ends:
// i <= min(norder/2, n - j + guard, j + guard).
#include <cstring>

#include "pxr_common.cuh"

namespace {

constexpr int MAX_HALF = 16;           // norder <= 32 per axis

struct YeeNParams {
  double *ex, *ey, *ez, *bx, *by, *bz;
  const double *jx, *jy, *jz;
  GridG G;                              // common shape of the nine arrays
  int nxs, nys, nzs;
  int hx, hy, hz;                       // norder / 2 per axis
  int ist;                              // 1 staggered grid, 0 nodal grid
  double mudt;
  double cx[MAX_HALF], cy[MAX_HALF], cz[MAX_HALF];
};

__device__ __forceinline__ int clip(int half, int n, int g, int j) {
  return min(min(half, (n - j) + g), j + g);
}

__global__ void __launch_bounds__(256) k_yee_e_norder(YeeNParams p) {
  const int j = -p.nxs + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int k = -p.nys + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int l = -p.nzs + (int)blockIdx.z;
  const GridG& G = p.G;
  const int nx = (int)G.nx, ny = (int)G.ny, nz = (int)G.nz;
  const int gx = (int)G.gx, gy = (int)G.gy, gz = (int)G.gz;
  if (j > nx + p.nxs || k > ny + p.nys) return;
  const i64 c = G.idx(j, k, l);
  const int st = p.ist;
  const int iy = clip(p.hy, ny, gy, k), iz = clip(p.hz, nz, gz, l), ix = clip(p.hx, nx, gx, j);
  double e = p.ex[c] - p.mudt * p.jx[c];
  for (int i = 1; i <= iy; ++i)
    e = e + p.cy[i - 1] * (p.bz[G.idx(j, k + i - st, l)] - p.bz[G.idx(j, k - i, l)]);
  for (int i = 1; i <= iz; ++i)
    e = e - p.cz[i - 1] * (p.by[G.idx(j, k, l + i - st)] - p.by[G.idx(j, k, l - i)]);
  p.ex[c] = e;
  e = p.ey[c] - p.mudt * p.jy[c];
  for (int i = 1; i <= ix; ++i)
    e = e - p.cx[i - 1] * (p.bz[G.idx(j + i - st, k, l)] - p.bz[G.idx(j - i, k, l)]);
  for (int i = 1; i <= iz; ++i)
    e = e + p.cz[i - 1] * (p.bx[G.idx(j, k, l + i - st)] - p.bx[G.idx(j, k, l - i)]);
  p.ey[c] = e;
  e = p.ez[c] - p.mudt * p.jz[c];
  for (int i = 1; i <= ix; ++i)
    e = e + p.cx[i - 1] * (p.by[G.idx(j + i - st, k, l)] - p.by[G.idx(j - i, k, l)]);
  for (int i = 1; i <= iy; ++i)
    e = e - p.cy[i - 1] * (p.bx[G.idx(j, k + i - st, l)] - p.bx[G.idx(j, k - i, l)]);
  p.ez[c] = e;
}

__global__ void __launch_bounds__(256) k_yee_b_norder(YeeNParams p) {
  const int j = -p.nxs + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int k = -p.nys + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int l = -p.nzs + (int)blockIdx.z;
  const GridG& G = p.G;
  const int nx = (int)G.nx, ny = (int)G.ny, nz = (int)G.nz;
  const int gx = (int)G.gx, gy = (int)G.gy, gz = (int)G.gz;
  if (j > nx + p.nxs || k > ny + p.nys) return;
  const i64 c = G.idx(j, k, l);
  const int st = p.ist;
  const int iy = clip(p.hy, ny, gy, k), iz = clip(p.hz, nz, gz, l), ix = clip(p.hx, nx, gx, j);
  double b = p.bx[c];
  for (int i = 1; i <= iy; ++i)
    b = b - p.cy[i - 1] * (p.ez[G.idx(j, k + i, l)] - p.ez[G.idx(j, k - i + st, l)]);
  for (int i = 1; i <= iz; ++i)
    b = b + p.cz[i - 1] * (p.ey[G.idx(j, k, l + i)] - p.ey[G.idx(j, k, l - i + st)]);
  p.bx[c] = b;
  b = p.by[c];
  for (int i = 1; i <= ix; ++i)
    b = b + p.cx[i - 1] * (p.ez[G.idx(j + i, k, l)] - p.ez[G.idx(j - i + st, k, l)]);
  for (int i = 1; i <= iz; ++i)
    b = b - p.cz[i - 1] * (p.ex[G.idx(j, k, l + i)] - p.ex[G.idx(j, k, l - i + st)]);
  p.by[c] = b;
  b = p.bz[c];
  for (int i = 1; i <= ix; ++i)
    b = b - p.cx[i - 1] * (p.ey[G.idx(j + i, k, l)] - p.ey[G.idx(j - i + st, k, l)]);
  for (int i = 1; i <= iy; ++i)
    b = b + p.cy[i - 1] * (p.ex[G.idx(j, k + i, l)] - p.ex[G.idx(j, k - i + st, l)]);
  p.bz[c] = b;
}

int setup(YeeNParams& p, const double* dtsdx, const double* dtsdy, const double* dtsdz,
          int64_t nx, int64_t ny, int64_t nz, int64_t norderx, int64_t nordery,
          int64_t norderz, int64_t nxguard, int64_t nyguard, int64_t nzguard, int64_t nxs,
          int64_t nys, int64_t nzs, int64_t l_nodalgrid) {
  const int64_t no[3] = {norderx, nordery, norderz};
  const double* cf[3] = {dtsdx, dtsdy, dtsdz};
  double* dst[3] = {p.cx, p.cy, p.cz};
  int* half[3] = {&p.hx, &p.hy, &p.hz};
  for (int a = 0; a < 3; ++a) {
    if (no[a] < 2 || no[a] % 2 || no[a] / 2 > MAX_HALF) return PXRB_EUNSUPPORTED;
    if (!cf[a]) return PXRB_EINVAL;
    *half[a] = (int)(no[a] / 2);
    std::memset(dst[a], 0, sizeof(double) * MAX_HALF);
    std::memcpy(dst[a], cf[a], sizeof(double) * (size_t)(no[a] / 2));
  }
  if (nx < 0 || ny < 0 || nz < 0 || nxguard < 0 || nyguard < 0 || nzguard < 0)
    return PXRB_EINVAL;
  // the loop range must stay inside the arrays
  if (nxs < 0 || nys < 0 || nzs < 0 || nxs > nxguard || nys > nyguard || nzs > nzguard)
    return PXRB_ERANGE;
  p.G = make_grid(nx, ny, nz, nxguard, nyguard, nzguard);
  p.nxs = (int)nxs; p.nys = (int)nys; p.nzs = (int)nzs;
  p.ist = l_nodalgrid ? 0 : 1;
  return PXRB_OK;
}

void launch_dims(const YeeNParams& p, dim3& grd, dim3& blk) {
  blk = dim3(32, 8, 1);
  grd = dim3((unsigned)((p.G.nx + 2 * p.nxs + 1 + 31) / 32),
             (unsigned)((p.G.ny + 2 * p.nys + 1 + 7) / 8), (unsigned)(p.G.nz + 2 * p.nzs + 1));
}

}  // namespace

extern "C" {

int pxrb_push_em3d_evec_norder(double* ex, double* ey, double* ez, const double* bx,
                               const double* by, const double* bz, const double* jx,
                               const double* jy, const double* jz, double mudt,
                               const double* dtsdx, const double* dtsdy, const double* dtsdz,
                               int64_t nx, int64_t ny, int64_t nz, int64_t norderx,
                               int64_t nordery, int64_t norderz, int64_t nxguard,
                               int64_t nyguard, int64_t nzguard, int64_t nxs, int64_t nys,
                               int64_t nzs, int64_t l_nodalgrid, void* stream) {
  if (!ex || !ey || !ez || !bx || !by || !bz || !jx || !jy || !jz) return PXRB_EINVAL;
  YeeNParams p;
  const int rc = setup(p, dtsdx, dtsdy, dtsdz, nx, ny, nz, norderx, nordery, norderz, nxguard,
                       nyguard, nzguard, nxs, nys, nzs, l_nodalgrid);
  if (rc) return rc;
  p.ex = ex; p.ey = ey; p.ez = ez;
  p.bx = const_cast<double*>(bx); p.by = const_cast<double*>(by); p.bz = const_cast<double*>(bz);
  p.jx = jx; p.jy = jy; p.jz = jz;
  p.mudt = mudt;
  dim3 grd, blk;
  launch_dims(p, grd, blk);
  k_yee_e_norder<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_push_em3d_bvec_norder(const double* ex, const double* ey, const double* ez,
                               double* bx, double* by, double* bz, const double* dtsdx,
                               const double* dtsdy, const double* dtsdz, int64_t nx, int64_t ny,
                               int64_t nz, int64_t norderx, int64_t nordery, int64_t norderz,
                               int64_t nxguard, int64_t nyguard, int64_t nzguard, int64_t nxs,
                               int64_t nys, int64_t nzs, int64_t l_nodalgrid, void* stream) {
  if (!ex || !ey || !ez || !bx || !by || !bz) return PXRB_EINVAL;
  YeeNParams p;
  const int rc = setup(p, dtsdx, dtsdy, dtsdz, nx, ny, nz, norderx, nordery, norderz, nxguard,
                       nyguard, nzguard, nxs, nys, nzs, l_nodalgrid);
  if (rc) return rc;
  p.ex = const_cast<double*>(ex); p.ey = const_cast<double*>(ey); p.ez = const_cast<double*>(ez);
  p.bx = bx; p.by = by; p.bz = bz;
  p.jx = p.jy = p.jz = nullptr;
  p.mudt = 0.0;
  dim3 grd, blk;
  launch_dims(p, grd, blk);
  k_yee_b_norder<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

// Fornberg's recursion (B. Fornberg, "Generation of finite difference
// formulas on arbitrarily spaced grids", Math. Comp. 51 (1988)) for the
// weights of the first derivative at z on the points x_i = i - n/2 + 1,
// i = 0..n-1, n = norder + 1; z = 1/2 on the staggered grid, 0 on the nodal
// one.  coeffs[i-1] = weight of point n/2 + i - 1 (i = 1..norder/2), as
// FD_weights returns them.  Host function.
int pxrb_fd_weights(double* coeffs, int64_t norder, int64_t l_nodal) {
  if (!coeffs || norder < 2 || norder % 2 || norder > 2 * MAX_HALF) return PXRB_EINVAL;
  const double z = l_nodal ? 0.0 : 0.5;
  const int n = (int)norder + 1;
  double x[2 * MAX_HALF + 1], d0[2 * MAX_HALF + 1], d1[2 * MAX_HALF + 1];
  for (int i = 0; i < n; ++i) { x[i] = (double)(i - n / 2 + 1); d0[i] = d1[i] = 0.0; }
  // d0 / d1: weights of the 0th / 1st derivative
  double c1 = 1.0, c4 = x[0] - z;
  d0[0] = 1.0;
  for (int i = 1; i < n; ++i) {
    double c2 = 1.0;
    const double c5 = c4;
    c4 = x[i] - z;
    for (int j = 0; j < i; ++j) {
      const double c3 = x[i] - x[j];
      c2 = c2 * c3;
      if (j == i - 1) {
        d1[i] = c1 * (1 * d0[i - 1] - c5 * d1[i - 1]) / c2;
        d0[i] = -c1 * c5 * d0[i - 1] / c2;
      }
      if (j == i - 1) {
        d1[j] = (c4 * d1[j] - 1 * d0[j]) / c3;
        d0[j] = c4 * d0[j] / c3;
      }
    }
    c1 = c2;
  }
  for (int i = 1; i <= (int)norder / 2; ++i) coeffs[i - 1] = d1[norder / 2 + i - 1];
  return PXRB_OK;
}

}  // extern "C"
