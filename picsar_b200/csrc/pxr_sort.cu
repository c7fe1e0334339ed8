// Bin sort of PICSAR's flat particle arrays (plain FP64 path): the B200 form
// of pxr_particle_bin_sorting (src/housekeeping/sorting.F90:247-361).
//
// The reference numbers the particles of a tile by bin, iz*nx3*ny3 + iy*nx3 +
// ix with (ix, iy, iz) = floor((x - xmin2) / dxf, ...), and reorders them by a
// counting sort that keeps the input order inside a bin (a stable sort by bin
// number).  Here the bin numbers are computed by one kernel, sorted with their
// particle indices by a stable device radix sort (CUB, compiled into this
// library), and every particle array is gathered through the sorted indices
// into a scratch column and copied back.  As in the reference, of the pid
// columns only the weight is carried along (sorting.F90:264, :336).
#include <cub/device/device_radix_sort.cuh>

#include "pxr_common.cuh"

namespace {

constexpr int SORT_TPB = 256;

struct BinParams {
  i64 np;
  const double *x, *y, *z;
  double x0, y0, z0;     // xmin2, ymin2, zmin2
  double dxi, dyi, dzi;  // 1 / bin size
  i64 nx3, ny3, nz3;
  int* key;
  int* idx;
};

__global__ void k_bin_keys(BinParams p) {
  const i64 nb = p.nx3 * p.ny3 * p.nz3;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    i64 ix = (i64)floor((p.x[i] - p.x0) * p.dxi);
    i64 iy = (i64)floor((p.y[i] - p.y0) * p.dyi);
    i64 iz = (i64)floor((p.z[i] - p.z0) * p.dzi);
    i64 b = iz * p.nx3 * p.ny3 + iy * p.nx3 + ix;
    // positions outside [min2, max2) (the reference checks only in DEBUG
    // builds) go to the nearest end bin
    b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
    p.key[i] = (int)b;
    p.idx[i] = (int)i;
  }
}

__global__ void k_gather_col(i64 np, const int* __restrict__ idx, const double* __restrict__ src,
                             double* __restrict__ dst) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < np;
       i += (i64)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

inline int sort_blocks(i64 n) {
  i64 b = (n + SORT_TPB - 1) / SORT_TPB;
  const i64 cap = 148 * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

size_t cub_bytes(i64 np) {
  size_t t = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t, (const int*)nullptr, (int*)nullptr,
                                  (const int*)nullptr, (int*)nullptr, (int)np);
  return t;
}

}  // namespace

extern "C" {

int64_t pxrb_particle_bin_sorting_scratch(int64_t np) {
  if (np < 0 || np > 0x7fffffff) return -1;
  const size_t col = align256((size_t)np * sizeof(int));
  return (int64_t)(4 * col + align256((size_t)np * sizeof(double)) + align256(cub_bytes(np)));
}

int pxrb_particle_bin_sorting(int64_t np, double* xp, double* yp, double* zp, double* ux,
                              double* uy, double* uz, double* gam, double* w, double xmin2,
                              double ymin2, double zmin2, double xmax2, double ymax2,
                              double zmax2, double dxf, double dyf, double dzf, void* scratch,
                              int64_t scratch_bytes, void* stream) {
  if (np < 0 || np > 0x7fffffff) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (!xp || !yp || !zp || !ux || !uy || !uz || !gam || !scratch) return PXRB_EINVAL;
  if (!(dxf > 0.0) || !(dyf > 0.0) || !(dzf > 0.0)) return PXRB_EINVAL;
  const int64_t need = pxrb_particle_bin_sorting_scratch(np);
  if (scratch_bytes < need) return PXRB_ESCRATCH;
  BinParams p;
  p.np = np; p.x = xp; p.y = yp; p.z = zp;
  p.x0 = xmin2; p.y0 = ymin2; p.z0 = zmin2;
  // dxi = 1./dxf as in the reference (a default-real 1 is exact)
  p.dxi = 1.0 / dxf; p.dyi = 1.0 / dyf; p.dzi = 1.0 / dzf;
  p.nx3 = (i64)ceil((xmax2 - xmin2) * p.dxi);
  p.ny3 = (i64)ceil((ymax2 - ymin2) * p.dyi);
  p.nz3 = (i64)ceil((zmax2 - zmin2) * p.dzi);
  if (p.nx3 < 1 || p.ny3 < 1 || p.nz3 < 1) return PXRB_EINVAL;
  const i64 nb = p.nx3 * p.ny3 * p.nz3;
  if (nb > 0x7fffffff) return PXRB_EINVAL;
  char* s = (char*)scratch;
  const size_t col = align256((size_t)np * sizeof(int));
  int* key_in = (int*)s;
  int* key_out = (int*)(s + col);
  int* idx_in = (int*)(s + 2 * col);
  int* idx_out = (int*)(s + 3 * col);
  double* tmp = (double*)(s + 4 * col);
  void* cub_tmp = s + 4 * col + align256((size_t)np * sizeof(double));
  size_t cub_len = cub_bytes(np);
  p.key = key_in; p.idx = idx_in;
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = sort_blocks(np);
  k_bin_keys<<<blocks, SORT_TPB, 0, st>>>(p);
  PXRB_CHECK_LAUNCH();
  int end_bit = 1;
  while (end_bit < 31 && ((i64)1 << end_bit) < nb) ++end_bit;
  if (cub::DeviceRadixSort::SortPairs(cub_tmp, cub_len, key_in, key_out, idx_in, idx_out,
                                      (int)np, 0, end_bit, st) != cudaSuccess)
    return PXRB_ELAUNCH;
  double* cols[8] = {xp, yp, zp, ux, uy, uz, gam, w};
  for (int c = 0; c < 8; ++c) {
    if (!cols[c]) continue;             // w (the pid weight column) is optional
    k_gather_col<<<blocks, SORT_TPB, 0, st>>>(np, idx_out, cols[c], tmp);
    PXRB_CHECK_LAUNCH();
    if (cudaMemcpyAsync(cols[c], tmp, (size_t)np * sizeof(double), cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess)
      return PXRB_ELAUNCH;
  }
  return PXRB_OK;
}

}  // extern "C"
