// Particle boundary conditions of one domain (plain FP64 path): the B200 form
// of the per-axis pbound cases of particle_bcs (src/boundary_conditions/
// particle_boundaries.F90:1098-1300, single domain, every side a domain
// boundary).  Per side, in the reference's order x-, x+, y-, y+, z-, z+:
//   0 periodic     x +- (xmax_part - xmin_part)
//   1 absorbing    the particle is removed (no further axis is looked at)
//   2 reflecting   x moved one cell inwards (x +- dx), u along the axis negated
//   3 reinjecting  x mirrored at the boundary, u = 0, position clamped into
//                  the tile's particle region less half a cell per axis (no
//                  further axis is looked at)
// The side tests use the position before any change along that axis, as the
// reference does (part_xyz).  Removed particles are compacted out with a
// stable prefix sum (the reference swaps the last particle into the hole; the
// particle set is the same).
#include <cub/device/device_scan.cuh>

#include "pxr_common.cuh"

namespace {

constexpr int BC_TPB = 256;

struct BcPart {
  i64 np;
  double *x, *y, *z, *ux, *uy, *uz;
  double lo[3], hi[3], d[3];
  double tlo[3], thi[3];    // tile particle region (reinjection clamps)
  int pb[6];
  int* keep;
};

__global__ void k_particle_bcs(BcPart p) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double* pos[3] = {p.x + i, p.y + i, p.z + i};
    double* mom[3] = {p.ux + i, p.uy + i, p.uz + i};
    int keep = 1;
    bool stop = false;
    for (int a = 0; a < 3 && !stop; ++a) {
      const double orig = *pos[a];
      const double len = p.hi[a] - p.lo[a];
      for (int side = 0; side < 2 && !stop; ++side) {
        const bool out = side == 0 ? orig < p.lo[a] : orig >= p.hi[a];
        if (!out) continue;
        const int code = p.pb[2 * a + side];
        const double sg = side == 0 ? 1.0 : -1.0;
        if (code == 1) {
          keep = 0;
          stop = true;
        } else if (code == 2) {
          *pos[a] = orig + sg * p.d[a];
          *mom[a] = -*mom[a];
        } else if (code == 3) {
          const double wall = side == 0 ? p.lo[a] : p.hi[a];
          *pos[a] = 2.0 * wall - *pos[a];
          *mom[0] = 0.0; *mom[1] = 0.0; *mom[2] = 0.0;
          for (int b = 0; b < 3; ++b) {
            *pos[b] = fmax(*pos[b], p.tlo[b] + 0.5 * p.d[b]);
            *pos[b] = fmin(*pos[b], p.thi[b] - 0.5 * p.d[b]);
          }
          stop = true;
        } else {
          *pos[a] = orig + sg * len;
        }
      }
    }
    p.keep[i] = keep;
  }
}

__global__ void k_compact_col(i64 np, const int* __restrict__ keep, const int* __restrict__ pos,
                              const double* __restrict__ src, double* __restrict__ dst) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < np;
       i += (i64)gridDim.x * blockDim.x)
    if (keep[i]) dst[pos[i]] = src[i];
}

__global__ void k_count(i64 np, const int* keep, const int* pos, int64_t* np_out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *np_out = (int64_t)pos[np - 1] + keep[np - 1];
}

__global__ void k_set_count(int64_t* np_out, i64 np) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *np_out = np;
}

inline int bc_blocks(i64 n) {
  i64 b = (n + BC_TPB - 1) / BC_TPB;
  const i64 cap = 148 * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

inline size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

size_t scan_bytes(i64 np) {
  size_t t = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, t, (const int*)nullptr, (int*)nullptr, (int)np);
  return t;
}

}  // namespace

extern "C" {

int64_t pxrb_particle_bcs_scratch(int64_t np) {
  if (np < 0 || np > 0x7fffffff) return -1;
  return (int64_t)(2 * al256((size_t)np * sizeof(int)) + al256((size_t)np * sizeof(double)) +
                   al256(scan_bytes(np)));
}

int pxrb_particle_bcs(int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
                      double* uzp, double* gaminv, double* w, double* pid, double xmin_part,
                      double ymin_part, double zmin_part, double xmax_part, double ymax_part,
                      double zmax_part, double dx, double dy, double dz, const int64_t* pbound,
                      const double* tile_lo, const double* tile_hi, void* scratch,
                      int64_t scratch_bytes, int64_t* np_out, void* stream) {
  if (np < 0 || np > 0x7fffffff || !pbound || !tile_lo || !tile_hi || !np_out)
    return PXRB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (np == 0) {
    if (cudaMemsetAsync(np_out, 0, sizeof(int64_t), st) != cudaSuccess) return PXRB_ELAUNCH;
    return PXRB_OK;
  }
  if (!xp || !yp || !zp || !uxp || !uyp || !uzp || !scratch) return PXRB_EINVAL;
  if (scratch_bytes < pxrb_particle_bcs_scratch(np)) return PXRB_ESCRATCH;
  BcPart p;
  p.np = np;
  p.x = xp; p.y = yp; p.z = zp; p.ux = uxp; p.uy = uyp; p.uz = uzp;
  p.lo[0] = xmin_part; p.lo[1] = ymin_part; p.lo[2] = zmin_part;
  p.hi[0] = xmax_part; p.hi[1] = ymax_part; p.hi[2] = zmax_part;
  p.d[0] = dx; p.d[1] = dy; p.d[2] = dz;
  for (int a = 0; a < 3; ++a) { p.tlo[a] = tile_lo[a]; p.thi[a] = tile_hi[a]; }
  bool removes = false;
  for (int s = 0; s < 6; ++s) {
    if (pbound[s] < 0 || pbound[s] > 3) return PXRB_EUNSUPPORTED;
    p.pb[s] = (int)pbound[s];
    removes = removes || pbound[s] == 1;
  }
  char* s = (char*)scratch;
  const size_t ci = al256((size_t)np * sizeof(int));
  p.keep = (int*)s;
  int* pos = (int*)(s + ci);
  double* tmp = (double*)(s + 2 * ci);
  void* scan_tmp = s + 2 * ci + al256((size_t)np * sizeof(double));
  size_t scan_len = scan_bytes(np);
  const int blocks = bc_blocks(np);
  k_particle_bcs<<<blocks, BC_TPB, 0, st>>>(p);
  PXRB_CHECK_LAUNCH();
  if (!removes) {
    k_set_count<<<1, 32, 0, st>>>(np_out, np);
    PXRB_CHECK_LAUNCH();
    return PXRB_OK;
  }
  if (cub::DeviceScan::ExclusiveSum(scan_tmp, scan_len, p.keep, pos, (int)np, st) !=
      cudaSuccess)
    return PXRB_ELAUNCH;
  double* cols[9] = {xp, yp, zp, uxp, uyp, uzp, gaminv, w, pid};
  for (int c = 0; c < 9; ++c) {
    if (!cols[c]) continue;
    k_compact_col<<<blocks, BC_TPB, 0, st>>>(np, p.keep, pos, cols[c], tmp);
    PXRB_CHECK_LAUNCH();
    if (cudaMemcpyAsync(cols[c], tmp, (size_t)np * sizeof(double), cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess)
      return PXRB_ELAUNCH;
  }
  k_count<<<1, 32, 0, st>>>(np, p.keep, pos, np_out);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"
