// Tiled engine: the B200-native per-step particle loop.
//
// Layout (see pxrb_tiled_job in picsar_b200.h): E/B in the engine precision R
// (float or double) with g periodic guard cells, J in FP64 without guards,
// particles sorted by cell tile as (packed cell, in-cell offset, u, w).
//
// One fused kernel per step does, for every tile: stage the tile's E/B window
// in shared memory, gather + push + position update + periodic wrap for each
// particle of the tile, and Esirkepov deposition from the exact old position
// into a shared-memory J window, flushed once to the global FP64 J with
// atomics.  Particles that drifted out of the tile window since the last sort
// use the global-memory path (same arithmetic, global loads/atomics).
//
// Formulas: gather/push particle_pusher_manager_3d.F90:1287-2193 (energy
// conserving, l_lower_order_in_v), Boris boris_3d.F90:96-131 + set_gamma,
// Vay vay_3d.F90:100-130, Esirkepov esirkepov_3d.F90:82-239, :1734-1918,
// :3263-3464, Yee yee.F90:637-740, :1258-1347.
#include "pxr_common.cuh"
#include "picsar_b200.h"

#include <cub/block/block_scan.cuh>
#include <mutex>
#include <algorithm>

namespace pxrt {
int launch_order1(int, int, int, int, const pxrb_tiled_job*, const int2*, int, const int*, int*, int, int, size_t, cudaStream_t);
int launch_order2(int, int, int, int, const pxrb_tiled_job*, const int2*, int, const int*, int*, int, int, size_t, cudaStream_t);
int launch_order3(int, int, int, int, const pxrb_tiled_job*, const int2*, int, const int*, int*, int, int, size_t, cudaStream_t);
}  // namespace pxrt

#include "pxr_tiled_kernel.cuh"

namespace {
using namespace pxrt;
// ---------------------------------------------------------------------------
// Yee on the guarded engine layout, all jobs in one launch.  Thread = cell.
// cell_off[j]: start of job j in the flat cell index space (multiple of the
// block size).  Writes the periodic images of each updated value into the
// guard cells.
// ---------------------------------------------------------------------------
constexpr int YEE_TPB = 256;

__device__ __forceinline__ int find_job(const int64_t* off, int njobs, int64_t gid) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= gid) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename R>
__device__ __forceinline__ void store_images(R* base, int i, int j, int k, int nx, int ny,
                                             int nz, int G, int pitch, int NYg, R v) {
  int ii[2] = {i, 0}, jj[2] = {j, 0}, kk[2] = {k, 0};
  int ni = 1, nj = 1, nk = 1;
  if (i < G) ii[ni++] = i + nx; else if (i >= nx - G) ii[ni++] = i - nx;
  if (j < G) jj[nj++] = j + ny; else if (j >= ny - G) jj[nj++] = j - ny;
  if (k < G) kk[nk++] = k + nz; else if (k >= nz - G) kk[nk++] = k - nz;
  for (int c = 0; c < nk; ++c)
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a)
        base[(ii[a] + G) + (i64)pitch * ((jj[b] + G) + (i64)NYg * (kk[c] + G))] = v;
}

// Cell (i, j, k) of a job's flat cell index (x fastest).  The flat index of
// one job is below 2^32 (2^32 cells of the engine's layout exceed any one
// GPU's memory), so 32-bit divisions suffice.
__device__ __forceinline__ void yee_ijk(int64_t lid, int nx, int ny, int& i, int& j, int& k) {
  const uint32_t l = (uint32_t)lid, ux = (uint32_t)nx, uy = (uint32_t)ny;
  const uint32_t t = l / ux;
  i = (int)(l - t * ux);
  const uint32_t kk = t / uy;
  j = (int)(t - kk * uy);
  k = (int)kk;
}

// Each thread updates YEE_CPT cells spaced by the block size, loading all of
// them before computing (memory-level parallelism); a block covers YEE_CPB
// consecutive cells of one job.
constexpr int YEE_CPT = 4;
constexpr int YEE_CPB = YEE_TPB * YEE_CPT;

template <typename R>
__global__ void __launch_bounds__(YEE_TPB)
    k_yee_b_t(const Job* __restrict__ jobs, int njobs, const int64_t* __restrict__ off, R frac) {
  __shared__ int s_job;
  __shared__ R s_c[3];
  const int64_t gid0 = (int64_t)blockIdx.x * YEE_CPB;
  if (threadIdx.x == 0) {
    const int jb = find_job(off, njobs, gid0);
    const Job& J0 = jobs[jb];
    s_job = jb;
    s_c[0] = (R)(frac * J0.dt / J0.dx);
    s_c[1] = (R)(frac * J0.dt / J0.dy);
    s_c[2] = (R)(frac * J0.dt / J0.dz);
  }
  __syncthreads();
  const Job& J = jobs[s_job];
  const int64_t l0 = gid0 - off[s_job] + threadIdx.x;
  const int nx = J.nx, ny = J.ny, nz = J.nz;
  const int64_t ncell = (int64_t)nx * ny * nz;
  const int G = J.g, pitch = J.pitch_x, NYg = J.pitch_y;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  const R* ex = (const R*)J.ex; const R* ey = (const R*)J.ey; const R* ez = (const R*)J.ez;
  R* bx = (R*)J.bx; R* by = (R*)J.by; R* bz = (R*)J.bz;
  const R dtsdx = s_c[0], dtsdy = s_c[1], dtsdz = s_c[2];
  int ci[YEE_CPT], cj[YEE_CPT], ck[YEE_CPT];
  R vbx[YEE_CPT], vby[YEE_CPT], vbz[YEE_CPT];
#pragma unroll
  for (int u = 0; u < YEE_CPT; ++u) {
    const int64_t lid = l0 + u * YEE_TPB;
    if (lid < ncell) {
      yee_ijk(lid, nx, ny, ci[u], cj[u], ck[u]);
      const i64 c = (ci[u] + G) + sy * (cj[u] + G) + sz * (ck[u] + G);
      const R ezc = ez[c], eyc = ey[c], exc = ex[c];
      vbx[u] = bx[c] - dtsdy * (ez[c + sy] - ezc) + dtsdz * (ey[c + sz] - eyc);
      vby[u] = by[c] + dtsdx * (ez[c + 1] - ezc) - dtsdz * (ex[c + sz] - exc);
      vbz[u] = bz[c] - dtsdx * (ey[c + 1] - eyc) + dtsdy * (ex[c + sy] - exc);
    }
  }
#pragma unroll
  for (int u = 0; u < YEE_CPT; ++u) {
    if (l0 + u * YEE_TPB < ncell) {
      store_images(bx, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vbx[u]);
      store_images(by, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vby[u]);
      store_images(bz, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vbz[u]);
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(YEE_TPB)
    k_yee_e_t(const Job* __restrict__ jobs, int njobs, const int64_t* __restrict__ off,
              int zero_j) {
  __shared__ int s_job;
  __shared__ R s_c[4];
  const int64_t gid0 = (int64_t)blockIdx.x * YEE_CPB;
  if (threadIdx.x == 0) {
    const int jb = find_job(off, njobs, gid0);
    const Job& J0 = jobs[jb];
    s_job = jb;
    const double c2 = J0.clight * J0.clight;
    s_c[0] = (R)(c2 * J0.mu0 * J0.dt);
    s_c[1] = (R)(c2 * J0.dt / J0.dx);
    s_c[2] = (R)(c2 * J0.dt / J0.dy);
    s_c[3] = (R)(c2 * J0.dt / J0.dz);
  }
  __syncthreads();
  const Job& J = jobs[s_job];
  const int64_t l0 = gid0 - off[s_job] + threadIdx.x;
  const int nx = J.nx, ny = J.ny, nz = J.nz;
  const int64_t ncell = (int64_t)nx * ny * nz;
  const int G = J.g, pitch = J.pitch_x, NYg = J.pitch_y;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  R* ex = (R*)J.ex; R* ey = (R*)J.ey; R* ez = (R*)J.ez;
  const R* bx = (const R*)J.bx; const R* by = (const R*)J.by; const R* bz = (const R*)J.bz;
  double* jxp = J.jx; double* jyp = J.jy; double* jzp = J.jz;
  const R mudt = s_c[0], dtsdx = s_c[1], dtsdy = s_c[2], dtsdz = s_c[3];
  int ci[YEE_CPT], cj[YEE_CPT], ck[YEE_CPT];
  R vex[YEE_CPT], vey[YEE_CPT], vez[YEE_CPT];
#pragma unroll
  for (int u = 0; u < YEE_CPT; ++u) {
    const int64_t lid = l0 + u * YEE_TPB;
    if (lid < ncell) {
      yee_ijk(lid, nx, ny, ci[u], cj[u], ck[u]);
      const i64 c = (ci[u] + G) + sy * (cj[u] + G) + sz * (ck[u] + G);
      const R jxv = (R)jxp[lid], jyv = (R)jyp[lid], jzv = (R)jzp[lid];
      const R bzc = bz[c], byc = by[c], bxc = bx[c];
      vex[u] = ex[c] + dtsdy * (bzc - bz[c - sy]) - dtsdz * (byc - by[c - sz]) - mudt * jxv;
      vey[u] = ey[c] - dtsdx * (bzc - bz[c - 1]) + dtsdz * (bxc - bx[c - sz]) - mudt * jyv;
      vez[u] = ez[c] + dtsdx * (byc - by[c - 1]) - dtsdy * (bxc - bx[c - sy]) - mudt * jzv;
    }
  }
#pragma unroll
  for (int u = 0; u < YEE_CPT; ++u) {
    const int64_t lid = l0 + u * YEE_TPB;
    if (lid < ncell) {
      if (zero_j) { jxp[lid] = 0.0; jyp[lid] = 0.0; jzp[lid] = 0.0; }
      store_images(ex, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vex[u]);
      store_images(ey, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vey[u]);
      store_images(ez, ci[u], cj[u], ck[u], nx, ny, nz, G, pitch, NYg, vez[u]);
    }
  }
}

// ---------------------------------------------------------------------------
// Counting sort by tile (cubic tiles, edge 4 or 8).
//   count:    per particle, its rank inside its cell (atomic on the cell's
//             counter, kept in rank_b);
//   cellscan: per tile, cell counts -> exclusive prefixes in place (cell_cnt)
//             and the tile total (tile_cnt);
//   scan:     tile totals -> tile_off;
//   perm:     perm[tile_off + prefix(cell) + rank] = p (cell-major order
//             inside the tile; only a 4-byte index moves);
//   map:      per tile (one warp), the bank-order destination of every
//             particle (k_tile_map, below), stored as its source in cell_b;
//   gather:   in destination order into the *_b buffers (coalesced writes),
//             which then trade places with the particle arrays in the
//             device descriptors (k_swap_particle_buffers).
// ---------------------------------------------------------------------------
struct TileCell {
  int t, lc;
};
__device__ __forceinline__ TileCell tile_cell(const Job& J, uint32_t cell) {
  int i, j, k;
  unpack_cell(cell, i, j, k);
  const int sh = __ffs(J.tx) - 1, m = J.tx - 1;      // power-of-two edge
  TileCell r;
  r.t = (i >> sh) + J.ntx * ((j >> sh) + J.nty * (k >> sh));
  r.lc = (i & m) + J.tx * ((j & m) + J.tx * (k & m));
  return r;
}

// Clears the tile counters and per-cell counters of every job of a batch
// (job = blockIdx.y), in place of the single-job path's memsets.
__global__ void k_sort_zero(const Job* __restrict__ jp) {
  const Job& J = jp[blockIdx.y];
  const i64 ntiles = (i64)J.ntx * J.nty * J.ntz;
  const i64 ncell = ntiles * J.tx * J.ty * J.tz;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < ncell + ntiles + 1;
       i += (i64)gridDim.x * blockDim.x) {
    if (i <= ntiles) J.tile_cnt[i] = 0;
    else J.cell_cnt[i - ntiles - 1] = 0;
  }
  if (J.tile_stats)        // tiles get new particles: the carried bounds are void
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < 4 * ntiles;
         i += (i64)gridDim.x * blockDim.x)
      J.tile_stats[i] = 0.f;
}

__global__ void k_sort_count(const Job* __restrict__ jp) {
  const Job J = jp[blockIdx.y];            // by value: fields stay in registers
  const int T3 = J.tx * J.tx * J.tx;
  const uint32_t* __restrict__ cell = J.cell;
  int* __restrict__ rank = J.rank_b;
  int* __restrict__ cc = J.cell_cnt;
  const i64 np = J.np;
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < np;
       p += (i64)gridDim.x * blockDim.x) {
    const TileCell tc = tile_cell(J, cell[p]);
    rank[p] = atomicAdd(&cc[(i64)tc.t * T3 + tc.lc], 1);
  }
}

// One warp per tile: exclusive prefix of the tile's cell counts, in place,
// and the tile total.
constexpr int CS_TPB = 256;
__global__ void __launch_bounds__(CS_TPB) k_sort_cellscan(const Job* __restrict__ jp) {
  const Job& J = jp[blockIdx.y];
  const int ntiles = J.ntx * J.nty * J.ntz;
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x * (CS_TPB / 32) + (threadIdx.x >> 5);
  if (t >= ntiles) return;
  const int T3 = J.tx * J.tx * J.tx, per = (T3 + 31) / 32;
  int* c = J.cell_cnt + (i64)t * T3;
  int v[16];
  int sum = 0;
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int lc = lane * per + u;
    v[u] = (u < per && lc < T3) ? c[lc] : 0;
    sum += v[u];
  }
  int incl = sum;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  int run = incl - sum;
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int lc = lane * per + u;
    if (u < per && lc < T3) { c[lc] = run; run += v[u]; }
  }
  if (lane == 31) J.tile_cnt[t] = incl;
}

constexpr int SCAN_TPB = 1024;

// exclusive scan of tile_cnt into tile_off
__global__ void __launch_bounds__(SCAN_TPB) k_sort_scan(const Job* __restrict__ jp) {
  typedef cub::BlockScan<int, SCAN_TPB> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry;
  const Job& J = jp[blockIdx.y];
  const int ntiles = J.ntx * J.nty * J.ntz;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ntiles; base += SCAN_TPB) {
    int t = base + threadIdx.x;
    int v = t < ntiles ? J.tile_cnt[t] : 0;
    int ex, tot;
    Scan(tmp).ExclusiveSum(v, ex, tot);
    int c0 = carry;
    if (t < ntiles) J.tile_off[t] = c0 + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry = c0 + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) J.tile_off[ntiles] = carry;
}

__global__ void k_sort_perm(const Job* __restrict__ jp) {
  const Job J = jp[blockIdx.y];
  const int T3 = J.tx * J.tx * J.tx;
  const uint32_t* __restrict__ cell = J.cell;
  const int* __restrict__ rank = J.rank_b;
  const int* __restrict__ cc = J.cell_cnt;
  const int* __restrict__ toff = J.tile_off;
  int* __restrict__ perm = J.perm;
  const i64 np = J.np;
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < np;
       p += (i64)gridDim.x * blockDim.x) {
    const TileCell tc = tile_cell(J, cell[p]);
    perm[toff[tc.t] + cc[(i64)tc.t * T3 + tc.lc] + rank[p]] = (int)p;
  }
}

// Bank-class layout inside each tile.  The class of a particle is the
// shared-memory window address of its stencil origin mod 32, i.e. of its cell
// in the particle kernel's padded window pitch (at order 2 the stencils start
// at the nearest node, so the cell is shifted by one along each axis where
// the in-cell offset is >= 1/2).  The tile's particles, taken cell-major, are
// numbered within their class (level) and laid out by (level, class): every
// 32 consecutive particles then sit in distinct classes, hence distinct banks
// for every gather load and deposit atomic of a warp, until the smallest
// class runs out; only the tail beyond it repeats classes, and cell-major
// numbering keeps those repeats mostly within one cell (one address, a
// broadcast for the loads).  k_tile_map (below) computes the destinations,
// k_relayout_gather moves the particles.
constexpr int RR_MAXC = 512;        // cells per tile (tile edge <= 8)

// Bank-order re-layout of every tile, between sorts (the tiles keep their
// particle ranges).  Particles that changed cell since the last layout put
// two lanes of a warp into one bank class, and the warp's window loads and
// atomics then replay: with thermal motion the step's cost grows by about a
// third within 20 steps.  This restores the sort's (level, class) order from
// the particles' current cells: k_tile_map numbers the classes in the tile's
// current order and finds every particle's destination; the gather then
// moves the particles into the *_b buffers in destination order, and those
// trade places with the particle arrays in the descriptors.

// One warp per tile: classes numbered in input order with per-class counters
// in shared memory (no block barriers), then the destination of every
// particle from the level table, stored as the source of that destination.
// CELL_MAJOR: the input order is the sort's cell-major permutation (perm);
// otherwise the tile's current order.  Scratch: rank_b (level and class per
// input slot); output: cell_b (source particle per destination).
constexpr int TM_WARPS = 4;         // tiles per CTA
constexpr int TM_LEVELS = 256;      // level table entries per tile
constexpr int TM_SEG = 4096;        // classes staged per tile segment

template <typename R, bool CELL_MAJOR>
__global__ void __launch_bounds__(TM_WARPS * 32) k_tile_map(const Job* __restrict__ jp) {
  __shared__ int s_cnt[TM_WARPS][32];
  __shared__ int s_P[TM_WARPS][TM_LEVELS];
  __shared__ unsigned s_M[TM_WARPS][TM_LEVELS];
  __shared__ unsigned char s_cls[TM_WARPS][TM_SEG];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const Job& J = jp[blockIdx.y];
  const int t = blockIdx.x * TM_WARPS + wid;
  const int ntl = J.ntx * J.nty * J.ntz;
  if (t >= ntl) return;                       // whole warp
  const int b0 = J.tile_off[t], b1 = J.tile_off[t + 1];
  if (b0 == b1) return;
  if (J.cell_order) {
    // cell order: the sort's permutation as it is; a re-layout keeps the
    // current order (the cell-grouped kernel groups by cell itself)
    for (int i = b0 + lane; i < b1; i += 32)
      J.cell_b[i] = CELL_MAJOR ? (uint32_t)J.perm[i] : (uint32_t)i;
    return;
  }
  const int T = J.tx, D = J.drift, nx = J.nx, ny = J.ny, nz = J.nz;
  const int L = J.order == 1 ? 0 : 1, H = J.order == 1 ? 1 : 2;
  const int W = T + 2 * D + L + H;
  const int SY = pxrt::win_sy(T, W), SZ = pxrt::win_sz(T, W);
  const int ntx = J.ntx, nty = J.nty;
  const int x0 = (t % ntx) * T, y0 = ((t / ntx) % nty) * T, z0 = (t / (ntx * nty)) * T;
  const int tex = min(T, nx - x0), tey = min(T, ny - y0), tez = min(T, nz - z0);
  const bool half = J.order == 2;
  const uint32_t* __restrict__ cell = J.cell;
  const R* __restrict__ ox = (const R*)J.ox;
  const R* __restrict__ oy = (const R*)J.oy;
  const R* __restrict__ oz = (const R*)J.oz;
  const int* __restrict__ perm = J.perm;
  int* key_at = J.rank_b;
  uint32_t* src_at = J.cell_b;
  int* cnt = s_cnt[wid];
  auto source = [&](int sl) { return CELL_MAJOR ? __ldg(perm + sl) : sl; };
  // class of a particle from its current cell (window-relative, periodic)
  auto class_of = [&](int p) {
    const uint32_t c = __ldg(cell + p);
    int x = (int)(c & 2047u) - x0, y = (int)((c >> 11) & 2047u) - y0, z = (int)(c >> 22) - z0;
    if (x > tex - 1 + D) x -= nx; else if (x < -D) x += nx;
    if (y > tey - 1 + D) y -= ny; else if (y < -D) y += ny;
    if (z > tez - 1 + D) z -= nz; else if (z < -D) z += nz;
    if (half) {
      x += __ldg(ox + p) >= (R)0.5 ? 1 : 0;
      y += __ldg(oy + p) >= (R)0.5 ? 1 : 0;
      z += __ldg(oz + p) >= (R)0.5 ? 1 : 0;
    }
    return (x + SY * y + SZ * z) & 31;
  };
  const bool packed = b1 - b0 < (1 << 26);    // level and class in one int
  cnt[lane] = 0;
  // per segment: the classes first (independent loads, several in flight)
  // into shared memory, then the numbering pass over them in order
  constexpr int U = 4;
  unsigned char* cls = s_cls[wid];
  for (int seg = b0; seg < b1; seg += TM_SEG) {
    const int sn = min(TM_SEG, b1 - seg);
    for (int i0 = 0; i0 < sn; i0 += 32 * U) {
      int kk[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + 32 * u + lane;
        kk[u] = i < sn ? class_of(source(seg + i)) : 0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + 32 * u + lane;
        if (i < sn) cls[i] = (unsigned char)kk[u];
      }
    }
    __syncwarp();
    for (int base = 0; base < sn; base += 32) {
      const int i = base + lane;
      const bool valid = i < sn;
      const int k = valid ? (int)cls[i] : 0;
      // lanes of the same class: five ballots over the class bits
      unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        const unsigned m = __ballot_sync(0xffffffffu, (k >> b) & 1);
        peers &= ((k >> b) & 1) ? m : ~m;
      }
      const int lev = valid ? cnt[k] + __popc(peers & ((1u << lane) - 1u)) : 0;
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) cnt[k] += __popc(peers);
      __syncwarp();
      if (valid) key_at[seg + i] = packed ? (lev << 5 | k) : lev;
    }
    __syncwarp();
  }
  int nmax = cnt[lane];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
  const bool table = nmax <= TM_LEVELS;
  auto level_row = [&](int l, int& P, unsigned& M) {
    P = 0; M = 0;
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const int c = cnt[k];
      P += min(c, l);
      M |= (c > l ? 1u : 0u) << k;
    }
  };
  if (table) {
    for (int l = lane; l < nmax; l += 32) level_row(l, s_P[wid][l], s_M[wid][l]);
    __syncwarp();
  }
  for (int s0 = b0; s0 < b1; s0 += 32 * U) {
    int kv[U], pp[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int sl = s0 + 32 * u + lane;
      kv[u] = sl < b1 ? key_at[sl] : 0;
      pp[u] = sl < b1 ? source(sl) : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int sl = s0 + 32 * u + lane;
      if (sl >= b1) continue;
      const int lev = packed ? kv[u] >> 5 : kv[u], k = packed ? kv[u] & 31 : class_of(pp[u]);
      int P;
      unsigned M;
      if (table) { P = s_P[wid][lev]; M = s_M[wid][lev]; }
      else level_row(lev, P, M);
      src_at[b0 + P + __popc(M & ((1u << k) - 1u))] = (uint32_t)pp[u];
    }
  }
}

// Exchange every job's particle arrays with their *_b buffers (after a
// gather into the *_b buffers, instead of copying back).
__global__ void k_swap_particle_buffers(pxrb_tiled_job* jp, int njobs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  Job& J = jp[j];
  { uint32_t* t = J.cell; J.cell = J.cell_b; J.cell_b = t; }
  { void* t = J.ox; J.ox = J.ox_b; J.ox_b = t; }
  { void* t = J.oy; J.oy = J.oy_b; J.oy_b = t; }
  { void* t = J.oz; J.oz = J.oz_b; J.oz_b = t; }
  { void* t = J.ux; J.ux = J.ux_b; J.ux_b = t; }
  { void* t = J.uy; J.uy = J.uy_b; J.uy_b = t; }
  { void* t = J.uz; J.uz = J.uz_b; J.uz_b = t; }
  { void* t = J.w; J.w = J.w_b; J.w_b = t; }
  if (J.pid) { int32_t* t = J.pid; J.pid = J.pid_b; J.pid_b = t; }
}

// Gather in destination order into the *_b buffers (all particles of a job):
// the source of destination d is read from cell_b[d] before the cell
// replaces it.
template <typename R>
__global__ void k_relayout_gather(const Job* __restrict__ jp) {
  const Job J = jp[blockIdx.y];
  const i64 np = J.np;
  const uint32_t* __restrict__ cell = J.cell;
  const R* __restrict__ ox = (const R*)J.ox;
  const R* __restrict__ oy = (const R*)J.oy;
  const R* __restrict__ oz = (const R*)J.oz;
  const R* __restrict__ ux = (const R*)J.ux;
  const R* __restrict__ uy = (const R*)J.uy;
  const R* __restrict__ uz = (const R*)J.uz;
  const R* __restrict__ w = (const R*)J.w;
  const int* __restrict__ pid = J.pid;
  uint32_t* cb = J.cell_b;             // source per destination, then its cell
  R* __restrict__ oxb = (R*)J.ox_b;
  R* __restrict__ oyb = (R*)J.oy_b;
  R* __restrict__ ozb = (R*)J.oz_b;
  R* __restrict__ uxb = (R*)J.ux_b;
  R* __restrict__ uyb = (R*)J.uy_b;
  R* __restrict__ uzb = (R*)J.uz_b;
  R* __restrict__ wb = (R*)J.w_b;
  int* __restrict__ pidb = J.pid_b;
  for (i64 d = blockIdx.x * (i64)blockDim.x + threadIdx.x; d < np;
       d += (i64)gridDim.x * blockDim.x) {
    const int p = (int)cb[d];
    cb[d] = __ldg(cell + p);
    oxb[d] = __ldg(ox + p); oyb[d] = __ldg(oy + p); ozb[d] = __ldg(oz + p);
    uxb[d] = __ldg(ux + p); uyb[d] = __ldg(uy + p); uzb[d] = __ldg(uz + p);
    wb[d] = __ldg(w + p);
    if (pid) pidb[d] = __ldg(pid + p);
  }
}

// ---------------------------------------------------------------------------
// Conversions
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_load_particles(Job J, const double* x, const double* y, const double* z,
                                 const double* ux, const double* uy, const double* uz,
                                 const double* w) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    double pos[3] = {(x[p] - J.xmin) / J.dx, (y[p] - J.ymin) / J.dy, (z[p] - J.zmin) / J.dz};
    int n[3] = {J.nx, J.ny, J.nz};
    int c[3];
    R o[3];
    for (int a = 0; a < 3; ++a) {
      double f = floor(pos[a]);
      int ci = (int)f;
      R oo = (R)(pos[a] - f);
      if (oo >= (R)1) { oo = (R)0; ci += 1; }
      ci %= n[a];
      if (ci < 0) ci += n[a];
      c[a] = ci; o[a] = oo;
    }
    J.cell[p] = pack_cell(c[0], c[1], c[2]);
    ((R*)J.ox)[p] = o[0]; ((R*)J.oy)[p] = o[1]; ((R*)J.oz)[p] = o[2];
    ((R*)J.ux)[p] = (R)ux[p]; ((R*)J.uy)[p] = (R)uy[p]; ((R*)J.uz)[p] = (R)uz[p];
    ((R*)J.w)[p] = (R)w[p];
  }
}

template <typename R>
__global__ void k_store_particles(Job J, double* x, double* y, double* z, double* ux,
                                  double* uy, double* uz, double* gaminv, double* w) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    int i, j, k;
    unpack_cell(J.cell[p], i, j, k);
    if (x) x[p] = J.xmin + ((double)i + (double)((const R*)J.ox)[p]) * J.dx;
    if (y) y[p] = J.ymin + ((double)j + (double)((const R*)J.oy)[p]) * J.dy;
    if (z) z[p] = J.zmin + ((double)k + (double)((const R*)J.oz)[p]) * J.dz;
    double a = ((const R*)J.ux)[p], b = ((const R*)J.uy)[p], c = ((const R*)J.uz)[p];
    if (ux) ux[p] = a;
    if (uy) uy[p] = b;
    if (uz) uz[p] = c;
    if (gaminv) gaminv[p] = 1.0 / sqrt(1.0 + (a * a + b * b + c * c) / (J.clight * J.clight));
    if (w) w[p] = ((const R*)J.w)[p];
  }
}

// Engine -> PICSAR arrays in id order: particle p goes to row pid[p].  The
// descriptor is read from device memory (one copy per block in shared memory).
template <typename R>
__global__ void k_store_particles_by_id(const Job* __restrict__ jd, i64 np, double* x,
                                        double* y, double* z, double* ux, double* uy,
                                        double* uz, double* gaminv, double* w) {
  __shared__ Job J;
  if (threadIdx.x == 0) J = *jd;
  __syncthreads();
  if (!J.pid) return;
  const i64 n = J.np < np ? J.np : np;
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < n;
       p += (i64)gridDim.x * blockDim.x) {
    const i64 d = J.pid[p];
    if (d < 0 || d >= np) continue;
    int i, j, k;
    unpack_cell(J.cell[p], i, j, k);
    if (x) x[d] = J.xmin + ((double)i + (double)((const R*)J.ox)[p]) * J.dx;
    if (y) y[d] = J.ymin + ((double)j + (double)((const R*)J.oy)[p]) * J.dy;
    if (z) z[d] = J.zmin + ((double)k + (double)((const R*)J.oz)[p]) * J.dz;
    const double a = ((const R*)J.ux)[p], b = ((const R*)J.uy)[p], c = ((const R*)J.uz)[p];
    if (ux) ux[d] = a;
    if (uy) uy[d] = b;
    if (uz) uz[d] = c;
    if (gaminv) gaminv[d] = 1.0 / sqrt(1.0 + (a * a + b * b + c * c) / (J.clight * J.clight));
    if (w) w[d] = ((const R*)J.w)[p];
  }
}

// Fortran guarded FP64 grid (ng guards) <-> engine.  dir 0: import, 1: export.
template <typename R>
__global__ void k_field_xfer(Job J, int which, double* f, int ng, int dir) {
  const int nx = J.nx, ny = J.ny, nz = J.nz, G = J.g;
  if (which < 6) {
    R* e = (R*)((&J.ex)[which]);
    const int ex_ = nx + 2 * G, ey_ = ny + 2 * G, ez_ = nz + 2 * G, py = J.pitch_y;
    const i64 total = (i64)ex_ * ey_ * ez_;
    const int sx = nx + 1 + 2 * ng, sy = ny + 1 + 2 * ng;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
      int a = (int)(t % ex_), b = (int)((t / ex_) % ey_), c = (int)(t / ((i64)ex_ * ey_));
      int i = a - G, j = b - G, k = c - G;
      int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
      i64 e_idx = a + (i64)J.pitch_x * (b + (i64)py * c);
      if (dir == 0) {
        e[e_idx] = (R)f[(pi + ng) + (i64)sx * ((pj + ng) + (i64)sy * (pk + ng))];
      } else if (i >= -ng && i <= nx + ng && j >= -ng && j <= ny + ng && k >= -ng &&
                 k <= nz + ng) {
        f[(i + ng) + (i64)sx * ((j + ng) + (i64)sy * (k + ng))] = (double)e[e_idx];
      }
    }
    if (dir == 1) {
      // nodes beyond the engine guards (ng > G) get periodic images
      const i64 tot2 = (i64)(nx + 1 + 2 * ng) * (ny + 1 + 2 * ng) * (nz + 1 + 2 * ng);
      for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < tot2;
           t += (i64)gridDim.x * blockDim.x) {
        int a = (int)(t % sx), b = (int)((t / sx) % sy), c = (int)(t / ((i64)sx * sy));
        int i = a - ng, j = b - ng, k = c - ng;
        if (i >= -G && i < nx + G && j >= -G && j < ny + G && k >= -G && k < nz + G) continue;
        int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
        f[t] = (double)e[(pi + G) + (i64)J.pitch_x * ((pj + G) + (i64)py * (pk + G))];
      }
    }
  } else {
    double* jj = (&J.jx)[which - 6];
    const int sx = nx + 1 + 2 * ng, sy = ny + 1 + 2 * ng;
    const i64 total = dir == 0 ? (i64)nx * ny * nz : (i64)sx * sy * (nz + 1 + 2 * ng);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
      if (dir == 0) {
        int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((i64)nx * ny));
        jj[t] = f[(i + ng) + (i64)sx * ((j + ng) + (i64)sy * (k + ng))];
      } else {
        int a = (int)(t % sx), b = (int)((t / sx) % sy), c = (int)(t / ((i64)sx * sy));
        int i = a - ng, j = b - ng, k = c - ng;
        int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
        f[t] = jj[pi + (i64)nx * (pj + (i64)ny * pk)];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Diagnostics
// ---------------------------------------------------------------------------
template <typename R, int ORDER>
__global__ void k_rho_t(Job J, double* rho) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    int ci, cj, ck;
    unpack_cell(J.cell[p], ci, cj, ck);
    NodeCO<ORDER, double> sx, sy, sz;
    sx.set((double)((const R*)J.ox)[p]);
    sy.set((double)((const R*)J.oy)[p]);
    sz.set((double)((const R*)J.oz)[p]);
    const double wq = J.q * (double)((const R*)J.w)[p] / (J.dx * J.dy * J.dz);
#pragma unroll
    for (int c = 0; c < ORDER + 1; ++c)
#pragma unroll
      for (int b = 0; b < ORDER + 1; ++b)
#pragma unroll
        for (int a = 0; a < ORDER + 1; ++a) {
          int i = GlobAcc::wrap(ci + sx.r0 + a, J.nx), j = GlobAcc::wrap(cj + sy.r0 + b, J.ny),
              k = GlobAcc::wrap(ck + sz.r0 + c, J.nz);
          atomicAdd(rho + i + (i64)J.nx * (j + (i64)J.ny * k), sx.s[a] * sy.s[b] * sz.s[c] * wq);
        }
  }
}

constexpr int RED_TPB = 256;

// per-block partial sums: [0..5] 0.5 F^2 of the six fields, [6] (divE eps0 - rho)^2,
// [7] rho^2; part[q * nblocks + block]
template <typename R>
__global__ void __launch_bounds__(RED_TPB) k_field_sums(Job J, const double* rho, double* part) {
  const int nx = J.nx, ny = J.ny, nz = J.nz, G = J.g, pitch = J.pitch_x, NYg = J.pitch_y;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  const i64 total = (i64)nx * ny * nz;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const R* F[6] = {(const R*)J.ex, (const R*)J.ey, (const R*)J.ez,
                   (const R*)J.bx, (const R*)J.by, (const R*)J.bz};
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
       t += (i64)gridDim.x * blockDim.x) {
    int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((i64)nx * ny));
    i64 c = (i + G) + sy * (j + G) + sz * (k + G);
    for (int q = 0; q < 6; ++q) {
      double v = (double)F[q][c];
      acc[q] += v * v * 0.5;
    }
    if (rho) {
      double dive = ((double)F[0][c] - (double)F[0][c - 1]) / J.dx +
                    ((double)F[1][c] - (double)F[1][c - sy]) / J.dy +
                    ((double)F[2][c] - (double)F[2][c - sz]) / J.dz;
      double r = rho[t];
      double d = dive * J.eps0 - r;
      acc[6] += d * d;
      acc[7] += r * r;
    }
  }
  {
    // kinetic energy: this block's fixed slice of the per-tile sums
    const int ntiles = J.ntx * J.nty * J.ntz;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < ntiles; b += gridDim.x * blockDim.x)
      acc[8] += J.ke_tile[b];
  }
  __shared__ double red[9][RED_TPB / 32];
  for (int q = 0; q < 9; ++q) {
    double v = acc[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0;
    for (int w = 0; w < RED_TPB / 32; ++w) s += red[threadIdx.x][w];
    part[threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

// Nine warps, one per quantity, each summing that quantity's block partials
// in a fixed order (deterministic results).
__global__ void __launch_bounds__(288) k_diag_final(Job J, const double* part, int nblocks,
                                                    double* out) {
  __shared__ double s[9];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double t = 0;
  for (int b = lane; b < nblocks; b += 32) t += part[q * nblocks + b];
  for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  if (lane == 0) s[q] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dv = J.dx * J.dy * J.dz;
    out[0] = s[8];
    for (int c = 0; c < 3; ++c) out[1 + c] = s[c] * dv * J.eps0;
    for (int c = 3; c < 6; ++c) out[1 + c] = s[c] * dv / J.mu0;
    out[7] = sqrt(s[6]);
    out[8] = sqrt(s[7]);
  }
}

// blocks of the diagnostics reduction: at most DIAG_MAX_BLOCKS (8 per SM of
// a B200), each writing 9 partial sums
constexpr int DIAG_MAX_BLOCKS = 1184;
int diag_blocks(const Job& J) {
  i64 total = (i64)J.nx * J.ny * J.nz;
  i64 b = (total + RED_TPB - 1) / RED_TPB;
  return (int)(b > DIAG_MAX_BLOCKS ? DIAG_MAX_BLOCKS : (b < 1 ? 1 : b));
}

template <int ORDER>
constexpr int reach_total() { return Reach<ORDER>::L + Reach<ORDER>::H; }

int64_t smem_bytes(int order, int prec, int acc, int tx, int ty, int tz, int drift) {
  (void)ty; (void)tz;                 // cubic tiles
  const int lh = order == 1 ? 1 : 3, W = tx + 2 * drift + lh;
  const i64 V = (i64)pxrt::win_sz(tx, W) * W;
  i64 r = prec ? 8 : 4;
  i64 a = acc == 3 ? 8 : 4, nw = acc == 2 ? 2 : 1;
  const i64 hb = tx + 2 * drift;      // next-step occupancy histogram (fixed point)
  if (acc == 4)                       // cell-grouped kernel (cg_smem_bytes)
    return V * 36 + hb * hb * hb * 12 + 4 + ((hb * hb * hb * 2 + 15) / 16) * 16 + 256 * 8;
  return V * (6 * r + 3 * a * nw) + ((acc == 1 || acc == 2) ? hb * hb * hb * 4 : 0);
}

inline int gs_blocks(i64 n, int tpb) {
  i64 b = (n + tpb - 1) / tpb;
  const i64 cap = 148 * 32;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

extern "C" {

int64_t pxrb_tiled_job_size(void) { return (int64_t)sizeof(pxrb_tiled_job); }

int64_t pxrb_tiled_smem_bytes(int32_t order, int32_t prec, int32_t acc, int32_t tx, int32_t ty,
                              int32_t tz, int32_t drift) {
  return smem_bytes(order, prec, acc, tx, ty, tz, drift);
}

int pxrb_tiled_particle_step(const pxrb_tiled_job* jobs_dev, int32_t order, int32_t prec,
                             int32_t tile, int32_t drift, int32_t acc, const int32_t* work,
                             int32_t nwork,
                             const int32_t* nwork_dev, int32_t* ctr, int32_t threads,
                             int32_t ctas, int64_t smem, void* stream) {
  if (!jobs_dev || !work || !ctr || nwork < 0 || smem < 0) return PXRB_EINVAL;
  if (nwork == 0) return PXRB_OK;
  if (threads < 32 || threads % 32 ||
      threads > (prec == 1 && acc != 4 ? MAX_THREADS_FP64 : MAX_THREADS))
    return PXRB_EINVAL;
  if (order < 1 || order > 3 || prec < 0 || prec > 1) return PXRB_EUNSUPPORTED;
  if (ctas < 1) ctas = 1;
  cudaStream_t s = (cudaStream_t)stream;
  const int2* w2 = reinterpret_cast<const int2*>(work);
  if (order == 1)
    return pxrt::launch_order1(prec, tile, drift, acc, jobs_dev, w2, nwork, nwork_dev, ctr,
                               threads, ctas, (size_t)smem, s);
  if (order == 2)
    return pxrt::launch_order2(prec, tile, drift, acc, jobs_dev, w2, nwork, nwork_dev, ctr,
                               threads, ctas, (size_t)smem, s);
  return pxrt::launch_order3(prec, tile, drift, acc, jobs_dev, w2, nwork, nwork_dev, ctr,
                             threads, ctas, (size_t)smem, s);
}

int pxrb_tiled_push_b(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, double frac,
                      void* stream) {
  if (!jobs_dev || !cell_off_dev || njobs < 1 || total_cells < 0 || total_cells % YEE_CPB)
    return PXRB_EINVAL;
  if (total_cells == 0) return PXRB_OK;
  int nb = (int)(total_cells / YEE_CPB);
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == 0) k_yee_b_t<float><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, (float)frac);
  else k_yee_b_t<double><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, frac);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_push_e(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, int32_t zero_j,
                      void* stream) {
  if (!jobs_dev || !cell_off_dev || njobs < 1 || total_cells < 0 || total_cells % YEE_CPB)
    return PXRB_EINVAL;
  if (total_cells == 0) return PXRB_OK;
  int nb = (int)(total_cells / YEE_CPB);
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == 0) k_yee_e_t<float><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, zero_j);
  else k_yee_e_t<double><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, zero_j);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_sort(const pxrb_tiled_job* job_host, pxrb_tiled_job* job_dev, void* stream) {
  if (!job_host || !job_dev) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np < 0 || !J.tile_cnt || !J.tile_off) return PXRB_EINVAL;
  const int ntiles = J.ntx * J.nty * J.ntz;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(J.tile_cnt, 0, sizeof(int32_t) * (ntiles + 1), s) != cudaSuccess)
    return PXRB_ELAUNCH;
  if (J.tx != J.ty || J.ty != J.tz || J.tx * J.tx * J.tx > RR_MAXC || !J.cell_cnt || (J.np > 0 && !J.rank_b))
    return PXRB_EINVAL;
  if (cudaMemsetAsync(J.cell_cnt, 0, sizeof(int32_t) * (size_t)ntiles * J.tx * J.tx * J.tx, s) !=
      cudaSuccess)
    return PXRB_ELAUNCH;
  if (J.tile_stats && cudaMemsetAsync(J.tile_stats, 0, sizeof(float) * 4 * (size_t)ntiles, s) !=
                          cudaSuccess)
    return PXRB_ELAUNCH;
  if (J.tx != 4 && J.tx != 8) return PXRB_EUNSUPPORTED;
  const int nb = gs_blocks(J.np, 256);
  if (J.np > 0) {
    k_sort_count<<<nb, 256, 0, s>>>(job_dev);
    k_sort_cellscan<<<(ntiles + CS_TPB / 32 - 1) / (CS_TPB / 32), CS_TPB, 0, s>>>(job_dev);
  }
  k_sort_scan<<<1, SCAN_TPB, 0, s>>>(job_dev);
  if (J.np > 0) {
    if (!J.perm) return PXRB_EINVAL;
    k_sort_perm<<<nb, 256, 0, s>>>(job_dev);
    if (J.prec == 0) {
      k_tile_map<float, true><<<(ntiles + TM_WARPS - 1) / TM_WARPS, TM_WARPS * 32, 0, s>>>(job_dev);
      k_relayout_gather<float><<<nb, 256, 0, s>>>(job_dev);
    } else {
      k_tile_map<double, true><<<(ntiles + TM_WARPS - 1) / TM_WARPS, TM_WARPS * 32, 0, s>>>(job_dev);
      k_relayout_gather<double><<<nb, 256, 0, s>>>(job_dev);
    }
    k_swap_particle_buffers<<<1, 32, 0, s>>>(job_dev, 1);
  }
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_sort_batch(pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                          int32_t max_tiles, int64_t max_np, void* stream) {
  if (!jobs_dev || njobs < 1 || njobs > 65535 || max_tiles < 1 || max_np < 0)
    return PXRB_EINVAL;
  if (prec < 0 || prec > 1) return PXRB_EUNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  // blocks per job: enough to cover the largest job, capped so that the whole
  // batch stays a few thousand CTAs (each CTA strides through its job)
  const int64_t want = (max_np + 255) / 256;
  const int cap = njobs >= 4096 ? 1 : 4096 / njobs;
  const int bx = (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
  const dim3 g_np(bx, njobs), g_one(1, njobs);
  const dim3 g_cs((max_tiles + CS_TPB / 32 - 1) / (CS_TPB / 32), njobs);
  k_sort_zero<<<g_np, 256, 0, s>>>(jobs_dev);
  k_sort_count<<<g_np, 256, 0, s>>>(jobs_dev);
  k_sort_cellscan<<<g_cs, CS_TPB, 0, s>>>(jobs_dev);
  k_sort_scan<<<g_one, SCAN_TPB, 0, s>>>(jobs_dev);
  k_sort_perm<<<g_np, 256, 0, s>>>(jobs_dev);
  if (prec == 0) {
    k_tile_map<float, true><<<dim3((max_tiles + TM_WARPS - 1) / TM_WARPS, njobs), TM_WARPS * 32, 0, s>>>(jobs_dev);
    k_relayout_gather<float><<<g_np, 256, 0, s>>>(jobs_dev);
  } else {
    k_tile_map<double, true><<<dim3((max_tiles + TM_WARPS - 1) / TM_WARPS, njobs), TM_WARPS * 32, 0, s>>>(jobs_dev);
    k_relayout_gather<double><<<g_np, 256, 0, s>>>(jobs_dev);
  }
  k_swap_particle_buffers<<<(njobs + 127) / 128, 128, 0, s>>>(jobs_dev, njobs);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_relayout(pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                        int32_t max_tiles, int64_t max_np, void* stream) {
  if (!jobs_dev || njobs < 1 || njobs > 65535 || max_tiles < 1 || max_np < 0)
    return PXRB_EINVAL;
  if (prec < 0 || prec > 1) return PXRB_EUNSUPPORTED;
  if (max_np == 0) return PXRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t want = (max_np + 255) / 256;
  const int cap = njobs >= 4096 ? 1 : 4096 / njobs;
  const int bx = (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
  const dim3 g_tiles((max_tiles + TM_WARPS - 1) / TM_WARPS, njobs), g_np(bx, njobs);
  if (prec == 0) {
    k_tile_map<float, false><<<g_tiles, TM_WARPS * 32, 0, s>>>(jobs_dev);
    k_relayout_gather<float><<<g_np, 256, 0, s>>>(jobs_dev);
  } else {
    k_tile_map<double, false><<<g_tiles, TM_WARPS * 32, 0, s>>>(jobs_dev);
    k_relayout_gather<double><<<g_np, 256, 0, s>>>(jobs_dev);
  }
  k_swap_particle_buffers<<<(njobs + 127) / 128, 128, 0, s>>>(jobs_dev, njobs);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_load_particles(const pxrb_tiled_job* job_host, const double* x, const double* y,
                              const double* z, const double* ux, const double* uy,
                              const double* uz, const double* w, void* stream) {
  if (!job_host) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np == 0) return PXRB_OK;
  if (!x || !y || !z || !ux || !uy || !uz || !w || !J.cell) return PXRB_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  if (J.prec == 0) k_load_particles<float><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, w);
  else k_load_particles<double><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, w);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_store_particles(const pxrb_tiled_job* job_host, double* x, double* y, double* z,
                               double* ux, double* uy, double* uz, double* gaminv, double* w,
                               void* stream) {
  if (!job_host) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np == 0) return PXRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (J.prec == 0)
    k_store_particles<float><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, gaminv, w);
  else
    k_store_particles<double><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, gaminv, w);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_store_particles_by_id(const pxrb_tiled_job* job_dev, int64_t np, int32_t prec,
                                     double* x, double* y, double* z, double* ux, double* uy,
                                     double* uz, double* gaminv, double* w, void* stream) {
  if (!job_dev || np < 0) return PXRB_EINVAL;
  if (prec < 0 || prec > 1) return PXRB_EUNSUPPORTED;
  if (np == 0) return PXRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == 0)
    k_store_particles_by_id<float><<<gs_blocks(np, 256), 256, 0, s>>>(job_dev, np, x, y, z, ux,
                                                                      uy, uz, gaminv, w);
  else
    k_store_particles_by_id<double><<<gs_blocks(np, 256), 256, 0, s>>>(job_dev, np, x, y, z, ux,
                                                                       uy, uz, gaminv, w);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static int field_xfer(const pxrb_tiled_job* job_host, int32_t which, double* f, int64_t ng,
                      int dir, void* stream) {
  if (!job_host || !f || which < 0 || which > 8 || ng < 0) return PXRB_EINVAL;
  const Job& J = *job_host;
  cudaStream_t s = (cudaStream_t)stream;
  i64 total = (i64)(J.nx + 1 + 2 * ng) * (J.ny + 1 + 2 * ng) * (J.nz + 1 + 2 * ng);
  i64 t2 = (i64)(J.nx + 2 * J.g) * (J.ny + 2 * J.g) * (J.nz + 2 * J.g);
  if (t2 > total) total = t2;
  if (J.prec == 0) k_field_xfer<float><<<gs_blocks(total, 256), 256, 0, s>>>(J, which, f, (int)ng, dir);
  else k_field_xfer<double><<<gs_blocks(total, 256), 256, 0, s>>>(J, which, f, (int)ng, dir);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_field_import(const pxrb_tiled_job* job_host, int32_t which, const double* src,
                            int64_t nguard_src, void* stream) {
  return field_xfer(job_host, which, const_cast<double*>(src), nguard_src, 0, stream);
}

int pxrb_tiled_field_export(const pxrb_tiled_job* job_host, int32_t which, double* dst,
                            int64_t nguard_dst, void* stream) {
  return field_xfer(job_host, which, dst, nguard_dst, 1, stream);
}

int64_t pxrb_tiled_diag_scratch(const pxrb_tiled_job* job_host) {
  if (!job_host) return -1;
  return 9 * (int64_t)diag_blocks(*job_host);
}

int pxrb_tiled_diagnostics(const pxrb_tiled_job* job_host, double* rho, double* scratch,
                           int64_t scratch_len, double* out, void* stream) {
  if (!job_host || !scratch || !out) return PXRB_EINVAL;
  const Job& J = *job_host;
  const int nb = diag_blocks(J);
  if (scratch_len < 9 * (int64_t)nb) return PXRB_ESCRATCH;
  cudaStream_t s = (cudaStream_t)stream;
  if (rho && cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)J.nx * J.ny * J.nz, s) != cudaSuccess)
    return PXRB_ELAUNCH;
  if (rho && J.np > 0) {
    const int pb = gs_blocks(J.np, 256);
#define PXRB_RHO(R_)                                                   \
    if (J.order == 1) k_rho_t<R_, 1><<<pb, 256, 0, s>>>(J, rho);       \
    else if (J.order == 2) k_rho_t<R_, 2><<<pb, 256, 0, s>>>(J, rho);  \
    else k_rho_t<R_, 3><<<pb, 256, 0, s>>>(J, rho);
    if (J.prec == 0) { PXRB_RHO(float) } else { PXRB_RHO(double) }
#undef PXRB_RHO
  }
  if (J.prec == 0) k_field_sums<float><<<nb, RED_TPB, 0, s>>>(J, rho, scratch);
  else k_field_sums<double><<<nb, RED_TPB, 0, s>>>(J, rho, scratch);
  k_diag_final<<<1, 288, 0, s>>>(J, scratch, nb, out);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Diagnostics without any allocation by the caller.
//
// Some callers cannot allocate device memory: a runtime that hands the library
// only a job descriptor (no allocator of its own), or code that runs inside a
// memory pool it must not grow.  This variant keeps its scratch -- the rho
// grid and the per-block partial sums -- in one file-scope device array, so
// the caller passes nothing but the job and the 9-double output.
//
// Limits and rules:
//  * the array holds PXRB_NOALLOC_RHO_MAX doubles of rho (with gauss != 0,
//    jobs of at most 1,048,576 cells, e.g. 96^3 or 128x128x64) plus the
//    partial sums of the reduction, whose block count is capped, so jobs of
//    any size fit with gauss = 0; a larger job with gauss != 0 is rejected
//    with PXRB_ETOOLARGE before any GPU work;
//  * every GPU that loads the library holds the array (~8.1 MiB) until exit;
//  * every call shares the array and it keeps the last call's contents, so
//    calls that overlap on the GPU (different streams, or a second call
//    enqueued before the first finished, from any thread) race;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (once per device); make that first call before any
//    stream capture;
//  * that address is cached per device index for the life of the process: it
//    does not survive cudaDeviceReset (or any other teardown of the device's
//    primary context), after which this entry point must not be called.
// ---------------------------------------------------------------------------
#define PXRB_NOALLOC_RHO_MAX (1 << 20)
#define PXRB_NOALLOC_PART_MAX (9 * DIAG_MAX_BLOCKS)
static __device__ __align__(256) double g_noalloc_scratch[PXRB_NOALLOC_RHO_MAX + PXRB_NOALLOC_PART_MAX];

static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[256];   // per device; host-side copy of the device address

extern "C" int pxrb_tiled_diagnostics_noalloc(const pxrb_tiled_job* job_host, int32_t gauss,
                                              double* out, void* stream) {
  if (!job_host || !out) return PXRB_EINVAL;
  const Job& J = *job_host;
  const i64 ncell = (i64)J.nx * J.ny * J.nz;
  static_assert(PXRB_NOALLOC_PART_MAX >= 9 * DIAG_MAX_BLOCKS,
                "the partial sums of the largest reduction must fit the static array");
  if (gauss && ncell > PXRB_NOALLOC_RHO_MAX) return PXRB_ETOOLARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return PXRB_ELAUNCH;
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PXRB_ELAUNCH;
      g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    base = g_noalloc_addr[dev];
  }
  double* rho = gauss ? base : nullptr;
  double* part = base + PXRB_NOALLOC_RHO_MAX;
  return pxrb_tiled_diagnostics(job_host, rho, part, PXRB_NOALLOC_PART_MAX, out, stream);
}
