// Device code of the tiled engine's cell-grouped particle kernel (FP32, int32
// fixed-point current, shape orders 1 and 3), included by pxr_tiled_o1.cu
// and pxr_tiled_o3.cu.
//
// At orders 1 and 3 every particle of a cell gathers from the same E/B nodes
// and, when it stays in its cell, deposits on the same J nodes.  The kernel
// therefore sorts each tile's particles by window cell in shared memory at
// the start of every step and hands each thread a group of CG_P particles of
// one cell (a packed f32x2 pair): every E/B value the thread loads from the
// window serves the group's gathers, and the group's Esirkepov contributions
// to a J node are summed in registers before one shared-memory atomic.  Per
// particle this takes 1/CG_P of the window loads and accumulator atomics of
// the one-particle-per-thread kernel (k_tile_step).
#pragma once
#include "pxr_tiled_kernel.cuh"

namespace pxrt {

__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
  f2_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
  f2_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_s(float v) { return f2_pack(v, v); }
__device__ __forceinline__ float f2_lo(f2_t v) { return __uint_as_float((unsigned)(v & 0xffffffffull)); }
__device__ __forceinline__ float f2_hi(f2_t v) { return __uint_as_float((unsigned)(v >> 32)); }

constexpr int CG_P = 2;                 // particles per group (1 or 2 pairs)
constexpr int CG_Q = CG_P / 2;          // packed pairs per group

// Node shape of orders 1 and 3 at in-cell offsets o (first node at c for
// order 1, c - 1 for order 3): NodeCO's formulas on a pair of particles.
// Esirkepov's shape of the same orders is the same function of the offset.
template <int ORDER>
__device__ __forceinline__ void node_pair(f2_t o, f2_t* s) {
  if (ORDER == 1) {
    s[0] = f2_sub(f2_s(1.f), o);
    s[1] = o;
  } else {
    const f2_t ox = f2_sub(f2_s(1.f), o), xs = f2_mul(o, o), oxs = f2_mul(ox, ox);
    s[0] = f2_mul(f2_mul(f2_s((float)(1.0 / 6.0)), oxs), ox);
    s[1] = f2_fma(xs, f2_fma(o, f2_s(0.5f), f2_s(-1.f)), f2_s((float)(2.0 / 3.0)));
    s[2] = f2_fma(oxs, f2_fma(ox, f2_s(0.5f), f2_s(-1.f)), f2_s((float)(2.0 / 3.0)));
    s[3] = f2_mul(f2_mul(f2_s((float)(1.0 / 6.0)), xs), o);
  }
}
// Staggered (one order lower) shape of StagCO on a pair; first node at c for
// order 1, c - 1 for order 3.
template <int ORDER>
__device__ __forceinline__ void stag_pair(f2_t o, f2_t* s) {
  if (ORDER == 1) {
    s[0] = f2_s(1.f);
  } else {
    const f2_t xi = f2_sub(o, f2_s(0.5f));
    const f2_t a = f2_sub(f2_s(0.5f), xi), b = f2_add(f2_s(0.5f), xi);
    s[0] = f2_mul(f2_mul(f2_s(0.5f), a), a);
    s[1] = f2_sub(f2_s(0.75f), f2_mul(xi, xi));
    s[2] = f2_mul(f2_mul(f2_s(0.5f), b), b);
  }
}

// One field component at the group's CG_P particles: window points
// base[t + b*SY + c*SZ], weights sa[q][t] * sb[q][b] * sc[q][c] of pair q.
// Each loaded value is splatted once and serves the group's pairs; per
// particle the sums run as gwin's (x, then y, then z).
template <int NA, int NB, int NC, int SY, int SZ>
__device__ __forceinline__ void cg_comp(const float* base, const f2_t (*sa)[4],
                                        const f2_t (*sb)[4], const f2_t (*sc)[4],
                                        f2_t* out) {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    f2_t a[CG_Q];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      f2_t F[NA];
#pragma unroll
      for (int t = 0; t < NA; ++t) F[t] = f2_s(base[t + b * SY + c * SZ]);
#pragma unroll
      for (int q = 0; q < CG_Q; ++q) {
        f2_t r = f2_mul(sa[q][0], F[0]);
#pragma unroll
        for (int t = 1; t < NA; ++t) r = f2_fma(sa[q][t], F[t], r);
        a[q] = b == 0 ? f2_mul(r, sb[q][0]) : f2_fma(r, sb[q][b], a[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < CG_Q; ++q)
      out[q] = c == 0 ? f2_mul(a[q], sc[q][0]) : f2_fma(a[q], sc[q][c], out[q]);
  }
}

// Fixed-point sum of a pair's contributions C*f to one J node: each term is
// rounded to the nearest integer by one FMA onto 1.5 * 2^23 (the FMA rounds
// the exact product once; |C f| <= 2^22 by the tile's scale), and the two
// integers are added exactly, so node sums do not depend on how the
// particles are grouped.
__device__ __forceinline__ int cg_fix(f2_t C, f2_t f) {
  const f2_t t = f2_fma(C, f, f2_s(12582912.0f));
  // the bit patterns are 0x4B400000 + round(C f); summed modulo 2^32
  return (int)((unsigned)(t & 0xffffffffull) + (unsigned)(t >> 32) - 2u * 0x4B400000u);
}

// Esirkepov deposit of a pair of particles that stay in their cell: boxes of
// ORDER+1 nodes per axis at base (the form of dep_window_same); t0 / t1 =
// shapes at the new / old offsets per axis, cq = charge factors (q w /
// (dt dA) times the window's fixed-point scale; zero for a particle that
// does not take part).  One shared atomic per node for the pair.
template <int ORDER, int SY, int SZ, int V>
__device__ __forceinline__ void cg_deposit(int* base, const f2_t (*t0)[4], const f2_t (*t1)[4],
                                           const f2_t* cq) {
  constexpr int N = ORDER + 1;
  const f2_t half = f2_s(0.5f), third = f2_s((float)(1.0 / 3.0));
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    // axes: a = prefix-sum (current) axis, b = weighted-sum axis, c = the third
    const int ax = comp, bx = (comp + 1) % 3, cx = (comp + 2) % 3;
    f2_t C[N - 1], A[N], B[N];
    f2_t run = f2_s(0.f);
#pragma unroll
    for (int i = 0; i < N - 1; ++i) {
      run = i == 0 ? f2_sub(t1[ax][0], t0[ax][0]) : f2_add(run, f2_sub(t1[ax][i], t0[ax][i]));
      C[i] = f2_mul(run, cq[comp]);
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const f2_t s0 = t0[bx][j], ds = f2_sub(t1[bx][j], s0);
      A[j] = f2_fma(half, ds, s0);
      B[j] = f2_fma(third, ds, f2_mul(half, s0));
    }
    // node (a, b, c) of this component at base + comp*V + its offsets along
    // the grid axes; the loops run over (c, b) then a
#pragma unroll
    for (int kc = 0; kc < N; ++kc) {
      const f2_t s0c = t0[cx][kc], dsc = f2_sub(t1[cx][kc], s0c);
#pragma unroll
      for (int kb = 0; kb < N; ++kb) {
        const f2_t f = f2_fma(A[kb], s0c, f2_mul(B[kb], dsc));
#pragma unroll
        for (int ka = 0; ka < N - 1; ++ka) {
          const int v = cg_fix(C[ka], f);
          const int ox = comp == 0 ? ka : (comp == 1 ? kc : kb);
          const int oy = comp == 0 ? kb : (comp == 1 ? ka : kc);
          const int oz = comp == 0 ? kc : (comp == 1 ? kb : ka);
          atomicAdd(base + comp * V + ox + oy * SY + oz * SZ, v);
        }
      }
    }
  }
}

// CTA size: 256 threads, two CTAs per SM (128 registers per thread).  Groups
// of two particles fit that; groups of four need 168 registers, so 12 warps
// per SM, and measured 17.8 against 15.0 ms per step at 256^3.
constexpr int CG_THREADS = 256;
constexpr int CG_MINB = 2;

// Entries of the per-tile level table of the group order (levels beyond it
// are placed by a loop over the 32 classes).
constexpr int CG_LT = 256;

// Particles per thread whose window cell and rank stay in registers between
// the count and the placement of a tile (20 x 256 threads: 5120 particles,
// a 8^3 tile at 10 per cell); beyond that they go through global scratch.
constexpr int CG_KR = 20;

// Dynamic shared memory of the cell-grouped kernel: E/B window, int32 J
// window, the next step's cell occupancy, per-cell counts and group
// prefixes, the window cells ordered by bank class, and the level table.
__host__ __device__ constexpr int cg_smem_bytes(int T, int D, int V) {
  return V * (6 * 4 + 3 * 4) + (T + 2 * D) * (T + 2 * D) * (T + 2 * D) * 4 * 3 + 4 +
         (((T + 2 * D) * (T + 2 * D) * (T + 2 * D) * 2 + 15) / 16) * 16 + CG_LT * 8;
}

// ---------------------------------------------------------------------------
// The cell-grouped particle kernel.  Persistent CTAs pull (job, tile) work
// items as k_tile_step does; per tile:
//   1. the E/B window is staged with cp.async while the tile's particles are
//      counted per window cell (one shared atomic each; particles outside
//      the window go to one more bucket), and the counts are scanned;
//   2. each window cell of n particles makes ceil(n/CG_P) groups; a group's
//      bank class is its cell's (the bank of the cell's window address, where
//      its gather loads and deposit atomics start); the groups are numbered
//      within their class (level) and laid out by (level, class), so 32
//      consecutive groups - a warp's - sit in distinct banks until classes
//      run out (the sort's particle layout, applied to groups);
//   3. each thread takes a group: gather, push, position, and the summed
//      deposit of the particles that stay in the cell; particles that change
//      cell join k_tile_step's node-change queue (window) or deposit on the
//      global grid; particles outside the window take the global path.
// Scratch, all in the tile's range of the sort buffers that are free between
// sorts: w_b (window cell and rank per particle); perm, ux_b, uy_b, uz_b (the
// CG_P particle slots of each group, in group order, so a warp reads its
// groups' slots with coalesced loads: tile-relative particle index | window
// cell << 21, -1 for an empty slot; particles outside the window follow the
// groups in perm); rank_b / cell_b / ox_b / oy_b / oz_b (the node-change
// queue, as in k_tile_step).  A tile holds fewer than 2^21 particles.
// ---------------------------------------------------------------------------
template <int ORDER, int T, int D>
__global__ void __launch_bounds__(CG_THREADS, CG_MINB)
    k_cell_step(const Job* __restrict__ jobs, const int2* __restrict__ work, int nwork,
                const int* __restrict__ nwork_dev, int* ctr) {
  typedef float R;
  constexpr int MODE = 1;
  typedef int A;
  constexpr int L = Reach<ORDER>::L, H = Reach<ORDER>::H;
  constexpr int W = T + 2 * D + L + H, SY = win_sy(T, W), SZ = win_sz(T, W), V = SZ * W;
  constexpr int HB = T + 2 * D, NH = HB * HB * HB;
  constexpr int N = ORDER + 1, S = ORDER;
  static_assert(ORDER == 1 || ORDER == 3, "stencils fixed per cell at orders 1 and 3 only");
  static_assert(NH < 2048, "window cell keys take 11 bits");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* Fs = reinterpret_cast<R*>(smem_raw);
  A* Js = reinterpret_cast<A*>(smem_raw + (size_t)6 * V * sizeof(R));
  int* nh = Js + 3 * V;                 // next step's occupancy of the window cells
  int* s_cnt = nh + NH;                 // particles per window cell; [NH]: outside
  int* s_pre = s_cnt + NH + 1;          // groups of the cell's class before its own
  unsigned short* s_tau = reinterpret_cast<unsigned short*>(s_pre + NH);  // by class
  int* s_lvP = reinterpret_cast<int*>(smem_raw + cg_smem_bytes(T, D, V) - CG_LT * 8);
  unsigned* s_lvM = reinterpret_cast<unsigned*>(s_lvP + CG_LT);
  __shared__ int s_have;
  __shared__ Job sj;
  __shared__ int s_item;
  __shared__ int s_qn;
  __shared__ float s_max[5][CG_THREADS / 32];
  __shared__ double s_red[CG_THREADS / 32];
  __shared__ int s_ncls[32];            // window cells per class
  __shared__ int s_coff[33];            // their start in s_tau
  __shared__ int s_G[32];               // groups per class
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  auto cls = [](int h) {
    const int hx = h % HB, hy = (h / HB) % HB, hz = h / (HB * HB);
    return (hx + hy * SY + hz * SZ) & 31;
  };

  if (nwork_dev) nwork = min(nwork, *nwork_dev);
  for (int r = threadIdx.x; r < 6 * V; r += blockDim.x) {
    const int q = r % V, c = q / SZ, b = (q - c * SZ) / SY, a = q - c * SZ - b * SY;
    if (a >= W || b >= W) Fs[r] = (R)0;
  }
  // the window cells ordered by (class, cell), once per CTA
  if (threadIdx.x < 32) s_ncls[threadIdx.x] = 0;
  __syncthreads();
  for (int h = threadIdx.x; h < NH; h += blockDim.x) atomicAdd(&s_ncls[cls(h)], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int c = 0; c < 32; ++c) { s_coff[c] = t; t += s_ncls[c]; }
    s_coff[32] = t;
  }
  __syncthreads();
  for (int q = wid; q < 32; q += nwarps) {
    int lev = s_coff[q];
    for (int h0 = 0; h0 < NH; h0 += 32) {
      const int h = h0 + lane;
      const bool m = h < NH && cls(h) == q;
      const unsigned b = __ballot_sync(0xffffffffu, m);
      if (m) s_tau[lev + __popc(b & ((1u << lane) - 1u))] = (unsigned short)h;
      lev += __popc(b);
    }
  }

  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(ctr, 1);
      s_qn = 0;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= nwork) break;
    const int2 wk = work[item];
    {
      const int nw = (int)(sizeof(Job) / sizeof(int));
      const int* src = reinterpret_cast<const int*>(jobs + wk.x);
      int* dst = reinterpret_cast<int*>(&sj);
      for (int t = threadIdx.x; t < nw; t += blockDim.x) dst[t] = src[t];
    }
    __syncthreads();
    const int nx = sj.nx, ny = sj.ny, nz = sj.nz, G = sj.g;
    const int tile = wk.y;
    const int ti = tile % sj.ntx, tj = (tile / sj.ntx) % sj.nty, tk = tile / (sj.ntx * sj.nty);
    const int c0x = ti * T, c0y = tj * T, c0z = tk * T;
    const int tex = min(T, nx - c0x), tey = min(T, ny - c0y), tez = min(T, nz - c0z);
    const int wox = c0x - D - L, woy = c0y - D - L, woz = c0z - D - L;
    const int pbeg = sj.tile_off[tile], pend = sj.tile_off[tile + 1];
    const int pitch = sj.pitch_x, NYg = sj.pitch_y;
    {
      const i64 base0 = (i64)(wox + G) + (i64)pitch * ((woy + G) + (i64)NYg * (woz + G));
#pragma unroll 1
      for (int comp = 0; comp < 6; ++comp) {
        const R* src = (const R*)(comp == 0 ? sj.ex : comp == 1 ? sj.ey : comp == 2 ? sj.ez
                                 : comp == 3 ? sj.bx : comp == 4 ? sj.by : sj.bz) + base0;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Fs + comp * V);
        for (int r = threadIdx.x; r < W * W * W; r += blockDim.x) {
          const int a = r % W, b = (r / W) % W, c = r / (W * W);
          const R* g = src + a + (i64)pitch * (b + (i64)NYg * c);
          const uint32_t d = dst + (uint32_t)((a + b * SY + c * SZ) * sizeof(R));
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(g),
                       "n"((int)sizeof(R)));
        }
      }
      asm volatile("cp.async.commit_group;\n" ::);
    }
    {
      constexpr size_t JB = (size_t)3 * V * sizeof(A);
      if (JB % 16 == 0 && ((size_t)6 * V * sizeof(R)) % 16 == 0) {
        uint4* j4 = reinterpret_cast<uint4*>(Js);
        for (int e = threadIdx.x; e < (int)(JB / 16); e += blockDim.x) j4[e] = make_uint4(0, 0, 0, 0);
      } else {
        for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) Js[e] = 0;
      }
    }
    for (int e = threadIdx.x; e < 2 * NH + 1; e += blockDim.x) nh[e] = 0;   // nh and s_cnt
    float* stats = sj.tile_stats ? sj.tile_stats + 4 * (size_t)tile : nullptr;
    if (threadIdx.x == 0) s_have = stats && stats[3] != 0.f;
    float umax2 = 0.f, wmax = 0.f, cmax = 0.f;
    __syncthreads();
    const bool have = s_have;
    const R* wp = (const R*)sj.w;
    uint32_t* cellp = sj.cell;
    R *oxp = (R*)sj.ox, *oyp = (R*)sj.oy, *ozp = (R*)sj.oz;
    R *uxp = (R*)sj.ux, *uyp = (R*)sj.uy, *uzp = (R*)sj.uz;
    int* keyrank = reinterpret_cast<int*>(sj.w_b);
    int* const gsl[4] = {sj.perm + pbeg, reinterpret_cast<int*>(sj.ux_b) + pbeg,
                         reinterpret_cast<int*>(sj.uy_b) + pbeg,
                         reinterpret_cast<int*>(sj.uz_b) + pbeg};
    int* const gs0 = gsl[0];
    // ---- particles per window cell (+ the fixed-point bounds after a sort) --
    int kr[CG_KR];
    {
      int* hist = reinterpret_cast<int*>(Js) + 2 * V;   // zero; re-zeroed below
      auto count = [&](int ip, uint32_t cell) {
        int ci, cj, ck;
        unpack_cell(cell, ci, cj, ck);
        int vx = ci - c0x, vy = cj - c0y, vz = ck - c0z;
        if (vx > tex - 1 + D) vx -= nx; else if (vx < -D) vx += nx;
        if (vy > tey - 1 + D) vy -= ny; else if (vy < -D) vy += ny;
        if (vz > tez - 1 + D) vz -= nz; else if (vz < -D) vz += nz;
        const bool in = vx >= -D && vx <= tex - 1 + D && vy >= -D && vy <= tey - 1 + D &&
                        vz >= -D && vz <= tez - 1 + D;
        const int key = in ? (vx + D) + HB * ((vy + D) + HB * (vz + D)) : NH;
        const int r = atomicAdd(&s_cnt[key], 1);
        if (!have) {
          const float a = uxp[ip], b = uyp[ip], c = uzp[ip];
          umax2 = fmaxf(umax2, a * a + b * b + c * c);
          wmax = fmaxf(wmax, fabsf(wp[ip]));
          if (in) atomicAdd(hist + (vx + D + L) + (vy + D + L) * SY + (vz + D + L) * SZ, 1);
        }
        return key | (r << 11);
      };
      // the first CG_KR particles of each thread: cells loaded together, cell
      // and rank kept in registers until the slots are written; the rest of a
      // large tile through keyrank
      uint32_t cc[CG_KR];
#pragma unroll
      for (int k = 0; k < CG_KR; ++k) {
        const int ip = pbeg + threadIdx.x + k * blockDim.x;
        cc[k] = ip < pend ? cellp[ip] : 0u;
      }
#pragma unroll
      for (int k = 0; k < CG_KR; ++k) {
        const int ip = pbeg + threadIdx.x + k * blockDim.x;
        kr[k] = ip < pend ? count(ip, cc[k]) : 0;
      }
      for (int ip = pbeg + threadIdx.x + CG_KR * blockDim.x; ip < pend; ip += blockDim.x)
        keyrank[ip] = count(ip, cellp[ip]);
      __syncthreads();
      if (!have) {
        for (int r = threadIdx.x; r < V; r += blockDim.x) {
          cmax = fmaxf(cmax, (float)hist[r]);
          hist[r] = 0;
        }
      } else {
        umax2 = stats[0]; wmax = stats[1]; cmax = stats[2];
      }
    }
    // ---- groups: per class, prefix of the cells' group counts ---------------
    for (int q = wid; q < 32; q += nwarps) {
      int run = 0;
      for (int j0 = s_coff[q]; j0 < s_coff[q + 1]; j0 += 32) {
        const int j = j0 + lane;
        const int h = j < s_coff[q + 1] ? s_tau[j] : 0;
        const int g = j < s_coff[q + 1] ? (s_cnt[h] + CG_P - 1) / CG_P : 0;
        int incl = g;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl += y;
        }
        if (j < s_coff[q + 1]) s_pre[h] = run + incl - g;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) s_G[q] = run;
    }
    __syncthreads();
    // level table: the first position of level l and the classes present
    // there, for the levels that occur (below the largest class)
    int NI = 0, Gmax = 0;
    for (int c = 0; c < 32; ++c) { NI += s_G[c]; Gmax = max(Gmax, s_G[c]); }
    for (int l = threadIdx.x; l < min(Gmax, CG_LT); l += blockDim.x) {
      int P = 0;
      unsigned M = 0;
      for (int c = 0; c < 32; ++c) {
        const int n = s_G[c];
        P += min(n, l);
        M |= (n > l ? 1u : 0u) << c;
      }
      s_lvP[l] = P; s_lvM[l] = M;
    }
    __syncthreads();
    // position of the group of level l in class c
    auto gpos = [&](int l, int c) {
      if (l < CG_LT) return s_lvP[l] + __popc(s_lvM[l] & ((1u << c) - 1u));
      int P = 0;
      for (int c2 = 0; c2 < 32; ++c2) {
        const int n = s_G[c2];
        P += min(n, l) + (c2 < c && n > l ? 1 : 0);
      }
      return P;
    };
    if (pend - pbeg >= (1 << 21)) {   // beyond the slot encoding: flag, leave the tile
      if (threadIdx.x == 0) atomicExch(&sj.counters[1], 1);
      NI = 0;
    } else {
      auto place = [&](int ip, int v) {
        const int h = v & 2047, r = v >> 11;
        if (h == NH) { gs0[NI + r] = ip - pbeg; return; }
        const int k = r / CG_P, p = r - k * CG_P;
        const int pos = gpos(s_pre[h] + k, cls(h));
        const int e = (ip - pbeg) | (h << 21);
        gsl[p][pos] = e;
        if (r == s_cnt[h] - 1)          // the cell's last particle closes its group
          for (int q = p + 1; q < CG_P; ++q) gsl[q][pos] = -1;
      };
#pragma unroll
      for (int k = 0; k < CG_KR; ++k) {
        const int ip = pbeg + threadIdx.x + k * blockDim.x;
        if (ip < pend) place(ip, kr[k]);
      }
      for (int ip = pbeg + threadIdx.x + CG_KR * blockDim.x; ip < pend; ip += blockDim.x)
        place(ip, keyrank[ip]);
    }
    // ---- window staged: |E|, |B| maxima and the fixed-point scale -----------
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    float emax = 0.f, bmax = 0.f;
    if ((3 * V) % 4 == 0) {
      const float4* e4 = reinterpret_cast<const float4*>(Fs);
      const float4* b4 = e4 + (3 * V) / 4;
      for (int r = threadIdx.x; r < (3 * V) / 4; r += blockDim.x) {
        const float4 e = e4[r], b = b4[r];
        emax = fmaxf(emax, fmaxf(fmaxf(fabsf(e.x), fabsf(e.y)), fmaxf(fabsf(e.z), fabsf(e.w))));
        bmax = fmaxf(bmax, fmaxf(fmaxf(fabsf(b.x), fabsf(b.y)), fmaxf(fabsf(b.z), fabsf(b.w))));
      }
    } else {
      for (int r = threadIdx.x; r < 3 * V; r += blockDim.x) {
        emax = fmaxf(emax, fabsf(Fs[r]));
        bmax = fmaxf(bmax, fabsf(Fs[r + 3 * V]));
      }
    }
    emax = warp_max(emax); bmax = warp_max(bmax); umax2 = warp_max(umax2); wmax = warp_max(wmax);
    cmax = warp_max(cmax);
    if (lane == 0) {
      s_max[0][wid] = emax; s_max[1][wid] = bmax; s_max[2][wid] = umax2; s_max[3][wid] = wmax;
      s_max[4][wid] = cmax;
    }
    __syncthreads();
    double scale[3];
    {
      float E = 0.f, B = 0.f, U2 = 0.f, Wm = 0.f, Cm = 0.f;
      for (int w = 0; w < nwarps; ++w) {
        E = fmaxf(E, s_max[0][w]); B = fmaxf(B, s_max[1][w]);
        U2 = fmaxf(U2, s_max[2][w]); Wm = fmaxf(Wm, s_max[3][w]); Cm = fmaxf(Cm, s_max[4][w]);
      }
      // the bound of k_tile_step's fixed-point scale (see there)
      const double c = sj.clight;
      const double qdm = fabs(sj.q) / sj.m * sj.dt;
      const double tau = 0.5 * qdm * 1.7320508075688772 * (double)B;
      const double ub = (sqrt((double)U2) * (1.0 + tau) + qdm * 1.7320508075688772 * (double)E) *
                        (1.0 + tau) * 1.0001;
      const double vb = ub / sqrt(1.0 + ub * ub / (c * c));
      const double dV = sj.dx * sj.dy * sj.dz;
      constexpr int reach = L + H + 3;
      const double np_ = fmax((double)Cm * (reach * reach * reach), 1.0);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double dq = q == 0 ? sj.dx : (q == 1 ? sj.dy : sj.dz);
        const double disp = fmin(vb * sj.dt / dq, 1.0);
        const double bound = fabs(sj.q) * (double)Wm * dq / (sj.dt * dV) * disp;
        const double s = scale_bits<MODE, ORDER>() / fmax(np_ * bound, 1e-300);
        scale[q] = fmin(s, 1e30);
      }
    }
    // ---- particles -----------------------------------------------------------
    const R dtdx = (R)(sj.dt / sj.dx), dtdy = (R)(sj.dt / sj.dy), dtdz = (R)(sj.dt / sj.dz);
    const R clghtisq = (R)(1.0 / (sj.clight * sj.clight));
    const R cst_b = (R)(sj.q * sj.dt * 0.5 / sj.m), cst_v = (R)(sj.q * sj.dt / sj.m);
    const R invc = (R)(1.0 / sj.clight);
    const R qdx = (R)(sj.q / (sj.dt * sj.dy * sj.dz)), qdy = (R)(sj.q / (sj.dt * sj.dx * sj.dz)),
            qdz = (R)(sj.q / (sj.dt * sj.dx * sj.dy));
    const R scx = (R)scale[0], scy = (R)scale[1], scz = (R)scale[2];
    const bool vay = sj.pusher == 1;
    int* q_list = sj.rank_b;
    uint32_t* q_pk = sj.cell_b;
    R *q_ox = (R*)sj.ox_b, *q_oy = (R*)sj.oy_b, *q_oz = (R*)sj.oz_b;
    double ke = 0.0;
    float nu2 = 0.f, nwm = 0.f;
    int nslow = 0, bad = 0;

    // what the next step's bounds need from a particle now in cell (nci, ncj, nck)
    auto next_bounds = [&](int nci, int ncj, int nck, float ux, float uy, float uz, float w) {
      if (!stats) return;
      int hx = nci - c0x, hy = ncj - c0y, hz = nck - c0z;
      if (hx > tex - 1 + D) hx -= nx; else if (hx < -D) hx += nx;
      if (hy > tey - 1 + D) hy -= ny; else if (hy < -D) hy += ny;
      if (hz > tez - 1 + D) hz -= nz; else if (hz < -D) hz += nz;
      if (hx >= -D && hx <= tex - 1 + D && hy >= -D && hy <= tey - 1 + D && hz >= -D &&
          hz <= tez - 1 + D)
        atomicAdd(nh + (hx + D) + (hy + D) * HB + (hz + D) * (HB * HB), 1);
      nu2 = fmaxf(nu2, ux * ux + uy * uy + uz * uz);
      nwm = fmaxf(nwm, fabsf(w));
    };

    // the slots of a thread's next group are read one group ahead
    int en[CG_P];
    if ((int)threadIdx.x < NI) {
#pragma unroll
      for (int p = 0; p < CG_P; ++p) en[p] = gsl[p][threadIdx.x];
    }
    for (int it = threadIdx.x; it < NI; it += blockDim.x) {
      int e[CG_P];
#pragma unroll
      for (int p = 0; p < CG_P; ++p) e[p] = en[p];
      if (it + (int)blockDim.x < NI) {
#pragma unroll
        for (int p = 0; p < CG_P; ++p) en[p] = gsl[p][it + blockDim.x];
      }
      const int h = (int)((unsigned)e[0] >> 21);
      int n = 1;
#pragma unroll
      for (int p = 1; p < CG_P; ++p) n += e[p] >= 0;
      const int hx = h % HB, hy = (h / HB) % HB, hz = h / (HB * HB);
      const int vx = hx - D, vy = hy - D, vz = hz - D;
      int ci = c0x + vx, cj = c0y + vy, ck = c0z + vz;
      ci = ci < 0 ? ci + nx : (ci >= nx ? ci - nx : ci);
      cj = cj < 0 ? cj + ny : (cj >= ny ? cj - ny : cj);
      ck = ck < 0 ? ck + nz : (ck >= nz ? ck - nz : ck);
      int ip[CG_P];
      R ox[CG_P], oy[CG_P], oz[CG_P], u0[CG_P], u1[CG_P], u2[CG_P], wg[CG_P];
#pragma unroll
      for (int p = 0; p < CG_P; ++p) {
        ip[p] = pbeg + ((e[p] >= 0 ? e[p] : e[0]) & 0x1FFFFF);
        ox[p] = oxp[ip[p]]; oy[p] = oyp[ip[p]]; oz[p] = ozp[ip[p]];
        u0[p] = uxp[ip[p]]; u1[p] = uyp[ip[p]]; u2[p] = uzp[ip[p]]; wg[p] = wp[ip[p]];
      }
      // ---- gather: each window value serves the group's particles -----------
      R eb[6][CG_P];
      {
        // node shapes for all six components; the staggered ones computed where
        // needed, in a component order that keeps at most two of them live
        f2_t ax[CG_Q], ay[CG_Q], az[CG_Q];
        f2_t nX[CG_Q][4], nY[CG_Q][4], nZ[CG_Q][4], sA[CG_Q][4], sB[CG_Q][4];
#pragma unroll
        for (int q = 0; q < CG_Q; ++q) {
          ax[q] = f2_pack(ox[2 * q], ox[2 * q + 1]); ay[q] = f2_pack(oy[2 * q], oy[2 * q + 1]);
          az[q] = f2_pack(oz[2 * q], oz[2 * q + 1]);
          node_pair<ORDER>(ax[q], nX[q]); node_pair<ORDER>(ay[q], nY[q]);
          node_pair<ORDER>(az[q], nZ[q]);
        }
        // gather and deposit stencils of a cell both start at its window address
        const float* F = Fs + hx + hy * SY + hz * SZ;
        f2_t o2[CG_Q];
#define PXRB_CG_COMP(c_, NA_, NB_, NC_, a_, b_, z_)                                          \
  cg_comp<NA_, NB_, NC_, SY, SZ>(F + (c_) * V, a_, b_, z_, o2);                               \
  _Pragma("unroll") for (int q = 0; q < CG_Q; ++q) {                                          \
    eb[c_][2 * q] = f2_lo(o2[q]); eb[c_][2 * q + 1] = f2_hi(o2[q]);                           \
  }
#define PXRB_CG_STAG(dst_, o_) \
  _Pragma("unroll") for (int q = 0; q < CG_Q; ++q) stag_pair<ORDER>(o_[q], dst_[q]);
        PXRB_CG_STAG(sA, ax)                         // sA = x
        PXRB_CG_COMP(0, S, N, N, sA, nY, nZ)         // Ex
        PXRB_CG_STAG(sB, az)                         // sB = z
        PXRB_CG_COMP(4, S, N, S, sA, nY, sB)         // By
        PXRB_CG_COMP(2, N, N, S, nX, nY, sB)         // Ez
        PXRB_CG_STAG(sA, ay)                         // sA = y
        PXRB_CG_COMP(3, N, S, S, nX, sA, sB)         // Bx
        PXRB_CG_COMP(1, N, S, N, nX, sA, nZ)         // Ey
        PXRB_CG_STAG(sB, ax)                         // sB = x
        PXRB_CG_COMP(5, S, S, N, sB, sA, nZ)         // Bz
#undef PXRB_CG_STAG
#undef PXRB_CG_COMP
      }
      // ---- push, position, store; deposit factors ------------------------------
      R nox[CG_P], noy[CG_P], noz[CG_P], cqx[CG_P], cqy[CG_P], cqz[CG_P];
#pragma unroll
      for (int p = 0; p < CG_P; ++p) {
        const bool valid = p < n;
        R ux = u0[p], uy = u1[p], uz = u2[p];
        const R wgt = wg[p];
        R gi;
        if (vay) {
          gi = inv_sqrt<R>((R)1 + (ux * ux + uy * uy + uz * uz) * clghtisq);
          vay_push(ux, uy, uz, gi, eb[0][p], eb[1][p], eb[2][p], eb[3][p], eb[4][p], eb[5][p],
                   cst_v, invc, clghtisq);
        } else {
          boris_push(ux, uy, uz, gi, eb[0][p], eb[1][p], eb[2][p], eb[3][p], eb[4][p], eb[5][p],
                     cst_b, clghtisq);
          set_gamma(ux, uy, uz, gi, clghtisq);
        }
        R px = ox[p], py = oy[p], pz = oz[p];
        int sx = 0, sy = 0, sz = 0;
        cell_step(px, sx, ux * gi * dtdx);
        cell_step(py, sy, uy * gi * dtdy);
        cell_step(pz, sz, uz * gi * dtdz);
        nox[p] = px; noy[p] = py; noz[p] = pz;
        // at orders 1 and 3 the Esirkepov node is the cell: a particle that
        // stays in its cell deposits on the group's box
        const bool same = sx == 0 && sy == 0 && sz == 0;
        const R wq = valid && same ? wgt : (R)0;
        cqx[p] = wq * qdx * scx; cqy[p] = wq * qdy * scy; cqz[p] = wq * qdz * scz;
        if (!valid) continue;
        if (!same) {
          if (sx < -1 || sx > 1 || sy < -1 || sy > 1 || sz < -1 || sz > 1) bad = 1;
          const bool in_new = vx + sx >= -D && vx + sx <= tex - 1 + D && vy + sy >= -D &&
                              vy + sy <= tey - 1 + D && vz + sz >= -D && vz + sz <= tez - 1 + D;
          if (in_new) {
            const int q = atomicAdd(&s_qn, 1);
            q_list[pbeg + q] = ip[p];
            q_pk[ip[p]] = (unsigned)(vx + D + L) | ((unsigned)(vy + D + L) << 8) |
                          ((unsigned)(vz + D + L) << 16) | ((unsigned)(sx + 1) << 24) |
                          ((unsigned)(sy + 1) << 26) | ((unsigned)(sz + 1) << 28);
            q_ox[ip[p]] = ox[p]; q_oy[ip[p]] = oy[p]; q_oz[ip[p]] = oz[p];
          } else {
            ++nslow;
            EsirAxis<ORDER, R> EX, EY, EZ;
            EX.set(ci + sx, px, ci, ox[p]);
            EY.set(cj + sy, py, cj, oy[p]);
            EZ.set(ck + sz, pz, ck, oz[p]);
            dep_global<ORDER, R>(sj, EX, EY, EZ, wgt * qdx, wgt * qdy, wgt * qdz);
          }
        }
        int nci = ci + sx, ncj = cj + sy, nck = ck + sz;
        nci = nci < 0 ? nci + nx : (nci >= nx ? nci - nx : nci);
        ncj = ncj < 0 ? ncj + ny : (ncj >= ny ? ncj - ny : ncj);
        nck = nck < 0 ? nck + nz : (nck >= nz ? nck - nz : nck);
        cellp[ip[p]] = pack_cell(nci, ncj, nck);
        oxp[ip[p]] = px; oyp[ip[p]] = py; ozp[ip[p]] = pz;
        uxp[ip[p]] = ux; uyp[ip[p]] = uy; uzp[ip[p]] = uz;
        next_bounds(nci, ncj, nck, ux, uy, uz, wgt);
        const R u2 = (ux * ux + uy * uy + uz * uz) * clghtisq;
        ke += (double)(quot<R>(u2, (R)1 + sqrt(u2 + (R)1)) * wgt);
      }
      // ---- summed deposit of the particles that stay in the cell, by pairs ----
#pragma unroll
      for (int q = 0; q < CG_Q; ++q) {
        if (cqx[2 * q] == (R)0 && cqx[2 * q + 1] == (R)0) continue;
        f2_t t0[3][4], t1[3][4];
        node_pair<ORDER>(f2_pack(nox[2 * q], nox[2 * q + 1]), t0[0]);
        node_pair<ORDER>(f2_pack(noy[2 * q], noy[2 * q + 1]), t0[1]);
        node_pair<ORDER>(f2_pack(noz[2 * q], noz[2 * q + 1]), t0[2]);
        node_pair<ORDER>(f2_pack(ox[2 * q], ox[2 * q + 1]), t1[0]);
        node_pair<ORDER>(f2_pack(oy[2 * q], oy[2 * q + 1]), t1[1]);
        node_pair<ORDER>(f2_pack(oz[2 * q], oz[2 * q + 1]), t1[2]);
        const f2_t cq[3] = {f2_pack(cqx[2 * q], cqx[2 * q + 1]), f2_pack(cqy[2 * q], cqy[2 * q + 1]),
                            f2_pack(cqz[2 * q], cqz[2 * q + 1])};
        cg_deposit<ORDER, SY, SZ, V>(Js + hx + hy * SY + hz * SZ, t0, t1, cq);
      }
    }
    // ---- particles outside the window: global gather and deposit ------------
    {
      const int n_out = s_cnt[NH];
      for (int s = threadIdx.x; s < n_out; s += blockDim.x) {
        const int p = pbeg + gs0[NI + s];
        int ci, cj, ck;
        unpack_cell(cellp[p], ci, cj, ck);
        const R ox = oxp[p], oy = oyp[p], oz = ozp[p];
        R ux = uxp[p], uy = uyp[p], uz = uzp[p];
        const R wgt = wp[p];
        R eb[6];
        gather_global<ORDER, R>(sj, ci, cj, ck, ox, oy, oz, eb);
        R gi;
        if (vay) {
          gi = inv_sqrt<R>((R)1 + (ux * ux + uy * uy + uz * uz) * clghtisq);
          vay_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_v, invc, clghtisq);
        } else {
          boris_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_b, clghtisq);
          set_gamma(ux, uy, uz, gi, clghtisq);
        }
        R px = ox, py = oy, pz = oz;
        int sx = 0, sy = 0, sz = 0;
        cell_step(px, sx, ux * gi * dtdx);
        cell_step(py, sy, uy * gi * dtdy);
        cell_step(pz, sz, uz * gi * dtdz);
        EsirAxis<ORDER, R> EX, EY, EZ;
        bool ok = EX.set(ci + sx, px, ci, ox);
        ok = EY.set(cj + sy, py, cj, oy) && ok;
        ok = EZ.set(ck + sz, pz, ck, oz) && ok;
        if (!ok) bad = 1;
        ++nslow;
        dep_global<ORDER, R>(sj, EX, EY, EZ, wgt * qdx, wgt * qdy, wgt * qdz);
        int nci = ci + sx, ncj = cj + sy, nck = ck + sz;
        nci = nci < 0 ? nci + nx : (nci >= nx ? nci - nx : nci);
        ncj = ncj < 0 ? ncj + ny : (ncj >= ny ? ncj - ny : ncj);
        nck = nck < 0 ? nck + nz : (nck >= nz ? nck - nz : nck);
        cellp[p] = pack_cell(nci, ncj, nck);
        oxp[p] = px; oyp[p] = py; ozp[p] = pz;
        uxp[p] = ux; uyp[p] = uy; uzp[p] = uz;
        next_bounds(nci, ncj, nck, ux, uy, uz, wgt);
        const R u2 = (ux * ux + uy * uy + uz * uz) * clghtisq;
        ke += (double)(quot<R>(u2, (R)1 + sqrt(u2 + (R)1)) * wgt);
      }
    }
    __syncthreads();
    // ---- window particles with a node change (k_tile_step's queue) -----------
    {
      const int nq = s_qn;
      for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int ip = q_list[pbeg + q];
        const unsigned pk = q_pk[ip];
        const int bx = pk & 255u, by = (pk >> 8) & 255u, bz = (pk >> 16) & 255u;
        const int sx = (int)((pk >> 24) & 3u) - 1, sy = (int)((pk >> 26) & 3u) - 1,
                  sz = (int)((pk >> 28) & 3u) - 1;
        const R ox = q_ox[ip], oy = q_oy[ip], oz = q_oz[ip];
        const R nox = oxp[ip], noy = oyp[ip], noz = ozp[ip], wq = wp[ip];
        int r0, r1;
        R a0, a1;
        EsirAxis<ORDER, R> EX, EY, EZ;
        esir_node<ORDER, R>(nox, r0, a0); esir_node<ORDER, R>(ox, r1, a1);
        bool ok = EX.set(bx + sx + r0, a0, bx + r1, a1);
        esir_node<ORDER, R>(noy, r0, a0); esir_node<ORDER, R>(oy, r1, a1);
        ok = EY.set(by + sy + r0, a0, by + r1, a1) && ok;
        esir_node<ORDER, R>(noz, r0, a0); esir_node<ORDER, R>(oz, r1, a1);
        ok = EZ.set(bz + sz + r0, a0, bz + r1, a1) && ok;
        if (!ok) bad = 1;
        dep_window<ORDER, R, MODE, SY, SZ, V>(Js, EX, EY, EZ, wq * qdx * scx, wq * qdy * scy,
                                              wq * qdz * scz);
      }
    }
    __syncthreads();
    // ---- flush the J window: FP64 atomics into the periodic grid -------------
    {
#pragma unroll 1
      for (int comp = 0; comp < 3; ++comp) {
        double* dst = comp == 0 ? sj.jx : comp == 1 ? sj.jy : sj.jz;
        const double inv = 1.0 / scale[comp];
        const A* src = Js + comp * V;
        for (int r = threadIdx.x; r < V; r += blockDim.x) {
          const int v = src[r];
          if (v == 0) continue;
          const int c = r / SZ, b = (r - c * SZ) / SY, a = r - c * SZ - b * SY;
          const int gi = GlobAcc::wrap(wox + a, nx), gj = GlobAcc::wrap(woy + b, ny),
                    gk = GlobAcc::wrap(woz + c, nz);
          atomicAdd(dst + gi + (i64)nx * (gj + (i64)ny * gk), (double)v * inv);
        }
      }
    }
    // ---- kinetic energy of the tile, the next step's bounds -------------------
    {
      double v = ke;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) s_red[wid] = v;
      if (nslow) atomicAdd(&sj.counters[0], nslow);
      if (bad) atomicExch(&sj.counters[1], 1);
      if (stats) {
        float c = 0.f;
        for (int r = threadIdx.x; r < NH; r += blockDim.x) c = fmaxf(c, (float)nh[r]);
        c = warp_max(c);
        const float a = warp_max(nu2), b = warp_max(nwm);
        if (lane == 0) { s_max[0][wid] = a; s_max[1][wid] = b; s_max[2][wid] = c; }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nwarps; ++w) t += s_red[w];
        sj.ke_tile[tile] = t * sj.m * sj.clight * sj.clight;
        if (stats) {
          float a = 0.f, b = 0.f, c = 0.f;
          for (int w = 0; w < nwarps; ++w) {
            a = fmaxf(a, s_max[0][w]); b = fmaxf(b, s_max[1][w]); c = fmaxf(c, s_max[2][w]);
          }
          stats[0] = a; stats[1] = b; stats[2] = c; stats[3] = 1.f;
        }
      }
    }
    __syncthreads();
  }
}

// Launch of the cell-grouped kernel on the persistent work list of
// pxrb_tiled_particle_step; threads <= CG_THREADS.
template <int ORDER, int T, int D>
int launch_cell(const Job* jobs, const int2* work, int nwork, const int* nwork_dev, int* ctr,
                int threads, int ctas, size_t smem, cudaStream_t s) {
  constexpr int W = T + 2 * D + Reach<ORDER>::L + Reach<ORDER>::H;
  if (threads > CG_THREADS || smem < (size_t)cg_smem_bytes(T, D, win_sz(T, W) * W))
    return PXRB_EINVAL;
  auto kern = k_cell_step<ORDER, T, D>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return PXRB_EUNSUPPORTED;
  if (cudaMemsetAsync(ctr, 0, sizeof(int), s) != cudaSuccess) return PXRB_ELAUNCH;
  kern<<<ctas, threads, smem, s>>>(jobs, work, nwork, nwork_dev, ctr);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // namespace pxrt
