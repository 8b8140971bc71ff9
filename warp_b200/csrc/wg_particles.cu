// Particle kernels: fixed-point CIC deposition, field gather, the fused
// gather + quad + Boris leapfrog push + boundaries kernel, and moments.
//
// Compiled with --fmad=false: gather and push evaluate the reference's
// expressions in its operand order, so with identical phi and particles the
// results match the CPU oracle bit for bit. Deposition accumulates
// round(weight * 2^46) in 64-bit integers, so rho does not depend on the
// order of the atomic adds (bit-identical run to run); it differs from an
// FP64 running sum only by the rounding of each weight to 2^-46.

#include <cmath>
#include <mutex>
#include <string>

#include "wg_internal.h"

namespace wg {

// 2^46: one particle's full CIC weight (1.0) in accumulator units. The
// convert kernel reports WG_EOVERFLOW once a node reaches 2^62, i.e. 65536
// full particle weights on one node (the unsigned sum wraps only at 2^64).
constexpr double kFixScale = 70368744177664.0;  // 2^46
constexpr double kFixInv = 1.0 / 70368744177664.0;

struct GridP {
  int nx, ny, nz;
  double dx, dy, dz, xmmin, ymmin, zmmin, zgrid;
  // 1/dx and 1/(2 dx) per axis, formed once on the host (IEEE divisions,
  // the same bits as the device's)
  double dxi, dyi, dzi, tdxi, tdyi, tdzi;
};

inline GridP make_gridp(int nx, int ny, int nz, double dx, double dy, double dz, double xmmin, double ymmin,
                        double zmmin, double zgrid) {
  return GridP{nx, ny, nz, dx, dy, dz, xmmin, ymmin, zmmin, zgrid,
               1. / dx, 1. / dy, 1. / dz, 1. / (2. * dx), 1. / (2. * dy), 1. / (2. * dz)};
}

namespace {

__device__ inline void cellfrac(double s, int n, int& i, double& f) {
  i = (int)s;
  if (i > n - 1) i = n - 1;
  if (i < 0) i = 0;
  f = s - i;
}

// setrho3ddirect1 (w3d.F:7757-7960) with 64-bit fixed-point weights. A CTA
// takes a chunk of DEP_NT*DEP_PPT consecutive particles; warp w of the CTA
// takes the DEP_PPT*32 consecutive particles starting at w*32*DEP_PPT, 32 at
// a time (coalesced loads). Each particle's 8 CIC weights are rounded to
// integers (2^46 per full weight) and summed three ways:
//  - while a whole warp-load of 32 particles sits in one cell and it is the
//    same cell as the previous warp-load (sorted particles: a cell holds
//    hundreds), every lane keeps adding its weights in registers; the warp
//    sums its lanes once, when the cell changes;
//  - otherwise each lane adds its own weights, visiting the 8 nodes in an
//    order rotated by lane (fewer same-address conflicts);
//  - the sums go to a shared-memory copy of the chunk's bounding box of
//    nodes, added to the global accumulator at the end, or straight to global
//    memory when the box is larger than DEP_BOX nodes (unsorted particles).
// Integer adds commute, so rho does not depend on any of these orders.
constexpr int DEP_NT = 256, DEP_PPT = 16, DEP_BOX = 3072;

// A box node holds its fixed-point sum as three 32-bit parts (bits 0-15,
// 16-31 and 32 up), so every shared-memory add is a 32-bit atomic: 64-bit
// shared atomics are several times slower. A chunk adds at most
// DEP_NT*DEP_PPT = 4096 contributions to a node, so the two 16-bit parts sum
// below 2^28 and the high part below 2^26 (total below 2^58): no part
// overflows, and the recombined 64-bit value is exact.
template <int NB>
struct DepBoxN {
  unsigned lo[NB], mid[NB], hi[NB];
};
using DepBox = DepBoxN<DEP_BOX>;
template <int NB>
__device__ inline void box_add(DepBoxN<NB>& b, int n, unsigned long long v) {
  const unsigned l = (unsigned)(v & 0xFFFFull), m = (unsigned)((v >> 16) & 0xFFFFull), h = (unsigned)(v >> 32);
  if (l) atomicAdd(&b.lo[n], l);
  if (m) atomicAdd(&b.mid[n], m);
  if (h) atomicAdd(&b.hi[n], h);
}

// Cell and fractions of particle i; FP32 positions are converted to FP64
// first (exactly), so both storages share the FP64 arithmetic below.
template <typename T>
__device__ inline bool dep_cell(const T* xp, const T* yp, const T* zp, const T* gaminv, int64_t i, int64_t np,
                                const GridP& g, int& ii, int& jj, int& kk, double& u1, double& v1, double& w1) {
  if (i >= np || gaminv[i] == (T)0) return false;
  cellfrac(((double)xp[i] - g.xmmin) * g.dxi, g.nx, ii, u1);
  cellfrac(((double)yp[i] - g.ymmin) * g.dyi, g.ny, jj, v1);
  cellfrac(((double)zp[i] - g.zgrid - g.zmmin) * g.dzi, g.nz, kk, w1);
  return true;
}

// The sum over the 32 lanes of a warp of v < 2^51, exact, as two 32-bit
// warp reductions of its bits 0-24 and 25 up (each sums below 2^31).
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  const unsigned lo = __reduce_add_sync(0xffffffffu, (unsigned)(v & 0x1FFFFFFull));
  const unsigned hi = __reduce_add_sync(0xffffffffu, (unsigned)(v >> 25));
  return ((unsigned long long)hi << 25) + lo;
}

// Adds v to node (i, j, k) of the box or of the global accumulator.
template <int NB>
__device__ inline void dep_add(DepBoxN<NB>& box, bool use_box, int ox, int oy, int oz, int bx, int by,
                               unsigned long long* acc, const GridP& g, int i, int j, int k, unsigned long long v) {
  if (use_box)
    box_add(box, (i - ox) + bx * ((j - oy) + by * (k - oz)), v);
  else
    atomicAdd(acc + i + (g.nx + 1) * (j + (g.ny + 1) * k), v);
}

// Four blocks per SM (64 registers): 1.37 -> 1.21 ms for 5e7 particles.
template <typename T>
__global__ void __launch_bounds__(DEP_NT, 4) k_deposit(const T* __restrict__ xp, const T* __restrict__ yp,
                                                    const T* __restrict__ zp, const T* __restrict__ gaminv,
                                                    int64_t np, GridP g, unsigned long long* __restrict__ acc) {
  __shared__ DepBox box;
  __shared__ int bmin[3], bmax[3];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t base = (int64_t)blockIdx.x * (DEP_NT * DEP_PPT) + (int64_t)warp * (32 * DEP_PPT) + lane;
  if (tid < 3) {
    bmin[tid] = 0x7fffffff;
    bmax[tid] = -1;
  }
  __syncthreads();
  int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-1, -1, -1};
  for (int j = 0; j < DEP_PPT; ++j) {
    int c[3];
    double f1, f2, f3;
    if (dep_cell(xp, yp, zp, gaminv, base + 32 * j, np, g, c[0], c[1], c[2], f1, f2, f3))
      for (int d = 0; d < 3; ++d) {
        lo[d] = min(lo[d], c[d]);
        hi[d] = max(hi[d], c[d]);
      }
  }
  for (int d = 0; d < 3; ++d) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  if (lane == 0 && hi[0] >= 0)
    for (int d = 0; d < 3; ++d) {
      atomicMin(&bmin[d], lo[d]);
      atomicMax(&bmax[d], hi[d]);
    }
  __syncthreads();
  // node box [bmin, bmax+1] in each direction
  const int ox = bmin[0], oy = bmin[1], oz = bmin[2];
  const int bx = bmax[0] - ox + 2, by = bmax[1] - oy + 2, bz = bmax[2] - oz + 2;
  const bool any = bmax[0] >= 0;
  const bool use_box = any && (long long)bx * by * bz <= DEP_BOX;
  if (use_box)
    for (int i = tid; i < bx * by * bz; i += DEP_NT) {
      box.lo[i] = 0u;
      box.mid[i] = 0u;
      box.hi[i] = 0u;
    }
  __syncthreads();
  if (any) {
    // register sums of the warp's current uniform cell (ci, cj, ck), or ci < 0
    unsigned long long s[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) s[n] = 0ull;
    int ci = -1, cj = 0, ck = 0;
    auto flush = [&]() {
      if (ci < 0) return;
#pragma unroll
      for (int n = 0; n < 8; ++n) s[n] = warp_sum_u64(s[n]);
      // lane n < 8 adds node n
      unsigned long long mine = 0ull;
#pragma unroll
      for (int n = 0; n < 8; ++n)
        if (lane == n) mine = s[n];
      if (lane < 8 && mine)
        dep_add(box, use_box, ox, oy, oz, bx, by, acc, g, ci + (lane & 1), cj + ((lane >> 1) & 1), ck + (lane >> 2),
                mine);
#pragma unroll
      for (int n = 0; n < 8; ++n) s[n] = 0ull;
      ci = -1;
    };
    for (int j = 0; j < DEP_PPT; ++j) {
      int ii = 0, jj = 0, kk = 0;
      double u1 = 0., v1 = 0., w1 = 0.;
      const bool live = dep_cell(xp, yp, zp, gaminv, base + 32 * j, np, g, ii, jj, kk, u1, v1, w1);
      const int key = live ? ii + (g.nx + 1) * (jj + (g.ny + 1) * kk) : -1;
      const double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
      const int key0 = __shfl_sync(0xffffffffu, key, 0);
      if (__all_sync(0xffffffffu, live && key == key0)) {
        unsigned long long w[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          const int dx = n & 1, dy = (n >> 1) & 1, dz = n >> 2;
          const double wgt = (dx ? u1 : u0) * (dy ? v1 : v0) * (dz ? w1 : w0);
          w[n] = (unsigned long long)llrint(wgt * kFixScale);
        }
        const int i0 = __shfl_sync(0xffffffffu, ii, 0), j0 = __shfl_sync(0xffffffffu, jj, 0),
                  k0 = __shfl_sync(0xffffffffu, kk, 0);
        if (ci != i0 || cj != j0 || ck != k0) {
          flush();
          ci = i0;
          cj = j0;
          ck = k0;
        }
#pragma unroll
        for (int n = 0; n < 8; ++n) s[n] += w[n];
        continue;
      }
      flush();
      // mixed cells: each lane adds its own 8 weights, visiting the nodes
      // in an order rotated by lane so that lanes of one cell hit
      // different nodes in the same instruction
      if (live) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = (j + lane) & 7;
          const int dx = n & 1, dy = (n >> 1) & 1, dz = n >> 2;
          const double wgt = (dx ? u1 : u0) * (dy ? v1 : v0) * (dz ? w1 : w0);
          const unsigned long long v = (unsigned long long)llrint(wgt * kFixScale);
          if (v) dep_add(box, use_box, ox, oy, oz, bx, by, acc, g, ii + dx, jj + dy, kk + dz, v);
        }
      }
    }
    flush();
  }
  if (use_box) {
    __syncthreads();
    for (int i = tid; i < bx * by * bz; i += DEP_NT) {
      const unsigned long long v =
          ((unsigned long long)box.hi[i] << 32) + ((unsigned long long)box.mid[i] << 16) + box.lo[i];
      if (v) {
        const int lx = i % bx, ly = (i / bx) % by, lz = i / (bx * by);
        atomicAdd(acc + (ox + lx) + (g.nx + 1) * ((oy + ly) + (g.ny + 1) * (oz + lz)), v);
      }
    }
  }
}

// rho (+)= acc * g * 2^-46; flags accumulator values at or above 2^62.
// Zeroing as a kernel: a cudaMemsetAsync may wait for a copy engine that a
// caller's bulk transfers on other streams keep busy.
__global__ void k_zero_u64(unsigned long long* __restrict__ u, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) u[i] = 0ull;
}

__global__ void k_publish_word(const unsigned long long* __restrict__ src, unsigned long long* dst) {
  *(volatile unsigned long long*)dst = *src;
  __threadfence_system();
}

__global__ void k_fix_to_rho(const unsigned long long* __restrict__ acc, double* __restrict__ rho, size_t n,
                             double scale, int add, unsigned long long* flag) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long a = acc[i];
  if (a >> 62) atomicOr(flag, 1ull);
  double v = (double)a * scale;
  rho[i] = add ? rho[i] + v : v;
}

// applyrhoboundaryconditions3d (w3d.F:2660-2750), serial, no rho guard:
// one thread per line perpendicular to the face, phases x, y, z in order.
__global__ void k_rhobc(double* __restrict__ rho, int nx, int ny, int nz, int axis, int blo, int bhi) {
  const size_t sx = 1, sy = nx + 1, sz = (size_t)(nx + 1) * (ny + 1);
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride, base;
  int n;
  if (axis == 0) {
    if (t >= (size_t)(ny + 1) * (nz + 1)) return;
    base = (t % (ny + 1)) * sy + (t / (ny + 1)) * sz;
    stride = sx;
    n = nx;
  } else if (axis == 1) {
    if (t >= (size_t)(nx + 1) * (nz + 1)) return;
    base = (t % (nx + 1)) * sx + (t / (nx + 1)) * sz;
    stride = sy;
    n = ny;
  } else {
    if (t >= (size_t)(nx + 1) * (ny + 1)) return;
    base = (t % (nx + 1)) * sx + (t / (nx + 1)) * sy;
    stride = sz;
    n = nz;
  }
  double* lo = rho + base;
  double* hi = rho + base + (size_t)n * stride;
  if (blo == 1) *lo = *lo + *lo;
  if (bhi == 1) *hi = *hi + *hi;
  if (blo == 2 || bhi == 2) {
    *lo = *lo + *hi;
    *hi = *lo;
  }
}

// sete_from_phi_linear3d (w3d.F:3963-4108), no symmetry: E from centred
// differences of phi at the 8 cell nodes, trilinearly weighted.
__device__ inline void gather_e(const double* __restrict__ phi, const GridP& g, double x, double y, double z,
                                double& ext, double& eyt, double& ezt) {
  const double tdxi = g.tdxi, tdyi = g.tdyi, tdzi = g.tdzi;
  const double dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
  int i, j, k;
  double u1, v1, w1;
  cellfrac((x - g.xmmin) * dxi, g.nx, i, u1);
  cellfrac((y - g.ymmin) * dyi, g.ny, j, v1);
  cellfrac((z - g.zgrid - g.zmmin) * dzi, g.nz, k, w1);
  const double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
  // phi(i+a, j+b, k+c) through one base pointer and 32-bit offsets (the
  // padded grid holds fewer than 2^31 nodes)
  const int sy = g.nx + 3, sz = sy * (g.ny + 3);
  const double* base = phi + ((i + 1) + sy * (j + 1) + sz * (k + 1));
  auto P = [&](int a, int b, int c) { return __ldg(base + ((a - i) + (b - j) * sy + (c - k) * sz)); };
  ext = tdxi * (u0 * v0 * w0 * (P(i - 1, j, k) - P(i + 1, j, k)) + u1 * v0 * w0 * (P(i, j, k) - P(i + 2, j, k)) +
                u0 * v1 * w0 * (P(i - 1, j + 1, k) - P(i + 1, j + 1, k)) +
                u1 * v1 * w0 * (P(i, j + 1, k) - P(i + 2, j + 1, k)) +
                u0 * v0 * w1 * (P(i - 1, j, k + 1) - P(i + 1, j, k + 1)) +
                u1 * v0 * w1 * (P(i, j, k + 1) - P(i + 2, j, k + 1)) +
                u0 * v1 * w1 * (P(i - 1, j + 1, k + 1) - P(i + 1, j + 1, k + 1)) +
                u1 * v1 * w1 * (P(i, j + 1, k + 1) - P(i + 2, j + 1, k + 1)));
  eyt = tdyi * (u0 * v0 * w0 * (P(i, j - 1, k) - P(i, j + 1, k)) + u1 * v0 * w0 * (P(i + 1, j - 1, k) - P(i + 1, j + 1, k)) +
                u0 * v1 * w0 * (P(i, j, k) - P(i, j + 2, k)) + u1 * v1 * w0 * (P(i + 1, j, k) - P(i + 1, j + 2, k)) +
                u0 * v0 * w1 * (P(i, j - 1, k + 1) - P(i, j + 1, k + 1)) +
                u1 * v0 * w1 * (P(i + 1, j - 1, k + 1) - P(i + 1, j + 1, k + 1)) +
                u0 * v1 * w1 * (P(i, j, k + 1) - P(i, j + 2, k + 1)) +
                u1 * v1 * w1 * (P(i + 1, j, k + 1) - P(i + 1, j + 2, k + 1)));
  ezt = tdzi * (u0 * v0 * w0 * (P(i, j, k - 1) - P(i, j, k + 1)) + u1 * v0 * w0 * (P(i + 1, j, k - 1) - P(i + 1, j, k + 1)) +
                u0 * v1 * w0 * (P(i, j + 1, k - 1) - P(i, j + 1, k + 1)) +
                u1 * v1 * w0 * (P(i + 1, j + 1, k - 1) - P(i + 1, j + 1, k + 1)) +
                u0 * v0 * w1 * (P(i, j, k) - P(i, j, k + 2)) + u1 * v0 * w1 * (P(i + 1, j, k) - P(i + 1, j, k + 2)) +
                u0 * v1 * w1 * (P(i, j + 1, k) - P(i, j + 1, k + 2)) +
                u1 * v1 * w1 * (P(i + 1, j + 1, k) - P(i + 1, j + 1, k + 2)));
}

// The FP32 push's field: E at every node 0..nx x 0..ny x 0..nz from the
// centred differences of the FP64 phi, rounded to FP32, one float4 a node
// (x, y, z, unused). gather_e's trilinear sum of node differences is the
// trilinear sum of these node fields, so the FP32 advance reads 8 vector
// loads a particle instead of 24 FP64 ones and interpolates in FP32.
// 32 x 8 blocks over (x, y); each thread takes ENODE_Z consecutive z planes
// of its (x, y) column, issuing all of its loads before the first store
// (the column's phi at k-1 .. k+ENODE_Z serves every plane's z difference).
// No index is divided.
constexpr int ENODE_Z = 4;
__global__ void __launch_bounds__(256) k_enode(const double* __restrict__ phi, GridP g, float4* __restrict__ en) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k0 = (int)blockIdx.z * ENODE_Z;
  if (i > g.nx || j > g.ny) return;
  const int sy = g.nx + 3, sz = sy * (g.ny + 3);
  const double* c = phi + ((i + 1) + sy * (j + 1) + (size_t)sz * (k0 + 1));
  const double tdxi = g.tdxi, tdyi = g.tdyi, tdzi = g.tdzi;
  double col[ENODE_Z + 2], xm[ENODE_Z], xp[ENODE_Z], ym[ENODE_Z], yp[ENODE_Z];
  const int nk = min(ENODE_Z, g.nz + 1 - k0);  // planes of this thread (k0 + nk - 1 <= nz)
#pragma unroll
  for (int q = 0; q < ENODE_Z + 2; ++q)
    if (q <= nk + 1) col[q] = __ldg(c + (ptrdiff_t)(q - 1) * sz);  // planes k0-1 .. k0+nk, inside -1..nz+1
#pragma unroll
  for (int q = 0; q < ENODE_Z; ++q)
    if (q < nk) {
      const double* cq = c + (ptrdiff_t)q * sz;
      xm[q] = __ldg(cq - 1);
      xp[q] = __ldg(cq + 1);
      ym[q] = __ldg(cq - sy);
      yp[q] = __ldg(cq + sy);
    }
  const size_t o = (size_t)i + (size_t)(g.nx + 1) * (j + (size_t)(g.ny + 1) * k0);
  const size_t so = (size_t)(g.nx + 1) * (g.ny + 1);
#pragma unroll
  for (int q = 0; q < ENODE_Z; ++q)
    if (q < nk)
      en[o + q * so] = make_float4((float)(tdxi * (xm[q] - xp[q])), (float)(tdyi * (ym[q] - yp[q])),
                                   (float)(tdzi * (col[q] - col[q + 2])), 0.f);
}

// gather_e from the node fields of k_enode, in FP32 (the cell and its
// fractions as gather_e finds them).
__device__ inline void gather_e_nodes(const float4* __restrict__ en, const GridP& g, double x, double y, double z,
                                      float& ext, float& eyt, float& ezt) {
  int i, j, k;
  double u1d, v1d, w1d;
  cellfrac((x - g.xmmin) * g.dxi, g.nx, i, u1d);
  cellfrac((y - g.ymmin) * g.dyi, g.ny, j, v1d);
  cellfrac((z - g.zgrid - g.zmmin) * g.dzi, g.nz, k, w1d);
  const float u1 = (float)u1d, v1 = (float)v1d, w1 = (float)w1d;
  const float u0 = 1.f - u1, v0 = 1.f - v1, w0 = 1.f - w1;
  const int sy = g.nx + 1, sz = sy * (g.ny + 1);
  const float4* b = en + (i + sy * j + (size_t)sz * k);
  const float4 e000 = __ldg(b), e100 = __ldg(b + 1), e010 = __ldg(b + sy), e110 = __ldg(b + sy + 1);
  const float4 e001 = __ldg(b + sz), e101 = __ldg(b + sz + 1), e011 = __ldg(b + sz + sy), e111 = __ldg(b + sz + sy + 1);
  const float a000 = u0 * v0 * w0, a100 = u1 * v0 * w0, a010 = u0 * v1 * w0, a110 = u1 * v1 * w0;
  const float a001 = u0 * v0 * w1, a101 = u1 * v0 * w1, a011 = u0 * v1 * w1, a111 = u1 * v1 * w1;
  // fused multiply-adds written out (this file is compiled without
  // contraction for the FP64 paths' sake)
  ext = __fmaf_rn(a111, e111.x, __fmaf_rn(a011, e011.x, __fmaf_rn(a101, e101.x, __fmaf_rn(a001, e001.x,
        __fmaf_rn(a110, e110.x, __fmaf_rn(a010, e010.x, __fmaf_rn(a100, e100.x, a000 * e000.x)))))));
  eyt = __fmaf_rn(a111, e111.y, __fmaf_rn(a011, e011.y, __fmaf_rn(a101, e101.y, __fmaf_rn(a001, e001.y,
        __fmaf_rn(a110, e110.y, __fmaf_rn(a010, e010.y, __fmaf_rn(a100, e100.y, a000 * e000.y)))))));
  ezt = __fmaf_rn(a111, e111.z, __fmaf_rn(a011, e011.z, __fmaf_rn(a101, e101.z, __fmaf_rn(a001, e001.z,
        __fmaf_rn(a110, e110.z, __fmaf_rn(a010, e010.z, __fmaf_rn(a100, e100.z, a000 * e000.z)))))));
}

// ---- lcorrectede: E next to conductors (sete3dwithconductor) -------------

// Level-0 conductor data read by the corrected gather.
struct CondE {
  const int* icg;   // icgrid over the level-0 nodes
  const double* e0e;  // efield0 of the even subgrid points, 3 per point
  const double* e0o;  // odd
  const double* ede;  // efieldd of the even points, 6 per point
  const double* edo;  // odd
};

// setupconductorfielddata (f3d_mgrid.F:4581-4632): one list into icgrid.
// value 0 writes kIcInterior; +1/-1 write +/-(list index + 1).
__global__ void k_icgrid_fill(const int32_t* __restrict__ ijk, int n, int value, int nx, int ny, int nz,
                              int* __restrict__ icg) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int ix = ijk[3 * t], iy = ijk[3 * t + 1], iz = ijk[3 * t + 2];
  if (ix < 0 || ix > nx || iy < 0 || iy > ny || iz < 0 || iz > nz) return;
  icg[(size_t)ix + (size_t)(nx + 1) * ((size_t)iy + (size_t)(ny + 1) * iz)] = value == 0 ? kIcInterior : value * (t + 1);
}

// getefieldatconductorsubgrid / SETEE (f3d_mgrid.F:4635-4735) at the level-0
// subgrid points of one list: efield0 per axis from the two sides (the
// conductor surface at dels with its volt, or the neighbour node), and
// efieldd towards each neighbour that is an interior node.
__global__ void k_efield_sub(const double* __restrict__ phi, GridP g, const int32_t* __restrict__ ijk,
                             const double* __restrict__ dels, const double* __restrict__ volt, int n,
                             const int* __restrict__ icg, double* __restrict__ e0, double* __restrict__ ed) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int ix = ijk[3 * t], iy = ijk[3 * t + 1], iz = ijk[3 * t + 2];
  if (ix < 0 || ix > g.nx || iy < 0 || iy > g.ny || iz < 0 || iz > g.nz) return;
  const int sy = g.nx + 3, sz = sy * (g.ny + 3);
  const double* p0 = phi + ((ix + 1) + sy * (iy + 1) + sz * (iz + 1));
  const int cy = g.nx + 1, cz = cy * (g.ny + 1);
  const int* c0 = icg + ((size_t)ix + (size_t)cy * iy + (size_t)cz * iz);
  const double ppp = p0[0];
#pragma unroll
  for (int id = 0; id < 3; ++id) {
    const int so = id == 0 ? 1 : id == 1 ? sy : sz;
    const int co = id == 0 ? 1 : id == 1 ? cy : cz;
    const int coord = id == 0 ? ix : id == 1 ? iy : iz;
    const int nmaxc = id == 0 ? g.nx : id == 1 ? g.ny : g.nz;
    const double di = id == 0 ? g.dxi : id == 1 ? g.dyi : g.dzi;
    const double dm = dels[6 * t + 2 * id], dp = dels[6 * t + 2 * id + 1];
    double vv0, dd0, vv1, dd1;
    if (0. < dm && dm <= 1.) {
      vv0 = volt[6 * t + 2 * id];
      dd0 = dm;
    } else {
      vv0 = p0[-so];
      dd0 = 1.;
    }
    if (0. < dp && dp <= 1.) {
      vv1 = volt[6 * t + 2 * id + 1];
      dd1 = dp;
    } else {
      vv1 = p0[so];
      dd1 = 1.;
    }
    e0[3 * t + id] = (dd1 / (dd0 + dd1) * (vv0 - ppp) / dd0 + dd0 / (dd0 + dd1) * (ppp - vv1) / dd1) * di;
    if (coord - 1 >= 0 && c0[-co] == kIcInterior)
      ed[6 * t + 2 * id] = ((vv0 - ppp) / dd0 - (2. - dd0) / (2. + dd1) * (ppp - vv1) / dd1) *
                           ((2. + dd1) / (dd1 + dd0)) * di;
    if (coord + 1 <= nmaxc && c0[co] == kIcInterior)
      ed[6 * t + 2 * id + 1] = ((ppp - vv1) / dd1 - (2. - dd1) / (2. + dd0) * (vv0 - ppp) / dd0) *
                               ((2. + dd0) / (dd0 + dd1)) * di;
  }
}

__device__ __forceinline__ double cond_e0(const CondE& ce, int ic, int id) {
  return ic > 0 ? __ldg(ce.e0e + 3 * (ic - 1) + id) : __ldg(ce.e0o + 3 * (-ic - 1) + id);
}
__device__ __forceinline__ double cond_ed(const CondE& ce, int ic, int k) {
  return ic > 0 ? __ldg(ce.ede + 6 * (ic - 1) + k) : __ldg(ce.edo + 6 * (-ic - 1) + k);
}

// GETEEFROME (f3d_mgrid.F:5160-5220): the cell edge from node a (phi at pa,
// icgrid value ca) to node a+p (icgrid value cb); ps is the phi stride of p.
__device__ __forceinline__ void cond_edge(const double* __restrict__ pa, int ps, int ca, int cb, const CondE& ce,
                                          int id, double di, double wm, double wp, double& ee, double& ww) {
  if (ca == 0) {
    ee = ee + wm * (__ldg(pa - ps) - __ldg(pa + ps)) * 0.5 * di;
    ww = ww + wm;
  } else if (ca != kIcInterior) {
    ee = ee + wm * cond_e0(ce, ca, id);
    ww = ww + wm;
    if (cb == kIcInterior) {
      ee = ee + wp * cond_ed(ce, ca, 2 * id + 1);
      ww = ww + wp;
    }
  }
  if (cb == 0) {
    ee = ee + wp * (__ldg(pa) - __ldg(pa + 2 * ps)) * 0.5 * di;
    ww = ww + wp;
  } else if (cb != kIcInterior) {
    ee = ee + wp * cond_e0(ce, cb, id);
    ww = ww + wp;
    if (ca == kIcInterior) {
      ee = ee + wm * cond_ed(ce, cb, 2 * id);
      ww = ww + wm;
    }
  }
}

// sete3dwithconductor, efetch = 1 (f3d_mgrid.F:4774-5020). Returns false for
// a particle outside the grid, which gets no field. All-vacuum cells use
// centred differences with each term scaled by 1/(2 dx); other cells weight
// the vacuum differences and the conductor points' fields per cell edge,
// normalized by the weights used. A particle on an upper face uses the last
// cell with fraction 1.
__device__ inline bool gather_e_cond(const double* __restrict__ phi, const GridP& g, const CondE& ce, double x,
                                     double y, double z, double& ext, double& eyt, double& ezt) {
  const double tdxi = g.tdxi, tdyi = g.tdyi, tdzi = g.tdzi;
  const double dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
  const double xi = (x - g.xmmin) * dxi, yj = (y - g.ymmin) * dyi, zk = (z - g.zgrid - g.zmmin) * dzi;
  if (xi < 0. || xi > g.nx || yj < 0. || yj > g.ny || zk < 0. || zk > g.nz) return false;
  int i, j, k;
  double u1, v1, w1;
  cellfrac(xi, g.nx, i, u1);
  cellfrac(yj, g.ny, j, v1);
  cellfrac(zk, g.nz, k, w1);
  const double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
  const int sy = g.nx + 3, sz = sy * (g.ny + 3);
  const double* b = phi + ((i + 1) + sy * (j + 1) + sz * (k + 1));
  auto P = [&](int a, int bb, int c) { return __ldg(b + (a + bb * sy + c * sz)); };
  const int cy = g.nx + 1, cz = cy * (g.ny + 1);
  const int* cb = ce.icg + ((size_t)i + (size_t)cy * j + (size_t)cz * k);
  const int c000 = __ldg(cb), c100 = __ldg(cb + 1), c010 = __ldg(cb + cy), c110 = __ldg(cb + 1 + cy);
  const int c001 = __ldg(cb + cz), c101 = __ldg(cb + 1 + cz), c011 = __ldg(cb + cy + cz),
            c111 = __ldg(cb + 1 + cy + cz);
  if ((c000 | c100 | c010 | c110 | c001 | c101 | c011 | c111) == 0) {
    ext = u0 * v0 * w0 * (P(-1, 0, 0) - P(1, 0, 0)) * tdxi + u1 * v0 * w0 * (P(0, 0, 0) - P(2, 0, 0)) * tdxi +
          u0 * v1 * w0 * (P(-1, 1, 0) - P(1, 1, 0)) * tdxi + u1 * v1 * w0 * (P(0, 1, 0) - P(2, 1, 0)) * tdxi +
          u0 * v0 * w1 * (P(-1, 0, 1) - P(1, 0, 1)) * tdxi + u1 * v0 * w1 * (P(0, 0, 1) - P(2, 0, 1)) * tdxi +
          u0 * v1 * w1 * (P(-1, 1, 1) - P(1, 1, 1)) * tdxi + u1 * v1 * w1 * (P(0, 1, 1) - P(2, 1, 1)) * tdxi;
    eyt = u0 * v0 * w0 * (P(0, -1, 0) - P(0, 1, 0)) * tdyi + u1 * v0 * w0 * (P(1, -1, 0) - P(1, 1, 0)) * tdyi +
          u0 * v1 * w0 * (P(0, 0, 0) - P(0, 2, 0)) * tdyi + u1 * v1 * w0 * (P(1, 0, 0) - P(1, 2, 0)) * tdyi +
          u0 * v0 * w1 * (P(0, -1, 1) - P(0, 1, 1)) * tdyi + u1 * v0 * w1 * (P(1, -1, 1) - P(1, 1, 1)) * tdyi +
          u0 * v1 * w1 * (P(0, 0, 1) - P(0, 2, 1)) * tdyi + u1 * v1 * w1 * (P(1, 0, 1) - P(1, 2, 1)) * tdyi;
    ezt = u0 * v0 * w0 * (P(0, 0, -1) - P(0, 0, 1)) * tdzi + u1 * v0 * w0 * (P(1, 0, -1) - P(1, 0, 1)) * tdzi +
          u0 * v1 * w0 * (P(0, 1, -1) - P(0, 1, 1)) * tdzi + u1 * v1 * w0 * (P(1, 1, -1) - P(1, 1, 1)) * tdzi +
          u0 * v0 * w1 * (P(0, 0, 0) - P(0, 0, 2)) * tdzi + u1 * v0 * w1 * (P(1, 0, 0) - P(1, 0, 2)) * tdzi +
          u0 * v1 * w1 * (P(0, 1, 0) - P(0, 1, 2)) * tdzi + u1 * v1 * w1 * (P(1, 1, 0) - P(1, 1, 2)) * tdzi;
    return true;
  }
  double ee = 0., ww = 0.;
  cond_edge(b, 1, c000, c100, ce, 0, dxi, u0 * v0 * w0, u1 * v0 * w0, ee, ww);
  cond_edge(b + sy, 1, c010, c110, ce, 0, dxi, u0 * v1 * w0, u1 * v1 * w0, ee, ww);
  cond_edge(b + sz, 1, c001, c101, ce, 0, dxi, u0 * v0 * w1, u1 * v0 * w1, ee, ww);
  cond_edge(b + sy + sz, 1, c011, c111, ce, 0, dxi, u0 * v1 * w1, u1 * v1 * w1, ee, ww);
  if (ww != 0.) ww = 1. / ww;
  ext = ee * ww;
  ee = 0.;
  ww = 0.;
  cond_edge(b, sy, c000, c010, ce, 1, dyi, u0 * v0 * w0, u0 * v1 * w0, ee, ww);
  cond_edge(b + 1, sy, c100, c110, ce, 1, dyi, u1 * v0 * w0, u1 * v1 * w0, ee, ww);
  cond_edge(b + sz, sy, c001, c011, ce, 1, dyi, u0 * v0 * w1, u0 * v1 * w1, ee, ww);
  cond_edge(b + 1 + sz, sy, c101, c111, ce, 1, dyi, u1 * v0 * w1, u1 * v1 * w1, ee, ww);
  if (ww != 0.) ww = 1. / ww;
  eyt = ee * ww;
  ee = 0.;
  ww = 0.;
  cond_edge(b, sz, c000, c001, ce, 2, dzi, u0 * v0 * w0, u0 * v0 * w1, ee, ww);
  cond_edge(b + 1, sz, c100, c101, ce, 2, dzi, u1 * v0 * w0, u1 * v0 * w1, ee, ww);
  cond_edge(b + sy, sz, c010, c011, ce, 2, dzi, u0 * v1 * w0, u0 * v1 * w1, ee, ww);
  cond_edge(b + 1 + sy, sz, c110, c111, ce, 2, dzi, u1 * v1 * w0, u1 * v1 * w1, ee, ww);
  if (ww != 0.) ww = 1. / ww;
  ezt = ee * ww;
  return true;
}

__global__ void k_fetch_e_cond(const double* __restrict__ phi, GridP g, CondE ce, const double* __restrict__ xp,
                               const double* __restrict__ yp, const double* __restrict__ zp,
                               double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez,
                               int64_t np) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  double a, b, c;
  if (!gather_e_cond(phi, g, ce, xp[i], yp[i], zp[i], a, b, c)) return;
  ex[i] = ex[i] + a;
  ey[i] = ey[i] + b;
  ez[i] = ez[i] + c;
}

__global__ void k_fetch_e(const double* __restrict__ phi, GridP g, const double* __restrict__ xp,
                          const double* __restrict__ yp, const double* __restrict__ zp, double* __restrict__ ex,
                          double* __restrict__ ey, double* __restrict__ ez, int64_t np) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  double a, b, c;
  gather_e(phi, g, xp[i], yp[i], zp[i], a, b, c);
  ex[i] = ex[i] + a;
  ey[i] = ey[i] + b;
  ez[i] = ez[i] + c;
}

struct PushP {
  double q, m, dt;
  double zmmin, zmmax;
  double prwall, prwallx, prwally;
  const double* czs;
  const double* cze;
  const double* cdb;
  int nzl;
  double zlmin, dzl;
  // formed once on the host (set_push_constants), in the expressions and
  // operand order of the push, so with the same bits as per particle:
  // q (dt/2) / m; the Boris factors q dt / 2 / m (fullv) and q (dt/2) / 2 / m
  // (halfv, synchv); 1/dzl; zmmax - zmmin and its inverse; zmmin and zmmax
  // rounded to FP32 towards the inside of the interval
  double cst, cbf, cbh, dzli, syslen, sysleni;
  float zminf, zmaxf;
};

// The FP32 image of a z bound of the periodic wrap, rounded towards the
// inside of [zmmin, zmmax] (a float rounded outward would let a wrapped
// particle sit just past the grid, where its CIC weights leave [0, 1]).
inline float inner_bound_f(double v, bool lower) {
  float f = (float)v;
  if (lower && (double)f < v) f = std::nextafter(f, INFINITY);
  if (!lower && (double)f > v) f = std::nextafter(f, -INFINITY);
  return f;
}

inline void set_push_constants(PushP& P) {
  P.cst = P.q * (0.5 * P.dt) / P.m;
  P.cbf = P.q * P.dt * 0.5 / P.m;
  P.cbh = P.q * (0.5 * P.dt) * 0.5 / P.m;
  P.dzli = 1. / P.dzl;
  P.syslen = P.zmmax - P.zmmin;
  P.sysleni = 1. / (P.zmmax - P.zmmin);
  P.zminf = inner_bound_f(P.zmmin, true);
  P.zmaxf = inner_bound_f(P.zmmax, false);
}

// The deposit of one advanced particle per thread (the CTA's 256 particles)
// into the fixed-point accumulator: the same cells, weights and integer
// sums as k_deposit, so the accumulated charge is the same bit for bit. The
// CTA's particles are consecutive, so when they are sorted by cell they
// cover a small box of nodes: the weights go to a shared-memory copy of the
// box (three 32-bit parts per node, as k_deposit) and the box is added to
// the accumulator at the end; when the box is larger than ADV_BOX nodes
// each lane adds to the accumulator directly. A warp whose 32 particles sit
// in one cell sums them in registers first. All threads of the CTA call it.
// A CTA adds at most 256 particles' weights (each below 2^46 + 1) to a node,
// so the box holds two 32-bit parts per node, bits 0-22 and 23 up: each part
// sums below 2^31, and the two adds per node weight are a third fewer shared
// atomics than k_deposit's three parts.
constexpr int ADV_BOX = 1536;
struct AdvBox {
  unsigned lo[ADV_BOX], hi[ADV_BOX];
};
__device__ inline void adv_add(AdvBox& box, bool use_box, int ox, int oy, int oz, int bx, int by,
                               unsigned long long* acc, const GridP& g, int i, int j, int k, unsigned long long v) {
  if (use_box) {
    const int n = (i - ox) + bx * ((j - oy) + by * (k - oz));
    const unsigned l = (unsigned)(v & 0x7FFFFFull), h = (unsigned)(v >> 23);
    if (l) atomicAdd(&box.lo[n], l);
    if (h) atomicAdd(&box.hi[n], h);
  } else {
    atomicAdd(acc + i + (g.nx + 1) * (j + (g.ny + 1) * k), v);
  }
}
__device__ inline void block_deposit(bool live, double x, double y, double z, const GridP& g,
                                     unsigned long long* __restrict__ acc, AdvBox& box, int* bmin, int* bmax) {
  const int tid = threadIdx.x, lane = tid & 31;
  int ii = 0, jj = 0, kk = 0;
  double u1 = 0., v1 = 0., w1 = 0.;
  if (live) {
    cellfrac((x - g.xmmin) * g.dxi, g.nx, ii, u1);
    cellfrac((y - g.ymmin) * g.dyi, g.ny, jj, v1);
    cellfrac((z - g.zgrid - g.zmmin) * g.dzi, g.nz, kk, w1);
  }
  int lo[3] = {live ? ii : 0x7fffffff, live ? jj : 0x7fffffff, live ? kk : 0x7fffffff};
  int hi[3] = {live ? ii : -1, live ? jj : -1, live ? kk : -1};
  for (int d = 0; d < 3; ++d) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  if (lane == 0 && hi[0] >= 0)
    for (int d = 0; d < 3; ++d) {
      atomicMin(&bmin[d], lo[d]);
      atomicMax(&bmax[d], hi[d]);
    }
  __syncthreads();
  const int ox = bmin[0], oy = bmin[1], oz = bmin[2];
  const int bx = bmax[0] - ox + 2, by = bmax[1] - oy + 2, bz = bmax[2] - oz + 2;
  const bool any = bmax[0] >= 0;
  const bool use_box = any && (long long)bx * by * bz <= ADV_BOX;
  if (use_box)
    for (int n = tid; n < bx * by * bz; n += blockDim.x) {
      box.lo[n] = 0u;
      box.hi[n] = 0u;
    }
  __syncthreads();
  if (any) {
    const double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
    const int key = live ? ii + (g.nx + 1) * (jj + (g.ny + 1) * kk) : -1;
    const int key0 = __shfl_sync(0xffffffffu, key, 0);
    if (__all_sync(0xffffffffu, live && key == key0)) {
      // one cell for the whole warp: lane n < 8 adds the warp's sum of node n
      unsigned long long mine = 0ull;
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        const int dx = n & 1, dy = (n >> 1) & 1, dz = n >> 2;
        const double wgt = (dx ? u1 : u0) * (dy ? v1 : v0) * (dz ? w1 : w0);
        const unsigned long long v = warp_sum_u64((unsigned long long)llrint(wgt * kFixScale));
        if (lane == n) mine = v;
      }
      if (lane < 8 && mine)
        adv_add(box, use_box, ox, oy, oz, bx, by, acc, g, ii + (lane & 1), jj + ((lane >> 1) & 1), kk + (lane >> 2),
                mine);
    } else if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int n = (j + lane) & 7;
        const int dx = n & 1, dy = (n >> 1) & 1, dz = n >> 2;
        const double wgt = (dx ? u1 : u0) * (dy ? v1 : v0) * (dz ? w1 : w0);
        const unsigned long long v = (unsigned long long)llrint(wgt * kFixScale);
        if (v) adv_add(box, use_box, ox, oy, oz, bx, by, acc, g, ii + dx, jj + dy, kk + dz, v);
      }
    }
  }
  if (use_box) {
    __syncthreads();
    for (int n = tid; n < bx * by * bz; n += blockDim.x) {
      const unsigned long long v = ((unsigned long long)box.hi[n] << 23) + box.lo[n];
      if (v) {
        const int lx = n % bx, ly = (n / bx) % by, lz = n / (bx * by);
        atomicAdd(acc + (ox + lx) + (g.nx + 1) * ((oy + ly) + (g.ny + 1) * (oz + lz)), v);
      }
    }
  }
}

// padvnc3d + particleboundaries3d for one particle per thread. CENTER 0 is
// "fullv" (w3d.F:1862-1987): quad window (-dt/2, dt/2), half E kick, full-dt
// Boris rotation, half E kick, drift. CENTER 1 is "halfv" (w3d.F:1989-2125),
// the first step after loading, velocities from t to t+dt/2: window
// (0, dt/2), half-dt rotation, half E kick, drift. CENTER 2 is "synchv"
// (w3d.F:2187-2310), velocities from t-dt/2 to t: window (-dt/2, 0), half E
// kick, half-dt rotation; no drift and no boundaries.
// COND selects the conductor-corrected gather (lcorrectede), which leaves E
// at 0 for a particle outside the grid. Four blocks per SM (64 registers and
// a few spills to L1): the kernel waits on memory, and the extra warps took
// it from 1.97 to 1.83 ms for 5e7 particles on the B200.
// T is the particle storage and push arithmetic: double is the reference's
// arithmetic (bit-identical to the oracle); float is the push of the mixed
// form, whose E is interpolated in FP32 from the FP32 node fields of k_enode
// (with lcorrectede: gathered in FP64 at the FP32 positions and rounded).
// The push constants (q dt / 2m, the lattice tables, the pipe radius) are
// formed in FP64 and rounded once.
// The z bounds of the periodic wrap in the particle type: FP64 as given; in
// FP32 rounded towards the inside of [zmmin, zmmax] (inner_bound_f).
template <typename T>
__device__ __forceinline__ T zbound(const PushP& P, bool lower) {
  if constexpr (sizeof(T) == 8) {
    return lower ? P.zmmin : P.zmmax;
  } else {
    return lower ? P.zminf : P.zmaxf;
  }
}

// One particle of k_advance; returns whether it is live after the advance
// (x, y, z are then its new position).
template <typename T, int CENTER, bool COND>
__device__ __forceinline__ bool advance_one(const double* __restrict__ phi, const float4* __restrict__ en,
                                            const GridP& g, const PushP& P,
                                            const CondE& ce, T* __restrict__ xp, T* __restrict__ yp,
                                            T* __restrict__ zp, T* __restrict__ uxp, T* __restrict__ uyp,
                                            T* __restrict__ uzp, T* __restrict__ gaminv, int64_t i, T& x, T& y,
                                            T& z) {
  T gi = gaminv[i];
  if (gi == (T)0) return false;
  x = xp[i];
  y = yp[i];
  z = zp[i];
  T ux = uxp[i], uy = uyp[i], uz = uzp[i];
  T ex, ey, ez;
  if constexpr (sizeof(T) == 4 && !COND) {
    gather_e_nodes(en, g, (double)x, (double)y, (double)z, ex, ey, ez);
  } else {
    double exd, eyd, ezd;
    if (COND) {
      if (!gather_e_cond(phi, g, ce, (double)x, (double)y, (double)z, exd, eyd, ezd)) exd = eyd = ezd = 0.;
    } else {
      gather_e(phi, g, (double)x, (double)y, (double)z, exd, eyd, ezd);
    }
    ex = (T)exd;
    ey = (T)eyd;
    ez = (T)ezd;
  }
  // fetche3d zeroes E before the gather (w3d.F:11015): E = 0 + gathered
  ex = (T)0 + ex;
  ey = (T)0 + ey;
  ez = (T)0 + ez;
  T bx = 0, by = 0, bz = 0;
  const T dt = (T)P.dt;
  const T halfdt = (T)(0.5 * P.dt), dtl = CENTER == 1 ? (T)0 : -halfdt, dtr = CENTER == 2 ? (T)0 : halfdt;
  if (P.czs) {
    // applyquad (top_lattice.F:2985-3120), one overlap level
    const T vz = uz * gi;
    const T a = vz * (dtr - dtl);
    const T dzi = fabs((T)1 / copysign(fabs(a) + (T)1.0e-36, a));
    int iz = (int)fmax((T)0, (z - (T)P.zlmin) * (T)P.dzli + (T)0.5);
    if (iz > P.nzl) iz = P.nzl;
    const T zs = (T)__ldg(P.czs + iz), ze = (T)__ldg(P.cze + iz);
    const T z1 = z + vz * dtl, z2 = z + vz * dtr;
    const T zl = fmin(z1, z2);
    const T fl = (zl >= zs && zl < ze) ? (T)1 : (T)0;
    const T zr = fmax(z1, z2);
    const T fr = (zr >= zs && zr < ze) ? (T)1 : (T)0;
    T frac = fl;
    if (fl > fr) frac = (ze - zl) * dzi;
    if (fr > fl) frac = (zr - zs) * dzi;
    if (frac > (T)0) {
      const T db = (T)__ldg(P.cdb + iz);
      bx = bx + db * frac * y;
      by = by + db * frac * x;
    }
  }
  // epush3d (half step), bpush3d (ibpush = 1), epush3d (half step)
  const T cst = (T)P.cst;
  if (CENTER != 1) {
    ux = ux + ex * cst;
    uy = uy + ey * cst;
    uz = uz + ez * cst;
  }
  const T cb = (T)(CENTER == 0 ? P.cbf : P.cbh);
  const T tx = gi * bx * cb, ty = gi * by * cb, tz = gi * bz * cb;
  const T tsqi = (T)2 / ((T)1 + tx * tx + ty * ty + tz * tz);
  const T sx = tx * tsqi, sy = ty * tsqi, sz = tz * tsqi;
  const T uxppr = ux + uy * tz - uz * ty;
  const T uyppr = uy + uz * tx - ux * tz;
  const T uzppr = uz + ux * ty - uy * tx;
  ux = ux + uyppr * sz - uzppr * sy;
  uy = uy + uzppr * sx - uxppr * sz;
  uz = uz + uxppr * sy - uyppr * sx;
  if (CENTER == 2) {
    uxp[i] = ux;
    uyp[i] = uy;
    uzp[i] = uz;
    return true;
  }
  ux = ux + ex * cst;
  uy = uy + ey * cst;
  uz = uz + ez * cst;
  // xpush3d
  x = x + ux * gi * dt;
  y = y + uy * gi * dt;
  z = z + uz * gi * dt;
  // periz (top.F:4015-4035)
  const T zmmin = zbound<T>(P, true), zmmax = zbound<T>(P, false);
  const T syslen = (T)P.syslen, sysleni = (T)P.sysleni;
  if (z < zmmin) z = z + syslen * (T)(int)((zmmax - z) * sysleni);
  if (z > zmmax) z = z - syslen * (T)(int)((z - zmmin) * sysleni);
  if constexpr (sizeof(T) == 4) {
    // the FP32 wrap itself rounds: keep z inside [zmmin, zmmax], where the
    // deposit's CIC fractions stay within [0, 1]
    z = fmin(fmax(z, zmmin), zmmax);
  }
  // stckxy3d round aperture
  const T rx = x - (T)P.prwallx, ry = y - (T)P.prwally;
  const T prw = (T)P.prwall;
  const bool lost = rx * rx + ry * ry >= prw * prw;
  if (lost) gaminv[i] = (T)0;
  xp[i] = x;
  yp[i] = y;
  zp[i] = z;
  uxp[i] = ux;
  uyp[i] = uy;
  uzp[i] = uz;
  return !lost;
}

// DEP: the advanced particles' charge is also added to the fixed-point
// accumulator acc (block_deposit), as a deposit after the advance would.
template <typename T, int CENTER, bool COND, bool DEP>
__global__ void __launch_bounds__(256, 4) k_advance(const double* __restrict__ phi, const float4* __restrict__ en,
                                                    GridP g, PushP P, CondE ce,
                                                 T* __restrict__ xp, T* __restrict__ yp, T* __restrict__ zp,
                                                 T* __restrict__ uxp, T* __restrict__ uyp, T* __restrict__ uzp,
                                                 T* __restrict__ gaminv, int64_t np,
                                                 unsigned long long* __restrict__ acc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (!DEP) {
    if (i >= np) return;
    T x, y, z;
    advance_one<T, CENTER, COND>(phi, en, g, P, ce, xp, yp, zp, uxp, uyp, uzp, gaminv, i, x, y, z);
  } else {
    __shared__ AdvBox box;
    __shared__ int bmin[3], bmax[3];
    if (threadIdx.x < 3) {
      bmin[threadIdx.x] = 0x7fffffff;
      bmax[threadIdx.x] = -1;
    }
    __syncthreads();
    T x = 0, y = 0, z = 0;
    const bool live = i < np && advance_one<T, CENTER, COND>(phi, en, g, P, ce, xp, yp, zp, uxp, uyp, uzp, gaminv,
                                                             i, x, y, z);
    block_deposit(live, (double)x, (double)y, (double)z, g, acc, box, bmin, bmax);
  }
}

// Cell key of particlesortxyzwithcopy (top.F:5095-5130):
// ix + (nx+1)*(iy + (ny+1)*iz); lost particles get the key past the last
// node so that a stable sort moves them behind the live ones.
template <typename T>
__global__ void k_cell_keys(const T* __restrict__ xp, const T* __restrict__ yp, const T* __restrict__ zp,
                            const T* __restrict__ gaminv, int64_t np, GridP g, int64_t* __restrict__ key) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  if (gaminv[i] == (T)0) {
    key[i] = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    return;
  }
  int ii, jj, kk;
  double f;
  cellfrac(((double)xp[i] - g.xmmin) * g.dxi, g.nx, ii, f);
  cellfrac(((double)yp[i] - g.ymmin) * g.dyi, g.ny, jj, f);
  cellfrac(((double)zp[i] - g.zgrid - g.zmmin) * g.dzi, g.nz, kk, f);
  key[i] = (int64_t)ii + (int64_t)(g.nx + 1) * ((int64_t)jj + (int64_t)(g.ny + 1) * kk);
}

// dst[k][i] = src[k][perm[i]] for the 7 particle arrays.
template <typename PS>
__global__ void k_permute(const int64_t* __restrict__ perm, int64_t np, PS src, PS dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int64_t j = perm[i];
  dst.x[i] = src.x[j];
  dst.y[i] = src.y[j];
  dst.z[i] = src.z[j];
  dst.ux[i] = src.ux[j];
  dst.uy[i] = src.uy[j];
  dst.uz[i] = src.uz[j];
  dst.gaminv[i] = src.gaminv[j];
}

// ---- z moments (getzmmnt, itask = 2, ifzmmnt = 2) --------------------------

constexpr int kZM = 33;              // moments per sum (the reference's NUMZMMNT)
constexpr int kZMSmemPlanes = 640;   // planes kept in shared memory (168 KB)

struct ZMomP {
  double dt, oneondt, dtscale, zbeam, zmmntmin, zmmntmax, dzm, dzmi, dtmax;
  int nzmmnt;
};

// The 33 moment contributions of one particle state (reference indices
// k+1), non-relativistic branch. For the global sums pass w = 1 and the
// unextrapolated state; vz is the value the velocity ratios divide by.
__device__ __forceinline__ void zm_terms(double qx, double qy, double qz, double px, double py, double pz,
                                         double w, double* m) {
  const double v = 1. / (pz + 1.0e-36);
  m[0] = w;
  m[1] = qx * w;
  m[2] = qy * w;
  m[3] = qz * w;
  m[6] = px * w;
  m[7] = py * w;
  m[8] = pz * w;
  m[9] = qx * qy * w;
  m[11] = qx * qx * w;
  m[12] = qy * qy * w;
  m[13] = qz * qz * w;
  m[16] = px * px * w;
  m[17] = py * py * w;
  m[18] = pz * pz * w;
  m[21] = qz * pz * w;
  m[24] = qx * pz * w;
  m[25] = qy * pz * w;
  m[26] = px * pz * w;
  m[27] = py * pz * w;
  m[4] = px * v * w;
  m[5] = py * v * w;
  m[10] = px * py * (v * v) * w;
  m[14] = (px * v) * (px * v) * w;
  m[15] = (py * v) * (py * v) * w;
  m[19] = qx * px * v * w;
  m[20] = qy * py * v * w;
  m[22] = qx * py * v * w;
  m[23] = qy * px * v * w;
  m[28] = qx * px * w;
  m[29] = qy * py * w;
  m[30] = qx * py * w;
  m[31] = qy * px * w;
  m[32] = px * py * w;
}

__device__ __forceinline__ void zm_add(double* dst, const double* m, bool warp_uniform, bool lead) {
  if (warp_uniform) {
#pragma unroll
    for (int k = 0; k < kZM; ++k) {
      double v = m[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lead) atomicAdd(dst + k, v);
    }
  } else {
#pragma unroll
    for (int k = 0; k < kZM; ++k) atomicAdd(dst + k, m[k]);
  }
}

// Sums over the live particles: the global sums (g, 33) and the two-plane
// extrapolated sums on the z grid (zm, (nzmmnt+1) x 33), accumulated in
// shared memory when the grid fits there, then added to the outputs. The
// floating-point addition order is not fixed, so the sums agree with the
// serial ones to rounding, not bit for bit.
template <typename T>
__global__ void __launch_bounds__(256) k_zmoments(const T* __restrict__ xp, const T* __restrict__ yp,
                                                  const T* __restrict__ zp, const T* __restrict__ uxp,
                                                  const T* __restrict__ uyp, const T* __restrict__ uzp,
                                                  const T* __restrict__ gaminv, const T* __restrict__ uxo,
                                                  const T* __restrict__ uyo, const T* __restrict__ uzo,
                                                  int64_t np, ZMomP P, double* __restrict__ g_out,
                                                  double* __restrict__ zm_out) {
  extern __shared__ double sh[];
  const bool in_smem = P.nzmmnt + 1 <= kZMSmemPlanes;
  double* gs = sh;
  double* zs = in_smem ? sh + kZM : zm_out;
  const int nsh = kZM + (in_smem ? (P.nzmmnt + 1) * kZM : 0);
  for (int i = threadIdx.x; i < nsh; i += blockDim.x) sh[i] = 0.;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (np + stride - 1) / stride;
  for (int64_t r = 0; r < nround; ++r) {
    const int64_t i = r * stride + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < np && gaminv[i] != (T)0;
    double x = 0., y = 0., z = 0., ux = 0., uy = 0., uz = 1., gi = 0.;
    if (live) {
      x = xp[i];
      y = yp[i];
      z = zp[i];
      ux = uxp[i];
      uy = uyp[i];
      uz = uzp[i];
      gi = gaminv[i];
    }
    double m[kZM];
    // global sums: the unextrapolated state, weight 1
    zm_terms(x, y, z, ux, uy, uz, live ? 1. : 0., m);
    const unsigned all = __ballot_sync(0xffffffffu, true);
    zm_add(gs, m, all == 0xffffffffu, lane == 0);
    // z grid
    const double zr = z - P.zbeam;
    const bool in = live && !(zr < P.zmmntmin || zr >= P.zmmntmax);
    int iz = -1;
    if (in) {
      iz = (int)((z - P.zbeam - P.zmmntmin) * P.dzmi);
      if (iz == P.nzmmnt) iz = P.nzmmnt - 1;
    }
    const int iz0 = __shfl_sync(0xffffffffu, iz, 0);
    const bool uniform = __all_sync(0xffffffffu, in && iz == iz0);
    if (!uniform && !in) continue;
    const double vzgi = 1. / (uz * gi + 1.0e-36);
    const double ux_o = in ? (double)uxo[i] : 0., uy_o = in ? (double)uyo[i] : 0., uz_o = in ? (double)uzo[i] : 0.;
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
      double dtx = ((iz + side) * P.dzm - z + P.zbeam + P.zmmntmin) * vzgi;
      dtx = fmax(-P.dtmax * P.dt, fmin(P.dtmax * P.dt, dtx));
      const double px = ux * (1. + dtx * P.oneondt) - ux_o * dtx * P.oneondt;
      const double py = uy * (1. + dtx * P.oneondt) - uy_o * dtx * P.oneondt;
      const double pz = uz * (1. + dtx * P.oneondt) - uz_o * dtx * P.oneondt;
      const double qx = x + ux * dtx * gi, qy = y + uy * dtx * gi, qz = z + uz * dtx * gi;
      const double w = side == 0 ? (1. - (z - P.zbeam - P.zmmntmin) * P.dzmi + iz) * P.dtscale
                                 : ((z - P.zbeam - P.zmmntmin) * P.dzmi - iz) * P.dtscale;
      zm_terms(qx, qy, qz, px, py, pz, w, m);
      zm_add(zs + (size_t)(iz + side) * kZM, m, uniform, lane == 0);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kZM; k += blockDim.x) atomicAdd(g_out + k, gs[k]);
  if (in_smem)
    for (int k = threadIdx.x; k < (P.nzmmnt + 1) * kZM; k += blockDim.x) atomicAdd(zm_out + k, zs[k]);
}

constexpr int kMomN = 11;

// Per-block partial sums of the moments of live particles (getzmmnt,
// top.F:690-721 with x' = ux/(uz+SMALLPOS)); fixed reduction tree per block.
template <typename T>
__global__ void k_moments(const T* __restrict__ xp, const T* __restrict__ yp, const T* __restrict__ uxp,
                          const T* __restrict__ uyp, const T* __restrict__ uzp, const T* __restrict__ gaminv,
                          int64_t np, double* __restrict__ part) {
  __shared__ double sm[kMomN][256];
  double s[kMomN];
#pragma unroll
  for (int k = 0; k < kMomN; ++k) s[k] = 0.;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    if (gaminv[i] == (T)0) continue;
    const double vzi = 1. / ((double)uzp[i] + 1.0e-36);
    const double x = xp[i], y = yp[i], xpr = (double)uxp[i] * vzi, ypr = (double)uyp[i] * vzi;
    s[0] += 1.;
    s[1] += x;
    s[2] += y;
    s[3] += xpr;
    s[4] += ypr;
    s[5] += x * x;
    s[6] += y * y;
    s[7] += xpr * xpr;
    s[8] += ypr * ypr;
    s[9] += x * xpr;
    s[10] += y * ypr;
  }
#pragma unroll
  for (int k = 0; k < kMomN; ++k) sm[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < kMomN; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < kMomN; ++k) part[(size_t)blockIdx.x * kMomN + k] = sm[k][0];
}

__global__ void k_moments_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[kMomN];
  for (int k = 0; k < kMomN; ++k) s[k] = 0.;
  for (int b = 0; b < nb; ++b)
    for (int k = 0; k < kMomN; ++k) s[k] += part[(size_t)b * kMomN + k];
  const double n = s[0] > 0. ? s[0] : 1.;
  const double xb = s[1] / n, yb = s[2] / n, xpb = s[3] / n, ypb = s[4] / n;
  const double dxsq = s[5] / n - xb * xb, dysq = s[6] / n - yb * yb;
  const double dxpsq = s[7] / n - xpb * xpb, dypsq = s[8] / n - ypb * ypb;
  const double dxxp = s[9] / n - xb * xpb, dyyp = s[10] / n - yb * ypb;
  out[0] = s[0];
  out[1] = xb;
  out[2] = yb;
  out[3] = sqrt(fmax(0., dxsq));
  out[4] = sqrt(fmax(0., dysq));
  out[5] = 4. * sqrt(fmax(0., dxsq * dxpsq - dxxp * dxxp));
  out[6] = 4. * sqrt(fmax(0., dysq * dypsq - dyyp * dyyp));
  out[7] = 0.;
}

inline unsigned cdiv64(int64_t a, unsigned b) { return (unsigned)((a + b - 1) / b); }

GridP gridp(const wg_ctx* c) {
  return make_gridp(c->grid.nx, c->grid.ny, c->grid.nz, c->dx, c->dy, c->dz, c->grid.xmmin, c->grid.ymmin,
                    c->grid.zmmin, 0.);
}

// Element type of a particle struct.
template <typename PS>
struct PElem;
template <>
struct PElem<wg_particles> {
  using T = double;
};
template <>
struct PElem<wg_particles_f32> {
  using T = float;
};

}  // namespace

template <typename PS>
int deposit_t(wg_ctx* c, const PS* p, int zero_first) {
  using T = typename PElem<PS>::T;
  if (!p || (p->np > 0 && (!p->x || !p->y || !p->z || !p->gaminv)) || p->np < 0) {
    set_error("wg_deposit: null particle arrays");
    return WG_EINVAL;
  }
  Level& L0 = c->lv[0];
  cudaStream_t s = c->stream;
  { ++c->nlaunch; k_zero_u64<<<(unsigned)std::min<size_t>((L0.nr + 255) / 256, 148 * 16), 256, 0, s>>>(c->racc, L0.nr); }
  { ++c->nlaunch; k_zero_u64<<<1, 32, 0, s>>>(c->dred + 3, 1); }
  GridP g = gridp(c);
  if (p->np > 0) {
    const int64_t maxblocks = 2147483647LL;
    if (cdiv64(p->np, 256) > maxblocks) { set_error("wg_deposit: too many particles"); return WG_ETOOLARGE; }
    { ++c->nlaunch; int pe = c->prof_begin(WG_PROF_DEPOSIT, (double)p->np); k_deposit<T><<<cdiv64(p->np, DEP_NT * DEP_PPT), DEP_NT, 0, s>>>(p->x, p->y, p->z, p->gaminv, p->np, g, c->racc); c->prof_end(pe); }
  }
  double gg = p->w * p->q;
  gg = gg / c->dx;
  gg = gg / c->dy;
  gg = gg / c->dz;
  { ++c->nlaunch; k_fix_to_rho<<<cdiv64((int64_t)L0.nr, 256), 256, 0, s>>>(c->racc, c->rho, L0.nr, gg * kFixInv, zero_first ? 0 : 1,
                                                           c->dred + 3); }
  WG_TRY_CUDA(cudaGetLastError());
  { ++c->nlaunch; k_publish_word<<<1, 1, 0, s>>>(c->dred + 3, c->hred_dev + 3); }
  WG_TRY_CUDA(cudaGetLastError());
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  if (c->hred[3]) {
    set_error("wg_deposit: fixed-point charge accumulator above 2^62 at some node (more than 65536 full "
              "particle weights on one node)");
    return WG_EOVERFLOW;
  }
  return WG_OK;
}

// Chunked deposit: the pieces accumulate in the same fixed-point grid and
// are converted once, so the result is the same as one deposit of all
// pieces, bit for bit. Nothing here synchronizes the stream; an overflow is
// flagged in dred[4] and reported by the next solve.
int deposit_begin(wg_ctx* c) {
  cudaStream_t s = c->stream;
  const size_t nr = c->lv[0].nr;
  { ++c->nlaunch; k_zero_u64<<<(unsigned)std::min<size_t>((nr + 255) / 256, 148 * 16), 256, 0, s>>>(c->racc, nr); }
  { ++c->nlaunch; k_zero_u64<<<1, 32, 0, s>>>(c->dred + 4, 1); }
  WG_TRY_CUDA(cudaGetLastError());
  c->dep_open = true;
  c->dep_gg_set = false;
  c->dep_gg = 0.;
  return WG_OK;
}

template <typename PS>
int deposit_add_t(wg_ctx* c, const PS* p) {
  using T = typename PElem<PS>::T;
  if (!p || (p->np > 0 && (!p->x || !p->y || !p->z || !p->gaminv)) || p->np < 0) {
    set_error("wg_deposit_add: null particle arrays");
    return WG_EINVAL;
  }
  if (!c->dep_open) {
    set_error("wg_deposit_add: no chunked deposit open (wg_deposit_begin)");
    return WG_ESTATE;
  }
  double gg = p->w * p->q;
  gg = gg / c->dx;
  gg = gg / c->dy;
  gg = gg / c->dz;
  if (c->dep_gg_set && gg != c->dep_gg) {
    set_error("wg_deposit_add: the pieces of one deposit must share q and w");
    return WG_EINVAL;
  }
  c->dep_gg = gg;
  c->dep_gg_set = true;
  if (p->np == 0) return WG_OK;
  if (cdiv64(p->np, 256) > 2147483647LL) { set_error("wg_deposit_add: too many particles"); return WG_ETOOLARGE; }
  { ++c->nlaunch; int pe = c->prof_begin(WG_PROF_DEPOSIT, (double)p->np); k_deposit<T><<<cdiv64(p->np, DEP_NT * DEP_PPT), DEP_NT, 0, c->stream>>>(p->x, p->y, p->z, p->gaminv, p->np, gridp(c), c->racc); c->prof_end(pe); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

int deposit_end(wg_ctx* c, int zero_first) {
  if (!c->dep_open) {
    set_error("wg_deposit_end: no chunked deposit open (wg_deposit_begin)");
    return WG_ESTATE;
  }
  c->dep_open = false;
  Level& L0 = c->lv[0];
  { ++c->nlaunch; k_fix_to_rho<<<cdiv64((int64_t)L0.nr, 256), 256, 0, c->stream>>>(c->racc, c->rho, L0.nr, c->dep_gg * kFixInv, zero_first ? 0 : 1, c->dred + 4); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

int finalize_rho(wg_ctx* c) {
  const wg_grid& G = c->grid;
  cudaStream_t s = c->stream;
  const int* b = G.bounds;
  size_t nyz = (size_t)(G.ny + 1) * (G.nz + 1), nxz = (size_t)(G.nx + 1) * (G.nz + 1),
         nxy = (size_t)(G.nx + 1) * (G.ny + 1);
  if (b[0] >= 1 || b[1] >= 1) { ++c->nlaunch; k_rhobc<<<cdiv64((int64_t)nyz, 256), 256, 0, s>>>(c->rho, G.nx, G.ny, G.nz, 0, b[0], b[1]); }
  if (b[2] >= 1 || b[3] >= 1) { ++c->nlaunch; k_rhobc<<<cdiv64((int64_t)nxz, 256), 256, 0, s>>>(c->rho, G.nx, G.ny, G.nz, 1, b[2], b[3]); }
  if (b[4] >= 1 || b[5] >= 1) { ++c->nlaunch; k_rhobc<<<cdiv64((int64_t)nxy, 256), 256, 0, s>>>(c->rho, G.nx, G.ny, G.nz, 2, b[4], b[5]); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

// lcorrectede setup before a corrected gather: rebuilds icgrid and the
// per-point field arrays when the conductors changed, then recomputes
// efield0/efieldd from the current phi (the reference does this after every
// solve, multigrid.py:602-616). Nothing is computed unless both subgrid
// lists (all levels) are non-empty, as in getefieldatconductorsubgrid; the
// fields then stay 0.
int prepare_correctede(wg_ctx* c, CondE* ce) {
  Level& L = c->lv[0];
  const LevelDims& d = L.d;
  cudaStream_t s = c->stream;
  const size_t nodes = (size_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  if (c->icgrid_version != c->cond_version || !c->icgrid) {
    if (!c->icgrid) WG_TRY_CUDA(cudaMalloc((void**)&c->icgrid, nodes * sizeof(int)));
    for (int p = 0; p < 2; ++p) {
      if (c->ef0[p]) cudaFree(c->ef0[p]);
      if (c->efd[p]) cudaFree(c->efd[p]);
      c->ef0[p] = c->efd[p] = nullptr;
      const size_t n = (size_t)L.sub[p].n;
      if (n) {
        WG_TRY_CUDA(cudaMalloc((void**)&c->ef0[p], 3 * n * sizeof(double)));
        WG_TRY_CUDA(cudaMalloc((void**)&c->efd[p], 6 * n * sizeof(double)));
        WG_TRY_CUDA(cudaMemsetAsync(c->ef0[p], 0, 3 * n * sizeof(double), s));
        WG_TRY_CUDA(cudaMemsetAsync(c->efd[p], 0, 6 * n * sizeof(double), s));
      }
    }
    WG_TRY_CUDA(cudaMemsetAsync(c->icgrid, 0, nodes * sizeof(int), s));
    if (L.n_int) { ++c->nlaunch; k_icgrid_fill<<<(L.n_int + 255) / 256, 256, 0, s>>>(L.int_ijk, L.n_int, 0, d.nx, d.ny, d.nz, c->icgrid); }
    if (L.sub[0].n) { ++c->nlaunch; k_icgrid_fill<<<(L.sub[0].n + 255) / 256, 256, 0, s>>>(L.sub[0].ijk, L.sub[0].n, 1, d.nx, d.ny, d.nz, c->icgrid); }
    if (L.sub[1].n) { ++c->nlaunch; k_icgrid_fill<<<(L.sub[1].n + 255) / 256, 256, 0, s>>>(L.sub[1].ijk, L.sub[1].n, -1, d.nx, d.ny, d.nz, c->icgrid); }
    WG_TRY_CUDA(cudaGetLastError());
    c->icgrid_version = c->cond_version;
  }
  if (!c->cond.even_indx.empty() && !c->cond.odd_indx.empty()) {
    for (int p = 0; p < 2; ++p) {
      const DevSubgrid& S = L.sub[p];
      if (!S.n) continue;
      { ++c->nlaunch; k_efield_sub<<<(S.n + 255) / 256, 256, 0, s>>>(L.phi, gridp(c), S.ijk, S.dels, S.volt, S.n, c->icgrid, c->ef0[p], c->efd[p]); }
    }
    WG_TRY_CUDA(cudaGetLastError());
  }
  ce->icg = c->icgrid;
  ce->e0e = c->ef0[0];
  ce->e0o = c->ef0[1];
  ce->ede = c->efd[0];
  ce->edo = c->efd[1];
  return WG_OK;
}

int fetch_e(wg_ctx* c, const double* x, const double* y, const double* z, double* ex, double* ey, double* ez,
            int64_t np) {
  if (np < 0 || (np > 0 && (!x || !y || !z || !ex || !ey || !ez))) {
    set_error("wg_fetch_e: null arrays");
    return WG_EINVAL;
  }
  if (np == 0) return WG_OK;
  if (c->correctede) {
    CondE ce{};
    WG_TRY(prepare_correctede(c, &ce));
    { ++c->nlaunch; k_fetch_e_cond<<<cdiv64(np, 256), 256, 0, c->stream>>>(c->lv[0].phi, gridp(c), ce, x, y, z, ex, ey, ez, np); }
    WG_TRY_CUDA(cudaGetLastError());
    return WG_OK;
  }
  { ++c->nlaunch; k_fetch_e<<<cdiv64(np, 256), 256, 0, c->stream>>>(c->lv[0].phi, gridp(c), x, y, z, ex, ey, ez, np); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

// deposit: also accumulate the advanced particles' charge into the open
// chunked deposit (wg_deposit_begin .. wg_deposit_end), as wg_deposit_add
// of the same particles after the advance would.
template <typename PS>
int advance_t(wg_ctx* c, const PS* p, const wg_push_params* prm, bool deposit = false) {
  using T = typename PElem<PS>::T;
  if (!p || !prm || p->np < 0 ||
      (p->np > 0 && (!p->x || !p->y || !p->z || !p->ux || !p->uy || !p->uz || !p->gaminv))) {
    set_error("wg_advance: null arguments");
    return WG_EINVAL;
  }
  if (prm->use_lattice && c->nzl < 0) {
    set_error("wg_advance: use_lattice set but no lattice installed (wg_set_lattice)");
    return WG_ESTATE;
  }
  if (prm->center != WG_CENTER_FULLV && prm->center != WG_CENTER_HALFV && prm->center != WG_CENTER_SYNCHV) {
    set_error("wg_advance: center must be WG_CENTER_FULLV, WG_CENTER_HALFV or WG_CENTER_SYNCHV");
    return WG_EINVAL;
  }
  if (deposit) {
    if (!c->dep_open) {
      set_error("wg_advance_deposit: no chunked deposit open (wg_deposit_begin)");
      return WG_ESTATE;
    }
    double gg = p->w * p->q;
    gg = gg / c->dx;
    gg = gg / c->dy;
    gg = gg / c->dz;
    if (c->dep_gg_set && gg != c->dep_gg) {
      set_error("wg_advance_deposit: the pieces of one deposit must share q and w");
      return WG_EINVAL;
    }
    c->dep_gg = gg;
    c->dep_gg_set = true;
  }
  if (p->np == 0) return WG_OK;
  if (cdiv64(p->np, 256) > 2147483647LL) { set_error("wg_advance: too many particles"); return WG_ETOOLARGE; }
  PushP P{p->q, p->m, prm->dt, c->grid.zmmin, c->grid.zmmax, prm->prwall, prm->prwallx, prm->prwally,
          prm->use_lattice ? c->czs : nullptr, c->cze, c->cdb, c->nzl, c->zlmin, c->dzl};
  set_push_constants(P);
  CondE ce{};
  if (c->correctede) WG_TRY(prepare_correctede(c, &ce));
  // the FP32 push without lcorrectede gathers from node fields formed from
  // phi on every call (k_enode)
  const bool nodes = sizeof(T) == 4 && !c->correctede;
  const size_t nn = (size_t)(c->grid.nx + 1) * (c->grid.ny + 1) * (c->grid.nz + 1);
  if (nodes && (c->grid.nz + 1 + ENODE_Z - 1) / ENODE_Z > 65535) {
    set_error("wg_advance_f32: nz too large for the node-field launch (65535 slices of 4 planes)");
    return WG_ETOOLARGE;
  }
  if (nodes && c->enode_n < nn) {
    if (c->enode) cudaFree(c->enode);
    c->enode = nullptr;
    c->enode_n = 0;
    cudaError_t e = cudaMalloc((void**)&c->enode, nn * sizeof(float4));
    if (e != cudaSuccess) {
      c->enode = nullptr;
      set_error(std::string("wg_advance: cudaMalloc of the node fields failed: ") + cudaGetErrorString(e));
      return WG_ENOMEM;
    }
    c->enode_n = nn;
  }
  using K = void (*)(const double*, const float4*, GridP, PushP, CondE, T*, T*, T*, T*, T*, T*, T*, int64_t,
                     unsigned long long*);
  // [correctede][deposit][center]
  static const K kerns[2][2][3] = {
      {{k_advance<T, 0, false, false>, k_advance<T, 1, false, false>, k_advance<T, 2, false, false>},
       {k_advance<T, 0, false, true>, k_advance<T, 1, false, true>, k_advance<T, 2, false, true>}},
      {{k_advance<T, 0, true, false>, k_advance<T, 1, true, false>, k_advance<T, 2, true, false>},
       {k_advance<T, 0, true, true>, k_advance<T, 1, true, true>, k_advance<T, 2, true, true>}}};
  const K kern = kerns[c->correctede ? 1 : 0][deposit ? 1 : 0][prm->center];
  {
    int pe = c->prof_begin(WG_PROF_ADVANCE, (double)p->np);
    if (nodes) {
      ++c->nlaunch;
      const dim3 eg((unsigned)((c->grid.nx + 1 + 31) / 32), (unsigned)((c->grid.ny + 1 + 7) / 8),
                    (unsigned)((c->grid.nz + 1 + ENODE_Z - 1) / ENODE_Z));
      k_enode<<<eg, dim3(32, 8), 0, c->stream>>>(c->lv[0].phi, gridp(c), c->enode);
    }
    ++c->nlaunch;
    kern<<<cdiv64(p->np, 256), 256, 0, c->stream>>>(c->lv[0].phi, nodes ? c->enode : nullptr, gridp(c), P, ce, p->x,
                                                   p->y, p->z, p->ux, p->uy, p->uz, p->gaminv, p->np,
                                                   deposit ? c->racc : nullptr);
    c->prof_end(pe);
  }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

template <typename PS, typename T = typename PElem<PS>::T>
int zmoments_t(wg_ctx* c, const PS* p, const T* uxo, const T* uyo, const T* uzo, double dt, double dtscale,
               double zbeam, double zmmntmin, double zmmntmax, int nzmmnt, double zmmntdtextmax, double* zmmnts0,
               double* zmmnts) {
  if (!p || p->np < 0 || !zmmnts0 || !zmmnts ||
      (p->np > 0 && (!p->x || !p->y || !p->z || !p->ux || !p->uy || !p->uz || !p->gaminv || !uxo || !uyo || !uzo))) {
    set_error("wg_zmoments: null arguments");
    return WG_EINVAL;
  }
  if (nzmmnt < 1 || !(zmmntmax > zmmntmin) || !(dt > 0.)) {
    set_error("wg_zmoments: need nzmmnt >= 1, zmmntmax > zmmntmin and dt > 0");
    return WG_EINVAL;
  }
  const size_t n = (size_t)(nzmmnt + 2) * kZM;
  if (c->zmom_n < n) {
    if (c->zmom) cudaFree(c->zmom);
    c->zmom = nullptr;
    c->zmom_n = 0;
    WG_TRY_CUDA(cudaMalloc((void**)&c->zmom, n * sizeof(double)));
    c->zmom_n = n;
  }
  cudaStream_t s = c->stream;
  WG_TRY_CUDA(cudaMemsetAsync(c->zmom, 0, n * sizeof(double), s));
  ZMomP P;
  P.dt = dt;
  P.oneondt = 1. / dt;
  P.dtscale = dtscale;
  P.zbeam = zbeam;
  P.zmmntmin = zmmntmin;
  P.zmmntmax = zmmntmax;
  P.dzm = (zmmntmax - zmmntmin) / nzmmnt;
  P.dzmi = 1. / P.dzm;
  P.dtmax = zmmntdtextmax;
  P.nzmmnt = nzmmnt;
  if (p->np > 0) {
    const bool in_smem = nzmmnt + 1 <= kZMSmemPlanes;
    const size_t smem = (size_t)(kZM + (in_smem ? (nzmmnt + 1) * kZM : 0)) * sizeof(double);
    WG_TRY_CUDA(cudaFuncSetAttribute(k_zmoments<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = in_smem ? 148u : 592u;
    { ++c->nlaunch; k_zmoments<T><<<blocks, 256, smem, s>>>(p->x, p->y, p->z, p->ux, p->uy, p->uz, p->gaminv, uxo, uyo, uzo, p->np, P, c->zmom, c->zmom + kZM); }
    WG_TRY_CUDA(cudaGetLastError());
  }
  WG_TRY_CUDA(cudaMemcpyAsync(zmmnts0, c->zmom, kZM * sizeof(double), cudaMemcpyDeviceToHost, s));
  WG_TRY_CUDA(cudaMemcpyAsync(zmmnts, c->zmom + kZM, (size_t)(nzmmnt + 1) * kZM * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  return WG_OK;
}

template <typename PS>
int moments_t(wg_ctx* c, const PS* p, double* out) {
  using T = typename PElem<PS>::T;
  if (!p || !out || p->np < 0) { set_error("wg_moments: null arguments"); return WG_EINVAL; }
  cudaStream_t s = c->stream;
  const int nb = c->mom_blocks;
  { ++c->nlaunch; k_moments<T><<<nb, 256, 0, s>>>(p->x, p->y, p->ux, p->uy, p->uz, p->gaminv, p->np, c->dmom); }
  { ++c->nlaunch; k_moments_final<<<1, 32, 0, s>>>(c->dmom, nb, c->dmom + (size_t)nb * kMomN); }
  WG_TRY_CUDA(cudaGetLastError());
  WG_TRY_CUDA(cudaMemcpyAsync(out, c->dmom + (size_t)nb * kMomN, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  return WG_OK;
}

int moments_scratch_doubles(int nb) { return nb * kMomN + 8; }

template <typename PS>
int cell_keys_t(wg_ctx* c, const PS* p, int64_t* keys) {
  using T = typename PElem<PS>::T;
  if (!p || !keys || p->np < 0) { set_error("wg_particle_keys: null arguments"); return WG_EINVAL; }
  if (p->np == 0) return WG_OK;
  { ++c->nlaunch; k_cell_keys<T><<<cdiv64(p->np, 256), 256, 0, c->stream>>>(p->x, p->y, p->z, p->gaminv, p->np, gridp(c), keys); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

template <typename PS>
int permute_t(wg_ctx* c, const int64_t* perm, const PS* src, const PS* dst) {
  if (!perm || !src || !dst || src->np != dst->np || src->np < 0) {
    set_error("wg_particle_permute: bad arguments");
    return WG_EINVAL;
  }
  if (src->np == 0) return WG_OK;
  { ++c->nlaunch; k_permute<PS><<<cdiv64(src->np, 256), 256, 0, c->stream>>>(perm, src->np, *src, *dst); }
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

int deposit(wg_ctx* c, const wg_particles* p, int zero_first) { return deposit_t(c, p, zero_first); }
int deposit_f32(wg_ctx* c, const wg_particles_f32* p, int zero_first) { return deposit_t(c, p, zero_first); }
int deposit_add(wg_ctx* c, const wg_particles* p) { return deposit_add_t(c, p); }
int deposit_add_f32(wg_ctx* c, const wg_particles_f32* p) { return deposit_add_t(c, p); }
int advance(wg_ctx* c, const wg_particles* p, const wg_push_params* prm) { return advance_t(c, p, prm); }
int advance_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm) { return advance_t(c, p, prm); }
int advance_deposit(wg_ctx* c, const wg_particles* p, const wg_push_params* prm) {
  return advance_t(c, p, prm, true);
}
int advance_deposit_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm) {
  return advance_t(c, p, prm, true);
}
int moments(wg_ctx* c, const wg_particles* p, double* out) { return moments_t(c, p, out); }
int moments_f32(wg_ctx* c, const wg_particles_f32* p, double* out) { return moments_t(c, p, out); }
int zmoments(wg_ctx* c, const wg_particles* p, const double* uxo, const double* uyo, const double* uzo, double dt,
             double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt, double zmmntdtextmax,
             double* zmmnts0, double* zmmnts) {
  return zmoments_t(c, p, uxo, uyo, uzo, dt, dtscale, zbeam, zmmntmin, zmmntmax, nzmmnt, zmmntdtextmax, zmmnts0,
                    zmmnts);
}
int zmoments_f32(wg_ctx* c, const wg_particles_f32* p, const float* uxo, const float* uyo, const float* uzo,
                 double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt,
                 double zmmntdtextmax, double* zmmnts0, double* zmmnts) {
  return zmoments_t(c, p, uxo, uyo, uzo, dt, dtscale, zbeam, zmmntmin, zmmntmax, nzmmnt, zmmntdtextmax, zmmnts0,
                    zmmnts);
}
int cell_keys(wg_ctx* c, const wg_particles* p, int64_t* keys) { return cell_keys_t(c, p, keys); }
int cell_keys_f32(wg_ctx* c, const wg_particles_f32* p, int64_t* keys) { return cell_keys_t(c, p, keys); }
int permute(wg_ctx* c, const int64_t* perm, const wg_particles* src, const wg_particles* dst) {
  return permute_t(c, perm, src, dst);
}
int permute_f32(wg_ctx* c, const int64_t* perm, const wg_particles_f32* src, const wg_particles_f32* dst) {
  return permute_t(c, perm, src, dst);
}

// ---- deposition into caller memory with no allocation ----------------------
//
// For callers that own every device buffer and cannot let a library allocate:
// a host code with its own device memory manager, or one that keeps a step
// free of cudaMalloc/cudaFree because those calls synchronize the device and
// would stall its other streams. The fixed-point accumulator lives in a
// file-scope device array instead of a context, so this path needs neither
// wg_create nor any allocation. Two calls that overlap on one device (other
// streams or host threads) share that array and race.

namespace {

constexpr int64_t kNoAllocMaxNodes = 1 << 20;  // (nx+1)(ny+1)(nz+1) limit: 8 MiB of accumulator
constexpr int kNoAllocMaxDevices = 64;

// accumulator nodes [0, kNoAllocMaxNodes), then the overflow flag
static __device__ __align__(256) unsigned long long g_noalloc_acc[kNoAllocMaxNodes + 32];

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kNoAllocMaxDevices] = {};

}  // namespace

int deposit_noalloc(const wg_grid* grid, const wg_particles* p, double* rho, int zero_first, void* stream) {
  if (!grid || !p || !rho) { set_error("wg_deposit_noalloc: null argument"); return WG_EINVAL; }
  const wg_grid& G = *grid;
  if (G.nx < 1 || G.ny < 1 || G.nz < 1 || !(G.xmmax > G.xmmin) || !(G.ymmax > G.ymmin) || !(G.zmmax > G.zmmin)) {
    set_error("wg_deposit_noalloc: need nx, ny, nz >= 1 and increasing mesh extents");
    return WG_EINVAL;
  }
  if (p->np < 0 || (p->np > 0 && (!p->x || !p->y || !p->z || !p->gaminv))) {
    set_error("wg_deposit_noalloc: null particle arrays");
    return WG_EINVAL;
  }
  const int64_t nr = (int64_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
  if (nr > kNoAllocMaxNodes) {
    set_error("wg_deposit_noalloc: grid has " + std::to_string(nr) + " nodes, above the fixed limit of " +
              std::to_string(kNoAllocMaxNodes) + " nodes ((nx+1)(ny+1)(nz+1)); use wg_deposit for larger grids");
    return WG_ETOOLARGE;
  }
  if (cdiv64(p->np, DEP_NT * DEP_PPT) > 2147483647LL) {
    set_error("wg_deposit_noalloc: too many particles");
    return WG_ETOOLARGE;
  }
  int dev = 0;
  WG_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("wg_deposit_noalloc: device ordinal above " + std::to_string(kNoAllocMaxDevices - 1));
    return WG_EINVAL;
  }
  unsigned long long* acc;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* a = nullptr;
      WG_TRY_CUDA(cudaGetSymbolAddress(&a, g_noalloc_acc));
      g_noalloc_ptr[dev] = static_cast<unsigned long long*>(a);
    }
    acc = g_noalloc_ptr[dev];
  }
  unsigned long long* flag = acc + kNoAllocMaxNodes;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // zeroed by kernels, as in wg_deposit: a cudaMemsetAsync may wait behind a
  // caller's bulk copies on a copy engine
  k_zero_u64<<<(unsigned)std::min<int64_t>((nr + 255) / 256, 148 * 16), 256, 0, s>>>(acc, (size_t)nr);
  k_zero_u64<<<1, 32, 0, s>>>(flag, 1);
  const double dx = (G.xmmax - G.xmmin) / G.nx, dy = (G.ymmax - G.ymmin) / G.ny, dz = (G.zmmax - G.zmmin) / G.nz;
  GridP g = make_gridp(G.nx, G.ny, G.nz, dx, dy, dz, G.xmmin, G.ymmin, G.zmmin, 0.);
  if (p->np > 0) k_deposit<double><<<cdiv64(p->np, DEP_NT * DEP_PPT), DEP_NT, 0, s>>>(p->x, p->y, p->z, p->gaminv, p->np, g, acc);
  double gg = p->w * p->q;
  gg = gg / dx;
  gg = gg / dy;
  gg = gg / dz;
  k_fix_to_rho<<<cdiv64(nr, 256), 256, 0, s>>>(acc, rho, (size_t)nr, gg * kFixInv, zero_first ? 0 : 1, flag);
  WG_TRY_CUDA(cudaGetLastError());
  unsigned long long hflag = 0;
  WG_TRY_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(hflag), cudaMemcpyDeviceToHost, s));
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  if (hflag) {
    set_error("wg_deposit_noalloc: fixed-point charge accumulator above 2^62 at some node (more than 65536 full "
              "particle weights on one node)");
    return WG_EOVERFLOW;
  }
  return WG_OK;
}

}  // namespace wg
