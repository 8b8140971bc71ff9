// Multigrid Poisson solver with subgrid conductors on one B200.
//
// Device kernels for the phases of multigrid3dsolve (pywarp90/f3d_mgrid.F:83-500):
// red-black SOR, subgrid conductor stencil, residual, restriction,
// prolongation and guard-plane boundary conditions, for FP64 and FP32 levels,
// plus the host-side V-cycle driver. This translation unit is compiled with
// --fmad=false and evaluates every expression in the reference's operand
// order, so with identical inputs the FP64 path reproduces the CPU oracle
// bit for bit.
//
// Layout: each level keeps phi and res as (nx+3)(ny+3)(nz+3) arrays with one
// guard cell and rhs as (nx+1)(ny+1)(nz+1), x fastest (the reference's
// Fortran layout), so the user-visible solver.phi needs no repacking.
//
// Conductor nodes are marked inside the rhs arrays: at an interior or
// subgrid node rhs holds a NaN whose payload is the node's index in its list
// (sign bit set for interior points) and the real rhs value is kept in the
// list record. A sweep therefore reads exactly phi and rhs per node and
// finds the conductor nodes without a separate tag array.
//
// sorpass3d is one kernel per colour (k_sor_bulk). With Dirichlet x and y,
// Dirichlet or periodic z and no Neumann-type conductor surface point, that
// kernel also updates the colour's subgrid points and writes the periodic
// images, so a half sweep is one launch; otherwise the subgrid and boundary
// kernels follow it.

#include <cmath>
#include <cstdio>
#include <cstring>

#include "wg_internal.h"

namespace wg {

namespace {

constexpr double kEps0 = 1. / (4. * 3.14159265358979323 * 1.e-7 * 2.99792458e+8 * 2.99792458e+8);

struct Bnd {
  int b[6];
};

__host__ __device__ inline size_t pix(int nx, int ny, int ix, int iy, int iz) {
  return (size_t)(ix + 1) + (size_t)(nx + 3) * ((size_t)(iy + 1) + (size_t)(ny + 3) * (size_t)(iz + 1));
}
__host__ __device__ inline size_t rix(int nx, int ny, int ix, int iy, int iz) {
  return (size_t)ix + (size_t)(nx + 1) * ((size_t)iy + (size_t)(ny + 1) * (size_t)iz);
}

// NaN boxes marking conductor nodes in rhs arrays.
template <typename T>
struct Box;
template <>
struct Box<double> {
  // the index takes the low 32 bits of the payload: any int count fits
  __device__ static double make(bool interior, uint32_t idx) {
    return __longlong_as_double((long long)(0x7FF8000000000000ull | (interior ? 0x8000000000000000ull : 0ull) |
                                            (unsigned long long)idx));
  }
  __device__ static uint32_t idx(double v) { return (uint32_t)((unsigned long long)__double_as_longlong(v)); }
  __device__ static bool interior(double v) { return __double_as_longlong(v) < 0; }
};
template <>
struct Box<float> {
  static constexpr uint32_t kMax = 0x3FFFFFu;
  __device__ static float make(bool interior, uint32_t idx) {
    return __uint_as_float(0x7FC00000u | (interior ? 0x80000000u : 0u) | (idx & 0x3FFFFFu));
  }
  __device__ static uint32_t idx(float v) { return __float_as_uint(v) & 0x3FFFFFu; }
  __device__ static bool interior(float v) { return __float_as_int(v) < 0; }
};
// z planes per thread of the bulk stencil kernels
template <typename T>
struct ZPlanes;
template <>
struct ZPlanes<double> {
  static constexpr int value = 2;
};
template <>
struct ZPlanes<float> {
  static constexpr int value = 4;
};

template <typename T>
__device__ inline bool isbox(T v) {
  return v != v;
}

__device__ inline void atomic_max_nonneg(unsigned long long* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}
__device__ inline double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Max reductions land in one of kRedSlots slots, kRedStride words apart
// (separate cache lines), so that the blocks of a large grid do not all
// serialise on one address; k_fold_max combines the slots.
constexpr int kRedSlots = 32, kRedStride = 16, kRedQ = kRedSlots * kRedStride;

// Block-wide max folded into the slot of this block under `base` (all
// threads must call). The atomic is skipped when the slot already holds a
// larger value.
__device__ inline void block_max_to(unsigned long long* base, double v) {
  __shared__ double sm[32];
  v = warp_max(v);
  int lane = threadIdx.x & 31, wid = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  int nw = (blockDim.x * blockDim.y + 31) >> 5;
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double w = (lane < nw) ? sm[lane] : 0.;
    w = warp_max(w);
    if (lane == 0 && w > 0.) {
      const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
      unsigned long long* addr = base + kRedStride * (bid % kRedSlots);
      const unsigned long long bits = (unsigned long long)__double_as_longlong(w);
      if (bits > *(volatile unsigned long long*)addr) atomic_max_nonneg(addr, w);
    }
  }
}

// out[q] = max over the slots of reduction q (q < nq).
// Programmatic dependent launch: wait until the grid this one depends on
// has finished and its writes are visible, then let the next grid of the
// stream be scheduled, so that its launch overlaps this grid's run. Both are
// no-ops for a grid launched without the attribute.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Reduction words into the mapped host copy (read after a stream sync).
__global__ void k_publish(const unsigned long long* __restrict__ src, unsigned long long* dst, int n) {
  pdl_entry();
  if ((int)threadIdx.x < n) ((volatile unsigned long long*)dst)[threadIdx.x] = src[threadIdx.x];
  __threadfence_system();
}

template <typename T>
__global__ void k_copy(const T* __restrict__ a, T* __restrict__ b, size_t n) {
  pdl_entry();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = a[i];
}

template <typename T>
__global__ void k_zero(T* __restrict__ u, size_t n) {
  pdl_entry();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) u[i] = (T)0.;
}

__global__ void k_fold_max(const unsigned long long* __restrict__ slots, unsigned long long* __restrict__ out,
                           int nq) {
  pdl_entry();
  const int q = threadIdx.x / 32, lane = threadIdx.x & 31;
  if (q >= nq) return;
  unsigned long long v = slots[q * kRedQ + kRedStride * lane];
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
    v = t > v ? t : v;
  }
  if (lane == 0) out[q] = v;
}

// ---------------------------------------------------------------------------
// applyboundaryconditions3d (f3d_mgrid.F:3847-3955), ncomp = 1, one guard.
// The x phase, then the y phase over all x (guards included), then the z
// phase over all x and y, exactly as the reference orders them.
template <typename T>
__global__ void k_bc_xy(T* __restrict__ u, int nx, int ny, Bnd B, int lwithdirichlet) {
  pdl_entry();
  const int iz = blockIdx.x;
  const size_t sy = nx + 3;
  const size_t base = (size_t)(ny + 3) * sy * (size_t)(iz + 1);
  for (int iy = threadIdx.x; iy <= ny; iy += blockDim.x) {
    T* r = u + base + sy * (iy + 1) + 1;  // r[ix] = u(ix,iy,iz)
    if (lwithdirichlet) {
      if (B.b[0] == 0) r[-1] = (T)2. * r[0] - r[1];
      if (B.b[1] == 0) r[nx + 1] = (T)2. * r[nx] - r[nx - 1];
    }
    if (B.b[0] == 1) r[-1] = r[1];
    if (B.b[1] == 1) r[nx + 1] = r[nx - 1];
    if (B.b[0] == 2 && B.b[1] == 2) {
      r[-1] = r[nx - 1];
      r[nx] = r[0];
      r[nx + 1] = r[1];
    }
  }
  __syncthreads();
  for (int ix = -1 + (int)threadIdx.x; ix <= nx + 1; ix += blockDim.x) {
    T* c = u + base + (ix + 1) + sy;  // c[iy*sy] = u(ix,iy,iz)
    auto C = [&](int iy) -> T& { return c[(ptrdiff_t)iy * (ptrdiff_t)sy]; };
    if (lwithdirichlet) {
      if (B.b[2] == 0) C(-1) = (T)2. * C(0) - C(1);
      if (B.b[3] == 0) C(ny + 1) = (T)2. * C(ny) - C(ny - 1);
    }
    if (B.b[2] == 1) C(-1) = C(1);
    if (B.b[3] == 1) C(ny + 1) = C(ny - 1);
    if (B.b[2] == 2 && B.b[3] == 2) {
      C(-1) = C(ny - 1);
      C(ny) = C(0);
      C(ny + 1) = C(1);
    }
  }
}

template <typename T>
__global__ void k_bc_z(T* __restrict__ u, int nx, int ny, int nz, Bnd B, int lwithdirichlet) {
  pdl_entry();
  const size_t nxy = (size_t)(nx + 3) * (ny + 3);
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxy) return;
  T* c = u + t + nxy;  // c[iz*nxy] = u(.,.,iz)
  auto C = [&](int iz) -> T& { return c[(ptrdiff_t)iz * (ptrdiff_t)nxy]; };
  if (lwithdirichlet) {
    if (B.b[4] == 0) C(-1) = (T)2. * C(0) - C(1);
    if (B.b[5] == 0) C(nz + 1) = (T)2. * C(nz) - C(nz - 1);
  }
  if (B.b[4] == 1) C(-1) = C(1);
  if (B.b[5] == 1) C(nz + 1) = C(nz - 1);
  if (B.b[4] == 2 && B.b[5] == 2) {
    C(-1) = C(nz - 1);
    C(nz) = C(0);
    C(nz + 1) = C(1);
  }
}


// handlesubgrid2 (f3d_mgrid.F:2628-2764).
template <typename T>
__device__ inline void handlesubgrid2(int im, int ip, T& pm, T& pp, T dsqicos, const double* dels, const double* volt,
                                      T voltfac, T& denom, T& ppp) {
  const T dm = (T)dels[im], dp = (T)dels[ip];
  const T one = (T)1., two = (T)2., half = (T)0.5, zero = (T)0.;
  const T nearone = (T)(1. - 1.e-9);
  if (zero < dm && dm < one && zero < dp && dp < one) {
    pm = voltfac * (T)volt[im] * two / (dm * (dp + dm));
    pp = voltfac * (T)volt[ip] * two / (dp * (dp + dm));
    denom = denom + two * (one - dp * dm) / (dp * dm) * dsqicos;
    ppp = fmin(ppp, dm);
    ppp = fmin(ppp, dp);
  } else if (zero >= dm && dm > -one && zero >= dp && dp > -one) {
    pm = zero;
    pp = zero;
    denom = denom - two * dsqicos;
    ppp = (fabs(dm) > zero) ? (T)fmin(ppp, (T)fabs(dm)) : (T)fmin(ppp, nearone);
    ppp = (fabs(dp) > zero) ? (T)fmin(ppp, (T)fabs(dp)) : (T)fmin(ppp, nearone);
  } else if (zero < dm && dm < one && zero >= dp && dp > -one) {
    const T adel = fabs(dp);
    pm = voltfac * (T)volt[im] / (dm * (adel + half * dm));
    pp = zero;
    denom = denom + (one - two * dm * adel - dm) / (dm * (adel + half * dm)) * dsqicos;
    ppp = fmin(ppp, dm);
    ppp = (adel > zero) ? (T)fmin(ppp, adel) : (T)fmin(ppp, nearone);
  } else if (zero >= dm && dm > -one && zero < dp && dp < one) {
    const T adel = fabs(dm);
    pm = zero;
    pp = voltfac * (T)volt[ip] / (dp * (adel + half * dp));
    denom = denom + (one - two * dp * adel - dp) / (dp * (adel + half * dp)) * dsqicos;
    ppp = (adel > zero) ? (T)fmin(ppp, adel) : (T)fmin(ppp, nearone);
    ppp = fmin(ppp, dp);
  } else {
    if (zero < dm && dm < one) {
      pm = voltfac * (T)volt[im] * two / (dm * (one + dm));
      pp = pp * (two / (one + dm));
      denom = denom + two * (one - dm) / dm * dsqicos;
      ppp = fmin(ppp, dm);
    } else if (zero >= dm && dm > -one) {
      const T adel = fabs(dm);
      pm = zero;
      pp = pp / (half + adel);
      denom = denom - two * adel / (adel + half) * dsqicos;
      ppp = (adel > zero) ? (T)fmin(ppp, adel) : (T)fmin(ppp, nearone);
    }
    if (zero < dp && dp < one) {
      pp = voltfac * (T)volt[ip] * two / (dp * (one + dp));
      pm = pm * (two / (one + dp));
      denom = denom + two * (one - dp) / dp * dsqicos;
      ppp = fmin(ppp, dp);
    } else if (zero >= dp && dp > -one) {
      const T adel = fabs(dp);
      pp = zero;
      pm = pm / (half + adel);
      denom = denom - two * adel / (adel + half) * dsqicos;
      ppp = (adel > zero) ? (T)fmin(ppp, adel) : (T)fmin(ppp, nearone);
    }
  }
}


struct SorCoef {
  double cx, cy, cz, spm1, mgparam;
};

// Conductor data of one level as kernel arguments.
template <typename T>
struct CondArgs {
  const int32_t* iijk;
  const double* ivolt;
  int nint;
  const int32_t* sijk[2];
  const double* sdels[2];
  const double* svolt[2];
  const T* srhs[2];
  int nsub[2];
};

// New value of subgrid point i of colour `par` (condbndymg with icndbndy = 2,
// f3d_mgrid.F:2874-2978): neighbours p[6] = xm,xp,ym,yp,zm,zp, prev = the
// point's value before the pass. Without lcndbndy the bulk update is used.
template <typename T>
__device__ __forceinline__ T subgrid_core(T r, const double* d, const double* v, T pxm, T pxp, T pym, T pyp, T pzm,
                                          T pzp, T prev, const SorCoef& c, int voltfac_on, int lcndbndy) {
  const T dxsqic = (T)c.cx, dysqic = (T)c.cy, dzsqic = (T)c.cz;
  if (lcndbndy) {
    const T dxsqicos = (T)(c.cx / c.mgparam), dysqicos = (T)(c.cy / c.mgparam), dzsqicos = (T)(c.cz / c.mgparam);
    const T voltfac = voltfac_on ? (T)1. : (T)0.;
    T denom = (T)1., ppp = (T)1.;
    handlesubgrid2<T>(0, 1, pxm, pxp, dxsqicos, d, v, voltfac, denom, ppp);
    handlesubgrid2<T>(2, 3, pym, pyp, dysqicos, d, v, voltfac, denom, ppp);
    handlesubgrid2<T>(4, 5, pzm, pzp, dzsqicos, d, v, voltfac, denom, ppp);
    if (ppp < (T)1.)
      return (r + (pxm + pxp) * dxsqic + (pym + pyp) * dysqic + (pzm + pzp) * dzsqic) / denom + (T)c.spm1 * prev;
  }
  return r + (pxm + pxp) * dxsqic + (pym + pyp) * dysqic + (pzm + pzp) * dzsqic + (T)c.spm1 * prev;
}

template <typename T>
__device__ __noinline__ T subgrid_value(const CondArgs<T>& C, int par, int i, T pxm, T pxp, T pym, T pyp, T pzm,
                                        T pzp, T prev, const SorCoef& c, int voltfac_on, int lcndbndy) {
  return subgrid_core<T>(C.srhs[par][i], C.sdels[par] + 6 * (size_t)i, C.svolt[par] + 6 * (size_t)i, pxm, pxp, pym,
                         pyp, pzm, pzp, prev, c, voltfac_on, lcndbndy);
}

// Marks the conductor nodes of one level in its rhs array (see the header
// comment) and saves their rhs values in the subgrid records.
template <typename T>
__global__ void k_box(T* __restrict__ rhs, int nx, int ny, CondArgs<T> C, T* __restrict__ srhs0,
                      T* __restrict__ srhs1) {
  pdl_entry();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < C.nint) {
    rhs[rix(nx, ny, C.iijk[3 * i], C.iijk[3 * i + 1], C.iijk[3 * i + 2])] = Box<T>::make(true, (uint32_t)i);
    return;
  }
  i -= C.nint;
  for (int par = 0; par < 2; ++par) {
    if (i < C.nsub[par]) {
      const int32_t* p = C.sijk[par] + 3 * (size_t)i;
      T& r = rhs[rix(nx, ny, p[0], p[1], p[2])];
      (par ? srhs1 : srhs0)[i] = r;
      r = Box<T>::make(false, (uint32_t)i);
      return;
    }
    i -= C.nsub[par];
  }
}

// ---------------------------------------------------------------------------
// Generic in-place path.

// Writes v to node p at plane iz and, when wtz is set (periodic z with
// non-periodic x and y), to its periodic images: plane nz (image of 0), and
// the guard planes nz+1 (image of 1) and -1 (image of nz-1). This is what
// applyboundaryconditions3d would copy afterwards.
template <typename T>
__device__ inline void store_wt(T* phi, int p, int iz, int nz, int sz, int wtz, T v) {
  phi[p] = v;
  if (wtz) {
    if (iz <= 1) phi[p + nz * sz] = v;
    if (iz == nz - 1) phi[p - nz * sz] = v;
  }
}

// condbndymg update of subgrid point i of colour par (no-op on Dirichlet
// boundary planes). With wtz the plane nz is left to the write-through of
// plane 0. ZERO: phi is taken as all zeros (nothing of it is read).
template <typename T, bool ZERO = false>
__device__ __forceinline__ void special_point(T* phi, int nx, int ny, int nz, const CondArgs<T>& C, int par, const Bnd& B,
                                     const SorCoef& c, int voltfac_on, int lcndbndy, int i, int wtz) {
  // pointers chosen without indexing the parameter arrays by a runtime value
  const int32_t* q = (par ? C.sijk[1] : C.sijk[0]) + 3 * (size_t)i;
  const double* dl = (par ? C.sdels[1] : C.sdels[0]) + 6 * (size_t)i;
  const double* vl = (par ? C.svolt[1] : C.svolt[0]) + 6 * (size_t)i;
  const T r = (par ? C.srhs[1] : C.srhs[0])[i];
  const int ix = q[0], iy = q[1], iz = q[2];
  if (ix == 0 && B.b[0] < 1) return;
  if (ix == nx && B.b[1] < 1) return;
  if (iy == 0 && B.b[2] < 1) return;
  if (iy == ny && B.b[3] < 1) return;
  if (iz == 0 && B.b[4] < 1) return;
  if (iz == nz && B.b[5] < 1) return;
  if (wtz && iz == nz) return;
  const int sy = nx + 3, sz = sy * (ny + 3);
  const int p = (ix + 1) + sy * (iy + 1) + sz * (iz + 1);
  const T z = (T)0.;
  const T v = ZERO ? subgrid_core<T>(r, dl, vl, z, z, z, z, z, z, z, c, voltfac_on, lcndbndy)
                   : subgrid_core<T>(r, dl, vl, phi[p - 1], phi[p + 1], phi[p - sy], phi[p + sy], phi[p - sz],
                                     phi[p + sz], phi[p], c, voltfac_on, lcndbndy);
  store_wt(phi, p, iz, nz, sz, wtz, v);
}

// sorhalfpass3d bulk loop (f3d_mgrid.F:2229-2243): one colour, in place.
// Conductor nodes are skipped here: they keep their old value, which is the
// prevphi of condbndymg, and k_special_sor updates them.
template <typename T, int ZPT>
__global__ void __launch_bounds__(256) k_sor_bulk(T* __restrict__ phi, const T* __restrict__ rhs, int nx, int ny,
                                                  int ixmin, int ixmax, int iymin, int iymax, int izmin, int izmax,
                                                  int parity, T cx, T cy, T cz, T spm1, int nz, int wtz, int nbz,
                                                  CondArgs<T> C, Bnd B, SorCoef sc, int voltfac_on, int lcndbndy) {
  pdl_entry();
  // the first nspz z-slices of blocks update the subgrid conductor points
  // of this colour (condbndymg); they read only nodes of the other colour
  // too, and go first so that their dependent loads overlap the bulk blocks
  const int nspz = (int)gridDim.z - nbz;
  if ((int)blockIdx.z < nspz) {
    const int i = (((int)blockIdx.z * (int)gridDim.y + (int)blockIdx.y) * (int)gridDim.x + (int)blockIdx.x) *
                      (int)(blockDim.x * blockDim.y) +
                  (int)(threadIdx.y * blockDim.x + threadIdx.x);
    if (i < (parity ? C.nsub[1] : C.nsub[0])) special_point<T>(phi, nx, ny, nz, C, parity, B, sc, voltfac_on, lcndbndy, i, wtz);
    return;
  }
  // ZPT consecutive planes per thread; every load of the thread is issued
  // before the first store (the nodes of one colour read only nodes of the
  // other colour, so the order within the half sweep does not matter).
  // Offsets are 32-bit (the level holds fewer than 2^31 padded nodes).
  const int iy = iymin + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (iy > iymax) return;
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iz0 = izmin + ((int)blockIdx.z - nspz) * ZPT;
  const int sy = nx + 3, sz = sy * (ny + 3), ry = nx + 1, rz = ry * (ny + 1);
  const int xb = ixmin + 2 * t, odd0 = (ixmin + iy + iz0 + parity) & 1;
  const int p0 = (xb + 1) + sy * (iy + 1) + sz * (iz0 + 1);
  const int q0 = xb + ry * iy + rz * iz0;
  T r[ZPT], c[ZPT], xm[ZPT], xp[ZPT], ym[ZPT], yp[ZPT], zm[ZPT], zp[ZPT];
  bool ok[ZPT];
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    const int sh = (odd0 + k) & 1;
    ok[k] = iz0 + k <= izmax && xb + sh <= ixmax;
    if (ok[k]) {
      const int p = p0 + k * sz + sh;
      r[k] = rhs[q0 + k * rz + sh];
      c[k] = phi[p];
      xm[k] = phi[p - 1];
      xp[k] = phi[p + 1];
      ym[k] = phi[p - sy];
      yp[k] = phi[p + sy];
      zm[k] = phi[p - sz];
      zp[k] = phi[p + sz];
    }
  }
#pragma unroll
  for (int k = 0; k < ZPT; ++k)
    if (ok[k] && !isbox(r[k]))
      store_wt(phi, p0 + k * sz + ((odd0 + k) & 1), iz0 + k, nz, sz, wtz,
               r[k] + (xm[k] + xp[k]) * cx + (ym[k] + yp[k]) * cy + (zm[k] + zp[k]) * cz + spm1 * c[k]);
}

// The first (red) half sweep of a pass whose phi is all zeros, for a level
// where k_sor_bulk does the whole half sweep (no Neumann-type subgrid
// points, Dirichlet x and y, periodic z with an even nz or Dirichlet z). It
// writes every node of the padded array once, reading rhs only, and so
// replaces the zeroing: a red node of the update range gets the bulk or
// subgrid formula evaluated with zero neighbours (the same expressions, so
// the same bits as zeroing the array and running k_sor_bulk), every other
// node 0, and with wtz the periodic images take their source plane's value.
// As in k_sor_bulk, the first nspz z-slices of blocks take the red subgrid
// points, one a thread; the bulk blocks skip those nodes. A bulk thread
// takes the x pair (2t-1, 2t) of one row in FZ consecutive planes: one node
// of a pair is red, and its rhs loads for all FZ planes are issued before
// the first store.
template <typename T, int FZ>
__global__ void __launch_bounds__(256) k_sor_from_zero(T* __restrict__ phi, const T* __restrict__ rhs, int nx, int ny,
                                                       int nz, int ixmin, int ixmax, int iymin, int iymax, int izmin,
                                                       int izmax, T cx, T cy, T cz, T spm1, int wtz, int nbz,
                                                       CondArgs<T> C, Bnd B, SorCoef sc, int lcndbndy) {
  pdl_entry();
  const int nspz = (int)gridDim.z - nbz;
  if ((int)blockIdx.z < nspz) {
    const int i = (((int)blockIdx.z * (int)gridDim.y + (int)blockIdx.y) * (int)gridDim.x + (int)blockIdx.x) *
                      (int)(blockDim.x * blockDim.y) +
                  (int)(threadIdx.y * blockDim.x + threadIdx.x);
    if (i < C.nsub[0]) special_point<T, true>(phi, nx, ny, nz, C, 0, B, sc, 0, lcndbndy, i, wtz);
    return;
  }
  const int x0 = 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x) - 1;
  const int iy = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 1;
  const int z0 = ((int)blockIdx.z - nspz) * FZ - 1;
  if (x0 > nx + 1 || iy > ny + 1) return;
  const bool yin = iy >= iymin && iy <= iymax;
  T r[FZ];
  int xr[FZ];
  bool upd[FZ];
#pragma unroll
  for (int k = 0; k < FZ; ++k) {
    const int iz = z0 + k;
    int src = iz;
    if (wtz) {
      if (iz == nz) src = 0;
      else if (iz == nz + 1) src = 1;
      else if (iz == -1) src = nz - 1;
    }
    xr[k] = x0 + ((x0 + iy + src) & 1);
    upd[k] = iz <= nz + 1 && yin && src >= izmin && src <= izmax && xr[k] >= ixmin && xr[k] <= ixmax;
    if (upd[k]) r[k] = rhs[(size_t)xr[k] + (size_t)(nx + 1) * ((size_t)iy + (size_t)(ny + 1) * src)];
  }
  const size_t sz = (size_t)(nx + 3) * (ny + 3);
  const size_t pr = (size_t)(x0 + 1) + (size_t)(nx + 3) * (iy + 1);
#pragma unroll
  for (int k = 0; k < FZ; ++k) {
    const int iz = z0 + k;
    if (iz > nz + 1) break;
    // a red subgrid point of the range is written by the subgrid blocks
    bool mine = true;
    T v = (T)0.;
    if (upd[k]) {
      if (!isbox(r[k])) {
        const T z = (T)0.;
        v = r[k] + (z + z) * cx + (z + z) * cy + (z + z) * cz + spm1 * z;
      } else {
        mine = Box<T>::interior(r[k]);
      }
    }
    // the pair's second node exists up to x = nx + 1 (an odd row length
    // leaves the last pair single)
    T* row = phi + pr + sz * (size_t)(iz + 1);
    const bool second = xr[k] != x0;
    if (second) row[0] = (T)0.;
    else if (mine) row[0] = v;
    if (x0 + 1 <= nx + 1) {
      if (!second) row[1] = (T)0.;
      else if (mine) row[1] = v;
    }
  }
}

// condbndymg for one colour then cond_potmg (f3d_mgrid.F:2874-2978,
// 2426-2470). Subgrid and interior sets are disjoint and only read the other
// colour, so one launch does both.
template <typename T>
__global__ void k_special_sor(T* __restrict__ phi, int nx, int ny, int nz, CondArgs<T> C, int par, Bnd B, SorCoef c,
                              int voltfac_on, int usev, int lcndbndy) {
  pdl_entry();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nsub = par ? C.nsub[1] : C.nsub[0];
  if (i < nsub) {
    special_point<T>(phi, nx, ny, nz, C, par, B, c, voltfac_on, lcndbndy, i, 0);
    return;
  }
  i -= nsub;
  if (i < C.nint) phi[pix(nx, ny, C.iijk[3 * i], C.iijk[3 * i + 1], C.iijk[3 * i + 2])] = usev ? (T)C.ivolt[i] : (T)0.;
}

// cond_potmg alone (start of sorpass3d and the mgform=2 initial phi).
template <typename T>
__global__ void k_interior(T* __restrict__ phi, int nx, int ny, const int32_t* __restrict__ iijk,
                           const double* __restrict__ ivolt, int nint, int usev, int nz = 0, int wtz = 0) {
  pdl_entry();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nint) return;
  const int ix = iijk[3 * i], iy = iijk[3 * i + 1], iz = iijk[3 * i + 2];
  const int sy = nx + 3, sz = sy * (ny + 3);
  if (wtz && iz == nz) return;
  store_wt(phi, (ix + 1) + sy * (iy + 1) + sz * (iz + 1), iz, nz, sz, wtz, usev ? (T)ivolt[i] : (T)0.);
}

// condbndymgint (f3d_mgrid.F:2982-3092): Neumann subgrid neighbours take the
// point's value.
template <typename T>
__global__ void k_condbndymgint(T* __restrict__ phi, int nx, int ny, int nz, const int32_t* __restrict__ ijk,
                                const double* __restrict__ dels, int n, Bnd B) {
  pdl_entry();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ix = ijk[3 * i], iy = ijk[3 * i + 1], iz = ijk[3 * i + 2];
  const double* d = dels + 6 * (size_t)i;
  const T p0 = phi[pix(nx, ny, ix, iy, iz)];
  if (!((ix - 1 == 0 && B.b[0] == 0) || (ix + 1 == nx && B.b[1] == 0) || (ix == 0 && B.b[0] < 1) ||
        (ix == nx && B.b[1] < 1))) {
    if (0. >= d[0] && d[0] > -1.) phi[pix(nx, ny, ix - 1, iy, iz)] = p0;
    if (0. >= d[1] && d[1] > -1.) phi[pix(nx, ny, ix + 1, iy, iz)] = p0;
  }
  if (!((iy - 1 == 0 && B.b[2] == 0) || (iy + 1 == ny && B.b[3] == 0) || (iy == 0 && B.b[2] < 1) ||
        (iy == ny && B.b[3] < 1))) {
    if (0. >= d[2] && d[2] > -1.) phi[pix(nx, ny, ix, iy - 1, iz)] = p0;
    if (0. >= d[3] && d[3] > -1.) phi[pix(nx, ny, ix, iy + 1, iz)] = p0;
  }
  if (!((iz - 1 == 0 && B.b[4] == 0) || (iz + 1 == nz && B.b[5] == 0) || (iz == 0 && B.b[4] < 1) ||
        (iz == nz && B.b[5] < 1))) {
    if (0. >= d[4] && d[4] > -1.) phi[pix(nx, ny, ix, iy, iz - 1)] = p0;
    if (0. >= d[5] && d[5] > -1.) phi[pix(nx, ny, ix, iy, iz + 1)] = p0;
  }
}

// ---------------------------------------------------------------------------
// residual3d bulk part (f3d_mgrid.F:3519-3586).
//   MODE 0: writes the padded res array (0 outside the updated range)
//   MODE 1: no store, only the max over non-conductor nodes (norm)
//   MODE 2: writes the unpadded FP32 rhs of the next correction solve
// Conductor nodes get 0 here; k_special_res fills them in.
// Six blocks per SM (40 registers): the kernel is bound by memory latency, and
// the extra resident warps took the FP32 residual of the finest 256x256x512
// level from 187 to 167 us on the B200.
// The bulk residual for the thread's node column of block (bx, by, bz).
// keep_sub: leave subgrid-point nodes unwritten (a merged kernel's
// subgrid blocks write them).
// wtz (MODE 0, periodic z with Dirichlet x and y): planes 0, 1 and nz-1 are
// also written to their images nz, nz+1 and -1, which are then not written
// from their own threads: the boundary copy that would follow is done.
template <typename T, int MODE, typename TO, int ZPT>
__device__ __forceinline__ void residual_bulk(const T* __restrict__ phi, const T* __restrict__ rhs,
                                              TO* __restrict__ out, int nx, int ny, int nz, int ixmin, int ixmax,
                                              int iymin, int iymax, int izmin, int izmax, T cx, T cy, T cz, T mgparam,
                                              int bx, int by, int bz, bool keep_sub, T& m, int wtz = 0) {
  // MODE 0 covers the padded array, the others the node array; ZPT planes
  // per thread with all loads issued first; 32-bit offsets
  const int g = (MODE == 0) ? 1 : 0;
  const int ix = (int)(bx * blockDim.x + threadIdx.x) - g;
  const int iy = (int)(by * blockDim.y + threadIdx.y) - g;
  const int iz0 = bz * ZPT - g;
  const bool live = ix <= nx + g && iy <= ny + g;
  const bool xyin = ix >= ixmin && ix <= ixmax && iy >= iymin && iy <= iymax;
  const int sy = nx + 3, sz = sy * (ny + 3), ry = nx + 1, rz = ry * (ny + 1);
  const int p0 = (ix + 1) + sy * (iy + 1) + sz * (iz0 + 1);
  const int q0 = ix + ry * iy + rz * iz0;
  T b[ZPT], c[ZPT], xm[ZPT], xp[ZPT], ym[ZPT], yp[ZPT], zm[ZPT], zp[ZPT];
  bool in[ZPT];
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    const int iz = iz0 + k;
    in[k] = live && xyin && iz >= izmin && iz <= izmax;
    if (in[k]) {
      const int p = p0 + k * sz;
      b[k] = rhs[q0 + k * rz];
      c[k] = phi[p];
      xm[k] = phi[p - 1];
      xp[k] = phi[p + 1];
      ym[k] = phi[p - sy];
      yp[k] = phi[p + sy];
      zm[k] = phi[p - sz];
      zp[k] = phi[p + sz];
    }
  }
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    if (!live || iz0 + k > nz + g) continue;
    T r = (T)0.;
    if (in[k]) {
      if (!isbox(b[k])) {
        r = b[k] + (xm[k] + xp[k]) * cx + (ym[k] + yp[k]) * cy + (zm[k] + zp[k]) * cz - c[k] * mgparam;
        m = fmax(m, fabs(r));
      } else if (keep_sub && !Box<T>::interior(b[k])) {
        continue;
      }
    }
    if (MODE == 0) {
      const int iz = iz0 + k;
      if (wtz && (iz < 0 || iz >= nz)) continue;
      const int p = p0 + k * sz;
      out[p] = (TO)r;
      if (wtz) {
        if (iz <= 1) out[p + nz * sz] = (TO)r;
        if (iz == nz - 1) out[p - nz * sz] = (TO)r;
      }
    }
    if (MODE == 2) out[q0 + k * rz] = (TO)r;
  }
}

template <typename T, int MODE, typename TO, int ZPT>
__global__ void __launch_bounds__(256, 6) k_residual(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                  TO* __restrict__ out, int nx, int ny, int nz, int ixmin,
                                                  int ixmax, int iymin, int iymax, int izmin, int izmax, T cx, T cy,
                                                  T cz, T mgparam, unsigned long long* maxout, int wtz) {
  pdl_entry();
  T m = (T)0.;
  residual_bulk<T, MODE, TO, ZPT>(phi, rhs, out, nx, ny, nz, ixmin, ixmax, iymin, iymax, izmin, izmax, cx, cy, cz,
                                  mgparam, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, false, m, wtz);
  if (maxout) block_max_to(maxout, (double)m);
}

// cond_potmgres (interior -> 0, f3d_mgrid.F:2472-2500) and condbndyres
// (icndbndy = 2, f3d_mgrid.F:3240-3362) for both colours.
template <typename T, int MODE, typename TO>
__device__ __forceinline__ double special_res_point(const T* __restrict__ phi, TO* __restrict__ out, int nx, int ny,
                                                    int nz, const CondArgs<T>& C, const Bnd& B, double dxsqi,
                                                    double dysqi, double dzsqi, double mgparam_d, int voltfac_on,
                                                    int mgform2init, int lcndbndy, int i, int wtz = 0) {
  double m = 0.;
  auto store = [&](int ix, int iy, int iz, T v) {
    if (MODE == 0) {
      // wtz: as in residual_bulk, image planes only through their sources
      if (wtz && (iz < 0 || iz >= nz)) return;
      const size_t q = pix(nx, ny, ix, iy, iz);
      out[q] = (TO)v;
      if (wtz) {
        const size_t nxy = (size_t)(nx + 3) * (ny + 3);
        if (iz <= 1) out[q + (size_t)nz * nxy] = (TO)v;
        if (iz == nz - 1) out[q - (size_t)nz * nxy] = (TO)v;
      }
    }
    if (MODE == 2 && ix >= 0 && ix <= nx && iy >= 0 && iy <= ny && iz >= 0 && iz <= nz)
      out[rix(nx, ny, ix, iy, iz)] = (TO)v;
  };
  const int n0 = C.nsub[0], n1 = C.nsub[1];
  if (i < C.nint) {
    store(C.iijk[3 * i], C.iijk[3 * i + 1], C.iijk[3 * i + 2], (T)0.);
  } else if (i < C.nint + n0 + n1) {
    int k = i - C.nint;
    const int par = (k < n0) ? 0 : 1;
    if (par) k -= n0;
    // parity arrays chosen without indexing the parameter arrays at run time
    const int32_t* sijk = par ? C.sijk[1] : C.sijk[0];
    const T* srhs = par ? C.srhs[1] : C.srhs[0];
    const double* sdels = par ? C.sdels[1] : C.sdels[0];
    const double* svolt = par ? C.svolt[1] : C.svolt[0];
    const int32_t* q = sijk + 3 * (size_t)k;
    const int ix = q[0], iy = q[1], iz = q[2];
    bool skip = (ix == 0 && B.b[0] == 0) || (ix == nx && B.b[1] == 0) || (iy == 0 && B.b[2] == 0) ||
                (iy == ny && B.b[3] == 0) || (iz == 0 && B.b[4] == 0) || (iz == nz && B.b[5] == 0);
    if (!skip) {
      const double cst = 0.5 / (dxsqi + dysqi + dzsqi);
      const T dxsqic = (T)(dxsqi * cst), dysqic = (T)(dysqi * cst), dzsqic = (T)(dzsqi * cst);
      const T dxsqics = (T)(mgparam_d * dxsqi * cst), dysqics = (T)(mgparam_d * dysqi * cst),
              dzsqics = (T)(mgparam_d * dzsqi * cst);
      const T mgparam = (T)mgparam_d;
      const size_t sy = nx + 3, sz = (size_t)(nx + 3) * (ny + 3);
      const size_t p = pix(nx, ny, ix, iy, iz);
      const T rhsv = srhs[k];
      T pxm = phi[p - 1], pxp = phi[p + 1], pym = phi[p - sy], pyp = phi[p + sy], pzm = phi[p - sz],
        pzp = phi[p + sz];
      T denom = (T)1., ppp = (T)1.;
      if (lcndbndy) {
        const T voltfac = voltfac_on ? (T)1. : (T)0.;
        const double* d = sdels + 6 * (size_t)k;
        const double* v = svolt + 6 * (size_t)k;
        handlesubgrid2<T>(0, 1, pxm, pxp, dxsqic, d, v, voltfac, denom, ppp);
        handlesubgrid2<T>(2, 3, pym, pyp, dysqic, d, v, voltfac, denom, ppp);
        handlesubgrid2<T>(4, 5, pzm, pzp, dzsqic, d, v, voltfac, denom, ppp);
      }
      if (ppp < (T)1.) {
        // the reported max always uses the ppp-scaled row (getresidual,
        // scripts/multigrid.py:940); the stored value drops the scaling for
        // the residual-correction set-up
        const T pppmax = ppp;
        if (mgform2init) ppp = (T)1.;
        const T inner = rhsv + (pxm + pxp) * dxsqics + (pym + pyp) * dysqics + (pzm + pzp) * dzsqics -
                        phi[p] * mgparam * denom;
        T r = ppp * inner;
        store(ix, iy, iz, r);
        m = fabs((double)(pppmax * inner));
        const double* d = sdels + 6 * (size_t)k;
        if (0. >= d[0] && d[0] >= -1.) store(ix - 1, iy, iz, (T)0.);
        if (0. >= d[1] && d[1] >= -1.) store(ix + 1, iy, iz, (T)0.);
        if (0. >= d[2] && d[2] >= -1.) store(ix, iy - 1, iz, (T)0.);
        if (0. >= d[3] && d[3] >= -1.) store(ix, iy + 1, iz, (T)0.);
        if (0. >= d[4] && d[4] >= -1.) store(ix, iy, iz - 1, (T)0.);
        if (0. >= d[5] && d[5] >= -1.) store(ix, iy, iz + 1, (T)0.);
      } else {
        // no special direction: the bulk residual the reference keeps
        T r = rhsv + (pxm + pxp) * dxsqics + (pym + pyp) * dysqics + (pzm + pzp) * dzsqics - phi[p] * mgparam;
        store(ix, iy, iz, r);
        m = fabs((double)r);
      }
    }
  }
  return m;
}

template <typename T, int MODE, typename TO>
__global__ void k_special_res(const T* __restrict__ phi, TO* __restrict__ out, int nx, int ny, int nz, CondArgs<T> C,
                              Bnd B, double dxsqi, double dysqi, double dzsqi, double mgparam_d, int voltfac_on,
                              int mgform2init, int lcndbndy, unsigned long long* maxout, int wtz) {
  pdl_entry();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double m = special_res_point<T, MODE, TO>(phi, out, nx, ny, nz, C, B, dxsqi, dysqi, dzsqi, mgparam_d,
                                                  voltfac_on, mgform2init, lcndbndy, i, wtz);
  if (maxout) block_max_to(maxout, m);
}

// The residual of a level without Neumann-type subgrid points in one launch:
// the first nspz z-slices of blocks compute the subgrid points
// (k_special_res), the others the bulk, which leaves those nodes unwritten.
template <typename T, int MODE, typename TO, int ZPT>
__global__ void __launch_bounds__(256) k_residual_sp(const T* __restrict__ phi, const T* __restrict__ rhs,
                                                     TO* __restrict__ out, int nx, int ny, int nz, int ixmin,
                                                     int ixmax, int iymin, int iymax, int izmin, int izmax, T cx,
                                                     T cy, T cz, T mgparam, int nbz, CondArgs<T> C, Bnd B,
                                                     double dxsqi, double dysqi, double dzsqi, double mgparam_d,
                                                     int voltfac_on, int mgform2init, int lcndbndy,
                                                     unsigned long long* maxout, int wtz) {
  pdl_entry();
  const int nspz = (int)gridDim.z - nbz;
  double md;
  if ((int)blockIdx.z < nspz) {
    const int i = (((int)blockIdx.z * (int)gridDim.y + (int)blockIdx.y) * (int)gridDim.x + (int)blockIdx.x) *
                      (int)(blockDim.x * blockDim.y) +
                  (int)(threadIdx.y * blockDim.x + threadIdx.x);
    md = special_res_point<T, MODE, TO>(phi, out, nx, ny, nz, C, B, dxsqi, dysqi, dzsqi, mgparam_d, voltfac_on,
                                        mgform2init, lcndbndy, i, wtz);
  } else {
    T m = (T)0.;
    residual_bulk<T, MODE, TO, ZPT>(phi, rhs, out, nx, ny, nz, ixmin, ixmax, iymin, iymax, izmin, izmax, cx, cy,
                                    cz, mgparam, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z - nspz, true, m,
                                    wtz);
    md = (double)m;
  }
  if (maxout) block_max_to(maxout, md);
}

// restrict3d (f3d_mgrid.F:1593-1775): one thread per coarse node, summing
// the tent-weighted fine residual in the reference's loop order (z, y, x).
// Windows and weights come from per-axis tables (Level::rlo/rn/rw) and are
// at most NT wide per axis; the loads of one fine plane are issued together
// before the ordered sums. The products keep the reference's order,
// (wx * wy) * wz, with wx * wy formed once per thread; 32-bit offsets.
template <typename T, int NT>
__global__ void __launch_bounds__(256) k_restrict(const T* __restrict__ res, T* __restrict__ rhoc, int nx, int ny,
                                                  int nxc, int nyc, int ixcmin, int ixcmax, int iycmin, int iycmax,
                                                  int izcmin, int izcmax, const int32_t* __restrict__ tlo,
                                                  const int32_t* __restrict__ tn, const double* __restrict__ tw,
                                                  double ff) {
  pdl_entry();
  const int ixc = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iyc = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int izc = blockIdx.z;
  if (ixc > nxc || iyc > nyc) return;
  const int o = ixc + (nxc + 1) * (iyc + (nyc + 1) * izc);
  if (ixc < ixcmin || ixc > ixcmax || iyc < iycmin || iyc > iycmax || izc < izcmin || izc > izcmax) {
    rhoc[o] = (T)0.;
    return;
  }
  const int ox = ixc, oy = nxc + 1 + iyc, oz = nxc + 1 + nyc + 1 + izc;
  const int lx = tlo[ox], ly = tlo[oy], lz = tlo[oz];
  const int cx = tn[ox], cy = tn[oy], cz = tn[oz];
  T wxy[NT][NT];
#pragma unroll
  for (int ky = 0; ky < NT; ++ky)
#pragma unroll
    for (int kx = 0; kx < NT; ++kx) wxy[ky][kx] = (T)tw[ox * kRestrictTaps + kx] * (T)tw[oy * kRestrictTaps + ky];
  const int sy = nx + 3, sz = sy * (ny + 3);
  const int b0 = (lx + 1) + sy * (ly + 1) + sz * (lz + 1);
  T r = (T)0., w = (T)0.;
  for (int kz = 0; kz < cz; ++kz) {
    const T wz = (T)tw[oz * kRestrictTaps + kz];
    const T* plane = res + (b0 + kz * sz);
    T v[NT][NT];
#pragma unroll
    for (int ky = 0; ky < NT; ++ky)
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) v[ky][kx] = (ky < cy && kx < cx) ? plane[ky * sy + kx] : (T)0.;
#pragma unroll
    for (int ky = 0; ky < NT; ++ky) {
      if (ky >= cy) break;
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) {
        if (kx >= cx) break;
        const T t = wxy[ky][kx] * wz;
        r = r + t * v[ky][kx];
        w = w + t;
      }
    }
  }
  if (w > (T)0.) {
    r = r / w;
    rhoc[o] = r * (T)ff;
  } else {
    rhoc[o] = (T)0.;
  }
}

// expand3d (f3d_mgrid.F:1777-1947): trilinear prolongation added to phi.
// Coarse indices and weights come from per-axis tables (Level::ej/ew); ZPT
// consecutive fine planes per thread, all loads issued before the sums;
// 32-bit offsets. The weight products keep the reference's left-to-right
// order, ((wx' * wy') * wz') * q, with the x-y part formed once per thread.
// restrict3d for a coarse level whose z is not coarsened (nzc == nz). The
// z window of a coarse plane is the fine plane itself with weight exactly 1,
// so each tap weight is (wx * wy) * 1 = wx * wy, and the sums below are the
// generic kernel's, operation for operation. The x-y weights and their sum
// are formed once and serve ZPT coarse planes per thread.
template <typename T, int NT, int ZPT>
__global__ void __launch_bounds__(256) k_restrict_xy(const T* __restrict__ res, T* __restrict__ rhoc, int nx, int ny,
                                                     int nxc, int nyc, int nzc, int ixcmin, int ixcmax, int iycmin,
                                                     int iycmax, int izcmin, int izcmax,
                                                     const int32_t* __restrict__ tlo, const int32_t* __restrict__ tn,
                                                     const double* __restrict__ tw, double ff) {
  pdl_entry();
  const int ixc = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iyc = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int izc0 = (int)blockIdx.z * ZPT;
  if (ixc > nxc || iyc > nyc) return;
  const bool xyin = ixc >= ixcmin && ixc <= ixcmax && iyc >= iycmin && iyc <= iycmax;
  const int ox = ixc, oy = nxc + 1 + iyc;
  int lx = 0, ly = 0, cx = 0, cy = 0;
  T wxy[NT][NT];
  T w = (T)0.;
  if (xyin) {
    lx = tlo[ox];
    ly = tlo[oy];
    cx = tn[ox];
    cy = tn[oy];
#pragma unroll
    for (int ky = 0; ky < NT; ++ky)
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) wxy[ky][kx] = (T)tw[ox * kRestrictTaps + kx] * (T)tw[oy * kRestrictTaps + ky];
#pragma unroll
    for (int ky = 0; ky < NT; ++ky) {
      if (ky >= cy) break;
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) {
        if (kx >= cx) break;
        w = w + wxy[ky][kx];
      }
    }
  }
  const int sy = nx + 3, sz = sy * (ny + 3);
  const int b0 = (lx + 1) + sy * (ly + 1);
  T v[ZPT][NT][NT];
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    const int izc = izc0 + k;
    const bool in = xyin && izc >= izcmin && izc <= izcmax;
    const T* plane = res + (b0 + sz * (izc + 1));
#pragma unroll
    for (int ky = 0; ky < NT; ++ky)
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) v[k][ky][kx] = (in && ky < cy && kx < cx) ? plane[ky * sy + kx] : (T)0.;
  }
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    const int izc = izc0 + k;
    if (izc > nzc) break;
    const int o = ixc + (nxc + 1) * (iyc + (nyc + 1) * izc);
    if (!xyin || izc < izcmin || izc > izcmax) {
      rhoc[o] = (T)0.;
      continue;
    }
    T r = (T)0.;
#pragma unroll
    for (int ky = 0; ky < NT; ++ky) {
      if (ky >= cy) break;
#pragma unroll
      for (int kx = 0; kx < NT; ++kx) {
        if (kx >= cx) break;
        r = r + wxy[ky][kx] * v[k][ky][kx];
      }
    }
    if (w > (T)0.) {
      r = r / w;
      rhoc[o] = r * (T)ff;
    } else {
      rhoc[o] = (T)0.;
    }
  }
}

// wtz: periodic z with Dirichlet x and y; the range stops at plane nz-1 and
// planes 0, 1 and nz-1 are also written to their images nz, nz+1 and -1 (the
// boundary copy that would follow).
template <typename T, int ZPT, bool ZC>
__global__ void __launch_bounds__(256) k_expand(T* __restrict__ phi, const T* __restrict__ pc, int nx, int ny,
                                                int nxc, int nyc, int ixmin, int ixmax, int iymin, int iymax,
                                                int izmin, int izmax, const int32_t* __restrict__ ej,
                                                const double* __restrict__ ew, int nz, int wtz) {
  pdl_entry();
  const int ix = ixmin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int iy = iymin + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int iz0 = izmin + (int)blockIdx.z * ZPT;
  if (ix > ixmax || iy > iymax) return;
  const int oy = nx + 3, oz = nx + 3 + ny + 3;
  const int jx = ej[ix + 1], jy = ej[oy + iy + 1];
  const T one = (T)1.;
  const T wx = (T)ew[ix + 1], wy = (T)ew[oy + iy + 1];
  const T a00 = (one - wx) * (one - wy), a10 = wx * (one - wy), a01 = (one - wx) * wy, a11 = wx * wy;
  const int sy = nx + 3, sz = sy * (ny + 3);
  const int syc = nxc + 3, szc = syc * (nyc + 3);
  const int cxy = (jx + 1) + syc * (jy + 1);
  const int f0 = (ix + 1) + sy * (iy + 1) + sz * (iz0 + 1);
  T q[ZPT][8], f[ZPT], wz[ZPT];
  bool ok[ZPT];
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    const int iz = iz0 + k;
    ok[k] = iz <= izmax;
    if (ok[k]) {
      // z not coarsened: the coarse plane is the fine plane and its weight
      // is exactly 0, so the tables need not be read
      const int jz = ZC ? ej[oz + iz + 1] : iz;
      wz[k] = ZC ? (T)ew[oz + iz + 1] : (T)0.;
      const T* b = pc + (cxy + szc * (jz + 1));
      q[k][0] = b[0];
      q[k][1] = b[1];
      q[k][2] = b[syc];
      q[k][3] = b[syc + 1];
      if (ZC) {
        q[k][4] = b[szc];
        q[k][5] = b[szc + 1];
        q[k][6] = b[szc + syc];
        q[k][7] = b[szc + syc + 1];
      }
      f[k] = phi[f0 + k * sz];
    }
  }
#pragma unroll
  for (int k = 0; k < ZPT; ++k) {
    if (!ok[k]) continue;
    const T z = wz[k], z1 = one - z;
    T v;
    if (ZC)
      v = f[k] + a00 * z1 * q[k][0] + a10 * z1 * q[k][1] + a01 * z1 * q[k][2] + a11 * z1 * q[k][3] +
          a00 * z * q[k][4] + a10 * z * q[k][5] + a01 * z * q[k][6] + a11 * z * q[k][7];
    else  // z not coarsened: wz = 0 and z1 = 1 exactly, the z+1 terms add zeros
      v = f[k] + a00 * q[k][0] + a10 * q[k][1] + a01 * q[k][2] + a11 * q[k][3];
    const int p = f0 + k * sz;
    phi[p] = v;
    if (wtz) {
      const int iz = iz0 + k;
      if (iz <= 1) phi[p + nz * sz] = v;
      if (iz == nz - 1) phi[p - nz * sz] = v;
    }
  }
}


// mgerror = max|phisave - phi| over nodes 0..n (f3d_mgrid.F:383-391).
__global__ void k_maxdiff(const double* __restrict__ a, const double* __restrict__ b, int nx, int ny,
                          unsigned long long* maxout) {
  pdl_entry();
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  double m = 0.;
  if (ix <= nx && iy <= ny) {
    size_t p = pix(nx, ny, ix, iy, iz);
    m = fabs(a[p] - b[p]);
  }
  block_max_to(maxout, m);
}

// rhs = rho * reps0c (f3d_mgrid.F:223) and max|rhs|; flags a non-finite rho.
// rhs (node layout) into the interior of a padded array: the source of the
// full multigrid's restriction of rho, whose windows stay inside 0..n.
__global__ void k_pad_copy(const double* __restrict__ src, double* __restrict__ dst, int nx, int ny) {
  pdl_entry();
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y, iz = blockIdx.z;
  if (ix > nx || iy > ny) return;
  dst[(size_t)(ix + 1) + (size_t)(nx + 3) * ((size_t)(iy + 1) + (size_t)(ny + 3) * (iz + 1))] =
      src[(size_t)ix + (size_t)(nx + 1) * ((size_t)iy + (size_t)(ny + 1) * iz)];
}

__global__ void k_scale_rhs(const double* __restrict__ rho, double* __restrict__ rhs, size_t n, double s,
                            unsigned long long* maxout, unsigned long long* flag) {
  pdl_entry();
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.;
  if (i < n) {
    double v = rho[i] * s;
    if (!isfinite(v)) atomicOr(flag, 2ull);
    rhs[i] = v;
    m = fabs(v);
  }
  block_max_to(maxout, m);
}

// Residual-correction update phi = e + phisave (f3d_mgrid.F:355-358) with
// e from an FP32 V-cycle; max|dphi| over nodes 0..n. Four planes per thread.
constexpr int kCorrPlanes = 4;
__global__ void __launch_bounds__(256) k_add_corr(double* __restrict__ phi, const float* __restrict__ e, int nx,
                                                  int ny, int nz, unsigned long long* maxout) {
  pdl_entry();
  const int ix = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 1;
  const int iy = (int)(blockIdx.y * blockDim.y + threadIdx.y) - 1;
  const int iz0 = (int)blockIdx.z * kCorrPlanes - 1;
  double m = 0.;
  if (ix <= nx + 1 && iy <= ny + 1) {
    const int sz = (nx + 3) * (ny + 3);
    const int p0 = (ix + 1) + (nx + 3) * (iy + 1) + sz * (iz0 + 1);
    double old[kCorrPlanes];
    float ev[kCorrPlanes];
#pragma unroll
    for (int k = 0; k < kCorrPlanes; ++k) {
      if (iz0 + k <= nz + 1) {
        old[k] = phi[p0 + k * sz];
        ev[k] = e[p0 + k * sz];
      }
    }
#pragma unroll
    for (int k = 0; k < kCorrPlanes; ++k) {
      const int iz = iz0 + k;
      if (iz > nz + 1) continue;
      const double nw = (double)ev[k] + old[k];
      phi[p0 + k * sz] = nw;
      if (ix >= 0 && ix <= nx && iy >= 0 && iy <= ny && iz >= 0 && iz <= nz) m = fmax(m, fabs(old[k] - nw));
    }
  }
  block_max_to(maxout, m);
}

inline unsigned cdiv(size_t a, unsigned b) { return (unsigned)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
template <typename T>
struct Arr;
template <>
struct Arr<double> {
  static double*& phi(Level& L) { return L.phi; }
  static double* rhs(Level& L) { return L.rhs; }
  static double* res(Level& L) { return L.res; }
  static double* srhs(DevSubgrid& S) { return S.rhs; }
};
template <>
struct Arr<float> {
  static float*& phi(Level& L) { return L.phif; }
  static float* rhs(Level& L) { return L.rhsf; }
  static float* res(Level& L) { return L.resf; }
  static float* srhs(DevSubgrid& S) { return S.rhsf; }
};

template <typename T>
CondArgs<T> cond_args(Level& L) {
  CondArgs<T> C;
  C.iijk = L.int_ijk;
  C.ivolt = L.int_volt;
  C.nint = L.n_int;
  for (int p = 0; p < 2; ++p) {
    C.sijk[p] = L.sub[p].ijk;
    C.sdels[p] = L.sub[p].dels;
    C.svolt[p] = L.sub[p].volt;
    C.srhs[p] = Arr<T>::srhs(L.sub[p]);
    C.nsub[p] = L.sub[p].n;
  }
  return C;
}

struct Ranges {
  int ixmin, ixmax, iymin, iymax, izmin, izmax;
};
// Loop limits: `le` = limits of sorhalfpass3d (bound <= 0 excludes the edge),
// else those of residual3d/expand3d/restrict3d (bound == 0 excludes it).
Ranges ranges(const LevelDims& d, const int* b, bool le) {
  Ranges r{0, d.nx, 0, d.ny, 0, d.nz};
  auto dir = [&](int v) { return le ? v <= 0 : v == 0; };
  if (dir(b[0])) r.ixmin = 1;
  if (dir(b[1])) r.ixmax = d.nx - 1;
  if (dir(b[2])) r.iymin = 1;
  if (dir(b[3])) r.iymax = d.ny - 1;
  if (dir(b[4])) r.izmin = 1;
  if (dir(b[5])) r.izmax = d.nz - 1;
  return r;
}

struct Solver {
  wg_ctx* c;
  const wg_solve_opts* o;
  Bnd B;
  cudaStream_t s;
  bool capturing = false;
  bool pdl = false;  // launch with programmatic dependent launch
  bool pdl_timed = false;  // the solve's PDL setting (pdl is off while profiling)
  cudaError_t lerr = cudaSuccess;  // first launch error

  // One kernel launch on the solver's stream; with pdl set, the kernel may
  // be scheduled while the previous one in the stream still runs (every
  // kernel launched here starts with pdl_entry()).
  template <typename... KArgs, typename... Args>
  void launch(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, Args&&... args) {
    ++c->nlaunch;
    cudaError_t e;
    if (pdl) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = g;
      cfg.blockDim = b;
      cfg.dynamicSmemBytes = smem;
      cfg.stream = s;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      e = cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
    } else {
      k<<<g, b, smem, s>>>(std::forward<Args>(args)...);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess && lerr == cudaSuccess) lerr = e;
  }

  // Zeroing and copying are kernels here, not cudaMemsetAsync or a
  // device-to-device cudaMemcpyAsync, so that a chain of launches stays PDL
  // and nothing in the solve waits for a copy engine that a caller's bulk
  // transfers keep busy.
  template <typename T>
  void zero(T* u, size_t n) {
    const unsigned nb = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    launch(k_zero<T>, dim3(nb), dim3(256), 0, u, n);
  }
  template <typename T>
  void copy(const T* a, T* b, size_t n) {
    const unsigned nb = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
    launch(k_copy<T>, dim3(nb), dim3(256), 0, a, b, n);
  }

  int prof_begin(int l, int kind, double units) { return (!capturing && l == 0) ? c->prof_begin(kind, units) : -1; }

  template <typename T>
  void bc(Level& L, T* u, bool lwithdirichlet) {
    const int* b = B.b;
    bool xy = lwithdirichlet || b[0] >= 1 || b[1] >= 1 || b[2] >= 1 || b[3] >= 1;
    bool z = lwithdirichlet || b[4] >= 1 || b[5] >= 1;
    if (xy) { launch(k_bc_xy<T>, L.d.nz + 1, 256, 0, u, L.d.nx, L.d.ny, B, (int)lwithdirichlet); }
    if (z) {
      size_t nxy = (size_t)(L.d.nx + 3) * (L.d.ny + 3);
      { launch(k_bc_z<T>, cdiv(nxy, 256), 256, 0, u, L.d.nx, L.d.ny, L.d.nz, B, (int)lwithdirichlet); }
    }
  }

  SorCoef coef(const LevelDims& d) const {
    double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
    double cst = o->mgparam * 0.5 / (dxsqi + dysqi + dzsqi);
    return SorCoef{dxsqi * cst, dysqi * cst, dzsqi * cst, 1. - o->mgparam, o->mgparam};
  }

  template <typename T>
  void neumann_int(Level& L, T* phi) {
    if (!L.has_neumann_sub) return;
    for (int par = 0; par < 2; ++par) {
      DevSubgrid& S = L.sub[par];
      if (S.n) {
        launch(k_condbndymgint<T>, cdiv(S.n, 128), 128, 0, phi, L.d.nx, L.d.ny, L.d.nz, S.ijk, S.dels, S.n, B);
      }
    }
  }

  // Marks conductor nodes in the rhs array of level l.
  template <typename T>
  void box(int l) {
    Level& L = c->lv[l];
    int n = L.n_int + L.sub[0].n + L.sub[1].n;
    if (!n) return;
    launch(k_box<T>, cdiv(n, 128), 128, 0, Arr<T>::rhs(L), L.d.nx, L.d.ny, cond_args<T>(L), Arr<T>::srhs(L.sub[0]),
                                          Arr<T>::srhs(L.sub[1]));
  }

  // Whether one launch per half pass does all of sorpass3d's half pass on
  // level L (k_sor_bulk with its subgrid slices): no Neumann subgrid
  // points, and the boundary copy after each half pass is either empty
  // (all Dirichlet) or the periodic-z copy, which the kernel then does
  // itself by writing every updated node of planes 0, 1 and nz-1 to its
  // images. That write-through needs an even nz: with an odd nz the nodes
  // (i, j, 0) and (i, j, nz-1) have the same colour, and the first reads the
  // image of the second within the half pass.
  bool merged_ok(const Level& L) const {
    const int* b = B.b;
    const bool xy_dir = b[0] == 0 && b[1] == 0 && b[2] == 0 && b[3] == 0;
    const bool zper = b[4] == 2 && b[5] == 2, zdir = b[4] == 0 && b[5] == 0;
    return !L.has_neumann_sub && xy_dir && (zdir || (zper && L.d.nz % 2 == 0)) && L.d.nz >= 2;
  }

  // Whether the boundary copy after a residual or a prolongation on level L
  // is only the periodic-z copy (Dirichlet x and y, periodic z, nz >= 2),
  // which those kernels then do themselves by writing planes 0, 1 and nz-1
  // through to their images.
  bool zper_wt(const Level& L) const {
    const int* b = B.b;
    return b[0] == 0 && b[1] == 0 && b[2] == 0 && b[3] == 0 && b[4] == 2 && b[5] == 2 && L.d.nz >= 2;
  }

  // Whether the first red half sweep of level l can start from an
  // unzeroed phi and write all of it (k_sor_from_zero).
  bool from_zero_ok(int l) const { return o->downpasses >= 1 && merged_ok(c->lv[l]); }

  // sorpass3d (f3d_mgrid.F:1949-2093)
  template <typename T>
  void sorpass(int l, bool usev, bool phi_zero = false) {
    Level& L = c->lv[l];
    const SorCoef k = coef(L.d);
    T* phi = Arr<T>::phi(L);
    const T* rhs = Arr<T>::rhs(L);
    // one launch per half pass (bulk nodes and subgrid points together)
    const bool merged = merged_ok(L);
    const int wtz = (merged && B.b[4] == 2) ? 1 : 0;
    // cond_potmg sets the interior nodes to their voltage or, below the
    // finest level, to 0: a no-op on a phi that was just zeroed
    if (L.n_int && !(phi_zero && !usev)) {
      launch(k_interior<T>, cdiv(L.n_int, 128), 128, 0, phi, L.d.nx, L.d.ny, L.int_ijk, L.int_volt, L.n_int, usev,
                                                        L.d.nz, wtz);
    }
    neumann_int<T>(L, phi);
    const Ranges R = ranges(L.d, B.b, true);
    const int izmax = wtz ? std::min(R.izmax, L.d.nz - 1) : R.izmax;
    const int nyr = R.iymax - R.iymin + 1, nzr = izmax - R.izmin + 1;
    const int nhalf = (R.ixmax - R.ixmin) / 2 + 1;
    for (int parity = 0; parity < 2; ++parity) {
      int nsub = L.sub[parity].n;
      // Interior conductor nodes were set by k_interior at the start of the
      // pass; no kernel of the pass writes them unless Neumann subgrid
      // points copy values into their neighbours, so only then are they
      // set again after each half pass.
      CondArgs<T> ca = cond_args<T>(L);
      if (!L.has_neumann_sub) ca.nint = 0;
      constexpr int zpt = ZPlanes<T>::value;
      const bool bulk = nyr > 0 && nzr > 0 && nhalf > 0;
      dim3 blk(32, 8);
      const unsigned gx = bulk ? cdiv(nhalf, 32) : 1, gy = bulk ? cdiv(nyr, 8) : 1;
      const int nbz = bulk ? (int)cdiv(nzr, zpt) : 0;
      const int nspz = merged ? (int)cdiv((size_t)nsub, 256u * gx * gy) : 0;
      if (parity == 0 && phi_zero && !usev && merged) {
        // phi was not zeroed: this launch writes all of it (from_zero_ok).
        // It is not timed as WG_PROF_SOR0, which times k_sor_bulk only.
        constexpr int fz = 4;
        const unsigned fgx = cdiv(cdiv(L.d.nx + 3, 2), 32), fgy = cdiv(L.d.ny + 3, 8);
        const int fbz = (int)cdiv(L.d.nz + 3, fz);
        const int fspz = (int)cdiv((size_t)nsub, 256u * fgx * fgy);
        launch(k_sor_from_zero<T, fz>, dim3(fgx, fgy, fbz + fspz), blk, 0, phi, rhs, L.d.nx, L.d.ny, L.d.nz, R.ixmin,
               R.ixmax, R.iymin, R.iymax, R.izmin, izmax, (T)k.cx, (T)k.cy, (T)k.cz, (T)k.spm1, wtz, fbz, ca, B, k,
               o->lcndbndy);
      } else if (nbz + nspz > 0) {
        int pe = prof_begin(l, WG_PROF_SOR0, (double)L.nr);
        launch(k_sor_bulk<T, zpt>, dim3(gx, gy, nbz + nspz), blk, 0, 
            phi, rhs, L.d.nx, L.d.ny, R.ixmin, R.ixmax, R.iymin, R.iymax, R.izmin, izmax, parity, (T)k.cx, (T)k.cy,
            (T)k.cz, (T)k.spm1, L.d.nz, wtz, nbz, ca, B, k, (int)usev, o->lcndbndy);
        c->prof_end(pe);
      }
      if (!merged && nsub + ca.nint) {
        launch(k_special_sor<T>, cdiv(nsub + ca.nint, 128), 128, 0, phi, L.d.nx, L.d.ny, L.d.nz, ca, parity, B, k,
                                                                    (int)usev, (int)usev, o->lcndbndy);
      }
      neumann_int<T>(L, phi);
      if (!merged) bc<T>(L, phi, false);
    }
  }

  // residual3d into the padded res array of level l (MODE 0), or a norm only
  // (MODE 1), or into the FP32 rhs of level 0 (MODE 2).
  template <typename T, int MODE, typename TO>
  void residual(int l, const T* phi, TO* out, bool mgform2init, bool voltfac_on, unsigned long long* maxout) {
    Level& L = c->lv[l];
    const T* rhs = Arr<T>::rhs(L);
    const Ranges R = ranges(L.d, B.b, false);
    double dxsqi = 1. / (L.d.dx * L.d.dx), dysqi = 1. / (L.d.dy * L.d.dy), dzsqi = 1. / (L.d.dz * L.d.dz);
    double cst = 0.5 / (dxsqi + dysqi + dzsqi);
    const int g = (MODE == 0) ? 1 : 0;
    constexpr int zpt = ZPlanes<T>::value;
    dim3 blk(32, 8), grd(cdiv(L.d.nx + 1 + 2 * g, 32), cdiv(L.d.ny + 1 + 2 * g, 8), cdiv(L.d.nz + 1 + 2 * g, zpt));
    // interior conductor nodes are boxed, so the bulk kernel already stored
    // their zero residual
    CondArgs<T> ca = cond_args<T>(L);
    ca.nint = 0;
    int n = L.sub[0].n + L.sub[1].n;
    const int wt = (MODE == 0 && zper_wt(L)) ? 1 : 0;
    if (sizeof(T) == 4 && l > 0 && MODE == 0 && n && !L.has_neumann_sub) {
      // FP32, below the finest level: bulk and subgrid points in one launch
      // (the FP64 form of the merged kernel needs 76 registers and is slower)
      const int nbz = (int)grd.z;
      const int nspz = (int)cdiv((size_t)n, 256u * grd.x * grd.y);
      launch(k_residual_sp<T, MODE, TO, zpt>, dim3(grd.x, grd.y, nbz + nspz), blk, 0, phi, rhs, out, L.d.nx, L.d.ny,
             L.d.nz, R.ixmin, R.ixmax, R.iymin, R.iymax, R.izmin, R.izmax, (T)(dxsqi * o->mgparam * cst),
             (T)(dysqi * o->mgparam * cst), (T)(dzsqi * o->mgparam * cst), (T)o->mgparam, nbz, ca, B, dxsqi, dysqi,
             dzsqi, o->mgparam, (int)voltfac_on, (int)mgform2init, o->lcndbndy, maxout, wt);
      if (!wt) bc<TO>(L, (TO*)out, false);
      return;
    }
    {
      int pe = prof_begin(l, WG_PROF_RESID0, (double)L.nr);
      launch(k_residual<T, MODE, TO, zpt>, grd, blk, 0, phi, rhs, out, L.d.nx, L.d.ny, L.d.nz, R.ixmin, R.ixmax, R.iymin,
                                                  R.iymax, R.izmin, R.izmax, (T)(dxsqi * o->mgparam * cst),
                                                  (T)(dysqi * o->mgparam * cst), (T)(dzsqi * o->mgparam * cst),
                                                  (T)o->mgparam, maxout, wt);
      c->prof_end(pe);
    }
    if (n) {
      launch(k_special_res<T, MODE, TO>, cdiv(n, 128), 128, 0, phi, out, L.d.nx, L.d.ny, L.d.nz, ca, B,
                                                              dxsqi, dysqi, dzsqi, o->mgparam, (int)voltfac_on,
                                                              (int)mgform2init, o->lcndbndy, maxout, wt);
    }
    if (MODE == 0 && !wt) bc<TO>(L, (TO*)out, false);
  }

  // Everything vcycle(l) does below level l: the conductor marks of level
  // l+1, its phi zeroed unless the first half sweep writes all of it, and
  // vcycle(l+1).
  template <typename T>
  void coarse_region(int l) {
    Level& Lc = c->lv[l + 1];
    box<T>(l + 1);
    if (!from_zero_ok(l + 1)) zero(Arr<T>::phi(Lc), Lc.np);
    vcycle<T>(l + 1, false, true);
  }

  // For WG_PROF_COARSE: the region below level 0 replayed from a captured
  // graph launched with the solve's PDL setting, so that its CUDA-event time
  // is the time it takes inside a replayed V-cycle. (Profiling otherwise
  // launches kernel by kernel, and these small kernels would then wait on
  // the host's launches.) Recaptured when the options or conductors change.
  template <typename T>
  void coarse_from_graph() {
    const int gi = sizeof(T) == 8 ? 0 : 1;
    unsigned long long mp;
    memcpy(&mp, &o->mgparam, sizeof(mp));
    unsigned long long key = mp;
    const long long parts[] = {o->mgmaxlevels, o->downpasses, o->uppasses, o->lcndbndy, c->cond_version,
                               (long long)pdl_timed};
    for (long long x : parts) key = (key ^ (unsigned long long)x) * 0x100000001B3ull;
    key |= 1ull;
    if (!c->cgraph[gi] || c->cgraph_key[gi] != key) {
      if (c->cgraph[gi]) cudaGraphExecDestroy(c->cgraph[gi]);
      c->cgraph[gi] = nullptr;
      cudaError_t e = cudaSuccess;
      if (!c->cap_stream) e = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        if (lerr == cudaSuccess) lerr = e;
        return;
      }
      Solver G = *this;
      G.s = c->cap_stream;
      G.capturing = true;
      G.pdl = pdl_timed;
      const long long n0 = c->nlaunch;
      G.coarse_region<T>(0);
      cudaGraph_t g;
      e = cudaStreamEndCapture(c->cap_stream, &g);
      c->cgraph_kernels[gi] = c->nlaunch - n0;
      c->nlaunch = n0;
      if (G.lerr != cudaSuccess) e = G.lerr;
      if (e == cudaSuccess) {
        e = cudaGraphInstantiate(&c->cgraph[gi], g, 0);
        cudaGraphDestroy(g);
      }
      if (e != cudaSuccess) {
        c->cgraph[gi] = nullptr;
        if (lerr == cudaSuccess) lerr = e;
        return;
      }
      c->cgraph_key[gi] = key;
    }
    cudaError_t e = cudaGraphLaunch(c->cgraph[gi], s);
    if (e != cudaSuccess && lerr == cudaSuccess) lerr = e;
    c->nlaunch += c->cgraph_kernels[gi];
  }

  // vcycle (f3d_mgrid.F:1101-1591)
  template <typename T>
  // phi_zero: phi of level l is all zeros on entry
  void vcycle(int l, bool usev, bool phi_zero = false) {
    Level& L = c->lv[l];
    for (int i = 0; i < o->downpasses; ++i) sorpass<T>(l, usev, phi_zero && i == 0);
    const LevelDims& d = L.d;
    if (d.nx >= 4 && d.ny >= 4 && d.nz >= 4 && l < o->mgmaxlevels && l + 1 < (int)c->lv.size()) {
      residual<T, 0, T>(l, Arr<T>::phi(L), Arr<T>::res(L), false, usev, nullptr);
      Level& Lc = c->lv[l + 1];
      const LevelDims& dc = Lc.d;
      double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
      double dxcsqi = 1. / (dc.dx * dc.dx), dycsqi = 1. / (dc.dy * dc.dy), dzcsqi = 1. / (dc.dz * dc.dz);
      double ff = (dxsqi + dysqi + dzsqi) / (dxcsqi + dycsqi + dzcsqi);
      Ranges Rc = ranges(dc, B.b, false);
      dim3 blk(32, 8), grd(cdiv(dc.nx + 1, 32), cdiv(dc.ny + 1, 8), dc.nz + 1);
      int pr = prof_begin(l, WG_PROF_RESTRICT0, (double)L.nr);
      if (dc.nz == d.nz && L.rmax <= 3) {
        // z not coarsened: x-y windows only, several coarse planes per thread
        constexpr int zpt = ZPlanes<T>::value;
        dim3 grdxy(cdiv(dc.nx + 1, 32), cdiv(dc.ny + 1, 8), cdiv(dc.nz + 1, zpt));
        launch(k_restrict_xy<T, 3, zpt>, grdxy, blk, 0, Arr<T>::res(L), Arr<T>::rhs(Lc), d.nx, d.ny, dc.nx, dc.ny,
               dc.nz, Rc.ixmin, Rc.ixmax, Rc.iymin, Rc.iymax, Rc.izmin, Rc.izmax, L.rlo, L.rn, L.rw, ff);
      } else if (L.rmax <= 3) {
        launch(k_restrict<T, 3>, grd, blk, 0, Arr<T>::res(L), Arr<T>::rhs(Lc), d.nx, d.ny, dc.nx, dc.ny, Rc.ixmin,
                                             Rc.ixmax, Rc.iymin, Rc.iymax, Rc.izmin, Rc.izmax, L.rlo, L.rn, L.rw, ff);
      } else {
        launch(k_restrict<T, kRestrictTaps>, grd, blk, 0, Arr<T>::res(L), Arr<T>::rhs(Lc), d.nx, d.ny, dc.nx, dc.ny,
                                                         Rc.ixmin, Rc.ixmax, Rc.iymin, Rc.iymax, Rc.izmin, Rc.izmax,
                                                         L.rlo, L.rn, L.rw, ff);
      }
      c->prof_end(pr);
      int pc = (l == 0) ? prof_begin(0, WG_PROF_COARSE, (double)Lc.nr) : -1;
      if (pc >= 0)
        coarse_from_graph<T>();
      else
        coarse_region<T>(l);
      c->prof_end(pc);
      expand<T>(l);
      if (!zper_wt(L)) bc<T>(L, Arr<T>::phi(L), false);
    }
    for (int i = 0; i < o->uppasses; ++i) sorpass<T>(l, usev);
  }

  // expand3d (f3d_mgrid.F:1777-1947): adds level l+1's phi, interpolated,
  // to level l's phi
  template <typename T>
  void expand(int l) {
    Level& L = c->lv[l];
    Level& Lc = c->lv[l + 1];
    const LevelDims& d = L.d;
    const LevelDims& dc = Lc.d;
    Ranges R = ranges(d, B.b, false);
    // periodic images written by the kernel (zper_wt): plane nz is the
    // image of plane 0, not a node of its own
    const int wt = zper_wt(L) ? 1 : 0;
    if (wt) R.izmax = std::min(R.izmax, d.nz - 1);
    constexpr int zpt = ZPlanes<T>::value;
    dim3 blk(32, 8);
    dim3 grd2(cdiv(R.ixmax - R.ixmin + 1, 32), cdiv(R.iymax - R.iymin + 1, 8), cdiv(R.izmax - R.izmin + 1, zpt));
    if (R.ixmax >= R.ixmin && R.iymax >= R.iymin && R.izmax >= R.izmin) {
      int pe = prof_begin(l, WG_PROF_EXPAND0, (double)L.nr);
      if (dc.nz == d.nz)
        launch(k_expand<T, zpt, false>, grd2, blk, 0, Arr<T>::phi(L), Arr<T>::phi(Lc), d.nx, d.ny, dc.nx, dc.ny,
                                                     R.ixmin, R.ixmax, R.iymin, R.iymax, R.izmin, R.izmax, L.ej, L.ew,
                                                     d.nz, wt);
      else
        launch(k_expand<T, zpt, true>, grd2, blk, 0, Arr<T>::phi(L), Arr<T>::phi(Lc), d.nx, d.ny, dc.nx, dc.ny,
                                                    R.ixmin, R.ixmax, R.iymin, R.iymax, R.izmin, R.izmax, L.ej, L.ew,
                                                    d.nz, wt);
      c->prof_end(pe);
    }
  }

  // The deepest level the recursion of vcycle and fullmultigrid3dsolve
  // reaches from level 0.
  int deepest() const {
    int l = 0;
    for (;;) {
      const LevelDims& d = c->lv[l].d;
      if (d.nx >= 4 && d.ny >= 4 && d.nz >= 4 && l < o->mgmaxlevels && l + 1 < (int)c->lv.size())
        ++l;
      else
        return l;
    }
  }

  // fullmultigrid3dsolve (f3d_mgrid.F:502-945), downward part: the source of
  // every level down to lmax, restricted from the scaled rho of level 0
  // (rho has no guard cells there, hence the ng = 0 tables).
  void fmg_restrict(int lmax) {
    for (int l = 0; l < lmax; ++l) {
      Level& L = c->lv[l];
      Level& Lc = c->lv[l + 1];
      const LevelDims& d = L.d;
      const LevelDims& dc = Lc.d;
      dim3 blk(32, 8);
      { launch(k_pad_copy, dim3(cdiv(d.nx + 1, 32), cdiv(d.ny + 1, 8), d.nz + 1), blk, 0, L.rhs, L.res, d.nx, d.ny); }
      double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
      double dxcsqi = 1. / (dc.dx * dc.dx), dycsqi = 1. / (dc.dy * dc.dy), dzcsqi = 1. / (dc.dz * dc.dz);
      double ff = (dxsqi + dysqi + dzsqi) / (dxcsqi + dycsqi + dzcsqi);
      Ranges Rc = ranges(dc, B.b, false);
      dim3 grd(cdiv(dc.nx + 1, 32), cdiv(dc.ny + 1, 8), dc.nz + 1);
      if (L.rmax0 <= 3)
        launch(k_restrict<double, 3>, grd, blk, 0, L.res, Lc.rhs, d.nx, d.ny, dc.nx, dc.ny, Rc.ixmin, Rc.ixmax,
                                                  Rc.iymin, Rc.iymax, Rc.izmin, Rc.izmax, L.rlo0, L.rn0, L.rw0, ff);
      else
        launch(k_restrict<double, kRestrictTaps>, grd, blk, 0, L.res, Lc.rhs, d.nx, d.ny, dc.nx, dc.ny, Rc.ixmin,
                                                              Rc.ixmax, Rc.iymin, Rc.iymax, Rc.izmin, Rc.izmax,
                                                              L.rlo0, L.rn0, L.rw0, ff);
    }
  }

  // Upward part: from the coarsest level (phi = 0) to level 1, each level's
  // phi is the expanded phi of the next coarser one followed by nvc
  // V-cycles without a convergence test (voltages zero below level 0, as in
  // every V-cycle); level 0 gets the expansion only. With a single level
  // phi is left as it is.
  int fmg_up(int lmax, int nvc) {
    for (int l = lmax; l >= 0; --l) {
      Level& L = c->lv[l];
      if (l < lmax) {
        zero(L.phi, L.np);
        expand<double>(l);
      } else if (l > 0) {
        zero(L.phi, L.np);
      }
      bc<double>(L, L.phi, false);
      if (l == 0) break;
      box<double>(l);
      for (int it = 0; it < nvc; ++it) vcycle<double>(l, false);
      bc<double>(L, L.phi, true);
    }
    return WG_OK;
  }

  // reduction slot area of quantity q: 0 max|dphi|, 1 max|res|, 2 max|rhs|
  unsigned long long* slotq(int q) { return c->dslot + (size_t)q * kRedQ; }
  int clear_slots(int q) {
    zero(slotq(q), (size_t)kRedQ);
    return WG_OK;
  }

  int fetch_red(double* out, int n) {
    { launch(k_fold_max, 1, 96, 0, c->dslot, c->dred, 3); }
    { launch(k_publish, 1, 32, 0, c->dred, c->hred_dev, 5); }
    WG_TRY_CUDA(cudaStreamSynchronize(s));
    WG_TRY_CUDA(lerr);
    for (int i = 0; i < n; ++i) {
      unsigned long long v = c->hred[i];
      double dv;
      memcpy(&dv, &v, sizeof(double));
      out[i] = dv;
    }
    return WG_OK;
  }

};

// The V-cycle of precision T from a captured CUDA graph (recaptured when the
// options or the conductor arrays change), or launched kernel by kernel.
template <typename T>
int run_vcycle(Solver& S, bool usev) {
  wg_ctx* c = S.c;
  const wg_solve_opts* o = S.o;
  if (!(o->flags & WG_SOLVE_GRAPH) || c->prof_mask) {
    S.vcycle<T>(0, usev, !usev);
    return WG_OK;
  }
  const int gi = sizeof(T) == 8 ? 0 : 1;
  unsigned long long mp;
  memcpy(&mp, &o->mgparam, sizeof(mp));
  unsigned long long key = mp ^ ((unsigned long long)o->mgmaxlevels << 1) ^ ((unsigned long long)o->downpasses << 9) ^
                           ((unsigned long long)o->uppasses << 17) ^ ((unsigned long long)o->lcndbndy << 25) ^
                           ((unsigned long long)usev << 28) ^
                           ((unsigned long long)S.pdl << 29) ^
                           ((unsigned long long)c->cond_version << 32);
  if (!c->vgraph[gi] || c->vgraph_key[gi] != key) {
    if (c->vgraph[gi]) cudaGraphExecDestroy(c->vgraph[gi]);
    c->vgraph[gi] = nullptr;
    if (!c->cap_stream) WG_TRY_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
    Solver G = S;
    G.s = c->cap_stream;
    G.capturing = true;
    const long long n0 = c->nlaunch;
    cudaGraph_t g;
    WG_TRY_CUDA(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
    G.vcycle<T>(0, usev, !usev);
    cudaError_t ce = cudaStreamEndCapture(c->cap_stream, &g);
    if (G.lerr != cudaSuccess) ce = G.lerr;
    WG_TRY_CUDA(ce);
    cudaError_t e = cudaGraphInstantiate(&c->vgraph[gi], g, 0);
    cudaGraphDestroy(g);
    WG_TRY_CUDA(e);
    c->vgraph_key[gi] = key;
    c->vgraph_kernels[gi] = c->nlaunch - n0;
    c->nlaunch = n0;
  }
  WG_TRY_CUDA(cudaGraphLaunch(c->vgraph[gi], S.s));
  c->nlaunch += c->vgraph_kernels[gi];
  return WG_OK;
}


}  // namespace

int ensure_fp32(wg_ctx* c);

int solve(wg_ctx* c, const wg_solve_opts* o, wg_solve_stats* st) {
  if (!o || !st) { set_error("wg_solve: null options or stats"); return WG_EINVAL; }
  if (!(o->mgparam > 0. && o->mgparam < 2.) || o->mgmaxiters < 0 || o->downpasses < 0 || o->uppasses < 0 ||
      (o->precision != 0 && o->precision != 1) || (o->tolkind != 0 && o->tolkind != 1) || o->mgmaxvcycles < 0) {
    set_error("wg_solve: invalid options");
    return WG_EINVAL;
  }
  if (o->precision == 1) {
    WG_TRY(ensure_fp32(c));
    for (Level& L : c->lv)
      for (DevSubgrid& S : L.sub)
        if ((uint32_t)S.n > Box<float>::kMax || (uint32_t)L.n_int > Box<float>::kMax) {
          set_error("wg_solve: more than 4194303 conductor points of one kind on a level (FP32 limit)");
          return WG_ETOOLARGE;
        }
  }
  Solver S{c, o, {}, c->stream, false};
  for (int k = 0; k < 6; ++k) S.B.b[k] = c->grid.bounds[k];
  S.pdl_timed = (o->flags & WG_SOLVE_PDL) != 0;
  S.pdl = S.pdl_timed && !c->prof_mask;
  cudaStream_t s = c->stream;
  Level& L0 = c->lv[0];
  const LevelDims& d = L0.d;
  double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
  double reps0c = o->mgparam / (kEps0 * 2. * (dxsqi + dysqi + dzsqi));
  S.zero(c->dred, (size_t)4);
  S.zero(c->dslot, (size_t)3 * kRedQ);
  { S.launch(k_scale_rhs, cdiv(L0.nr, 256), 256, 0, c->rho, L0.rhs, L0.nr, reps0c, S.slotq(2), c->dred + 3); }
  const bool fmg = o->mgmaxvcycles > 0;
  const int lmax = fmg ? S.deepest() : 0;
  if (fmg) S.fmg_restrict(lmax);
  S.box<double>(0);
  S.bc<double>(L0, L0.phi, false);
  dim3 blk(32, 8), grdn(cdiv(d.nx + 1, 32), cdiv(d.ny + 1, 8), d.nz + 1);
  int it = 0;
  double err = 2. * o->mgtol + 1., relres = -1.;
  bool conv = false;
  double rv[4];
  WG_TRY(S.fetch_red(rv, 3));
  if (c->hred[3] & 2ull) {
    set_error("wg_solve: rho contains NaN or Inf");
    return WG_EINVAL;
  }
  if (c->hred[4]) {
    S.zero(c->dred + 4, (size_t)1);
    set_error("wg_solve: the last chunked deposit overflowed the fixed-point accumulator (more than 65536 full "
              "particle weights on one node)");
    return WG_EOVERFLOW;
  }
  if (fmg) WG_TRY(S.fmg_up(lmax, o->mgmaxvcycles));
  if (o->precision == 0) {
    for (;;) {
      if (o->tolkind == 1) {
        WG_TRY(S.clear_slots(1));
        S.residual<double, 1, double>(0, L0.phi, nullptr, false, true, S.slotq(1));
        WG_TRY(S.fetch_red(rv, 3));
        relres = rv[2] > 0. ? rv[1] / rv[2] : rv[1];
        if (relres <= o->mgtol) { conv = true; break; }
      }
      if (it >= o->mgmaxiters) break;
      if (o->tolkind == 0)
        S.copy(L0.phi, c->phisave, L0.np);
      WG_TRY(run_vcycle<double>(S, true));
      it += 1;
      if (o->tolkind == 0) {
        WG_TRY(S.clear_slots(0));
        { S.launch(k_maxdiff, grdn, blk, 0, c->phisave, L0.phi, d.nx, d.ny, S.slotq(0)); }
        WG_TRY(S.fetch_red(rv, 1));
        err = rv[0];
        if (!(err > o->mgtol)) { conv = true; break; }
      }
    }
  } else {
    for (;;) {
      // residual of the FP64 solution with actual voltages (mgform = 2 set-up)
      if (L0.n_int) {
        S.launch(k_interior<double>, cdiv(L0.n_int, 128), 128, 0, L0.phi, d.nx, d.ny, L0.int_ijk, L0.int_volt, L0.n_int, 1, 0, 0);
      }
      S.neumann_int<double>(L0, L0.phi);
      WG_TRY(S.clear_slots(1));
      S.residual<double, 2, float>(0, L0.phi, L0.rhsf, true, true, S.slotq(1));
      if (o->tolkind == 1 || it >= o->mgmaxiters) {
        WG_TRY(S.fetch_red(rv, 3));
        relres = rv[2] > 0. ? rv[1] / rv[2] : rv[1];
        if (o->tolkind == 1 && relres <= o->mgtol) { conv = true; break; }
      }
      if (it >= o->mgmaxiters) break;
      S.box<float>(0);
      if (!S.from_zero_ok(0)) S.zero(L0.phif, L0.np);
      WG_TRY(run_vcycle<float>(S, false));
      WG_TRY(S.clear_slots(0));
      {
        dim3 grdc(cdiv(d.nx + 3, 32), cdiv(d.ny + 3, 8), cdiv(d.nz + 3, kCorrPlanes));
        int pe = S.prof_begin(0, WG_PROF_CORR, (double)L0.nr);
        S.launch(k_add_corr, grdc, blk, 0, L0.phi, L0.phif, d.nx, d.ny, d.nz, S.slotq(0));
        c->prof_end(pe);
      }
      S.bc<double>(L0, L0.phi, false);
      it += 1;
      if (o->tolkind == 0) {
        WG_TRY(S.fetch_red(rv, 1));
        err = rv[0];
        if (!(err > o->mgtol)) { conv = true; break; }
      }
    }
  }
  S.bc<double>(L0, L0.phi, true);
  WG_TRY_CUDA(S.lerr);
  WG_TRY_CUDA(cudaGetLastError());
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  st->mgiters = it;
  st->converged = conv ? 1 : 0;
  st->mgerror = (o->tolkind == 0) ? err : -1.;
  st->relres = relres;
  return WG_OK;
}

int relresidual(wg_ctx* c, double mgparam, double* out) {
  wg_solve_opts o{mgparam, 0., 0, 101, 1, 1, 1, 0, 1, 0};
  Solver S{c, &o, {}, c->stream, false};
  for (int k = 0; k < 6; ++k) S.B.b[k] = c->grid.bounds[k];
  cudaStream_t s = c->stream;
  Level& L0 = c->lv[0];
  const LevelDims& d = L0.d;
  double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
  double reps0c = mgparam / (kEps0 * 2. * (dxsqi + dysqi + dzsqi));
  S.zero(c->dred, (size_t)4);
  S.zero(c->dslot, (size_t)3 * kRedQ);
  { ++c->nlaunch; k_scale_rhs<<<cdiv(L0.nr, 256), 256, 0, s>>>(c->rho, L0.rhs, L0.nr, reps0c, S.slotq(2), c->dred + 3); }
  S.box<double>(0);
  // residual of a copy with the conductor voltages imposed, as the solver sees it
  S.copy(L0.phi, c->phisave, L0.np);
  if (L0.n_int) {
    ++c->nlaunch;
    k_interior<double><<<cdiv(L0.n_int, 128), 128, 0, s>>>(c->phisave, d.nx, d.ny, L0.int_ijk, L0.int_volt, L0.n_int, 1);
  }
  S.residual<double, 1, double>(0, c->phisave, nullptr, false, true, S.slotq(1));
  double rv[4];
  WG_TRY(S.fetch_red(rv, 3));
  *out = rv[2] > 0. ? rv[1] / rv[2] : rv[1];
  return WG_OK;
}

// Residual field of the current phi on the finest level into out (rho
// layout, device memory): rhs - A phi with the conductor voltages imposed,
// the right-hand side of the correction equation of the residual-correction
// form (mgform = 2, f3d_mgrid.F:340-358). Zero at conductor and boundary
// nodes that are not updated.
int residual_field(wg_ctx* c, double mgparam, double* out) {
  wg_solve_opts o{mgparam, 0., 0, 101, 1, 1, 1, 0, 1, 0};
  Solver S{c, &o, {}, c->stream, false};
  for (int k = 0; k < 6; ++k) S.B.b[k] = c->grid.bounds[k];
  cudaStream_t s = c->stream;
  Level& L0 = c->lv[0];
  const LevelDims& d = L0.d;
  double dxsqi = 1. / (d.dx * d.dx), dysqi = 1. / (d.dy * d.dy), dzsqi = 1. / (d.dz * d.dz);
  double reps0c = mgparam / (kEps0 * 2. * (dxsqi + dysqi + dzsqi));
  S.zero(c->dred, (size_t)4);
  S.zero(c->dslot, (size_t)3 * kRedQ);
  { ++c->nlaunch; k_scale_rhs<<<cdiv(L0.nr, 256), 256, 0, s>>>(c->rho, L0.rhs, L0.nr, reps0c, S.slotq(2), c->dred + 3); }
  S.box<double>(0);
  S.copy(L0.phi, c->phisave, L0.np);
  if (L0.n_int) {
    ++c->nlaunch;
    k_interior<double><<<cdiv(L0.n_int, 128), 128, 0, s>>>(c->phisave, d.nx, d.ny, L0.int_ijk, L0.int_volt, L0.n_int, 1);
  }
  S.residual<double, 2, double>(0, c->phisave, out, true, true, nullptr);
  WG_TRY_CUDA(cudaGetLastError());
  return WG_OK;
}

// getese3dfromrhophi (dw3d.F:708-777) without symmetry, in the reference's
// summation order: per (x, y) column over z, then over y into row 0, then
// over x; the result is bit-identical to the serial loops.
__global__ void k_ese_cols(const double* __restrict__ rho, const double* __restrict__ phi, int nx, int ny, int nz,
                           double* __restrict__ scr) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y;
  if (ix > nx) return;
  const size_t sy = nx + 3, sz = (size_t)(nx + 3) * (ny + 3), rz = (size_t)(nx + 1) * (ny + 1);
  const double* r = rho + ix + (size_t)(nx + 1) * iy;
  const double* p = phi + (ix + 1) + sy * (iy + 1) + sz;
  double c = 0.;
  for (int iz = 0; iz <= nz; ++iz) c = c + r[rz * iz] * p[sz * iz];
  scr[ix + (size_t)(nx + 1) * iy] = c;
}

__global__ void k_ese_rows(double* __restrict__ scr, int nx, int ny, double dvol, double* __restrict__ out) {
  for (int ix = threadIdx.x; ix <= nx; ix += blockDim.x) {
    double c = scr[ix];
    for (int iy = 1; iy <= ny; ++iy) c = c + scr[ix + (size_t)(nx + 1) * iy];
    scr[ix] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ese = 0.;
    for (int ix = 0; ix <= nx; ++ix) ese = ese + scr[ix];
    *out = dvol * 0.5 * ese;
  }
}

int field_energy(wg_ctx* c, double* out) {
  cudaStream_t s = c->stream;
  const LevelDims& d = c->lv[0].d;
  ++c->nlaunch;
  k_ese_cols<<<dim3(cdiv(d.nx + 1, 128), d.ny + 1), 128, 0, s>>>(c->rho, c->lv[0].phi, d.nx, d.ny, d.nz, c->dese);
  ++c->nlaunch;
  k_ese_rows<<<1, 256, 0, s>>>(c->dese, d.nx, d.ny, c->dx * c->dy * c->dz, c->dese + (size_t)(d.nx + 1) * (d.ny + 1));
  WG_TRY_CUDA(cudaGetLastError());
  WG_TRY_CUDA(cudaMemcpyAsync(out, c->dese + (size_t)(d.nx + 1) * (d.ny + 1), sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  WG_TRY_CUDA(cudaStreamSynchronize(s));
  return WG_OK;
}

// Per-kernel attributes set once per context (none needed at present).
int configure_kernels() { return WG_OK; }

}  // namespace wg
