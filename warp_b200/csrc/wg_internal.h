// Internal declarations shared by the warp_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/warp_b200.h"

namespace wg {

void set_error(const std::string& msg);

#define WG_TRY_CUDA(expr)                                                   \
  do {                                                                      \
    cudaError_t e_ = (expr);                                                \
    if (e_ != cudaSuccess) {                                                \
      ::wg::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));  \
      return WG_ECUDA;                                                      \
    }                                                                       \
  } while (0)

#define WG_TRY(expr)            \
  do {                          \
    int r_ = (expr);            \
    if (r_ != WG_OK) return r_; \
  } while (0)

// Host-side conductor lists (ConductorType, f3d.v:105-164), all levels.
struct HostConductors {
  std::vector<int32_t> int_indx;  // 3 per point
  std::vector<double> int_volt;
  std::vector<int32_t> int_level;
  std::vector<int32_t> sub_indx;  // 3 per point
  std::vector<double> sub_dels;   // 6 per point
  std::vector<double> sub_volt;   // 6 per point
  std::vector<int32_t> sub_level;
  // after finalize: points sorted by level; even and odd separated
  std::vector<int32_t> istart_int, istart_even, istart_odd;
  std::vector<int32_t> even_indx, odd_indx;
  std::vector<double> even_dels, odd_dels, even_volt, odd_volt;
  std::vector<int32_t> even_level, odd_level;
  bool finalized = false;
};

struct LevelDims {
  int nx, ny, nz;
  double dx, dy, dz;
};

// Device conductor data of one level (one parity for subgrid lists).
// The rhs arrays of a level hold, at every conductor node, a NaN whose
// payload is the node's index in its list (sign bit set for interior
// points); the node's real rhs value is kept here in `rhs`/`rhsf`.
struct DevSubgrid {
  int n = 0;
  int32_t* ijk = nullptr;   // 3 per point
  double* dels = nullptr;   // 6 per point
  double* volt = nullptr;   // 6 per point
  double* rhs = nullptr;    // rhs value at the point (FP64 levels)
  float* rhsf = nullptr;    // rhs value at the point (FP32 levels)
};

struct Level {
  LevelDims d;
  size_t np = 0;  // (nx+3)(ny+3)(nz+3)
  size_t nr = 0;  // (nx+1)(ny+1)(nz+1)
  double* phi = nullptr;
  double* rhs = nullptr;
  double* res = nullptr;
  float* phif = nullptr;
  float* rhsf = nullptr;
  float* resf = nullptr;
  int n_int = 0;
  int32_t* int_ijk = nullptr;
  double* int_volt = nullptr;
  DevSubgrid sub[2];   // 0 even, 1 odd
  bool has_neumann_sub = false;
  // prolongation from the next coarser level: per fine index i = -1..n+1
  // (stored at i+1) the coarse cell j = (i*nc)/n and weight 1.*(i*nc)/n - j,
  // x entries first, then y, then z
  int32_t* ej = nullptr;
  double* ew = nullptr;
  // restriction into the next coarser level: per coarse index ic = 0..nc
  // the first fine index, the tap count (<= kRestrictTaps) and the tap
  // weights 1 - |ic - i*nc/n|, x entries first, then y, then z
  int32_t* rlo = nullptr;
  int32_t* rn = nullptr;
  double* rw = nullptr;
  int rmax = 0;  // widest x or y window
  // the same for a source without guard cells (rho in the full multigrid)
  int32_t* rlo0 = nullptr;
  int32_t* rn0 = nullptr;
  double* rw0 = nullptr;
  int rmax0 = 0;
};

constexpr int kRestrictTaps = 4;
// icgrid value of a level-0 conductor interior node (the reference's nmax+1)
constexpr int kIcInterior = 0x7fffffff;

std::vector<LevelDims> mglevels(int nx, int ny, int nz, double dx, double dy, double dz);

// Conductor generation and checking (wg_conductors.cpp).
int add_shape(HostConductors& C, const std::vector<LevelDims>& lv, double xmmin, double ymmin, double zmmin,
              int kind, double radius, double length, double voltage, double xcent, double ycent, double zcent,
              int condid, double dfill);
int finalize_conductors(HostConductors& C, const std::vector<LevelDims>& lv);

}  // namespace wg

struct wg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  wg_grid grid;
  double dx, dy, dz;
  std::vector<wg::Level> lv;
  wg::HostConductors cond;
  // level-0 work arrays
  double* phisave = nullptr;          // copy of phi at the start of a V-cycle
  double* rho = nullptr;              // user-visible rho (Fortran layout)
  unsigned long long* racc = nullptr; // fixed-point deposit accumulator
  // reductions: [0] max|dphi| bits, [1] max|res| bits, [2] max|rhs| bits, [3] flags,
  // [4] accumulator overflow of the last chunked deposit (reported by wg_solve)
  unsigned long long* dred = nullptr;
  unsigned long long* dslot = nullptr; // per-block max slots of [0..2], folded into dred
  unsigned long long* hred = nullptr;      // mapped pinned host copy, written by kernels
  unsigned long long* hred_dev = nullptr;  // device address of hred
  double* dmom = nullptr;              // moment partial sums
  double* dese = nullptr;              // field-energy row sums ((nx+1)(ny+1) + 1)
  double* zmom = nullptr;              // z-moment sums (33 global, then 33 per plane)
  size_t zmom_n = 0;
  int mom_blocks = 0;
  // lattice tables
  double* czs = nullptr;
  double* cze = nullptr;
  double* cdb = nullptr;
  int nzl = -1;
  double zlmin = 0., dzl = 1.;
  bool have_fp32 = false;
  // chunked deposit (wg_deposit_begin/add/end): open, and the q*w/(dx dy dz)
  // that every piece shares
  bool dep_open = false;
  bool dep_gg_set = false;
  double dep_gg = 0.;
  // lcorrectede: E next to conductors from the subgrid data
  int correctede = 0;
  int* icgrid = nullptr;                 // level-0 nodes: 0 vacuum, kIcInterior, +/- (subgrid index + 1)
  double* ef0[2] = {nullptr, nullptr};   // efield0 of the level-0 even/odd subgrid points, 3 per point
  double* efd[2] = {nullptr, nullptr};   // efieldd, 6 per point
  long long icgrid_version = 0;          // cond_version the icgrid was built for
  // kernels launched by this context (cumulative; a graph replay counts its kernels)
  long long nlaunch = 0;
  // captured V-cycles (index 0: FP64, 1: FP32), valid for vgraph_key
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t vgraph[2] = {nullptr, nullptr};
  unsigned long long vgraph_key[2] = {0ull, 0ull};
  long long vgraph_kernels[2] = {0, 0};
  // the work below level 0 of a V-cycle, captured for WG_PROF_COARSE timing
  cudaGraphExec_t cgraph[2] = {nullptr, nullptr};
  unsigned long long cgraph_key[2] = {0ull, 0ull};
  long long cgraph_kernels[2] = {0, 0};
  long long cond_version = 1;  // bumped whenever device conductor arrays change
  // node fields of the FP32 push (k_enode), (nx+1)(ny+1)(nz+1) float4
  float4* enode = nullptr;
  size_t enode_n = 0;
  // CUDA-event timing of selected kernel kinds (WG_PROF_* bits)
  int prof_mask = 0;
  std::vector<cudaEvent_t> prof_ev;  // start/stop pairs
  std::vector<int> prof_kind;
  std::vector<double> prof_units;
  size_t prof_used = 0;

  // Records a start event for a launch of `kind`; returns the pair index or -1.
  int prof_begin(int kind, double units) {
    if (!(prof_mask & (1 << kind)) || prof_used >= prof_kind.size()) return -1;
    size_t i = prof_used++;
    prof_kind[i] = kind;
    prof_units[i] = units;
    cudaEventRecord(prof_ev[2 * i], stream);
    return (int)i;
  }
  void prof_end(int i) {
    if (i >= 0) cudaEventRecord(prof_ev[2 * (size_t)i + 1], stream);
  }
};
