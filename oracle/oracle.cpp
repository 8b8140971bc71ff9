// CPU oracle for the 3D electrostatic PIC step of WARP.
//
// TEST INFRASTRUCTURE ONLY. This file is a plain FP64 restatement of the
// reference Fortran, used by the test suite, by __graft_entry__.smoke() and by
// the CPU-baseline leg of bench.py as the checker. The product (warp_b200)
// never links, loads or calls it.
//
// Parity pin: the multigrid part is pinned against the reference's own
// known-answer test (warp_test/MutltiGrid3D_test.py with
// warp_test/fieldsolvertesttools.py: discrete manufactured solution, every
// boundary combination, error < 1e-10 at mgtol = 1e-12). The reference itself
// cannot be compiled here (Fortran + Forthon, no Fortran compiler), so no
// reference-produced vectors exist; the conductor stencil, deposit, gather and
// push are pinned by this restatement plus physics invariants.
//
// Arrays use the reference's Fortran layout, x fastest:
//   phi(-1:nx+1,-1:ny+1,-1:nz+1)   (nxguardphi = 1)
//   rho(0:nx,0:ny,0:nz)            (nxguardrho = 0)
// Conductor data uses the ConductorType layout of pywarp90/f3d.v:105-164.
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off, no fast-math).
//
// Loops whose iterations are independent (the red-black sweeps, residual,
// restriction, prolongation, gather, push and the maxima) run on all host
// threads; their results do not depend on the thread count. The deposit runs
// over z slabs in two phases; its sums on the planes shared by two slabs are
// ordered by slab, so its last bits depend on the thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <thread>
#include <vector>

namespace {

// Host threads for the loops whose iterations are independent (the CPU
// baseline uses every core of the host). ORACLE_THREADS sets the count;
// default: all hardware threads.
int nthreads() {
  static const int n = [] {
    const char* e = std::getenv("ORACLE_THREADS");
    int v = e ? std::atoi(e) : 0;
    if (v <= 0) v = (int)std::thread::hardware_concurrency();
    return std::max(1, v);
  }();
  return n;
}

// f(i) for i in [lo, hi), split into contiguous ranges over the threads;
// serial when the loop holds less than kParMin units of work (grain = work
// units per iteration, e.g. the nodes of a plane).
constexpr int64_t kParMin = 1 << 17;

template <typename F>
void par_for(int64_t lo, int64_t hi, F f, int64_t grain = 1) {
  const int64_t n = hi - lo;
  int nt = nthreads();
  if (nt <= 1 || n < 2 || n * grain < kParMin) {
    for (int64_t i = lo; i < hi; ++i) f(i);
    return;
  }
  nt = (int)std::min<int64_t>(nt, n);
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      const int64_t a = lo + n * t / nt, b = lo + n * (t + 1) / nt;
      for (int64_t i = a; i < b; ++i) f(i);
    });
  for (auto& x : th) x.join();
}

// max over i in [lo, hi) of f(i) (non-negative values), in parallel
template <typename F>
double par_max(int64_t lo, int64_t hi, F f, int64_t grain = 1) {
  if ((hi - lo) * grain < kParMin || nthreads() <= 1) {
    double m = 0.;
    for (int64_t i = lo; i < hi; ++i) m = std::max(m, f(i));
    return m;
  }
  const int nt = std::max(1, (int)std::min<int64_t>(nthreads(), std::max<int64_t>(1, hi - lo)));
  std::vector<double> part(nt, 0.);
  par_for(0, nt, [&](int64_t t) {
    const int64_t n = hi - lo, a = lo + n * t / nt, b = lo + n * (t + 1) / nt;
    double m = 0.;
    for (int64_t i = a; i < b; ++i) m = std::max(m, f(i));
    part[t] = m;
  }, kParMin);
  double m = 0.;
  for (double v : part) m = std::max(m, v);
  return m;
}

const double LARGEPOS = 1.0e36;   // pywarp90/top.h:3
const double SMALLPOS = 1.0e-36;  // pywarp90/top.h:4
const double PI = 3.14159265358979323;
const double CLIGHT = 2.99792458e+8;
const double MU0 = 4. * PI * 1.e-7;               // pywarp90/top.F:380
const double EPS0 = 1. / (MU0 * CLIGHT * CLIGHT);  // pywarp90/top.F:384

struct Level {
  int nx, ny, nz;
  double dx, dy, dz;
};

// getnextcoarselevel3d, pywarp90/f3d_mgrid.F:3601-3652 (mgcoarsening = 2).
void next_coarse(const Level& f, Level& c) {
  c.nx = (f.nx + 1) / 2;
  if (c.nx % 2 == 1) c.nx += 1;
  c.ny = (f.ny + 1) / 2;
  if (c.ny % 2 == 1) c.ny += 1;
  c.nz = (f.nz + 1) / 2;
  if (c.nz % 2 == 1) c.nz += 1;
  double mingridsize = std::min(f.dx, f.dy);
  mingridsize = std::min(mingridsize, f.dz);
  if (f.dx > 4. / 3. * mingridsize) c.nx = f.nx;
  if (f.dy > 4. / 3. * mingridsize) c.ny = f.ny;
  if (f.dz > 4. / 3. * mingridsize) c.nz = f.nz;
  c.dx = f.dx * f.nx / c.nx;
  c.dy = (c.ny == 0) ? c.dx : f.dy * f.ny / c.ny;
  c.dz = f.dz * f.nz / c.nz;
}

// getmglevels, pywarp90/f3d_mgrid.F:3654-3845 (serial branch).
std::vector<Level> mglevels(int nx, int ny, int nz, double dx, double dy, double dz) {
  std::vector<Level> lv;
  Level f{nx, ny, nz, dx, dy, dz};
  for (int lev = 0;; ++lev) {
    lv.push_back(f);
    if (f.nx < 4 || (f.ny < 4 && f.ny > 0) || f.nz < 4 || lev == 100) break;
    Level c;
    next_coarse(f, c);
    f = c;
  }
  return lv;
}

// ---------------------------------------------------------------------------
// Conductor data (ConductorType, pywarp90/f3d.v:105-164)
// ---------------------------------------------------------------------------
struct Interior {
  std::vector<int> indx;  // 3 per point
  std::vector<double> volt;
  std::vector<int> numb;
  std::vector<int> ilevel;
  std::vector<int> istart;  // per level, 0-based, size levels+1
  size_t n() const { return volt.size(); }
};
struct Subgrid {
  std::vector<int> indx;     // 3 per point
  std::vector<double> dels;  // 6 per point: mx,px,my,py,mz,pz
  std::vector<double> volt;  // 6 per point
  std::vector<int> numb;     // 6 per point
  std::vector<int> ilevel;
  std::vector<double> prevphi;
  std::vector<int> istart;
  size_t n() const { return ilevel.size(); }
};
struct Conductors {
  Interior interior;
  Subgrid even, odd;
  int levels = 0;
  std::vector<Level> lv;
};

struct Grid {
  int nx, ny, nz;
  double xmmin, ymmin, zmmin, dx, dy, dz;
  int bounds[6];
};

inline size_t pidx(int nx, int ny, int ix, int iy, int iz) {
  return (size_t)(ix + 1) + (size_t)(nx + 3) * ((size_t)(iy + 1) + (size_t)(ny + 3) * (size_t)(iz + 1));
}
inline size_t ridx(int nx, int ny, int ix, int iy, int iz) {
  return (size_t)ix + (size_t)(nx + 1) * ((size_t)iy + (size_t)(ny + 1) * (size_t)iz);
}

// Cell index and fraction of a particle coordinate s = (x - xmin)/dx, as
// int() truncation followed by s - i (w3d.F:7820-7830). The index is clamped
// to [0, n-1] so that a particle sitting exactly on the upper grid edge
// deposits into the last cell with fraction 1 instead of writing past the
// array (the reference writes a zero weight one node past the edge there).
inline void cellfrac(double s, int n, int& i, double& f) {
  i = (int)s;
  if (i > n - 1) i = n - 1;
  if (i < 0) i = 0;
  f = s - i;
}

// ---------------------------------------------------------------------------
// Conductor generation. Intercepts along every grid line of each MG level are
// computed analytically for the supported shapes (ZCylinderOut, ZCylinder,
// Sphere), then converted by conductordelfromintercepts
// (pywarp90/f3d_conductors.F:12-729) with fuzz = 1e-13
// (scripts/generateconductors.py:1856) and dfill (default 2.,
// scripts/generateconductors.py:184).
// ---------------------------------------------------------------------------
struct Shape {
  int kind;  // 0 = ZCylinderOut, 1 = ZCylinder, 2 = Sphere
  double radius, length, voltage, xcent, ycent, zcent;
  int condid;
};

// Intercept pairs (entry, exit) of the solid along a line. Lines parallel to
// an axis; `axis` is 0,1,2 and (a,b) are the two fixed coordinates in the
// order (y,z) for x lines, (x,z) for y lines, (x,y) for z lines.
void shape_line_intercepts(const Shape& s, int axis, double a, double b,
                           std::vector<double>& out) {
  out.clear();
  double zmin = s.zcent - 0.5 * s.length, zmax = s.zcent + 0.5 * s.length;
  if (s.kind == 2) {  // Sphere
    double c0, c1, c2;  // along-line center, and the two fixed offsets
    if (axis == 0) { c0 = s.xcent; c1 = a - s.ycent; c2 = b - s.zcent; }
    else if (axis == 1) { c0 = s.ycent; c1 = a - s.xcent; c2 = b - s.zcent; }
    else { c0 = s.zcent; c1 = a - s.xcent; c2 = b - s.ycent; }
    double d2 = s.radius * s.radius - c1 * c1 - c2 * c2;
    if (d2 <= 0.) return;
    double h = std::sqrt(d2);
    out.push_back(c0 - h);
    out.push_back(c0 + h);
    return;
  }
  // cylinders along z
  if (axis == 2) {
    double rr = (a - s.xcent) * (a - s.xcent) + (b - s.ycent) * (b - s.ycent);
    bool inside_r = rr < s.radius * s.radius;
    if (s.kind == 1) {  // ZCylinder: solid for r < radius, zmin <= z <= zmax
      if (inside_r) { out.push_back(zmin); out.push_back(zmax); }
    } else {  // ZCylinderOut: solid for r > radius, zmin <= z <= zmax
      if (!inside_r) { out.push_back(zmin); out.push_back(zmax); }
    }
    return;
  }
  double fixedz = b;
  if (fixedz < zmin || fixedz > zmax) return;
  double c0, c1;
  if (axis == 0) { c0 = s.xcent; c1 = a - s.ycent; }
  else { c0 = s.ycent; c1 = a - s.xcent; }
  double d2 = s.radius * s.radius - c1 * c1;
  if (s.kind == 1) {
    if (d2 <= 0.) return;
    double h = std::sqrt(d2);
    out.push_back(c0 - h);
    out.push_back(c0 + h);
  } else {
    if (d2 <= 0.) { out.push_back(-LARGEPOS); out.push_back(LARGEPOS); return; }
    double h = std::sqrt(d2);
    out.push_back(-LARGEPOS);
    out.push_back(c0 - h);
    out.push_back(c0 + h);
    out.push_back(LARGEPOS);
  }
}

// conductordelfromintercepts for one shape on one level.
void delfromintercepts(const Shape& s, const Level& L, double xmmin, double ymmin, double zmmin,
                       int mglevel, double dfill, double fuzz, Conductors& C) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const double dx = L.dx, dy = L.dy, dz = L.dz;
  const double xmmax = xmmin + nx * dx, ymmax = ymmin + ny * dy, zmmax = zmmin + nz * dz;
  const double dxi = 1. / dx, dyi = 1. / dy, dzi = 1. / dz;
  // Precompute all intercept lists (x lines indexed by (iy,iz), etc.).
  std::vector<std::vector<double>> xi((size_t)(ny + 1) * (nz + 1)), yi((size_t)(nx + 1) * (nz + 1)),
      zi((size_t)(nx + 1) * (ny + 1));
  for (int iz = 0; iz <= nz; ++iz)
    for (int iy = 0; iy <= ny; ++iy)
      shape_line_intercepts(s, 0, ymmin + iy * dy, zmmin + iz * dz, xi[iy + (size_t)(ny + 1) * iz]);
  for (int iz = 0; iz <= nz; ++iz)
    for (int ix = 0; ix <= nx; ++ix)
      shape_line_intercepts(s, 1, xmmin + ix * dx, zmmin + iz * dz, yi[ix + (size_t)(nx + 1) * iz]);
  for (int iy = 0; iy <= ny; ++iy)
    for (int ix = 0; ix <= nx; ++ix)
      shape_line_intercepts(s, 2, xmmin + ix * dx, ymmin + iy * dy, zi[ix + (size_t)(nx + 1) * iy]);
  auto X = [&](int iy, int iz) -> const std::vector<double>& { return xi[iy + (size_t)(ny + 1) * iz]; };
  auto Y = [&](int ix, int iz) -> const std::vector<double>& { return yi[ix + (size_t)(nx + 1) * iz]; };
  auto Z = [&](int ix, int iy) -> const std::vector<double>& { return zi[ix + (size_t)(nx + 1) * iy]; };
  const double V = s.voltage;

  // Interior points (f3d_conductors.F:190-258).
  for (int iz = 0; iz <= nz; ++iz) {
    double zz = zmmin + iz * dz;
    for (int iy = 0; iy <= ny; ++iy) {
      double yy = ymmin + iy * dy;
      const auto& xs = X(iy, iz);
      for (size_t ii = 0; ii + 1 < xs.size(); ii += 2) {
        double x1 = xs[ii], x2 = xs[ii + 1];
        if (!(x2 >= xmmin && x1 <= xmmax)) continue;
        int ix1 = (int)((std::max(x1 - fuzz, xmmin) - xmmin) * dxi);
        int ix2 = (int)((std::min(x2 + fuzz, xmmax) - xmmin) * dxi);
        if (xmmin + ix1 * dx <= x1 && ix1 < nx) ix1 += 1;
        if (xmmin + (ix2 + 1) * dx <= x2 && ix2 < nx) ix2 += 1;
        for (int ix = ix1; ix <= ix2; ++ix) {
          double delx, dely, delz;
          if (dfill < LARGEPOS) {
            double xx = xmmin + ix * dx;
            delx = std::min(xx - x1, x2 - xx);
            dely = LARGEPOS;
            delz = LARGEPOS;
            for (double v : Y(ix, iz)) { dely = std::min(dely, std::fabs(yy - v)); if (v > yy) break; }
            for (double v : Z(ix, iy)) { delz = std::min(delz, std::fabs(zz - v)); if (v > zz) break; }
          } else {
            delx = dely = delz = 0.;
          }
          if (delx < dfill * dx || dely < dfill * dy || delz < dfill * dz) {
            C.interior.indx.push_back(ix); C.interior.indx.push_back(iy); C.interior.indx.push_back(iz);
            C.interior.volt.push_back(V);
            C.interior.numb.push_back(s.condid);
            C.interior.ilevel.push_back(mglevel);
          }
        }
      }
    }
  }

  auto save = [&](int ix, int iy, int iz, const double* dels, const double* volt, const int* numb) {
    Subgrid& S = ((ix + iy + iz) % 2 == 0) ? C.even : C.odd;
    S.indx.push_back(ix); S.indx.push_back(iy); S.indx.push_back(iz);
    for (int k = 0; k < 6; ++k) { S.dels.push_back(dels[k]); S.volt.push_back(volt[k]); S.numb.push_back(numb[k]); }
    S.ilevel.push_back(mglevel);
    S.prevphi.push_back(0.);
  };
  // Scan of a crossing list in the perpendicular direction for the nearest
  // intercept, f3d_conductors.F:334-397 (side-alternating form).
  auto scan_perp = [&](const std::vector<double>& ics, double pos, double di, int idel_minus, int idel_plus,
                       double* dels, double* volt, int* numb) {
    int n = (int)ics.size();
    double side = +1.;
    for (int i1 = 0; i1 < n; ++i1) {
      double d;
      int idel;
      if (side > 0.) {
        if (i1 == 0) d = (ics[i1] - pos) * di;
        else if (pos > ics[i1 - 1]) d = (ics[i1] - pos) * di;
        else d = LARGEPOS;
        idel = idel_plus;
      } else {
        if (i1 == n - 1) d = (pos - ics[i1]) * di;
        else if (pos < ics[i1 + 1]) d = (pos - ics[i1]) * di;
        else d = LARGEPOS;
        idel = idel_minus;
      }
      if (0. < d && d < 1. - fuzz && d < dels[idel]) { dels[idel] = d; volt[idel] = V; numb[idel] = s.condid; }
      side = -side;
    }
  };
  // First-intercept scan used to skip points already found (f3d_conductors.F:471-486).
  auto first_del = [&](const std::vector<double>& ics, double pos, double di) {
    double d = 2.;
    double side = +1.;
    for (size_t i1 = 0; i1 < ics.size(); ++i1) {
      if (d < 1.) break;
      if (side > 0.) { if (ics[i1] >= pos) d = (ics[i1] - pos) * di; }
      else { if (ics[i1] <= pos) d = (pos - ics[i1]) * di; }
      side = -side;
    }
    return d;
  };
  // Finds the grid point next to intercept ii of a line and its delta
  // (f3d_conductors.F:277-320). Returns false when the point is skipped.
  auto line_point = [&](const std::vector<double>& ics, size_t ii, double side, double mmin, double mmax,
                        double d, double di, int n, int& ipt, double& del, int& idel, int idm, int idp) {
    double icpt = ics[ii];
    if (!(mmin - d < icpt && icpt < mmax + d)) return false;
    int i = (int)std::floor((icpt - mmin) * di);
    if (side > 0.) {
      if (i < 0) return false;
      double xx = mmin + i * d;
      if (ii == 0) del = (icpt - mmin) * di - i;
      else if (xx > ics[ii - 1]) del = (icpt - mmin) * di - i;
      else del = LARGEPOS;
      idel = idp;
    } else {
      i = i + 1;
      if (i > n) return false;
      double xx = mmin + i * d;
      if (ii == ics.size() - 1) del = i - (icpt - mmin) * di;
      else if (xx < ics[ii + 1]) del = i - (icpt - mmin) * di;
      else del = LARGEPOS;
      idel = idm;
    }
    ipt = i;
    return true;
  };

  // x lines (f3d_conductors.F:263-416)
  for (int iz = 0; iz <= nz; ++iz) {
    double zz = zmmin + iz * dz;
    for (int iy = 0; iy <= ny; ++iy) {
      double yy = ymmin + iy * dy;
      const auto& xs = X(iy, iz);
      double side = -1.;
      for (size_t ii = 0; ii < xs.size(); ++ii) {
        side = -side;
        int ix, idel;
        double delx;
        if (!line_point(xs, ii, side, xmmin, xmmax, dx, dxi, nx, ix, delx, idel, 0, 1)) continue;
        if (0. < delx && delx < 1. - fuzz) {
          double dels[6], volt[6];
          int numb[6];
          for (int k = 0; k < 6; ++k) { dels[k] = LARGEPOS; volt[k] = 0.; numb[k] = 0; }
          dels[idel] = delx; volt[idel] = V; numb[idel] = s.condid;
          scan_perp(Y(ix, iz), yy, dyi, 2, 3, dels, volt, numb);
          scan_perp(Z(ix, iy), zz, dzi, 4, 5, dels, volt, numb);
          save(ix, iy, iz, dels, volt, numb);
        }
      }
    }
  }
  // y lines (f3d_conductors.F:418-557)
  for (int iz = 0; iz <= nz; ++iz) {
    double zz = zmmin + iz * dz;
    for (int ix = 0; ix <= nx; ++ix) {
      double xx = xmmin + ix * dx;
      const auto& ys = Y(ix, iz);
      double side = -1.;
      for (size_t ii = 0; ii < ys.size(); ++ii) {
        side = -side;
        int iy, idel;
        double dely;
        if (!line_point(ys, ii, side, ymmin, ymmax, dy, dyi, ny, iy, dely, idel, 2, 3)) continue;
        double delx = first_del(X(iy, iz), xx, dxi);
        if (0. < dely && dely < 1. - fuzz && delx >= 1. - fuzz) {
          double dels[6], volt[6];
          int numb[6];
          for (int k = 0; k < 6; ++k) { dels[k] = LARGEPOS; volt[k] = 0.; numb[k] = 0; }
          dels[idel] = dely; volt[idel] = V; numb[idel] = s.condid;
          scan_perp(Z(ix, iy), zz, dzi, 4, 5, dels, volt, numb);
          save(ix, iy, iz, dels, volt, numb);
        }
      }
    }
  }
  // z lines (f3d_conductors.F:559-720)
  for (int iy = 0; iy <= ny; ++iy) {
    double yy = ymmin + iy * dy;
    for (int ix = 0; ix <= nx; ++ix) {
      double xx = xmmin + ix * dx;
      const auto& zs = Z(ix, iy);
      double side = -1.;
      for (size_t ii = 0; ii < zs.size(); ++ii) {
        side = -side;
        int iz, idel;
        double delz;
        if (!line_point(zs, ii, side, zmmin, zmmax, dz, dzi, nz, iz, delz, idel, 4, 5)) continue;
        double delx = first_del(X(iy, iz), xx, dxi);
        double dely = first_del(Y(ix, iz), yy, dyi);
        if (0. < delz && delz < 1. - fuzz && delx >= 1. - fuzz && dely >= 1. - fuzz) {
          double dels[6], volt[6];
          int numb[6];
          for (int k = 0; k < 6; ++k) { dels[k] = LARGEPOS; volt[k] = 0.; numb[k] = 0; }
          dels[idel] = delz; volt[idel] = V; numb[idel] = s.condid;
          save(ix, iy, iz, dels, volt, numb);
        }
      }
    }
  }
}

// checkconductors_work, pywarp90/f3d_mgrid.F:4141-4326, for one level.
void checkconductors_work(Conductors& C, int nxl, int nyl, int nzl, int mglevel) {
  const int BIG = -2;  // marks a conductor interior point
  std::vector<int> iii((size_t)(nxl + 1) * (nyl + 1) * (nzl + 1), -1);
  auto at = [&](int ix, int iy, int iz) -> int& { return iii[ridx(nxl, nyl, ix, iy, iz)]; };
  Interior& I = C.interior;
  for (size_t ic = 0; ic < I.n(); ++ic) {
    if (I.ilevel[ic] != mglevel) continue;
    int ix = I.indx[3 * ic], iy = I.indx[3 * ic + 1], iz = I.indx[3 * ic + 2];
    if (ix < 0 || nxl < ix || iy < 0 || nyl < iy || iz < 0 || nzl < iz) { I.ilevel[ic] = -1; continue; }
    if (at(ix, iy, iz) == BIG) { I.ilevel[ic] = -1; continue; }
    at(ix, iy, iz) = BIG;
  }
  for (Subgrid* S : {&C.even, &C.odd}) {
    for (size_t ic = 0; ic < S->n(); ++ic) {
      if (S->ilevel[ic] != mglevel) continue;
      int ix = S->indx[3 * ic], iy = S->indx[3 * ic + 1], iz = S->indx[3 * ic + 2];
      if (ix < 0 || nxl < ix || iy < 0 || nyl < iy || iz < 0 || nzl < iz) { S->ilevel[ic] = -1; continue; }
      int& cell = at(ix, iy, iz);
      if (cell == BIG) { S->ilevel[ic] = -1; continue; }
      if (cell == -1) { cell = (int)ic; continue; }
      int i = cell;
      if (S->ilevel[ic] != S->ilevel[i]) { cell = (int)ic; continue; }
      for (int id = 0; id < 6; ++id) {
        double d = S->dels[6 * ic + id];
        if (std::fabs(d) < 1. && std::fabs(d) < std::fabs(S->dels[6 * i + id])) {
          S->dels[6 * i + id] = d;
          S->volt[6 * i + id] = S->volt[6 * ic + id];
          S->numb[6 * i + id] = S->numb[6 * ic + id];
        }
      }
      S->ilevel[ic] = -1;
    }
    // The reference uses one work array for both parities; even and odd
    // points never share a node on one level, so a fresh map per parity is
    // equivalent except that interior marks must persist.
    for (auto& v : iii) if (v != BIG) v = -1;
  }
}

// Stable sort by level (isortconductor / iswapconductor, f3d_mgrid.F:4052-4110),
// dropping points with ilevel = -1.
template <typename T>
void gather_rows(std::vector<T>& a, const std::vector<size_t>& order, int w) {
  std::vector<T> b;
  b.reserve(order.size() * w);
  for (size_t i : order) for (int k = 0; k < w; ++k) b.push_back(a[i * w + k]);
  a.swap(b);
}
void sort_interior(Interior& I, int levels) {
  std::vector<size_t> order;
  I.istart.assign(levels + 1, 0);
  for (int l = 0; l < levels; ++l) {
    I.istart[l] = (int)order.size();
    for (size_t ic = 0; ic < I.n(); ++ic) if (I.ilevel[ic] == l) order.push_back(ic);
  }
  I.istart[levels] = (int)order.size();
  gather_rows(I.indx, order, 3);
  gather_rows(I.volt, order, 1);
  gather_rows(I.numb, order, 1);
  gather_rows(I.ilevel, order, 1);
}
void sort_subgrid(Subgrid& S, int levels) {
  std::vector<size_t> order;
  S.istart.assign(levels + 1, 0);
  for (int l = 0; l < levels; ++l) {
    S.istart[l] = (int)order.size();
    for (size_t ic = 0; ic < S.n(); ++ic) if (S.ilevel[ic] == l) order.push_back(ic);
  }
  S.istart[levels] = (int)order.size();
  gather_rows(S.indx, order, 3);
  gather_rows(S.dels, order, 6);
  gather_rows(S.volt, order, 6);
  gather_rows(S.numb, order, 6);
  gather_rows(S.ilevel, order, 1);
  S.prevphi.assign(S.ilevel.size(), 0.);
}

// ---------------------------------------------------------------------------
// Multigrid solver (pywarp90/f3d_mgrid.F)
// ---------------------------------------------------------------------------

// applyboundaryconditions3d, f3d_mgrid.F:3847-3955, ncomp = 1.
void applybc(int nx, int ny, int nz, int ng, double* u, const int* b, bool lwithdirichlet, bool lzerodirichlet) {
  const int sx = nx + 1 + 2 * ng, sy = ny + 1 + 2 * ng;
  auto U = [&](int ix, int iy, int iz) -> double& {
    return u[(size_t)(ix + ng) + (size_t)sx * ((size_t)(iy + ng) + (size_t)sy * (size_t)(iz + ng))];
  };
  if (ng > 0) {
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy) {
        if (lwithdirichlet) {
          if (b[0] == 0) for (int ix = -1; ix >= -ng; --ix) U(ix, iy, iz) = 2. * U(ix + 1, iy, iz) - U(ix + 2, iy, iz);
          if (b[1] == 0) for (int ix = nx + 1; ix <= nx + ng; ++ix) U(ix, iy, iz) = 2. * U(ix - 1, iy, iz) - U(ix - 2, iy, iz);
        }
      }
    if (!lwithdirichlet && lzerodirichlet) {
      for (int iz = -ng; iz <= nz + ng; ++iz)
        for (int iy = -ng; iy <= ny + ng; ++iy) {
          if (b[0] == 0) for (int ix = -ng; ix <= -1; ++ix) U(ix, iy, iz) = 0.;
          if (b[1] == 0) for (int ix = nx + 1; ix <= nx + ng; ++ix) U(ix, iy, iz) = 0.;
        }
    }
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy) {
        if (b[0] == 1) for (int k = 1; k <= ng; ++k) U(-k, iy, iz) = U(k, iy, iz);
        if (b[1] == 1) for (int k = 1; k <= ng; ++k) U(nx + k, iy, iz) = U(nx - k, iy, iz);
        if (b[0] == 2 && b[1] == 2) {
          for (int k = 1; k <= ng; ++k) U(-k, iy, iz) = U(nx - k, iy, iz);
          for (int k = 0; k <= ng; ++k) U(nx + k, iy, iz) = U(k, iy, iz);
        }
      }
  }
  if (ng > 0) {
    for (int iz = 0; iz <= nz; ++iz)
      for (int ix = -ng; ix <= nx + ng; ++ix) {
        if (lwithdirichlet) {
          if (b[2] == 0) for (int iy = -1; iy >= -ng; --iy) U(ix, iy, iz) = 2. * U(ix, iy + 1, iz) - U(ix, iy + 2, iz);
          if (b[3] == 0) for (int iy = ny + 1; iy <= ny + ng; ++iy) U(ix, iy, iz) = 2. * U(ix, iy - 1, iz) - U(ix, iy - 2, iz);
        }
      }
    if (!lwithdirichlet && lzerodirichlet) {
      for (int iz = -ng; iz <= nz + ng; ++iz)
        for (int ix = -ng; ix <= nx + ng; ++ix) {
          if (b[2] == 0) for (int iy = -ng; iy <= -1; ++iy) U(ix, iy, iz) = 0.;
          if (b[3] == 0) for (int iy = ny + 1; iy <= ny + ng; ++iy) U(ix, iy, iz) = 0.;
        }
    }
    for (int iz = 0; iz <= nz; ++iz)
      for (int ix = -ng; ix <= nx + ng; ++ix) {
        if (b[2] == 1) for (int k = 1; k <= ng; ++k) U(ix, -k, iz) = U(ix, k, iz);
        if (b[3] == 1) for (int k = 1; k <= ng; ++k) U(ix, ny + k, iz) = U(ix, ny - k, iz);
        if (b[2] == 2 && b[3] == 2) {
          for (int k = 1; k <= ng; ++k) U(ix, -k, iz) = U(ix, ny - k, iz);
          for (int k = 0; k <= ng; ++k) U(ix, ny + k, iz) = U(ix, k, iz);
        }
      }
  }
  if (ng > 0) {
    for (int iy = -ng; iy <= ny + ng; ++iy)
      for (int ix = -ng; ix <= nx + ng; ++ix) {
        if (lwithdirichlet) {
          if (b[4] == 0) for (int iz = -1; iz >= -ng; --iz) U(ix, iy, iz) = 2. * U(ix, iy, iz + 1) - U(ix, iy, iz + 2);
          if (b[5] == 0) for (int iz = nz + 1; iz <= nz + ng; ++iz) U(ix, iy, iz) = 2. * U(ix, iy, iz - 1) - U(ix, iy, iz - 2);
        } else if (lzerodirichlet) {
          if (b[4] == 0) for (int iz = -ng; iz <= -1; ++iz) U(ix, iy, iz) = 0.;
          if (b[5] == 0) for (int iz = nz + 1; iz <= nz + ng; ++iz) U(ix, iy, iz) = 0.;
        }
        if (b[4] == 1) for (int k = 1; k <= ng; ++k) U(ix, iy, -k) = U(ix, iy, k);
        if (b[5] == 1) for (int k = 1; k <= ng; ++k) U(ix, iy, nz + k) = U(ix, iy, nz - k);
        if (b[4] == 2 && b[5] == 2) {
          for (int k = 1; k <= ng; ++k) U(ix, iy, -k) = U(ix, iy, nz - k);
          for (int k = 0; k <= ng; ++k) U(ix, iy, nz + k) = U(ix, iy, k);
        }
      }
  }
}

struct MGParams {
  double mgparam;
  int mgform, mgmaxiters, mgmaxlevels, downpasses, uppasses, icndbndy, lcndbndy;
  double mgtol;
};

// cond_potmg, f3d_mgrid.F:2426-2470
void cond_potmg(const Interior& I, int nx, int ny, double* phi, int mglevel, int mgform, bool mgform2init) {
  bool usev = (mglevel == 0 && (mgform == 1 || mgform2init));
  par_for(I.istart[mglevel], I.istart[mglevel + 1], [&](int64_t ic) {
    phi[pidx(nx, ny, I.indx[3 * ic], I.indx[3 * ic + 1], I.indx[3 * ic + 2])] = usev ? I.volt[ic] : 0.;
  });
}

// handlesubgrid2, f3d_mgrid.F:2628-2764
void handlesubgrid2(int im, int ip, double& pm, double& pp, double dsqicos, const double* dels,
                    const double* volt, double voltfac, double& denom, double& ppp) {
  double dm = dels[im], dp = dels[ip];
  if (0. < dm && dm < +1. && 0. < dp && dp < +1.) {
    pm = voltfac * volt[im] * 2. / (dm * (dp + dm));
    pp = voltfac * volt[ip] * 2. / (dp * (dp + dm));
    denom = denom + 2. * (1. - dp * dm) / (dp * dm) * dsqicos;
    ppp = std::min(ppp, dm);
    ppp = std::min(ppp, dp);
  } else if (0. >= dm && dm > -1. && 0. >= dp && dp > -1.) {
    pm = 0.;
    pp = 0.;
    denom = denom - 2. * dsqicos;
    ppp = (std::fabs(dm) > 0.) ? std::min(ppp, std::fabs(dm)) : std::min(ppp, 1. - 1.e-9);
    ppp = (std::fabs(dp) > 0.) ? std::min(ppp, std::fabs(dp)) : std::min(ppp, 1. - 1.e-9);
  } else if (0. < dm && dm < +1. && 0. >= dp && dp > -1.) {
    double adel = std::fabs(dp);
    pm = voltfac * volt[im] / (dm * (adel + 0.5 * dm));
    pp = 0.;
    denom = denom + (1. - 2. * dm * adel - dm) / (dm * (adel + 0.5 * dm)) * dsqicos;
    ppp = std::min(ppp, dm);
    ppp = (adel > 0.) ? std::min(ppp, adel) : std::min(ppp, 1. - 1.e-9);
  } else if (0. >= dm && dm > -1. && 0. < dp && dp < +1.) {
    double adel = std::fabs(dm);
    pm = 0.;
    pp = voltfac * volt[ip] / (dp * (adel + 0.5 * dp));
    denom = denom + (1. - 2. * dp * adel - dp) / (dp * (adel + 0.5 * dp)) * dsqicos;
    ppp = (adel > 0.) ? std::min(ppp, adel) : std::min(ppp, 1. - 1.e-9);
    ppp = std::min(ppp, dp);
  } else {
    if (0. < dm && dm < +1.) {
      pm = voltfac * volt[im] * 2. / (dm * (1. + dm));
      pp = pp * (2. / (1. + dm));
      denom = denom + 2. * (1. - dm) / dm * dsqicos;
      ppp = std::min(ppp, dm);
    } else if (0. >= dm && dm > -1.) {
      double adel = std::fabs(dm);
      pm = 0.;
      pp = pp / (0.5 + adel);
      denom = denom - 2. * adel / (adel + 0.5) * dsqicos;
      ppp = (adel > 0.) ? std::min(ppp, adel) : std::min(ppp, 1. - 1.e-9);
    }
    if (0. < dp && dp < +1.) {
      pp = voltfac * volt[ip] * 2. / (dp * (1. + dp));
      pm = pm * (2. / (1. + dp));
      denom = denom + 2. * (1. - dp) / dp * dsqicos;
      ppp = std::min(ppp, dp);
    } else if (0. >= dp && dp > -1.) {
      double adel = std::fabs(dp);
      pp = 0.;
      pm = pm / (0.5 + adel);
      denom = denom - 2. * adel / (adel + 0.5) * dsqicos;
      ppp = (adel > 0.) ? std::min(ppp, adel) : std::min(ppp, 1. - 1.e-9);
    }
  }
}

// condbndymg with icndbndy = 2, f3d_mgrid.F:2766-2980
void condbndymg(Subgrid& S, int nx, int ny, int nz, double* phi, const double* rho, double dxsqic,
                double dysqic, double dzsqic, double spm1, double mgparam, const int* lb, int mglevel,
                int mgform) {
  double dxsqicos = dxsqic / mgparam, dysqicos = dysqic / mgparam, dzsqicos = dzsqic / mgparam;
  double voltfac = (mglevel == 0 && mgform == 1) ? 1. : 0.;
  // subgrid points of one colour read only the other colour
  par_for(S.istart[mglevel], S.istart[mglevel + 1], [&](int64_t ic) {
    int ix = S.indx[3 * ic], iy = S.indx[3 * ic + 1], iz = S.indx[3 * ic + 2];
    if (ix == 0 && lb[0] < 1) return;
    if (ix == nx && lb[1] < 1) return;
    if (iy == 0 && lb[2] < 1) return;
    if (iy == ny && lb[3] < 1) return;
    if (iz == 0 && lb[4] < 1) return;
    if (iz == nz && lb[5] < 1) return;
    double pxm = phi[pidx(nx, ny, ix - 1, iy, iz)], pxp = phi[pidx(nx, ny, ix + 1, iy, iz)];
    double pym = phi[pidx(nx, ny, ix, iy - 1, iz)], pyp = phi[pidx(nx, ny, ix, iy + 1, iz)];
    double pzm = phi[pidx(nx, ny, ix, iy, iz - 1)], pzp = phi[pidx(nx, ny, ix, iy, iz + 1)];
    double denom = 1., ppp = 1.;
    const double* dels = &S.dels[6 * ic];
    const double* volt = &S.volt[6 * ic];
    handlesubgrid2(0, 1, pxm, pxp, dxsqicos, dels, volt, voltfac, denom, ppp);
    handlesubgrid2(2, 3, pym, pyp, dysqicos, dels, volt, voltfac, denom, ppp);
    handlesubgrid2(4, 5, pzm, pzp, dzsqicos, dels, volt, voltfac, denom, ppp);
    if (ppp < 1.) {
      phi[pidx(nx, ny, ix, iy, iz)] =
          (rho[ridx(nx, ny, ix, iy, iz)] + (pxm + pxp) * dxsqic + (pym + pyp) * dysqic + (pzm + pzp) * dzsqic) / denom +
          spm1 * S.prevphi[ic];
    }
  });
}

// condbndymgint, f3d_mgrid.F:2982-3092 (Neumann subgrid neighbours)
void condbndymgint(Conductors& C, int nx, int ny, int nz, double* phi, const int* lb, int mglevel) {
  for (Subgrid* S : {&C.even, &C.odd}) {
    for (int ic = S->istart[mglevel]; ic < S->istart[mglevel + 1]; ++ic) {
      int ix = S->indx[3 * ic], iy = S->indx[3 * ic + 1], iz = S->indx[3 * ic + 2];
      const double* d = &S->dels[6 * ic];
      double p0 = phi[pidx(nx, ny, ix, iy, iz)];
      if (!((ix - 1 == 0 && lb[0] == 0) || (ix + 1 == nx && lb[1] == 0) || (ix == 0 && lb[0] < 1) || (ix == nx && lb[1] < 1))) {
        if (0. >= d[0] && d[0] > -1.) phi[pidx(nx, ny, ix - 1, iy, iz)] = p0;
        if (0. >= d[1] && d[1] > -1.) phi[pidx(nx, ny, ix + 1, iy, iz)] = p0;
      }
      if (!((iy - 1 == 0 && lb[2] == 0) || (iy + 1 == ny && lb[3] == 0) || (iy == 0 && lb[2] < 1) || (iy == ny && lb[3] < 1))) {
        if (0. >= d[2] && d[2] > -1.) phi[pidx(nx, ny, ix, iy - 1, iz)] = p0;
        if (0. >= d[3] && d[3] > -1.) phi[pidx(nx, ny, ix, iy + 1, iz)] = p0;
      }
      if (!((iz - 1 == 0 && lb[4] == 0) || (iz + 1 == nz && lb[5] == 0) || (iz == 0 && lb[4] < 1) || (iz == nz && lb[5] < 1))) {
        if (0. >= d[4] && d[4] > -1.) phi[pidx(nx, ny, ix, iy, iz - 1)] = p0;
        if (0. >= d[5] && d[5] > -1.) phi[pidx(nx, ny, ix, iy, iz + 1)] = p0;
      }
    }
  }
}

// sorhalfpass3d (no bends, no precalculated coefficients), f3d_mgrid.F:2095-2291
void sorhalfpass3d(int parity, int mglevel, int nx, int ny, int nz, double* phi, const double* rho,
                   double dxsqi, double dysqi, double dzsqi, const int* lb, const MGParams& P, Conductors& C) {
  double cst = P.mgparam * 0.5 / (dxsqi + dysqi + dzsqi);
  double dxsqic = dxsqi * cst, dysqic = dysqi * cst, dzsqic = dzsqi * cst;
  double spm1 = 1. - P.mgparam;
  int ixmin = 0, ixmax = nx, iymin = 0, iymax = ny, izmin = 0, izmax = nz;
  if (lb[0] <= 0) ixmin = 1;
  if (lb[1] <= 0) ixmax = nx - 1;
  if (lb[2] <= 0) iymin = 1;
  if (lb[3] <= 0) iymax = ny - 1;
  if (lb[4] <= 0) izmin = 1;
  if (lb[5] <= 0) izmax = nz - 1;
  Subgrid& S = (parity == 0) ? C.even : C.odd;
  if (P.lcndbndy)
    par_for(S.istart[mglevel], S.istart[mglevel + 1], [&](int64_t ic) {
      S.prevphi[ic] = phi[pidx(nx, ny, S.indx[3 * ic], S.indx[3 * ic + 1], S.indx[3 * ic + 2])];
    });
  const size_t sx = 1, sy = nx + 3, sz = (size_t)(nx + 3) * (ny + 3);
  // one colour reads only the other colour: planes are independent
  par_for(izmin, izmax + 1, [&](int64_t iz64) {
    const int iz = (int)iz64;
    for (int iy = iymin; iy <= iymax; ++iy) {
      int ix1 = ixmin + (((ixmin + iy + iz + parity) % 2) + 2) % 2;
      for (int ix = ix1; ix <= ixmax; ix += 2) {
        size_t p = pidx(nx, ny, ix, iy, iz);
        phi[p] = rho[ridx(nx, ny, ix, iy, iz)] + (phi[p - sx] + phi[p + sx]) * dxsqic +
                 (phi[p - sy] + phi[p + sy]) * dysqic + (phi[p - sz] + phi[p + sz]) * dzsqic + spm1 * phi[p];
      }
    }
  }, (int64_t)(nx + 1) * (ny + 1) / 2);
  if (P.lcndbndy) condbndymg(S, nx, ny, nz, phi, rho, dxsqic, dysqic, dzsqic, spm1, P.mgparam, lb, mglevel, P.mgform);
  cond_potmg(C.interior, nx, ny, phi, mglevel, P.mgform, false);
  condbndymgint(C, nx, ny, nz, phi, lb, mglevel);
}

// sorpass3d, f3d_mgrid.F:1949-2093
void sorpass3d(int mglevel, int nx, int ny, int nz, double* phi, const double* rho, double dxsqi, double dysqi,
               double dzsqi, const int* lb, const MGParams& P, Conductors& C) {
  cond_potmg(C.interior, nx, ny, phi, mglevel, P.mgform, false);
  condbndymgint(C, nx, ny, nz, phi, lb, mglevel);
  for (int parity = 0; parity <= 1; ++parity) {
    sorhalfpass3d(parity, mglevel, nx, ny, nz, phi, rho, dxsqi, dysqi, dzsqi, lb, P, C);
    applybc(nx, ny, nz, 1, phi, lb, false, false);
  }
}

// condbndyres with icndbndy = 2, f3d_mgrid.F:3094-3365
void condbndyres(Conductors& C, int nx, int ny, int nz, const double* phi, const double* rho, double* res,
                 double dxsqi, double dysqi, double dzsqi, double mgparam, const int* lb, int mglevel, int mgform,
                 bool mgform2init) {
  double cst = 0.5 / (dxsqi + dysqi + dzsqi);
  double dxsqic = dxsqi * cst, dysqic = dysqi * cst, dzsqic = dzsqi * cst;
  double dxsqics = mgparam * dxsqi * cst, dysqics = mgparam * dysqi * cst, dzsqics = mgparam * dzsqi * cst;
  double voltfac = (mglevel == 0 && (mgform == 1 || mgform2init)) ? 1. : 0.;
  for (Subgrid* S : {&C.even, &C.odd}) {
    for (int ic = S->istart[mglevel]; ic < S->istart[mglevel + 1]; ++ic) {
      int ix = S->indx[3 * ic], iy = S->indx[3 * ic + 1], iz = S->indx[3 * ic + 2];
      if (ix == 0 && lb[0] == 0) continue;
      if (ix == nx && lb[1] == 0) continue;
      if (iy == 0 && lb[2] == 0) continue;
      if (iy == ny && lb[3] == 0) continue;
      if (iz == 0 && lb[4] == 0) continue;
      if (iz == nz && lb[5] == 0) continue;
      double pxm = phi[pidx(nx, ny, ix - 1, iy, iz)], pxp = phi[pidx(nx, ny, ix + 1, iy, iz)];
      double pym = phi[pidx(nx, ny, ix, iy - 1, iz)], pyp = phi[pidx(nx, ny, ix, iy + 1, iz)];
      double pzm = phi[pidx(nx, ny, ix, iy, iz - 1)], pzp = phi[pidx(nx, ny, ix, iy, iz + 1)];
      double denom = 1., ppp = 1.;
      const double* d = &S->dels[6 * ic];
      const double* v = &S->volt[6 * ic];
      handlesubgrid2(0, 1, pxm, pxp, dxsqic, d, v, voltfac, denom, ppp);
      handlesubgrid2(2, 3, pym, pyp, dysqic, d, v, voltfac, denom, ppp);
      handlesubgrid2(4, 5, pzm, pzp, dzsqic, d, v, voltfac, denom, ppp);
      if (ppp < 1.) {
        if (mgform2init) ppp = 1.;
        res[pidx(nx, ny, ix, iy, iz)] =
            ppp * (rho[ridx(nx, ny, ix, iy, iz)] + (pxm + pxp) * dxsqics + (pym + pyp) * dysqics +
                   (pzm + pzp) * dzsqics - phi[pidx(nx, ny, ix, iy, iz)] * mgparam * denom);
        if (0. >= d[0] && d[0] >= -1.) res[pidx(nx, ny, ix - 1, iy, iz)] = 0.;
        if (0. >= d[1] && d[1] >= -1.) res[pidx(nx, ny, ix + 1, iy, iz)] = 0.;
        if (0. >= d[2] && d[2] >= -1.) res[pidx(nx, ny, ix, iy - 1, iz)] = 0.;
        if (0. >= d[3] && d[3] >= -1.) res[pidx(nx, ny, ix, iy + 1, iz)] = 0.;
        if (0. >= d[4] && d[4] >= -1.) res[pidx(nx, ny, ix, iy, iz - 1)] = 0.;
        if (0. >= d[5] && d[5] >= -1.) res[pidx(nx, ny, ix, iy, iz + 1)] = 0.;
      }
    }
  }
}

// residual3d (no precalculated coefficients), f3d_mgrid.F:3367-3598.
// res has one guard cell and is fully rewritten (entries the reference leaves
// untouched are zero, matching a freshly zeroed array).
void residual3d(int nx, int ny, int nz, double dxsqi, double dysqi, double dzsqi, const double* phi,
                const double* rho, double* res, int mglevel, const int* lb, const MGParams& P, bool mgform2init,
                Conductors& C) {
  double cst = 0.5 / (dxsqi + dysqi + dzsqi);
  double dxsqic = dxsqi * P.mgparam * cst, dysqic = dysqi * P.mgparam * cst, dzsqic = dzsqi * P.mgparam * cst;
  int ixmin = 0, ixmax = nx, iymin = 0, iymax = ny, izmin = 0, izmax = nz;
  if (lb[0] == 0) ixmin = 1;
  if (lb[1] == 0) ixmax = nx - 1;
  if (lb[2] == 0) iymin = 1;
  if (lb[3] == 0) iymax = ny - 1;
  if (lb[4] == 0) izmin = 1;
  if (lb[5] == 0) izmax = nz - 1;
  const int64_t npad = (int64_t)(nx + 3) * (ny + 3) * (nz + 3);
  par_for(0, npad, [&](int64_t i) { res[i] = 0.; });
  const size_t sx = 1, sy = nx + 3, sz = (size_t)(nx + 3) * (ny + 3);
  par_for(izmin, izmax + 1, [&](int64_t iz64) {
    const int iz = (int)iz64;
    for (int iy = iymin; iy <= iymax; ++iy)
      for (int ix = ixmin; ix <= ixmax; ++ix) {
        size_t p = pidx(nx, ny, ix, iy, iz);
        res[p] = rho[ridx(nx, ny, ix, iy, iz)] + (phi[p - sx] + phi[p + sx]) * dxsqic +
                 (phi[p - sy] + phi[p + sy]) * dysqic + (phi[p - sz] + phi[p + sz]) * dzsqic - phi[p] * P.mgparam;
      }
  }, (int64_t)(nx + 1) * (ny + 1));
  const Interior& I = C.interior;
  for (int ic = I.istart[mglevel]; ic < I.istart[mglevel + 1]; ++ic)
    res[pidx(nx, ny, I.indx[3 * ic], I.indx[3 * ic + 1], I.indx[3 * ic + 2])] = 0.;
  if (P.lcndbndy)
    condbndyres(C, nx, ny, nz, phi, rho, res, dxsqi, dysqi, dzsqi, P.mgparam, lb, mglevel, P.mgform, mgform2init);
  applybc(nx, ny, nz, 1, res, lb, false, false);
}

// restrict3d, f3d_mgrid.F:1593-1775 (serial: offsets 0, nguardres = 1)
// The source has `ng` guard cells (1 for the V-cycle's residual, 0 for rho
// in the full multigrid) and is passed in the padded layout. Windows are
// clipped to the guard; the weights stay indexed from the unclipped window
// start, as the reference's precalculated wxa/wya/wza are, so a window
// clipped at its low end takes the weights of the taps below it. (With
// ng = 1 and coarsening ratios up to 2 no window is clipped.)
void restrict3d(int nx, int ny, int nz, const double* res, int nxc, int nyc, int nzc, double* rhoc, double ff,
                const int* lbc, int ng = 1) {
  int ixcmin = 0, ixcmax = nxc, iycmin = 0, iycmax = nyc, izcmin = 0, izcmax = nzc;
  if (lbc[0] == 0) ixcmin = 1;
  if (lbc[1] == 0) ixcmax = nxc - 1;
  if (lbc[2] == 0) iycmin = 1;
  if (lbc[3] == 0) iycmax = nyc - 1;
  if (lbc[4] == 0) izcmin = 1;
  if (lbc[5] == 0) izcmax = nzc - 1;
  double dxi = 1. * nxc / nx, dyi = 1. * nyc / ny, dzi = 1. * nzc / nz;
  std::fill(rhoc, rhoc + (size_t)(nxc + 1) * (nyc + 1) * (nzc + 1), 0.);
  auto lim = [ng](int ic, int n, int nc, int& lo, int& hi, int& lo0) {
    lo0 = ((ic - 1) * n + 4 * nc) / nc - 3;
    hi = ((ic + 1) * n - 1) / nc;
    lo = std::max(lo0, -ng);
    hi = std::min(hi, n + ng);
  };
  par_for(izcmin, izcmax + 1, [&](int64_t izc64) {
    const int izc = (int)izc64;
    int izmin, izmax, iz0;
    lim(izc, nz, nzc, izmin, izmax, iz0);
    for (int iyc = iycmin; iyc <= iycmax; ++iyc) {
      int iymin, iymax, iy0;
      lim(iyc, ny, nyc, iymin, iymax, iy0);
      for (int ixc = ixcmin; ixc <= ixcmax; ++ixc) {
        int ixmin, ixmax, ix0;
        lim(ixc, nx, nxc, ixmin, ixmax, ix0);
        double r = 0., w = 0.;
        for (int iz = izmin; iz <= izmax; ++iz) {
          double wz = 1. - std::fabs(izc - (iz0 + (iz - izmin) + 0.) * dzi);
          for (int iy = iymin; iy <= iymax; ++iy) {
            double wy = 1. - std::fabs(iyc - (iy0 + (iy - iymin) + 0.) * dyi);
            for (int ix = ixmin; ix <= ixmax; ++ix) {
              double wx = 1. - std::fabs(ixc - (ix0 + (ix - ixmin) + 0.) * dxi);
              r = r + wx * wy * wz * res[pidx(nx, ny, ix, iy, iz)];
              w = w + wx * wy * wz;
            }
          }
        }
        if (w > 0.) {
          r = r / w;
          rhoc[ridx(nxc, nyc, ixc, iyc, izc)] = r * ff;
        } else {
          rhoc[ridx(nxc, nyc, ixc, iyc, izc)] = 0.;
        }
      }
    }
  }, (int64_t)(nxc + 1) * (nyc + 1) * 9);
}

// expand3d (no precalculated coefficients), f3d_mgrid.F:1777-1947
void expand3d(int nx, int ny, int nz, double* phi, int nxc, int nyc, int nzc, const double* phic, const int* lb) {
  int ixmin = 0, ixmax = nx, iymin = 0, iymax = ny, izmin = 0, izmax = nz;
  if (lb[0] == 0) ixmin = 1;
  if (lb[1] == 0) ixmax = nx - 1;
  if (lb[2] == 0) iymin = 1;
  if (lb[3] == 0) iymax = ny - 1;
  if (lb[4] == 0) izmin = 1;
  if (lb[5] == 0) izmax = nz - 1;
  par_for(izmin, izmax + 1, [&](int64_t iz64) {
    const int iz = (int)iz64;
    int jz = (iz * nzc) / nz;
    double wz = 1. * (iz * nzc) / nz - jz;
    for (int iy = iymin; iy <= iymax; ++iy) {
      int jy = (iy * nyc) / ny;
      double wy = 1. * (iy * nyc) / ny - jy;
      for (int ix = ixmin; ix <= ixmax; ++ix) {
        int jx = (ix * nxc) / nx;
        double wx = 1. * (ix * nxc) / nx - jx;
        double& p = phi[pidx(nx, ny, ix, iy, iz)];
        p = p + (1. - wx) * (1. - wy) * (1. - wz) * phic[pidx(nxc, nyc, jx, jy, jz)] +
            wx * (1. - wy) * (1. - wz) * phic[pidx(nxc, nyc, jx + 1, jy, jz)] +
            (1. - wx) * wy * (1. - wz) * phic[pidx(nxc, nyc, jx, jy + 1, jz)] +
            wx * wy * (1. - wz) * phic[pidx(nxc, nyc, jx + 1, jy + 1, jz)] +
            (1. - wx) * (1. - wy) * wz * phic[pidx(nxc, nyc, jx, jy, jz + 1)] +
            wx * (1. - wy) * wz * phic[pidx(nxc, nyc, jx + 1, jy, jz + 1)] +
            (1. - wx) * wy * wz * phic[pidx(nxc, nyc, jx, jy + 1, jz + 1)] +
            wx * wy * wz * phic[pidx(nxc, nyc, jx + 1, jy + 1, jz + 1)];
      }
    }
  }, (int64_t)(nx + 1) * (ny + 1));
}

// vcycle, f3d_mgrid.F:1101-1591 (serial; recursive)
void vcycle(int mglevel, const std::vector<Level>& lv, double* phi, const double* rho, const int* bounds,
            const MGParams& P, Conductors& C) {
  const Level& L = lv[mglevel];
  int nx = L.nx, ny = L.ny, nz = L.nz;
  double dxsqi = 1. / (L.dx * L.dx), dysqi = 1. / (L.dy * L.dy), dzsqi = 1. / (L.dz * L.dz);
  for (int i = 0; i < P.downpasses; ++i) sorpass3d(mglevel, nx, ny, nz, phi, rho, dxsqi, dysqi, dzsqi, bounds, P, C);
  if (nx >= 4 && ny >= 4 && nz >= 4 && mglevel < P.mgmaxlevels && mglevel + 1 < (int)lv.size()) {
    std::vector<double> res((size_t)(nx + 3) * (ny + 3) * (nz + 3));
    residual3d(nx, ny, nz, dxsqi, dysqi, dzsqi, phi, rho, res.data(), mglevel, bounds, P, false, C);
    const Level& Lc = lv[mglevel + 1];
    double dxcsqi = 1. / (Lc.dx * Lc.dx), dycsqi = 1. / (Lc.dy * Lc.dy), dzcsqi = 1. / (Lc.dz * Lc.dz);
    std::vector<double> phic((size_t)(Lc.nx + 3) * (Lc.ny + 3) * (Lc.nz + 3), 0.);
    std::vector<double> rhoc((size_t)(Lc.nx + 1) * (Lc.ny + 1) * (Lc.nz + 1), 0.);
    double ff = (dxsqi + dysqi + dzsqi) / (dxcsqi + dycsqi + dzcsqi);
    restrict3d(nx, ny, nz, res.data(), Lc.nx, Lc.ny, Lc.nz, rhoc.data(), ff, bounds);
    vcycle(mglevel + 1, lv, phic.data(), rhoc.data(), bounds, P, C);
    expand3d(nx, ny, nz, phi, Lc.nx, Lc.ny, Lc.nz, phic.data(), bounds);
    applybc(nx, ny, nz, 1, phi, bounds, false, false);
  }
  for (int i = 0; i < P.uppasses; ++i) sorpass3d(mglevel, nx, ny, nz, phi, rho, dxsqi, dysqi, dzsqi, bounds, P, C);
}

// fullmultigrid3dsolve below the finest level (f3d_mgrid.F:502-945): rho is
// this level's source (already scaled), phi its potential. Coarser levels are
// solved first from the restricted rho (ghost width 0), their phi expanded
// into a zeroed phi here; a coarse level then does mgmaxvcycles V-cycles
// without a convergence test. Level 0 stops after the expansion: the caller
// iterates it to convergence.
void fmg_level(int mglevel, const std::vector<Level>& lv, double* phi, const double* rho, const int* bounds,
               const MGParams& P, Conductors& C, int mgmaxvcycles) {
  const Level& L = lv[mglevel];
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  if (nx >= 4 && ny >= 4 && nz >= 4 && mglevel < P.mgmaxlevels && mglevel + 1 < (int)lv.size()) {
    const Level& Lc = lv[mglevel + 1];
    double dxsqi = 1. / (L.dx * L.dx), dysqi = 1. / (L.dy * L.dy), dzsqi = 1. / (L.dz * L.dz);
    double dxcsqi = 1. / (Lc.dx * Lc.dx), dycsqi = 1. / (Lc.dy * Lc.dy), dzcsqi = 1. / (Lc.dz * Lc.dz);
    double ff = (dxsqi + dysqi + dzsqi) / (dxcsqi + dycsqi + dzcsqi);
    std::vector<double> rpad((size_t)(nx + 3) * (ny + 3) * (nz + 3), 0.);
    for (int iz = 0; iz <= nz; ++iz)
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) rpad[pidx(nx, ny, ix, iy, iz)] = rho[ridx(nx, ny, ix, iy, iz)];
    std::vector<double> rhoc((size_t)(Lc.nx + 1) * (Lc.ny + 1) * (Lc.nz + 1), 0.);
    restrict3d(nx, ny, nz, rpad.data(), Lc.nx, Lc.ny, Lc.nz, rhoc.data(), ff, bounds, 0);
    std::vector<double> phic((size_t)(Lc.nx + 3) * (Lc.ny + 3) * (Lc.nz + 3), 0.);
    fmg_level(mglevel + 1, lv, phic.data(), rhoc.data(), bounds, P, C, mgmaxvcycles);
    std::fill(phi, phi + (size_t)(nx + 3) * (ny + 3) * (nz + 3), 0.);
    expand3d(nx, ny, nz, phi, Lc.nx, Lc.ny, Lc.nz, phic.data(), bounds);
  }
  applybc(nx, ny, nz, 1, phi, bounds, false, false);
  if (mglevel == 0) return;
  for (int it = 0; it < mgmaxvcycles; ++it) vcycle(mglevel, lv, phi, rho, bounds, P, C);
  applybc(nx, ny, nz, 1, phi, bounds, true, false);
}

}  // namespace

// ===========================================================================
// C ABI of the oracle (ctypes)
// ===========================================================================
extern "C" {

struct or_conductors;  // opaque

int or_mglevels(int nx, int ny, int nz, double dx, double dy, double dz, int* out_n, double* out_d, int maxlev) {
  auto lv = mglevels(nx, ny, nz, dx, dy, dz);
  int n = std::min((int)lv.size(), maxlev);
  for (int i = 0; i < n; ++i) {
    out_n[3 * i] = lv[i].nx; out_n[3 * i + 1] = lv[i].ny; out_n[3 * i + 2] = lv[i].nz;
    out_d[3 * i] = lv[i].dx; out_d[3 * i + 1] = lv[i].dy; out_d[3 * i + 2] = lv[i].dz;
  }
  return (int)lv.size();
}

or_conductors* or_cond_new(int nx, int ny, int nz, double dx, double dy, double dz) {
  Conductors* C = new Conductors();
  C->lv = mglevels(nx, ny, nz, dx, dy, dz);
  C->levels = (int)C->lv.size();
  return reinterpret_cast<or_conductors*>(C);
}
void or_cond_free(or_conductors* c) { delete reinterpret_cast<Conductors*>(c); }

// Adds a shape on every MG level: kind 0 ZCylinderOut, 1 ZCylinder, 2 Sphere.
int or_cond_add_shape(or_conductors* c, int kind, double radius, double length, double voltage, double xcent,
                      double ycent, double zcent, int condid, double xmmin, double ymmin, double zmmin,
                      double dfill) {
  Conductors* C = reinterpret_cast<Conductors*>(c);
  Shape s{kind, radius, length, voltage, xcent, ycent, zcent, condid};
  for (int l = 0; l < C->levels; ++l) delfromintercepts(s, C->lv[l], xmmin, ymmin, zmmin, l, dfill, 1.e-13, *C);
  return 0;
}

// Adds raw conductor points (same layout as ConductorType).
int or_cond_add_points(or_conductors* c, int kind, int64_t n, const int* indx, const double* dels,
                       const double* volt, const int* ilevel) {
  Conductors* C = reinterpret_cast<Conductors*>(c);
  for (int64_t i = 0; i < n; ++i) {
    int ix = indx[3 * i], iy = indx[3 * i + 1], iz = indx[3 * i + 2];
    if (kind == 0) {
      C->interior.indx.insert(C->interior.indx.end(), {ix, iy, iz});
      C->interior.volt.push_back(volt[i]);
      C->interior.numb.push_back(0);
      C->interior.ilevel.push_back(ilevel[i]);
    } else {
      Subgrid& S = ((ix + iy + iz) % 2 == 0) ? C->even : C->odd;
      S.indx.insert(S.indx.end(), {ix, iy, iz});
      for (int k = 0; k < 6; ++k) { S.dels.push_back(dels[6 * i + k]); S.volt.push_back(volt[6 * i + k]); S.numb.push_back(0); }
      S.ilevel.push_back(ilevel[i]);
      S.prevphi.push_back(0.);
    }
  }
  return 0;
}

// checkconductors, f3d_mgrid.F:3964-4050
int or_cond_finalize(or_conductors* c) {
  Conductors* C = reinterpret_cast<Conductors*>(c);
  for (int l = 0; l < C->levels; ++l) checkconductors_work(*C, C->lv[l].nx, C->lv[l].ny, C->lv[l].nz, l);
  sort_interior(C->interior, C->levels);
  sort_subgrid(C->even, C->levels);
  sort_subgrid(C->odd, C->levels);
  return 0;
}

// Counts: out[0] interior, out[1] even subgrid, out[2] odd subgrid.
void or_cond_counts(or_conductors* c, int64_t* out) {
  Conductors* C = reinterpret_cast<Conductors*>(c);
  out[0] = (int64_t)C->interior.n();
  out[1] = (int64_t)C->even.n();
  out[2] = (int64_t)C->odd.n();
}
// which: 0 interior, 1 even, 2 odd. dels/volt arrays are 6 per point for
// subgrid and 1 per point (volt) for interior.
void or_cond_export(or_conductors* c, int which, int* indx, double* dels, double* volt, int* ilevel) {
  Conductors* C = reinterpret_cast<Conductors*>(c);
  if (which == 0) {
    const Interior& I = C->interior;
    std::memcpy(indx, I.indx.data(), I.indx.size() * sizeof(int));
    std::memcpy(volt, I.volt.data(), I.volt.size() * sizeof(double));
    std::memcpy(ilevel, I.ilevel.data(), I.ilevel.size() * sizeof(int));
  } else {
    const Subgrid& S = (which == 1) ? C->even : C->odd;
    std::memcpy(indx, S.indx.data(), S.indx.size() * sizeof(int));
    std::memcpy(dels, S.dels.data(), S.dels.size() * sizeof(double));
    std::memcpy(volt, S.volt.data(), S.volt.size() * sizeof(double));
    std::memcpy(ilevel, S.ilevel.data(), S.ilevel.size() * sizeof(int));
  }
}

// multigrid3dsolve, f3d_mgrid.F:83-500 (serial, no bends, no precalculated
// coefficients; mgform 1 or 2). phi is (nx+3)(ny+3)(nz+3) with guards, rho is
// (nx+1)(ny+1)(nz+1). rho is not modified (the reference scales it in place
// and unscales it afterwards). cond may be NULL.
// multigrid3dsolve (f3d_mgrid.F:83-500), or with mgmaxvcycles > 0 the full
// multigrid fullmultigrid3dsolve (:502-945, mgform 1 only): the coarse
// levels give the starting phi, then level 0 iterates as multigrid3dsolve.
int or_mgsolve(int nx, int ny, int nz, double dx, double dy, double dz, const int* bounds, double* phi,
               const double* rho, or_conductors* cond, double mgparam, double mgtol, int mgmaxiters,
               int mgmaxlevels, int downpasses, int uppasses, int mgform, int lcndbndy, int* mgiters_out,
               double* mgerror_out, int mgmaxvcycles) {
  Conductors empty;
  Conductors* C = cond ? reinterpret_cast<Conductors*>(cond) : &empty;
  std::vector<Level> lv = mglevels(nx, ny, nz, dx, dy, dz);
  if (!cond) {
    empty.levels = (int)lv.size();
    empty.lv = lv;
    sort_interior(empty.interior, empty.levels);
    sort_subgrid(empty.even, empty.levels);
    sort_subgrid(empty.odd, empty.levels);
  }
  if (C->levels != (int)lv.size()) return -3;
  MGParams P{mgparam, mgform, mgmaxiters, mgmaxlevels, downpasses, uppasses, 2, lcndbndy};
  P.mgtol = mgtol;
  double dxsqi = 1. / (dx * dx), dysqi = 1. / (dy * dy), dzsqi = 1. / (dz * dz);
  double reps0c = mgparam / (EPS0 * 2. * (dxsqi + dysqi + dzsqi));
  const size_t nr = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
  const size_t np = (size_t)(nx + 3) * (ny + 3) * (nz + 3);
  std::vector<double> rhs(nr);
  for (size_t i = 0; i < nr; ++i) rhs[i] = rho[i] * reps0c;
  if (mgmaxvcycles > 0) {
    if (mgform != 1) return -4;
    fmg_level(0, lv, phi, rhs.data(), bounds, P, *C, mgmaxvcycles);
  } else {
    applybc(nx, ny, nz, 1, phi, bounds, false, false);
  }
  std::vector<double> rhosave, res;
  if (mgform == 2) { rhosave = rhs; res.resize(np); }
  std::vector<double> phisave(np);
  int mgiters = 0;
  double mgerror = 2. * mgtol + 1.;
  while (mgerror > mgtol && mgiters < mgmaxiters) {
    mgiters += 1;
    std::copy(phi, phi + np, phisave.begin());
    if (mgform == 2) {
      cond_potmg(C->interior, nx, ny, phisave.data(), 0, mgform, true);
      condbndymgint(*C, nx, ny, nz, phisave.data(), bounds, 0);
      residual3d(nx, ny, nz, dxsqi, dysqi, dzsqi, phisave.data(), rhosave.data(), res.data(), 0, bounds, P, true, *C);
      for (int iz = 0; iz <= nz; ++iz)
        for (int iy = 0; iy <= ny; ++iy)
          for (int ix = 0; ix <= nx; ++ix) rhs[ridx(nx, ny, ix, iy, iz)] = res[pidx(nx, ny, ix, iy, iz)];
      std::fill(phi, phi + np, 0.);
    }
    vcycle(0, lv, phi, rhs.data(), bounds, P, *C);
    if (mgform == 2) {
      par_for(0, (int64_t)np, [&](int64_t i) { phi[i] = phi[i] + phisave[i]; });
      applybc(nx, ny, nz, 1, phi, bounds, false, false);
    }
    mgerror = par_max(0, nz + 1, [&](int64_t iz) {
      double m = 0.;
      for (int iy = 0; iy <= ny; ++iy)
        for (int ix = 0; ix <= nx; ++ix) {
          size_t p = pidx(nx, ny, ix, iy, (int)iz);
          m = std::max(m, std::fabs(phisave[p] - phi[p]));
        }
      return m;
    }, (int64_t)(nx + 1) * (ny + 1));
  }
  applybc(nx, ny, nz, 1, phi, bounds, true, false);
  *mgiters_out = mgiters;
  *mgerror_out = mgerror;
  return 0;
}

// Relative residual max|res| / max|rhs| over the nodes 0..n, where res is
// the reference's own level-0 residual (getresidual) and rhs = rho*reps0c;
// both carry the same scale factor, which cancels in the ratio.
double or_relresidual(int nx, int ny, int nz, double dx, double dy, double dz, const int* bounds,
                      const double* phi, const double* rho, or_conductors* cond, double mgparam) {
  Conductors empty;
  Conductors* C = cond ? reinterpret_cast<Conductors*>(cond) : &empty;
  std::vector<Level> lv = mglevels(nx, ny, nz, dx, dy, dz);
  if (!cond) {
    empty.levels = (int)lv.size();
    sort_interior(empty.interior, empty.levels);
    sort_subgrid(empty.even, empty.levels);
    sort_subgrid(empty.odd, empty.levels);
  }
  MGParams P{mgparam, 1, 1, 101, 1, 1, 2, 1};
  double dxsqi = 1. / (dx * dx), dysqi = 1. / (dy * dy), dzsqi = 1. / (dz * dz);
  double reps0c = mgparam / (EPS0 * 2. * (dxsqi + dysqi + dzsqi));
  const size_t nr = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<double> rhs(nr), res((size_t)(nx + 3) * (ny + 3) * (nz + 3));
  std::vector<double> ph(phi, phi + res.size());
  for (size_t i = 0; i < nr; ++i) rhs[i] = rho[i] * reps0c;
  // residual of MultiGrid3D.getresidual (scripts/multigrid.py:940-950):
  // level-0 residual3d with mgform = 1, so rows next to conductors carry
  // the ppp = min(dels) scaling of condbndyres
  residual3d(nx, ny, nz, dxsqi, dysqi, dzsqi, ph.data(), rhs.data(), res.data(), 0, bounds, P, false, *C);
  const double rmax = par_max(0, nz + 1, [&](int64_t iz) {
    double m = 0.;
    for (int iy = 0; iy <= ny; ++iy)
      for (int ix = 0; ix <= nx; ++ix) m = std::max(m, std::fabs(res[pidx(nx, ny, ix, iy, (int)iz)]));
    return m;
  }, (int64_t)(nx + 1) * (ny + 1));
  const double bmax = par_max(0, nz + 1, [&](int64_t iz) {
    double m = 0.;
    for (int iy = 0; iy <= ny; ++iy)
      for (int ix = 0; ix <= nx; ++ix) m = std::max(m, std::fabs(rhs[ridx(nx, ny, ix, iy, (int)iz)]));
    return m;
  }, (int64_t)(nx + 1) * (ny + 1));
  return bmax > 0. ? rmax / bmax : rmax;
}

// setrho3ddirect1 (no symmetry, ny > 0), pywarp90/w3d.F:7757-7960. Adds into
// rho(0:nx,0:ny,0:nz). Particles with gaminv == 0 (lost) are skipped.
void or_setrho(int nx, int ny, int nz, double dx, double dy, double dz, double xmmin, double ymmin, double zmmin,
               double zgrid, double* rho, int64_t np, const double* xp, const double* yp, const double* zp,
               const double* gaminv, double q, double wght) {
  double g = wght * q;
  g = g / dx;
  g = g / dy;
  g = g / dz;
  double dxi = 1. / dx, dyi = 1. / dy, dzi = 1. / dz;
  auto deposit = [&](int64_t ip) {
    if (gaminv && gaminv[ip] == 0.) return;
    int ii, jj, kk;
    double u1, v1, w1;
    cellfrac((xp[ip] - xmmin) * dxi, nx, ii, u1);
    cellfrac((yp[ip] - ymmin) * dyi, ny, jj, v1);
    cellfrac((zp[ip] - zgrid - zmmin) * dzi, nz, kk, w1);
    double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
    rho[ridx(nx, ny, ii, jj, kk)] += u0 * v0 * w0 * g;
    rho[ridx(nx, ny, ii + 1, jj, kk)] += u1 * v0 * w0 * g;
    rho[ridx(nx, ny, ii, jj + 1, kk)] += u0 * v1 * w0 * g;
    rho[ridx(nx, ny, ii + 1, jj + 1, kk)] += u1 * v1 * w0 * g;
    rho[ridx(nx, ny, ii, jj, kk + 1)] += u0 * v0 * w1 * g;
    rho[ridx(nx, ny, ii + 1, jj, kk + 1)] += u1 * v0 * w1 * g;
    rho[ridx(nx, ny, ii, jj + 1, kk + 1)] += u0 * v1 * w1 * g;
    rho[ridx(nx, ny, ii + 1, jj + 1, kk + 1)] += u1 * v1 * w1 * g;
  };
  const int nt = nthreads();
  if (nt <= 1 || np < kParMin || nz < 2) {
    for (int64_t ip = 0; ip < np; ++ip) deposit(ip);
    return;
  }
  // Parallel over z slabs of cells. A particle in cell kk writes node planes
  // kk and kk + 1, so slabs two apart never share a plane: the even slabs
  // run at once, then the odd ones. Within a slab the particles keep their
  // order, so the result is fixed for a given thread count; it differs from
  // the serial loop only by the order of the adds on the shared planes.
  const int nslab = std::min(2 * nt, nz);
  std::vector<int> slab(np);
  par_for(0, np, [&](int64_t ip) {
    int kk;
    double w1;
    cellfrac((zp[ip] - zgrid - zmmin) * dzi, nz, kk, w1);
    slab[ip] = (int)((int64_t)kk * nslab / nz);
  });
  std::vector<int64_t> start(nslab + 1, 0);
  for (int64_t ip = 0; ip < np; ++ip) ++start[slab[ip] + 1];
  for (int b = 0; b < nslab; ++b) start[b + 1] += start[b];
  std::vector<int64_t> order(np), fill(start.begin(), start.end() - 1);
  for (int64_t ip = 0; ip < np; ++ip) order[fill[slab[ip]]++] = ip;
  for (int phase = 0; phase < 2; ++phase)
    par_for(0, (nslab - phase + 1) / 2, [&](int64_t h) {
      const int b = 2 * (int)h + phase;
      for (int64_t t = start[b]; t < start[b + 1]; ++t) deposit(order[t]);
    }, kParMin);
}

// applyrhoboundaryconditions3d (serial, nguardrho = 0), w3d.F:2660-2750
void or_rhobc(int nx, int ny, int nz, double* rho, const int* bounds) {
  auto R = [&](int ix, int iy, int iz) -> double& { return rho[ridx(nx, ny, ix, iy, iz)]; };
  if (bounds[0] == 1) for (int iz = 0; iz <= nz; ++iz) for (int iy = 0; iy <= ny; ++iy) R(0, iy, iz) += R(0, iy, iz);
  if (bounds[1] == 1) for (int iz = 0; iz <= nz; ++iz) for (int iy = 0; iy <= ny; ++iy) R(nx, iy, iz) += R(nx, iy, iz);
  if (bounds[0] == 2 || bounds[1] == 2)
    for (int iz = 0; iz <= nz; ++iz) for (int iy = 0; iy <= ny; ++iy) { R(0, iy, iz) += R(nx, iy, iz); R(nx, iy, iz) = R(0, iy, iz); }
  if (bounds[2] == 1) for (int iz = 0; iz <= nz; ++iz) for (int ix = 0; ix <= nx; ++ix) R(ix, 0, iz) += R(ix, 0, iz);
  if (bounds[3] == 1) for (int iz = 0; iz <= nz; ++iz) for (int ix = 0; ix <= nx; ++ix) R(ix, ny, iz) += R(ix, ny, iz);
  if (bounds[2] == 2 || bounds[3] == 2)
    for (int iz = 0; iz <= nz; ++iz) for (int ix = 0; ix <= nx; ++ix) { R(ix, 0, iz) += R(ix, ny, iz); R(ix, ny, iz) = R(ix, 0, iz); }
  if (bounds[4] == 1) for (int iy = 0; iy <= ny; ++iy) for (int ix = 0; ix <= nx; ++ix) R(ix, iy, 0) += R(ix, iy, 0);
  if (bounds[5] == 1) for (int iy = 0; iy <= ny; ++iy) for (int ix = 0; ix <= nx; ++ix) R(ix, iy, nz) += R(ix, iy, nz);
  if (bounds[4] == 2 || bounds[5] == 2)
    for (int iy = 0; iy <= ny; ++iy) for (int ix = 0; ix <= nx; ++ix) { R(ix, iy, 0) += R(ix, iy, nz); R(ix, iy, nz) = R(ix, iy, 0); }
}

// sete_from_phi_linear3d (no symmetry), w3d.F:3963-4108. E is ADDED to ex,ey,ez.
void or_sete(int nx, int ny, int nz, double dx, double dy, double dz, double xmmin, double ymmin, double zmmin,
             double zgrid, const double* phi, int64_t np, const double* xp, const double* yp, const double* zp,
             double* ex, double* ey, double* ez) {
  double tdxi = 1. / (2. * dx), tdyi = 1. / (2. * dy), tdzi = 1. / (2. * dz);
  double dxi = 1. / dx, dyi = 1. / dy, dzi = 1. / dz;
  auto P = [&](int ix, int iy, int iz) { return phi[pidx(nx, ny, ix, iy, iz)]; };
  // particles are independent
  par_for(0, np, [&](int64_t ip) {
    int i, j, k;
    double u1, v1, w1;
    cellfrac((xp[ip] - xmmin) * dxi, nx, i, u1);
    cellfrac((yp[ip] - ymmin) * dyi, ny, j, v1);
    cellfrac((zp[ip] - zgrid - zmmin) * dzi, nz, k, w1);
    double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
    double ext = tdxi * (u0 * v0 * w0 * (P(i - 1, j, k) - P(i + 1, j, k)) + u1 * v0 * w0 * (P(i, j, k) - P(i + 2, j, k)) +
                         u0 * v1 * w0 * (P(i - 1, j + 1, k) - P(i + 1, j + 1, k)) +
                         u1 * v1 * w0 * (P(i, j + 1, k) - P(i + 2, j + 1, k)) +
                         u0 * v0 * w1 * (P(i - 1, j, k + 1) - P(i + 1, j, k + 1)) +
                         u1 * v0 * w1 * (P(i, j, k + 1) - P(i + 2, j, k + 1)) +
                         u0 * v1 * w1 * (P(i - 1, j + 1, k + 1) - P(i + 1, j + 1, k + 1)) +
                         u1 * v1 * w1 * (P(i, j + 1, k + 1) - P(i + 2, j + 1, k + 1)));
    double eyt = tdyi * (u0 * v0 * w0 * (P(i, j - 1, k) - P(i, j + 1, k)) + u1 * v0 * w0 * (P(i + 1, j - 1, k) - P(i + 1, j + 1, k)) +
                         u0 * v1 * w0 * (P(i, j, k) - P(i, j + 2, k)) + u1 * v1 * w0 * (P(i + 1, j, k) - P(i + 1, j + 2, k)) +
                         u0 * v0 * w1 * (P(i, j - 1, k + 1) - P(i, j + 1, k + 1)) +
                         u1 * v0 * w1 * (P(i + 1, j - 1, k + 1) - P(i + 1, j + 1, k + 1)) +
                         u0 * v1 * w1 * (P(i, j, k + 1) - P(i, j + 2, k + 1)) +
                         u1 * v1 * w1 * (P(i + 1, j, k + 1) - P(i + 1, j + 2, k + 1)));
    double ezt = tdzi * (u0 * v0 * w0 * (P(i, j, k - 1) - P(i, j, k + 1)) + u1 * v0 * w0 * (P(i + 1, j, k - 1) - P(i + 1, j, k + 1)) +
                         u0 * v1 * w0 * (P(i, j + 1, k - 1) - P(i, j + 1, k + 1)) +
                         u1 * v1 * w0 * (P(i + 1, j + 1, k - 1) - P(i + 1, j + 1, k + 1)) +
                         u0 * v0 * w1 * (P(i, j, k) - P(i, j, k + 2)) + u1 * v0 * w1 * (P(i + 1, j, k) - P(i + 1, j, k + 2)) +
                         u0 * v1 * w1 * (P(i, j + 1, k) - P(i, j + 1, k + 2)) +
                         u1 * v1 * w1 * (P(i + 1, j + 1, k) - P(i + 1, j + 1, k + 2)));
    ex[ip] = ex[ip] + ext;
    ey[ip] = ey[ip] + eyt;
    ez[ip] = ez[ip] + ezt;
  });
}

// Per-lattice-cell quad tables as built by setlattzt (top_lattice.F:1852-2030)
// for a hard-edge quad lattice repeated with period zlatperi: each lattice
// cell iz (centre zlmin + iz*dzl) takes the element whose territory (bounded
// by the midpoints of the drifts on either side) contains the centre.
// zs/ze/db describe one period of elements (sorted by zs).
void or_quad_table(int nquad, const double* zs, const double* ze, const double* db, double zlatperi,
                   double zlatstrt, double zlmin, double dzl, int nzl, double* czs, double* cze, double* cdb) {
  for (int iz = 0; iz <= nzl; ++iz) {
    double zz = zlmin + iz * dzl;
    double offset = std::floor((zz - zlatstrt) / zlatperi) * zlatperi + zlatstrt;
    double zloc = zz - offset;
    int best = 0;
    double left0 = 0.5 * (zs[0] + ze[nquad - 1] - zlatperi);
    if (zloc < left0) {
      best = nquad - 1;
      offset -= zlatperi;
    } else if (zloc >= left0 + zlatperi) {
      best = 0;
      offset += zlatperi;
    } else {
      for (int k = 0; k < nquad; ++k) {
        double left = (k == 0) ? left0 : 0.5 * (zs[k] + ze[k - 1]);
        double right = (k == nquad - 1) ? 0.5 * (ze[k] + zs[0] + zlatperi) : 0.5 * (ze[k] + zs[k + 1]);
        if (zloc >= left && zloc < right) { best = k; break; }
      }
    }
    czs[iz] = zs[best] + offset;
    cze[iz] = ze[best] + offset;
    cdb[iz] = db[best];
  }
}

// One particle advance of padvnc3d followed by the particle boundaries.
// center 0, "fullv" (w3d.F:1862-1987): E (already gathered, passed in
//   ex,ey,ez), B from applyquad (top_lattice.F:2985-3120) over the residence
//   window (-dt/2, +dt/2), epush3d half step, bpush3d (ibpush = 1) full step,
//   epush3d half step, xpush3d (gaminv fixed: lrelativ false), periz
//   (top.F:4015-4035), stckxy3d round pipe (w3d.F:11520-11535).
// center 1, "halfv" (w3d.F:1989-2125), the first step after loading, which
//   takes velocities from t to t+dt/2: window (0, +dt/2), bpush3d half step,
//   epush3d half step, then the same xpush3d, periz and pipe.
// center 2, "synchv" (w3d.F:2187-2310), which takes velocities from t-dt/2
//   back to t for diagnostics: window (-dt/2, 0), epush3d half step, bpush3d
//   half step; positions are not pushed and no boundary is applied.
// Lost particles get gaminv = 0 and are skipped.
void or_push(int center, int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp, double* uzp,
             double* gaminv, const double* ex, const double* ey, const double* ez, double q, double m, double dt,
             const double* czs, const double* cze, const double* cdb, int nzl, double zlmin, double dzl,
             double zmmin, double zmmax, double prwall, double prwallx, double prwally) {
  const double halfdt = 0.5 * dt;
  const double dtl = center == 1 ? 0. : -halfdt, dtr = center == 2 ? 0. : halfdt;
  const double bdt = center == 0 ? dt : halfdt;
  const double dzli = 1. / dzl;
  // particles are independent
  par_for(0, np, [&](int64_t ip) {
    if (gaminv[ip] == 0.) return;
    double bx = 0., by = 0., bz = 0.;
    if (czs) {
      double vz = uzp[ip] * gaminv[ip];
      double a = vz * (dtr - dtl);
      double dzi = std::fabs(1. / std::copysign(std::fabs(a) + SMALLPOS, a));
      int iz = (int)std::max(0., (zp[ip] - zlmin) * dzli + 0.5);
      if (iz > nzl) iz = nzl;
      double z1 = zp[ip] + vz * dtl, z2 = zp[ip] + vz * dtr;
      double zl = std::min(z1, z2);
      double fl = (zl >= czs[iz] && zl < cze[iz]) ? 1. : 0.;
      double zr = std::max(z1, z2);
      double fr = (zr >= czs[iz] && zr < cze[iz]) ? 1. : 0.;
      double frac = fl;
      if (fl > fr) frac = (cze[iz] - zl) * dzi;
      if (fr > fl) frac = (zr - czs[iz]) * dzi;
      if (frac > 0.) {
        bx = bx + cdb[iz] * frac * yp[ip];
        by = by + cdb[iz] * frac * xp[ip];
      }
    }
    const double cst = q * halfdt / m;
    if (center != 1) {
      // epush3d, half step
      uxp[ip] = uxp[ip] + ex[ip] * cst;
      uyp[ip] = uyp[ip] + ey[ip] * cst;
      uzp[ip] = uzp[ip] + ez[ip] * cst;
    }
    // bpush3d, ibpush = 1
    double cb = q * bdt * 0.5 / m;
    double tx = gaminv[ip] * bx * cb, ty = gaminv[ip] * by * cb, tz = gaminv[ip] * bz * cb;
    double tsqi = 2. / (1. + tx * tx + ty * ty + tz * tz);
    double sx = tx * tsqi, sy = ty * tsqi, sz = tz * tsqi;
    double uxppr = uxp[ip] + uyp[ip] * tz - uzp[ip] * ty;
    double uyppr = uyp[ip] + uzp[ip] * tx - uxp[ip] * tz;
    double uzppr = uzp[ip] + uxp[ip] * ty - uyp[ip] * tx;
    uxp[ip] = uxp[ip] + uyppr * sz - uzppr * sy;
    uyp[ip] = uyp[ip] + uzppr * sx - uxppr * sz;
    uzp[ip] = uzp[ip] + uxppr * sy - uyppr * sx;
    if (center == 2) return;
    // epush3d, half step
    uxp[ip] = uxp[ip] + ex[ip] * cst;
    uyp[ip] = uyp[ip] + ey[ip] * cst;
    uzp[ip] = uzp[ip] + ez[ip] * cst;
    // xpush3d
    xp[ip] = xp[ip] + uxp[ip] * gaminv[ip] * dt;
    yp[ip] = yp[ip] + uyp[ip] * gaminv[ip] * dt;
    zp[ip] = zp[ip] + uzp[ip] * gaminv[ip] * dt;
    // periz
    double syslen = zmmax - zmmin, sysleni = 1. / syslen;
    if (zp[ip] < zmmin) zp[ip] = zp[ip] + syslen * (int)((zmmax - zp[ip]) * sysleni);
    if (zp[ip] > zmmax) zp[ip] = zp[ip] - syslen * (int)((zp[ip] - zmmin) * sysleni);
    // stckxy3d, round aperture (prwelip = 1)
    double rx = xp[ip] - prwallx, ry = yp[ip] - prwally;
    if (rx * rx + ry * ry >= prwall * prwall) gaminv[ip] = 0.;
  });
}

// lcorrectede: E at particles next to conductors from the subgrid data.
// 1. icgrid over the level-0 nodes (setupconductorfielddata,
//    f3d_mgrid.F:4581-4632): 0 in vacuum, nmax+1 at level-0 interior points,
//    then the 1-based list index at even subgrid points and minus it at odd
//    ones, written in that order.
// 2. At every level-0 subgrid point, efield0 (centred, one per axis) and
//    efieldd (one-sided, one per direction, only towards an interior
//    neighbour) from phi and the conductor's dels/volt
//    (getefieldatconductorsubgrid and SETEE, f3d_mgrid.F:4635-4735). Nothing is
//    computed unless both subgrid lists are non-empty; the fields stay 0.
// 3. The efetch = 1 gather of sete3dwithconductor (f3d_mgrid.F:4774-5020,
//    GETEEFROME :5160-5220): particles outside the grid get nothing; cells
//    whose 8 nodes are all vacuum use centred differences with each term
//    scaled by 1/(2 dx); other cells weight, per edge of the cell, the
//    vacuum differences and the conductor points' fields by the particle's
//    weights, normalized by the weights used.
// A particle on an upper grid face uses the last cell with fraction 1 (the
// reference reads one node past the array there). E is ADDED to ex,ey,ez.
void or_sete_cond(or_conductors* hc, int nx, int ny, int nz, double dx, double dy, double dz, double xmmin,
                  double ymmin, double zmmin, double zgrid, const double* phi, int64_t np, const double* xp,
                  const double* yp, const double* zp, double* ex, double* ey, double* ez) {
  const Conductors& C = *reinterpret_cast<Conductors*>(hc);
  auto P = [&](int ix, int iy, int iz) { return phi[pidx(nx, ny, ix, iy, iz)]; };
  const int nmax = (int)std::max(C.even.n(), C.odd.n());
  std::vector<int> icgrid((size_t)(nx + 1) * (ny + 1) * (nz + 1), 0);
  auto ICG = [&](int ix, int iy, int iz) -> int& { return icgrid[ridx(nx, ny, ix, iy, iz)]; };
  const Interior& I = C.interior;
  for (int ic = I.istart[0]; ic < I.istart[1]; ++ic) ICG(I.indx[3 * ic], I.indx[3 * ic + 1], I.indx[3 * ic + 2]) = nmax + 1;
  for (int ie = C.even.istart[0]; ie < C.even.istart[1]; ++ie)
    ICG(C.even.indx[3 * ie], C.even.indx[3 * ie + 1], C.even.indx[3 * ie + 2]) = ie + 1;
  for (int io = C.odd.istart[0]; io < C.odd.istart[1]; ++io)
    ICG(C.odd.indx[3 * io], C.odd.indx[3 * io + 1], C.odd.indx[3 * io + 2]) = -(io + 1);

  std::vector<double> e0[2], ed[2];
  const Subgrid* L[2] = {&C.even, &C.odd};
  for (int s = 0; s < 2; ++s) {
    e0[s].assign(3 * L[s]->n(), 0.);
    ed[s].assign(6 * L[s]->n(), 0.);
  }
  if (C.even.n() > 0 && C.odd.n() > 0) {
    for (int s = 0; s < 2; ++s) {
      const Subgrid& S = *L[s];
      for (int ic = S.istart[0]; ic < S.istart[1]; ++ic) {
        const int ix = S.indx[3 * ic], iy = S.indx[3 * ic + 1], iz = S.indx[3 * ic + 2];
        const double* dels = &S.dels[6 * ic];
        const double* volt = &S.volt[6 * ic];
        for (int id = 0; id < 3; ++id) {
          const int mx = id == 0 ? -1 : 0, my = id == 1 ? -1 : 0, mz = id == 2 ? -1 : 0;
          const int px = -mx, py = -my, pz = -mz;
          const double di = id == 0 ? 1. / dx : id == 1 ? 1. / dy : 1. / dz;
          const int im = 2 * id, ip = 2 * id + 1;
          double vv0, dd0, vv1, dd1;
          if (0. < dels[im] && dels[im] <= 1.) { vv0 = volt[im]; dd0 = dels[im]; }
          else { vv0 = P(ix + mx, iy + my, iz + mz); dd0 = 1.; }
          if (0. < dels[ip] && dels[ip] <= 1.) { vv1 = volt[ip]; dd1 = dels[ip]; }
          else { vv1 = P(ix + px, iy + py, iz + pz); dd1 = 1.; }
          const double ppp = P(ix, iy, iz);
          e0[s][3 * ic + id] = (dd1 / (dd0 + dd1) * (vv0 - ppp) / dd0 + dd0 / (dd0 + dd1) * (ppp - vv1) / dd1) * di;
          if (ix + mx >= 0 && iy + my >= 0 && iz + mz >= 0 && ICG(ix + mx, iy + my, iz + mz) > nmax)
            ed[s][6 * ic + im] = ((vv0 - ppp) / dd0 - (2. - dd0) / (2. + dd1) * (ppp - vv1) / dd1) *
                                 ((2. + dd1) / (dd1 + dd0)) * di;
          if (ix + px <= nx && iy + py <= ny && iz + pz <= nz && ICG(ix + px, iy + py, iz + pz) > nmax)
            ed[s][6 * ic + ip] = ((ppp - vv1) / dd1 - (2. - dd1) / (2. + dd0) * (vv0 - ppp) / dd0) *
                                 ((2. + dd0) / (dd0 + dd1)) * di;
        }
      }
    }
  }
  auto E0 = [&](int ic, int id) { return ic < 0 ? e0[1][3 * (-ic - 1) + id] : e0[0][3 * (ic - 1) + id]; };
  auto ED = [&](int ic, int k) { return ic < 0 ? ed[1][6 * (-ic - 1) + k] : ed[0][6 * (ic - 1) + k]; };

  const double tdxi = 1. / (2. * dx), tdyi = 1. / (2. * dy), tdzi = 1. / (2. * dz);
  const double dxi = 1. / dx, dyi = 1. / dy, dzi = 1. / dz;
  // particles are independent
  par_for(0, np, [&](int64_t ip) {
    const double xi = (xp[ip] - xmmin) * dxi, yj = (yp[ip] - ymmin) * dyi, zk = (zp[ip] - zgrid - zmmin) * dzi;
    if (xi < 0. || xi > nx || yj < 0. || yj > ny || zk < 0. || zk > nz) return;
    int i, j, k;
    double u1, v1, w1;
    cellfrac(xi, nx, i, u1);
    cellfrac(yj, ny, j, v1);
    cellfrac(zk, nz, k, w1);
    const double u0 = 1. - u1, v0 = 1. - v1, w0 = 1. - w1;
    double ext, eyt, ezt;
    if (ICG(i, j, k) == 0 && ICG(i + 1, j, k) == 0 && ICG(i, j + 1, k) == 0 && ICG(i + 1, j + 1, k) == 0 &&
        ICG(i, j, k + 1) == 0 && ICG(i + 1, j, k + 1) == 0 && ICG(i, j + 1, k + 1) == 0 &&
        ICG(i + 1, j + 1, k + 1) == 0) {
      ext = u0 * v0 * w0 * (P(i - 1, j, k) - P(i + 1, j, k)) * tdxi + u1 * v0 * w0 * (P(i, j, k) - P(i + 2, j, k)) * tdxi +
            u0 * v1 * w0 * (P(i - 1, j + 1, k) - P(i + 1, j + 1, k)) * tdxi +
            u1 * v1 * w0 * (P(i, j + 1, k) - P(i + 2, j + 1, k)) * tdxi +
            u0 * v0 * w1 * (P(i - 1, j, k + 1) - P(i + 1, j, k + 1)) * tdxi +
            u1 * v0 * w1 * (P(i, j, k + 1) - P(i + 2, j, k + 1)) * tdxi +
            u0 * v1 * w1 * (P(i - 1, j + 1, k + 1) - P(i + 1, j + 1, k + 1)) * tdxi +
            u1 * v1 * w1 * (P(i, j + 1, k + 1) - P(i + 2, j + 1, k + 1)) * tdxi;
      eyt = u0 * v0 * w0 * (P(i, j - 1, k) - P(i, j + 1, k)) * tdyi + u1 * v0 * w0 * (P(i + 1, j - 1, k) - P(i + 1, j + 1, k)) * tdyi +
            u0 * v1 * w0 * (P(i, j, k) - P(i, j + 2, k)) * tdyi + u1 * v1 * w0 * (P(i + 1, j, k) - P(i + 1, j + 2, k)) * tdyi +
            u0 * v0 * w1 * (P(i, j - 1, k + 1) - P(i, j + 1, k + 1)) * tdyi +
            u1 * v0 * w1 * (P(i + 1, j - 1, k + 1) - P(i + 1, j + 1, k + 1)) * tdyi +
            u0 * v1 * w1 * (P(i, j, k + 1) - P(i, j + 2, k + 1)) * tdyi +
            u1 * v1 * w1 * (P(i + 1, j, k + 1) - P(i + 1, j + 2, k + 1)) * tdyi;
      ezt = u0 * v0 * w0 * (P(i, j, k - 1) - P(i, j, k + 1)) * tdzi + u1 * v0 * w0 * (P(i + 1, j, k - 1) - P(i + 1, j, k + 1)) * tdzi +
            u0 * v1 * w0 * (P(i, j + 1, k - 1) - P(i, j + 1, k + 1)) * tdzi +
            u1 * v1 * w0 * (P(i + 1, j + 1, k - 1) - P(i + 1, j + 1, k + 1)) * tdzi +
            u0 * v0 * w1 * (P(i, j, k) - P(i, j, k + 2)) * tdzi + u1 * v0 * w1 * (P(i + 1, j, k) - P(i + 1, j, k + 2)) * tdzi +
            u0 * v1 * w1 * (P(i, j + 1, k) - P(i, j + 1, k + 2)) * tdzi +
            u1 * v1 * w1 * (P(i + 1, j + 1, k) - P(i + 1, j + 1, k + 2)) * tdzi;
    } else {
      double ee[3] = {0., 0., 0.}, ww[3] = {0., 0., 0.};
      // GETEEFROME: the cell edge from node a = (i+ox, j+oy, k+oz) to a + p
      auto edge = [&](int id, int ox, int oy, int oz, int px, int py, int pz, double di, double wm, double wp) {
        const int ax = i + ox, ay = j + oy, az = k + oz;
        int ic = ICG(ax, ay, az);
        if (ic == 0) {
          ee[id] = ee[id] + wm * (P(ax - px, ay - py, az - pz) - P(ax + px, ay + py, az + pz)) * 0.5 * di;
          ww[id] = ww[id] + wm;
        } else if (ic < nmax + 1) {
          ee[id] = ee[id] + wm * E0(ic, id);
          ww[id] = ww[id] + wm;
          if (ICG(ax + px, ay + py, az + pz) > nmax) {
            ee[id] = ee[id] + wp * ED(ic, 2 * id + 1);
            ww[id] = ww[id] + wp;
          }
        }
        ic = ICG(ax + px, ay + py, az + pz);
        if (ic == 0) {
          ee[id] = ee[id] + wp * (P(ax, ay, az) - P(ax + 2 * px, ay + 2 * py, az + 2 * pz)) * 0.5 * di;
          ww[id] = ww[id] + wp;
        } else if (ic < nmax + 1) {
          ee[id] = ee[id] + wp * E0(ic, id);
          ww[id] = ww[id] + wp;
          if (ICG(ax, ay, az) > nmax) {
            ee[id] = ee[id] + wm * ED(ic, 2 * id);
            ww[id] = ww[id] + wm;
          }
        }
      };
      edge(0, 0, 0, 0, 1, 0, 0, dxi, u0 * v0 * w0, u1 * v0 * w0);
      edge(0, 0, 1, 0, 1, 0, 0, dxi, u0 * v1 * w0, u1 * v1 * w0);
      edge(0, 0, 0, 1, 1, 0, 0, dxi, u0 * v0 * w1, u1 * v0 * w1);
      edge(0, 0, 1, 1, 1, 0, 0, dxi, u0 * v1 * w1, u1 * v1 * w1);
      if (ww[0] != 0.) ww[0] = 1. / ww[0];
      edge(1, 0, 0, 0, 0, 1, 0, dyi, u0 * v0 * w0, u0 * v1 * w0);
      edge(1, 1, 0, 0, 0, 1, 0, dyi, u1 * v0 * w0, u1 * v1 * w0);
      edge(1, 0, 0, 1, 0, 1, 0, dyi, u0 * v0 * w1, u0 * v1 * w1);
      edge(1, 1, 0, 1, 0, 1, 0, dyi, u1 * v0 * w1, u1 * v1 * w1);
      if (ww[1] != 0.) ww[1] = 1. / ww[1];
      edge(2, 0, 0, 0, 0, 0, 1, dzi, u0 * v0 * w0, u0 * v0 * w1);
      edge(2, 1, 0, 0, 0, 0, 1, dzi, u1 * v0 * w0, u1 * v0 * w1);
      edge(2, 0, 1, 0, 0, 0, 1, dzi, u0 * v1 * w0, u0 * v1 * w1);
      edge(2, 1, 1, 0, 0, 0, 1, dzi, u1 * v1 * w0, u1 * v1 * w1);
      if (ww[2] != 0.) ww[2] = 1. / ww[2];
      ext = ee[0] * ww[0];
      eyt = ee[1] * ww[1];
      ezt = ee[2] * ww[2];
    }
    ex[ip] = ex[ip] + ext;
    ey[ip] = ey[ip] + eyt;
    ez[ip] = ez[ip] + ezt;
  });
}

// The moment sums of getzmmnt, itask = 2 (top.F:814-860 and 880-1160), for
// a non-relativistic species (lrelativ false: the velocities are the u
// themselves and the factors pp(13), pp(18) are 1) with ifzmmnt = 2. Lost particles (gaminv = 0) are
// skipped. zmmnts0[33]: the global sums over all particles. zmmnts
// [(nzmmnt+1)*33], moment fastest: each particle in [zmmntmin, zmmntmax)
// (relative to zbeam) is extrapolated in time to the two z-grid planes
// around it, with the velocity change between uo (the velocities dt earlier)
// and u, and adds to both planes with its linear weights times dtscale.
// The moment index k (0-based) is the reference's index k+1.
void or_zmoments(int64_t np, const double* xp, const double* yp, const double* zp, const double* uxp,
                 const double* uyp, const double* uzp, const double* gaminv, const double* uxpo, const double* uypo,
                 const double* uzpo, double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax,
                 int nzmmnt, double zmmntdtextmax, double* zmmnts0, double* zmmnts) {
  const int NM = 33;
  const double dzm = (zmmntmax - zmmntmin) / nzmmnt, dzmi = 1. / dzm;
  const double oneondt = 1. / dt;
  std::fill(zmmnts0, zmmnts0 + NM, 0.);
  std::fill(zmmnts, zmmnts + (size_t)(nzmmnt + 1) * NM, 0.);
  for (int64_t ip = 0; ip < np; ++ip) {
    if (gaminv[ip] == 0.) continue;
    const double x = xp[ip], y = yp[ip], z = zp[ip], ux = uxp[ip], uy = uyp[ip], uz = uzp[ip];
    double vzi = 1. / (uz + SMALLPOS);
    double* g = zmmnts0;
    g[0] += 1.;
    g[1] += x;
    g[2] += y;
    g[3] += z;
    g[6] += ux;
    g[7] += uy;
    g[8] += uz;
    g[9] += x * y;
    g[11] += x * x;
    g[12] += y * y;
    g[13] += z * z;
    g[16] += ux * ux;
    g[17] += uy * uy;
    g[18] += uz * uz;
    g[21] += z * uz;
    g[24] += x * uz;
    g[25] += y * uz;
    g[26] += ux * uz;
    g[27] += uy * uz;
    g[4] += ux * vzi;
    g[5] += uy * vzi;
    g[10] += ux * uy * (vzi * vzi);
    g[14] += (ux * vzi) * (ux * vzi);
    g[15] += (uy * vzi) * (uy * vzi);
    g[19] += x * ux * vzi;
    g[20] += y * uy * vzi;
    g[22] += x * uy * vzi;
    g[23] += y * ux * vzi;
    g[28] += x * ux;
    g[29] += y * uy;
    g[30] += x * uy;
    g[31] += y * ux;
    g[32] += ux * uy;
    if ((z - zbeam) < zmmntmin || (z - zbeam) >= zmmntmax) continue;
    const double vzgi = 1. / (uz * gaminv[ip] + SMALLPOS);
    int iz = (int)((z - zbeam - zmmntmin) * dzmi);
    if (iz == nzmmnt) iz = nzmmnt - 1;
    for (int side = 0; side < 2; ++side) {
      double dtx = ((iz + side) * dzm - z + zbeam + zmmntmin) * vzgi;
      dtx = std::max(-zmmntdtextmax * dt, std::min(zmmntdtextmax * dt, dtx));
      const double px = ux * (1. + dtx * oneondt) - uxpo[ip] * dtx * oneondt;
      const double py = uy * (1. + dtx * oneondt) - uypo[ip] * dtx * oneondt;
      const double pz = uz * (1. + dtx * oneondt) - uzpo[ip] * dtx * oneondt;
      const double qx = x + ux * dtx * gaminv[ip];
      const double qy = y + uy * dtx * gaminv[ip];
      const double qz = z + uz * dtx * gaminv[ip];
      const double w = side == 0 ? (1. - (z - zbeam - zmmntmin) * dzmi + iz) * dtscale
                                 : ((z - zbeam - zmmntmin) * dzmi - iz) * dtscale;
      const double v = 1. / (pz + SMALLPOS);
      double* m = zmmnts + (size_t)(iz + side) * NM;
      m[0] += w;
      m[1] += qx * w;
      m[2] += qy * w;
      m[3] += qz * w;
      m[6] += px * w;
      m[7] += py * w;
      m[8] += pz * w;
      m[9] += qx * qy * w;
      m[11] += qx * qx * w;
      m[12] += qy * qy * w;
      m[13] += qz * qz * w;
      m[16] += px * px * w;
      m[17] += py * py * w;
      m[18] += pz * pz * w;
      m[21] += qz * pz * w;
      m[24] += qx * pz * w;
      m[25] += qy * pz * w;
      m[26] += px * pz * w;
      m[27] += py * pz * w;
      m[4] += px * v * w;
      m[5] += py * v * w;
      m[10] += px * py * (v * v) * w;
      m[14] += (px * v) * (px * v) * w;
      m[15] += (py * v) * (py * v) * w;
      m[19] += qx * px * v * w;
      m[20] += qy * py * v * w;
      m[22] += qx * py * v * w;
      m[23] += qy * px * v * w;
      m[28] += qx * px * w;
      m[29] += qy * py * w;
      m[30] += qx * py * w;
      m[31] += qy * px * w;
      m[32] += px * py * w;
    }
  }
}

// Global moments of the live particles (getzmmnt, top.F:521-1444). out[]:
// 0 n, 1 xbar, 2 ybar, 3 xrms, 4 yrms, 5 epsx, 6 epsy (x' = ux/uz).
void or_moments(int64_t np, const double* xp, const double* yp, const double* uxp, const double* uyp,
                const double* uzp, const double* gaminv, double* out) {
  double s[12] = {0};
  for (int64_t ip = 0; ip < np; ++ip) {
    if (gaminv[ip] == 0.) continue;
    double vzi = 1. / (uzp[ip] + SMALLPOS);
    double xpr = uxp[ip] * vzi, ypr = uyp[ip] * vzi;
    s[0] += 1.;
    s[1] += xp[ip]; s[2] += yp[ip];
    s[3] += xpr; s[4] += ypr;
    s[5] += xp[ip] * xp[ip]; s[6] += yp[ip] * yp[ip];
    s[7] += xpr * xpr; s[8] += ypr * ypr;
    s[9] += xp[ip] * xpr; s[10] += yp[ip] * ypr;
  }
  double n = s[0] > 0. ? s[0] : 1.;
  double xb = s[1] / n, yb = s[2] / n, xpb = s[3] / n, ypb = s[4] / n;
  double dxsq = s[5] / n - xb * xb, dysq = s[6] / n - yb * yb;
  double dxpsq = s[7] / n - xpb * xpb, dypsq = s[8] / n - ypb * ypb;
  double dxxp = s[9] / n - xb * xpb, dyyp = s[10] / n - yb * ypb;
  out[0] = s[0];
  out[1] = xb;
  out[2] = yb;
  out[3] = std::sqrt(std::max(0., dxsq));
  out[4] = std::sqrt(std::max(0., dysq));
  out[5] = 4. * std::sqrt(std::max(0., dxsq * dxpsq - dxxp * dxxp));
  out[6] = 4. * std::sqrt(std::max(0., dysq * dypsq - dyyp * dyyp));
}

// getese3dfromrhophi (dw3d.F:708-777), no symmetry: ese = dx dy dz / 2 times
// the sum of rho*phi over nodes 0..n, summed over z per (x, y) column first,
// then over y into row 0, then over x, in that order.
double or_ese(int nx, int ny, int nz, const double* rho, const double* phi, double dx, double dy, double dz) {
  std::vector<double> scr((size_t)(nx + 1) * (ny + 1), 0.);
  const size_t sy = nx + 3, sz = (size_t)(nx + 3) * (ny + 3);
  for (int iz = 0; iz <= nz; ++iz)
    for (int iy = 0; iy <= ny; ++iy)
      for (int ix = 0; ix <= nx; ++ix) {
        const double r = rho[ix + (size_t)(nx + 1) * (iy + (size_t)(ny + 1) * iz)];
        const double p = phi[(ix + 1) + sy * (iy + 1) + sz * (iz + 1)];
        double& c = scr[ix + (size_t)(nx + 1) * iy];
        c = c + r * p;
      }
  for (int iy = 1; iy <= ny; ++iy)
    for (int ix = 0; ix <= nx; ++ix) scr[ix] = scr[ix] + scr[ix + (size_t)(nx + 1) * iy];
  double ese = 0.;
  for (int ix = 0; ix <= nx; ++ix) ese = ese + scr[ix];
  return dx * dy * dz * 0.5 * ese;
}

double or_eps0() { return EPS0; }

int or_threads() { return nthreads(); }

}  // extern "C"
