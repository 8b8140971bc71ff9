// Host-side conductor set-up: shapes -> per-level ConductorType lists.
//
// Runs once per installconductor (gridmode = 1, scripts/multigrid.py:743-783),
// not on the per-step path. The grid-line crossing rules follow
// conductordelfromintercepts (pywarp90/f3d_conductors.F:12-729) and the clean-up
// follows checkconductors (pywarp90/f3d_mgrid.F:3964-4326), because the
// solver's subgrid stencil consumes exactly those dels/volt values. The three
// grid-line directions are handled by one routine over a coordinate
// permutation.

#include <algorithm>
#include <array>
#include <cmath>
#include <map>

#include "wg_internal.h"

namespace wg {
namespace {

const double kLarge = 1.0e36;  // LARGEPOS, pywarp90/top.h:3
const double kFuzz = 1.0e-13;  // scripts/generateconductors.py:1856

struct ShapeDef {
  int kind;  // 0 ZCylinderOut, 1 ZCylinder, 2 Sphere
  double r, len, v, xc, yc, zc;
  int id;
};

// Crossing coordinates of the solid along a grid line in direction `axis`,
// through the point whose other two coordinates are p[] (p[axis] ignored).
// Returned as (entry, exit) pairs in increasing order.
void crossings(const ShapeDef& s, int axis, const double p[3], std::vector<double>& out) {
  out.clear();
  const double c[3] = {s.xc, s.yc, s.zc};
  if (s.kind == 2) {
    // offsets along the two other axes, lower axis first
    int lo = (axis == 0) ? 1 : 0, hi = (axis == 2) ? 1 : 2;
    double a = p[lo] - c[lo], b = p[hi] - c[hi];
    double d2 = s.r * s.r - a * a - b * b;
    if (d2 <= 0.) return;
    double h = std::sqrt(d2);
    out.push_back(c[axis] - h);
    out.push_back(c[axis] + h);
    return;
  }
  const double zmin = s.zc - 0.5 * s.len, zmax = s.zc + 0.5 * s.len;
  if (axis == 2) {
    double rr = (p[0] - s.xc) * (p[0] - s.xc) + (p[1] - s.yc) * (p[1] - s.yc);
    bool inside = rr < s.r * s.r;
    if ((s.kind == 1) == inside) {
      out.push_back(zmin);
      out.push_back(zmax);
    }
    return;
  }
  if (p[2] < zmin || p[2] > zmax) return;
  double off = (axis == 0) ? p[1] - s.yc : p[0] - s.xc;
  double d2 = s.r * s.r - off * off;
  double c0 = (axis == 0) ? s.xc : s.yc;
  if (s.kind == 1) {
    if (d2 <= 0.) return;
    double h = std::sqrt(d2);
    out.push_back(c0 - h);
    out.push_back(c0 + h);
  } else {
    if (d2 <= 0.) {
      out.push_back(-kLarge);
      out.push_back(kLarge);
      return;
    }
    double h = std::sqrt(d2);
    out.insert(out.end(), {-kLarge, c0 - h, c0 + h, kLarge});
  }
}

struct Sub {
  std::array<int, 3> ijk;
  std::array<double, 6> dels, volt;
};

// Per-level generator.
struct LevelGen {
  const ShapeDef& s;
  int n[3];
  double d[3], mn[3], mx[3], di[3];
  // crossing lists per axis, indexed by the two other node indices
  std::vector<std::vector<double>> lines[3];

  LevelGen(const ShapeDef& sh, const LevelDims& L, const double mins[3]) : s(sh) {
    n[0] = L.nx; n[1] = L.ny; n[2] = L.nz;
    d[0] = L.dx; d[1] = L.dy; d[2] = L.dz;
    for (int a = 0; a < 3; ++a) {
      mn[a] = mins[a];
      mx[a] = mins[a] + n[a] * d[a];
      di[a] = 1. / d[a];
    }
    for (int a = 0; a < 3; ++a) {
      int a1 = (a == 0) ? 1 : 0, a2 = (a == 2) ? 1 : 2;
      lines[a].resize((size_t)(n[a1] + 1) * (n[a2] + 1));
      for (int j2 = 0; j2 <= n[a2]; ++j2)
        for (int j1 = 0; j1 <= n[a1]; ++j1) {
          double p[3] = {0., 0., 0.};
          p[a1] = mn[a1] + j1 * d[a1];
          p[a2] = mn[a2] + j2 * d[a2];
          crossings(s, a, p, lines[a][(size_t)j1 + (size_t)(n[a1] + 1) * j2]);
        }
    }
  }
  // crossing list of the line along `a` through node ijk
  const std::vector<double>& line(int a, const int ijk[3]) const {
    int a1 = (a == 0) ? 1 : 0, a2 = (a == 2) ? 1 : 2;
    return lines[a][(size_t)ijk[a1] + (size_t)(n[a1] + 1) * ijk[a2]];
  }

  // Nearest-crossing update in direction a for a point at position pos
  // (side-alternating scan, f3d_conductors.F:334-397).
  void perp_update(int a, const std::vector<double>& ics, double pos, Sub& S) const {
    int cnt = (int)ics.size();
    bool plus = true;
    for (int k = 0; k < cnt; ++k, plus = !plus) {
      double dd;
      if (plus) dd = (k == 0 || pos > ics[k - 1]) ? (ics[k] - pos) * di[a] : kLarge;
      else dd = (k == cnt - 1 || pos < ics[k + 1]) ? (pos - ics[k]) * di[a] : kLarge;
      int slot = 2 * a + (plus ? 1 : 0);
      if (0. < dd && dd < 1. - kFuzz && dd < S.dels[slot]) {
        S.dels[slot] = dd;
        S.volt[slot] = s.v;
      }
    }
  }
  // Distance to the first crossing that brackets pos (f3d_conductors.F:471-486).
  double first_dist(int a, const std::vector<double>& ics, double pos) const {
    double dd = 2.;
    bool plus = true;
    for (size_t k = 0; k < ics.size() && !(dd < 1.); ++k, plus = !plus) {
      if (plus) { if (ics[k] >= pos) dd = (ics[k] - pos) * di[a]; }
      else { if (ics[k] <= pos) dd = (pos - ics[k]) * di[a]; }
    }
    return dd;
  }

  void subgrid_points(int a, std::vector<Sub>& out) const {
    int a1 = (a == 0) ? 1 : 0, a2 = (a == 2) ? 1 : 2;
    // loop order of the reference: outer index is the slower of the two
    for (int j2 = 0; j2 <= n[a2]; ++j2)
      for (int j1 = 0; j1 <= n[a1]; ++j1) {
        const auto& ics = lines[a][(size_t)j1 + (size_t)(n[a1] + 1) * j2];
        bool plus = false;
        for (size_t k = 0; k < ics.size(); ++k) {
          plus = !plus;
          double c = ics[k];
          if (!(mn[a] - d[a] < c && c < mx[a] + d[a])) continue;
          int i = (int)std::floor((c - mn[a]) * di[a]);
          double del;
          int slot;
          if (plus) {
            if (i < 0) continue;
            double xx = mn[a] + i * d[a];
            del = (k == 0 || xx > ics[k - 1]) ? (c - mn[a]) * di[a] - i : kLarge;
            slot = 2 * a + 1;
          } else {
            i = i + 1;
            if (i > n[a]) continue;
            double xx = mn[a] + i * d[a];
            del = (k == ics.size() - 1 || xx < ics[k + 1]) ? i - (c - mn[a]) * di[a] : kLarge;
            slot = 2 * a;
          }
          int ijk[3];
          ijk[a] = i;
          ijk[a1] = j1;
          ijk[a2] = j2;
          double pos[3] = {mn[0] + ijk[0] * d[0], mn[1] + ijk[1] * d[1], mn[2] + ijk[2] * d[2]};
          // points with a closer crossing along a lower axis were found there
          bool skip = false;
          for (int b = 0; b < a; ++b)
            if (first_dist(b, line(b, ijk), pos[b]) < 1. - kFuzz) skip = true;
          if (skip || !(0. < del && del < 1. - kFuzz)) continue;
          Sub S;
          S.ijk = {ijk[0], ijk[1], ijk[2]};
          S.dels.fill(kLarge);
          S.volt.fill(0.);
          S.dels[slot] = del;
          S.volt[slot] = s.v;
          for (int b = a + 1; b < 3; ++b) perp_update(b, line(b, ijk), pos[b], S);
          out.push_back(S);
        }
      }
  }

  void interior_points(double dfill, std::vector<std::array<int, 3>>& out) const {
    for (int iz = 0; iz <= n[2]; ++iz)
      for (int iy = 0; iy <= n[1]; ++iy) {
        int ijk0[3] = {0, iy, iz};
        const auto& xs = line(0, ijk0);
        for (size_t k = 0; k + 1 < xs.size(); k += 2) {
          double x1 = xs[k], x2 = xs[k + 1];
          if (!(x2 >= mn[0] && x1 <= mx[0])) continue;
          int i1 = (int)((std::max(x1 - kFuzz, mn[0]) - mn[0]) * di[0]);
          int i2 = (int)((std::min(x2 + kFuzz, mx[0]) - mn[0]) * di[0]);
          if (mn[0] + i1 * d[0] <= x1 && i1 < n[0]) i1 += 1;
          if (mn[0] + (i2 + 1) * d[0] <= x2 && i2 < n[0]) i2 += 1;
          for (int ix = i1; ix <= i2; ++ix) {
            double ddx = 0., ddy = 0., ddz = 0.;
            if (dfill < kLarge) {
              double xx = mn[0] + ix * d[0], yy = mn[1] + iy * d[1], zz = mn[2] + iz * d[2];
              int ijk[3] = {ix, iy, iz};
              ddx = std::min(xx - x1, x2 - xx);
              ddy = kLarge;
              ddz = kLarge;
              for (double v : line(1, ijk)) { ddy = std::min(ddy, std::fabs(yy - v)); if (v > yy) break; }
              for (double v : line(2, ijk)) { ddz = std::min(ddz, std::fabs(zz - v)); if (v > zz) break; }
            }
            if (ddx < dfill * d[0] || ddy < dfill * d[1] || ddz < dfill * d[2]) out.push_back({ix, iy, iz});
          }
        }
      }
  }
};

}  // namespace

int add_shape(HostConductors& C, const std::vector<LevelDims>& lv, double xmmin, double ymmin, double zmmin,
              int kind, double radius, double length, double voltage, double xcent, double ycent, double zcent,
              int condid, double dfill) {
  if (kind < 0 || kind > 2 || !(radius > 0.)) {
    set_error("wg_conductors_add_shape: unknown kind or non-positive radius");
    return WG_EINVAL;
  }
  ShapeDef s{kind, radius, length, voltage, xcent, ycent, zcent, condid};
  const double mins[3] = {xmmin, ymmin, zmmin};
  for (size_t l = 0; l < lv.size(); ++l) {
    LevelGen g(s, lv[l], mins);
    std::vector<std::array<int, 3>> ins;
    g.interior_points(dfill, ins);
    for (auto& p : ins) {
      C.int_indx.insert(C.int_indx.end(), {p[0], p[1], p[2]});
      C.int_volt.push_back(voltage);
      C.int_level.push_back((int32_t)l);
    }
    std::vector<Sub> subs;
    for (int a = 0; a < 3; ++a) g.subgrid_points(a, subs);
    for (auto& S : subs) {
      C.sub_indx.insert(C.sub_indx.end(), S.ijk.begin(), S.ijk.end());
      C.sub_dels.insert(C.sub_dels.end(), S.dels.begin(), S.dels.end());
      C.sub_volt.insert(C.sub_volt.end(), S.volt.begin(), S.volt.end());
      C.sub_level.push_back((int32_t)l);
    }
  }
  C.finalized = false;
  return WG_OK;
}

// checkconductors: per level, drop points off the mesh, drop subgrid points on
// interior points, merge duplicate subgrid points (nearest crossing per
// direction wins), then order everything by level.
int finalize_conductors(HostConductors& C, const std::vector<LevelDims>& lv) {
  const int nlev = (int)lv.size();
  const size_t nint = C.int_volt.size(), nsub = C.sub_level.size();
  std::vector<int32_t> ilev(C.int_level), slev(C.sub_level);
  for (int l = 0; l < nlev; ++l) {
    const LevelDims& L = lv[l];
    auto key = [&](int ix, int iy, int iz) {
      return (int64_t)ix + (int64_t)(L.nx + 1) * ((int64_t)iy + (int64_t)(L.ny + 1) * iz);
    };
    auto onmesh = [&](const int32_t* p) {
      return p[0] >= 0 && p[0] <= L.nx && p[1] >= 0 && p[1] <= L.ny && p[2] >= 0 && p[2] <= L.nz;
    };
    std::map<int64_t, int64_t> owner;  // node -> -1 interior, else subgrid index
    for (size_t i = 0; i < nint; ++i) {
      if (ilev[i] != l) continue;
      const int32_t* p = &C.int_indx[3 * i];
      if (!onmesh(p)) { ilev[i] = -1; continue; }
      auto it = owner.find(key(p[0], p[1], p[2]));
      if (it != owner.end()) { ilev[i] = -1; continue; }
      owner[key(p[0], p[1], p[2])] = -1;
    }
    for (int parity = 0; parity < 2; ++parity) {
      for (size_t i = 0; i < nsub; ++i) {
        if (slev[i] != l) continue;
        const int32_t* p = &C.sub_indx[3 * i];
        if (((p[0] + p[1] + p[2]) % 2 + 2) % 2 != parity) continue;
        if (!onmesh(p)) { slev[i] = -1; continue; }
        auto it = owner.find(key(p[0], p[1], p[2]));
        if (it == owner.end()) { owner[key(p[0], p[1], p[2])] = (int64_t)i; continue; }
        if (it->second == -1) { slev[i] = -1; continue; }
        size_t j = (size_t)it->second;
        for (int k = 0; k < 6; ++k) {
          double dn = C.sub_dels[6 * i + k];
          if (std::fabs(dn) < 1. && std::fabs(dn) < std::fabs(C.sub_dels[6 * j + k])) {
            C.sub_dels[6 * j + k] = dn;
            C.sub_volt[6 * j + k] = C.sub_volt[6 * i + k];
          }
        }
        slev[i] = -1;
      }
    }
  }
  C.istart_int.assign(nlev + 1, 0);
  C.istart_even.assign(nlev + 1, 0);
  C.istart_odd.assign(nlev + 1, 0);
  std::vector<int32_t> iidx, ilv;
  std::vector<double> ivolt;
  C.even_indx.clear(); C.odd_indx.clear(); C.even_dels.clear(); C.odd_dels.clear();
  C.even_volt.clear(); C.odd_volt.clear(); C.even_level.clear(); C.odd_level.clear();
  for (int l = 0; l < nlev; ++l) {
    C.istart_int[l] = (int32_t)ivolt.size();
    for (size_t i = 0; i < nint; ++i)
      if (ilev[i] == l) {
        iidx.insert(iidx.end(), &C.int_indx[3 * i], &C.int_indx[3 * i] + 3);
        ivolt.push_back(C.int_volt[i]);
        ilv.push_back(l);
      }
    C.istart_even[l] = (int32_t)C.even_level.size();
    C.istart_odd[l] = (int32_t)C.odd_level.size();
    for (size_t i = 0; i < nsub; ++i) {
      if (slev[i] != l) continue;
      const int32_t* p = &C.sub_indx[3 * i];
      bool even = ((p[0] + p[1] + p[2]) % 2) == 0;
      auto& ix = even ? C.even_indx : C.odd_indx;
      auto& ds = even ? C.even_dels : C.odd_dels;
      auto& vs = even ? C.even_volt : C.odd_volt;
      auto& lv2 = even ? C.even_level : C.odd_level;
      ix.insert(ix.end(), p, p + 3);
      ds.insert(ds.end(), &C.sub_dels[6 * i], &C.sub_dels[6 * i] + 6);
      vs.insert(vs.end(), &C.sub_volt[6 * i], &C.sub_volt[6 * i] + 6);
      lv2.push_back(l);
    }
  }
  C.istart_int[nlev] = (int32_t)ivolt.size();
  C.istart_even[nlev] = (int32_t)C.even_level.size();
  C.istart_odd[nlev] = (int32_t)C.odd_level.size();
  // keep the finalized interior lists in place of the raw ones
  C.int_indx.swap(iidx);
  C.int_volt.swap(ivolt);
  C.int_level.swap(ilv);
  // raw subgrid lists are rebuilt from even+odd so that a second finalize works
  C.sub_indx = C.even_indx;
  C.sub_indx.insert(C.sub_indx.end(), C.odd_indx.begin(), C.odd_indx.end());
  C.sub_dels = C.even_dels;
  C.sub_dels.insert(C.sub_dels.end(), C.odd_dels.begin(), C.odd_dels.end());
  C.sub_volt = C.even_volt;
  C.sub_volt.insert(C.sub_volt.end(), C.odd_volt.begin(), C.odd_volt.end());
  C.sub_level = C.even_level;
  C.sub_level.insert(C.sub_level.end(), C.odd_level.begin(), C.odd_level.end());
  C.finalized = true;
  return WG_OK;
}

}  // namespace wg
