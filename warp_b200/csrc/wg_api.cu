// C ABI entry points (include/warp_b200.h): context, level allocation,
// conductor upload, and dispatch to the solver and particle kernels.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "wg_internal.h"

namespace wg {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int solve(wg_ctx* c, const wg_solve_opts* o, wg_solve_stats* st);
int relresidual(wg_ctx* c, double mgparam, double* out);
int residual_field(wg_ctx* c, double mgparam, double* out);
int field_energy(wg_ctx* c, double* out);
int deposit(wg_ctx* c, const wg_particles* p, int zero_first);
int deposit_noalloc(const wg_grid* grid, const wg_particles* p, double* rho, int zero_first, void* stream);
int finalize_rho(wg_ctx* c);
int deposit_begin(wg_ctx* c);
int deposit_add(wg_ctx* c, const wg_particles* p);
int deposit_end(wg_ctx* c, int zero_first);
int fetch_e(wg_ctx* c, const double* x, const double* y, const double* z, double* ex, double* ey, double* ez,
            int64_t np);
int advance(wg_ctx* c, const wg_particles* p, const wg_push_params* prm);
int moments(wg_ctx* c, const wg_particles* p, double* out);
int zmoments(wg_ctx* c, const wg_particles* p, const double* uxo, const double* uyo, const double* uzo, double dt,
             double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt, double zmmntdtextmax,
             double* zmmnts0, double* zmmnts);
int moments_scratch_doubles(int nb);
int configure_kernels();
int deposit_f32(wg_ctx* c, const wg_particles_f32* p, int zero_first);
int deposit_add_f32(wg_ctx* c, const wg_particles_f32* p);
int advance_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm);
int advance_deposit(wg_ctx* c, const wg_particles* p, const wg_push_params* prm);
int advance_deposit_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm);
int moments_f32(wg_ctx* c, const wg_particles_f32* p, double* out);
int zmoments_f32(wg_ctx* c, const wg_particles_f32* p, const float* uxo, const float* uyo, const float* uzo,
                 double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt,
                 double zmmntdtextmax, double* zmmnts0, double* zmmnts);
int cell_keys_f32(wg_ctx* c, const wg_particles_f32* p, int64_t* keys);
int permute_f32(wg_ctx* c, const int64_t* perm, const wg_particles_f32* src, const wg_particles_f32* dst);

// getnextcoarselevel3d / getmglevels (f3d_mgrid.F:3601-3845), serial,
// mgcoarsening = 2.
std::vector<LevelDims> mglevels(int nx, int ny, int nz, double dx, double dy, double dz) {
  std::vector<LevelDims> lv;
  LevelDims f{nx, ny, nz, dx, dy, dz};
  for (int lev = 0;; ++lev) {
    lv.push_back(f);
    if (f.nx < 4 || (f.ny < 4 && f.ny > 0) || f.nz < 4 || lev == 100) break;
    LevelDims c;
    c.nx = (f.nx + 1) / 2;
    if (c.nx % 2 == 1) c.nx += 1;
    c.ny = (f.ny + 1) / 2;
    if (c.ny % 2 == 1) c.ny += 1;
    c.nz = (f.nz + 1) / 2;
    if (c.nz % 2 == 1) c.nz += 1;
    double mg = f.dx < f.dy ? f.dx : f.dy;
    mg = mg < f.dz ? mg : f.dz;
    if (f.dx > 4. / 3. * mg) c.nx = f.nx;
    if (f.dy > 4. / 3. * mg) c.ny = f.ny;
    if (f.dz > 4. / 3. * mg) c.nz = f.nz;
    c.dx = f.dx * f.nx / c.nx;
    c.dy = (c.ny == 0) ? c.dx : f.dy * f.ny / c.ny;
    c.dz = f.dz * f.nz / c.nz;
    f = c;
  }
  return lv;
}

template <typename T>
int dalloc(T** p, size_t n) {
  if (n == 0) { *p = nullptr; return WG_OK; }
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error(std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    return WG_ENOMEM;
  }
  e = cudaMemset(*p, 0, n * sizeof(T));
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return WG_ECUDA; }
  return WG_OK;
}
template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void free_conductor_data(wg_ctx* c) {
  for (Level& L : c->lv) {
    dfree(L.int_ijk);
    dfree(L.int_volt);
    L.n_int = 0;
    for (DevSubgrid& S : L.sub) {
      dfree(S.ijk);
      dfree(S.dels);
      dfree(S.volt);
      dfree(S.rhs);
      dfree(S.rhsf);
      S.n = 0;
    }
    L.has_neumann_sub = false;
  }
}

// Index and weight tables of expand3d (f3d_mgrid.F:1777-1947) from coarse
// level dc into level L, evaluated with the same integer and double
// expressions the reference uses per node.
int expand_tables(Level& L, const LevelDims& dc) {
  const int n[3] = {L.d.nx, L.d.ny, L.d.nz}, nc[3] = {dc.nx, dc.ny, dc.nz};
  const size_t tot = (size_t)(n[0] + 3) + (n[1] + 3) + (n[2] + 3);
  std::vector<int32_t> j(tot);
  std::vector<double> w(tot);
  size_t o = 0;
  for (int a = 0; a < 3; ++a)
    for (int i = -1; i <= n[a] + 1; ++i, ++o) {
      j[o] = (i * nc[a]) / n[a];
      w[o] = 1. * (i * nc[a]) / n[a] - j[o];
    }
  WG_TRY(dalloc(&L.ej, tot));
  WG_TRY(dalloc(&L.ew, tot));
  WG_TRY_CUDA(cudaMemcpy(L.ej, j.data(), tot * sizeof(int32_t), cudaMemcpyHostToDevice));
  WG_TRY_CUDA(cudaMemcpy(L.ew, w.data(), tot * sizeof(double), cudaMemcpyHostToDevice));
  return WG_OK;
}

// Window and weight tables of restrict3d (f3d_mgrid.F:1593-1775) from level
// L into coarse level dc, with the reference's per-node expressions.
// Index and weight tables of restrict3d (f3d_mgrid.F:1593-1775) from level L
// into coarse level dc, for a source with ng guard cells: ng = 1 for the
// V-cycle's residual, ng = 0 for rho in the full multigrid. A window clipped
// at its low end keeps the weights indexed from its unclipped start, as the
// reference's precalculated wxa/wya/wza are.
int restrict_tables_ng(const LevelDims& d, const LevelDims& dc, int ng, int32_t** dlo, int32_t** dn, double** dw,
                       int* rmax) {
  const int n[3] = {d.nx, d.ny, d.nz}, nc[3] = {dc.nx, dc.ny, dc.nz};
  const size_t tot = (size_t)(nc[0] + 1) + (nc[1] + 1) + (nc[2] + 1);
  std::vector<int32_t> lo(tot), cnt(tot);
  std::vector<double> w(tot * kRestrictTaps, 0.);
  size_t o = 0;
  *rmax = 0;
  for (int a = 0; a < 3; ++a) {
    const double dci = 1. * nc[a] / n[a];
    for (int ic = 0; ic <= nc[a]; ++ic, ++o) {
      const int l0 = ((ic - 1) * n[a] + 4 * nc[a]) / nc[a] - 3;
      int h = ((ic + 1) * n[a] - 1) / nc[a];
      const int l = std::max(l0, -ng);
      h = std::min(h, n[a] + ng);
      const int k = std::max(0, h - l + 1);
      if (k > kRestrictTaps) {
        set_error("wg_create: restriction window wider than 4 fine cells (coarsening ratio above 2)");
        return WG_EINVAL;
      }
      lo[o] = l;
      cnt[o] = k;
      if (a < 2) *rmax = std::max(*rmax, k);
      for (int t = 0; t < k; ++t) w[o * kRestrictTaps + t] = 1. - std::fabs(ic - (l0 + t + 0.) * dci);
    }
  }
  WG_TRY(dalloc(dlo, tot));
  WG_TRY(dalloc(dn, tot));
  WG_TRY(dalloc(dw, tot * kRestrictTaps));
  WG_TRY_CUDA(cudaMemcpy(*dlo, lo.data(), tot * sizeof(int32_t), cudaMemcpyHostToDevice));
  WG_TRY_CUDA(cudaMemcpy(*dn, cnt.data(), tot * sizeof(int32_t), cudaMemcpyHostToDevice));
  WG_TRY_CUDA(cudaMemcpy(*dw, w.data(), tot * kRestrictTaps * sizeof(double), cudaMemcpyHostToDevice));
  return WG_OK;
}

int restrict_tables(Level& L, const LevelDims& dc) {
  WG_TRY(restrict_tables_ng(L.d, dc, 1, &L.rlo, &L.rn, &L.rw, &L.rmax));
  return restrict_tables_ng(L.d, dc, 0, &L.rlo0, &L.rn0, &L.rw0, &L.rmax0);
}

void free_graphs(wg_ctx* c) {
  for (int i = 0; i < 2; ++i) {
    if (c->vgraph[i]) cudaGraphExecDestroy(c->vgraph[i]);
    c->vgraph[i] = nullptr;
    c->vgraph_key[i] = 0ull;
    if (c->cgraph[i]) cudaGraphExecDestroy(c->cgraph[i]);
    c->cgraph[i] = nullptr;
    c->cgraph_key[i] = 0ull;
  }
}

void free_all(wg_ctx* c) {
  free_graphs(c);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  c->cap_stream = nullptr;
  free_conductor_data(c);
  for (auto& e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  for (Level& L : c->lv) {
    dfree(L.phi);
    dfree(L.rhs);
    dfree(L.res);
    dfree(L.phif);
    dfree(L.rhsf);
    dfree(L.resf);
    dfree(L.ej);
    dfree(L.ew);
    dfree(L.rlo);
    dfree(L.rn);
    dfree(L.rw);
    dfree(L.rlo0);
    dfree(L.rn0);
    dfree(L.rw0);
  }
  dfree(c->phisave);
  dfree(c->rho);
  dfree(c->racc);
  dfree(c->dred);
  dfree(c->dslot);
  dfree(c->dmom);
  dfree(c->dese);
  dfree(c->zmom);
  dfree(c->czs);
  dfree(c->cze);
  dfree(c->cdb);
  dfree(c->icgrid);
  for (int s = 0; s < 2; ++s) {
    dfree(c->ef0[s]);
    dfree(c->efd[s]);
  }
  if (c->enode) cudaFree(c->enode);
  c->enode = nullptr;
  c->enode_n = 0;
  if (c->hred) cudaFreeHost(c->hred);
  c->hred = nullptr;
}

template <typename T>
int upload(T** d, const T* h, size_t n) {
  WG_TRY(dalloc(d, n));
  if (n) WG_TRY_CUDA(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return WG_OK;
}

int upload_conductors(wg_ctx* c) {
  free_graphs(c);
  c->cond_version += 1;
  free_conductor_data(c);
  HostConductors& C = c->cond;
  for (size_t l = 0; l < c->lv.size(); ++l) {
    Level& L = c->lv[l];
    int a = C.istart_int[l], b = C.istart_int[l + 1];
    L.n_int = b - a;
    WG_TRY(upload(&L.int_ijk, C.int_indx.data() + 3 * (size_t)a, 3 * (size_t)L.n_int));
    WG_TRY(upload(&L.int_volt, C.int_volt.data() + a, (size_t)L.n_int));
    for (int par = 0; par < 2; ++par) {
      const std::vector<int32_t>& ist = par ? C.istart_odd : C.istart_even;
      const std::vector<int32_t>& idx = par ? C.odd_indx : C.even_indx;
      const std::vector<double>& dl = par ? C.odd_dels : C.even_dels;
      const std::vector<double>& vl = par ? C.odd_volt : C.even_volt;
      DevSubgrid& S = L.sub[par];
      int s0 = ist[l], s1 = ist[l + 1];
      S.n = s1 - s0;
      WG_TRY(upload(&S.ijk, idx.data() + 3 * (size_t)s0, 3 * (size_t)S.n));
      WG_TRY(upload(&S.dels, dl.data() + 6 * (size_t)s0, 6 * (size_t)S.n));
      WG_TRY(upload(&S.volt, vl.data() + 6 * (size_t)s0, 6 * (size_t)S.n));
      WG_TRY(dalloc(&S.rhs, (size_t)S.n));
      if (c->have_fp32) WG_TRY(dalloc(&S.rhsf, (size_t)S.n));
      for (int i = s0; i < s1; ++i)
        for (int k = 0; k < 6; ++k) {
          double d = dl[6 * (size_t)i + k];
          if (0. >= d && d > -1.) L.has_neumann_sub = true;
        }
    }
  }
  return WG_OK;
}

}  // namespace wg

using namespace wg;

int ensure_fp32_impl(wg_ctx* c) {
  if (c->have_fp32) return WG_OK;
  free_graphs(c);
  c->cond_version += 1;
  for (Level& L : c->lv) {
    WG_TRY(dalloc(&L.phif, L.np));
    WG_TRY(dalloc(&L.rhsf, L.nr));
    WG_TRY(dalloc(&L.resf, L.np));
    for (DevSubgrid& S : L.sub)
      if (S.n && !S.rhsf) WG_TRY(dalloc(&S.rhsf, (size_t)S.n));
  }
  c->have_fp32 = true;
  return WG_OK;
}
namespace wg {
int ensure_fp32(wg_ctx* c) { return ensure_fp32_impl(c); }
}  // namespace wg

extern "C" {

const char* wg_last_error(void) { return g_last_error.c_str(); }

int wg_create(const wg_grid* grid, wg_ctx** out) {
  if (!grid || !out) { set_error("wg_create: null argument"); return WG_EINVAL; }
  *out = nullptr;
  const wg_grid& G = *grid;
  if (G.nx < 2 || G.ny < 2 || G.nz < 2 || !(G.xmmax > G.xmmin) || !(G.ymmax > G.ymmin) || !(G.zmmax > G.zmmin)) {
    set_error("wg_create: need nx, ny, nz >= 2 and increasing mesh extents (2D XZ/RZ meshes are not supported)");
    return WG_EINVAL;
  }
  for (int k = 0; k < 6; ++k)
    if (G.bounds[k] < 0 || G.bounds[k] > 2) { set_error("wg_create: bounds must be 0, 1 or 2"); return WG_EINVAL; }
  for (int a = 0; a < 3; ++a)
    if ((G.bounds[2 * a] == 2) != (G.bounds[2 * a + 1] == 2)) {
      set_error("wg_create: periodic bounds must be set on both sides of an axis");
      return WG_EINVAL;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("wg_create: no CUDA device");
    return WG_ENODEV;
  }
  wg_ctx* c = new (std::nothrow) wg_ctx();
  if (!c) { set_error("wg_create: out of host memory"); return WG_ENOMEM; }
  cudaGetDevice(&c->device);
  c->grid = G;
  c->dx = (G.xmmax - G.xmmin) / G.nx;
  c->dy = (G.ymmax - G.ymmin) / G.ny;
  c->dz = (G.zmmax - G.zmmin) / G.nz;
  if ((double)(G.nx + 3) * (G.ny + 3) * (G.nz + 3) >= 2147483647.) {
    set_error("wg_create: the padded grid (nx+3)(ny+3)(nz+3) must hold fewer than 2^31 nodes");
    delete c;
    return WG_ETOOLARGE;
  }
  std::vector<LevelDims> dims = mglevels(G.nx, G.ny, G.nz, c->dx, c->dy, c->dz);
  c->lv.resize(dims.size());
  int rc = WG_OK;
  for (size_t l = 0; l < dims.size() && rc == WG_OK; ++l) {
    Level& L = c->lv[l];
    L.d = dims[l];
    L.np = (size_t)(L.d.nx + 3) * (L.d.ny + 3) * (L.d.nz + 3);
    L.nr = (size_t)(L.d.nx + 1) * (L.d.ny + 1) * (L.d.nz + 1);
    rc = dalloc(&L.phi, L.np);
    if (rc == WG_OK) rc = dalloc(&L.rhs, L.nr);
    if (rc == WG_OK && l + 1 < dims.size()) rc = dalloc(&L.res, L.np);
    if (rc == WG_OK && l + 1 < dims.size()) rc = expand_tables(L, dims[l + 1]);
    if (rc == WG_OK && l + 1 < dims.size()) rc = restrict_tables(L, dims[l + 1]);
  }
  Level& L0 = c->lv[0];
  if (rc == WG_OK) rc = dalloc(&c->phisave, L0.np);
  if (rc == WG_OK) rc = dalloc(&c->rho, L0.nr);
  if (rc == WG_OK) rc = dalloc(&c->racc, L0.nr);
  if (rc == WG_OK) rc = dalloc(&c->dred, (size_t)5);
  if (rc == WG_OK) rc = dalloc(&c->dese, (size_t)(G.nx + 1) * (G.ny + 1) + 1);
  if (rc == WG_OK) rc = dalloc(&c->dslot, (size_t)3 * 32 * 16);
  if (rc == WG_OK) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, c->device);
    c->mom_blocks = prop.multiProcessorCount * 4;
    rc = dalloc(&c->dmom, (size_t)moments_scratch_doubles(c->mom_blocks));
  }
  // The reduction words reach the host through mapped pinned memory written
  // by a kernel, not through a copy: a small device-to-host copy would queue
  // behind the bulk copies of a caller's other streams on the copy engines.
  if (rc == WG_OK && cudaHostAlloc((void**)&c->hred, 5 * sizeof(unsigned long long), cudaHostAllocMapped) != cudaSuccess) {
    set_error("wg_create: cudaHostAlloc failed");
    rc = WG_ENOMEM;
  }
  if (rc == WG_OK && cudaHostGetDevicePointer((void**)&c->hred_dev, c->hred, 0) != cudaSuccess) {
    set_error("wg_create: cudaHostGetDevicePointer failed");
    rc = WG_ECUDA;
  }
  if (rc == WG_OK) rc = configure_kernels();
  if (rc == WG_OK) {
    // empty conductor set so the solver can run without installconductor
    rc = finalize_conductors(c->cond, dims);
    if (rc == WG_OK) rc = upload_conductors(c);
  }
  if (rc != WG_OK) {
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return WG_OK;
}

int wg_destroy(wg_ctx* c) {
  if (!c) return WG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
  return WG_OK;
}

int wg_set_stream(wg_ctx* c, void* stream) {
  if (!c) { set_error("wg_set_stream: null context"); return WG_EINVAL; }
  c->stream = (cudaStream_t)stream;
  return WG_OK;
}

int wg_level_info(wg_ctx* c, int* nlevels, int* dims, double* deltas, int maxlevels) {
  if (!c || !nlevels) { set_error("wg_level_info: null argument"); return WG_EINVAL; }
  *nlevels = (int)c->lv.size();
  for (int l = 0; l < (int)c->lv.size() && l < maxlevels; ++l) {
    if (dims) { dims[3 * l] = c->lv[l].d.nx; dims[3 * l + 1] = c->lv[l].d.ny; dims[3 * l + 2] = c->lv[l].d.nz; }
    if (deltas) { deltas[3 * l] = c->lv[l].d.dx; deltas[3 * l + 1] = c->lv[l].d.dy; deltas[3 * l + 2] = c->lv[l].d.dz; }
  }
  return WG_OK;
}

int wg_arrays(wg_ctx* c, double** phi, double** rho) {
  if (!c) { set_error("wg_arrays: null context"); return WG_EINVAL; }
  if (phi) *phi = c->lv[0].phi;
  if (rho) *rho = c->rho;
  return WG_OK;
}

static std::vector<LevelDims> dims_of(wg_ctx* c) {
  std::vector<LevelDims> d;
  for (auto& L : c->lv) d.push_back(L.d);
  return d;
}

int wg_conductors_add_shape(wg_ctx* c, int kind, double radius, double length, double voltage, double xcent,
                            double ycent, double zcent, int condid, double dfill) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  if (!(dfill > 0.)) dfill = 2.0;
  return add_shape(c->cond, dims_of(c), c->grid.xmmin, c->grid.ymmin, c->grid.zmmin, kind, radius, length, voltage,
                   xcent, ycent, zcent, condid, dfill);
}

int wg_conductors_add_points(wg_ctx* c, int kind, int64_t n, const int32_t* indx, const double* dels,
                             const double* volt, const int32_t* ilevel) {
  if (!c || n < 0 || (n > 0 && (!indx || !volt || !ilevel || (kind == 1 && !dels))) || (kind != 0 && kind != 1)) {
    set_error("wg_conductors_add_points: bad arguments");
    return WG_EINVAL;
  }
  HostConductors& C = c->cond;
  if (kind == 0) {
    C.int_indx.insert(C.int_indx.end(), indx, indx + 3 * n);
    C.int_volt.insert(C.int_volt.end(), volt, volt + n);
    C.int_level.insert(C.int_level.end(), ilevel, ilevel + n);
  } else {
    C.sub_indx.insert(C.sub_indx.end(), indx, indx + 3 * n);
    C.sub_dels.insert(C.sub_dels.end(), dels, dels + 6 * n);
    C.sub_volt.insert(C.sub_volt.end(), volt, volt + 6 * n);
    C.sub_level.insert(C.sub_level.end(), ilevel, ilevel + n);
  }
  C.finalized = false;
  return WG_OK;
}

int wg_conductors_finalize(wg_ctx* c) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  WG_TRY(finalize_conductors(c->cond, dims_of(c)));
  return upload_conductors(c);
}

int wg_conductors_clear(wg_ctx* c) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  c->cond = HostConductors();
  return wg_conductors_finalize(c);
}

int wg_conductors_counts(wg_ctx* c, int64_t* out) {
  if (!c || !out) { set_error("null argument"); return WG_EINVAL; }
  if (!c->cond.finalized) { set_error("wg_conductors_counts: call wg_conductors_finalize first"); return WG_ESTATE; }
  out[0] = (int64_t)c->cond.int_volt.size();
  out[1] = (int64_t)c->cond.even_level.size();
  out[2] = (int64_t)c->cond.odd_level.size();
  return WG_OK;
}

int wg_conductors_export(wg_ctx* c, int which, int32_t* indx, double* dels, double* volt, int32_t* ilevel) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  const HostConductors& C = c->cond;
  if (!C.finalized) { set_error("wg_conductors_export: not finalized"); return WG_ESTATE; }
  if (which == 0) {
    if (indx) memcpy(indx, C.int_indx.data(), C.int_indx.size() * sizeof(int32_t));
    if (volt) memcpy(volt, C.int_volt.data(), C.int_volt.size() * sizeof(double));
    if (ilevel) memcpy(ilevel, C.int_level.data(), C.int_level.size() * sizeof(int32_t));
  } else if (which == 1 || which == 2) {
    const auto& I = which == 1 ? C.even_indx : C.odd_indx;
    const auto& D = which == 1 ? C.even_dels : C.odd_dels;
    const auto& V = which == 1 ? C.even_volt : C.odd_volt;
    const auto& L = which == 1 ? C.even_level : C.odd_level;
    if (indx) memcpy(indx, I.data(), I.size() * sizeof(int32_t));
    if (dels) memcpy(dels, D.data(), D.size() * sizeof(double));
    if (volt) memcpy(volt, V.data(), V.size() * sizeof(double));
    if (ilevel) memcpy(ilevel, L.data(), L.size() * sizeof(int32_t));
  } else {
    set_error("wg_conductors_export: which must be 0, 1 or 2");
    return WG_EINVAL;
  }
  return WG_OK;
}

int wg_solve(wg_ctx* c, const wg_solve_opts* opts, wg_solve_stats* stats) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  if (!c->cond.finalized) { set_error("wg_solve: conductors added but not finalized"); return WG_ESTATE; }
  return solve(c, opts, stats);
}

int wg_field_energy(wg_ctx* c, double* out) {
  if (!c || !out) { set_error("null argument"); return WG_EINVAL; }
  return field_energy(c, out);
}

int wg_residual_field(wg_ctx* c, double mgparam, double* out) {
  if (!c || !out) { set_error("null argument"); return WG_EINVAL; }
  return residual_field(c, mgparam, out);
}

int wg_relresidual(wg_ctx* c, double mgparam, double* out) {
  if (!c || !out) { set_error("null argument"); return WG_EINVAL; }
  return relresidual(c, mgparam, out);
}

int wg_deposit(wg_ctx* c, const wg_particles* p, int zero_first) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  if (c->dep_open) { set_error("wg_deposit: a chunked deposit is open (wg_deposit_end first)"); return WG_ESTATE; }
  return deposit(c, p, zero_first);
}

int wg_deposit_begin(wg_ctx* c) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return deposit_begin(c);
}

int wg_deposit_add(wg_ctx* c, const wg_particles* p) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return deposit_add(c, p);
}

int wg_deposit_end(wg_ctx* c, int zero_first) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return deposit_end(c, zero_first);
}

int wg_deposit_noalloc(const wg_grid* grid, const wg_particles* p, double* rho, int zero_first, void* stream) {
  return deposit_noalloc(grid, p, rho, zero_first, stream);
}

int wg_finalize_rho(wg_ctx* c) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return finalize_rho(c);
}

int wg_fetch_e(wg_ctx* c, const double* x, const double* y, const double* z, double* ex, double* ey, double* ez,
               int64_t np) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return fetch_e(c, x, y, z, ex, ey, ez, np);
}

int wg_set_lattice(wg_ctx* c, const double* czs, const double* cze, const double* cdb, int nzl, double zlmin,
                   double dzl) {
  if (!c || nzl < 0 || !czs || !cze || !cdb || !(dzl > 0.)) {
    set_error("wg_set_lattice: bad arguments");
    return WG_EINVAL;
  }
  dfree(c->czs);
  dfree(c->cze);
  dfree(c->cdb);
  WG_TRY(upload(&c->czs, czs, (size_t)nzl + 1));
  WG_TRY(upload(&c->cze, cze, (size_t)nzl + 1));
  WG_TRY(upload(&c->cdb, cdb, (size_t)nzl + 1));
  c->nzl = nzl;
  c->zlmin = zlmin;
  c->dzl = dzl;
  return WG_OK;
}

int wg_set_correctede(wg_ctx* c, int on) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  c->correctede = on ? 1 : 0;
  return WG_OK;
}

int wg_advance(wg_ctx* c, const wg_particles* p, const wg_push_params* prm) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return advance(c, p, prm);
}

int wg_zmoments(wg_ctx* c, const wg_particles* p, const double* uxo, const double* uyo, const double* uzo, double dt,
                double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt, double zmmntdtextmax,
                double* zmmnts0, double* zmmnts) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return zmoments(c, p, uxo, uyo, uzo, dt, dtscale, zbeam, zmmntmin, zmmntmax, nzmmnt, zmmntdtextmax, zmmnts0, zmmnts);
}

int wg_moments(wg_ctx* c, const wg_particles* p, double* out) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return moments(c, p, out);
}

int wg_deposit_f32(wg_ctx* c, const wg_particles_f32* p, int zero_first) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  if (c->dep_open) { set_error("wg_deposit_f32: a chunked deposit is open (wg_deposit_end first)"); return WG_ESTATE; }
  return deposit_f32(c, p, zero_first);
}

int wg_deposit_add_f32(wg_ctx* c, const wg_particles_f32* p) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return deposit_add_f32(c, p);
}

int wg_advance_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return advance_f32(c, p, prm);
}

int wg_advance_deposit(wg_ctx* c, const wg_particles* p, const wg_push_params* prm) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return advance_deposit(c, p, prm);
}

int wg_advance_deposit_f32(wg_ctx* c, const wg_particles_f32* p, const wg_push_params* prm) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return advance_deposit_f32(c, p, prm);
}

int wg_moments_f32(wg_ctx* c, const wg_particles_f32* p, double* out) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return moments_f32(c, p, out);
}

int wg_zmoments_f32(wg_ctx* c, const wg_particles_f32* p, const float* uxo, const float* uyo, const float* uzo,
                    double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt,
                    double zmmntdtextmax, double* zmmnts0, double* zmmnts) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return zmoments_f32(c, p, uxo, uyo, uzo, dt, dtscale, zbeam, zmmntmin, zmmntmax, nzmmnt, zmmntdtextmax, zmmnts0,
                      zmmnts);
}

}  // extern "C"

extern "C" {

int wg_prof_enable(wg_ctx* c, int mask) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (mask && c->prof_ev.empty()) {
    const size_t npairs = 1 << 14;
    c->prof_ev.resize(2 * npairs);
    for (auto& e : c->prof_ev) WG_TRY_CUDA(cudaEventCreate(&e));
    c->prof_kind.assign(npairs, -1);
    c->prof_units.assign(npairs, 0.);
  }
  c->prof_mask = mask;
  c->prof_used = 0;
  return WG_OK;
}

int wg_prof_read(wg_ctx* c, int kind, double* total_ms, int64_t* launches, double* units) {
  if (!c || !total_ms || !launches) { set_error("null argument"); return WG_EINVAL; }
  WG_TRY_CUDA(cudaStreamSynchronize(c->stream));
  double ms = 0., u = 0.;
  int64_t n = 0;
  for (size_t i = 0; i < c->prof_used; ++i) {
    if (c->prof_kind[i] != kind) continue;
    float t = 0.f;
    WG_TRY_CUDA(cudaEventElapsedTime(&t, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]));
    ms += t;
    u += c->prof_units[i];
    ++n;
  }
  *total_ms = ms;
  *launches = n;
  if (units) *units = u;
  return WG_OK;
}

int wg_launch_count(wg_ctx* c, int64_t* n) {
  if (!c || !n) { set_error("null argument"); return WG_EINVAL; }
  *n = c->nlaunch;
  return WG_OK;
}

}  // extern "C"

namespace wg {
int cell_keys(wg_ctx* c, const wg_particles* p, int64_t* keys);
int permute(wg_ctx* c, const int64_t* perm, const wg_particles* src, const wg_particles* dst);
}  // namespace wg

extern "C" {

int wg_particle_keys(wg_ctx* c, const wg_particles* p, int64_t* keys) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return cell_keys(c, p, keys);
}

int wg_particle_permute(wg_ctx* c, const int64_t* perm, const wg_particles* src, const wg_particles* dst) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return permute(c, perm, src, dst);
}

int wg_particle_keys_f32(wg_ctx* c, const wg_particles_f32* p, int64_t* keys) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return cell_keys_f32(c, p, keys);
}

int wg_particle_permute_f32(wg_ctx* c, const int64_t* perm, const wg_particles_f32* src,
                            const wg_particles_f32* dst) {
  if (!c) { set_error("null context"); return WG_EINVAL; }
  return permute_f32(c, perm, src, dst);
}

}  // extern "C"
