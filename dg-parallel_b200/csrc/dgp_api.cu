// C ABI of libdgp.so (include/dgp.h): handles, host preprocessing, device
// buffers in the internal (Morton) cell order, and the device-resident time
// loop captured in CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_host.h"
#include "dgp_handles.h"
#include "dgp_adjoint.cuh"
#include "dgp_limiter.cuh"
#include "dgp_solver.h"

namespace dgp {

std::map<OpsKey, Ops>& ops_registry() {
  static std::map<OpsKey, Ops> r;
  return r;
}

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

namespace {
void ensure_registry() {
  static std::once_flag once;
  std::call_once(once, [] {
    register_scalar_ops();
    register_burgers_ops();
    register_euler2d_godunov_ops();
    register_euler2d_roe_ops();
    register_euler2d_llf_ops();
    register_euler3d_ops();
    register_maxwell3d_ops();
    register_maxwell2d_ops();
    register_burgers_tile_ops();
    register_euler2d_roe_tile_ops();
  });
}

// Autotuner results: the tile shape (threads of the element and face kernels)
// that measured fastest for a (law, flux, element, order, precision) at a
// problem size (bucket: floor(log2(cells))).  Consulted when solvers and
// ensemble groups are created; filled by dgp_autotune / dgp_autotune_ensemble.
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int, int>, int> g_tune;

int size_bucket(long long cells) {
  int b = 0;
  while ((1LL << (b + 1)) <= cells) ++b;
  return b;
}

int tuned_block(int law, int flux, int dim, int order, int precision, long long cells) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tune.find(std::make_tuple(law, flux, dim, order, precision, size_bucket(cells)));
  return it == g_tune.end() ? kDefaultBlock : it->second;
}

void set_tuned_block(int law, int flux, int dim, int order, int precision, long long cells, int block) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune[std::make_tuple(law, flux, dim, order, precision, size_bucket(cells))] = block;
}

// Fused stage kernel or separate face and element kernels, per (law, flux,
// element, order, precision, size bucket): the autotuner's measurement where
// there is one, else the default below.  The default follows measurements on
// B200 (128-thread tiles, 131k-180k triangles, 196k-663k tets; step time of
// the separate kernels over the fused one): the fused kernel wins for the 2D
// Euler (Roe, LLF), scalar and Maxwell laws at P2-P3 (1.10-1.45x), Euler P1
// (1.08x) and P1 on tets (scalar P2: 1.11x, 1.21-1.38x); the separate kernels
// win for Burgers (up to 1.56x), the exact Godunov flux, P4 on triangles (up to
// 2x), the 3D Euler law and tets of higher order (1.07-1.43x), where the fused
// tile's halo (rows read and faces evaluated by two tiles) and its larger
// shared memory cost more than the face data the separate kernels pass
// through device memory.
std::map<std::tuple<int, int, int, int, int, int>, int> g_tune_fused;

bool fused_default(int law, int flux, int dim, int order) {
  if (law == DGP_LAW_BURGERS2D || law == DGP_LAW_EULER3D || flux == DGP_FLUX_GODUNOV) return false;
  if (dim == 2) return order == 2 || order == 3 || (order == 1 && law == DGP_LAW_EULER2D);
  return order == 1 || (law == DGP_LAW_SCALAR && order == 2);
}

bool tuned_fused(int law, int flux, int dim, int order, int precision, long long cells) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tune_fused.find(std::make_tuple(law, flux, dim, order, precision, size_bucket(cells)));
  return it == g_tune_fused.end() ? fused_default(law, flux, dim, order) : it->second != 0;
}

void set_tuned_fused(int law, int flux, int dim, int order, int precision, long long cells, bool fused) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_fused[std::make_tuple(law, flux, dim, order, precision, size_bucket(cells))] = fused ? 1 : 0;
}

bool has_block(int law, int flux, int dim, int order, int precision, int block) {
  ensure_registry();
  return ops_registry().count(OpsKey(law, flux, dim, order, precision, block, DGP_RULE_REFERENCE)) != 0;
}

// gather cells by `perm` and convert the arithmetic type
template <typename Tin, typename Tout>
__global__ void gather_cells(const Tin* in, Tout* out, const int* perm, int E, int mnp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)E * mnp) return;
  const int e = static_cast<int>(i / mnp), r = static_cast<int>(i - (long long)e * mnp);
  out[i] = static_cast<Tout>(in[(size_t)perm[e] * mnp + r]);
}

// device clock mark of a run's start (ensembles time their instances from it)
__global__ void mark_clock(TimeCtl* c) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  c->t_mark_ns = t;
}

// controls of one adjoint segment: time and step of the forward recompute,
// a step's start time for the fixed-step forward, its recomputation and the
// reversed stages: t0 + k dt from the host for step k, so all three see the
// same boundary times bit for bit (values travel as kernel parameters, so
// steps queued without a host sync do not race)
__global__ void set_segment_time(TimeCtl* c, double t, double dt, double* t_seg) {
  c->t = t;
  c->dt = dt;
  c->tend = 0.0;
  c->max_steps = 0;
  c->done = 0;
  c->blocks_done = 0;
  *t_seg = t;
}

uint64_t spread2(uint32_t x) {
  uint64_t v = x;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
  v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}

uint64_t spread3(uint32_t x) {
  uint64_t v = x & 0x1FFFFF;
  v = (v | (v << 32)) & 0x1F00000000FFFFull;
  v = (v | (v << 16)) & 0x1F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}
}  // namespace
}  // namespace dgp

using namespace dgp;


// Triangle moment limiter data in the internal cell order: neighbours by
// bounding boxes (DGLimiter.cc:970-993, DGCell.cc:76-86), FP64 geometry of the
// derivative transforms and the bounding-box centres, degree tables.  Padding
// cells of an ensemble keep no neighbours and zero geometry.
static int setup_limiter(dgp_solver s) {
  const int Etot = s->b.E;
  std::vector<int> nb(4 * (size_t)Etot, -1);
  std::vector<double> geo(static_cast<size_t>(Etot) * kLimGeo, 0.0);
  for (size_t ii = 0; ii < s->meshes.size(); ++ii) {
    const HostMesh& m = s->meshes[ii];
    const int E = m.E, uf = s->inst_ufirst[ii], off = s->inst_off[ii];
    std::vector<double> bmin(2 * (size_t)E), bmax(2 * (size_t)E), bbc(2 * (size_t)E);
    for (int e = 0; e < E; ++e) {
      const int* c = &m.cv[static_cast<size_t>(e) * m.nvc];
      for (int k = 0; k < 2; ++k) bmin[2 * e + k] = bmax[2 * e + k] = m.X[3 * c[0] + k];
      for (int v = 1; v < m.nvc; ++v)
        for (int k = 0; k < 2; ++k) {
          const double x = m.X[3 * c[v] + k];
          if (x < bmin[2 * e + k]) bmin[2 * e + k] = x;
          if (x > bmax[2 * e + k]) bmax[2 * e + k] = x;
        }
      for (int k = 0; k < 2; ++k) bbc[2 * e + k] = (bmin[2 * e + k] + bmax[2 * e + k]) / 2.;
    }
    std::vector<int> cf(3 * (size_t)E, -1);  // face of (cell, local face)
    for (int f = 0; f < m.F; ++f) {
      cf[3 * (size_t)m.eL[f] + m.lfL[f]] = f;
      if (m.eR[f] >= 0) cf[3 * (size_t)m.eR[f] + m.lfR[f]] = f;
    }
    for (int e = 0; e < E; ++e) {
      const int i = s->f2i[uf + e];
      (void)off;
      const double px = bbc[2 * e], py = bbc[2 * e + 1];
      int* n = &nb[4 * (size_t)i];
      for (int lf = 0; lf < 3; ++lf) {
        const int f = cf[3 * (size_t)e + lf];
        if (f < 0 || m.eR[f] < 0) continue;
        const int o = (m.eL[f] == e) ? m.eR[f] : m.eL[f];
        const int oi = s->f2i[uf + o];
        if (px > bmax[2 * o]) n[0] = oi;
        if (px < bmin[2 * o]) n[1] = oi;
        if (py > bmax[2 * o + 1]) n[2] = oi;
        if (py < bmin[2 * o + 1]) n[3] = oi;
      }
      double X0[3], J[9], Ji[9];
      cell_frame(m, e, X0, J);
      invert3(J, Ji);
      double* g = &geo[static_cast<size_t>(i) * kLimGeo];
      g[0] = Ji[0];
      g[1] = Ji[1];
      g[2] = Ji[3];
      g[3] = Ji[4];
      g[4] = J[0];
      g[5] = J[1];
      g[6] = J[3];
      g[7] = J[4];
      g[8] = px;
      g[9] = py;
    }
  }
  std::vector<double> D, Dinv;
  build_limiter_tables(s->tab, D, Dinv);
  DeviceBuffers& b = s->b;
  int rc = DGP_OK;
  if ((rc = s->upload(&b.nb, nb)) || (rc = s->upload(&b.lgeo, geo)) || (rc = s->upload(&b.limD, D)) ||
      (rc = s->upload(&b.limDinv, Dinv)) || (rc = s->alloc(&b.trig, static_cast<size_t>(Etot) * b.M)) ||
      (rc = s->alloc(&b.lbig, static_cast<size_t>(Etot) * b.M)) || (rc = s->alloc(&b.lmo, s->state_count())))
    return rc;
  DGP_CUDA(cudaMemset(b.trig, 0, static_cast<size_t>(Etot) * b.M));
  return DGP_OK;
}

// Morton code of the cell centroids of one mesh (locality of neighbours)
static std::vector<int> morton_order(const HostMesh& m) {
  const int E = m.E, dim = m.dim, nvc = m.nvc;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  std::vector<double> cen(static_cast<size_t>(E) * 3);
  for (int e = 0; e < E; ++e)
    for (int c = 0; c < 3; ++c) {
      double x = 0;
      for (int k = 0; k < nvc; ++k) x += m.X[3 * m.cv[static_cast<size_t>(e) * nvc + k] + c];
      x /= nvc;
      cen[3 * e + c] = x;
      lo[c] = std::min(lo[c], x);
      hi[c] = std::max(hi[c], x);
    }
  std::vector<uint64_t> key(E);
  for (int e = 0; e < E; ++e) {
    uint32_t qv[3];
    for (int c = 0; c < 3; ++c) {
      double span = hi[c] - lo[c];
      double u = span > 0 ? (cen[3 * e + c] - lo[c]) / span : 0.0;
      double scale = dim == 2 ? 4294967295.0 : 2097151.0;
      qv[c] = static_cast<uint32_t>(std::min(scale, std::max(0.0, u * scale)));
    }
    key[e] = dim == 2 ? (spread2(qv[0]) | (spread2(qv[1]) << 1))
                      : (spread3(qv[0]) | (spread3(qv[1]) << 1) | (spread3(qv[2]) << 2));
  }
  std::vector<int> order(E);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return key[a] < key[c]; });
  return order;
}

// Face records and halos of the fused stage kernel's tiles (TileMesh): for
// tile t, every face with a side among its cells, in face order, with both
// sides as local rows (own cells first, then the halo in order of first use)
// and the face's FP64 normal and measure.  The fused kernel is built for the
// solver (fused_ok) when every tile's halo fits in shared memory; whether the
// stages then use it or the face and element kernels is tuned_fused's choice
// (dgp_set_fused switches).
static int build_tiles(dgp_solver s, int Etot, const std::vector<int>& fel, const std::vector<int>& fcode,
                       const std::vector<double>& fnrm, const std::vector<double>& fj, const std::vector<int>& bpart,
                       const std::vector<int>& cface) {
  const int TE = s->ops.TE, nlf = s->tab.nlf, dim = s->b.dim;
  const int ntiles = (Etot + TE - 1) / TE;
  std::vector<int> tf_off(1, 0), tf_side, tf_code, tf_bnd, th_off(1, 0), th_cell;
  std::vector<double> tf_nrm, tf_fj;
  std::vector<int> flist, halo;
  int nh_max = 0;
  for (int t = 0; t < ntiles; ++t) {
    const int e0 = t * TE, e1 = std::min(e0 + TE, Etot);
    flist.clear();
    halo.clear();
    for (int e = e0; e < e1; ++e)
      for (int lf = 0; lf < nlf; ++lf) {
        const int k = cface[static_cast<size_t>(e) * nlf + lf];
        if (k >= 0) flist.push_back(k);
      }
    std::sort(flist.begin(), flist.end());
    flist.erase(std::unique(flist.begin(), flist.end()), flist.end());
    auto local = [&](int e) {
      if (e >= e0 && e < e1) return e - e0;
      for (size_t h = 0; h < halo.size(); ++h)
        if (halo[h] == e) return TE + static_cast<int>(h);
      halo.push_back(e);
      return TE + static_cast<int>(halo.size()) - 1;
    };
    for (int k : flist) {
      const int eL = fel[2 * static_cast<size_t>(k)], eR = fel[2 * static_cast<size_t>(k) + 1];
      const int lL = local(eL);
      const int ownL = (eL >= e0 && eL < e1) ? 1 : 0;
      int side = lL, ownR = 0, kind = 0, bnd = -1;
      if (eR >= 0) {
        side |= (local(eR) + 1) << 16;
        ownR = (eR >= e0 && eR < e1) ? 1 : 0;
      } else {
        bnd = -eR - 1;
        if (bpart[bnd] >= 0) {
          kind = 2;
          side |= (local(bpart[bnd]) + 1) << 16;
        } else {
          kind = 1;
        }
      }
      tf_side.push_back(side);
      tf_code.push_back((fcode[k] & 0xfff) | (ownL << 12) | (ownR << 13) | (kind << 14));
      tf_bnd.push_back(bnd);
      for (int c = 0; c < dim; ++c) tf_nrm.push_back(fnrm[static_cast<size_t>(k) * dim + c]);
      tf_fj.push_back(fj[k]);
    }
    tf_off.push_back(static_cast<int>(tf_side.size()));
    th_cell.insert(th_cell.end(), halo.begin(), halo.end());
    th_off.push_back(static_cast<int>(th_cell.size()));
    nh_max = std::max(nh_max, static_cast<int>(halo.size()));
  }
  s->fused_ok = s->ops.fused != nullptr && nh_max <= TE * nlf && s->ops.fused_smem(nh_max) + 8 * 1024 <= 227 * 1024;
  long long cells = 0;
  for (const auto& hm : s->meshes) cells += hm.E;
  s->fused = s->fused_ok && tuned_fused(s->law, s->flux, dim, s->order, s->precision, cells);
  if (!s->fused_ok) return DGP_OK;
  TileMesh& tm = s->b.tm;
  int rc = DGP_OK;
  int *d_tf_off, *d_tf_side, *d_tf_code, *d_tf_bnd, *d_th_off, *d_th_cell;
  double *d_tf_nrm, *d_tf_fj;
  if (th_cell.empty()) th_cell.push_back(0);
  if (tf_side.empty()) {
    tf_side.push_back(0);
    tf_code.push_back(0);
    tf_bnd.push_back(-1);
    tf_fj.push_back(0.0);
    tf_nrm.resize(dim, 0.0);
  }
  if ((rc = s->upload(&d_tf_off, tf_off)) || (rc = s->upload(&d_tf_side, tf_side)) ||
      (rc = s->upload(&d_tf_code, tf_code)) || (rc = s->upload(&d_tf_bnd, tf_bnd)) ||
      (rc = s->upload(&d_tf_nrm, tf_nrm)) || (rc = s->upload(&d_tf_fj, tf_fj)) ||
      (rc = s->upload(&d_th_off, th_off)) || (rc = s->upload(&d_th_cell, th_cell)))
    return rc;
  tm.tf_off = d_tf_off;
  tm.tf_side = d_tf_side;
  tm.tf_code = d_tf_code;
  tm.tf_bnd = d_tf_bnd;
  tm.tf_nrm = d_tf_nrm;
  tm.tf_fj = d_tf_fj;
  tm.th_off = d_th_off;
  tm.th_cell = d_th_cell;
  tm.nh_max = nh_max;
  return DGP_OK;
}

// Builds the device state of a solver over the instances already in s->meshes
// (one mesh for a single solver).  Instance i owns internal cells
// [inst_off[i], inst_off[i] + E_i), each instance starting on an
// element-kernel tile; ensemble=false keeps the single-solver layout (no
// per-instance arrays, kernels see cell_inst == nullptr).
static int build_solver(dgp_solver s, const std::vector<LawParams>& lps, int field, bool ensemble) {
  const int n = static_cast<int>(s->meshes.size());
  const int dim = s->meshes[0].dim;
  const int TE = s->ops.TE;
  const RefTables& t = s->tab;
  s->inst_off.resize(n);
  s->inst_ufirst.resize(n);
  int Etot = 0, uf = 0, Ftot = 0;
  for (int i = 0; i < n; ++i) {
    s->inst_off[i] = Etot;
    s->inst_ufirst[i] = uf;
    const int Ei = s->meshes[i].E;
    uf += Ei;
    Etot += ensemble ? (Ei + TE - 1) / TE * TE : Ei;
    Ftot += s->meshes[i].F;
  }
  DeviceBuffers& b = s->b;
  b.E = Etot;
  b.dim = dim;
  b.order = s->order;
  b.M = s->ops.M;
  b.NP = s->ops.NP;
  s->i2f.assign(Etot, -1);
  s->f2i.assign(uf, -1);
  std::vector<int> cell_inst(Etot, -1);
  for (int i = 0; i < n; ++i) {
    const std::vector<int> ord = morton_order(s->meshes[i]);
    for (int r = 0; r < static_cast<int>(ord.size()); ++r) {
      const int internal = s->inst_off[i] + r, ufile = s->inst_ufirst[i] + ord[r];
      s->i2f[internal] = ufile;
      s->f2i[ufile] = internal;
      cell_inst[internal] = i;
    }
  }

  // cell geometry (FP64 on the host); padding cells stay zero
  std::vector<double> jinv(static_cast<size_t>(Etot) * dim * dim, 0.0), detj(Etot, 0.0), csize(Etot, 0.0),
      x0(3 * (size_t)Etot, 0.0), jac(9 * (size_t)Etot, 0.0);
  for (int i = 0; i < Etot; ++i) {
    if (s->i2f[i] < 0) continue;
    const int inst = cell_inst[i];
    const HostMesh& m = s->meshes[inst];
    const int e = s->i2f[i] - s->inst_ufirst[inst];
    const int nvc = m.nvc;
    double X0[3], J[9], Ji[9];
    cell_frame(m, e, X0, J);
    double d = invert3(J, Ji);
    detj[i] = std::fabs(d);
    for (int r = 0; r < dim; ++r)
      for (int c = 0; c < dim; ++c) jinv[static_cast<size_t>(i) * dim * dim + r * dim + c] = Ji[r * 3 + c];
    for (int k = 0; k < 3; ++k) x0[3 * i + k] = X0[k];
    for (int k = 0; k < 9; ++k) jac[9 * i + k] = J[k];
    const int* c = &m.cv[static_cast<size_t>(e) * nvc];
    auto len = [&](int a, int bb) {
      const double *p = &m.X[3 * c[a]], *q = &m.X[3 * c[bb]];
      return std::sqrt((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) +
                       (q[2] - p[2]) * (q[2] - p[2]));
    };
    if (dim == 2) {  // DGCell::computeCellSize (DGCell.cc:1211-1229)
      double a = len(0, 1), bb = len(1, 2), cc = len(2, 0);
      double hp = 0.5 * (a + bb + cc);
      csize[i] = std::sqrt(hp * (hp - a) * (hp - bb) * (hp - cc)) / hp * 2.;
    } else {  // minimum edge (DGCell.cc:1239-1256)
      double L[6] = {len(0, 1), len(1, 2), len(2, 0), len(0, 3), len(1, 3), len(2, 3)};
      double mn = L[0];
      for (int k = 1; k < 6; ++k) mn = std::min(mn, L[k]);
      csize[i] = mn;
    }
  }
  // faces of all instances, sorted by internal left cell
  struct FRef {
    int inst, f;
  };
  std::vector<FRef> faces;
  faces.reserve(Ftot);
  for (int i = 0; i < n; ++i)
    for (int f = 0; f < s->meshes[i].F; ++f) faces.push_back({i, f});
  auto left_internal = [&](const FRef& r) {
    return s->f2i[s->inst_ufirst[r.inst] + s->meshes[r.inst].eL[r.f]];
  };
  std::stable_sort(faces.begin(), faces.end(), [&](const FRef& a, const FRef& c) {
    const int ia = left_internal(a), ic = left_internal(c);
    return ia != ic ? ia < ic : s->meshes[a.inst].lfL[a.f] < s->meshes[c.inst].lfL[c.f];
  });
  std::vector<int> fel(2 * (size_t)Ftot), fcode(Ftot), bbid, bpart;
  std::vector<int> cface(static_cast<size_t>(Etot) * t.nlf, -1);  // local face -> face, per cell
  std::vector<double> fnrm(static_cast<size_t>(Ftot) * dim), fj(Ftot), bpts, bpphi;
  int nb = 0;
  for (int k = 0; k < Ftot; ++k) {
    const HostMesh& m = s->meshes[faces[k].inst];
    const int f = faces[k].f, ufo = s->inst_ufirst[faces[k].inst];
    fel[2 * k] = s->f2i[ufo + m.eL[f]];
    cface[static_cast<size_t>(fel[2 * k]) * t.nlf + m.lfL[f]] = k;
    if (m.eR[f] >= 0) {
      fel[2 * k + 1] = s->f2i[ufo + m.eR[f]];
      cface[static_cast<size_t>(fel[2 * k + 1]) * t.nlf + m.lfR[f]] = k;
    } else {
      fel[2 * k + 1] = -(nb + 1);
      bbid.push_back(m.bid[f]);
      const int* fv = &m.fv[static_cast<size_t>(f) * m.nfv];
      for (int q = 0; q < t.nqf; ++q) {
        const double *pa = &m.X[3 * fv[0]], *pb = &m.X[3 * fv[1]];
        double x[3];
        if (dim == 2) {
          double sp = t.fqp[2 * q];
          for (int c = 0; c < 3; ++c) x[c] = pa[c] * (1 - sp) * 0.5 + pb[c] * (1 + sp) * 0.5;
        } else {
          const double* pc = &m.X[3 * fv[2]];
          double u = t.fqp[2 * q], v = t.fqp[2 * q + 1];
          for (int c = 0; c < 3; ++c) x[c] = pa[c] * (1 - u - v) + pb[c] * u + pc[c] * v;
        }
        bpts.insert(bpts.end(), x, x + 3);
      }
      // periodic partner: its left cell's basis at the mirrored points
      // (DGBoundaryCell::setPeriodicBC, DGCell.cc:557-577)
      const int pf = m.pface.empty() ? -1 : m.pface[f];
      bpart.push_back(pf >= 0 ? s->f2i[ufo + m.eL[pf]] : -1);
      std::vector<double> ph(static_cast<size_t>(t.nqf) * t.Np, 0.0);
      if (pf >= 0) {
        const int pe = m.eL[pf];
        double X0[3], J[9], Ji[9];
        cell_frame(m, pe, X0, J);
        invert3(J, Ji);
        for (int q = 0; q < t.nqf; ++q) {
          const double* x = &bpts[bpts.size() - 3 * static_cast<size_t>(t.nqf) + 3 * q];
          double xm[3] = {x[0], x[1], x[2]};
          if (m.bid[f] == 510) xm[0] = -x[0];
          else xm[1] = -x[1];
          double d[3] = {xm[0] - X0[0], xm[1] - X0[1], xm[2] - X0[2]}, xi[3] = {0, 0, 0};
          for (int r = 0; r < dim; ++r) xi[r] = Ji[0 * 3 + r] * d[0] + Ji[1 * 3 + r] * d[1] + Ji[2 * 3 + r] * d[2];
          basis_eval(t, xi, &ph[static_cast<size_t>(q) * t.Np]);
        }
      }
      bpphi.insert(bpphi.end(), ph.begin(), ph.end());
      ++nb;
    }
    fcode[k] = m.lfL[f] | ((m.eR[f] >= 0 ? m.lfR[f] : 0) << 4) | (m.rperm[f] << 8);
    for (int c = 0; c < dim; ++c) fnrm[static_cast<size_t>(k) * dim + c] = m.fn[3 * f + c];
    fj[k] = dim == 2 ? 0.5 * m.fmeas[f] : 2.0 * m.fmeas[f];  // |J_f| of the face map
  }
  b.F = Ftot;
  b.NB = nb;
  if (int rc = build_tiles(s, Etot, fel, fcode, fnrm, fj, bpart, cface)) return rc;
  // per-cell geometry padded to whole tiles (the element kernel copies a
  // tile's J^{-1} and |J| in one piece)
  {
    const size_t ecap = (static_cast<size_t>(Etot) + TE - 1) / TE * TE;
    jinv.resize(ecap * dim * dim, 0.0);
    detj.resize(ecap, 1.0);
  }

  // reference tables
  std::vector<double> qpd(static_cast<size_t>(t.nq) * 3);
  for (int q = 0; q < t.nq; ++q)
    for (int c = 0; c < 3; ++c) qpd[3 * q + c] = t.qp[3 * q + c];
  int rc = DGP_OK;
  if ((rc = s->upload_t(&b.jinv, jinv)) || (rc = s->upload_t(&b.detj, detj)) ||
      (rc = s->upload(&b.detjd, detj)) ||
      (rc = s->upload(&b.csize, csize)) || (rc = s->upload(&b.x0, x0)) || (rc = s->upload(&b.jac, jac)) ||
      (rc = s->upload(&b.fel, fel)) || (rc = s->upload(&b.fcode, fcode)) ||
      (rc = s->upload_t(&b.fnrm, fnrm)) || (rc = s->upload_t(&b.fj, fj)) ||
      (rc = s->upload(&b.bpts, bpts.empty() ? std::vector<double>(3, 0.0) : bpts)) ||
      (rc = s->upload(&b.bbid, bbid.empty() ? std::vector<int>(1, 0) : bbid)) ||
      (rc = s->upload(&b.bpart, bpart.empty() ? std::vector<int>(1, -1) : bpart)) ||
      (rc = s->upload_t(&b.bpphi, bpphi.empty() ? std::vector<double>(1, 0.0) : bpphi)) ||
      (rc = s->upload_t(&b.phi, t.phi)) || (rc = s->upload_t(&b.dphi, t.dphi)) ||
      (rc = s->upload_t(&b.qw, t.qw)) || (rc = s->upload_t(&b.phif, t.phif)) ||
      (rc = s->upload_t(&b.fqw, t.fqw)) || (rc = s->upload(&b.qmap, t.qmap)) ||
      (rc = s->upload(&b.phiv, t.phiv)) || (rc = s->upload(&b.phiq, t.phi)) ||
      (rc = s->upload(&b.qwd, t.qw)) || (rc = s->upload(&b.qpd, qpd)) ||
      (rc = s->upload(&b.eqp, t.eqp)) || (rc = s->upload(&b.eqw, t.eqw)) ||
      (rc = s->upload(&b.ephi, t.ephi)) || (rc = s->upload(&s->d_i2f, s->i2f)) ||
      (rc = s->upload(&s->d_f2i, s->f2i)))
    return rc;
  {
    // largest |phi_k| over the volume points and every local face's points
    const size_t np = static_cast<size_t>(t.Np);
    std::vector<double> phimax(np, 0.0);
    for (size_t i = 0; i < t.phi.size(); ++i) phimax[i % np] = std::max(phimax[i % np], std::fabs(t.phi[i]));
    for (size_t i = 0; i < t.phif.size(); ++i) phimax[i % np] = std::max(phimax[i % np], std::fabs(t.phif[i]));
    if ((rc = s->upload_t(&b.phimax, phimax))) return rc;
  }
  {
    std::vector<double> blob(s->ops.blob_elems);
    s->ops.fill_blob(t.dphi.data(), t.phif.data(), t.phi.data(), t.qw.data(), blob.data());
    if ((rc = s->upload_t(&b.blob, blob))) return rc;
    std::vector<double> fblob(s->ops.fused_blob_elems, 0.0);
    s->ops.fill_fused_blob(t.dphi.data(), t.phif.data(), t.phi.data(), t.qw.data(), fblob.data());
    if ((rc = s->upload_t(&b.fblob, fblob))) return rc;
    b.blob_bytes = static_cast<int>(s->ops.blob_elems * s->ops.tsize);
  }
  b.nqe = t.nqe;
  b.phi0 = t.phi0;
  b.law = lps[0];
  b.law.field = field;

  const size_t nstate = s->state_count();
  // slots are tile-transposed over whole tiles of TE cells; state buffers get
  // 256 bytes of tail so the bulk copy of the last tile may round up to 16 bytes
  const size_t ntiles = (static_cast<size_t>(Etot) + TE - 1) / TE;
  const size_t nslot = ntiles * TE * t.nlf * t.nqf * b.M;
  unsigned char *C, *U0, *slots, *tr, *rhs, *scratch;
  const size_t ts = s->ops.tsize;  // slots and traces hold the RHS arithmetic type; the state is FP64
  if ((rc = s->alloc(&C, nstate * 8 + 256)) || (rc = s->alloc(&U0, nstate * 8 + 256)) ||
      (rc = s->alloc(&slots, nslot * ts)) || (rc = s->alloc(&tr, nslot * ts)) ||
      (rc = s->alloc(&rhs, nstate * 8 + 256)) || (rc = s->alloc(&scratch, nstate * 8 + 256)))
    return rc;
  DGP_CUDA(cudaMemset(tr, 0, nslot * ts));
  DGP_CUDA(cudaMemset(C, 0, nstate * 8 + 256));
  DGP_CUDA(cudaMemset(U0, 0, nstate * 8 + 256));
  if (s->fused_ok) {  // stage states u1, u2 (with the same tail as the state)
    unsigned char *X1, *X2;
    if ((rc = s->alloc(&X1, nstate * 8 + 256)) || (rc = s->alloc(&X2, nstate * 8 + 256))) return rc;
    DGP_CUDA(cudaMemset(X1, 0, nstate * 8 + 256));
    DGP_CUDA(cudaMemset(X2, 0, nstate * 8 + 256));
    b.X1 = X1;
    b.X2 = X2;
  }
  b.C = C;
  b.U0 = U0;
  b.slots = slots;
  b.tr = tr;
  b.rhs = rhs;
  b.scratch = scratch;
  b.npartials = std::max(s->ops.grid_elem(Etot), (Etot + 255) / 256) * std::max(b.M, 3) + 1;
  const int nctl = ensemble ? n + 1 : 1;
  if ((rc = s->alloc(&b.partials, b.npartials)) || (rc = s->alloc(&b.ctl, nctl)) ||
      (rc = s->alloc(&b.status, 1)))
    return rc;
  DGP_CUDA(cudaMemset(slots, 0, nslot * ts));
  {
    std::vector<TimeCtl> c0(nctl);
    for (auto& c : c0) {
      c = TimeCtl{};
      c.dtmin_bits = 0x7FF0000000000000ull;
    }
    DGP_CUDA(cudaMemcpy(b.ctl, c0.data(), nctl * sizeof(TimeCtl), cudaMemcpyHostToDevice));
  }
  b.gctl = b.ctl + (ensemble ? n : 0);
  if (ensemble) {
    std::vector<int> inst_end(n), tile_first(n + 1);
    for (int i = 0; i < n; ++i) {
      inst_end[i] = s->inst_off[i] + s->meshes[i].E;
      tile_first[i] = s->inst_off[i] / TE;
    }
    tile_first[n] = (Etot + TE - 1) / TE;
    if ((rc = s->upload(&b.cell_inst, cell_inst)) || (rc = s->upload(&b.inst_end, inst_end)) ||
        (rc = s->upload(&b.tile_first, tile_first)) || (rc = s->upload(&b.laws, lps)))
      return rc;
    b.ninst = n;
  }
  Status st0{0, INT32_MAX};
  DGP_CUDA(cudaMemcpy(b.status, &st0, sizeof(Status), cudaMemcpyHostToDevice));
  // P0 fallback marks (DGCell::setToZero), on by default for the Euler laws
  // whose isPhysical can fail
  if ((rc = s->alloc(&b.bad, static_cast<size_t>(Etot)))) return rc;
  DGP_CUDA(cudaMemset(b.bad, 0, Etot));
  b.p0 = (s->law == DGP_LAW_EULER2D || s->law == DGP_LAW_EULER3D) ? 1 : 0;
  b.limiter_kind = s->order >= 1 ? s->limiter : DGP_LIMITER_NONE;
  if (s->limiter == DGP_LIMITER_MOMENT && s->order >= 1) {
    if ((rc = setup_limiter(s))) return rc;
  }
  if (s->limiter == DGP_LIMITER_BARTH && s->order >= 1) {
    // FP64 face-point basis values and each cell's faces; triggers per row
    if ((rc = s->upload(&b.cface, cface)) || (rc = s->upload(&b.bphif, t.phif)) ||
        (rc = s->alloc(&b.trig, static_cast<size_t>(Etot) * b.M)))
      return rc;
    DGP_CUDA(cudaMemset(b.trig, 0, static_cast<size_t>(Etot) * b.M));
  }
  if (cudaError_t e = s->ops.prepare()) return fail(DGP_ERR_CUDA, cudaGetErrorString(e));
  // DGAnalysis::DGAnalysis projects the far field as the initial state
  s->ops.project(b, 0.0, s->stream);
  s->ops.trace(b, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

// common part of solver and ensemble-group creation: kernels, tables, stream
static int solver_begin(dgp_solver s, int law, int flux, int dim, int order, int precision, int limiter,
                        int block, int rule = DGP_RULE_REFERENCE) {
  ensure_registry();
  auto it = ops_registry().find(OpsKey(law, flux, dim, order, precision, block, rule));
  if (it == ops_registry().end())
    return fail(DGP_ERR_UNSUPPORTED, rule == DGP_RULE_REFERENCE
                                         ? "no kernels for this law/flux/element/order/precision"
                                         : "no kernels with this quadrature rule for this configuration");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(DGP_ERR_CUDA, "no CUDA device available");
  s->ops = it->second;
  s->law = law;
  s->flux = flux;
  s->order = order;
  s->precision = precision;
  s->limiter = limiter;
  cudaGetDevice(&s->device);
  std::string err;
  s->rule = rule;
  if (int rc = build_tables(dim, order, s->tab, err, rule)) return fail(rc, err);
  const RefTables& t = s->tab;
  if (t.nq != s->ops.NQ || t.nqf != s->ops.NQF || t.Np != s->ops.NP)
    return fail(DGP_ERR_UNSUPPORTED, "table/kernel shape mismatch");
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(DGP_ERR_CUDA, "stream creation failed");
  if (cudaMallocHost(&s->h_ctl, 2 * sizeof(TimeCtl)) != cudaSuccess)
    return fail(DGP_ERR_CUDA, "pinned allocation failed");
  return DGP_OK;
}

extern "C" {

const char* dgp_last_error(void) { return g_err.c_str(); }
int dgp_version(void) { return 1; }

int dgp_set_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
    return fail(DGP_ERR_INVALID, "no CUDA device " + std::to_string(device));
  DGP_CUDA(cudaSetDevice(device));
  return DGP_OK;
}

int dgp_mesh_from_msh(const char* path, dgp_mesh* out) { return dgp_mesh_from_msh_ex(path, 0, out); }

int dgp_mesh_from_msh_ex(const char* path, int gpu_faces, dgp_mesh* out) {
  if (!path || !out) return fail(DGP_ERR_INVALID, "null argument");
  auto* h = new dgp_mesh_s;
  std::string err;
  int rc = read_msh_v1(path, h->m, err, gpu_faces != 0);
  if (rc != DGP_OK) {
    delete h;
    return fail(rc, err);
  }
  *out = h;
  return DGP_OK;
}

int dgp_mesh_from_arrays(int dim, int nv, const double* xyz, const int* vertex_ids, int ncells,
                         const int* cells, int cell_tag, int nbfaces, const int* bfaces,
                         const int* btags, dgp_mesh* out) {
  return dgp_mesh_from_arrays_ex(dim, nv, xyz, vertex_ids, ncells, cells, cell_tag, nbfaces, bfaces, btags, 0,
                                 out);
}

int dgp_mesh_from_arrays_ex(int dim, int nv, const double* xyz, const int* vertex_ids, int ncells,
                            const int* cells, int cell_tag, int nbfaces, const int* bfaces, const int* btags,
                            int gpu_faces, dgp_mesh* out) {
  if (!out) return fail(DGP_ERR_INVALID, "null output handle");
  auto* h = new dgp_mesh_s;
  std::string err;
  int rc = mesh_from_arrays(dim, nv, xyz, vertex_ids, ncells, cells, cell_tag, nbfaces, bfaces, btags,
                            h->m, err, gpu_faces != 0);
  if (rc != DGP_OK) {
    delete h;
    return fail(rc, err);
  }
  *out = h;
  return DGP_OK;
}

int dgp_mesh_info(dgp_mesh m, int* dim, int* ncells, int* nfaces, int* nvertices) {
  if (!m) return fail(DGP_ERR_INVALID, "null mesh");
  if (dim) *dim = m->m.dim;
  if (ncells) *ncells = m->m.E;
  if (nfaces) *nfaces = m->m.F;
  if (nvertices) *nvertices = static_cast<int>(m->m.vid.size());
  return DGP_OK;
}

int dgp_mesh_connectivity(dgp_mesh mh, int* out) {
  if (!mh || !out) return fail(DGP_ERR_INVALID, "null argument");
  const HostMesh& m = mh->m;
  size_t w = 0;
  for (int f = 0; f < m.F; ++f) {
    int v[3];
    for (int k = 0; k < m.nfv; ++k) v[k] = m.vid[m.fv[static_cast<size_t>(f) * m.nfv + k]];
    std::sort(v, v + m.nfv);
    for (int k = 0; k < m.nfv; ++k) out[w++] = v[k];
    out[w++] = m.eL[f];
    out[w++] = m.eR[f];
    out[w++] = m.lfL[f];
    out[w++] = m.lfR[f];
    out[w++] = m.bid[f];
  }
  return DGP_OK;
}

int dgp_mesh_face_geometry(dgp_mesh mh, double* out) {
  if (!mh || !out) return fail(DGP_ERR_INVALID, "null argument");
  const HostMesh& m = mh->m;
  for (int f = 0; f < m.F; ++f) {
    for (int k = 0; k < 3; ++k) out[4 * f + k] = m.fn[3 * f + k];
    out[4 * f + 3] = m.fmeas[f];
  }
  return DGP_OK;
}

int dgp_mesh_destroy(dgp_mesh m) {
  delete m;
  return DGP_OK;
}

int dgp_law_create(int kind, int flux, int field, const double* params, dgp_law* out) {
  if (!out) return fail(DGP_ERR_INVALID, "null output handle");
  if (kind < DGP_LAW_SCALAR || kind > DGP_LAW_MAXWELL2D) return fail(DGP_ERR_INVALID, "unknown law");
  if (flux < DGP_FLUX_UPWIND || flux > DGP_FLUX_LLF) return fail(DGP_ERR_INVALID, "unknown flux");
  if (field < DGP_FIELD_GAUSS || field > DGP_FIELD_TM2D) return fail(DGP_ERR_INVALID, "unknown field");
  auto* l = new dgp_law_s;
  l->kind = kind;
  l->flux = flux;
  l->field = field;
  for (int i = 0; i < DGP_NPARAMS; ++i) l->p[i] = params ? params[i] : 0.0;
  if (!(l->p[7] > 0.0)) l->p[7] = 1.4;  // gamma default (EulerLaw.h:14)
  *out = l;
  return DGP_OK;
}

int dgp_law_set_bc(dgp_law l, int boundary_id, int bc_kind) {
  if (!l) return fail(DGP_ERR_INVALID, "null law");
  if (bc_kind < DGP_BC_DEFAULT || bc_kind > DGP_BC_WALL) return fail(DGP_ERR_INVALID, "unknown boundary condition");
  if (boundary_id == 510 || boundary_id == 610)
    return fail(DGP_ERR_INVALID, "510 and 610 are periodic edges, not boundary conditions");
  if (bc_kind == DGP_BC_WALL && (l->kind == DGP_LAW_SCALAR || l->kind == DGP_LAW_BURGERS2D))
    return fail(DGP_ERR_UNSUPPORTED, "no wall condition for the scalar laws");
  for (int i = 0; i < l->nbc; ++i)
    if (l->bc_id[i] == boundary_id) {
      l->bc_kind[i] = bc_kind;
      return DGP_OK;
    }
  if (l->nbc == DGP_MAX_BC) return fail(DGP_ERR_INVALID, "too many boundary settings on one law");
  l->bc_id[l->nbc] = boundary_id;
  l->bc_kind[l->nbc] = bc_kind;
  ++l->nbc;
  return DGP_OK;
}

int dgp_law_destroy(dgp_law l) {
  delete l;
  return DGP_OK;
}

int dgp_solver_create(dgp_mesh mh, dgp_law law, int order, int precision, int limiter,
                      dgp_solver* out) {
  return dgp_solver_create_ex(mh, law, order, precision, limiter, DGP_RULE_REFERENCE, out);
}

int dgp_solver_create_ex(dgp_mesh mh, dgp_law law, int order, int precision, int limiter, int rule,
                         dgp_solver* out) {
  if (!mh || !law || !out) return fail(DGP_ERR_INVALID, "null argument");
  if (rule != DGP_RULE_REFERENCE && rule != DGP_RULE_WORKLOAD) return fail(DGP_ERR_INVALID, "unknown rule");
  if (precision != DGP_PRECISION_FP64 && precision != DGP_PRECISION_MIXED)
    return fail(DGP_ERR_INVALID, "unknown precision");
  if (limiter != DGP_LIMITER_NONE && limiter != DGP_LIMITER_MOMENT && limiter != DGP_LIMITER_BARTH)
    return fail(DGP_ERR_INVALID, "unknown limiter");
  const HostMesh& m = mh->m;
  if (limiter == DGP_LIMITER_MOMENT && m.dim != 2)
    return fail(DGP_ERR_UNSUPPORTED, "the moment limiter is built for triangles only");
  if ((law->kind == DGP_LAW_EULER2D || law->kind == DGP_LAW_BURGERS2D || law->kind == DGP_LAW_MAXWELL2D) &&
      m.dim != 2)
    return fail(DGP_ERR_UNSUPPORTED, "2D law on a 3D mesh");
  if ((law->kind == DGP_LAW_EULER3D || law->kind == DGP_LAW_MAXWELL3D) && m.dim != 3)
    return fail(DGP_ERR_UNSUPPORTED, "3D law on a 2D mesh");
  auto s = new dgp_solver_s;
  // the other rule is built for the default tile shape only
  const int block = rule == DGP_RULE_REFERENCE ? tuned_block(law->kind, law->flux, m.dim, order, precision, m.E)
                                               : kDefaultBlock;
  if (int rc = solver_begin(s, law->kind, law->flux, m.dim, order, precision, limiter, block, rule)) {
    delete s;
    return rc;
  }
  s->meshes.push_back(m);
  const LawParams lp = law->params();
  if (int rc = build_solver(s, {lp}, law->field, false)) {
    delete s;
    return rc;
  }
  *out = s;
  return DGP_OK;
}

int dgp_solver_destroy(dgp_solver s) {
  if (s) {
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
  }
  delete s;
  return DGP_OK;
}

int dgp_solver_info(dgp_solver s, int* nfields, int* nmodes, int* ncells, int* nfaces) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (nfields) *nfields = s->b.M;
  if (nmodes) *nmodes = s->b.NP;
  if (ncells) *ncells = s->b.E;
  if (nfaces) *nfaces = s->b.F;
  return DGP_OK;
}

static int set_ctl(dgp_solver s, double t, double dt, double tend, double cfl, int max_steps) {
  TimeCtl c{};
  c.t = t;
  c.dt = dt;
  c.tend = tend;
  c.cfl = cfl;
  c.max_steps = max_steps;
  c.lts_shift = s->lts.on ? s->lts.nb - 1 : 0;  // mode-5 step: CFL minimum times 2^(bins-1)
  c.dtmin_bits = 0x7FF0000000000000ull;
  s->h_ctl[0] = c;
  DGP_CUDA(cudaMemcpyAsync(s->b.ctl, &s->h_ctl[0], sizeof(TimeCtl), cudaMemcpyHostToDevice, s->stream));
  return DGP_OK;
}

static int read_ctl(dgp_solver s, TimeCtl* out) {
  DGP_CUDA(cudaMemcpyAsync(&s->h_ctl[1], s->b.ctl, sizeof(TimeCtl), cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  *out = s->h_ctl[1];
  return DGP_OK;
}

int dgp_project(dgp_solver s, double t) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  DGP_CUDA(cudaSetDevice(s->device));
  s->ops.project(s->b, t, s->stream);
  // DGAnalysis::DGAnalysis limits the projected state once (DGAnalysis.cc:276-291)
  if (s->limiter != DGP_LIMITER_NONE && s->ops.limit) s->ops.limit(s->b, 0, s->stream);
  s->ops.trace(s->b, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

// host FP64 [cell][field][mode] in file order <-> device state in internal order:
// one copy of the whole array through the state-sized staging buffer, the
// reordering by a gather kernel on the solver's stream
static int host_to_state(dgp_solver s, const double* in, void* dst) {
  const int mnp = s->b.M * s->b.NP;
  const size_t n = s->state_count();
  DGP_CUDA(cudaMemcpyAsync(s->b.scratch, in, n * 8, cudaMemcpyHostToDevice, s->stream));
  const int grid = static_cast<int>((n + 255) / 256);
  gather_cells<double, double><<<grid, 256, 0, s->stream>>>(static_cast<const double*>(s->b.scratch),
                                                            static_cast<double*>(dst), s->d_i2f, s->b.E, mnp);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

static int state_to_host(dgp_solver s, const void* src, double* out) {
  const int mnp = s->b.M * s->b.NP;
  const size_t n = s->state_count();
  const int grid = static_cast<int>((n + 255) / 256);
  gather_cells<double, double><<<grid, 256, 0, s->stream>>>(static_cast<const double*>(src),
                                                            static_cast<double*>(s->b.scratch), s->d_f2i, s->b.E,
                                                            mnp);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaMemcpyAsync(out, s->b.scratch, n * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

// ---------------------------------------------------------------------------
// Checkpoints in the data format of DGAnalysis::write / read (DGPref.cc:712-766,
// DGCell::write / read DGCell.cc:1523-1540, mMesh::writeMEntity / readMEntity
// mMesh.cc:401-455): TACT, ITER, "dim cells faces", then per cell its entity
// (type, geometric order, vertex ids) followed by "order" and the coefficients
// [field][mode], then the face entities.  DGAnalysis::write omits the geometric
// order that readMEntity expects; files are written the way readMEntity reads
// them, and both layouts are read.
static const int kTypeEdge = 1, kTypeTri = 2, kTypeTet = 4;  // mEntity::mType

int dgp_checkpoint_write(dgp_solver s, const char* path, double t, int iter) {
  if (!s || !path) return fail(DGP_ERR_INVALID, "null argument");
  if (s->b.ninst) return fail(DGP_ERR_UNSUPPORTED, "checkpoints are written for a single solver");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  const HostMesh& m = s->meshes[0];
  const size_t mnp = static_cast<size_t>(s->b.M) * s->b.NP;
  std::vector<double> c(static_cast<size_t>(m.E) * mnp);
  if (int rc = state_to_host(s, s->b.C, c.data())) return rc;
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(DGP_ERR_IO, std::string("cannot write ") + path);
  const int ctype = m.dim == 2 ? kTypeTri : kTypeTet, ftype = m.dim == 2 ? kTypeEdge : kTypeTri;
  std::fprintf(f, "%.17g\n%d\n%d %d %d\n", t, iter, m.dim, m.E, m.F);
  for (int e = 0; e < m.E; ++e) {
    std::fprintf(f, "%d 1 ", ctype);
    for (int k = 0; k < m.nvc; ++k) std::fprintf(f, "%d ", m.vid[m.cv[static_cast<size_t>(e) * m.nvc + k]]);
    std::fprintf(f, "\n%d ", s->order);
    for (size_t i = 0; i < mnp; ++i) std::fprintf(f, "%.17g ", c[e * mnp + i]);
  }
  for (int fc = 0; fc < m.F; ++fc) {
    std::fprintf(f, "%d 1 ", ftype);
    for (int k = 0; k < m.nfv; ++k) std::fprintf(f, "%d ", m.vid[m.fv[static_cast<size_t>(fc) * m.nfv + k]]);
    std::fprintf(f, "\n");
  }
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? DGP_OK : fail(DGP_ERR_IO, std::string("write failed: ") + path);
}

int dgp_checkpoint_read(dgp_solver s, const char* path, double* t, int* iter) {
  if (!s || !path) return fail(DGP_ERR_INVALID, "null argument");
  if (s->b.ninst) return fail(DGP_ERR_UNSUPPORTED, "checkpoints are read into a single solver");
  std::ifstream in(path);
  if (!in) return fail(DGP_ERR_IO, std::string("cannot read ") + path);
  std::vector<std::string> tok;
  for (std::string w; in >> w;) tok.push_back(w);
  const HostMesh& m = s->meshes[0];
  const size_t mnp = static_cast<size_t>(s->b.M) * s->b.NP;
  if (tok.size() < 5) return fail(DGP_ERR_IO, "checkpoint header is incomplete");
  double tt = std::strtod(tok[0].c_str(), nullptr);
  const int it = std::atoi(tok[1].c_str()), dim = std::atoi(tok[2].c_str());
  const int ncell = std::atoi(tok[3].c_str()), nface = std::atoi(tok[4].c_str());
  if (dim != m.dim || ncell != m.E) return fail(DGP_ERR_IO, "checkpoint does not match the solver's mesh");
  // layout: with or without the geometric order after each type, with or
  // without the face list
  const size_t rest = tok.size() - 5;
  int go = -1;
  for (int g = 1; g >= 0 && go < 0; --g)
    for (int fl = 1; fl >= 0 && go < 0; --fl) {
      const size_t need = static_cast<size_t>(ncell) * (1 + g + m.nvc + 1 + mnp) +
                          (fl ? static_cast<size_t>(nface) * (1 + g + m.nfv) : 0);
      if (need == rest) go = g;
    }
  if (go < 0) return fail(DGP_ERR_IO, "checkpoint size does not match the solver's fields and order");
  // cells by their sorted vertex ids
  std::map<std::vector<int>, int> byv;
  for (int e = 0; e < m.E; ++e) {
    std::vector<int> key(m.nvc);
    for (int k = 0; k < m.nvc; ++k) key[k] = m.vid[m.cv[static_cast<size_t>(e) * m.nvc + k]];
    std::sort(key.begin(), key.end());
    byv[key] = e;
  }
  std::vector<double> c(static_cast<size_t>(m.E) * mnp, 0.0);
  std::vector<char> seen(m.E, 0);
  size_t p = 5;
  for (int i = 0; i < ncell; ++i) {
    ++p;  // type
    p += go;
    std::vector<int> key(m.nvc);
    for (int k = 0; k < m.nvc; ++k) key[k] = std::atoi(tok[p++].c_str());
    std::sort(key.begin(), key.end());
    const int order = std::atoi(tok[p++].c_str());
    auto f = byv.find(key);
    if (f == byv.end()) return fail(DGP_ERR_IO, "checkpoint cell " + std::to_string(i) + " is not in the mesh");
    if (order != s->order) return fail(DGP_ERR_UNSUPPORTED, "checkpoint cell order differs from the solver's");
    const int e = f->second;
    seen[e] = 1;
    for (size_t k = 0; k < mnp; ++k) c[e * mnp + k] = std::strtod(tok[p++].c_str(), nullptr);
  }
  for (int e = 0; e < m.E; ++e)
    if (!seen[e]) return fail(DGP_ERR_IO, "checkpoint misses cell " + std::to_string(e));
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (int rc = host_to_state(s, c.data(), s->b.C)) return rc;
  s->ops.trace(s->b, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (t) *t = tt;
  if (iter) *iter = it;
  return DGP_OK;
}

// the face-point traces after the state was set from outside the stages:
// the separate face kernel reads them at once; the fused stage kernel keeps
// none, so they are only marked stale (refreshed by whatever reads them next:
// local time stepping, a switch to the separate form)
static void traces_after_state_change(dgp_solver s) {
  if (s->fused && !s->lts.on) {
    s->tr_stale = true;
    return;
  }
  s->ops.trace(s->b, nullptr, s->stream);
  s->tr_stale = false;
}

int dgp_set_state(dgp_solver s, const double* host_state) {
  if (!s || !host_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (int rc = host_to_state(s, host_state, s->b.C)) return rc;
  traces_after_state_change(s);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_get_state(dgp_solver s, double* host_state) {
  if (!s || !host_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return state_to_host(s, s->b.C, host_state);
}

int dgp_set_state_device(dgp_solver s, const double* dev_state) {
  if (!s || !dev_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const int mnp = s->b.M * s->b.NP;
  const long long n = static_cast<long long>(s->b.E) * mnp;
  const int grid = static_cast<int>((n + 255) / 256);
  gather_cells<double, double><<<grid, 256, 0, s->stream>>>(dev_state, static_cast<double*>(s->b.C),
                                                            s->d_i2f, s->b.E, mnp);
  traces_after_state_change(s);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_get_state_device(dgp_solver s, double* dev_state) {
  if (!s || !dev_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const int mnp = s->b.M * s->b.NP;
  const long long n = static_cast<long long>(s->b.E) * mnp;
  const int grid = static_cast<int>((n + 255) / 256);
  gather_cells<double, double><<<grid, 256, 0, s->stream>>>(static_cast<const double*>(s->b.C), dev_state,
                                                            s->d_f2i, s->b.E, mnp);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_rhs(dgp_solver s, double t, double* host_rhs) {
  if (!s || !host_rhs) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  if (int rc = set_ctl(s, t, 0.0, 0.0, 0.0, 0)) return rc;
  if (s->fused) {
    const double* C = static_cast<const double*>(s->b.C);
    s->ops.fused(s->b, C, C, static_cast<double*>(s->b.rhs), nullptr, 0, 0.0, 0, s->stream);
  } else {
    // the P0 fallback's second face pass zeroes the marked cells' modes in
    // the state: the assembly runs on a copy, the state stays as it was
    const size_t bytes = s->state_count() * 8;
    if (s->b.p0)
      DGP_CUDA(cudaMemcpyAsync(s->b.scratch, s->b.C, bytes, cudaMemcpyDeviceToDevice, s->stream));
    s->ops.stage(s->b, 0, 0.0, 0, s->stream);
    if (s->b.p0)
      DGP_CUDA(cudaMemcpyAsync(s->b.C, s->b.scratch, bytes, cudaMemcpyDeviceToDevice, s->stream));
  }
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return state_to_host(s, s->b.rhs, host_rhs);
}

int dgp_cfl_dt(dgp_solver s, double cfl, double* dt) {
  if (!s || !dt || !(cfl > 0)) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  if (int rc = set_ctl(s, 0.0, 0.0, 0.0, cfl, 0)) return rc;
  s->ops.cfl(s->b, s->stream);
  DGP_CUDA(cudaGetLastError());
  TimeCtl c;
  if (int rc = read_ctl(s, &c)) return rc;
  *dt = c.dt;
  return DGP_OK;
}

// RungeKuttaTVD3::advanceInTime: with the limiter, TimeIntegrator::limit
// follows every stage and the next step's CFL reduction runs on the limited
// state (instead of inside the last stage's element kernel)
static void launch_step(dgp_solver s, int fuse_cfl) {
  if (s->lts.on) {  // RungeKuttaTVD2adaptive::advanceInTime
    dgp::launch_lts_step(s, fuse_cfl != 0);
    if (!s->probes.empty()) launch_probe_recorders(s);
    return;
  }
  const bool lim = s->limiter != DGP_LIMITER_NONE && s->ops.limit;
  if (s->fused) {
    // u_n (C) -> u1 (X1) -> u2 (X2) -> u_n+1 (C, own rows in place); the
    // limiter runs on each stage's output
    DeviceBuffers& b = s->b;
    double* C = static_cast<double*>(b.C);
    double* X1 = static_cast<double*>(b.X1);
    double* X2 = static_cast<double*>(b.X2);
    DeviceBuffers bl = b;
    s->ops.fused(b, C, C, X1, nullptr, 1, 0.0, 0, s->stream);
    if (lim) {
      bl.C = X1;
      s->ops.limit(bl, 1, s->stream);
    }
    s->ops.fused(b, X1, C, X2, nullptr, 2, 1.0, 0, s->stream);
    if (lim) {
      bl.C = X2;
      s->ops.limit(bl, 1, s->stream);
    }
    s->ops.fused(b, X2, C, C, nullptr, 3, 0.5, lim ? 0 : fuse_cfl, s->stream);
    if (lim) {
      s->ops.limit(b, 1, s->stream);
      if (fuse_cfl) s->ops.cfl(b, s->stream);
    }
    s->tr_stale = true;
  } else {
    s->ops.stage(s->b, 1, 0.0, 0, s->stream);
    if (lim) s->ops.limit(s->b, 1, s->stream);
    s->ops.stage(s->b, 2, 1.0, 0, s->stream);
    if (lim) s->ops.limit(s->b, 1, s->stream);
    s->ops.stage(s->b, 3, 0.5, lim ? 0 : fuse_cfl, s->stream);
    if (lim) {
      s->ops.limit(s->b, 1, s->stream);
      if (fuse_cfl) s->ops.cfl(s->b, s->stream);
    }
  }
  if (!s->probes.empty()) launch_probe_recorders(s);
}

// the local time stepping kernels read the face-point traces, which the fused
// stage kernel does not keep
static void refresh_traces(dgp_solver s) {
  if (!s->tr_stale) return;
  s->ops.trace(s->b, nullptr, s->stream);
  s->tr_stale = false;
}

int dgp_launches_per_step(dgp_solver s, int* n) {
  if (!s || !n) return fail(DGP_ERR_INVALID, "null argument");
  if (s->lts.on) {
    *n = dgp::launch_lts_step(s, true, true);
    return DGP_OK;
  }
  const bool lim = s->limiter != DGP_LIMITER_NONE && s->ops.limit;
  const int per_pass = s->limiter == DGP_LIMITER_BARTH ? 1 : 2;
  *n = (s->fused ? 4 : 3 * (s->b.p0 ? 4 : 2)) + (lim ? 3 * per_pass + 1 : 0);
  return DGP_OK;
}

int dgp_step(dgp_solver s, double t, double dt, double* resid) {
  if (!s || !(dt > 0)) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  if (int rc = set_ctl(s, t, dt, 0.0, 0.0, 0)) return rc;
  if (s->lts.on) refresh_traces(s);
  launch_step(s, 0);
  DGP_CUDA(cudaGetLastError());
  TimeCtl c;
  if (int rc = read_ctl(s, &c)) return rc;
  if (resid) *resid = c.resid;
  return DGP_OK;
}

int dgp_run(dgp_solver s, double t0, double tend, double cfl, int max_steps, double* t_out,
            int* steps_out) {
  if (!s || !(cfl > 0)) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  if (tend <= 0 && max_steps <= 0) {
    if (t_out) *t_out = t0;
    if (steps_out) *steps_out = 0;
    return DGP_OK;
  }
  // K steps per graph; finished steps turn the remaining kernels into no-ops.
  // The last steps of a run with a step limit go through a one-step graph.
  const int K = 8;
  auto capture = [&](int steps, cudaGraphExec_t* out) -> int {
    cudaGraph_t g;
    DGP_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < steps; ++k) launch_step(s, 1);
    DGP_CUDA(cudaStreamEndCapture(s->stream, &g));
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(DGP_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
    return DGP_OK;
  };
  const bool tail = max_steps > 0 && max_steps % K != 0;
  if (s->lts.on) refresh_traces(s);
  if (!s->graph) {
    if (int rc = capture(K, &s->graph)) return rc;
    s->graph_steps = K;
  }
  if (tail && !s->graph1)
    if (int rc = capture(1, &s->graph1)) return rc;
  if (int rc = set_ctl(s, t0, 0.0, tend, cfl, max_steps)) return rc;
  if (int rc = reset_probe_recorders(s)) return rc;
  s->ops.cfl(s->b, s->stream);
  DGP_CUDA(cudaGetLastError());
  TimeCtl c{};
  for (long long guard = 0;; ++guard) {
    const bool one = tail && max_steps - c.steps < K;
    DGP_CUDA(cudaGraphLaunch(one ? s->graph1 : s->graph, s->stream));
    if (int rc = read_ctl(s, &c)) return rc;
    if (c.done) break;
    if (!std::isfinite(c.dt) || !(c.dt > 0))
      return fail(DGP_ERR_NONPHYSICAL, "time step is not positive and finite");
  }
  if (t_out) *t_out = c.t;
  if (steps_out) *steps_out = c.steps;
  return DGP_OK;
}

int dgp_limit(dgp_solver s, unsigned char* triggers) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (s->limiter == DGP_LIMITER_NONE) return fail(DGP_ERR_INVALID, "solver created without a limiter");
  DGP_CUDA(cudaSetDevice(s->device));
  if (s->ops.limit) s->ops.limit(s->b, 0, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return triggers ? dgp_limiter_triggers(s, triggers) : DGP_OK;
}

int dgp_limiter_triggers(dgp_solver s, unsigned char* out) {
  if (!s || !out) return fail(DGP_ERR_INVALID, "null argument");
  if (s->limiter == DGP_LIMITER_NONE) return fail(DGP_ERR_INVALID, "solver created without a limiter");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  const int E = s->b.E;
  if (!s->b.trig) {  // P0: nothing is ever limited
    std::memset(out, 0, E);
    return DGP_OK;
  }
  // per row on the device; a cell's trigger is the lowest over its fields
  const int M = s->b.M;
  std::vector<unsigned char> t(static_cast<size_t>(E) * M);
  DGP_CUDA(cudaMemcpy(t.data(), s->b.trig, t.size(), cudaMemcpyDeviceToHost));
  // 0 (untouched) maps to 255 so that the minimum over the fields is the
  // lowest limited degree
  const int* i2f = s->i2f.data();
  const unsigned char* tp = t.data();
  if (M == 1) {
    for (int i = 0; i < E; ++i) out[i2f[i]] = tp[i];
  } else {
    for (int i = 0; i < E; ++i) {
      unsigned v = 255;
      for (int j = 0; j < M; ++j) v = std::min(v, (unsigned)(unsigned char)(tp[static_cast<size_t>(i) * M + j] - 1));
      out[i2f[i]] = static_cast<unsigned char>(v + 1);
    }
  }
  return DGP_OK;
}

int dgp_set_p0_fallback(dgp_solver s, int on) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (on && s->lts.on)
    return fail(DGP_ERR_UNSUPPORTED, "the P0 fallback is not built for local time stepping");
  s->drop_graphs();
  s->b.p0 = on ? 1 : 0;
  return DGP_OK;
}

int dgp_set_tensor_cores(dgp_solver s, int on) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (on && !(s->fused && s->ops.tensor_cores_ok))
    return fail(DGP_ERR_UNSUPPORTED,
                "no tensor-core contraction for this solver (mixed form, 128-thread tiles, at most 16 modes)");
  s->drop_graphs();
  s->b.tensor_cores = on ? 1 : 0;
  return DGP_OK;
}

int dgp_set_rounding_probe(dgp_solver s, int mask) {
  if (!s || mask < 0 || mask > 127) return fail(DGP_ERR_INVALID, "bad argument");
  if (mask && !(s->fused && s->ops.probe_ok && s->meshes.size() == 1))
    return fail(DGP_ERR_UNSUPPORTED, "the rounding probe is built for the FP64 P3 Euler (Roe) solver "
                                     "with 128-thread tiles");
  s->drop_graphs();
  s->b.round_mask = mask;
  return DGP_OK;
}

int dgp_set_copy_wait_limit(dgp_solver s, int polls) {
  if (!s || polls < 0) return fail(DGP_ERR_INVALID, "bad argument");
  s->drop_graphs();
  s->b.mbar_polls = polls;
  return DGP_OK;
}

int dgp_status(dgp_solver s, int* nonphysical, int* first_bad_cell) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  DGP_CUDA(cudaSetDevice(s->device));
  Status st;
  DGP_CUDA(cudaMemcpyAsync(&st, s->b.status, sizeof(Status), cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  // each call reports what happened since the previous one
  Status st0{0, INT32_MAX};
  DGP_CUDA(cudaMemcpy(s->b.status, &st0, sizeof(Status), cudaMemcpyHostToDevice));
  if (st.timeouts > 0)
    return fail(DGP_ERR_CUDA, "a bounded wait on a bulk copy gave up in " + std::to_string(st.timeouts) +
                                  " CTA(s); results of that launch are incomplete");
  if (nonphysical) *nonphysical = st.nonphysical;
  if (first_bad_cell) *first_bad_cell = st.nonphysical ? s->i2f[std::min(st.first_bad, s->b.E - 1)] : -1;
  return DGP_OK;
}

int dgp_l2_error(dgp_solver s, double t, int field, double* err) {
  if (!s || !err || field < 0 || field >= s->b.M) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  s->ops.l2err(s->b, t, field, 0, s->b.E, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  const int nblk = (s->b.E + 255) / 256;
  std::vector<double> p(nblk);
  DGP_CUDA(cudaMemcpyAsync(p.data(), s->b.partials, nblk * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  double acc = 0.0;
  for (double v : p) acc += v;
  *err = std::sqrt(acc);
  return DGP_OK;
}

int dgp_error_norms(dgp_solver s, double t, int quantity, int rule, double* norms) {
  if (!s || !norms || (rule != 0 && rule != 1) || quantity >= s->b.M || quantity < -2)
    return fail(DGP_ERR_INVALID, "bad argument");
  if (quantity < 0 && s->law != DGP_LAW_EULER2D && s->law != DGP_LAW_EULER3D)
    return fail(DGP_ERR_INVALID, "pressure and entropy errors are defined for the Euler laws");
  DGP_CUDA(cudaSetDevice(s->device));
  s->ops.norms(s->b, t, quantity, rule, 0, s->b.E, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  const int nblk = (s->b.E + 255) / 256;
  std::vector<double> p(3 * static_cast<size_t>(nblk));
  DGP_CUDA(cudaMemcpyAsync(p.data(), s->b.partials, p.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  double l1 = 0.0, l2 = 0.0, li = 0.0;
  for (int k = 0; k < nblk; ++k) {
    l1 += p[3 * k];
    l2 += p[3 * k + 1];
    li = std::max(li, p[3 * k + 2]);
  }
  norms[0] = l1;
  norms[1] = std::sqrt(l2);
  norms[2] = li;
  return DGP_OK;
}

int dgp_totals(dgp_solver s, double* totals) {
  if (!s || !totals) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const double refm = s->b.dim == 2 ? 0.5 : 1.0 / 6.0;
  s->ops.totals(s->b, refm, 0, s->b.E, s->stream);
  DGP_CUDA(cudaGetLastError());
  const int nblk = (s->b.E + 255) / 256;
  std::vector<double> p(static_cast<size_t>(nblk) * s->b.M);
  DGP_CUDA(cudaMemcpyAsync(p.data(), s->b.partials, p.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  for (int j = 0; j < s->b.M; ++j) {
    double acc = 0.0;
    for (int k = 0; k < nblk; ++k) acc += p[static_cast<size_t>(k) * s->b.M + j];
    totals[j] = acc;
  }
  return DGP_OK;
}

int dgp_solver_stream(dgp_solver s, void** stream) {
  if (!s || !stream) return fail(DGP_ERR_INVALID, "null argument");
  *stream = static_cast<void*>(s->stream);
  return DGP_OK;
}

int dgp_profile_kernels(dgp_solver s, int iters, float* ms) {
  if (!s || !ms || iters <= 0) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const size_t bytes = s->state_count() * 8;
  // the element kernel updates the state in place: run it with dt = 0 and
  // u_n = u so every launch leaves the state as it found it, then restore it
  DGP_CUDA(cudaMemcpyAsync(s->b.scratch, s->b.C, bytes, cudaMemcpyDeviceToDevice, s->stream));
  DGP_CUDA(cudaMemcpyAsync(s->b.U0, s->b.C, bytes, cudaMemcpyDeviceToDevice, s->stream));
  if (int rc = set_ctl(s, 0.0, 0.0, 0.0, 0.1, 0)) return rc;
  cudaEvent_t ev[4];
  for (auto& e : ev) DGP_CUDA(cudaEventCreate(&e));
  if (s->fused) {
    // stage 1, stage 2 and the last stage with the CFL reduction, each reading
    // the state and writing a stage buffer (the state is left as it is)
    double* C = static_cast<double*>(s->b.C);
    double* X1 = static_cast<double*>(s->b.X1);
    double* X2 = static_cast<double*>(s->b.X2);
    auto run = [&](int k) {
      if (k == 0) s->ops.fused(s->b, C, C, X1, nullptr, 1, 0.0, 0, s->stream);
      if (k == 1) s->ops.fused(s->b, C, C, X2, nullptr, 2, 1.0, 0, s->stream);
      if (k == 2) s->ops.fused(s->b, C, C, X2, nullptr, 3, 0.5, 1, s->stream);
    };
    for (int k = 0; k < 3; ++k) run(k);  // warm-up
    for (int k = 0; k < 3; ++k) {
      DGP_CUDA(cudaEventRecord(ev[k], s->stream));
      for (int i = 0; i < iters; ++i) run(k);
    }
    DGP_CUDA(cudaEventRecord(ev[3], s->stream));
    DGP_CUDA(cudaGetLastError());
    DGP_CUDA(cudaEventSynchronize(ev[3]));
    for (int k = 0; k < 3; ++k) {
      float t = 0;
      DGP_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      ms[k] = t / iters;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    DGP_CUDA(cudaMemcpyAsync(s->b.C, s->b.scratch, bytes, cudaMemcpyDeviceToDevice, s->stream));
    DGP_CUDA(cudaStreamSynchronize(s->stream));
    return DGP_OK;
  }
  s->ops.face(s->b, 2, 1.0, s->stream);  // warm-up
  s->ops.elem(s->b, 2, 0, s->stream);
  s->ops.elem(s->b, 3, 1, s->stream);
  DGP_CUDA(cudaEventRecord(ev[0], s->stream));
  for (int i = 0; i < iters; ++i) s->ops.face(s->b, 2, 1.0, s->stream);
  DGP_CUDA(cudaEventRecord(ev[1], s->stream));
  for (int i = 0; i < iters; ++i) s->ops.elem(s->b, 2, 0, s->stream);
  DGP_CUDA(cudaEventRecord(ev[2], s->stream));
  for (int i = 0; i < iters; ++i) s->ops.elem(s->b, 3, 1, s->stream);
  DGP_CUDA(cudaEventRecord(ev[3], s->stream));
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaEventSynchronize(ev[3]));
  for (int k = 0; k < 3; ++k) {
    float t = 0;
    DGP_CUDA(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
    ms[k] = t / iters;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  DGP_CUDA(cudaMemcpyAsync(s->b.C, s->b.scratch, bytes, cudaMemcpyDeviceToDevice, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_synchronize(dgp_solver s) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}


// ---------------------------------------------------------------------------
// Ensembles: independent instances of uneven size run batched.  Instances of
// one (law, flux, element, order) form a group whose cells, faces and state
// live in one index space (each instance from a tile boundary), so that one
// face kernel and one element kernel per stage serve the whole group; each
// instance keeps its own time control (CFL step, end time, done flag, finish
// clock).  Groups run on their own streams; a run is a loop of CUDA-graph
// launches of 8 steps per group until every instance is done.

int dgp_ensemble_create(int n, const dgp_mesh* meshes, const dgp_law* laws, const int* orders, int precision,
                        int limiter, dgp_ensemble* out) {
  if (n <= 0 || !meshes || !laws || !orders || !out) return fail(DGP_ERR_INVALID, "bad argument");
  if (precision != DGP_PRECISION_FP64 && precision != DGP_PRECISION_MIXED)
    return fail(DGP_ERR_INVALID, "unknown precision");
  if (limiter != DGP_LIMITER_NONE && limiter != DGP_LIMITER_MOMENT && limiter != DGP_LIMITER_BARTH)
    return fail(DGP_ERR_INVALID, "unknown limiter");
  std::map<std::tuple<int, int, int, int>, std::vector<int>> groups;
  for (int i = 0; i < n; ++i) {
    if (!meshes[i] || !laws[i]) return fail(DGP_ERR_INVALID, "null mesh or law");
    const HostMesh& m = meshes[i]->m;
    const dgp_law_s* l = laws[i];
    if ((l->kind == DGP_LAW_EULER2D || l->kind == DGP_LAW_BURGERS2D || l->kind == DGP_LAW_MAXWELL2D) &&
        m.dim != 2)
      return fail(DGP_ERR_UNSUPPORTED, "2D law on a 3D mesh");
    if ((l->kind == DGP_LAW_EULER3D || l->kind == DGP_LAW_MAXWELL3D) && m.dim != 3)
      return fail(DGP_ERR_UNSUPPORTED, "3D law on a 2D mesh");
    if (limiter == DGP_LIMITER_MOMENT && m.dim != 2)
      return fail(DGP_ERR_UNSUPPORTED, "the moment limiter is built for triangles only");
    groups[std::make_tuple(l->kind, l->flux, m.dim, orders[i])].push_back(i);
  }
  auto e = new dgp_ensemble_s;
  e->inst_group.assign(n, -1);
  e->inst_index.assign(n, -1);
  for (auto& kv : groups) {
    const auto& members = kv.second;
    const dgp_law_s* l0 = laws[members[0]];
    for (int i : members)
      if (laws[i]->p[7] != l0->p[7]) {
        delete e;
        return fail(DGP_ERR_INVALID, "instances of one law/order group must share gamma");
      }
    auto s = new dgp_solver_s;
    long long cells = 0;
    for (int i : members) cells += meshes[i]->m.E;
    const int block = tuned_block(std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                                  std::get<3>(kv.first), precision, cells);
    if (int rc = solver_begin(s, std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                              std::get<3>(kv.first), precision, limiter, block)) {
      delete s;
      delete e;
      return rc;
    }
    std::vector<LawParams> lps;
    for (size_t k = 0; k < members.size(); ++k) {
      const int i = members[k];
      s->meshes.push_back(meshes[i]->m);
      lps.push_back(laws[i]->params());
      e->inst_group[i] = static_cast<int>(e->groups.size());
      e->inst_index[i] = static_cast<int>(k);
    }
    if (int rc = build_solver(s, lps, l0->field, true)) {
      delete s;
      delete e;
      return rc;
    }
    e->groups.push_back(s);
  }
  e->n = n;
  *out = e;
  return DGP_OK;
}

int dgp_ensemble_destroy(dgp_ensemble e) {
  if (!e) return DGP_OK;
  for (dgp_solver s : e->groups) dgp_solver_destroy(s);
  delete e;
  return DGP_OK;
}

int dgp_ensemble_info(dgp_ensemble e, int i, int* nfields, int* nmodes, int* ncells, int* group) {
  if (!e || i < 0 || i >= e->n) return fail(DGP_ERR_INVALID, "bad instance");
  dgp_solver s = e->groups[e->inst_group[i]];
  if (nfields) *nfields = s->b.M;
  if (nmodes) *nmodes = s->b.NP;
  if (ncells) *ncells = s->meshes[e->inst_index[i]].E;
  if (group) *group = e->inst_group[i];
  return DGP_OK;
}

int dgp_ensemble_project(dgp_ensemble e, double t) {
  if (!e) return fail(DGP_ERR_INVALID, "null ensemble");
  for (dgp_solver s : e->groups)
    if (int rc = dgp_project(s, t)) return rc;
  return DGP_OK;
}

static int ens_rows(dgp_ensemble e, int i, dgp_solver* s, int* k, size_t* mnp) {
  if (!e || i < 0 || i >= e->n) return fail(DGP_ERR_INVALID, "bad instance");
  *s = e->groups[e->inst_group[i]];
  *k = e->inst_index[i];
  *mnp = static_cast<size_t>((*s)->b.M) * (*s)->b.NP;
  return DGP_OK;
}

int dgp_ensemble_get_state(dgp_ensemble e, int i, double* host_state) {
  dgp_solver s;
  int k;
  size_t mnp;
  if (int rc = ens_rows(e, i, &s, &k, &mnp)) return rc;
  if (!host_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  const int E = s->meshes[k].E, off = s->inst_off[k], uf = s->inst_ufirst[k];
  std::vector<double> tmp(static_cast<size_t>(E) * mnp);
  DGP_CUDA(cudaMemcpy(tmp.data(), static_cast<double*>(s->b.C) + static_cast<size_t>(off) * mnp,
                      tmp.size() * 8, cudaMemcpyDeviceToHost));
  for (int r = 0; r < E; ++r)
    std::memcpy(&host_state[static_cast<size_t>(s->i2f[off + r] - uf) * mnp], &tmp[r * mnp], mnp * 8);
  return DGP_OK;
}

int dgp_ensemble_set_state(dgp_ensemble e, int i, const double* host_state) {
  dgp_solver s;
  int k;
  size_t mnp;
  if (int rc = ens_rows(e, i, &s, &k, &mnp)) return rc;
  if (!host_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  const int E = s->meshes[k].E, off = s->inst_off[k], uf = s->inst_ufirst[k];
  std::vector<double> tmp(static_cast<size_t>(E) * mnp);
  for (int r = 0; r < E; ++r)
    std::memcpy(&tmp[r * mnp], &host_state[static_cast<size_t>(s->i2f[off + r] - uf) * mnp], mnp * 8);
  DGP_CUDA(cudaMemcpy(static_cast<double*>(s->b.C) + static_cast<size_t>(off) * mnp, tmp.data(),
                      tmp.size() * 8, cudaMemcpyHostToDevice));
  s->ops.trace(s->b, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_ensemble_totals(dgp_ensemble e, int i, double* totals) {
  dgp_solver s;
  int k;
  size_t mnp;
  if (int rc = ens_rows(e, i, &s, &k, &mnp)) return rc;
  if (!totals) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const double refm = s->b.dim == 2 ? 0.5 : 1.0 / 6.0;
  const int e0 = s->inst_off[k], e1 = e0 + s->meshes[k].E;
  s->ops.totals(s->b, refm, e0, e1, s->stream);
  DGP_CUDA(cudaGetLastError());
  const int nblk = (e1 - e0 + 255) / 256;
  std::vector<double> p(static_cast<size_t>(nblk) * s->b.M);
  DGP_CUDA(cudaMemcpyAsync(p.data(), s->b.partials, p.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  for (int j = 0; j < s->b.M; ++j) {
    double acc = 0.0;
    for (int q = 0; q < nblk; ++q) acc += p[static_cast<size_t>(q) * s->b.M + j];
    totals[j] = acc;
  }
  return DGP_OK;
}

int dgp_ensemble_l2_error(dgp_ensemble e, int i, double t, int field, double* err) {
  dgp_solver s;
  int k;
  size_t mnp;
  if (int rc = ens_rows(e, i, &s, &k, &mnp)) return rc;
  if (!err || field < 0 || field >= s->b.M) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const int e0 = s->inst_off[k], e1 = e0 + s->meshes[k].E;
  s->ops.l2err(s->b, t, field, e0, e1, s->b.laws + k, s->stream);
  DGP_CUDA(cudaGetLastError());
  const int nblk = (e1 - e0 + 255) / 256;
  std::vector<double> p(nblk);
  DGP_CUDA(cudaMemcpyAsync(p.data(), s->b.partials, nblk * 8, cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  double acc = 0.0;
  for (double v : p) acc += v;
  *err = std::sqrt(acc);
  return DGP_OK;
}

int dgp_ensemble_run(dgp_ensemble e, double t0, double tend, double cfl, int max_steps, double* t_out,
                     int* steps_out, double* ms_out, double* total_ms) {
  if (!e || !(cfl > 0)) return fail(DGP_ERR_INVALID, "bad argument");
  if (tend <= 0 && max_steps <= 0) return fail(DGP_ERR_INVALID, "need an end time or a step count");
  const int G = static_cast<int>(e->groups.size());
  dgp_solver s0 = e->groups[0];
  DGP_CUDA(cudaSetDevice(s0->device));
  for (dgp_solver s : e->groups) {
    // drain earlier work (set_state, project) before the controls change
    DGP_CUDA(cudaStreamSynchronize(s->stream));
    if (!s->graph) {
      const int K = 8;
      cudaGraph_t g;
      DGP_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < K; ++k) launch_step(s, 1);
      DGP_CUDA(cudaStreamEndCapture(s->stream, &g));
      cudaError_t err = cudaGraphInstantiate(&s->graph, g, 0);
      cudaGraphDestroy(g);
      if (err != cudaSuccess) return fail(DGP_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(err));
      s->graph_steps = K;
    }
    const int n = s->b.ninst;
    std::vector<TimeCtl> c(n + 1);
    for (auto& x : c) {
      x = TimeCtl{};
      x.t = t0;
      x.tend = tend;
      x.cfl = cfl;
      x.max_steps = max_steps;
      x.dtmin_bits = 0x7FF0000000000000ull;
    }
    DGP_CUDA(cudaMemcpy(s->b.ctl, c.data(), c.size() * sizeof(TimeCtl), cudaMemcpyHostToDevice));
  }
  // common start: every group waits for the clock mark on the first stream
  cudaEvent_t start;
  DGP_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  mark_clock<<<1, 1, 0, s0->stream>>>(s0->b.gctl);
  DGP_CUDA(cudaEventRecord(start, s0->stream));
  for (dgp_solver s : e->groups) {
    if (s != s0) DGP_CUDA(cudaStreamWaitEvent(s->stream, start, 0));
    s->ops.cfl(s->b, s->stream);
  }
  DGP_CUDA(cudaGetLastError());
  std::vector<int> done(G, 0);
  std::vector<TimeCtl*> gpin(G);
  for (int g = 0; g < G; ++g) gpin[g] = &e->groups[g]->h_ctl[1];
  for (;;) {
    int all = 1;
    for (int g = 0; g < G; ++g)
      if (!done[g]) {
        dgp_solver s = e->groups[g];
        DGP_CUDA(cudaGraphLaunch(s->graph, s->stream));
        DGP_CUDA(cudaMemcpyAsync(gpin[g], s->b.gctl, sizeof(TimeCtl), cudaMemcpyDeviceToHost, s->stream));
      }
    for (int g = 0; g < G; ++g)
      if (!done[g]) {
        DGP_CUDA(cudaStreamSynchronize(e->groups[g]->stream));
        done[g] = gpin[g]->done;
        all &= done[g];
      }
    if (all) break;
  }
  cudaEventDestroy(start);
  // per-instance results
  TimeCtl g0;
  DGP_CUDA(cudaMemcpy(&g0, s0->b.gctl, sizeof(TimeCtl), cudaMemcpyDeviceToHost));
  double tmax = 0.0;
  for (int g = 0; g < G; ++g) {
    dgp_solver s = e->groups[g];
    const int n = s->b.ninst;
    std::vector<TimeCtl> c(n);
    DGP_CUDA(cudaMemcpy(c.data(), s->b.ctl, n * sizeof(TimeCtl), cudaMemcpyDeviceToHost));
    for (int i = 0; i < e->n; ++i) {
      if (e->inst_group[i] != g) continue;
      const TimeCtl& x = c[e->inst_index[i]];
      const double ms = (static_cast<double>(x.t_mark_ns) - static_cast<double>(g0.t_mark_ns)) * 1e-6;
      if (!std::isfinite(x.dt) || !(x.dt > 0))
        return fail(DGP_ERR_NONPHYSICAL, "instance " + std::to_string(i) + ": time step not positive and finite");
      if (t_out) t_out[i] = x.t;
      if (steps_out) steps_out[i] = x.steps;
      if (ms_out) ms_out[i] = ms;
      tmax = std::max(tmax, ms);
    }
  }
  if (total_ms) *total_ms = tmax;
  return DGP_OK;
}

int dgp_ensemble_launches_per_step(dgp_ensemble e, int* n) {
  if (!e || !n) return fail(DGP_ERR_INVALID, "null argument");
  int tot = 0;
  for (dgp_solver s : e->groups) {
    int k = 0;
    if (int rc = dgp_launches_per_step(s, &k)) return rc;
    tot += k;
  }
  *n = tot;
  return DGP_OK;
}


// ---------------------------------------------------------------------------
// Autotuner: times `iters` SSP-RK3 steps (after 2 warm-up steps) of every
// tile shape built for the configuration, on the caller's mesh(es), with CUDA
// events on the solver's stream, and records the fastest for later creations.

// mean ms per step of a built solver (single or ensemble group)
static int time_steps(dgp_solver s, int iters, float* ms) {
  DGP_CUDA(cudaSetDevice(s->device));
  // controls: t = 0, no end, the CFL step of the current state
  const int nctl = s->b.ninst ? s->b.ninst + 1 : 1;
  std::vector<TimeCtl> c(nctl);
  for (auto& x : c) {
    x = TimeCtl{};
    x.cfl = 0.1;
    x.dtmin_bits = 0x7FF0000000000000ull;
  }
  DGP_CUDA(cudaMemcpy(s->b.ctl, c.data(), nctl * sizeof(TimeCtl), cudaMemcpyHostToDevice));
  s->ops.cfl(s->b, s->stream);
  launch_step(s, 0);
  launch_step(s, 0);
  cudaEvent_t e0, e1;
  DGP_CUDA(cudaEventCreate(&e0));
  DGP_CUDA(cudaEventCreate(&e1));
  DGP_CUDA(cudaEventRecord(e0, s->stream));
  for (int k = 0; k < iters; ++k) launch_step(s, 0);
  DGP_CUDA(cudaEventRecord(e1, s->stream));
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  DGP_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / iters;
  return DGP_OK;
}

static const int kTileBlocks[3] = {64, 128, 256};

int dgp_autotune(dgp_mesh mh, dgp_law law, int order, int precision, int limiter, int iters, int* best_block,
                 float* ms_per_step) {
  if (!mh || !law || iters <= 0) return fail(DGP_ERR_INVALID, "bad argument");
  const HostMesh& m = mh->m;
  int best = 0;
  float best_ms = 0;
  bool best_fused = false;
  for (int v = 0; v < 3; ++v) {
    if (ms_per_step) ms_per_step[v] = -1.0f;
    const int block = kTileBlocks[v];
    if (!has_block(law->kind, law->flux, m.dim, order, precision, block)) continue;
    set_tuned_block(law->kind, law->flux, m.dim, order, precision, m.E, block);
    dgp_solver s = nullptr;
    if (int rc = dgp_solver_create(mh, law, order, precision, limiter, &s)) return rc;
    // both stage forms where the fused kernel is built
    float ms = 0;
    bool fused = false;
    int rc = DGP_OK;
    for (int f = 0; f < (s->fused_ok ? 2 : 1) && !rc; ++f) {
      if (s->fused_ok) rc = dgp_set_fused(s, f);
      float t = 0;
      if (!rc) rc = time_steps(s, iters, &t);
      if (!rc && (f == 0 || t < ms)) {
        ms = t;
        fused = f == 1;
      }
    }
    dgp_solver_destroy(s);
    if (rc) return rc;
    if (ms_per_step) ms_per_step[v] = ms;
    if (!best || ms < best_ms) {
      best = block;
      best_ms = ms;
      best_fused = fused;
    }
  }
  if (!best) return fail(DGP_ERR_UNSUPPORTED, "no kernels for this law/flux/element/order/precision");
  set_tuned_block(law->kind, law->flux, m.dim, order, precision, m.E, best);
  set_tuned_fused(law->kind, law->flux, m.dim, order, precision, m.E, best_fused);
  if (best_block) *best_block = best;
  return DGP_OK;
}

int dgp_autotune_ensemble(int n, const dgp_mesh* meshes, const dgp_law* laws, const int* orders, int precision,
                          int limiter, int iters) {
  if (n <= 0 || !meshes || !laws || !orders || iters <= 0) return fail(DGP_ERR_INVALID, "bad argument");
  // one candidate ensemble per group key, timed group by group
  std::map<std::tuple<int, int, int, int>, std::vector<int>> groups;
  for (int i = 0; i < n; ++i) {
    if (!meshes[i] || !laws[i]) return fail(DGP_ERR_INVALID, "null mesh or law");
    groups[std::make_tuple(laws[i]->kind, laws[i]->flux, meshes[i]->m.dim, orders[i])].push_back(i);
  }
  for (auto& kv : groups) {
    const int law = std::get<0>(kv.first), flux = std::get<1>(kv.first), dim = std::get<2>(kv.first),
              order = std::get<3>(kv.first);
    std::vector<dgp_mesh> ms;
    std::vector<dgp_law> ls;
    std::vector<int> os;
    long long cells = 0;
    for (int i : kv.second) {
      ms.push_back(meshes[i]);
      ls.push_back(laws[i]);
      os.push_back(order);
      cells += meshes[i]->m.E;
    }
    int best = 0;
    float best_ms = 0;
    bool best_fused = false;
    for (int block : kTileBlocks) {
      if (!has_block(law, flux, dim, order, precision, block)) continue;
      set_tuned_block(law, flux, dim, order, precision, cells, block);
      dgp_ensemble e = nullptr;
      if (int rc = dgp_ensemble_create(static_cast<int>(ms.size()), ms.data(), ls.data(), os.data(), precision,
                                       limiter, &e))
        return rc;
      dgp_solver g = e->groups[0];
      int rc = DGP_OK;
      for (int f = 0; f < (g->fused_ok ? 2 : 1) && !rc; ++f) {
        if (g->fused_ok) rc = dgp_set_fused(g, f);
        float t = 0;
        if (!rc) rc = time_steps(g, iters, &t);
        if (!rc && (!best || t < best_ms)) {
          best = block;
          best_ms = t;
          best_fused = g->fused_ok && f == 1;
        }
      }
      dgp_ensemble_destroy(e);
      if (rc) return rc;
    }
    if (best) {
      set_tuned_block(law, flux, dim, order, precision, cells, best);
      set_tuned_fused(law, flux, dim, order, precision, cells, best_fused);
    }
  }
  return DGP_OK;
}

int dgp_tune_set(int law, int flux, int dim, int order, int precision, int cells, int block) {
  if (!has_block(law, flux, dim, order, precision, block))
    return fail(DGP_ERR_UNSUPPORTED, "no kernels with this tile shape for this configuration");
  set_tuned_block(law, flux, dim, order, precision, cells, block);
  return DGP_OK;
}

int dgp_solver_block(dgp_solver s, int* block, int* cells_per_tile) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (block) *block = s->ops.elem_block;
  if (cells_per_tile) *cells_per_tile = s->ops.TE;
  return DGP_OK;
}

int dgp_solver_fused(dgp_solver s, int* fused) {
  if (!s || !fused) return fail(DGP_ERR_INVALID, "null argument");
  *fused = s->fused ? 1 : 0;
  return DGP_OK;
}

int dgp_set_fused(dgp_solver s, int on) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (on && !s->fused_ok)
    return fail(DGP_ERR_UNSUPPORTED, "no fused stage kernel for this solver (a tile's halo does not fit)");
  if (on == (s->fused ? 1 : 0)) return DGP_OK;
  DGP_CUDA(cudaSetDevice(s->device));
  s->drop_graphs();
  if (!on) {
    // the face kernel reads the face-point traces, which fused stages do not keep
    s->ops.trace(s->b, nullptr, s->stream);
    DGP_CUDA(cudaGetLastError());
    s->tr_stale = false;
    s->b.tensor_cores = 0;
    s->b.round_mask = 0;
  }
  s->fused = on != 0;
  return DGP_OK;
}

int dgp_ensemble_group_block(dgp_ensemble e, int group, int* block, int* cells_per_tile) {
  if (!e || group < 0 || group >= static_cast<int>(e->groups.size())) return fail(DGP_ERR_INVALID, "bad group");
  return dgp_solver_block(e->groups[group], block, cells_per_tile);
}


// ---------------------------------------------------------------------------
// Discrete adjoint (no counterpart in DG-Parallel): gradient of an objective of
// the final state with respect to the initial coefficients, through the
// SSP-RK3 steps with a fixed time step, by checkpoint and recompute.

static int adj_buffer(dgp_solver s, double** p, size_t* have, size_t states) {
  if (*have >= states && *p) return DGP_OK;
  if (*p) {
    cudaFree(*p);
    s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), static_cast<void*>(*p)), s->allocs.end());
    *p = nullptr;
  }
  if (int rc = s->alloc(p, states * s->state_count() + 32)) return rc;
  *have = states;
  return DGP_OK;
}

// the Barth slope factors of `stages` stages ([stage][E][M] doubles)
static int adj_slopes(dgp_solver s, size_t stages) {
  AdjointState& a = s->adj;
  const size_t n = stages * static_cast<size_t>(s->b.E) * s->b.M;
  if (a.slopes && a.slopes_n >= n) return DGP_OK;
  if (a.slopes) {
    cudaFree(a.slopes);
    s->allocs.erase(std::remove(s->allocs.begin(), s->allocs.end(), static_cast<void*>(a.slopes)), s->allocs.end());
    a.slopes = nullptr;
  }
  if (int rc = s->alloc(&a.slopes, n)) return rc;
  a.slopes_n = n;
  return DGP_OK;
}

int dgp_adjoint_freeze_limiter(dgp_solver s, int on) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (on && s->limiter != DGP_LIMITER_BARTH) return fail(DGP_ERR_UNSUPPORTED, "no Barth limiter to freeze");
  s->adj.freeze = on != 0;
  return DGP_OK;
}

int dgp_adjoint_set_receivers(dgp_solver s, int n, const double* points, const double* observed) {
  if (!s || n <= 0 || !points || !observed) return fail(DGP_ERR_INVALID, "bad argument");
  if (s->b.ninst) return fail(DGP_ERR_UNSUPPORTED, "receivers are set on a single solver");
  DGP_CUDA(cudaSetDevice(s->device));
  std::vector<int> cell;
  std::vector<double> phi;
  if (int rc = locate_points(s, n, points, cell, phi)) return rc;
  for (int r = 0; r < n; ++r)
    if (cell[r] < 0) return fail(DGP_ERR_INVALID, "receiver " + std::to_string(r) + " lies outside the mesh");
  AdjointState& a = s->adj;
  std::vector<double> obs(observed, observed + n);
  int rc = DGP_OK;
  if ((rc = s->upload(&a.rcell, cell)) || (rc = s->upload(&a.rphi, phi)) || (rc = s->upload(&a.robs, obs)) ||
      (rc = s->alloc(&a.rrho, static_cast<size_t>(n))) || (rc = s->alloc(&a.rJ, 1)))
    return rc;
  a.nrec = n;
  return DGP_OK;
}

static Receivers receivers_of(dgp_solver s) {
  Receivers r;
  r.n = s->adj.nrec;
  r.cell = s->adj.rcell;
  r.phi = s->adj.rphi;
  r.obs = s->adj.robs;
  r.np = s->b.NP;
  r.mnp = s->b.M * s->b.NP;
  return r;
}

int dgp_receiver_values(dgp_solver s, double* rho, double* J) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (!s->adj.nrec) return fail(DGP_ERR_INVALID, "no receivers set");
  DGP_CUDA(cudaSetDevice(s->device));
  receiver_values_kernel<<<1, 256, 0, s->stream>>>(receivers_of(s), static_cast<const double*>(s->b.C),
                                                    s->adj.rrho, s->adj.rJ);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (rho) DGP_CUDA(cudaMemcpy(rho, s->adj.rrho, s->adj.nrec * 8, cudaMemcpyDeviceToHost));
  double j = 0;
  DGP_CUDA(cudaMemcpy(&j, s->adj.rJ, 8, cudaMemcpyDeviceToHost));
  if (J) *J = j;
  return DGP_OK;
}

// one SSP-RK3 step from X back into X, keeping u_n, u1, u2 in S (three
// consecutive states).  With the Barth limiter it follows every stage, its
// slope factors going to slopes[3][E][M] (replay: applied from there).
static void step_keeping_stages(dgp_solver s, double* X, double* S, size_t ns, double* slopes = nullptr,
                                bool replay = false) {
  const bool lim = s->limiter == DGP_LIMITER_BARTH && s->ops.limit;
  const size_t em = static_cast<size_t>(s->b.E) * s->b.M;
  auto limit = [&](double* u, int k) {
    if (!lim) return;
    DeviceBuffers bl = s->b;
    bl.C = u;
    bl.lim_slope = slopes ? slopes + static_cast<size_t>(k) * em : nullptr;
    bl.lim_replay = replay ? 1 : 0;
    s->ops.limit(bl, 0, s->stream);
  };
  if (s->fused) {
    s->ops.fused(s->b, X, X, S + ns, S, 1, 0.0, 0, s->stream);
    limit(S + ns, 0);
    s->ops.fused(s->b, S + ns, S, S + 2 * ns, nullptr, 2, 1.0, 0, s->stream);
    limit(S + 2 * ns, 1);
    s->ops.fused(s->b, S + 2 * ns, S, X, nullptr, 3, 0.5, 0, s->stream);
    limit(X, 2);
    s->tr_stale = true;
    return;
  }
  // the separate kernels read the face-point traces of each stage's input
  auto traces = [&](double* u) {
    if (!replay) return;  // the limiter pass refreshed the traces of the cells it changed
    DeviceBuffers bt = s->b;
    bt.C = u;
    s->ops.trace(bt, nullptr, s->stream);
  };
  DeviceBuffers b = s->b;
  b.U0 = S;
  b.C = X;
  b.Cout = S + ns;
  s->ops.stage(b, 1, 0.0, 0, s->stream);
  limit(S + ns, 0);
  if (lim) traces(S + ns);
  b.C = S + ns;
  b.Cout = S + 2 * ns;
  s->ops.stage(b, 2, 1.0, 0, s->stream);
  limit(S + 2 * ns, 1);
  if (lim) traces(S + 2 * ns);
  b.C = S + 2 * ns;
  b.Cout = X;
  s->ops.stage(b, 3, 0.5, 0, s->stream);
  limit(X, 2);
  if (lim) traces(X);
}

int dgp_forward_checkpointed(dgp_solver s, double t0, double dt, int nsteps, int every, double* J) {
  if (s && s->lts.on) return fail(DGP_ERR_UNSUPPORTED, "the discrete adjoint follows SSP-RK3, not local time stepping");
  if (!s || !(dt > 0) || nsteps <= 0 || every < 0) return fail(DGP_ERR_INVALID, "bad argument");
  if (s->b.ninst) return fail(DGP_ERR_UNSUPPORTED, "the adjoint runs on a single solver");
  if (!s->ops.adj_stage) return fail(DGP_ERR_UNSUPPORTED, "no discrete adjoint for this law/flux");
  if (s->limiter == DGP_LIMITER_MOMENT)
    return fail(DGP_ERR_UNSUPPORTED, "the adjoint's frozen limiter is built for the Barth limiter");
  for (const HostMesh& hm : s->meshes)
    for (int pf : hm.pface)
      if (pf >= 0) return fail(DGP_ERR_UNSUPPORTED, "adjoint on a mesh with periodic edges");
  DGP_CUDA(cudaSetDevice(s->device));
  AdjointState& a = s->adj;
  // every == 0: one segment whose stage states are all kept (no recompute)
  const bool record = every == 0;
  const bool lim = s->limiter == DGP_LIMITER_BARTH;
  if (a.freeze && !(record && lim && a.slopes && a.slopes_n >= static_cast<size_t>(3) * nsteps * s->b.E * s->b.M))
    return fail(DGP_ERR_INVALID, "a frozen limiter replays the factors of a recorded pass (every = 0) of as many steps");
  if (record) every = nsteps;
  const int nseg = (nsteps + every - 1) / every;
  if (int rc = adj_buffer(s, &a.ckpt, &a.ckpt_states, static_cast<size_t>(nseg) + 1)) return rc;
  if (record)
    if (int rc = adj_buffer(s, &a.store, &a.store_states, static_cast<size_t>(3) * nsteps)) return rc;
  if (record && lim && !a.freeze)
    if (int rc = adj_slopes(s, static_cast<size_t>(3) * nsteps)) return rc;
  a.recorded = record;
  if (!a.t_seg && (s->alloc(&a.t_seg, 1) != DGP_OK)) return DGP_ERR_NOMEM;
  a.nsteps = nsteps;
  a.every = every;
  a.nseg = nseg;
  a.t0 = t0;
  a.dt = dt;
  const size_t ns = s->state_count(), bytes = ns * 8;
  const size_t em = static_cast<size_t>(s->b.E) * s->b.M;
  const int p0 = s->b.p0;
  s->b.p0 = 0;  // the adjoint differentiates the plain operator
  for (int seg = 0; seg < nseg; ++seg) {
    DGP_CUDA(cudaMemcpyAsync(a.ckpt + static_cast<size_t>(seg) * ns, s->b.C, bytes, cudaMemcpyDeviceToDevice,
                             s->stream));
    const int len = std::min(every, nsteps - seg * every);
    double* X = static_cast<double*>(s->b.C);
    for (int k = 0; k < len; ++k) {
      const double tk = t0 + static_cast<double>(seg * every + k) * dt;
      set_segment_time<<<1, 1, 0, s->stream>>>(s->b.ctl, tk, dt, a.t_seg);
      if (record)
        step_keeping_stages(s, X, a.store + static_cast<size_t>(k) * 3 * ns, ns,
                            lim ? a.slopes + static_cast<size_t>(k) * 3 * em : nullptr, a.freeze);
      else
        launch_step(s, 0);
    }
  }
  DGP_CUDA(cudaMemcpyAsync(a.ckpt + static_cast<size_t>(nseg) * ns, s->b.C, bytes, cudaMemcpyDeviceToDevice,
                           s->stream));
  s->b.p0 = p0;
  DGP_CUDA(cudaGetLastError());
  a.ready = true;
  if (a.nrec) return dgp_receiver_values(s, nullptr, J);
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (J) *J = 0.0;
  return DGP_OK;
}

int dgp_backward(dgp_solver s, const double* dJ_duT, double* dJ_du0) {
  if (!s || !dJ_du0) return fail(DGP_ERR_INVALID, "null argument");
  AdjointState& a = s->adj;
  if (!a.ready) return fail(DGP_ERR_INVALID, "run dgp_forward_checkpointed first");
  if (!dJ_duT && !a.nrec) return fail(DGP_ERR_INVALID, "no seed and no receivers");
  DGP_CUDA(cudaSetDevice(s->device));
  const size_t ns = s->state_count(), bytes = ns * 8;
  if (int rc = adj_buffer(s, &a.store, &a.store_states, static_cast<size_t>(3) * a.every)) return rc;
  const bool lim = s->limiter == DGP_LIMITER_BARTH;
  const size_t em = static_cast<size_t>(s->b.E) * s->b.M;
  if (lim && !a.recorded)
    if (int rc = adj_slopes(s, static_cast<size_t>(3) * a.every)) return rc;
  // the frozen limiter of stage k of step j: its recorded linear map (diagonal
  // in the modes) applied to the cotangent of the stage's limited output
  auto frozen = [&](double* mu, int j, int k) {
    if (!lim) return;
    DeviceBuffers bl = s->b;
    bl.C = mu;
    bl.tr = nullptr;
    bl.trig = nullptr;
    bl.lim_slope = a.slopes + (static_cast<size_t>(j) * 3 + k) * em;
    bl.lim_replay = 1;
    s->ops.limit(bl, 0, s->stream);
  };
  if (!a.lam) {
    size_t one = 0;
    if (int rc = adj_buffer(s, &a.lam, &one, 1)) return rc;
    one = 0;
    if (int rc = adj_buffer(s, &a.lam2, &one, 1)) return rc;
    one = 0;
    if (int rc = adj_buffer(s, &a.lam1, &one, 1)) return rc;
    one = 0;
    if (int rc = adj_buffer(s, &a.acc, &one, 1)) return rc;
  }
  // seed: dJ/du_T
  if (dJ_duT) {
    if (int rc = host_to_state(s, dJ_duT, a.lam)) return rc;
  } else {
    DGP_CUDA(cudaMemsetAsync(a.lam, 0, bytes, s->stream));
    const double* uT = a.ckpt + static_cast<size_t>(a.nseg) * ns;
    receiver_values_kernel<<<1, 256, 0, s->stream>>>(receivers_of(s), uT, a.rrho, a.rJ);
    receiver_seed_kernel<<<1, 32, 0, s->stream>>>(receivers_of(s), a.rrho, a.lam);
  }
  const int p0 = s->b.p0;
  s->b.p0 = 0;
  double* X = static_cast<double*>(s->b.C);
  for (int seg = a.nseg - 1; seg >= 0; --seg) {
    const int len = std::min(a.every, a.nsteps - seg * a.every);
    auto step_time = [&](int j) { return a.t0 + static_cast<double>(seg * a.every + j) * a.dt; };
    if (!a.recorded) {
      // recompute the segment from its checkpoint, keeping every stage state
      DGP_CUDA(cudaMemcpyAsync(X, a.ckpt + static_cast<size_t>(seg) * ns, bytes, cudaMemcpyDeviceToDevice,
                               s->stream));
      s->ops.trace(s->b, nullptr, s->stream);
      for (int j = 0; j < len; ++j) {
        set_segment_time<<<1, 1, 0, s->stream>>>(s->b.ctl, step_time(j), a.dt, a.t_seg);
        step_keeping_stages(s, X, a.store + static_cast<size_t>(j) * 3 * ns, ns,
                            lim ? a.slopes + static_cast<size_t>(j) * 3 * em : nullptr);
      }
    }
    // reversed steps
    for (int j = len - 1; j >= 0; --j) {
      set_segment_time<<<1, 1, 0, s->stream>>>(s->b.ctl, step_time(j), a.dt, a.t_seg);
      DeviceBuffers b = s->b;
      AdjStage g{};
      g.dt = a.dt;
      g.t_seg = a.t_seg;
      // u3 = (2 (u2 + dt L(u2)) + u) / 3
      b.C = a.store + (static_cast<size_t>(j) * 3 + 2) * ns;
      frozen(a.lam, j, 2);
      g.mu = a.lam;
      g.out = a.lam2;
      g.acc = a.acc;
      g.ca = 2.0 / 3.0;
      g.cb = 2.0 / 3.0;
      g.cc = 0.0;
      g.cd = 0.0;
      g.ce = 1.0 / 3.0;
      g.t_factor = 0.5;
      s->ops.adj_stage(b, g, s->stream);
      // u2 = (u1 + dt L(u1) + 3 u) / 4
      b.C = a.store + (static_cast<size_t>(j) * 3 + 1) * ns;
      frozen(a.lam2, j, 1);
      g.mu = a.lam2;
      g.out = a.lam1;
      g.ca = 0.25;
      g.cb = 0.25;
      g.cc = 0.0;
      g.cd = 1.0;
      g.ce = 0.75;
      g.t_factor = 1.0;
      s->ops.adj_stage(b, g, s->stream);
      // u1 = u + dt L(u)
      b.C = a.store + (static_cast<size_t>(j) * 3 + 0) * ns;
      frozen(a.lam1, j, 0);
      g.mu = a.lam1;
      g.out = a.lam;
      g.ca = 1.0;
      g.cb = 1.0;
      g.cc = 1.0;
      g.cd = 0.0;
      g.ce = 0.0;
      g.t_factor = 0.0;
      s->ops.adj_stage(b, g, s->stream);
    }
  }
  s->b.p0 = p0;
  // the forward state is left at u_T
  DGP_CUDA(cudaMemcpyAsync(X, a.ckpt + static_cast<size_t>(a.nseg) * ns, bytes, cudaMemcpyDeviceToDevice,
                           s->stream));
  s->ops.trace(s->b, nullptr, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return state_to_host(s, a.lam, dJ_du0);
}

}  // extern "C"
