// C ABI of libdgp.so (include/dgp.h): handles, host preprocessing, device
// buffers in the internal (Morton) cell order, and the device-resident time
// loop captured in CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_host.h"
#include "dgp_handles.h"
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
  });
}

// gather cells by `perm` and convert the arithmetic type
template <typename Tin, typename Tout>
__global__ void gather_cells(const Tin* in, Tout* out, const int* perm, int E, int mnp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)E * mnp) return;
  const int e = static_cast<int>(i / mnp), r = static_cast<int>(i - (long long)e * mnp);
  out[i] = static_cast<Tout>(in[(size_t)perm[e] * mnp + r]);
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
// derivative transforms and the bounding-box centres, degree tables.
static int setup_limiter(dgp_solver s) {
  const HostMesh& m = s->mesh;
  const int E = m.E;
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
  std::vector<int> nb(4 * (size_t)E, -1);
  std::vector<double> geo(static_cast<size_t>(E) * kLimGeo);
  for (int i = 0; i < E; ++i) {
    const int e = s->i2f[i];
    const double px = bbc[2 * e], py = bbc[2 * e + 1];
    int* n = &nb[4 * (size_t)i];
    for (int lf = 0; lf < 3; ++lf) {
      const int f = cf[3 * (size_t)e + lf];
      if (f < 0 || m.eR[f] < 0) continue;
      const int o = (m.eL[f] == e) ? m.eR[f] : m.eL[f];
      const int oi = s->f2i[o];
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
  std::vector<double> D, Dinv;
  build_limiter_tables(s->tab, D, Dinv);
  DeviceBuffers& b = s->b;
  int rc = DGP_OK;
  if ((rc = s->upload(&b.nb, nb)) || (rc = s->upload(&b.lgeo, geo)) || (rc = s->upload(&b.limD, D)) ||
      (rc = s->upload(&b.limDinv, Dinv)) || (rc = s->alloc(&b.trig, static_cast<size_t>(E))) ||
      (rc = s->alloc(&b.L, s->state_count())))
    return rc;
  DGP_CUDA(cudaMemset(b.trig, 0, E));
  return DGP_OK;
}

extern "C" {

const char* dgp_last_error(void) { return g_err.c_str(); }
int dgp_version(void) { return 1; }

int dgp_mesh_from_msh(const char* path, dgp_mesh* out) {
  if (!path || !out) return fail(DGP_ERR_INVALID, "null argument");
  auto* h = new dgp_mesh_s;
  std::string err;
  int rc = read_msh_v1(path, h->m, err);
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
  if (!out) return fail(DGP_ERR_INVALID, "null output handle");
  auto* h = new dgp_mesh_s;
  std::string err;
  int rc = mesh_from_arrays(dim, nv, xyz, vertex_ids, ncells, cells, cell_tag, nbfaces, bfaces, btags,
                            h->m, err);
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
  if (kind < DGP_LAW_SCALAR || kind > DGP_LAW_MAXWELL3D) return fail(DGP_ERR_INVALID, "unknown law");
  if (flux < DGP_FLUX_UPWIND || flux > DGP_FLUX_LLF) return fail(DGP_ERR_INVALID, "unknown flux");
  if (field < DGP_FIELD_GAUSS || field > DGP_FIELD_TM110) return fail(DGP_ERR_INVALID, "unknown field");
  auto* l = new dgp_law_s;
  l->kind = kind;
  l->flux = flux;
  l->field = field;
  for (int i = 0; i < DGP_NPARAMS; ++i) l->p[i] = params ? params[i] : 0.0;
  if (!(l->p[7] > 0.0)) l->p[7] = 1.4;  // gamma default (EulerLaw.h:14)
  *out = l;
  return DGP_OK;
}

int dgp_law_destroy(dgp_law l) {
  delete l;
  return DGP_OK;
}

int dgp_solver_create(dgp_mesh mh, dgp_law law, int order, int precision, int limiter,
                      dgp_solver* out) {
  if (!mh || !law || !out) return fail(DGP_ERR_INVALID, "null argument");
  if (precision != DGP_PRECISION_FP64 && precision != DGP_PRECISION_MIXED)
    return fail(DGP_ERR_INVALID, "unknown precision");
  if (limiter != DGP_LIMITER_NONE && limiter != DGP_LIMITER_MOMENT) return fail(DGP_ERR_INVALID, "unknown limiter");
  const HostMesh& m = mh->m;
  if (limiter == DGP_LIMITER_MOMENT && m.dim != 2)
    return fail(DGP_ERR_UNSUPPORTED, "the moment limiter is built for triangles only");
  if ((law->kind == DGP_LAW_EULER2D || law->kind == DGP_LAW_BURGERS2D) && m.dim != 2)
    return fail(DGP_ERR_UNSUPPORTED, "2D law on a 3D mesh");
  if ((law->kind == DGP_LAW_EULER3D || law->kind == DGP_LAW_MAXWELL3D) && m.dim != 3)
    return fail(DGP_ERR_UNSUPPORTED, "3D law on a 2D mesh");
  ensure_registry();
  auto it = ops_registry().find(OpsKey(law->kind, law->flux, m.dim, order, precision));
  if (it == ops_registry().end())
    return fail(DGP_ERR_UNSUPPORTED, "no kernels for this law/flux/element/order/precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(DGP_ERR_CUDA, "no CUDA device available");

  auto s = new dgp_solver_s;
  auto bail = [&](int rc) {
    delete s;
    return rc;
  };
  s->mesh = m;
  s->ops = it->second;
  s->law = law->kind;
  s->flux = law->flux;
  s->order = order;
  s->precision = precision;
  s->limiter = limiter;
  cudaGetDevice(&s->device);
  std::string err;
  if (int rc = build_tables(m.dim, order, s->tab, err)) return bail(fail(rc, err));
  const RefTables& t = s->tab;
  if (t.nq != s->ops.NQ || t.nqf != s->ops.NQF || t.Np != s->ops.NP)
    return bail(fail(DGP_ERR_UNSUPPORTED, "table/kernel shape mismatch"));
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(DGP_ERR_CUDA, "stream creation failed"));
  if (cudaMallocHost(&s->h_ctl, 2 * sizeof(TimeCtl)) != cudaSuccess)
    return bail(fail(DGP_ERR_CUDA, "pinned allocation failed"));

  const int dim = m.dim, E = m.E, nvc = m.nvc;
  DeviceBuffers& b = s->b;
  b.E = E;
  b.dim = dim;
  b.order = order;
  b.M = s->ops.M;
  b.NP = s->ops.NP;

  // internal order: Morton code of the cell centroids (locality of neighbours)
  {
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
    s->i2f.resize(E);
    std::iota(s->i2f.begin(), s->i2f.end(), 0);
    std::stable_sort(s->i2f.begin(), s->i2f.end(), [&](int a, int c) { return key[a] < key[c]; });
    s->f2i.resize(E);
    for (int i = 0; i < E; ++i) s->f2i[s->i2f[i]] = i;
  }

  // cell geometry (FP64 on the host)
  std::vector<double> jinv(static_cast<size_t>(E) * dim * dim), detj(E), csize(E), x0(3 * (size_t)E),
      jac(9 * (size_t)E);
  for (int i = 0; i < E; ++i) {
    const int e = s->i2f[i];
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
  // faces sorted by internal left cell
  std::vector<int> forder(m.F);
  std::iota(forder.begin(), forder.end(), 0);
  std::stable_sort(forder.begin(), forder.end(), [&](int a, int c) {
    int ia = s->f2i[m.eL[a]], ic = s->f2i[m.eL[c]];
    return ia != ic ? ia < ic : m.lfL[a] < m.lfL[c];
  });
  std::vector<int> fel(2 * (size_t)m.F), fcode(m.F), bbid;
  std::vector<double> fnrm(static_cast<size_t>(m.F) * dim), fj(m.F), bpts;
  int nb = 0;
  for (int k = 0; k < m.F; ++k) {
    const int f = forder[k];
    fel[2 * k] = s->f2i[m.eL[f]];
    if (m.eR[f] >= 0) {
      fel[2 * k + 1] = s->f2i[m.eR[f]];
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
      ++nb;
    }
    fcode[k] = m.lfL[f] | ((m.eR[f] >= 0 ? m.lfR[f] : 0) << 4) | (m.rperm[f] << 8);
    for (int c = 0; c < dim; ++c) fnrm[static_cast<size_t>(k) * dim + c] = m.fn[3 * f + c];
    fj[k] = dim == 2 ? 0.5 * m.fmeas[f] : 2.0 * m.fmeas[f];  // |J_f| of the face map
  }
  b.F = m.F;
  b.NB = nb;

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
      (rc = s->upload_t(&b.phi, t.phi)) || (rc = s->upload_t(&b.dphi, t.dphi)) ||
      (rc = s->upload_t(&b.qw, t.qw)) || (rc = s->upload_t(&b.phif, t.phif)) ||
      (rc = s->upload_t(&b.fqw, t.fqw)) || (rc = s->upload(&b.qmap, t.qmap)) ||
      (rc = s->upload(&b.phiv, t.phiv)) || (rc = s->upload(&b.phiq, t.phi)) ||
      (rc = s->upload(&b.qwd, t.qw)) || (rc = s->upload(&b.qpd, qpd)) ||
      (rc = s->upload(&b.eqp, t.eqp)) || (rc = s->upload(&b.eqw, t.eqw)) ||
      (rc = s->upload(&b.ephi, t.ephi)) || (rc = s->upload(&s->d_i2f, s->i2f)) ||
      (rc = s->upload(&s->d_f2i, s->f2i)))
    return bail(rc);
  {
    std::vector<double> blob(s->ops.blob_elems);
    s->ops.fill_blob(t.dphi.data(), t.phif.data(), t.phi.data(), t.qw.data(), blob.data());
    if ((rc = s->upload_t(&b.blob, blob))) return bail(rc);
    b.blob_bytes = static_cast<int>(s->ops.blob_elems * s->ops.tsize);
  }
  b.nqe = t.nqe;
  b.phi0 = t.phi0;
  b.law.field = law->field;
  for (int i = 0; i < DGP_NPARAMS; ++i) b.law.p[i] = law->p[i];

  const size_t nstate = s->state_count();
  // slots are tile-transposed over whole tiles of TE cells; state buffers get
  // 256 bytes of tail so the bulk copy of the last tile may round up to 16 bytes
  const size_t ntiles = (static_cast<size_t>(E) + s->ops.TE - 1) / s->ops.TE;
  const size_t nslot = ntiles * s->ops.TE * t.nlf * t.nqf * b.M;
  unsigned char *C, *U0, *slots, *rhs, *scratch;
  const size_t ts = s->ops.tsize;  // slots hold the RHS arithmetic type; the state is FP64
  if ((rc = s->alloc(&C, nstate * 8 + 256)) || (rc = s->alloc(&U0, nstate * 8 + 256)) ||
      (rc = s->alloc(&slots, nslot * ts)) || (rc = s->alloc(&rhs, nstate * 8 + 256)) ||
      (rc = s->alloc(&scratch, nstate * 8 + 256)))
    return bail(rc);
  b.C = C;
  b.U0 = U0;
  b.slots = slots;
  b.rhs = rhs;
  b.scratch = scratch;
  b.npartials = std::max(s->ops.grid_elem(E), (E + 255) / 256) * std::max(b.M, 1) + 1;
  if ((rc = s->alloc(&b.partials, b.npartials)) || (rc = s->alloc(&b.ctl, 1)) ||
      (rc = s->alloc(&b.status, 1)))
    return bail(rc);
  DGP_CUDA(cudaMemset(slots, 0, nslot * ts));
  // P0 fallback marks (DGCell::setToZero), on by default for the Euler laws
  // whose isPhysical can fail
  if ((rc = s->alloc(&b.bad, static_cast<size_t>(E)))) return bail(rc);
  DGP_CUDA(cudaMemset(b.bad, 0, E));
  b.p0 = (law->kind == DGP_LAW_EULER2D || law->kind == DGP_LAW_EULER3D) ? 1 : 0;
  if (limiter == DGP_LIMITER_MOMENT && order >= 1) {
    if ((rc = setup_limiter(s))) return bail(rc);
  }
  TimeCtl c0{};
  c0.dtmin_bits = 0x7FF0000000000000ull;
  DGP_CUDA(cudaMemcpy(b.ctl, &c0, sizeof(TimeCtl), cudaMemcpyHostToDevice));
  Status st0{0, INT32_MAX};
  DGP_CUDA(cudaMemcpy(b.status, &st0, sizeof(Status), cudaMemcpyHostToDevice));
  if (cudaError_t e = s->ops.prepare()) return bail(fail(DGP_ERR_CUDA, cudaGetErrorString(e)));
  // DGAnalysis::DGAnalysis projects the far field as the initial state
  s->ops.project(b, 0.0, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
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
  if (s->limiter == DGP_LIMITER_MOMENT && s->ops.limit) s->ops.limit(s->b, 0, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

// host FP64 [cell][field][mode] in file order <-> device state in internal order
static int host_to_state(dgp_solver s, const double* in, void* dst) {
  const size_t mnp = static_cast<size_t>(s->b.M) * s->b.NP, n = s->state_count();
  std::vector<double> tmp(n);
  for (int i = 0; i < s->b.E; ++i)
    std::memcpy(&tmp[i * mnp], &in[static_cast<size_t>(s->i2f[i]) * mnp], mnp * 8);
  DGP_CUDA(cudaMemcpy(dst, tmp.data(), n * 8, cudaMemcpyHostToDevice));
  return DGP_OK;
}

static int state_to_host(dgp_solver s, const void* src, double* out) {
  const size_t mnp = static_cast<size_t>(s->b.M) * s->b.NP, n = s->state_count();
  std::vector<double> tmp(n);
  DGP_CUDA(cudaMemcpy(tmp.data(), src, n * 8, cudaMemcpyDeviceToHost));
  for (int i = 0; i < s->b.E; ++i)
    std::memcpy(&out[static_cast<size_t>(s->i2f[i]) * mnp], &tmp[i * mnp], mnp * 8);
  return DGP_OK;
}

int dgp_set_state(dgp_solver s, const double* host_state) {
  if (!s || !host_state) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return host_to_state(s, host_state, s->b.C);
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
  s->ops.stage(s->b, 0, 0.0, 0, s->stream);
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
  const bool lim = s->limiter == DGP_LIMITER_MOMENT && s->ops.limit;
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

int dgp_launches_per_step(dgp_solver s, int* n) {
  if (!s || !n) return fail(DGP_ERR_INVALID, "null argument");
  const bool lim = s->limiter == DGP_LIMITER_MOMENT && s->ops.limit;
  *n = 3 * (s->b.p0 ? 3 : 2) + (lim ? 3 * 2 + 1 : 0);
  return DGP_OK;
}

int dgp_step(dgp_solver s, double t, double dt, double* resid) {
  if (!s || !(dt > 0)) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  if (int rc = set_ctl(s, t, dt, 0.0, 0.0, 0)) return rc;
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
  if (!s->graph) {
    // K steps per graph; finished steps turn the remaining kernels into no-ops
    const int K = 8;
    cudaGraph_t g;
    DGP_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K; ++k) launch_step(s, 1);
    DGP_CUDA(cudaStreamEndCapture(s->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(DGP_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
    s->graph_steps = K;
  }
  if (int rc = set_ctl(s, t0, 0.0, tend, cfl, max_steps)) return rc;
  s->ops.cfl(s->b, s->stream);
  DGP_CUDA(cudaGetLastError());
  TimeCtl c;
  for (long long guard = 0;; ++guard) {
    DGP_CUDA(cudaGraphLaunch(s->graph, s->stream));
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
  if (s->limiter != DGP_LIMITER_MOMENT) return fail(DGP_ERR_INVALID, "solver created without a limiter");
  DGP_CUDA(cudaSetDevice(s->device));
  if (s->ops.limit) s->ops.limit(s->b, 0, s->stream);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return triggers ? dgp_limiter_triggers(s, triggers) : DGP_OK;
}

int dgp_limiter_triggers(dgp_solver s, unsigned char* out) {
  if (!s || !out) return fail(DGP_ERR_INVALID, "null argument");
  if (s->limiter != DGP_LIMITER_MOMENT) return fail(DGP_ERR_INVALID, "solver created without a limiter");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  const int E = s->b.E;
  if (!s->b.trig) {  // P0: nothing is ever limited
    std::memset(out, 0, E);
    return DGP_OK;
  }
  std::vector<unsigned char> t(E);
  DGP_CUDA(cudaMemcpy(t.data(), s->b.trig, E, cudaMemcpyDeviceToHost));
  for (int i = 0; i < E; ++i) out[s->i2f[i]] = t[i];
  return DGP_OK;
}

int dgp_set_p0_fallback(dgp_solver s, int on) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  s->b.p0 = on ? 1 : 0;
  return DGP_OK;
}

int dgp_status(dgp_solver s, int* nonphysical, int* first_bad_cell) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  DGP_CUDA(cudaSetDevice(s->device));
  Status st;
  DGP_CUDA(cudaMemcpyAsync(&st, s->b.status, sizeof(Status), cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (st.timeouts > 0)
    return fail(DGP_ERR_CUDA, "a bounded wait on a bulk copy gave up in " + std::to_string(st.timeouts) +
                                  " CTA(s); results of that launch are incomplete");
  if (nonphysical) *nonphysical = st.nonphysical;
  if (first_bad_cell) *first_bad_cell = st.nonphysical ? s->i2f[std::min(st.first_bad, s->b.E - 1)] : -1;
  Status st0{0, INT32_MAX};
  DGP_CUDA(cudaMemcpy(s->b.status, &st0, sizeof(Status), cudaMemcpyHostToDevice));
  return DGP_OK;
}

int dgp_l2_error(dgp_solver s, double t, int field, double* err) {
  if (!s || !err || field < 0 || field >= s->b.M) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  s->ops.l2err(s->b, t, field, s->stream);
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

int dgp_totals(dgp_solver s, double* totals) {
  if (!s || !totals) return fail(DGP_ERR_INVALID, "bad argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const double refm = s->b.dim == 2 ? 0.5 : 1.0 / 6.0;
  s->ops.totals(s->b, refm, s->stream);
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

}  // extern "C"
