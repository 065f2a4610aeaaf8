// Host-side preprocessing of the dgp solver (FP64): Gmsh v1 import, the face
// table with DG-Parallel's left/right convention, geometry and the
// reference-element tables.
#include "dgp_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "../../include/dgp.h"
#include "quadrature_rules.h"

namespace dgp {

uint32_t glibc_rand_first(uint32_t seed) {
  // TYPE_3 state of 31 words seeded by the Park-Miller LCG (16807 mod 2^31-1,
  // Schrage form), r[i] = r[i-31] + r[i-3] mod 2^32, first output r[344] >> 1.
  int32_t r[345];
  r[0] = static_cast<int32_t>(seed ? seed : 1);
  for (int i = 1; i < 31; ++i) {
    int64_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
    int64_t w = 16807 * lo - 2836 * hi;
    if (w < 0) w += 2147483647;
    r[i] = static_cast<int32_t>(w);
  }
  for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
  for (int i = 34; i < 345; ++i)
    r[i] = static_cast<int32_t>(static_cast<uint32_t>(r[i - 31]) + static_cast<uint32_t>(r[i - 3]));
  return static_cast<uint32_t>(r[344]) >> 1;
}

namespace {

const int kTriFace[3][2] = {{0, 1}, {1, 2}, {2, 0}};
const int kTetFace[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
// the 6 permutations of a triangle's vertices; entry p lists, for the right
// cell's local vertices 0,1,2, their position in the face frame
const int kPerm3[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

struct FaceKey {
  int v[3];
  int cell, lf;
  bool operator<(const FaceKey& o) const {
    if (v[0] != o.v[0]) return v[0] < o.v[0];
    if (v[1] != o.v[1]) return v[1] < o.v[1];
    return v[2] < o.v[2];
  }
  bool same(const FaceKey& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};

void sort_small(int* a, int n) {
  for (int i = 1; i < n; ++i)
    for (int j = i; j > 0 && a[j - 1] > a[j]; --j) std::swap(a[j - 1], a[j]);
}

// mEntity::lessthan (mEntity.cc:173-200): compare the int-truncated sum of
// rand(vertex id), then the sorted vertex ids.
struct CellOrder {
  const HostMesh& m;
  const std::vector<uint32_t>& rk;
  int32_t key(int e) const {
    uint64_t s = 0;
    for (int k = 0; k < m.nvc; ++k) s += rk[m.cv[e * m.nvc + k]];
    return static_cast<int32_t>(static_cast<uint32_t>(s));
  }
  bool less(int a, int b) const {
    int32_t ka = key(a), kb = key(b);
    if (ka != kb) return ka < kb;
    int va[4], vb[4];
    for (int k = 0; k < m.nvc; ++k) {
      va[k] = m.vid[m.cv[a * m.nvc + k]];
      vb[k] = m.vid[m.cv[b * m.nvc + k]];
    }
    sort_small(va, m.nvc);
    sort_small(vb, m.nvc);
    for (int k = 0; k < m.nvc; ++k)
      if (va[k] != vb[k]) return va[k] < vb[k];
    return false;
  }
};

int local_vertex(const HostMesh& m, int lf, int k) {
  return m.dim == 2 ? kTriFace[lf][k] : kTetFace[lf][k];
}

// classification of every face: a boundary face takes the tag of the boundary
// element with its vertices, any other face the cells' tag
void boundary_ids(HostMesh& m, const std::vector<FaceKey>& sorted_bkeys) {
  m.bid.assign(m.F, m.ctag);
  for (int f = 0; f < m.F; ++f) {
    if (m.eR[f] >= 0) continue;
    FaceKey k{{INT32_MAX, INT32_MAX, INT32_MAX}, 0, 0};
    for (int j = 0; j < m.nfv; ++j) k.v[j] = m.vid[m.fv[static_cast<size_t>(f) * m.nfv + j]];
    sort_small(k.v, m.nfv);
    auto it = std::lower_bound(sorted_bkeys.begin(), sorted_bkeys.end(), k);
    if (it != sorted_bkeys.end() && it->same(k)) m.bid[f] = it->cell;
  }
}

void periodic_pairs(HostMesh& m) {
  // periodic pairs (mMesh::setPeriodicBC, mMesh.cc:457-524): a boundary edge
  // tagged 510 pairs with the first other 510 edge whose two vertices have the
  // same y coordinates (within 1e-10, either order), 610 likewise with x
  m.pface.assign(m.F, -1);
  if (m.dim == 2) {
    const double SN = 1.0e-10;
    for (int f = 0; f < m.F; ++f) {
      const int id = m.bid[f];
      if (m.eR[f] >= 0 || (id != 510 && id != 610)) continue;
      const int c = (id == 510) ? 1 : 0;
      const double* v1 = &m.X[3 * m.fv[2 * f]];
      const double* v2 = &m.X[3 * m.fv[2 * f + 1]];
      for (int g = 0; g < m.F; ++g) {
        if (g == f || m.eR[g] >= 0 || m.bid[g] != id) continue;
        const double* a1 = &m.X[3 * m.fv[2 * g]];
        const double* a2 = &m.X[3 * m.fv[2 * g + 1]];
        if ((std::fabs(v1[c] - a1[c]) < SN && std::fabs(v2[c] - a2[c]) < SN) ||
            (std::fabs(v1[c] - a2[c]) < SN && std::fabs(v2[c] - a1[c]) < SN)) {
          m.pface[f] = g;
          break;
        }
      }
    }
  }
}

int build_faces(HostMesh& m, const std::vector<FaceKey>& bkeys_in, std::string& err) {
  std::vector<FaceKey> bkeys = bkeys_in;
  std::sort(bkeys.begin(), bkeys.end());
  std::vector<FaceKey> keys(static_cast<size_t>(m.E) * m.nlf);
  for (int e = 0; e < m.E; ++e)
    for (int lf = 0; lf < m.nlf; ++lf) {
      FaceKey k{{INT32_MAX, INT32_MAX, INT32_MAX}, e, lf};
      for (int j = 0; j < m.nfv; ++j) k.v[j] = m.vid[m.cv[e * m.nvc + local_vertex(m, lf, j)]];
      sort_small(k.v, m.nfv);
      keys[static_cast<size_t>(e) * m.nlf + lf] = k;
    }
  std::sort(keys.begin(), keys.end());
  std::vector<uint32_t> rk(m.vid.size());
  for (size_t i = 0; i < m.vid.size(); ++i) rk[i] = glibc_rand_first(static_cast<uint32_t>(m.vid[i]));
  CellOrder order{m, rk};
  m.F = 0;
  m.fv.clear(); m.eL.clear(); m.eR.clear(); m.lfL.clear(); m.lfR.clear(); m.bid.clear();
  m.rperm.clear();
  for (size_t i = 0; i < keys.size();) {
    size_t j = i + 1;
    while (j < keys.size() && keys[i].same(keys[j])) ++j;
    if (j - i > 2) {
      err = "non-manifold face shared by more than two cells";
      return DGP_ERR_IO;
    }
    int a = keys[i].cell, la = keys[i].lf, b = -1, lb = -1;
    if (j - i == 2) {
      b = keys[i + 1].cell;
      lb = keys[i + 1].lf;
      if (order.less(b, a)) {
        std::swap(a, b);
        std::swap(la, lb);
      }
    }
    int frame[3];
    for (int k = 0; k < m.nfv; ++k) frame[k] = m.cv[a * m.nvc + local_vertex(m, la, k)];
    int perm = 0;
    if (b >= 0) {
      int rv[3];
      for (int k = 0; k < m.nfv; ++k) rv[k] = m.cv[b * m.nvc + local_vertex(m, lb, k)];
      if (m.dim == 2) {
        perm = (rv[0] == frame[0]) ? 0 : 1;
      } else {
        int pos[3];
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l)
            if (rv[k] == frame[l]) pos[k] = l;
        perm = -1;
        for (int p = 0; p < 6; ++p)
          if (kPerm3[p][0] == pos[0] && kPerm3[p][1] == pos[1] && kPerm3[p][2] == pos[2]) perm = p;
        if (perm < 0) {
          err = "inconsistent face vertices";
          return DGP_ERR_IO;
        }
      }
    }
    for (int k = 0; k < m.nfv; ++k) m.fv.push_back(frame[k]);
    m.eL.push_back(a);
    m.eR.push_back(b);
    m.lfL.push_back(la);
    m.lfR.push_back(lb);
    m.rperm.push_back(perm);
    m.F++;
    i = j;
  }
  // normals and measures (Mapping::normalVector, Mapping.cc:660-685: outward
  // from the left cell; DGBoundaryCell::computeSize)
  m.fn.assign(static_cast<size_t>(m.F) * 3, 0.0);
  m.fmeas.assign(m.F, 0.0);
  for (int f = 0; f < m.F; ++f) {
    const int* fv = &m.fv[static_cast<size_t>(f) * m.nfv];
    const double* a = &m.X[3 * fv[0]];
    const double* b = &m.X[3 * fv[1]];
    int opp = -1;
    for (int k = 0; k < m.nvc; ++k) {
      int v = m.cv[m.eL[f] * m.nvc + k];
      bool on = false;
      for (int j = 0; j < m.nfv; ++j) on |= (fv[j] == v);
      if (!on) opp = v;
    }
    const double* po = &m.X[3 * opp];
    double n[3], meas;
    if (m.dim == 2) {
      double t0 = b[0] - a[0], t1 = b[1] - a[1];
      meas = std::sqrt(t0 * t0 + t1 * t1);
      n[0] = t1 / meas;
      n[1] = -t0 / meas;
      n[2] = 0.0;
    } else {
      const double* c = &m.X[3 * fv[2]];
      double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
      double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
      double l = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      for (int k = 0; k < 3; ++k) n[k] = cr[k] / l;
      meas = 0.5 * l;
    }
    double d = (po[0] - a[0]) * n[0] + (po[1] - a[1]) * n[1] + (po[2] - a[2]) * n[2];
    if (d > 0)
      for (double& x : n) x = -x;
    for (int k = 0; k < 3; ++k) m.fn[3 * f + k] = n[k];
    m.fmeas[f] = meas;
  }
  boundary_ids(m, bkeys);
  periodic_pairs(m);
  return DGP_OK;
}

// minimal fast tokenizer over the whole file
struct Scanner {
  const char* p;
  const char* end;
  bool word(std::string& out) {
    while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
    if (p >= end) return false;
    const char* s = p;
    while (p < end && !std::isspace(static_cast<unsigned char>(*p))) ++p;
    out.assign(s, p);
    return true;
  }
  bool integer(long& v) {
    while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
    char* e = nullptr;
    v = std::strtol(p, &e, 10);
    if (e == p) return false;
    p = e;
    return true;
  }
  bool real(double& v) {
    while (p < end && std::isspace(static_cast<unsigned char>(*p))) ++p;
    char* e = nullptr;
    v = std::strtod(p, &e);
    if (e == p) return false;
    p = e;
    return true;
  }
};

}  // namespace

int read_msh_v1(const std::string& path, HostMesh& m, std::string& err, bool gpu_faces) {
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    err = "cannot open mesh file " + path;
    return DGP_ERR_IO;
  }
  std::string buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  buf.push_back('\0');
  Scanner sc{buf.data(), buf.data() + buf.size() - 1};
  std::string tok;
  std::vector<double> X;
  std::vector<int> ids;
  std::vector<int> tri, tet, lines, btri;
  std::vector<int> tri_tag, tet_tag, line_tag, btri_tag;
  bool have_nod = false, have_elm = false;
  while (sc.word(tok)) {
    if (tok == "$NOD" || tok == "$NOE") {
      long n;
      if (!sc.integer(n) || n < 0) { err = "bad $NOD count"; return DGP_ERR_IO; }
      X.resize(static_cast<size_t>(n) * 3);
      ids.resize(n);
      for (long i = 0; i < n; ++i) {
        long id;
        if (!sc.integer(id) || !sc.real(X[3 * i]) || !sc.real(X[3 * i + 1]) || !sc.real(X[3 * i + 2])) {
          err = "truncated $NOD section";
          return DGP_ERR_IO;
        }
        ids[i] = static_cast<int>(id);
      }
      have_nod = true;
    } else if (tok == "$ELM") {
      long n;
      if (!sc.integer(n) || n < 0) { err = "bad $ELM count"; return DGP_ERR_IO; }
      for (long i = 0; i < n; ++i) {
        long num, typ, phys, elem, nn;
        if (!sc.integer(num) || !sc.integer(typ) || !sc.integer(phys) || !sc.integer(elem) ||
            !sc.integer(nn) || nn < 0 || nn > 64) {
          err = "truncated $ELM section";
          return DGP_ERR_IO;
        }
        long v[64];
        for (long k = 0; k < nn; ++k)
          if (!sc.integer(v[k])) { err = "truncated element line"; return DGP_ERR_IO; }
        switch (typ) {
          case 1:
            lines.insert(lines.end(), v, v + 2);
            line_tag.push_back(static_cast<int>(phys));
            break;
          case 2:
            tri.insert(tri.end(), v, v + 3);
            tri_tag.push_back(static_cast<int>(phys));
            break;
          case 4:
            tet.insert(tet.end(), v, v + 4);
            tet_tag.push_back(static_cast<int>(phys));
            break;
          default:
            err = "element type " + std::to_string(typ) + " is not a straight triangle/tet/line";
            return DGP_ERR_UNSUPPORTED;
        }
      }
      have_elm = true;
    }
  }
  if (!have_nod || !have_elm) {
    err = "mesh file lacks $NOD or $ELM";
    return DGP_ERR_IO;
  }
  int maxid = 0;
  for (int id : ids) maxid = std::max(maxid, id);
  std::vector<int> id2idx(static_cast<size_t>(maxid) + 1, -1);
  for (size_t i = 0; i < ids.size(); ++i) id2idx[ids[i]] = static_cast<int>(i);
  auto map_ids = [&](std::vector<int>& a) -> bool {
    for (int& x : a) {
      if (x < 0 || x > maxid || id2idx[x] < 0) return false;
      x = id2idx[x];
    }
    return true;
  };
  const bool is3d = !tet.empty();
  std::vector<int>& cells = is3d ? tet : tri;
  std::vector<int>& ctags = is3d ? tet_tag : tri_tag;
  std::vector<int>& bf = is3d ? tri : lines;
  std::vector<int>& bt = is3d ? tri_tag : line_tag;
  if (cells.empty()) {
    err = "mesh has no triangles or tets";
    return DGP_ERR_IO;
  }
  if (!map_ids(cells) || !map_ids(bf)) {
    err = "element references an unknown node id";
    return DGP_ERR_IO;
  }
  const int dim = is3d ? 3 : 2;
  return mesh_from_arrays(dim, static_cast<int>(ids.size()), X.data(), ids.data(),
                          static_cast<int>(ctags.size()), cells.data(), ctags.empty() ? 0 : ctags.back(),
                          static_cast<int>(bt.size()), bf.data(), bt.data(), m, err, gpu_faces);
}

int mesh_from_arrays(int dim, int nv, const double* xyz, const int* vids, int ncells,
                     const int* cells, int cell_tag, int nbf, const int* bfaces,
                     const int* btags, HostMesh& m, std::string& err, bool gpu_faces) {
  if ((dim != 2 && dim != 3) || nv <= 0 || ncells <= 0 || !xyz || !cells) {
    err = "invalid mesh arrays";
    return DGP_ERR_INVALID;
  }
  m = HostMesh();
  m.dim = dim;
  m.nvc = dim + 1;
  m.nfv = dim;
  m.nlf = dim + 1;
  m.X.assign(xyz, xyz + static_cast<size_t>(nv) * 3);
  m.vid.resize(nv);
  for (int i = 0; i < nv; ++i) m.vid[i] = vids ? vids[i] : i + 1;
  m.E = ncells;
  m.cv.assign(cells, cells + static_cast<size_t>(ncells) * m.nvc);
  for (int x : m.cv)
    if (x < 0 || x >= nv) {
      err = "cell vertex index out of range";
      return DGP_ERR_INVALID;
    }
  m.ctag = cell_tag;
  std::vector<FaceKey> bkeys;
  for (int i = 0; i < nbf; ++i) {
    FaceKey k{{INT32_MAX, INT32_MAX, INT32_MAX}, btags ? btags[i] : cell_tag, 0};
    for (int j = 0; j < dim; ++j) {
      int v = bfaces[static_cast<size_t>(i) * dim + j];
      if (v < 0 || v >= nv) {
        err = "boundary face vertex index out of range";
        return DGP_ERR_INVALID;
      }
      k.v[j] = m.vid[v];
    }
    sort_small(k.v, dim);
    bkeys.push_back(k);
  }
  // degenerate cells make the affine map singular
  for (int e = 0; e < m.E; ++e) {
    double x0[3], J[9], Ji[9];
    cell_frame(m, e, x0, J);
    double d = invert3(J, Ji);
    if (!(std::fabs(d) > 0.0) || !std::isfinite(d)) {
      err = "degenerate cell " + std::to_string(e);
      return DGP_ERR_INVALID;
    }
  }
  if (gpu_faces) {
    const int rc = build_faces_gpu(m, err);
    if (rc == DGP_OK) {
      std::sort(bkeys.begin(), bkeys.end());
      boundary_ids(m, bkeys);
      periodic_pairs(m);
      return DGP_OK;
    }
    if (rc != DGP_ERR_UNSUPPORTED) return rc;
    err.clear();
  }
  return build_faces(m, bkeys, err);
}

void cell_frame(const HostMesh& m, int e, double* x0, double* J) {
  const int* c = &m.cv[static_cast<size_t>(e) * m.nvc];
  const double* p0 = &m.X[3 * c[0]];
  static const int tet_node[3] = {3, 2, 1};
  for (int k = 0; k < 3; ++k) x0[k] = p0[k];
  for (int i = 0; i < 9; ++i) J[i] = 0.0;
  for (int r = 0; r < m.dim; ++r) {
    int node = (m.dim == 2) ? r + 1 : tet_node[r];
    const double* p = &m.X[3 * c[node]];
    for (int k = 0; k < 3; ++k) J[r * 3 + k] = p[k] - p0[k];
  }
  if (m.dim == 2) J[8] = 1.0;
}

void PointLocator::build(const HostMesh& mesh) {
  m = &mesh;
  const int dim = mesh.dim, E = mesh.E;
  double hi[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k) {
    lo[k] = 1e300;
    hi[k] = -1e300;
  }
  for (int v = 0; v < (int)(mesh.X.size() / 3); ++v)
    for (int k = 0; k < dim; ++k) {
      lo[k] = std::min(lo[k], mesh.X[3 * v + k]);
      hi[k] = std::max(hi[k], mesh.X[3 * v + k]);
    }
  // about one cell per bucket
  const double per = std::pow(std::max(E, 1), 1.0 / dim);
  for (int k = 0; k < 3; ++k) {
    n[k] = k < dim ? std::max(1, (int)per) : 1;
    const double ext = k < dim ? std::max(hi[k] - lo[k], 1e-300) : 1.0;
    h[k] = ext / n[k];
  }
  auto bucket_range = [&](int e, int* b0, int* b1) {
    const int* c = &mesh.cv[static_cast<size_t>(e) * mesh.nvc];
    for (int k = 0; k < 3; ++k) {
      if (k >= dim) {
        b0[k] = b1[k] = 0;
        continue;
      }
      double mn = 1e300, mx = -1e300;
      for (int v = 0; v < mesh.nvc; ++v) {
        mn = std::min(mn, mesh.X[3 * c[v] + k]);
        mx = std::max(mx, mesh.X[3 * c[v] + k]);
      }
      b0[k] = std::max(0, std::min(n[k] - 1, (int)std::floor((mn - lo[k]) / h[k])));
      b1[k] = std::max(0, std::min(n[k] - 1, (int)std::floor((mx - lo[k]) / h[k])));
    }
  };
  const size_t nb = static_cast<size_t>(n[0]) * n[1] * n[2];
  std::vector<int> cnt(nb + 1, 0);
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      off.assign(nb + 1, 0);
      for (size_t b = 0; b < nb; ++b) off[b + 1] = off[b] + cnt[b];
      ids.assign(off[nb], 0);
      std::fill(cnt.begin(), cnt.end(), 0);
    }
    for (int e = 0; e < E; ++e) {
      int b0[3], b1[3];
      bucket_range(e, b0, b1);
      for (int z = b0[2]; z <= b1[2]; ++z)
        for (int y = b0[1]; y <= b1[1]; ++y)
          for (int x = b0[0]; x <= b1[0]; ++x) {
            const size_t b = (static_cast<size_t>(z) * n[1] + y) * n[0] + x;
            if (pass == 1) ids[off[b] + cnt[b]] = e;
            cnt[b]++;
          }
    }
  }
}

int PointLocator::locate(const double* x, double* xi) const {
  const int dim = m->dim;
  int bi[3] = {0, 0, 0};
  for (int k = 0; k < dim; ++k) {
    const double u = (x[k] - lo[k]) / h[k];
    if (u < -1e-9 * n[k] || u > n[k] * (1 + 1e-9)) return -1;
    bi[k] = std::max(0, std::min(n[k] - 1, (int)std::floor(u)));
  }
  const size_t b = (static_cast<size_t>(bi[2]) * n[1] + bi[1]) * n[0] + bi[0];
  int best = -1;
  for (int i = off[b]; i < off[b + 1]; ++i) {
    const int e = ids[i];
    if (best >= 0 && e >= best) continue;
    double X0[3], J[9], Ji[9], r[3] = {0, 0, 0};
    cell_frame(*m, e, X0, J);
    invert3(J, Ji);
    for (int q = 0; q < dim; ++q)
      for (int c = 0; c < dim; ++c) r[q] += Ji[c * 3 + q] * (x[c] - X0[c]);
    double sum = 0.0, mn = 1.0;
    for (int q = 0; q < dim; ++q) {
      sum += r[q];
      mn = std::min(mn, r[q]);
    }
    if (mn >= -1e-12 && sum <= 1.0 + 1e-12) {
      best = e;
      for (int q = 0; q < 3; ++q) xi[q] = q < dim ? r[q] : 0.0;
    }
  }
  return best;
}

double invert3(const double* A, double* B) {
  double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
               A[2] * (A[3] * A[7] - A[4] * A[6]);
  double id = 1.0 / det;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * id;
  B[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = (A[5] * A[6] - A[3] * A[8]) * id;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  B[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * id;
  B[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return det;
}

// ---------------------------------------------------------------------------
// orthonormal basis: Gram-Schmidt of the monomials in DG-Parallel's order
// (SHF::PascalgetFct ShapeFunctionList.cc:311, SHF::getTetFct :666) under
// int_ref a b, in long double.
namespace {
const int kTriMono[15][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}, {3, 0}, {2, 1},
                             {1, 2}, {0, 3}, {4, 0}, {3, 1}, {2, 2}, {1, 3}, {0, 4}};
const int kTetMono[35][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1},
    {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2},
    {0, 1, 2}, {1, 1, 1}, {4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {3, 1, 0}, {3, 0, 1}, {1, 3, 0}, {0, 3, 1},
    {1, 0, 3}, {0, 1, 3}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};

long double factl(int n) {
  long double r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

double mono_val(const int* e, const double* x) {
  double r = 1;
  for (int k = 0; k < 3; ++k)
    for (int p = 0; p < e[k]; ++p) r *= x[k];
  return r;
}

double mono_der(const int* e, const double* x, int dir) {
  if (e[dir] == 0) return 0.0;
  double r = e[dir];
  for (int k = 0; k < 3; ++k) {
    int p = e[k] - (k == dir);
    for (int q = 0; q < p; ++q) r *= x[k];
  }
  return r;
}

const dgp_q_rule* find_rule(int dim, int degree) {
  if (degree < 1) degree = 1;
  if (dim == 2) {
    for (const auto& r : dgp_q_tri_rules)
      if (r.degree == degree) return &r;
  } else {
    for (const auto& r : dgp_q_tet_rules)
      if (r.degree == degree) return &r;
  }
  return nullptr;
}

// reference coordinates of the element vertices (node order of the affine map)
void ref_vertex(int dim, int node, double* xi) {
  xi[0] = xi[1] = xi[2] = 0.0;
  if (dim == 2) {
    if (node == 1) xi[0] = 1.0;
    if (node == 2) xi[1] = 1.0;
  } else {
    if (node == 3) xi[0] = 1.0;
    if (node == 2) xi[1] = 1.0;
    if (node == 1) xi[2] = 1.0;
  }
}
}  // namespace

void basis_eval(const RefTables& t, const double* xi, double* out) {
  for (int i = 0; i < t.Np; ++i) {
    double r = 0.0;
    for (int j = 0; j <= i; ++j) r += mono_val(t.mono[j], xi) * t.G[i][j];
    out[i] = r;
  }
}

void build_limiter_tables(const RefTables& t, std::vector<double>& D, std::vector<double>& Dinv) {
  const int P = t.order;
  const size_t total = static_cast<size_t>((P + 1) * (P + 2) * (2 * P + 3) / 6);
  D.assign(total, 0.0);
  Dinv.assign(total, 0.0);
  for (int n = 0; n <= P; ++n) {
    const int base = n * (n + 1) / 2, w = n + 1, off = n * (n + 1) * (2 * n + 1) / 6;
    long double A[5][5], X[5][5];
    for (int i = 0; i <= n; ++i)
      for (int m = 0; m <= n; ++m) {
        const double f = static_cast<double>(factl(n - i) * factl(i));
        D[off + i * w + m] = f * t.G[base + m][base + i];
        A[i][m] = static_cast<long double>(D[off + i * w + m]);
      }
    for (int k = 0; k <= n; ++k)  // column k of the inverse, back substitution
      for (int i = n; i >= 0; --i) {
        long double r = (i == k) ? 1.0L : 0.0L;
        for (int m = i + 1; m <= n; ++m) r -= A[i][m] * X[m][k];
        X[i][k] = r / A[i][i];
      }
    for (int m = 0; m <= n; ++m)
      for (int i = 0; i <= n; ++i) Dinv[off + m * w + i] = static_cast<double>(X[m][i]);
  }
}

int build_tables(int dim, int order, RefTables& t, std::string& err, int rule) {
  t = RefTables();
  t.dim = dim;
  t.order = order;
  t.Np = dim == 2 ? (order + 1) * (order + 2) / 2 : (order + 1) * (order + 2) * (order + 3) / 6;
  t.nlf = dim + 1;
  if (order < 0 || (dim == 2 && order > 4) || (dim == 3 && order > 3)) {
    err = "supported orders: P0-P4 on triangles, P0-P3 on tets";
    return DGP_ERR_UNSUPPORTED;
  }
  const int N = t.Np;
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) t.mono[i][k] = (k < dim) ? (dim == 2 ? kTriMono[i][k] : kTetMono[i][k]) : 0;
  static long double M[kMaxNp][kMaxNp], V[kMaxNp][kMaxNp];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      int tot = 0;
      long double num = 1;
      for (int k = 0; k < 3; ++k) {
        int e = t.mono[i][k] + t.mono[j][k];
        num *= factl(e);
        tot += e;
      }
      M[i][j] = num / factl(tot + dim);
    }
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < N; ++j) V[i][j] = (i == j) ? 1.0L : 0.0L;
    for (int pass = 0; pass < 2; ++pass)
      for (int j = 0; j < i; ++j) {
        long double p = 0;
        for (int a = 0; a < N; ++a)
          for (int b = 0; b < N; ++b) p += V[i][a] * V[j][b] * M[a][b];
        for (int a = 0; a < N; ++a) V[i][a] -= p * V[j][a];
      }
    long double nn = 0;
    for (int a = 0; a < N; ++a)
      for (int b = 0; b < N; ++b) nn += V[i][a] * V[i][b] * M[a][b];
    long double inv = 1.0L / std::sqrt(nn);
    for (int a = 0; a < N; ++a) V[i][a] *= inv;
  }
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) t.G[i][j] = static_cast<double>(V[i][j]);
  t.phi0 = t.G[0][0];

  const double refm = dim == 2 ? 0.5 : 1.0 / 6.0;
  const bool alt = rule == 1 && order == 2;
  const dgp_q_rule* vr = !alt ? find_rule(dim, 2 * order) : dim == 2 ? find_rule(2, 5) : &dgp_q_tet_alt_rules[0];
  const dgp_q_rule* er = find_rule(dim, 2 * (order + 1));
  if (!vr || !er) {
    err = "no quadrature rule for this order";
    return DGP_ERR_UNSUPPORTED;
  }
  t.nq = vr->npts;
  t.qp.assign(static_cast<size_t>(t.nq) * 3, 0.0);
  t.qw.resize(t.nq);
  t.phi.resize(static_cast<size_t>(t.nq) * N);
  t.dphi.resize(static_cast<size_t>(t.nq) * dim * N);
  for (int q = 0; q < t.nq; ++q) {
    double* x = &t.qp[3 * q];
    for (int k = 0; k < dim; ++k) x[k] = vr->data[q * (dim + 1) + k];
    t.qw[q] = refm * vr->data[q * (dim + 1) + dim];
    basis_eval(t, x, &t.phi[static_cast<size_t>(q) * N]);
    for (int r = 0; r < dim; ++r)
      for (int i = 0; i < N; ++i) {
        double v = 0.0;
        for (int j = 0; j <= i; ++j) v += mono_der(t.mono[j], x, r) * t.G[i][j];
        t.dphi[(static_cast<size_t>(q) * dim + r) * N + i] = v;
      }
  }
  t.nqe = er->npts;
  t.eqp.assign(static_cast<size_t>(t.nqe) * 3, 0.0);
  t.eqw.resize(t.nqe);
  t.ephi.resize(static_cast<size_t>(t.nqe) * N);
  for (int q = 0; q < t.nqe; ++q) {
    double* x = &t.eqp[3 * q];
    for (int k = 0; k < dim; ++k) x[k] = er->data[q * (dim + 1) + k];
    t.eqw[q] = refm * er->data[q * (dim + 1) + dim];
    basis_eval(t, x, &t.ephi[static_cast<size_t>(q) * N]);
  }

  // face rule: Gauss-Legendre n = p+1 on [-1,1] (getNGQ1DPts(2p+1)) for edges,
  // the triangle rule of degree 2p+1 for tet faces (weights incl. 1/2)
  if (dim == 2) {
    t.nqf = order + 1;
    const double* gl = dgp_q_gauss_legendre[t.nqf];
    t.fqp.assign(static_cast<size_t>(t.nqf) * 2, 0.0);
    t.fqw.resize(t.nqf);
    for (int q = 0; q < t.nqf; ++q) {
      t.fqp[2 * q] = gl[2 * q];
      t.fqw[q] = gl[2 * q + 1];
    }
  } else {
    const dgp_q_rule* fr = find_rule(2, alt ? 4 : 2 * order + 1);
    if (!fr) {
      err = "no face rule";
      return DGP_ERR_UNSUPPORTED;
    }
    t.nqf = fr->npts;
    t.fqp.resize(static_cast<size_t>(t.nqf) * 2);
    t.fqw.resize(t.nqf);
    for (int q = 0; q < t.nqf; ++q) {
      t.fqp[2 * q] = fr->data[3 * q];
      t.fqp[2 * q + 1] = fr->data[3 * q + 1];
      t.fqw[q] = 0.5 * fr->data[3 * q + 2];
    }
  }
  // traces on each local face, in the face's own (element-local) point order
  t.phif.resize(static_cast<size_t>(t.nlf) * t.nqf * N);
  for (int lf = 0; lf < t.nlf; ++lf)
    for (int q = 0; q < t.nqf; ++q) {
      double xi[3] = {0, 0, 0};
      if (dim == 2) {
        double a[3], b[3], s = t.fqp[2 * q];
        ref_vertex(2, kTriFace[lf][0], a);
        ref_vertex(2, kTriFace[lf][1], b);
        for (int k = 0; k < 3; ++k) xi[k] = a[k] * (1 - s) * 0.5 + b[k] * (1 + s) * 0.5;
      } else {
        double a[3], b[3], c[3], u = t.fqp[2 * q], v = t.fqp[2 * q + 1];
        ref_vertex(3, kTetFace[lf][0], a);
        ref_vertex(3, kTetFace[lf][1], b);
        ref_vertex(3, kTetFace[lf][2], c);
        for (int k = 0; k < 3; ++k) xi[k] = a[k] * (1 - u - v) + b[k] * u + c[k] * v;
      }
      basis_eval(t, xi, &t.phif[(static_cast<size_t>(lf) * t.nqf + q) * N]);
    }
  // orientation maps: frame point q -> index of the same physical point in the
  // right cell's local-face order
  t.nperm = dim == 2 ? 2 : 6;
  t.qmap.resize(static_cast<size_t>(t.nperm) * t.nqf);
  for (int p = 0; p < t.nperm; ++p)
    for (int q = 0; q < t.nqf; ++q) {
      double target[2];
      if (dim == 2) {
        target[0] = (p == 0) ? t.fqp[2 * q] : -t.fqp[2 * q];
        target[1] = 0.0;
      } else {
        double lam[3] = {1.0 - t.fqp[2 * q] - t.fqp[2 * q + 1], t.fqp[2 * q], t.fqp[2 * q + 1]};
        // right-local vertex k sits at frame position kPerm3[p][k]
        target[0] = lam[kPerm3[p][1]];
        target[1] = lam[kPerm3[p][2]];
      }
      int best = -1;
      double bd = 1e300;
      for (int r = 0; r < t.nqf; ++r) {
        double d = std::fabs(t.fqp[2 * r] - target[0]) + std::fabs(t.fqp[2 * r + 1] - target[1]);
        if (d < bd) {
          bd = d;
          best = r;
        }
      }
      if (bd > 1e-12) {
        err = "face rule is not symmetric under vertex permutations";
        return DGP_ERR_UNSUPPORTED;
      }
      t.qmap[static_cast<size_t>(p) * t.nqf + q] = best;
    }
  // basis at the reference vertices (DGCell::computeMAXEV evaluates the state there)
  t.phiv.resize(static_cast<size_t>(dim + 1) * N);
  for (int node = 0; node <= dim; ++node) {
    double xi[3];
    ref_vertex(dim, node, xi);
    basis_eval(t, xi, &t.phiv[static_cast<size_t>(node) * N]);
  }
  return DGP_OK;
}

}  // namespace dgp
