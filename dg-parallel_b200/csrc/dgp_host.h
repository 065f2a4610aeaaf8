// Host-side data of the dgp solver: mesh, connectivity, FP64 geometry and the
// reference-element tables that the CUDA kernels consume.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace dgp {

constexpr int kMaxNp = 35;   // tet P4
constexpr int kMaxQ = 64;

// Mesh as imported (mImportExport::importGmshFile, mImportExport.cc:77-170)
// plus the face table DG-Parallel derives from it (mMesh::createCellBoundaries
// and createConnections, mMesh.cc:321-378; DGBoundaryCell::check,
// DGCell.cc:355-391).  Cells keep file order here; the solver reorders them.
struct HostMesh {
  int dim = 0, nvc = 0, nfv = 0, nlf = 0;
  std::vector<double> X;     // nv x 3
  std::vector<int> vid;      // file vertex ids
  int E = 0;
  std::vector<int> cv;       // E x nvc vertex indices (file node order)
  int ctag = 0;              // physical tag of the cells
  int F = 0;
  std::vector<int> fv;       // F x nfv: vertices in the left cell's local-face order
  std::vector<int> eL, eR, lfL, lfR, bid;
  std::vector<int> rperm;    // right local face orientation w.r.t. the face frame
  std::vector<double> fn;    // F x 3 unit normal, outward from the left cell
  std::vector<double> fmeas; // F face length / area
  std::vector<int> pface;    // F periodic partner face of a 510/610 boundary edge (-1: none)
};

// Reads a Gmsh v1 file; returns 0 or a DGP_ERR_* code with `err` set.
// gpu_faces: match the faces on the current CUDA device (build_faces_gpu).
int read_msh_v1(const std::string& path, HostMesh& m, std::string& err, bool gpu_faces = false);
// Builds from arrays (0-based indices); vertex ids default to 1..nv.
int mesh_from_arrays(int dim, int nv, const double* xyz, const int* vids, int ncells,
                     const int* cells, int cell_tag, int nbf, const int* bfaces,
                     const int* btags, HostMesh& m, std::string& err, bool gpu_faces = false);
// Face matching on the GPU (dgp_meshprep.cu): fills F, fv, eL, eR, lfL, lfR,
// rperm, fn, fmeas exactly as the host matching does (classification ids and
// periodic pairs are added on the host).  DGP_ERR_UNSUPPORTED when the vertex
// count does not fit the packed face keys (the caller then matches on the host).
int build_faces_gpu(HostMesh& m, std::string& err);

// glibc srand(seed); rand(): the TYPE_3 additive generator of the C library,
// which DG-Parallel sums over vertex ids to order its entities
// (Vertex::getRAND, Vertex.cc:26-31).
uint32_t glibc_rand_first(uint32_t seed);

// Reference-element tables for one (dimension, order).
struct RefTables {
  int dim = 0, order = 0, Np = 0, nlf = 0;
  double G[kMaxNp][kMaxNp];          // basis i = sum_j G[i][j] monomial_j
  int mono[kMaxNp][3];
  int nq = 0;                        // volume rule of degree 2p
  std::vector<double> qp, qw;        // nq x 3 (u,v,w), weight incl. reference measure
  std::vector<double> phi;           // nq x Np
  std::vector<double> dphi;          // nq x dim x Np  (d phi / d xi_r)
  int nqf = 0;                       // face rule of degree 2p+1
  std::vector<double> fqw;           // nqf face weights (incl. reference measure)
  std::vector<double> fqp;           // nqf x 2 face-local coordinates
  std::vector<double> phif;          // nlf x nqf x Np: traces on each local face
  int nperm = 0;                     // face orientations (2 edge, 6 triangle)
  std::vector<int> qmap;             // nperm x nqf: frame point -> right-local point
  std::vector<double> phiv;          // (dim+1) x Np basis at the reference vertices
  double phi0 = 0;                   // constant basis value (sqrt 2 / sqrt 6)
  int nqe = 0;                       // error rule of degree 2(p+1)
  std::vector<double> eqp, eqw, ephi;
};

// rule 0: DG-Parallel's quadrature (volume degree 2p, tet faces degree 2p + 1);
// rule 1: at P2 the workloads' point counts (triangle volume: the 7-point rule
// of degree 5; tets: the 11-point volume and 6-point face rules of degree 4)
int build_tables(int dim, int order, RefTables& t, std::string& err, int rule = 0);
void basis_eval(const RefTables& t, const double* xi, double* out);
// triangle moment limiter tables, per degree n a (n+1)^2 block at
// n(n+1)(2n+1)/6: D[i][m] = d^n phi_(n,m) / du^(n-i) dv^i (constant on the
// cell) and its inverse (D is upper triangular)
void build_limiter_tables(const RefTables& t, std::vector<double>& D, std::vector<double>& Dinv);

// Affine frame of a cell: x = x0 + sum_r xi_r J[r][:], with the node order of
// MeshMapping::GeomShapeFunctionTri/Tet (Mapping.cc:40-71, 94-103).
void cell_frame(const HostMesh& m, int e, double* x0, double* J);
double invert3(const double* A, double* B);

// Point location over the cells of one mesh (DGCell::inCell, DGCell.cc:1499-1521:
// bounding box, then the reference coordinates of the point inside the
// reference simplex).  A uniform grid of buckets holds every cell whose
// bounding box meets the bucket; a point takes the lowest-index cell whose
// reference coordinates are all >= -1e-12 (points on shared faces resolve the
// same way whatever the bucketing).
struct PointLocator {
  const HostMesh* m = nullptr;
  double lo[3] = {0, 0, 0}, h[3] = {1, 1, 1};
  int n[3] = {1, 1, 1};
  std::vector<int> off, ids;  // bucket -> cells (CSR)
  void build(const HostMesh& mesh);
  // cell index (file order of the mesh) or -1; xi: reference coordinates
  int locate(const double* x, double* xi) const;
};

}  // namespace dgp
