// Oracle driver around DG-Parallel's own C++ code (TEST INFRASTRUCTURE ONLY).
//
// This file is linked against objects compiled unchanged from the DG-Parallel
// sources (see oracle/Makefile); it is never part of the product.  It rebuilds
// the time loop that ships commented out in DGAnalysis::run
// (DGAnalysis.cc:480-731) and dumps what the parity tests compare:
//
//   --conn FILE    one line per mesh face: sorted face vertex ids, left and
//                  right cell (0-based file order of the cell elements, -1 for
//                  none), local face index on each side, classification id,
//                  the left-outward unit normal and the face measure.
//   --rhs FILE     theRightHandSide of every cell after one assembly
//                  (TimeIntegrator::assembleVolume + assembleBoundary) of the
//                  projected initial state, in file order.
//   --state FILE   coefficients of every cell ([field][mode], file order) of
//                  the projected initial state and after every --every steps.
//   --log FILE     per step: dt, time, residual returned by advanceInTime.
//   --barth FILE   after the steps: DGBarthLimiter::limit on every cell of the
//                  state (means computed first, each cell's faces as its
//                  allSubs list as DGAnalysis.cc:244-253 builds it), then the
//                  coefficients of every cell ([field][mode], file order) and
//                  the cell's per-field slope factors (details->limSlope).  The
//                  limiter writes the coefficients in place; TimeIntegrator::
//                  limit's copy of the unwritten second slot is not applied.
//   --state-bin F  after the steps: the coefficients of every cell as raw
//                  native doubles, [cell][field][mode] in file order.
//   --l2 FILE      after the steps: DGAnalysis::densityErrorL2 (DGPref.cc:370-380)
//                  at the final time, then every cell's DGCell::densityErrorL2
//                  (DGError.cc:805-826; the squared error) in file order.
//   --ckpt-out F   after the steps: the data stream of DGAnalysis::write
//                  (DGPref.cc:712-739) -- TACT, ITER, sizes, every cell's
//                  writeMEntity + DGCell::write, every face's writeMEntity.
//   --ckpt-in F    before the steps: the coefficients of every cell read the
//                  way DGAnalysis::read does (DGPref.cc:741-766:
//                  mMesh::readMEntity, the order, DGCell::read) in place of the
//                  projection.
//   --gpu 1        (built as ref_driver_gpu only) step with GpuTimeIntegrator,
//                  the shim of dg-parallel_b200/integration, on the reference's
//                  own cells and CFL steps instead of RungeKuttaTVD3
//   --lts 1        (built as ref_driver_lts only) local time stepping: the
//                  cells binned by size as DGAnalysis::sortCellsBySize does
//                  (DGAnalysis.cc:749-890), the time step of mode 5
//                  (DGAnalysis.cc:514-593: CFL minimum times 2^(bins-1)) and
//                  RungeKuttaTVD2adaptive::advanceInTime (TimeIntegrator.cc:
//                  442-836).  The reference ships the two range helpers that
//                  integrator calls, TimeIntegrator::assembleVolume(begin, end,
//                  t) and assembleBoundary(begin, end, t) (TimeIntegrator.cc:
//                  1438-1487), with their bodies commented out, so its local
//                  time stepping never assembles a right-hand side and leaves
//                  the state unchanged.  This build defines them below with the
//                  bodies of the whole-mesh versions (TimeIntegrator.cc:
//                  1332-1412) restricted to the range, and links them ahead of
//                  TimeIntegrator.cc compiled without inlining (oracle/Makefile).
//   --bins FILE    (with --lts) per cell in file order: bin, role (0 inner,
//                  1 large on an interface, 2 small on an interface).
//   --bench N      time N steps (after --warmup W untimed ones) (CFL dt + RungeKuttaTVD3::advanceInTime)
//                  with --threads workers of the reference pthreads path
//                  (parallel.cc, chunked as main.cc) and print one "BENCH ..."
//                  line.  Without --bench a single worker thread runs every
//                  chunk, so results are deterministic and use the stage time.
//
// Cases (--case): the analytic fields below are this driver's own and are
// restated identically by the C oracle and the product.
//   gauss     scalar advection u_t + a.grad u = 0 (ScalarLaw), a = (ax, ay),
//             u0 = exp(-((x-cx)^2+(y-cy)^2)/s), exact u0(x - a t) as far field.
//   vortex    2D Euler isentropic vortex (Euler2d exact Godunov, or
//             Euler2dRoe with --flux roe); exact solution as far field.
//   pulse3d   3D Euler (Euler3d) density pulse advected by a uniform flow.
//   sine      Burgers2D with u0 = 0.5 + A sin(2 pi (x+y)) as far field.
//   tm2d      Maxwell2d (MaxwellLaw.cc) with a TM cavity mode (TM2DField) as
//             initial state and far field; faces tagged 40000 reflect.
//   gauss3d   scalar advection on tets, 3D Gaussian.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <set>
#include <string>
#include <vector>
#include <algorithm>
#include <fstream>
#include <unistd.h>

#include "mImportExport.h"
#include "mDGMesh.h"
#include "mEntity.h"
#include "Vertex.h"
#include "gEntity.h"
#include "parallel.h"
#include "DGCell.h"
#include "FunctionSpace.h"
#include "Mapping.h"
#include "Integrator.h"
#include "TimeIntegrator.h"
#include "ScalarLaw.h"
#include "EulerLaw.h"
#include "MaxwellLaw.h"
#include "Burgers.h"
#include "FieldEvaluator.h"
#include "DGLimiter.h"
#ifdef DGP_GPU_INTEGRATOR
#include "GpuTimeIntegrator.h"
#endif
#include "mPoint.h"

// Globals that the reference's threading code declares extern (main.cc owns
// them in the shipped program).
unsigned int numCPU = 1;
unsigned int numThreads = 1;
vector<infoWrapper> threadInfo[4];
vector<infoWrapper> threadInfoBoundary[4];
double timeRK = 0;

static const double kPi = 3.14159265358979323846;

#ifdef DGP_REF_LTS
// The range helpers RungeKuttaTVD2adaptive calls, with the bodies of the
// whole-mesh versions (TimeIntegrator.cc:1332-1412) on one thread.
void TimeIntegrator::assembleVolume(const mMesh::iter begin, const mMesh::iter end, double t) {
  for (mMesh::iter it = begin; it != end; ++it) ((DGCell*)(*it)->getCell())->computeVolumeContribution(t);
}

void TimeIntegrator::assembleBoundary(const mMesh::iter begin, const mMesh::iter end, double t) {
  for (mMesh::iter it = begin; it != end; ++it) {
    DGBoundaryCell* cell = (DGBoundaryCell*)(*it)->getCell();
    switch (cell->computeBoundaryContributions(t)) {
      case 0: break;
      case 1: cell->getLeftCell()->setToZero(t); break;
      case 2: cell->getRightCell()->setToZero(t); break;
      default: cell->getLeftCell()->setToZero(t); cell->getRightCell()->setToZero(t); break;
    }
  }
}

// Size bins as DGAnalysis::sortCellsBySize (DGAnalysis.cc:749-890) forms them:
// bins = ceil(log2(max size / min size)) (the minimum starts at 1.0), bin i
// holds sizes in (B_{i+1} * 1.0001, B_i * 1.0001] with B_i = max / 2^i; a face
// whose cells differ by one bin goes to the interface list of the larger bin,
// its cells leave their bins for the large / small on-interface lists.
// Returns the number of bins; exits as the reference does when cells are
// lost or neighbours differ by more than one bin.
static int ltsSortCells(mDGMesh* mesh, int n) {
  double maxSize = 0.0, minSize = 1.0;
  for (mMesh::iter it = mesh->begin(n); it != mesh->end(n); ++it) {
    double sz = ((DGCell*)(*it)->getCell())->getSize();
    if (maxSize < sz) maxSize = sz;
    if (minSize > sz) minSize = sz;
  }
  const int nb = (int)ceil(log(maxSize / minSize) / log(2.));
  mesh->setNbBins(nb);
  std::vector<double> B(nb + 1);
  B[0] = maxSize;
  if (nb > 1) {
    for (int i = 1; i <= nb; ++i) B[i] = B[i - 1] * 0.5;
    for (mMesh::iter it = mesh->begin(n); it != mesh->end(n); ++it) {
      DGCell* cell = (DGCell*)(*it)->getCell();
      double sz = cell->getSize();
      for (int i = 1; i <= nb; ++i)
        if (sz <= B[i - 1] * 1.0001 && sz > B[i] * 1.0001) {
          mesh->addToBin(i - 1, *it);
          cell->setBinNb(i - 1);
        }
    }
  }
  for (mMesh::iter it = mesh->begin(n - 1); it != mesh->end(n - 1); ++it) {
    DGBoundaryCell* bc = (DGBoundaryCell*)(*it)->getCell();
    mEntity* left = bc->getLeft();
    mEntity* right = bc->getRight();
    int lb = ((DGCell*)left->getCell())->getBinNb();
    int rb = right ? ((DGCell*)right->getCell())->getBinNb() : 0;
    if (lb == rb || !right) {
      mesh->addToBin(lb, *it);
    } else if (lb - rb == 1 || rb - lb == 1) {
      mesh->addToInterfaceBin(lb < rb ? lb : rb, *it);
      if (lb < rb) {
        mesh->addToLargeOnInterface(lb, left);
        mesh->addToSmallOnInterface(lb, right);
      } else {
        mesh->addToLargeOnInterface(rb, right);
        mesh->addToSmallOnInterface(rb, left);
      }
      mesh->delFromBin(lb, left);
      mesh->delFromBin(rb, right);
    } else {
      printf("Too big a difference between elements\n");
      exit(0);
    }
  }
  int total = 0;
  for (int i = 0; i < nb; ++i)
    total += mesh->sizeOfBin(i, n) + mesh->sizeOfLargeOnInterface(i, n) + mesh->sizeOfSmallOnInterface(i, n);
  if (total != mesh->size(n)) {
    printf("Cells were lost in sorting!");
    exit(0);
  }
  return nb;
}
#endif

struct Params {
  std::string mesh, caseName = "gauss", flux = "exact", conn, rhs, state, log, barth, ckptOut, ckptIn, l2, stateBin;
  std::string p0rhs, p0cells;  // P0 fallback fixture: output file, perturbed cells
  std::string probeOut, probePts;  // point sensors: output file, "x,y,z;x,y,z;..."
  std::string norms;  // the DGError.cc error norms at the final time
  double p0amp = 3.0;
  int order = 2, steps = 0, every = 1, threads = 1, bench = 0, warmup = 0, gpu = 0, lts = 0;
  std::string bins;
  double cfl = 0.1, tend = -1.0;
  // scalar
  double ax = 1.0, ay = 0.5, az = 0.0, cx = 0.3, cy = 0.3, cz = 0.3, s = 0.01;
  // vortex
  double gamma = 1.4, beta = 5.0, vx0 = 5.0, vy0 = 5.0;
  // burgers
  double amp = 1.0;
  double L = 1.0;  // tm2d cavity side
};
static Params P;

class ConstVelocity : public FieldEvaluator {
 public:
  void eval(const mPoint&, double, double* v) const { v[0] = P.ax; v[1] = P.ay; v[2] = P.az; }
  int order() const { return 0; }
};

class GaussField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double t, double* v) const {
    mPoint& p = const_cast<mPoint&>(x);
    double dx = p(0) - P.ax * t - P.cx, dy = p(1) - P.ay * t - P.cy;
    v[0] = exp(-(dx * dx + dy * dy) / P.s);
  }
  int order() const { return 0; }
};

class Gauss3DField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double t, double* v) const {
    mPoint& p = const_cast<mPoint&>(x);
    double dx = p(0) - P.ax * t - P.cx, dy = p(1) - P.ay * t - P.cy, dz = p(2) - P.az * t - P.cz;
    v[0] = exp(-(dx * dx + dy * dy + dz * dz) / P.s);
  }
  int order() const { return 0; }
};

// Isentropic vortex (free stream rho=u=v=p=1) advected with velocity (1,1).
class VortexField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double t, double* q) const {
    mPoint& p = const_cast<mPoint&>(x);
    const double g = P.gamma, b = P.beta;
    double dx = p(0) - (P.vx0 + t), dy = p(1) - (P.vy0 + t);
    double r2 = dx * dx + dy * dy;
    double e = exp(0.5 * (1.0 - r2));
    double u = 1.0 - b / (2.0 * kPi) * e * dy;
    double v = 1.0 + b / (2.0 * kPi) * e * dx;
    double T = 1.0 - (g - 1.0) * b * b / (8.0 * g * kPi * kPi) * e * e;
    double rho = pow(T, 1.0 / (g - 1.0));
    double pr = pow(rho, g);
    q[0] = rho;
    q[1] = rho * u;
    q[2] = rho * v;
    q[3] = pr / (g - 1.0) + 0.5 * rho * (u * u + v * v);
  }
  int order() const { return 0; }
};

// 3D Euler density pulse rho = 1 + 0.2 exp(-|x-c-Ut|^2/s), U = (ax,ay,az), p = 1.
// Field order of Euler3d: (rho, rho u, rho v, E, rho w).
class Pulse3DField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double t, double* q) const {
    mPoint& p = const_cast<mPoint&>(x);
    double dx = p(0) - P.ax * t - P.cx, dy = p(1) - P.ay * t - P.cy, dz = p(2) - P.az * t - P.cz;
    double rho = 1.0 + 0.2 * exp(-(dx * dx + dy * dy + dz * dz) / P.s);
    double pr = 1.0;
    q[0] = rho;
    q[1] = rho * P.ax;
    q[2] = rho * P.ay;
    q[4] = rho * P.az;
    q[3] = pr / (P.gamma - 1.0) + 0.5 * rho * (P.ax * P.ax + P.ay * P.ay + P.az * P.az);
  }
  int order() const { return 0; }
};

// the TM mode Ez = sin(pi x/L) sin(pi y/L) cos(w t), w = pi sqrt(2)/L, of
// Maxwell2d's equations (dHx/dt = -dEz/dy, dHy/dt = dEz/dx, dEz/dt = dHy/dx -
// dHx/dy), fields (Hx, Hy, Ez); L = --L (default 1)
class TM2DField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double t, double* v) const {
    mPoint& p = const_cast<mPoint&>(x);
    const double L = P.L > 0 ? P.L : 1.0;
    const double k = kPi / L, w = kPi * sqrt(2.0) / L;
    const double sx = sin(k * p(0)), cx = cos(k * p(0)), sy = sin(k * p(1)), cy = cos(k * p(1));
    v[0] = -(k / w) * sx * cy * sin(w * t);
    v[1] = (k / w) * cx * sy * sin(w * t);
    v[2] = sx * sy * cos(w * t);
  }
  int order() const { return 0; }
};

class SineField : public FieldEvaluator {
 public:
  void eval(const mPoint& x, double, double* v) const {
    mPoint& p = const_cast<mPoint&>(x);
    v[0] = 0.5 + P.amp * sin(2.0 * kPi * (p(0) + p(1)));
  }
  int order() const { return 0; }
};

// ---- file-order bookkeeping -------------------------------------------------
struct MshCells {
  int dim = 0;
  std::map<std::vector<int>, int> index;  // sorted vertex ids -> file order of the cell
  std::vector<std::vector<int> > verts;    // file vertex order per cell
};

static MshCells readCells(const char* path) {
  MshCells out;
  FILE* f = fopen(path, "r");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  char tok[256];
  std::vector<std::vector<int> > tris, tets;
  while (fscanf(f, "%255s", tok) == 1) {
    if (!strcmp(tok, "$NOD")) {
      int n; if (fscanf(f, "%d", &n) != 1) exit(2);
      for (int i = 0; i < n; ++i) { int id; double x, y, z; if (fscanf(f, "%d %lf %lf %lf", &id, &x, &y, &z) != 4) exit(2); }
    } else if (!strcmp(tok, "$ELM")) {
      int n; if (fscanf(f, "%d", &n) != 1) exit(2);
      for (int i = 0; i < n; ++i) {
        int num, typ, phys, elem, nn;
        if (fscanf(f, "%d %d %d %d %d", &num, &typ, &phys, &elem, &nn) != 5) exit(2);
        std::vector<int> v(nn);
        for (int k = 0; k < nn; ++k) if (fscanf(f, "%d", &v[k]) != 1) exit(2);
        if (typ == 2) tris.push_back(v);
        if (typ == 4) tets.push_back(v);
      }
    }
  }
  fclose(f);
  out.dim = tets.empty() ? 2 : 3;
  out.verts = tets.empty() ? tris : tets;
  for (size_t i = 0; i < out.verts.size(); ++i) {
    std::vector<int> k = out.verts[i];
    std::sort(k.begin(), k.end());
    out.index[k] = (int)i;
  }
  return out;
}

static int cellIndex(const MshCells& mc, mEntity* e) {
  std::vector<int> k;
  for (int i = 0; i < e->size(0); ++i) k.push_back(e->get(0, i)->getId());
  std::sort(k.begin(), k.end());
  std::map<std::vector<int>, int>::const_iterator it = mc.index.find(k);
  if (it == mc.index.end()) { fprintf(stderr, "cell not found\n"); exit(3); }
  return it->second;
}

// local face index of face entity f in cell c: triangle edge k = (v_k, v_{k+1});
// tet faces {0,1,2},{0,1,3},{0,2,3},{1,2,3} (mTet.cc Tfv1).
static int localFace(mEntity* c, mEntity* f) {
  std::set<int> fv;
  for (int i = 0; i < f->size(0); ++i) fv.insert(f->get(0, i)->getId());
  int nv = c->size(0);
  static const int tri[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  static const int tet[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  if (nv == 3) {
    for (int k = 0; k < 3; ++k) {
      std::set<int> s;
      s.insert(c->get(0, tri[k][0])->getId());
      s.insert(c->get(0, tri[k][1])->getId());
      if (s == fv) return k;
    }
  } else {
    for (int k = 0; k < 4; ++k) {
      std::set<int> s;
      for (int j = 0; j < 3; ++j) s.insert(c->get(0, tet[k][j])->getId());
      if (s == fv) return k;
    }
  }
  return -1;
}

static double nowSec() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void usage() {
  fprintf(stderr, "usage: ref_driver --mesh F.msh [--case gauss|vortex|pulse3d|sine|gauss3d] "
                  "[--flux exact|roe] [--order p] [--steps n | --tend T] [--cfl c] "
                  "[--conn F] [--rhs F] [--state F --every k] [--log F] [--barth F] [--l2 F] [--state-bin F] [--ckpt-in F] [--ckpt-out F] "
                  "[--p0-rhs F --p0-cells e,e,... [--p0-amp a]] [--probe-out F --probe-pts x,y,z;...] [--norms F] "
                  "[--threads k --bench n]\n");
  exit(1);
}

int main(int argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    const char* v = (i + 1 < argc) ? argv[i + 1] : 0;
    if (!v) usage();
    if (a == "--mesh") P.mesh = v;
    else if (a == "--case") P.caseName = v;
    else if (a == "--flux") P.flux = v;
    else if (a == "--order") P.order = atoi(v);
    else if (a == "--steps") P.steps = atoi(v);
    else if (a == "--tend") P.tend = atof(v);
    else if (a == "--cfl") P.cfl = atof(v);
    else if (a == "--every") P.every = atoi(v);
    else if (a == "--threads") P.threads = atoi(v);
    else if (a == "--bench") P.bench = atoi(v);
    else if (a == "--warmup") P.warmup = atoi(v);
    else if (a == "--conn") P.conn = v;
    else if (a == "--rhs") P.rhs = v;
    else if (a == "--state") P.state = v;
    else if (a == "--log") P.log = v;
    else if (a == "--barth") P.barth = v;
    else if (a == "--l2") P.l2 = v;
    else if (a == "--state-bin") P.stateBin = v;
    else if (a == "--p0-rhs") P.p0rhs = v;
    else if (a == "--p0-cells") P.p0cells = v;
    else if (a == "--p0-amp") P.p0amp = atof(v);
    else if (a == "--probe-out") P.probeOut = v;
    else if (a == "--norms") P.norms = v;
    else if (a == "--probe-pts") P.probePts = v;
    else if (a == "--ckpt-out") P.ckptOut = v;
    else if (a == "--ckpt-in") P.ckptIn = v;
    else if (a == "--gpu") P.gpu = atoi(v);
    else if (a == "--lts") P.lts = atoi(v);
    else if (a == "--bins") P.bins = v;
    else if (a == "--ax") P.ax = atof(v);
    else if (a == "--ay") P.ay = atof(v);
    else if (a == "--az") P.az = atof(v);
    else if (a == "--cx") P.cx = atof(v);
    else if (a == "--cy") P.cy = atof(v);
    else if (a == "--cz") P.cz = atof(v);
    else if (a == "--s") P.s = atof(v);
    else if (a == "--beta") P.beta = atof(v);
    else if (a == "--x0") P.vx0 = atof(v);
    else if (a == "--y0") P.vy0 = atof(v);
    else if (a == "--amp") P.amp = atof(v);
    else if (a == "--L") P.L = atof(v);
    else usage();
    ++i;
  }
  if (P.mesh.empty()) usage();
  numCPU = sysconf(_SC_NPROCESSORS_ONLN);
  numThreads = P.threads > 0 ? P.threads : 1;

  MshCells mc = readCells(P.mesh.c_str());
  mImportExport io;
  mDGMesh* mesh = new mDGMesh;
  io.import((char*)P.mesh.c_str(), mesh);
  const int dim = mesh->size(3) ? 3 : 2;
  mesh->createCellBoundaries(dim, dim - 1);
  mesh->createConnections(dim - 1, dim);
  mesh->createConnections(0, dim - 1);
  mesh->setPeriodicBC(dim);

  // Thread chunks.  --bench uses the chunking of main.cc:137-159.  Otherwise
  // (parity runs) one forked worker owns every entity and the master's chunk
  // is empty: TimeIntegrator::assembleBoundary hands the master chunk
  // info->_t, which it never updates (TimeIntegrator.cc:1366-1384), so with
  // main.cc's chunking the master's faces see boundary data at t = 0.
  if (P.bench <= 0) {
    numThreads = 2;
    for (int i = 0; i < 4; ++i) {
      if (mesh->size(i) == 0) continue;
      threadInfo[i].push_back(infoWrapper(mesh->begin(i), mesh->end(i), 0, 0));
      threadInfo[i].push_back(infoWrapper(mesh->end(i), mesh->end(i), 0, 0));
    }
  }
  for (int i = 0; i < 4 && P.bench > 0; ++i) {
    if (mesh->size(i) == 0) continue;
    int chunk = mesh->size(i) / numThreads;
    mMesh::iter it = mesh->begin(i);
    for (unsigned j = 0; j + 1 < numThreads; ++j) {
      mMesh::iter head = it;
      for (int k = 0; k < chunk; ++k) ++it;
      threadInfo[i].push_back(infoWrapper(head, it, 0, 0));
    }
    threadInfo[i].push_back(infoWrapper(it, mesh->end(i), 0, 0));
  }

  ConstVelocity vel;
  GaussField gauss;
  Gauss3DField gauss3;
  VortexField vortex;
  Pulse3DField pulse;
  SineField sine;
  TM2DField tm2d;
  std::set<int> walls;
  ConservationLaw* law = 0;
  if (P.caseName == "gauss") law = new ScalarLaw(&gauss, &vel, &gauss);
  else if (P.caseName == "gauss3d") law = new ScalarLaw(&gauss3, &vel, &gauss3);
  else if (P.caseName == "vortex") {
    if (P.flux == "roe") law = new Euler2dRoe(walls, &vortex, P.gamma);
    else law = new Euler2d(walls, &vortex, P.gamma);
  } else if (P.caseName == "pulse3d") law = new Euler3d(walls, &pulse, P.gamma);
  else if (P.caseName == "sine") law = new Burgers2D(&sine, &sine);
  else if (P.caseName == "tm2d") law = new Maxwell2d(walls, &tm2d);
  else usage();
  const int m = law->getNbFields();

  GaussIntegrator gi;
  int DOF = 0;
  const int E = (int)mc.verts.size();
  std::vector<DGCell*> byFile(E, (DGCell*)0);
  for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it) {
    mEntity* ent = *it;
    FunctionSpace* fs;
    if (dim == 2) fs = new OrthogonalTriangleFunctionSpace(P.order);
    else fs = new OrthogonalTetFunctionSpace(P.order);
    ConstantMeshMapping* map = new ConstantMeshMapping(ent);
    DGCell* cell = new DGCell(law, ent, fs, 0, map, &gi);
    ent->setCell(cell);
    DOF += m * fs->size();
    cell->L2ProjInitial(law->getFarField());
    cell->computeMean();
    cell->ZeroRHS();
    byFile[cellIndex(mc, ent)] = cell;
  }
  for (mMesh::iter it = mesh->begin(dim - 1); it != mesh->end(dim - 1); ++it) {
    mEntity* ent = *it;
    DGBoundaryCell* bc = new DGBoundaryCell(ent, new MeshMapping(ent), &gi);
    ent->setCell(bc);
  }
  // partner traces of periodic faces (DGAnalysis::setPeriodicBC, DGPref.cc:1389-1403)
  for (mMesh::iter it = mesh->begin(dim - 1); it != mesh->end(dim - 1); ++it) {
    mEntity* ent = *it;
    const int id = ent->getClassification()->getId();
    if ((id == 510 || id == 610) && ent->getAttachedEntity(TYPE_CELL))
      ((DGBoundaryCell*)ent->getCell())->setPeriodicBC();
  }
  const int Np = byFile[0]->fSize;

  if (!P.conn.empty()) {
    FILE* f = fopen(P.conn.c_str(), "w");
    for (mMesh::iter it = mesh->begin(dim - 1); it != mesh->end(dim - 1); ++it) {
      mEntity* ent = *it;
      DGBoundaryCell* bc = (DGBoundaryCell*)ent->getCell();
      std::vector<int> fv;
      for (int i = 0; i < ent->size(0); ++i) fv.push_back(ent->get(0, i)->getId());
      std::sort(fv.begin(), fv.end());
      mEntity* L = bc->getLeft();
      mEntity* R = bc->getRight();
      int eL = cellIndex(mc, L), eR = R ? cellIndex(mc, R) : -1;
      int lfL = localFace(L, ent), lfR = R ? localFace(R, ent) : -1;
      double meas = 0;
      for (int q = 0; q < bc->getNbPtGauss(); ++q) meas += bc->pt(q)->JacTimesWeight;
      mVector& n = bc->pt(0)->n;
      for (size_t i = 0; i < fv.size(); ++i) fprintf(f, "%d ", fv[i]);
      fprintf(f, "%d %d %d %d %d %.17g %.17g %.17g %.17g\n", eL, eR, lfL, lfR,
              ent->getClassification()->getId(), n(0), n(1), n(2), meas);
    }
    fclose(f);
  }

  RungeKuttaTVD3 rk(mesh, 0, m, DOF);
#ifdef DGP_REF_LTS
  RungeKuttaTVD2adaptive* lts = 0;
  int ltsBins = 0;
  if (P.lts) {
    ltsBins = ltsSortCells(mesh, dim);
    lts = new RungeKuttaTVD2adaptive(mesh, 0, m, DOF);
    if (!P.bins.empty()) {
      std::vector<int> bin(E, -1), role(E, -1);
      for (int b = 0; b < ltsBins; ++b) {
        for (mMesh::iter it = mesh->beginBin(b, dim); it != mesh->endBin(b, dim); ++it)
          bin[cellIndex(mc, *it)] = b, role[cellIndex(mc, *it)] = 0;
        for (mMesh::iter it = mesh->beginLargeOnInterface(b, dim); it != mesh->endLargeOnInterface(b, dim); ++it)
          bin[cellIndex(mc, *it)] = b, role[cellIndex(mc, *it)] = 1;
        for (mMesh::iter it = mesh->beginSmallOnInterface(b, dim); it != mesh->endSmallOnInterface(b, dim); ++it)
          bin[cellIndex(mc, *it)] = b + 1, role[cellIndex(mc, *it)] = 2;
      }
      FILE* f = fopen(P.bins.c_str(), "w");
      fprintf(f, "%d %d\n", E, ltsBins);
      for (int e = 0; e < E; ++e) fprintf(f, "%d %d\n", bin[e], role[e]);
      fclose(f);
    }
  }
#endif

  double TACT = 0.0;
  if (!P.ckptIn.empty()) {
    std::ifstream is(P.ckptIn.c_str());
    int iter = 0, nd = 0, nvol = 0, nbnd = 0, order = 0;
    is >> TACT >> iter >> nd >> nvol >> nbnd;
    for (int i = 0; i < nvol; ++i) {
      mEntity* ent = mesh->readMEntity(is);
      is >> order;
      DGCell* cell = (DGCell*)ent->getCell();
      cell->read(is);
      cell->computeMean();
    }
  }

  // The P0 fallback as DGAnalysis's serial assembly applies it
  // (DGAnalysis.cc:392-417): every volume and face contribution first,
  // collecting the cells with a non-physical trace, then DGCell::setToZero on
  // each of them.  The state: the projection with the listed cells' first
  // field pushed away from its mean (modes k >= 1 += a|c_0|, the sign
  // alternating over the list).  Writes "E m Np n", the n zeroed cells (file
  // order, as listed), the perturbed state, the state after the fallback
  // (the volume correction zeroes cells too) and the right-hand side.
  if (!P.p0rhs.empty()) {
    std::vector<int> pert;
    for (const char* c = P.p0cells.c_str(); *c;) {
      pert.push_back(atoi(c));
      while (*c && *c != ',') ++c;
      if (*c == ',') ++c;
    }
    for (size_t k = 0; k < pert.size(); ++k) {
      DGCell* cell = byFile[pert[k]];
      const double a = (k % 2 ? -1.0 : 1.0) * P.p0amp * fabs(cell->theFieldsCoefficients->get(0, 0));
      for (int j = 1; j < Np; ++j) cell->theFieldsCoefficients->get(0, j) += a;
      cell->computeMean();
    }
    std::vector<double> perturbed((size_t)E * m * Np);
    for (int e = 0; e < E; ++e)
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < Np; ++j) perturbed[((size_t)e * m + i) * Np + j] = byFile[e]->theFieldsCoefficients->get(i, j);
    for (int e = 0; e < E; ++e) byFile[e]->ZeroRHS();
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it)
      ((DGCell*)(*it)->getCell())->computeVolumeContribution(0.0);
    std::vector<DGCell*> zero;
    for (mMesh::iter it = mesh->begin(dim - 1); it != mesh->end(dim - 1); ++it) {
      DGBoundaryCell* bc = (DGBoundaryCell*)(*it)->getCell();
      const int np = bc->computeBoundaryContributions(0.0);
      if (np == 1 || np == 3) zero.push_back((DGCell*)bc->getLeftCell());
      if (np == 2 || np == 3) zero.push_back((DGCell*)bc->getRightCell());
    }
    for (size_t k = 0; k < zero.size(); ++k) zero[k]->setToZero(0.0);
    FILE* f = fopen(P.p0rhs.c_str(), "w");
    fprintf(f, "%d %d %d %d\n", E, m, Np, (int)zero.size());
    for (size_t k = 0; k < zero.size(); ++k) fprintf(f, "%d ", cellIndex(mc, zero[k]->getMeshEntity()));
    fprintf(f, "\n");
    for (int e = 0; e < E; ++e) {
      for (int j = 0; j < m * Np; ++j) fprintf(f, "%.17g ", perturbed[(size_t)e * m * Np + j]);
      fprintf(f, "\n");
    }
    for (int e = 0; e < E; ++e) {
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < Np; ++j) fprintf(f, "%.17g ", byFile[e]->theFieldsCoefficients->get(i, j));
      fprintf(f, "\n");
    }
    for (int e = 0; e < E; ++e) {
      for (int j = 0; j < m * Np; ++j) fprintf(f, "%.17g ", byFile[e]->theRightHandSide[j]);
      fprintf(f, "\n");
    }
    fclose(f);
    return 0;
  }

  if (!P.rhs.empty()) {
    rk.assembleVolume(0.0);
    rk.assembleBoundary(0.0);
    FILE* f = fopen(P.rhs.c_str(), "w");
    fprintf(f, "%d %d %d\n", E, m, Np);
    for (int e = 0; e < E; ++e) {
      for (int j = 0; j < m * Np; ++j) fprintf(f, "%.17g ", byFile[e]->theRightHandSide[j]);
      fprintf(f, "\n");
    }
    fclose(f);
    for (int e = 0; e < E; ++e) byFile[e]->ZeroRHS();
  }

#ifdef DGP_GPU_INTEGRATOR
  GpuTimeIntegrator* gti = 0;
  if (P.gpu) {
    // the same case as the reference law, in the library's parameter layout
    double prm[DGP_NPARAMS] = {0};
    int kind = DGP_LAW_SCALAR, flux = DGP_FLUX_UPWIND, field = DGP_FIELD_GAUSS;
    prm[0] = P.ax; prm[1] = P.ay; prm[2] = P.az;
    prm[3] = P.cx; prm[4] = P.cy; prm[5] = P.cz;
    prm[6] = P.s; prm[7] = P.gamma; prm[8] = P.beta; prm[9] = P.amp; prm[10] = 1.0;
    if (P.caseName == "gauss3d") field = DGP_FIELD_GAUSS3D;
    else if (P.caseName == "vortex") {
      kind = DGP_LAW_EULER2D;
      flux = P.flux == "roe" ? DGP_FLUX_ROE : DGP_FLUX_GODUNOV;
      field = DGP_FIELD_VORTEX;
      prm[0] = 1.0; prm[1] = 1.0; prm[2] = 0.0;
      prm[3] = P.vx0; prm[4] = P.vy0; prm[5] = 0.0;
    } else if (P.caseName == "pulse3d") {
      kind = DGP_LAW_EULER3D;
      flux = DGP_FLUX_GODUNOV;
      field = DGP_FIELD_PULSE3D;
    } else if (P.caseName == "sine") {
      kind = DGP_LAW_BURGERS2D;
      flux = DGP_FLUX_CENTRAL;
      field = DGP_FIELD_SINE;
    } else if (P.caseName == "tm2d") {
      kind = DGP_LAW_MAXWELL2D;
      flux = DGP_FLUX_UPWIND;
      field = DGP_FIELD_TM2D;
      prm[10] = P.L;
    }
    // the law and flux ids come from the reference law object itself
    // (GpuConservationLaw); they must agree with this driver's case table
    int mk = -1, mf = -1;
    if (!GpuConservationLaw::map(law, &mk, &mf) || mk != kind || mf != flux) {
      fprintf(stderr, "GpuConservationLaw maps this law to (%d, %d), the case table says (%d, %d)\n", mk, mf,
              kind, flux);
      return 2;
    }
    gti = new GpuTimeIntegrator(mesh, law, P.order, P.mesh.c_str(), byFile, field, prm);
  }
#endif
  FILE* fs = P.state.empty() ? 0 : fopen(P.state.c_str(), "w");
  FILE* fl = P.log.empty() ? 0 : fopen(P.log.c_str(), "w");
  if (fs) fprintf(fs, "%d %d %d\n", E, m, Np);
  struct Dump {
    static void state(FILE* f, int step, double t, std::vector<DGCell*>& cells, int m, int Np) {
      fprintf(f, "step %d %.17g\n", step, t);
      for (size_t e = 0; e < cells.size(); ++e) {
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < Np; ++j) fprintf(f, "%.17g ", cells[e]->theFieldsCoefficients->get(i, j));
        fprintf(f, "\n");
      }
    }
  };
  if (fs) Dump::state(fs, 0, 0.0, byFile, m, Np);

  const int nsteps = P.bench > 0 ? P.bench + P.warmup : P.steps;
  double t0 = nowSec();
  for (int step = 1; nsteps <= 0 || step <= nsteps; ++step) {
    if (P.bench > 0 && step == P.warmup + 1) t0 = nowSec();
    if (P.tend > 0 && TACT >= P.tend) break;
    if (nsteps <= 0 && P.tend <= 0) break;
    // CFL time step (DGAnalysis.cc:514-548, mode 0)
    double dt = 500;
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it)
      ((DGCell*)(*it)->getCell())->adaptTimeStep(P.cfl, dt);
#ifdef DGP_REF_LTS
    if (lts) dt *= pow(2., ltsBins - 1);  // DGAnalysis.cc:590
#endif
    if (P.tend > 0) {
      int N = (int)ceil((P.tend - TACT) / dt);
      dt = (P.tend - TACT) / N;
    }
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it)
      ((DGCell*)(*it)->getCell())->setTimeStep(dt);
#if defined(DGP_GPU_INTEGRATOR)
    double resid = gti ? gti->advanceInTime(TACT, dt) : rk.advanceInTime(TACT, dt);
#elif defined(DGP_REF_LTS)
    double resid = lts ? lts->advanceInTime(TACT, dt) : rk.advanceInTime(TACT, dt);
#else
    double resid = rk.advanceInTime(TACT, dt);
#endif
    TACT += dt;
    if (fl) fprintf(fl, "%d %.17g %.17g %.17g\n", step, dt, TACT, resid);
    if (fs && (step % P.every == 0)) Dump::state(fs, step, TACT, byFile, m, Np);
  }
  double elapsed = nowSec() - t0;
  if (!P.ckptOut.empty()) {
    std::ofstream data(P.ckptOut.c_str());
    data.precision(16);
    data << TACT << "\n";
    data << (nsteps > 0 ? nsteps : 0) << "\n";
    data << dim << " " << mesh->size(dim) << " " << mesh->size(dim - 1) << "\n";
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it) {
      mesh->writeMEntity(data, *it);
      ((DGCell*)(*it)->getCell())->write(data);
    }
    for (mMesh::iter it = mesh->begin(dim - 1); it != mesh->end(dim - 1); ++it) mesh->writeMEntity(data, *it);
  }
  if (!P.stateBin.empty()) {
    FILE* f = fopen(P.stateBin.c_str(), "wb");
    std::vector<double> row(m * Np);
    for (int e = 0; e < E; ++e) {
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < Np; ++j) row[i * Np + j] = byFile[e]->theFieldsCoefficients->get(i, j);
      fwrite(row.data(), sizeof(double), row.size(), f);
    }
    fclose(f);
  }
  if (!P.norms.empty()) {
    // DGAnalysis::ExactError, LinfError, PressureError, entropyErrorL1,
    // pressureErrorL2, densityErrorL2, entropyErrorL2 (DGPref.cc:249-381) at
    // the final time, summed over the cells as there (one thread); the
    // pressure and entropy norms for the 2D Euler case only
    double l1 = 0.0, linf = 0.0, pl1 = 0.0, el1 = 0.0, pl2 = 0.0, dl2 = 0.0, el2 = 0.0;
    const bool euler = P.caseName == "vortex";
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it) {
      DGCell* cell = (DGCell*)(*it)->getCell();
      l1 += cell->L1exact(TACT);
      const double li = cell->LinfError(TACT);
      if (linf < li) linf = li;
      dl2 += cell->densityErrorL2(TACT);
      if (euler) {
        pl1 += cell->L1exactPressure(TACT);
        el1 += cell->entropyErrorL1_2D(TACT);
        pl2 += cell->pressureErrorL2(TACT);
        el2 += cell->entropyErrorL2_2D(TACT);
      }
    }
    FILE* f = fopen(P.norms.c_str(), "w");
    fprintf(f, "t %.17g\nExactError %.17g\nLinfError %.17g\ndensityErrorL2 %.17g\n", TACT, l1, linf, sqrt(dl2));
    if (euler)
      fprintf(f, "PressureError %.17g\nentropyErrorL1 %.17g\npressureErrorL2 %.17g\nentropyErrorL2 %.17g\n", pl1,
              el1, sqrt(pl2), sqrt(el2));
    fclose(f);
  }
  if (!P.probeOut.empty()) {
    // DGPointSensor::eval (DGSensor.cc:170-186) at the final time: the field
    // values at each point from DGCell::inCell (DGCell.cc:1499-1521) of the
    // first cell (file order) that contains it; "i cell v_0 .. v_m-1", cell -1
    // (and no values) for a point outside the mesh
    FILE* f = fopen(P.probeOut.c_str(), "w");
    int i = 0;
    for (const char* c = P.probePts.c_str(); *c; ++i) {
      double x[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < 3 && *c; ++k) {
        x[k] = atof(c);
        while (*c && *c != ',' && *c != ';') ++c;
        if (*c == ',') ++c;
      }
      if (*c == ';') ++c;
      double val[MaxNbEqn];
      int found = -1;
      for (int e = 0; e < E && found < 0; ++e)
        if (byFile[e]->inCell(mPoint(x[0], x[1], x[2]), val)) found = e;
      fprintf(f, "%d %d", i, found);
      if (found >= 0)
        for (int k = 0; k < m; ++k) fprintf(f, " %.17g", val[k]);
      fprintf(f, "\n");
    }
    fclose(f);
  }
  if (!P.l2.empty()) {
    // DGAnalysis::densityErrorL2 (DGPref.cc:370-380): sqrt of the sum over
    // cells of DGCell::densityErrorL2 (DGError.cc:805-826) at the final time;
    // the total first, then each cell's squared error in file order
    double total = 0.0;
    std::vector<double> per(E, 0.0);
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it) {
      DGCell* cell = (DGCell*)(*it)->getCell();
      const double v = cell->densityErrorL2(TACT);
      per[cellIndex(mc, *it)] = v;
      total += v;
    }
    FILE* f = fopen(P.l2.c_str(), "w");
    fprintf(f, "%.17g %.17g\n", TACT, sqrt(total));
    for (int e = 0; e < E; ++e) fprintf(f, "%.17g\n", per[e]);
    fclose(f);
  }
  if (!P.barth.empty()) {
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it) {
      DGCell* cell = (DGCell*)(*it)->getCell();
      cell->computeMean();
      cell->details->allSubs.clear();
      for (int k = 0; k < cell->theMeshEntity->size(dim - 1); ++k)
        cell->details->allSubs.push_back(cell->theMeshEntity->get(dim - 1, k));
    }
    DGBarthLimiter barth;
    for (mMesh::iter it = mesh->begin(dim); it != mesh->end(dim); ++it)
      barth.limit((DGCell*)(*it)->getCell(), TACT);
    FILE* f = fopen(P.barth.c_str(), "w");
    fprintf(f, "%d %d %d\n", E, m, Np);
    for (int e = 0; e < E; ++e) {
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < Np; ++j) fprintf(f, "%.17g ", byFile[e]->theFieldsCoefficients->get(i, j));
      for (int i = 0; i < m; ++i) fprintf(f, "%.17g ", byFile[e]->details->limSlope[i]);
      fprintf(f, "\n");
    }
    fclose(f);
  }
  if (fs) fclose(fs);
  if (fl) fclose(fl);
  if (P.bench > 0)
    printf("BENCH elements=%d fields=%d modes=%d steps=%d threads=%u seconds=%.6f "
           "dof_stage_per_s=%.6e\n", E, m, Np, P.bench, numThreads, elapsed,
           (double)E * m * Np * 3.0 * P.bench / elapsed);
  return 0;
}
