// Point and line probes on the device (DGPointSensor / DGLineSensor,
// DGSensor.cc:88-186, with the point location of DGCell::inCell).
//
// The points are located once on the host (uniform-grid PointLocator); their
// cells and basis values live on the device.  dgp_probe_eval evaluates every
// field at every point of the current state; a recorder samples inside every
// step of dgp_run / dgp_step (the kernel is part of the captured step graph),
// so a run records its time series without a host round trip per sample.
#include <cmath>
#include <limits>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_handles.h"

namespace {

using dgp::TimeCtl;

// values[p][j] = sum_k phi[p][k] c[cell p][j][k] (k in order); NaN outside
__global__ void probe_eval_kernel(const int* cell, const double* phi, const double* C, int n, int M, int NP,
                                  double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * M) return;
  const int p = i / M, j = i - p * M;
  const int e = cell[p];
  if (e < 0) {
    out[i] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  const double* c = C + ((size_t)e * M + j) * NP;
  const double* ph = phi + (size_t)p * NP;
  double v = 0.0;
  for (int k = 0; k < NP; ++k) v += ph[k] * c[k];
  out[i] = v;
}

// the recorder: after a step, sample s = steps / every - 1 when steps is a
// multiple of every (a step that did not run -- the run is done -- leaves
// steps and the state unchanged, so writing the same sample again is harmless)
__global__ void probe_record_kernel(const int* cell, const double* phi, const double* C, int n, int M, int NP,
                                    const TimeCtl* ctl, int every, int max_samples, double* rec, double* rec_t,
                                    int* rec_n) {
  const int steps = ctl->steps;
  if (steps <= 0 || steps % every != 0) return;
  const int s = steps / every - 1;
  if (s >= max_samples) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n * M) {
    const int p = i / M, j = i - p * M;
    const int e = cell[p];
    double v = __longlong_as_double(0x7ff8000000000000ll);
    if (e >= 0) {
      const double* c = C + ((size_t)e * M + j) * NP;
      const double* ph = phi + (size_t)p * NP;
      v = 0.0;
      for (int k = 0; k < NP; ++k) v += ph[k] * c[k];
    }
    rec[(size_t)s * n * M + i] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    rec_t[s] = ctl->t;
    atomicMax(rec_n, s + 1);
  }
}

int probe_alloc(dgp_probe p, void** ptr, size_t bytes) {
  if (cudaMalloc(ptr, bytes ? bytes : 1) != cudaSuccess) return dgp::fail(DGP_ERR_NOMEM, "probe allocation failed");
  p->allocs.push_back(*ptr);
  return DGP_OK;
}

}  // namespace

namespace dgp {

// locate points on the solver's (single) mesh: internal cells and basis values
int locate_points(dgp_solver s, int n, const double* points, std::vector<int>& cell, std::vector<double>& phi) {
  if (s->meshes.size() != 1) return fail(DGP_ERR_UNSUPPORTED, "points are located on a single solver's mesh");
  const HostMesh& m = s->meshes[0];
  if (!s->locator_ready) {
    s->locator.build(m);
    s->locator_ready = true;
  }
  const int dim = m.dim, NP = s->b.NP;
  cell.assign(n, -1);
  phi.assign(static_cast<size_t>(n) * NP, 0.0);
  for (int r = 0; r < n; ++r) {
    double x[3] = {0, 0, 0}, xi[3];
    for (int k = 0; k < dim; ++k) x[k] = points[static_cast<size_t>(r) * dim + k];
    const int e = s->locator.locate(x, xi);
    if (e < 0) continue;
    cell[r] = s->f2i[e];
    basis_eval(s->tab, xi, &phi[static_cast<size_t>(r) * NP]);
  }
  return DGP_OK;
}

// inside launch_step: every recorder of the solver samples the new state
void launch_probe_recorders(dgp_solver s) {
  for (dgp_probe_s* p : s->probes) {
    if (p->every <= 0 || p->n == 0) continue;
    const int M = s->b.M, NP = s->b.NP;
    const int grid = (p->n * M + 127) / 128;
    probe_record_kernel<<<grid, 128, 0, s->stream>>>(p->cell, p->phi, static_cast<const double*>(s->b.C), p->n, M,
                                                     NP, s->b.ctl, p->every, p->max_samples, p->rec, p->rec_t,
                                                     p->rec_n);
  }
}

// a run starts its recorders from sample 0
int reset_probe_recorders(dgp_solver s) {
  for (dgp_probe_s* p : s->probes)
    if (p->every > 0) DGP_CUDA(cudaMemsetAsync(p->rec_n, 0, sizeof(int), s->stream));
  return DGP_OK;
}

}  // namespace dgp

using namespace dgp;

extern "C" {

int dgp_probe_create(dgp_solver s, int n, const double* points, dgp_probe* out, int* found) {
  if (!s || n <= 0 || !points || !out) return fail(DGP_ERR_INVALID, "bad argument");
  if (s->b.ninst) return fail(DGP_ERR_UNSUPPORTED, "probes are set on a single solver");
  DGP_CUDA(cudaSetDevice(s->device));
  std::vector<int> cell;
  std::vector<double> phi;
  if (int rc = locate_points(s, n, points, cell, phi)) return rc;
  dgp_probe p = new dgp_probe_s;
  p->s = s;
  p->n = n;
  for (int r = 0; r < n; ++r) {
    p->found += cell[r] >= 0;
    if (found) found[r] = cell[r] >= 0 ? 1 : 0;
  }
  const size_t M = s->b.M;
  int rc = DGP_OK;
  if ((rc = probe_alloc(p, reinterpret_cast<void**>(&p->cell), cell.size() * sizeof(int))) ||
      (rc = probe_alloc(p, reinterpret_cast<void**>(&p->phi), phi.size() * sizeof(double))) ||
      (rc = probe_alloc(p, reinterpret_cast<void**>(&p->vals), n * M * sizeof(double)))) {
    delete p;
    return rc;
  }
  cudaMemcpy(p->cell, cell.data(), cell.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(p->phi, phi.data(), phi.size() * sizeof(double), cudaMemcpyHostToDevice);
  s->probes.push_back(p);
  *out = p;
  return DGP_OK;
}

int dgp_probe_destroy(dgp_probe p) {
  if (!p) return DGP_OK;
  if (p->s) {
    dgp_solver s = p->s;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    if (p->every > 0) s->drop_graphs();
    for (size_t i = 0; i < s->probes.size(); ++i)
      if (s->probes[i] == p) {
        s->probes.erase(s->probes.begin() + i);
        break;
      }
  }
  delete p;
  return DGP_OK;
}

int dgp_probe_info(dgp_probe p, int* n, int* found) {
  if (!p) return fail(DGP_ERR_INVALID, "null probe");
  if (n) *n = p->n;
  if (found) *found = p->found;
  return DGP_OK;
}

int dgp_probe_eval(dgp_probe p, double* values) {
  if (!p || !values) return fail(DGP_ERR_INVALID, "null argument");
  dgp_solver s = p->s;
  if (!s) return fail(DGP_ERR_INVALID, "the probe's solver was destroyed");
  DGP_CUDA(cudaSetDevice(s->device));
  const int M = s->b.M, NP = s->b.NP;
  probe_eval_kernel<<<(p->n * M + 127) / 128, 128, 0, s->stream>>>(p->cell, p->phi,
                                                                   static_cast<const double*>(s->b.C), p->n, M, NP,
                                                                   p->vals);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaMemcpyAsync(values, p->vals, static_cast<size_t>(p->n) * M * sizeof(double),
                           cudaMemcpyDeviceToHost, s->stream));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}

int dgp_probe_record(dgp_probe p, int every, int max_samples) {
  if (!p || every < 0 || (every > 0 && max_samples <= 0)) return fail(DGP_ERR_INVALID, "bad argument");
  dgp_solver s = p->s;
  if (!s) return fail(DGP_ERR_INVALID, "the probe's solver was destroyed");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  if (every > 0 && max_samples > p->max_samples) {
    const size_t M = s->b.M;
    if (int rc = probe_alloc(p, reinterpret_cast<void**>(&p->rec), static_cast<size_t>(max_samples) * p->n * M * 8))
      return rc;
    if (int rc = probe_alloc(p, reinterpret_cast<void**>(&p->rec_t), static_cast<size_t>(max_samples) * 8)) return rc;
    if (!p->rec_n)
      if (int rc = probe_alloc(p, reinterpret_cast<void**>(&p->rec_n), sizeof(int))) return rc;
  }
  if (every > 0) {
    p->max_samples = std::max(p->max_samples, max_samples);
    DGP_CUDA(cudaMemset(p->rec_n, 0, sizeof(int)));
  }
  p->every = every;
  s->drop_graphs();  // the step graphs capture the recorders
  return DGP_OK;
}

int dgp_probe_samples(dgp_probe p, int* nsamples, double* times, double* values) {
  if (!p || !nsamples) return fail(DGP_ERR_INVALID, "null argument");
  dgp_solver s = p->s;
  if (!s) return fail(DGP_ERR_INVALID, "the probe's solver was destroyed");
  DGP_CUDA(cudaSetDevice(s->device));
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  int k = 0;
  if (p->rec_n) DGP_CUDA(cudaMemcpy(&k, p->rec_n, sizeof(int), cudaMemcpyDeviceToHost));
  k = std::min(k, p->max_samples);
  *nsamples = k;
  const size_t M = s->b.M;
  if (k > 0 && times) DGP_CUDA(cudaMemcpy(times, p->rec_t, static_cast<size_t>(k) * 8, cudaMemcpyDeviceToHost));
  if (k > 0 && values)
    DGP_CUDA(cudaMemcpy(values, p->rec, static_cast<size_t>(k) * p->n * M * 8, cudaMemcpyDeviceToHost));
  return DGP_OK;
}

}  // extern "C"
