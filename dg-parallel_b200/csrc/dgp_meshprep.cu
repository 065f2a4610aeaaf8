// Face matching on the GPU (mMesh::createCellBoundaries / createConnections,
// mMesh.cc:321-378, and DGBoundaryCell::init's frame, orientation and normal,
// DGCell.cc:423-555), producing the same faces as the host matching in
// dgp_host.cpp:
//   1. every (cell, local face) writes a packed key of its sorted vertex
//      indices and the value cell * nlf + lf;
//   2. a stable radix sort of the pairs groups each face's one or two entries
//      (ties keep (cell, lf) ascending, as the host's sort);
//   3. group heads and an exclusive scan number the faces;
//   4. one thread per face: left / right by the reference's entity order
//      (mEntity::lessthan: int-truncated sum of glibc rand() of the vertex ids,
//      then the sorted ids), the left cell's face frame, the right cell's
//      orientation, the unit normal (outward from the left cell) and measure,
//      with single-rounding arithmetic in the host's operation order.
// A third entry with the same key flags a non-manifold face.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_host.h"

namespace dgp {
namespace {

__constant__ int c_tri_face[3][2] = {{0, 1}, {1, 2}, {2, 0}};
__constant__ int c_tet_face[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
__constant__ int c_perm3[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

__device__ __forceinline__ int local_vertex(int dim, int lf, int k) {
  return dim == 2 ? c_tri_face[lf][k] : c_tet_face[lf][k];
}

template <int N>
__device__ __forceinline__ void sort_small(int* a) {
#pragma unroll
  for (int i = 1; i < N; ++i)
#pragma unroll
    for (int j = i; j > 0; --j)
      if (a[j - 1] > a[j]) {
        const int t = a[j - 1];
        a[j - 1] = a[j];
        a[j] = t;
      }
}

__global__ void face_keys_kernel(const int* cv, int E, int dim, unsigned long long* keys, int* vals) {
  const int nlf = dim + 1, nvc = dim + 1;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)E * nlf) return;
  const int e = static_cast<int>(i / nlf), lf = static_cast<int>(i - (long long)e * nlf);
  unsigned long long key;
  if (dim == 2) {
    int v[2] = {cv[e * nvc + local_vertex(2, lf, 0)], cv[e * nvc + local_vertex(2, lf, 1)]};
    sort_small<2>(v);
    key = ((unsigned long long)v[0] << 32) | (unsigned long long)v[1];
  } else {
    int v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] = cv[e * nvc + local_vertex(3, lf, k)];
    sort_small<3>(v);
    key = ((unsigned long long)v[0] << 42) | ((unsigned long long)v[1] << 21) | (unsigned long long)v[2];
  }
  keys[i] = key;
  vals[i] = static_cast<int>(i);
}

__global__ void face_heads_kernel(const unsigned long long* keys, long long n, int* head, int* bad) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
  if (i + 2 < n && keys[i] == keys[i + 2]) atomicExch(bad, 1);
}

// mEntity::lessthan on two cells: key sum, then sorted vertex ids
__device__ bool cell_less(int a, int b, const int* cv, int nvc, const unsigned* rk, const int* vid) {
  unsigned long long sa = 0, sb = 0;
  for (int k = 0; k < nvc; ++k) {
    sa += rk[cv[a * nvc + k]];
    sb += rk[cv[b * nvc + k]];
  }
  const int ka = static_cast<int>(static_cast<unsigned>(sa)), kb = static_cast<int>(static_cast<unsigned>(sb));
  if (ka != kb) return ka < kb;
  int va[4], vb[4];
  for (int k = 0; k < nvc; ++k) {
    va[k] = vid[cv[a * nvc + k]];
    vb[k] = vid[cv[b * nvc + k]];
  }
  if (nvc == 3) {
    sort_small<3>(va);
    sort_small<3>(vb);
  } else {
    sort_small<4>(va);
    sort_small<4>(vb);
  }
  for (int k = 0; k < nvc; ++k)
    if (va[k] != vb[k]) return va[k] < vb[k];
  return false;
}

struct FaceOut {
  int* fv;
  int* eL;
  int* eR;
  int* lfL;
  int* lfR;
  int* rperm;
  double* fn;
  double* fmeas;
  int* bad;
};

__global__ void face_build_kernel(const unsigned long long* keys, const int* vals, const int* head, const int* fid,
                                  long long n, const int* cv, const double* X, const unsigned* rk, const int* vid,
                                  int dim, FaceOut o) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  const int nlf = dim + 1, nvc = dim + 1, nfv = dim;
  const int f = fid[i];
  int a = vals[i] / nlf, la = vals[i] - (vals[i] / nlf) * nlf, b = -1, lb = -1;
  if (i + 1 < n && !head[i + 1]) {
    b = vals[i + 1] / nlf;
    lb = vals[i + 1] - b * nlf;
    if (cell_less(b, a, cv, nvc, rk, vid)) {
      int t = a;
      a = b;
      b = t;
      t = la;
      la = lb;
      lb = t;
    }
  }
  int frame[3];
  for (int k = 0; k < nfv; ++k) frame[k] = cv[a * nvc + local_vertex(dim, la, k)];
  int perm = 0;
  if (b >= 0) {
    int rv[3];
    for (int k = 0; k < nfv; ++k) rv[k] = cv[b * nvc + local_vertex(dim, lb, k)];
    if (dim == 2) {
      perm = (rv[0] == frame[0]) ? 0 : 1;
    } else {
      int pos[3] = {-1, -1, -1};
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          if (rv[k] == frame[l]) pos[k] = l;
      perm = -1;
      for (int p = 0; p < 6; ++p)
        if (c_perm3[p][0] == pos[0] && c_perm3[p][1] == pos[1] && c_perm3[p][2] == pos[2]) perm = p;
      if (perm < 0) {
        atomicExch(o.bad, 2);
        perm = 0;
      }
    }
  }
  for (int k = 0; k < nfv; ++k) o.fv[(size_t)f * nfv + k] = frame[k];
  o.eL[f] = a;
  o.eR[f] = b;
  o.lfL[f] = la;
  o.lfR[f] = lb;
  o.rperm[f] = perm;
  // unit normal outward from the left cell, and the face measure
  const double* pa = X + 3 * (size_t)frame[0];
  const double* pb = X + 3 * (size_t)frame[1];
  int opp = -1;
  for (int k = 0; k < nvc; ++k) {
    const int v = cv[a * nvc + k];
    bool on = false;
    for (int j = 0; j < nfv; ++j) on |= (frame[j] == v);
    if (!on) opp = v;
  }
  const double* po = X + 3 * (size_t)opp;
  double nn[3], meas;
  if (dim == 2) {
    const double t0 = __dsub_rn(pb[0], pa[0]), t1 = __dsub_rn(pb[1], pa[1]);
    meas = __dsqrt_rn(__dadd_rn(__dmul_rn(t0, t0), __dmul_rn(t1, t1)));
    nn[0] = __ddiv_rn(t1, meas);
    nn[1] = __ddiv_rn(-t0, meas);
    nn[2] = 0.0;
  } else {
    const double* pc = X + 3 * (size_t)frame[2];
    const double u[3] = {__dsub_rn(pb[0], pa[0]), __dsub_rn(pb[1], pa[1]), __dsub_rn(pb[2], pa[2])};
    const double v[3] = {__dsub_rn(pc[0], pa[0]), __dsub_rn(pc[1], pa[1]), __dsub_rn(pc[2], pa[2])};
    const double cr[3] = {__dsub_rn(__dmul_rn(u[1], v[2]), __dmul_rn(u[2], v[1])),
                          __dsub_rn(__dmul_rn(u[2], v[0]), __dmul_rn(u[0], v[2])),
                          __dsub_rn(__dmul_rn(u[0], v[1]), __dmul_rn(u[1], v[0]))};
    const double l = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(cr[0], cr[0]), __dmul_rn(cr[1], cr[1])), __dmul_rn(cr[2], cr[2])));
    for (int k = 0; k < 3; ++k) nn[k] = __ddiv_rn(cr[k], l);
    meas = __dmul_rn(0.5, l);
  }
  const double d = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(po[0], pa[0]), nn[0]),
                                       __dmul_rn(__dsub_rn(po[1], pa[1]), nn[1])),
                             __dmul_rn(__dsub_rn(po[2], pa[2]), nn[2]));
  if (d > 0)
    for (int k = 0; k < 3; ++k) nn[k] = -nn[k];
  for (int k = 0; k < 3; ++k) o.fn[3 * (size_t)f + k] = nn[k];
  o.fmeas[f] = meas;
}

// device buffers freed on every return path
struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  cudaError_t get(T** out, size_t n) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, (n ? n : 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(v);
    *out = static_cast<T*>(v);
    return e;
  }
};

}  // namespace

int build_faces_gpu(HostMesh& m, std::string& err) {
  const int dim = m.dim, nlf = m.nlf, nfv = m.nfv;
  const long long n = static_cast<long long>(m.E) * nlf;
  const size_t nv = m.vid.size();
  if ((dim == 3 && nv >= (1u << 21)) || n >= (1ll << 31)) return DGP_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DGP_ERR_UNSUPPORTED;
  std::vector<unsigned> rk(nv);
  for (size_t i = 0; i < nv; ++i) rk[i] = glibc_rand_first(static_cast<uint32_t>(m.vid[i]));
  DevBufs B;
  int *d_cv, *d_vid, *d_vals, *d_vals2, *d_head, *d_fid, *d_bad;
  unsigned long long *d_keys, *d_keys2;
  unsigned* d_rk;
  double* d_X;
  auto ck = [&](cudaError_t e) {
    if (e != cudaSuccess) err = std::string("GPU face matching: ") + cudaGetErrorString(e);
    return e == cudaSuccess;
  };
  if (!ck(B.get(&d_cv, m.cv.size())) || !ck(B.get(&d_vid, nv)) || !ck(B.get(&d_rk, nv)) ||
      !ck(B.get(&d_X, m.X.size())) || !ck(B.get(&d_keys, n)) || !ck(B.get(&d_keys2, n)) ||
      !ck(B.get(&d_vals, n)) || !ck(B.get(&d_vals2, n)) || !ck(B.get(&d_head, n)) || !ck(B.get(&d_fid, n)) ||
      !ck(B.get(&d_bad, 1)))
    return DGP_ERR_CUDA;
  if (!ck(cudaMemcpy(d_cv, m.cv.data(), m.cv.size() * 4, cudaMemcpyHostToDevice)) ||
      !ck(cudaMemcpy(d_vid, m.vid.data(), nv * 4, cudaMemcpyHostToDevice)) ||
      !ck(cudaMemcpy(d_rk, rk.data(), nv * 4, cudaMemcpyHostToDevice)) ||
      !ck(cudaMemcpy(d_X, m.X.data(), m.X.size() * 8, cudaMemcpyHostToDevice)) ||
      !ck(cudaMemset(d_bad, 0, 4)))
    return DGP_ERR_CUDA;
  const int T = 256;
  const int G = static_cast<int>((n + T - 1) / T);
  face_keys_kernel<<<G, T>>>(d_cv, m.E, dim, d_keys, d_vals);
  // stable radix sort on the significant key bits
  const int bits = dim == 2 ? 64 : 63;
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_keys, d_keys2, d_vals, d_vals2, static_cast<int>(n), 0,
                                  bits);
  void* d_tmp;
  if (!ck(B.get(reinterpret_cast<unsigned char**>(&d_tmp), tmp_bytes))) return DGP_ERR_CUDA;
  if (!ck(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_keys, d_keys2, d_vals, d_vals2, static_cast<int>(n),
                                          0, bits)))
    return DGP_ERR_CUDA;
  face_heads_kernel<<<G, T>>>(d_keys2, n, d_head, d_bad);
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_head, d_fid, static_cast<int>(n));
  void* d_scan;
  if (!ck(B.get(reinterpret_cast<unsigned char**>(&d_scan), scan_bytes))) return DGP_ERR_CUDA;
  if (!ck(cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_head, d_fid, static_cast<int>(n))))
    return DGP_ERR_CUDA;
  int last_fid = 0, last_head = 0, bad = 0;
  if (!ck(cudaMemcpy(&last_fid, d_fid + n - 1, 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(&last_head, d_head + n - 1, 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(&bad, d_bad, 4, cudaMemcpyDeviceToHost)))
    return DGP_ERR_CUDA;
  if (bad) {
    err = "non-manifold face shared by more than two cells";
    return DGP_ERR_IO;
  }
  const int F = last_fid + last_head;
  FaceOut o;
  if (!ck(B.get(&o.fv, static_cast<size_t>(F) * nfv)) || !ck(B.get(&o.eL, F)) || !ck(B.get(&o.eR, F)) ||
      !ck(B.get(&o.lfL, F)) || !ck(B.get(&o.lfR, F)) || !ck(B.get(&o.rperm, F)) ||
      !ck(B.get(&o.fn, static_cast<size_t>(F) * 3)) || !ck(B.get(&o.fmeas, F)))
    return DGP_ERR_CUDA;
  o.bad = d_bad;
  face_build_kernel<<<G, T>>>(d_keys2, d_vals2, d_head, d_fid, n, d_cv, d_X, d_rk, d_vid, dim, o);
  if (!ck(cudaGetLastError()) || !ck(cudaDeviceSynchronize())) return DGP_ERR_CUDA;
  if (!ck(cudaMemcpy(&bad, d_bad, 4, cudaMemcpyDeviceToHost))) return DGP_ERR_CUDA;
  if (bad) {
    err = "inconsistent face vertices";
    return DGP_ERR_IO;
  }
  m.F = F;
  m.fv.resize(static_cast<size_t>(F) * nfv);
  m.eL.resize(F);
  m.eR.resize(F);
  m.lfL.resize(F);
  m.lfR.resize(F);
  m.rperm.resize(F);
  m.fn.resize(static_cast<size_t>(F) * 3);
  m.fmeas.resize(F);
  if (!ck(cudaMemcpy(m.fv.data(), o.fv, m.fv.size() * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.eL.data(), o.eL, F * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.eR.data(), o.eR, F * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.lfL.data(), o.lfL, F * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.lfR.data(), o.lfR, F * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.rperm.data(), o.rperm, F * 4, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.fn.data(), o.fn, m.fn.size() * 8, cudaMemcpyDeviceToHost)) ||
      !ck(cudaMemcpy(m.fmeas.data(), o.fmeas, F * 8, cudaMemcpyDeviceToHost)))
    return DGP_ERR_CUDA;
  return DGP_OK;
}

}  // namespace dgp
