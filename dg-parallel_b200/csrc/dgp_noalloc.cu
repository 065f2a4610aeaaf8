// dgp_rhs_noalloc: the assembled right-hand side without any device
// allocation.
//
// Who needs it: callers that cannot call cudaMalloc when they need a DG
// right-hand side -- a host code whose device memory is owned by another
// allocator (a framework caching allocator that has reserved nearly all of the
// GPU, so a raw cudaMalloc fails or fragments it), a time-critical loop where
// the implicit device synchronisation of cudaMalloc/cudaFree is not
// acceptable, or a plugin host that forbids libraries from allocating after
// initialisation.  dgp_rhs (and the stepping entry points) use buffers the
// solver allocates; this entry point does not allocate at all.
//
// How: the caller passes the state and the output as device buffers.  Every
// intermediate -- the state in the solver's internal cell order, the per-cell
// face slots written by the face kernel, the face-point traces, the RHS in
// internal order -- lives in one file-scope __device__ array of kScratchBytes
// (32 MiB).  The array is part of the library image: every GPU that loads
// libdgp.so holds it until the process exits.  Meshes whose intermediates do
// not fit are rejected.
//
// The array is shared by all calls and keeps the last call's contents; every
// byte a call reads is written earlier in the same call, so nothing has to be
// cleared.  Calls that overlap on the GPU (from several threads or streams)
// race on the array; the entry point synchronises the solver's stream before
// returning so that consecutive calls from one thread do not overlap.
//
// The host-side name of the array is only a stand-in for the device symbol;
// its device address is taken once per device with cudaGetSymbolAddress (with
// that device current) on the first call made on that device.  That first call
// therefore does host-side setup and should come before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "dgp_handles.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// device address of g_scratch on `device` (the current device), looked up once
// per device; a device reset frees the module and with it this address, as it
// frees every other device buffer the library's handles hold
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return fail(DGP_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess)
      return fail(DGP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return DGP_OK;
}

size_t round256(size_t n) { return (n + 255) / 256 * 256; }

// out[i][:] = in[perm[i]][:], converting the arithmetic type
template <typename Tin, typename Tout>
__global__ void permute_rows(const Tin* in, Tout* out, const int* perm, int E, int mnp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)E * mnp) return;
  const int e = static_cast<int>(i / mnp), r = static_cast<int>(i - (long long)e * mnp);
  out[i] = static_cast<Tout>(in[(size_t)perm[e] * mnp + r]);
}

}  // namespace

extern "C" int dgp_rhs_noalloc(dgp_solver s, const double* dev_state, double t, double* dev_rhs) {
  if (!s || !dev_state || !dev_rhs) return fail(DGP_ERR_INVALID, "null argument");
  DGP_CUDA(cudaSetDevice(s->device));
  const size_t tsize = s->ops.tsize;
  const int E = s->b.E, mnp = s->b.M * s->b.NP;
  // FP64 state and RHS, each with the 256-byte tail the solver's own state
  // buffers carry: the element kernel's bulk copy of the last tile rounds its
  // length up to 16 bytes and must stay inside the region
  const size_t state_b = round256(s->state_count() * 8 + 256);
  const size_t ntiles = (static_cast<size_t>(E) + s->ops.TE - 1) / s->ops.TE;
  // the fused stage kernel keeps face data in shared memory: state and RHS
  // only; the separate kernels also need the face slots and traces
  const size_t slot_b =
      s->fused ? 0 : round256(ntiles * s->ops.TE * s->tab.nlf * s->tab.nqf * s->b.M * tsize);
  const size_t need = 2 * state_b + 2 * slot_b;
  if (need > kScratchBytes)
    return fail(DGP_ERR_INVALID, "dgp_rhs_noalloc: this mesh needs " + std::to_string(need) +
                                     " bytes of scratch; the static scratch holds " +
                                     std::to_string(kScratchBytes) + " bytes (32 MiB)");
  void* base = nullptr;
  if (int rc = scratch_address(s->device, &base)) return rc;
  unsigned char* p = static_cast<unsigned char*>(base);
  dgp::DeviceBuffers b = s->b;  // geometry and tables of the solver, intermediates in scratch
  // the separate form's P0 second pass would zero modes of the state copy in
  // place before the element kernel reads it, which the fused kernel does in
  // shared memory only: the fallback applies in the fused form
  if (!s->fused) b.p0 = 0;
  b.C = p;
  b.slots = p + state_b;
  b.rhs = p + state_b + slot_b;
  b.tr = p + 2 * state_b + slot_b;
  const long long n = static_cast<long long>(E) * mnp;
  const int grid = static_cast<int>((n + 255) / 256);
  permute_rows<double, double><<<grid, 256, 0, s->stream>>>(dev_state, static_cast<double*>(b.C),
                                                             s->d_i2f, E, mnp);
  dgp::TimeCtl c{};
  c.t = t;
  c.dtmin_bits = 0x7FF0000000000000ull;
  s->h_ctl[0] = c;
  DGP_CUDA(cudaMemcpyAsync(s->b.ctl, &s->h_ctl[0], sizeof(dgp::TimeCtl), cudaMemcpyHostToDevice, s->stream));
  if (s->fused) {
    const double* C = static_cast<const double*>(b.C);
    s->ops.fused(b, C, C, static_cast<double*>(b.rhs), nullptr, 0, 0.0, 0, s->stream);
  } else {
    s->ops.trace(b, nullptr, s->stream);
    s->ops.face(b, 0, 0.0, s->stream);
    s->ops.elem(b, 0, 0, s->stream);
  }
  permute_rows<double, double><<<grid, 256, 0, s->stream>>>(static_cast<const double*>(b.rhs), dev_rhs,
                                                             s->d_f2i, E, mnp);
  DGP_CUDA(cudaGetLastError());
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  return DGP_OK;
}
