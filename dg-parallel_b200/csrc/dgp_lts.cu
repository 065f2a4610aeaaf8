// Local time stepping on the host side: the size bins of
// DGAnalysis::sortCellsBySize (DGAnalysis.cc:749-890), the cell groups and face
// classes RungeKuttaTVD2adaptive walks (TimeIntegrator.cc:442-836), and the
// launch sequence of one advanceInTime (kernels in dgp_lts.cuh).
//
// The sequence follows the integrator call for call: every assembleVolume of a
// group is one lts_vol_kernel, every assembleBoundary of a face class one
// face-kernel pass over the class plus one lift into the cells touching it,
// every coefficient loop one lts_update_kernel.  The reference's range helpers
// ship with empty bodies (TimeIntegrator.cc:1438-1487); here they assemble what
// their whole-mesh versions (TimeIntegrator.cc:1332-1412) assemble on the range.
// Empty groups and classes launch nothing.  dt of bin b is DT * 2^-b, exact, so
// the kernels get 2^-k factors of the device-resident step.
#include <algorithm>
#include <cmath>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_handles.h"
#include "dgp_lts.cuh"

namespace {

using dgp::TimeCtl;

constexpr int kMaxBins = 10;  // the integrator's per-bin arrays (TimeIntegrator.h:47-50)

// end of a step: t += dt, one more step, residual 0 (advanceInTime returns 0)
__global__ void lts_advance_kernel(TimeCtl* c) {
  if (c->done) return;
  c->t = c->t + c->dt;
  c->steps += 1;
  c->resid = 0.0;
}

// The integrator's calls, batched: between two coefficient updates all
// assembly calls commute (they read the state and add to accumulators), and
// between two assembly calls the updates touch disjoint cell groups, so a run
// of assembly calls is one volume launch (a segment per group), one face launch
// (a segment per face class, each with its boundary time) and one lift over
// the cells touching those classes, and a run of updates is one update launch
// (a segment per group, each with its operation and dt).  A group or class
// that repeats inside a run starts a new launch.
struct Seq {
  enum Mode { LAUNCH, COUNT, PLAN };
  dgp_solver s;
  Mode mode;
  std::vector<unsigned>* masks = nullptr;  // PLAN: the class sets of the lifts
  int launches = 0;
  std::vector<int> vg;                          // pending volume groups (3 b + g)
  std::vector<std::pair<int, int>> fc;          // pending face classes and their k
  std::vector<std::tuple<int, int, int>> up;    // pending updates: group, op, k
  const LtsState& L() const { return s->lts; }
  static double fac(int k) { return std::ldexp(1.0, -k); }
  // assembleVolume over group (g, b)
  void vol(int g, int b) {
    flush_updates();
    const int i = 3 * b + g;
    if (L().gn[i] == 0) return;
    if (std::find(vg.begin(), vg.end(), i) != vg.end() || static_cast<int>(vg.size()) == dgp::kLtsMaxSegs)
      flush_assembly();
    vg.push_back(i);
  }
  // assembleBoundary over face class c at t + DT * 2^-k
  void bnd(int c, int k) {
    flush_updates();
    if (L().fn[c] == 0) return;
    bool again = static_cast<int>(fc.size()) == dgp::kLtsMaxSegs;
    for (const auto& p : fc) again |= p.first == c;
    if (again) flush_assembly();
    fc.push_back({c, k});
  }
  // a coefficient loop over group (g, b) with dt = DT * 2^-k
  void upd(int g, int b, int op, int k) {
    flush_assembly();
    const int i = 3 * b + g;
    if (L().gn[i] == 0) return;
    bool again = static_cast<int>(up.size()) == dgp::kLtsMaxSegs;
    for (const auto& u : up) again |= std::get<0>(u) == i;
    if (again) flush_updates();
    up.push_back({i, op, k});
  }
  void flush_assembly() {
    if (!vg.empty()) {
      ++launches;
      if (mode == LAUNCH) {
        dgp::LtsSegs S{};
        S.nseg = static_cast<int>(vg.size());
        for (int j = 0; j < S.nseg; ++j) {
          S.off[j] = L().goff[vg[j]];
          S.cnt[j] = L().gn[vg[j]];
        }
        s->ops.lts_vol(s->b, L().lists, S, L().racc, s->stream);
      }
      vg.clear();
    }
    if (!fc.empty()) {
      launches += 2;
      unsigned mask = 0;
      for (const auto& p : fc) mask |= 1u << p.first;
      if (mode == PLAN) masks->push_back(mask);
      if (mode == LAUNCH) {
        dgp::LtsSegs S{};
        S.nseg = static_cast<int>(fc.size());
        for (int j = 0; j < S.nseg; ++j) {
          S.off[j] = L().foff[fc[j].first];
          S.cnt[j] = L().fn[fc[j].first];
          S.fac[j] = fac(fc[j].second);
        }
        s->ops.lts_face(s->b, L().lists, S, s->stream);
        const auto& u = L().lift.at(mask);
        s->ops.lts_lift(s->b, L().lists + u.first, u.second, L().cface, L().fcls, mask, L().racc, s->stream);
      }
      fc.clear();
    }
  }
  void flush_updates() {
    if (up.empty()) return;
    ++launches;
    if (mode == LAUNCH) {
      dgp::LtsSegs S{};
      S.nseg = static_cast<int>(up.size());
      for (int j = 0; j < S.nseg; ++j) {
        const int i = std::get<0>(up[j]);
        S.off[j] = L().goff[i];
        S.cnt[j] = L().gn[i];
        S.op[j] = std::get<1>(up[j]);
        S.fac[j] = fac(std::get<2>(up[j]));
      }
      s->ops.lts_update(s->b, L().lists, S, L().c1, L().save, L().racc, s->stream);
    }
    up.clear();
  }
  void finish() {
    flush_assembly();
    flush_updates();
  }
  // RungeKuttaTVD2adaptive::firstStage (TimeIntegrator.cc:442-591)
  void first(int from, int to) {
    const int nb = L().nb;
    int k = from;
    if (from) vol(2, from - 1);
    for (int b = from; b < to; ++b) {
      vol(0, b);
      vol(1, b);
      vol(2, b);
      bnd(b, k);
      bnd(nb + b, k);
      ++k;
    }
    if (from) bnd(nb + from - 1, k);
    k = from;
    for (int b = from; b < to; ++b) upd(0, b, dgp::LTS_EULER_IN, k++);
    k = from;
    for (int b = from; b < to - 1; ++b) upd(1, b, dgp::LTS_TWO_HALF, ++k);
    k = from;
    if (from) upd(2, from - 1, dgp::LTS_EULER, k);
    for (int b = from; b < to - 1; ++b) upd(2, b, dgp::LTS_TWO_HALF, ++k);
  }
  // RungeKuttaTVD2adaptive::secondStage (TimeIntegrator.cc:594-715)
  void second(int from, int to) {
    const int nb = L().nb;
    int k = from;
    for (int b = from; b < to; ++b, ++k) {
      if (b > from) upd(2, b - 1, dgp::LTS_COPYBACK_ZERO, k);
      vol(0, b);
      vol(1, b);
      if (b > 0) vol(2, b - 1);
      bnd(b, k);
      bnd(nb + b, k);
      if (b > 0) bnd(nb + b - 1, k);
      upd(0, b, dgp::LTS_SECOND, k);
      upd(1, b, dgp::LTS_SECOND_SWAP, k);
      if (b > 0) upd(2, b - 1, dgp::LTS_SECOND, k);
    }
  }
  // RungeKuttaTVD2adaptive::advanceInTime (TimeIntegrator.cc:784-836)
  void step() {
    const int nb = L().nb;
    bool flat[kMaxBins];
    first(0, nb);
    second(0, nb);
    flat[0] = true;
    for (int i = 1; i < nb; ++i) flat[i] = false;
    int i = nb - 1;
    while (i > 0) {
      for (i = nb - 1; i >= 1; i--)
        if (!flat[i]) {
          upd(1, i - 1, dgp::LTS_LI_HALF, 0);
          first(i, nb);
          upd(1, i - 1, dgp::LTS_RESTORE, 0);
          second(i, nb);
          upd(1, i - 1, dgp::LTS_FINAL_RESET, 0);
          flat[i] = true;
          for (int j = i + 1; j < nb; ++j) flat[j] = false;
          break;
        }
    }
  }
};

}  // namespace

namespace dgp {

int launch_lts_step(dgp_solver s, bool next_dt, bool dry) {
  Seq q{s, dry ? Seq::COUNT : Seq::LAUNCH};
  q.step();
  q.finish();
  q.launches += 1 + (next_dt ? 1 : 0);
  if (!dry) {
    lts_advance_kernel<<<1, 1, 0, s->stream>>>(s->b.ctl);
    if (next_dt) s->ops.cfl(s->b, s->stream);
  }
  return q.launches;
}

}  // namespace dgp

// Bins as DGAnalysis::sortCellsBySize: bins = ceil(log2(max / min)) with the
// minimum starting at 1.0 (DGAnalysis.cc:756-771); bin i - 1 holds sizes in
// (B_i * 1.0001, B_{i-1} * 1.0001] with B_i = max / 2^i; a face between cells
// one bin apart goes to the interface class of the larger cell's bin, its
// cells become large / small on that interface.
static int lts_setup(dgp_solver s, int* nbins) {
  LtsState& L = s->lts;
  const int E = s->b.E, F = s->b.F, NLF = s->b.dim + 1;
  std::vector<double> csize(E);
  std::vector<int> fel(2 * static_cast<size_t>(F)), fcode(F);
  DGP_CUDA(cudaStreamSynchronize(s->stream));
  DGP_CUDA(cudaMemcpy(csize.data(), s->b.csize, E * sizeof(double), cudaMemcpyDeviceToHost));
  DGP_CUDA(cudaMemcpy(fel.data(), s->b.fel, fel.size() * sizeof(int), cudaMemcpyDeviceToHost));
  DGP_CUDA(cudaMemcpy(fcode.data(), s->b.fcode, F * sizeof(int), cudaMemcpyDeviceToHost));
  double maxS = 0.0, minS = 1.0;
  for (int e = 0; e < E; ++e) {
    if (maxS < csize[e]) maxS = csize[e];
    if (minS > csize[e]) minS = csize[e];
  }
  const int nb = static_cast<int>(std::ceil(std::log(maxS / minS) / std::log(2.)));
  if (nb < 2) return fail(DGP_ERR_INVALID, "local time stepping: fewer than 2 size bins (no cell is binned)");
  if (nb > kMaxBins) return fail(DGP_ERR_INVALID, "local time stepping: more than 10 size bins");
  double B[kMaxBins + 1];
  B[0] = maxS;
  for (int i = 1; i <= nb; ++i) B[i] = B[i - 1] * 0.5;
  std::vector<int> bin(E, -1), role(E, 0), fcls(F);
  for (int e = 0; e < E; ++e) {
    for (int i = 1; i <= nb; ++i)
      if (csize[e] <= B[i - 1] * 1.0001 && csize[e] > B[i] * 1.0001) bin[e] = i - 1;
    if (bin[e] < 0) return fail(DGP_ERR_INVALID, "local time stepping: a cell falls in no size bin");
  }
  std::vector<int> cface(static_cast<size_t>(E) * NLF, -1);
  for (int f = 0; f < F; ++f) {
    const int eL = fel[2 * f], eR = fel[2 * f + 1];
    cface[static_cast<size_t>(eL) * NLF + (fcode[f] & 15)] = f;
    if (eR >= 0) cface[static_cast<size_t>(eR) * NLF + ((fcode[f] >> 4) & 15)] = f;
    const int lb = bin[eL], rb = eR >= 0 ? bin[eR] : 0;
    if (eR < 0 || lb == rb) {
      fcls[f] = lb;
    } else if (lb - rb == 1 || rb - lb == 1) {
      const int lo = std::min(lb, rb);
      const int large = lb < rb ? eL : eR, small = lb < rb ? eR : eL;
      if (role[large] == 2 || role[small] == 1)
        return fail(DGP_ERR_INVALID, "local time stepping: a cell lies on two bin interfaces");
      fcls[f] = nb + lo;
      role[large] = 1;
      role[small] = 2;
    } else {
      return fail(DGP_ERR_INVALID, "local time stepping: neighbouring cells more than one size bin apart");
    }
  }
  // lists: groups (3 per bin), face classes (2 per bin)
  std::vector<int> all;
  L.goff.assign(3 * nb, 0);
  L.gn.assign(3 * nb, 0);
  for (int b = 0; b < nb; ++b)
    for (int g = 0; g < 3; ++g) {
      L.goff[3 * b + g] = static_cast<int>(all.size());
      for (int e = 0; e < E; ++e)
        if (role[e] == g && bin[e] == (g == 2 ? b + 1 : b)) all.push_back(e);
      L.gn[3 * b + g] = static_cast<int>(all.size()) - L.goff[3 * b + g];
    }
  L.nb = nb;
  L.foff.assign(2 * nb, 0);
  L.fn.assign(2 * nb, 0);
  for (int c = 0; c < 2 * nb; ++c) {
    L.foff[c] = static_cast<int>(all.size());
    for (int f = 0; f < F; ++f)
      if (fcls[f] == c) all.push_back(f);
    L.fn[c] = static_cast<int>(all.size()) - L.foff[c];
  }
  // the cells each batched lift covers: every cell touching a face of one of
  // the classes of the run (found by walking the step once without launches)
  {
    std::vector<unsigned> masks;
    Seq plan{s, Seq::PLAN};
    plan.masks = &masks;
    plan.step();
    plan.finish();
    std::sort(masks.begin(), masks.end());
    masks.erase(std::unique(masks.begin(), masks.end()), masks.end());
    L.lift.clear();
    for (unsigned mask : masks) {
      std::vector<int> touch;
      for (int f = 0; f < F; ++f)
        if ((mask >> fcls[f]) & 1u) {
          touch.push_back(fel[2 * f]);
          if (fel[2 * f + 1] >= 0) touch.push_back(fel[2 * f + 1]);
        }
      std::sort(touch.begin(), touch.end());
      touch.erase(std::unique(touch.begin(), touch.end()), touch.end());
      L.lift[mask] = {static_cast<int>(all.size()), static_cast<int>(touch.size())};
      all.insert(all.end(), touch.begin(), touch.end());
    }
  }
  if (!L.lists) {  // first setup: device buffers live as long as the solver
    const size_t n = s->state_count();
    if (int rc = s->alloc(&L.c1, n)) return rc;
    if (int rc = s->alloc(&L.save, n)) return rc;
    if (int rc = s->alloc(&L.racc, n)) return rc;
    if (int rc = s->upload(&L.lists, all)) return rc;
    if (int rc = s->upload(&L.fcls, fcls)) return rc;
    if (int rc = s->upload(&L.cface, cface)) return rc;
    DGP_CUDA(cudaMemset(L.c1, 0, n * sizeof(double)));
    DGP_CUDA(cudaMemset(L.save, 0, n * sizeof(double)));
  }
  // the right-hand sides start at zero (DGCell::ZeroRHS after the projection)
  DGP_CUDA(cudaMemset(L.racc, 0, s->state_count() * sizeof(double)));
  L.bin = bin;
  L.role = role;
  if (nbins) *nbins = nb;
  return DGP_OK;
}

int dgp_set_time_stepping(dgp_solver s, int mode, int* nbins) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (mode != DGP_STEPPING_SSPRK3 && mode != DGP_STEPPING_LOCAL)
    return fail(DGP_ERR_INVALID, "unknown time stepping mode " + std::to_string(mode));
  DGP_CUDA(cudaSetDevice(s->device));
  s->drop_graphs();
  if (mode == DGP_STEPPING_SSPRK3) {
    s->lts.on = false;
    if (nbins) *nbins = 0;
    return DGP_OK;
  }
  if (!s->ops.lts_vol)
    return fail(DGP_ERR_UNSUPPORTED, "local time stepping is built for FP64 solvers with 128-thread tiles");
  if (s->limiter != DGP_LIMITER_NONE)
    return fail(DGP_ERR_UNSUPPORTED, "local time stepping runs without a limiter");
  if (s->meshes.size() != 1) return fail(DGP_ERR_UNSUPPORTED, "local time stepping runs on single solvers");
  if (s->b.p0)
    return fail(DGP_ERR_UNSUPPORTED,
                "local time stepping runs without the P0 fallback: turn it off first (dgp_set_p0_fallback(s, 0))");
  if (int rc = lts_setup(s, nbins)) return rc;
  s->lts.on = true;
  return DGP_OK;
}

int dgp_lts_bins(dgp_solver s, int* bin, int* role) {
  if (!s) return fail(DGP_ERR_INVALID, "null solver");
  if (!s->lts.on) return fail(DGP_ERR_INVALID, "local time stepping is off");
  for (int i = 0; i < s->b.E; ++i) {
    if (bin) bin[s->i2f[i]] = s->lts.bin[i];
    if (role) role[s->i2f[i]] = s->lts.role[i];
  }
  return DGP_OK;
}
