// Batched solves of many bodies of uneven size on one device.
//
// A batch owns nslots contexts (each with its own streams and device
// buffers, sized by the largest body it has met). fp_batch_solve hands the
// bodies out, largest first, to one host thread per slot; each thread runs
// set-geometry, set-wake and fp_solve_body for its bodies on its own context,
// so up to nslots solves share the GPU at any time. Every body is solved by
// exactly the kernels of a single fp_solve_body call, so the results equal
// those of solving the bodies one by one.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "fp_internal.cuh"

struct fp_batch {
  int device = 0;
  std::vector<fp_ctx*> slots;
  std::string err;
};

extern "C" {

int fp_batch_create(int device, int nslots, fp_batch** out) {
  if (!out || nslots <= 0 || nslots > 64) return FP_EINVAL;
  *out = nullptr;
  fp_batch* b = new fp_batch();
  b->device = device;
  for (int s = 0; s < nslots; ++s) {
    fp_ctx* c = nullptr;
    const int rc = fp_ctx_create(device, &c);
    if (rc) {
      for (fp_ctx* x : b->slots) fp_ctx_destroy(x);
      delete b;
      return rc;
    }
    b->slots.push_back(c);
  }
  *out = b;
  return FP_OK;
}

int fp_batch_destroy(fp_batch* b) {
  if (!b) return FP_EINVAL;
  for (fp_ctx* c : b->slots) fp_ctx_destroy(c);
  delete b;
  return FP_OK;
}

const char* fp_batch_last_error(fp_batch* b) { return b ? b->err.c_str() : "null batch"; }

int fp_batch_solve(fp_batch* b, int element, double kerneloffset, double kernelcutoff, int64_t nbody,
                   const fp_body_desc* bodies, const fp_solve_opts* opts, fp_stats* stats) {
  if (!b) return FP_EINVAL;
  b->err.clear();
  if (nbody < 0 || (nbody > 0 && !bodies)) {
    b->err = "fp_batch_solve: bad arguments";
    return FP_EINVAL;
  }
  for (int64_t i = 0; i < nbody; ++i)
    if (!bodies[i].x || !bodies[i].Uinfs) {
      b->err = "fp_batch_solve: body " + std::to_string(i) + " has no Uinfs or no output";
      return FP_EINVAL;
    }
  // largest bodies first: the last ones to finish are then the small ones
  std::vector<int64_t> order(nbody);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t a, int64_t c) { return bodies[a].npanels > bodies[c].npanels; });
  std::atomic<int64_t> next{0};
  std::mutex mu;
  int first_rc = FP_OK;
  int64_t first_body = -1;
  auto worker = [&](fp_ctx* c) {
    for (;;) {
      const int64_t q = next.fetch_add(1);
      if (q >= nbody) return;
      const int64_t i = order[q];
      const fp_body_desc& d = bodies[i];
      fp_stats st{};
      int rc = fp_set_geometry(c, d.nodes, d.nnodes, d.panel_offsets, d.panel_nodes, d.npanels, d.cps,
                               d.normals, nullptr);
      if (!rc && element == FP_ELEMENT_VORTEXRING) rc = fp_set_wake(c, d.shedding, d.nsh, d.Das, d.Dbs);
      if (!rc) rc = fp_solve_body(c, element, kerneloffset, kernelcutoff, d.Uinfs, 1, opts, d.x, &st);
      if (stats) stats[i] = st;
      if (rc) {
        std::lock_guard<std::mutex> lock(mu);
        if (first_rc == FP_OK || i < first_body) {
          first_rc = rc;
          first_body = i;
          b->err = "body " + std::to_string(i) + ": " + fp_last_error(c);
        }
      }
    }
  };
  std::vector<std::thread> threads;
  const int64_t nt = std::min<int64_t>((int64_t)b->slots.size(), nbody);
  for (int64_t s = 0; s < nt; ++s) threads.emplace_back(worker, b->slots[s]);
  for (std::thread& t : threads) t.join();
  return first_rc;
}

}  // extern "C"
