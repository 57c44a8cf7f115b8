// Batches: many resident simulations advanced together, one CUDA graph
// launch per time step for all of them.
//
// Each session captures its steady step as a CUDA graph the first time it
// reaches a graphable step (Session::enqueue_step).  A batch builds one
// parent graph whose child nodes are those graphs, with no edges between
// them, so the device runs the simulations' kernels side by side and the
// host issues one launch per step however many simulations there are.
// Steps that are not graphable (an initial-pressure start, a simulation's
// last step, steps of a per-point corrected source) run on their own,
// ordered on the batch stream.  When the set of members changes (a
// simulation finishes, or re-captures its step after a schedule change) the
// parent graph is built again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kwave_b200.h"
#include "solver_internal.h"

namespace kwb {

namespace {
void bk(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw KwError(KW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

class Batch {
 public:
  explicit Batch(std::vector<Session*> s) : ss(std::move(s)) {
    if (ss.empty()) throw KwError(KW_ERR_INVALID_ARGUMENT, "a batch needs at least one session");
    for (size_t i = 0; i < ss.size(); ++i) {
      if (!ss[i]) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL session in batch");
      for (size_t j = 0; j < i; ++j)
        if (ss[j] == ss[i]) throw KwError(KW_ERR_INVALID_ARGUMENT, "a session appears twice in the batch");
      if (ss[i]->ring_rows) throw KwError(KW_ERR_INVALID_ARGUMENT, "streamed sessions cannot be batched");
    }
    bk(cudaStreamCreateWithFlags(&bst, cudaStreamNonBlocking), "cudaStreamCreate");
    bk(cudaEventCreate(&ev0), "cudaEventCreate");
    bk(cudaEventCreate(&ev1), "cudaEventCreate");
    bk(cudaEventCreateWithFlags(&order, cudaEventDisableTiming), "cudaEventCreate");
  }
  ~Batch() {
    if (bst) cudaStreamSynchronize(bst);
    drop_parent();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (order) cudaEventDestroy(order);
    if (bst) cudaStreamDestroy(bst);
  }

  // Advance every member that has steps left by up to n steps (members
  // stop at their own Nt).  Asynchronous: the work is ordered after each
  // member's queued work, and each member's later work after this.
  void advance(uint64_t n) {
    for (Session* s : ss) {  // the batch stream waits for every member's queued work
      bk(cudaEventRecord(order, s->st), "cudaEventRecord");
      bk(cudaStreamWaitEvent(bst, order, 0), "cudaStreamWaitEvent");
    }
    std::vector<cudaStream_t> own(ss.size());
    for (size_t i = 0; i < ss.size(); ++i) {  // members' own launches go to the batch stream meanwhile
      own[i] = ss[i]->st;
      ss[i]->st = bst;
    }
    bk(cudaEventRecord(ev0, bst), "cudaEventRecord");
    try {
      for (uint64_t k = 0; k < n; ++k) step();
    } catch (...) {
      // the steps already enqueued on the batch stream still write the
      // members' buffers: each member's own stream waits for them before
      // its next work (best effort; the original error is what is reported)
      const bool marked = cudaEventRecord(ev1, bst) == cudaSuccess;
      for (size_t i = 0; i < ss.size(); ++i) {
        ss[i]->st = own[i];
        if (!marked || cudaStreamWaitEvent(own[i], ev1, 0) != cudaSuccess) cudaStreamSynchronize(bst);
      }
      throw;
    }
    bk(cudaEventRecord(ev1, bst), "cudaEventRecord");
    for (size_t i = 0; i < ss.size(); ++i) {
      ss[i]->st = own[i];
      bk(cudaStreamWaitEvent(ss[i]->st, ev1, 0), "cudaStreamWaitEvent");
    }
  }

  float elapsed_ms() {
    bk(cudaEventSynchronize(ev1), "cudaEventSynchronize");
    float ms = 0.f;
    bk(cudaEventElapsedTime(&ms, ev0, ev1), "cudaEventElapsedTime");
    return ms;
  }

  void sync() {
    bk(cudaStreamSynchronize(bst), "sync");
    for (Session* s : ss) s->sync();  // also reads each member's device error word
  }

  uint64_t graph_launches = 0;  // parent-graph launches so far (one per batched step)
  uint64_t rebuilds = 0;        // parent graphs built

 private:
  void step() {
    members.clear();
    for (Session* s : ss) {
      if (s->t_done >= s->Nt) continue;
      const uint64_t t = s->t_done + 1;
      if (s->graphable(t) && s->graph_exec)
        members.push_back(s);
      else
        s->enqueue_step();  // alone (captures the member's graph at its first graphable step)
    }
    if (members.empty()) return;
    std::vector<std::pair<cudaGraph_t, uint64_t>> gs;
    for (Session* s : members) gs.push_back({s->graph, s->graph_gen});
    if (gs != parent_of) build(gs);
    bk(cudaGraphLaunch(parent_exec, bst), "cudaGraphLaunch");
    ++graph_launches;
    for (Session* s : members) {
      s->launches_ += s->graph_launches;
      ++s->t_done;
    }
  }

  void build(const std::vector<std::pair<cudaGraph_t, uint64_t>>& gs) {
    drop_parent();
    bk(cudaGraphCreate(&parent, 0), "cudaGraphCreate");
    for (auto& g : gs) {
      cudaGraphNode_t node = nullptr;
      bk(cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, g.first), "cudaGraphAddChildGraphNode");
    }
    bk(cudaGraphInstantiate(&parent_exec, parent, 0), "cudaGraphInstantiate");
    parent_of = gs;
    ++rebuilds;
  }

  void drop_parent() {
    if (parent_exec) cudaGraphExecDestroy(parent_exec);
    if (parent) cudaGraphDestroy(parent);
    parent_exec = nullptr;
    parent = nullptr;
    parent_of.clear();
  }

  std::vector<Session*> ss, members;
  cudaStream_t bst = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, order = nullptr;
  cudaGraph_t parent = nullptr;
  cudaGraphExec_t parent_exec = nullptr;
  std::vector<std::pair<cudaGraph_t, uint64_t>> parent_of;  // member graphs (and capture numbers) it was built from
};

}  // namespace kwb

struct kw_batch {
  std::unique_ptr<kwb::Batch> b;
};

namespace {

int bstatus(kw_status* st, int code, const char* msg) {
  if (st) {
    st->code = code;
    std::snprintf(st->message, sizeof(st->message), "%s", msg);
  }
  return code;
}

template <class F>
int bguard(kw_status* st, F&& f) {
  try {
    f();
    return bstatus(st, KW_OK, "");
  } catch (const kwb::KwError& e) {
    return bstatus(st, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return bstatus(st, KW_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return bstatus(st, KW_ERR_INTERNAL, e.what());
  }
}

}  // namespace

extern "C" {

int kw_batch_create(kw_session* const* sessions, int n, kw_batch** batch, kw_status* status) {
  return bguard(status, [&] {
    if (!batch || !sessions || n < 1) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "sessions, n >= 1 and batch needed");
    *batch = nullptr;
    std::vector<kwb::Session*> ss;
    for (int i = 0; i < n; ++i) ss.push_back(sessions[i] ? sessions[i]->s.get() : nullptr);
    auto h = std::make_unique<kw_batch>();
    h->b = std::make_unique<kwb::Batch>(ss);
    *batch = h.release();
  });
}

int kw_batch_advance(kw_batch* b, uint64_t nsteps, kw_status* status) {
  return bguard(status, [&] {
    if (!b) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL batch");
    b->b->advance(nsteps);
  });
}

int kw_batch_elapsed_ms(kw_batch* b, float* ms, kw_status* status) {
  return bguard(status, [&] {
    if (!b || !ms) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    *ms = b->b->elapsed_ms();
  });
}

int kw_batch_sync(kw_batch* b, kw_status* status) {
  return bguard(status, [&] {
    if (!b) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL batch");
    b->b->sync();
  });
}

uint64_t kw_batch_graph_launches(const kw_batch* b) { return b ? b->b->graph_launches : 0; }

void kw_batch_destroy(kw_batch* b) { delete b; }

}  // extern "C"
