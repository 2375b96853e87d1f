// Serving pool: continuous batching of independent model runs on one device.
//
// A request is a model directory plus an end time.  Its host-side preparation
// (reading the inputs, building the dense layout) happens outside the pool,
// on any host thread, so it overlaps with device work.  The pool admits a
// prepared model into a free slot when the model's exact device footprint
// fits the HBM budget, uploads it, and from then on advances it together with
// every other resident model in the same launches (one scenario table, one
// tile list, per-model dt).  Finished models stay resident until the caller
// has read their results and releases the slot.  Membership changes take
// effect between chunks of steps: the runner (scenario table, tiles, tensor
// maps, CUDA graph) is rebuilt over the current members; the models' states
// live in their own device memory and are untouched by a rebuild.  Regular
// grids and quadtree meshes run in two runners on two streams, so the two
// kinds of request overlap on the device too.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/sfincs_bmi.h"
#include "model.h"

namespace sfg {
void launch_gather_f32_f64(const float* src, const int32_t* cmp, double* out, long long n, cudaStream_t s);
void launch_gather_f32(const float* src, const int32_t* cmp, float* out, long long n, cudaStream_t s);
void launch_gather_f64(const double* src, const int32_t* cmp, double* out, long long n, cudaStream_t s);
void set_last_error(const std::string& msg);

namespace {

struct Prepared {
  std::unique_ptr<HostModel> host;
  size_t bytes = 0;
};

struct Slot {
  std::unique_ptr<HostModel> host;
  std::unique_ptr<DeviceModel> dev;
  double t_end = 0.0;
  bool used = false, finished = false;
  StepState last{};
};

struct Pool {
  int max_slots;
  size_t budget, used_bytes = 0;
  std::vector<Slot> slots;
  std::vector<int> members[2];  // slot of each runner scenario: regular grids, quadtree meshes
  std::unique_ptr<Runner> runner[2];
  bool dirty = false;
  cudaStream_t stream = nullptr;   // regular-grid runner, uploads and reads
  cudaStream_t stream_qt = nullptr;  // quadtree runner
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  StepState* h_states = nullptr;

  Pool(int n, size_t b) : max_slots(n), budget(b), slots((size_t)n) {
    check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "pool stream");
    check_cuda(cudaStreamCreateWithFlags(&stream_qt, cudaStreamNonBlocking), "pool stream");
    check_cuda(cudaMallocHost(&h_states, (size_t)n * sizeof(StepState)), "pinned states");
  }
  void sync_all() {
    check_cuda(cudaStreamSynchronize(stream), "pool sync");
    check_cuda(cudaStreamSynchronize(stream_qt), "pool sync");
  }
  ~Pool() {
    if (stream) cudaStreamSynchronize(stream);
    if (stream_qt) cudaStreamSynchronize(stream_qt);
    runner[0].reset();
    runner[1].reset();
    for (auto& s : slots) s.dev.reset();
    if (d_stage) cudaFree(d_stage);
    if (h_states) cudaFreeHost(h_states);
    if (stream) cudaStreamDestroy(stream);
    if (stream_qt) cudaStreamDestroy(stream_qt);
  }

  int admit(Prepared* pr, double t_end) {
    if (pr->bytes > budget - std::min(budget, used_bytes)) return -1;
    int k = -1;
    for (int i = 0; i < max_slots; i++)
      if (!slots[i].used) {
        k = i;
        break;
      }
    if (k < 0) return -1;
    Slot& s = slots[k];
    s.dev = std::make_unique<DeviceModel>(*pr->host);
    s.host = std::move(pr->host);
    s.t_end = (t_end >= 0.0) ? t_end : s.host->t1;  // negative or NaN: the model's own tstop
    s.used = true;
    s.finished = false;
    s.last = StepState{};
    used_bytes += s.dev->bytes();
    // run target of the new member (the runner applies nothing to it before a rebuild)
    const int left = -1;
    check_cuda(cudaMemcpyAsync(&s.dev->state()->tend, &s.t_end, sizeof(double), cudaMemcpyHostToDevice, stream),
               "tend");
    check_cuda(cudaMemcpyAsync(&s.dev->state()->steps_left, &left, sizeof(int), cudaMemcpyHostToDevice, stream),
               "steps_left");
    dirty = true;
    return k;
  }

  void rebuild() {
    sync_all();
    for (int k = 0; k < 2; k++) {
      runner[k].reset();
      members[k].clear();
      std::vector<DeviceModel*> devs;
      for (int i = 0; i < max_slots; i++)
        if (slots[i].used && !slots[i].finished && (slots[i].host->p.quadtree != 0) == (k == 1)) {
          members[k].push_back(i);
          devs.push_back(slots[i].dev.get());
        }
      if (!devs.empty()) runner[k] = std::make_unique<Runner>(devs, 8, k == 0 ? stream : stream_qt);
    }
    dirty = false;
  }

  // Advance the running members by up to nsteps steps; returns how many are
  // still running afterwards.  Both runners are queued before either is
  // waited for.
  int advance(int nsteps) {
    if (dirty) rebuild();
    if (!runner[0] && !runner[1]) return 0;
    size_t j = 0;
    for (int k = 0; k < 2; k++) {
      if (!runner[k]) continue;
      runner[k]->issue(nsteps);
      for (int slot : members[k])
        check_cuda(cudaMemcpyAsync(&h_states[j++], slots[slot].dev->state(), sizeof(StepState),
                                   cudaMemcpyDeviceToHost, k == 0 ? stream : stream_qt),
                   "read state");
    }
    sync_all();
    int running = 0;
    j = 0;
    for (int k = 0; k < 2; k++) {
      if (!runner[k]) continue;
      for (int slot : members[k]) {
        Slot& s = slots[slot];
        s.last = h_states[j];
        const StepState& st = h_states[j++];
        if (st.stop_pending || !(st.t < st.tend) || st.error || st.fault) {
          s.finished = true;
          dirty = true;
        } else {
          running++;
        }
      }
    }
    return running;
  }

  Slot& at(int k) {
    if (k < 0 || k >= max_slots || !slots[k].used) throw std::runtime_error("no model in pool slot " + std::to_string(k));
    return slots[k];
  }

  void release(int k) {
    Slot& s = at(k);
    sync_all();
    runner[0].reset();  // they may still reference the model; rebuilt on the next advance
    runner[1].reset();
    dirty = true;
    used_bytes -= s.dev->bytes();
    s.dev.reset();
    s.host.reset();
    s.used = false;
    s.finished = false;
  }

  void get(int k, const std::string& name, void* dst, size_t bytes) {
    Slot& s = at(k);
    const long long n = s.host->np;
    ScnDev& D = s.dev->dev();
    sync_all();
    check_cuda(cudaMemcpyAsync(&s.last, s.dev->state(), sizeof(StepState), cudaMemcpyDeviceToHost, stream), "state");
    check_cuda(cudaStreamSynchronize(stream), "pool sync");
    const int p = s.last.run ? (s.last.parity ^ 1) : s.last.parity;
    const size_t need8 = (size_t)n * 8;
    if (stage_bytes < need8) {
      if (d_stage) cudaFree(d_stage);
      d_stage = nullptr;
      check_cuda(cudaMalloc(&d_stage, need8), "pool stage");
      stage_bytes = need8;
    }
    auto need = [&](size_t b) {
      if (bytes != b) throw std::runtime_error("pool get('" + name + "'): expected " + std::to_string(b) + " bytes");
    };
    auto f32 = [&](const float* src, const int32_t* map = nullptr) {
      need((size_t)n * 4);
      launch_gather_f32(src, map ? map : s.dev->d_cmp_off(), (float*)d_stage, n, stream);
    };
    if (name == "zs") {
      need(need8);
      launch_gather_f32_f64(D.zs, s.dev->d_cmp_off(), (double*)d_stage, n, stream);
    } else if (name == "z_volume" && D.zvol) {
      need(need8);
      launch_gather_f64(D.zvol, s.dev->d_cmp_off(), (double*)d_stage, n, stream);
    } else if (name == "zsmax") {
      f32(D.zsmax);
    } else if ((name == "vmax" && D.vmax) || (name == "qmax" && D.qmax) || (name == "twet" && D.twet) ||
               (name == "tzsmax" && D.tzsmax)) {
      f32(name == "vmax" ? D.vmax : name == "qmax" ? D.qmax : name == "twet" ? D.twet : D.tzsmax);
    } else if (name == "qx") {
      f32(D.qu[p], s.dev->face_map(0));
    } else if (name == "qy") {
      f32(D.qv[p], s.dev->face_map(1));
    } else if (name == "uvx") {
      f32(D.uu[p], s.dev->face_map(0));
    } else if (name == "uvy") {
      f32(D.vv[p], s.dev->face_map(1));
    } else {
      throw std::runtime_error("pool get: unknown variable '" + name + "'");
    }
    check_cuda(cudaMemcpyAsync(dst, d_stage, bytes, cudaMemcpyDeviceToHost, stream), "pool get");
    check_cuda(cudaStreamSynchronize(stream), "pool sync");
  }

  void scalars(int k, double* out) {
    Slot& s = at(k);
    sync_all();
    check_cuda(cudaMemcpyAsync(&s.last, s.dev->state(), sizeof(StepState), cudaMemcpyDeviceToHost, stream), "state");
    check_cuda(cudaStreamSynchronize(stream), "pool sync");
    const HostModel& h = *s.host;
    const StepState& st = s.last;
    double t = st.t;
    if (st.stop_pending) t = h.t1 + 1.0;
    double v[19] = {t, st.dt, st.min_dt, (double)st.nt, (double)st.error, h.t0, h.t1, (double)h.np, (double)h.npuv,
                    (double)h.p.nkcuv2, (double)h.p.ngbnd, (double)h.p.subgrid, st.bflux_vol,
                    st.rain_vol * h.area_total_kcs1, st.src_vol, h.p.dtmax, h.p.dtmin, (double)s.dev->bytes(),
                    (double)(h.p.quadtree ? h.np : (long long)h.tiles.size())};
    std::memcpy(out, v, sizeof(v));
  }
};

template <class F>
int pool_guarded(F&& f) {
  try {
    return f();
  } catch (std::exception& e) {
    set_last_error(e.what());
    return -2;
  }
}

void copy_msg(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) {
    std::strncpy(err, msg, (size_t)errlen - 1);
    err[errlen - 1] = 0;
  }
}

}  // namespace
}  // namespace sfg

using sfg::pool_guarded;

extern "C" {

void* sfg_pool_create(int max_slots, double hbm_budget_bytes, char* err, int errlen) {
  try {
    if (max_slots < 1) throw std::runtime_error("max_slots must be >= 1");
    if (!(hbm_budget_bytes > 0)) throw std::runtime_error("hbm budget must be positive");
    return new sfg::Pool(max_slots, (size_t)hbm_budget_bytes);
  } catch (std::exception& e) {
    sfg::copy_msg(err, errlen, e.what());
    return nullptr;
  }
}
void sfg_pool_destroy(void* pool) { delete static_cast<sfg::Pool*>(pool); }

void* sfg_prepare(const char* model_dir, int bmi, char* err, int errlen) {
  try {
    auto* p = new sfg::Prepared();
    p->host = sfg::load_model(model_dir ? model_dir : ".", bmi != 0);
    p->bytes = sfg::device_bytes_needed(*p->host);
    return p;
  } catch (std::exception& e) {
    sfg::copy_msg(err, errlen, e.what());
    return nullptr;
  }
}
double sfg_prepared_bytes(void* prepared) { return (double)static_cast<sfg::Prepared*>(prepared)->bytes; }
double sfg_prepared_cells(void* prepared) { return (double)static_cast<sfg::Prepared*>(prepared)->host->np; }
void sfg_prepared_destroy(void* prepared) { delete static_cast<sfg::Prepared*>(prepared); }

int sfg_pool_admit(void* pool, void* prepared, double t_end) {
  return pool_guarded([&] {
    auto* pr = static_cast<sfg::Prepared*>(prepared);
    const int k = static_cast<sfg::Pool*>(pool)->admit(pr, t_end);
    if (k >= 0) delete pr;  // consumed
    return k;
  });
}
int sfg_pool_advance(void* pool, int nsteps) {
  return pool_guarded([&] { return static_cast<sfg::Pool*>(pool)->advance(nsteps); });
}
int sfg_pool_finished(void* pool, int* slots, int cap) {
  return pool_guarded([&] {
    auto* P = static_cast<sfg::Pool*>(pool);
    int c = 0;
    for (int i = 0; i < P->max_slots && c < cap; i++)
      if (P->slots[i].used && P->slots[i].finished) slots[c++] = i;
    return c;
  });
}
int sfg_pool_scalars(void* pool, int slot, double out[19]) {
  return pool_guarded([&] {
    static_cast<sfg::Pool*>(pool)->scalars(slot, out);
    return 0;
  });
}
int sfg_pool_get(void* pool, int slot, const char* name, void* dst, size_t bytes) {
  return pool_guarded([&] {
    static_cast<sfg::Pool*>(pool)->get(slot, name ? name : "", dst, bytes);
    return 0;
  });
}
int sfg_pool_release(void* pool, int slot) {
  return pool_guarded([&] {
    static_cast<sfg::Pool*>(pool)->release(slot);
    return 0;
  });
}
double sfg_pool_used_bytes(void* pool) { return (double)static_cast<sfg::Pool*>(pool)->used_bytes; }
int sfg_pool_resident(void* pool) {
  auto* P = static_cast<sfg::Pool*>(pool);
  int c = 0;
  for (auto& s : P->slots) c += s.used ? 1 : 0;
  return c;
}
void* sfg_pool_stream(void* pool) { return (void*)static_cast<sfg::Pool*>(pool)->stream; }

}  // extern "C"
