// C-ABI of libsfincs_gpu.so: the reference's BMI surface (sfincs_bmi.f90)
// re-implemented over the B200 core, plus model and ensemble handles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/sfincs_bmi.h"
#include "model.h"
#include "output.h"

namespace sfg {
void launch_gather_f32_f64(const float* src, const int32_t* cmp, double* out, long long n, cudaStream_t s);
void launch_gather_f32(const float* src, const int32_t* cmp, float* out, long long n, cudaStream_t s);
void launch_gather_f64(const double* src, const int32_t* cmp, double* out, long long n, cudaStream_t s);
void launch_gather_u8(const uint8_t* ku, const uint8_t* kv, const int32_t* cmp, float* out, long long n,
                      cudaStream_t s);
void launch_or_u8(uint8_t* a, uint8_t mask, long long n, cudaStream_t s);
void launch_scatter_f32(const float* in, const int32_t* cmp, float* dst, long long n, cudaStream_t s);
void launch_scatter_f64_f32(const double* in, const int32_t* cmp, float* dst, long long n, cudaStream_t s);
int volume_parts(long long n);
void launch_volume(const ScnDev* d_scn, const int32_t* cmp, long long n, double* part, double* out, cudaStream_t s);
int volume_noalloc(const ScnDev* d_scn, const int32_t* cmp, long long n, cudaStream_t s, double* host_out,
                   const char** why);

namespace {

thread_local std::string g_err = "no error";

// time_to_string (sfincs_date.f90:298-327): "yyyymmdd.HHMMSS" of tref + t
// seconds, with the reference's real*4 arithmetic for the time of day.
std::string restart_time_string(double t_sec, const std::string& tref) {
  const int yyyy = std::atoi(tref.substr(0, 4).c_str()), mm = std::atoi(tref.substr(4, 2).c_str()),
            dd = std::atoi(tref.substr(6, 2).c_str()), hh0 = std::atoi(tref.substr(9, 2).c_str()),
            mn0 = std::atoi(tref.substr(11, 2).c_str()), ss0 = std::atoi(tref.substr(13, 2).c_str());
  const float ref_fraction = (float)hh0 / 24.0f + (float)mn0 / 1440.0f + (float)ss0 / 86400.0f;
  const float sec_add = (float)((double)(ref_fraction * 86400.0f) + t_sec);
  const int ndays_add = (int)(sec_add / 86400.0f);
  const float secs_time = sec_add - (float)ndays_add * 86400.0f;
  // civil date of the reference day + ndays_add (proleptic Gregorian)
  auto days_from_civil = [](long long y, long long m, long long d) {
    y -= m <= 2;
    const long long era = (y >= 0 ? y : y - 399) / 400, yoe = y - era * 400;
    const long long doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1, doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + doe - 719468;
  };
  long long z = days_from_civil(yyyy, mm, dd) + ndays_add + 719468;
  const long long era = (z >= 0 ? z : z - 146096) / 146097, doe = z - era * 146097;
  const long long yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365, doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const long long mp = (5 * doy + 2) / 153, d = doy - (153 * mp + 2) / 5 + 1, m = mp + (mp < 10 ? 3 : -9);
  const long long y = yoe + era * 400 + (m <= 2);
  const int hh = (int)(secs_time / 3600.0f);
  const int mn = (int)((secs_time - (float)(hh * 3600)) / 60.0f);
  const int ss = (int)(secs_time - (float)(hh * 3600) - (float)(mn * 60));
  char buf[96];
  std::snprintf(buf, sizeof buf, "%04lld%02lld%02lld.%02d%02d%02d", y, m, d, hh, mn, ss);
  return buf;
}

// One model with its runner and data-interface staging buffers.
struct ModelHandle {
  std::unique_ptr<HostModel> host;
  std::unique_ptr<DeviceModel> dev;
  std::unique_ptr<Runner> runner;
  void* d_stage = nullptr;  // 8*np bytes
  double* d_part = nullptr;
  double* d_vol = nullptr;
  // BMI host mirrors (pinned)
  double* h_zs = nullptr;
  float* h_qext = nullptr;
  bool zs_exported = false, qext_exported = false;
  // update(): the exported qext crosses PCIe on its own stream while the step's
  // boundary and momentum kernels run; continuity waits for it.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t main_tail = nullptr, qext_ready = nullptr;
  // map / his / max output (off the step's critical path)
  std::unique_ptr<OutputWriter> out;
  bool finalized = false;

  ModelHandle(const std::string& dir, bool bmi) {
    host = load_model(dir, bmi);
    dev = std::make_unique<DeviceModel>(*host);
    runner = std::make_unique<Runner>(std::vector<DeviceModel*>{dev.get()});
    const size_t np = (size_t)std::max<long long>(host->np, 1);
    check_cuda(cudaMalloc(&d_stage, np * 8 * 2), "stage");
    check_cuda(cudaMalloc(&d_part, (size_t)volume_parts((long long)np) * sizeof(double)), "parts");
    check_cuda(cudaMalloc(&d_vol, sizeof(double)), "vol");
    check_cuda(cudaMallocHost(&h_zs, np * sizeof(double)), "pinned zs");
    check_cuda(cudaMallocHost(&h_qext, np * sizeof(float)), "pinned qext");
    std::memset(h_qext, 0, np * sizeof(float));
    check_cuda(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "copy stream");
    check_cuda(cudaEventCreateWithFlags(&main_tail, cudaEventDisableTiming), "event");
    check_cuda(cudaEventCreateWithFlags(&qext_ready, cudaEventDisableTiming), "event");
    refresh_zs();
    out = std::make_unique<OutputWriter>(*host, *dev, s());
  }
  ~ModelHandle() {
    try {
      finalize_output();
    } catch (...) {
    }
    out.reset();
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    runner.reset();
    if (qext_ready) cudaEventDestroy(qext_ready);
    if (main_tail) cudaEventDestroy(main_tail);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    dev.reset();
    if (d_stage) cudaFree(d_stage);
    if (d_part) cudaFree(d_part);
    if (d_vol) cudaFree(d_vol);
    if (h_zs) cudaFreeHost(h_zs);
    if (h_qext) cudaFreeHost(h_qext);
  }
  long long np() const { return host->np; }
  cudaStream_t s() const { return runner->stream(); }
  int latest(const StepState& st) const { return st.run ? (st.parity ^ 1) : st.parity; }

  void refresh_zs() {
    launch_gather_f32_f64(dev->dev().zs, dev->d_cmp_off(), (double*)d_stage, np(), s());
    check_cuda(cudaMemcpyAsync(h_zs, d_stage, (size_t)np() * 8, cudaMemcpyDeviceToHost, s()), "zs to host");
    runner->sync();
  }
  void push_qext() {
    if (!dev->dev().qext) return;
    check_cuda(cudaMemcpyAsync(d_stage, h_qext, (size_t)np() * 4, cudaMemcpyHostToDevice, s()), "qext to device");
    launch_scatter_f32((const float*)d_stage, dev->d_cmp_off(), const_cast<float*>(dev->dev().qext), np(), s());
  }
  void before_update() {
    if (qext_exported) push_qext();
  }
  // One step with the exported qext pushed concurrently: the copy and the
  // scatter into the model's qext start after everything queued before on the
  // model's stream (the previous step's continuity reads qext), and only the
  // step's continuity kernel waits for them.
  void step_once() {
    if (!(qext_exported && dev->dev().qext)) {
      runner->step_once();
      return;
    }
    check_cuda(cudaEventRecord(main_tail, s()), "record");
    check_cuda(cudaStreamWaitEvent(copy_stream, main_tail, 0), "copy stream wait");
    check_cuda(cudaMemcpyAsync(d_stage, h_qext, (size_t)np() * 4, cudaMemcpyHostToDevice, copy_stream), "qext to device");
    launch_scatter_f32((const float*)d_stage, dev->d_cmp_off(), const_cast<float*>(dev->dev().qext), np(), copy_stream);
    check_cuda(cudaEventRecord(qext_ready, copy_stream), "record");
    runner->step_once(qext_ready);
  }
  void after_update() {
    if (zs_exported) refresh_zs();
  }
  double next_output() const {
    return std::min({host->trstout, out->tmapout, out->tmaxout, out->thisout});
  }
  // Runs to tend (or max_steps steps), stopping at every output time on the
  // step that reaches it (t >= tout after the step, as sfincs_lib.f90:419-476
  // checks), where it writes the map / max / his output and the restart file.
  void run(double tend, long long max_steps, int chunk) {
    if (next_output() >= 1.0e9) {
      runner->run({tend}, max_steps, chunk);
      check_fault();
      return;
    }
    long long left = max_steps;
    for (;;) {
      const StepState s0 = runner->read_state(0);
      if (!(s0.t < tend) || left == 0) break;
      const double tnext = next_output();
      if (tnext <= s0.t)
        runner->run({tend}, 1, 1);  // the output falls on the next step
      else
        runner->run({std::min(tend, tnext)}, left, chunk);
      const StepState s1 = runner->read_state(0);
      if (left > 0) left = std::max(0LL, left - (long long)(s1.nt - s0.nt));
      check_fault();
      after_step_output();
      if (s1.nt == s0.nt) break;  // stopped (instability or end of the run)
    }
  }
  // A staged kernel whose bounded wait for its tile data gave up skipped that
  // tile and set the fault flag: the run is reported as failed.
  void check_fault() {
    if (runner->read_state(0).fault)
      throw std::runtime_error("a staged kernel gave up waiting for its tile data (fault flag set); the state of "
                               "this model is incomplete");
  }
  // The output checks after a step (sfincs_lib.f90:419-476), in the
  // reference's order: each due output sets the output time, the last one
  // set is the time every file of this step is written with.
  void after_step_output() {
    if (next_output() >= 1.0e9) return;
    const StepState st = runner->read_state(0);
    const double t = st.t, dt = (double)st.dt;
    const OutputSpec& o = host->out;
    bool wmap = false, wmax = false, wrst = false, whis = false;
    double tout = t;
    if (t >= out->tmapout) {
      wmap = true;
      out->ntmapout++;
      tout = std::max(out->tmapout, t - dt);
      out->tmapout += o.dtmapout;
    }
    if (t >= out->tmaxout) {
      wmax = true;
      out->ntmaxout++;
      tout = std::max(out->tmaxout, t - dt);
      if (t < (double)(float)host->t1) out->tmaxout += o.dtmaxout;
    }
    if (t >= host->trstout) {
      wrst = true;
      tout = host->trstout;
      host->trstout = host->dtrstout > 1.0e-6 ? host->trstout + host->dtrstout : 1.0e9;
    }
    if (t >= out->thisout) {
      whis = true;
      out->nthisout++;
      tout = std::max(out->thisout, t - dt);
      out->thisout += o.dthisout;
    }
    if (wmap || wmax || whis) out->write(wmap, wmax, whis, tout, latest(st));
    if (wrst) write_restart(tout);
  }
  // finalize_output (sfincs_output.f90:260-296): once, at finalize
  void finalize_output() {
    if (finalized || !out) return;
    finalized = true;
    const StepState st = runner->read_state(0);
    const float avg = st.nt > 0 ? (float)((st.t - host->t0) / (double)st.nt) : 0.0f;
    out->finalize(st.t, (double)(float)host->t1, latest(st), avg, st.error);
  }
  // write_rst_file (sfincs_output.f90:657-733), flavour 1: zs, q, uvmean
  void write_restart(double t) {
    const HostModel& H = *host;
    const ScnDev& D = dev->dev();
    const StepState st = runner->read_state(0);
    const int p = latest(st);
    const size_t NA = H.p.quadtree ? (size_t)H.np : (size_t)H.p.nalloc;  // storage length of a cell array
    std::vector<float> zs4((size_t)H.np), q, uvm;
    std::vector<int32_t> ident;  // quadtree: cells are stored in the reference's order
    const std::vector<int32_t>* cells = &H.cmp_off;
    if (H.p.quadtree) {
      // zs, q of the uv points, combined points and dummy, uvmean: all in the reference's order already
      const size_t NQ = (size_t)(H.npuv + H.p.ncuv + 1);
      q.resize(NQ);
      uvm.resize((size_t)H.p.nkcuv2);
      check_cuda(cudaMemcpy(zs4.data(), D.zs, (size_t)H.np * 4, cudaMemcpyDeviceToHost), "restart zs");
      check_cuda(cudaMemcpy(q.data(), D.qu[p], NQ * 4, cudaMemcpyDeviceToHost), "restart q");
      if (H.p.nkcuv2 > 0)
        check_cuda(cudaMemcpy(uvm.data(), D.uvmean, uvm.size() * 4, cudaMemcpyDeviceToHost), "restart uvmean");
      ident.resize((size_t)H.np);
      for (long long i = 0; i < H.np; i++) ident[(size_t)i] = (int32_t)i;
      cells = &ident;
    } else {
      std::vector<float> zsd(NA), qu(NA), qv(NA), um((size_t)std::max(H.p.nkcuv2, 1));
      check_cuda(cudaMemcpy(zsd.data(), D.zs, NA * 4, cudaMemcpyDeviceToHost), "restart zs");
      check_cuda(cudaMemcpy(qu.data(), D.qu[p], NA * 4, cudaMemcpyDeviceToHost), "restart qu");
      check_cuda(cudaMemcpy(qv.data(), D.qv[p], NA * 4, cudaMemcpyDeviceToHost), "restart qv");
      if (H.p.nkcuv2 > 0)
        check_cuda(cudaMemcpy(um.data(), D.uvmean, (size_t)H.p.nkcuv2 * 4, cudaMemcpyDeviceToHost), "restart uvmean");
      q.assign((size_t)H.npuv + 1, 0.0f);
      uvm.assign(H.kb_bface.size(), 0.0f);
      for (long long i = 0; i < H.np; i++) zs4[(size_t)i] = zsd[(size_t)H.cmp_off[i]];
      for (size_t f = 0; f < H.face_off.size(); f++) q[f] = (H.face_dir[f] == 0 ? qu : qv)[(size_t)H.face_off[f]];
      for (size_t ib = 0; ib < H.kb_bface.size(); ib++)
        if (H.kb_bface[ib] >= 0) uvm[ib] = um[(size_t)H.kb_bface[ib]];
    }
    const std::string name = H.dir + "/sfincs." + restart_time_string(1.0 * (double)(long long)t, H.tref) + ".rst";
    FILE* fp = std::fopen(name.c_str(), "wb");
    if (!fp) throw std::runtime_error("cannot write restart file " + name);
    auto rec = [&](const void* data, size_t bytes) {
      const int32_t n = (int32_t)bytes;
      std::fwrite(&n, 4, 1, fp);
      std::fwrite(data, 1, bytes, fp);
      std::fwrite(&n, 4, 1, fp);
    };
    // flavour 1, or 4 / 5 / 6 with the state of the cnb / gai / hor infiltration (sfincs_output.f90:690-722)
    const int32_t type = H.p.inftype == 3 ? 4 : H.p.inftype == 4 ? 5 : H.p.inftype == 5 ? 6 : 1;
    rec(&type, 4);
    rec(zs4.data(), zs4.size() * 4);
    rec(q.data(), q.size() * 4);
    rec(uvm.data(), uvm.size() * 4);
    for (int j = 0; j < (type == 5 ? 2 : (type == 1 ? 0 : 1)); j++) {
      std::vector<float> sd(NA), s4((size_t)H.np);
      check_cuda(cudaMemcpy(sd.data(), D.inf_st[j], NA * 4, cudaMemcpyDeviceToHost), "restart infiltration state");
      for (long long i = 0; i < H.np; i++) s4[(size_t)i] = sd[(size_t)(*cells)[(size_t)i]];
      rec(s4.data(), s4.size() * 4);
    }
    std::fclose(fp);
  }

  void scalars(double* out) {
    StepState st = runner->read_state(0);
    const HostModel& h = *host;
    double t = st.t;
    if (st.stop_pending) t = h.t1 + 1.0;  // sfincs_lib.f90:646 takes effect at the end of the step
    double v[19] = {t,
                    st.dt,
                    st.min_dt,
                    (double)st.nt,
                    (double)st.error,
                    h.t0,
                    h.t1,
                    (double)h.np,
                    (double)h.npuv,
                    (double)h.p.nkcuv2,
                    (double)h.p.ngbnd,
                    (double)h.p.subgrid,
                    st.bflux_vol,
                    st.rain_vol * h.area_total_kcs1,
                    st.src_vol,
                    h.p.dtmax,
                    h.p.dtmin,
                    (double)dev->bytes(),
                    (double)runner->ntiles()};
    std::memcpy(out, v, sizeof(v));
  }

  double volume() {
    launch_volume(runner->d_scns(), dev->d_cmp_off(), np(), d_part, d_vol, s());
    double v = 0.0;
    check_cuda(cudaMemcpyAsync(&v, d_vol, sizeof(double), cudaMemcpyDeviceToHost, s()), "volume");
    runner->sync();
    return v;
  }

  void get(const std::string& name, void* dst, size_t bytes) {
    const long long n = np();
    ScnDev& D = dev->dev();
    StepState st = runner->read_state(0);
    const int p = latest(st);
    auto need = [&](size_t b) {
      if (bytes != b) throw std::runtime_error("get_var('" + name + "'): expected " + std::to_string(b) + " bytes");
    };
    auto f32 = [&](const float* src, const int32_t* map = nullptr) {
      need((size_t)n * 4);
      launch_gather_f32(src, map ? map : dev->d_cmp_off(), (float*)d_stage, n, s());
      check_cuda(cudaMemcpyAsync(dst, d_stage, (size_t)n * 4, cudaMemcpyDeviceToHost, s()), "get");
    };
    if (name == "zs") {
      need((size_t)n * 8);
      launch_gather_f32_f64(D.zs, dev->d_cmp_off(), (double*)d_stage, n, s());
      check_cuda(cudaMemcpyAsync(dst, d_stage, (size_t)n * 8, cudaMemcpyDeviceToHost, s()), "get");
    } else if (name == "zsmax") {
      f32(D.zsmax);
    } else if (name == "vmax" || name == "qmax" || name == "twet" || name == "tzsmax" || name == "cumprcp" ||
               name == "cuminf") {
      const float* a = name == "vmax" ? D.vmax : name == "qmax" ? D.qmax : name == "twet" ? D.twet
                       : name == "tzsmax" ? D.tzsmax : name == "cumprcp" ? D.cumprcp : D.cuminf;
      if (!a) throw std::runtime_error("'" + name + "' is not stored by this model (store switch off)");
      f32(a);
    } else if (name == "qext") {
      if (!D.qext) throw std::runtime_error("qext is not enabled for this model");
      f32(D.qext);
    } else if (name == "z_volume") {
      if (!D.zvol) throw std::runtime_error("z_volume exists only for subgrid models");
      need((size_t)n * 8);
      launch_gather_f64(D.zvol, dev->d_cmp_off(), (double*)d_stage, n, s());
      check_cuda(cudaMemcpyAsync(dst, d_stage, (size_t)n * 8, cudaMemcpyDeviceToHost, s()), "get");
    } else if (name == "qx") {
      f32(D.qu[p], dev->face_map(0));
    } else if (name == "qy") {
      f32(D.qv[p], dev->face_map(1));
    } else if (name == "uvx") {
      f32(D.uu[p], dev->face_map(0));
    } else if (name == "uvy") {
      f32(D.vv[p], dev->face_map(1));
    } else if (name == "zs0" && D.zs0) {
      f32(D.zs0);
    } else if (name == "zsderv" && D.zsderv) {
      f32(D.zsderv);
    } else if (name == "kfuv") {
      if (D.quadtree) throw std::runtime_error("kfuv is not available per cell on quadtree meshes");
      need((size_t)n * 8);
      launch_gather_u8(D.kf[0], D.kf[1], dev->d_cmp_off(), (float*)d_stage, n, s());
      check_cuda(cudaMemcpyAsync(dst, d_stage, (size_t)n * 8, cudaMemcpyDeviceToHost, s()), "get");
    } else {
      throw std::runtime_error("unknown variable '" + name + "'");
    }
    runner->sync();
  }

  void set(const std::string& name, const void* src, size_t bytes) {
    const long long n = np();
    ScnDev& D = dev->dev();
    StepState st = runner->read_state(0);
    const int p = latest(st);
    if (D.quadtree && name != "zs" && name != "qext")
      throw std::runtime_error("set_var('" + name + "') is not available on quadtree meshes");
    auto put32 = [&](float* dstp) {
      if (bytes != (size_t)n * 4) throw std::runtime_error("set_var('" + name + "'): wrong size");
      check_cuda(cudaMemcpyAsync(d_stage, src, bytes, cudaMemcpyHostToDevice, s()), "set");
      launch_scatter_f32((const float*)d_stage, dev->d_cmp_off(), dstp, n, s());
    };
    if (name == "zs") {
      if (bytes != (size_t)n * 8) throw std::runtime_error("set_var('zs'): wrong size");
      check_cuda(cudaMemcpyAsync(d_stage, src, bytes, cudaMemcpyHostToDevice, s()), "set");
      launch_scatter_f64_f32((const double*)d_stage, dev->d_cmp_off(), D.zs, n, s());
    } else if (name == "qext") {
      if (!D.qext) throw std::runtime_error("qext is not enabled for this model");
      put32(const_cast<float*>(D.qext));
      std::memcpy(h_qext, src, bytes);
    } else if (name == "qx") {
      put32(D.qu[p]);
    } else if (name == "qy") {
      put32(D.qv[p]);
    } else if (name == "uvx") {
      put32(D.uu[p]);
    } else if (name == "uvy") {
      put32(D.vv[p]);
    } else {
      throw std::runtime_error("variable '" + name + "' cannot be set");
    }
    if (name == "qx" || name == "qy" || name == "uvx" || name == "uvy") {
      // host-written fluxes: make every face write its buffers on the next two steps
      launch_or_u8(D.kf[0], KF_WET2, (long long)D.nalloc, s());
      launch_or_u8(D.kf[1], KF_WET2, (long long)D.nalloc, s());
    }
    runner->sync();
    if (zs_exported && name == "zs") refresh_zs();
  }

  // find_quadtree_cell on a single-level grid (sfincs_quadtree.F90:764-820)
  int cell_index(double xd, double yd) const { return sfg::cell_index(*host, xd, yd); }

  void update_zbuv() {
    HostModel& h = *host;
    if (h.p.subgrid) return;  // zbuvmx exists only for regular bathymetry
    if (h.p.quadtree) throw std::runtime_error("update_zbuv is not available on quadtree meshes");
    for (long long i = 0; i < h.np; i++) h.zb[h.cmp_off[i]] = h.zb_cmp[i];
    const int ld = h.p.ld;
    for (int m = 1; m <= h.p.mmax; m++)
      for (int n = 1; n <= h.p.nmax; n++) {
        const size_t c = (size_t)m * ld + kGhostPad + n;
        if (!(h.flags[c] & F_ACT)) continue;
        if (m < h.p.mmax && (h.flags[c + ld] & F_ACT)) h.zbmx_u[c] = std::max(h.zb[c], h.zb[c + ld]) + h.p.huthresh;
        if (n < h.p.nmax && (h.flags[c + 1] & F_ACT)) h.zbmx_v[c] = std::max(h.zb[c], h.zb[c + 1]) + h.p.huthresh;
      }
    const size_t NA = (size_t)h.p.nalloc;
    check_cuda(cudaMemcpy((void*)dev->dev().zb, h.zb.data(), NA * 4, cudaMemcpyHostToDevice), "zb");
    check_cuda(cudaMemcpy((void*)dev->dev().zbmx_u, h.zbmx_u.data(), NA * 4, cudaMemcpyHostToDevice), "zbmx_u");
    check_cuda(cudaMemcpy((void*)dev->dev().zbmx_v, h.zbmx_v.data(), NA * 4, cudaMemcpyHostToDevice), "zbmx_v");
  }
};

struct EnsembleHandle {
  std::vector<std::unique_ptr<HostModel>> hosts;
  std::vector<std::unique_ptr<DeviceModel>> devs;
  std::unique_ptr<Runner> runner;
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
};

ModelHandle* g_bmi = nullptr;

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

void copy_err(char* err, int errlen, const std::string& msg) {
  if (err && errlen > 0) {
    std::strncpy(err, msg.c_str(), (size_t)errlen - 1);
    err[errlen - 1] = 0;
  }
}

int require_bmi() {
  if (!g_bmi) throw std::runtime_error("model not initialized (call initialize first)");
  return 0;
}

}  // namespace

void set_last_error(const std::string& msg) { g_err = msg; }

}  // namespace sfg

using sfg::g_bmi;
using sfg::g_err;
using sfg::guarded;

extern "C" {

int BMI_LENVARADDRESS = 64;
int BMI_LENVARTYPE = 64;
int BMI_LENGRIDTYPE = 64;
int BMI_LENCOMPONENTNAME = 64;
int BMI_LENVERSION = 256;
int BMI_LENERRMESSAGE = 1024;

int initialize_config(const char* model_dir) {
  return guarded([&] {
    if (g_bmi) throw std::runtime_error("model already initialized (call finalize first)");
    g_bmi = new sfg::ModelHandle(model_dir ? model_dir : ".", true);
    return 0;
  });
}

int initialize(void) { return initialize_config("."); }

int update(void) {
  return guarded([&] {
    sfg::require_bmi();
    g_bmi->step_once();
    g_bmi->after_update();
    g_bmi->runner->sync();  // the step is complete when update() returns, as in the reference
    g_bmi->check_fault();
    g_bmi->after_step_output();
    return 0;
  });
}

int update_until(double t_target) {
  return guarded([&] {
    sfg::require_bmi();
    g_bmi->before_update();
    g_bmi->run(t_target, -1, 32);
    g_bmi->after_update();
    return 0;
  });
}

int finalize(void) {
  int err = 0;
  int rc = guarded([&] {
    if (!g_bmi) return 0;
    double s[19];
    g_bmi->scalars(s);
    err = (int)s[4];
    g_bmi->finalize_output();
    delete g_bmi;
    g_bmi = nullptr;
    return 0;
  });
  return rc != 0 ? rc : err;
}

int get_value_ptr(const char* name, void** ptr) {
  *ptr = nullptr;
  return guarded([&]() -> int {
    sfg::require_bmi();
    std::string n(name);
    sfg::HostModel& h = *g_bmi->host;
    if (n == "z_xz")
      *ptr = h.z_xz.data();
    else if (n == "z_yz")
      *ptr = h.z_yz.data();
    else if (n == "zs") {
      g_bmi->zs_exported = true;
      g_bmi->refresh_zs();
      *ptr = g_bmi->h_zs;
    } else if (n == "zb" && !h.p.subgrid)
      *ptr = h.zb_cmp.data();
    else if (n == "subgrid_z_zmin" && h.p.subgrid)
      *ptr = h.zmin_cmp.data();
    else if (n == "qext" && h.p.use_qext) {
      g_bmi->qext_exported = true;
      *ptr = g_bmi->h_qext;
    } else
      return -1;
    return 0;
  });
}

int get_var_shape(const char* name, int shape[6]) {
  for (int i = 0; i < 6; i++) shape[i] = 0;
  return guarded([&]() -> int {
    sfg::require_bmi();
    std::string n(name);
    if (n == "z_xz" || n == "z_yz" || n == "zs" || n == "zb" || n == "uorb" || n == "subgrid_z_zmin" || n == "qext" ||
        n == "z_index_z_n" || n == "z_index_z_m") {
      shape[0] = (int)g_bmi->np();
      return 0;
    }
    return -1;
  });
}

int get_var_type(const char* name, char* type) {
  std::string n(name), t;
  if (n == "z_xz" || n == "z_yz" || n == "zb" || n == "subgrid_z_zmin" || n == "qext" || n == "uorb")
    t = "float";
  else if (n == "zs")
    t = "double";
  else if (n == "z_index_z_n" || n == "z_index_z_m")
    t = "integer";
  else {
    if (type) type[0] = 0;
    return -1;
  }
  std::strcpy(type, t.c_str());
  return 0;
}

int get_var_rank(const char* name, int* rank) {
  std::string n(name);
  if (n == "z_xz" || n == "z_yz" || n == "zs" || n == "zb" || n == "subgrid_z_zmin" || n == "qext" || n == "uorb") {
    *rank = 1;
    return 0;
  }
  return -1;
}

int set_logical(const char* name, const int* value) {
  return guarded([&]() -> int {
    sfg::require_bmi();
    if (std::string(name) != "qext") return -1;
    const bool on = value[0] != 0;
    sfg::ScnDev& D = g_bmi->dev->dev();
    if (on && !D.qext) throw std::runtime_error("qext array was not allocated for this model");
    D.use_qext = on ? 1 : 0;
    g_bmi->runner->refresh_params();
    return 0;
  });
}

int get_start_time(double* t) {
  return guarded([&] {
    sfg::require_bmi();
    *t = g_bmi->host->t0;
    return 0;
  });
}
int get_end_time(double* t) {
  return guarded([&] {
    sfg::require_bmi();
    *t = g_bmi->host->t1;
    return 0;
  });
}
int get_time_step(double* dt) {
  return guarded([&] {
    sfg::require_bmi();
    double s[19];
    g_bmi->scalars(s);
    *dt = s[1];
    return 0;
  });
}
int get_current_time(double* t) {
  return guarded([&] {
    sfg::require_bmi();
    double s[19];
    g_bmi->scalars(s);
    *t = s[0];
    return 0;
  });
}

int update_zbuv(void) {
  return guarded([&] {
    sfg::require_bmi();
    g_bmi->update_zbuv();
    return 0;
  });
}

int update_apparent_roughness(void) { return 0; }

int get_sfincs_cell_index(const double* x, const double* y, int* index) {
  return guarded([&] {
    sfg::require_bmi();
    *index = g_bmi->cell_index(*x, *y);
    return 0;
  });
}

int get_sfincs_cell_indices(const double* x, const double* y, int* index, int n) {
  return guarded([&] {
    sfg::require_bmi();
    for (int i = 0; i < n; i++) index[i] = g_bmi->cell_index(x[i], y[i]);
    return 0;
  });
}

int get_sfincs_cell_area(const int* index, double* area) {
  return guarded([&] {
    sfg::require_bmi();
    if (*index < 1 || *index > g_bmi->np()) throw std::runtime_error("cell index out of range");
    const sfg::HostModel& h = *g_bmi->host;
    if (h.p.geo)  // cell_area_m2 (sfincs_bmi.f90:359-362)
      *area = (double)h.geo_area[(size_t)h.cmp_off[(size_t)*index - 1]];
    else if (h.p.quadtree)
      *area = (double)h.cell_area[(size_t)*index - 1];
    else
      *area = (double)h.p.area;
    return 0;
  });
}

int get_last_bmi_error(char* msg) {
  sfg::copy_err(msg, BMI_LENERRMESSAGE, g_err);
  return 0;
}

int get_var(const char* name, void* dst, size_t bytes) {
  return guarded([&] {
    sfg::require_bmi();
    g_bmi->get(name, dst, bytes);
    return 0;
  });
}

int set_var(const char* name, const void* src, size_t bytes) {
  return guarded([&] {
    sfg::require_bmi();
    g_bmi->set(name, src, bytes);
    return 0;
  });
}

// ---------------------------------------------------------------- model handles
void* sfg_model_create(const char* model_dir, int bmi, char* err, int errlen) {
  try {
    return new sfg::ModelHandle(model_dir, bmi != 0);
  } catch (std::exception& e) {
    sfg::copy_err(err, errlen, e.what());
    g_err = e.what();
    return nullptr;
  }
}
void sfg_model_destroy(void* m) { delete static_cast<sfg::ModelHandle*>(m); }
int sfg_model_finalize(void* m) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->finalize_output();
    return 0;
  });
}
int sfg_model_run(void* m, double t_end, long long max_steps, int chunk) {
  return guarded([&] {
    auto* h = static_cast<sfg::ModelHandle*>(m);
    h->run(t_end, max_steps, chunk > 0 ? chunk : 32);
    return 0;
  });
}
int sfg_model_set_autotune(void* m, int on) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->runner->set_autotune(on != 0);
    return 0;
  });
}
int sfg_model_variant(void* m) { return static_cast<sfg::ModelHandle*>(m)->runner->variant(); }
int sfg_model_set_variant(void* m, int variant) {
  return guarded([&] {
    if (variant < 2 || variant > 5) throw std::runtime_error("kernel variant must be 2, 3, 4 or 5");
    static_cast<sfg::ModelHandle*>(m)->runner->set_variant(variant);
    return 0;
  });
}
int sfg_model_issue(void* m, int nsteps) {
  return guarded([&] {
    auto* h = static_cast<sfg::ModelHandle*>(m);
    // unbounded target so that issued steps always execute
    const double big = 1.0e300;
    const int left = -1;
    sfg::check_cuda(cudaMemcpyAsync(&h->dev->state()->tend, &big, 8, cudaMemcpyHostToDevice, h->s()), "tend");
    sfg::check_cuda(cudaMemcpyAsync(&h->dev->state()->steps_left, &left, 4, cudaMemcpyHostToDevice, h->s()), "left");
    h->runner->issue(nsteps);
    sfg::check_cuda(cudaGetLastError(), "issue");
    return 0;
  });
}
int sfg_model_sync(void* m) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->runner->sync();
    static_cast<sfg::ModelHandle*>(m)->check_fault();
    return 0;
  });
}
int sfg_model_scalars(void* m, double out[19]) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->scalars(out);
    return 0;
  });
}
int sfg_model_get(void* m, const char* name, void* dst, size_t bytes) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->get(name, dst, bytes);
    return 0;
  });
}
int sfg_model_set(void* m, const char* name, const void* src, size_t bytes) {
  return guarded([&] {
    static_cast<sfg::ModelHandle*>(m)->set(name, src, bytes);
    return 0;
  });
}
int sfg_model_volume(void* m, double* v) {
  return guarded([&] {
    *v = static_cast<sfg::ModelHandle*>(m)->volume();
    return 0;
  });
}
// No try/catch wrapper and no std::string on the success path: this entry
// point allocates nothing (see volume_noalloc in aux_kernels.cu).
int sfg_model_volume_noalloc(void* m, double* v) {
  if (!m || !v) {
    sfg::g_err = "sfg_model_volume_noalloc: null model or output pointer";
    return 1;
  }
  auto* h = static_cast<sfg::ModelHandle*>(m);
  const char* why = nullptr;
  if (sfg::volume_noalloc(h->runner->d_scns(), h->dev->d_cmp_off(), h->np(), h->s(), v, &why)) {
    sfg::g_err = std::string("sfg_model_volume_noalloc: ") + (why ? why : "failed");
    return 1;
  }
  return 0;
}
void* sfg_model_stream(void* m) { return (void*)static_cast<sfg::ModelHandle*>(m)->s(); }
int sfg_model_kernel_times(void* m, int nsteps, double ms_out[4], int* launches_per_step) {
  return guarded([&] {
    auto* h = static_cast<sfg::ModelHandle*>(m);
    const double big = 1.0e300;
    const int left = -1;
    sfg::check_cuda(cudaMemcpyAsync(&h->dev->state()->tend, &big, 8, cudaMemcpyHostToDevice, h->s()), "tend");
    sfg::check_cuda(cudaMemcpyAsync(&h->dev->state()->steps_left, &left, 4, cudaMemcpyHostToDevice, h->s()), "left");
    auto t = h->runner->time_kernels(nsteps);
    for (int k = 0; k < 4; k++) ms_out[k] = t[k];
    if (launches_per_step) *launches_per_step = h->runner->launches_per_step();
    return 0;
  });
}

// ---------------------------------------------------------------- ensembles
void* sfg_ensemble_create(const char* const* dirs, int n, int bmi, char* err, int errlen) {
  auto* e = new sfg::EnsembleHandle();
  try {
    std::vector<sfg::DeviceModel*> ptrs;
    size_t maxnp = 1;
    for (int i = 0; i < n; i++) {
      e->hosts.push_back(sfg::load_model(dirs[i], bmi != 0));
      e->devs.push_back(std::make_unique<sfg::DeviceModel>(*e->hosts.back()));
      ptrs.push_back(e->devs.back().get());
      maxnp = std::max(maxnp, (size_t)e->hosts.back()->np);
    }
    e->runner = std::make_unique<sfg::Runner>(ptrs);
    e->stage_bytes = maxnp * 8 * 2;
    sfg::check_cuda(cudaMalloc(&e->d_stage, e->stage_bytes), "stage");
    return e;
  } catch (std::exception& ex) {
    sfg::copy_err(err, errlen, ex.what());
    g_err = ex.what();
    e->runner.reset();
    e->devs.clear();
    delete e;
    return nullptr;
  }
}
void sfg_ensemble_destroy(void* ev) {
  auto* e = static_cast<sfg::EnsembleHandle*>(ev);
  if (!e) return;
  e->runner.reset();
  e->devs.clear();
  if (e->d_stage) cudaFree(e->d_stage);
  delete e;
}
int sfg_ensemble_run(void* ev, const double* t_end, long long max_steps, int chunk) {
  return guarded([&] {
    auto* e = static_cast<sfg::EnsembleHandle*>(ev);
    std::vector<double> te(t_end, t_end + e->devs.size());
    e->runner->run(te, max_steps, chunk > 0 ? chunk : 32);
    for (int i = 0; i < (int)e->devs.size(); i++)
      if (e->runner->read_state(i).fault)
        throw std::runtime_error("ensemble member " + std::to_string(i) +
                                 ": a staged kernel gave up waiting for its tile data (fault flag set)");
    return 0;
  });
}
int sfg_ensemble_set_autotune(void* ev, int on) {
  return guarded([&] {
    static_cast<sfg::EnsembleHandle*>(ev)->runner->set_autotune(on != 0);
    return 0;
  });
}
int sfg_ensemble_variant(void* ev) { return static_cast<sfg::EnsembleHandle*>(ev)->runner->variant(); }
int sfg_ensemble_set_variant(void* ev, int variant) {
  return guarded([&] {
    if (variant < 2 || variant > 5) throw std::runtime_error("kernel variant must be 2, 3, 4 or 5");
    static_cast<sfg::EnsembleHandle*>(ev)->runner->set_variant(variant);
    return 0;
  });
}
int sfg_ensemble_issue(void* ev, int nsteps) {
  return guarded([&] {
    auto* e = static_cast<sfg::EnsembleHandle*>(ev);
    const double big = 1.0e300;
    const int left = -1;
    for (auto& d : e->devs) {
      sfg::check_cuda(cudaMemcpyAsync(&d->state()->tend, &big, 8, cudaMemcpyHostToDevice, e->runner->stream()), "tend");
      sfg::check_cuda(cudaMemcpyAsync(&d->state()->steps_left, &left, 4, cudaMemcpyHostToDevice, e->runner->stream()),
                      "left");
    }
    e->runner->issue(nsteps);
    sfg::check_cuda(cudaGetLastError(), "issue");
    return 0;
  });
}
int sfg_ensemble_sync(void* ev) {
  return guarded([&] {
    static_cast<sfg::EnsembleHandle*>(ev)->runner->sync();
    return 0;
  });
}
int sfg_ensemble_scalars(void* ev, int i, double out[19]) {
  return guarded([&] {
    auto* e = static_cast<sfg::EnsembleHandle*>(ev);
    if (i < 0 || i >= (int)e->devs.size()) throw std::runtime_error("member index out of range");
    sfg::StepState st = e->runner->read_state(i);
    const sfg::HostModel& h = *e->hosts[i];
    double t = st.stop_pending ? h.t1 + 1.0 : st.t;
    double v[19] = {t, st.dt, st.min_dt, (double)st.nt, (double)st.error, h.t0, h.t1, (double)h.np, (double)h.npuv,
                    (double)h.p.nkcuv2, (double)h.p.ngbnd, (double)h.p.subgrid, st.bflux_vol,
                    st.rain_vol * h.area_total_kcs1, st.src_vol, h.p.dtmax, h.p.dtmin, (double)e->devs[i]->bytes(),
                    (double)e->runner->ntiles()};
    std::memcpy(out, v, sizeof(v));
    return 0;
  });
}
int sfg_ensemble_get(void* ev, int i, const char* name, void* dst, size_t bytes) {
  return guarded([&] {
    auto* e = static_cast<sfg::EnsembleHandle*>(ev);
    if (i < 0 || i >= (int)e->devs.size()) throw std::runtime_error("member index out of range");
    sfg::DeviceModel& d = *e->devs[i];
    const long long n = e->hosts[i]->np;
    sfg::StepState st = e->runner->read_state(i);
    const int p = st.run ? (st.parity ^ 1) : st.parity;
    std::string nm(name);
    cudaStream_t s = e->runner->stream();
    if (nm == "zs") {
      if (bytes != (size_t)n * 8) throw std::runtime_error("wrong size for zs");
      sfg::launch_gather_f32_f64(d.dev().zs, d.d_cmp_off(), (double*)e->d_stage, n, s);
    } else if (nm == "z_volume") {
      if (!d.dev().zvol) throw std::runtime_error("z_volume exists only for subgrid models");
      if (bytes != (size_t)n * 8) throw std::runtime_error("wrong size for z_volume");
      sfg::launch_gather_f64(d.dev().zvol, d.d_cmp_off(), (double*)e->d_stage, n, s);
    } else {
      const float* src = nullptr;
      const int32_t* map = d.d_cmp_off();
      if (nm == "zsmax") src = d.dev().zsmax;
      else if (nm == "vmax" && d.dev().vmax) src = d.dev().vmax;
      else if (nm == "qmax" && d.dev().qmax) src = d.dev().qmax;
      else if (nm == "twet" && d.dev().twet) src = d.dev().twet;
      else if (nm == "tzsmax" && d.dev().tzsmax) src = d.dev().tzsmax;
      else if (nm == "qx") src = d.dev().qu[p], map = d.face_map(0);
      else if (nm == "qy") src = d.dev().qv[p], map = d.face_map(1);
      else if (nm == "uvx") src = d.dev().uu[p], map = d.face_map(0);
      else if (nm == "uvy") src = d.dev().vv[p], map = d.face_map(1);
      else throw std::runtime_error("unknown ensemble variable " + nm);
      if (bytes != (size_t)n * 4) throw std::runtime_error("wrong size for " + nm);
      sfg::launch_gather_f32(src, map, (float*)e->d_stage, n, s);
    }
    sfg::check_cuda(cudaMemcpyAsync(dst, e->d_stage, bytes, cudaMemcpyDeviceToHost, s), "get");
    e->runner->sync();
    return 0;
  });
}
void* sfg_ensemble_stream(void* ev) { return (void*)static_cast<sfg::EnsembleHandle*>(ev)->runner->stream(); }
int sfg_ensemble_kernel_times(void* ev, int nsteps, double ms_out[4], int* launches_per_step) {
  return guarded([&] {
    auto* e = static_cast<sfg::EnsembleHandle*>(ev);
    const double big = 1.0e300;
    const int left = -1;
    for (auto& d : e->devs) {
      sfg::check_cuda(cudaMemcpyAsync(&d->state()->tend, &big, 8, cudaMemcpyHostToDevice, e->runner->stream()), "tend");
      sfg::check_cuda(cudaMemcpyAsync(&d->state()->steps_left, &left, 4, cudaMemcpyHostToDevice, e->runner->stream()),
                      "left");
    }
    auto t = e->runner->time_kernels(nsteps);
    for (int k = 0; k < 4; k++) ms_out[k] = t[k];
    if (launches_per_step) *launches_per_step = e->runner->launches_per_step();
    return 0;
  });
}

int sfg_layout_get(const char* model_dir, int bmi, const char* name, double* dst, size_t n) {
  return guarded([&]() -> int {
    auto H = sfg::load_model(model_dir, bmi != 0);
    const sfg::HostModel& h = *H;
    const std::string nm(name);
    std::vector<double> out;
    const size_t NA = (size_t)h.p.nalloc;
    auto per_cell = [&](auto get) {
      out.resize((size_t)h.np);
      for (long long i = 0; i < h.np; i++) out[i] = (double)get((size_t)h.cmp_off[i]);
    };
    if (nm == "counts") {
      out = {(double)h.np,    (double)h.npuv,  (double)h.p.ngbnd, (double)h.p.nkcuv2, (double)h.p.nlev,
             (double)NA,      (double)h.p.dtmax, (double)h.p.dtmin, h.t0, h.t1};
    } else if (nm == "flags") {
      per_cell([&](size_t c) { return h.flags[c]; });
    } else if (nm == "zs") {
      per_cell([&](size_t c) { return h.zs[c]; });
    } else if (nm == "zvol") {
      if (h.zvol.empty()) return -1;
      per_cell([&](size_t c) { return h.zvol[c]; });
    } else if (nm == "zbmx" || nm == "gn2") {
      const auto& u = nm == "zbmx" ? h.zbmx_u : h.gn2_u;
      const auto& v = nm == "zbmx" ? h.zbmx_v : h.gn2_v;
      if (u.empty()) return -1;
      out.resize((size_t)h.np * 2);
      for (long long i = 0; i < h.np; i++) {
        out[i] = u[h.cmp_off[i]];
        out[h.np + i] = v[h.cmp_off[i]];
      }
    } else if (nm == "uvmean0") {  // initial boundary mean fluxes, boundary-face order
      out.assign(h.uvmean0.begin(), h.uvmean0.end());
      out.resize(h.bfaces.size(), 0.0);
    } else if (nm == "uv0" || nm == "q0") {  // initial u then v face values per cell (restart)
      const auto& u = nm == "uv0" ? h.uv0u : h.q0u;
      const auto& v = nm == "uv0" ? h.uv0v : h.q0v;
      out.assign((size_t)h.np * 2, 0.0);
      if (!u.empty())
        for (long long i = 0; i < h.np; i++) {
          out[i] = u[h.cmp_off[i]];
          out[h.np + i] = v[h.cmp_off[i]];
        }
    } else if (nm == "nstruc") {
      out = {(double)h.struc.size()};
    } else if (nm == "struc") {
      // per weir face: compact cell (0-based; on a quadtree the uv point), direction, crest level, Cd,
      // relative length
      for (auto& w : h.struc)
        for (double v : {h.p.quadtree ? (double)w.face : (double)h.dense2cmp[w.face], (double)w.dir, (double)w.height,
                         (double)w.cd, (double)w.len})
          out.push_back(v);
    } else if (nm == "crs_faces") {  // per crossed face: cross-section, cell (0-based compact), direction, sign
      for (size_t c = 0; c < h.out.crs.size(); c++)
        for (const auto& f : h.out.crs[c].faces) {
          const double cell = h.p.quadtree ? (double)h.qface[(size_t)f.face].nm : (double)h.dense2cmp[(size_t)f.face];
          for (double v : {(double)c, cell, (double)f.dir, (double)f.idir}) out.push_back(v);
        }
    } else if (nm == "tide_omega") {
      out.assign(h.tide.omega.begin(), h.tide.omega.end());
    } else if (nm == "tide_amp") {
      out.assign(h.tide.amp.begin(), h.tide.amp.end());
    } else if (nm == "tide_phase") {
      out.assign(h.tide.phase.begin(), h.tide.phase.end());
    } else if (nm == "gb_cell") {
      for (auto c : h.gb_cmp) out.push_back((double)c);
    } else if (nm == "kb_cell") {
      for (auto& b : h.bfaces)
        out.push_back(h.p.quadtree ? (double)h.qface[b.face].nm : (double)h.dense2cmp[b.face]);
    } else if (h.p.quadtree && nm == "qt_counts") {
      out = {(double)h.np, (double)h.npuv, (double)h.p.ncuv, (double)h.p.nref};
    } else if (h.p.quadtree && nm.compare(0, 3, "uv_") == 0) {
      // uv-point arrays, 1-based indices as in the reference
      for (auto& f : h.qface) {
        double v;
        if (nm == "uv_nm") v = f.nm + 1;
        else if (nm == "uv_nmu") v = f.nmu + 1;
        else if (nm == "uv_dir") v = (f.info & sfg::QF_DIR) ? 1 : 0;
        else if (nm == "uv_iref") v = (double)(((f.info >> 8) & 15u) + 1);
        else if (nm == "uv_trans") v = (f.info & sfg::QF_TRANS) ? 1 : 0;
        else if (nm == "uv_act") v = (f.info & sfg::QF_ACT) ? 1 : 0;
        else if (nm == "uv_adv") v = (f.info & sfg::QF_ADV) ? 1 : 0;
        else if (nm == "uv_th") v = (f.info & sfg::QF_TH) ? 1 : 0;
        else if (nm == "uv_u_nmd") v = f.u_nmd + 1;
        else if (nm == "uv_u_nmu") v = f.u_nmu + 1;
        else if (nm == "uv_u_ndm") v = f.u_ndm + 1;
        else if (nm == "uv_u_num") v = f.u_num + 1;
        else if (nm == "uv_v_ndm") v = f.v_ndm + 1;
        else if (nm == "uv_v_nm") v = f.v_nm + 1;
        else if (nm == "uv_v_ndmu") v = f.v_ndmu + 1;
        else if (nm == "uv_v_nmu") v = f.v_nmu + 1;
        else return -1;
        out.push_back(v);
      }
    } else if (h.p.quadtree && nm.compare(0, 5, "z_uv_") == 0) {
      for (auto& c : h.qcell) {
        if (nm == "z_uv_md") out.push_back(c.x + 1);
        else if (nm == "z_uv_mu") out.push_back(c.y + 1);
        else if (nm == "z_uv_nd") out.push_back(c.z + 1);
        else if (nm == "z_uv_nu") out.push_back(c.w + 1);
        else return -1;
      }
    } else if (h.p.quadtree && (nm == "cuv_uv1" || nm == "cuv_uv2")) {
      for (auto& c : h.qcuv) out.push_back((nm == "cuv_uv1" ? c.x : c.y) + 1);
    } else if (h.p.quadtree && (nm == "zbuvmx" || nm == "gn2uv")) {
      const auto& v = nm == "zbuvmx" ? h.zbmx_q : h.gn2_q;
      if (v.empty()) return -1;
      out.assign(v.begin(), v.end());
    } else if (nm == "kb_dir") {
      for (auto& b : h.bfaces) out.push_back((double)(b.info & 1));
    } else if (nm == "kb_sign") {
      for (auto& b : h.bfaces) out.push_back((b.info & 2) ? 1.0 : -1.0);
    } else if (nm == "kb_fac") {
      for (auto& b : h.bfaces) out.push_back((double)b.fac);
    } else {
      return -1;
    }
    if (out.size() != n) throw std::runtime_error("sfg_layout_get(" + nm + "): size is " + std::to_string(out.size()));
    std::memcpy(dst, out.data(), n * sizeof(double));
    return 0;
  });
}

}  // extern "C"
