// Map, his and max output of one model (sfincs_output.f90:8-258,
// sfincs_ncoutput.F90:148-1590): netCDF files (sfincs_map.nc,
// sfincs_his.nc) or the reference's binary / text files, written off the
// step's critical path.  At an output time the fields are gathered on the
// device into staging buffers (a few microseconds on the model's stream),
// the max fields are reset there, and the device-to-host copies and the file
// writes run on a copy stream and a writer thread while the model keeps
// stepping.
#pragma once
#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "model.h"

namespace sfg {

class NcWriter;

class OutputWriter {
 public:
  OutputWriter(const HostModel& h, DeviceModel& d, cudaStream_t main);
  ~OutputWriter();
  OutputWriter(const OutputWriter&) = delete;
  OutputWriter& operator=(const OutputWriter&) = delete;

  // next output times (1e9: none) and counts (sfincs_lib.f90:419-476)
  double tmapout = 1.0e9, tmaxout = 1.0e9, thisout = 1.0e9;
  int ntmapout = 0, ntmaxout = 0, nthisout = 0;

  // Writes the outputs flagged, at time tout, from the model's state after
  // the step; parity: the flux buffer that holds the latest q / uv.
  void write(bool map, bool max, bool his, double tout, int parity);
  // finalize_output (sfincs_output.f90:260-296): the max fields at the end
  // when an interval was not completed, the run's scalars, the files closed.
  void finalize(double t, double t1, int parity, float average_dt, int status);
  // Waits for the copies and file writes in flight.
  void drain();

 private:
  struct Slot {  // one gathered field
    void* dev = nullptr;
    void* host = nullptr;  // pinned
    size_t n = 0, esize = 4;
  };
  const HostModel& h_;
  DeviceModel& d_;
  cudaStream_t main_ = nullptr, copy_ = nullptr;
  cudaEvent_t gathered_ = nullptr, copied_ = nullptr;
  int32_t* d_maps_ = nullptr;  // device gather maps: md, nd, mu, nu uv points of every cell; obs cells
  size_t np_ = 0, nobs_ = 0, ncrs_ = 0, ncrs_faces_ = 0, ndrn_ = 0, nrug_ = 0, nrug_pts_ = 0;
  bool map_net_ = false, map_bin_ = false, his_net_ = false, his_txt_ = false, max_on_ = false;
  int infstate_ = 0;  // map state of the infiltration: 3 Seff, 4 sigma, 5 f
  std::unique_ptr<NcWriter> map_nc_, his_nc_;
  FILE* zs_dat_ = nullptr;
  FILE* zvol_dat_ = nullptr;
  std::vector<FILE*> max_dat_;
  std::vector<Slot> slots_;
  std::vector<int> max_vars_;  // netCDF ids: timemax, zsmax, cumprcp, tmax, t_zsmax, hmax, vmax, qmax, cuminf (-1: off)
  std::vector<int> rec_ids_;   // netCDF ids: time, zs, h, u, v, subgrid_volume, infiltration state (-1: off)
  std::vector<int> his_ids_;   // netCDF ids: time, point_zs, point_h, point_u, point_v, point_uvmag, point_uvdir,
                               // point_qinf, point_S, crosssection_discharge, drainage_discharge,
                               // runup_gauge_zs
  std::vector<size_t> file_idx_;  // file position (n, m) or quadtree point of every compact cell
  size_t ncells_file_ = 0;
  float huthresh_ = 0;
  // worker
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> jobs_;
  bool busy_ = false, stop_ = false;
  std::string error_;

  // a compact cell field in the file's cell layout: fill where skipped
  std::vector<float> scatter(const float* v, const std::vector<uint8_t>* keep = nullptr) const;
  size_t file_index(size_t i) const { return file_idx_[i]; }
  size_t cells_total() const { return ncells_file_; }
  void post(std::function<void()> job);
  void run_worker();
  Slot& slot(int k) { return slots_[(size_t)k]; }
  void gather(int k, const void* src, const int32_t* map, bool f64 = false);
  void open_map();
  void open_his();
  void open_max_bin();
  void write_map_files(double tout, int rec);
  void write_max_files(double tout, int rec);
  void write_his_files(double tout, int rec);
  // discharge through each cross-section from the gathered face fluxes
  std::vector<float> crs_discharges();
};

}  // namespace sfg
