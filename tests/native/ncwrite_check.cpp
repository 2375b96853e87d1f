// Writes a small netCDF file through the core's CDF-2 writer (sfincs_b200/csrc/host/ncwrite.h):
// fixed and record variables of every type the output files use, attributes, a partial
// hyperslab of a fixed variable and three records.
#include <cstdio>
#include <vector>

#include "ncwrite.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  sfg::NcWriter nc;
  const int dn = nc.def_dim("n", 3), dm = nc.def_dim("m", 5), dt = nc.def_dim("time", sfg::NcWriter::UNLIMITED),
            dk = nc.def_dim("timemax", 2), dl = nc.def_dim("len", 7);
  nc.att_text(sfg::NcWriter::GLOBAL, "title", "writer check");
  const int vx = nc.def_var("x", sfg::NcWriter::FLOAT, {dn, dm});
  nc.att_float(vx, "_FillValue", -99999.0f);
  nc.att_text(vx, "units", "m");
  const int vi = nc.def_var("msk", sfg::NcWriter::INT, {dn, dm});
  nc.att_int(vi, "flag_values", {0, 1, 2});
  const int vd = nc.def_var("xd", sfg::NcWriter::DOUBLE, {dm});
  const int vc = nc.def_var("name", sfg::NcWriter::CHAR, {dn, dl});
  const int vk = nc.def_var("zsmax", sfg::NcWriter::FLOAT, {dk, dn, dm});
  nc.att_float(vk, "_FillValue", -99999.0f);
  const int vs = nc.def_var("scalar", sfg::NcWriter::INT, {});
  const int vt = nc.def_var("time", sfg::NcWriter::FLOAT, {dt});
  const int vz = nc.def_var("zs", sfg::NcWriter::FLOAT, {dt, dn, dm});
  const int vq = nc.def_var("qd", sfg::NcWriter::DOUBLE, {dt, dm});
  nc.create(argv[1]);
  std::vector<float> x(15);
  std::vector<int32_t> msk(15);
  for (int i = 0; i < 15; i++) x[i] = 0.5f * (float)i, msk[i] = i % 3;
  nc.put(vx, x.data(), x.size());
  nc.put(vi, msk.data(), msk.size());
  std::vector<double> xd = {1.0, 2.5, -3.25, 1e300, -0.0};
  nc.put(vd, xd.data(), xd.size());
  const char names[22] = "abc    de     fghijkl";
  nc.put(vc, names, 21);
  std::vector<float> z(15);
  for (int i = 0; i < 15; i++) z[i] = 100.0f + (float)i;
  nc.put(vk, z.data(), 15, 15);  // the second timemax slab only
  const int32_t one = 42;
  nc.put(vs, &one, 1);
  for (int r = 0; r < 3; r++) {
    const float t = 600.0f * (float)r;
    nc.put_record(vt, r, &t, 1);
    for (int i = 0; i < 15; i++) z[i] = (float)(r * 100 + i);
    nc.put_record(vz, r, z.data(), 15);
    std::vector<double> q(5, (double)r + 0.125);
    nc.put_record(vq, r, q.data(), 5);
  }
  nc.close();
  return 0;
}
