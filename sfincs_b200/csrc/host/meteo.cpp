// Gridded meteo input: the ASCII equidistant-grid files of the reference
// (amu / amv wind components, amp pressure, ampr rain; read_amuv_dimensions
// and read_amuv_file, sfincs_spiderweb.f90:135-230 and 320-403, with the
// TIME lines of compute_time_in_seconds, :409-458).  The grids go to the
// device as they are; the update-window fields are interpolated there.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "inputs.h"
#include "model.h"

namespace sfg {

// Seconds after tref of a "TIME = <v> <unit> since yyyy-mm-dd HH:MM:SS" line:
// v times the unit less (tref - that date), in the reference's real*4 and
// integer*8 steps (the difference truncated to whole seconds).
static float meteo_time(const std::string& line, const std::string& tref) {
  const size_t eq = line.find('='), since = line.find("since");
  const char* units[4] = {"seconds", "minutes", "hours", "days"};
  const long facs[4] = {1, 60, 3600, 86400};
  size_t ju = std::string::npos;
  long fac = 1;
  for (int u = 0; u < 4 && ju == std::string::npos; u++) {
    ju = line.find(units[u]);
    fac = facs[u];
  }
  if (eq == std::string::npos || since == std::string::npos || ju == std::string::npos || ju < eq ||
      line.size() < since + 25)
    throw std::runtime_error("meteo file: cannot read the time line '" + line + "'");
  const float tim = std::strtof(line.substr(eq + 1, ju - eq - 1).c_str(), nullptr);
  const std::string d = line.substr(since + 6, 19);  // yyyy-mm-dd HH:MM:SS
  const std::string date = d.substr(0, 4) + d.substr(5, 2) + d.substr(8, 2) + " " + d.substr(11, 2) +
                           d.substr(14, 2) + d.substr(17, 2);
  const long long shift = seconds_between(date, tref);  // tref - date
  const float v = tim * (float)fac - (float)shift;
  return (float)(long long)v;
}

void read_meteo_grid(const std::string& file, const std::string& tref, MeteoGridHost& g, int q) {
  std::ifstream f(file);
  if (!f) throw std::runtime_error("cannot open meteo file " + file);
  std::vector<std::string> lines;
  for (std::string l; std::getline(f, l);) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines.push_back(l);
  }
  // header keys up to the first line that starts with TIME
  std::map<std::string, std::string> kv;
  size_t i = 0;
  for (; i < lines.size() && lines[i].compare(0, 4, "TIME") != 0; i++) {
    const size_t e = lines[i].find('=');
    if (e == std::string::npos) continue;
    std::string k = lines[i].substr(0, e);
    k.erase(0, k.find_first_not_of(" \t"));
    k.erase(k.find_last_not_of(" \t") + 1);
    for (auto& ch : k) ch = (char)std::tolower((unsigned char)ch);
    kv[k] = lines[i].substr(e + 1);
  }
  auto num = [&](const char* k) {
    auto it = kv.find(k);
    return it == kv.end() ? 0.0 : std::strtod(it->second.c_str(), nullptr);
  };
  const int ncols = (int)num("n_cols"), nrows = (int)num("n_rows");
  if (ncols < 2 || nrows < 2) throw std::runtime_error("meteo file " + file + ": needs n_cols and n_rows >= 2");
  std::vector<float> times, vals;
  const size_t need = (size_t)nrows * ncols;
  while (i < lines.size()) {
    if (lines[i].compare(0, 4, "TIME") != 0) {
      i++;
      continue;
    }
    times.push_back(meteo_time(lines[i], tref));
    i++;
    size_t got = 0;
    while (got < need && i < lines.size()) {  // list-directed: values may span lines
      std::istringstream ls(lines[i++]);
      double x;
      while (got < need && ls >> x) {
        vals.push_back((float)x);
        got++;
      }
    }
    if (got < need) throw std::runtime_error("meteo file " + file + ": a time block is incomplete");
  }
  if (times.empty()) throw std::runtime_error("meteo file " + file + " holds no TIME blocks");
  if (q == 0) {
    g.nt = (int)times.size();
    g.nrows = nrows;
    g.ncols = ncols;
    g.x_ll = (float)num("x_llcorner");
    g.y_ll = (float)num("y_llcorner");
    g.dx = (float)num("dx");
    g.dy = (float)num("dy");
    g.times = times;
  } else if ((int)times.size() != g.nt || nrows != g.nrows || ncols != g.ncols) {
    throw std::runtime_error("meteo file " + file + ": the second wind component has another grid or times");
  }
  g.v[q] = vals;
}

}  // namespace sfg
