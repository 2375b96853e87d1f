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
float meteo_time(const std::string& line, const std::string& tref) {
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

namespace sfg {

// Value of a "key = value" eye line: the twelve characters after '=' (read_spw_file,
// sfincs_spiderweb.f90:96-108).
static float spw_eye_value(const std::string& line, const std::string& file) {
  const size_t e = line.find('=');
  if (e == std::string::npos) throw std::runtime_error("spiderweb file " + file + ": no value in '" + line + "'");
  return std::strtof(line.substr(e + 1, 12).c_str(), nullptr);
}

void read_spw_file(const std::string& file, const std::string& tref, bool use_precip, SpwHost& s) {
  std::ifstream f(file);
  if (!f) throw std::runtime_error("cannot open spiderweb file " + file);
  std::vector<std::string> lines;
  for (std::string l; std::getline(f, l);) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines.push_back(l);
  }
  // header keys (read_spw_dimensions, sfincs_spiderweb.f90:231-255)
  std::map<std::string, std::string> kv;
  for (const std::string& l : lines) {
    if (l.compare(0, 4, "TIME") == 0) break;
    const size_t e = l.find('=');
    if (e == std::string::npos) continue;
    std::string k = l.substr(0, e);
    k.erase(0, k.find_first_not_of(" \t"));
    k.erase(k.find_last_not_of(" \t") + 1);
    for (auto& ch : k) ch = (char)std::tolower((unsigned char)ch);
    kv[k] = l.substr(e + 1);
  }
  auto num = [&](const char* k) {
    auto it = kv.find(k);
    return it == kv.end() ? 0.0 : std::strtod(it->second.c_str(), nullptr);
  };
  s.ncols = (int)num("n_cols");
  s.nrows = (int)num("n_rows");
  s.nquant = (int)num("n_quantity");
  s.radius = (float)num("spw_radius");
  if (s.ncols < 1 || s.nrows < 2 || (s.nquant != 3 && s.nquant != 4) || !(s.radius > 0.0f))
    throw std::runtime_error("spiderweb file " + file + ": needs n_cols, n_rows >= 2, n_quantity 3 or 4 and spw_radius");
  // the first TIME line within the first 30 lines ends the header, else 16 / 18 lines (:50-79)
  size_t nheader = 0;
  bool found = false;
  for (size_t ip = 0; ip < 30 && ip < lines.size(); ip++)
    if (lines[ip].compare(0, 4, "TIME") == 0) {
      nheader = ip;
      found = true;
      break;
    }
  if (!found) nheader = s.nquant == 4 ? 18 : 16;
  // blocks: TIME, eye x, eye y, eye pressure drop, then nrows lines per quantity (:86-128)
  const size_t block = 4 + (size_t)s.nrows * s.nquant;
  size_t i = nheader;
  const size_t rec = (size_t)s.nrows * s.ncols;
  std::vector<float> vmag, vdir, pdrp;
  while (i < lines.size()) {
    if (i + block > lines.size()) throw std::runtime_error("spiderweb file " + file + ": a time block is incomplete");
    s.times.push_back(meteo_time(lines[i], tref));
    s.xe.push_back(spw_eye_value(lines[i + 1], file));
    s.ye.push_back(spw_eye_value(lines[i + 2], file));
    i += 4;
    for (int q = 0; q < s.nquant; q++) {
      std::vector<float>& dst = q == 0 ? vmag : q == 1 ? vdir : q == 2 ? pdrp : s.prcp;
      for (int r = 0; r < s.nrows; r++) {  // list-directed: a row starts on a new line
        int got = 0;
        while (got < s.ncols) {
          if (i >= lines.size()) throw std::runtime_error("spiderweb file " + file + ": a row is incomplete");
          std::istringstream ls(lines[i++]);
          double x;
          while (got < s.ncols && ls >> x) {
            dst.push_back((float)x);
            got++;
          }
        }
      }
    }
    // rows spread over several lines shift the block grid; the reference counts one line per row
    if (i != nheader + s.times.size() * block)
      throw std::runtime_error("spiderweb file " + file + ": rows must be one line each");
  }
  s.nt = (int)s.times.size();
  if (s.nt == 0) throw std::runtime_error("spiderweb file " + file + " holds no TIME blocks");
  if (s.nquant < 4) s.prcp.assign(rec * s.nt, 0.0f);
  // wind components from speed and nautical direction (sfincs_meteo.f90:72-81)
  s.wu.resize(rec * s.nt);
  s.wv.resize(rec * s.nt);
  s.pdrp = pdrp;
  const float pi = 3.14159f;
  for (size_t k = 0; k < rec * s.nt; k++) {
    const float a = pi * (270.0f - vdir[k]) / 180.0f;
    s.wu[k] = vmag[k] * std::cos(a);
    s.wv[k] = vmag[k] * std::sin(a);
  }
  s.precip = s.nquant == 4 && use_precip;
}

}  // namespace sfg
