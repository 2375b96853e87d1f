// Input readers of the B200 core: sfincs.inp keyword file, stream-binary
// arrays, ASCII time series and netCDF-3 classic variables.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace sfg {

// sfincs.inp: "keyword = value" lines; '#', '!' or '@' in column 1 comment a
// line, a trailing '#' starts a comment, tabs expand to 8-column stops and the
// first occurrence of a keyword wins (sfincs_read.f90:5-249).  Logical values
// are true when the first character is one of 1yYtT (sfincs_read.f90:178).
class InpFile {
 public:
  explicit InpFile(const std::string& path);
  bool has(const std::string& key) const { return kv_.count(key) != 0; }
  float real(const std::string& key, float def) const;
  int integer(const std::string& key, int def) const;
  std::string str(const std::string& key, const std::string& def) const;
  bool logical(const std::string& key, bool def) const;
  const std::map<std::string, std::string>& all() const { return kv_; }

 private:
  std::map<std::string, std::string> kv_;
};

// Seconds between two "yyyymmdd HHMMSS" strings (sfincs_date.f90:183-215).
long long seconds_between(const std::string& a, const std::string& b);

std::vector<std::vector<double>> read_table(const std::string& path);

template <class X>
std::vector<X> read_binary(const std::string& path, size_t n, size_t offset_bytes = 0);

// netCDF-3 classic (CDF-1/CDF-2) reader for fixed-size variables.
class NcFile {
 public:
  explicit NcFile(const std::string& path);
  long long dim(const std::string& name) const;
  bool has(const std::string& name) const { return vars_.count(name) != 0; }
  std::vector<float> floats(const std::string& name) const;
  std::vector<double> doubles(const std::string& name) const;
  double att(const std::string& name) const;  // numeric global attribute (first value)

 private:
  struct Var {
    int type;
    uint64_t begin, count;
  };
  std::string path_;
  std::map<std::string, long long> dims_;
  std::map<std::string, Var> vars_;
  std::map<std::string, double> gatts_;
  static double value_of(int type, const uint8_t* p);
};

}  // namespace sfg
