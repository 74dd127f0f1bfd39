// gs_data.h -- named fields and string variables of the front end.
//
// Field: a host array with a dimension header, the reference's Data<Real>
// as far as scripts see it (include/datamain.th:114-192): `ndim d1..dn`,
// N = product, row-major with the last index fastest, float values.  The
// device copy lives in the plugin's gs_sim handle, not here.
// Text file: first line "ndim d1 .. dn " then one value per line, printed
// with six significant digits (DumpFile, :338-354); binary file: int32 ndim,
// int32 dims[ndim], float values (BinaryDumpFile, :356-369).
#pragma once
#include <cstdint>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "gs_util.h"

namespace gsfe {

struct Field {
  std::vector<int> dims;
  std::vector<float> v;
  bool empty() const { return dims.empty(); }
  size_t n() const {
    size_t k = dims.empty() ? 0 : 1;
    for (int d : dims) k *= (size_t)d;
    return k;
  }
  void init(const std::vector<int>& d, float fill = 0.0f) {
    dims = d;
    v.assign(n(), fill);
  }
  float sum() const {
    float s = 0;  // a float accumulator, as Data::TotalHost
    for (float x : v) s += x;
    return s;
  }
  void print(std::ostream& os) const {
    os << dims.size() << " ";
    for (int d : dims) os << d << " ";
    os << "\n";
    for (float x : v) os << x << "\n";
  }
  bool write_text(const std::string& path) const {
    std::ofstream os(path);
    if (!os) return false;
    print(os);
    return true;
  }
  bool write_binary(const std::string& path) const {
    std::ofstream os(path, std::ios::binary);
    if (!os) return false;
    int32_t nd = (int32_t)dims.size();
    os.write((const char*)&nd, 4);
    for (int d : dims) {
      int32_t x = d;
      os.write((const char*)&x, 4);
    }
    os.write((const char*)v.data(), (std::streamsize)(v.size() * sizeof(float)));
    return true;
  }
  bool read_text(const std::string& path) {
    std::ifstream is(path);
    if (!is) return false;
    int nd = 0;
    is >> nd;
    std::vector<int> d(nd);
    for (auto& x : d) is >> x;
    init(d);
    for (auto& x : v) is >> x;
    return true;
  }
  bool read_binary(const std::string& path) {
    std::ifstream is(path, std::ios::binary);
    if (!is) return false;
    int32_t nd = 0;
    is.read((char*)&nd, 4);
    std::vector<int> d(nd);
    for (auto& x : d) {
      int32_t y;
      is.read((char*)&y, 4);
      x = y;
    }
    init(d);
    is.read((char*)v.data(), (std::streamsize)(v.size() * sizeof(float)));
    return true;
  }
};

// string-keyed store with aliases: `link target alias` makes alias resolve to
// target (include/datamap.th:6-164)
template <class V> class Store {
 public:
  V& operator[](const std::string& key) { return items_[resolve(key)]; }
  bool has(const std::string& key) const { return items_.count(resolve(key)) > 0; }
  V* find(const std::string& key) {
    auto it = items_.find(resolve(key));
    return it == items_.end() ? nullptr : &it->second;
  }
  int link(const std::string& target, const std::string& alias) {
    if (!has(target)) return -1;
    items_.erase(alias);
    alias_[alias] = target;
    return 0;
  }

 private:
  std::string resolve(const std::string& k) const {
    std::string cur = k;
    for (int i = 0; i < 16; ++i) {
      auto it = alias_.find(cur);
      if (it == alias_.end()) break;
      cur = it->second;
    }
    return cur;
  }
  std::map<std::string, V> items_;
  std::map<std::string, std::string> alias_;
};

}  // namespace gsfe
