// host_util.cpp — see host_util.h.
#include "host_util.h"

#include <fstream>
#include <sstream>

namespace cupf_host {

template <typename T>
static bool get_param_impl(const std::string& lineText, const std::string& key, T& param) {
  std::istringstream iss(lineText);
  std::string word;
  bool found = false;
  while (iss >> word) {
    if (word != key) continue;
    if (!(iss >> word) || word != "=") continue;
    if (!(iss >> word)) break;
    try {
      param = static_cast<T>(std::stof(word));
      found = true;
    } catch (...) {
    }
  }
  return found;
}

bool getParam(const std::string& lineText, const std::string& key, float& param) {
  return get_param_impl(lineText, key, param);
}

bool getParam(const std::string& lineText, const std::string& key, int& param) {
  return get_param_impl(lineText, key, param);
}

int read_input(const std::string& path, float* target, int cap) {
  // float targets are parsed as float, exactly as `ss >> float` in the reference
  std::ifstream f(path);
  if (!f.good()) return -1;
  std::string line;
  int n = 0;
  while (n < cap && std::getline(f, line)) {
    std::istringstream ss(line);
    float v = 0.0f;
    ss >> v;
    target[n++] = v;
  }
  return n;
}

int read_input(const std::string& path, int* target, int cap) {
  std::ifstream f(path);
  if (!f.good()) return -1;
  std::string line;
  int n = 0;
  while (n < cap && std::getline(f, line)) {
    std::istringstream ss(line);
    int v = 0;
    ss >> v;
    target[n++] = v;
  }
  return n;
}

std::vector<float> read_column(const std::string& path) {
  std::vector<float> out;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    float v = 0.0f;
    ss >> v;
    out.push_back(v);
  }
  return out;
}

}  // namespace cupf_host
